"""Continuous collision of fast bodies against static shapes (the reference's continuous.rs:337
solve_continuous with collision/time_of_impact.rs:391), on the oracle and on the device.

- the oracle's time of impact against the reference's known answers (distance_tests.rs:182-280:
  states, normals and iteration counts of a translating, a receding and a rotating box);
- the reference's fast-body scene (ccd_tests.rs:30-85: a box at 200 m/s at a 0.2 m wall, 30
  steps of one substep) on both engines: it stays on the approach side with finite state and
  no live contact, and without the continuous pass it tunnels;
- the device's continuous pass bit for bit against the oracle's, step by step, on that scene and
  on a pile dropped onto a thin ground with a thousand fast bodies a step;
- bullets (body_def.rs:74 is_bullet; solver_integration.rs:949-958): the same scene as a bullet
  (ccd_tests.rs:85-100), a bullet shot at a free box (it stops at the box, where a plain fast
  body passes through it), and the reference's fast-movers scene (parallel_solver_tests.rs:
  280-322: 640 cubes between two walls, 24 spheres at 300 m/s, every third a bullet), device
  against oracle bit for bit every step.
"""
import math

import numpy as np
import pytest

from natsel_b200 import scenes
from oracle import pyoracle

DT = 1.0 / 60.0
ENGINES = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]
BOX = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float32)
ID = (0.0, 0.0, 0.0, 1.0)
ZERO = (0.0, 0.0, 0.0)


def _toi(sweep_b):
    """distance_tests.rs:182 run_time_of_impact: a 2 m box at rest against a 2 m box on sweep_b."""
    return pyoracle.time_of_impact(BOX, 0.0, BOX, 0.0, (ZERO, ZERO, ZERO, ID, ID), sweep_b, 1.0)


def test_toi_translation_known_answer():
    """distance_tests.rs:200-228: hit, normal exactly +x, 2 distance / 1 push-back / 2 root
    iterations; the fraction puts the faces the target (one linear slop) apart."""
    out = _toi((ZERO, (5.0, 0.0, 0.0), ZERO, ID, ID))
    assert out["state"] == "hit"
    assert out["normal"].tolist() == [1.0, 0.0, 0.0]
    assert (out["distance_iterations"], out["push_back_iterations"], out["root_iterations"]) == (2, 1, 2)
    gap = 5.0 * (1.0 - float(out["fraction"])) - 2.0
    assert abs(gap - 0.005) <= 0.25 * 0.005


def test_toi_receding_known_answer():
    """distance_tests.rs:231-254: separated after one distance iteration, fraction 1."""
    out = _toi((ZERO, (5.0, 0.0, 0.0), (10.0, 0.0, 0.0), ID, ID))
    assert out["state"] == "separated" and out["distance_iterations"] == 1 and out["fraction"] == 1.0


def test_toi_rotation_known_answer():
    """distance_tests.rs:257-280: a box turning 45 degrees about z while closing: hit, normal
    exactly +x, 2 distance iterations and 4 root iterations."""
    a = 0.785398163
    q = (0.0, 0.0, math.sin(0.5 * a), math.cos(0.5 * a))
    out = _toi((ZERO, (4.0, 0.0, 0.0), ZERO, ID, q))
    assert out["state"] == "hit"
    assert out["normal"].tolist() == [1.0, 0.0, 0.0]
    assert out["distance_iterations"] == 2 and out["root_iterations"] == 4


def _world(engine, **kw):
    if engine == "oracle":
        return pyoracle.OracleWorld(**kw)
    from natsel_b200.world import World, default_world_def
    kw = dict(kw)
    kw["enable_continuous"] = int(kw.get("enable_continuous", True))
    return World(default_world_def(**kw))


def _fast_box(w, bullet=False):
    """ccd_tests.rs:30-51: a static wall (half extents 0.1, 2, 2) and a 0.4 m box of density 1000
    at x = -5 moving at 200 m/s toward it."""
    wall = w.create_body(type=0)
    w.create_box(wall, 0.1, 2.0, 2.0)
    b = w.create_body(type=2, position=(-5.0, 0.0, 0.0), linear_velocity=(200.0, 0.0, 0.0), is_bullet=bullet)
    w.create_box(b, 0.2, 0.2, 0.2, density=1000.0)
    return b


@pytest.mark.parametrize("bullet", [False, True], ids=["fast_body", "bullet"])
@pytest.mark.parametrize("engine", ENGINES)
def test_fast_body_does_not_tunnel(engine, bullet):
    """ccd_tests.rs:52-68 and :85-118: after 30 steps of one substep the box, plain or a bullet,
    is still on the approach side of the wall (x < 0), its state finite and no contact alive;
    with continuous collision off the same box passes the wall."""
    w = _world(engine, gravity=(0.0, -10.0, 0.0), enable_continuous=True)
    b = _fast_box(w, bullet)
    for _ in range(30):
        w.step(DT, 1)
    pos, rot, lin, ang = w.bodies()
    assert pos[b, 0] < 0.0
    assert np.isfinite(lin[b]).all() and np.isfinite(ang[b]).all()
    assert w.counters()[0] == 0
    off = _world(engine, gravity=(0.0, -10.0, 0.0), enable_continuous=False)
    b = _fast_box(off)
    for _ in range(30):
        off.step(DT, 1)
    assert off.bodies()[0][b, 0] > 10.0


@pytest.mark.gpu
@pytest.mark.parametrize("bullet", [False, True], ids=["fast_body", "bullet"])
def test_fast_body_scene_matches_oracle_every_step(bullet):
    g = _world("gpu", gravity=(0.0, -10.0, 0.0), enable_continuous=True)
    o = _world("oracle", gravity=(0.0, -10.0, 0.0), enable_continuous=True)
    for w in (g, o):
        _fast_box(w, bullet)
    for _ in range(30):
        g.step(DT, 1)
        o.step(DT, 1)
        assert g.state_hash() == o.state_hash()
    assert g.counters()[26] == o.counters()[26] > 0


def _shot_at_a_box(w, bullet):
    """No gravity: a free 1 m box at rest at the origin and a 0.1 m sphere at x = -5 moving at
    300 m/s toward it (5 m per step)."""
    box = w.create_body(type=2, enable_sleep=False)
    w.create_box(box, 0.5, 0.5, 0.5, density=1000.0)
    ball = w.create_body(type=2, position=(-5.0, 0.0, 0.0), linear_velocity=(300.0, 0.0, 0.0), is_bullet=bullet,
                         enable_sleep=False)
    w.create_sphere(ball, 0.1, density=1000.0)
    return box, ball


@pytest.mark.parametrize("engine", ENGINES)
def test_bullet_stops_at_a_dynamic_body(engine):
    """A bullet is swept against dynamic bodies too (continuous.rs:429-448): the ball stops at the
    box's face in the step it would pass it, then pushes the box; a plain fast body only sweeps
    against static shapes and passes through the box, leaving it at rest."""
    w = _world(engine, gravity=(0.0, 0.0, 0.0), enable_continuous=True)
    box, ball = _shot_at_a_box(w, True)
    w.step(DT, 4)
    pos, rot, lin, ang = w.bodies()
    assert -0.65 < pos[ball, 0] < -0.55  # touching the face at x = -0.5 (radius 0.1)
    for _ in range(3):
        w.step(DT, 4)
    pos, rot, lin, ang = w.bodies()
    assert lin[box, 0] > 1.0 and pos[ball, 0] < pos[box, 0]
    w = _world(engine, gravity=(0.0, 0.0, 0.0), enable_continuous=True)
    box, ball = _shot_at_a_box(w, False)
    for _ in range(4):
        w.step(DT, 4)
    pos, rot, lin, ang = w.bodies()
    assert pos[ball, 0] > 10.0 and lin[box, 0] == 0.0


def _fast_movers(w):
    """parallel_solver_tests.rs:280-322 build_fast_and_sleepy: a ground, two walls, 640 cubes of
    0.4 m half extent and 24 spheres of radius 0.1 at 300 m/s across them, every third a bullet."""
    g = w.create_body(type=0, position=(0.0, -1.0, 0.0))
    w.create_box(g, 50.0, 1.0, 50.0)
    for x in (-16.0, 16.0):
        wall = w.create_body(type=0, position=(x, 4.0, 0.0))
        w.create_box(wall, 0.25, 4.0, 20.0)
    for i in range(640):
        b = w.create_body(type=2, position=((i % 16) - 7.5, 0.4 + (i // 256) * 0.8, ((i // 16) % 16) - 7.5),
                          enable_sleep=False)
        w.create_box(b, 0.4, 0.4, 0.4)
    for i in range(24):
        b = w.create_body(type=2, position=(-12.0 if i % 2 == 0 else 12.0, 1.0 + (i // 2) * 0.5, (i % 5) - 2.0),
                          linear_velocity=(300.0 if i % 2 == 0 else -300.0, 0.0, (i % 3) - 1.0),
                          is_bullet=i % 3 == 0, enable_sleep=False)
        w.create_sphere(b, 0.1)


@pytest.mark.gpu
def test_fast_movers_scene_matches_oracle_every_step():
    """The reference's fast-movers scene, gravity -10, 60 Hz, 4 substeps: the device equals the
    oracle bit for bit every step for 60 steps; a sphere found beyond a wall's plane went around
    the wall (cubes deflect some sideways), not through it."""
    s = dict(gravity=(0.0, -10.0, 0.0), enable_continuous=True)
    g, o = _world("gpu", **s), _world("oracle", **s)
    for w in (g, o):
        _fast_movers(w)
    pyoracle.set_threads(8)
    try:
        for k in range(60):
            g.step(DT, 4)
            o.step(DT, 4)
            assert g.state_hash() == o.state_hash(), k
    finally:
        pyoracle.set_threads(1)
    assert g.counters()[26] == o.counters()[26] > 0
    pos = g.bodies()[0][-24:]
    beyond = np.abs(pos[:, 0]) > 16.0
    assert ((np.abs(pos[beyond, 2]) > 20.0) | (pos[beyond, 1] > 8.0)).all()


@pytest.mark.gpu
def test_pile_on_a_thin_ground_matches_oracle_with_continuous_collision():
    """3 000 bodies of the pile's mix dropped from up to 61 m onto a 0.2 m slab with continuous
    collision on (about a thousand fast bodies a step during the drop): the device's state
    equals the oracle's bit for bit every step for 150 steps, and the fast-body counts agree."""
    s = dict(gravity=(0.0, -9.81, 0.0), enable_continuous=True)
    g, o = _world("gpu", **s), _world("oracle", **s)
    for w in (g, o):
        scenes.large_pile(w, n=3000, seed=5, ground_half_height=0.1)
    pyoracle.set_threads(8)
    try:
        for k in range(150):
            g.step(DT, 4)
            o.step(DT, 4)
            assert g.state_hash() == o.state_hash(), k
    finally:
        pyoracle.set_threads(1)
    assert g.counters()[26] == o.counters()[26] > 10000
    assert (g.bodies()[0][1:, 1] > -0.2).all()
