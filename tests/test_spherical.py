"""Spherical joints (spherical_joint.rs; SphericalJointDef, types/joint_defs.rs:169).

- the reference's joint_grid golden hash (Tools/Benchmarks/reference-hashes.json: a 100 x 100
  grid of spheres on default spherical joints, 100 steps) on the device, through the C ABI;
- a hanging chain of boxes whose joints carry each feature in turn (cone limit, twist limit,
  spring to a target rotation, motor): on the oracle the cone limit holds and the motor drives
  its body's spin; the device equals the oracle bit for bit every step.
"""
import json
import math
import os

import numpy as np
import pytest

from natsel_b200 import scenes
from oracle import pyoracle

DT = 1.0 / 60.0
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ENGINES = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]
DOWN = (math.sin(math.pi / 4), 0.0, 0.0, math.cos(math.pi / 4))  # frame rotation taking z to -y
CONE = 0.2


def _world(engine, **kw):
    if engine == "oracle":
        return pyoracle.OracleWorld(**kw)
    from natsel_b200.world import World, default_world_def
    kw = dict(kw)
    kw["enable_continuous"] = int(kw.get("enable_continuous", False))
    return World(default_world_def(**kw))


@pytest.mark.gpu
def test_joint_grid_golden_hash_on_gpu():
    case = json.load(open(os.path.join(GOLDEN, "reference_hashes.json")))["cases"]["joint_grid"]
    w = _world("gpu", **scenes.WORLD_SETTINGS["joint_grid"])
    scenes.joint_grid(w)
    for _ in range(case["steps"]):
        w.step(DT, 4)
    assert "%016x" % w.state_hash() == case["hash"]


def _chain(w, cone=True):
    """A static anchor and six 0.1 x 0.3 x 0.1 m boxes hanging below it, each joined to the one
    above at their ends; joint k has the cone limit (k % 4 == 0), the twist limit (1), a spring
    towards a 0.4 rad turn about x (2) or a motor spinning it about the chain at 1 rad/s (3).
    The bodies start swinging and twisting, the top one hard enough to reach its cone."""
    a = w.create_body(type=0, position=(0.0, 5.0, 0.0))
    w.create_box(a, 0.1, 0.1, 0.1)
    prev, bodies = a, []
    for k in range(6):
        v = (6.0, 0.0, 2.0) if k == 0 else (1.0, 0.0, 0.5 - 0.2 * k)
        b = w.create_body(type=2, position=(0.0, 4.7 - 0.6 * k, 0.0), linear_velocity=v,
                          angular_velocity=(0.3, 1.5 - 0.4 * k, 0.0), enable_sleep=False)
        w.create_box(b, 0.1, 0.3, 0.1)
        top = (0.0, -0.1, 0.0) if k == 0 else (0.0, -0.3, 0.0)
        f = k % 4
        kw = {}
        if f == 0:
            kw = dict(enable_cone_limit=cone, cone_angle=CONE)
        elif f == 1:
            kw = dict(enable_twist_limit=True, lower_twist_angle=-0.3, upper_twist_angle=0.3)
        elif f == 2:
            kw = dict(enable_spring=True, hertz=2.0, damping_ratio=0.5,
                      target_rotation=(math.sin(0.2), 0.0, 0.0, math.cos(0.2)))
        else:
            kw = dict(enable_motor=True, max_motor_torque=5.0, motor_velocity=(0.0, 1.0, 0.0))
        w.create_spherical(prev, b, top + DOWN, (0.0, 0.3, 0.0) + DOWN, **kw)
        prev = b
        bodies.append(b)
    return bodies


def _axis(q, v):
    x, y, z, s = (float(c) for c in q)
    u = np.array([x, y, z])
    v = np.asarray(v, float)
    return v + 2.0 * np.cross(u, np.cross(u, v) + s * v)


def _swing(engine, cone):
    """The largest angle between the anchor's frame z axis (-y) and box 0's over 3 s."""
    w = _world(engine, gravity=(0.0, -9.81, 0.0))
    bodies = _chain(w, cone)
    worst = 0.0
    for _ in range(180):
        w.step(DT, 4)
        pos, rot, lin, ang = w.bodies()
        zb = _axis(rot[bodies[0]], (0.0, -1.0, 0.0))
        worst = max(worst, math.acos(max(-1.0, min(1.0, -float(zb[1])))))
    return worst, w, bodies


@pytest.mark.parametrize("engine", ENGINES)
def test_cone_limit_holds_and_motor_spins(engine):
    free, _, _ = _swing(engine, False)
    worst, w, bodies = _swing(engine, True)
    assert free > CONE + 0.05 and worst < CONE + 0.03, (free, worst)
    pos, rot, lin, ang = w.bodies()
    # joint 3's motor: box 3 spins about the chain relative to box 2 near 1 rad/s
    rel = ang[bodies[3]] - ang[bodies[2]]
    axis = _axis(rot[bodies[2]], (0.0, -1.0, 0.0))
    assert 0.5 < abs(float(np.dot(rel, axis))) < 1.5
    assert np.isfinite(pos).all()


@pytest.mark.gpu
def test_spherical_chain_matches_oracle_every_step():
    s = dict(gravity=(0.0, -9.81, 0.0))
    g, o = _world("gpu", **s), _world("oracle", **s)
    for w in (g, o):
        _chain(w)
    for k in range(240):
        g.step(DT, 4)
        o.step(DT, 4)
        assert g.state_hash() == o.state_hash(), k
