"""Kinematic bodies (BodyType::KinematicBody): zero mass (body_api.rs:670-689), pairs only with a
dynamic body (contact_creation.rs:113), coloured like static bodies (constraint_graph.rs:113),
no gravity (solver_integration.rs:282), never changed by a constraint or a warm start; swept by
bullets (continuous.rs:429-448). On the oracle and on the device, and the device bit for bit
against the oracle.

- step_tests.rs:71-142: a kinematic sphere with linear and angular velocity moves at its
  velocity and ignores gravity;
- a platform moving at constant velocity carries a stack of boxes by friction and keeps its own
  velocity; a kinematic body overlapping a static one and another kinematic body makes no contact;
- device against oracle every step on a scene with a moving platform, a spinning paddle, a
  pendulum hinged to a moving kinematic anchor and bullets fired at a kinematic wall.
"""
import numpy as np
import pytest

from oracle import pyoracle

DT = 1.0 / 60.0
ENGINES = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]
KIN, DYN, STA = 1, 2, 0


def _world(engine, **kw):
    if engine == "oracle":
        return pyoracle.OracleWorld(**kw)
    from natsel_b200.world import World, default_world_def
    kw = dict(kw)
    kw["enable_continuous"] = int(kw.get("enable_continuous", False))
    return World(default_world_def(**kw))


@pytest.mark.parametrize("engine", ENGINES)
def test_kinematic_body_moves_at_its_velocity_and_ignores_gravity(engine):
    """step_tests.rs:71-82 and :136-138: a kinematic sphere at (2, 0, 0) with velocity (0, 0, 1)
    and angular velocity (0.3, 0, 0) under gravity -10, 5 steps of 4 substeps."""
    w = _world(engine, gravity=(0.0, -10.0, 0.0), enable_continuous=False)
    b = w.create_body(type=KIN, position=(2.0, 0.0, 0.0), linear_velocity=(0.0, 0.0, 1.0),
                      angular_velocity=(0.3, 0.0, 0.0))
    w.create_sphere(b, 0.25)
    for _ in range(5):
        w.step(DT, 4)
    pos, rot, lin, ang = w.bodies()
    assert lin[b].tolist() == [0.0, 0.0, 1.0] and ang[b].tolist() == [np.float32(0.3), 0.0, 0.0]
    assert pos[b, 0] == 2.0 and pos[b, 1] == 0.0
    assert abs(pos[b, 2] - 5 * DT) < 1e-6
    assert abs(rot[b, 0] - np.sin(0.5 * 0.3 * 5 * DT)) < 1e-5


def _platform(w):
    """A 4 x 0.4 x 4 m kinematic platform moving at 1 m/s along x, three boxes stacked on it,
    a static box and a second kinematic box overlapping the platform's far end."""
    p = w.create_body(type=KIN, position=(0.0, 0.0, 0.0), linear_velocity=(1.0, 0.0, 0.0))
    w.create_box(p, 2.0, 0.2, 2.0, friction=0.8)
    boxes = []
    for k in range(3):
        b = w.create_body(type=DYN, position=(0.0, 0.698 + 0.996 * k, 0.0), enable_sleep=False)
        w.create_box(b, 0.5, 0.5, 0.5, friction=0.8)
        boxes.append(b)
    s = w.create_body(type=STA, position=(3.0, -1.0, 0.0))
    w.create_box(s, 0.5, 0.5, 0.5)
    k2 = w.create_body(type=KIN, position=(-3.0, -1.0, 0.0), linear_velocity=(2.0, 0.0, 0.0))
    w.create_box(k2, 0.5, 0.5, 0.5)
    return p, boxes, k2


@pytest.mark.parametrize("engine", ENGINES)
def test_moving_platform_carries_boxes_and_keeps_its_velocity(engine):
    w = _world(engine, gravity=(0.0, -9.81, 0.0), enable_continuous=False)
    p, boxes, k2 = _platform(w)
    for _ in range(180):  # the stack rocks for about two seconds, then rides along
        w.step(DT, 4)
    pos, rot, lin, ang = w.bodies()
    assert lin[p].tolist() == [1.0, 0.0, 0.0] and ang[p].tolist() == [0.0, 0.0, 0.0]
    assert abs(pos[p, 0] - 180 * DT) < 1e-4 and pos[p, 1] == 0.0
    for b in boxes:
        assert abs(lin[b, 0] - 1.0) < 0.02, lin[b]
        assert abs(pos[b, 0] - pos[p, 0]) < 0.05
    assert pos[boxes[0], 1] > 0.6
    # the platform against the static box and the other kinematic box: no contact (shape ids
    # equal body ids here: one shape per body, created in order)
    ints = w.contacts()[0]
    shapes = set()
    for row in ints:
        shapes.update(int(x) for x in row[1:3])
    assert len(ints) > 0 and k2 not in shapes and 4 not in shapes


def _mixed(w):
    """A ground, a platform moving along z carrying boxes, a paddle spinning about y sweeping
    boxes on the ground, a pendulum hinged to a kinematic anchor moving along x, and two spheres
    fired at 300 m/s at a thin kinematic wall (one a bullet)."""
    g = w.create_body(type=STA, position=(0.0, -1.0, 0.0))
    w.create_box(g, 30.0, 1.0, 30.0)
    p = w.create_body(type=KIN, position=(-6.0, 0.5, 0.0), linear_velocity=(0.0, 0.0, 0.8))
    w.create_box(p, 1.5, 0.2, 1.5)
    for k in range(4):
        b = w.create_body(type=DYN, position=(-6.0 + 0.9 * (k % 2) - 0.45, 1.2 + 0.6 * (k // 2), 0.2 * k),
                          enable_sleep=False)
        w.create_box(b, 0.25, 0.25, 0.25)
    paddle = w.create_body(type=KIN, position=(4.0, 0.3, 0.0), angular_velocity=(0.0, 2.0, 0.0))
    w.create_box(paddle, 2.0, 0.3, 0.1)
    for k in range(6):
        b = w.create_body(type=DYN, position=(4.0 + 0.7 * (k - 2.5), 0.25, 1.0 + 0.3 * (k % 2)), enable_sleep=False)
        w.create_sphere(b, 0.25) if k % 2 else w.create_box(b, 0.25, 0.25, 0.25)
    anchor = w.create_body(type=KIN, position=(0.0, 5.0, -5.0), linear_velocity=(0.5, 0.0, 0.0))
    w.create_box(anchor, 0.1, 0.1, 0.1)
    bob = w.create_body(type=DYN, position=(0.0, 4.0, -5.0), linear_velocity=(0.0, 0.0, 2.0), enable_sleep=False)
    w.create_box(bob, 0.2, 0.4, 0.2)
    w.create_revolute(anchor, bob, (0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0), (0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0))
    wall = w.create_body(type=KIN, position=(10.0, 2.0, 8.0), linear_velocity=(0.0, 0.0, -0.1))
    w.create_box(wall, 0.1, 2.0, 2.0)
    for k in range(2):
        b = w.create_body(type=DYN, position=(2.0, 1.5 + k, 8.0), linear_velocity=(300.0, 0.0, 0.0),
                          is_bullet=k == 1, enable_sleep=False)
        w.create_sphere(b, 0.1)


@pytest.mark.parametrize("engine", ENGINES)
def test_bullet_stops_at_a_kinematic_wall(engine):
    """The bullet sweeps against the kinematic wall and stays on its near side; the plain fast
    sphere only sweeps against static shapes and passes through it."""
    w = _world(engine, gravity=(0.0, -9.81, 0.0), enable_continuous=True)
    _mixed(w)
    for _ in range(10):
        w.step(DT, 4)
    pos = w.bodies()[0]
    plain, bullet = len(pos) - 2, len(pos) - 1
    assert pos[bullet, 0] < 10.0 and pos[plain, 0] > 12.0


@pytest.mark.gpu
def test_mixed_kinematic_scene_matches_oracle_every_step():
    s = dict(gravity=(0.0, -9.81, 0.0), enable_continuous=True)
    g, o = _world("gpu", **s), _world("oracle", **s)
    for w in (g, o):
        _mixed(w)
    for k in range(120):
        g.step(DT, 4)
        o.step(DT, 4)
        assert g.state_hash() == o.state_hash(), k
    assert g.counters()[0] == o.counters()[0] > 0
