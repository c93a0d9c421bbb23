"""Parity of the CUDA step (through the C ABI) with the oracle and the reference's golden
vectors. Everything integer (pairs, contact ids, feature ids, colours, counters) must match
bit for bit; the body state is compared bit for bit too (the per-step world hash), which is
stricter than the 1e-5 relative / 1e-6 m absolute per-step tolerance the path is held to
(test_body_state_within_tolerance states that bar explicitly)."""
import json
import os

import numpy as np
import pytest

from natsel_b200 import narrowphase, scenes
from natsel_b200.world import NsError, World, default_world_def, load_library
from oracle import pyoracle

import _pairgen

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DT = 1.0 / 60.0


def gpu_world(name, world_kw=None, **kw):
    s = scenes.WORLD_SETTINGS[name]
    w = World(default_world_def(gravity=s["gravity"], enable_continuous=int(s["enable_continuous"]),
                                **(world_kw or {})))
    info = scenes.BUILDERS[name](w, **kw)
    return w, info


def oracle_world(name, **kw):
    w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS[name])
    info = scenes.BUILDERS[name](w, **kw)
    return w, info


def step_hashes(w, name, steps):
    out = []
    for _ in range(steps):
        w.step(DT, scenes.SUBSTEPS[name])
        out.append("%016x" % w.state_hash())
    return out


@pytest.mark.parametrize("name", ["large_pyramid", "many_pyramids"])
def test_reference_golden_hash_on_gpu(name):
    case = json.load(open(os.path.join(GOLDEN, "reference_hashes.json")))["cases"][name]
    w, _ = gpu_world(name)
    for _ in range(case["steps"]):
        w.step(DT, 4)
    assert "%016x" % w.state_hash() == case["hash"]


def _fixture_cases():
    cases = json.load(open(os.path.join(GOLDEN, "oracle_hashes.json")))["cases"]
    return [pytest.param(c, id="%s-%s" % (c["scene"], "-".join("%s%s" % kv for kv in c["kw"].items()) or "default"))
            for c in cases]


@pytest.mark.parametrize("case", _fixture_cases())
def test_every_step_matches_oracle_fixture(case):
    w, _ = gpu_world(case["scene"], **case["kw"])
    got = step_hashes(w, case["scene"], case["steps"])
    first_bad = next((i for i, (a, b) in enumerate(zip(got, case["hashes"])) if a != b), None)
    assert first_bad is None, "first differing step %s" % first_bad


def test_contacts_features_colors_match_oracle():
    """Full 10 000-body pile: after 3 steps every live contact (id, shapes, colour, point
    count, flags, SAT cache type), every feature id and every manifold float agree."""
    g, _ = gpu_world("large_pile")
    o, _ = oracle_world("large_pile")
    for step in range(3):
        g.step(DT, 4)
        o.step(DT, 4)
        gi, gf, gx = g.contacts()
        oi, of, ox = o.contacts()
        assert len(gi) == len(oi) and len(gi) > 1000
        np.testing.assert_array_equal(gi, oi)
        np.testing.assert_array_equal(gf, of)
        assert gx.tobytes() == ox.tobytes()
        gc, oc = g.counters(), o.counters()
        np.testing.assert_array_equal(gc[:26], oc[:26])


def test_body_state_within_tolerance():
    """North-star per-step bar: positions and velocities within 1e-5 relative with a 1e-6 m
    absolute floor after one step (here they are also bit-identical)."""
    g, _ = gpu_world("large_pile")
    o, _ = oracle_world("large_pile")
    for _ in range(20):
        g.step(DT, 4)
        o.step(DT, 4)
    for a, b in zip(g.bodies(), o.bodies()):
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6)
        assert a.tobytes() == b.tobytes()


def _pairs(seed, n):
    return _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, n, seed)


def test_pairs_fixture_on_gpu():
    z = np.load(os.path.join(GOLDEN, "pairs.npz"))
    jobs = z["jobs0"].view(narrowphase.PAIR_JOB_DTYPE).copy()
    r1 = narrowphase.collide_pairs(jobs)
    assert r1.tobytes() == z["res1"].tobytes()
    assert jobs.tobytes() == z["jobs1"].tobytes()
    r2 = narrowphase.collide_pairs(jobs)
    assert r2.tobytes() == z["res2"].tobytes()
    assert jobs.tobytes() == z["jobs2"].tobytes()


@pytest.mark.parametrize("reach", [0.9, 1.6])
def test_pairs_random_match_oracle(reach):
    """120 000 random pairs of every type combination, cold then warm caches."""
    n = 120000
    jg = _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, n, 100 + int(reach * 10), reach)
    jo = jg.copy().view(pyoracle.PAIR_JOB_DTYPE)
    for _ in range(2):
        rg = narrowphase.collide_pairs(jg)
        ro = pyoracle.collide_pairs(jo)
        bad = np.nonzero((rg.view(np.uint8).reshape(n, -1) != ro.view(np.uint8).reshape(n, -1)).any(1))[0]
        assert len(bad) == 0, "%d pairs differ, first %s types %s" % (len(bad), bad[:5], jg["type_a"][bad[:5]])
        assert jg.tobytes() == jo.tobytes()
        assert (rg["point_count"] > 0).sum() > n // 10


def test_narrowphase_known_answers_on_gpu():
    """The reference's manifold known-answer cases (convex_manifold_tests.rs:35-100,
    shape_collision_tests.rs:25-192), run on the GPU and compared with the oracle."""
    rows = [
        (3, 3, (1, 1, 1), (1, 1, 1), (1.5, 0, 0), (0, 0, 0, 1)),
        (3, 3, (1, 1, 1), (1, 1, 1), (1.2, 0.7, 0.3), scenes.quat_from_axis_angle((0.0, 1.0, 0.0), 0.785398163)),
        (5, 5, (0, 0, 0, 1), (0, 0, 0, 1), (1.5, 0, 0), (0, 0, 0, 1)),
        (0, 0, (0, -1, 0, 0, 1, 0, 0.5), (0, -1, 0, 0, 1, 0, 0.5), (0.8, 0, 0), (0, 0, 0, 1)),
        (0, 5, (0, 0, 0, 0, 0, 0, 0.5), (0, 0, 0, 1), (1.2, 0.3, 0), (0, 0, 0, 1)),
        (3, 5, (1, 1, 1), (0, 0, 0, 1), (1.2, 0.5, 0), (0, 0, 0, 1)),
        (3, 0, (1, 1, 1), (0, 0, 0, 0, 0, 0, 0.25), (1.1, 0, 0), (0, 0, 0, 1)),
    ]
    jobs = np.zeros(len(rows), narrowphase.PAIR_JOB_DTYPE)
    for k, (ta, tb, ga, gb, p, q) in enumerate(rows):
        jobs["type_a"][k], jobs["type_b"][k] = ta, tb
        jobs["geom_a"][k, :len(ga)] = ga
        jobs["geom_b"][k, :len(gb)] = gb
        jobs["xf"][k] = tuple(p) + tuple(q)
    jo = jobs.copy().view(pyoracle.PAIR_JOB_DTYPE)
    for _ in range(2):  # second pass: warm SAT cache (face_contact expects a hit)
        rg = narrowphase.collide_pairs(jobs)
        ro = pyoracle.collide_pairs(jo)
        assert rg.tobytes() == ro.tobytes() and jobs.tobytes() == jo.tobytes()
    assert list(rg["point_count"]) == [4, 4, 1, 2, 1, 1, 2]
    assert jobs["sat_hit"][0] == 1 and jobs["sat_type"][1] == 2


def test_overflow_color_pile_on_gpu():
    w, _ = gpu_world("overflow_pile")
    for _ in range(10):
        w.step(DT, 4)
    c = w.counters()
    assert w.body_count == 27 and c[0] == 65 and c[2 + 23] == 5


def test_restitution_phase_on_gpu():
    for e in (0.25, 0.5, 0.9):
        vals = []
        for i in range(16):
            gap = float(np.float32(np.float32(i) / np.float32(16)) * np.float32(5.0) * np.float32(DT))
            w, info = gpu_world("restitution_ball", restitution=e, gap=gap)
            for _ in range(60):
                w.step(DT, 4)
            vals.append(float(w.bodies()[2][info["ball"], 1] / np.float32(5.0)))
            w.close()
        assert max(vals) - min(vals) <= 0.05 and abs(np.mean(vals) - e) <= 0.05


# ----- edge cases ---------------------------------------------------------------------------
def _both(build, steps=5, dt=DT, substeps=4):
    g = World(default_world_def(gravity=(0.0, -9.81, 0.0), enable_continuous=0))
    o = pyoracle.OracleWorld(gravity=(0.0, -9.81, 0.0), enable_continuous=False)
    build(g)
    build(o)
    for _ in range(steps):
        g.step(dt, substeps)
        o.step(dt, substeps)
        assert g.state_hash() == o.state_hash()
    return g, o


def test_rollout_scene_matches_oracle():
    # 1024 cubes with random velocities on the ground (the adjoint's rollout scene); this body
    # count also needs the state pass's shared-memory limit raised above the 48 KB default
    g, _ = gpu_world("differentiable_rollout")
    o, _ = oracle_world("differentiable_rollout")
    for _ in range(10):
        g.step(DT, 4)
        o.step(DT, 4)
        assert g.state_hash() == o.state_hash()
    g.close()


def test_empty_world():
    _both(lambda w: None)


def test_static_only_world():
    def build(w):
        b = w.create_body(type=0, position=(0.0, -1.0, 0.0))
        w.create_box(b, 10.0, 1.0, 10.0)
    _both(build)


def test_single_body_free_fall():
    def build(w):
        b = w.create_body(type=2, position=(0.0, 5.0, 0.0), angular_velocity=(0.3, 1.0, -0.2))
        w.create_box(b, 0.3, 0.6, 0.9)
    g, o = _both(build, steps=30)
    assert g.bodies()[2][0, 1] < 0


def test_zero_dt_step():
    def build(w):
        scenes.box_pyramid(w, base=4)
    _both(build, steps=3, dt=0.0)


def test_one_substep_and_many_substeps():
    for sub in (1, 8):
        _both(lambda w: scenes.box_pyramid(w, base=6), steps=10, substeps=sub)


def test_applied_forces_match_oracle():
    """ns_world_apply_forces (apply_body_force_to_center + apply_body_torque for every body)
    before each step gives the oracle's trajectory bit for bit, before and after upload."""
    rng = np.random.Generator(np.random.PCG64(9))
    g = World(default_world_def(gravity=(0.0, -9.81, 0.0), enable_continuous=0))
    o = pyoracle.OracleWorld(gravity=(0.0, -9.81, 0.0), enable_continuous=False)
    for w in (g, o):
        scenes.box_pyramid(w, base=8)
    for k in range(12):
        f = rng.normal(0.0, 200.0, (g.body_count, 3)).astype(np.float32)
        t = rng.normal(0.0, 20.0, (g.body_count, 3)).astype(np.float32)
        for w in (g, o):
            w.apply_forces(f, t if k % 3 else None)
            w.step(DT, 4)
        assert g.state_hash() == o.state_hash()


@pytest.mark.parametrize("solver_blocks", [64, 4])
def test_solver_launch_shapes_match_oracle(solver_blocks):
    """A cooperative grid of 64 blocks and a cluster of 4 CTAs give the same bits as the default."""
    g, _ = gpu_world("large_pile", world_kw={"solver_blocks": solver_blocks}, n=3000, seed=4)
    o, _ = oracle_world("large_pile", n=3000, seed=4)
    for _ in range(40):
        g.step(DT, 4)
        o.step(DT, 4)
    assert g.state_hash() == o.state_hash()
    assert g.solver_counts()[14] == (1 if solver_blocks > 16 else 0)


@pytest.mark.parametrize("n", [3000, 500])
def test_default_solver_shape_follows_world_size(n):
    """solver_blocks 0: a cooperative grid over every SM for a world of 2 048 awake bodies or more
    (it stages each colour's constraints in shared memory), the 16-CTA cluster below (its barrier
    is the cheaper); the same bits either way."""
    g, _ = gpu_world("large_pile", n=n, seed=5)
    o, _ = oracle_world("large_pile", n=n, seed=5)
    for _ in range(30):
        g.step(DT, 4)
        o.step(DT, 4)
    assert g.state_hash() == o.state_hash()
    assert g.solver_counts()[14] == (1 if n >= 2048 else 0)


def test_eager_path_matches_oracle(monkeypatch):
    """Without a CUDA graph (the fallback when stream capture is refused) the step is the same."""
    monkeypatch.setenv("NATSEL_EAGER", "1")
    g, o = _both(lambda w: scenes.box_pyramid(w, base=8), steps=20)
    assert g.phase_times().sum() > 0


def test_contact_capacity_exceeded_is_reported():
    w = World(default_world_def(contact_capacity=1024))
    scenes.large_pyramid(w)  # about 15 000 contacts on the first step
    with pytest.raises(NsError) as err:
        for _ in range(5):
            w.step(DT, 4)
        w.synchronize()
    assert err.value.code == 3


def test_invalid_ids_are_rejected():
    w = World(default_world_def())
    with pytest.raises(NsError):
        w.create_box(7, 0.5, 0.5, 0.5)
    b = w.create_body(type=2)
    with pytest.raises(NsError):
        w.create_revolute(b, 99, (0,) * 6 + (1,), (0,) * 6 + (1,))


def test_barrier_timeout_is_reported_and_context_survives():
    lib = load_library()
    assert lib.ns_selftest_barrier_timeout(0, 50) == 4  # NS_ERR_TIMEOUT
    _both(lambda w: scenes.box_pyramid(w, base=3), steps=2)


def test_spring_limit_motor_revolute_matches_oracle():
    """The scene of revolute_joint_tests.rs:21-62 (spring 4 Hz / 0.6, motor 50 N m at 1 rad/s,
    limit +-0.5 rad, initial spin) built through ns_create_revolute_joint_def: 120 steps equal
    to the oracle's, bit for bit, every step."""
    g = World(default_world_def(gravity=(0.0, -10.0, 0.0)))
    o = pyoracle.OracleWorld(gravity=(0.0, -10.0, 0.0), enable_continuous=True)
    for w in (g, o):
        a = w.create_body(type=0, position=(0.0, 3.0, 0.0))
        b = w.create_body(type=2, position=(1.5, 3.0, 0.0), angular_velocity=(1.0, 0.5, 0.0))
        w.create_box(b, 0.2, 0.2, 0.2, density=1000.0)
        w.create_revolute(a, b, (1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0), (-0.5, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0),
                          enable_spring=True, hertz=4.0, damping_ratio=0.6, enable_motor=True,
                          max_motor_torque=50.0, motor_speed=1.0, enable_limit=True, lower=-0.5, upper=0.5)
    for _ in range(120):
        g.step(DT, 4)
        o.step(DT, 4)
        assert g.state_hash() == o.state_hash()
    g.close()


def test_nonfinite_state_is_reported():
    """A NaN force reaches finalize's finite check (the reference asserts finite velocities
    there, solver_integration.rs:626-627): the next synchronising call reports
    NS_ERR_NONFINITE. Only the one step with the NaN runs; its bodies keep their old fat AABBs."""
    g = World(default_world_def(gravity=(0.0, -9.81, 0.0)))
    scenes.box_pyramid(g, base=4)
    for _ in range(3):
        g.step(DT, 4)
    g.synchronize()
    f = np.zeros((g.body_count, 3), np.float32)
    f[g.body_count - 1, 0] = np.nan
    g.apply_forces(f)
    g.step(DT, 4)
    with pytest.raises(NsError) as err:
        g.synchronize()
    assert err.value.code == 5 and "NaN" in str(err.value)
    g.close()


# ----- full-size properties -----------------------------------------------------------------
def test_large_pile_settles():
    """600 steps of the 10 000-body pile (the workload's full length): state stays finite,
    nothing falls through the ground, contacts stay shallow and the pile comes to rest."""
    w, _ = gpu_world("large_pile")
    for _ in range(600):
        w.step(DT, 4)
    pos, rot, lin, ang = w.bodies()
    assert np.isfinite(pos).all() and np.isfinite(lin).all() and np.isfinite(ang).all()
    dyn = np.array(w.body_types) == 2
    # bodies still above the 100 x 100 m ground box (a few roll off its edge and fall)
    on_ground = dyn & (np.abs(pos[:, 0]) < 49.0) & (np.abs(pos[:, 2]) < 49.0)
    assert on_ground.sum() > 9900
    assert pos[on_ground, 1].min() > -0.05
    _, _, fl = w.contacts()
    ints = w.contacts()[0]
    touching = ints[:, 4] > 0
    seps = [fl[i, 6 + 5 * k] for i in np.nonzero(touching)[0] for k in range(ints[i, 4])]
    assert min(seps) > -0.25 and np.percentile(seps, 0.1) > -0.05
    assert np.median(np.linalg.norm(lin[on_ground], axis=1)) < 0.1


def test_jointed_chains_full_size_hold_together():
    """52 000 bodies and 48 000 limited revolute joints: 30 steps stay finite and each
    link's upper end stays attached to the previous link's lower end."""
    w, info = gpu_world("jointed_chains")
    for _ in range(30):
        w.step(DT, 8)
    pos, rot, lin, ang = w.bodies()
    assert np.isfinite(pos).all() and np.isfinite(lin).all()
    # body 0 is the ground; then per chain 1 static anchor + 24 links
    chain = pos[1:1 + 2000 * 25].reshape(2000, 25, 3)
    q = rot[1:1 + 2000 * 25].reshape(2000, 25, 4)

    def rotate(qv, v):
        u, s = qv[..., :3], qv[..., 3:4]
        t = 2.0 * np.cross(u, v)
        return v + s * t + np.cross(u, t)

    up = chain[:, 1:] + rotate(q[:, 1:], np.array([0.0, 0.25, 0.0]))
    down = chain[:, 1:-1] + rotate(q[:, 1:-1], np.array([0.0, -0.25, 0.0]))
    gap = np.linalg.norm(up[:, 1:] - down, axis=-1)
    anchor_gap = np.linalg.norm(up[:, 0] - chain[:, 0], axis=-1)
    assert np.percentile(gap, 99) < 0.02 and np.percentile(anchor_gap, 99) < 0.02


def test_box_pyramid_long_run_statistics():
    """1000 steps of the 210-cube pyramid: identical to the oracle at the end, so energy,
    penetration and resting-contact statistics agree exactly; the pyramid stands."""
    g, _ = gpu_world("box_pyramid")
    o, _ = oracle_world("box_pyramid")
    for _ in range(1000):
        g.step(DT, 4)
        o.step(DT, 4)
    assert g.state_hash() == o.state_hash()
    pos = g.bodies()[0]
    assert pos[1:, 1].max() > 19.0  # the top cube is still up
