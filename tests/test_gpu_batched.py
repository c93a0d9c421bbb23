"""Batched worlds: independent sub-worlds stepped together in one world object must each give
the bits of the same world stepped on its own (per-sub-world world_state_hash equal to the
oracle's), including their overflow colours, joints and restitution."""
import numpy as np
import pytest

from natsel_b200 import scenes
from natsel_b200.world import NsError, World, default_world_def
from oracle import pyoracle

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0
SETTINGS = dict(gravity=(0.0, -9.81, 0.0), enable_continuous=False)

MIXED = [
    ("overflow_pile", {}),
    ("box_pyramid", {"base": 6}),
    ("jointed_chains", {"chains": 6, "boxes": 12, "grid": 3, "height": 8.0}),
    ("large_pile", {"n": 300, "seed": 9, "restitution": 0.4, "spread": 4.0, "drop": (1.0, 9.0), "ground_half": 15.0}),
    ("box_pyramid", {"base": 3}),
]


def oracle_hash(build, steps, substeps):
    o = pyoracle.OracleWorld(**SETTINGS)
    build(o)
    for _ in range(steps):
        o.step(DT, substeps)
    return o.state_hash()


def test_mixed_batch_matches_each_world_alone():
    g = World(default_world_def(gravity=SETTINGS["gravity"], enable_continuous=0))
    for k, (name, kw) in enumerate(MIXED):
        if k:
            g.begin_subworld()
        scenes.BUILDERS[name](g, **kw)
    assert g.subworld_count == len(MIXED)
    for _ in range(40):
        g.step(DT, 4)
    got = g.subworld_hashes()
    for k, (name, kw) in enumerate(MIXED):
        want = oracle_hash(lambda w: scenes.BUILDERS[name](w, **kw), 40, 4)
        assert int(got[k]) == want, "sub-world %d (%s) differs" % (k, name)
    c = g.counters()
    assert c[2 + 23] > 0  # the overflow pile's overflow colour is populated inside the batch


def test_batched_worlds_workload_sample_matches():
    """The 4096-world workload (log-uniform 32..512 bodies each): after 12 steps a sample of
    sub-worlds equals the same worlds stepped alone."""
    g = World(default_world_def(gravity=SETTINGS["gravity"], enable_continuous=0))
    info = scenes.batched_worlds(g, count=4096, seed=4)
    assert g.subworld_count == 4096 and info["dynamic_bodies"] > 500000
    for _ in range(12):
        g.step(DT, 4)
    got = g.subworld_hashes()
    for k in [0, 1, 2, 3, 511, 1024, 2047, 3000, 4095]:
        want = oracle_hash(lambda w: scenes.batch_world(w, k, 4), 12, 4)
        assert int(got[k]) == want, "sub-world %d differs" % k


def test_subworld_rules():
    g = World(default_world_def())
    b0 = g.create_body(type=2)
    assert g.begin_subworld() == 1
    b1 = g.create_body(type=2, position=(0.0, 2.0, 0.0))
    from natsel_b200.world import NsError
    with pytest.raises(NsError):
        g.create_box(b0, 0.5, 0.5, 0.5)  # a body of an earlier sub-world
    with pytest.raises(NsError):
        g.create_revolute(b0, b1, (0,) * 6 + (1,), (0,) * 6 + (1,))
    g.create_box(b1, 0.5, 0.5, 0.5)
    assert list(g.subworld_bodies()) == [0, 1, 2]


@pytest.mark.parametrize("batched", [True, False], ids=["batch", "single-world"])
def test_autotune_keeps_the_world_and_its_trajectory(batched):
    """ns_world_autotune times the solver's candidate launch shapes from a copy of the world's
    state and keeps the fastest: the world is left as it was, and the steps after it are
    bit-identical to those of a world that was never tuned."""
    def build():
        g = World(default_world_def(gravity=SETTINGS["gravity"], enable_continuous=0))
        if batched:
            scenes.batched_worlds(g, count=96, seed=4)
        else:
            scenes.large_pile(g, n=1500, seed=5, spread=8.0, drop=(1.0, 15.0))
        return g
    tuned, plain = build(), build()
    for w in (tuned, plain):
        for _ in range(5):
            w.step(DT, 4)
    before = tuned.state_hash()
    table = tuned.autotune(DT, 4, steps=3)
    assert len(table) >= 2 and all(ms > 0 or (not grid and ms == -1.0) for _, grid, ms in table)
    assert tuned.state_hash() == before
    chosen = tuned.solver_counts()
    fastest = min((ms, b, grid) for b, grid, ms in table if ms > 0)
    assert (int(chosen[13]), bool(chosen[14])) == (fastest[1], fastest[2])
    # the other tuned kernels: every candidate timed, the fastest (or the default on a tie) kept
    rows = tuned.autotune_table()
    shapes = tuned.launch_shapes()
    keys = {"recycle_pass": ("recycle_threads", "recycle_per_sm"), "manifold_updates": ("update_threads", "update_per_sm"),
            "prepare": ("prepare_threads", "prepare_per_sm")}
    for dim, (kt, kb) in keys.items():
        cands = [r for r in rows if r["dimension"] == dim]
        assert len(cands) == 5 and all(r["ms_per_step"] > 0 for r in cands)
        best = min(cands, key=lambda r: r["ms_per_step"])
        assert (shapes[kt], shapes[kb]) == (best["a"], best["b"])
    # the same shapes applied to a fresh world of the same scene (ns_world_set_launch_shapes)
    applied = build()
    applied.set_launch_shapes(shapes)
    assert applied.launch_shapes() == shapes
    for _ in range(5):
        applied.step(DT, 4)
    for _ in range(10):
        tuned.step(DT, 4)
        plain.step(DT, 4)
        applied.step(DT, 4)
        assert tuned.state_hash() == plain.state_hash() == applied.state_hash()
    bad = dict(shapes, update_threads=96)  # above k_collide_update's launch bound
    with pytest.raises(NsError):
        applied.set_launch_shapes(bad)
    for w in (tuned, plain, applied):
        w.close()


def test_batch_with_kinematic_bodies_and_bullets_matches_each_world_alone():
    """Sub-worlds with continuous collision on: kinematic platforms, a spinning paddle and a
    kinematic wall hit by a bullet; the reference's fast-movers scene with bullets among cubes;
    a pyramid. The bullet pass and the kinematic rules stay inside each sub-world."""
    from test_continuous import _fast_movers
    from test_kinematic import _mixed
    settings = dict(gravity=(0.0, -9.81, 0.0), enable_continuous=True)
    builders = [_mixed, _fast_movers, lambda w: scenes.BUILDERS["box_pyramid"](w, base=4), _mixed]
    g = World(default_world_def(gravity=settings["gravity"], enable_continuous=1))
    for k, build in enumerate(builders):
        if k:
            g.begin_subworld()
        build(g)
    for _ in range(30):
        g.step(DT, 4)
    got = g.subworld_hashes()
    for k, build in enumerate(builders):
        o = pyoracle.OracleWorld(**settings)
        build(o)
        for _ in range(30):
            o.step(DT, 4)
        assert int(got[k]) == o.state_hash(), "sub-world %d differs" % k
