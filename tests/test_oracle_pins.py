"""The oracle (CPU restatement of the reference step) against the reference's own golden
vectors and known-answer tests, and against the committed fixtures. CPU only."""
import json
import os

import numpy as np
import pytest

from natsel_b200 import scenes
from oracle import pyoracle

import _pairgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _world(name, **kw):
    w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS[name])
    info = scenes.BUILDERS[name](w, **kw)
    return w, info


def _hashes(name, kw, steps):
    w, _ = _world(name, **kw)
    out = []
    for _ in range(steps):
        w.step(1.0 / 60.0, scenes.SUBSTEPS[name])
        out.append("%016x" % w.state_hash())
    return out


@pytest.mark.parametrize("name", ["large_pyramid", "many_pyramids", "joint_grid"])
def test_reference_golden_hash(name):
    """Tools/Benchmarks/reference-hashes.json: state hash after N steps of the benchmark scene."""
    case = json.load(open(os.path.join(GOLDEN, "reference_hashes.json")))["cases"][name]
    assert _hashes(name, {}, case["steps"])[-1] == case["hash"]


@pytest.mark.parametrize("name", ["large_pyramid", "many_pyramids", "joint_grid"])
def test_colour_parallel_oracle_reproduces_golden_hash(name):
    """The oracle's colour-parallel loops (the reference arm's CPU path) give the same bits on
    four threads: every parallel loop touches disjoint data."""
    case = json.load(open(os.path.join(GOLDEN, "reference_hashes.json")))["cases"][name]
    pyoracle.set_threads(4)
    try:
        assert _hashes(name, {}, case["steps"])[-1] == case["hash"]
    finally:
        pyoracle.set_threads(1)


def test_colour_parallel_oracle_matches_one_thread():
    kw = {"n": 2000, "seed": 7}
    one = _hashes("large_pile", kw, 30)
    pyoracle.set_threads(4)
    try:
        assert _hashes("large_pile", kw, 30) == one
    finally:
        pyoracle.set_threads(1)


def _fixture_cases():
    cases = json.load(open(os.path.join(GOLDEN, "oracle_hashes.json")))["cases"]
    return [pytest.param(c, id="%s-%s" % (c["scene"], "-".join("%s%s" % kv for kv in c["kw"].items()) or "default"))
            for c in cases]


@pytest.mark.parametrize("case", _fixture_cases())
def test_oracle_matches_fixture(case):
    steps = min(case["steps"], 40)
    assert _hashes(case["scene"], case["kw"], steps) == case["hashes"][:steps]


def test_overflow_color_pile():
    """overflow_color_tests.rs:83-100: 10 steps -> 27 bodies, 65 contacts, 5 in the overflow colour."""
    w, info = _world("overflow_pile")
    for _ in range(10):
        w.step(1.0 / 60.0, 4)
    c = w.counters()
    assert w.body_count == 27
    assert c[0] == 65
    assert c[2 + 23] == 5


@pytest.mark.parametrize("restitution", [0.25, 0.5, 0.9])
def test_restitution_phase(restitution):
    """restitution_phase_tests.rs:96-130: over 16 impact phases the recovered coefficient has
    spread <= 0.05 and mean within 0.05 of the restitution."""
    speed = np.float32(5.0)
    vals = []
    for i in range(16):
        gap = float(np.float32(np.float32(i) / np.float32(16)) * speed * np.float32(1.0 / 60.0))
        w, info = _world("restitution_ball", restitution=restitution, gap=gap)
        for _ in range(60):
            w.step(1.0 / 60.0, 4)
        vals.append(float(w.bodies()[2][info["ball"], 1] / speed))
    assert max(vals) - min(vals) <= 0.05
    assert abs(np.mean(vals) - restitution) <= 0.05


# ----- narrowphase known answers (convex_manifold_tests.rs, shape_collision_tests.rs) -----
FACE_AXIS_A, FACE_AXIS_B = 2, 3  # SeparatingFeature (collision_types.rs:65)


def _job(ta, tb, ga, gb, p, q=(0.0, 0.0, 0.0, 1.0)):
    j = np.zeros(1, pyoracle.PAIR_JOB_DTYPE)
    j["type_a"], j["type_b"] = ta, tb
    j["geom_a"][0, :len(ga)] = ga
    j["geom_b"][0, :len(gb)] = gb
    j["xf"][0] = tuple(p) + tuple(q)
    return j


def _bits(x):
    return int(np.float32(x).view(np.uint32))


def test_kat_face_contact():
    """convex_manifold_tests.rs:35: unit boxes 1.5 apart -> FaceAxisB 0/0, then a cache hit, 4 points."""
    j = _job(3, 3, (1, 1, 1), (1, 1, 1), (1.5, 0, 0))
    r = pyoracle.collide_pairs(j)
    assert j["sat_type"][0] == FACE_AXIS_B and j["sat_index_a"][0] == 0 and j["sat_index_b"][0] == 0
    assert j["sat_hit"][0] == 0
    r = pyoracle.collide_pairs(j)
    assert j["sat_hit"][0] == 1 and r["point_count"][0] == 4


def test_kat_rotated_contact():
    """convex_manifold_tests.rs:76: B turned 45 deg about y at (1.2, 0.7, 0.3) -> FaceAxisA 1/5,
    normal along x exactly, 4 points."""
    q = scenes.quat_from_axis_angle((0.0, 1.0, 0.0), 0.785398163)
    j = _job(3, 3, (1, 1, 1), (1, 1, 1), (1.2, 0.7, 0.3), q)
    r = pyoracle.collide_pairs(j)
    assert _bits(r["normal"][0, 1]) == 0 and _bits(r["normal"][0, 2]) == 0
    assert j["sat_type"][0] == FACE_AXIS_A and j["sat_index_a"][0] == 1 and j["sat_index_b"][0] == 5
    assert r["point_count"][0] == 4


def test_kat_spheres():
    """shape_collision_tests.rs:25: unit spheres 1.5 apart -> normal +x (y, z bits 0), 1 point on
    the x axis, feature id 0."""
    r = pyoracle.collide_pairs(_job(5, 5, (0, 0, 0, 1), (0, 0, 0, 1), (1.5, 0, 0)))
    assert r["point_count"][0] == 1
    assert _bits(r["normal"][0, 1]) == 0 and _bits(r["normal"][0, 2]) == 0
    assert _bits(r["points"][0, 0, 1]) == 0
    assert r["feature_ids"][0, 0] == 0
    assert r["normal"][0, 0] == 1.0 and r["points"][0, 0, 3] == np.float32(-0.5)


def test_kat_capsules():
    """shape_collision_tests.rs:52: parallel capsules 0.8 apart -> 2 points."""
    g = (0, -1, 0, 0, 1, 0, 0.5)
    r = pyoracle.collide_pairs(_job(0, 0, g, g, (0.8, 0, 0)))
    assert r["point_count"][0] == 2


def test_kat_capsule_sphere():
    """shape_collision_tests.rs:90: 1 point."""
    r = pyoracle.collide_pairs(_job(0, 5, (0, 0, 0, 0, 0, 0, 0.5), (0, 0, 0, 1), (1.2, 0.3, 0)))
    assert r["point_count"][0] == 1


def test_kat_hull_sphere():
    """shape_collision_tests.rs:123: 1 point."""
    r = pyoracle.collide_pairs(_job(3, 5, (1, 1, 1), (0, 0, 0, 1), (1.2, 0.5, 0)))
    assert r["point_count"][0] == 1


def test_kat_hull_capsule():
    """shape_collision_tests.rs:157: point-like capsule r 0.25 at x 1.1 against a unit box -> 2 points."""
    r = pyoracle.collide_pairs(_job(3, 0, (1, 1, 1), (0, 0, 0, 0, 0, 0, 0.25), (1.1, 0, 0)))
    assert r["point_count"][0] == 2


def test_pairs_fixture():
    z = np.load(os.path.join(GOLDEN, "pairs.npz"))
    jobs = z["jobs0"].view(pyoracle.PAIR_JOB_DTYPE).copy()
    fresh = _pairgen.make_jobs(pyoracle.PAIR_JOB_DTYPE, len(jobs), 21)
    assert fresh.tobytes() == jobs.tobytes()
    r1 = pyoracle.collide_pairs(jobs)
    assert r1.tobytes() == z["res1"].tobytes() and jobs.tobytes() == z["jobs1"].tobytes()
    r2 = pyoracle.collide_pairs(jobs)
    assert r2.tobytes() == z["res2"].tobytes() and jobs.tobytes() == z["jobs2"].tobytes()


def test_native_timing_build_keeps_the_golden_hash():
    """The CPU baselines time an -O3 -march=native build of the oracle made on the timing host;
    without contraction it must give the same bits (here: many_pyramids, 100 steps, 4 threads)."""
    import subprocess
    import sys
    from conftest import ROOT, TESTS
    script = (
        "import sys, json; sys.path[:0] = [%r, %r]\n"
        "from oracle import pyoracle\n"
        "desc = pyoracle.use_host_native()\n"
        "assert 'march=native' in desc, desc\n"
        "pyoracle.set_threads(4)\n"
        "from test_oracle_pins import _hashes\n"
        "case = json.load(open(%r))['cases']['many_pyramids']\n"
        "assert _hashes('many_pyramids', {}, case['steps'])[-1] == case['hash']\n"
        "print('native ok')\n" % (ROOT, TESTS, os.path.join(GOLDEN, "reference_hashes.json")))
    out = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0 and "native ok" in out.stdout, out.stdout + out.stderr
