"""Regenerate the golden fixtures in this folder from the CPU oracle.

    python tests/golden/make_golden.py

Writes ``oracle_hashes.json`` (per-step FNV-1a world hashes of seeded scenes,
the digest of the reference's World::world_state_hash, body_queries.rs:432)
and ``pairs.npz`` (seeded narrowphase jobs with the oracle's manifolds and
updated caches, two passes so the second runs from warm caches). The oracle is
pinned first: it must reproduce the reference's own published hashes in
``reference_hashes.json`` before anything is written.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from natsel_b200 import scenes  # noqa: E402
from oracle import pyoracle  # noqa: E402
import _pairgen  # noqa: E402

# name, builder kwargs, steps
HASH_CASES = [
    ("box_pyramid", {}, 200),
    ("large_pile", {}, 40),
    ("large_pile", {"n": 2000, "seed": 5, "restitution": 0.4}, 60),
    ("jointed_chains", {"chains": 200, "boxes": 400}, 30),
    ("overflow_pile", {}, 30),
    ("restitution_ball", {"restitution": 0.5, "gap": 0.03}, 60),
]
PAIR_COUNT = 1800
PAIR_SEED = 21


def run_hashes(name, kw, steps):
    w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS[name])
    scenes.BUILDERS[name](w, **kw)
    out = []
    for _ in range(steps):
        w.step(1.0 / 60.0, scenes.SUBSTEPS[name])
        out.append("%016x" % w.state_hash())
    return out


def main():
    ref = json.load(open(os.path.join(HERE, "reference_hashes.json")))
    for name, case in ref["cases"].items():
        got = run_hashes(name, {}, case["steps"])[-1]
        assert got == case["hash"], (name, got, case["hash"])
        print("oracle pinned:", name, got)
    cases = []
    for name, kw, steps in HASH_CASES:
        hashes = run_hashes(name, kw, steps)
        cases.append({"scene": name, "kw": kw, "steps": steps, "substeps": scenes.SUBSTEPS[name],
                      "dt": 1.0 / 60.0, "settings": scenes.WORLD_SETTINGS[name], "hashes": hashes})
        print(name, kw, steps, hashes[-1])
    with open(os.path.join(HERE, "oracle_hashes.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=1)
    jobs = _pairgen.make_jobs(pyoracle.PAIR_JOB_DTYPE, PAIR_COUNT, PAIR_SEED)
    jobs0 = jobs.copy()
    res1 = pyoracle.collide_pairs(jobs)
    jobs1 = jobs.copy()
    res2 = pyoracle.collide_pairs(jobs)
    np.savez_compressed(os.path.join(HERE, "pairs.npz"), jobs0=jobs0.view(np.uint8), res1=res1.view(np.uint8),
                        jobs1=jobs1.view(np.uint8), res2=res2.view(np.uint8), jobs2=jobs.view(np.uint8))
    print("pairs", PAIR_COUNT, "touching", int((res1["point_count"] > 0).sum()))


if __name__ == "__main__":
    main()
