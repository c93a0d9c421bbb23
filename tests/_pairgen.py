"""Seeded random narrowphase jobs for parity tests (shape sizes as in the 10 000-body pile)."""
import numpy as np

CAPSULE, HULL, SPHERE = 0, 3, 5
# (primary A, B): capsule > sphere, hull > sphere/capsule (contact_creation.rs:88-96)
COMBOS = [(HULL, HULL), (HULL, SPHERE), (HULL, CAPSULE), (SPHERE, SPHERE), (CAPSULE, SPHERE), (CAPSULE, CAPSULE)]


def make_jobs(dtype, n, seed, reach=1.6):
    """``n`` jobs cycling through COMBOS; B is placed uniformly within ``reach`` of A with a
    uniform random orientation, so separated, touching and deeply overlapping pairs all occur."""
    rng = np.random.Generator(np.random.PCG64(seed))
    jobs = np.zeros(n, dtype)
    combo = np.array([COMBOS[i % len(COMBOS)] for i in range(n)], np.int32).reshape(n, 2)
    jobs["type_a"], jobs["type_b"] = combo[:, 0], combo[:, 1]
    for side, key in ((0, "geom_a"), (1, "geom_b")):
        t = combo[:, side]
        g = np.zeros((n, 7), np.float32)
        h = rng.uniform(0.25, 0.75, (n, 3))
        r_s = rng.uniform(0.2, 0.6, n)
        hh = rng.uniform(0.2, 0.8, n)
        r_c = rng.uniform(0.15, 0.4, n)
        m = t == HULL
        g[m, 0:3] = h[m]
        m = t == SPHERE
        g[m, 3] = r_s[m]
        m = t == CAPSULE
        g[m, 1] = -hh[m]
        g[m, 4] = hh[m]
        g[m, 6] = r_c[m]
        jobs[key] = g
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    p = rng.uniform(-reach, reach, (n, 3))
    xf = np.concatenate([p, q], 1).astype(np.float32)
    jobs["xf"] = xf
    return jobs
