"""Batch narrowphase over the C ABI (``ns_collide_pairs``).

One call collides many independent shape pairs on the GPU, one device thread
per pair, with the same routines the world step uses: the reference's
``collide_hulls_with_scratch`` (collision/convex_manifold.rs:1445),
``collide_spheres`` / ``collide_capsule_and_sphere`` / ``collide_capsules`` /
``collide_hull_and_sphere`` / ``collide_hull_and_capsule``
(collision/convex_manifold_shapes.rs:21-643). Jobs are a numpy structured
array laid out exactly like ``ns_pair_job``; the SAT and simplex caches in the
jobs are read and written back, as the reference's ``&mut SATCache`` /
``&mut SimplexCache`` arguments are.
"""
import ctypes

import numpy as np

from .world import NsError, load_library

CAPSULE = 0
HULL = 3
SPHERE = 5

PAIR_JOB_DTYPE = np.dtype([
    ("type_a", "<i4"), ("type_b", "<i4"),
    ("geom_a", "<f4", 7), ("geom_b", "<f4", 7),
    ("xf", "<f4", 7),
    ("sat_separation", "<f4"), ("sat_type", "<i4"), ("sat_index_a", "<i4"), ("sat_index_b", "<i4"),
    ("sat_hit", "<i4"),
    ("simplex_metric", "<f4"), ("simplex_count", "<i4"), ("simplex_ia", "<i4", 4), ("simplex_ib", "<i4", 4),
])
PAIR_RESULT_DTYPE = np.dtype([
    ("normal", "<f4", 3), ("point_count", "<i4"), ("points", "<f4", (4, 4)), ("feature_ids", "<u4", 4),
])
assert PAIR_JOB_DTYPE.itemsize == 152 and PAIR_RESULT_DTYPE.itemsize == 96


def collide_pairs(jobs):
    """Collide ``jobs`` (PAIR_JOB_DTYPE array, updated in place) and return the results."""
    if jobs.dtype != PAIR_JOB_DTYPE or not jobs.flags.c_contiguous:
        raise ValueError("jobs must be a C-contiguous PAIR_JOB_DTYPE array")
    lib = load_library()
    results = np.zeros(len(jobs), PAIR_RESULT_DTYPE)
    if len(jobs) == 0:
        return results
    status = lib.ns_collide_pairs(jobs.ctypes.data_as(ctypes.c_void_p), results.ctypes.data_as(ctypes.c_void_p),
                                  len(jobs))
    if status != 0:
        raise NsError(status, lib.ns_last_error(None).decode())
    return results


NOALLOC_MAX_PAIRS = 4096


def collide_pairs_noalloc(jobs):
    """Same as :func:`collide_pairs` through ``ns_collide_pairs_noalloc``, which allocates no
    device memory (it works in a fixed scratch area inside the library) and therefore takes at
    most NOALLOC_MAX_PAIRS jobs per call. For hosts that cannot call cudaMalloc while running."""
    if jobs.dtype != PAIR_JOB_DTYPE or not jobs.flags.c_contiguous:
        raise ValueError("jobs must be a C-contiguous PAIR_JOB_DTYPE array")
    lib = load_library()
    results = np.zeros(len(jobs), PAIR_RESULT_DTYPE)
    status = lib.ns_collide_pairs_noalloc(jobs.ctypes.data_as(ctypes.c_void_p),
                                          results.ctypes.data_as(ctypes.c_void_p), len(jobs))
    if status != 0:
        raise NsError(status, lib.ns_last_error(None).decode())
    return results
