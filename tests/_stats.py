"""Trajectory statistics for comparing an FP32 run with the FP64 oracle run of the same scene:
chaos rules out pointwise agreement over hundreds of steps, so the runs are compared by energy,
penetration and resting-contact statistics (the reference's own tolerance tests follow the same
pattern, e.g. restitution_quality_tests.rs:138-175)."""
import numpy as np


def trajectory_stats(world, gravity=9.81, ground_half=50.0):
    """Statistics of one world state (a natsel_b200 World or an oracle world):

    - ``energy``: sum over dynamic bodies still above the ground box of 0.5 |v|^2 + g y
      (energy per unit mass; bodies that rolled off the ground's edge are counted apart);
    - ``speed``: mean linear speed of those bodies;
    - ``median_height``: their median centre height;
    - ``off_ground``: dynamic bodies that left the ground box (fell past its edge);
    - ``touching``: touching contacts (manifolds with at least one point), the resting-contact
      count of a settled pile;
    - ``max_penetration`` / ``p999_penetration`` / ``p99_penetration``: the deepest, the
      99.9th- and the 99th-percentile depth over every manifold point (depth = -separation)."""
    pos, rot, lin, ang = world.bodies()
    dyn = np.array(world.body_types) == 2
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    on = dyn & (np.abs(x) < ground_half) & (np.abs(z) < ground_half) & (y > -1.0)
    v = lin.astype(np.float64)
    energy = float(np.sum(0.5 * np.sum(v[on] ** 2, 1) + gravity * y[on]))
    ints, feats, fl = world.contacts()
    pc = ints[:, 4]
    seps = np.concatenate([fl[pc > k, 3 + 5 * k + 3] for k in range(4)]).astype(np.float64)
    depth = -seps if len(seps) else np.zeros(1)
    return {
        "energy": energy,
        "speed": float(np.mean(np.linalg.norm(v[on], axis=1))) if on.any() else 0.0,
        "median_height": float(np.median(y[on])) if on.any() else 0.0,
        "off_ground": int((dyn & ~on).sum()),
        "touching": int((pc > 0).sum()),
        "max_penetration": float(depth.max()),
        "p999_penetration": float(np.quantile(depth, 0.999)),
        "p99_penetration": float(np.quantile(depth, 0.99)),
    }


def mean_stats(rows):
    return {k: float(np.mean([r[k] for r in rows])) for k in rows[0]}
