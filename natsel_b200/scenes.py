"""Seeded synthetic scenes for the rigid-body step.

Every builder takes a world object exposing ``create_body``, ``create_box``,
``create_sphere``, ``create_capsule`` and ``create_revolute`` and returns a
dict describing the scene. Values are generated as float32 (positions
widened to float64 exactly) so the same call sequence builds bit-identical
scenes in any world implementation with this interface.

- :func:`large_pyramid`, :func:`many_pyramids`: the reference benchmark scenes
  (src/bin/benchmarks/scenes.rs:105 and :170), used with the reference's
  golden state hashes.
- :func:`box_pyramid`: a 20-wide pyramid of 1 m cubes (210 bodies).
- :func:`large_pile`: 10 000 mixed boxes/spheres/capsules dropped onto a
  ground box.
- :func:`jointed_chains`: capsule chains linked by limited revolute joints
  with loose boxes falling onto them.
- :func:`overflow_pile`, :func:`restitution_ball`: the reference's own test
  scenes for the overflow colour (tests/simulation/overflow_color_tests.rs:15)
  and restitution (tests/simulation/restitution_phase_tests.rs:36-70).
"""
import numpy as np

STATIC = 0
DYNAMIC = 2
F = np.float32


def _f(x):
    return float(np.float32(x))


def joint_grid(world, n=100):
    """scenes.rs:49 create_joint_grid (default world: gravity -10): an n x n grid of 0.4 m spheres
    (the first row static) in the xy plane, each joined to its upper and left neighbours by a
    spherical joint with the default definition (a point constraint); the spheres' filters keep
    them from colliding with one another."""
    ids = []
    for k in range(n):
        for i in range(n):
            b = world.create_body(type=STATIC if i == 0 else DYNAMIC, position=(float(k), float(-i), 0.0),
                                  enable_sleep=False)
            world.create_sphere(b, 0.4, category_bits=2, mask_bits=0xFFFFFFFFFFFFFFFD)
            if i > 0:
                world.create_spherical(ids[-1], b, (0.0, -0.5, 0.0, 0.0, 0.0, 0.0, 1.0), (0.0, 0.5, 0.0, 0.0, 0.0, 0.0, 1.0))
            if k > 0:
                world.create_spherical(ids[-n], b, (0.5, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0), (-0.5, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0))
            ids.append(b)
    return {"name": "joint_grid", "dynamic_bodies": n * (n - 1)}


def large_pyramid(world, base_count=100):
    """scenes.rs:105 create_large_pyramid (default world: gravity -10)."""
    g = world.create_body(type=STATIC, position=(0.0, -1.0, 0.0))
    world.create_box(g, 400.0, 1.0, 400.0)
    h = F(0.5)
    shift = h
    n = 0
    for i in range(base_count):
        y = (F(2.0) * F(i) + F(1.0)) * shift
        for j in range(i, base_count):
            x = (F(i) + F(1.0)) * shift + F(2.0) * F(j - i) * shift - h * F(base_count)
            b = world.create_body(type=DYNAMIC, position=(float(x), float(y), 0.0))
            world.create_box(b, float(h), float(h), float(h), density=100.0)
            n += 1
    return {"name": "large_pyramid", "dynamic_bodies": n}


def many_pyramids(world, base_count=10, rows=14, cols=14):
    """scenes.rs:170 create_many_pyramids."""
    extent = F(0.5)
    ground_extent = extent * F(cols) * (F(base_count) + F(1.0))
    g = world.create_body(type=STATIC, position=(0.0, -1.0, 0.0))
    world.create_box(g, float(ground_extent), 1.0, float(ground_extent))
    base_width = F(2.0) * extent * F(base_count)
    base_z = -ground_extent + F(2.0) * extent
    delta_z = F(2.0) * (ground_extent - F(2.0) * extent) / F(rows - 1)
    z = base_z
    n = 0
    for _ in range(rows):
        for j in range(cols):
            cx = -ground_extent + F(j) * (base_width + F(2.0) * extent) + F(2.0) * extent
            for i in range(base_count):
                y = (F(2.0) * F(i) + F(1.0)) * extent
                for k in range(i, base_count):
                    x = (F(i) + F(1.0)) * extent + F(2.0) * F(k - i) * extent + cx - F(0.5)
                    b = world.create_body(type=DYNAMIC, position=(float(x), float(y), float(z)), enable_sleep=False)
                    world.create_box(b, float(extent), float(extent), float(extent), density=100.0)
                    n += 1
        z = z + delta_z
    return {"name": "many_pyramids", "dynamic_bodies": n}


def box_pyramid(world, base=20, seed=1):
    """20-wide pyramid of 1 m cubes (base 20 -> 210 cubes), 1.05 m spacing with x/z jitter."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = world.create_body(type=STATIC, position=(0.0, -0.5, 0.0))
    world.create_box(g, 50.0, 0.5, 50.0, friction=0.6)
    n = 0
    for i in range(base):
        count = base - i
        for j in range(count):
            jx, jz = rng.uniform(-0.01, 0.01, 2).astype(np.float32)
            x = F((F(j) - F(0.5) * F(count - 1)) * F(1.05)) + jx
            y = F(0.5) + F(1.0) * F(i)
            b = world.create_body(type=DYNAMIC, position=(float(x), float(y), float(jz)))
            world.create_box(b, 0.5, 0.5, 0.5, density=1000.0, friction=0.6, restitution=0.0)
            n += 1
    return {"name": "box_pyramid", "dynamic_bodies": n}


def _random_quats(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.astype(np.float32)


GROUND_HALF_HEIGHT = 5.0


def large_pile(world, n=10000, seed=2, ground_half=50.0, restitution=0.0, spread=20.0, drop=(1.0, 61.0),
               ground_half_height=0.5):
    """10 000 dynamic bodies (60% boxes, 25% spheres, 15% capsules) dropped from a 40x60x40 m volume
    onto a 100 x 1 x 100 m ground box with its top at y = 0 (``ground_half_height`` sets its half
    thickness). ``restitution`` > 0 gives every shape that coefficient (exercises the restitution
    stage). Bodies dropped from 61 m arrive at up to 35 m/s (0.58 m per step); the world runs
    with continuous collision on (the reference's default), which sweeps the fast ones against
    the ground."""
    rng = np.random.Generator(np.random.PCG64(seed))
    hy = float(ground_half_height)
    g = world.create_body(type=STATIC, position=(0.0, -hy, 0.0))
    world.create_box(g, ground_half, hy, ground_half, friction=0.6)
    n_box = int(round(0.6 * n))
    n_sph = int(round(0.25 * n))
    kinds = np.array([0] * n_box + [1] * n_sph + [2] * (n - n_box - n_sph))
    rng.shuffle(kinds)
    pos = np.stack([rng.uniform(-spread, spread, n), rng.uniform(drop[0], drop[1], n), rng.uniform(-spread, spread, n)],
                   1).astype(np.float32)
    quats = _random_quats(rng, n)
    box_h = rng.uniform(0.25, 0.75, (n, 3)).astype(np.float32)
    sph_r = rng.uniform(0.2, 0.6, n).astype(np.float32)
    cap_r = rng.uniform(0.15, 0.4, n).astype(np.float32)
    cap_hh = rng.uniform(0.2, 0.8, n).astype(np.float32)
    density = rng.uniform(500.0, 2000.0, n).astype(np.float32)
    friction = rng.uniform(0.3, 0.9, n).astype(np.float32)
    for i in range(n):
        b = world.create_body(type=DYNAMIC, position=tuple(float(v) for v in pos[i]),
                              rotation=tuple(float(v) for v in quats[i]))
        mat = dict(density=float(density[i]), friction=float(friction[i]), restitution=float(restitution))
        if kinds[i] == 0:
            world.create_box(b, float(box_h[i, 0]), float(box_h[i, 1]), float(box_h[i, 2]), **mat)
        elif kinds[i] == 1:
            world.create_sphere(b, float(sph_r[i]), **mat)
        else:
            hh = float(cap_hh[i])
            world.create_capsule(b, (0.0, -hh, 0.0), (0.0, hh, 0.0), float(cap_r[i]), **mat)
    return {"name": "large_pile", "dynamic_bodies": n, "boxes": n_box, "spheres": n_sph,
            "capsules": n - n_box - n_sph}


def _axis_angle_quat(axis, angle):
    s, c = np.sin(0.5 * angle), np.cos(0.5 * angle)
    return (float(F(axis[0] * s)), float(F(axis[1] * s)), float(F(axis[2] * s)), float(F(c)))


def jointed_chains(world, chains=2000, links=24, boxes=4000, seed=3, grid=45, spacing=2.0, height=30.0):
    """Capsule chains (r 0.1, half-height 0.25) on revolute joints limited to +-60 degrees,
    plus loose boxes (half-extent 0.3) falling onto them. The ground is 10 m thick (top at
    y = 0) for the same reason as in :func:`large_pile`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = world.create_body(type=STATIC, position=(0.0, -GROUND_HALF_HEIGHT, 0.0))
    world.create_box(g, 100.0, GROUND_HALF_HEIGHT, 100.0, friction=0.6)
    r, hh = 0.1, 0.25
    link = 2.0 * hh
    limit = float(F(np.pi / 3.0))
    n_joints = 0
    half = 0.5 * (grid - 1) * spacing
    for c in range(chains):
        gx, gz = c % grid, c // grid
        ax, az = gx * spacing - half, gz * spacing - half
        anchor = world.create_body(type=STATIC, position=(float(F(ax)), float(F(height)), float(F(az))))
        prev = anchor
        prev_frame = (0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0)
        angles = rng.uniform(-0.3, 0.3, links).astype(np.float32)
        for k in range(links):
            y = height - (k + 0.5) * link
            b = world.create_body(type=DYNAMIC, position=(float(F(ax)), float(F(y)), float(F(az))))
            world.create_capsule(b, (0.0, -hh, 0.0), (0.0, hh, 0.0), r, density=1000.0, friction=0.6)
            q = _axis_angle_quat((0.0, 0.0, 1.0), float(angles[k]))
            frame_b = (0.0, hh, 0.0) + q
            world.create_revolute(prev, b, prev_frame, frame_b, enable_limit=True, lower=-limit, upper=limit)
            n_joints += 1
            prev = b
            prev_frame = (0.0, -hh, 0.0, 0.0, 0.0, 0.0, 1.0)
    pos = np.stack([rng.uniform(-half, half, boxes), rng.uniform(height + 2.0, height + 22.0, boxes),
                    rng.uniform(-half, half, boxes)], 1).astype(np.float32)
    quats = _random_quats(rng, boxes)
    for i in range(boxes):
        b = world.create_body(type=DYNAMIC, position=tuple(float(v) for v in pos[i]),
                              rotation=tuple(float(v) for v in quats[i]))
        world.create_box(b, 0.3, 0.3, 0.3, density=1000.0, friction=0.6)
    return {"name": "jointed_chains", "dynamic_bodies": chains * links + boxes, "joints": n_joints}


def _batch_plan(index, seed):
    """The seeded draws of batch world ``index``: (kind, N, rng positioned after them)."""
    rng = np.random.Generator(np.random.PCG64([seed, index]))
    n = int(np.exp(rng.uniform(np.log(32.0), np.log(512.0))))
    kind = "pyramid" if rng.uniform() < 0.5 else "drop"
    return kind, n, rng


def _pyramid_base(n):
    return max(2, int((np.sqrt(8 * n + 1) - 1) / 2))


def batch_world_size(index, seed=4):
    """Dynamic bodies of batch world ``index`` without building it (a pyramid of base b holds
    b (b + 1) / 2 cubes; a drop holds N bodies)."""
    kind, n, _ = _batch_plan(index, seed)
    if kind == "pyramid":
        b = _pyramid_base(n)
        return b * (b + 1) // 2
    return n


def batch_world(world, index, seed=4):
    """One world of the batched-worlds workload: N ~ log-uniform(32, 512) bodies, either a box
    pyramid of about N cubes or a random drop of N bodies with the 10 000-body pile's shape mix
    and parameter ranges (dropped from its volume scaled to N at the same density), seeded by
    (seed, index)."""
    kind, n, rng = _batch_plan(index, seed)
    if kind == "pyramid":
        info = box_pyramid(world, base=_pyramid_base(n), seed=int(rng.integers(1 << 30)))
        return {"kind": "pyramid", "dynamic_bodies": info["dynamic_bodies"]}
    # the 10 000-body pile's 40 x 60 x 40 m volume scaled to N at the same initial density
    scale = (n / 10000.0) ** (1.0 / 3.0)
    spread = float(np.float32(20.0 * scale))
    height = float(np.float32(60.0 * scale))
    info = large_pile(world, n=n, seed=int(rng.integers(1 << 30)), ground_half=max(10.0, 2.5 * spread),
                      spread=spread, drop=(1.0, 1.0 + height), ground_half_height=GROUND_HALF_HEIGHT)
    return {"kind": "drop", "dynamic_bodies": info["dynamic_bodies"]}


def batched_worlds(world, count=4096, seed=4, indices=None):
    """``count`` independent worlds (batch_world) in one world object, one sub-world each;
    ``indices`` builds only those worlds of the batch (one rank's share), in that order."""
    total, kinds = 0, []
    picks = range(count) if indices is None else indices
    for k, index in enumerate(picks):
        if k > 0:
            world.begin_subworld()
        info = batch_world(world, int(index), seed)
        total += info["dynamic_bodies"]
        kinds.append(info["kind"])
    return {"name": "batched_worlds", "worlds": len(kinds), "dynamic_bodies": total, "kinds": kinds}


PI = F(3.14159265359)  # base/constants.rs:6


def unwind_angle(radians):
    """math/functions.rs:134 unwind_angle: IEEE remainder by 2*pi, computed exactly in float64."""
    x = float(F(radians))
    period = float(F(2.0) * PI)
    n = float(np.round(x / period))  # numpy rounds half to even
    r = x - n * period
    if r > 0.5 * period:
        n += 1.0
        r = x - n * period
    elif r < -0.5 * period:
        n -= 1.0
        r = x - n * period
    return F(r)


def compute_cos_sin(radians):
    """math/functions.rs:101 compute_cos_sin (rational approximation, float32 throughout)."""
    x = unwind_angle(radians)
    pi2 = PI * PI
    if x < F(-0.5) * PI:
        y = x + PI
        y2 = y * y
        c = -(pi2 - F(4.0) * y2) / (pi2 + y2)
    elif x > F(0.5) * PI:
        y = x - PI
        y2 = y * y
        c = -(pi2 - F(4.0) * y2) / (pi2 + y2)
    else:
        y2 = x * x
        c = (pi2 - F(4.0) * y2) / (pi2 + y2)
    if x < F(0.0):
        y = x + PI
        s = F(-16.0) * y * (PI - y) / (F(5.0) * pi2 - F(4.0) * y * (PI - y))
    else:
        s = F(16.0) * x * (PI - x) / (F(5.0) * pi2 - F(4.0) * x * (PI - x))
    mag = np.sqrt(s * s + c * c)
    inv = F(1.0) / mag if mag > F(0.0) else F(0.0)
    return F(c * inv), F(s * inv)


def quat_from_axis_angle(axis, radians):
    """math/functions.rs:461 make_quat_from_axis_angle, as (x, y, z, s)."""
    c, s = compute_cos_sin(F(0.5) * F(radians))
    return (float(F(s * F(axis[0]))), float(F(s * F(axis[1]))), float(F(s * F(axis[2]))), float(c))


def overflow_pile(world, ring_count=5, per_ring=5):
    """overflow_color_tests.rs:15 create_overflow_color_pile: a tall hub box ringed by 25 small
    boxes in 5 staggered layers, enough dynamic neighbours to populate the overflow colour."""
    g = world.create_body(type=STATIC, position=(0.0, -1.0, 0.0))
    world.create_box(g, 20.0, 1.0, 20.0)
    hub = world.create_body(type=DYNAMIC, position=(0.0, 2.5, 0.0))
    world.create_box(hub, 0.5, 2.5, 0.5, density=50.0)
    half = F(0.2)
    ring_radius = F(0.5) + half - F(0.03)
    base_y = half + F(0.05)
    n = 0
    for ring in range(ring_count):
        y = base_y + F(0.5) * F(ring)
        offset = PI / F(per_ring) if ring & 1 else F(0.0)
        for slot in range(per_ring):
            theta = offset + (F(2.0) * PI * F(slot)) / F(per_ring)
            c, s = compute_cos_sin(theta)
            b = world.create_body(type=DYNAMIC, position=(float(F(ring_radius * c)), float(y), float(F(ring_radius * s))))
            world.create_box(b, float(half), float(half), float(half))
            n += 1
    return {"name": "overflow_pile", "dynamic_bodies": n + 1}


def restitution_ball(world, restitution=0.5, gap=0.0, speed=5.0):
    """restitution_phase_tests.rs:36-70: a frictionless ball of radius 0.5 driven at ``speed``
    into a frictionless static ground (top at y = 0) from ``gap`` above contact; run with
    gravity 0. Returns the ball's body id."""
    g = world.create_body(type=STATIC, position=(0.0, -1.0, 0.0))
    world.create_box(g, 40.0, 1.0, 40.0, friction=0.0, restitution=float(restitution))
    ball = world.create_body(type=DYNAMIC, position=(0.0, float(F(F(0.5) + F(gap))), 0.0),
                             linear_velocity=(0.0, -float(speed), 0.0))
    world.create_sphere(ball, 0.5, friction=0.0, restitution=float(restitution))
    return {"name": "restitution_ball", "dynamic_bodies": 1, "ball": ball}


def differentiable_rollout(world, count=1024, seed=5, spacing=1.25, perturb=None):
    """1024 unit cubes (half-extent 0.5 m) on a 32 x 32 grid, resting 2 mm into a ground box,
    with initial linear velocities N(0, 2^2) m/s and angular velocities N(0, 1) rad/s per
    component; density 1000, friction 0.6. Returns the seeded target positions of the
    rollout's loss sum |x_final - x_target|^2 (the initial positions plus N(0, 0.5^2) m).
    ``perturb`` = (what, body, component, delta) moves one input ("v0", "density" or
    "friction") for finite differences; the value applied (f32 where the API takes f32) is
    returned as ``perturbed_value``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = world.create_body(type=STATIC, position=(0.0, -0.5, 0.0))
    world.create_box(g, 40.0, 0.5, 40.0, friction=0.6)
    side = int(round(count ** 0.5))
    pos = np.zeros((count, 3))
    v0 = rng.normal(0.0, 2.0, (count, 3)).astype(np.float32)
    w0 = rng.normal(0.0, 1.0, (count, 3)).astype(np.float32)
    density = np.full(count, 1000.0)
    friction = np.full(count, 0.6)
    value = None
    if perturb is not None:
        what, body, comp, delta = perturb
        if what == "v0":
            v0[body, comp] = np.float32(float(v0[body, comp]) + delta)
            value = float(v0[body, comp])
        elif what == "density":
            density[body] += delta
            value = float(np.float32(density[body]))
        else:
            friction[body] += delta
            value = float(np.float32(friction[body]))
    for k in range(count):
        i, j = divmod(k, side)
        pos[k] = ((i - 0.5 * (side - 1)) * spacing, 0.498, (j - 0.5 * (side - 1)) * spacing)
        b = world.create_body(type=DYNAMIC, position=tuple(pos[k]), linear_velocity=tuple(map(float, v0[k])),
                              angular_velocity=tuple(map(float, w0[k])), enable_sleep=False)
        world.create_box(b, 0.5, 0.5, 0.5, density=float(density[k]), friction=float(friction[k]))
    targets = pos + rng.normal(0.0, 0.5, (count, 3))
    return {"name": "differentiable_rollout", "dynamic_bodies": count, "targets": targets, "perturbed_value": value}


WORLD_SETTINGS = {
    # gravity per scene: the reference scenes use the World default (-10); the synthetic
    # configurations use -9.81. The 10 000-body pile runs with continuous collision on, as the
    # reference World does by default; the other synthetic scenes keep it off (their bodies never
    # move fast enough to need it: the batched worlds' drops are short and sit on a 10 m ground).
    "large_pyramid": dict(gravity=(0.0, -10.0, 0.0), enable_continuous=True),
    "joint_grid": dict(gravity=(0.0, -10.0, 0.0), enable_continuous=True),
    "many_pyramids": dict(gravity=(0.0, -10.0, 0.0), enable_continuous=True),
    "box_pyramid": dict(gravity=(0.0, -9.81, 0.0), enable_continuous=False),
    "large_pile": dict(gravity=(0.0, -9.81, 0.0), enable_continuous=True),
    "jointed_chains": dict(gravity=(0.0, -9.81, 0.0), enable_continuous=False),
    "overflow_pile": dict(gravity=(0.0, -10.0, 0.0), enable_continuous=True),
    "batched_worlds": dict(gravity=(0.0, -9.81, 0.0), enable_continuous=False),
    "restitution_ball": dict(gravity=(0.0, 0.0, 0.0), enable_continuous=True),
    "differentiable_rollout": dict(gravity=(0.0, -9.81, 0.0), enable_continuous=False),
}

SUBSTEPS = {"joint_grid": 4, "large_pyramid": 4, "many_pyramids": 4, "box_pyramid": 4, "large_pile": 4, "jointed_chains": 8,
            "overflow_pile": 4, "restitution_ball": 4, "batched_worlds": 4, "differentiable_rollout": 4}

BUILDERS = {
    "joint_grid": joint_grid,
    "large_pyramid": large_pyramid,
    "many_pyramids": many_pyramids,
    "box_pyramid": box_pyramid,
    "large_pile": large_pile,
    "jointed_chains": jointed_chains,
    "overflow_pile": overflow_pile,
    "restitution_ball": restitution_ball,
    "batched_worlds": batched_worlds,
    "differentiable_rollout": differentiable_rollout,
}
