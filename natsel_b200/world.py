"""Python view of libnatsel_gpu.so, mirroring the reference World API.

The reference engine exposes ``World::create_body``, ``create_hull_shape``
(boxes via ``make_box_hull``), ``create_sphere_shape``,
``create_capsule_shape``, ``create_revolute_joint`` and ``step(dt, substeps)``
(src/simulation/world_runtime.rs:1506, shape_creation.rs:504-569,
revolute_joint.rs:162, solver_integration.rs:807). :class:`World` offers the
same calls over the C ABI declared in ``include/natsel_gpu.h``; there is no
CPU fallback: constructing a World without the CUDA library or a GPU raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnatsel_gpu.so")

STATIC_BODY = 0
KINEMATIC_BODY = 1
DYNAMIC_BODY = 2


class NsError(RuntimeError):
    """A natsel_gpu call returned a non-zero status."""

    def __init__(self, code, message):
        super().__init__(f"natsel_gpu error {code}: {message}")
        self.code = code


class WorldDef(ctypes.Structure):
    _fields_ = [
        ("gravity", ctypes.c_float * 3),
        ("enable_sleep", ctypes.c_int),
        ("enable_continuous", ctypes.c_int),
        ("enable_warm_starting", ctypes.c_int),
        ("contact_hertz", ctypes.c_float),
        ("contact_damping_ratio", ctypes.c_float),
        ("contact_speed", ctypes.c_float),
        ("max_linear_speed", ctypes.c_float),
        ("restitution_threshold", ctypes.c_float),
        ("restitution_iterations", ctypes.c_int),
        ("joint_hertz", ctypes.c_float),
        ("joint_damping_ratio", ctypes.c_float),
        ("contact_capacity", ctypes.c_int),
        ("solver_blocks", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class BodyDef(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int),
        ("position", ctypes.c_double * 3),
        ("rotation", ctypes.c_float * 4),
        ("linear_velocity", ctypes.c_float * 3),
        ("angular_velocity", ctypes.c_float * 3),
        ("linear_damping", ctypes.c_float),
        ("angular_damping", ctypes.c_float),
        ("gravity_scale", ctypes.c_float),
        ("enable_sleep", ctypes.c_int),
        ("is_bullet", ctypes.c_int),
    ]


class ShapeDef(ctypes.Structure):
    _fields_ = [
        ("density", ctypes.c_float),
        ("friction", ctypes.c_float),
        ("restitution", ctypes.c_float),
        ("rolling_resistance", ctypes.c_float),
        ("category_bits", ctypes.c_uint64),
        ("mask_bits", ctypes.c_uint64),
        ("group_index", ctypes.c_int),
    ]


class SphericalJointDef(ctypes.Structure):
    """ns_spherical_joint_def (the reference's SphericalJointDef, types/joint_defs.rs:169)."""
    _fields_ = [
        ("body_a", ctypes.c_int), ("body_b", ctypes.c_int),
        ("local_frame_a", ctypes.c_float * 7), ("local_frame_b", ctypes.c_float * 7),
        ("constraint_hertz", ctypes.c_float), ("constraint_damping_ratio", ctypes.c_float),
        ("collide_connected", ctypes.c_int),
        ("enable_spring", ctypes.c_int), ("hertz", ctypes.c_float), ("damping_ratio", ctypes.c_float),
        ("target_rotation", ctypes.c_float * 4),
        ("enable_cone_limit", ctypes.c_int), ("cone_angle", ctypes.c_float),
        ("enable_twist_limit", ctypes.c_int), ("lower_twist_angle", ctypes.c_float),
        ("upper_twist_angle", ctypes.c_float),
        ("enable_motor", ctypes.c_int), ("max_motor_torque", ctypes.c_float), ("motor_velocity", ctypes.c_float * 3),
    ]


class RevoluteJointDef(ctypes.Structure):
    """ns_revolute_joint_def (the reference's RevoluteJointDef, types/joint_defs.rs:154)."""
    _fields_ = [
        ("body_a", ctypes.c_int), ("body_b", ctypes.c_int),
        ("local_frame_a", ctypes.c_float * 7), ("local_frame_b", ctypes.c_float * 7),
        ("constraint_hertz", ctypes.c_float), ("constraint_damping_ratio", ctypes.c_float),
        ("collide_connected", ctypes.c_int),
        ("target_angle", ctypes.c_float),
        ("enable_spring", ctypes.c_int), ("hertz", ctypes.c_float), ("damping_ratio", ctypes.c_float),
        ("enable_limit", ctypes.c_int), ("lower_angle", ctypes.c_float), ("upper_angle", ctypes.c_float),
        ("enable_motor", ctypes.c_int), ("max_motor_torque", ctypes.c_float), ("motor_speed", ctypes.c_float),
    ]


def revolute_def(cls, default_hertz, default_zeta, body_a, body_b, frame_a, frame_b, enable_limit, lower, upper,
                 enable_spring, hertz, damping_ratio, max_motor_torque, collide_connected, enable_motor,
                 motor_speed, target_angle, constraint_hertz, constraint_damping_ratio):
    """Fill a revolute joint definition struct (``cls``: this module's or the oracle's mirror)."""
    d = cls()
    d.body_a, d.body_b = body_a, body_b
    d.local_frame_a = (ctypes.c_float * 7)(*frame_a)
    d.local_frame_b = (ctypes.c_float * 7)(*frame_b)
    d.constraint_hertz = default_hertz if constraint_hertz is None else constraint_hertz
    d.constraint_damping_ratio = default_zeta if constraint_damping_ratio is None else constraint_damping_ratio
    d.collide_connected = int(collide_connected)
    d.target_angle = target_angle
    d.enable_spring, d.hertz, d.damping_ratio = int(enable_spring), hertz, damping_ratio
    d.enable_limit, d.lower_angle, d.upper_angle = int(enable_limit), lower, upper
    d.enable_motor = int(max_motor_torque > 0.0) if enable_motor is None else int(enable_motor)
    d.max_motor_torque, d.motor_speed = max_motor_torque, motor_speed
    return d


_F3 = ctypes.c_float * 3
_F7 = ctypes.c_float * 7
_lib = None

EXPORTED = [
    "ns_default_world_def", "ns_world_create", "ns_world_destroy", "ns_last_error",
    "ns_create_body", "ns_create_box_shape", "ns_create_sphere_shape", "ns_create_capsule_shape",
    "ns_create_revolute_joint", "ns_default_revolute_joint_def", "ns_create_revolute_joint_def",
    "ns_default_spherical_joint_def", "ns_create_spherical_joint_def", "ns_world_step", "ns_world_synchronize", "ns_world_get_bodies",
    "ns_world_body_count", "ns_world_state_hash", "ns_world_contact_capacity", "ns_world_get_contacts",
    "ns_world_counters", "ns_world_phase_times", "ns_world_stream", "ns_world_solver_counts",
    "ns_collide_pairs", "ns_selftest_barrier_timeout", "ns_world_apply_forces", "ns_collide_pairs_noalloc",
    "ns_world_begin_subworld", "ns_world_subworld_count", "ns_world_subworld_bodies", "ns_world_subworld_hashes",
    "ns_world_tape_begin", "ns_world_tape_end", "ns_world_tape_free", "ns_world_tape_info", "ns_world_vjp",
    "ns_world_vjp_f64", "ns_world_vjp_restitution", "ns_world_autotune", "ns_world_autotune_table", "ns_world_launch_shapes", "ns_world_set_launch_shapes",
    "ns_adjoint_selfcheck",
]


def load_library(path=LIB_PATH):
    """Load libnatsel_gpu.so and declare its signatures. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with natsel_b200._build.build()")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    lib.ns_default_world_def.argtypes = [ctypes.POINTER(WorldDef)]
    lib.ns_world_create.argtypes = [ctypes.POINTER(WorldDef)]
    lib.ns_world_create.restype = P
    lib.ns_world_destroy.argtypes = [P]
    lib.ns_last_error.argtypes = [P]
    lib.ns_last_error.restype = ctypes.c_char_p
    lib.ns_create_body.argtypes = [P, ctypes.POINTER(BodyDef)]
    lib.ns_create_box_shape.argtypes = [P, ctypes.c_int, ctypes.POINTER(ShapeDef)] + [ctypes.c_float] * 3
    lib.ns_create_sphere_shape.argtypes = [P, ctypes.c_int, ctypes.POINTER(ShapeDef), _F3, ctypes.c_float]
    lib.ns_create_capsule_shape.argtypes = [P, ctypes.c_int, ctypes.POINTER(ShapeDef), _F3, _F3, ctypes.c_float]
    lib.ns_create_revolute_joint.argtypes = [P, ctypes.c_int, ctypes.c_int, _F7, _F7, ctypes.c_int,
                                             ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                                             ctypes.c_float, ctypes.c_float, ctypes.c_int]
    lib.ns_default_revolute_joint_def.argtypes = [ctypes.POINTER(RevoluteJointDef)]
    lib.ns_default_revolute_joint_def.restype = None
    lib.ns_create_revolute_joint_def.argtypes = [P, ctypes.POINTER(RevoluteJointDef)]
    lib.ns_default_spherical_joint_def.argtypes = [ctypes.POINTER(SphericalJointDef)]
    lib.ns_default_spherical_joint_def.restype = None
    lib.ns_create_spherical_joint_def.argtypes = [P, ctypes.POINTER(SphericalJointDef)]
    lib.ns_world_autotune_table.argtypes = [P, P, P, P, P, ctypes.c_int]
    lib.ns_world_launch_shapes.argtypes = [P, P]
    lib.ns_world_set_launch_shapes.argtypes = [P, P]
    lib.ns_world_step.argtypes = [P, ctypes.c_float, ctypes.c_int]
    lib.ns_world_synchronize.argtypes = [P]
    lib.ns_world_get_bodies.argtypes = [P, P, P, P, P]
    lib.ns_world_body_count.argtypes = [P]
    lib.ns_world_state_hash.argtypes = [P, ctypes.POINTER(ctypes.c_uint64)]
    lib.ns_world_contact_capacity.argtypes = [P]
    lib.ns_world_get_contacts.argtypes = [P, P, P, P, ctypes.c_int]
    lib.ns_world_counters.argtypes = [P, P]
    lib.ns_world_phase_times.argtypes = [P, P]
    lib.ns_world_stream.argtypes = [P]
    lib.ns_world_stream.restype = P
    lib.ns_world_solver_counts.argtypes = [P, P]
    lib.ns_collide_pairs.argtypes = [P, P, ctypes.c_int]
    lib.ns_collide_pairs_noalloc.argtypes = [P, P, ctypes.c_int]
    lib.ns_selftest_barrier_timeout.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.ns_world_apply_forces.argtypes = [P, P, P]
    lib.ns_world_begin_subworld.argtypes = [P]
    lib.ns_world_subworld_count.argtypes = [P]
    lib.ns_world_subworld_bodies.argtypes = [P, P]
    lib.ns_world_subworld_hashes.argtypes = [P, P]
    lib.ns_world_tape_begin.argtypes = [P, ctypes.c_int]
    lib.ns_world_tape_end.argtypes = [P]
    lib.ns_world_tape_free.argtypes = [P]
    lib.ns_world_tape_info.argtypes = [P, P]
    lib.ns_world_vjp.argtypes = [P] * 11
    lib.ns_world_vjp_f64.argtypes = [P] * 11
    lib.ns_world_vjp_restitution.argtypes = [P, P]
    lib.ns_world_autotune.argtypes = [P, ctypes.c_float, ctypes.c_int, ctypes.c_int, P, P, P, ctypes.c_int]
    lib.ns_adjoint_selfcheck.argtypes = [ctypes.c_int, ctypes.c_int, P]
    _lib = lib
    return lib


def default_world_def(**overrides):
    lib = load_library()
    d = WorldDef()
    lib.ns_default_world_def(ctypes.byref(d))
    for k, v in overrides.items():
        if k == "gravity":
            d.gravity = (ctypes.c_float * 3)(*v)
        else:
            setattr(d, k, v)
    return d


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class World:
    """A device-resident world. Methods follow the reference World API."""

    def __init__(self, world_def=None, **overrides):
        self._lib = load_library()
        d = world_def if world_def is not None else default_world_def(**overrides)
        self._def = d
        self._w = self._lib.ns_world_create(ctypes.byref(d))
        if not self._w:
            raise NsError(1, self._lib.ns_last_error(None).decode())
        self.body_types = []

    def close(self):
        if getattr(self, "_w", None):
            self._lib.ns_world_destroy(self._w)
            self._w = None

    def __del__(self):
        self.close()

    def _check(self, status):
        if status != 0:
            raise NsError(status, self._lib.ns_last_error(self._w).decode())

    def _id(self, value):
        if value < 0:
            raise NsError(1, self._lib.ns_last_error(self._w).decode())
        return value

    # scene construction -------------------------------------------------
    def create_body(self, type=DYNAMIC_BODY, position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0, 1.0),
                    linear_velocity=(0.0, 0.0, 0.0), angular_velocity=(0.0, 0.0, 0.0),
                    linear_damping=0.0, angular_damping=0.0, gravity_scale=1.0, enable_sleep=True,
                    is_bullet=False):
        b = BodyDef()
        b.type = type
        b.position = (ctypes.c_double * 3)(*position)
        b.rotation = (ctypes.c_float * 4)(*rotation)
        b.linear_velocity = (ctypes.c_float * 3)(*linear_velocity)
        b.angular_velocity = (ctypes.c_float * 3)(*angular_velocity)
        b.linear_damping, b.angular_damping, b.gravity_scale = linear_damping, angular_damping, gravity_scale
        b.enable_sleep = 1 if enable_sleep else 0
        b.is_bullet = 1 if is_bullet else 0
        self.body_types.append(type)
        return self._id(self._lib.ns_create_body(self._w, ctypes.byref(b)))

    @staticmethod
    def shape_def(density=1000.0, friction=0.6, restitution=0.0, rolling_resistance=0.0,
                  category_bits=1, mask_bits=0xFFFFFFFFFFFFFFFF, group_index=0):
        s = ShapeDef()
        s.density, s.friction, s.restitution, s.rolling_resistance = density, friction, restitution, rolling_resistance
        s.category_bits, s.mask_bits, s.group_index = category_bits, mask_bits, group_index
        return s

    def create_box(self, body, hx, hy, hz, **shape):
        return self._id(self._lib.ns_create_box_shape(self._w, body, ctypes.byref(self.shape_def(**shape)), hx, hy, hz))

    def create_sphere(self, body, radius, center=(0.0, 0.0, 0.0), **shape):
        return self._id(self._lib.ns_create_sphere_shape(self._w, body, ctypes.byref(self.shape_def(**shape)),
                                                         _F3(*center), radius))

    def create_capsule(self, body, center1, center2, radius, **shape):
        return self._id(self._lib.ns_create_capsule_shape(self._w, body, ctypes.byref(self.shape_def(**shape)),
                                                          _F3(*center1), _F3(*center2), radius))

    def create_revolute(self, body_a, body_b, frame_a, frame_b, enable_limit=False, lower=0.0, upper=0.0,
                        enable_spring=False, hertz=0.0, damping_ratio=0.0, max_motor_torque=0.0,
                        collide_connected=False, enable_motor=None, motor_speed=0.0, target_angle=0.0,
                        constraint_hertz=None, constraint_damping_ratio=None):
        """A revolute joint. With only the first arguments this is ns_create_revolute_joint (a
        positive max_motor_torque is a drag motor of speed 0, softness from the world); any of
        enable_motor, motor_speed, target_angle or the constraint softness goes through
        ns_create_revolute_joint_def with the whole definition."""
        if enable_motor is None and motor_speed == 0.0 and target_angle == 0.0 and constraint_hertz is None \
                and constraint_damping_ratio is None:
            return self._id(self._lib.ns_create_revolute_joint(
                self._w, body_a, body_b, _F7(*frame_a), _F7(*frame_b), int(enable_limit), lower, upper,
                int(enable_spring), hertz, damping_ratio, max_motor_torque, int(collide_connected)))
        d = revolute_def(RevoluteJointDef, self._def.joint_hertz, self._def.joint_damping_ratio, body_a, body_b,
                         frame_a, frame_b, enable_limit, lower, upper, enable_spring, hertz, damping_ratio,
                         max_motor_torque, collide_connected, enable_motor, motor_speed, target_angle,
                         constraint_hertz, constraint_damping_ratio)
        return self._id(self._lib.ns_create_revolute_joint_def(self._w, ctypes.byref(d)))

    def create_spherical(self, body_a, body_b, frame_a, frame_b, collide_connected=False, enable_spring=False,
                         hertz=0.0, damping_ratio=0.0, target_rotation=(0.0, 0.0, 0.0, 1.0), enable_cone_limit=False,
                         cone_angle=0.0, enable_twist_limit=False, lower_twist_angle=0.0, upper_twist_angle=0.0,
                         enable_motor=False, max_motor_torque=0.0, motor_velocity=(0.0, 0.0, 0.0),
                         constraint_hertz=None, constraint_damping_ratio=None):
        """A spherical joint (ns_create_spherical_joint_def; spherical_joint.rs:119). The
        constraint softness defaults to the world's joint softness."""
        d = SphericalJointDef()
        self._lib.ns_default_spherical_joint_def(ctypes.byref(d))
        d.body_a, d.body_b = body_a, body_b
        d.local_frame_a = (ctypes.c_float * 7)(*frame_a)
        d.local_frame_b = (ctypes.c_float * 7)(*frame_b)
        d.constraint_hertz = self._def.joint_hertz if constraint_hertz is None else constraint_hertz
        d.constraint_damping_ratio = (self._def.joint_damping_ratio if constraint_damping_ratio is None
                                      else constraint_damping_ratio)
        d.collide_connected = int(collide_connected)
        d.enable_spring, d.hertz, d.damping_ratio = int(enable_spring), hertz, damping_ratio
        d.target_rotation = (ctypes.c_float * 4)(*target_rotation)
        d.enable_cone_limit, d.cone_angle = int(enable_cone_limit), cone_angle
        d.enable_twist_limit = int(enable_twist_limit)
        d.lower_twist_angle, d.upper_twist_angle = lower_twist_angle, upper_twist_angle
        d.enable_motor, d.max_motor_torque = int(enable_motor), max_motor_torque
        d.motor_velocity = (ctypes.c_float * 3)(*motor_velocity)
        return self._id(self._lib.ns_create_spherical_joint_def(self._w, ctypes.byref(d)))

    # stepping and readback ----------------------------------------------
    def step(self, dt=1.0 / 60.0, substeps=4):
        self._check(self._lib.ns_world_step(self._w, dt, substeps))

    # batched worlds ------------------------------------------------------
    def begin_subworld(self):
        """Start the next independent sub-world; later bodies, shapes and joints belong to it."""
        return self._id(self._lib.ns_world_begin_subworld(self._w))

    @property
    def subworld_count(self):
        return self._lib.ns_world_subworld_count(self._w)

    def subworld_bodies(self):
        """First body id of each sub-world followed by the total body count."""
        out = np.zeros(self.subworld_count + 1, np.int32)
        self._check(self._lib.ns_world_subworld_bodies(self._w, _ptr(out)))
        return out

    def subworld_hashes(self):
        out = np.zeros(self.subworld_count, np.uint64)
        self._check(self._lib.ns_world_subworld_hashes(self._w, _ptr(out)))
        return out

    def apply_forces(self, force=None, torque=None):
        """Add per-body force / torque (float32 arrays, n_bodies x 3) for the next step."""
        f = None if force is None else np.ascontiguousarray(force, np.float32)
        t = None if torque is None else np.ascontiguousarray(torque, np.float32)
        for a in (f, t):
            if a is not None and a.shape != (self.body_count, 3):
                raise ValueError("force/torque must be n_bodies x 3")
        self._check(self._lib.ns_world_apply_forces(self._w, _ptr(f), _ptr(t)))

    def get_bodies_into(self, pos, rot, lin, ang):
        """Readback into caller-owned arrays (for example pinned host buffers); any may be None."""
        def addr(a):
            if a is None:
                return None
            return ctypes.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data)
        self._check(self._lib.ns_world_get_bodies(self._w, addr(pos), addr(rot), addr(lin), addr(ang)))

    def synchronize(self):
        self._check(self._lib.ns_world_synchronize(self._w))

    @property
    def body_count(self):
        return self._lib.ns_world_body_count(self._w)

    def bodies(self):
        n = self.body_count
        pos = np.zeros((n, 3), np.float64)
        rot = np.zeros((n, 4), np.float32)
        lin = np.zeros((n, 3), np.float32)
        ang = np.zeros((n, 3), np.float32)
        self._check(self._lib.ns_world_get_bodies(self._w, _ptr(pos), _ptr(rot), _ptr(lin), _ptr(ang)))
        return pos, rot, lin, ang

    def state_hash(self):
        out = ctypes.c_uint64(0)
        self._check(self._lib.ns_world_state_hash(self._w, ctypes.byref(out)))
        return out.value

    def contacts(self):
        cap = self._lib.ns_world_contact_capacity(self._w)
        cap = max(cap, 1)
        ints = np.zeros((cap, 8), np.int32)
        feats = np.zeros((cap, 4), np.uint32)
        fl = np.zeros((cap, 24), np.float32)
        n = self._lib.ns_world_get_contacts(self._w, _ptr(ints), _ptr(feats), _ptr(fl), cap)
        if n < 0:
            raise NsError(2, self._lib.ns_last_error(self._w).decode())
        return ints[:n], feats[:n], fl[:n]

    def counters(self):
        out = np.zeros(32, np.int32)
        self._check(self._lib.ns_world_counters(self._w, _ptr(out)))
        return out

    def phase_times(self):
        out = np.zeros(5, np.float32)
        self._check(self._lib.ns_world_phase_times(self._w, _ptr(out)))
        return out

    def solver_counts(self):
        out = np.zeros(16, np.int64)
        self._check(self._lib.ns_world_solver_counts(self._w, _ptr(out)))
        return out

    def stream(self):
        return self._lib.ns_world_stream(self._w)

    def autotune(self, dt=1.0 / 60.0, substeps=4, steps=5):
        """Time the solver's candidate launch shapes on this world and keep the fastest (the world
        state is unchanged). Returns [(blocks, cooperative_grid, ms_per_step), ...]."""
        blocks = np.zeros(8, np.int32)
        grid = np.zeros(8, np.int32)
        ms = np.zeros(8, np.float32)
        r = self._lib.ns_world_autotune(self._w, dt, substeps, steps, _ptr(blocks), _ptr(grid), _ptr(ms), 8)
        if r < 0:
            raise NsError(-r, self._lib.ns_last_error(self._w).decode())
        return [(int(blocks[c]), bool(grid[c]), float(ms[c])) for c in range(min(r, 8))]

    TUNE_DIMENSIONS = {0: "solver", 1: "recycle_pass", 2: "manifold_updates", 3: "prepare"}

    def autotune_table(self):
        """Every candidate the last autotune timed: dicts of dimension, a, b, ms_per_step (for the
        solver a = blocks and b = cooperative grid; otherwise threads per block and blocks per SM)."""
        n = self._lib.ns_world_autotune_table(self._w, None, None, None, None, 0)
        if n < 0:
            raise NsError(-n, "autotune_table")
        dim, a, b = (np.zeros(max(n, 1), np.int32) for _ in range(3))
        ms = np.zeros(max(n, 1), np.float32)
        self._lib.ns_world_autotune_table(self._w, _ptr(dim), _ptr(a), _ptr(b), _ptr(ms), n)
        return [{"dimension": self.TUNE_DIMENSIONS[int(dim[r])], "a": int(a[r]), "b": int(b[r]),
                 "ms_per_step": float(ms[r])} for r in range(n)]

    def launch_shapes(self):
        """The launch shapes in use: solver blocks and grid flag, then threads per block and blocks
        per SM of the recycle pass, the manifold updates and the preparation."""
        out = np.zeros(8, np.int32)
        self._check(self._lib.ns_world_launch_shapes(self._w, _ptr(out)))
        keys = ["solver_blocks", "solver_grid", "recycle_threads", "recycle_per_sm", "update_threads",
                "update_per_sm", "prepare_threads", "prepare_per_sm"]
        return {k: int(v) for k, v in zip(keys, out)}

    def set_launch_shapes(self, shapes):
        """Apply launch shapes (a dict as launch_shapes() returns) chosen elsewhere."""
        keys = ["solver_blocks", "solver_grid", "recycle_threads", "recycle_per_sm", "update_threads",
                "update_per_sm", "prepare_threads", "prepare_per_sm"]
        arr = np.array([int(shapes[k]) for k in keys], np.int32)
        self._check(self._lib.ns_world_set_launch_shapes(self._w, _ptr(arr)))

    # ---- adjoint ---------------------------------------------------------------------------
    def tape_begin(self, checkpoint_substeps=8):
        """Record the following steps for vjp(), with a checkpoint every checkpoint_substeps."""
        self._check(self._lib.ns_world_tape_begin(self._w, int(checkpoint_substeps)))

    def tape_end(self):
        self._check(self._lib.ns_world_tape_end(self._w))

    def tape_free(self):
        self._check(self._lib.ns_world_tape_free(self._w))

    def tape_info(self):
        """steps, checkpoints, replay mismatches, vjp calls, recording, checkpoint interval,
        kernel launches of the last vjp, 0."""
        out = np.zeros(8, np.int64)
        self._check(self._lib.ns_world_tape_info(self._w, _ptr(out)))
        return out

    def vjp(self, dpos=None, drot=None, dlin=None, dang=None):
        """Pull cotangents of the final state (body id order) back to the tape's start.

        Returns a dict of float32 arrays: lin0, ang0 (n x 3), mass, friction, restitution (n),
        pos0 (n x 3), rot0 (n x 4)."""
        n = self.body_count
        def arr(a, w):
            if a is None:
                return None
            a = np.ascontiguousarray(a, np.float32)
            if a.shape != (n, w):
                raise ValueError(f"cotangent must be n_bodies x {w}")
            return a
        ins = [arr(dpos, 3), arr(drot, 4), arr(dlin, 3), arr(dang, 3)]
        out = dict(lin0=np.zeros((n, 3), np.float32), ang0=np.zeros((n, 3), np.float32),
                   mass=np.zeros(n, np.float32), friction=np.zeros(n, np.float32),
                   pos0=np.zeros((n, 3), np.float32), rot0=np.zeros((n, 4), np.float32))
        self._check(self._lib.ns_world_vjp(self._w, *[_ptr(a) for a in ins], _ptr(out["lin0"]), _ptr(out["ang0"]),
                                           _ptr(out["mass"]), _ptr(out["friction"]), _ptr(out["pos0"]),
                                           _ptr(out["rot0"])))
        out["restitution"] = np.zeros(n, np.float32)
        self._check(self._lib.ns_world_vjp_restitution(self._w, _ptr(out["restitution"])))
        return out

    def vjp_f64(self, dpos=None, drot=None, dlin=None, dang=None):
        """vjp() with the reverse pass run on the host in f64 (the reference for vjp's f32 pass)."""
        n = self.body_count
        def arr(a, w):
            if a is None:
                return None
            a = np.ascontiguousarray(a, np.float32)
            if a.shape != (n, w):
                raise ValueError(f"cotangent must be n_bodies x {w}")
            return a
        ins = [arr(dpos, 3), arr(drot, 4), arr(dlin, 3), arr(dang, 3)]
        out = dict(lin0=np.zeros((n, 3)), ang0=np.zeros((n, 3)), mass=np.zeros(n), friction=np.zeros(n),
                   pos0=np.zeros((n, 3)), rot0=np.zeros((n, 4)))
        self._check(self._lib.ns_world_vjp_f64(self._w, *[_ptr(a) for a in ins], _ptr(out["lin0"]),
                                               _ptr(out["ang0"]), _ptr(out["mass"]), _ptr(out["friction"]),
                                               _ptr(out["pos0"]), _ptr(out["rot0"])))
        return out


ADJOINT_CHECKS = ["warm_start", "push", "relax", "prepare", "integrate_velocities", "integrate_positions",
                  "finalize_rotation", "inverse_inertia", "recycle", "box_face", "box_any", "box_edge",
                  "warm_start_reverse_sweep", "push_reverse_sweep", "relax_reverse_sweep",
                  "integrate_positions_reverse_sweep", "integrate_velocities_reverse_sweep", "restitution",
                  "relative_velocity_reverse_sweep", "sphere_sphere", "capsule_sphere", "capsule_capsule",
                  "box_sphere", "box_capsule", "joint_solve", "joint_warm_start", "joint_prepare"]


def adjoint_selfcheck(which, seed):
    """f64 check of one local derivative of the adjoint on the host (no GPU): returns the
    worst relative difference between the dual-number VJP and central differences, and the
    separating-axis kind of the box cases (-1 otherwise)."""
    lib = load_library()
    out = np.array([-1.0, -1.0])
    st = lib.ns_adjoint_selfcheck(int(which), int(seed), _ptr(out))
    if st != 0:
        raise NsError(st, lib.ns_last_error(None).decode())
    return float(out[0]), int(out[1])
