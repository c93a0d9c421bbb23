"""ctypes wrapper of the oracle (libns_oracle.so).

TEST INFRASTRUCTURE ONLY. The oracle is the CPU restatement of the
reference's scalar world step; tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it as the parity checker. The product package never
imports this module. The method names match natsel_b200.world.World so one
scene builder drives both.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libns_oracle.so")
SOURCES = ["ns_world.cpp", "ns_math.hpp", "ns_collide.hpp", "ns_joint.hpp", "ns_oracle.h"]

STATIC_BODY = 0
KINEMATIC_BODY = 1
DYNAMIC_BODY = 2


LIB64_PATH = os.path.join(HERE, "libns_oracle64.so")


def build(force=False):
    """Compile libns_oracle.so (IEEE f32, no contraction) and libns_oracle64.so (the same sources
    in f64) with g++."""
    if not force and all(os.path.exists(p) for p in (LIB_PATH, LIB64_PATH)):
        t = min(os.path.getmtime(LIB_PATH), os.path.getmtime(LIB64_PATH))
        if all(os.path.getmtime(os.path.join(HERE, s)) <= t for s in SOURCES):
            return LIB_PATH
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


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


class RevoluteDef(ctypes.Structure):
    """nso_revolute_def: the reference's RevoluteJointDef (types/joint_defs.rs:154)."""
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


class SphericalDef(ctypes.Structure):
    """nso_spherical_def: the reference's SphericalJointDef (types/joint_defs.rs:169)."""
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


def fill_spherical_def(d, default_hertz, default_zeta, body_a, body_b, frame_a, frame_b, collide_connected=False,
                       enable_spring=False, hertz=0.0, damping_ratio=0.0, target_rotation=(0.0, 0.0, 0.0, 1.0),
                       enable_cone_limit=False, cone_angle=0.0, enable_twist_limit=False, lower_twist_angle=0.0,
                       upper_twist_angle=0.0, enable_motor=False, max_motor_torque=0.0,
                       motor_velocity=(0.0, 0.0, 0.0), constraint_hertz=None, constraint_damping_ratio=None):
    """Fill a spherical joint definition (the oracle's or the product's mirror struct)."""
    d.body_a, d.body_b = body_a, body_b
    d.local_frame_a = (ctypes.c_float * 7)(*frame_a)
    d.local_frame_b = (ctypes.c_float * 7)(*frame_b)
    d.constraint_hertz = default_hertz if constraint_hertz is None else constraint_hertz
    d.constraint_damping_ratio = default_zeta if constraint_damping_ratio is None else constraint_damping_ratio
    d.collide_connected = int(collide_connected)
    d.enable_spring, d.hertz, d.damping_ratio = int(enable_spring), hertz, damping_ratio
    d.target_rotation = (ctypes.c_float * 4)(*target_rotation)
    d.enable_cone_limit, d.cone_angle = int(enable_cone_limit), cone_angle
    d.enable_twist_limit = int(enable_twist_limit)
    d.lower_twist_angle, d.upper_twist_angle = lower_twist_angle, upper_twist_angle
    d.enable_motor, d.max_motor_torque = int(enable_motor), max_motor_torque
    d.motor_velocity = (ctypes.c_float * 3)(*motor_velocity)
    return d


def _revolute_def(default_hertz, default_zeta, body_a, body_b, frame_a, frame_b, enable_limit, lower, upper,
                  enable_spring, hertz, damping_ratio, max_motor_torque, collide_connected, enable_motor,
                  motor_speed, target_angle, constraint_hertz, constraint_damping_ratio):
    d = RevoluteDef()
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
_lib_path = None


def use_host_native():
    """Switch this process to an oracle built with -march=native for the host it runs on (the
    CPU-baseline timing build: -O3 -ffp-contract=off, as the portable build, plus the host's
    vector extensions, which change no bits without contraction). Must run before the first
    oracle call. Returns a one-line description of the build that will be used."""
    global _lib_path
    if _lib is not None:
        raise RuntimeError("use_host_native() must run before the oracle is loaded")
    import tempfile
    out = os.path.join(tempfile.mkdtemp(prefix="ns_oracle_"), "libns_oracle_native.so")
    r = subprocess.run(["make", "-s", "-C", HERE, "native", "OUT=" + out], capture_output=True, text=True)
    if r.returncode != 0 or not os.path.exists(out):
        build()
        return "portable -O3 build (the -march=native build failed: %s)" % (r.stderr.strip().splitlines() or ["?"])[-1]
    _lib_path = out
    return "-O3 -march=native -ffp-contract=off, built on this host"


_lib64 = None


def load(precision="f32"):
    """The oracle library: "f32" is the parity oracle (the reference's arithmetic), "f64" the
    same step with every scalar in double (the trajectory-statistics reference)."""
    global _lib, _lib64
    if precision == "f64":
        if _lib64 is None:
            build()
            _lib64 = _declare(ctypes.CDLL(LIB64_PATH))
        return _lib64
    if _lib is not None:
        return _lib
    if _lib_path is None:
        build()
    _lib = _declare(ctypes.CDLL(_lib_path or LIB_PATH))
    return _lib


def _declare(lib):
    P = ctypes.c_void_p
    lib.nso_default_world_def.argtypes = [ctypes.POINTER(WorldDef)]
    lib.nso_create.argtypes = [ctypes.POINTER(WorldDef)]
    lib.nso_create.restype = P
    lib.nso_destroy.argtypes = [P]
    lib.nso_set_threads.argtypes = [ctypes.c_int]
    lib.nso_create_body.argtypes = [P, ctypes.POINTER(BodyDef)]
    lib.nso_create_box.argtypes = [P, ctypes.c_int, ctypes.POINTER(ShapeDef)] + [ctypes.c_float] * 3
    lib.nso_create_sphere.argtypes = [P, ctypes.c_int, ctypes.POINTER(ShapeDef), _F3, ctypes.c_float]
    lib.nso_create_capsule.argtypes = [P, ctypes.c_int, ctypes.POINTER(ShapeDef), _F3, _F3, ctypes.c_float]
    lib.nso_create_revolute.argtypes = [P, ctypes.c_int, ctypes.c_int, _F7, _F7, ctypes.c_int, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_int]
    lib.nso_create_revolute_def.argtypes = [P, ctypes.POINTER(RevoluteDef)]
    lib.nso_create_spherical_def.argtypes = [P, ctypes.POINTER(SphericalDef)]
    lib.nso_step.argtypes = [P, ctypes.c_float, ctypes.c_int]
    lib.nso_state_hash.argtypes = [P]
    lib.nso_state_hash.restype = ctypes.c_uint64
    lib.nso_body_count.argtypes = [P]
    lib.nso_get_bodies.argtypes = [P, P, P, P, P]
    lib.nso_contact_capacity.argtypes = [P]
    lib.nso_get_contacts.argtypes = [P, P, P, P]
    lib.nso_counters.argtypes = [P, P]
    lib.nso_collide_pairs.argtypes = [P, P, ctypes.c_int]
    lib.nso_apply_forces.argtypes = [P, P, P]
    lib.nso_time_of_impact.argtypes = [P, ctypes.c_int, ctypes.c_float, P, ctypes.c_int, ctypes.c_float, P, P,
                                       ctypes.c_float, P]
    lib.nso_time_of_impact.restype = None
    return lib


TOI_STATES = {0: "unknown", 1: "failed", 2: "overlapped", 3: "hit", 4: "separated"}


def time_of_impact(points_a, radius_a, points_b, radius_b, sweep_a, sweep_b, max_fraction=1.0, precision="f32"):
    """collision/time_of_impact.rs:391 on two point proxies and sweeps (local_center, c1, c2, q1,
    q2 with quaternions as x, y, z, s). Returns a dict of the TOIOutput fields."""
    pa = np.ascontiguousarray(points_a, np.float32).reshape(-1, 3)
    pb = np.ascontiguousarray(points_b, np.float32).reshape(-1, 3)
    sa = np.ascontiguousarray(np.concatenate([np.ravel(x) for x in sweep_a]), np.float32)
    sb = np.ascontiguousarray(np.concatenate([np.ravel(x) for x in sweep_b]), np.float32)
    assert sa.size == 17 and sb.size == 17
    out = np.zeros(13, np.float32)
    load(precision).nso_time_of_impact(_ptr(pa), len(pa), radius_a, _ptr(pb), len(pb), radius_b, _ptr(sa), _ptr(sb),
                                       max_fraction, _ptr(out))
    return {"state": TOI_STATES[int(out[0])], "fraction": out[1], "distance": out[2], "point": out[3:6].copy(),
            "normal": out[6:9].copy(), "distance_iterations": int(out[9]), "push_back_iterations": int(out[10]),
            "root_iterations": int(out[11])}


def set_threads(threads):
    """Host threads of the oracle's colour-parallel loops (every world in the process; default 1).
    Any count gives the same bits: each parallel loop touches disjoint data."""
    load().nso_set_threads(int(threads))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleWorld:
    """CPU oracle world with the same scene-building calls as natsel_b200.World."""

    def __init__(self, gravity=(0.0, -10.0, 0.0), enable_continuous=True, enable_warm_starting=True,
                 precision="f32", **overrides):
        self._lib = load(precision)
        d = WorldDef()
        self._lib.nso_default_world_def(ctypes.byref(d))
        d.gravity = (ctypes.c_float * 3)(*gravity)
        d.enable_continuous = int(enable_continuous)
        d.enable_warm_starting = int(enable_warm_starting)
        for k, v in overrides.items():
            if hasattr(d, k):
                setattr(d, k, v)
        self._def = d
        self._w = self._lib.nso_create(ctypes.byref(d))
        self.body_types = []

    def close(self):
        if getattr(self, "_w", None):
            self._lib.nso_destroy(self._w)
            self._w = None

    def __del__(self):
        self.close()

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
        return self._lib.nso_create_body(self._w, ctypes.byref(b))

    @staticmethod
    def shape_def(density=1000.0, friction=0.6, restitution=0.0, rolling_resistance=0.0,
                  category_bits=1, mask_bits=0xFFFFFFFFFFFFFFFF, group_index=0):
        s = ShapeDef()
        s.density, s.friction, s.restitution, s.rolling_resistance = density, friction, restitution, rolling_resistance
        s.category_bits, s.mask_bits, s.group_index = category_bits, mask_bits, group_index
        return s

    def create_box(self, body, hx, hy, hz, **shape):
        return self._lib.nso_create_box(self._w, body, ctypes.byref(self.shape_def(**shape)), hx, hy, hz)

    def create_sphere(self, body, radius, center=(0.0, 0.0, 0.0), **shape):
        return self._lib.nso_create_sphere(self._w, body, ctypes.byref(self.shape_def(**shape)), _F3(*center), radius)

    def create_capsule(self, body, center1, center2, radius, **shape):
        return self._lib.nso_create_capsule(self._w, body, ctypes.byref(self.shape_def(**shape)),
                                            _F3(*center1), _F3(*center2), radius)

    def create_revolute(self, body_a, body_b, frame_a, frame_b, enable_limit=False, lower=0.0, upper=0.0,
                        enable_spring=False, hertz=0.0, damping_ratio=0.0, max_motor_torque=0.0,
                        collide_connected=False, enable_motor=None, motor_speed=0.0, target_angle=0.0,
                        constraint_hertz=None, constraint_damping_ratio=None):
        if enable_motor is None and motor_speed == 0.0 and target_angle == 0.0 and constraint_hertz is None \
                and constraint_damping_ratio is None:
            return self._lib.nso_create_revolute(self._w, body_a, body_b, _F7(*frame_a), _F7(*frame_b),
                                                 int(enable_limit), lower, upper, int(enable_spring), hertz,
                                                 damping_ratio, max_motor_torque, int(collide_connected))
        d = _revolute_def(self._def.joint_hertz, self._def.joint_damping_ratio, body_a, body_b, frame_a, frame_b,
                          enable_limit, lower, upper, enable_spring, hertz, damping_ratio, max_motor_torque,
                          collide_connected, enable_motor, motor_speed, target_angle, constraint_hertz,
                          constraint_damping_ratio)
        return self._lib.nso_create_revolute_def(self._w, ctypes.byref(d))

    def create_spherical(self, body_a, body_b, frame_a, frame_b, **kw):
        """A spherical joint (spherical_joint.rs:119); keywords as fill_spherical_def."""
        d = fill_spherical_def(SphericalDef(), self._def.joint_hertz, self._def.joint_damping_ratio, body_a, body_b,
                               frame_a, frame_b, **kw)
        return self._lib.nso_create_spherical_def(self._w, ctypes.byref(d))

    def step(self, dt=1.0 / 60.0, substeps=4):
        self._lib.nso_step(self._w, dt, substeps)

    def apply_forces(self, force=None, torque=None):
        f = None if force is None else np.ascontiguousarray(force, np.float32)
        t = None if torque is None else np.ascontiguousarray(torque, np.float32)
        self._lib.nso_apply_forces(self._w, None if f is None else _ptr(f), None if t is None else _ptr(t))

    @property
    def body_count(self):
        return self._lib.nso_body_count(self._w)

    def bodies(self):
        n = self.body_count
        pos = np.zeros((n, 3), np.float64)
        rot = np.zeros((n, 4), np.float32)
        lin = np.zeros((n, 3), np.float32)
        ang = np.zeros((n, 3), np.float32)
        self._lib.nso_get_bodies(self._w, _ptr(pos), _ptr(rot), _ptr(lin), _ptr(ang))
        return pos, rot, lin, ang

    def state_hash(self):
        return self._lib.nso_state_hash(self._w)

    def contacts(self):
        cap = max(self._lib.nso_contact_capacity(self._w), 1)
        ints = np.zeros((cap, 8), np.int32)
        feats = np.zeros((cap, 4), np.uint32)
        fl = np.zeros((cap, 24), np.float32)
        n = self._lib.nso_get_contacts(self._w, _ptr(ints), _ptr(feats), _ptr(fl))
        return ints[:n], feats[:n], fl[:n]

    def counters(self):
        out = np.zeros(32, np.int32)
        self._lib.nso_counters(self._w, _ptr(out))
        return out


# One narrowphase pair per row, laid out like nso_pair_job / nso_pair_result (ns_oracle.h).
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


def collide_pairs(jobs):
    """Oracle narrowphase for each job (caches in ``jobs`` are updated in place)."""
    assert jobs.dtype == PAIR_JOB_DTYPE and jobs.flags.c_contiguous
    lib = load()
    results = np.zeros(len(jobs), PAIR_RESULT_DTYPE)
    if len(jobs):
        lib.nso_collide_pairs(_ptr(jobs), _ptr(results), len(jobs))
    return results
