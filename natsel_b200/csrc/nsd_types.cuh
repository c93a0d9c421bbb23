// Device-resident world layout for the B200 step.
//
// Bodies: the awake set keeps the reference's 64-byte BodyState rows
// (world_runtime.rs:209) as four float4 so one body is two 32-byte sectors;
// body sims (world_runtime.rs:261) are AoS records read once per body per
// phase. Contacts are AoS records indexed by contact id (only the narrowphase
// touches them); the solver reads prepared constraints from float4 SoA planes
// ordered by graph color so every warp load is coalesced.
#pragma once
#include "nsd_geom.cuh"

namespace nsd {

// world_runtime.rs:87-121 body flags
enum : uint32_t {
  kLockLinX = 0x1, kLockLinY = 0x2, kLockLinZ = 0x4, kLockAngX = 0x8, kLockAngY = 0x10,
  kLockAngZ = 0x20, kIsFast = 0x40, kIsBullet = 0x80, kIsSpeedCapped = 0x100,
  kHadToi = 0x200, kAllowFastRotation = 0x400, kDynamicFlag = 0x1000, kEnableSleepFlag = 0x2000,
  kEnableRecycling = 0x4000, kDirtyMass = 0x8000, kGyroscopic = 0x10000,
  kTransient = kIsSpeedCapped | kHadToi,
};
// body_api.rs:25-39 contact flags
enum : uint32_t {
  cTouching = 0x1, cStatic = 0x8, cRecycle = 0x10, cSimTouching = 0x10000,
  cSimDisjoint = 0x20000, cSimStarted = 0x40000, cSimStopped = 0x80000,
  cRelativeValid = 0x800000, cSpeculative = 0x1000000,
};
enum ShapeKind { kCapsule = 0, kHull = 3, kSphere = 5 };  // shape_def.rs:64

struct alignas(16) DSim {
  double px, py, pz;   // transform.p
  double cx, cy, cz;   // center of mass, world
  Q q;                 // transform.q
  V3 local_center;
  V3 force, torque;
  float inv_mass;
  uint32_t flags;
  float min_extent;
  V3 max_extent;
  M3 inertia;          // local inertia (gyroscopic Newton step)
  M3 inv_inertia_local;
  M3 inv_inertia_world;
  float linear_damping, angular_damping, gravity_scale;
  float safety_factor;
  int body_id;
  int shape_begin, shape_end;  // range in the body->shape index table
  double cx0, cy0, cz0;        // centre and rotation at the start of the sweep (center0,
  Q q0;                        // rotation0): the last pose finalize accepted without a sweep test
};

struct alignas(16) DState {
  V3 v; float pad1;
  V3 w; float pad2;
  V3 dp; uint32_t flags;
  Q dq;
};

struct DShape {
  int type, body, enc, is_static;
  float aabb_margin, friction, restitution, rolling;
  uint64_t category, mask;
  int group, hull;
  int world;           // sub-world of the shape (0 for a single world)
  Sphere sphere;
  Capsule capsule;
};

struct ManifoldPoint {
  V3 anchor_a, anchor_b;
  float separation, normal_impulse, total_normal_impulse, normal_velocity, base_separation;
  uint32_t feature_id;
  int persisted;
};
struct Manifold {
  ManifoldPoint points[4];
  V3 normal;
  float twist_impulse;
  V3 friction_impulse, rolling_impulse;
  int point_count;
};

struct alignas(16) DContact {
  int shape_a, shape_b, enc_a, enc_b;
  int body_a, body_b;
  uint32_t flags;
  int color;
  int local;           // position in the overflow list (overflow color only)
  int manifold_count;
  int alive;
  int kind;            // pair kind (shape type combination), fixed at creation
  float friction, restitution, rolling;
  V3 tangent_velocity;
  Q cached_rot_a, cached_rot_b;
  Xf cached_rel;
  SATCache sat;
  SimplexCache simplex;
  Manifold manifold;
};

struct Softness { float bias_rate, mass_scale, impulse_scale; };

// solver_integration.rs:72 make_soft
NSD_HD Softness make_soft(float hertz, float zeta, float h) {
  Softness s = {0, 0, 0};
  if (hertz == 0.0f) return s;
  float omega = 2.0f * kPi * hertz;
  float a1 = 2.0f * zeta + h * omega;
  float a2 = h * omega * a1;
  float a3 = 1.0f / (1.0f + a2);
  s.bias_rate = omega / a1;
  s.mass_scale = a2 * a3;
  s.impulse_scale = a3;
  return s;
}

// contact_solver.rs:38-139 symmetric 3x3 (upper triangle, wide-solver association order)
struct Sym { float xx, xy, xz, yy, yz, zz; };
NSD_HD Sym sym_from(M3 m) { Sym s = {m.cx.x, m.cx.y, m.cx.z, m.cy.y, m.cy.z, m.cz.z}; return s; }
NSD_HD Sym sym_zero() { Sym s = {0, 0, 0, 0, 0, 0}; return s; }
NSD_HD V3 sym_mv(Sym s, V3 a) {
  return v3(s.xx * a.x + (s.xy * a.y + s.xz * a.z), s.xy * a.x + (s.yy * a.y + s.yz * a.z),
            s.xz * a.x + (s.yz * a.y + s.zz * a.z));
}
NSD_HD Sym sym_add(Sym a, Sym b) {
  Sym s = {a.xx + b.xx, a.xy + b.xy, a.xz + b.xz, a.yy + b.yy, a.yz + b.yz, a.zz + b.zz};
  return s;
}
NSD_HD Sym sym_invert(Sym m) {
  float cxx = m.yy * m.zz - m.yz * m.yz;
  float cxy = m.xz * m.yz - m.xy * m.zz;
  float cxz = m.xy * m.yz - m.xz * m.yy;
  float cyy = m.xx * m.zz - m.xz * m.xz;
  float cyz = m.xy * m.xz - m.xx * m.yz;
  float czz = m.xx * m.yy - m.xy * m.xy;
  float d = m.xx * cxx + (m.xy * cxy + m.xz * cxz);
  bool valid = absf(d) > 1000.0f * kMinPositive;
  float inv = valid ? 1.0f / d : 0.0f;
  Sym s = {inv * cxx, inv * cxy, inv * cxz, inv * cyy, inv * cyz, inv * czz};
  return s;
}
// contact_solver.rs:291 inv_rotate_vector_wide
NSD_HD V3 inv_rotate_wide(Q q, V3 a) {
  V3 t0 = cross(q.v, a);
  V3 t = v3(t0.x + t0.x, t0.y + t0.y, t0.z + t0.z);
  V3 u = cross(q.v, t);
  return v3((a.x - q.s * t.x) + u.x, (a.y - q.s * t.y) + u.y, (a.z - q.s * t.z) + u.z);
}

// Colored contact constraints as SoA planes (index = slot in the color-ordered list).
struct CPlanes {
  int4* idx;      // index_a, index_b, contact id, point_count | is_static << 8
  float4* mass;   // inv_mass_a, inv_mass_b, friction, restitution
  float4* ia0;    // inv_ia xx, xy, xz, yy
  float4* ia1;    // inv_ia yz, zz, inv_ib xx, xy
  float4* ib1;    // inv_ib xz, yy, yz, zz
  float4* n;      // normal xyz, rolling resistance
  float4* t1;     // tangent1 xyz, tangent velocity 1
  float4* t2;     // tangent2 xyz, tangent velocity 2
  float4* ca;     // friction center a xyz, twist mass
  float4* cb;     // friction center b xyz, twist impulse (updated)
  float4* tm;     // tangent mass cx.x, cx.y, cy.x, cy.y
  float4* fr;     // friction impulse x, y (updated); rolling mass xx, xy
  float4* roll;   // rolling impulse xyz (updated); rolling mass xz
  float4* rm;     // rolling mass yy, yz, zz, unused
  // points, index p * cap + slot
  float4* pra;    // r_a xyz, base separation
  float4* prb;    // r_b xyz, normal mass
  float4* pimp;   // normal impulse, total normal impulse, lever arm, relative velocity
  float* prest;   // restitution impulse
  int cap;
};

// Overflow constraints keep full 3x3 inertia and are solved by one thread in list order
// (overflow_contact_solver.rs:41).
struct ConstraintPoint {
  V3 r_a, r_b;
  float base_separation, relative_velocity, normal_impulse, total_normal_impulse,
      restitution_impulse, normal_mass, lever_arm;
};
struct ManifoldConstraint {
  ConstraintPoint points[4];
  int point_count;
  V3 normal, tangent1, tangent2, center_a, center_b;
  float twist_mass, twist_impulse;
  M2 tangent_mass;
  V2 friction_impulse;
  V3 rolling_impulse;
  float tangent_velocity1, tangent_velocity2;
};
struct DOverflow {
  int contact_id, index_a, index_b, manifold_count;
  float inv_mass_a, inv_mass_b;
  M3 inv_ia, inv_ib, rolling_mass;
  Softness softness;
  float friction, restitution, rolling_resistance;
  ManifoldConstraint m;
};

// Revolute joint rows (revolute_joint.rs:28 RevoluteJointSim + JointSim base fields).
struct DJoint {
  int body_a, body_b, color, enc_a, enc_b, index_a, index_b;
  int world;           // sub-world of both bodies
  int enable_spring, enable_motor, enable_limit, fixed_rotation;
  Xf local_frame_a, local_frame_b;
  float constraint_hertz, constraint_damping_ratio;
  Softness constraint_softness, spring_softness;
  float inv_mass_a, inv_mass_b;
  M3 inv_ia, inv_ib;
  V3 linear_impulse;
  V2 perp_impulse;
  float spring_impulse, motor_impulse, lower_impulse, upper_impulse;
  float hertz, damping_ratio, max_motor_torque, motor_speed, target_angle, lower_angle, upper_angle;
  Xf frame_a, frame_b;
  V3 rotation_axis_z, perp_axis_x, perp_axis_y, delta_center;
  float axial_mass;
  // kJointSpherical (spherical_joint.rs:40 SphericalJointSim): lower_impulse / upper_impulse hold
  // the twist limit impulses, the spring and motor impulses are vectors
  int type;
  int enable_cone_limit, enable_twist_limit;
  float cone_angle, lower_twist_angle, upper_twist_angle;
  Q target_rotation;
  V3 motor_velocity, spring_impulse3, motor_impulse3;
  float swing_impulse, swing_mass, twist_mass;
  V3 swing_axis, twist_jacobian;
  M3 rotation_mass;
};
enum : int { kJointRevolute = 0, kJointSpherical = 1 };

// Per-step scalars (solver_integration.rs:1024 StepContext plus world settings).
struct StepParams {
  float dt, inv_dt, h, inv_h;
  int substeps;
  Softness contact_softness, static_softness;
  float contact_speed, max_linear_speed, restitution_threshold;
  float warm_start;
  int restitution_iterations;
  int enable_continuous;
  float contact_hertz, contact_damping_ratio;
  V3 gravity;
};

// Device-side counters and error flags.
struct Control {
  int error;              // NS_ERR_* raised on the device
  int barrier_count;      // grid barrier arrivals
  int moved_count;        // proxies enlarged since the last pair update
  int new_pairs;          // pairs found by the last pair update
  int cand_count;         // candidate slots used by the last pair update
  int changed_count;      // contact state changes in the last collide
  int overflow_count;     // contacts in the overflow color, all sub-worlds
  int recycled;           // contacts recycled in the last collide
  int fast_flags;         // fast-body flags raised by finalize
  int any_restitution;    // a prepared contact has restitution
  int tombstones;         // erased pair-set slots since the last rebuild
  int hs_rebuild;         // rebuild the pair set this step
  int color_count[24];    // constraints per color (colors 0..22)
  int color_offset[25];
  int live_contacts;
  int collide_count[17];  // contacts queued for a full manifold update: pair kinds 0..2, the
                          // hull-sphere and hull-capsule pairs by their simplex cache's size
                          // (0..3), then the hull pairs by the type of their SAT cache (0..5)
  int long_segments;      // candidate segments handed to the block sort this pair update
  int fast_count;         // fast bodies queued by finalize for the continuous pass (this step)
  int bullet_count;       // fast bullets queued by finalize for the bullet pass (this step)
};

}  // namespace nsd
