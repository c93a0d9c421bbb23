// Oracle world step. TEST INFRASTRUCTURE ONLY: a single-threaded C++
// restatement of the reference's World::step restricted to the hot path
// (sleep disabled; CCD only flags fast bodies). Used as the parity checker;
// the product never links it. Each block cites the reference function it
// follows; operand order matches the reference so results are bit-identical.
#ifdef _OPENMP
#include <omp.h>
#endif
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <unordered_set>
#include <vector>

#include "ns_collide.hpp"
#include "ns_joint.hpp"
#include "ns_toi.hpp"
#include "ns_oracle.h"

namespace nso {

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

struct BodySim {
  WXf transform;
  Pos center;
  uint32_t flags;
  real min_extent;
  V3 max_extent;
  Q rotation0;
  Pos center0;
  V3 local_center, force, torque;
  real inv_mass;
  M3 inertia, inv_inertia_local, inv_inertia_world;
  real linear_damping, angular_damping, gravity_scale;
  int body_id;
};
struct BodyState { V3 v; V3 w; V3 dp; uint32_t flags; Q dq; };

struct Body {
  int id = -1, type = 0, set_index = -1, local_index = -1;
  int head_shape = -1, shape_count = 0;
  int joint_count = 0;
  uint32_t flags = 0;
  real sleep_threshold = 0, sleep_time = 0, safety_factor = 0.5f, mass = 0;
};

struct Shape {
  int id = -1, body_id = -1, next_shape = -1, type = kSphere;
  real density = 0, aabb_margin = 0;
  AABB aabb;
  real friction = 0.6f, restitution = 0, rolling = 0;
  uint64_t category = 1, mask = ~0ull;
  int group = 0;
  Hull hull;
  Sphere sphere;
  Capsule capsule;
  bool is_static = false;
};

struct ManifoldPoint {
  V3 anchor_a, anchor_b;
  real separation, normal_impulse, total_normal_impulse, normal_velocity, base_separation;
  uint32_t feature_id;
  bool persisted;
};
struct Manifold {
  ManifoldPoint points[4];
  V3 normal;
  real twist_impulse;
  V3 friction_impulse, rolling_impulse;
  int point_count;
};

struct Contact {
  int contact_id = -1, color_index = -1, local_index = -1;
  int shape_a = -1, shape_b = -1, body_a = -1, body_b = -1;
  int encoded_a = -1, encoded_b = -1;
  uint32_t flags = 0;
  Manifold manifold;
  int manifold_count = 0;
  Q cached_rot_a, cached_rot_b;
  Xf cached_rel;
  real friction = 0, restitution = 0, rolling = 0;
  V3 tangent_velocity = {0, 0, 0};
  SATCache sat;
  SimplexCache simplex;
};

struct Softness { real bias_rate, mass_scale, impulse_scale; };

// solver_integration.rs:72 make_soft
static Softness make_soft(real hertz, real zeta, real h) {
  Softness s = {0, 0, 0};
  if (hertz == 0.0f) return s;
  real omega = 2.0f * kPi * hertz;
  real a1 = 2.0f * zeta + h * omega;
  real a2 = h * omega * a1;
  real a3 = 1.0f / (1.0f + a2);
  s.bias_rate = omega / a1;
  s.mass_scale = a2 * a3;
  s.impulse_scale = a3;
  return s;
}

// contact_solver.rs:38-139 symmetric 3x3
struct Sym { real xx, xy, xz, yy, yz, zz; };
static Sym sym_from(M3 m) { Sym s = {m.cx.x, m.cx.y, m.cx.z, m.cy.y, m.cy.z, m.cz.z}; return s; }
static Sym sym_zero() { Sym s = {0, 0, 0, 0, 0, 0}; return s; }
static V3 sym_mv(Sym s, V3 a) {
  return v3(s.xx * a.x + (s.xy * a.y + s.xz * a.z), s.xy * a.x + (s.yy * a.y + s.yz * a.z),
            s.xz * a.x + (s.yz * a.y + s.zz * a.z));
}
static Sym sym_add(Sym a, Sym b) {
  Sym s = {a.xx + b.xx, a.xy + b.xy, a.xz + b.xz, a.yy + b.yy, a.yz + b.yz, a.zz + b.zz};
  return s;
}
static Sym sym_invert(Sym m) {
  real cxx = m.yy * m.zz - m.yz * m.yz;
  real cxy = m.xz * m.yz - m.xy * m.zz;
  real cxz = m.xy * m.yz - m.xz * m.yy;
  real cyy = m.xx * m.zz - m.xz * m.xz;
  real cyz = m.xy * m.xz - m.xx * m.yz;
  real czz = m.xx * m.yy - m.xy * m.xy;
  real d = m.xx * cxx + (m.xy * cxy + m.xz * cxz);
  bool valid = absf(d) > 1000.0f * kMinPositive;
  real inv = valid ? 1.0f / d : 0.0f;
  Sym s = {inv * cxx, inv * cxy, inv * cxz, inv * cyy, inv * cyz, inv * czz};
  return s;
}
// contact_solver.rs:291
static V3 inv_rotate_wide(Q q, V3 a) {
  V3 t0 = cross(q.v, a);
  V3 t = v3(t0.x + t0.x, t0.y + t0.y, t0.z + t0.z);
  V3 u = cross(q.v, t);
  return v3((a.x - q.s * t.x) + u.x, (a.y - q.s * t.y) + u.y, (a.z - q.s * t.z) + u.z);
}

struct ConstraintPoint {
  V3 r_a, r_b;
  real base_separation, relative_velocity, normal_impulse, total_normal_impulse,
      restitution_impulse, normal_mass, lever_arm;
};
struct ManifoldConstraint {
  ConstraintPoint points[4];
  int point_count;
  V3 normal, tangent1, tangent2, center_a, center_b;
  real twist_mass, twist_impulse;
  M2 tangent_mass;
  V2 friction_impulse;
  V3 rolling_impulse;
  real tangent_velocity1, tangent_velocity2;
};
struct ContactConstraint {
  int contact_id, index_a, index_b;
  real inv_mass_a, inv_mass_b;
  Sym inv_ia, inv_ib, rolling_mass;
  Softness softness;
  real friction, restitution, rolling_resistance;
  bool is_static;
  ManifoldConstraint m;  // convex contacts carry exactly one manifold
};
struct OverflowConstraint {
  int contact_id, index_a, index_b;
  real inv_mass_a, inv_mass_b;
  M3 inv_ia, inv_ib, rolling_mass;
  Softness softness;
  real friction, restitution, rolling_resistance;
  int manifold_count;
  ManifoldConstraint m;
};

struct StepContext {
  real dt, inv_dt, h, inv_h;
  int sub_step_count;
  Softness contact_softness, static_softness;
  bool enable_warm_starting;
};

struct IdPool {  // id_pool.rs
  std::vector<int> free_list;
  int next = 0;
  int alloc() {
    if (!free_list.empty()) { int id = free_list.back(); free_list.pop_back(); return id; }
    return next++;
  }
  void release(int id) { free_list.push_back(id); }
};

struct GraphColor {
  std::vector<int> convex;         // convex contact ids, append + swap-remove order
  std::vector<int> overflow;       // scalar contact specs (overflow color only)
  std::vector<int> joints;         // joint ids
};

}  // namespace nso

using namespace nso;

struct nso_world {
  nso_world_def def;
  std::vector<Body> bodies;
  std::vector<BodySim> static_sims, awake_sims;
  std::vector<BodyState> awake_states;
  std::vector<Shape> shapes;
  std::vector<AABB> fat;
  std::vector<uint8_t> proxy_moved;
  std::vector<Contact> contacts;
  IdPool contact_ids;
  std::unordered_set<uint64_t> pair_set;
  std::vector<GraphColor> colors;
  std::vector<std::vector<uint64_t>> color_bits;  // per color, bit per body id
  std::vector<Joint> joints;
  std::vector<std::vector<int>> body_joints;
  // per-step solver data
  std::vector<std::vector<ContactConstraint>> constraints;
  std::vector<OverflowConstraint> overflow;
  bool any_restitution = false;
  StepContext ctx;
  int fast_flags_seen = 0;
  int sat_calls = 0;
  int recycled = 0;
  bool static_moved = false;
};

namespace {

// constraint graph bitset helpers (constraint_graph.rs:92-110)
bool get_bit(nso_world* w, int c, int b) {
  const std::vector<uint64_t>& v = w->color_bits[c];
  size_t blk = (size_t)b >> 6;
  if (blk >= v.size()) return false;
  return (v[blk] >> (b & 63)) & 1ull;
}
// Host threads for the colour-parallel loops (collide per contact, prepare and the solver stages
// per constraint of a colour, the body stages per body). The reference runs its stages the same
// way (solver_stages.rs:227-231, collide_pass.rs:209); every such loop touches disjoint data, so
// any thread count gives the same bits. One thread unless nso_set_threads raises it.
int g_threads = 1;
constexpr int kParMin = 64;
int thread_index() {
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

void set_bit(nso_world* w, int c, int b) {
  std::vector<uint64_t>& v = w->color_bits[c];
  size_t blk = (size_t)b >> 6;
  if (blk >= v.size()) v.resize(blk + 1, 0);
  v[blk] |= 1ull << (b & 63);
}
void clear_bit(nso_world* w, int c, int b) {
  std::vector<uint64_t>& v = w->color_bits[c];
  size_t blk = (size_t)b >> 6;
  if (blk >= v.size()) return;
  v[blk] &= ~(1ull << (b & 63));
}

int encode_body(const Body& b) {  // world_runtime.rs:900
  if (b.set_index == 2) return b.local_index;
  if (b.set_index == 0) return -(b.local_index + 2);
  return -1;
}

BodySim& sim_of(nso_world* w, const Body& b) {
  return b.set_index == 2 ? w->awake_sims[b.local_index] : w->static_sims[b.local_index];
}

// world_runtime.rs:1479 sync_body_flags
void sync_body_flags(nso_world* w, int bi) {
  Body& b = w->bodies[bi];
  BodySim& s = sim_of(w, b);
  s.flags = (s.flags & (kIsFast | kHadToi)) | (b.flags & ~kTransient);
  if (b.set_index == 2) w->awake_states[b.local_index].flags = b.flags & ~kTransient;
}

// shape_runtime.rs:370 compute_shape_aabb
AABB shape_aabb_xf(const Shape& s, Xf t) {
  if (s.type == kHull) return aabb_transform(t, s.hull.bounds);  // hull_queries.rs:16
  if (s.type == kSphere) {  // sphere.rs:27
    V3 c = xf_point(t, s.sphere.center);
    real r = s.sphere.radius;
    V3 e = v3(r, r, r);
    return aabb(c - e, c + e);
  }
  V3 c1 = xf_point(t, s.capsule.c1), c2 = xf_point(t, s.capsule.c2);  // capsule.rs:66
  real r = s.capsule.radius;
  V3 e = v3(r, r, r);
  return aabb(min3(c1, c2) - e, max3(c1, c2) + e);
}
// shape_runtime.rs:405 compute_shape_aabb in a rotation-only frame
AABB shape_local_aabb(const Shape& s, Q q) { return shape_aabb_xf(s, xf(v3(0, 0, 0), q)); }
// shape_runtime.rs:420 compute_fat_shape_aabb
AABB fat_shape_aabb(const Shape& s, WXf t, real extra) {
  return offset_aabb(aabb_inflate(shape_local_aabb(s, t.q), extra), t.p);
}

struct MassData { real mass; V3 center; M3 inertia; };
MassData shape_mass(const Shape& s) {
  MassData md;
  if (s.type == kHull) {  // shape_runtime.rs:312
    md.mass = s.density * s.hull.volume;
    md.center = s.hull.center;
    md.inertia = mul_sm(s.density, s.hull.central_inertia);
  } else if (s.type == kSphere) {  // sphere.rs:13
    real r = s.sphere.radius;
    real volume = 4.0f / 3.0f * kPi * r * r * r;
    real mass = volume * s.density;
    real ixx = 0.4f * mass * r * r;
    md.mass = mass;
    md.center = s.sphere.center;
    md.inertia = diag(ixx, ixx, ixx);
  } else {  // capsule.rs:27
    V3 c1 = s.capsule.c1, c2 = s.capsule.c2;
    real r = s.capsule.radius;
    real h = distance(c1, c2);
    real cyl_vol = kPi * r * r * h;
    real cyl_mass = cyl_vol * s.density;
    real sph_vol = (4.0f / 3.0f) * kPi * r * r * r;
    real sph_mass = sph_vol * s.density;
    // geometry_queries.rs cylinder_inertia / sphere_inertia
    real cyl_lateral = cyl_mass * (3.0f * r * r + h * h) / 12.0f;
    real cyl_axial = 0.5f * cyl_mass * r * r;
    M3 cyl = diag(cyl_lateral, cyl_axial, cyl_lateral);
    real sph_i = 0.4f * sph_mass * r * r;
    M3 sph = diag(sph_i, sph_i, sph_i);
    M3 inertia = add_mm(cyl, sph);
    real st = 0.125f * sph_mass * (3.0f * r + 2.0f * h) * h;
    inertia.cx.x += st;
    inertia.cz.z += st;
    M3 rot = identity_m3();
    if (h * h > 1000.0f * kMinPositive) {
      V3 dir = normalize(c2 - c1);
      Q q = quat_between_unit_vectors(v3(0, 1, 0), dir);
      rot = matrix_from_quat(q);
    }
    md.mass = sph_mass + cyl_mass;
    md.center = 0.5f * (c1 + c2);
    md.inertia = mul_mm(rot, mul_mm(inertia, transpose(rot)));
  }
  return md;
}

struct Extent { real min_extent; V3 max_extent; };
Extent shape_extent(const Shape& s, V3 lc) {  // shape_runtime.rs:499
  Extent e;
  if (s.type == kCapsule) {
    real r = s.capsule.radius;
    e.min_extent = r;
    V3 c1 = s.capsule.c1 - lc, c2 = s.capsule.c2 - lc;
    e.max_extent = max3(abs3(c1), abs3(c2)) + v3(r, r, r);
  } else if (s.type == kSphere) {
    real r = s.sphere.radius;
    e.min_extent = r;
    e.max_extent = abs3(s.sphere.center - lc) + v3(r, r, r);
  } else {  // hull_queries.rs:101
    e.min_extent = s.hull.inner_radius;
    e.max_extent = v3(0, 0, 0);
    for (int i = 0; i < s.hull.vertex_count; ++i)
      e.max_extent = max3(e.max_extent, abs3(s.hull.points[i] - lc));
  }
  return e;
}

// body_api.rs:611 update_isotropic_inertia
void update_isotropic_inertia(nso_world* w, int bi) {
  Body& b = w->bodies[bi];
  BodySim& s = sim_of(w, b);
  M3 I = s.inertia;
  real mean = (I.cx.x + I.cy.y + I.cz.z) / 3.0f;
  real dx = I.cx.x - mean, dy = I.cy.y - mean, dz = I.cz.z - mean;
  real off = I.cy.x * I.cy.x + I.cz.x * I.cz.x + I.cz.y * I.cz.y;
  real dev = dx * dx + dy * dy + dz * dz + 2.0f * off;
  real tol = 0.2f;  // world isotropic_inertia_tolerance default (world_runtime.rs:1256)
  if (2.0f * dev > 3.0f * tol * tol * mean * mean) b.flags |= kGyroscopic;
  else b.flags &= ~kGyroscopic;
  sync_body_flags(w, bi);
}

// body_api.rs:642 update_body_mass_data
void update_body_mass(nso_world* w, int bi) {
  Body& b = w->bodies[bi];
  b.flags &= ~kDirtyMass;
  b.flags &= ~kGyroscopic;
  sync_body_flags(w, bi);
  b.mass = 0.0f;
  BodySim& s = sim_of(w, b);
  s.inertia = m3zero(); s.inv_mass = 0.0f;
  s.inv_inertia_local = m3zero(); s.inv_inertia_world = m3zero();
  s.local_center = v3(0, 0, 0);
  s.min_extent = huge_value();
  s.max_extent = v3(0, 0, 0);
  if (b.head_shape == -1) return;
  if (b.type != 2) {
    // body_api.rs:670-689: zero mass; a kinematic body keeps its shapes' extents about its origin
    s.center = s.transform.p;
    s.center0 = s.center;
    if (b.type == 1)
      for (int sid = b.head_shape; sid != -1; sid = w->shapes[sid].next_shape) {
        Extent e = shape_extent(w->shapes[sid], v3(0, 0, 0));
        s.min_extent = minf(s.min_extent, e.min_extent);
        s.max_extent = max3(s.max_extent, e.max_extent);
      }
    return;
  }
  std::vector<MassData> masses;
  V3 lc = v3(0, 0, 0);
  for (int sid = b.head_shape; sid != -1;) {
    const Shape& sh = w->shapes[sid];
    sid = sh.next_shape;
    if (sh.density == 0.0f) { MassData z = {0, v3(0, 0, 0), m3zero()}; masses.push_back(z); continue; }
    MassData md = shape_mass(sh);
    b.mass += md.mass;
    lc = mul_add(lc, md.mass, md.center);
    masses.push_back(md);
  }
  if (b.mass > 0.0f) {
    s.inv_mass = 1.0f / b.mass;
    lc = s.inv_mass * lc;
  }
  for (const MassData& md : masses) {
    if (md.mass == 0.0f) continue;
    V3 off = lc - md.center;
    M3 I = add_mm(md.inertia, steiner(md.mass, off));
    s.inertia = add_mm(s.inertia, I);
  }
  real d = det(s.inertia);
  if (d > 0.0f) {
    s.inv_inertia_local = invert_t(s.inertia);
    M3 R = matrix_from_quat(s.transform.q);
    s.inv_inertia_world = mul_mm(mul_mm(R, s.inv_inertia_local), transpose(R));
  }
  Pos old_center = s.center;
  s.local_center = lc;
  s.center = world_point(s.transform, s.local_center);
  s.center0 = s.center;
  BodyState& st = w->awake_states[b.local_index];
  V3 dl = cross(st.w, sub_pos(s.center, old_center));
  st.v = st.v + dl;
  for (int sid = b.head_shape; sid != -1;) {
    const Shape& sh = w->shapes[sid];
    Extent e = shape_extent(sh, lc);
    s.min_extent = minf(s.min_extent, e.min_extent);
    s.max_extent = max3(s.max_extent, e.max_extent);
    sid = sh.next_shape;
  }
  if ((s.flags & (kLockAngX | kLockAngY | kLockAngZ)) == (kLockAngX | kLockAngY | kLockAngZ)) {
    s.inertia = m3zero(); s.inv_inertia_local = m3zero(); s.inv_inertia_world = m3zero();
  }
  update_isotropic_inertia(w, bi);
}

// shape_creation.rs:199 compute_shape_margin
real shape_margin(const Shape& s) {
  real margin = 0.0f;
  if (s.type == kSphere) margin = s.sphere.radius;
  else if (s.type == kCapsule) margin = 0.5f * distance(s.capsule.c2, s.capsule.c1) + s.capsule.radius;
  else {
    real mx = 0.0f;
    for (int i = 0; i < s.hull.vertex_count; ++i)
      mx = maxf(mx, distance_sq(s.hull.points[i], s.hull.center));
    margin = std::sqrt(mx);
  }
  return minf(max_aabb_margin(), kAabbMarginFraction * margin);
}

int create_shape(nso_world* w, int bi, const nso_shape_def* def, Shape sh) {
  int sid = (int)w->shapes.size();
  Body& b = w->bodies[bi];
  sh.id = sid;
  sh.body_id = bi;
  sh.density = def->density;
  sh.friction = def->friction;
  sh.restitution = def->restitution;
  sh.rolling = def->rolling_resistance;
  sh.category = def->category_bits;
  sh.mask = def->mask_bits;
  sh.group = def->group_index;
  sh.aabb_margin = shape_margin(sh);
  sh.is_static = b.type == 0;
  // shape_creation.rs:236 update_shape_aabbs at the body's current transform
  const BodySim& s = sim_of(w, b);
  real spec = speculative_distance();
  AABB a = fat_shape_aabb(sh, s.transform, spec);
  sh.aabb = a;
  real margin = b.type == 0 ? spec : sh.aabb_margin;
  w->fat.push_back(aabb_inflate(a, margin));
  // broad_phase.rs:73 -- static proxies are marked only when contact creation is forced,
  // which ShapeDef's default (invoke_contact_creation = true) does.
  w->proxy_moved.push_back(1);
  if (b.type == 0) w->static_moved = true;
  sh.next_shape = b.head_shape;
  b.head_shape = sid;
  b.shape_count++;
  w->shapes.push_back(sh);
  update_body_mass(w, bi);
  return sid;
}

// hash_set.rs:25 shape_pair_key with child 0
uint64_t pair_key(int s1, int s2) {
  const uint64_t mask = (1ull << 22) - 1;
  uint64_t a = mask & (uint64_t)(int64_t)s1, b = mask & (uint64_t)(int64_t)s2;
  if (s1 < s2) return (a << 42) | (b << 20);
  return (b << 42) | (a << 20);
}

// contact_creation.rs:151 should_create_pair (minus sensors/custom filters, absent here)
bool should_create_pair(nso_world* w, int sa, int sb) {
  const Shape& a = w->shapes[sa];
  const Shape& b = w->shapes[sb];
  if (a.body_id == b.body_id) return false;
  // shape_runtime.rs:284 should_shapes_collide
  if (a.group == b.group && a.group != 0) {
    if (!(a.group > 0)) return false;
  } else if (!((a.mask & b.category) != 0 && (a.category & b.mask) != 0)) {
    return false;
  }
  // contact_creation.rs:113 should_bodies_collide
  const Body& ba = w->bodies[a.body_id];
  const Body& bb = w->bodies[b.body_id];
  if (ba.type != 2 && bb.type != 2) return false;
  const Body& scan = ba.joint_count < bb.joint_count ? ba : bb;
  int other = ba.joint_count < bb.joint_count ? bb.id : ba.id;
  if (scan.id < (int)w->body_joints.size()) {
    for (int jid : w->body_joints[scan.id]) {
      const Joint& j = w->joints[jid];
      int o = j.body_a == scan.id ? j.body_b : j.body_a;
      if (!j.collide_connected && o == other) return false;
    }
  }
  return true;
}

// contact_creation.rs:219 create_contact (+ :248 create_contact_with_shapes)
void create_contact(nso_world* w, int sa, int sb) {
  // contact_creation.rs:65 contact registers: capsule>sphere, hull>sphere, hull>capsule.
  int ta = w->shapes[sa].type, tb = w->shapes[sb].type;
  auto primary = [](int a, int b) {
    if (a == b) return true;
    if (a == kCapsule && b == kSphere) return true;
    if (a == kHull && (b == kSphere || b == kCapsule)) return true;
    return false;
  };
  if (!primary(ta, tb)) std::swap(sa, sb);
  const Shape& A = w->shapes[sa];
  const Shape& B = w->shapes[sb];
  int cid = w->contact_ids.alloc();
  if (cid == (int)w->contacts.size()) w->contacts.push_back(Contact());
  Contact c;
  c.contact_id = cid;
  c.shape_a = sa; c.shape_b = sb;
  c.body_a = A.body_id; c.body_b = B.body_id;
  const Body& ba = w->bodies[A.body_id];
  const Body& bb = w->bodies[B.body_id];
  c.encoded_a = encode_body(ba);
  c.encoded_b = encode_body(bb);
  if (ba.type == 0 || bb.type == 0) c.flags |= cStatic;
  c.flags |= cSpeculative;  // enable_speculative world + shape defaults
  if ((ba.flags & kEnableRecycling) && (bb.flags & kEnableRecycling)) c.flags |= cRecycle;
  real ra = A.type == kSphere ? A.sphere.radius : (A.type == kCapsule ? A.capsule.radius : 0.0f);
  real rb = B.type == kSphere ? B.sphere.radius : (B.type == kCapsule ? B.capsule.radius : 0.0f);
  c.rolling = maxf(A.rolling, B.rolling) * maxf(ra, rb);
  w->pair_set.insert(pair_key(sa, sb));
  w->contacts[cid] = c;
}

// contact_creation.rs:901 update_broad_phase_pairs. The candidate set of the reference's
// tree traversal is every overlapping fat-AABB pair (dynamic vs dynamic/static) with at least one
// moved proxy; keys are sorted before creation, so the search order does not matter. The oracle
// finds the same set with a sort-and-sweep along x.
void update_pairs(nso_world* w) {
  int n = (int)w->shapes.size();
  bool any = w->static_moved;
  for (int i = 0; i < n && !any; ++i) any = w->proxy_moved[i] != 0;
  if (!any) return;
  std::vector<int> small, large;
  for (int i = 0; i < n; ++i) {
    real wx = w->fat[i].hi.x - w->fat[i].lo.x;
    if (w->shapes[i].is_static && wx > 8.0f) large.push_back(i);
    else small.push_back(i);
  }
  std::sort(small.begin(), small.end(), [&](int a, int b) {
    if (w->fat[a].lo.x != w->fat[b].lo.x) return w->fat[a].lo.x < w->fat[b].lo.x;
    return a < b;
  });
  std::vector<uint64_t> keys;
  auto consider = [&](int a, int b, std::vector<uint64_t>& out) {
    const Shape& A = w->shapes[a];
    const Shape& B = w->shapes[b];
    if (A.is_static && B.is_static) return;
    if (!w->proxy_moved[a] && !w->proxy_moved[b]) return;
    if (!aabb_overlaps(w->fat[a], w->fat[b])) return;
    int lo = std::min(a, b), hi = std::max(a, b);
    uint64_t k = pair_key(lo, hi);
    if (w->pair_set.count(k)) return;
    if (!should_create_pair(w, lo, hi)) return;
    out.push_back(k);
  };
  // small vs small: each pair once (i < j in sweep order); the search only reads the world, so
  // threads collect into their own lists and the keys are sorted below
  const int ns_ = (int)small.size();
  std::vector<std::vector<uint64_t>> found(g_threads);
#pragma omp parallel num_threads(g_threads) if (g_threads > 1 && ns_ >= 1024)
  {
    std::vector<uint64_t>& mine = found[thread_index()];
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < ns_; ++i) {
      int a = small[i];
      real hx = w->fat[a].hi.x;
      for (int j = i + 1; j < ns_; ++j) {
        int b = small[j];
        if (w->fat[b].lo.x > hx) break;
        consider(a, b, mine);
      }
    }
  }
  for (const std::vector<uint64_t>& f : found) keys.insert(keys.end(), f.begin(), f.end());
  for (int L : large)
    for (int s : small) consider(L, s, keys);
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  for (int i = 0; i < n; ++i) w->proxy_moved[i] = 0;
  w->static_moved = false;
  for (uint64_t k : keys) {
    int sa = (int)((k >> 42) & ((1ull << 22) - 1));
    int sb = (int)((k >> 20) & ((1ull << 22) - 1));
    create_contact(w, sa, sb);
  }
}

// constraint_graph.rs:113 add_contact_to_graph
void add_contact_to_graph(nso_world* w, int cid) {
  Contact& c = w->contacts[cid];
  int color = kOverflowIndex;
  int a = c.body_a, b = c.body_b;
  int ta = w->bodies[a].type, tb = w->bodies[b].type;
  if (ta == 2 && tb == 2) {
    for (int i = 0; i < kDynamicColorCount; ++i) {
      if (get_bit(w, i, a) || get_bit(w, i, b)) continue;
      set_bit(w, i, a); set_bit(w, i, b);
      color = i;
      break;
    }
  } else if (ta == 2) {
    for (int i = kOverflowIndex - 1; i >= 1; --i)
      if (!get_bit(w, i, a)) { set_bit(w, i, a); color = i; break; }
  } else if (tb == 2) {
    for (int i = kOverflowIndex - 1; i >= 1; --i)
      if (!get_bit(w, i, b)) { set_bit(w, i, b); color = i; break; }
  }
  c.color_index = color;
  if (color == kOverflowIndex) {
    c.local_index = (int)w->colors[color].overflow.size();
    w->colors[color].overflow.push_back(cid);
  } else {
    c.local_index = (int)w->colors[color].convex.size();
    w->colors[color].convex.push_back(cid);
  }
  c.encoded_a = encode_body(w->bodies[a]);
  c.encoded_b = encode_body(w->bodies[b]);
}

// constraint_graph.rs:200 remove_contact_from_graph (swap-remove keeps local indices valid)
void remove_contact_from_graph(nso_world* w, int a, int b, int color, int local) {
  if (color != kOverflowIndex) { clear_bit(w, color, a); clear_bit(w, color, b); }
  std::vector<int>& list = color == kOverflowIndex ? w->colors[color].overflow : w->colors[color].convex;
  int last = (int)list.size() - 1;
  if (local != last) {
    list[local] = list[last];
    list.pop_back();
    w->contacts[list[local]].local_index = local;
  } else {
    list.pop_back();
  }
}

// contact_creation.rs:428 destroy_contact
void destroy_contact(nso_world* w, int cid) {
  Contact& c = w->contacts[cid];
  w->pair_set.erase(pair_key(c.shape_a, c.shape_b));
  c.manifold_count = 0;
  if (c.color_index != -1) remove_contact_from_graph(w, c.body_a, c.body_b, c.color_index, c.local_index);
  c.contact_id = -1;
  c.color_index = -1;
  c.local_index = -1;
  w->contact_ids.release(cid);
}

// contact_update.rs:43 compute_convex_manifold + :243 update_convex_contact + :393 update_contact
bool update_contact(nso_world* w, Contact& c, V3 lca, WXf xa, V3 lcb, WXf xb) {
  const Shape& A = w->shapes[c.shape_a];
  const Shape& B = w->shapes[c.shape_b];
  LocalManifold lm;
  Xf b2a = inv_mul_wxf(xa, xb);
  if (A.type == kSphere) {
    collide_spheres(&lm, A.sphere, B.sphere, b2a);
  } else if (A.type == kCapsule) {
    if (B.type == kSphere) collide_capsule_sphere(&lm, A.capsule, B.sphere, b2a);
    else collide_capsules(&lm, A.capsule, B.capsule, b2a);
  } else {
    if (B.type == kSphere) collide_hull_sphere(&lm, A.hull, B.sphere, b2a, &c.simplex);
    else if (B.type == kCapsule) collide_hull_capsule(&lm, A.hull, B.capsule, b2a, &c.simplex);
    else collide_hulls(&lm, A.hull, B.hull, b2a, &c.sat, &w->sat_calls);
  }
  if (lm.point_count == 0) {
    c.manifold_count = 0;
    c.flags &= ~cSimTouching;
    return false;
  }
  ManifoldPoint old_points[4];
  int old_count = 0;
  if (c.manifold_count == 0) {
    Manifold fresh;
    std::memset(&fresh, 0, sizeof(fresh));
    c.manifold = fresh;
    c.manifold_count = 1;
  } else {
    old_count = c.manifold.point_count;
    for (int i = 0; i < old_count; ++i) old_points[i] = c.manifold.points[i];
  }
  Manifold& m = c.manifold;
  m.point_count = lm.point_count;
  M3 ma = matrix_from_quat(xa.q);
  m.normal = mul_mv(ma, lm.normal);
  for (int i = 0; i < lm.point_count; ++i) {
    ManifoldPoint t;
    std::memset(&t, 0, sizeof(t));
    t.anchor_a = mul_mv(ma, lm.points[i].point);
    t.anchor_b = t.anchor_a + sub_pos(xa.p, xb.p);
    t.separation = lm.points[i].separation;
    t.feature_id = make_feature_id(lm.points[i].pair);
    t.normal_velocity = 0.0f;
    m.points[i] = t;
  }
  for (int i = 0; i < lm.point_count; ++i) {
    ManifoldPoint p2 = m.points[i];
    p2.total_normal_impulse = 0.0f;
    p2.persisted = false;
    for (int j = 0; j < old_count; ++j) {
      if (p2.feature_id == old_points[j].feature_id) {
        p2.normal_impulse = old_points[j].normal_impulse;
        p2.persisted = true;
        old_points[j].feature_id = 0xffffffffu;
        break;
      }
    }
    if (!p2.persisted) p2.normal_impulse = 0.0f;
    m.points[i] = p2;
  }
  // material mixing (world_runtime.rs:1305 mix_friction / mix_restitution)
  c.friction = std::sqrt(A.friction * B.friction);
  c.restitution = maxf(A.restitution, B.restitution);
  if (A.rolling > 0.0f || B.rolling > 0.0f) {
    auto radius = [](const Shape& s) {
      if (s.type == kSphere) return s.sphere.radius;
      if (s.type == kCapsule) return s.capsule.radius;
      return 0.25f * s.hull.inner_radius;
    };
    c.rolling = maxf(A.rolling, B.rolling) * maxf(radius(A), radius(B));
  } else {
    c.rolling = 0.0f;
  }
  V3 tva = rotate(xa.q, v3(0, 0, 0));
  V3 tvb = rotate(xb.q, v3(0, 0, 0));
  c.tangent_velocity = tva - tvb;
  // anchors relative to the centers of mass
  V3 ca = rotate(xa.q, lca), cb = rotate(xb.q, lcb);
  for (int j = 0; j < m.point_count; ++j) {
    m.points[j].anchor_a = m.points[j].anchor_a - ca;
    m.points[j].anchor_b = m.points[j].anchor_b - cb;
  }
  c.flags |= cSimTouching;
  return true;
}

// collide_pass.rs:541 collide_one_contact
void collide_one(nso_world* w, int cid, std::vector<uint8_t>& bits) {
  Contact& c = w->contacts[cid];
  if (!aabb_overlaps(w->fat[c.shape_a], w->fat[c.shape_b])) {
    c.flags |= cSimDisjoint;
    c.flags &= ~cSimTouching;
    bits[cid] = 1;
    return;
  }
  const Body& ba = w->bodies[c.body_a];
  const Body& bb = w->bodies[c.body_b];
  const BodySim& sa = ba.set_index == 2 ? w->awake_sims[ba.local_index] : w->static_sims[ba.local_index];
  const BodySim& sb = bb.set_index == 2 ? w->awake_sims[bb.local_index] : w->static_sims[bb.local_index];
  bool was_touching = (c.flags & cSimTouching) != 0;
  WXf xa = sa.transform, xb = sb.transform;
  bool is_fast = ((sa.flags | sb.flags) & kIsFast) != 0;
  real recycle = contact_recycle_distance();
  real spec = speculative_distance();
  real recycle_nt = minf(recycle, spec);
  real tol = was_touching ? recycle : recycle_nt;
  if (!is_fast && recycle > 0.0f && (c.flags & cRelativeValid) && (c.flags & cRecycle)) {
    real ang_a = dot_quat(xa.q, c.cached_rot_a);
    real ang_b = dot_quat(xb.q, c.cached_rot_b);
    real ang = minf(ang_a * ang_a, ang_b * ang_b);
    Xf x = inv_mul_wxf(xa, xb);
    Xf xc = c.cached_rel;
    V3 mea = c.encoded_a < -1 ? v3(0, 0, 0) : sa.max_extent;
    V3 meb = c.encoded_b < -1 ? v3(0, 0, 0) : sb.max_extent;
    V3 me = max3(mea, meb);
    real dsq = distance_sq(x.p, xc.p);
    if (ang > kRecycleAngular && dsq < tol * tol) {
      real dist = std::sqrt(dsq);
      real slack = tol - dist;
      Q qr = inv_mul_quat(xc.q, x.q);
      V3 arc = modified_cross(abs3(qr.v), me);
      real arc_sq = 4.0f * length_sq(arc);
      if (arc_sq < slack * slack) {
        Q dqa = mul_quat(xa.q, conjugate(c.cached_rot_a));
        Q dqb = mul_quat(xb.q, conjugate(c.cached_rot_b));
        M3 ma = matrix_from_quat(dqa), mb = matrix_from_quat(dqb);
        V3 dc = sub_pos(sb.center, sa.center);
        if (c.manifold_count > 0) {
          Manifold& m = c.manifold;
          V3 n = m.normal;
          for (int i = 0; i < m.point_count; ++i) {
            V3 ra = mul_mv(ma, m.points[i].anchor_a);
            V3 rb = mul_mv(mb, m.points[i].anchor_b);
            V3 dp = dc + (rb - ra);
            m.points[i].separation = m.points[i].base_separation + dot(dp, n);
            m.points[i].normal_velocity = 0.0f;
            m.points[i].persisted = true;
          }
        }
#pragma omp atomic
        w->recycled++;
        return;
      }
    }
  }
  c.cached_rot_a = xa.q;
  c.cached_rot_b = xb.q;
  c.cached_rel = inv_mul_wxf(xa, xb);
  c.flags |= cRelativeValid;
  bool touching = update_contact(w, c, sa.local_center, xa, sb.local_center, xb);
  if (touching && !was_touching) { c.flags |= cSimStarted; bits[cid] = 1; }
  else if (!touching && was_touching) { c.flags |= cSimStopped; bits[cid] = 1; }
  if (touching && c.manifold_count > 0) {
    for (int i = 0; i < c.manifold.point_count; ++i)
      c.manifold.points[i].base_separation = c.manifold.points[i].separation;
  }
}

// collide_pass.rs:164 collide + :386 collide_state_pass
void collide(nso_world* w) {
  w->recycled = 0;
  std::vector<uint8_t> bits(w->contacts.size(), 0);
  const int n_ = (int)w->contacts.size();
#pragma omp parallel for schedule(dynamic, 64) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int i = 0; i < n_; ++i)
    if (w->contacts[i].contact_id != -1) collide_one(w, i, bits);
  for (size_t i = 0; i < bits.size(); ++i) {
    if (!bits[i]) continue;
    Contact& c = w->contacts[i];
    uint32_t f = c.flags;
    if (f == 0) continue;
    if (f & cSimDisjoint) {
      destroy_contact(w, (int)i);
    } else if (f & cSimStarted) {
      c.flags &= ~cSimStarted;
      c.flags |= cTouching;
      add_contact_to_graph(w, (int)i);
    } else if (f & cSimStopped) {
      c.flags &= ~cSimStopped;
      c.flags &= ~cTouching;
      int color = c.color_index, local = c.local_index;
      c.color_index = -1;
      c.local_index = -1;
      remove_contact_from_graph(w, c.body_a, c.body_b, color, local);
    }
  }
}

BodyState state_at(nso_world* w, int i) {
  if (i >= 0) return w->awake_states[i];
  BodyState s;
  s.v = v3(0, 0, 0); s.w = v3(0, 0, 0); s.dp = v3(0, 0, 0); s.flags = 0; s.dq = qid();
  return s;
}
void set_state(nso_world* w, int i, const BodyState& s) {
  if (i >= 0 && (s.flags & kDynamicFlag)) w->awake_states[i] = s;
}

// contact_solver.rs:445 prepare_contact_constraint
ContactConstraint prepare_contact(nso_world* w, int cid, Softness soft, Softness static_soft, real ws) {
  real inv_tau = 1.0f / speculative_distance();
  const Contact& ct = w->contacts[cid];
  ContactConstraint c;
  std::memset(&c, 0, sizeof(c));
  c.contact_id = cid;
  int ia = ct.encoded_a >= 0 ? ct.encoded_a : -1;
  int ib = ct.encoded_b >= 0 ? ct.encoded_b : -1;
  c.index_a = ia; c.index_b = ib;
  if (ia >= 0) { c.inv_mass_a = w->awake_sims[ia].inv_mass; c.inv_ia = sym_from(w->awake_sims[ia].inv_inertia_world); }
  else { c.inv_mass_a = 0.0f; c.inv_ia = sym_zero(); }
  if (ib >= 0) { c.inv_mass_b = w->awake_sims[ib].inv_mass; c.inv_ib = sym_from(w->awake_sims[ib].inv_inertia_world); }
  else { c.inv_mass_b = 0.0f; c.inv_ib = sym_zero(); }
  c.friction = ct.friction;
  c.restitution = ct.restitution;
  c.rolling_resistance = ct.rolling;
  c.is_static = (ct.flags & cStatic) != 0;
  c.softness = c.is_static ? static_soft : soft;
  Sym inv_iab = sym_add(c.inv_ia, c.inv_ib);
  c.rolling_mass = c.rolling_resistance > 0.0f ? sym_invert(inv_iab) : sym_zero();
  const Manifold& man = ct.manifold;
  ManifoldConstraint& mc = c.m;
  mc.point_count = man.point_count;
  mc.normal = man.normal;
  mc.tangent1 = perp(man.normal);
  mc.tangent2 = cross(mc.tangent1, man.normal);
  mc.tangent_velocity1 = dot(ct.tangent_velocity, mc.tangent1);
  mc.tangent_velocity2 = dot(ct.tangent_velocity, mc.tangent2);
  mc.twist_impulse = ws * man.twist_impulse;
  mc.rolling_impulse = c.rolling_resistance > 0.0f ? ws * man.rolling_impulse : v3(0, 0, 0);
  mc.friction_impulse = v2(ws * dot(man.friction_impulse, mc.tangent1), ws * dot(man.friction_impulse, mc.tangent2));
  V3 normal = mc.normal, t1 = mc.tangent1, t2 = mc.tangent2;
  V3 ca = v3(0, 0, 0), cb = v3(0, 0, 0);
  real tw = 0.0f;
  for (int i = 0; i < man.point_count; ++i) {
    const ManifoldPoint& mp = man.points[i];
    ConstraintPoint& cp = mc.points[i];
    cp.r_a = mp.anchor_a;
    cp.r_b = mp.anchor_b;
    cp.base_separation = mp.separation - dot(cp.r_b - cp.r_a, normal);
    cp.normal_impulse = ws * mp.normal_impulse;
    cp.total_normal_impulse = 0.0f;
    cp.relative_velocity = 0.0f;
    cp.restitution_impulse = 0.0f;
    real weight = clampf(2.0f - mp.separation * inv_tau, kMinFrictionWeight, 1.0f);
    ca = ca + weight * cp.r_a;
    cb = cb + weight * cp.r_b;
    tw += weight;
    V3 rna = cross(cp.r_a, normal), rnb = cross(cp.r_b, normal);
    real k = c.inv_mass_a + c.inv_mass_b;
    k += dot(rna, sym_mv(c.inv_ia, rna));
    k += dot(rnb, sym_mv(c.inv_ib, rnb));
    cp.normal_mass = k > 0.0f ? 1.0f / k : 0.0f;
  }
  if (tw > 0.0f) {
    ca = (1.0f / tw) * ca;
    cb = (1.0f / tw) * cb;
    mc.center_a = ca; mc.center_b = cb;
  } else {
    mc.center_a = v3(0, 0, 0); mc.center_b = v3(0, 0, 0);
  }
  for (int i = 0; i < man.point_count; ++i) {
    V3 d = mc.points[i].r_a - mc.center_a;
    mc.points[i].lever_arm = std::sqrt(dot(d, d));
  }
  {
    V3 rta1 = cross(mc.center_a, t1), rta2 = cross(mc.center_a, t2);
    V3 rtb1 = cross(mc.center_b, t1), rtb2 = cross(mc.center_b, t2);
    V3 ia1 = sym_mv(c.inv_ia, rta1), ia2 = sym_mv(c.inv_ia, rta2);
    V3 ib1 = sym_mv(c.inv_ib, rtb1), ib2 = sym_mv(c.inv_ib, rtb2);
    real msum = c.inv_mass_a + c.inv_mass_b;
    real kxx = (msum + dot(rta1, ia1)) + dot(rtb1, ib1);
    real kyy = (msum + dot(rta2, ia2)) + dot(rtb2, ib2);
    real kxy = dot(rta1, ia2) + dot(rtb1, ib2);
    real d = kxx * kyy - kxy * kxy;
    bool valid = absf(d) > 1000.0f * kMinPositive && tw > 0.0f;
    real inv = valid ? 1.0f / d : 0.0f;
    mc.tangent_mass.cx = v2(inv * kyy, -(inv * kxy));
    mc.tangent_mass.cy = v2(-(inv * kxy), inv * kxx);
  }
  real ktw = dot(normal, sym_mv(inv_iab, normal));
  mc.twist_mass = ktw > 0.0f ? 1.0f / ktw : 0.0f;
  if (ct.restitution > 0.0f) {
    BodyState sa = state_at(w, ia), sb = state_at(w, ib);
    for (int i = 0; i < man.point_count; ++i) {
      ConstraintPoint& cp = mc.points[i];
      V3 vra = sa.v + cross(sa.w, cp.r_a);
      V3 vrb = sb.v + cross(sb.w, cp.r_b);
      cp.relative_velocity = dot(normal, vrb - vra);
    }
  }
  return c;
}

// overflow_contact_solver.rs:92 prepare_overflow_contacts
void prepare_overflow(nso_world* w, Softness soft, Softness static_soft) {
  w->overflow.clear();
  real ws = w->def.enable_warm_starting ? 1.0f : 0.0f;
  real inv_tau = 1.0f / speculative_distance();
  for (int cid : w->colors[kOverflowIndex].overflow) {
    Contact& ct = w->contacts[cid];
    OverflowConstraint c;
    std::memset(&c, 0, sizeof(c));
    int ia = ct.encoded_a >= 0 ? ct.encoded_a : -1;
    int ib = ct.encoded_b >= 0 ? ct.encoded_b : -1;
    c.contact_id = cid; c.index_a = ia; c.index_b = ib;
    c.inv_ia = m3zero(); c.inv_ib = m3zero();
    if (ia >= 0) { c.inv_mass_a = w->awake_sims[ia].inv_mass; c.inv_ia = w->awake_sims[ia].inv_inertia_world; }
    if (ib >= 0) { c.inv_mass_b = w->awake_sims[ib].inv_mass; c.inv_ib = w->awake_sims[ib].inv_inertia_world; }
    real mA = c.inv_mass_a, mB = c.inv_mass_b;
    M3 iA = c.inv_ia, iB = c.inv_ib;
    c.rolling_mass = invert_matrix(add_mm(iA, iB));
    c.softness = (ct.flags & cStatic) ? static_soft : soft;
    c.friction = ct.friction; c.restitution = ct.restitution; c.rolling_resistance = ct.rolling;
    bool sample = ct.restitution > 0.0f;
    if (sample) w->any_restitution = true;
    V3 va = v3(0, 0, 0), wa = v3(0, 0, 0), vb = v3(0, 0, 0), wb = v3(0, 0, 0);
    if (sample) {
      if (ia >= 0) { va = w->awake_states[ia].v; wa = w->awake_states[ia].w; }
      if (ib >= 0) { vb = w->awake_states[ib].v; wb = w->awake_states[ib].w; }
    }
    c.manifold_count = ct.manifold_count;
    if (ct.manifold_count > 0) {
      Manifold& man = ct.manifold;
      ManifoldConstraint& mc = c.m;
      int pc = man.point_count;
      V3 n = man.normal, t1 = perp(n), t2 = cross(t1, n);
      mc.point_count = pc; mc.normal = n; mc.tangent1 = t1; mc.tangent2 = t2;
      mc.tangent_velocity1 = dot(ct.tangent_velocity, t1);
      mc.tangent_velocity2 = dot(ct.tangent_velocity, t2);
      V3 ca = v3(0, 0, 0), cb = v3(0, 0, 0);
      real tw = 0.0f;
      for (int i = 0; i < pc; ++i) {
        ConstraintPoint cp;
        std::memset(&cp, 0, sizeof(cp));
        const ManifoldPoint& mp = man.points[i];
        cp.r_a = mp.anchor_a; cp.r_b = mp.anchor_b;
        real s = mp.separation;
        cp.base_separation = s - dot(cp.r_b - cp.r_a, n);
        cp.normal_impulse = ws * mp.normal_impulse;
        V3 ra = cp.r_a, rb = cp.r_b;
        V3 rna = cross(ra, n), rnb = cross(rb, n);
        real k = mA + mB + dot(rna, mul_mv(iA, rna)) + dot(rnb, mul_mv(iB, rnb));
        cp.normal_mass = k > 0.0f ? 1.0f / k : 0.0f;
        if (sample) {
          V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
          cp.relative_velocity = dot(n, vrb - vra);
        } else {
          cp.relative_velocity = 0.0f;
        }
        man.points[i].normal_velocity = 0.0f;
        real weight = clampf(2.0f - s * inv_tau, kMinFrictionWeight, 1.0f);
        ca = mul_add(ca, weight, ra);
        cb = mul_add(cb, weight, rb);
        tw += weight;
        mc.points[i] = cp;
      }
      real iw = 1.0f / tw;
      ca = iw * ca; cb = iw * cb;
      mc.center_a = ca; mc.center_b = cb;
      for (int i = 0; i < pc; ++i) mc.points[i].lever_arm = distance(mc.points[i].r_a, ca);
      V3 rta1 = cross(ca, t1), rta2 = cross(ca, t2), rtb1 = cross(cb, t1), rtb2 = cross(cb, t2);
      M2 k;
      k.cx.x = mA + mB + dot(rta1, mul_mv(iA, rta1)) + dot(rtb1, mul_mv(iB, rtb1));
      k.cy.y = mA + mB + dot(rta2, mul_mv(iA, rta2)) + dot(rtb2, mul_mv(iB, rtb2));
      k.cx.y = dot(rta1, mul_mv(iA, rta2)) + dot(rtb1, mul_mv(iB, rtb2));
      k.cy.x = k.cx.y;
      mc.tangent_mass = invert2(k);
      mc.friction_impulse = v2(ws * dot(man.friction_impulse, t1), ws * dot(man.friction_impulse, t2));
      real ktw = dot(n, mul_mv(add_mm(iA, iB), n));
      mc.twist_mass = ktw > 0.0f ? 1.0f / ktw : 0.0f;
      mc.twist_impulse = ws * man.twist_impulse;
      mc.rolling_impulse = ws * man.rolling_impulse;
    }
    w->overflow.push_back(c);
  }
}

// solver_prepare.rs:269 prepare_all_contacts (joints first, overflow, then colors)
void prepare_all(nso_world* w) {
  w->any_restitution = false;
  prepare_joints(w->joints, w->awake_sims, w->static_sims, w->bodies.data(), w->ctx.h, w->ctx.inv_h,
                 w->def.enable_warm_starting ? 1.0f : 0.0f);
  real hz = minf(w->def.contact_hertz, 0.125f * w->ctx.inv_h);
  Softness soft = make_soft(hz, w->def.contact_damping_ratio, w->ctx.h);
  Softness stat = make_soft(2.0f * hz, 0.5f * w->def.contact_damping_ratio, w->ctx.h);
  prepare_overflow(w, soft, stat);
  real ws = w->def.enable_warm_starting ? 1.0f : 0.0f;
  for (int ci = 0; ci < kOverflowIndex; ++ci) {
    const std::vector<int>& ids = w->colors[ci].convex;
    std::vector<ContactConstraint>& out = w->constraints[ci];
    out.resize(ids.size());
    const int n_ = (int)ids.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
    for (int k = 0; k < n_; ++k) out[k] = prepare_contact(w, ids[k], soft, stat, ws);
    for (int cid : ids)
      if (w->contacts[cid].restitution > 0.0f) w->any_restitution = true;
  }
}

// solver_integration.rs:263 integrate_velocities_range
void integrate_velocities(nso_world* w, real h) {
  V3 g = v3(w->def.gravity[0], w->def.gravity[1], w->def.gravity[2]);
  const int n_ = (int)w->awake_sims.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int i = 0; i < n_; ++i) {
    const BodySim& sim = w->awake_sims[i];
    BodyState& st = w->awake_states[i];
    V3 v = st.v, wv = st.w;
    real ld = 1.0f / (1.0f + h * sim.linear_damping);
    real ad = 1.0f / (1.0f + h * sim.angular_damping);
    real gs = sim.inv_mass > 0.0f ? sim.gravity_scale : 0.0f;
    V3 lvd = blend2(h * sim.inv_mass, sim.force, h * gs, g);
    v = mul_add(lvd, ld, v);
    V3 avd = h * mul_mv(sim.inv_inertia_world, sim.torque);
    wv = mul_add(avd, ad, wv);
    if (sim.flags & kGyroscopic) {
      Q q0 = sim.transform.q;
      Q q = mul_quat(st.dq, q0);
      V3 om1 = inv_rotate(q, wv);
      V3 om2 = om1;
      real i00 = sim.inertia.cx.x, i01 = sim.inertia.cy.x, i02 = sim.inertia.cz.x;
      real i11 = sim.inertia.cy.y, i12 = sim.inertia.cz.y, i22 = sim.inertia.cz.z;
      {
        real w1 = om2.x, w2 = om2.y, w3 = om2.z;
        real iw1 = i00 * w1 + i01 * w2 + i02 * w3;
        real iw2 = i01 * w1 + i11 * w2 + i12 * w3;
        real iw3 = i02 * w1 + i12 * w2 + i22 * w3;
        V3 dw = om2 - om1;
        V3 b = v3(i00 * dw.x + i01 * dw.y + i02 * dw.z + h * (w2 * iw3 - w3 * iw2),
                  i01 * dw.x + i11 * dw.y + i12 * dw.z + h * (w3 * iw1 - w1 * iw3),
                  i02 * dw.x + i12 * dw.y + i22 * dw.z + h * (w1 * iw2 - w2 * iw1));
        M3 J = m3(v3(i00 + h * (w2 * i02 - w3 * i01), i01 + h * (w3 * i00 - w1 * i02 - iw3),
                     i02 + h * (w1 * i01 - w2 * i00 + iw2)),
                  v3(i01 + h * (w2 * i12 - w3 * i11 + iw3), i11 + h * (w3 * i01 - w1 * i12),
                     i12 + h * (w1 * i11 - w2 * i01 - iw1)),
                  v3(i02 + h * (w2 * i22 - w3 * i12 - iw2), i12 + h * (w3 * i02 - w1 * i22 + iw1),
                     i22 + h * (w1 * i12 - w2 * i02)));
        om2 = om2 - solve3(J, b);
      }
      wv = rotate(q, om2);
    }
    st.v = v;
    st.w = wv;
  }
}

// solver_integration.rs:377 integrate_positions_range
void integrate_positions(nso_world* w, real h, real inv_dt) {
  real maxl = w->def.max_linear_speed;
  real maxa = kMaxRotation * inv_dt;
  real maxl2 = maxl * maxl, maxa2 = maxa * maxa;
  const int n_ = (int)w->awake_states.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int i_ = 0; i_ < n_; ++i_) {
    BodyState& st = w->awake_states[i_];
    V3 v = st.v, wv = st.w;
    v.x = (st.flags & kLockLinX) ? 0.0f : v.x;
    v.y = (st.flags & kLockLinY) ? 0.0f : v.y;
    v.z = (st.flags & kLockLinZ) ? 0.0f : v.z;
    wv.x = (st.flags & kLockAngX) ? 0.0f : wv.x;
    wv.y = (st.flags & kLockAngY) ? 0.0f : wv.y;
    wv.z = (st.flags & kLockAngZ) ? 0.0f : wv.z;
    if (dot(v, v) > maxl2) {
      real ratio = maxl / length(v);
      v = ratio * v;
      st.flags |= kIsSpeedCapped;
    }
    if (dot(wv, wv) > maxa2 && (st.flags & kAllowFastRotation) == 0) {
      real ratio = maxa / length(wv);
      wv = ratio * wv;
      st.flags |= kIsSpeedCapped;
    }
    st.v = v;
    st.w = wv;
    st.dp = mul_add(st.dp, h, v);
    st.dq = integrate_rotation(st.dq, h * wv);
  }
}

// contact_solver.rs:697 warm_start_contacts_body
void warm_start_color(nso_world* w, int ci) {
  auto& list_ = w->constraints[ci];
  const int n_ = (int)list_.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int k_ = 0; k_ < n_; ++k_) {
    const ContactConstraint& c = list_[k_];
    const ManifoldConstraint& cm = c.m;
    V3 li = v3(0, 0, 0), aia = v3(0, 0, 0), aib = v3(0, 0, 0);
    real tni = 0.0f;
    V3 moa = v3(0, 0, 0), mob = v3(0, 0, 0);
    for (int p = 0; p < cm.point_count; ++p) {
      const ConstraintPoint& cp = cm.points[p];
      tni += cp.normal_impulse;
      moa = mul_add(moa, cp.normal_impulse, cp.r_a);
      mob = mul_add(mob, cp.normal_impulse, cp.r_b);
    }
    V3 n = cm.normal;
    V3 fi = cm.friction_impulse.x * cm.tangent1;
    fi = mul_add(fi, cm.friction_impulse.y, cm.tangent2);
    V3 lin = mul_add(fi, tni, n);
    V3 twi = cm.twist_impulse * n;
    V3 anga = cross(moa, n) + cross(cm.center_a, fi) + twi;
    V3 angb = cross(mob, n) + cross(cm.center_b, fi) + twi;
    if (c.rolling_resistance > 0.0f) { anga = anga + cm.rolling_impulse; angb = angb + cm.rolling_impulse; }
    li = li + lin; aia = aia + anga; aib = aib + angb;
    BodyState ba = state_at(w, c.index_a), bb = state_at(w, c.index_b);
    ba.w = ba.w - sym_mv(c.inv_ia, aia);
    ba.v = ba.v - c.inv_mass_a * li;
    bb.w = bb.w + sym_mv(c.inv_ib, aib);
    bb.v = bb.v + c.inv_mass_b * li;
    set_state(w, c.index_a, ba);
    set_state(w, c.index_b, bb);
  }
}

// contact_solver.rs:796 push_contacts_body
void push_color(nso_world* w, int ci) {
  const StepContext& ctx = w->ctx;
  real inv_h = ctx.inv_h;
  real cs = -w->def.contact_speed;
  real dbr = ctx.contact_softness.mass_scale * ctx.contact_softness.bias_rate;
  real dms = ctx.contact_softness.mass_scale, dis = ctx.contact_softness.impulse_scale;
  real sbr = ctx.static_softness.mass_scale * ctx.static_softness.bias_rate;
  real sms = ctx.static_softness.mass_scale, sis = ctx.static_softness.impulse_scale;
  auto& list_ = w->constraints[ci];
  const int n_ = (int)list_.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int k_ = 0; k_ < n_; ++k_) {
    ContactConstraint& c = list_[k_];
    BodyState ba = state_at(w, c.index_a), bb = state_at(w, c.index_b);
    real br = c.is_static ? sbr : dbr, ms = c.is_static ? sms : dms, is = c.is_static ? sis : dis;
    V3 dp = bb.dp - ba.dp;
    real im = c.inv_mass_a + c.inv_mass_b;
    ManifoldConstraint& cm = c.m;
    V3 n = cm.normal;
    real ns = dot(n, dp);
    V3 na = inv_rotate_wide(ba.dq, n), nb = inv_rotate_wide(bb.dq, n);
    real lnv = dot(n, bb.v - ba.v);
    real mi = 0.0f;
    for (int p = 0; p < cm.point_count; ++p) {
      ConstraintPoint& cp = cm.points[p];
      real s = (ns + (dot(nb, cp.r_b) - dot(na, cp.r_a))) + cp.base_separation;
      bool sep = s > 0.0f;
      real spec_bias = s * inv_h;
      real ovl = maxf(br * s, cs);
      real vb = sep ? spec_bias : ovl;
      real pms = sep ? 1.0f : ms;
      real pis = sep ? 0.0f : is;
      V3 ua = cross(cp.r_a, n), ub = cross(cp.r_b, n);
      V3 ga = sym_mv(c.inv_ia, ua), gb = sym_mv(c.inv_ib, ub);
      real vn = lnv + (dot(ub, bb.w) - dot(ua, ba.w));
      real neg = cp.normal_mass * (pms * vn + vb) + pis * cp.normal_impulse;
      real imp = maxf(-neg, -cp.normal_impulse);
      cp.normal_impulse = cp.normal_impulse + imp;
      lnv += im * imp;
      mi += imp;
      ba.w = ba.w - imp * ga;
      bb.w = bb.w + imp * gb;
    }
    V3 P = mi * n;
    ba.v = ba.v - c.inv_mass_a * P;
    bb.v = bb.v + c.inv_mass_b * P;
    set_state(w, c.index_a, ba);
    set_state(w, c.index_b, bb);
  }
}

// contact_solver.rs:927 solve_contacts_body (relax)
void relax_color(nso_world* w, int ci) {
  real inv_h = w->ctx.inv_h;
  real eps = kEps;
  auto& list_ = w->constraints[ci];
  const int n_ = (int)list_.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int k_ = 0; k_ < n_; ++k_) {
    ContactConstraint& c = list_[k_];
    BodyState ba = state_at(w, c.index_a), bb = state_at(w, c.index_b);
    bool any_rolling = c.rolling_resistance > 0.0f;
    V3 dp = bb.dp - ba.dp;
    real im = c.inv_mass_a + c.inv_mass_b;
    ManifoldConstraint& cm = c.m;
    V3 n = cm.normal;
    real ns = dot(n, dp);
    V3 na = inv_rotate_wide(ba.dq, n), nb = inv_rotate_wide(bb.dq, n);
    V3 dv = bb.v - ba.v;
    real lnv = dot(n, dv);
    real lt1 = dot(cm.tangent1, dv) - cm.tangent_velocity1;
    real lt2 = dot(cm.tangent2, dv) - cm.tangent_velocity2;
    real mi = 0.0f, tni = 0.0f, ttl = 0.0f;
    for (int p = 0; p < cm.point_count; ++p) {
      ConstraintPoint& cp = cm.points[p];
      real s = (ns + (dot(nb, cp.r_b) - dot(na, cp.r_a))) + cp.base_separation;
      real vb = maxf(0.0f, s * inv_h);
      V3 ua = cross(cp.r_a, n), ub = cross(cp.r_b, n);
      V3 ga = sym_mv(c.inv_ia, ua), gb = sym_mv(c.inv_ib, ub);
      real vn = lnv + (dot(ub, bb.w) - dot(ua, ba.w));
      real neg = cp.normal_mass * (vn + vb);
      real imp = maxf(-neg, -cp.normal_impulse);
      real ni = cp.normal_impulse + imp;
      cp.normal_impulse = ni;
      cp.total_normal_impulse = cp.total_normal_impulse + ni;
      tni += ni;
      ttl += cp.lever_arm * ni;
      lnv += im * imp;
      mi += imp;
      ba.w = ba.w - imp * ga;
      bb.w = bb.w + imp * gb;
    }
    if (any_rolling) {
      V3 di = sym_mv(c.rolling_mass, ba.w - bb.w);
      V3 old = cm.rolling_impulse;
      cm.rolling_impulse = old + di;
      real mx = c.rolling_resistance * tni;
      real lsq = dot(cm.rolling_impulse, cm.rolling_impulse);
      bool mask = lsq > eps + mx * mx;
      real nrm = mx / (std::sqrt(lsq) + eps);
      real sc = mask ? nrm : 1.0f;
      V3 scaled = sc * cm.rolling_impulse;
      if (c.rolling_resistance == 0.0f) scaled = v3(0, 0, 0);
      cm.rolling_impulse = scaled;
      di = cm.rolling_impulse - old;
      ba.w = ba.w - sym_mv(c.inv_ia, di);
      bb.w = bb.w + sym_mv(c.inv_ib, di);
    }
    {
      real ts = dot(n, bb.w - ba.w);
      real ml = c.friction * ttl;
      real old = cm.twist_impulse;
      real imp = -(cm.twist_mass * ts);
      imp = maxf(-ml - old, minf(imp, ml - old));
      cm.twist_impulse = old + imp;
      ba.w = ba.w - imp * sym_mv(c.inv_ia, n);
      bb.w = bb.w + imp * sym_mv(c.inv_ib, n);
    }
    {
      V3 t1 = cm.tangent1, t2 = cm.tangent2;
      V3 ra = cm.center_a, rb = cm.center_b;
      V3 arv = cross(bb.w, rb) - cross(ba.w, ra);
      V2 vt = v2(lt1 + dot(arv, t1), lt2 + dot(arv, t2));
      V2 di = mul_mv2(cm.tangent_mass, vt);
      di = v2(-di.x, -di.y);
      V2 ni = v2(cm.friction_impulse.x + di.x, cm.friction_impulse.y + di.y);
      real mx = c.friction * tni;
      real lsq = ni.x * ni.x + ni.y * ni.y;
      bool mask = lsq > mx * mx;
      real nrm = mx / (std::sqrt(lsq) + eps);
      real sc = mask ? nrm : 1.0f;
      ni = v2(sc * ni.x, sc * ni.y);
      di = v2(ni.x - cm.friction_impulse.x, ni.y - cm.friction_impulse.y);
      cm.friction_impulse = ni;
      V3 P = di.x * t1;
      P = P + di.y * t2;
      ba.w = ba.w - sym_mv(c.inv_ia, cross(ra, P));
      bb.w = bb.w + sym_mv(c.inv_ib, cross(rb, P));
      P = P + mi * n;
      ba.v = ba.v - c.inv_mass_a * P;
      bb.v = bb.v + c.inv_mass_b * P;
    }
    set_state(w, c.index_a, ba);
    set_state(w, c.index_b, bb);
  }
}

// contact_solver.rs:1135 apply_restitution_body
void restitution_color(nso_world* w, int ci) {
  real inv_h = w->ctx.inv_h;
  real nrt = -w->def.restitution_threshold;
  auto& list_ = w->constraints[ci];
  const int n_ = (int)list_.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int k_ = 0; k_ < n_; ++k_) {
    ContactConstraint& c = list_[k_];
    if (c.restitution == 0.0f) continue;
    BodyState ba = state_at(w, c.index_a), bb = state_at(w, c.index_b);
    bool rmask = c.restitution > 0.0f;
    V3 dp = bb.dp - ba.dp;
    ManifoldConstraint& cm = c.m;
    V3 n = cm.normal;
    real ns = dot(n, dp);
    V3 na = inv_rotate_wide(ba.dq, n), nb = inv_rotate_wide(bb.dq, n);
    for (int p = 0; p < cm.point_count; ++p) {
      ConstraintPoint& cp = cm.points[p];
      real s = (ns + (dot(nb, cp.r_b) - dot(na, cp.r_a))) + cp.base_separation;
      real nm = rmask ? cp.normal_mass : 0.0f;
      real comp = cp.total_normal_impulse - cp.restitution_impulse;
      bool armed = rmask && cp.relative_velocity < nrt && comp > 0.0f;
      real sb = maxf(0.0f, s * inv_h);
      real vb = armed ? c.restitution * cp.relative_velocity : sb;
      V3 vra = ba.v + cross(ba.w, cp.r_a), vrb = bb.v + cross(bb.w, cp.r_b);
      real vn = dot(vrb - vra, n);
      real neg = nm * (vn + vb);
      real ni = maxf(cp.normal_impulse - neg, 0.0f);
      real imp = ni - cp.normal_impulse;
      real app = minf(maxf(-nm * vn, 0.0f), maxf(imp, 0.0f));
      real allow = c.restitution * (comp + app) - cp.restitution_impulse;
      real mx = app + maxf(allow, 0.0f);
      imp = armed ? minf(imp, mx) : imp;
      cp.normal_impulse = cp.normal_impulse + imp;
      cp.restitution_impulse = cp.restitution_impulse + (imp - app);
      cp.total_normal_impulse = cp.total_normal_impulse + imp;
      V3 P = imp * n;
      ba.w = ba.w - sym_mv(c.inv_ia, cross(cp.r_a, P));
      ba.v = ba.v - c.inv_mass_a * P;
      bb.w = bb.w + sym_mv(c.inv_ib, cross(cp.r_b, P));
      bb.v = bb.v + c.inv_mass_b * P;
    }
    set_state(w, c.index_a, ba);
    set_state(w, c.index_b, bb);
  }
}

// contact_solver.rs:1258 store_impulses_body
void store_color(nso_world* w, int ci) {
  auto& list_ = w->constraints[ci];
  const int n_ = (int)list_.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int k_ = 0; k_ < n_; ++k_) {
    const ContactConstraint& c = list_[k_];
    Contact& ct = w->contacts[c.contact_id];
    if (ct.manifold_count <= 0) continue;
    const ManifoldConstraint& cm = c.m;
    Manifold& out = ct.manifold;
    int cnt = min_i(out.point_count, cm.point_count);
    for (int p = 0; p < cnt; ++p) {
      out.points[p].normal_impulse = cm.points[p].normal_impulse;
      out.points[p].total_normal_impulse = cm.points[p].total_normal_impulse;
    }
    out.twist_impulse = cm.twist_impulse;
    out.friction_impulse = cm.friction_impulse.x * cm.tangent1 + cm.friction_impulse.y * cm.tangent2;
    out.rolling_impulse = cm.rolling_impulse;
  }
}

// overflow_contact_solver.rs:308-700 sequential overflow color
void overflow_store_velocity(nso_world* w, int i, uint32_t flags, V3 v, V3 wv) {
  if (i >= 0 && (flags & kDynamicFlag)) { w->awake_states[i].v = v; w->awake_states[i].w = wv; }
}
void warm_start_overflow(nso_world* w) {
  for (const OverflowConstraint& c : w->overflow) {
    V3 li = v3(0, 0, 0), aia = v3(0, 0, 0), aib = v3(0, 0, 0);
    for (int mi = 0; mi < c.manifold_count; ++mi) {
      const ManifoldConstraint& mc = c.m;
      V3 n = mc.normal;
      real tni = 0.0f;
      V3 moa = v3(0, 0, 0), mob = v3(0, 0, 0);
      for (int j = 0; j < mc.point_count; ++j) {
        const ConstraintPoint& cp = mc.points[j];
        tni += cp.normal_impulse;
        moa = mul_add(moa, cp.normal_impulse, cp.r_a);
        mob = mul_add(mob, cp.normal_impulse, cp.r_b);
      }
      V3 fi = mc.friction_impulse.x * mc.tangent1;
      fi = mul_add(fi, mc.friction_impulse.y, mc.tangent2);
      li = li + mul_add(fi, tni, n);
      V3 twi = mc.twist_impulse * n;
      V3 anga = (cross(moa, n) + cross(mc.center_a, fi)) + twi;
      V3 angb = (cross(mob, n) + cross(mc.center_b, fi)) + twi;
      aia = aia + (anga + mc.rolling_impulse);
      aib = aib + (angb + mc.rolling_impulse);
    }
    if (c.index_a >= 0 && (w->awake_states[c.index_a].flags & kDynamicFlag)) {
      BodyState& s = w->awake_states[c.index_a];
      s.v = mul_sub(s.v, c.inv_mass_a, li);
      s.w = s.w - mul_mv(c.inv_ia, aia);
    }
    if (c.index_b >= 0 && (w->awake_states[c.index_b].flags & kDynamicFlag)) {
      BodyState& s = w->awake_states[c.index_b];
      s.v = mul_add(s.v, c.inv_mass_b, li);
      s.w = s.w + mul_mv(c.inv_ib, aib);
    }
  }
}
void push_overflow(nso_world* w) {
  real inv_h = w->ctx.inv_h;
  real cs = w->def.contact_speed;
  for (OverflowConstraint& c : w->overflow) {
    real mA = c.inv_mass_a, mB = c.inv_mass_b;
    M3 iA = c.inv_ia, iB = c.inv_ib;
    BodyState sa = state_at(w, c.index_a), sb = state_at(w, c.index_b);
    V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
    Q dqa = sa.dq, dqb = sb.dq;
    V3 dp = sb.dp - sa.dp;
    Softness soft = c.softness;
    for (int mi = 0; mi < c.manifold_count; ++mi) {
      ManifoldConstraint& mc = c.m;
      V3 n = mc.normal;
      for (int p = 0; p < mc.point_count; ++p) {
        ConstraintPoint& cp = mc.points[p];
        V3 ra = cp.r_a, rb = cp.r_b;
        V3 ds = dp + (rotate(dqb, rb) - rotate(dqa, ra));
        real s = dot(ds, n) + cp.base_separation;
        real vbias, mscale, iscale;
        if (s > 0.0f) { vbias = s * inv_h; mscale = 1.0f; iscale = 0.0f; }
        else {
          vbias = maxf(soft.mass_scale * soft.bias_rate * s, -cs);
          mscale = soft.mass_scale; iscale = soft.impulse_scale;
        }
        V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
        real vn = dot(vrb - vra, n);
        real ni0 = cp.normal_impulse;
        real di = -cp.normal_mass * (mscale * vn + vbias) - iscale * ni0;
        real ni = maxf(ni0 + di, 0.0f);
        di = ni - ni0;
        cp.normal_impulse = ni;
        V3 P = di * n;
        va = mul_sub(va, mA, P);
        wa = wa - mul_mv(iA, cross(ra, P));
        vb = mul_add(vb, mB, P);
        wb = wb + mul_mv(iB, cross(rb, P));
      }
    }
    overflow_store_velocity(w, c.index_a, sa.flags, va, wa);
    overflow_store_velocity(w, c.index_b, sb.flags, vb, wb);
  }
}
void relax_overflow(nso_world* w) {
  real inv_h = w->ctx.inv_h;
  for (OverflowConstraint& c : w->overflow) {
    real mA = c.inv_mass_a, mB = c.inv_mass_b;
    M3 iA = c.inv_ia, iB = c.inv_ib;
    BodyState sa = state_at(w, c.index_a), sb = state_at(w, c.index_b);
    V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
    Q dqa = sa.dq, dqb = sb.dq;
    V3 dp = sb.dp - sa.dp;
    real fr = c.friction, rr = c.rolling_resistance;
    for (int mi = 0; mi < c.manifold_count; ++mi) {
      ManifoldConstraint& mc = c.m;
      V3 n = mc.normal;
      real tni = 0.0f, ttl = 0.0f;
      for (int p = 0; p < mc.point_count; ++p) {
        ConstraintPoint& cp = mc.points[p];
        V3 ra = cp.r_a, rb = cp.r_b;
        V3 ds = dp + (rotate(dqb, rb) - rotate(dqa, ra));
        real s = dot(ds, n) + cp.base_separation;
        real vbias = s > 0.0f ? s * inv_h : 0.0f;
        V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
        real vn = dot(vrb - vra, n);
        real ni0 = cp.normal_impulse;
        real di = -cp.normal_mass * (vn + vbias);
        real ni = maxf(ni0 + di, 0.0f);
        di = ni - ni0;
        cp.normal_impulse = ni;
        cp.total_normal_impulse += ni;
        tni += ni;
        ttl += cp.lever_arm * ni;
        V3 P = di * n;
        va = mul_sub(va, mA, P);
        wa = wa - mul_mv(iA, cross(ra, P));
        vb = mul_add(vb, mB, P);
        wb = wb + mul_mv(iB, cross(rb, P));
      }
      {
        real ts = dot(n, wb - wa);
        real mx = fr * ttl;
        real di = -mc.twist_mass * ts;
        real old = mc.twist_impulse;
        mc.twist_impulse = clampf(old + di, -mx, mx);
        di = mc.twist_impulse - old;
        wa = wa - mul_mv(iA, di * n);
        wb = wb + mul_mv(iB, di * n);
      }
      if (rr > 0.0f) {
        V3 di = -mul_mv(c.rolling_mass, wb - wa);
        V3 old = mc.rolling_impulse;
        mc.rolling_impulse = old + di;
        real mx = rr * tni;
        real msq = dot(mc.rolling_impulse, mc.rolling_impulse);
        if (msq > mx * mx + kEps) mc.rolling_impulse = (mx / std::sqrt(msq)) * mc.rolling_impulse;
        di = mc.rolling_impulse - old;
        wa = wa - mul_mv(iA, di);
        wb = wb + mul_mv(iB, di);
      }
      {
        V3 t1 = mc.tangent1, t2 = mc.tangent2, ra = mc.center_a, rb = mc.center_b;
        V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
        V3 vr = vrb - vra;
        V2 vt = v2(dot(vr, t1) - mc.tangent_velocity1, dot(vr, t2) - mc.tangent_velocity2);
        V2 tm = mul_mv2(mc.tangent_mass, vt);
        V2 di = v2(-tm.x, -tm.y);
        V2 ni = v2(mc.friction_impulse.x + di.x, mc.friction_impulse.y + di.y);
        real mx = fr * tni;
        real lsq = dot2(ni, ni);
        if (lsq > mx * mx) {
          real sc = mx / std::sqrt(lsq);
          ni.x *= sc; ni.y *= sc;
        }
        di = v2(ni.x - mc.friction_impulse.x, ni.y - mc.friction_impulse.y);
        mc.friction_impulse = ni;
        V3 P = blend2(di.x, t1, di.y, t2);
        va = mul_sub(va, mA, P);
        wa = wa - mul_mv(iA, cross(ra, P));
        vb = mul_add(vb, mB, P);
        wb = wb + mul_mv(iB, cross(rb, P));
      }
    }
    overflow_store_velocity(w, c.index_a, sa.flags, va, wa);
    overflow_store_velocity(w, c.index_b, sb.flags, vb, wb);
  }
}
void restitution_overflow(nso_world* w) {
  real thr = w->def.restitution_threshold;
  real inv_h = w->ctx.inv_h;
  for (OverflowConstraint& c : w->overflow) {
    real rest = c.restitution;
    if (rest == 0.0f) continue;
    real mA = c.inv_mass_a, mB = c.inv_mass_b;
    M3 iA = c.inv_ia, iB = c.inv_ib;
    BodyState sa = state_at(w, c.index_a), sb = state_at(w, c.index_b);
    V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
    Q dqa = sa.dq, dqb = sb.dq;
    V3 dp = sb.dp - sa.dp;
    for (int mi = 0; mi < c.manifold_count; ++mi) {
      ManifoldConstraint& mc = c.m;
      V3 n = mc.normal;
      for (int p = 0; p < mc.point_count; ++p) {
        ConstraintPoint cp = mc.points[p];
        V3 ra = cp.r_a, rb = cp.r_b;
        real comp = cp.total_normal_impulse - cp.restitution_impulse;
        bool armed = rest > 0.0f && cp.relative_velocity < -thr && comp > 0.0f;
        real vbias;
        if (armed) vbias = rest * cp.relative_velocity;
        else {
          V3 ds = dp + (rotate(dqb, rb) - rotate(dqa, ra));
          real s = dot(ds, n) + cp.base_separation;
          vbias = s > 0.0f ? s * inv_h : 0.0f;
        }
        V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
        real vn = dot(vrb - vra, n);
        real imp = -cp.normal_mass * (vn + vbias);
        real ni = maxf(cp.normal_impulse + imp, 0.0f);
        imp = ni - cp.normal_impulse;
        real app = minf(maxf(-cp.normal_mass * vn, 0.0f), maxf(imp, 0.0f));
        if (armed) {
          real allow = rest * (comp + app) - cp.restitution_impulse;
          imp = minf(imp, app + maxf(allow, 0.0f));
        }
        mc.points[p].normal_impulse += imp;
        mc.points[p].restitution_impulse += imp - app;
        mc.points[p].total_normal_impulse += imp;
        V3 P = imp * n;
        va = mul_sub(va, mA, P);
        wa = wa - mul_mv(iA, cross(ra, P));
        vb = mul_add(vb, mB, P);
        wb = wb + mul_mv(iB, cross(rb, P));
      }
    }
    overflow_store_velocity(w, c.index_a, sa.flags, va, wa);
    overflow_store_velocity(w, c.index_b, sb.flags, vb, wb);
  }
}
void store_overflow(nso_world* w) {
  for (const OverflowConstraint& c : w->overflow) {
    if (c.manifold_count == 0) continue;
    Manifold& m = w->contacts[c.contact_id].manifold;
    const ManifoldConstraint& mc = c.m;
    m.twist_impulse = mc.twist_impulse;
    m.friction_impulse = blend2(mc.friction_impulse.x, mc.tangent1, mc.friction_impulse.y, mc.tangent2);
    m.rolling_impulse = mc.rolling_impulse;
    for (int p = 0; p < mc.point_count; ++p) {
      m.points[p].normal_impulse = mc.points[p].normal_impulse;
      m.points[p].total_normal_impulse = mc.points[p].total_normal_impulse;
    }
  }
}

// solver_stages.rs:543 solve_constraint_stages
void solve_stages(nso_world* w) {
  const StepContext& ctx = w->ctx;
  for (int sub = 0; sub < ctx.sub_step_count; ++sub) {
    integrate_velocities(w, ctx.h);
    warm_start_joints_color(w->joints, w->colors[kOverflowIndex].joints, w->awake_states, ctx.h);
    warm_start_overflow(w);
    for (int ci = 0; ci < kOverflowIndex; ++ci) {
      warm_start_joints_color(w->joints, w->colors[ci].joints, w->awake_states, ctx.h);
      warm_start_color(w, ci);
    }
    solve_joints_color(w->joints, w->colors[kOverflowIndex].joints, w->awake_states, ctx.h, ctx.inv_h, true);
    push_overflow(w);
    for (int ci = 0; ci < kOverflowIndex; ++ci) {
      solve_joints_color(w->joints, w->colors[ci].joints, w->awake_states, ctx.h, ctx.inv_h, true);
      push_color(w, ci);
    }
    integrate_positions(w, ctx.h, ctx.inv_dt);
    solve_joints_color(w->joints, w->colors[kOverflowIndex].joints, w->awake_states, ctx.h, ctx.inv_h, false);
    relax_overflow(w);
    for (int ci = 0; ci < kOverflowIndex; ++ci) {
      solve_joints_color(w->joints, w->colors[ci].joints, w->awake_states, ctx.h, ctx.inv_h, false);
      relax_color(w, ci);
    }
  }
  if (w->any_restitution && w->def.restitution_iterations > 0) {
    for (int it = 0; it < w->def.restitution_iterations; ++it) {
      restitution_overflow(w);
      for (int ci = 0; ci < kOverflowIndex; ++ci) restitution_color(w, ci);
    }
  }
  store_overflow(w);
  for (int ci = 0; ci < kOverflowIndex; ++ci) store_color(w, ci);
}

// ---------------------------------------------------------------------------------------------
// Continuous collision: continuous.rs:337 solve_continuous. Fast non-bullet bodies sweep their
// fast shapes against static shapes, in body order after finalize (solver_integration.rs:
// 540-566); then fast bullets sweep all their shapes against static shapes and the shapes of
// non-bullet dynamic bodies at their final poses, in body order (solver_integration.rs:949-958).

// shape_runtime.rs:434 get_shape_centroid
V3 shape_centroid(const Shape& s) {
  if (s.type == kHull) return s.hull.center;
  if (s.type == kSphere) return s.sphere.center;
  return lerp(s.capsule.c1, s.capsule.c2, 0.5f);
}

// shape_runtime.rs:643 make_shape_proxy
Proxy shape_proxy(const Shape& s) {
  Proxy p;
  if (s.type == kHull) {
    p.count = s.hull.vertex_count;
    for (int i = 0; i < p.count; ++i) p.pts[i] = s.hull.points[i];
    p.radius = 0.0f;
  } else if (s.type == kSphere) {
    p.count = 1;
    p.pts[0] = s.sphere.center;
    p.radius = s.sphere.radius;
  } else {
    p.count = 2;
    p.pts[0] = s.capsule.c1;
    p.pts[1] = s.capsule.c2;
    p.radius = s.capsule.radius;
  }
  return p;
}

// world_runtime.rs:929 make_relative_sweep
Sweep relative_sweep(const BodySim& b, Pos base) {
  Sweep s;
  s.c1 = sub_pos(b.center0, base);
  s.c2 = sub_pos(b.center, base);
  s.q1 = b.rotation0;
  s.q2 = b.transform.q;
  s.local_center = b.local_center;
  return s;
}

// continuous.rs:124 is_shape_fast (convex shapes)
bool is_shape_fast(const Shape& s, V3 centroid1, V3 centroid2, real rotation_chord, real safety_factor) {
  real radius;
  V3 lc = shape_centroid(s);
  if (s.type == kSphere) {
    radius = s.sphere.radius;
  } else if (s.type == kCapsule) {
    radius = 0.5f * distance(s.capsule.c1, s.capsule.c2) + s.capsule.radius;
  } else {
    const AABB& b = s.hull.bounds;  // internal_math.rs:426 farthest_point_on_aabb
    V3 f = v3((lc.x - b.lo.x) > (b.hi.x - lc.x) ? b.lo.x : b.hi.x, (lc.y - b.lo.y) > (b.hi.y - lc.y) ? b.lo.y : b.hi.y,
              (lc.z - b.lo.z) > (b.hi.z - lc.z) ? b.lo.z : b.hi.z);
    radius = distance(f, lc);
  }
  // shape_runtime.rs:547 compute_shape_min_extent
  real min_extent = s.type == kCapsule ? s.capsule.radius : s.type == kSphere ? s.sphere.radius : s.hull.inner_radius;
  real max_motion = distance(centroid1, centroid2) + rotation_chord * radius;
  return max_motion > safety_factor * min_extent;
}

// contact_creation.rs:113 should_bodies_collide (joints without collide_connected)
bool bodies_collide(nso_world* w, int ia, int ib) {
  const Body& ba = w->bodies[ia];
  const Body& bb = w->bodies[ib];
  if (ba.type != 2 && bb.type != 2) return false;
  const Body& scan = ba.joint_count < bb.joint_count ? ba : bb;
  int other = ba.joint_count < bb.joint_count ? bb.id : ba.id;
  if (scan.id < (int)w->body_joints.size())
    for (int jid : w->body_joints[scan.id]) {
      const Joint& j = w->joints[jid];
      int o = j.body_a == scan.id ? j.body_b : j.body_a;
      if (!j.collide_connected && o == other) return false;
    }
  return true;
}

// shape_runtime.rs:284 should_shapes_collide
bool shapes_collide(const Shape& a, const Shape& b) {
  if (a.group == b.group && a.group != 0) return a.group > 0;
  return (a.mask & b.category) != 0 && (a.category & b.mask) != 0;
}

// continuous.rs:210-302 continuous_query_callback: the filters, then the time of impact of the
// fast shape against one candidate at its own sweep, the best fraction so far as the bound
void continuous_candidate(nso_world* w, const Shape& fs, const Proxy& fp, const Sweep& sweep, Pos base,
                          int sid, real& fraction) {
  const Shape& ss = w->shapes[sid];
  if (ss.body_id == fs.body_id || !shapes_collide(fs, ss)) return;
  const Body& other = w->bodies[ss.body_id];
  if (sim_of(w, other).flags & kIsBullet) return;
  if (!bodies_collide(w, fs.body_id, ss.body_id)) return;
  Proxy sp = shape_proxy(ss);
  ToiOut o = time_of_impact(sp, fp, relative_sweep(sim_of(w, other), base), sweep, fraction);
  if (0.0f < o.fraction && o.fraction < fraction) fraction = o.fraction;
}

void solve_continuous(nso_world* w, int i) {
  BodySim& sim = w->awake_sims[i];
  BodyState& st = w->awake_states[i];
  Body& body = w->bodies[sim.body_id];
  const bool bullet = (sim.flags & kIsBullet) != 0;
  Pos base = sim.center0;
  Sweep sweep = relative_sweep(sim, base);
  Xf xf1 = xf(sweep.c1 - rotate(sweep.q1, sweep.local_center), sweep.q1);
  Xf xf2 = xf(sweep.c2 - rotate(sweep.q2, sweep.local_center), sweep.q2);
  real fraction = 1.0f;
  real rotation_chord = 2.0f * length(inv_mul_quat(sweep.q1, sweep.q2).v);
  for (int fid = body.head_shape; fid != -1; fid = w->shapes[fid].next_shape) {
    Shape& fs = w->shapes[fid];
    V3 lc = shape_centroid(fs);
    V3 centroid1 = xf_point(xf1, lc), centroid2 = xf_point(xf2, lc);
    AABB box1 = fs.aabb;
    AABB box2 = offset_aabb(shape_aabb_xf(fs, xf2), base);
    fs.aabb = box2;
    if (!bullet && !is_shape_fast(fs, centroid1, centroid2, rotation_chord, body.safety_factor)) continue;
    AABB swept = aabb(min3(box1.lo, box2.lo), max3(box1.hi, box2.hi));
    Proxy fp = shape_proxy(fs);
    // the static tree's proxies whose fat bounds overlap the swept box, in shape order (the
    // reference walks its tree; each time of impact is bounded by the best fraction so far)
    for (int sid = 0; sid < (int)w->shapes.size(); ++sid)
      if (w->shapes[sid].is_static && aabb_overlaps(w->fat[sid], swept))
        continuous_candidate(w, fs, fp, sweep, base, sid, fraction);
    // bullets also query the kinematic tree, then the dynamic tree (continuous.rs:429-448)
    if (bullet)
      for (int type = 1; type <= 2; ++type)
        for (int sid = 0; sid < (int)w->shapes.size(); ++sid)
          if (w->bodies[w->shapes[sid].body_id].type == type && aabb_overlaps(w->fat[sid], swept))
            continuous_candidate(w, fs, fp, sweep, base, sid, fraction);
  }
  real spec = speculative_distance();
  if (fraction < 1.0f) {
    Q q = nlerp(sweep.q1, sweep.q2, fraction);
    V3 c = lerp(sweep.c1, sweep.c2, fraction);
    V3 origin = c - rotate(q, sweep.local_center);
    WXf t = {offset_pos(base, origin), q};
    Pos center = offset_pos(base, c);
    sim.transform = t;
    sim.center = center;
    sim.rotation0 = q;
    sim.center0 = center;
    sim.flags |= kHadToi;
    // the gravity lost in the remaining time (other forces ignored, as the reference does)
    real time_loss = (1.0f - fraction) * w->ctx.dt;
    V3 g = v3(w->def.gravity[0], w->def.gravity[1], w->def.gravity[2]);
    V3 dv = (-time_loss * sim.gravity_scale) * g;
    dv.x = (st.flags & kLockLinX) ? 0.0f : dv.x;
    dv.y = (st.flags & kLockLinY) ? 0.0f : dv.y;
    dv.z = (st.flags & kLockLinZ) ? 0.0f : dv.z;
    st.v = st.v + dv;
    for (int sid = body.head_shape; sid != -1; sid = w->shapes[sid].next_shape) {
      Shape& sh = w->shapes[sid];
      AABB a = fat_shape_aabb(sh, t, spec);
      sh.aabb = a;
      if (!aabb_contains(w->fat[sid], a)) {
        w->fat[sid] = aabb_inflate(a, sh.aabb_margin);
        w->proxy_moved[sid] = 1;
      }
    }
  } else {
    sim.rotation0 = sim.transform.q;
    sim.center0 = sim.center;
    for (int sid = body.head_shape; sid != -1; sid = w->shapes[sid].next_shape) {
      Shape& sh = w->shapes[sid];
      if (!aabb_contains(w->fat[sid], sh.aabb)) {
        w->fat[sid] = aabb_inflate(sh.aabb, sh.aabb_margin);
        w->proxy_moved[sid] = 1;
      }
    }
  }
  // solver_integration.rs:556-564: the world inertia at the (possibly moved back) rotation
  M3 R = matrix_from_quat(sim.transform.q);
  sim.inv_inertia_world = mul_mm(mul_mm(R, sim.inv_inertia_local), transpose(R));
}

// solver_integration.rs:587 finalize_body_range (sleep disabled), then the continuous pass of
// the fast bodies in body order (solver_integration.rs:540-566)
void finalize(nso_world* w) {
  real dt = w->ctx.dt, inv_dt = w->ctx.inv_dt;
  real spec = speculative_distance();
  const int n_ = (int)w->awake_sims.size();
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n_ >= kParMin)
  for (int i = 0; i < n_; ++i) {
    BodyState& st = w->awake_states[i];
    BodySim& sim = w->awake_sims[i];
    V3 v = st.v, wv = st.w;
    V3 lom = inv_rotate(sim.transform.q, wv);
    V3 ldr = inv_rotate(sim.transform.q, st.dq.v);
    sim.center = offset_pos(sim.center, st.dp);
    sim.transform.q = normalize_quat(mul_quat(st.dq, sim.transform.q));
    V3 varc = modified_cross(abs3(lom), sim.max_extent);
    real maxv = length(v) + length(varc);
    V3 rarc = modified_cross(abs3(ldr), sim.max_extent);
    real maxdp = length(st.dp) + 2.0f * length(rarc);
    st.dp = v3(0, 0, 0);
    st.dq = qid();
    sim.transform.p = offset_pos(sim.center, -rotate(sim.transform.q, sim.local_center));
    Body& body = w->bodies[sim.body_id];
    sim.force = v3(0, 0, 0);
    sim.torque = v3(0, 0, 0);
    body.flags &= ~kTransient;
    sim.flags &= ~(kIsFast | kTransient);
    body.flags |= st.flags & kIsSpeedCapped;
    st.flags &= ~kTransient;
    body.sleep_time = 0.0f;
    real max_motion = maxf(maxdp, maxv * dt);
    (void)inv_dt;
    if (body.type == 2 && w->def.enable_continuous && max_motion > body.safety_factor * sim.min_extent) {
      sim.flags |= kIsFast;
#pragma omp atomic
      w->fast_flags_seen++;
    } else {
      sim.center0 = sim.center;
      sim.rotation0 = sim.transform.q;
    }
    M3 R = matrix_from_quat(sim.transform.q);
    sim.inv_inertia_world = mul_mm(mul_mm(R, sim.inv_inertia_local), transpose(R));
    if ((sim.flags & kIsFast) == 0) {
      for (int sid = body.head_shape; sid != -1; sid = w->shapes[sid].next_shape) {
        Shape& sh = w->shapes[sid];
        AABB a = fat_shape_aabb(sh, sim.transform, spec);
        sh.aabb = a;
        if (!aabb_contains(w->fat[sid], a)) {
          w->fat[sid] = aabb_inflate(a, sh.aabb_margin);
          w->proxy_moved[sid] = 1;
        }
      }
    }
  }
  for (int i = 0; i < n_; ++i)
    if ((w->awake_sims[i].flags & (kIsFast | kIsBullet)) == kIsFast) solve_continuous(w, i);
  // solver_integration.rs:949-958: the bullets, after every other body is final
  for (int i = 0; i < n_; ++i)
    if ((w->awake_sims[i].flags & (kIsFast | kIsBullet)) == (kIsFast | kIsBullet)) solve_continuous(w, i);
}

}  // namespace

extern "C" {

void nso_default_world_def(nso_world_def* d) {
  d->gravity[0] = 0.0f; d->gravity[1] = -10.0f; d->gravity[2] = 0.0f;
  d->enable_sleep = 0;
  d->enable_continuous = 1;
  d->enable_warm_starting = 1;
  d->contact_hertz = 30.0f;
  d->contact_damping_ratio = 10.0f;
  d->contact_speed = 3.0f;
  d->max_linear_speed = 400.0f;
  d->restitution_threshold = 1.0f;
  d->restitution_iterations = 2;
  d->joint_hertz = 60.0f;
  d->joint_damping_ratio = 2.0f;
}

nso_world* nso_create(const nso_world_def* def) {
  nso_world* w = new nso_world();
  w->def = *def;
  w->colors.resize(kGraphColorCount);
  w->color_bits.resize(kGraphColorCount);
  w->constraints.resize(kGraphColorCount);
  return w;
}

void nso_destroy(nso_world* w) { delete w; }

void nso_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }

// world_runtime.rs:1506 create_body (awake or static set only)
int nso_create_body(nso_world* w, const nso_body_def* d) {
  int id = (int)w->bodies.size();
  Body b;
  b.id = id;
  b.type = d->type;
  b.set_index = d->type == 0 ? 0 : 2;
  b.safety_factor = 0.5f;
  b.sleep_threshold = 0.05f;
  BodySim s;
  std::memset(&s, 0, sizeof(s));
  s.transform.p.x = d->position[0]; s.transform.p.y = d->position[1]; s.transform.p.z = d->position[2];
  s.transform.q = quat(v3(d->rotation[0], d->rotation[1], d->rotation[2]), d->rotation[3]);
  s.center = s.transform.p;
  s.rotation0 = s.transform.q;
  s.center0 = s.center;
  s.min_extent = huge_value();
  s.linear_damping = d->linear_damping;
  s.angular_damping = d->angular_damping;
  s.gravity_scale = d->gravity_scale;
  s.body_id = id;
  s.inertia = m3zero(); s.inv_inertia_local = m3zero(); s.inv_inertia_world = m3zero();
  s.flags = 0;
  if (d->type == 2) s.flags |= kDynamicFlag;
  if (d->enable_sleep) s.flags |= kEnableSleepFlag;
  if (d->is_bullet) s.flags |= kIsBullet;  // world_runtime.rs:1570
  s.flags |= kEnableRecycling;
  if (b.set_index == 2) {
    b.local_index = (int)w->awake_sims.size();
    w->awake_sims.push_back(s);
    BodyState st;
    st.v = v3(d->linear_velocity[0], d->linear_velocity[1], d->linear_velocity[2]);
    st.w = v3(d->angular_velocity[0], d->angular_velocity[1], d->angular_velocity[2]);
    st.dp = v3(0, 0, 0);
    st.dq = qid();
    st.flags = s.flags;
    w->awake_states.push_back(st);
  } else {
    b.local_index = (int)w->static_sims.size();
    w->static_sims.push_back(s);
  }
  b.flags = s.flags;
  w->bodies.push_back(b);
  return id;
}

int nso_create_box(nso_world* w, int body, const nso_shape_def* def, float hx, float hy, float hz) {
  Shape s;
  s.type = kHull;
  s.hull = make_box_hull(hx, hy, hz);
  return create_shape(w, body, def, s);
}

int nso_create_sphere(nso_world* w, int body, const nso_shape_def* def, const float c[3], float r) {
  Shape s;
  s.type = kSphere;
  s.sphere.center = v3(c[0], c[1], c[2]);
  s.sphere.radius = r;
  return create_shape(w, body, def, s);
}

int nso_create_capsule(nso_world* w, int body, const nso_shape_def* def, const float c1[3],
                       const float c2[3], float r) {
  Shape s;
  V3 a = v3(c1[0], c1[1], c1[2]), b = v3(c2[0], c2[1], c2[2]);
  if (distance(a, b) < min_capsule_length()) {  // shape_creation.rs:522
    s.type = kSphere;
    s.sphere.center = 0.5f * (a + b);
    s.sphere.radius = r;
  } else {
    s.type = kCapsule;
    s.capsule.c1 = a; s.capsule.c2 = b; s.capsule.radius = r;
  }
  return create_shape(w, body, def, s);
}

static int add_revolute(nso_world* w, Joint j);

int nso_create_revolute(nso_world* w, int body_a, int body_b, const float fa[7], const float fb[7],
                        int enable_limit, float lower, float upper, int enable_spring, float hertz,
                        float damping_ratio, float drag_torque, int collide_connected) {
  Joint j = make_revolute_joint(body_a, body_b, fa, fb, enable_limit != 0, lower, upper,
                                enable_spring != 0, hertz, damping_ratio, drag_torque,
                                collide_connected != 0, w->def.joint_hertz, w->def.joint_damping_ratio);
  return add_revolute(w, j);
}

// revolute_joint.rs:161-181 create_revolute_joint: every RevoluteJointDef field is copied
int nso_create_revolute_def(nso_world* w, const nso_revolute_def* d) {
  Joint j = make_revolute_joint(d->body_a, d->body_b, d->local_frame_a, d->local_frame_b, d->enable_limit != 0,
                                d->lower_angle, d->upper_angle, d->enable_spring != 0, d->hertz, d->damping_ratio,
                                d->max_motor_torque, d->collide_connected != 0, d->constraint_hertz,
                                d->constraint_damping_ratio);
  j.enable_motor = d->enable_motor != 0;
  j.motor_speed = d->motor_speed;
  j.target_angle = d->target_angle;
  return add_revolute(w, j);
}

int nso_create_spherical_def(nso_world* w, const nso_spherical_def* d) {
  const float* t = d->target_rotation;
  Joint j = make_spherical_joint(d->body_a, d->body_b, d->local_frame_a, d->local_frame_b, d->collide_connected != 0,
                                 d->constraint_hertz, d->constraint_damping_ratio, d->enable_spring != 0, d->hertz,
                                 d->damping_ratio, quat(v3(t[0], t[1], t[2]), t[3]), d->enable_cone_limit != 0,
                                 d->cone_angle, d->enable_twist_limit != 0, d->lower_twist_angle,
                                 d->upper_twist_angle, d->enable_motor != 0, d->max_motor_torque,
                                 v3(d->motor_velocity[0], d->motor_velocity[1], d->motor_velocity[2]));
  return add_revolute(w, j);
}

static int add_revolute(nso_world* w, Joint j) {
  int body_a = j.body_a, body_b = j.body_b;
  int id = (int)w->joints.size();
  j.id = id;
  // joint.rs:164 create_joint: awake joints go to the graph; bodies' joint counts grow.
  Body& ba = w->bodies[body_a];
  Body& bb = w->bodies[body_b];
  ba.joint_count++;
  bb.joint_count++;
  if ((int)w->body_joints.size() < (int)w->bodies.size()) w->body_joints.resize(w->bodies.size());
  w->body_joints[body_a].push_back((int)w->joints.size());
  w->body_joints[body_b].push_back((int)w->joints.size());
  int color = kOverflowIndex;
  if (ba.type == 2 && bb.type == 2) {
    for (int i = 0; i < kDynamicColorCount; ++i) {
      if (get_bit(w, i, body_a) || get_bit(w, i, body_b)) continue;
      set_bit(w, i, body_a); set_bit(w, i, body_b);
      color = i;
      break;
    }
  } else if (ba.type == 2) {
    for (int i = kOverflowIndex - 1; i >= 1; --i)
      if (!get_bit(w, i, body_a)) { set_bit(w, i, body_a); color = i; break; }
  } else if (bb.type == 2) {
    for (int i = kOverflowIndex - 1; i >= 1; --i)
      if (!get_bit(w, i, body_b)) { set_bit(w, i, body_b); color = i; break; }
  }
  // joint.rs:251-262: a joint not attached to a dynamic body stays in the static set, unsolved
  if (ba.type != 2 && bb.type != 2) color = -1;
  j.color = color;
  if (color >= 0) w->colors[color].joints.push_back(id);
  w->joints.push_back(j);
  return id;
}

// solver_integration.rs:807 World::step
void nso_step(nso_world* w, float dt, int substeps) {
  update_pairs(w);
  StepContext& c = w->ctx;
  c.dt = dt;
  c.sub_step_count = substeps < 1 ? 1 : substeps;
  if (dt > 0.0f) {
    c.inv_dt = 1.0f / dt;
    c.h = dt / (real)c.sub_step_count;
    c.inv_h = (real)c.sub_step_count * c.inv_dt;
  } else {
    c.inv_dt = 0.0f; c.h = 0.0f; c.inv_h = 0.0f;
  }
  real hz = minf(w->def.contact_hertz, 0.125f * c.inv_h);
  c.contact_softness = make_soft(hz, w->def.contact_damping_ratio, c.h);
  c.static_softness = make_soft(2.0f * hz, 0.5f * w->def.contact_damping_ratio, c.h);
  c.enable_warm_starting = w->def.enable_warm_starting != 0;
  if (dt > 0.0f) collide(w);
  if (dt <= 0.0f) return;
  if (w->awake_sims.empty()) return;
  prepare_all(w);
  solve_stages(w);
  finalize(w);
}

// body_queries.rs:432 world_state_hash
uint64_t nso_state_hash(const nso_world* w) {
  const uint64_t prime = 1099511628211ull;
  uint64_t h = 14695981039346656037ull;
  auto mixf = [&](float f) { uint32_t b; std::memcpy(&b, &f, 4); h = (h ^ (uint64_t)b) * prime; };
  auto mixd = [&](double d) { uint64_t b; std::memcpy(&b, &d, 8); h = (h ^ b) * prime; };
  for (const Body& b : w->bodies) {
    const BodySim& s = b.set_index == 2 ? w->awake_sims[b.local_index] : w->static_sims[b.local_index];
    mixd(s.transform.p.x); mixd(s.transform.p.y); mixd(s.transform.p.z);
    mixf(s.transform.q.v.x); mixf(s.transform.q.v.y); mixf(s.transform.q.v.z); mixf(s.transform.q.s);
    if (b.set_index == 2) {
      const BodyState& st = w->awake_states[b.local_index];
      mixf(st.v.x); mixf(st.v.y); mixf(st.v.z);
      mixf(st.w.x); mixf(st.w.y); mixf(st.w.z);
    }
  }
  return h;
}

int nso_body_count(const nso_world* w) { return (int)w->bodies.size(); }

int nso_get_bodies(const nso_world* w, double* pos, float* rot, float* lin, float* ang) {
  int n = (int)w->bodies.size();
  for (int i = 0; i < n; ++i) {
    const Body& b = w->bodies[i];
    const BodySim& s = b.set_index == 2 ? w->awake_sims[b.local_index] : w->static_sims[b.local_index];
    pos[3 * i] = s.transform.p.x; pos[3 * i + 1] = s.transform.p.y; pos[3 * i + 2] = s.transform.p.z;
    rot[4 * i] = s.transform.q.v.x; rot[4 * i + 1] = s.transform.q.v.y;
    rot[4 * i + 2] = s.transform.q.v.z; rot[4 * i + 3] = s.transform.q.s;
    V3 v = v3(0, 0, 0), wv = v3(0, 0, 0);
    if (b.set_index == 2) { v = w->awake_states[b.local_index].v; wv = w->awake_states[b.local_index].w; }
    lin[3 * i] = v.x; lin[3 * i + 1] = v.y; lin[3 * i + 2] = v.z;
    ang[3 * i] = wv.x; ang[3 * i + 1] = wv.y; ang[3 * i + 2] = wv.z;
  }
  return n;
}

int nso_contact_capacity(const nso_world* w) { return (int)w->contacts.size(); }

int nso_get_contacts(const nso_world* w, int32_t* ints, uint32_t* feats, float* fl) {
  int n = 0;
  for (size_t i = 0; i < w->contacts.size(); ++i) {
    const Contact& c = w->contacts[i];
    if (c.contact_id == -1) continue;
    int32_t* I = ints + 8 * n;
    uint32_t* F = feats + 4 * n;
    float* D = fl + 24 * n;
    int pc = c.manifold_count > 0 ? c.manifold.point_count : 0;
    I[0] = (int32_t)i; I[1] = c.shape_a; I[2] = c.shape_b; I[3] = c.color_index; I[4] = pc;
    I[5] = (int32_t)c.flags; I[6] = c.sat.type; I[7] = c.manifold_count;
    for (int k = 0; k < 4; ++k) F[k] = k < pc ? c.manifold.points[k].feature_id : 0u;
    for (int k = 0; k < 24; ++k) D[k] = 0.0f;
    if (pc > 0) {
      D[0] = c.manifold.normal.x; D[1] = c.manifold.normal.y; D[2] = c.manifold.normal.z;
      for (int k = 0; k < pc; ++k) {
        D[3 + 5 * k] = c.manifold.points[k].anchor_a.x;
        D[4 + 5 * k] = c.manifold.points[k].anchor_a.y;
        D[5 + 5 * k] = c.manifold.points[k].anchor_a.z;
        D[6 + 5 * k] = c.manifold.points[k].separation;
        D[7 + 5 * k] = c.manifold.points[k].normal_impulse;
      }
    }
    n++;
  }
  return n;
}

void nso_counters(const nso_world* w, int32_t* out) {
  for (int i = 0; i < 32; ++i) out[i] = 0;
  for (const Contact& c : w->contacts) {
    if (c.contact_id == -1) continue;
    out[0]++;
    if (c.flags & cTouching) out[1]++;
  }
  for (int ci = 0; ci < kGraphColorCount; ++ci)
    out[2 + ci] = (int)(w->colors[ci].convex.size() + w->colors[ci].overflow.size());
  out[26] = w->fast_flags_seen;
  out[27] = w->sat_calls;
  out[28] = w->recycled;
}

// body_api.rs:351 apply_body_force_to_center and :366 apply_body_torque, every body in id order
void nso_apply_forces(nso_world* w, const float* force, const float* torque) {
  for (size_t i = 0; i < w->bodies.size(); ++i) {
    const Body& b = w->bodies[i];
    if (b.set_index != 2) continue;
    BodySim& s = w->awake_sims[b.local_index];
    if (force) s.force = s.force + v3(force[3 * i], force[3 * i + 1], force[3 * i + 2]);
    if (torque) s.torque = s.torque + v3(torque[3 * i], torque[3 * i + 1], torque[3 * i + 2]);
  }
}

void nso_time_of_impact(const float* pa, int na, float ra, const float* pb, int nb, float rb, const float* sa,
                        const float* sb, float max_fraction, float* out) {
  Proxy a, b;
  a.count = na < 1 ? 1 : (na > 8 ? 8 : na);
  b.count = nb < 1 ? 1 : (nb > 8 ? 8 : nb);
  for (int i = 0; i < a.count; ++i) a.pts[i] = v3(pa[3 * i], pa[3 * i + 1], pa[3 * i + 2]);
  for (int i = 0; i < b.count; ++i) b.pts[i] = v3(pb[3 * i], pb[3 * i + 1], pb[3 * i + 2]);
  a.radius = ra;
  b.radius = rb;
  auto sweep = [](const float* f) {
    Sweep s;
    s.local_center = v3(f[0], f[1], f[2]);
    s.c1 = v3(f[3], f[4], f[5]);
    s.c2 = v3(f[6], f[7], f[8]);
    s.q1 = quat(v3(f[9], f[10], f[11]), f[12]);
    s.q2 = quat(v3(f[13], f[14], f[15]), f[16]);
    return s;
  };
  ToiOut o = time_of_impact(a, b, sweep(sa), sweep(sb), max_fraction);
  float r[13] = {(float)o.state, (float)o.fraction, (float)o.distance, (float)o.point.x, (float)o.point.y,
                 (float)o.point.z, (float)o.normal.x, (float)o.normal.y, (float)o.normal.z,
                 (float)o.distance_iterations, (float)o.push_back_iterations, (float)o.root_iterations, 0.0f};
  for (int i = 0; i < 13; ++i) out[i] = r[i];
}

void nso_collide_pairs(nso_pair_job* jobs, nso_pair_result* results, int count) {
  for (int i = 0; i < count; ++i) {
    nso_pair_job& j = jobs[i];
    nso_pair_result& r = results[i];
    std::memset(&r, 0, sizeof(r));
    Xf x = xf(v3(j.xf[0], j.xf[1], j.xf[2]), quat(v3(j.xf[3], j.xf[4], j.xf[5]), j.xf[6]));
    LocalManifold lm;
    auto sphere = [](const float* g) { Sphere s; s.center = v3(g[0], g[1], g[2]); s.radius = g[3]; return s; };
    auto capsule = [](const float* g) { Capsule c; c.c1 = v3(g[0], g[1], g[2]); c.c2 = v3(g[3], g[4], g[5]); c.radius = g[6]; return c; };
    SATCache sat;
    sat.separation = j.sat_separation; sat.type = (uint8_t)j.sat_type;
    sat.index_a = (uint8_t)j.sat_index_a; sat.index_b = (uint8_t)j.sat_index_b; sat.hit = (uint8_t)j.sat_hit;
    SimplexCache sc;
    sc.metric = j.simplex_metric; sc.count = (uint16_t)j.simplex_count;
    for (int k = 0; k < 4; ++k) { sc.ia[k] = (uint8_t)j.simplex_ia[k]; sc.ib[k] = (uint8_t)j.simplex_ib[k]; }
    if (j.type_a == kSphere) {
      collide_spheres(&lm, sphere(j.geom_a), sphere(j.geom_b), x);
    } else if (j.type_a == kCapsule) {
      if (j.type_b == kSphere) collide_capsule_sphere(&lm, capsule(j.geom_a), sphere(j.geom_b), x);
      else collide_capsules(&lm, capsule(j.geom_a), capsule(j.geom_b), x);
    } else {
      Hull ha = make_box_hull(j.geom_a[0], j.geom_a[1], j.geom_a[2]);
      if (j.type_b == kSphere) collide_hull_sphere(&lm, ha, sphere(j.geom_b), x, &sc);
      else if (j.type_b == kCapsule) collide_hull_capsule(&lm, ha, capsule(j.geom_b), x, &sc);
      else {
        Hull hb = make_box_hull(j.geom_b[0], j.geom_b[1], j.geom_b[2]);
        collide_hulls(&lm, ha, hb, x, &sat, nullptr);
      }
    }
    j.sat_separation = sat.separation; j.sat_type = sat.type; j.sat_index_a = sat.index_a;
    j.sat_index_b = sat.index_b; j.sat_hit = sat.hit;
    j.simplex_metric = sc.metric; j.simplex_count = sc.count;
    for (int k = 0; k < 4; ++k) { j.simplex_ia[k] = sc.ia[k]; j.simplex_ib[k] = sc.ib[k]; }
    r.normal[0] = lm.normal.x; r.normal[1] = lm.normal.y; r.normal[2] = lm.normal.z;
    r.point_count = lm.point_count;
    for (int k = 0; k < lm.point_count; ++k) {
      r.points[k][0] = lm.points[k].point.x; r.points[k][1] = lm.points[k].point.y;
      r.points[k][2] = lm.points[k].point.z; r.points[k][3] = lm.points[k].separation;
      r.feature_ids[k] = make_feature_id(lm.points[k].pair);
    }
  }
}

}  // extern "C"
