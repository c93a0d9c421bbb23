// libnatsel_gpu: host side of the B200 step behind the C ABI in include/natsel_gpu.h.
//
// Scene construction mirrors the reference World API (world_runtime.rs:1506 create_body,
// shape_creation.rs:287 create_shape_internal, body_api.rs:642 update_body_mass_data,
// joint.rs:164 create_joint) so ids, mass properties and initial graph colors match.
// The first step uploads the scene; every step after that is one CUDA graph launch
// with no host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/natsel_gpu.h"
#include "nsd_solve.cuh"
#include "nsd_adjoint.cuh"
#include "nsd_adjoint_host.h"

using namespace nsd;

namespace {

thread_local std::string g_create_error;

struct HostBody {
  int type = 0, set = 0, local = 0;
  int world = 0;            // sub-world
  uint32_t flags = 0;
  int joint_count = 0;
  float mass = 0;
  std::vector<int> shapes;  // creation order
};

struct HostShape {
  DShape d;
  Hull hull;
  float density = 0;
  float bound_radius = 0;  // radius about the shape's origin holding its local box in any rotation
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
};

}  // namespace

struct ns_world {
  ns_world_def def;
  std::string err;
  std::vector<HostBody> bodies;
  std::vector<DSim> asims, ssims;
  std::vector<DState> states;
  std::vector<HostShape> shapes;
  std::vector<AABB> fat;
  std::vector<AABB> saabb;  // each shape's bounds at creation (shape.aabb; continuous pass input)
  std::vector<DJoint> joints;
  std::vector<uint32_t> body_mask;
  std::vector<std::vector<int>> joint_partners;  // per body: bodies a joint keeps from colliding

  bool uploaded = false;
  int device = 0, sm_count = 0;
  cudaStream_t stream = nullptr;
  DW dw;
  JointRanges jr;
  std::vector<void*> allocations;
  std::vector<size_t> allocation_bytes;
  struct AdTape* tape = nullptr;   // rollout record for the adjoint (ns_world_tape_begin)
  std::vector<float> vjp_restitution;  // the last f32 VJP's restitution cotangents, body id order
  int n_bullets = 0;                   // dynamic bodies created as bullets
  // Device buffers kept for reuse by later tapes and VJPs and freed with the world: checkpoint
  // buffers (with their copy tables, valid for the world's allocation set, which is fixed once
  // uploaded), the VJP's step tapes and its cotangent buffers.
  std::vector<char*> ckpt_pool;
  char* tapes_buf = nullptr; size_t tapes_cap = 0;
  char* adj_buf = nullptr; size_t adj_cap = 0;
  // Snapshot layout of the allocations (device table, written once) and its total size.
  SnapOp* snap_ops = nullptr; size_t snap_bytes = 0;
  void* cub_sort_tmp = nullptr;
  size_t cub_sort_bytes = 0;
  void* cub_scan_tmp = nullptr;
  size_t cub_scan_bytes = 0;
  int solver_blocks = 1;           // blocks of the solver launch
  bool solver_grid = true;         // cooperative grid (true) or one thread-block cluster
  // launch shapes of the grid-stride step kernels (threads per block, blocks per SM at most),
  // chosen by ns_world_autotune; every shape gives the same bits
  int recycle_threads = kCollideThreads, recycle_per_sm = 16;       // k_collide
  int update_threads = kCollideUpdateThreads, update_per_sm = 32;   // k_collide_update
  int prepare_threads = kPrepareThreads, prepare_per_sm = 16;       // k_prepare_slots
  std::vector<std::array<float, 4>> tune_rows;  // last autotune: dimension, a, b, ms per step
  int sort_bits = 32;              // key bits of the broadphase sort (bucket index + large flag)
  int state_mode = 0;
  size_t state_smem = 0;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  float graph_dt = -1.0f;
  int graph_substeps = -1;
  cudaEvent_t ev[6] = {};
  int steps_done = 0;
  int last_substeps = 0;
  bool eager = false;
  // readback: body id -> awake index (>= 0) or -(static index + 1); packed output staging
  int* body_loc = nullptr;
  char* out_stage = nullptr;
  Control* host_ctl = nullptr;  // pinned
  // per-step external forces: pinned host staging -> device staging (force xyz | torque xyz)
  float* host_in = nullptr;     // pinned, 6 floats per body
  float* in_stage = nullptr;
  cudaEvent_t in_done = nullptr;
  // accounting
  int pair_kernels = 0, step_kernels = 0;  // own kernel launches per pair update / full step
  int64_t kernel_launches = 0;
  int64_t n_gyroscopic = 0;
  // sub-worlds: the first body and shape of each (bodies, shapes and joints are added to the
  // newest sub-world only, so each sub-world's ids are contiguous)
  std::vector<int> sub_body_begin = {0}, sub_shape_begin = {0};
};

namespace {

int fail(ns_world* w, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (w) w->err = buf; else g_create_error = buf;
  return code;
}

#define NS_CUDA(w, call)                                                                   \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail((w), NS_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));       \
  } while (0)

DSim& sim_ref(ns_world* w, const HostBody& b) { return b.set == 2 ? w->asims[b.local] : w->ssims[b.local]; }

int encode(const HostBody& b) { return b.set == 2 ? b.local : -(b.local + 2); }

// world_runtime.rs:1479 sync_body_flags
void sync_flags(ns_world* w, int bi) {
  HostBody& b = w->bodies[bi];
  DSim& s = sim_ref(w, b);
  s.flags = (s.flags & (kIsFast | kHadToi)) | (b.flags & ~kTransient);
  if (b.set == 2) w->states[b.local].flags = b.flags & ~kTransient;
}

struct MassData { float mass; V3 center; M3 inertia; };

MassData shape_mass(const HostShape& hs) {
  const DShape& s = hs.d;
  MassData md;
  if (s.type == kHull) {  // shape_runtime.rs:312 compute_hull_mass
    md.mass = hs.density * hs.hull.volume;
    md.center = hs.hull.center;
    md.inertia = mul_sm(hs.density, hs.hull.central_inertia);
  } else if (s.type == kSphere) {  // sphere.rs:13 compute_sphere_mass
    float r = s.sphere.radius;
    float volume = 4.0f / 3.0f * kPi * r * r * r;
    float mass = volume * hs.density;
    float ixx = 0.4f * mass * r * r;
    md.mass = mass;
    md.center = s.sphere.center;
    md.inertia = diag(ixx, ixx, ixx);
  } else {  // capsule.rs:27 compute_capsule_mass
    V3 c1 = s.capsule.c1, c2 = s.capsule.c2;
    float r = s.capsule.radius;
    float h = distance(c1, c2);
    float cyl_mass = kPi * r * r * h * hs.density;
    float sph_mass = (4.0f / 3.0f) * kPi * r * r * r * hs.density;
    // geometry_queries.rs cylinder_inertia / sphere_inertia
    float lateral = cyl_mass * (3.0f * r * r + h * h) / 12.0f;
    float axial = 0.5f * cyl_mass * r * r;
    M3 inertia = add_mm(diag(lateral, axial, lateral),
                        diag(0.4f * sph_mass * r * r, 0.4f * sph_mass * r * r, 0.4f * sph_mass * r * r));
    float st = 0.125f * sph_mass * (3.0f * r + 2.0f * h) * h;
    inertia.cx.x += st;
    inertia.cz.z += st;
    M3 rot = identity_m3();
    if (h * h > 1000.0f * kMinPositive) rot = matrix_from_quat(quat_between_unit_vectors(v3(0, 1, 0), normalize(c2 - c1)));
    md.mass = sph_mass + cyl_mass;
    md.center = 0.5f * (c1 + c2);
    md.inertia = mul_mm(rot, mul_mm(inertia, transpose(rot)));
  }
  return md;
}

void shape_extent(const HostShape& hs, V3 lc, float* min_e, V3* max_e) {  // shape_runtime.rs:499
  const DShape& s = hs.d;
  if (s.type == kCapsule) {
    float r = s.capsule.radius;
    *min_e = r;
    *max_e = max3(abs3(s.capsule.c1 - lc), abs3(s.capsule.c2 - lc)) + v3(r, r, r);
  } else if (s.type == kSphere) {
    float r = s.sphere.radius;
    *min_e = r;
    *max_e = abs3(s.sphere.center - lc) + v3(r, r, r);
  } else {  // hull_queries.rs:101
    *min_e = hs.hull.inner_radius;
    V3 m = v3(0, 0, 0);
    for (int i = 0; i < kHullVertexCount; ++i) m = max3(m, abs3(hs.hull.points[i] - lc));
    *max_e = m;
  }
}

// body_api.rs:642 update_body_mass_data (+ :611 update_isotropic_inertia)
void update_mass(ns_world* w, int bi) {
  HostBody& b = w->bodies[bi];
  b.flags &= ~kDirtyMass;
  b.flags &= ~kGyroscopic;
  sync_flags(w, bi);
  b.mass = 0.0f;
  DSim& s = sim_ref(w, b);
  s.inertia = m3zero(); s.inv_mass = 0.0f;
  s.inv_inertia_local = m3zero(); s.inv_inertia_world = m3zero();
  s.local_center = v3(0, 0, 0);
  s.min_extent = huge_value();
  s.max_extent = v3(0, 0, 0);
  if (b.shapes.empty()) return;
  if (b.type != NS_DYNAMIC_BODY) {
    // body_api.rs:670-689: static and kinematic sims have zero mass; a kinematic body keeps its
    // shapes' extents about its origin (contact recycling reads them)
    s.cx = s.px; s.cy = s.py; s.cz = s.pz;
    if (b.type == NS_KINEMATIC_BODY)
      for (int sid : b.shapes) {
        float mn;
        V3 mx;
        shape_extent(w->shapes[sid], v3(0, 0, 0), &mn, &mx);
        s.min_extent = minf(s.min_extent, mn);
        s.max_extent = max3(s.max_extent, mx);
      }
    return;
  }
  std::vector<MassData> masses;
  V3 lc = v3(0, 0, 0);
  for (auto it = b.shapes.rbegin(); it != b.shapes.rend(); ++it) {  // head of list = newest
    const HostShape& hs = w->shapes[*it];
    if (hs.density == 0.0f) { MassData z = {0, v3(0, 0, 0), m3zero()}; masses.push_back(z); continue; }
    MassData md = shape_mass(hs);
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
    s.inertia = add_mm(s.inertia, add_mm(md.inertia, steiner(md.mass, lc - md.center)));
  }
  Q q = s.q;
  if (det(s.inertia) > 0.0f) {
    s.inv_inertia_local = invert_t(s.inertia);
    M3 R = matrix_from_quat(q);
    s.inv_inertia_world = mul_mm(mul_mm(R, s.inv_inertia_local), transpose(R));
  }
  Pos old_center = {s.cx, s.cy, s.cz};
  s.local_center = lc;
  WXf t;
  t.p.x = s.px; t.p.y = s.py; t.p.z = s.pz; t.q = q;
  Pos c = world_point(t, lc);
  s.cx = c.x; s.cy = c.y; s.cz = c.z;
  DState& st = w->states[b.local];
  st.v = st.v + cross(st.w, sub_pos(c, old_center));
  for (auto it = b.shapes.rbegin(); it != b.shapes.rend(); ++it) {
    float mn; V3 mx;
    shape_extent(w->shapes[*it], lc, &mn, &mx);
    s.min_extent = minf(s.min_extent, mn);
    s.max_extent = max3(s.max_extent, mx);
  }
  if ((s.flags & (kLockAngX | kLockAngY | kLockAngZ)) == (kLockAngX | kLockAngY | kLockAngZ)) {
    s.inertia = m3zero(); s.inv_inertia_local = m3zero(); s.inv_inertia_world = m3zero();
  }
  // body_api.rs:611 update_isotropic_inertia (tolerance 0.2, world_runtime.rs:1256)
  M3 I = s.inertia;
  float mean = (I.cx.x + I.cy.y + I.cz.z) / 3.0f;
  float dx = I.cx.x - mean, dy = I.cy.y - mean, dz = I.cz.z - mean;
  float off = I.cy.x * I.cy.x + I.cz.x * I.cz.x + I.cz.y * I.cz.y;
  float dev = dx * dx + dy * dy + dz * dz + 2.0f * off;
  float tol = 0.2f;
  if (2.0f * dev > 3.0f * tol * tol * mean * mean) b.flags |= kGyroscopic;
  else b.flags &= ~kGyroscopic;
  sync_flags(w, bi);
}

AABB shape_local_aabb(const HostShape& hs, Q q) {  // shape_runtime.rs:405
  Xf t = xf(v3(0, 0, 0), q);
  const DShape& s = hs.d;
  if (s.type == kHull) return aabb_transform(t, hs.hull.bounds);
  if (s.type == kSphere) {
    V3 c = xf_point(t, s.sphere.center);
    float r = s.sphere.radius;
    return aabb(c - v3(r, r, r), c + v3(r, r, r));
  }
  V3 c1 = xf_point(t, s.capsule.c1), c2 = xf_point(t, s.capsule.c2);
  float r = s.capsule.radius;
  return aabb(min3(c1, c2) - v3(r, r, r), max3(c1, c2) + v3(r, r, r));
}

int create_shape(ns_world* w, int bi, const ns_shape_def* def, HostShape hs) {
  if (w->uploaded) return fail(w, -1, "scene changes after the first step are not supported"), -1;
  if (bi < 0 || bi >= (int)w->bodies.size() || !def) return fail(w, -1, "invalid body or shape def"), -1;
  // pair keys hold two 22-bit shape ids
  if (w->shapes.size() >= (1u << 22) - 1) return fail(w, -1, "at most 4194303 shapes per world"), -1;
  int sid = (int)w->shapes.size();
  HostBody& b = w->bodies[bi];
  if (b.world != (int)w->sub_body_begin.size() - 1)
    return fail(w, -1, "shapes can only be added to bodies of the newest sub-world"), -1;
  DShape& s = hs.d;
  s.body = bi;
  s.world = b.world;
  s.enc = encode(b);
  s.is_static = b.type == NS_STATIC_BODY;
  hs.density = def->density;
  s.friction = def->friction;
  s.restitution = def->restitution;
  s.rolling = def->rolling_resistance;
  s.category = def->category_bits;
  s.mask = def->mask_bits;
  s.group = def->group_index;
  // shape_creation.rs:199 compute_shape_margin
  float margin;
  if (s.type == kSphere) margin = s.sphere.radius;
  else if (s.type == kCapsule) margin = 0.5f * distance(s.capsule.c2, s.capsule.c1) + s.capsule.radius;
  else {
    float mx = 0.0f;
    for (int i = 0; i < kHullVertexCount; ++i) mx = maxf(mx, distance_sq(hs.hull.points[i], hs.hull.center));
    margin = sqrtf(mx);
  }
  s.aabb_margin = minf(max_aabb_margin(), kAabbMarginFraction * margin);
  if (s.type == kHull) {
    // the tight box rotates the hull's local bounds about the shape origin
    V3 lo = hs.hull.bounds.lo, hi = hs.hull.bounds.hi;
    V3 far_corner = v3(maxf(absf(lo.x), absf(hi.x)), maxf(absf(lo.y), absf(hi.y)), maxf(absf(lo.z), absf(hi.z)));
    hs.bound_radius = length(far_corner);
  } else {
    hs.bound_radius = margin;
  }
  // shape_creation.rs:236 update_shape_aabbs
  const DSim& sim = sim_ref(w, b);
  float spec = speculative_distance();
  Pos p = {sim.px, sim.py, sim.pz};
  AABB a = offset_aabb(aabb_inflate(shape_local_aabb(hs, sim.q), spec), p);
  w->fat.push_back(aabb_inflate(a, s.is_static ? spec : s.aabb_margin));
  w->saabb.push_back(a);
  s.hull = s.type == kHull ? sid : -1;
  w->shapes.push_back(hs);
  b.shapes.push_back(sid);
  update_mass(w, bi);
  return sid;
}

template <class T>
T* dalloc(ns_world* w, size_t n, int* status) {
  void* p = nullptr;
  size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    *status = fail(w, NS_ERR_CUDA, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    return nullptr;
  }
  cudaMemsetAsync(p, 0, bytes, w->stream);
  w->allocations.push_back(p);
  w->allocation_bytes.push_back(bytes);
  return (T*)p;
}

template <class T>
int upload(ns_world* w, T* dst, const std::vector<T>& src) {
  if (src.empty()) return NS_OK;
  NS_CUDA(w, cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, w->stream));
  return NS_OK;
}

// The narrowphase keeps the reference's 64-vertex clip buffers on the thread stack (about
// 2.5 KB). The default per-thread stack limit is 1 KB, so the limit is raised to the largest
// local-memory size of the step kernels before anything runs.
int ensure_stack(ns_world* w) {
  size_t need = 0;
  cudaFuncAttributes a;
  const void* kernels[] = {(const void*)k_collide, (const void*)k_collide_update, (const void*)k_collide_jobs,
                           (const void*)k_solve<true, false>,
                           (const void*)k_solve<false, false>,
                           (const void*)k_solve<true, true>,
                           (const void*)k_solve<false, true>,
                           (const void*)k_prepare_overflow, (const void*)k_color_scatter, (const void*)k_prepare_slots,
                           (const void*)k_warm_slots,
                           (const void*)k_finalize, (const void*)k_continuous, (const void*)k_bullets, (const void*)k_state_pass,
                           (const void*)k_adj_solve<true, false>, (const void*)k_adj_solve<false, false>,
                           (const void*)k_adj_solve<true, true>, (const void*)k_adj_solve<false, true>,
                           (const void*)k_adj_narrow, (const void*)k_adj_prepare, (const void*)k_adj_consts,
                           (const void*)k_adj_restitution, (const void*)k_adj_joint_prepare};
  for (const void* k : kernels) {
    cudaError_t e = cudaFuncGetAttributes(&a, k);
    if (e != cudaSuccess) return fail(w, NS_ERR_CUDA, "cudaFuncGetAttributes: %s", cudaGetErrorString(e));
    if (a.localSizeBytes > need) need = a.localSizeBytes;
  }
  need = ((need + 1023) / 1024) * 1024 + 1024;
  size_t cur = 0;
  cudaDeviceGetLimit(&cur, cudaLimitStackSize);
  if (cur < need) {
    cudaError_t e = cudaDeviceSetLimit(cudaLimitStackSize, need);
    if (e != cudaSuccess) return fail(w, NS_ERR_CUDA, "cudaDeviceSetLimit(stack %zu): %s", need, cudaGetErrorString(e));
  }
  return NS_OK;
}

int upload_world(ns_world* w) {
  if (w->def.enable_sleep) return fail(w, NS_ERR_UNSUPPORTED, "sleeping islands are not supported");
  NS_CUDA(w, cudaSetDevice(w->def.device));
  {
    int st0 = ensure_stack(w);
    if (st0) return st0;
  }
  NS_CUDA(w, cudaDeviceGetAttribute(&w->sm_count, cudaDevAttrMultiProcessorCount, w->def.device));
  NS_CUDA(w, cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
  for (int i = 0; i < 6; ++i) NS_CUDA(w, cudaEventCreate(&w->ev[i]));
  int st = NS_OK;
  DW& d = w->dw;
  memset(&d, 0, sizeof(d));
  int na = (int)w->asims.size(), ns = (int)w->ssims.size(), nsh = (int)w->shapes.size();
  int nb = (int)w->bodies.size(), nj = (int)w->joints.size();
  d.n_awake = na; d.n_static = ns; d.n_shapes = nsh; d.n_bodies = nb; d.n_joints = nj;
  // contact id ranges: one world keeps the reference-sized capacity; each sub-world of a batch
  // gets 12 contacts per shape + 64 (or contact_capacity), a multiple of 32 so its changed
  // bits fill whole words; the last range is padded to a multiple of 1024
  int n_worlds = (int)w->sub_body_begin.size();
  std::vector<int> world_shape(w->sub_shape_begin), world_cbase(n_worlds + 1, 0);
  world_shape.push_back(nsh);
  int cap;
  if (n_worlds == 1) {
    cap = w->def.contact_capacity > 0 ? w->def.contact_capacity : 8 * nsh + 4096;
    cap = (cap + 1023) & ~1023;
  } else {
    for (int k = 0; k < n_worlds; ++k) {
      int ns_k = world_shape[k + 1] - world_shape[k];
      int c = w->def.contact_capacity > 0 ? w->def.contact_capacity : 12 * ns_k + 64;
      world_cbase[k + 1] = world_cbase[k] + ((c + 31) & ~31);
    }
    cap = (world_cbase[n_worlds] + 1023) & ~1023;
  }
  world_cbase[n_worlds] = cap;
  d.cap = cap;
  d.n_worlds = n_worlds;
  int hs_size = 1;
  while (hs_size < 4 * cap) hs_size <<= 1;
  d.hs_mask = hs_size - 1;
  d.n_words = (cap + 31) / 32;
  d.cand_cap = cap;
  d.n_color_blocks = cap / kColorBlock;

  // body -> shape table for finalize (awake bodies)
  std::vector<int> body_shapes;
  for (int i = 0; i < nb; ++i) {
    HostBody& b = w->bodies[i];
    if (b.set != 2) continue;
    DSim& s = w->asims[b.local];
    s.shape_begin = (int)body_shapes.size();
    for (auto it = b.shapes.rbegin(); it != b.shapes.rend(); ++it) body_shapes.push_back(*it);
    s.shape_end = (int)body_shapes.size();
  }
  std::vector<DShape> dshapes(nsh);
  std::vector<Hull> hulls(nsh);
  std::vector<int> large;
  for (int i = 0; i < nsh; ++i) {
    dshapes[i] = w->shapes[i].d;
    hulls[i] = w->shapes[i].hull;
    if (dshapes[i].is_static && (w->fat[i].hi.x - w->fat[i].lo.x) > 8.0f) large.push_back(i);
  }
  d.n_large = (int)large.size();
  d.n_small = nsh - d.n_large;
  // static shapes per sub-world, for the continuous pass
  std::vector<int> static_list, static_off(n_worlds + 1, 0);
  for (int i = 0; i < nsh; ++i)
    if (dshapes[i].is_static) static_off[dshapes[i].world + 1]++;
  for (int k = 0; k < n_worlds; ++k) static_off[k + 1] += static_off[k];
  {
    std::vector<int> cursor(static_off.begin(), static_off.end() - 1);
    static_list.resize(static_off[n_worlds]);
    for (int i = 0; i < nsh; ++i)
      if (dshapes[i].is_static) static_list[cursor[dshapes[i].world]++] = i;
  }
  // shapes of moving bodies per sub-world for the bullets' continuous pass: the kinematic
  // bodies' in shape order, then the dynamic bodies' (the reference queries its kinematic tree,
  // then its dynamic tree, continuous.rs:429-448)
  std::vector<int> dyn_list, dyn_off(n_worlds + 1, 0);
  for (int i = 0; i < nsh; ++i)
    if (w->bodies[dshapes[i].body].type != NS_STATIC_BODY) dyn_off[dshapes[i].world + 1]++;
  for (int k = 0; k < n_worlds; ++k) dyn_off[k + 1] += dyn_off[k];
  {
    std::vector<int> cursor(dyn_off.begin(), dyn_off.end() - 1);
    dyn_list.resize(dyn_off[n_worlds]);
    for (int type : {NS_KINEMATIC_BODY, NS_DYNAMIC_BODY})
      for (int i = 0; i < nsh; ++i)
        if (w->bodies[dshapes[i].body].type == type) dyn_list[cursor[dshapes[i].world]++] = i;
  }
  // the sweep of a body starts at its pose at upload (body_api.rs:221, :533 center0/rotation0)
  for (DSim& s : w->asims) { s.cx0 = s.cx; s.cy0 = s.cy; s.cz0 = s.cz; s.q0 = s.q; }
  for (DSim& s : w->ssims) { s.cx0 = s.cx; s.cy0 = s.cy; s.cz0 = s.cz; s.q0 = s.q; }
  std::vector<int> large_off(n_worlds + 1, 0);
  for (int i : large) large_off[dshapes[i].world + 1]++;
  for (int k = 0; k < n_worlds; ++k) large_off[k + 1] += large_off[k];
  // grid cell edge: a bound on every small proxy's fat-AABB extent on any axis. A moving shape's
  // tight box lies within twice its bounding radius (the shape margin of
  // shape_creation.rs:199), and finalize grows it by the speculative distance and the shape's
  // AABB margin on each side; a static shape keeps its creation-time box.
  {
    float ext = 1e-3f;
    for (int i = 0; i < nsh; ++i) {
      const HostShape& h = w->shapes[i];
      if (std::find(large.begin(), large.end(), i) != large.end()) continue;
      float e;
      if (h.d.is_static) {
        const AABB& f = w->fat[i];
        e = maxf(f.hi.x - f.lo.x, maxf(f.hi.y - f.lo.y, f.hi.z - f.lo.z));
      } else {
        e = 2.0f * h.bound_radius + 2.0f * (speculative_distance() + h.d.aabb_margin);
      }
      ext = maxf(ext, e);
    }
    d.cell = ext * 1.001f + 1e-3f;
    d.inv_cell = 1.0f / d.cell;
    // at least twice as many buckets as small proxies: the keys of a 10 000-shape world fit in 16
    // bits, two passes of the radix sort (proxies met through a hash collision are filtered by
    // their cell)
    int buckets = 1024;
    while (buckets < 2 * std::max(d.n_small, 1)) buckets <<= 1;
    d.cell_mask = buckets - 1;
    w->sort_bits = 1;
    while ((1u << w->sort_bits) <= (unsigned)buckets) ++w->sort_bits;
  }
  // joint partner CSR (joint.rs:164: joints without collide_connected disable the pair)
  std::vector<int> joff(nb + 1, 0), jother;
  for (int i = 0; i < nb; ++i) {
    joff[i] = (int)jother.size();
    if (i < (int)w->joint_partners.size())
      for (int o : w->joint_partners[i]) jother.push_back(o);
  }
  joff[nb] = (int)jother.size();
  // joints grouped by graph color
  std::vector<int> jlist;
  for (int c = 0; c < kGraphColorCount; ++c) {
    w->jr.off[c] = (int)jlist.size();
    for (int j = 0; j < nj; ++j)
      if (w->joints[j].color == c) jlist.push_back(j);
  }
  w->jr.off[kGraphColorCount] = (int)jlist.size();

#define ALLOC(field, T, n) do { d.field = dalloc<T>(w, (n), &st); if (!d.field) return st; } while (0)
  ALLOC(asims, DSim, na); ALLOC(states, DState, na); ALLOC(ssims, DSim, ns);
  ALLOC(shapes, DShape, nsh); ALLOC(hulls, Hull, nsh); ALLOC(fat, AABB, nsh); ALLOC(moved, int, nsh);
  ALLOC(body_shapes, int, body_shapes.size()); ALLOC(body_mask, uint32_t, nb); ALLOC(body_dyn, uint8_t, nb);
  ALLOC(body_joint_off, int, nb + 1); ALLOC(body_joint_other, int, jother.size());
  ALLOC(contacts, DContact, cap); ALLOC(free_stack, int, cap);
  ALLOC(hs, unsigned long long, hs_size);
  ALLOC(changed_bits, uint32_t, d.n_words); ALLOC(changed_list, int, cap); ALLOC(destroyed, int, cap);
  ALLOC(overflow_list, int, cap); ALLOC(ovf, DOverflow, cap);
  ALLOC(joints, DJoint, nj); ALLOC(joint_list, int, jlist.size());
  ALLOC(bp_keys_in, uint32_t, nsh); ALLOC(bp_keys_out, uint32_t, nsh);
  ALLOC(bp_vals_in, int, nsh); ALLOC(bp_vals_out, int, nsh);
  ALLOC(bp_xy, float4, nsh); ALLOC(bp_z, float2, nsh); ALLOC(bp_meta, int, nsh);
  ALLOC(cells, int2, (size_t)d.cell_mask + 1); ALLOC(bp_world, int, nsh);
  ALLOC(collide_list, int, (size_t)kCollideQueues * cap);
  ALLOC(world_cbase, int, n_worlds + 1); ALLOC(world_shape, int, n_worlds + 1);
  ALLOC(pool_top, int, n_worlds); ALLOC(pool_next, int, n_worlds); ALLOC(ovf_count, int, n_worlds);
  ALLOC(large_off, int, n_worlds + 1);
  ALLOC(large_list, int, large.size());
  ALLOC(fast_list, int, std::max(na, 1)); ALLOC(bullet_list, int, std::max(na, 1));
  ALLOC(dyn_off, int, n_worlds + 1); ALLOC(dyn_list, int, std::max<size_t>(dyn_list.size(), 1));
  ALLOC(static_off, int, n_worlds + 1);
  ALLOC(static_list, int, std::max<size_t>(static_list.size(), 1)); ALLOC(saabb, AABB, nsh);
  ALLOC(seg_count, int, nsh); ALLOC(seg_off, int, nsh); ALLOC(seg_cursor, int, nsh);
  ALLOC(cand, unsigned long long, cap); ALLOC(sorted_keys, unsigned long long, cap);
  ALLOC(block_color, int, (size_t)d.n_color_blocks * 24);
  ALLOC(long_segment, int, kLongSegmentCap);
  ALLOC(ctl, Control, 1);
  ALLOC(bwd, float4, 48 * (size_t)na); ALLOC(bw_mask, uint32_t, na); ALLOC(slot_cid, int, cap); ALLOC(slot_state, uint8_t, cap);
  CPlanes& P = d.cp;
  P.cap = cap;
#define PALLOC(field, T, n) do { P.field = dalloc<T>(w, (n), &st); if (!P.field) return st; } while (0)
  PALLOC(idx, int4, cap); PALLOC(mass, float4, cap); PALLOC(ia0, float4, cap); PALLOC(ia1, float4, cap);
  PALLOC(ib1, float4, cap); PALLOC(n, float4, cap); PALLOC(t1, float4, cap); PALLOC(t2, float4, cap);
  PALLOC(ca, float4, cap); PALLOC(cb, float4, cap); PALLOC(tm, float4, cap); PALLOC(fr, float4, cap);
  PALLOC(roll, float4, cap); PALLOC(rm, float4, cap);
  PALLOC(pra, float4, 4 * (size_t)cap); PALLOC(prb, float4, 4 * (size_t)cap);
  PALLOC(pimp, float4, 4 * (size_t)cap); PALLOC(prest, float, 4 * (size_t)cap);
#undef PALLOC
#undef ALLOC
  if ((st = upload(w, d.asims, w->asims))) return st;
  if ((st = upload(w, d.states, w->states))) return st;
  if ((st = upload(w, d.ssims, w->ssims))) return st;
  if ((st = upload(w, d.shapes, dshapes))) return st;
  if ((st = upload(w, d.hulls, hulls))) return st;
  if ((st = upload(w, d.fat, w->fat))) return st;
  if ((st = upload(w, d.body_shapes, body_shapes))) return st;
  if ((st = upload(w, d.body_mask, w->body_mask))) return st;
  {
    std::vector<uint8_t> dyn(w->bodies.size());
    for (size_t i = 0; i < w->bodies.size(); ++i) dyn[i] = w->bodies[i].type == NS_DYNAMIC_BODY ? 1 : 0;
    if ((st = upload(w, d.body_dyn, dyn))) return st;
  }
  if ((st = upload(w, d.body_joint_off, joff))) return st;
  if ((st = upload(w, d.body_joint_other, jother))) return st;
  if ((st = upload(w, d.large_list, large))) return st;
  if ((st = upload(w, d.world_cbase, world_cbase))) return st;
  if ((st = upload(w, d.world_shape, world_shape))) return st;
  if ((st = upload(w, d.large_off, large_off))) return st;
  if ((st = upload(w, d.static_off, static_off))) return st;
  if ((st = upload(w, d.static_list, static_list))) return st;
  if ((st = upload(w, d.dyn_off, dyn_off))) return st;
  if ((st = upload(w, d.dyn_list, dyn_list))) return st;
  if ((st = upload(w, d.saabb, w->saabb))) return st;
  {
    std::vector<int> zeros(n_worlds, 0);
    if ((st = upload(w, d.pool_top, zeros))) return st;
    if ((st = upload(w, d.pool_next, zeros))) return st;
    if ((st = upload(w, d.ovf_count, zeros))) return st;
  }
  if ((st = upload(w, d.joint_list, jlist))) return st;
  std::vector<DJoint> dj = w->joints;
  if ((st = upload(w, d.joints, dj))) return st;
  std::vector<int> moved(nsh, 1);
  if ((st = upload(w, d.moved, moved))) return st;
  NS_CUDA(w, cudaMemsetAsync(d.hs, 0xff, sizeof(unsigned long long) * (size_t)hs_size, w->stream));
  Control c0;
  memset(&c0, 0, sizeof(c0));
  c0.moved_count = nsh;
  NS_CUDA(w, cudaMemcpyAsync(d.ctl, &c0, sizeof(Control), cudaMemcpyHostToDevice, w->stream));
  NS_CUDA(w, cudaFuncSetAttribute(k_bp_segsort_long, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(kLongSegmentKeys * sizeof(unsigned long long))));
  // CUB scratch (sizes depend only on the shape count)
  NS_CUDA(w, cub::DeviceRadixSort::SortPairs(nullptr, w->cub_sort_bytes, d.bp_keys_in, d.bp_keys_out,
                                              d.bp_vals_in, d.bp_vals_out, nsh));
  NS_CUDA(w, cub::DeviceScan::ExclusiveSum(nullptr, w->cub_scan_bytes, d.seg_count, d.seg_off, nsh));
  NS_CUDA(w, cudaMalloc(&w->cub_sort_tmp, std::max<size_t>(w->cub_sort_bytes, 16)));
  w->allocations.push_back(w->cub_sort_tmp);
  w->allocation_bytes.push_back(std::max<size_t>(w->cub_sort_bytes, 16));
  NS_CUDA(w, cudaMalloc(&w->cub_scan_tmp, std::max<size_t>(w->cub_scan_bytes, 16)));
  w->allocations.push_back(w->cub_scan_tmp);
  w->allocation_bytes.push_back(std::max<size_t>(w->cub_scan_bytes, 16));
  // state pass: staged change chunks always live in shared memory; every body's color
  // mask joins them there when it fits, and with it a per-body word for the parallel rounds
  // when that fits too (state_mode 2; 1: masks only, serial walk; 0: masks in global memory)
  int max_smem = 0;
  NS_CUDA(w, cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, w->def.device));
  size_t stage_bytes = (size_t)kStateChunk * 5 * sizeof(int);
  size_t need = stage_bytes + (size_t)nb * sizeof(uint32_t);
  size_t need2 = need + (size_t)nb * sizeof(int);
  w->state_mode = need2 + 16 * 1024 <= (size_t)max_smem ? 2 : need + 16 * 1024 <= (size_t)max_smem ? 1 : 0;
  w->state_smem = w->state_mode == 2 ? need2 : w->state_mode == 1 ? need : stage_bytes;
  // the kernel's static shared memory counts against the same 48 KB default, so the limit is
  // always raised to what this launch needs
  NS_CUDA(w, cudaFuncSetAttribute(k_state_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w->state_smem));
  // solver launch shape. solver_blocks 0: a cooperative grid over every SM for a batch of
  // sub-worlds or a world of kGridSolveBodies awake bodies or more, else one cluster of the
  // largest size that fits (16 CTAs on B200); 1..16: one thread-block cluster of that many CTAs
  // (non-portable sizes above 8); above 16: a cooperative grid of that many blocks, capped at
  // what fits co-resident. A colour phase costs about what one constraint's chain costs: the
  // cluster's barrier is the cheaper (0.3 against 1.2 us), the grid stages every colour of up to
  // 32 items per block in shared memory (on the 10 000-body pile: 0.61 against 0.68 ms per step).
  {
    constexpr int kGridSolveBodies = 2048;
    int want = w->def.solver_blocks > 0 ? w->def.solver_blocks
               : ((n_worlds > 1 || na >= kGridSolveBodies) ? std::max(w->sm_count, kMaxSolveCluster + 1)
                                                           : kMaxSolveCluster);
    if (want >= 1 && want <= kMaxSolveCluster) {
      NS_CUDA(w, cudaFuncSetAttribute(k_solve<false, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
      NS_CUDA(w, cudaFuncSetAttribute(k_solve<false, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
      int best = 0;
      for (int cs = want; cs >= 1; --cs) {
        cudaLaunchConfig_t cfg = {};
        cfg.blockDim = dim3(kSolveThreads);
        cfg.gridDim = dim3(cs);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        cudaError_t e = cudaOccupancyMaxActiveClusters(&clusters, k_solve<false, false>, &cfg);
        if (e == cudaSuccess && clusters >= 1) { best = cs; break; }
        cudaGetLastError();
      }
      if (best == 0) return fail(w, NS_ERR_CUDA, "the solver cluster does not fit on this device");
      w->solver_blocks = best;
      w->solver_grid = false;
    } else {
      int per_sm = 0;
      NS_CUDA(w, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve<true, false>, kSolveThreads, 0));
      int max_blocks = per_sm * w->sm_count;
      if (max_blocks < 1) return fail(w, NS_ERR_CUDA, "the solver block does not fit on this device");
      int blocks_ = std::min(want, max_blocks);
      w->solver_blocks = blocks_;
      w->solver_grid = true;
    }
  }
  // readback staging (64 B per body) and the body location table
  {
    std::vector<int> loc(nb);
    for (int i = 0; i < nb; ++i) loc[i] = w->bodies[i].set == 2 ? w->bodies[i].local : -(w->bodies[i].local + 1);
    w->body_loc = dalloc<int>(w, nb, &st);
    if (!w->body_loc) return st;
    if ((st = upload(w, w->body_loc, loc))) return st;
    w->out_stage = dalloc<char>(w, (size_t)std::max(nb, 1) * 64, &st);
    if (!w->out_stage) return st;
    NS_CUDA(w, cudaHostAlloc((void**)&w->host_ctl, sizeof(Control), cudaHostAllocDefault));
    NS_CUDA(w, cudaHostAlloc((void**)&w->host_in, sizeof(float) * 6 * (size_t)std::max(nb, 1), cudaHostAllocDefault));
    w->in_stage = dalloc<float>(w, 6 * (size_t)std::max(nb, 1), &st);
    if (!w->in_stage) return st;
    NS_CUDA(w, cudaEventCreateWithFlags(&w->in_done, cudaEventDisableTiming));
    w->n_gyroscopic = 0;
    for (const DSim& a : w->asims) w->n_gyroscopic += (a.flags & kGyroscopic) ? 1 : 0;
  }
  NS_CUDA(w, cudaStreamSynchronize(w->stream));
  const char* eager = getenv("NATSEL_EAGER");
  w->eager = eager && eager[0] == '1';
  w->uploaded = true;
  return NS_OK;
}

// Broadphase pair update (contact_creation.rs:901 update_broad_phase_pairs): new pairs of
// overlapping fat AABBs with a moved proxy become contacts, in pair-key order.
int enqueue_pair_update(ns_world* w) {
  DW d = w->dw;
  cudaStream_t s = w->stream;
  int nsh = d.n_shapes;
  auto blocks = [](int n, int t) { return std::max(1, (n + t - 1) / t); };
  int nk = 0;
  NS_CUDA(w, cudaMemsetAsync(d.seg_count, 0, sizeof(int) * (size_t)nsh, s));
  NS_CUDA(w, cudaMemsetAsync(d.seg_cursor, 0, sizeof(int) * (size_t)nsh, s));
  k_hs_rebuild_clear<<<4 * w->sm_count, 256, 0, s>>>(d); ++nk;
  k_hs_rebuild_insert<<<4 * w->sm_count, 256, 0, s>>>(d); ++nk;
  k_bp_keys<<<blocks(nsh, 256), 256, 0, s>>>(d); ++nk;
  NS_CUDA(w, cub::DeviceRadixSort::SortPairs(w->cub_sort_tmp, w->cub_sort_bytes, d.bp_keys_in, d.bp_keys_out,
                                              d.bp_vals_in, d.bp_vals_out, nsh, 0, w->sort_bits, s));
  NS_CUDA(w, cudaMemsetAsync(d.cells, 0, sizeof(int2) * ((size_t)d.cell_mask + 1), s));
  k_bp_gather<<<blocks(d.n_small, 256), 256, 0, s>>>(d); ++nk;
  k_bp_query<<<blocks(d.n_small, kQueryThreads / 32), kQueryThreads, 0, s>>>(d); ++nk;
  k_bp_large<<<blocks(nsh, 256), 256, 0, s>>>(d); ++nk;
  NS_CUDA(w, cub::DeviceScan::ExclusiveSum(w->cub_scan_tmp, w->cub_scan_bytes, d.seg_count, d.seg_off, nsh, s));
  k_bp_scatter<<<4 * w->sm_count, 256, 0, s>>>(d); ++nk;
  NS_CUDA(w, cudaMemsetAsync(&d.ctl->long_segments, 0, sizeof(int), s));
  k_bp_segsort<<<blocks(nsh, 256), 256, 0, s>>>(d); ++nk;
  k_bp_segsort_long<<<32, 1024, kLongSegmentKeys * sizeof(unsigned long long), s>>>(d); ++nk;
  k_bp_create<<<4 * w->sm_count, 256, 0, s>>>(d); ++nk;
  k_bp_pools<<<blocks(d.n_worlds, 256), 256, 0, s>>>(d); ++nk;
  k_bp_finish<<<1, 1, 0, s>>>(d); ++nk;
  NS_CUDA(w, cudaMemsetAsync(d.moved, 0, sizeof(int) * (size_t)nsh, s));
  w->pair_kernels = nk;
  return NS_OK;
}

StepParams make_step_params(const ns_world* w, float dt, int substeps) {
  StepParams p;
  memset(&p, 0, sizeof(p));
  p.dt = dt;
  p.substeps = substeps < 1 ? 1 : substeps;
  if (dt > 0.0f) {
    p.inv_dt = 1.0f / dt;
    p.h = dt / (float)p.substeps;
    p.inv_h = (float)p.substeps * p.inv_dt;
  }
  float hz = minf(w->def.contact_hertz, 0.125f * p.inv_h);
  p.contact_softness = make_soft(hz, w->def.contact_damping_ratio, p.h);
  p.static_softness = make_soft(2.0f * hz, 0.5f * w->def.contact_damping_ratio, p.h);
  p.contact_speed = w->def.contact_speed;
  p.max_linear_speed = w->def.max_linear_speed;
  p.restitution_threshold = w->def.restitution_threshold;
  p.warm_start = w->def.enable_warm_starting ? 1.0f : 0.0f;
  p.restitution_iterations = w->def.restitution_iterations;
  p.enable_continuous = w->def.enable_continuous;
  p.gravity = v3(w->def.gravity[0], w->def.gravity[1], w->def.gravity[2]);
  return p;
}

// Device copies of one step's inputs that the adjoint replays (nsd_adjoint.cuh StepTape).
struct HostStepTape {
  StepTape dev;
  SolveTape solve;
  CopyOp* plane_ops = nullptr;  // device table: the prepared planes -> dev.planes
  int n_plane_ops = 0;
};

// One step. With a tape the narrowphase outcomes, the contacts before the narrowphase and
// after the state pass, the prepared planes and the solver's inputs are recorded as well
// (the arithmetic is unchanged).
int enqueue_step(ns_world* w, float dt, int substeps, const HostStepTape* tape = nullptr) {
  DW d = w->dw;
  cudaStream_t s = w->stream;
  StepParams p = make_step_params(w, dt, substeps);
  auto blocks = [](int n, int t) { return std::max(1, (n + t - 1) / t); };
  int nk = 0;
  if (tape) {
    d.np_mode = tape->dev.mode;
    NS_CUDA(w, cudaMemsetAsync(tape->dev.mode, 0, (size_t)d.cap, s));
    NS_CUDA(w, cudaMemcpyAsync(tape->dev.sims, d.asims, sizeof(DSim) * (size_t)d.n_awake, cudaMemcpyDeviceToDevice, s));
  }
  // phase events: graph nodes that record externally when captured, plain records otherwise
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  NS_CUDA(w, cudaStreamIsCapturing(s, &capturing));
  unsigned ev_flags = capturing == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
  NS_CUDA(w, cudaEventRecordWithFlags(w->ev[0], s, ev_flags));
  {
    int st = enqueue_pair_update(w);
    if (st) return st;
  }
  NS_CUDA(w, cudaEventRecordWithFlags(w->ev[1], s, ev_flags));
  if (tape)
    NS_CUDA(w, cudaMemcpyAsync(tape->dev.pre, d.contacts, sizeof(DContact) * (size_t)d.cap, cudaMemcpyDeviceToDevice, s));
  // narrowphase (collide_pass.rs:164)
  NS_CUDA(w, cudaMemsetAsync(d.ctl->collide_count, 0, sizeof(d.ctl->collide_count), s));
  k_collide<<<std::min(blocks(d.cap, w->recycle_threads), w->recycle_per_sm * w->sm_count), w->recycle_threads, 0, s>>>(d);
  ++nk;
  k_collide_update<<<std::min(blocks(d.cap, w->update_threads), w->update_per_sm * w->sm_count), w->update_threads, 0,
                     s>>>(d);
  ++nk;
  NS_CUDA(w, cudaEventRecordWithFlags(w->ev[2], s, ev_flags));
  // state pass, colors, prepare (collide_pass.rs:386, solver_prepare.rs:269)
  if (d.n_worlds == 1) {
    k_state_pass<<<1, kStatePassThreads, w->state_smem, s>>>(d, w->state_mode); ++nk;
  } else {
    NS_CUDA(w, cudaMemsetAsync(&d.ctl->changed_count, 0, sizeof(int), s));
    NS_CUDA(w, cudaMemsetAsync(&d.ctl->overflow_count, 0, sizeof(int), s));
    k_state_worlds<<<blocks(d.n_worlds, 128), 128, 0, s>>>(d); ++nk;
    k_state_finish<<<1, 1, 0, s>>>(d); ++nk;
  }
  if (tape)
    NS_CUDA(w, cudaMemcpyAsync(tape->dev.post, d.contacts, sizeof(DContact) * (size_t)d.cap, cudaMemcpyDeviceToDevice, s));
  k_color_count<<<d.n_color_blocks, kColorBlock, 0, s>>>(d); ++nk;
  k_color_scan<<<kOverflowIndex, kColorScanThreads, 0, s>>>(d); ++nk;
  k_color_scatter<<<d.n_color_blocks, kColorBlock, 0, s>>>(d); ++nk;
  k_prepare_slots<<<std::min(blocks(d.cap, w->prepare_threads), w->prepare_per_sm * w->sm_count), w->prepare_threads, 0,
                    s>>>(d, p);
  ++nk;
  k_prepare_overflow<<<std::min(std::max(d.n_worlds, 8), 4096), 128, 0, s>>>(d, p); ++nk;
  if (d.n_joints > 0) {
    k_prepare_joints<<<blocks(d.n_joints, 128), 128, 0, s>>>(d, p);
    ++nk;
    if (tape)
      NS_CUDA(w, cudaMemcpyAsync(tape->dev.joints, d.joints, sizeof(DJoint) * (size_t)d.n_joints,
                                 cudaMemcpyDeviceToDevice, s));
  }
  NS_CUDA(w, cudaEventRecordWithFlags(w->ev[3], s, ev_flags));
  if (tape) {
    k_multi_copy<<<4 * w->sm_count, 256, 0, s>>>(tape->plane_ops, tape->n_plane_ops);
    NS_CUDA(w, cudaMemcpyAsync(tape->dev.ctl, d.ctl, sizeof(Control), cudaMemcpyDeviceToDevice, s));
  }
  // solver stages (solver_stages.rs:543)
  {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(w->solver_blocks);
    cfg.blockDim = dim3(kSolveThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    if (d.n_awake > 0) {
      NS_CUDA(w, cudaMemsetAsync(d.bw_mask, 0, sizeof(uint32_t) * d.n_awake, s));
      k_warm_slots<<<4 * w->sm_count, 256, 0, s>>>(d, w->jr); ++nk;
    }
    if (w->solver_grid) {
      NS_CUDA(w, cudaMemsetAsync(&d.ctl->barrier_count, 0, sizeof(int), s));
      attr[0].id = cudaLaunchAttributeCooperative;
      attr[0].val.cooperative = 1;
    } else {
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = w->solver_blocks;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
    }
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SolveTape tp;
    memset(&tp, 0, sizeof(tp));
    if (tape) tp = tape->solve;
    if (tape && w->solver_grid) NS_CUDA(w, cudaLaunchKernelEx(&cfg, k_solve<true, true>, d, p, w->jr, tp));
    else if (tape) NS_CUDA(w, cudaLaunchKernelEx(&cfg, k_solve<false, true>, d, p, w->jr, tp));
    else if (w->solver_grid) NS_CUDA(w, cudaLaunchKernelEx(&cfg, k_solve<true, false>, d, p, w->jr, tp));
    else NS_CUDA(w, cudaLaunchKernelEx(&cfg, k_solve<false, false>, d, p, w->jr, tp));
    ++nk;
  }
  NS_CUDA(w, cudaEventRecordWithFlags(w->ev[4], s, ev_flags));
  // finalize (solver_integration.rs:435)
  if (w->def.enable_continuous) NS_CUDA(w, cudaMemsetAsync(&d.ctl->fast_count, 0, 2 * sizeof(int), s));
  k_finalize<<<blocks(d.n_awake, 128), 128, 0, s>>>(d, p); ++nk;
  if (w->def.enable_continuous) {
    // continuous.rs:337 for the fast bodies finalize queued (solver_integration.rs:540-566)
    k_continuous<<<blocks(d.n_awake, 64), 64, 0, s>>>(d, p); ++nk;
    // then the fast bullets, one warp each, after every other body is final (:949-958)
    if (w->n_bullets > 0) { k_bullets<<<blocks(32 * w->n_bullets, 128), 128, 0, s>>>(d, p); ++nk; }
  }
  NS_CUDA(w, cudaEventRecordWithFlags(w->ev[5], s, ev_flags));
  NS_CUDA(w, cudaGetLastError());
  w->step_kernels = w->pair_kernels + nk;
  return NS_OK;
}

// body_api.rs:351 apply_body_force_to_center and :366 apply_body_torque for every body at
// once: awake bodies accumulate force and torque until finalize clears them.
__global__ void k_apply_forces(DW d, const int* body_loc, int nb, const float* force, const float* torque) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    int loc = body_loc[i];
    if (loc < 0) continue;
    DSim& s = d.asims[loc];
    if (force) s.force = s.force + v3(force[3 * i], force[3 * i + 1], force[3 * i + 2]);
    if (torque) s.torque = s.torque + v3(torque[3 * i], torque[3 * i + 1], torque[3 * i + 2]);
  }
}

// Packs the body state in id order for readback: pos f64x3 | rot f32x4 | lin f32x3 | ang f32x3.
__global__ void k_gather_bodies(DW d, const int* body_loc, int nb, double* pos, float* rot, float* lin,
                                float* ang) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    int loc = body_loc[i];
    const DSim& s = loc >= 0 ? d.asims[loc] : d.ssims[-loc - 1];
    pos[3 * i] = s.px; pos[3 * i + 1] = s.py; pos[3 * i + 2] = s.pz;
    rot[4 * i] = s.q.v.x; rot[4 * i + 1] = s.q.v.y; rot[4 * i + 2] = s.q.v.z; rot[4 * i + 3] = s.q.s;
    V3 v = v3(0, 0, 0), wv = v3(0, 0, 0);
    if (loc >= 0) { v = d.states[loc].v; wv = d.states[loc].w; }
    lin[3 * i] = v.x; lin[3 * i + 1] = v.y; lin[3 * i + 2] = v.z;
    ang[3 * i] = wv.x; ang[3 * i + 1] = wv.y; ang[3 * i + 2] = wv.z;
  }
}

int control_status(ns_world* w, const Control& c) {
  if (c.error == kErrCapacity) return fail(w, NS_ERR_CAPACITY, "device capacity exceeded (contacts or pairs)");
  if (c.error == kErrTimeout) return fail(w, NS_ERR_TIMEOUT, "solver grid barrier timed out");
  if (c.error == kErrNonFinite)
    return fail(w, NS_ERR_NONFINITE, "a body velocity, position or rotation became NaN or Inf in finalize");
  if (c.error) return fail(w, c.error, "device error %d", c.error);
  return NS_OK;
}

int read_control(ns_world* w, Control* c) {
  NS_CUDA(w, cudaStreamSynchronize(w->stream));
  NS_CUDA(w, cudaMemcpy(c, w->dw.ctl, sizeof(Control), cudaMemcpyDeviceToHost));
  return NS_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Rollout tape and adjoint (ns_world_tape_begin / ns_world_vjp).
//
// While a tape records, every step is logged and the world's device buffers are copied to a
// checkpoint whenever `every` substeps have passed since the last one. The vector-Jacobian
// product walks the checkpoint segments backwards: it restores a checkpoint, replays the
// segment's steps with the solver tape on (bit-identical to the recorded steps: same kernels,
// same inputs), and runs the reverse kernels step by step from the segment's end. The world is
// put back in its final state afterwards.
struct AdStepRec { float dt; int substeps; };
struct AdCheckpoint {
  char* data = nullptr;      // snapshot of every allocation (layout in ns_world::snap_ops)
};
struct AdTape {
  int every = 8;
  bool recording = false;
  std::vector<AdStepRec> steps;
  std::vector<int> ckpt_at;           // index of the first step after each checkpoint
  std::vector<AdCheckpoint> ckpt;
  int since = 0;
  int64_t replay_mismatch = 0;        // narrowphase replays that missed the recorded manifold
  int64_t vjp_calls = 0;
  int64_t vjp_launches = 0;           // own kernel launches of the last VJP
};

namespace {

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device scratch for checkpoints and the VJP comes from one stream-ordered memory pool per
// device, shared by all worlds of the process: memory a destroyed world gave back is reused by
// the next without a cudaMalloc, and up to kPoolKeep bytes stay reserved between uses.
constexpr uint64_t kPoolKeep = 16ull << 30;
cudaMemPool_t scratch_pool(int device) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(device);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) { cudaGetLastError(); pool = nullptr; }
  if (pool) {
    uint64_t keep = kPoolKeep;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  pools[device] = pool;
  return pool;
}

int scratch_alloc(ns_world* w, char** p, size_t bytes) {
  cudaMemPool_t pool = scratch_pool(w->def.device);
  if (!pool) return fail(w, NS_ERR_CUDA, "no memory pool on device %d", w->def.device);
  NS_CUDA(w, cudaMallocFromPoolAsync((void**)p, bytes, pool, w->stream));
  return NS_OK;
}

void scratch_free(ns_world* w, char* p) {
  if (p) cudaFreeAsync(p, w->stream);
}

int take_checkpoint(ns_world* w, AdCheckpoint* ck) {
  if (w->allocation_bytes.size() != w->allocations.size())
    return fail(w, NS_ERR_INVALID, "device allocation table is inconsistent");
  const size_t n = w->allocations.size();
  if (!w->snap_ops) {
    std::vector<SnapOp> ops(n);
    size_t bytes = 0;
    for (size_t i = 0; i < n; ++i) {
      ops[i] = {(char*)w->allocations[i], bytes, w->allocation_bytes[i]};
      bytes += align256(w->allocation_bytes[i]);
    }
    char* table = nullptr;
    int st = scratch_alloc(w, &table, std::max<size_t>(n, 1) * sizeof(SnapOp));
    if (st) return st;
    w->snap_ops = (SnapOp*)table;
    w->snap_bytes = bytes;
    NS_CUDA(w, cudaMemcpyAsync(w->snap_ops, ops.data(), n * sizeof(SnapOp), cudaMemcpyHostToDevice, w->stream));
    NS_CUDA(w, cudaStreamSynchronize(w->stream));
  }
  if (!ck->data && !w->ckpt_pool.empty()) {
    ck->data = w->ckpt_pool.back();
    w->ckpt_pool.pop_back();
  }
  if (!ck->data) {
    int st = scratch_alloc(w, &ck->data, w->snap_bytes);
    if (st) return st;
  }
  k_snapshot<<<4 * w->sm_count, 256, 0, w->stream>>>(w->snap_ops, (int)n, ck->data, 1);
  NS_CUDA(w, cudaGetLastError());
  return NS_OK;
}

int restore_checkpoint(ns_world* w, const AdCheckpoint& ck) {
  k_snapshot<<<4 * w->sm_count, 256, 0, w->stream>>>(w->snap_ops, (int)w->allocations.size(), ck.data, 0);
  NS_CUDA(w, cudaGetLastError());
  return NS_OK;
}

// A checkpoint buffer goes back to the world's pool (the stream must be past its last use).
void release_checkpoint(ns_world* w, AdCheckpoint* ck) {
  if (ck->data) w->ckpt_pool.push_back(ck->data);
  ck->data = nullptr;
}

void free_tape(ns_world* w) {
  if (!w->tape) return;
  cudaStreamSynchronize(w->stream);
  for (AdCheckpoint& c : w->tape->ckpt) release_checkpoint(w, &c);
  delete w->tape;
  w->tape = nullptr;
}

// Device scratch of at least `bytes`, kept in *buf / *cap for later calls.
int reuse_buffer(ns_world* w, char** buf, size_t* cap, size_t bytes) {
  if (*cap >= bytes && *buf) return NS_OK;
  scratch_free(w, *buf);
  *buf = nullptr;
  *cap = 0;
  int st = scratch_alloc(w, buf, bytes);
  if (st) return st;
  *cap = bytes;
  return NS_OK;
}

int tape_after_step(ns_world* w, float dt, int substeps) {
  AdTape* t = w->tape;
  t->steps.push_back({dt, substeps});
  t->since += substeps;
  if (t->since >= t->every) {
    t->ckpt.emplace_back();
    int st = take_checkpoint(w, &t->ckpt.back());
    if (st) return st;
    t->ckpt_at.push_back((int)t->steps.size());
    t->since = 0;
  }
  return NS_OK;
}

// The adjoint covers one world of boxes, spheres and capsules with revolute joints, without
// rolling resistance, continuous collision, or joints in the overflow colour.
int check_adjoint_scope(ns_world* w) {
  if (w->sub_body_begin.size() > 1) return fail(w, NS_ERR_UNSUPPORTED, "the adjoint takes a single world");
  if (w->jr.off[kOverflowIndex + 1] > w->jr.off[kOverflowIndex])
    return fail(w, NS_ERR_UNSUPPORTED, "joints in the overflow colour; the adjoint does not cover them");
  for (const DJoint& j : w->joints)
    if (j.type != kJointRevolute) return fail(w, NS_ERR_UNSUPPORTED, "the adjoint covers revolute joints only");
  if (w->def.enable_continuous) return fail(w, NS_ERR_UNSUPPORTED, "the adjoint needs enable_continuous = 0");
  for (const HostBody& b : w->bodies)
    if (b.type == NS_KINEMATIC_BODY) return fail(w, NS_ERR_UNSUPPORTED, "the adjoint does not cover kinematic bodies");
  for (const HostShape& hs : w->shapes)
    if (hs.d.rolling != 0.0f) return fail(w, NS_ERR_UNSUPPORTED, "the adjoint does not cover rolling resistance");
  for (const DSim& a : w->asims) {
    if (a.local_center.x != 0.0f || a.local_center.y != 0.0f || a.local_center.z != 0.0f)
      return fail(w, NS_ERR_UNSUPPORTED, "the adjoint needs each body's centre of mass at its origin");
  }
  return NS_OK;
}

// Device storage of the step tapes of one segment.
struct TapeSet {
  char* data = nullptr;
  size_t bytes = 0;
  std::vector<HostStepTape> steps;
};

int alloc_tapes(ns_world* w, int count, int max_substeps, TapeSet* ts) {
  const DW& d = w->dw;
  size_t cap = (size_t)d.cap, n = (size_t)std::max(d.n_awake, 1);
  std::vector<std::pair<size_t*, size_t>> parts;
  size_t per = 0;
  auto take = [&](size_t b) { size_t o = per; per += align256(b); return o; };
  size_t o_sims = take(sizeof(DSim) * n), o_pre = take(sizeof(DContact) * cap), o_post = take(sizeof(DContact) * cap);
  size_t o_ctl = take(sizeof(Control));
  size_t o_pl = take(sizeof(int4) * cap + 13 * sizeof(float4) * cap + 3 * 4 * sizeof(float4) * cap + 4 * sizeof(float) * cap + 16 * 20);
  size_t o_body = take(sizeof(DState) * 3 * n * max_substeps);
  size_t o_push = take(sizeof(float4) * 4 * cap * max_substeps);
  size_t o_relax = take(sizeof(float4) * 5 * cap * max_substeps);
  size_t o_fin = take(sizeof(float4) * cap), o_mode = take(cap), o_ops = take(sizeof(CopyOp) * 20);
  const int rest_its = std::max(w->def.restitution_iterations, 0);
  size_t o_rest = take(sizeof(float4) * 6 * cap * (size_t)std::max(rest_its, 1));
  const size_t nj = (size_t)std::max(d.n_joints, 1);
  size_t o_joints = take(sizeof(DJoint) * nj);
  size_t o_jrow = take(sizeof(float4) * 2 * 6 * nj * max_substeps), o_jwarm = take(sizeof(float4) * 4 * nj * max_substeps);
  int st = reuse_buffer(w, &w->tapes_buf, &w->tapes_cap, per * (size_t)count);
  if (st) return st;
  ts->data = w->tapes_buf;
  ts->bytes = per * (size_t)count;
  ts->steps.resize(count);
  for (int j = 0; j < count; ++j) {
    char* b = ts->data + per * (size_t)j;
    HostStepTape& h = ts->steps[j];
    StepTape& t = h.dev;
    t.sims = (DSim*)(b + o_sims); t.pre = (DContact*)(b + o_pre); t.post = (DContact*)(b + o_post);
    t.ctl = (Control*)(b + o_ctl);
    char* pl = b + o_pl;
    auto carve = [&](size_t bytes) { char* r = pl; pl += (bytes + 15) & ~(size_t)15; return r; };
    CPlanes& P = t.planes;
    const CPlanes& L = d.cp;
    P.cap = L.cap;
    P.idx = (int4*)carve(sizeof(int4) * cap);
    float4** f4[] = {&P.mass, &P.ia0, &P.ia1, &P.ib1, &P.n, &P.t1, &P.t2, &P.ca, &P.cb, &P.tm, &P.fr, &P.roll, &P.rm};
    for (float4** f : f4) *f = (float4*)carve(sizeof(float4) * cap);
    P.pra = (float4*)carve(sizeof(float4) * 4 * cap);
    P.prb = (float4*)carve(sizeof(float4) * 4 * cap);
    P.pimp = (float4*)carve(sizeof(float4) * 4 * cap);
    P.prest = (float*)carve(sizeof(float) * 4 * cap);
    std::vector<CopyOp> ops;
    ops.push_back({(const char*)L.idx, (char*)P.idx, sizeof(int4) * cap});
    float4* const* lf4[] = {&L.mass, &L.ia0, &L.ia1, &L.ib1, &L.n, &L.t1, &L.t2, &L.ca, &L.cb, &L.tm, &L.fr, &L.roll, &L.rm};
    for (int i = 0; i < 13; ++i) ops.push_back({(const char*)*lf4[i], (char*)*f4[i], sizeof(float4) * cap});
    ops.push_back({(const char*)L.pra, (char*)P.pra, sizeof(float4) * 4 * cap});
    ops.push_back({(const char*)L.prb, (char*)P.prb, sizeof(float4) * 4 * cap});
    ops.push_back({(const char*)L.pimp, (char*)P.pimp, sizeof(float4) * 4 * cap});
    t.body = (DState*)(b + o_body);
    t.push = (float4*)(b + o_push);
    t.relax = (float4*)(b + o_relax);
    t.fin = (float4*)(b + o_fin);
    t.mode = (uint8_t*)(b + o_mode);
    t.rest = (float4*)(b + o_rest);
    t.rest_iterations = rest_its;
    t.joints = (DJoint*)(b + o_joints);
    t.joint = (float4*)(b + o_jrow);
    t.jwarm = (float4*)(b + o_jwarm);
    t.n_joints = d.n_joints;
    t.substeps = 0;
    h.solve.body = t.body; h.solve.push = t.push; h.solve.relax = t.relax; h.solve.fin = t.fin;
    h.solve.rest = t.rest;
    h.solve.joint = d.n_joints > 0 ? t.joint : nullptr;
    h.solve.jwarm = d.n_joints > 0 ? t.jwarm : nullptr;
    h.plane_ops = (CopyOp*)(b + o_ops);
    h.n_plane_ops = (int)ops.size();
    NS_CUDA(w, cudaMemcpy(h.plane_ops, ops.data(), ops.size() * sizeof(CopyOp), cudaMemcpyHostToDevice));
  }
  return NS_OK;
}

// The reverse solve runs on the forward solver's launch shape (one thread-block cluster, or a
// cooperative grid when the world uses one): its phases are bounded by the barrier and one
// warp's latency chain, and a grid over every SM measured 2.4x slower on the 1024-box rollout.
template <bool kJoints>
int launch_adj_solve_t(ns_world* w, const StepTape& t, const AdjBufs& a, const StepParams& p) {
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(kAdjThreads);
  cfg.stream = w->stream;
  cudaLaunchAttribute attr[1];
  int blocks = w->solver_blocks;
  if (w->solver_grid) {
    int per_sm = 0;
    NS_CUDA(w, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adj_solve<true, kJoints>, kAdjThreads, 0));
    blocks = std::max(1, std::min(blocks, per_sm * w->sm_count));
    NS_CUDA(w, cudaMemsetAsync(&w->dw.ctl->barrier_count, 0, sizeof(int), w->stream));
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
  } else {
    NS_CUDA(w, cudaFuncSetAttribute(k_adj_solve<false, kJoints>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = blocks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
  }
  cfg.gridDim = dim3(blocks);
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (w->solver_grid) NS_CUDA(w, cudaLaunchKernelEx(&cfg, k_adj_solve<true, kJoints>, t, a, p, w->dw.ctl));
  else NS_CUDA(w, cudaLaunchKernelEx(&cfg, k_adj_solve<false, kJoints>, t, a, p, w->dw.ctl));
  return NS_OK;
}
int launch_adj_solve(ns_world* w, const StepTape& t, const AdjBufs& a, const StepParams& p) {
  return a.n_joints > 0 ? launch_adj_solve_t<true>(w, t, a, p) : launch_adj_solve_t<false>(w, t, a, p);
}

// Host check of the adjoint's local derivatives in f64: for each input direction i the
// dual-number VJP component sum_j ybar_j dy_j/dx_i is compared with the central difference of
// the same function evaluated in plain f64.
struct Rng64 {
  uint64_t s;
  double next() {  // uniform in [0, 1)
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
  }
  double range(double a, double b) { return a + (b - a) * next(); }
};

template <class Fn>
double vjp_fd_error(const std::vector<double>& x0, int ny, Fn fn, Rng64& rng, int n_dirs = -1) {
  const int nx = (int)x0.size();
  std::vector<double> ybar(ny);
  for (double& v : ybar) v = rng.range(-1.0, 1.0);
  std::vector<ad::Dual<double, 1>> yd(ny);
  std::vector<double> yp(ny), ym(ny), xp(x0), xm(x0);
  double worst = 0.0;
  for (int i = 0; i < (n_dirs < 0 ? nx : n_dirs); ++i) {
    ad::SeedIn<double, 1> in;
    in.x = x0.data();
    in.dir[0] = i;
    fn(in, yd.data());
    double g = 0.0;
    for (int j = 0; j < ny; ++j) g += ybar[j] * yd[j].d[0];
    const double h = 1e-6 * std::max(1.0, std::fabs(x0[i]));
    xp = x0; xm = x0;
    xp[i] += h; xm[i] -= h;
    ad::PlainIn<double> ip{xp.data()}, im{xm.data()};
    fn(ip, yp.data());
    fn(im, ym.data());
    double fd = 0.0;
    for (int j = 0; j < ny; ++j) fd += ybar[j] * (yp[j] - ym[j]) / (2.0 * h);
    double err = std::fabs(g - fd) / std::max(1.0, std::fabs(fd));
    worst = std::max(worst, err);
  }
  return worst;
}

void random_unit(Rng64& r, double* v, int n) {
  double l = 0.0;
  for (int i = 0; i < n; ++i) { v[i] = r.range(-1.0, 1.0); l += v[i] * v[i]; }
  l = std::sqrt(l);
  for (int i = 0; i < n; ++i) v[i] /= l;
}
void random_spd(Rng64& r, double* s /* xx xy xz yy yz zz */) {
  s[0] = r.range(0.5, 2.0); s[3] = r.range(0.5, 2.0); s[5] = r.range(0.5, 2.0);
  s[1] = r.range(-0.1, 0.1); s[2] = r.range(-0.1, 0.1); s[4] = r.range(-0.1, 0.1);
}
void random_constraint(Rng64& r, std::vector<double>& x) {
  using namespace ad;
  x.assign(kCV, 0.0);
  for (int i = 0; i < 12; ++i) x[i] = r.range(-1.0, 1.0);
  for (int i = 0; i < 3; ++i) { x[cvDpA + i] = r.range(-0.01, 0.01); x[cvDpB + i] = r.range(-0.01, 0.01); }
  for (int b = 0; b < 2; ++b) {
    double* q = &x[b ? cvDqB : cvDqA];
    q[0] = r.range(-0.02, 0.02); q[1] = r.range(-0.02, 0.02); q[2] = r.range(-0.02, 0.02);
    q[3] = std::sqrt(1.0 - q[0] * q[0] - q[1] * q[1] - q[2] * q[2]);
  }
  for (int q = 0; q < 4; ++q) x[cvLam + q] = r.range(0.05, 1.0);
  x[cvFr] = r.range(-0.1, 0.1); x[cvFr + 1] = r.range(-0.1, 0.1); x[cvTwist] = r.range(-0.01, 0.01);
  x[cvIma] = r.range(0.5, 2.0); x[cvImb] = r.range(0.5, 2.0);
  random_spd(r, &x[cvSa]); random_spd(r, &x[cvSb]);
  random_unit(r, &x[cvN], 3);
  for (int i = 0; i < 3; ++i) { x[cvCa + i] = r.range(-0.5, 0.5); x[cvCb + i] = r.range(-0.5, 0.5); }
  x[cvTwistMass] = r.range(0.3, 1.0);
  x[cvTm] = r.range(0.5, 1.0); x[cvTm + 1] = r.range(-0.1, 0.1); x[cvTm + 2] = x[cvTm + 1]; x[cvTm + 3] = r.range(0.5, 1.0);
  x[cvFriction] = r.range(0.3, 0.9);
  {
    // tangents from the normal, as prepare builds them
    ad::PlainIn<double> in{&x[cvN]};
    ad::TV3<double> n = ad::in3<double>(in, 0);
    ad::TV3<double> t1 = ad::perp(n), t2 = ad::cross(t1, n);
    x[cvT1] = t1.x; x[cvT1 + 1] = t1.y; x[cvT1 + 2] = t1.z;
    x[cvT2] = t2.x; x[cvT2 + 1] = t2.y; x[cvT2 + 2] = t2.z;
  }
  for (int q = 0; q < 4; ++q) {
    for (int f = 0; f < 6; ++f) x[cv_point(q, f)] = r.range(-0.5, 0.5);
    x[cv_point(q, 6)] = r.range(-0.02, 0.01);
    x[cv_point(q, 7)] = r.range(0.3, 1.0);
    x[cv_point(q, 8)] = r.range(0.05, 0.7);
  }
}

}  // namespace

extern "C" int ns_adjoint_selfcheck(int which, int seed, double* worst) {
  using namespace ad;
  if (!worst) return NS_ERR_INVALID;
  Rng64 r{0x9E3779B97F4A7C15ull ^ ((uint64_t)seed * 0xD1B54A32D192ED03ull + 1)};
  CParams cp;
  cp.pc = 4; cp.is_static = seed & 1;
  float h = 1.0f / 240.0f;
  cp.inv_h = 240.0f; cp.contact_speed = 3.0f;
  cp.contact_softness = make_soft(30.0f, 10.0f, h);
  cp.static_softness = make_soft(60.0f, 5.0f, h);
  std::vector<double> x;
  double e = -1.0;
  switch (which) {
    case 0:  // warm start
      random_constraint(r, x);
      e = vjp_fd_error(x, kWarmOut, [&](const auto& in, auto* y) { warm_fn(in, cp, y); }, r);
      break;
    case 1:  // push
      random_constraint(r, x);
      e = vjp_fd_error(x, kPushOut, [&](const auto& in, auto* y) { push_fn(in, cp, y); }, r);
      break;
    case 2:  // relax
      random_constraint(r, x);
      e = vjp_fd_error(x, kRelaxOut, [&](const auto& in, auto* y) { relax_fn(in, cp, y); }, r);
      break;
    case 3: {  // prepare
      x.assign(kPI, 0.0);
      random_unit(r, &x[piN], 3);
      for (int q = 0; q < 4; ++q) {
        for (int f = 0; f < 6; ++f) x[pi_point(q, f)] = r.range(-0.5, 0.5);
        x[pi_point(q, 6)] = r.range(-0.02, 0.015);
        x[pi_point(q, 7)] = r.range(0.0, 1.0);
      }
      for (int f = 0; f < 3; ++f) x[piFrictionImpulse + f] = r.range(-0.2, 0.2);
      x[piTwist] = r.range(-0.05, 0.05);
      x[piIma] = r.range(0.5, 2.0); x[piImb] = r.range(0.5, 2.0);
      random_spd(r, &x[piSa]); random_spd(r, &x[piSb]);
      x[piFriction] = r.range(0.3, 0.9);
      PParams pp = {4, 0, 1.0f};
      e = vjp_fd_error(x, kCVOwn, [&](const auto& in, auto* y) { prepare_fn(in, pp, y); }, r);
      break;
    }
    case 4: {  // integrate velocities
      x.assign(kIVIn, 0.0);
      for (int i = 0; i < 6; ++i) x[i] = r.range(-2.0, 2.0);
      x[6] = r.range(0.5, 2.0);
      for (int i = 0; i < 9; ++i) x[7 + i] = r.range(-0.2, 0.2) + ((i % 4) == 0 ? 1.0 : 0.0);
      for (int i = 16; i < 22; ++i) x[i] = r.range(-5.0, 5.0);
      random_unit(r, &x[22], 4);
      x[26] = r.range(-0.02, 0.02); x[27] = r.range(-0.02, 0.02); x[28] = r.range(-0.02, 0.02); x[29] = 1.0;
      {
        double s6[6];
        random_spd(r, s6);
        const int at[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int i = 0; i < 9; ++i) x[30 + i] = s6[at[i]];
      }
      BParams bp = {};
      bp.h = h; bp.lin_damp = 0.1f; bp.ang_damp = 0.05f; bp.grav_scale = 1.0f; bp.gravity = v3(0, -9.81f, 0);
      bp.flags = (seed & 1) ? kGyroscopic : 0u;  // odd seeds take the gyroscopic step
      e = vjp_fd_error(x, kIVOut, [&](const auto& in, auto* y) { iv_fn(in, bp, y); }, r);
      break;
    }
    case 5: {  // integrate positions
      x.assign(kIP, 0.0);
      for (int i = 0; i < 6; ++i) x[i] = r.range(-3.0, 3.0);
      for (int i = 6; i < 9; ++i) x[i] = r.range(-0.05, 0.05);
      random_unit(r, &x[9], 4);
      BParams bp = {};
      bp.h = h; bp.inv_dt = 60.0f; bp.max_linear_speed = (seed & 1) ? 1.0f : 400.0f;  // odd seeds cap the speed
      e = vjp_fd_error(x, kIP, [&](const auto& in, auto* y) { ip_fn(in, bp, y); }, r);
      break;
    }
    case 6: {  // finalize rotation
      x.assign(8, 0.0);
      random_unit(r, &x[0], 4);
      x[4] = r.range(-0.02, 0.02); x[5] = r.range(-0.02, 0.02); x[6] = r.range(-0.02, 0.02); x[7] = 1.0;
      e = vjp_fd_error(x, 4, [&](const auto& in, auto* y) { final_rot_fn(in, y); }, r);
      break;
    }
    case 7: {  // inverse world inertia
      x.assign(13, 0.0);
      random_unit(r, &x[0], 4);
      for (int i = 0; i < 9; ++i) x[4 + i] = r.range(-0.1, 0.1) + ((i % 4) == 0 ? 1.0 : 0.0);
      e = vjp_fd_error(x, 9, [&](const auto& in, auto* y) { inv_inertia_fn(in, y); }, r);
      break;
    }
    case 8: {  // recycled separations
      x.assign(kRI, 0.0);
      for (int i = 0; i < 6; ++i) x[i] = 0.0;
      for (int b = 0; b < 4; ++b) random_unit(r, &x[riQa + 4 * b], 4);
      random_unit(r, &x[riN], 3);
      for (int q = 0; q < 4; ++q) {
        for (int f = 0; f < 6; ++f) x[ri_point(q, f)] = r.range(-0.5, 0.5);
        x[ri_point(q, 6)] = r.range(-0.02, 0.02);
      }
      Pos ca = {r.range(-5, 5), r.range(0, 5), r.range(-5, 5)};
      Pos cb = {ca.x + r.range(-1, 1), ca.y + r.range(-1, 1), ca.z + r.range(-1, 1)};
      e = vjp_fd_error(x, 4, [&](const auto& in, auto* y) { recycle_fn(in, ca, cb, 4, y); }, r);
      break;
    }
    case 9: case 10: case 11: {  // box-box narrowphase replay: face contact (9), any axis (10), edges (11)
      Hull ha = make_box_hull(2.0f, 0.5f, 2.0f), hb = make_box_hull(0.5f, 0.4f, 0.3f);
      x.assign(kFI, 0.0);
      Pos ca = {0.0, 0.0, 0.0};
      double tilt = which == 9 ? 0.05 : 0.6;
      double qa[4], qb[4];
      qa[0] = r.range(-0.02, 0.02); qa[1] = r.range(-0.02, 0.02); qa[2] = r.range(-0.02, 0.02);
      qa[3] = std::sqrt(1 - qa[0] * qa[0] - qa[1] * qa[1] - qa[2] * qa[2]);
      qb[0] = r.range(-tilt, tilt); qb[1] = r.range(-tilt, tilt); qb[2] = r.range(-tilt, tilt);
      double l = std::sqrt(qb[0] * qb[0] + qb[1] * qb[1] + qb[2] * qb[2] + 1.0);
      for (int i = 0; i < 3; ++i) qb[i] /= l;
      qb[3] = 1.0 / l;
      for (int i = 0; i < 4; ++i) { x[fiQa + i] = qa[i]; x[fiQb + i] = qb[i]; }
      // place B just touching the top face of A
      Q qbf = {v3((float)qb[0], (float)qb[1], (float)qb[2]), (float)qb[3]};
      float low = 1e30f;
      for (int v = 0; v < 8; ++v) low = std::min(low, nsd::rotate(qbf, hb.points[v]).y);
      Pos cb = {r.range(-0.5, 0.5), 0.5 - (double)low - 0.005, r.range(-0.5, 0.5)};
      if (which == 11) {
        // B turned 45 degrees about x, then -25 degrees about z: its edge along the turned x
        // axis, sloping down towards +x, is placed across A's top edge (x = 2, y = 0.5) with a
        // gap of 3 mm along the edge pair's normal, so the separating axis is an edge pair.
        double th = -25.0 * M_PI / 180.0 * 0.5, ph = 45.0 * M_PI / 180.0 * 0.5;
        double qz[4] = {0, 0, std::sin(th), std::cos(th)}, qx[4] = {std::sin(ph), 0, 0, std::cos(ph)};
        qb[0] = qz[3] * qx[0] + qz[0] * qx[3] + qz[1] * qx[2] - qz[2] * qx[1];
        qb[1] = qz[3] * qx[1] - qz[0] * qx[2] + qz[1] * qx[3] + qz[2] * qx[0];
        qb[2] = qz[3] * qx[2] + qz[0] * qx[1] - qz[1] * qx[0] + qz[2] * qx[3];
        qb[3] = qz[3] * qx[3] - qz[0] * qx[0] - qz[1] * qx[1] - qz[2] * qx[2];
        qb[0] += r.range(-0.005, 0.005); qb[1] += r.range(-0.005, 0.005);
        double lq = std::sqrt(qb[0] * qb[0] + qb[1] * qb[1] + qb[2] * qb[2] + qb[3] * qb[3]);
        for (int i = 0; i < 4; ++i) { qb[i] /= lq; x[fiQb + i] = qb[i]; }
        qbf = Q{v3((float)qb[0], (float)qb[1], (float)qb[2]), (float)qb[3]};
        double a25 = 25.0 * M_PI / 180.0;
        V3 nrm = v3((float)std::sin(a25), (float)std::cos(a25), 0.0f);
        float best = -1e30f;
        for (int v = 0; v < 8; ++v) best = std::max(best, -nsd::dot(nsd::rotate(qbf, hb.points[v]), nrm));
        V3 mid = v3(0, 0, 0);
        int cnt = 0;
        for (int v = 0; v < 8; ++v) {
          V3 pv = nsd::rotate(qbf, hb.points[v]);
          if (-nsd::dot(pv, nrm) > best - 1e-3f) { mid = mid + pv; ++cnt; }
        }
        mid = (1.0f / (float)cnt) * mid;
        double gap = 0.003;
        cb = {2.0 + gap * nrm.x - mid.x, 0.5 + gap * nrm.y - mid.y, r.range(-0.5, 0.5) - mid.z};
      }
      WXf xa = {ca, Q{v3((float)qa[0], (float)qa[1], (float)qa[2]), (float)qa[3]}}, xbw = {cb, qbf};
      Xf b2a = inv_mul_wxf(xa, xbw);
      LocalManifold lm;
      SATCache cache;
      collide_hulls(&lm, ha, hb, b2a, &cache, nullptr);
      if (lm.point_count == 0) { e = 0.0; break; }
      NarrowCase nc = {cache.type, cache.index_a, cache.index_b, cache.hit};
      worst[1] = (double)cache.type;
      int pc = -1;
      {
        ad::PlainIn<double> in{x.data()};
        double y[kFO];
        pc = narrow_box_fn(in, ca, cb, ha, hb, nc, y);
      }
      if (pc < 1) return fail(nullptr, NS_ERR_INVALID, "narrowphase replay found no manifold");
      e = vjp_fd_error(x, 3 + 7 * pc,
                       [&](const auto& in, auto* y) { narrow_box_fn(in, ca, cb, ha, hb, nc, y); }, r);
      break;
    }
    case 12: case 13: case 14: {  // hand-written reverse sweeps against the dual numbers
      random_constraint(r, x);
      if (seed % 3 == 1) for (int q = 0; q < 4; ++q) x[cv_point(q, 6)] = r.range(0.0005, 0.01);  // speculative
      if (seed % 4 == 2) cp.pc = 1 + seed % 3;
      const int ny = which == 12 ? kWarmOut : which == 13 ? kPushOut : kRelaxOut;
      std::vector<double> yb(ny), hand(kCV, 0.0), crit(kCV, 0.0);
      for (double& v : yb) v = r.range(-1.0, 1.0);
      if (which == 12) { warm_vjp(x.data(), cp, yb.data(), hand.data()); warm_vjp<double, false>(x.data(), cp, yb.data(), crit.data()); }
      else if (which == 13) { push_vjp(x.data(), cp, yb.data(), hand.data()); push_vjp<double, false>(x.data(), cp, yb.data(), crit.data()); }
      else { relax_vjp(x.data(), cp, yb.data(), hand.data()); relax_vjp<double, false>(x.data(), cp, yb.data(), crit.data()); }
      std::vector<Dual<double, 1>> y(ny);
      e = 0.0;
      for (int i = 0; i < kCV; ++i) {
        SeedIn<double, 1> in;
        in.x = x.data();
        in.dir[0] = i;
        if (which == 12) warm_fn(in, cp, y.data());
        else if (which == 13) push_fn(in, cp, y.data());
        else relax_fn(in, cp, y.data());
        double g = 0.0;
        for (int j = 0; j < ny; ++j) g += yb[j] * y[j].d[0];
        e = std::max(e, std::fabs(g - hand[i]) / std::max(1.0, std::fabs(g)));
        // the critical-path variant keeps exactly the state and impulse entries
        double c = i < cvIma ? g : 0.0;
        e = std::max(e, std::fabs(c - crit[i]) / std::max(1.0, std::fabs(c)));
      }
      break;
    }
    case 15: case 16: {  // hand-written reverse of integrate positions / velocities
      const int nx = which == 15 ? kIP : kIVIn, ny = which == 15 ? kIP : kIVOut;
      x.assign(nx, 0.0);
      BParams bp = {};
      bp.h = h; bp.inv_dt = 60.0f; bp.lin_damp = 0.1f; bp.ang_damp = 0.05f; bp.grav_scale = 1.0f;
      bp.gravity = v3(0, -9.81f, 0);
      if (which == 15) {
        for (int i = 0; i < 6; ++i) x[i] = r.range(-3.0, 3.0);
        for (int i = 6; i < 9; ++i) x[i] = r.range(-0.05, 0.05);
        random_unit(r, &x[9], 4);
        bp.max_linear_speed = (seed & 1) ? 1.0f : 400.0f;
        if (seed % 3 == 2) { bp.flags = kLockAngX | kLockLinZ; for (int i = 3; i < 6; ++i) x[i] *= 300.0; }
      } else {
        for (int i = 0; i < 6; ++i) x[i] = r.range(-2.0, 2.0);
        x[6] = r.range(0.5, 2.0);
        for (int i = 0; i < 9; ++i) x[7 + i] = r.range(-0.2, 0.2) + ((i % 4) == 0 ? 1.0 : 0.0);
        for (int i = 16; i < 22; ++i) x[i] = r.range(-5.0, 5.0);
        random_unit(r, &x[22], 4);
        x[29] = 1.0;
      }
      std::vector<double> yb(ny), hand(nx, 0.0);
      for (double& v : yb) v = r.range(-1.0, 1.0);
      if (which == 15) ip_vjp(x.data(), bp, yb.data(), hand.data());
      else iv_vjp_plain(x.data(), bp, yb.data(), hand.data());
      std::vector<Dual<double, 1>> y(ny);
      e = 0.0;
      for (int i = 0; i < nx; ++i) {
        if (which == 16 && i >= 16) continue;  // force, torque (not returned); rotation, inertia (gyroscopic only)
        SeedIn<double, 1> in;
        in.x = x.data();
        in.dir[0] = i;
        if (which == 15) ip_fn(in, bp, y.data()); else iv_fn(in, bp, y.data());
        double g = 0.0;
        for (int j = 0; j < ny; ++j) g += yb[j] * y[j].d[0];
        e = std::max(e, std::fabs(g - hand[i]) / std::max(1.0, std::fabs(g)));
      }
      break;
    }
    case 17: {  // restitution (dual numbers against central differences)
      x.assign(kRV, 0.0);
      for (int i = 0; i < 12; ++i) x[i] = r.range(-1.0, 1.0);
      for (int i = 0; i < 3; ++i) { x[rvDpA + i] = r.range(-0.01, 0.01); x[rvDpB + i] = r.range(-0.01, 0.01); }
      for (int b = 0; b < 2; ++b) {
        double* q = &x[b ? rvDqB : rvDqA];
        q[0] = r.range(-0.02, 0.02); q[1] = r.range(-0.02, 0.02); q[2] = r.range(-0.02, 0.02);
        q[3] = std::sqrt(1.0 - q[0] * q[0] - q[1] * q[1] - q[2] * q[2]);
      }
      for (int q = 0; q < 4; ++q) {
        x[rvLam + q] = r.range(0.05, 1.0);
        x[rvTot + q] = r.range(0.5, 3.0);
        x[rvRest + q] = r.range(0.0, 0.4);
      }
      x[rvIma] = r.range(0.5, 2.0); x[rvImb] = r.range(0.5, 2.0);
      random_spd(r, &x[rvSa]); random_spd(r, &x[rvSb]);
      random_unit(r, &x[rvN], 3);
      x[rvE] = r.range(0.2, 0.9);
      for (int q = 0; q < 4; ++q) {
        for (int f = 0; f < 6; ++f) x[rv_point(q, f)] = r.range(-0.5, 0.5);
        x[rv_point(q, 6)] = r.range(-0.02, 0.01);
        x[rv_point(q, 7)] = r.range(0.3, 1.0);
        // even seeds: every point approaches faster than the threshold (the bounce is armed)
        x[rv_point(q, 8)] = (seed & 1) ? r.range(-4.0, 0.5) : r.range(-4.0, -1.2);
      }
      RParams rp = {1 + seed % 4, 240.0f, 1.0f};
      e = vjp_fd_error(x, kRestOut, [&](const auto& in, auto* y) { restitution_fn(in, rp, y); }, r);
      break;
    }
    case 18: {  // hand-written reverse of the relative normal velocity against the dual numbers
      x.assign(kRL, 0.0);
      for (int i = 0; i < kRL; ++i) x[i] = r.range(-1.0, 1.0);
      random_unit(r, &x[rlN], 3);
      const double yb = r.range(-1.0, 1.0);
      std::vector<double> hand(kRL, 0.0);
      relvel_vjp(x.data(), yb, hand.data());
      Dual<double, 1> y[1];
      e = 0.0;
      for (int i = 0; i < kRL; ++i) {
        SeedIn<double, 1> in;
        in.x = x.data();
        in.dir[0] = i;
        relvel_fn(in, y);
        double g = yb * y[0].d[0];
        e = std::max(e, std::fabs(g - hand[i]) / std::max(1.0, std::fabs(g)));
      }
      break;
    }
    case 19: case 20: case 21: case 22: case 23: {
      // manifolds of sphere-sphere (19), capsule-sphere (20), capsule-capsule (21), box-sphere
      // (22) and box-capsule (23) at random touching poses; worst[1] = the point count (19..21)
      // or the replayed path (22, 23)
      DShape A, B;
      std::memset(&A, 0, sizeof(A));
      std::memset(&B, 0, sizeof(B));
      Hull box = make_box_hull(0.6f, 0.4f, 0.5f);
      const Sphere sa = {v3(0, 0, 0), 0.5f}, sb = {v3(0, 0, 0), 0.3f};
      const Capsule capa = {v3(-0.5f, 0, 0), v3(0.5f, 0, 0), 0.3f}, capb = {v3(-0.4f, 0, 0), v3(0.4f, 0, 0), 0.2f};
      A.type = which == 19 ? kSphere : (which <= 21 ? kCapsule : kHull);
      B.type = (which == 19 || which == 20 || which == 22) ? kSphere : kCapsule;
      A.sphere = sa; A.capsule = capa;
      B.sphere = sb; B.capsule = capb;
      const Hull* ha = A.type == kHull ? &box : nullptr;
      // box-capsule cycles through its four paths by seed; the others take what comes
      const int want = which == 23 ? kRoundGjk + seed % 4 : (which == 22 ? (seed % 4 == 3 ? kRoundDeepFace : kRoundGjk) : -1);
      Pos ca = {0.0, 0.0, 0.0}, cb = {0.0, 0.0, 0.0};
      double qa[4], qb[4];
      RoundCase rc;
      rc.path = kRoundNone;
      for (int attempt = 0; attempt < 4000; ++attempt) {
        for (int i = 0; i < 3; ++i) qa[i] = r.range(-0.3, 0.3);
        qa[3] = 1.0;
        // near-parallel capsules on even seeds (the two-point branch)
        double tilt = (which == 21 && (seed & 1) == 0) ? 0.02 : 1.0;
        for (int i = 0; i < 3; ++i) qb[i] = r.range(-tilt, tilt);
        qb[3] = 1.0;
        if (which == 21 && (seed & 1) == 0)  // B turned like A plus a little
          for (int i = 0; i < 3; ++i) qb[i] += qa[i];
        double la = std::sqrt(qa[0] * qa[0] + qa[1] * qa[1] + qa[2] * qa[2] + qa[3] * qa[3]);
        double lb = std::sqrt(qb[0] * qb[0] + qb[1] * qb[1] + qb[2] * qb[2] + qb[3] * qb[3]);
        for (int i = 0; i < 4; ++i) { qa[i] /= la; qb[i] /= lb; }
        double reach = which == 19 ? 0.81 : (which == 20 ? 1.05 : 1.0);
        double dir[3];
        random_unit(r, dir, 3);
        double rad = which <= 21 ? r.range(0.3, reach) : r.range(0.0, 1.1);
        cb = {rad * dir[0], rad * dir[1], rad * dir[2]};
        Q fqa = {v3((float)qa[0], (float)qa[1], (float)qa[2]), (float)qa[3]};
        Q fqb = {v3((float)qb[0], (float)qb[1], (float)qb[2]), (float)qb[3]};
        WXf wa = {ca, fqa}, wb = {cb, fqb};
        rc = round_case(A, B, ha, inv_mul_wxf(wa, wb), SimplexCache());
        if (rc.path == kRoundNone || (want >= 0 && rc.path != want)) continue;
        std::vector<double> xt(kFI, 0.0);
        const float fa[4] = {fqa.v.x, fqa.v.y, fqa.v.z, fqa.s}, fb[4] = {fqb.v.x, fqb.v.y, fqb.v.z, fqb.s};
        for (int i = 0; i < 4; ++i) { xt[fiQa + i] = fa[i]; xt[fiQb + i] = fb[i]; }
        ad::PlainIn<double> in{xt.data()};
        double y[kFO];
        if (narrow_round_fn(in, ca, cb, A, B, ha, rc, y) < 1) { rc.path = kRoundNone; continue; }
        x = xt;
        break;
      }
      if (rc.path == kRoundNone) return fail(nullptr, NS_ERR_INVALID, "no touching pose found");
      int pc;
      {
        ad::PlainIn<double> in{x.data()};
        double y[kFO];
        pc = narrow_round_fn(in, ca, cb, A, B, ha, rc, y);
      }
      worst[1] = which <= 21 ? (double)pc : (double)rc.path;
      e = vjp_fd_error(x, 3 + 7 * pc, [&](const auto& in, auto* y) { narrow_round_fn(in, ca, cb, A, B, ha, rc, y); }, r);
      break;
    }
    case 24: case 25: case 26: {
      // revolute joint: the solve (24; even seeds push with bias, odd relax; the spring, motor
      // and limit rows by seed), its warm start (25) and its prepare (26)
      auto rand_quat = [&](double* q, double tilt) {
        for (int i = 0; i < 3; ++i) q[i] = r.range(-tilt, tilt);
        q[3] = 1.0;
        double l = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + 1.0);
        for (int i = 0; i < 4; ++i) q[i] /= l;
      };
      auto rand_m3 = [&](double* m) {  // symmetric positive definite, columns cx cy cz
        double s6[6];
        random_spd(r, s6);
        const int at[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int i = 0; i < 9; ++i) m[i] = s6[at[i]];
      };
      if (which == 26) {
        x.assign(kJPI, 0.0);
        rand_quat(&x[jpQa], 0.6);
        rand_quat(&x[jpQb], 0.6);
        x[jpIma] = r.range(0.5, 2.0); x[jpImb] = r.range(0.5, 2.0);
        rand_m3(&x[jpIA]); rand_m3(&x[jpIB]);
        Xf lfa = xf(v3((float)r.range(-0.5, 0.5), (float)r.range(-0.5, 0.5), (float)r.range(-0.5, 0.5)), qid());
        Xf lfb = xf(v3((float)r.range(-0.5, 0.5), (float)r.range(-0.5, 0.5), (float)r.range(-0.5, 0.5)),
                    quat(v3(0.0f, (float)std::sin(0.3), 0.0f), (float)std::cos(0.3)));
        Pos ca = {r.range(-2, 2), r.range(0, 3), r.range(-2, 2)}, cb = {r.range(-2, 2), r.range(0, 3), r.range(-2, 2)};
        e = vjp_fd_error(x, kJPO, [&](const auto& in, auto* y) {
          joint_prepare_fn(in, lfa, lfb, v3(0, 0, 0), v3(0, 0, 0), ca, cb, y);
        }, r);
        break;
      }
      x.assign(kJX, 0.0);
      for (int i = 0; i < 12; ++i) x[i] = r.range(-1.0, 1.0);
      for (int i = 0; i < 3; ++i) { x[jxDpA + i] = r.range(-0.01, 0.01); x[jxDpB + i] = r.range(-0.01, 0.01); }
      rand_quat(&x[jxDqA], 0.02);
      rand_quat(&x[jxDqB], 0.02);
      for (int i = 0; i < 3; ++i) x[jxLin + i] = r.range(-0.5, 0.5);
      x[jxPerp] = r.range(-0.2, 0.2); x[jxPerp + 1] = r.range(-0.2, 0.2);
      x[jxSpring] = r.range(-0.1, 0.1); x[jxMotor] = r.range(-0.05, 0.05);
      x[jxLower] = r.range(0.0, 0.2); x[jxUpper] = r.range(0.0, 0.2);
      for (int i = 0; i < 3; ++i) { x[jxPx + i] = r.range(-0.5, 0.5); x[jxPy + i] = r.range(-0.5, 0.5); }
      x[jxIma] = r.range(0.5, 2.0); x[jxImb] = r.range(0.5, 2.0);
      rand_m3(&x[jxIA]); rand_m3(&x[jxIB]);
      rand_quat(&x[jxFqA], 0.5);
      rand_quat(&x[jxFqB], 0.5);
      for (int i = 0; i < 3; ++i) { x[jxFpA + i] = r.range(-0.5, 0.5); x[jxFpB + i] = r.range(-0.5, 0.5); x[jxDc + i] = r.range(-1.0, 1.0); }
      {
        // the axis and axial mass as prepare makes them
        ad::PlainIn<double> in{x.data()};
        ad::TQ<double> fq = ad::in4<double>(in, jxFqA);
        ad::TV3<double> axis = ad::rotate(fq, ad::tv3<double>(0.0, 0.0, 1.0));
        ad::TM3<double> ia = ad::in_m3<double>(in, jxIA), ib = ad::in_m3<double>(in, jxIB);
        ad::TM3<double> sum = ad::tm3<double>(ia.cx + ib.cx, ia.cy + ib.cy, ia.cz + ib.cz);
        x[jxAxis] = axis.x; x[jxAxis + 1] = axis.y; x[jxAxis + 2] = axis.z;
        x[jxAxial] = 1.0 / ad::dot(axis, ad::mul_mv(sum, axis));
      }
      if (which == 25) {
        e = vjp_fd_error(x, 12, [&](const auto& in, auto* y) { joint_warm_fn(in, y); }, r);
        break;
      }
      JParams jp;
      jp.use_bias = (seed & 1) == 0;
      jp.fixed = false;
      jp.spring = seed % 3 == 0;
      jp.motor = seed % 3 == 1;
      jp.limit = seed % 3 != 1;
      jp.cs = make_soft(60.0f, 2.0f, h);
      jp.ss = make_soft(2.0f, 0.3f, h);
      jp.target = (float)r.range(-0.3, 0.3);
      jp.lower = (float)r.range(-0.6, 0.0);
      jp.upper = (float)r.range(0.0, 0.6);
      if (seed % 6 == 2) { jp.lower = 0.4f; jp.upper = 0.8f; }  // the angle below the lower limit
      jp.motor_speed = (float)r.range(-1.0, 1.0);
      jp.max_torque_h = (seed % 4 == 1) ? 1e-3f : 10.0f * h;  // odd motors clamp
      jp.inv_h = 1.0f / h;
      e = vjp_fd_error(x, kJSolveOut, [&](const auto& in, auto* y) { joint_solve_fn(in, jp, y); }, r);
      break;
    }
    default:
      return fail(nullptr, NS_ERR_INVALID, "unknown check %d", which);
  }
  *worst = e;
  return NS_OK;
}

// Host-side check of a batch narrowphase job before any GPU work: the kernel indexes local
// arrays with the caller's cache fields (a face plane per SAT face index, a half-edge pair per
// edge index, simplex vertices per cached index), so every one must lie inside its shape.
// Pairs follow the reference's primary-type order (contact_creation.rs:88-96).
static int shape_vertex_count(int type) { return type == kHull ? kHullVertexCount : type == kCapsule ? 2 : 1; }

static int validate_pair_jobs(const ns_pair_job* jobs, int count, const char* who) {
  for (int i = 0; i < count; ++i) {
    const ns_pair_job& j = jobs[i];
    bool pair_ok = (j.type_a == kSphere && j.type_b == kSphere) ||
                   (j.type_a == kCapsule && (j.type_b == kSphere || j.type_b == kCapsule)) ||
                   (j.type_a == kHull && (j.type_b == kSphere || j.type_b == kCapsule || j.type_b == kHull));
    if (!pair_ok)
      return fail(nullptr, NS_ERR_INVALID, "%s: job %d pairs shape types (%d, %d), not a primary-first pair of "
                  "0 capsule, 3 box hull, 5 sphere", who, i, j.type_a, j.type_b);
    if (j.sat_type < kInvalidAxis || j.sat_type > kManualEdgePairAxis || j.sat_hit < 0 || j.sat_hit > 1)
      return fail(nullptr, NS_ERR_INVALID, "%s: job %d has SAT cache type %d / hit %d", who, i, j.sat_type, j.sat_hit);
    bool face_a = j.sat_type == kFaceAxisA, face_b = j.sat_type == kFaceAxisB, edge = j.sat_type == kEdgePairAxis;
    // face caches index a face plane; edge caches index the first half-edge of a twin pair
    if ((face_a && (j.sat_index_a < 0 || j.sat_index_a >= kHullFaceCount)) ||
        (face_b && (j.sat_index_b < 0 || j.sat_index_b >= kHullFaceCount)) ||
        (edge && (j.sat_index_a < 0 || j.sat_index_a >= kHullEdgeCount - 1 || (j.sat_index_a & 1) ||
                  j.sat_index_b < 0 || j.sat_index_b >= kHullEdgeCount - 1 || (j.sat_index_b & 1))) ||
        j.sat_index_a < 0 || j.sat_index_a > 255 || j.sat_index_b < 0 || j.sat_index_b > 255)
      return fail(nullptr, NS_ERR_INVALID, "%s: job %d has SAT cache indices (%d, %d) outside the box for type %d",
                  who, i, j.sat_index_a, j.sat_index_b, j.sat_type);
    if (j.simplex_count < 0 || j.simplex_count > 3)
      return fail(nullptr, NS_ERR_INVALID, "%s: job %d has simplex cache count %d (0..3)", who, i, j.simplex_count);
    int na = shape_vertex_count(j.type_a), nb = shape_vertex_count(j.type_b);
    for (int k = 0; k < 4; ++k) {
      bool used = k < j.simplex_count;
      int ia = j.simplex_ia[k], ib = j.simplex_ib[k];
      if (ia < 0 || ia > 255 || ib < 0 || ib > 255 || (used && (ia >= na || ib >= nb)))
        return fail(nullptr, NS_ERR_INVALID, "%s: job %d simplex vertex %d indexes (%d, %d) of shapes with %d and %d "
                    "vertices", who, i, k, ia, ib, na, nb);
    }
  }
  return NS_OK;
}

// Fixed device scratch of ns_collide_pairs_noalloc: the device copies of one call's jobs
// (first kNoAllocPairs * sizeof(PairJob) bytes) and results (the rest). Every GPU that loads
// the library holds it until the process exits; all calls on a device share it.
constexpr int kNoAllocPairs = 4096;
constexpr size_t kNoAllocJobBytes = (size_t)kNoAllocPairs * sizeof(nsd::PairJob);
static_assert(kNoAllocJobBytes % 256 == 0, "results must start 256-byte aligned");
static __device__ __align__(256) unsigned char g_pair_scratch[kNoAllocJobBytes + (size_t)kNoAllocPairs * sizeof(nsd::PairResult)];

// In host code g_pair_scratch is only a host-side stand-in, never a device address: each call
// asks the runtime for the address on the current device. The stack set-up is done once per
// device (under the mutex).
constexpr int kNoAllocMaxDevices = 64;
static bool g_pair_stack_ready[kNoAllocMaxDevices];
static std::mutex g_pair_scratch_mutex;

extern "C" {

void ns_default_world_def(ns_world_def* d) {
  memset(d, 0, sizeof(*d));
  d->gravity[1] = -10.0f;
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

ns_world* ns_world_create(const ns_world_def* def) {
  if (!def) { g_create_error = "null world def"; return nullptr; }
  if (def->enable_sleep) { g_create_error = "enable_sleep must be 0: sleeping islands are not supported"; return nullptr; }
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    g_create_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
    return nullptr;
  }
  if (def->device < 0 || def->device >= count) { g_create_error = "invalid device ordinal"; return nullptr; }
  ns_world* w = new ns_world();
  w->def = *def;
  return w;
}

void ns_world_destroy(ns_world* w) {
  if (!w) return;
  if (w->uploaded) {
    cudaSetDevice(w->def.device);
    cudaStreamSynchronize(w->stream);
    if (w->graph_exec) cudaGraphExecDestroy(w->graph_exec);
    if (w->graph) cudaGraphDestroy(w->graph);
    free_tape(w);
    for (char* p : w->ckpt_pool) scratch_free(w, p);
    scratch_free(w, w->tapes_buf);
    scratch_free(w, w->adj_buf);
    scratch_free(w, (char*)w->snap_ops);
    cudaStreamSynchronize(w->stream);
    for (void* p : w->allocations) cudaFree(p);
    if (w->host_ctl) cudaFreeHost(w->host_ctl);
    if (w->host_in) cudaFreeHost(w->host_in);
    if (w->in_done) cudaEventDestroy(w->in_done);
    for (int i = 0; i < 6; ++i) if (w->ev[i]) cudaEventDestroy(w->ev[i]);
    cudaStreamDestroy(w->stream);
  }
  delete w;
}

const char* ns_last_error(const ns_world* w) { return w ? w->err.c_str() : g_create_error.c_str(); }

int ns_create_body(ns_world* w, const ns_body_def* d) {
  if (!w || !d) return -1;
  if (w->uploaded) { w->err = "scene changes after the first step are not supported"; return -1; }
  if (d->type != NS_STATIC_BODY && d->type != NS_KINEMATIC_BODY && d->type != NS_DYNAMIC_BODY) {
    w->err = "body type must be NS_STATIC_BODY, NS_KINEMATIC_BODY or NS_DYNAMIC_BODY";
    return -1;
  }
  int id = (int)w->bodies.size();
  HostBody b;
  b.type = d->type;
  b.set = d->type == NS_STATIC_BODY ? 0 : 2;
  DSim s;
  memset(&s, 0, sizeof(s));
  s.px = d->position[0]; s.py = d->position[1]; s.pz = d->position[2];
  s.q = quat(v3(d->rotation[0], d->rotation[1], d->rotation[2]), d->rotation[3]);
  s.cx = s.px; s.cy = s.py; s.cz = s.pz;
  s.min_extent = huge_value();
  s.linear_damping = d->linear_damping;
  s.angular_damping = d->angular_damping;
  s.gravity_scale = d->gravity_scale;
  s.safety_factor = 0.5f;
  s.body_id = id;
  s.flags = 0;
  if (d->type == NS_DYNAMIC_BODY) s.flags |= kDynamicFlag;
  if (d->enable_sleep) s.flags |= kEnableSleepFlag;
  if (d->is_bullet) s.flags |= kIsBullet;  // world_runtime.rs:1570
  s.flags |= kEnableRecycling;
  b.flags = s.flags;
  if (d->is_bullet && d->type == NS_DYNAMIC_BODY) ++w->n_bullets;
  if (b.set == 2) {
    b.local = (int)w->asims.size();
    w->asims.push_back(s);
    DState st;
    memset(&st, 0, sizeof(st));
    st.v = v3(d->linear_velocity[0], d->linear_velocity[1], d->linear_velocity[2]);
    st.w = v3(d->angular_velocity[0], d->angular_velocity[1], d->angular_velocity[2]);
    st.dq = qid();
    st.flags = s.flags;
    w->states.push_back(st);
  } else {
    b.local = (int)w->ssims.size();
    w->ssims.push_back(s);
  }
  b.world = (int)w->sub_body_begin.size() - 1;
  w->bodies.push_back(b);
  w->body_mask.push_back(0u);
  return id;
}

int ns_create_box_shape(ns_world* w, int body, const ns_shape_def* def, float hx, float hy, float hz) {
  if (!w) return -1;
  HostShape hs;
  memset(&hs.d, 0, sizeof(hs.d));
  hs.d.type = kHull;
  hs.hull = make_box_hull(hx, hy, hz);
  return create_shape(w, body, def, hs);
}

int ns_create_sphere_shape(ns_world* w, int body, const ns_shape_def* def, const float c[3], float r) {
  if (!w || !c) return -1;
  HostShape hs;
  memset(&hs.d, 0, sizeof(hs.d));
  memset(&hs.hull, 0, sizeof(hs.hull));
  hs.d.type = kSphere;
  hs.d.sphere.center = v3(c[0], c[1], c[2]);
  hs.d.sphere.radius = r;
  return create_shape(w, body, def, hs);
}

int ns_create_capsule_shape(ns_world* w, int body, const ns_shape_def* def, const float c1[3],
                            const float c2[3], float r) {
  if (!w || !c1 || !c2) return -1;
  HostShape hs;
  memset(&hs.d, 0, sizeof(hs.d));
  memset(&hs.hull, 0, sizeof(hs.hull));
  V3 a = v3(c1[0], c1[1], c1[2]), b = v3(c2[0], c2[1], c2[2]);
  if (distance(a, b) < min_capsule_length()) {  // shape_creation.rs:522
    hs.d.type = kSphere;
    hs.d.sphere.center = 0.5f * (a + b);
    hs.d.sphere.radius = r;
  } else {
    hs.d.type = kCapsule;
    hs.d.capsule.c1 = a; hs.d.capsule.c2 = b; hs.d.capsule.radius = r;
  }
  return create_shape(w, body, def, hs);
}

int ns_create_revolute_joint(ns_world* w, int body_a, int body_b, const float fa[7], const float fb[7],
                             int enable_limit, float lower, float upper, int enable_spring, float hertz,
                             float damping_ratio, float max_motor_torque, int collide_connected) {
  if (!w || !fa || !fb) return -1;
  ns_revolute_joint_def d;
  ns_default_revolute_joint_def(&d);
  d.body_a = body_a; d.body_b = body_b;
  memcpy(d.local_frame_a, fa, sizeof(d.local_frame_a));
  memcpy(d.local_frame_b, fb, sizeof(d.local_frame_b));
  d.constraint_hertz = w->def.joint_hertz;
  d.constraint_damping_ratio = w->def.joint_damping_ratio;
  d.collide_connected = collide_connected;
  d.enable_spring = enable_spring; d.hertz = hertz; d.damping_ratio = damping_ratio;
  d.enable_limit = enable_limit; d.lower_angle = lower; d.upper_angle = upper;
  // a motor with zero speed (a drag torque) whenever a torque is given
  d.enable_motor = max_motor_torque > 0.0f; d.max_motor_torque = max_motor_torque; d.motor_speed = 0.0f;
  return ns_create_revolute_joint_def(w, &d);
}

void ns_default_revolute_joint_def(ns_revolute_joint_def* d) {
  memset(d, 0, sizeof(*d));
  d->body_a = d->body_b = -1;
  d->local_frame_a[6] = 1.0f;
  d->local_frame_b[6] = 1.0f;
  d->constraint_hertz = 60.0f;          // joint_defs.rs:54-55
  d->constraint_damping_ratio = 2.0f;
}

static int add_joint(ns_world* w, DJoint j, int collide_connected);

// revolute_joint.rs:161 create_revolute_joint with the whole RevoluteJointDef
int ns_create_revolute_joint_def(ns_world* w, const ns_revolute_joint_def* def) {
  if (!w || !def) return -1;
  DJoint j;
  memset(&j, 0, sizeof(j));
  j.type = kJointRevolute;
  j.body_a = def->body_a; j.body_b = def->body_b;
  const float* fa = def->local_frame_a;
  const float* fb = def->local_frame_b;
  j.local_frame_a = xf(v3(fa[0], fa[1], fa[2]), quat(v3(fa[3], fa[4], fa[5]), fa[6]));
  j.local_frame_b = xf(v3(fb[0], fb[1], fb[2]), quat(v3(fb[3], fb[4], fb[5]), fb[6]));
  j.constraint_hertz = def->constraint_hertz;
  j.constraint_damping_ratio = def->constraint_damping_ratio;
  j.enable_limit = def->enable_limit != 0; j.lower_angle = def->lower_angle; j.upper_angle = def->upper_angle;
  j.enable_spring = def->enable_spring != 0; j.hertz = def->hertz; j.damping_ratio = def->damping_ratio;
  j.target_angle = def->target_angle;
  j.max_motor_torque = def->max_motor_torque; j.enable_motor = def->enable_motor != 0;
  j.motor_speed = def->motor_speed;
  return add_joint(w, j, def->collide_connected);
}

void ns_default_spherical_joint_def(ns_spherical_joint_def* d) {
  memset(d, 0, sizeof(*d));
  d->body_a = d->body_b = -1;
  d->local_frame_a[6] = 1.0f;
  d->local_frame_b[6] = 1.0f;
  d->constraint_hertz = 60.0f;          // joint_defs.rs:54-55
  d->constraint_damping_ratio = 2.0f;
  d->target_rotation[3] = 1.0f;         // joint_defs.rs:185-203
}

// spherical_joint.rs:119 create_spherical_joint
int ns_create_spherical_joint_def(ns_world* w, const ns_spherical_joint_def* def) {
  if (!w || !def) return -1;
  DJoint j;
  memset(&j, 0, sizeof(j));
  j.type = kJointSpherical;
  j.body_a = def->body_a; j.body_b = def->body_b;
  const float* fa = def->local_frame_a;
  const float* fb = def->local_frame_b;
  j.local_frame_a = xf(v3(fa[0], fa[1], fa[2]), quat(v3(fa[3], fa[4], fa[5]), fa[6]));
  j.local_frame_b = xf(v3(fb[0], fb[1], fb[2]), quat(v3(fb[3], fb[4], fb[5]), fb[6]));
  j.constraint_hertz = def->constraint_hertz;
  j.constraint_damping_ratio = def->constraint_damping_ratio;
  j.enable_spring = def->enable_spring != 0; j.hertz = def->hertz; j.damping_ratio = def->damping_ratio;
  const float* t = def->target_rotation;
  j.target_rotation = quat(v3(t[0], t[1], t[2]), t[3]);
  j.enable_cone_limit = def->enable_cone_limit != 0; j.cone_angle = def->cone_angle;
  j.enable_twist_limit = def->enable_twist_limit != 0;
  j.lower_twist_angle = def->lower_twist_angle; j.upper_twist_angle = def->upper_twist_angle;
  j.enable_motor = def->enable_motor != 0; j.max_motor_torque = def->max_motor_torque;
  j.motor_velocity = v3(def->motor_velocity[0], def->motor_velocity[1], def->motor_velocity[2]);
  return add_joint(w, j, def->collide_connected);
}

// joint.rs:164 create_joint: checks, the graph colour (constraint_graph.rs:256) and the bodies'
// joint bookkeeping, for any joint type
static int add_joint(ns_world* w, DJoint j, int collide_connected) {
  const int body_a = j.body_a, body_b = j.body_b;
  if (w->uploaded) { w->err = "scene changes after the first step are not supported"; return -1; }
  int nb = (int)w->bodies.size();
  if (body_a < 0 || body_b < 0 || body_a >= nb || body_b >= nb || body_a == body_b) { w->err = "invalid joint bodies"; return -1; }
  HostBody& ba = w->bodies[body_a];
  HostBody& bb = w->bodies[body_b];
  if (ba.world != bb.world || ba.world != (int)w->sub_body_begin.size() - 1) {
    w->err = "joint bodies must belong to the newest sub-world";
    return -1;
  }
  j.world = ba.world;
  j.enc_a = encode(ba); j.enc_b = encode(bb);
  j.constraint_softness.bias_rate = 0.0f; j.constraint_softness.mass_scale = 1.0f; j.constraint_softness.impulse_scale = 0.0f;
  // constraint_graph.rs:256 assign_joint_color
  uint32_t& ma = w->body_mask[body_a];
  uint32_t& mb = w->body_mask[body_b];
  int color = kOverflowIndex;
  if (ba.type != NS_DYNAMIC_BODY && bb.type != NS_DYNAMIC_BODY) {
    color = -1;  // joint.rs:251-262: not attached to a dynamic body, kept in the static set, never solved
  } else if (ba.type == NS_DYNAMIC_BODY && bb.type == NS_DYNAMIC_BODY) {
    uint32_t avail = ~(ma | mb) & ((1u << kDynamicColorCount) - 1u);
    if (avail) { color = __builtin_ctz(avail); ma |= 1u << color; mb |= 1u << color; }
  } else {
    uint32_t& m = ba.type == NS_DYNAMIC_BODY ? ma : mb;
    uint32_t avail = ~m & (((1u << kOverflowIndex) - 1u) & ~1u);
    if (avail) { color = 31 - __builtin_clz(avail); m |= 1u << color; }
  }
  j.color = color;
  ba.joint_count++;
  bb.joint_count++;
  if (!collide_connected) {
    if ((int)w->joint_partners.size() < nb) w->joint_partners.resize(nb);
    w->joint_partners[body_a].push_back(body_b);
    w->joint_partners[body_b].push_back(body_a);
  }
  w->joints.push_back(j);
  return (int)w->joints.size() - 1;
}

static int world_step(ns_world* w, float dt, int substeps);

int ns_world_step(ns_world* w, float dt, int substeps) {
  if (!w) return NS_ERR_INVALID;
  bool rec = w->tape && w->tape->recording;
  if (rec && !(dt > 0.0f)) return fail(w, NS_ERR_UNSUPPORTED, "a recording tape needs dt > 0");
  int st = world_step(w, dt, substeps);
  if (st || !rec) return st;
  return tape_after_step(w, dt, substeps < 1 ? 1 : substeps);
}

static int world_step(ns_world* w, float dt, int substeps) {
  if (!(dt >= 0.0f)) return fail(w, NS_ERR_INVALID, "dt must be >= 0");
  if (!w->uploaded) {
    int st = upload_world(w);
    if (st) return st;
  }
  NS_CUDA(w, cudaSetDevice(w->def.device));
  if (w->asims.empty()) return NS_OK;
  if (dt == 0.0f) {
    // solver_integration.rs:807 with a zero time step: pairs are updated, nothing else runs
    int st = enqueue_pair_update(w);
    if (st) return st;
    NS_CUDA(w, cudaGetLastError());
    w->kernel_launches += w->pair_kernels;
    return NS_OK;
  }
  if (w->eager) {
    int st = enqueue_step(w, dt, substeps);
    if (st) return st;
    w->steps_done++;
    w->last_substeps = substeps;
    w->kernel_launches += w->step_kernels;
    return NS_OK;
  }
  if (!w->graph_exec || w->graph_dt != dt || w->graph_substeps != substeps) {
    if (w->graph_exec) { cudaGraphExecDestroy(w->graph_exec); w->graph_exec = nullptr; }
    if (w->graph) { cudaGraphDestroy(w->graph); w->graph = nullptr; }
    NS_CUDA(w, cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
    int st = enqueue_step(w, dt, substeps);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(w->stream, &g);
    cudaGetLastError();
    bool ok = st == NS_OK && e == cudaSuccess && g != nullptr;
    if (ok && cudaGraphInstantiate(&w->graph_exec, g, 0) != cudaSuccess) {
      cudaGetLastError();
      w->graph_exec = nullptr;
      ok = false;
    }
    if (!ok) {
      // The step runs without a graph when capture is refused (for example a driver that
      // does not capture cooperative launches); results are identical, launches cost more.
      if (g) cudaGraphDestroy(g);
      w->eager = true;
      w->err = "graph capture unavailable; stepping without a CUDA graph";
      int st2 = enqueue_step(w, dt, substeps);
      if (st2) return st2;
      w->steps_done++;
      w->last_substeps = substeps;
      w->kernel_launches += w->step_kernels;
      return NS_OK;
    }
    w->graph = g;
    w->graph_dt = dt;
    w->graph_substeps = substeps;
  }
  NS_CUDA(w, cudaGraphLaunch(w->graph_exec, w->stream));
  w->steps_done++;
  w->last_substeps = substeps;
  w->kernel_launches += w->step_kernels;
  return NS_OK;
}

int ns_world_synchronize(ns_world* w) {
  if (!w) return NS_ERR_INVALID;
  if (!w->uploaded) return NS_OK;
  Control c;
  int st = read_control(w, &c);
  if (st) return st;
  return control_status(w, c);
}

int ns_world_body_count(const ns_world* w) { return w ? (int)w->bodies.size() : -1; }

int ns_world_apply_forces(ns_world* w, const float* force, const float* torque) {
  if (w && w->tape && w->tape->recording)
    return fail(w, NS_ERR_UNSUPPORTED, "forces cannot be applied while a tape records");
  if (!w) return NS_ERR_INVALID;
  int nb = (int)w->bodies.size();
  if (nb == 0 || (!force && !torque)) return NS_OK;
  if (!w->uploaded) {
    for (int i = 0; i < nb; ++i) {
      const HostBody& b = w->bodies[i];
      if (b.set != 2) continue;
      DSim& s = w->asims[b.local];
      if (force) s.force = s.force + v3(force[3 * i], force[3 * i + 1], force[3 * i + 2]);
      if (torque) s.torque = s.torque + v3(torque[3 * i], torque[3 * i + 1], torque[3 * i + 2]);
    }
    return NS_OK;
  }
  NS_CUDA(w, cudaSetDevice(w->def.device));
  // the pinned staging buffer is reused: wait for the previous upload from it to finish
  NS_CUDA(w, cudaEventSynchronize(w->in_done));
  size_t n3 = 3 * (size_t)nb;
  if (force) memcpy(w->host_in, force, sizeof(float) * n3);
  if (torque) memcpy(w->host_in + n3, torque, sizeof(float) * n3);
  size_t off = force ? 0 : n3, len = (force && torque) ? 2 * n3 : n3;
  NS_CUDA(w, cudaMemcpyAsync(w->in_stage + off, w->host_in + off, sizeof(float) * len, cudaMemcpyHostToDevice,
                             w->stream));
  NS_CUDA(w, cudaEventRecord(w->in_done, w->stream));
  k_apply_forces<<<std::min(4 * w->sm_count, (nb + 255) / 256), 256, 0, w->stream>>>(
      w->dw, w->body_loc, nb, force ? w->in_stage : nullptr, torque ? w->in_stage + n3 : nullptr);
  w->kernel_launches++;
  NS_CUDA(w, cudaGetLastError());
  return NS_OK;
}

int ns_world_get_bodies(ns_world* w, double* pos, float* rot, float* lin, float* ang) {
  if (!w) return NS_ERR_INVALID;
  int nb = (int)w->bodies.size();
  if (w->uploaded && nb > 0) {
    // one gather kernel packs the state, then one copy per requested array and one sync
    NS_CUDA(w, cudaSetDevice(w->def.device));
    double* dpos = (double*)w->out_stage;
    float* drot = (float*)(dpos + 3 * (size_t)nb);
    float* dlin = drot + 4 * (size_t)nb;
    float* dang = dlin + 3 * (size_t)nb;
    k_gather_bodies<<<std::min(4 * w->sm_count, (nb + 255) / 256), 256, 0, w->stream>>>(w->dw, w->body_loc, nb, dpos,
                                                                                        drot, dlin, dang);
    w->kernel_launches++;
    NS_CUDA(w, cudaGetLastError());
    if (pos) NS_CUDA(w, cudaMemcpyAsync(pos, dpos, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost, w->stream));
    if (rot) NS_CUDA(w, cudaMemcpyAsync(rot, drot, sizeof(float) * 4 * nb, cudaMemcpyDeviceToHost, w->stream));
    if (lin) NS_CUDA(w, cudaMemcpyAsync(lin, dlin, sizeof(float) * 3 * nb, cudaMemcpyDeviceToHost, w->stream));
    if (ang) NS_CUDA(w, cudaMemcpyAsync(ang, dang, sizeof(float) * 3 * nb, cudaMemcpyDeviceToHost, w->stream));
    NS_CUDA(w, cudaMemcpyAsync(w->host_ctl, w->dw.ctl, sizeof(Control), cudaMemcpyDeviceToHost, w->stream));
    NS_CUDA(w, cudaStreamSynchronize(w->stream));
    return control_status(w, *w->host_ctl);
  }
  for (int i = 0; i < nb; ++i) {
    const HostBody& b = w->bodies[i];
    const DSim& s = b.set == 2 ? w->asims[b.local] : w->ssims[b.local];
    if (pos) { pos[3 * i] = s.px; pos[3 * i + 1] = s.py; pos[3 * i + 2] = s.pz; }
    if (rot) { rot[4 * i] = s.q.v.x; rot[4 * i + 1] = s.q.v.y; rot[4 * i + 2] = s.q.v.z; rot[4 * i + 3] = s.q.s; }
    V3 v = v3(0, 0, 0), wv = v3(0, 0, 0);
    if (b.set == 2) { v = w->states[b.local].v; wv = w->states[b.local].w; }
    if (lin) { lin[3 * i] = v.x; lin[3 * i + 1] = v.y; lin[3 * i + 2] = v.z; }
    if (ang) { ang[3 * i] = wv.x; ang[3 * i + 1] = wv.y; ang[3 * i + 2] = wv.z; }
  }
  return NS_OK;
}

// body_queries.rs:432 world_state_hash over the bodies [b0, b1) of host arrays
static uint64_t state_hash_range(const ns_world* w, const double* pos, const float* rot, const float* lin,
                                 const float* ang, size_t b0, size_t b1) {
  const uint64_t prime = 1099511628211ull;
  uint64_t h = 14695981039346656037ull;
  auto mixf = [&](float f) { uint32_t b; memcpy(&b, &f, 4); h = (h ^ (uint64_t)b) * prime; };
  auto mixd = [&](double d) { uint64_t b; memcpy(&b, &d, 8); h = (h ^ b) * prime; };
  for (size_t i = b0; i < b1; ++i) {
    mixd(pos[3 * i]); mixd(pos[3 * i + 1]); mixd(pos[3 * i + 2]);
    mixf(rot[4 * i]); mixf(rot[4 * i + 1]); mixf(rot[4 * i + 2]); mixf(rot[4 * i + 3]);
    if (w->bodies[i].set == 2) {
      mixf(lin[3 * i]); mixf(lin[3 * i + 1]); mixf(lin[3 * i + 2]);
      mixf(ang[3 * i]); mixf(ang[3 * i + 1]); mixf(ang[3 * i + 2]);
    }
  }
  return h;
}

int ns_world_state_hash(ns_world* w, uint64_t* out) {
  if (!w || !out) return NS_ERR_INVALID;
  size_t n = w->bodies.size();
  std::vector<double> pos(3 * n);
  std::vector<float> rot(4 * n), lin(3 * n), ang(3 * n);
  int st = ns_world_get_bodies(w, pos.data(), rot.data(), lin.data(), ang.data());
  if (st) return st;
  *out = state_hash_range(w, pos.data(), rot.data(), lin.data(), ang.data(), 0, n);
  return NS_OK;
}

int ns_world_begin_subworld(ns_world* w) {
  if (!w) return -1;
  if (w->uploaded) { w->err = "scene changes after the first step are not supported"; return -1; }
  w->sub_body_begin.push_back((int)w->bodies.size());
  w->sub_shape_begin.push_back((int)w->shapes.size());
  return (int)w->sub_body_begin.size() - 1;
}

int ns_world_subworld_count(const ns_world* w) { return w ? (int)w->sub_body_begin.size() : -1; }

int ns_world_subworld_bodies(const ns_world* w, int* first_body) {
  if (!w || !first_body) return NS_ERR_INVALID;
  for (size_t k = 0; k < w->sub_body_begin.size(); ++k) first_body[k] = w->sub_body_begin[k];
  first_body[w->sub_body_begin.size()] = (int)w->bodies.size();
  return NS_OK;
}

int ns_world_subworld_hashes(ns_world* w, uint64_t* out) {
  if (!w || !out) return NS_ERR_INVALID;
  size_t n = w->bodies.size();
  std::vector<double> pos(3 * n);
  std::vector<float> rot(4 * n), lin(3 * n), ang(3 * n);
  int st = ns_world_get_bodies(w, pos.data(), rot.data(), lin.data(), ang.data());
  if (st) return st;
  size_t nw = w->sub_body_begin.size();
  for (size_t k = 0; k < nw; ++k) {
    size_t b1 = k + 1 < nw ? (size_t)w->sub_body_begin[k + 1] : n;
    out[k] = state_hash_range(w, pos.data(), rot.data(), lin.data(), ang.data(), (size_t)w->sub_body_begin[k], b1);
  }
  return NS_OK;
}

int ns_world_contact_capacity(ns_world* w) {
  if (!w) return -1;
  if (!w->uploaded) return 0;
  return w->dw.cap;
}

int ns_world_get_contacts(ns_world* w, int32_t* ints, uint32_t* feats, float* fl, int capacity) {
  if (!w || !ints || !feats || !fl) return -1;
  if (!w->uploaded) return 0;
  if (ns_world_synchronize(w)) return -1;
  std::vector<DContact> cs(w->dw.cap);
  if (cudaMemcpy(cs.data(), w->dw.contacts, sizeof(DContact) * cs.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  int n = 0;
  for (size_t i = 0; i < cs.size() && n < capacity; ++i) {
    const DContact& c = cs[i];
    if (!c.alive) continue;
    int32_t* I = ints + 8 * n;
    uint32_t* F = feats + 4 * n;
    float* D = fl + 24 * n;
    int pc = c.manifold_count > 0 ? c.manifold.point_count : 0;
    I[0] = (int32_t)i; I[1] = c.shape_a; I[2] = c.shape_b; I[3] = c.color; I[4] = pc;
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

int ns_world_counters(ns_world* w, int32_t* out) {
  if (!w || !out) return NS_ERR_INVALID;
  for (int i = 0; i < 32; ++i) out[i] = 0;
  if (!w->uploaded) return NS_OK;
  Control c;
  int st = read_control(w, &c);
  if (st) return st;
  std::vector<DContact> cs(w->dw.cap);
  NS_CUDA(w, cudaMemcpy(cs.data(), w->dw.contacts, sizeof(DContact) * cs.size(), cudaMemcpyDeviceToHost));
  for (const DContact& ct : cs) {
    if (!ct.alive) continue;
    out[0]++;
    if (ct.flags & cTouching) out[1]++;
  }
  for (int k = 0; k < kOverflowIndex; ++k) out[2 + k] = c.color_count[k] + 0;
  for (int k = 0; k < kOverflowIndex; ++k) out[2 + k] = 0;
  for (const DContact& ct : cs)
    if (ct.alive && (ct.flags & cTouching) && ct.color >= 0) out[2 + ct.color]++;
  out[26] = c.fast_flags;
  out[27] = 0;
  out[28] = c.recycled;
  out[29] = c.overflow_count;
  out[30] = c.new_pairs;
  out[31] = c.changed_count;
  return NS_OK;
}

int ns_world_phase_times(ns_world* w, float* ms) {
  if (!w || !ms) return NS_ERR_INVALID;
  if (!w->uploaded || w->steps_done == 0) { for (int i = 0; i < 5; ++i) ms[i] = 0; return NS_OK; }
  NS_CUDA(w, cudaStreamSynchronize(w->stream));
  for (int i = 0; i < 5; ++i) NS_CUDA(w, cudaEventElapsedTime(&ms[i], w->ev[i], w->ev[i + 1]));
  return NS_OK;
}

void* ns_world_stream(ns_world* w) { return w ? (void*)w->stream : nullptr; }

int ns_world_solver_counts(ns_world* w, int64_t* out) {
  if (!w || !out) return NS_ERR_INVALID;
  for (int i = 0; i < 16; ++i) out[i] = 0;
  out[0] = (int64_t)w->asims.size();
  out[1] = w->last_substeps;
  out[5] = (int64_t)w->joints.size();
  out[8] = w->n_gyroscopic;
  out[11] = w->step_kernels;
  out[12] = w->kernel_launches;
  out[13] = w->solver_blocks;
  out[14] = w->solver_grid ? 1 : 0;
  if (!w->uploaded) return NS_OK;
  Control c;
  int st = read_control(w, &c);
  if (st) return st;
  {
    // the dependent phases of the last solver launch, listed as k_solve lists them: per substep
    // integrate velocities (+ the overflow warm start and the body warm start when there is
    // overflow work), push colours, integrate positions, relax colours; then the restitution
    // iterations' colours
    const JointRanges& jr = w->jr;
    bool ovf_work = c.overflow_count > 0 || jr.off[kOverflowIndex + 1] > jr.off[kOverflowIndex];
    int64_t n = ovf_work ? 3 : 1, m = 0;
    for (int stage = 0; stage < 2; ++stage) {
      if (stage == 1) n++;
      if (ovf_work) n++;
      for (int col = 0; col < kOverflowIndex; ++col)
        if (c.color_offset[col + 1] != c.color_offset[col] || jr.off[col + 1] != jr.off[col]) n++;
    }
    if (c.any_restitution && w->def.restitution_iterations > 0) {
      if (c.overflow_count > 0) m++;
      for (int col = 0; col < kOverflowIndex; ++col)
        if (c.color_offset[col + 1] != c.color_offset[col]) m++;
    }
    out[15] = (int64_t)w->last_substeps * n + (int64_t)w->def.restitution_iterations * m;
  }
  int total = c.color_offset[kOverflowIndex];
  std::vector<int4> idx(std::max(total, 1));
  if (total > 0)
    NS_CUDA(w, cudaMemcpy(idx.data(), w->dw.cp.idx, sizeof(int4) * total, cudaMemcpyDeviceToHost));
  int64_t points = 0, stat = 0;
  for (int k = 0; k < total; ++k) {
    points += idx[k].w & 255;
    stat += (idx[k].x < 0) + (idx[k].y < 0);
  }
  out[2] = total;
  out[3] = points;
  out[4] = stat;
  out[6] = c.overflow_count;
  out[7] = c.any_restitution;
  if (c.overflow_count > 0) {
    int nw = w->dw.n_worlds;
    std::vector<int> cnt(nw), base(nw + 1);
    NS_CUDA(w, cudaMemcpy(cnt.data(), w->dw.ovf_count, sizeof(int) * nw, cudaMemcpyDeviceToHost));
    NS_CUDA(w, cudaMemcpy(base.data(), w->dw.world_cbase, sizeof(int) * (nw + 1), cudaMemcpyDeviceToHost));
    for (int k = 0; k < nw; ++k) {
      if (cnt[k] == 0) continue;
      std::vector<DOverflow> ov(cnt[k]);
      NS_CUDA(w, cudaMemcpy(ov.data(), w->dw.ovf + base[k], sizeof(DOverflow) * ov.size(), cudaMemcpyDeviceToHost));
      for (const DOverflow& o : ov) {
        out[9] += o.manifold_count > 0 ? o.m.point_count : 0;
        out[10] += (o.index_a < 0) + (o.index_b < 0);
      }
    }
  }
  return NS_OK;
}

int ns_collide_pairs(ns_pair_job* jobs, ns_pair_result* results, int count) {
  static_assert(sizeof(ns_pair_job) == sizeof(PairJob), "pair job layout");
  static_assert(sizeof(ns_pair_result) == sizeof(PairResult), "pair result layout");
  if (count < 0 || (count > 0 && (!jobs || !results))) return fail(nullptr, NS_ERR_INVALID, "invalid pair batch");
  if (count == 0) return NS_OK;
  {
    int st0 = validate_pair_jobs(jobs, count, "ns_collide_pairs");
    if (st0) return st0;
    st0 = ensure_stack(nullptr);
    if (st0) return st0;
  }
  PairJob* dj = nullptr;
  PairResult* dr = nullptr;
  cudaError_t e = cudaMalloc(&dj, sizeof(PairJob) * (size_t)count);
  if (e == cudaSuccess) e = cudaMalloc(&dr, sizeof(PairResult) * (size_t)count);
  if (e == cudaSuccess) e = cudaMemcpy(dj, jobs, sizeof(PairJob) * (size_t)count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_collide_jobs<<<(count + 127) / 128, 128>>>(dj, dr, count);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(jobs, dj, sizeof(PairJob) * (size_t)count, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(results, dr, sizeof(PairResult) * (size_t)count, cudaMemcpyDeviceToHost);
  if (dj) cudaFree(dj);
  if (dr) cudaFree(dr);
  if (e != cudaSuccess) return fail(nullptr, NS_ERR_CUDA, "ns_collide_pairs: %s", cudaGetErrorString(e));
  return NS_OK;
}

// See natsel_gpu.h: the batch narrowphase without any device allocation. The first call on a
// device raises that device's per-thread stack limit to what the narrowphase kernels need (the
// same set-up ns_collide_pairs and world creation do; the driver may allocate the larger
// local-memory reservation then) and, with lazy module loading, makes the module and its
// scratch array resident there. Every call looks the scratch address up again with the device
// current (cheap), so a reset device or another context never sees a stale address. Then two
// copies in, one launch and two copies out, all on the legacy default stream, so each call has
// finished when it returns.
int ns_collide_pairs_noalloc(ns_pair_job* jobs, ns_pair_result* results, int count) {
  if (count < 0 || (count > 0 && (!jobs || !results))) return fail(nullptr, NS_ERR_INVALID, "invalid pair batch");
  if (count > kNoAllocPairs)
    return fail(nullptr, NS_ERR_CAPACITY, "ns_collide_pairs_noalloc: %d pairs exceed its fixed scratch of %d pairs",
                count, kNoAllocPairs);
  if (count == 0) return NS_OK;
  {
    int st0 = validate_pair_jobs(jobs, count, "ns_collide_pairs_noalloc");
    if (st0) return st0;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(nullptr, NS_ERR_CUDA, "ns_collide_pairs_noalloc: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(nullptr, NS_ERR_INVALID, "device %d out of range", dev);
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pair_scratch_mutex);
    if (!g_pair_stack_ready[dev]) {
      int st0 = ensure_stack(nullptr);
      if (st0) return st0;
      g_pair_stack_ready[dev] = true;
    }
  }
  e = cudaGetSymbolAddress((void**)&base, g_pair_scratch);
  if (e != cudaSuccess)
    return fail(nullptr, NS_ERR_CUDA, "ns_collide_pairs_noalloc scratch address: %s", cudaGetErrorString(e));
  // every slot below count is overwritten (jobs by the copy, results by the kernel), so nothing
  // left from an earlier call is read
  PairJob* dj = reinterpret_cast<PairJob*>(base);
  PairResult* dr = reinterpret_cast<PairResult*>(base + kNoAllocJobBytes);
  e = cudaMemcpy(dj, jobs, sizeof(PairJob) * (size_t)count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_collide_jobs<<<(count + 127) / 128, 128>>>(dj, dr, count);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(jobs, dj, sizeof(PairJob) * (size_t)count, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(results, dr, sizeof(PairResult) * (size_t)count, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(nullptr, NS_ERR_CUDA, "ns_collide_pairs_noalloc: %s", cudaGetErrorString(e));
  return NS_OK;
}

int ns_selftest_barrier_timeout(int device, int timeout_ms) {
  if (timeout_ms <= 0 || timeout_ms > 2000) return fail(nullptr, NS_ERR_INVALID, "timeout_ms must be in 1..2000");
  cudaError_t e = cudaSetDevice(device);
  Control* ctl = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&ctl, sizeof(Control));
  if (e == cudaSuccess) e = cudaMemset(ctl, 0, sizeof(Control));
  if (e == cudaSuccess) {
    k_barrier_selftest<<<2, 32>>>(ctl, (unsigned long long)timeout_ms * 1000000ull);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  Control c;
  memset(&c, 0, sizeof(c));
  if (e == cudaSuccess) e = cudaMemcpy(&c, ctl, sizeof(Control), cudaMemcpyDeviceToHost);
  if (ctl) cudaFree(ctl);
  if (e != cudaSuccess) return fail(nullptr, NS_ERR_CUDA, "barrier self-test: %s", cudaGetErrorString(e));
  if (c.error == kErrTimeout) return fail(nullptr, NS_ERR_TIMEOUT, "grid barrier gave up after %d ms as designed", timeout_ms);
  return fail(nullptr, NS_ERR_INVALID, "barrier self-test did not time out (error %d)", c.error);
}


// Times `steps` steps (after one untimed step) from the checkpoint, eagerly with the world's
// current launch shapes; ms per step, or a negative status.
static int time_from_checkpoint(ns_world* w, const AdCheckpoint& snap, float dt, int substeps, int steps,
                                cudaEvent_t e0, cudaEvent_t e1, float* ms) {
  int st = restore_checkpoint(w, snap);
  if (st) return st;
  if ((st = enqueue_step(w, dt, substeps))) return st;
  NS_CUDA(w, cudaEventRecord(e0, w->stream));
  for (int k = 0; k < steps && !st; ++k) st = enqueue_step(w, dt, substeps);
  if (st) return st;
  NS_CUDA(w, cudaEventRecord(e1, w->stream));
  NS_CUDA(w, cudaEventSynchronize(e1));
  float t = 0.0f;
  NS_CUDA(w, cudaEventElapsedTime(&t, e0, e1));
  *ms = t / (float)steps;
  Control ctl;
  if ((st = read_control(w, &ctl))) return st;
  return control_status(w, ctl);
}

static int autotune(ns_world* w, float dt, int substeps, int steps, int* blocks_out, int* grid_out,
                    float* ms_out, int max_candidates, int* count) {
  if (!w) return NS_ERR_INVALID;
  if (!(dt > 0.0f) || steps < 1) return fail(w, NS_ERR_INVALID, "autotune needs dt > 0 and steps >= 1");
  if (w->tape && w->tape->recording) return fail(w, NS_ERR_UNSUPPORTED, "autotune while a tape records");
  if (!w->uploaded) {
    int st = upload_world(w);
    if (st) return st;
  }
  NS_CUDA(w, cudaSetDevice(w->def.device));
  // candidate solver launch shapes: thread-block clusters of 8 and 16 CTAs, cooperative grids
  // over half the SMs and of 1..4 blocks per SM (as many as can be co-resident)
  int per_sm = 0;
  NS_CUDA(w, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve<true, false>, kSolveThreads, 0));
  NS_CUDA(w, cudaFuncSetAttribute(k_solve<false, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  std::vector<std::pair<int, bool>> cand = {{8, false}, {kMaxSolveCluster, false}, {w->sm_count / 2, true}};
  for (int k = 1; k <= std::min(per_sm, 4); ++k) cand.push_back({k * w->sm_count, true});
  const int old_blocks = w->solver_blocks;
  const bool old_grid = w->solver_grid, old_eager = w->eager;
  const int old_shapes[6] = {w->recycle_threads, w->recycle_per_sm, w->update_threads, w->update_per_sm,
                             w->prepare_threads, w->prepare_per_sm};
  w->tune_rows.clear();
  AdCheckpoint snap;
  int st = take_checkpoint(w, &snap);
  std::vector<float> ms(cand.size(), 0.0f);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!st && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    st = fail(w, NS_ERR_CUDA, "autotune events");
  for (size_t c = 0; c < cand.size() && !st; ++c) {
    w->solver_blocks = cand[c].first;
    w->solver_grid = cand[c].second;
    if (!w->solver_grid) {
      cudaLaunchConfig_t cfg = {};
      cfg.blockDim = dim3(kSolveThreads);
      cfg.gridDim = dim3(w->solver_blocks);
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = w->solver_blocks;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, k_solve<false, false>, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        ms[c] = -1.0f;  // this cluster size does not fit
        w->tune_rows.push_back({0.0f, (float)cand[c].first, 0.0f, -1.0f});
        continue;
      }
    }
    st = time_from_checkpoint(w, snap, dt, substeps, steps, e0, e1, &ms[c]);
    w->tune_rows.push_back({0.0f, (float)cand[c].first, cand[c].second ? 1.0f : 0.0f, ms[c]});
  }
  // keep the fastest solver shape
  int best = -1;
  for (size_t c = 0; c < cand.size(); ++c)
    if (ms[c] > 0.0f && (best < 0 || ms[c] < ms[best])) best = (int)c;
  if (!st && best < 0) st = fail(w, NS_ERR_CUDA, "no solver launch shape could be timed");
  if (!st) {
    w->solver_blocks = cand[best].first;
    w->solver_grid = cand[best].second;
  }
  // then, one kernel at a time with the others kept, the launch shapes of the recycle pass, the
  // full manifold updates and the constraint preparation (threads per block within each
  // kernel's launch bound, blocks per SM at most); the default stays unless a shape is faster
  struct Dim { int id; int* threads; int* per_sm; std::vector<std::pair<int, int>> opts; };
  std::vector<Dim> dims = {
      {1, &w->recycle_threads, &w->recycle_per_sm, {{256, 16}, {128, 16}, {256, 8}, {256, 32}, {128, 32}}},
      {2, &w->update_threads, &w->update_per_sm, {{64, 32}, {32, 32}, {64, 16}, {64, 64}, {32, 64}}},
      {3, &w->prepare_threads, &w->prepare_per_sm, {{128, 16}, {64, 16}, {128, 8}, {128, 32}, {64, 32}}}};
  for (Dim& dm : dims) {
    float best_ms = -1.0f;
    std::pair<int, int> keep = {*dm.threads, *dm.per_sm};
    for (const auto& o : dm.opts) {
      if (st) break;
      *dm.threads = o.first;
      *dm.per_sm = o.second;
      float t = -1.0f;
      st = time_from_checkpoint(w, snap, dt, substeps, steps, e0, e1, &t);
      w->tune_rows.push_back({(float)dm.id, (float)o.first, (float)o.second, t});
      if (!st && (best_ms < 0.0f || t < best_ms)) { best_ms = t; keep = o; }
    }
    *dm.threads = keep.first;
    *dm.per_sm = keep.second;
  }
  // put the world back as it was
  if (snap.data) {
    int st2 = restore_checkpoint(w, snap);
    cudaStreamSynchronize(w->stream);
    release_checkpoint(w, &snap);
    if (!st) st = st2;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  w->eager = old_eager;
  if (st) {
    w->solver_blocks = old_blocks;
    w->solver_grid = old_grid;
    w->recycle_threads = old_shapes[0]; w->recycle_per_sm = old_shapes[1];
    w->update_threads = old_shapes[2]; w->update_per_sm = old_shapes[3];
    w->prepare_threads = old_shapes[4]; w->prepare_per_sm = old_shapes[5];
    return st;
  }
  if (w->graph_exec) { cudaGraphExecDestroy(w->graph_exec); w->graph_exec = nullptr; }
  if (w->graph) { cudaGraphDestroy(w->graph); w->graph = nullptr; }
  int n = std::min<int>((int)cand.size(), max_candidates);
  for (int c = 0; c < n; ++c) {
    if (blocks_out) blocks_out[c] = cand[c].first;
    if (grid_out) grid_out[c] = cand[c].second ? 1 : 0;
    if (ms_out) ms_out[c] = ms[c];
  }
  *count = (int)cand.size();
  return NS_OK;
}

int ns_world_autotune(ns_world* w, float dt, int substeps, int steps, int* blocks_out, int* grid_out,
                      float* ms_out, int max_candidates) {
  int count = 0;
  int st = autotune(w, dt, substeps, steps, blocks_out, grid_out, ms_out, max_candidates, &count);
  return st ? -st : count;
}

int ns_world_autotune_table(const ns_world* w, int* dimension, int* value_a, int* value_b, float* ms, int max_rows) {
  if (!w || max_rows < 0) return -NS_ERR_INVALID;
  int n = std::min<int>((int)w->tune_rows.size(), max_rows);
  for (int r = 0; r < n; ++r) {
    if (dimension) dimension[r] = (int)w->tune_rows[r][0];
    if (value_a) value_a[r] = (int)w->tune_rows[r][1];
    if (value_b) value_b[r] = (int)w->tune_rows[r][2];
    if (ms) ms[r] = w->tune_rows[r][3];
  }
  return (int)w->tune_rows.size();
}

int ns_world_set_launch_shapes(ns_world* w, const int* in8) {
  if (!w || !in8) return NS_ERR_INVALID;
  if (!w->uploaded) {
    int st = upload_world(w);
    if (st) return st;
  }
  NS_CUDA(w, cudaSetDevice(w->def.device));
  const int blocks_ = in8[0], grid = in8[1];
  auto threads_ok = [](int t, int most) { return t >= 32 && t <= most && t % 32 == 0; };
  if (!threads_ok(in8[2], kCollideThreads) || !threads_ok(in8[4], kCollideUpdateThreads) ||
      !threads_ok(in8[6], kPrepareThreads))
    return fail(w, NS_ERR_INVALID, "threads per block must be a multiple of 32 within the kernel's launch bound");
  for (int k : {3, 5, 7})
    if (in8[k] < 1 || in8[k] > 64) return fail(w, NS_ERR_INVALID, "blocks per SM must be in 1..64");
  if (grid != 0 && grid != 1) return fail(w, NS_ERR_INVALID, "the solver grid flag must be 0 or 1");
  if (grid) {
    int per_sm = 0;
    NS_CUDA(w, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve<true, false>, kSolveThreads, 0));
    if (blocks_ < 1 || blocks_ > per_sm * w->sm_count)
      return fail(w, NS_ERR_INVALID, "a cooperative solver grid of %d blocks is not co-resident", blocks_);
  } else {
    if (blocks_ < 1 || blocks_ > kMaxSolveCluster) return fail(w, NS_ERR_INVALID, "cluster of %d CTAs", blocks_);
    NS_CUDA(w, cudaFuncSetAttribute(k_solve<false, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(kSolveThreads);
    cfg.gridDim = dim3(blocks_);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = blocks_;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_solve<false, false>, &cfg) != cudaSuccess || clusters < 1) {
      cudaGetLastError();
      return fail(w, NS_ERR_INVALID, "a cluster of %d CTAs does not fit on this device", blocks_);
    }
  }
  w->solver_blocks = blocks_;
  w->solver_grid = grid != 0;
  w->recycle_threads = in8[2]; w->recycle_per_sm = in8[3];
  w->update_threads = in8[4]; w->update_per_sm = in8[5];
  w->prepare_threads = in8[6]; w->prepare_per_sm = in8[7];
  if (w->graph_exec) { cudaGraphExecDestroy(w->graph_exec); w->graph_exec = nullptr; }
  if (w->graph) { cudaGraphDestroy(w->graph); w->graph = nullptr; }
  return NS_OK;
}

int ns_world_launch_shapes(const ns_world* w, int* out8) {
  if (!w || !out8) return NS_ERR_INVALID;
  int v[8] = {w->solver_blocks, w->solver_grid ? 1 : 0, w->recycle_threads, w->recycle_per_sm, w->update_threads,
              w->update_per_sm, w->prepare_threads, w->prepare_per_sm};
  for (int i = 0; i < 8; ++i) out8[i] = v[i];
  return NS_OK;
}

int ns_world_tape_begin(ns_world* w, int checkpoint_substeps) {
  if (!w) return NS_ERR_INVALID;
  if (checkpoint_substeps < 1) return fail(w, NS_ERR_INVALID, "checkpoint_substeps must be >= 1");
  if (!w->uploaded) {
    int st = upload_world(w);
    if (st) return st;
  }
  NS_CUDA(w, cudaSetDevice(w->def.device));
  int st = check_adjoint_scope(w);
  if (st) return st;
  free_tape(w);
  w->tape = new AdTape();
  w->tape->every = checkpoint_substeps;
  w->tape->ckpt.emplace_back();
  st = take_checkpoint(w, &w->tape->ckpt.back());
  if (st) { free_tape(w); return st; }
  w->tape->ckpt_at.push_back(0);
  w->tape->recording = true;
  return NS_OK;
}

int ns_world_tape_end(ns_world* w) {
  if (!w) return NS_ERR_INVALID;
  if (!w->tape) return fail(w, NS_ERR_INVALID, "no tape");
  w->tape->recording = false;
  return NS_OK;
}

int ns_world_tape_free(ns_world* w) {
  if (!w) return NS_ERR_INVALID;
  free_tape(w);
  return NS_OK;
}

int ns_world_tape_info(ns_world* w, int64_t* out) {
  if (!w || !out) return NS_ERR_INVALID;
  for (int i = 0; i < 8; ++i) out[i] = 0;
  if (!w->tape) return NS_OK;
  const AdTape* t = w->tape;
  out[0] = (int64_t)t->steps.size();
  out[1] = (int64_t)t->ckpt.size();
  out[2] = t->replay_mismatch;
  out[3] = t->vjp_calls;
  out[4] = t->recording ? 1 : 0;
  out[5] = t->every;
  out[6] = t->vjp_launches;
  return NS_OK;
}

}  // extern "C"

// A copy of a step tape whose pointers point into a host copy of the tape buffer.
static StepTape rebase_tape(const StepTape& t, const char* dev_base, char* host_base) {
  auto rb = [&](auto* p) { return (decltype(p))(host_base + ((const char*)p - dev_base)); };
  StepTape h = t;
  h.sims = rb(t.sims); h.pre = rb(t.pre); h.post = rb(t.post); h.ctl = rb(t.ctl);
  h.body = rb(t.body); h.push = rb(t.push); h.relax = rb(t.relax); h.fin = rb(t.fin); h.mode = rb(t.mode);
  h.rest = rb(t.rest);
  h.joints = rb(t.joints); h.joint = rb(t.joint); h.jwarm = rb(t.jwarm);
  CPlanes& P = h.planes;
  P.idx = rb(t.planes.idx); P.mass = rb(t.planes.mass); P.ia0 = rb(t.planes.ia0); P.ia1 = rb(t.planes.ia1);
  P.ib1 = rb(t.planes.ib1); P.n = rb(t.planes.n); P.t1 = rb(t.planes.t1); P.t2 = rb(t.planes.t2);
  P.ca = rb(t.planes.ca); P.cb = rb(t.planes.cb); P.tm = rb(t.planes.tm); P.fr = rb(t.planes.fr);
  P.roll = rb(t.planes.roll); P.rm = rb(t.planes.rm); P.pra = rb(t.planes.pra); P.prb = rb(t.planes.prb);
  P.pimp = rb(t.planes.pimp); P.prest = rb(t.planes.prest);
  return h;
}

// The vector-Jacobian product of the recorded rollout: replay each checkpoint segment with the
// solver tape on, then reverse its steps on the device in f32 (f64 false) or on the host in f64
// from a copy of the segment's tapes. out: 16 values per body id (lin 3, ang 3, mass, friction,
// pos 3, rot 4, 0).
static int vjp_run(ns_world* w, const float* const seeds_in[4], bool f64, std::vector<double>& out) {
  if (!w) return NS_ERR_INVALID;
  if (!w->tape || w->tape->steps.empty()) return fail(w, NS_ERR_INVALID, "no recorded steps");
  NS_CUDA(w, cudaSetDevice(w->def.device));
  AdTape* tp = w->tape;
  if (f64 && w->dw.n_joints > 0) return fail(w, NS_ERR_UNSUPPORTED, "the f64 reverse pass does not cover joints");
  tp->recording = false;
  tp->vjp_calls++;
  const DW& d = w->dw;
  const int nb = (int)w->bodies.size(), n = d.n_awake, cap = d.cap;
  auto blocks = [](int count, int t) { return std::max(1, (count + t - 1) / t); };
  // segments between checkpoints
  std::vector<std::pair<int, int>> segs;
  for (size_t c = 0; c < tp->ckpt_at.size(); ++c) {
    int a = tp->ckpt_at[c];
    int b = c + 1 < tp->ckpt_at.size() ? tp->ckpt_at[c + 1] : (int)tp->steps.size();
    segs.push_back({a, b});
  }
  int max_len = 0, max_sub = 1;
  for (auto& sg : segs) max_len = std::max(max_len, sg.second - sg.first);
  for (const AdStepRec& r : tp->steps) max_sub = std::max(max_sub, r.substeps);
  AdCheckpoint final_state;
  TapeSet ts;
  char* buf = nullptr;
  int st = NS_OK;
  out.assign((size_t)16 * std::max(nb, 1), 0.0);
  std::vector<float> host_out((size_t)16 * std::max(nb, 1));
  // the host reverse pass (f64)
  host_adj::Bufs ha;
  std::vector<DShape> hshapes;
  std::vector<Hull> hhulls;
  std::vector<char> host_tape;
  host_adj::Consts hc = {};
  if (f64) {
    ha.init(n, cap);
    for (const HostShape& hs : w->shapes) { hshapes.push_back(hs.d); hhulls.push_back(hs.hull); }
    hc.shapes = hshapes.data(); hc.hulls = hhulls.data(); hc.ssims = w->ssims.data();
    for (int i = 0; i < nb; ++i) {
      const HostBody& b = w->bodies[i];
      if (b.set != 2) continue;
      int loc = b.local;
      for (int f = 0; f < 3; ++f) {
        ha.CQ(loc, f) = seeds_in[0] ? seeds_in[0][3 * i + f] : 0.0;
        ha.BB(loc, f) = seeds_in[2] ? seeds_in[2][3 * i + f] : 0.0;
        ha.BB(loc, 4 + f) = seeds_in[3] ? seeds_in[3][3 * i + f] : 0.0;
      }
      for (int f = 0; f < 4; ++f) ha.CQ(loc, 4 + f) = seeds_in[1] ? seeds_in[1][4 * i + f] : 0.0;
    }
  }
  do {
    if ((st = take_checkpoint(w, &final_state))) break;
    if ((st = alloc_tapes(w, std::max(max_len, 1), max_sub, &ts))) break;
    if (f64) host_tape.resize(ts.bytes);
    // cotangent buffers and staging
    size_t o = 0;
    auto take = [&](size_t b) { size_t r = o; o += align256(b); return r; };
    size_t o_bb = take(sizeof(float) * 16 * (size_t)n), o_cq = take(sizeof(float) * 8 * (size_t)n);
    size_t o_pb = take(sizeof(float) * kPB * (size_t)n), o_kb = take(sizeof(float) * ad::kCVOwn * (size_t)cap);
    size_t o_mb = take(sizeof(float) * kMB * (size_t)cap), o_mis = take(sizeof(int));
    size_t o_yrec = take(sizeof(float) * 3 * ad::kRelaxOut * (size_t)cap * max_sub);
    size_t o_tot = take(sizeof(float) * 4 * (size_t)cap), o_restb = take(sizeof(float) * 4 * (size_t)cap);
    size_t o_rel = take(sizeof(float) * 4 * (size_t)cap);
    const size_t nj = (size_t)std::max(d.n_joints, 1);
    size_t o_jb = take(sizeof(float) * ad::kJState * nj), o_jc = take(sizeof(float) * ad::kJConst * nj);
    size_t o_seed = take(sizeof(float) * 13 * (size_t)nb), o_out = take(sizeof(float) * 16 * (size_t)nb);
    if (reuse_buffer(w, &w->adj_buf, &w->adj_cap, o) != NS_OK) { st = fail(w, NS_ERR_CUDA, "adjoint buffers (%zu bytes)", o); break; }
    buf = w->adj_buf;
    NS_CUDA(w, cudaMemsetAsync(buf, 0, o, w->stream));
    AdjBufs a;
    a.bb = (float*)(buf + o_bb); a.cq = (float*)(buf + o_cq); a.pb = (float*)(buf + o_pb);
    a.kb = (float*)(buf + o_kb); a.mb = (float*)(buf + o_mb); a.mismatch = (int*)(buf + o_mis);
    a.yrec = (float*)(buf + o_yrec);
    bool any_rest = false;
    for (const HostShape& hs : w->shapes) any_rest = any_rest || hs.d.restitution > 0.0f;
    a.totb = any_rest ? (float*)(buf + o_tot) : nullptr;
    a.restb = (float*)(buf + o_restb); a.relb = (float*)(buf + o_rel);
    a.jb = (float*)(buf + o_jb); a.jc = (float*)(buf + o_jc);
    a.joint_list = d.joint_list; a.jr = w->jr; a.n_joints = d.n_joints;
    a.cap = cap; a.n_awake = n;
    float* seed = (float*)(buf + o_seed);
    float* dev_out = (float*)(buf + o_out);
    const int width[4] = {3, 4, 3, 3};
    float* dst[4] = {seed, seed + 3 * (size_t)nb, seed + 7 * (size_t)nb, seed + 10 * (size_t)nb};
    int64_t launches = 2;  // the final-state snapshot and the seeds
    if (!f64) {
      for (int i = 0; i < 4; ++i)
        if (seeds_in[i])
          NS_CUDA(w, cudaMemcpyAsync(dst[i], seeds_in[i], sizeof(float) * width[i] * (size_t)nb, cudaMemcpyHostToDevice, w->stream));
      k_adj_seed<<<blocks(nb, 256), 256, 0, w->stream>>>(a, w->body_loc, nb, seeds_in[0] ? dst[0] : nullptr,
                                                          seeds_in[1] ? dst[1] : nullptr, seeds_in[2] ? dst[2] : nullptr,
                                                          seeds_in[3] ? dst[3] : nullptr);
    }
    for (int sgi = (int)segs.size() - 1; sgi >= 0 && st == NS_OK; --sgi) {
      int s0 = segs[sgi].first, s1 = segs[sgi].second;
      if (s1 <= s0) continue;
      if ((st = restore_checkpoint(w, tp->ckpt[sgi]))) break;
      launches += 1;
      for (int j = s0; j < s1 && st == NS_OK; ++j) {
        HostStepTape& h = ts.steps[j - s0];
        h.dev.substeps = tp->steps[j].substeps;
        st = enqueue_step(w, tp->steps[j].dt, tp->steps[j].substeps, &h);
        launches += w->step_kernels + 1;  // the step and its plane copy
      }
      if (st) break;
      // the recorded steps must stay inside the adjoint's scope
      std::vector<Control> ctl(s1 - s0);
      for (int j = s0; j < s1; ++j)
        NS_CUDA(w, cudaMemcpyAsync(&ctl[j - s0], ts.steps[j - s0].dev.ctl, sizeof(Control), cudaMemcpyDeviceToHost, w->stream));
      NS_CUDA(w, cudaStreamSynchronize(w->stream));
      for (int j = s0; j < s1 && st == NS_OK; ++j) {
        const Control& c = ctl[j - s0];
        if (c.error) st = control_status(w, c);
        else if (c.overflow_count > 0) st = fail(w, NS_ERR_UNSUPPORTED, "step %d has overflow constraints; the adjoint does not cover them", j);
        else if (c.any_restitution && f64)
          st = fail(w, NS_ERR_UNSUPPORTED, "step %d has restitution; the f64 reverse pass does not cover it", j);
      }
      if (st) break;
      if (f64) {
        NS_CUDA(w, cudaMemcpy(host_tape.data(), ts.data, ts.bytes, cudaMemcpyDeviceToHost));
        for (int j = s1 - 1; j >= s0; --j) {
          StepTape t = rebase_tape(ts.steps[j - s0].dev, ts.data, host_tape.data());
          StepParams p = make_step_params(w, tp->steps[j].dt, tp->steps[j].substeps);
          host_adj::step(t, ha, hc, p);
        }
        continue;
      }
      for (int j = s1 - 1; j >= s0 && st == NS_OK; --j) {
        const StepTape& t = ts.steps[j - s0].dev;
        StepParams p = make_step_params(w, tp->steps[j].dt, tp->steps[j].substeps);
        const Control& c = ctl[j - s0];
        int n_slots = c.color_offset[kOverflowIndex];
        bool rest = n_slots > 0 && c.any_restitution;
        if (n > 0) k_adj_finalize<<<blocks(n, 128), 128, 0, w->stream>>>(t, a, n);
        if (n_slots > 0) k_adj_store<<<blocks(n_slots, 128), 128, 0, w->stream>>>(t, a, n_slots);
        // the restitution iterations ran after the substeps, colours in order: reverse them
        if (rest && p.restitution_iterations > 0) {
          const ad::RParams rp = {0, p.inv_h, p.restitution_threshold};
          const int per_block = kAdjThreads / 32;
          for (int it = p.restitution_iterations - 1; it >= 0; --it)
            for (int col = kOverflowIndex - 1; col >= 0; --col) {
              int cnt = c.color_offset[col + 1] - c.color_offset[col];
              if (cnt <= 0) continue;
              k_adj_restitution<<<blocks(cnt, per_block), kAdjThreads, 0, w->stream>>>(t, a, d, rp, it, col);
              launches += 1;
            }
        }
        if ((st = launch_adj_solve(w, t, a, p))) break;
        // prepare's relative velocities read the velocities at the step's start
        if (rest) {
          k_adj_relvel<<<blocks(n_slots, 128), 128, 0, w->stream>>>(t, a, n_slots);
          launches += 1;
        }
        if (n_slots > 0) k_adj_consts<<<blocks(n_slots, 64), 64, 0, w->stream>>>(t, a, p, n_slots);
        if (n_slots > 0) k_adj_prepare<<<blocks(n_slots, kAdjThreads / 32), kAdjThreads, 0, w->stream>>>(t, a, d, p, n_slots);
        if (d.n_joints > 0) {
          k_adj_joint_prepare<<<blocks(d.n_joints, kAdjThreads / 32), kAdjThreads, 0, w->stream>>>(t, a, d, p);
          launches += 1;
        }
        if (n > 0) k_adj_inertia<<<blocks(n, kAdjThreads / 32), kAdjThreads, 0, w->stream>>>(t, a);
        k_adj_narrow<<<blocks(cap, kAdjThreads / 32), kAdjThreads, 0, w->stream>>>(t, a, d);
        NS_CUDA(w, cudaGetLastError());
        launches += 2 + (n > 0 ? 2 : 0) + (n_slots > 0 ? 3 : 0);  // solve, narrowphase, per-body, per-slot
      }
    }
    if (st) break;
    int mismatch = 0;
    if (!f64) {
      k_adj_result<<<blocks(nb, 256), 256, 0, w->stream>>>(a, d, w->body_loc, nb, dev_out);
      launches += 2;  // the result and the final restore
      tp->vjp_launches = launches;
      NS_CUDA(w, cudaMemcpyAsync(host_out.data(), dev_out, sizeof(float) * 16 * (size_t)nb, cudaMemcpyDeviceToHost, w->stream));
      NS_CUDA(w, cudaMemcpyAsync(&mismatch, a.mismatch, sizeof(int), cudaMemcpyDeviceToHost, w->stream));
    }
    if ((st = restore_checkpoint(w, final_state))) break;
    NS_CUDA(w, cudaStreamSynchronize(w->stream));
    tp->replay_mismatch += f64 ? ha.mismatch : mismatch;
    Control c;
    if ((st = read_control(w, &c))) break;
    if ((st = control_status(w, c))) break;
  } while (0);
  if (st) {
    // put the world back even when the reverse pass failed
    if (final_state.data) { restore_checkpoint(w, final_state); cudaStreamSynchronize(w->stream); }
  }
  cudaStreamSynchronize(w->stream);
  release_checkpoint(w, &final_state);
  if (st) return st;
  if (!f64) {
    for (size_t i = 0; i < out.size(); ++i) out[i] = host_out[i];
    return NS_OK;
  }
  // results of the host pass (as k_adj_result)
  for (int i = 0; i < nb; ++i) {
    const HostBody& b = w->bodies[i];
    if (b.set != 2) continue;
    int loc = b.local;
    double* o = &out[(size_t)16 * i];
    for (int f = 0; f < 3; ++f) { o[f] = ha.BB(loc, f); o[3 + f] = ha.BB(loc, 4 + f); o[8 + f] = ha.CQ(loc, f); }
    for (int f = 0; f < 4; ++f) o[11 + f] = ha.CQ(loc, 4 + f);
    const DSim& s = w->asims[loc];
    double im = s.inv_mass;
    const float* il = &s.inv_inertia_local.cx.x;
    const float* ii = &s.inertia.cx.x;
    double dot_ii = 0.0, dot_i = 0.0;
    for (int f = 0; f < 9; ++f) { dot_ii += ha.PB(loc, pbIinv + f) * il[f]; dot_i += ha.PB(loc, pbInertia + f) * ii[f]; }
    o[6] = -ha.PB(loc, pbInvMass) * im * im - dot_ii * im + dot_i * im;
    o[7] = ha.PB(loc, pbFriction);
  }
  return NS_OK;
}

extern "C" {

int ns_world_vjp(ns_world* w, const float* dpos, const float* drot, const float* dlin, const float* dang,
                 float* dlin0, float* dang0, float* dmass, float* dfriction, float* dpos0, float* drot0) {
  const float* seeds[4] = {dpos, drot, dlin, dang};
  std::vector<double> o;
  int st = vjp_run(w, seeds, false, o);
  if (st) return st;
  for (int i = 0; i < (int)w->bodies.size(); ++i) {
    const double* r = &o[(size_t)16 * i];
    for (int f = 0; f < 3; ++f) {
      if (dlin0) dlin0[3 * i + f] = (float)r[f];
      if (dang0) dang0[3 * i + f] = (float)r[3 + f];
      if (dpos0) dpos0[3 * i + f] = (float)r[8 + f];
    }
    for (int f = 0; f < 4; ++f) if (drot0) drot0[4 * i + f] = (float)r[11 + f];
    if (dmass) dmass[i] = (float)r[6];
    if (dfriction) dfriction[i] = (float)r[7];
  }
  w->vjp_restitution.assign(w->bodies.size(), 0.0f);
  for (size_t i = 0; i < w->bodies.size(); ++i) w->vjp_restitution[i] = (float)o[16 * i + 15];
  return NS_OK;
}

int ns_world_vjp_restitution(const ns_world* w, float* drestitution) {
  if (!w || !drestitution) return NS_ERR_INVALID;
  if (w->vjp_restitution.size() != w->bodies.size())
    return fail(const_cast<ns_world*>(w), NS_ERR_INVALID, "no ns_world_vjp result for the current bodies");
  std::copy(w->vjp_restitution.begin(), w->vjp_restitution.end(), drestitution);
  return NS_OK;
}

int ns_world_vjp_f64(ns_world* w, const float* dpos, const float* drot, const float* dlin, const float* dang,
                     double* dlin0, double* dang0, double* dmass, double* dfriction, double* dpos0, double* drot0) {
  const float* seeds[4] = {dpos, drot, dlin, dang};
  std::vector<double> o;
  int st = vjp_run(w, seeds, true, o);
  if (st) return st;
  for (int i = 0; i < (int)w->bodies.size(); ++i) {
    const double* r = &o[(size_t)16 * i];
    for (int f = 0; f < 3; ++f) {
      if (dlin0) dlin0[3 * i + f] = r[f];
      if (dang0) dang0[3 * i + f] = r[3 + f];
      if (dpos0) dpos0[3 * i + f] = r[8 + f];
    }
    for (int f = 0; f < 4; ++f) if (drot0) drot0[4 * i + f] = r[11 + f];
    if (dmass) dmass[i] = r[6];
    if (dfriction) dfriction[i] = r[7];
  }
  return NS_OK;
}

}  // extern "C"
