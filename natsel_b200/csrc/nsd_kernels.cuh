// Step kernels. One world step is: pair update (sort-and-sweep) -> contact
// creation -> collide -> ordered state pass (graph coloring) -> color
// partition + constraint prepare -> persistent colored solver -> finalize.
// Each kernel cites the reference stage it replaces; arithmetic keeps the
// reference operand order so results match the reference bit for bit.
#pragma once
#include <climits>
#include <cub/cub.cuh>
#include "nsd_types.cuh"

namespace nsd {

constexpr int kStatePassThreads = 1024;

// Warp-aggregated counters. A counter that every element of a large pass bumps serialises one
// atomic per element at its L2 slice; here the threads that reach the call together (the
// active mask) add their total with one atomic. add_converged adds 1 per thread;
// slot_converged hands each thread a distinct slot of counters[key] (slots within a group in
// lane order, groups in atomic order: for lists whose order does not matter).
__device__ __forceinline__ void add_converged(int* counter) {
  const unsigned am = __activemask();
  if ((int)(threadIdx.x & 31) == __ffs(am) - 1) atomicAdd(counter, __popc(am));
}
__device__ __forceinline__ int slot_converged(int* counters, int key) {
  const unsigned am = __activemask();
  const unsigned peers = __match_any_sync(am, key);
  const int lane = (int)(threadIdx.x & 31), leader = __ffs(peers) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(&counters[key], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}

// DW::slot_state: bit 7 alive, bits 0..4 the colour + 1 of a touching contact in colours 0..22.
constexpr uint8_t kSlotAlive = 0x80;
__device__ __forceinline__ uint8_t slot_state_of(bool alive, bool touching, int color) {
  return (uint8_t)((alive ? kSlotAlive : 0) |
                   (alive && touching && color >= 0 && color < kOverflowIndex ? color + 1 : 0));
}
__device__ __forceinline__ int slot_color_of(uint8_t s) { return (s & kSlotAlive) ? (int)(s & 31) - 1 : -1; }
constexpr int kColorBlock = 1024;
constexpr int kSolveThreads = 256;   // per CTA of the solver cluster
constexpr int kMaxSolveCluster = 16;
constexpr unsigned long long kHsEmpty = ~0ull;
constexpr unsigned long long kHsTomb = ~0ull - 1ull;

// Error codes mirrored from natsel_gpu.h.
constexpr int kErrCapacity = 3;
constexpr int kErrTimeout = 4;
constexpr int kErrNonFinite = 5;

struct DW {
  DSim* asims; DState* states; int n_awake;
  DSim* ssims; int n_static;
  DShape* shapes; Hull* hulls; AABB* fat; int* moved; int n_shapes;
  int* body_shapes;                 // shape ids grouped per awake body (DSim shape range)
  uint32_t* body_mask; int n_bodies;
  uint8_t* body_dyn;  // [body id] 1 for a dynamic body (kinematic and static bodies are not)
  int* body_joint_off; int* body_joint_other;  // joint partners with collision disabled
  DContact* contacts; int cap;
  int* free_stack;
  unsigned long long* hs; int hs_mask;
  uint32_t* changed_bits; int* changed_list; int* destroyed; int n_words;
  int* overflow_list;
  CPlanes cp;
  DOverflow* ovf;
  DJoint* joints; int n_joints; int* joint_list;
  // broadphase scratch
  uint32_t* bp_keys_in; uint32_t* bp_keys_out; int* bp_vals_in; int* bp_vals_out;
  // small proxies sorted by grid cell: (lo.x, hi.x, lo.y, hi.y), (lo.z, hi.z), shape id | flags
  float4* bp_xy; float2* bp_z; int* bp_meta;
  // uniform grid over small proxies: cell edge >= every small proxy's extent; cells hashed into
  // cell_mask + 1 buckets holding [first, end) ranges of the sorted proxies
  float cell, inv_cell; int cell_mask; int2* cells;
  int n_small; int* large_list; int n_large;
  int* seg_count; int* seg_off; int* seg_cursor;
  unsigned long long* cand; unsigned long long* sorted_keys; int cand_cap;
  int* block_color;                 // per color-partition block x 24
  int n_color_blocks;
  Control* ctl;
  // Sub-worlds (independent worlds stepped together; one for a plain world). World w owns the
  // shapes [world_shape[w], world_shape[w+1]), the contact ids [world_cbase[w],
  // world_cbase[w+1]) (multiples of 32), a LIFO id pool on free_stack at world_cbase[w] with
  // pool_top[w] free ids and pool_next[w] the next never-used local id, an overflow list at
  // overflow_list + world_cbase[w] with ovf_count[w] entries, and the large static proxies
  // large_list[large_off[w] .. large_off[w+1]).
  int n_worlds;
  int* world_cbase; int* world_shape; int* pool_top; int* pool_next; int* ovf_count; int* large_off;
  int* bp_world;  // sub-world of each sorted small proxy
  int* collide_list;  // per pair kind k: ids at collide_list + k * cap needing a full update
  // Optional record of each contact's narrowphase outcome (0 none or disjoint, 1 recycled,
  // 2 new manifold, 3 no points), written only while the adjoint replays a step.
  uint8_t* np_mode;
  // Warm start by body: slot (body, colour c) of bwd holds the velocity change that body's
  // constraint or joint of colour c applies at the next warm start, (dv, dw) at
  // 2 * (24 * body + c) + {0, 1}, signed for the body's side; bit c of bw_mask[body] marks the
  // slot as used this step.
  float4* bwd; uint32_t* bw_mask;
  int* slot_cid;  // contact id of each coloured constraint slot (this step)
  // One byte per contact slot, kept with the contact: bit 7 alive, bits 0..4 the colour + 1 of a
  // touching contact in colours 0..22 (0 otherwise). Read by passes over every slot instead of
  // the 400-byte contact records.
  uint8_t* slot_state;
  int* long_segment;  // candidate segments of more than kShortSegment keys (this pair update)
  // Continuous collision: the fast bodies finalize queues (awake indices, this step), the
  // static shapes of each sub-world (static_list[static_off[w] .. static_off[w + 1])) and each
  // shape's last bounds (shape.aabb in the reference: the speculative-inflated box finalize
  // computes, or the swept end box of the continuous pass).
  int* fast_list; int* static_list; int* static_off; AABB* saabb;
  int* bullet_list; int* dyn_list; int* dyn_off;  // fast bullets; dynamic bodies' shapes per sub-world
};

struct JointRanges { int off[25]; };

// ---------------------------------------------------------------------------
// Small device helpers

__device__ __forceinline__ uint32_t float_sort_key(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ void raise_error(Control* c, int code) { atomicCAS(&c->error, 0, code); }

// hash_set.rs:25 shape_pair_key with child 0
__device__ __forceinline__ unsigned long long pair_key(int s1, int s2) {
  const unsigned long long mask = (1ull << 22) - 1ull;
  unsigned long long a = mask & (unsigned long long)(long long)s1;
  unsigned long long b = mask & (unsigned long long)(long long)s2;
  if (s1 < s2) return (a << 42) | (b << 20);
  return (b << 42) | (a << 20);
}

__device__ __forceinline__ uint32_t hs_hash(unsigned long long k) {
  k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
  return (uint32_t)k;
}
__device__ bool hs_contains(const DW& w, unsigned long long k) {
  uint32_t i = hs_hash(k) & (uint32_t)w.hs_mask;
  for (int probe = 0; probe <= w.hs_mask; ++probe) {
    unsigned long long v = w.hs[i];
    if (v == k) return true;
    if (v == kHsEmpty) return false;
    i = (i + 1) & (uint32_t)w.hs_mask;
  }
  return false;
}
__device__ void hs_insert(const DW& w, unsigned long long k) {
  uint32_t i = hs_hash(k) & (uint32_t)w.hs_mask;
  for (int probe = 0; probe <= w.hs_mask; ++probe) {
    unsigned long long v = w.hs[i];
    if (v == kHsEmpty || v == kHsTomb) {
      if (atomicCAS(&w.hs[i], v, k) == v) return;
      continue;  // lost the race for this slot; re-read it
    }
    i = (i + 1) & (uint32_t)w.hs_mask;
  }
  raise_error(w.ctl, kErrCapacity);
}
__device__ void hs_erase(const DW& w, unsigned long long k) {
  uint32_t i = hs_hash(k) & (uint32_t)w.hs_mask;
  for (int probe = 0; probe <= w.hs_mask; ++probe) {
    unsigned long long v = w.hs[i];
    if (v == k) { w.hs[i] = kHsTomb; atomicAdd(&w.ctl->tombstones, 1); return; }
    if (v == kHsEmpty) return;
    i = (i + 1) & (uint32_t)w.hs_mask;
  }
}

__device__ __forceinline__ const DSim& sim_of(const DW& w, int enc) {
  return enc >= 0 ? w.asims[enc] : w.ssims[-enc - 2];
}

// ---------------------------------------------------------------------------
// Pair update (contact_creation.rs:901 update_broad_phase_pairs). The reference's tree
// traversal yields every overlapping fat-AABB pair with at least one moved proxy; keys are
// sorted before contacts are created, so any search that finds the same set is equivalent.
// Here: a sort-and-sweep along x over the small proxies plus a direct test against the few
// large static proxies.

__global__ void k_hs_rebuild_clear(DW w) {
  if (w.ctl->hs_rebuild == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= w.hs_mask; i += gridDim.x * blockDim.x)
    w.hs[i] = kHsEmpty;
}
__global__ void k_hs_rebuild_insert(DW w) {
  if (w.ctl->hs_rebuild == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w.cap; i += gridDim.x * blockDim.x) {
    const DContact& c = w.contacts[i];
    if (c.alive) hs_insert(w, pair_key(c.shape_a, c.shape_b));
  }
}

// Grid cell of a coordinate (monotone in x, so order-preserving comparisons stay valid).
__device__ __forceinline__ int grid_coord(float x, float inv_cell) { return __float2int_rd(x * inv_cell); }
__device__ __forceinline__ uint32_t cell_hash(int world, int cx, int cy, int cz) {
  return ((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^ ((uint32_t)cz * 83492791u) ^
         ((uint32_t)world * 2654435761u);
}

// Sort keys: the hashed grid cell of each small proxy's lower corner; large static proxies
// (the ground) sort after all of them and are paired by k_bp_large.
__global__ void k_bp_keys(DW w) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n_shapes) return;
  const DShape& s = w.shapes[i];
  AABB f = w.fat[i];
  float width = f.hi.x - f.lo.x;
  bool large = s.is_static && width > 8.0f;
  uint32_t key = (uint32_t)w.cell_mask + 1u;
  if (!large)
    key = cell_hash(s.world, grid_coord(f.lo.x, w.inv_cell), grid_coord(f.lo.y, w.inv_cell),
                    grid_coord(f.lo.z, w.inv_cell)) & (uint32_t)w.cell_mask;
  w.bp_keys_in[i] = key;
  w.bp_vals_in[i] = i;
}

// contact_creation.rs:151 should_create_pair for the filters this path supports
__device__ bool should_create_pair(const DW& w, int a, int b) {
  const DShape& A = w.shapes[a];
  const DShape& B = w.shapes[b];
  if (A.body == B.body) return false;
  if (A.group == B.group && A.group != 0) {
    if (!(A.group > 0)) return false;
  } else if (!((A.mask & B.category) != 0 && (A.category & B.mask) != 0)) {
    return false;
  }
  // contact_creation.rs:113 should_bodies_collide: at least one dynamic body
  if (!w.body_dyn[A.body] && !w.body_dyn[B.body]) return false;
  for (int j = w.body_joint_off[A.body]; j < w.body_joint_off[A.body + 1]; ++j)
    if (w.body_joint_other[j] == B.body) return false;
  return true;
}

// Appends the pair {a, b} (fat AABBs known to overlap) when the filters accept it and it is
// not already a contact.
__device__ void emit_overlapping_pair(const DW& w, int a, int b) {
  int lo = a < b ? a : b, hi = a < b ? b : a;
  // most overlapping pairs are existing contacts: test the pair set before the filters
  unsigned long long k = pair_key(lo, hi);
  if (hs_contains(w, k)) return;
  if (!should_create_pair(w, lo, hi)) return;
  int slot = atomicAdd(&w.ctl->cand_count, 1);
  if (slot >= w.cand_cap) { raise_error(w.ctl, kErrCapacity); return; }
  w.cand[slot] = k;
  atomicAdd(&w.seg_count[lo], 1);
}

__device__ void emit_pair(const DW& w, int a, int b) {
  if (!aabb_overlaps(w.fat[a], w.fat[b])) return;
  emit_overlapping_pair(w, a, b);
}

constexpr int kMetaMoved = 1 << 30;
constexpr int kMetaStatic = 1 << 29;
constexpr int kMetaId = (1 << 29) - 1;

// Sorted small proxies as contiguous arrays, and each occupied bucket's [first, end) range
// (the bucket table is zeroed before this kernel).
__global__ void k_bp_gather(DW w) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= w.n_small) return;
  int b = w.bp_vals_out[j];
  AABB f = w.fat[b];
  w.bp_xy[j] = make_float4(f.lo.x, f.hi.x, f.lo.y, f.hi.y);
  w.bp_z[j] = make_float2(f.lo.z, f.hi.z);
  w.bp_meta[j] = b | (w.moved[b] ? kMetaMoved : 0) | (w.shapes[b].is_static ? kMetaStatic : 0);
  w.bp_world[j] = w.shapes[b].world;
  uint32_t key = w.bp_keys_out[j];
  if (j == 0 || w.bp_keys_out[j - 1] != key) w.cells[key].x = j;
  if (j == w.n_small - 1 || w.bp_keys_out[j + 1] != key) w.cells[key].y = j + 1;
}

// Cell range [lo, hi] of one axis, at most three cells: every proxy that can overlap a box
// with bounds [lo, hi] has its own lower bound in [lo - extent, hi], and extents stay below
// cell / 1.001, so rounding lo - cell cannot exclude one. Non-finite bounds give a clamped
// range instead of a runaway loop.
__device__ __forceinline__ void axis_cells(float lo, float hi, const DW& w, int* c0, int* c1) {
  int a = grid_coord(lo - w.cell, w.inv_cell);
  int b = grid_coord(hi, w.inv_cell);
  if (b - a > 2 || b < a) b = a + 2;
  *c0 = a;
  *c1 = b;
}

// contact_creation.rs:1000 find_pairs for each moved proxy (the reference queries its dynamic
// trees; the set of pairs is the same): every small proxy whose fat AABB overlaps the moved
// proxy's lies in the grid cells around it. Each overlapping pair with at least one moved
// proxy is reported once (by the smaller moved shape id when both moved); a proxy met again
// through a hash collision is skipped by checking its own cell and sub-world (proxies of
// different sub-worlds never pair). One warp per proxy, lane l < 27 scanning cell
// (x0 + l / 9, y0 + l / 3 % 3, z0 + l % 3) of the at most 3 x 3 x 3 around it; the pairs are
// sorted per shape afterwards, so the order they are found in does not matter.
constexpr int kQueryThreads = 128;
__global__ void __launch_bounds__(kQueryThreads) k_bp_query(DW w) {
  if (w.ctl->moved_count == 0) return;
  const int i = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int lane = (int)(threadIdx.x & 31u);
  if (i >= w.n_small || lane >= 27) return;
  int mm = w.bp_meta[i];
  if (!(mm & kMetaMoved)) return;
  int m = mm & kMetaId;
  bool m_static = (mm & kMetaStatic) != 0;
  int mw = w.bp_world[i];
  float4 A = w.bp_xy[i];
  float2 Az = w.bp_z[i];
  int x0, x1, y0, y1, z0, z1;
  axis_cells(A.x, A.y, w, &x0, &x1);
  axis_cells(A.z, A.w, w, &y0, &y1);
  axis_cells(Az.x, Az.y, w, &z0, &z1);
  const int cx = x0 + lane / 9, cy = y0 + (lane / 3) % 3, cz = z0 + lane % 3;
  if (cx > x1 || cy > y1 || cz > z1) return;
  int2 r = w.cells[cell_hash(mw, cx, cy, cz) & (uint32_t)w.cell_mask];
  for (int j = r.x; j < r.y; ++j) {
    if (j == i) continue;
    int bm = w.bp_meta[j];
    int b = bm & kMetaId;
    if ((bm & kMetaMoved) && b < m) continue;  // the smaller moved proxy of a pair reports it
    if (m_static && (bm & kMetaStatic)) continue;
    float4 B = w.bp_xy[j];
    if (A.y < B.x || A.x > B.y) continue;  // aabb_overlaps (collision/aabb.rs:903), axis by axis
    if (A.w < B.z || A.z > B.w) continue;
    float2 Bz = w.bp_z[j];
    if (Az.y < Bz.x || Az.x > Bz.y) continue;
    if (grid_coord(B.x, w.inv_cell) != cx || grid_coord(B.z, w.inv_cell) != cy ||
        grid_coord(Bz.x, w.inv_cell) != cz || w.bp_world[j] != mw)
      continue;
    emit_overlapping_pair(w, m, b);
  }
}

__global__ void k_bp_large(DW w) {
  if (w.ctl->moved_count == 0 || w.n_large == 0) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= w.n_shapes) return;
  const DShape& S = w.shapes[s];
  if (S.is_static && (w.fat[s].hi.x - w.fat[s].lo.x) > 8.0f) return;  // large itself
  if (S.is_static) return;                                             // static vs static
  for (int k = w.large_off[S.world]; k < w.large_off[S.world + 1]; ++k) {
    int L = w.large_list[k];
    if (!w.moved[s] && !w.moved[L]) continue;
    emit_pair(w, s, L);
  }
}

__global__ void k_bp_scatter(DW w) {
  int n = w.ctl->cand_count;
  if (n > w.cand_cap) n = w.cand_cap;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned long long k = w.cand[i];
    int lo = (int)((k >> 42) & ((1ull << 22) - 1ull));
    int pos = w.seg_off[lo] + atomicAdd(&w.seg_cursor[lo], 1);
    w.sorted_keys[pos] = k;
  }
}

// Each shape's candidate segment is sorted by its pair keys. Short segments (most of them) are
// sorted by one thread; longer ones (a large shape meeting many new partners at once, such as
// a ground box on the first step) are listed for k_bp_segsort_long, which sorts each with one
// block in shared memory.
constexpr int kShortSegment = 32, kLongSegmentCap = 256, kLongSegmentKeys = 8192;

__device__ void insertion_sort_keys(unsigned long long* a, int n) {
  for (int i = 1; i < n; ++i) {
    unsigned long long v = a[i];
    int j = i - 1;
    while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; --j; }
    a[j + 1] = v;
  }
}

__global__ void k_bp_segsort(DW w) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= w.n_shapes) return;
  int n = w.seg_count[s];
  if (n < 2) return;
  if (n > kShortSegment && n <= kLongSegmentKeys) {
    int slot = atomicAdd(&w.ctl->long_segments, 1);
    if (slot < kLongSegmentCap) {
      w.long_segment[slot] = s;
      return;
    }
  }
  insertion_sort_keys(w.sorted_keys + w.seg_off[s], n);
}

// Bitonic sort of one long segment per block (keys padded to a power of two with the largest
// key; equal keys are equal values, so the result is the segment's sorted order).
__global__ void __launch_bounds__(1024) k_bp_segsort_long(DW w) {
  extern __shared__ unsigned long long keys[];
  int count = min(w.ctl->long_segments, kLongSegmentCap);
  for (int li = blockIdx.x; li < count; li += gridDim.x) {
    int s = w.long_segment[li];
    int n = w.seg_count[s];
    unsigned long long* a = w.sorted_keys + w.seg_off[s];
    int p2 = 1;
    while (p2 < n) p2 <<= 1;
    for (int i = threadIdx.x; i < p2; i += blockDim.x) keys[i] = i < n ? a[i] : ~0ull;
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < p2; i += blockDim.x) {
          int ixj = i ^ j;
          if (ixj > i) {
            unsigned long long x = keys[i], y = keys[ixj];
            bool up = (i & k) == 0;
            if ((x > y) == up) { keys[i] = y; keys[ixj] = x; }
          }
        }
        __syncthreads();
      }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = keys[i];
    __syncthreads();
  }
}

// Six pair kinds, A being the primary shape: sphere-sphere, capsule-sphere, capsule-capsule,
// hull-sphere, hull-capsule, hull-hull.
constexpr int kPairKinds = 6;
// Queues of the narrowphase's update pass: kinds 0..2, the GJK pairs (kinds 3, 4) split by the
// size of their simplex cache and the hull pairs (kind 5) by the type of their SAT cache, so the
// lanes of a warp mostly take the same path through the update. Within a kind the pairs without
// a cache (new pairs: a full SAT or GJK from scratch) get the highest queue, run first.
constexpr int kCollideQueues = 17;
__device__ __forceinline__ int collide_queue(const DContact& c) {
  if (c.kind < 3) return c.kind;
  if (c.kind < 5) return 3 + 4 * (c.kind - 3) + 3 - min((int)c.simplex.count, 3);
  return 11 + 5 - min((int)c.sat.type, 5);
}
__device__ __forceinline__ int pair_kind(int ta, int tb) {
  if (ta == kSphere) return 0;
  if (ta == kCapsule) return tb == kSphere ? 1 : 2;
  return tb == kSphere ? 3 : (tb == kCapsule ? 4 : 5);
}

// contact_creation.rs:219 create_contact. Contact ids come from the LIFO id pool
// (id_pool.rs): the k-th new pair in key order takes the k-th id popped.
// First sorted candidate whose smaller shape is >= shape (candidate keys sort by that shape).
__device__ int first_candidate_of_shape(const DW& w, int n, int shape) {
  unsigned long long v = (unsigned long long)shape << 42;
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (w.sorted_keys[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void k_bp_create(DW w) {
  int n = w.ctl->cand_count;
  if (n > w.cand_cap) n = w.cand_cap;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    unsigned long long key = w.sorted_keys[k];
    int wi = w.shapes[(int)((key >> 42) & ((1ull << 22) - 1ull))].world;
    // the pair's rank among its sub-world's new pairs decides which id it pops
    int rank = k - first_candidate_of_shape(w, n, w.world_shape[wi]);
    int base = w.world_cbase[wi];
    int F = w.pool_top[wi], N0 = w.pool_next[wi];
    int local = rank < F ? -1 : N0 + (rank - F);
    if (local >= w.world_cbase[wi + 1] - base) { raise_error(w.ctl, kErrCapacity); continue; }
    int id = rank < F ? w.free_stack[base + F - 1 - rank] : base + local;
    int sa = (int)((key >> 42) & ((1ull << 22) - 1ull));
    int sb = (int)((key >> 20) & ((1ull << 22) - 1ull));
    int ta = w.shapes[sa].type, tb = w.shapes[sb].type;
    // contact_creation.rs:65 registers: capsule > sphere, hull > sphere, hull > capsule
    bool primary = ta == tb || (ta == kCapsule && tb == kSphere) ||
                   (ta == kHull && (tb == kSphere || tb == kCapsule));
    if (!primary) { int t = sa; sa = sb; sb = t; }
    const DShape& A = w.shapes[sa];
    const DShape& B = w.shapes[sb];
    DContact c;
    memset(&c, 0, sizeof(c));
    c.shape_a = sa; c.shape_b = sb;
    c.body_a = A.body; c.body_b = B.body;
    c.enc_a = A.enc; c.enc_b = B.enc;
    c.color = -1; c.local = -1; c.alive = 1;
    c.kind = pair_kind(A.type, B.type);
    const DSim& simA = sim_of(w, A.enc);
    const DSim& simB = sim_of(w, B.enc);
    uint32_t flags = 0;
    if (A.is_static || B.is_static) flags |= cStatic;
    flags |= cSpeculative;
    if ((simA.flags & kEnableRecycling) && (simB.flags & kEnableRecycling)) flags |= cRecycle;
    c.flags = flags;
    float ra = A.type == kSphere ? A.sphere.radius : (A.type == kCapsule ? A.capsule.radius : 0.0f);
    float rb = B.type == kSphere ? B.sphere.radius : (B.type == kCapsule ? B.capsule.radius : 0.0f);
    c.rolling = maxf(A.rolling, B.rolling) * maxf(ra, rb);
    c.sat = SATCache();
    c.simplex = SimplexCache();
    w.contacts[id] = c;
    w.slot_state[id] = slot_state_of(true, false, -1);
    hs_insert(w, key);
  }
}

// Per sub-world pool update for the pairs k_bp_create just made.
__global__ void k_bp_pools(DW w) {
  int wi = blockIdx.x * blockDim.x + threadIdx.x;
  if (wi >= w.n_worlds) return;
  int n = w.ctl->cand_count;
  if (n > w.cand_cap) n = w.cand_cap;
  int nw = first_candidate_of_shape(w, n, w.world_shape[wi + 1]) - first_candidate_of_shape(w, n, w.world_shape[wi]);
  int F = w.pool_top[wi], N0 = w.pool_next[wi];
  w.pool_top[wi] = F > nw ? F - nw : 0;
  w.pool_next[wi] = N0 + (nw > F ? nw - F : 0);
}

__global__ void k_bp_finish(DW w) {
  Control* c = w.ctl;
  int n = c->cand_count;
  if (n > w.cand_cap) n = w.cand_cap;
  c->new_pairs = n;
  c->cand_count = 0;
  c->moved_count = 0;
  c->recycled = 0;
  c->hs_rebuild = 0;
}

// ---------------------------------------------------------------------------
// Narrowphase (collide_pass.rs:541 collide_one_contact, contact_update.rs:43-468)

__device__ bool update_contact(const DW& w, DContact& c, V3 lca, WXf xa, V3 lcb, WXf xb) {
  const DShape& A = w.shapes[c.shape_a];
  const DShape& B = w.shapes[c.shape_b];
  LocalManifold lm;
  Xf b2a = inv_mul_wxf(xa, xb);
  if (A.type == kSphere) {
    collide_spheres(&lm, A.sphere, B.sphere, b2a);
  } else if (A.type == kCapsule) {
    if (B.type == kSphere) collide_capsule_sphere(&lm, A.capsule, B.sphere, b2a);
    else collide_capsules(&lm, A.capsule, B.capsule, b2a);
  } else {
    const Hull& ha = w.hulls[A.hull];
    if (B.type == kSphere) collide_hull_sphere(&lm, ha, B.sphere, b2a, &c.simplex);
    else if (B.type == kCapsule) collide_hull_capsule(&lm, ha, B.capsule, b2a, &c.simplex);
    else collide_hulls(&lm, ha, w.hulls[B.hull], b2a, &c.sat, nullptr);
  }
  if (lm.point_count == 0) {
    c.manifold_count = 0;
    c.flags &= ~cSimTouching;
    return false;
  }
  ManifoldPoint old_points[4];
  int old_count = 0;
  if (c.manifold_count == 0) {
    memset(&c.manifold, 0, sizeof(Manifold));
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
    memset(&t, 0, sizeof(t));
    t.anchor_a = mul_mv(ma, lm.points[i].point);
    t.anchor_b = t.anchor_a + sub_pos(xa.p, xb.p);
    t.separation = lm.points[i].separation;
    t.feature_id = make_feature_id(lm.points[i].pair);
    m.points[i] = t;
  }
  for (int i = 0; i < lm.point_count; ++i) {
    ManifoldPoint p2 = m.points[i];
    p2.total_normal_impulse = 0.0f;
    p2.persisted = 0;
    for (int j = 0; j < old_count; ++j) {
      if (p2.feature_id == old_points[j].feature_id) {
        p2.normal_impulse = old_points[j].normal_impulse;
        p2.persisted = 1;
        old_points[j].feature_id = 0xffffffffu;
        break;
      }
    }
    if (!p2.persisted) p2.normal_impulse = 0.0f;
    m.points[i] = p2;
  }
  // world_runtime.rs:1305 mix_friction / mix_restitution
  c.friction = sqrtf(A.friction * B.friction);
  c.restitution = maxf(A.restitution, B.restitution);
  if (A.rolling > 0.0f || B.rolling > 0.0f) {
    float rA = A.type == kSphere ? A.sphere.radius
               : (A.type == kCapsule ? A.capsule.radius : 0.25f * w.hulls[A.hull].inner_radius);
    float rB = B.type == kSphere ? B.sphere.radius
               : (B.type == kCapsule ? B.capsule.radius : 0.25f * w.hulls[B.hull].inner_radius);
    c.rolling = maxf(A.rolling, B.rolling) * maxf(rA, rB);
  } else {
    c.rolling = 0.0f;
  }
  V3 tva = rotate(xa.q, v3(0, 0, 0));
  V3 tvb = rotate(xb.q, v3(0, 0, 0));
  c.tangent_velocity = tva - tvb;
  V3 ca = rotate(xa.q, lca), cb = rotate(xb.q, lcb);
  for (int j = 0; j < m.point_count; ++j) {
    m.points[j].anchor_a = m.points[j].anchor_a - ca;
    m.points[j].anchor_b = m.points[j].anchor_b - cb;
  }
  c.flags |= cSimTouching;
  return true;
}

// collide_pass.rs:541 collide_one_contact, first half, for one live contact: the AABB
// re-check and the recycling test (collide_pass.rs:606-687). Returns true when the contact
// needs a full manifold update (collide_full).
__device__ bool collide_recycle(const DW& w, int cid) {
  DContact& c = w.contacts[cid];
  // Every read is issued before the first write, in two dependent rounds (the contact, then
  // its shapes' fat AABBs and its bodies' poses): the contact and body records are far apart in
  // memory and mostly come from DRAM, so one round trip per field would dominate the pass.
  const int shape_a = c.shape_a, shape_b = c.shape_b, enc_a = c.enc_a, enc_b = c.enc_b;
  const uint32_t flags = c.flags;
  const int manifold_count = c.manifold_count;
  const Q cached_rot_a = c.cached_rot_a, cached_rot_b = c.cached_rot_b;
  const Xf xc = c.cached_rel;
  const int point_count = c.manifold.point_count;
  const V3 n = c.manifold.normal;
  V3 anchor_a[4], anchor_b[4];
  float base_sep[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    anchor_a[i] = c.manifold.points[i].anchor_a;
    anchor_b[i] = c.manifold.points[i].anchor_b;
    base_sep[i] = c.manifold.points[i].base_separation;
  }
  const AABB fat_a = w.fat[shape_a], fat_b = w.fat[shape_b];
  const DSim& sa = sim_of(w, enc_a);
  const DSim& sb = sim_of(w, enc_b);
  WXf xa, xb;
  xa.p.x = sa.px; xa.p.y = sa.py; xa.p.z = sa.pz; xa.q = sa.q;
  xb.p.x = sb.px; xb.p.y = sb.py; xb.p.z = sb.pz; xb.q = sb.q;
  const uint32_t flags_a = sa.flags, flags_b = sb.flags;
  const V3 max_extent_a = sa.max_extent, max_extent_b = sb.max_extent;
  const Pos ca = {sa.cx, sa.cy, sa.cz}, cb = {sb.cx, sb.cy, sb.cz};
  if (!aabb_overlaps(fat_a, fat_b)) {
    c.flags = (flags | cSimDisjoint) & ~cSimTouching;
    atomicOr(&w.changed_bits[cid >> 5], 1u << (cid & 31));
    if (w.np_mode) w.np_mode[cid] = 0;
    return false;
  }
  bool was_touching = (flags & cSimTouching) != 0;
  bool is_fast = ((flags_a | flags_b) & kIsFast) != 0;
  float recycle = contact_recycle_distance();
  float spec = speculative_distance();
  float recycle_nt = minf(recycle, spec);
  float tol = was_touching ? recycle : recycle_nt;
  bool recycled = false;
  if (!is_fast && recycle > 0.0f && (flags & cRelativeValid) && (flags & cRecycle)) {
    // collide_pass.rs:606-687 contact recycling
    float ang_a = dot_quat(xa.q, cached_rot_a);
    float ang_b = dot_quat(xb.q, cached_rot_b);
    float ang = minf(ang_a * ang_a, ang_b * ang_b);
    Xf x = inv_mul_wxf(xa, xb);
    V3 mea = enc_a < -1 ? v3(0, 0, 0) : max_extent_a;
    V3 meb = enc_b < -1 ? v3(0, 0, 0) : max_extent_b;
    V3 me = max3(mea, meb);
    float dsq = distance_sq(x.p, xc.p);
    if (ang > kRecycleAngular && dsq < tol * tol) {
      float dist = sqrtf(dsq);
      float slack = tol - dist;
      Q qr = inv_mul_quat(xc.q, x.q);
      V3 arc = modified_cross(abs3(qr.v), me);
      float arc_sq = 4.0f * length_sq(arc);
      if (arc_sq < slack * slack) {
        Q dqa = mul_quat(xa.q, conjugate(cached_rot_a));
        Q dqb = mul_quat(xb.q, conjugate(cached_rot_b));
        M3 ma = matrix_from_quat(dqa), mb = matrix_from_quat(dqb);
        V3 dc = sub_pos(cb, ca);
        if (manifold_count > 0) {
          Manifold& m = c.manifold;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            if (i < point_count) {
              V3 ra = mul_mv(ma, anchor_a[i]);
              V3 rb = mul_mv(mb, anchor_b[i]);
              V3 dp = dc + (rb - ra);
              m.points[i].separation = base_sep[i] + dot(dp, n);
              m.points[i].normal_velocity = 0.0f;
              m.points[i].persisted = 1;
            }
          }
        }
        recycled = true;
        add_converged(&w.ctl->recycled);
        if (w.np_mode) w.np_mode[cid] = 1;
      }
    }
  }
  return !recycled;
}

// collide_pass.rs:541 collide_one_contact, second half: a new manifold from the narrowphase
// routines and the touch transition.
__device__ void collide_full(const DW& w, int cid) {
  DContact& c = w.contacts[cid];
  const DSim& sa = sim_of(w, c.enc_a);
  const DSim& sb = sim_of(w, c.enc_b);
  bool was_touching = (c.flags & cSimTouching) != 0;
  WXf xa, xb;
  xa.p.x = sa.px; xa.p.y = sa.py; xa.p.z = sa.pz; xa.q = sa.q;
  xb.p.x = sb.px; xb.p.y = sb.py; xb.p.z = sb.pz; xb.q = sb.q;
  bool changed = false;
  {
    c.cached_rot_a = xa.q;
    c.cached_rot_b = xb.q;
    c.cached_rel = inv_mul_wxf(xa, xb);
    c.flags |= cRelativeValid;
    bool touching = update_contact(w, c, sa.local_center, xa, sb.local_center, xb);
    if (w.np_mode) w.np_mode[cid] = touching ? 2 : 3;
    if (touching && !was_touching) { c.flags |= cSimStarted; changed = true; }
    else if (!touching && was_touching) { c.flags |= cSimStopped; changed = true; }
    if (touching && c.manifold_count > 0) {
      for (int i = 0; i < c.manifold.point_count; ++i)
        c.manifold.points[i].base_separation = c.manifold.points[i].separation;
    }
  }
  if (changed) atomicOr(&w.changed_bits[cid >> 5], 1u << (cid & 31));
}

// Narrowphase, first pass over all contact slots: recycle what can be recycled and queue the
// rest by pair kind.
constexpr int kCollideThreads = 256;
__global__ void __launch_bounds__(kCollideThreads) k_collide(DW w) {
  for (int cid = blockIdx.x * blockDim.x + threadIdx.x; cid < w.cap; cid += gridDim.x * blockDim.x) {
    if (!(w.slot_state[cid] & kSlotAlive)) continue;
    if (collide_recycle(w, cid)) {
      int q = collide_queue(w.contacts[cid]);
      int slot = slot_converged(w.ctl->collide_count, q);
      w.collide_list[(size_t)q * w.cap + slot] = cid;
    }
  }
}

// Narrowphase, second pass: full updates, kind by kind, so a warp runs one shape
// combination. Contacts are independent here: the order only changes which warp runs what.
// The queues go from the costliest (the hull pairs) to the cheapest (sphere-sphere), so the
// last blocks to start are the short ones and the launch does not wait on a tail of hull pairs.
// Small blocks spread the updates over every SM: a thread keeps ~2 KB of clip polygons on its
// stack, and fewer warps per SM keep more of it in L1. The minimum of one block per SM lets the
// compiler keep the manifold routines in 213 registers without spills (it targets 168 with
// spills otherwise).
constexpr int kCollideUpdateThreads = 64;
__global__ void __launch_bounds__(kCollideUpdateThreads, 1) k_collide_update(DW w) {
  __shared__ int start[kCollideQueues + 1];
  if (threadIdx.x == 0) {  // start[r]: first item of the r-th queue in cost order (queue 16 - r)
    int acc = 0;
    for (int r = 0; r < kCollideQueues; ++r) { start[r] = acc; acc += w.ctl->collide_count[kCollideQueues - 1 - r]; }
    start[kCollideQueues] = acc;
  }
  __syncthreads();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < start[kCollideQueues]; t += gridDim.x * blockDim.x) {
    int r = 0;
    while (t >= start[r + 1]) ++r;
    collide_full(w, w.collide_list[(size_t)(kCollideQueues - 1 - r) * w.cap + (t - start[r])]);
  }
}

// ---------------------------------------------------------------------------
// Ordered state pass (collide_pass.rs:386) with greedy coloring
// (constraint_graph.rs:113/200). One block: the changed ids are compacted in id order,
// then one thread applies the transitions in that order, keeping every body's color
// membership as a 24-bit mask (bit c == the reference's colors[c].body_set bit).

// collide_pass.rs:386-430: contact state changes in contact-id order. Begin-touch adds the
// contact to the constraint graph (constraint_graph.rs:113 greedy color from the bodies'
// color masks), end-touch removes it (:200), disjoint contacts are destroyed
// (contact_creation.rs:428). The coloring is order dependent, so one thread walks the
// changes; the contact fields it needs are staged in shared memory by the whole block
// chunk by chunk, and the results are written back by the whole block.
constexpr int kStateChunk = 2048;
struct StateStage {
  int* cid; uint32_t* flags; int* info; int* ba; int* bb;
};
// info: bits 0..7 color + 1 (0 = none), bit 8 dynamic A, bit 9 dynamic B; after the walk
// bits 16..23 hold the new color + 1 and bit 24 marks a destroyed contact.
template <typename MaskT>
__device__ int state_walk(const DW& w, MaskT mask, const StateStage& st, int n, int ovf) {
  for (int i = 0; i < n; ++i) {
    uint32_t f = st.flags[i];
    int info = st.info[i];
    int old_color = (info & 255) - 1;
    int a = st.ba[i], b = st.bb[i];
    int cid = st.cid[i];
    int new_color = old_color, destroyed = 0;
    auto remove = [&](int color) {  // constraint_graph.rs:200
      if (color != kOverflowIndex) {
        mask[a] &= ~(1u << color);
        mask[b] &= ~(1u << color);
      } else {
        int local = w.contacts[cid].local;
        int last = ovf - 1;
        if (local != last) {
          int moved = w.overflow_list[last];
          w.overflow_list[local] = moved;
          w.contacts[moved].local = local;
        }
        ovf = last;
      }
    };
    if (f == 0) {
    } else if (f & cSimDisjoint) {
      if (old_color != -1) remove(old_color);
      new_color = -1;
      destroyed = 1;
    } else if (f & cSimStarted) {
      bool dyn_a = (info >> 8) & 1, dyn_b = (info >> 9) & 1;
      int color = kOverflowIndex;
      if (dyn_a && dyn_b) {
        uint32_t avail = ~(mask[a] | mask[b]) & ((1u << kDynamicColorCount) - 1u);
        if (avail) {
          color = __ffs(avail) - 1;
          mask[a] |= 1u << color;
          mask[b] |= 1u << color;
        }
      } else {
        int d = dyn_a ? a : b;
        uint32_t avail = ~mask[d] & (((1u << kOverflowIndex) - 1u) & ~1u);  // colors 22..1
        if (avail) {
          color = 31 - __clz(avail);
          mask[d] |= 1u << color;
        }
      }
      new_color = color;
      if (color == kOverflowIndex) {
        w.contacts[cid].local = ovf;
        w.overflow_list[ovf] = cid;
        ovf++;
      }
    } else if (f & cSimStopped) {
      remove(old_color);
      new_color = -1;
    }
    st.info[i] = (info & 0xffff) | ((new_color + 1) << 16) | (destroyed << 24);
  }
  return ovf;
}

// The same transitions with the whole block, in rounds: a change is applied once it is the
// lowest-numbered change still pending on each of its dynamic bodies (minp[body], kept in shared
// memory), so every body's mask sees its changes in id order, as in state_walk, and changes on
// disjoint bodies run together. Static and kinematic bodies never hold colour bits, so only
// dynamic bodies order the changes. Edits of the overflow list depend on the order of all of
// them, so the rounds only mark them (bit 26 append, bit 27 remove) and one thread applies them
// in id order afterwards. Bit 25 marks an applied change. Returns the new overflow count.
constexpr int kStateDone = 1 << 25, kStateOvfAppend = 1 << 26, kStateOvfRemove = 1 << 27;
__device__ int state_walk_rounds(const DW& w, uint32_t* mask, int* minp, const StateStage& st, int n, int ovf) {
  const int t = threadIdx.x;
  for (;;) {
    int pending = 0;
    for (int i = t; i < n; i += kStatePassThreads) {
      int info = st.info[i];
      if (info & kStateDone) continue;
      pending = 1;
      if ((info >> 8) & 1) atomicMin(&minp[st.ba[i]], i);
      if ((info >> 9) & 1) atomicMin(&minp[st.bb[i]], i);
    }
    if (!__syncthreads_or(pending)) break;
    for (int i = t; i < n; i += kStatePassThreads) {
      int info = st.info[i];
      if (info & kStateDone) continue;
      const bool dyn_a = (info >> 8) & 1, dyn_b = (info >> 9) & 1;
      const int a = st.ba[i], b = st.bb[i];
      if ((dyn_a && minp[a] != i) || (dyn_b && minp[b] != i)) continue;
      uint32_t f = st.flags[i];
      int old_color = (info & 255) - 1;
      int new_color = old_color, destroyed = 0, ovf_op = 0;
      auto remove = [&](int color) {  // constraint_graph.rs:200
        if (color != kOverflowIndex) {
          if (dyn_a) mask[a] &= ~(1u << color);
          if (dyn_b) mask[b] &= ~(1u << color);
        } else {
          ovf_op = kStateOvfRemove;
        }
      };
      if (f == 0) {
      } else if (f & cSimDisjoint) {
        if (old_color != -1) remove(old_color);
        new_color = -1;
        destroyed = 1;
      } else if (f & cSimStarted) {
        int color = kOverflowIndex;
        if (dyn_a && dyn_b) {
          uint32_t avail = ~(mask[a] | mask[b]) & ((1u << kDynamicColorCount) - 1u);
          if (avail) {
            color = __ffs(avail) - 1;
            mask[a] |= 1u << color;
            mask[b] |= 1u << color;
          }
        } else {
          int d = dyn_a ? a : b;
          uint32_t avail = ~mask[d] & (((1u << kOverflowIndex) - 1u) & ~1u);  // colors 22..1
          if (avail) {
            color = 31 - __clz(avail);
            mask[d] |= 1u << color;
          }
        }
        new_color = color;
        if (color == kOverflowIndex) ovf_op = kStateOvfAppend;
      } else if (f & cSimStopped) {
        remove(old_color);
        new_color = -1;
      }
      st.info[i] = (info & 0xffff) | ((new_color + 1) << 16) | (destroyed << 24) | kStateDone | ovf_op;
    }
    __syncthreads();
    for (int i = t; i < n; i += kStatePassThreads) {
      minp[st.ba[i]] = INT_MAX;
      minp[st.bb[i]] = INT_MAX;
    }
    __syncthreads();
  }
  __shared__ int ovf_s2;
  if (t == 0) {
    for (int i = 0; i < n; ++i) {
      int info = st.info[i];
      int cid = st.cid[i];
      if (info & kStateOvfRemove) {
        int local = w.contacts[cid].local;
        int last = ovf - 1;
        if (local != last) {
          int moved = w.overflow_list[last];
          w.overflow_list[local] = moved;
          w.contacts[moved].local = local;
        }
        ovf = last;
      } else if (info & kStateOvfAppend) {
        w.contacts[cid].local = ovf;
        w.overflow_list[ovf] = cid;
        ovf++;
      }
    }
    ovf_s2 = ovf;
  }
  __syncthreads();
  return ovf_s2;
}

__global__ void __launch_bounds__(kStatePassThreads) k_state_pass(DW w, int use_shared) {
  extern __shared__ uint32_t dyn_smem[];
  typedef cub::BlockScan<int, kStatePassThreads> Scan;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ int total_s, ovf_s;
  int t = threadIdx.x;
  int per = (w.n_words + kStatePassThreads - 1) / kStatePassThreads;
  int w0 = t * per, w1 = min(w0 + per, w.n_words);
  int mine = 0;
  for (int k = w0; k < w1; ++k) mine += __popc(w.changed_bits[k]);
  int off, total;
  Scan(scan_tmp).ExclusiveSum(mine, off, total);
  for (int k = w0; k < w1; ++k) {
    uint32_t bits = w.changed_bits[k];
    while (bits) {
      int b = __ffs(bits) - 1;
      w.changed_list[off++] = (k << 5) + b;
      bits &= bits - 1;
    }
    w.changed_bits[k] = 0;
  }
  if (t == 0) { total_s = total; w.ctl->changed_count = total; ovf_s = w.ovf_count[0]; }
  __syncthreads();
  total = total_s;
  if (total == 0) return;
  StateStage st;
  st.cid = (int*)dyn_smem;
  st.flags = (uint32_t*)(st.cid + kStateChunk);
  st.info = (int*)(st.flags + kStateChunk);
  st.ba = st.info + kStateChunk;
  st.bb = st.ba + kStateChunk;
  uint32_t* smask = (uint32_t*)(st.bb + kStateChunk);
  int* minp = (int*)(smask + w.n_bodies);  // use_shared == 2: the rounds' per-body minimum
  if (use_shared) {
    for (int b = t; b < w.n_bodies; b += kStatePassThreads) smask[b] = w.body_mask[b];
  }
  if (use_shared == 2) {
    for (int b = t; b < w.n_bodies; b += kStatePassThreads) minp[b] = INT_MAX;
  }
  for (int base = 0; base < total; base += kStateChunk) {
    int n = min(kStateChunk, total - base);
    for (int i = t; i < n; i += kStatePassThreads) {
      int cid = w.changed_list[base + i];
      const DContact& c = w.contacts[cid];
      st.cid[i] = cid;
      st.flags[i] = c.flags;
      st.ba[i] = c.body_a;
      st.bb[i] = c.body_b;
      st.info[i] = (c.color + 1) | ((int)w.body_dyn[c.body_a] << 8) | ((int)w.body_dyn[c.body_b] << 9);
    }
    __syncthreads();
    if (use_shared == 2) {
      int o = state_walk_rounds(w, smask, minp, st, n, ovf_s);
      if (t == 0) ovf_s = o;
    } else if (t == 0) {
      ovf_s = use_shared ? state_walk(w, smask, st, n, ovf_s) : state_walk(w, w.body_mask, st, n, ovf_s);
    }
    __syncthreads();
    for (int i = t; i < n; i += kStatePassThreads) {
      DContact& c = w.contacts[st.cid[i]];
      uint32_t f = st.flags[i];
      int info = st.info[i];
      int color = ((info >> 16) & 255) - 1;
      int destroyed = (info >> 24) & 1;
      if (f == 0) {
      } else if (f & cSimDisjoint) {
        c.manifold_count = 0;
        c.alive = 0;
        c.color = -1;
        c.local = -1;
        w.slot_state[st.cid[i]] = slot_state_of(false, false, -1);
      } else if (f & cSimStarted) {
        c.flags = (f & ~cSimStarted) | cTouching;
        c.color = color;
        if (color != kOverflowIndex) c.local = -1;
        w.slot_state[st.cid[i]] = slot_state_of(true, true, color);
      } else if (f & cSimStopped) {
        c.flags = f & ~(cSimStopped | cTouching);
        c.color = -1;
        c.local = -1;
        w.slot_state[st.cid[i]] = slot_state_of(true, false, -1);
      }
      w.destroyed[base + i] = destroyed;
    }
    __syncthreads();
  }
  if (use_shared) {
    for (int b = t; b < w.n_bodies; b += kStatePassThreads) w.body_mask[b] = smask[b];
  }
  if (t == 0) { w.ovf_count[0] = ovf_s; w.ctl->overflow_count = ovf_s; }
  __syncthreads();
  // Destroyed ids go back on the LIFO pool in id order (contact_creation.rs:543 free).
  int nd = 0;
  int per2 = (total + kStatePassThreads - 1) / kStatePassThreads;
  int i0 = t * per2, i1 = min(i0 + per2, total);
  for (int i = i0; i < i1; ++i) nd += w.destroyed[i];
  int doff, dtotal;
  __syncthreads();
  Scan(scan_tmp).ExclusiveSum(nd, doff, dtotal);
  int top = w.pool_top[0];
  for (int i = i0; i < i1; ++i) {
    if (!w.destroyed[i]) continue;
    int cid = w.changed_list[i];
    w.free_stack[top + doff] = cid;
    doff++;
    const DContact& c = w.contacts[cid];
    hs_erase(w, pair_key(c.shape_a, c.shape_b));
  }
  __syncthreads();
  if (t == 0) {
    w.pool_top[0] = top + dtotal;
    w.ctl->hs_rebuild = w.ctl->tombstones > (w.hs_mask + 1) / 4 ? 1 : 0;
    if (w.ctl->hs_rebuild) w.ctl->tombstones = 0;
  }
}

// The ordered state pass for several sub-worlds: one thread per sub-world walks the changed
// contacts of its own id range in id order (its bitmap words), with the same transitions as
// k_state_pass, its own overflow list and its own id pool. Sub-worlds share no bodies, so
// their walks are independent. ctl->changed_count and ctl->overflow_count are zeroed before.
__global__ void k_state_worlds(DW w) {
  int wi = blockIdx.x * blockDim.x + threadIdx.x;
  if (wi >= w.n_worlds) return;
  int base = w.world_cbase[wi], end = w.world_cbase[wi + 1];
  int ovf = w.ovf_count[wi], top = w.pool_top[wi], changes = 0;
  int* olist = w.overflow_list + base;
  for (int word = base >> 5; word < (end >> 5); ++word) {
    uint32_t bits = w.changed_bits[word];
    if (!bits) continue;
    w.changed_bits[word] = 0;
    while (bits) {
      int cid = (word << 5) + __ffs(bits) - 1;
      bits &= bits - 1;
      ++changes;
      DContact& c = w.contacts[cid];
      uint32_t f = c.flags;
      auto remove = [&](int color) {  // constraint_graph.rs:200
        if (color != kOverflowIndex) {
          w.body_mask[c.body_a] &= ~(1u << color);
          w.body_mask[c.body_b] &= ~(1u << color);
        } else {
          int local = c.local, last = ovf - 1;
          if (local != last) {
            int moved = olist[last];
            olist[local] = moved;
            w.contacts[moved].local = local;
          }
          ovf = last;
        }
      };
      if (f == 0) {
      } else if (f & cSimDisjoint) {  // contact_creation.rs:428 destroy_contact
        if (c.color != -1) remove(c.color);
        c.manifold_count = 0;
        c.alive = 0;
        c.color = -1;
        c.local = -1;
        w.slot_state[cid] = slot_state_of(false, false, -1);
        w.free_stack[base + top++] = cid;  // contact_creation.rs:543: ids go back in id order
        hs_erase(w, pair_key(c.shape_a, c.shape_b));
      } else if (f & cSimStarted) {   // constraint_graph.rs:113 add_contact_to_graph
        c.flags = (f & ~cSimStarted) | cTouching;
        bool dyn_a = w.body_dyn[c.body_a] != 0, dyn_b = w.body_dyn[c.body_b] != 0;
        int color = kOverflowIndex;
        if (dyn_a && dyn_b) {
          uint32_t avail = ~(w.body_mask[c.body_a] | w.body_mask[c.body_b]) & ((1u << kDynamicColorCount) - 1u);
          if (avail) {
            color = __ffs(avail) - 1;
            w.body_mask[c.body_a] |= 1u << color;
            w.body_mask[c.body_b] |= 1u << color;
          }
        } else {
          int d = dyn_a ? c.body_a : c.body_b;
          uint32_t avail = ~w.body_mask[d] & (((1u << kOverflowIndex) - 1u) & ~1u);  // colors 22..1
          if (avail) {
            color = 31 - __clz(avail);
            w.body_mask[d] |= 1u << color;
          }
        }
        c.color = color;
        w.slot_state[cid] = slot_state_of(true, true, color);
        if (color == kOverflowIndex) {
          c.local = ovf;
          olist[ovf++] = cid;
        } else {
          c.local = -1;
        }
      } else if (f & cSimStopped) {
        c.flags = f & ~(cSimStopped | cTouching);
        int color = c.color;
        remove(color);
        c.color = -1;
        c.local = -1;
        w.slot_state[cid] = slot_state_of(true, false, -1);
      }
    }
  }
  w.ovf_count[wi] = ovf;
  w.pool_top[wi] = top;
  if (changes) atomicAdd(&w.ctl->changed_count, changes);
  if (ovf) atomicAdd(&w.ctl->overflow_count, ovf);
}

// After k_state_worlds: rebuild the pair set when erased slots pass a quarter.
__global__ void k_state_finish(DW w) {
  w.ctl->hs_rebuild = w.ctl->tombstones > (w.hs_mask + 1) / 4 ? 1 : 0;
  if (w.ctl->hs_rebuild) w.ctl->tombstones = 0;
}

// ---------------------------------------------------------------------------
// Color partition and constraint preparation (solver_prepare.rs:269/335,
// contact_solver.rs:445 prepare_contact_constraint). Constraints of color c occupy
// slots [color_offset[c], color_offset[c+1]); order inside a color does not change
// results because a color's constraints share no dynamic body.

__device__ __forceinline__ int colored_color(const DContact& c) {
  return (c.alive && (c.flags & cTouching) && c.color >= 0 && c.color < kOverflowIndex) ? c.color : -1;
}

__global__ void __launch_bounds__(kColorBlock) k_color_count(DW w) {
  __shared__ int wc[kColorBlock / 32][24];
  int cid = blockIdx.x * kColorBlock + threadIdx.x;
  int col = cid < w.cap ? slot_color_of(w.slot_state[cid]) : -1;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < kOverflowIndex; ++k) {
    unsigned m = __ballot_sync(0xffffffffu, col == k);
    if (lane == 0) wc[warp][k] = __popc(m);
  }
  __syncthreads();
  if (threadIdx.x < kOverflowIndex) {
    int s = 0;
    for (int q = 0; q < kColorBlock / 32; ++q) s += wc[q][threadIdx.x];
    w.block_color[blockIdx.x * 24 + threadIdx.x] = s;
  }
}

// Exclusive prefix over the partition blocks of each colour's counts: block c scans colour c's
// column. Thread t owns a run of consecutive partition blocks; the runs' sums are scanned
// across the block (warp shuffles, then the warps' totals) and each thread writes its run's
// prefixes. The colour offsets follow from the totals (k_color_scatter).
constexpr int kColorScanThreads = 1024;
__global__ void __launch_bounds__(kColorScanThreads) k_color_scan(DW w) {
  __shared__ int warp_sum[kColorScanThreads / 32];
  const int k = blockIdx.x;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int nb = w.n_color_blocks;
  const int per = (nb + kColorScanThreads - 1) / kColorScanThreads;
  const int b0 = min(nb, t * per), b1 = min(nb, b0 + per);
  int own = 0;
  for (int b = b0; b < b1; ++b) own += w.block_color[b * 24 + k];
  int x = own;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int s0 = warp_sum[lane], z = s0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += y;
    }
    warp_sum[lane] = z - s0;  // exclusive prefix of the warps
    if (lane == 31) w.ctl->color_count[k] = z;
  }
  __syncthreads();
  int run = warp_sum[warp] + x - own;  // exclusive prefix of this thread's run
  for (int b = b0; b < b1; ++b) {
    int v = w.block_color[b * 24 + k];
    w.block_color[b * 24 + k] = run;
    run += v;
  }
}

__device__ __forceinline__ DState* state_ptr(const DW& w, int i) { return &w.states[i]; }
__device__ __forceinline__ DState state_at(const DW& w, int i) {
  if (i >= 0) return *state_ptr(w, i);
  DState s;
  s.v = v3(0, 0, 0); s.w = v3(0, 0, 0); s.dp = v3(0, 0, 0); s.flags = 0; s.dq = qid();
  s.pad1 = 0; s.pad2 = 0;
  return s;
}

__device__ void prepare_constraint(const DW& w, const StepParams& p, int cid, int slot) {
  const DContact& ct = w.contacts[cid];
  const CPlanes& P = w.cp;
  float inv_tau = 1.0f / speculative_distance();
  float ws = p.warm_start;
  // The contact's fields, then its bodies' masses, are read before the first plane is written:
  // with the writes in between, each read would wait for its own trip to DRAM.
  const int enc_a = ct.enc_a, enc_b = ct.enc_b;
  const uint32_t flags = ct.flags;
  const float rolling = ct.rolling, friction = ct.friction, restitution = ct.restitution;
  const V3 tangent_velocity = ct.tangent_velocity;
  const Manifold& man = ct.manifold;
  const V3 n = man.normal;
  const float twist_impulse = man.twist_impulse;
  const V3 rolling_impulse = man.rolling_impulse, friction_impulse = man.friction_impulse;
  const int pc = man.point_count;
  V3 ra_[4], rb_[4];
  float sep_[4], nimp_[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    ra_[i] = man.points[i].anchor_a;
    rb_[i] = man.points[i].anchor_b;
    sep_[i] = man.points[i].separation;
    nimp_[i] = man.points[i].normal_impulse;
  }
  int ia = enc_a >= 0 ? enc_a : -1;
  int ib = enc_b >= 0 ? enc_b : -1;
  float ima = 0.0f, imb = 0.0f;
  Sym sa = sym_zero(), sb = sym_zero();
  if (ia >= 0) { ima = w.asims[ia].inv_mass; sa = sym_from(w.asims[ia].inv_inertia_world); }
  if (ib >= 0) { imb = w.asims[ib].inv_mass; sb = sym_from(w.asims[ib].inv_inertia_world); }
  bool is_static = (flags & cStatic) != 0;
  Sym inv_iab = sym_add(sa, sb);
  Sym rm = rolling > 0.0f ? sym_invert(inv_iab) : sym_zero();
  V3 t1 = perp(n);
  V3 t2 = cross(t1, n);
  float tv1 = dot(tangent_velocity, t1), tv2 = dot(tangent_velocity, t2);
  float twist = ws * twist_impulse;
  V3 rimp = rolling > 0.0f ? ws * rolling_impulse : v3(0, 0, 0);
  V2 fi = v2(ws * dot(friction_impulse, t1), ws * dot(friction_impulse, t2));
  V3 ca = v3(0, 0, 0), cb = v3(0, 0, 0);
  float tw = 0.0f;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i >= pc) break;
    V3 ra = ra_[i], rb = rb_[i];
    float base_sep = sep_[i] - dot(rb - ra, n);
    float weight = clampf(2.0f - sep_[i] * inv_tau, kMinFrictionWeight, 1.0f);
    ca = ca + weight * ra;
    cb = cb + weight * rb;
    tw += weight;
    V3 rna = cross(ra, n), rnb = cross(rb, n);
    float k = ima + imb;
    k += dot(rna, sym_mv(sa, rna));
    k += dot(rnb, sym_mv(sb, rnb));
    float nm = k > 0.0f ? 1.0f / k : 0.0f;
    P.pra[i * P.cap + slot] = make_float4(ra.x, ra.y, ra.z, base_sep);
    P.prb[i * P.cap + slot] = make_float4(rb.x, rb.y, rb.z, nm);
  }
  if (tw > 0.0f) {
    ca = (1.0f / tw) * ca;
    cb = (1.0f / tw) * cb;
  } else {
    ca = v3(0, 0, 0); cb = v3(0, 0, 0);
  }
  float rv[4] = {0, 0, 0, 0};
  if (restitution > 0.0f) {
    DState s_a = state_at(w, ia), s_b = state_at(w, ib);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (i >= pc) break;
      V3 vra = s_a.v + cross(s_a.w, ra_[i]);
      V3 vrb = s_b.v + cross(s_b.w, rb_[i]);
      rv[i] = dot(n, vrb - vra);
    }
    atomicOr(&w.ctl->any_restitution, 1);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i >= pc) break;
    V3 d = ra_[i] - ca;
    float lever = sqrtf(dot(d, d));
    P.pimp[i * P.cap + slot] = make_float4(ws * nimp_[i], 0.0f, lever, rv[i]);
    P.prest[i * P.cap + slot] = 0.0f;
  }
  V3 rta1 = cross(ca, t1), rta2 = cross(ca, t2), rtb1 = cross(cb, t1), rtb2 = cross(cb, t2);
  V3 ia1 = sym_mv(sa, rta1), ia2 = sym_mv(sa, rta2), ib1 = sym_mv(sb, rtb1), ib2 = sym_mv(sb, rtb2);
  float msum = ima + imb;
  float kxx = (msum + dot(rta1, ia1)) + dot(rtb1, ib1);
  float kyy = (msum + dot(rta2, ia2)) + dot(rtb2, ib2);
  float kxy = dot(rta1, ia2) + dot(rtb1, ib2);
  float det2 = kxx * kyy - kxy * kxy;
  bool valid = absf(det2) > 1000.0f * kMinPositive && tw > 0.0f;
  float inv = valid ? 1.0f / det2 : 0.0f;
  float ktw = dot(n, sym_mv(inv_iab, n));
  float twist_mass = ktw > 0.0f ? 1.0f / ktw : 0.0f;
  P.idx[slot] = make_int4(ia, ib, cid, pc | (is_static ? 256 : 0));
  P.mass[slot] = make_float4(ima, imb, friction, restitution);
  P.ia0[slot] = make_float4(sa.xx, sa.xy, sa.xz, sa.yy);
  P.ia1[slot] = make_float4(sa.yz, sa.zz, sb.xx, sb.xy);
  P.ib1[slot] = make_float4(sb.xz, sb.yy, sb.yz, sb.zz);
  P.n[slot] = make_float4(n.x, n.y, n.z, rolling);
  P.t1[slot] = make_float4(t1.x, t1.y, t1.z, tv1);
  P.t2[slot] = make_float4(t2.x, t2.y, t2.z, tv2);
  P.ca[slot] = make_float4(ca.x, ca.y, ca.z, twist_mass);
  P.cb[slot] = make_float4(cb.x, cb.y, cb.z, twist);
  P.tm[slot] = make_float4(inv * kyy, -(inv * kxy), -(inv * kxy), inv * kxx);
  P.fr[slot] = make_float4(fi.x, fi.y, rm.xx, rm.xy);
  P.roll[slot] = make_float4(rimp.x, rimp.y, rimp.z, rm.xz);
  P.rm[slot] = make_float4(rm.yy, rm.yz, rm.zz, 0.0f);
}

// Slot of every coloured contact (its colour's offset, the partition block's prefix, its rank in
// the block); the constraint is prepared by k_prepare_slots in slot order.
__global__ void __launch_bounds__(kColorBlock) k_color_scatter(DW w) {
  __shared__ int wc[kColorBlock / 32][24];
  __shared__ int offset_s[kOverflowIndex + 1];
  if (threadIdx.x == 0) {
    int run = 0;
    for (int c = 0; c < kOverflowIndex; ++c) { offset_s[c] = run; run += w.ctl->color_count[c]; }
    offset_s[kOverflowIndex] = run;
    if (blockIdx.x == 0) {
      for (int c = 0; c <= kOverflowIndex; ++c) w.ctl->color_offset[c] = offset_s[c];
      w.ctl->color_offset[24] = run;
      w.ctl->color_count[kOverflowIndex] = w.ctl->overflow_count;
      w.ctl->any_restitution = 0;
    }
  }
  int cid = blockIdx.x * kColorBlock + threadIdx.x;
  int col = cid < w.cap ? slot_color_of(w.slot_state[cid]) : -1;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned my_mask = 0;
  for (int k = 0; k < kOverflowIndex; ++k) {
    unsigned m = __ballot_sync(0xffffffffu, col == k);
    if (lane == 0) wc[warp][k] = __popc(m);
    if (col == k) my_mask = m;
  }
  __syncthreads();
  if (col < 0) return;
  int before = 0;
  for (int q = 0; q < warp; ++q) before += wc[q][col];
  int rank = __popc(my_mask & ((1u << lane) - 1u));
  int slot = offset_s[col] + w.block_color[blockIdx.x * 24 + col] + before + rank;
  w.slot_cid[slot] = cid;
}

// solver_prepare.rs:269 prepare per constraint slot (small blocks: the arithmetic keeps its
// registers instead of the 64 a 1024-thread block allows, and the planes are written in order).
constexpr int kPrepareThreads = 128;
__global__ void __launch_bounds__(kPrepareThreads) k_prepare_slots(DW w, StepParams p) {
  const int n = w.ctl->color_offset[kOverflowIndex];
  for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x)
    prepare_constraint(w, p, w.slot_cid[slot], slot);
}

// overflow_contact_solver.rs:92 prepare_overflow_contacts
__global__ void k_prepare_overflow(DW w, StepParams p) {
  float ws = p.warm_start;
  float inv_tau = 1.0f / speculative_distance();
  Softness soft = p.contact_softness, stat = p.static_softness;
  for (int wi = blockIdx.x; wi < w.n_worlds; wi += gridDim.x)
  for (int i = w.world_cbase[wi] + threadIdx.x; i < w.world_cbase[wi] + w.ovf_count[wi]; i += blockDim.x) {
    int cid = w.overflow_list[i];
    DContact& ct = w.contacts[cid];
    DOverflow c;
    memset(&c, 0, sizeof(c));
    int ia = ct.enc_a >= 0 ? ct.enc_a : -1;
    int ib = ct.enc_b >= 0 ? ct.enc_b : -1;
    c.contact_id = cid; c.index_a = ia; c.index_b = ib;
    c.inv_ia = m3zero(); c.inv_ib = m3zero();
    if (ia >= 0) { c.inv_mass_a = w.asims[ia].inv_mass; c.inv_ia = w.asims[ia].inv_inertia_world; }
    if (ib >= 0) { c.inv_mass_b = w.asims[ib].inv_mass; c.inv_ib = w.asims[ib].inv_inertia_world; }
    float mA = c.inv_mass_a, mB = c.inv_mass_b;
    M3 iA = c.inv_ia, iB = c.inv_ib;
    c.rolling_mass = invert_matrix(add_mm(iA, iB));
    c.softness = (ct.flags & cStatic) ? stat : soft;
    c.friction = ct.friction; c.restitution = ct.restitution; c.rolling_resistance = ct.rolling;
    bool sample = ct.restitution > 0.0f;
    if (sample) atomicOr(&w.ctl->any_restitution, 1);
    V3 va = v3(0, 0, 0), wa = v3(0, 0, 0), vb = v3(0, 0, 0), wb = v3(0, 0, 0);
    if (sample) {
      if (ia >= 0) { va = w.states[ia].v; wa = w.states[ia].w; }
      if (ib >= 0) { vb = w.states[ib].v; wb = w.states[ib].w; }
    }
    c.manifold_count = ct.manifold_count;
    if (ct.manifold_count > 0) {
      Manifold& man = ct.manifold;
      ManifoldConstraint& mc = c.m;
      int pc = man.point_count;
      V3 nn = man.normal, t1 = perp(nn), t2 = cross(t1, nn);
      mc.point_count = pc; mc.normal = nn; mc.tangent1 = t1; mc.tangent2 = t2;
      mc.tangent_velocity1 = dot(ct.tangent_velocity, t1);
      mc.tangent_velocity2 = dot(ct.tangent_velocity, t2);
      V3 ca = v3(0, 0, 0), cb = v3(0, 0, 0);
      float tw = 0.0f;
      for (int q = 0; q < pc; ++q) {
        ConstraintPoint cp;
        memset(&cp, 0, sizeof(cp));
        const ManifoldPoint& mp = man.points[q];
        cp.r_a = mp.anchor_a; cp.r_b = mp.anchor_b;
        float s = mp.separation;
        cp.base_separation = s - dot(cp.r_b - cp.r_a, nn);
        cp.normal_impulse = ws * mp.normal_impulse;
        V3 ra = cp.r_a, rb = cp.r_b;
        V3 rna = cross(ra, nn), rnb = cross(rb, nn);
        float k = mA + mB + dot(rna, mul_mv(iA, rna)) + dot(rnb, mul_mv(iB, rnb));
        cp.normal_mass = k > 0.0f ? 1.0f / k : 0.0f;
        if (sample) {
          V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
          cp.relative_velocity = dot(nn, vrb - vra);
        } else {
          cp.relative_velocity = 0.0f;
        }
        man.points[q].normal_velocity = 0.0f;
        float weight = clampf(2.0f - s * inv_tau, kMinFrictionWeight, 1.0f);
        ca = mul_add(ca, weight, ra);
        cb = mul_add(cb, weight, rb);
        tw += weight;
        mc.points[q] = cp;
      }
      float iw = 1.0f / tw;
      ca = iw * ca; cb = iw * cb;
      mc.center_a = ca; mc.center_b = cb;
      for (int q = 0; q < pc; ++q) mc.points[q].lever_arm = distance(mc.points[q].r_a, ca);
      V3 rta1 = cross(ca, t1), rta2 = cross(ca, t2), rtb1 = cross(cb, t1), rtb2 = cross(cb, t2);
      M2 k;
      k.cx.x = mA + mB + dot(rta1, mul_mv(iA, rta1)) + dot(rtb1, mul_mv(iB, rtb1));
      k.cy.y = mA + mB + dot(rta2, mul_mv(iA, rta2)) + dot(rtb2, mul_mv(iB, rtb2));
      k.cx.y = dot(rta1, mul_mv(iA, rta2)) + dot(rtb1, mul_mv(iB, rtb2));
      k.cy.x = k.cx.y;
      mc.tangent_mass = invert2(k);
      mc.friction_impulse = v2(ws * dot(man.friction_impulse, t1), ws * dot(man.friction_impulse, t2));
      float ktw = dot(nn, mul_mv(add_mm(iA, iB), nn));
      mc.twist_mass = ktw > 0.0f ? 1.0f / ktw : 0.0f;
      mc.twist_impulse = ws * man.twist_impulse;
      mc.rolling_impulse = ws * man.rolling_impulse;
    }
    w.ovf[i] = c;
  }
}

// distance_joint_solver.rs:74 prepare_joint + revolute_joint.rs:183 prepare_revolute_joint
__global__ void k_prepare_joints(DW w, StepParams p) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n_joints) return;
  DJoint j = w.joints[i];
  float hz = minf(j.constraint_hertz, 0.25f * p.inv_h);
  j.constraint_softness = make_soft(hz, j.constraint_damping_ratio, p.h);
  const DSim& sa = sim_of(w, j.enc_a);
  const DSim& sb = sim_of(w, j.enc_b);
  j.index_a = j.enc_a >= 0 ? j.enc_a : -1;
  j.index_b = j.enc_b >= 0 ? j.enc_b : -1;
  j.inv_mass_a = sa.inv_mass; j.inv_mass_b = sb.inv_mass;
  j.inv_ia = sa.inv_inertia_world; j.inv_ib = sb.inv_inertia_world;
  M3 sum = add_mm(j.inv_ia, j.inv_ib);
  j.fixed_rotation = det(sum) < 1000.0f * kMinPositive;
  j.frame_a.q = mul_quat(sa.q, j.local_frame_a.q);
  j.frame_a.p = rotate(sa.q, j.local_frame_a.p - sa.local_center);
  j.frame_b.q = mul_quat(sb.q, j.local_frame_b.q);
  j.frame_b.p = rotate(sb.q, j.local_frame_b.p - sb.local_center);
  Pos ca = {sa.cx, sa.cy, sa.cz}, cb = {sb.cx, sb.cy, sb.cz};
  j.delta_center = sub_pos(cb, ca);
  if (j.type == kJointSpherical) {
    // spherical_joint.rs:183-230
    V3 cone_axis = rotate(j.frame_a.q, v3(0, 0, 1));
    V3 twist_axis = rotate(j.frame_b.q, v3(0, 0, 1));
    if (j.enable_cone_limit) {
      V3 swing_axis = normalize(cross(cone_axis, twist_axis));
      float k = dot(swing_axis, mul_mv(sum, swing_axis));
      j.swing_mass = k > 0.0f ? 1.0f / k : 0.0f;
      j.swing_axis = swing_axis;
    }
    if (j.enable_twist_limit) {
      Q rel_q = inv_mul_quat(j.frame_a.q, j.frame_b.q);
      float tan_half = sqrtf((rel_q.v.x * rel_q.v.x + rel_q.v.y * rel_q.v.y) /
                             (rel_q.v.z * rel_q.v.z + rel_q.s * rel_q.s));
      V3 swing_axis = normalize(cross(cone_axis, twist_axis));
      V3 perp_axis = cross(swing_axis, cone_axis);
      V3 jac = mul_add(cone_axis, tan_half, perp_axis);
      float k = dot(jac, mul_mv(sum, jac));
      j.twist_mass = k > 0.0f ? 1.0f / k : 0.0f;
      j.twist_jacobian = jac;
    }
    j.rotation_mass = !j.fixed_rotation ? invert_matrix(sum) : m3zero();
    j.spring_softness = make_soft(j.hertz, j.damping_ratio, p.h);
    if (p.warm_start == 0.0f) {
      j.linear_impulse = v3(0, 0, 0); j.motor_impulse3 = v3(0, 0, 0); j.spring_impulse3 = v3(0, 0, 0);
      j.swing_impulse = 0; j.lower_impulse = 0; j.upper_impulse = 0;
    }
    w.joints[i] = j;
    return;
  }
  V3 axis = rotate(j.frame_a.q, v3(0, 0, 1));
  float k = dot(axis, mul_mv(sum, axis));
  j.axial_mass = k > 0.0f ? 1.0f / k : 0.0f;
  j.rotation_axis_z = axis;
  Q rq = inv_mul_quat(j.frame_a.q, j.frame_b.q);
  j.perp_axis_x = 0.5f * rotate(j.frame_a.q, rq.s * v3(1, 0, 0) + cross(rq.v, v3(1, 0, 0)));
  j.perp_axis_y = 0.5f * rotate(j.frame_a.q, rq.s * v3(0, 1, 0) + cross(rq.v, v3(0, 1, 0)));
  j.spring_softness = make_soft(j.hertz, j.damping_ratio, p.h);
  if (p.warm_start == 0.0f) {
    j.linear_impulse = v3(0, 0, 0); j.perp_impulse = v2(0, 0);
    j.motor_impulse = 0; j.spring_impulse = 0; j.lower_impulse = 0; j.upper_impulse = 0;
  }
  w.joints[i] = j;
}

// Batch narrowphase over explicit pair jobs (the same routines k_collide calls).
struct PairJob {
  int32_t type_a, type_b;
  float geom_a[7], geom_b[7];
  float xf[7];
  float sat_separation;
  int32_t sat_type, sat_index_a, sat_index_b, sat_hit;
  float simplex_metric;
  int32_t simplex_count, simplex_ia[4], simplex_ib[4];
};
struct PairResult {
  float normal[3];
  int32_t point_count;
  float points[4][4];
  uint32_t feature_ids[4];
};

__global__ void __launch_bounds__(128) k_collide_jobs(PairJob* jobs, PairResult* results, int count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  PairJob j = jobs[i];
  PairResult r;
  memset(&r, 0, sizeof(r));
  Xf x = xf(v3(j.xf[0], j.xf[1], j.xf[2]), quat(v3(j.xf[3], j.xf[4], j.xf[5]), j.xf[6]));
  LocalManifold lm;
  Sphere sa = {v3(j.geom_a[0], j.geom_a[1], j.geom_a[2]), j.geom_a[3]};
  Sphere sb = {v3(j.geom_b[0], j.geom_b[1], j.geom_b[2]), j.geom_b[3]};
  Capsule ca = {v3(j.geom_a[0], j.geom_a[1], j.geom_a[2]), v3(j.geom_a[3], j.geom_a[4], j.geom_a[5]), j.geom_a[6]};
  Capsule cb = {v3(j.geom_b[0], j.geom_b[1], j.geom_b[2]), v3(j.geom_b[3], j.geom_b[4], j.geom_b[5]), j.geom_b[6]};
  SATCache sat;
  sat.separation = j.sat_separation; sat.type = (uint8_t)j.sat_type;
  sat.index_a = (uint8_t)j.sat_index_a; sat.index_b = (uint8_t)j.sat_index_b; sat.hit = (uint8_t)j.sat_hit;
  SimplexCache sc;
  sc.metric = j.simplex_metric; sc.count = (uint16_t)j.simplex_count;
  for (int k = 0; k < 4; ++k) { sc.ia[k] = (uint8_t)j.simplex_ia[k]; sc.ib[k] = (uint8_t)j.simplex_ib[k]; }
  if (j.type_a == kSphere) {
    collide_spheres(&lm, sa, sb, x);
  } else if (j.type_a == kCapsule) {
    if (j.type_b == kSphere) collide_capsule_sphere(&lm, ca, sb, x);
    else collide_capsules(&lm, ca, cb, x);
  } else {
    Hull ha = make_box_hull(j.geom_a[0], j.geom_a[1], j.geom_a[2]);
    if (j.type_b == kSphere) collide_hull_sphere(&lm, ha, sb, x, &sc);
    else if (j.type_b == kCapsule) collide_hull_capsule(&lm, ha, cb, x, &sc);
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
  for (int k = 0; k < lm.point_count && k < 4; ++k) {
    r.points[k][0] = lm.points[k].point.x; r.points[k][1] = lm.points[k].point.y;
    r.points[k][2] = lm.points[k].point.z; r.points[k][3] = lm.points[k].separation;
    r.feature_ids[k] = make_feature_id(lm.points[k].pair);
  }
  jobs[i] = j;
  results[i] = r;
}

}  // namespace nsd
