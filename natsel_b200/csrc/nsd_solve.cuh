// Persistent colored solver (solver_stages.rs:543 solve_constraint_stages) and body
// finalization (solver_integration.rs:587 finalize_body_range).
//
// One persistent launch runs every substep: integrate velocities together with each body's
// warm start (the changes its constraints recorded, applied in colour order; the overflow
// colour's warm start, when there is overflow work, runs on one thread per world between the
// two), then per stage (push, relax) the overflow color on one thread followed by colors
// 0..22, each color one phase separated by a barrier over the whole launch (a grid-wide
// barrier for a cooperative launch over the GPU, or the hardware barrier of one thread-block
// cluster), integrate positions between the stages; then restitution and impulse storage.
// Every block takes the same path through the phases (the loop bounds are read identically
// by all of them), so every block reaches every barrier; colors with no work are skipped by
// all blocks alike.
#pragma once
#include "nsd_kernels.cuh"
#include "nsd_toi.cuh"

namespace nsd {

// barrier.cluster with release/acquire semantics: global-memory writes of every thread of
// the cluster before the barrier are visible to every thread of the cluster after it.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Grid-wide barrier of the cooperative solver launch: thread 0 of each block adds its arrival
// with release semantics and polls the counter with acquire loads; the block's other threads
// are ordered by __syncthreads on both sides. Barrier k completes at (k + 1) * gridDim.x
// arrivals (the counter is zeroed before each launch; ``missing`` is only set by the barrier
// self-test, to wait for arrivals that never come). The wait is bounded: after limit_ns (2 s),
// 2^26 polls or another block's error it raises NS_ERR_TIMEOUT and returns false, and every
// block then leaves the kernel at its next barrier.
__device__ __forceinline__ void grid_arrive(Control* ctl) {
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(&ctl->barrier_count) : "memory");
}

__device__ __forceinline__ bool grid_wait(Control* ctl, int& index, int missing = 0,
                                          unsigned long long limit_ns = 2000000000ull) {
  __shared__ int ok_s;
  if (threadIdx.x == 0) {
    int target = (index + 1) * (int)gridDim.x + missing;
    int* cnt = &ctl->barrier_count;
    int ok = 1;
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (long long spins = 1;; ++spins) {
      int v;
      asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
      if (v >= target) break;
      if ((spins & 255) == 0) {
        unsigned long long t1;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
        if (*((volatile int*)&ctl->error) != 0 || t1 - t0 > limit_ns || spins > (1ll << 26)) { ok = 0; break; }
      }
    }
    if (!ok) atomicCAS(&ctl->error, 0, kErrTimeout);
    ok_s = ok;
  }
  __syncthreads();
  index++;
  return ok_s != 0;
}

__device__ __forceinline__ bool grid_sync_acq_rel(Control* ctl, int& index, int missing = 0,
                                                  unsigned long long limit_ns = 2000000000ull) {
  grid_arrive(ctl);
  return grid_wait(ctl, index, missing, limit_ns);
}

// Self-test of the solver's bounded grid barrier: every block arrives, but the barrier also
// waits for one arrival that nothing makes, so each block gives up after ``limit_ns`` and the
// kernel returns with ctl->error = kErrTimeout.
__global__ void k_barrier_selftest(Control* ctl, unsigned long long limit_ns) {
  int bar = 0;
  grid_sync_acq_rel(ctl, bar, 1, limit_ns);
}

template <bool kGrid>
__device__ __forceinline__ bool phase_sync(Control* ctl, int& index) {
  if (kGrid) return grid_sync_acq_rel(ctl, index);
  cluster_sync_all();
  return true;
}

__device__ __forceinline__ void store_state_vw(const DW& w, int i, const DState& s) {
  if (i >= 0 && (s.flags & kDynamicFlag)) {
    w.states[i].v = s.v;
    w.states[i].w = s.w;
  }
}

// solver_integration.rs:263 integrate_velocities_range. Split into a load and an update so
// a thread can issue the loads of all its bodies before the first update.
struct IVIn {
  float lin_damp, ang_damp, inv_mass, grav_scale;
  V3 force, torque;
  M3 iiw;
  uint32_t flags;
  Q q;
  M3 inertia;
  V3 v, w;
  Q dq;
  uint32_t state_flags;
};
__device__ __forceinline__ IVIn load_iv(const DW& w, int i) {
  const DSim& sim = w.asims[i];
  const DState& st = w.states[i];
  IVIn r;
  r.lin_damp = sim.linear_damping; r.ang_damp = sim.angular_damping;
  r.inv_mass = sim.inv_mass; r.grav_scale = sim.gravity_scale;
  r.force = sim.force; r.torque = sim.torque;
  r.iiw = sim.inv_inertia_world;
  r.flags = sim.flags;
  r.q = sim.q;
  r.inertia = sim.inertia;
  r.v = st.v; r.w = st.w; r.dq = st.dq;
  r.state_flags = st.flags;
  return r;
}
__device__ __forceinline__ void integrate_velocity(const StepParams& p, const IVIn& sim, V3& v_out, V3& w_out) {
  float h = p.h;
  V3 v = sim.v, wv = sim.w;
  float ld = 1.0f / (1.0f + h * sim.lin_damp);
  float ad = 1.0f / (1.0f + h * sim.ang_damp);
  float gs = sim.inv_mass > 0.0f ? sim.grav_scale : 0.0f;
  V3 lvd = blend2(h * sim.inv_mass, sim.force, h * gs, p.gravity);
  v = mul_add(lvd, ld, v);
  V3 avd = h * mul_mv(sim.iiw, sim.torque);
  wv = mul_add(avd, ad, wv);
  if (sim.flags & kGyroscopic) {
    Q q = mul_quat(sim.dq, sim.q);
    V3 om1 = inv_rotate(q, wv);
    V3 om2 = om1;
    float i00 = sim.inertia.cx.x, i01 = sim.inertia.cy.x, i02 = sim.inertia.cz.x;
    float i11 = sim.inertia.cy.y, i12 = sim.inertia.cz.y, i22 = sim.inertia.cz.z;
    float w1 = om2.x, w2 = om2.y, w3 = om2.z;
    float iw1 = i00 * w1 + i01 * w2 + i02 * w3;
    float iw2 = i01 * w1 + i11 * w2 + i12 * w3;
    float iw3 = i02 * w1 + i12 * w2 + i22 * w3;
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
    wv = rotate(q, om2);
  }
  v_out = v;
  w_out = wv;
}

// solver_integration.rs:377 integrate_positions_range (the state row is the only input)
__device__ __forceinline__ void apply_ip(const DW& w, const StepParams& p, int i, DState st) {
  float maxl = p.max_linear_speed;
  float maxa = kMaxRotation * p.inv_dt;
  float maxl2 = maxl * maxl, maxa2 = maxa * maxa;
  V3 v = st.v, wv = st.w;
  v.x = (st.flags & kLockLinX) ? 0.0f : v.x;
  v.y = (st.flags & kLockLinY) ? 0.0f : v.y;
  v.z = (st.flags & kLockLinZ) ? 0.0f : v.z;
  wv.x = (st.flags & kLockAngX) ? 0.0f : wv.x;
  wv.y = (st.flags & kLockAngY) ? 0.0f : wv.y;
  wv.z = (st.flags & kLockAngZ) ? 0.0f : wv.z;
  if (dot(v, v) > maxl2) {
    float ratio = maxl / length(v);
    v = ratio * v;
    st.flags |= kIsSpeedCapped;
  }
  if (dot(wv, wv) > maxa2 && (st.flags & kAllowFastRotation) == 0) {
    float ratio = maxa / length(wv);
    wv = ratio * wv;
    st.flags |= kIsSpeedCapped;
  }
  st.v = v;
  st.w = wv;
  st.dp = mul_add(st.dp, p.h, v);
  st.dq = integrate_rotation(st.dq, p.h * wv);
  w.states[i] = st;
}

// Contact constraint data in registers. load_direct issues every load of a constraint
// before the first store and before the dependent body-state loads, so one L2 round trip
// brings all the planes instead of one per point behind each impulse store. Read-only
// planes (written by prepare, never by the solver) go through the non-coherent path;
// impulse planes are read and written only by the thread that processes the constraint in
// a phase, with phase barriers in between.
struct CLoad {
  int ia, ib, pc;
  bool is_static;
  float ima, imb, friction, restitution, rolling;
  Sym sa, sb;
  V3 n;
};
__device__ __forceinline__ CLoad unpack_constraint(int4 idx, float4 m, float4 a0, float4 a1, float4 b1, float4 nn) {
  CLoad c;
  c.ia = idx.x; c.ib = idx.y; c.pc = idx.w & 255; c.is_static = (idx.w & 256) != 0;
  c.ima = m.x; c.imb = m.y; c.friction = m.z; c.restitution = m.w;
  c.sa.xx = a0.x; c.sa.xy = a0.y; c.sa.xz = a0.z; c.sa.yy = a0.w; c.sa.yz = a1.x; c.sa.zz = a1.y;
  c.sb.xx = a1.z; c.sb.xy = a1.w; c.sb.xz = b1.x; c.sb.yy = b1.y; c.sb.yz = b1.z; c.sb.zz = b1.w;
  c.n = v3(nn.x, nn.y, nn.z);
  c.rolling = nn.w;
  return c;
}

enum Stage { kWarm = 0, kPush = 1, kRelax = 2, kRestitution = 3 };

struct CData {
  CLoad c;
  float4 t1, t2, ca, cb, fr, roll, rm, tm;
  float4 pra[4], prb[4], pimp[4];
  float prest[4];
};

// Every field is written (zero where the stage reads nothing). Only the manifold's points are
// read: the cluster's 16 SMs move every phase's constraints from L2, so bytes count.
__device__ __forceinline__ void load_direct(const CPlanes& P, int k, int stage, CData& d) {
  const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  d.c = unpack_constraint(__ldg(&P.idx[k]), __ldg(&P.mass[k]), __ldg(&P.ia0[k]), __ldg(&P.ia1[k]),
                          __ldg(&P.ib1[k]), __ldg(&P.n[k]));
  d.t1 = z; d.t2 = z; d.ca = z; d.cb = z; d.fr = z; d.roll = z; d.rm = z; d.tm = z;
  if (stage == kWarm || stage == kRelax) {
    d.t1 = __ldg(&P.t1[k]); d.t2 = __ldg(&P.t2[k]); d.ca = __ldg(&P.ca[k]);
    d.cb = P.cb[k]; d.fr = P.fr[k]; d.roll = P.roll[k];
  }
  if (stage == kRelax) { d.rm = __ldg(&P.rm[k]); d.tm = __ldg(&P.tm[k]); }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    d.pra[q] = z; d.prb[q] = z; d.pimp[q] = z; d.prest[q] = 0.0f;
    if (q < d.c.pc) {
      d.pra[q] = __ldg(&P.pra[q * P.cap + k]);
      d.prb[q] = __ldg(&P.prb[q * P.cap + k]);
      d.pimp[q] = P.pimp[q * P.cap + k];
      if (stage == kRestitution) d.prest[q] = P.prest[q * P.cap + k];
    }
  }
}

// A constraint's planes staged in shared memory ahead of its phase: one column per lane of the
// block's first warp, rows idx, mass, ia0, ia1, ib1, n, t1, t2, ca, cb, fr, roll, rm, tm, then
// pra, prb and pimp of the four points (all four are copied: the point count is in idx).
constexpr int kStageRows = 26;
typedef float4 StageBuf[kStageRows][32];
__device__ __forceinline__ void cp_async16(float4* smem, const void* gmem) {
  unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
// Issue the copies of constraint k for the given stage (push or relax). The planes other than
// the impulses are constant during the launch and the impulses are written only by the thread
// that owns the constraint (this one), in earlier phases.
__device__ __forceinline__ void stage_constraint(const CPlanes& P, int k, int stage, StageBuf& b, int lane) {
  cp_async16(&b[0][lane], &P.idx[k]);
  cp_async16(&b[1][lane], &P.mass[k]);
  cp_async16(&b[2][lane], &P.ia0[k]);
  cp_async16(&b[3][lane], &P.ia1[k]);
  cp_async16(&b[4][lane], &P.ib1[k]);
  cp_async16(&b[5][lane], &P.n[k]);
  if (stage == kRelax) {
    cp_async16(&b[6][lane], &P.t1[k]);
    cp_async16(&b[7][lane], &P.t2[k]);
    cp_async16(&b[8][lane], &P.ca[k]);
    cp_async16(&b[9][lane], &P.cb[k]);
    cp_async16(&b[10][lane], &P.fr[k]);
    cp_async16(&b[11][lane], &P.roll[k]);
    cp_async16(&b[12][lane], &P.rm[k]);
    cp_async16(&b[13][lane], &P.tm[k]);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    cp_async16(&b[14 + q][lane], &P.pra[q * P.cap + k]);
    cp_async16(&b[18 + q][lane], &P.prb[q * P.cap + k]);
    cp_async16(&b[22 + q][lane], &P.pimp[q * P.cap + k]);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}
// load_direct's result (push or relax) from the staged copy.
__device__ __forceinline__ void load_staged(const StageBuf& b, int lane, int stage, CData& d) {
  asm volatile("cp.async.wait_all;" ::: "memory");
  const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float4 i4 = b[0][lane];
  int4 idx = make_int4(__float_as_int(i4.x), __float_as_int(i4.y), __float_as_int(i4.z), __float_as_int(i4.w));
  d.c = unpack_constraint(idx, b[1][lane], b[2][lane], b[3][lane], b[4][lane], b[5][lane]);
  d.t1 = z; d.t2 = z; d.ca = z; d.cb = z; d.fr = z; d.roll = z; d.rm = z; d.tm = z;
  if (stage == kRelax) {
    d.t1 = b[6][lane]; d.t2 = b[7][lane]; d.ca = b[8][lane]; d.cb = b[9][lane];
    d.fr = b[10][lane]; d.roll = b[11][lane]; d.rm = b[12][lane]; d.tm = b[13][lane];
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    d.pra[q] = z; d.prb[q] = z; d.pimp[q] = z; d.prest[q] = 0.0f;
    if (q < d.c.pc) {
      d.pra[q] = b[14 + q][lane];
      d.prb[q] = b[18 + q][lane];
      d.pimp[q] = b[22 + q][lane];
    }
  }
}

// Change of the two bodies' velocities by one warm start: body a gets v - dva, w - dwa and
// body b v + dvb, w + dvb. It depends on the constraint's planes and impulses only, not on the
// bodies' velocities, so it can be formed when the impulses are last updated and applied later
// by each body in colour order with the same operations.
struct WarmDelta { V3 dva, dwa, dvb, dwb; };

// contact_solver.rs:697 warm_start_contacts_body (the per-body change; ni the points' normal
// impulses, fr the friction impulses, cbf.w the twist impulse, roll the rolling impulse)
__device__ __forceinline__ WarmDelta contact_warm_delta(const CLoad& c, float4 t1f, float4 t2f, float4 caf,
                                                        float4 cbf, float4 fr, float4 roll, const float4* pra,
                                                        const float4* prb, const float* ni) {
  V3 t1 = v3(t1f.x, t1f.y, t1f.z), t2 = v3(t2f.x, t2f.y, t2f.z);
  V3 center_a = v3(caf.x, caf.y, caf.z), center_b = v3(cbf.x, cbf.y, cbf.z);
  float twist = cbf.w;
  V3 li = v3(0, 0, 0), aia = v3(0, 0, 0), aib = v3(0, 0, 0);
  float tni = 0.0f;
  V3 moa = v3(0, 0, 0), mob = v3(0, 0, 0);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (q < c.pc) {
      tni += ni[q];
      moa = mul_add(moa, ni[q], v3(pra[q].x, pra[q].y, pra[q].z));
      mob = mul_add(mob, ni[q], v3(prb[q].x, prb[q].y, prb[q].z));
    }
  }
  V3 n = c.n;
  V3 fi = fr.x * t1;
  fi = mul_add(fi, fr.y, t2);
  V3 lin = mul_add(fi, tni, n);
  V3 twi = twist * n;
  V3 anga = cross(moa, n) + cross(center_a, fi) + twi;
  V3 angb = cross(mob, n) + cross(center_b, fi) + twi;
  if (c.rolling > 0.0f) {
    V3 ri = v3(roll.x, roll.y, roll.z);
    anga = anga + ri;
    angb = angb + ri;
  }
  li = li + lin; aia = aia + anga; aib = aib + angb;
  WarmDelta r;
  r.dwa = sym_mv(c.sa, aia);
  r.dva = c.ima * li;
  r.dwb = sym_mv(c.sb, aib);
  r.dvb = c.imb * li;
  return r;
}

// Record a warm-start change in the slots of colour `color` of both bodies (a static body, index
// -1, has none). Body a's change is stored negated: v + (-x) is v - x exactly.
__device__ __forceinline__ void put_warm_delta(const DW& w, int ia, int ib, int color, const WarmDelta& x) {
  if (ia >= 0) {
    float4* s = w.bwd + 2 * (24 * (size_t)ia + color);
    s[0] = make_float4(-x.dva.x, -x.dva.y, -x.dva.z, 0.0f);
    s[1] = make_float4(-x.dwa.x, -x.dwa.y, -x.dwa.z, 0.0f);
  }
  if (ib >= 0) {
    float4* s = w.bwd + 2 * (24 * (size_t)ib + color);
    s[0] = make_float4(x.dvb.x, x.dvb.y, x.dvb.z, 0.0f);
    s[1] = make_float4(x.dwb.x, x.dwb.y, x.dwb.z, 0.0f);
  }
}

// The solver index of a dynamic body, -1 for a static or kinematic one
__device__ __forceinline__ int dynamic_index(const DW& w, int i) {
  return i >= 0 && (w.states[i].flags & kDynamicFlag) ? i : -1;
}

__device__ __forceinline__ void mark_warm_slot(const DW& w, int body, int color) {
  if (body >= 0) atomicOr(&w.bw_mask[body], 1u << color);
}

// A dynamic body's warm start: the changes of its constraints and joints in colour order (the
// order the colour phases would apply them; one item per colour). load_warm_slots fetches up
// to kSlotBatch slots and clears their bits from m; apply_warm_slots adds them in order.
constexpr int kSlotBatch = 8;
struct WarmSlots {
  float4 dv[kSlotBatch], dw[kSlotBatch];
  int count;
};
__device__ __forceinline__ void load_warm_slots(const DW& w, int i, uint32_t& m, WarmSlots& ws) {
  const float4* row = w.bwd + 48 * (size_t)i;
  ws.count = 0;
#pragma unroll
  for (int q = 0; q < kSlotBatch; ++q) {
    ws.dv[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    ws.dw[q] = ws.dv[q];
    if (m != 0u) {
      int c = __ffs(m) - 1;
      m &= m - 1u;
      ws.dv[q] = row[2 * c];
      ws.dw[q] = row[2 * c + 1];
      ws.count = q + 1;
    }
  }
}
__device__ __forceinline__ void apply_warm_slots(const WarmSlots& ws, V3& v, V3& wv) {
#pragma unroll
  for (int q = 0; q < kSlotBatch; ++q) {
    if (q < ws.count) {
      wv = wv + v3(ws.dw[q].x, ws.dw[q].y, ws.dw[q].z);
      v = v + v3(ws.dv[q].x, ws.dv[q].y, ws.dv[q].z);
    }
  }
}
__device__ __forceinline__ void warm_body(const DW& w, int i, uint32_t m, WarmSlots& ws, V3& v, V3& wv) {
  apply_warm_slots(ws, v, wv);
  while (m != 0u) {
    load_warm_slots(w, i, m, ws);
    apply_warm_slots(ws, v, wv);
  }
}

// contact_solver.rs:796 push_contacts_body
__device__ void push_constraint(const DW& w, const StepParams& p, int k, const CData& d) {
  const CPlanes& P = w.cp;
  const CLoad& c = d.c;
  DState ba = state_at(w, c.ia), bb = state_at(w, c.ib);
  float inv_h = p.inv_h;
  float cs = -p.contact_speed;
  float br = c.is_static ? p.static_softness.mass_scale * p.static_softness.bias_rate
                         : p.contact_softness.mass_scale * p.contact_softness.bias_rate;
  float ms = c.is_static ? p.static_softness.mass_scale : p.contact_softness.mass_scale;
  float is = c.is_static ? p.static_softness.impulse_scale : p.contact_softness.impulse_scale;
  V3 dp = bb.dp - ba.dp;
  float im = c.ima + c.imb;
  V3 n = c.n;
  float ns = dot(n, dp);
  V3 na = inv_rotate_wide(ba.dq, n), nb = inv_rotate_wide(bb.dq, n);
  float lnv = dot(n, bb.v - ba.v);
  float mi = 0.0f;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (q < c.pc) {
      float4 raf = d.pra[q], rbf = d.prb[q];
      float4 imp4 = d.pimp[q];
      V3 ra = v3(raf.x, raf.y, raf.z), rb = v3(rbf.x, rbf.y, rbf.z);
      float base_sep = raf.w, nmass = rbf.w, nimp = imp4.x;
      float s = (ns + (dot(nb, rb) - dot(na, ra))) + base_sep;
      bool sep = s > 0.0f;
      float spec_bias = s * inv_h;
      float ovl = maxf(br * s, cs);
      float vb = sep ? spec_bias : ovl;
      float pms = sep ? 1.0f : ms;
      float pis = sep ? 0.0f : is;
      V3 ua = cross(ra, n), ub = cross(rb, n);
      V3 ga = sym_mv(c.sa, ua), gb = sym_mv(c.sb, ub);
      float vn = lnv + (dot(ub, bb.w) - dot(ua, ba.w));
      float neg = nmass * (pms * vn + vb) + pis * nimp;
      float impulse = maxf(-neg, -nimp);
      imp4.x = nimp + impulse;
      P.pimp[q * P.cap + k] = imp4;
      lnv += im * impulse;
      mi += impulse;
      ba.w = ba.w - impulse * ga;
      bb.w = bb.w + impulse * gb;
    }
  }
  V3 Pv = mi * n;
  ba.v = ba.v - c.ima * Pv;
  bb.v = bb.v + c.imb * Pv;
  store_state_vw(w, c.ia, ba);
  store_state_vw(w, c.ib, bb);
}

// contact_solver.rs:927 solve_contacts_body (relax)
// warm_color >= 0: also record the warm-start change of the next substep from the updated
// impulses in the bodies' slots of that colour.
__device__ void relax_constraint(const DW& w, const StepParams& p, int k, const CData& d, int warm_color) {
  const CPlanes& P = w.cp;
  const CLoad& c = d.c;
  DState ba = state_at(w, c.ia), bb = state_at(w, c.ib);
  float4 cbf = d.cb, fr = d.fr, ro = d.roll, rmv = d.rm, caf = d.ca, tmf = d.tm;
  bool any_rolling = c.rolling > 0.0f;
  float inv_h = p.inv_h;
  const float eps = kEps;
  V3 dp = bb.dp - ba.dp;
  float im = c.ima + c.imb;
  V3 n = c.n;
  V3 t1 = v3(d.t1.x, d.t1.y, d.t1.z), t2 = v3(d.t2.x, d.t2.y, d.t2.z);
  float ns = dot(n, dp);
  V3 na = inv_rotate_wide(ba.dq, n), nb = inv_rotate_wide(bb.dq, n);
  V3 dv = bb.v - ba.v;
  float lnv = dot(n, dv);
  float lt1 = dot(t1, dv) - d.t1.w;
  float lt2 = dot(t2, dv) - d.t2.w;
  float mi = 0.0f, tni = 0.0f, ttl = 0.0f;
  float nis[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (q < c.pc) {
      float4 raf = d.pra[q], rbf = d.prb[q];
      float4 imp4 = d.pimp[q];
      V3 ra = v3(raf.x, raf.y, raf.z), rb = v3(rbf.x, rbf.y, rbf.z);
      float s = (ns + (dot(nb, rb) - dot(na, ra))) + raf.w;
      float vb = maxf(0.0f, s * inv_h);
      V3 ua = cross(ra, n), ub = cross(rb, n);
      V3 ga = sym_mv(c.sa, ua), gb = sym_mv(c.sb, ub);
      float vn = lnv + (dot(ub, bb.w) - dot(ua, ba.w));
      float neg = rbf.w * (vn + vb);
      float impulse = maxf(-neg, -imp4.x);
      float ni = imp4.x + impulse;
      imp4.x = ni;
      imp4.y = imp4.y + ni;
      P.pimp[q * P.cap + k] = imp4;
      nis[q] = ni;
      tni += ni;
      ttl += imp4.z * ni;
      lnv += im * impulse;
      mi += impulse;
      ba.w = ba.w - impulse * ga;
      bb.w = bb.w + impulse * gb;
    }
  }
  if (any_rolling) {
    Sym rm = {fr.z, fr.w, ro.w, rmv.x, rmv.y, rmv.z};
    V3 di = sym_mv(rm, ba.w - bb.w);
    V3 old = v3(ro.x, ro.y, ro.z);
    V3 rimp = old + di;
    float mx = c.rolling * tni;
    float lsq = dot(rimp, rimp);
    bool mask = lsq > eps + mx * mx;
    float nrm = mx / (sqrtf(lsq) + eps);
    float sc = mask ? nrm : 1.0f;
    V3 scaled = sc * rimp;
    if (c.rolling == 0.0f) scaled = v3(0, 0, 0);
    rimp = scaled;
    di = rimp - old;
    ba.w = ba.w - sym_mv(c.sa, di);
    bb.w = bb.w + sym_mv(c.sb, di);
    P.roll[k] = make_float4(rimp.x, rimp.y, rimp.z, ro.w);
    ro = make_float4(rimp.x, rimp.y, rimp.z, ro.w);
  }
  {
    float ts = dot(n, bb.w - ba.w);
    float ml = c.friction * ttl;
    float old = cbf.w;
    float impulse = -(caf.w * ts);
    impulse = maxf(-ml - old, minf(impulse, ml - old));
    cbf.w = old + impulse;
    P.cb[k] = cbf;
    ba.w = ba.w - impulse * sym_mv(c.sa, n);
    bb.w = bb.w + impulse * sym_mv(c.sb, n);
    V3 ra = v3(caf.x, caf.y, caf.z), rb = v3(cbf.x, cbf.y, cbf.z);
    M2 tm;
    tm.cx = v2(tmf.x, tmf.y);
    tm.cy = v2(tmf.z, tmf.w);
    V3 arv = cross(bb.w, rb) - cross(ba.w, ra);
    V2 vt = v2(lt1 + dot(arv, t1), lt2 + dot(arv, t2));
    V2 di = mul_mv2(tm, vt);
    di = v2(-di.x, -di.y);
    V2 ni = v2(fr.x + di.x, fr.y + di.y);
    float mx = c.friction * tni;
    float lsq = ni.x * ni.x + ni.y * ni.y;
    bool mask = lsq > mx * mx;
    float nrm = mx / (sqrtf(lsq) + eps);
    float sc = mask ? nrm : 1.0f;
    ni = v2(sc * ni.x, sc * ni.y);
    di = v2(ni.x - fr.x, ni.y - fr.y);
    fr.x = ni.x; fr.y = ni.y;
    P.fr[k] = fr;
    V3 Pv = di.x * t1;
    Pv = Pv + di.y * t2;
    ba.w = ba.w - sym_mv(c.sa, cross(ra, Pv));
    bb.w = bb.w + sym_mv(c.sb, cross(rb, Pv));
    Pv = Pv + mi * n;
    ba.v = ba.v - c.ima * Pv;
    bb.v = bb.v + c.imb * Pv;
  }
  store_state_vw(w, c.ia, ba);
  store_state_vw(w, c.ib, bb);
  if (warm_color >= 0)  // only a dynamic body takes a warm start (kinematic bodies share colours)
    put_warm_delta(w, (ba.flags & kDynamicFlag) ? c.ia : -1, (bb.flags & kDynamicFlag) ? c.ib : -1, warm_color,
                   contact_warm_delta(c, d.t1, d.t2, caf, cbf, fr, ro, d.pra, d.prb, nis));
}

// contact_solver.rs:1135 apply_restitution_body
__device__ void restitution_constraint(const DW& w, const StepParams& p, int k, const CData& d) {
  const CPlanes& P = w.cp;
  const CLoad& c = d.c;
  if (c.restitution == 0.0f) return;
  DState ba = state_at(w, c.ia), bb = state_at(w, c.ib);
  float inv_h = p.inv_h;
  float nrt = -p.restitution_threshold;
  bool rmask = c.restitution > 0.0f;
  V3 dp = bb.dp - ba.dp;
  V3 n = c.n;
  float ns = dot(n, dp);
  V3 na = inv_rotate_wide(ba.dq, n), nb = inv_rotate_wide(bb.dq, n);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (q < c.pc) {
      float4 raf = d.pra[q], rbf = d.prb[q];
      float4 imp4 = d.pimp[q];
      float rest_imp = d.prest[q];
      V3 ra = v3(raf.x, raf.y, raf.z), rb = v3(rbf.x, rbf.y, rbf.z);
      float s = (ns + (dot(nb, rb) - dot(na, ra))) + raf.w;
      float nm = rmask ? rbf.w : 0.0f;
      float comp = imp4.y - rest_imp;
      bool armed = rmask && imp4.w < nrt && comp > 0.0f;
      float sb = maxf(0.0f, s * inv_h);
      float vb = armed ? c.restitution * imp4.w : sb;
      V3 vra = ba.v + cross(ba.w, ra), vrb = bb.v + cross(bb.w, rb);
      float vn = dot(vrb - vra, n);
      float neg = nm * (vn + vb);
      float ni = maxf(imp4.x - neg, 0.0f);
      float impulse = ni - imp4.x;
      float app = minf(maxf(-nm * vn, 0.0f), maxf(impulse, 0.0f));
      float allow = c.restitution * (comp + app) - rest_imp;
      float mx = app + maxf(allow, 0.0f);
      impulse = armed ? minf(impulse, mx) : impulse;
      imp4.x = imp4.x + impulse;
      rest_imp = rest_imp + (impulse - app);
      imp4.y = imp4.y + impulse;
      P.pimp[q * P.cap + k] = imp4;
      P.prest[q * P.cap + k] = rest_imp;
      V3 Pv = impulse * n;
      ba.w = ba.w - sym_mv(c.sa, cross(ra, Pv));
      ba.v = ba.v - c.ima * Pv;
      bb.w = bb.w + sym_mv(c.sb, cross(rb, Pv));
      bb.v = bb.v + c.imb * Pv;
    }
  }
  store_state_vw(w, c.ia, ba);
  store_state_vw(w, c.ib, bb);
}

__device__ __forceinline__ void run_contact(const DW& w, const StepParams& p, int k, int stage, const CData& d,
                                            int warm_color) {
  if (stage == kPush) push_constraint(w, p, k, d);
  else if (stage == kRelax) relax_constraint(w, p, k, d, warm_color);
  else restitution_constraint(w, p, k, d);
}

// contact_solver.rs:1258 store_impulses_body
__device__ void store_constraint(const DW& w, int k) {
  const CPlanes& P = w.cp;
  int4 idx = P.idx[k];
  DContact& ct = w.contacts[idx.z];
  if (ct.manifold_count <= 0) return;
  int pc = idx.w & 255;
  Manifold& out = ct.manifold;
  int cnt = min_i(out.point_count, pc);
  for (int q = 0; q < cnt; ++q) {
    float4 imp4 = P.pimp[q * P.cap + k];
    out.points[q].normal_impulse = imp4.x;
    out.points[q].total_normal_impulse = imp4.y;
  }
  float4 cbf = P.cb[k], t1f = P.t1[k], t2f = P.t2[k], fr = P.fr[k], ro = P.roll[k];
  out.twist_impulse = cbf.w;
  out.friction_impulse = fr.x * v3(t1f.x, t1f.y, t1f.z) + fr.y * v3(t2f.x, t2f.y, t2f.z);
  out.rolling_impulse = v3(ro.x, ro.y, ro.z);
}

// overflow_contact_solver.rs:308-700 sequential overflow color
__device__ void ovf_store_velocity(const DW& w, int i, uint32_t flags, V3 v, V3 wv) {
  if (i >= 0 && (flags & kDynamicFlag)) { DState* d = state_ptr(w, i); d->v = v; d->w = wv; }
}
__device__ void warm_start_overflow(const DW& w, int base, int n) {
  for (int i = base; i < base + n; ++i) {
    const DOverflow& c = w.ovf[i];
    V3 li = v3(0, 0, 0), aia = v3(0, 0, 0), aib = v3(0, 0, 0);
    for (int mi = 0; mi < c.manifold_count; ++mi) {
      const ManifoldConstraint& mc = c.m;
      V3 nn = mc.normal;
      float tni = 0.0f;
      V3 moa = v3(0, 0, 0), mob = v3(0, 0, 0);
      for (int j = 0; j < mc.point_count; ++j) {
        const ConstraintPoint& cp = mc.points[j];
        tni += cp.normal_impulse;
        moa = mul_add(moa, cp.normal_impulse, cp.r_a);
        mob = mul_add(mob, cp.normal_impulse, cp.r_b);
      }
      V3 fi = mc.friction_impulse.x * mc.tangent1;
      fi = mul_add(fi, mc.friction_impulse.y, mc.tangent2);
      li = li + mul_add(fi, tni, nn);
      V3 twi = mc.twist_impulse * nn;
      V3 anga = (cross(moa, nn) + cross(mc.center_a, fi)) + twi;
      V3 angb = (cross(mob, nn) + cross(mc.center_b, fi)) + twi;
      aia = aia + (anga + mc.rolling_impulse);
      aib = aib + (angb + mc.rolling_impulse);
    }
    if (c.index_a >= 0 && (state_ptr(w, c.index_a)->flags & kDynamicFlag)) {
      DState& s = *state_ptr(w, c.index_a);
      s.v = mul_sub(s.v, c.inv_mass_a, li);
      s.w = s.w - mul_mv(c.inv_ia, aia);
    }
    if (c.index_b >= 0 && (state_ptr(w, c.index_b)->flags & kDynamicFlag)) {
      DState& s = *state_ptr(w, c.index_b);
      s.v = mul_add(s.v, c.inv_mass_b, li);
      s.w = s.w + mul_mv(c.inv_ib, aib);
    }
  }
}
__device__ void push_overflow(const DW& w, const StepParams& p, int base, int n) {
  float inv_h = p.inv_h;
  float cs = p.contact_speed;
  for (int i = base; i < base + n; ++i) {
    DOverflow& c = w.ovf[i];
    float mA = c.inv_mass_a, mB = c.inv_mass_b;
    M3 iA = c.inv_ia, iB = c.inv_ib;
    DState sa = state_at(w, c.index_a), sb = state_at(w, c.index_b);
    V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
    Q dqa = sa.dq, dqb = sb.dq;
    V3 dp = sb.dp - sa.dp;
    Softness soft = c.softness;
    for (int mi = 0; mi < c.manifold_count; ++mi) {
      ManifoldConstraint& mc = c.m;
      V3 nn = mc.normal;
      for (int q = 0; q < mc.point_count; ++q) {
        ConstraintPoint& cp = mc.points[q];
        V3 ra = cp.r_a, rb = cp.r_b;
        V3 ds = dp + (rotate(dqb, rb) - rotate(dqa, ra));
        float s = dot(ds, nn) + cp.base_separation;
        float vbias, mscale, iscale;
        if (s > 0.0f) { vbias = s * inv_h; mscale = 1.0f; iscale = 0.0f; }
        else {
          vbias = maxf(soft.mass_scale * soft.bias_rate * s, -cs);
          mscale = soft.mass_scale; iscale = soft.impulse_scale;
        }
        V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
        float vn = dot(vrb - vra, nn);
        float ni0 = cp.normal_impulse;
        float di = -cp.normal_mass * (mscale * vn + vbias) - iscale * ni0;
        float ni = maxf(ni0 + di, 0.0f);
        di = ni - ni0;
        cp.normal_impulse = ni;
        V3 Pv = di * nn;
        va = mul_sub(va, mA, Pv);
        wa = wa - mul_mv(iA, cross(ra, Pv));
        vb = mul_add(vb, mB, Pv);
        wb = wb + mul_mv(iB, cross(rb, Pv));
      }
    }
    ovf_store_velocity(w, c.index_a, sa.flags, va, wa);
    ovf_store_velocity(w, c.index_b, sb.flags, vb, wb);
  }
}
__device__ void relax_overflow(const DW& w, const StepParams& p, int base, int n) {
  float inv_h = p.inv_h;
  for (int i = base; i < base + n; ++i) {
    DOverflow& c = w.ovf[i];
    float mA = c.inv_mass_a, mB = c.inv_mass_b;
    M3 iA = c.inv_ia, iB = c.inv_ib;
    DState sa = state_at(w, c.index_a), sb = state_at(w, c.index_b);
    V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
    Q dqa = sa.dq, dqb = sb.dq;
    V3 dp = sb.dp - sa.dp;
    float fr = c.friction, rr = c.rolling_resistance;
    for (int mi = 0; mi < c.manifold_count; ++mi) {
      ManifoldConstraint& mc = c.m;
      V3 nn = mc.normal;
      float tni = 0.0f, ttl = 0.0f;
      for (int q = 0; q < mc.point_count; ++q) {
        ConstraintPoint& cp = mc.points[q];
        V3 ra = cp.r_a, rb = cp.r_b;
        V3 ds = dp + (rotate(dqb, rb) - rotate(dqa, ra));
        float s = dot(ds, nn) + cp.base_separation;
        float vbias = s > 0.0f ? s * inv_h : 0.0f;
        V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
        float vn = dot(vrb - vra, nn);
        float ni0 = cp.normal_impulse;
        float di = -cp.normal_mass * (vn + vbias);
        float ni = maxf(ni0 + di, 0.0f);
        di = ni - ni0;
        cp.normal_impulse = ni;
        cp.total_normal_impulse += ni;
        tni += ni;
        ttl += cp.lever_arm * ni;
        V3 Pv = di * nn;
        va = mul_sub(va, mA, Pv);
        wa = wa - mul_mv(iA, cross(ra, Pv));
        vb = mul_add(vb, mB, Pv);
        wb = wb + mul_mv(iB, cross(rb, Pv));
      }
      {
        float ts = dot(nn, wb - wa);
        float mx = fr * ttl;
        float di = -mc.twist_mass * ts;
        float old = mc.twist_impulse;
        mc.twist_impulse = clampf(old + di, -mx, mx);
        di = mc.twist_impulse - old;
        wa = wa - mul_mv(iA, di * nn);
        wb = wb + mul_mv(iB, di * nn);
      }
      if (rr > 0.0f) {
        V3 di = -mul_mv(c.rolling_mass, wb - wa);
        V3 old = mc.rolling_impulse;
        mc.rolling_impulse = old + di;
        float mx = rr * tni;
        float msq = dot(mc.rolling_impulse, mc.rolling_impulse);
        if (msq > mx * mx + kEps) mc.rolling_impulse = (mx / sqrtf(msq)) * mc.rolling_impulse;
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
        float mx = fr * tni;
        float lsq = dot2(ni, ni);
        if (lsq > mx * mx) {
          float sc = mx / sqrtf(lsq);
          ni.x *= sc; ni.y *= sc;
        }
        di = v2(ni.x - mc.friction_impulse.x, ni.y - mc.friction_impulse.y);
        mc.friction_impulse = ni;
        V3 Pv = blend2(di.x, t1, di.y, t2);
        va = mul_sub(va, mA, Pv);
        wa = wa - mul_mv(iA, cross(ra, Pv));
        vb = mul_add(vb, mB, Pv);
        wb = wb + mul_mv(iB, cross(rb, Pv));
      }
    }
    ovf_store_velocity(w, c.index_a, sa.flags, va, wa);
    ovf_store_velocity(w, c.index_b, sb.flags, vb, wb);
  }
}
__device__ void restitution_overflow(const DW& w, const StepParams& p, int base, int n) {
  float thr = p.restitution_threshold;
  float inv_h = p.inv_h;
  for (int i = base; i < base + n; ++i) {
    DOverflow& c = w.ovf[i];
    float rest = c.restitution;
    if (rest == 0.0f) continue;
    float mA = c.inv_mass_a, mB = c.inv_mass_b;
    M3 iA = c.inv_ia, iB = c.inv_ib;
    DState sa = state_at(w, c.index_a), sb = state_at(w, c.index_b);
    V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
    Q dqa = sa.dq, dqb = sb.dq;
    V3 dp = sb.dp - sa.dp;
    for (int mi = 0; mi < c.manifold_count; ++mi) {
      ManifoldConstraint& mc = c.m;
      V3 nn = mc.normal;
      for (int q = 0; q < mc.point_count; ++q) {
        ConstraintPoint cp = mc.points[q];
        V3 ra = cp.r_a, rb = cp.r_b;
        float comp = cp.total_normal_impulse - cp.restitution_impulse;
        bool armed = rest > 0.0f && cp.relative_velocity < -thr && comp > 0.0f;
        float vbias;
        if (armed) vbias = rest * cp.relative_velocity;
        else {
          V3 ds = dp + (rotate(dqb, rb) - rotate(dqa, ra));
          float s = dot(ds, nn) + cp.base_separation;
          vbias = s > 0.0f ? s * inv_h : 0.0f;
        }
        V3 vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
        float vn = dot(vrb - vra, nn);
        float imp = -cp.normal_mass * (vn + vbias);
        float ni = maxf(cp.normal_impulse + imp, 0.0f);
        imp = ni - cp.normal_impulse;
        float app = minf(maxf(-cp.normal_mass * vn, 0.0f), maxf(imp, 0.0f));
        if (armed) {
          float allow = rest * (comp + app) - cp.restitution_impulse;
          imp = minf(imp, app + maxf(allow, 0.0f));
        }
        mc.points[q].normal_impulse += imp;
        mc.points[q].restitution_impulse += imp - app;
        mc.points[q].total_normal_impulse += imp;
        V3 Pv = imp * nn;
        va = mul_sub(va, mA, Pv);
        wa = wa - mul_mv(iA, cross(ra, Pv));
        vb = mul_add(vb, mB, Pv);
        wb = wb + mul_mv(iB, cross(rb, Pv));
      }
    }
    ovf_store_velocity(w, c.index_a, sa.flags, va, wa);
    ovf_store_velocity(w, c.index_b, sb.flags, vb, wb);
  }
}
__device__ void store_overflow(const DW& w, int base, int n) {
  for (int i = base; i < base + n; ++i) {
    const DOverflow& c = w.ovf[i];
    if (c.manifold_count == 0) continue;
    Manifold& m = w.contacts[c.contact_id].manifold;
    const ManifoldConstraint& mc = c.m;
    m.twist_impulse = mc.twist_impulse;
    m.friction_impulse = blend2(mc.friction_impulse.x, mc.tangent1, mc.friction_impulse.y, mc.tangent2);
    m.rolling_impulse = mc.rolling_impulse;
    for (int q = 0; q < mc.point_count; ++q) {
      m.points[q].normal_impulse = mc.points[q].normal_impulse;
      m.points[q].total_normal_impulse = mc.points[q].total_normal_impulse;
    }
  }
}

// revolute_joint.rs:95 solve_point_constraint
__device__ V3 solve_point_constraint(float ma, float mb, M3 ia, M3 ib, V3 ra, V3 rb, V3 rhs) {
  float axy = ra.z * ia.cy.y - ra.y * ia.cz.y;
  float axz = ra.z * ia.cy.z - ra.y * ia.cz.z;
  V3 ay = ra.x * ia.cz - ra.z * ia.cx;
  V3 az = ra.y * ia.cx - ra.x * ia.cy;
  float bxy = rb.z * ib.cy.y - rb.y * ib.cz.y;
  float bxz = rb.z * ib.cy.z - rb.y * ib.cz.z;
  V3 by = rb.x * ib.cz - rb.z * ib.cx;
  V3 bz = rb.y * ib.cx - rb.x * ib.cy;
  float m = ma + mb;
  float kxx = (axy * ra.z - axz * ra.y) + (bxy * rb.z - bxz * rb.y) + m;
  float kyy = (ay.z * ra.x - ay.x * ra.z) + (by.z * rb.x - by.x * rb.z) + m;
  float kzz = (az.x * ra.y - az.y * ra.x) + (bz.x * rb.y - bz.y * rb.x) + m;
  float kxy = (ay.y * ra.z - ay.z * ra.y) + (by.y * rb.z - by.z * rb.y);
  float kxz = (az.y * ra.z - az.z * ra.y) + (bz.y * rb.z - bz.z * rb.y);
  float kyz = (az.z * ra.x - az.x * ra.z) + (bz.z * rb.x - bz.x * rb.z);
  float cxx = kyy * kzz - kyz * kyz;
  float cyy = kxx * kzz - kxz * kxz;
  float czz = kxx * kyy - kxy * kxy;
  float cxy = kxz * kyz - kxy * kzz;
  float cxz = kxy * kyz - kyy * kxz;
  float cyz = kxy * kxz - kxx * kyz;
  float d = kxx * cxx + kxy * cxy + kxz * cxz;
  if (absf(d) > 1000.0f * kMinPositive) {
    float inv = 1.0f / d;
    return v3(inv * (cxx * rhs.x + cxy * rhs.y + cxz * rhs.z),
              inv * (cxy * rhs.x + cyy * rhs.y + cyz * rhs.z),
              inv * (cxz * rhs.x + cyz * rhs.y + czz * rhs.z));
  }
  return v3(0, 0, 0);
}

// revolute_joint.rs:261 warm_start_revolute_joint, the per-body change (dqa, dqb: the bodies'
// rotation increments, which no stage between a joint's last update and the next warm start
// changes)
__device__ __forceinline__ WarmDelta joint_warm_delta(const DJoint& j, Q dqa, Q dqb) {
  float mA = j.inv_mass_a, mB = j.inv_mass_b;
  V3 ra = rotate(dqa, j.frame_a.p), rb = rotate(dqb, j.frame_b.p);
  V3 ang;
  if (j.type == kJointSpherical) {  // spherical_joint.rs:233 warm_start_spherical_joint
    ang = j.spring_impulse3 + j.motor_impulse3;
    ang = ang - j.swing_impulse * j.swing_axis;
    ang = mul_add(ang, j.lower_impulse - j.upper_impulse, j.twist_jacobian);
  } else {
    float axial = j.spring_impulse + j.motor_impulse + j.lower_impulse - j.upper_impulse;
    ang = j.perp_impulse.x * j.perp_axis_x + j.perp_impulse.y * j.perp_axis_y;
    ang = mul_add(ang, axial, j.rotation_axis_z);
  }
  WarmDelta r;
  r.dva = mA * j.linear_impulse;
  r.dwa = mul_mv(j.inv_ia, cross(ra, j.linear_impulse) + ang);
  r.dvb = mB * j.linear_impulse;
  r.dwb = mul_mv(j.inv_ib, cross(rb, j.linear_impulse) + ang);
  return r;
}

// The same applied at once (the overflow colour's joints).
__device__ __noinline__ void warm_start_joint(const DW& w, DJoint& j) {
  DState sa = state_at(w, j.index_a), sb = state_at(w, j.index_b);
  WarmDelta x = joint_warm_delta(j, sa.dq, sb.dq);
  if (sa.flags & kDynamicFlag) { sa.v = sa.v - x.dva; sa.w = sa.w - x.dwa; }
  if (sb.flags & kDynamicFlag) { sb.v = sb.v + x.dvb; sb.w = sb.w + x.dwb; }
  store_state_vw(w, j.index_a, sa);
  store_state_vw(w, j.index_b, sb);
}

// spherical_joint.rs:315-438: the spring, motor, twist limit and cone limit rows of
// solve_spherical_joint (its point constraint is the revolute joint's)
__device__ void spherical_angular(DJoint& j, const StepParams& p, Q qa, Q qb, M3 iA, M3 iB, bool use_bias, V3& wa,
                                  V3& wb) {
  Q rel_q = inv_mul_quat(qa, qb);
  if (j.fixed_rotation || !(j.enable_spring || j.enable_motor || j.enable_twist_limit || j.enable_cone_limit)) return;
  M3 sum = add_mm(iA, iB);
  V3 cdot = wb - wa;
  V3 ang = v3(0, 0, 0);
  if (j.enable_spring) {
    V3 dr = delta_quat_to_rotation(rel_q, j.target_rotation);
    V3 c = -(rotate(qa, dr));
    V3 bias = j.spring_softness.bias_rate * c;
    float ms = j.spring_softness.mass_scale, is = j.spring_softness.impulse_scale;
    V3 imp = (-ms) * mul_mv(j.rotation_mass, cdot + bias) - is * j.spring_impulse3;
    j.spring_impulse3 = j.spring_impulse3 + imp;
    cdot = cdot + mul_mv(sum, imp);
    ang = ang + imp;
  }
  if (j.enable_motor) {
    V3 lambda = -(mul_mv(j.rotation_mass, cdot - j.motor_velocity));
    V3 next = j.motor_impulse3 + lambda;
    float len = length(next);
    float mx = j.max_motor_torque * p.h;
    if (len > mx) next = (mx / len) * next;
    lambda = next - j.motor_impulse3;
    j.motor_impulse3 = next;
    cdot = cdot + mul_mv(sum, lambda);
    ang = ang + lambda;
  }
  if (j.enable_twist_limit) {
    float twist = get_twist_angle(rel_q);
    V3 jac = j.twist_jacobian;
    V3 resp = mul_mv(sum, jac);
    for (int side = 0; side < 2; ++side) {
      float c = side == 0 ? twist - j.lower_twist_angle : j.upper_twist_angle - twist;
      float bias = 0.0f, ms = 1.0f, is = 0.0f;
      if (c > 0.0f) bias = c * p.inv_h;
      else if (use_bias) {
        bias = j.constraint_softness.bias_rate * c;
        ms = j.constraint_softness.mass_scale;
        is = j.constraint_softness.impulse_scale;
      }
      float tcd = side == 0 ? dot(cdot, jac) : -dot(cdot, jac);
      float& imp = side == 0 ? j.lower_impulse : j.upper_impulse;
      float old = imp;
      float di = maxf(-ms * j.twist_mass * (tcd + bias) - is * old, -old);
      imp = old + di;
      if (side == 0) {
        cdot = mul_add(cdot, di, resp);
        ang = mul_add(ang, di, jac);
      } else {
        cdot = cdot - di * resp;
        ang = ang - di * jac;
      }
    }
  }
  if (j.enable_cone_limit) {
    float swing = get_swing_angle(rel_q);
    float c = j.cone_angle - swing;
    float bias = 0.0f, ms = 1.0f, is = 0.0f;
    if (c > 0.0f) bias = c * p.inv_h;
    else if (use_bias) {
      bias = j.constraint_softness.bias_rate * c;
      ms = j.constraint_softness.mass_scale;
      is = j.constraint_softness.impulse_scale;
    }
    float scd = -dot(cdot, j.swing_axis);
    float old = j.swing_impulse;
    float di = maxf(-ms * j.swing_mass * (scd + bias) - is * old, -old);
    j.swing_impulse = old + di;
    ang = ang - di * j.swing_axis;
  }
  wa = wa - mul_mv(iA, ang);
  wb = wb + mul_mv(iB, ang);
}

// revolute_joint.rs:316 solve_revolute_joint
__device__ __noinline__ void solve_joint(const DW& w, const StepParams& p, DJoint& j, bool use_bias) {
  float mA = j.inv_mass_a, mB = j.inv_mass_b;
  M3 iA = j.inv_ia, iB = j.inv_ib;
  DState sa = state_at(w, j.index_a), sb = state_at(w, j.index_b);
  V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
  bool fixed = j.fixed_rotation != 0;
  Q qa = mul_quat(sa.dq, j.frame_a.q);
  Q qb = mul_quat(sb.dq, j.frame_b.q);
  if (j.type == kJointSpherical) {
    spherical_angular(j, p, qa, qb, iA, iB, use_bias, wa, wb);
    fixed = true;  // the revolute rows below do not apply
  }
  if (dot_quat(qa, qb) < 0.0f) qb = quat(v3(-qb.v.x, -qb.v.y, -qb.v.z), -qb.s);
  Q rq = inv_mul_quat(qa, qb);
  if (!fixed && (j.enable_spring || j.enable_motor || j.enable_limit)) {
    V3 axis = j.rotation_axis_z;
    V3 ga = mul_mv(iA, axis), gb = mul_mv(iB, axis);
    float k = dot(axis, ga + gb);
    float acd = dot(wb - wa, axis);
    float ai = 0.0f;
    if (j.enable_spring) {
      float angle = get_twist_angle(rq);
      float c = angle - j.target_angle;
      float bias = j.spring_softness.bias_rate * c;
      float ms = j.spring_softness.mass_scale, is = j.spring_softness.impulse_scale;
      float di = -ms * j.axial_mass * (acd + bias) - is * j.spring_impulse;
      j.spring_impulse += di;
      acd += k * di;
      ai += di;
    }
    if (j.enable_motor) {
      float cdot = acd - j.motor_speed;
      float old = j.motor_impulse;
      float mx = j.max_motor_torque * p.h;
      float di = clampf(-j.axial_mass * cdot, -mx - old, mx - old);
      j.motor_impulse = old + di;
      acd += k * di;
      ai += di;
    }
    if (j.enable_limit) {
      float angle = get_twist_angle(rq);
      {
        float c = angle - j.lower_angle;
        float bias = 0.0f, ms = 1.0f, is = 0.0f;
        if (c > 0.0f) bias = c * p.inv_h;
        else if (use_bias) {
          bias = j.constraint_softness.bias_rate * c;
          ms = j.constraint_softness.mass_scale;
          is = j.constraint_softness.impulse_scale;
        }
        float old = j.lower_impulse;
        float di = maxf(-ms * j.axial_mass * (acd + bias) - is * old, -old);
        j.lower_impulse = old + di;
        acd += k * di;
        ai += di;
      }
      {
        float c = j.upper_angle - angle;
        float bias = 0.0f, ms = 1.0f, is = 0.0f;
        if (c > 0.0f) bias = c * p.inv_h;
        else if (use_bias) {
          bias = j.constraint_softness.bias_rate * c;
          ms = j.constraint_softness.mass_scale;
          is = j.constraint_softness.impulse_scale;
        }
        float cdot = -acd;
        float old = j.upper_impulse;
        float di = maxf(-ms * j.axial_mass * (cdot + bias) - is * old, -old);
        j.upper_impulse = old + di;
        ai -= di;
      }
    }
    wa = wa - ai * ga;
    wb = wb + ai * gb;
  }
  if (!fixed) {
    V2 bias = v2(0, 0);
    float ms = 1.0f, is = 0.0f;
    if (use_bias) {
      V2 c = v2(rq.v.x, rq.v.y);
      bias = v2(j.constraint_softness.bias_rate * c.x, j.constraint_softness.bias_rate * c.y);
      ms = j.constraint_softness.mass_scale;
      is = j.constraint_softness.impulse_scale;
    }
    V3 px = 0.5f * rotate(qa, rq.s * v3(1, 0, 0) + cross(rq.v, v3(1, 0, 0)));
    V3 py = 0.5f * rotate(qa, rq.s * v3(0, 1, 0) + cross(rq.v, v3(0, 1, 0)));
    j.perp_axis_x = px;
    j.perp_axis_y = py;
    M3 sum = add_mm(iA, iB);
    float kxx = dot(px, mul_mv(sum, px));
    float kyy = dot(py, mul_mv(sum, py));
    float kxy = dot(px, mul_mv(sum, py));
    M2 K;
    K.cx = v2(kxx, kxy);
    K.cy = v2(kxy, kyy);
    V3 wr = wb - wa;
    V2 cdot = v2(dot(wr, px), dot(wr, py));
    V2 old = j.perp_impulse;
    V2 sol = solve2(K, v2(cdot.x + bias.x, cdot.y + bias.y));
    V2 di = v2((-ms) * sol.x - is * old.x, (-ms) * sol.y - is * old.y);
    j.perp_impulse = v2(j.perp_impulse.x + di.x, j.perp_impulse.y + di.y);
    V3 ang = di.x * px + di.y * py;
    wa = wa - mul_mv(iA, ang);
    wb = wb + mul_mv(iB, ang);
  }
  {
    V3 ra = rotate(sa.dq, j.frame_a.p), rb = rotate(sb.dq, j.frame_b.p);
    V3 cdot = (vb + cross(wb, rb)) - va - cross(wa, ra);
    V3 bias = v3(0, 0, 0);
    float ms = 1.0f, is = 0.0f;
    if (use_bias) {
      V3 sep = ((sb.dp - sa.dp) + (rb - ra)) + j.delta_center;
      bias = j.constraint_softness.bias_rate * sep;
      ms = j.constraint_softness.mass_scale;
      is = j.constraint_softness.impulse_scale;
    }
    V3 b = solve_point_constraint(mA, mB, j.inv_ia, j.inv_ib, ra, rb, cdot + bias);
    V3 imp = (-ms) * b - is * j.linear_impulse;
    j.linear_impulse = j.linear_impulse + imp;
    va = va - mA * imp;
    wa = wa - mul_mv(iA, cross(ra, imp));
    vb = vb + mB * imp;
    wb = wb + mul_mv(iB, cross(rb, imp));
  }
  if (sa.flags & kDynamicFlag) { sa.v = va; sa.w = wa; }
  if (sb.flags & kDynamicFlag) { sb.v = vb; sb.w = wb; }
  store_state_vw(w, j.index_a, sa);
  store_state_vw(w, j.index_b, sb);
}

// First position in [lo, hi) of joint_list whose joint belongs to sub-world >= wi (the list of
// one color is in joint id order, and joint ids are grouped by sub-world).
__device__ int first_joint_of_world(const DW& w, int lo, int hi, int wi) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (w.joints[w.joint_list[mid]].world < wi) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// The overflow color: in each sub-world, one thread runs its overflow joints then its overflow
// contacts in list order (overflow_contact_solver.rs:41); sub-worlds run side by side.
__device__ void run_overflow(const DW& w, const StepParams& p, const JointRanges& jr, int stage) {
  int stride = gridDim.x * blockDim.x;
  for (int wi = blockIdx.x * blockDim.x + threadIdx.x; wi < w.n_worlds; wi += stride) {
    if (stage != kRestitution && jr.off[kOverflowIndex + 1] > jr.off[kOverflowIndex]) {
      int j0 = first_joint_of_world(w, jr.off[kOverflowIndex], jr.off[kOverflowIndex + 1], wi);
      int j1 = first_joint_of_world(w, j0, jr.off[kOverflowIndex + 1], wi + 1);
      for (int t = j0; t < j1; ++t) {
        DJoint& j = w.joints[w.joint_list[t]];
        if (stage == kWarm) warm_start_joint(w, j);
        else solve_joint(w, p, j, stage == kPush);
      }
    }
    int base = w.world_cbase[wi], n = w.ovf_count[wi];
    if (n == 0) continue;
    if (stage == kWarm) warm_start_overflow(w, base, n);
    else if (stage == kPush) push_overflow(w, p, base, n);
    else if (stage == kRelax) relax_overflow(w, p, base, n);
    else restitution_overflow(w, p, base, n);
  }
}

// Warm start of a step's first substep: every coloured constraint and joint records its change
// in its bodies' slots and marks them (later substeps' changes are recorded by the relax
// updates before them). bw_mask is zero at launch.
__global__ void __launch_bounds__(256) k_warm_slots(DW w, JointRanges jr) {
  __shared__ int coff[kOverflowIndex + 1];
  if (threadIdx.x <= kOverflowIndex) coff[threadIdx.x] = w.ctl->color_offset[threadIdx.x];
  __syncthreads();
  const int n_col = coff[kOverflowIndex], n_jnt = jr.off[kOverflowIndex];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_col + n_jnt; i += gridDim.x * blockDim.x) {
    if (i < n_col) {
      const int k = i;
      int c = 0;
      while (coff[c + 1] <= k) ++c;
      CData d;
      load_direct(w.cp, k, kWarm, d);
      float ni[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) ni[q] = d.pimp[q].x;
      // only a dynamic body takes a warm start (a kinematic body may have several constraints
      // in one colour)
      const int ia = dynamic_index(w, d.c.ia), ib = dynamic_index(w, d.c.ib);
      put_warm_delta(w, ia, ib, c,
                     contact_warm_delta(d.c, d.t1, d.t2, d.ca, d.cb, d.fr, d.roll, d.pra, d.prb, ni));
      mark_warm_slot(w, ia, c);
      mark_warm_slot(w, ib, c);
    } else {
      const int t = i - n_col;
      int c = 0;
      while (jr.off[c + 1] <= t) ++c;
      const DJoint& j = w.joints[w.joint_list[t]];
      DState sa = state_at(w, j.index_a), sb = state_at(w, j.index_b);
      const int ia = (sa.flags & kDynamicFlag) ? j.index_a : -1, ib = (sb.flags & kDynamicFlag) ? j.index_b : -1;
      put_warm_delta(w, ia, ib, c, joint_warm_delta(j, sa.dq, sb.dq));
      mark_warm_slot(w, ia, c);
      mark_warm_slot(w, ib, c);
    }
  }
}

// Phase codes: contact phases stage * 32 + color; the rest as below.
// kPhaseIntegrateVelocityWarm: integrate velocities, then each body's warm start from its
// slots; kPhaseBodyWarm: the slots alone (after the overflow colour's warm start).
constexpr int kPhaseIntegrateVelocity = 1000, kPhaseIntegratePosition = 1001, kPhaseIntegrateVelocityWarm = 1002,
              kPhaseBodyWarm = 1003, kPhaseOverflow = 2000;

// Record of the solver's inputs kept while the adjoint replays a step (kTape): per substep
// three body rows (before integrate-velocities, before and after integrate-positions), the
// velocities and normal impulses each push and relax update reads, the friction and twist
// impulses each relax update reads, and the final friction and twist impulses.
struct SolveTape {
  DState* body;    // [substep][3][n_awake]
  float4* push;    // [substep][4][cap]: vA|l0, wA|l1, vB|l2, wB|l3
  float4* relax;   // [substep][5][cap]: the same, then fr.x, fr.y, twist
  float4* fin;     // [cap]
  float4* rest;    // [iteration][6][cap]: vA|l0, wA|l1, vB|l2, wB|l3, the points' total normal
                   // impulses, their restitution impulses (before each restitution update)
  float4* joint;   // [substep][push, relax][6][n_joints]: vA|lin.x, wA|lin.y, vB|lin.z, wB|perp.x,
                   // perp.y spring motor lower, upper (before each joint solve)
  float4* jwarm;   // [substep][4][n_joints]: the state the next substep's warm start reads, after
                   // relax: lin|perp.x, perp.y spring motor lower, upper|px, py|0
};

// A revolute joint's inputs before a push or relax solve (the adjoint replays it)
__device__ __forceinline__ void tape_joint(const DW& w, const SolveTape& tp, int sub, int stage, int ji,
                                           const DJoint& j) {
  const size_t nj = (size_t)w.n_joints;
  const DState sa = state_at(w, j.index_a), sb = state_at(w, j.index_b);
  float4* rows = tp.joint + (size_t)(sub * 2 + (stage == kRelax ? 1 : 0)) * 6 * nj;
  rows[ji] = make_float4(sa.v.x, sa.v.y, sa.v.z, j.linear_impulse.x);
  rows[nj + ji] = make_float4(sa.w.x, sa.w.y, sa.w.z, j.linear_impulse.y);
  rows[2 * nj + ji] = make_float4(sb.v.x, sb.v.y, sb.v.z, j.linear_impulse.z);
  rows[3 * nj + ji] = make_float4(sb.w.x, sb.w.y, sb.w.z, j.perp_impulse.x);
  rows[4 * nj + ji] = make_float4(j.perp_impulse.y, j.spring_impulse, j.motor_impulse, j.lower_impulse);
  rows[5 * nj + ji] = make_float4(j.upper_impulse, 0.0f, 0.0f, 0.0f);
}
// A joint's state after a relax solve, which the warm start of the next substep reads
__device__ __forceinline__ void tape_joint_warm(const DW& w, const SolveTape& tp, int sub, int ji, const DJoint& j) {
  const size_t nj = (size_t)w.n_joints;
  float4* rows = tp.jwarm + (size_t)sub * 4 * nj;
  rows[ji] = make_float4(j.linear_impulse.x, j.linear_impulse.y, j.linear_impulse.z, j.perp_impulse.x);
  rows[nj + ji] = make_float4(j.perp_impulse.y, j.spring_impulse, j.motor_impulse, j.lower_impulse);
  rows[2 * nj + ji] = make_float4(j.upper_impulse, j.perp_axis_x.x, j.perp_axis_x.y, j.perp_axis_x.z);
  rows[3 * nj + ji] = make_float4(j.perp_axis_y.x, j.perp_axis_y.y, j.perp_axis_y.z, 0.0f);
}

__device__ __forceinline__ void tape_restitution(const DW& w, const SolveTape& tp, int it, int k, const CData& d) {
  const int cap = w.cp.cap;
  DState ba = state_at(w, d.c.ia), bb = state_at(w, d.c.ib);
  float l[4], tot[4], rest[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    bool on = q < d.c.pc;
    l[q] = on ? d.pimp[q].x : 0.0f;
    tot[q] = on ? d.pimp[q].y : 0.0f;
    rest[q] = on ? d.prest[q] : 0.0f;
  }
  float4* rows = tp.rest + (size_t)it * 6 * cap;
  rows[k] = make_float4(ba.v.x, ba.v.y, ba.v.z, l[0]);
  rows[(size_t)cap + k] = make_float4(ba.w.x, ba.w.y, ba.w.z, l[1]);
  rows[2 * (size_t)cap + k] = make_float4(bb.v.x, bb.v.y, bb.v.z, l[2]);
  rows[3 * (size_t)cap + k] = make_float4(bb.w.x, bb.w.y, bb.w.z, l[3]);
  rows[4 * (size_t)cap + k] = make_float4(tot[0], tot[1], tot[2], tot[3]);
  rows[5 * (size_t)cap + k] = make_float4(rest[0], rest[1], rest[2], rest[3]);
}

__device__ __forceinline__ void tape_contact(const DW& w, const SolveTape& tp, int sub, int stage, int k,
                                             const CData& d) {
  const int cap = w.cp.cap;
  DState ba = state_at(w, d.c.ia), bb = state_at(w, d.c.ib);
  float l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) l[q] = q < d.c.pc ? d.pimp[q].x : 0.0f;
  float4* rows = stage == kPush ? tp.push + (size_t)sub * 4 * cap : tp.relax + (size_t)sub * 5 * cap;
  rows[k] = make_float4(ba.v.x, ba.v.y, ba.v.z, l[0]);
  rows[(size_t)cap + k] = make_float4(ba.w.x, ba.w.y, ba.w.z, l[1]);
  rows[2 * (size_t)cap + k] = make_float4(bb.v.x, bb.v.y, bb.v.z, l[2]);
  rows[3 * (size_t)cap + k] = make_float4(bb.w.x, bb.w.y, bb.w.z, l[3]);
  if (stage == kRelax) rows[4 * (size_t)cap + k] = make_float4(d.fr.x, d.fr.y, d.cb.w, 0.0f);
}

// Persistent solver. kGrid: one cooperative launch over the whole GPU, phases separated by
// grid_sync_acq_rel, compiled for two blocks per SM (128 registers; the batch's colours hold
// more items than one block per SM has threads); otherwise one thread-block cluster separated
// by barrier.cluster.
template <bool kGrid, bool kTape>
__global__ void __launch_bounds__(kSolveThreads, kGrid ? 2 : 1) k_solve(DW w, StepParams p, JointRanges jr, SolveTape tp) {
  __shared__ int coff[25];
  __shared__ int phases[3 * 25 + 2];  // one substep
  __shared__ int rphases[25];         // one restitution iteration
  __shared__ int n_ph_s, n_rph_s, n_ovf_s;
  if (threadIdx.x < 25) coff[threadIdx.x] = threadIdx.x < 24 ? w.ctl->color_offset[threadIdx.x] : w.ctl->color_offset[23];
  __syncthreads();
  if (threadIdx.x == 0) {
    int n_ovf = w.ctl->overflow_count;
    bool ovf_work = n_ovf > 0 || jr.off[kOverflowIndex + 1] > jr.off[kOverflowIndex];
    int n = 0;
    if (ovf_work) {
      phases[n++] = kPhaseIntegrateVelocity;
      phases[n++] = kPhaseOverflow + kWarm;
      phases[n++] = kPhaseBodyWarm;
    } else {
      phases[n++] = kPhaseIntegrateVelocityWarm;
    }
    for (int stage = kPush; stage <= kRelax; ++stage) {
      if (stage == kRelax) phases[n++] = kPhaseIntegratePosition;
      if (ovf_work) phases[n++] = kPhaseOverflow + stage;
      for (int c = 0; c < kOverflowIndex; ++c)
        if (coff[c + 1] != coff[c] || jr.off[c + 1] != jr.off[c]) phases[n++] = stage * 32 + c;
    }
    int m = 0;
    if (w.ctl->any_restitution && p.restitution_iterations > 0) {
      if (n_ovf > 0) rphases[m++] = kPhaseOverflow + kRestitution;
      for (int c = 0; c < kOverflowIndex; ++c)
        if (coff[c + 1] != coff[c]) rphases[m++] = kRestitution * 32 + c;
    }
    n_ph_s = n;
    n_rph_s = m;
    n_ovf_s = n_ovf;
  }
  __syncthreads();
  const int n_ph = n_ph_s, n_rph = n_rph_s;
  const int main_phases = p.substeps * n_ph;
  const int total_phases = main_phases + (n_rph > 0 ? p.restitution_iterations * n_rph : 0);
  auto phase_at = [&](int s) { return s < main_phases ? phases[s % n_ph] : rphases[(s - main_phases) % n_rph]; };
  // Items of colour c: t < nj is joint t, t in [nj, total) constraint coff[c] + t - nj, in every
  // stage (restitution skips the joints), so one thread owns a constraint in all its phases.
  auto contact_range = [&](int ph, int& nj, int& total) {
    const int c = ph & 31;
    nj = jr.off[c + 1] - jr.off[c];
    total = nj + (coff[c + 1] - coff[c]);
  };
  const int stride = gridDim.x * blockDim.x;
  // Items go to threads 32 at a time, dealt across the blocks (chunk j to block j % gridDim.x):
  // a colour with fewer items than the launch has threads occupies every SM with a few warps
  // instead of filling the first blocks, and a phase's time follows the warps per SM.
  const int g = (((int)threadIdx.x >> 5) * (int)gridDim.x + (int)blockIdx.x) * 32 + ((int)threadIdx.x & 31);
  // The contact that a thread of a block's first warp holds in the next phase (when the phase's
  // items are at most one per thread) is staged in shared memory while the phase before it
  // ends, so after the barrier only the body states are fetched.
  __shared__ StageBuf stage_buf;
  bool staged = false;
  // The warm-start slots a body uses are marked by k_warm_slots before the launch and do not
  // change during it: the mask of the thread's first body is read once, so the integrate-velocity
  // phases can issue the slot loads without waiting for it.
  const uint32_t first_mask = g < w.n_awake ? w.bw_mask[g] : 0u;
  int bar = 0;
  for (int s = 0; s < total_phases; ++s) {
    int ph = phase_at(s);
    const int sub = s / n_ph;
    if (ph == kPhaseIntegrateVelocity || ph == kPhaseIntegrateVelocityWarm) {
      for (int i = g; i < w.n_awake; i += stride) {
        if (kTape) tp.body[((size_t)sub * 3) * w.n_awake + i] = w.states[i];
        IVIn in = load_iv(w, i);
        uint32_t m = ph == kPhaseIntegrateVelocityWarm ? (i == g ? first_mask : w.bw_mask[i]) : 0u;
        WarmSlots ws;
        load_warm_slots(w, i, m, ws);  // in flight while the velocity is integrated
        V3 v, wv;
        integrate_velocity(p, in, v, wv);
        warm_body(w, i, m, ws, v, wv);
        DState& st = w.states[i];
        st.v = v;
        st.w = wv;
      }
    } else if (ph == kPhaseBodyWarm) {
      for (int i = g; i < w.n_awake; i += stride) {
        uint32_t m = w.bw_mask[i];
        DState st = w.states[i];
        if ((st.flags & kDynamicFlag) && m != 0u) {
          V3 v = st.v, wv = st.w;
          WarmSlots ws;
          load_warm_slots(w, i, m, ws);
          warm_body(w, i, m, ws, v, wv);
          w.states[i].v = v;
          w.states[i].w = wv;
        }
      }
    } else if (ph == kPhaseIntegratePosition) {
      for (int i = g; i < w.n_awake; i += stride) {
        DState st = w.states[i];
        if (kTape) tp.body[((size_t)sub * 3 + 1) * w.n_awake + i] = st;
        apply_ip(w, p, i, st);
        if (kTape) tp.body[((size_t)sub * 3 + 2) * w.n_awake + i] = w.states[i];
      }
    } else if (ph >= kPhaseOverflow) {
      run_overflow(w, p, jr, ph - kPhaseOverflow);
    } else {
      int stage = ph >> 5, c = ph & 31;
      int nj, total;
      contact_range(ph, nj, total);
      const int warm_color = stage == kRelax && s < main_phases && sub + 1 < p.substeps ? c : -1;
      // The colour's contacts, then its joints: no two items of one colour share a dynamic
      // body, so their order does not change any result. Each thread keeps its items of the
      // colour (t = g, g + stride, ...).
      for (int t = g >= nj ? g : g + ((nj - g + stride - 1) / stride) * stride; t < total; t += stride) {
        int k = coff[c] + (t - nj);
        CData d;
        if (staged && t == g) load_staged(stage_buf, (int)threadIdx.x, stage, d);
        else load_direct(w.cp, k, stage, d);
        if (kTape && (stage == kPush || stage == kRelax) && s < main_phases) tape_contact(w, tp, sub, stage, k, d);
        if (kTape && stage == kRestitution && tp.rest && d.c.restitution > 0.0f)
          tape_restitution(w, tp, (s - main_phases) / n_rph, k, d);
        run_contact(w, p, k, stage, d, warm_color);
      }
      for (int tj = g; stage != kRestitution && tj < nj; tj += stride) {
        const int ji = w.joint_list[jr.off[c] + tj];
        DJoint& j = w.joints[ji];
        if (kTape && tp.joint && s < main_phases) tape_joint(w, tp, sub, stage, ji, j);
        solve_joint(w, p, j, stage == kPush);
        if (kTape && tp.joint && warm_color >= 0) tape_joint_warm(w, tp, sub, ji, j);
        if (warm_color >= 0) {
          DState sa = state_at(w, j.index_a), sb = state_at(w, j.index_b);
          put_warm_delta(w, (sa.flags & kDynamicFlag) ? j.index_a : -1, (sb.flags & kDynamicFlag) ? j.index_b : -1, c,
                         joint_warm_delta(j, sa.dq, sb.dq));
        }
      }
    }
    staged = false;
    if (s + 1 < total_phases) {
      const int nph = phase_at(s + 1);
      const int nstage = nph >> 5;
      if (nph < kPhaseIntegrateVelocity && (nstage == kPush || nstage == kRelax)) {
        int nj2, total2;
        contact_range(nph, nj2, total2);
        // the contacts follow the colour's joints (items nj2..total2-1); a thread's first
        // contact of the colour is item g when g >= nj2, and its only one when total2 <= stride
        if (total2 <= stride && threadIdx.x < 32 && g >= nj2 && g < total2) {
          stage_constraint(w.cp, coff[nph & 31] + (g - nj2), nstage, stage_buf, (int)threadIdx.x);
          staged = true;
        }
      }
    }
    if (!phase_sync<kGrid>(w.ctl, bar)) {
      asm volatile("cp.async.wait_all;" ::: "memory");
      return;
    }
  }
  // store impulses (contact_solver.rs:1258; overflow_contact_solver.rs:688)
  for (int wi = g; wi < w.n_worlds; wi += stride) store_overflow(w, w.world_cbase[wi], w.ovf_count[wi]);
  for (int k = g; k < coff[kOverflowIndex]; k += stride) {
    if (kTape) tp.fin[k] = make_float4(w.cp.fr[k].x, w.cp.fr[k].y, w.cp.cb[k].w, 0.0f);
    store_constraint(w, k);
  }
}

// shape_runtime.rs:370 compute_shape_aabb of a shape under a transform
__device__ AABB shape_box(const DW& w, const DShape& sh, Xf t) {
  if (sh.type == kHull) return aabb_transform(t, w.hulls[sh.hull].bounds);  // hull_queries.rs:16
  if (sh.type == kSphere) {                                                   // sphere.rs:27
    V3 c = xf_point(t, sh.sphere.center);
    float r = sh.sphere.radius;
    V3 e = v3(r, r, r);
    return aabb(c - e, c + e);
  }
  V3 c1 = xf_point(t, sh.capsule.c1), c2 = xf_point(t, sh.capsule.c2);          // capsule.rs:66
  float r = sh.capsule.radius;
  V3 e = v3(r, r, r);
  return aabb(min3(c1, c2) - e, max3(c1, c2) + e);
}

// solver_integration.rs:587 finalize_body_range (sleep disabled: bodies never sleep). A fast
// body is queued for the continuous pass, which sets its bounds (solver_integration.rs:540-566).
__global__ void k_finalize(DW w, StepParams p) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n_awake) return;
  DState st = w.states[i];
  DSim sim = w.asims[i];
  float dt = p.dt;
  V3 v = st.v, wv = st.w;
  V3 lom = inv_rotate(sim.q, wv);
  V3 ldr = inv_rotate(sim.q, st.dq.v);
  Pos center = {sim.cx, sim.cy, sim.cz};
  center = offset_pos(center, st.dp);
  sim.cx = center.x; sim.cy = center.y; sim.cz = center.z;
  sim.q = normalize_quat(mul_quat(st.dq, sim.q));
  V3 varc = modified_cross(abs3(lom), sim.max_extent);
  float maxv = length(v) + length(varc);
  V3 rarc = modified_cross(abs3(ldr), sim.max_extent);
  float maxdp = length(st.dp) + 2.0f * length(rarc);
  st.dp = v3(0, 0, 0);
  st.dq = qid();
  Pos tp = offset_pos(center, -rotate(sim.q, sim.local_center));
  sim.px = tp.x; sim.py = tp.y; sim.pz = tp.z;
  sim.force = v3(0, 0, 0);
  sim.torque = v3(0, 0, 0);
  sim.flags &= ~(kIsFast | kTransient);
  st.flags &= ~kTransient;
  float max_motion = maxf(maxdp, maxv * dt);
  // solver_integration.rs:626-627 asserts finite velocities here; the device raises
  // NS_ERR_NONFINITE instead (first error wins) and keeps the body's old fat AABB, so a
  // non-finite pose never reaches the broadphase grid or the continuous pass
  bool finite = isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(wv.x) && isfinite(wv.y) &&
                isfinite(wv.z) && isfinite(sim.cx) && isfinite(sim.cy) && isfinite(sim.cz) &&
                isfinite(sim.q.v.x) && isfinite(sim.q.v.y) && isfinite(sim.q.v.z) && isfinite(sim.q.s);
  if (!finite) atomicCAS(&w.ctl->error, 0, kErrNonFinite);
  if (finite && p.enable_continuous && (sim.flags & kDynamicFlag) && max_motion > sim.safety_factor * sim.min_extent) {
    sim.flags |= kIsFast;
    add_converged(&w.ctl->fast_flags);
    // the continuous pass (k_continuous, or k_bullets for a bullet) sweeps it from (cx0, q0)
    // and updates its bounds
    if (sim.flags & kIsBullet) w.bullet_list[atomicAdd(&w.ctl->bullet_count, 1)] = i;
    else w.fast_list[atomicAdd(&w.ctl->fast_count, 1)] = i;
  } else {
    sim.cx0 = sim.cx; sim.cy0 = sim.cy; sim.cz0 = sim.cz;
    sim.q0 = sim.q;
  }
  M3 R = matrix_from_quat(sim.q);
  sim.inv_inertia_world = mul_mm(mul_mm(R, sim.inv_inertia_local), transpose(R));
  if (finite && (sim.flags & kIsFast) == 0) {
    WXf xf_;
    xf_.p = tp; xf_.q = sim.q;
    float spec = speculative_distance();
    for (int k = sim.shape_begin; k < sim.shape_end; ++k) {
      int sid = w.body_shapes[k];
      const DShape& sh = w.shapes[sid];
      // shape_runtime.rs:405-427 compute_fat_shape_aabb
      AABB a = offset_aabb(aabb_inflate(shape_box(w, sh, xf(v3(0, 0, 0), xf_.q)), spec), xf_.p);
      w.saabb[sid] = a;
      if (!aabb_contains(w.fat[sid], a)) {
        w.fat[sid] = aabb_inflate(a, sh.aabb_margin);
        w.moved[sid] = 1;
        add_converged(&w.ctl->moved_count);
      }
    }
  }
  w.states[i] = st;
  w.asims[i] = sim;
}

// The proxy of a shape (shape_runtime.rs:643 make_shape_proxy) and its centroid
// (shape_runtime.rs:434 get_shape_centroid), both in the body's frame.
__device__ void shape_proxy(const DW& w, const DShape& sh, Proxy* p, V3* centroid) {
  if (sh.type == kHull) {
    const Hull& h = w.hulls[sh.hull];
    for (int k = 0; k < kHullVertexCount; ++k) p->pts[k] = h.points[k];
    p->count = kHullVertexCount;
    p->radius = 0.0f;
    *centroid = h.center;
  } else if (sh.type == kSphere) {
    p->pts[0] = sh.sphere.center;
    p->count = 1;
    p->radius = sh.sphere.radius;
    *centroid = sh.sphere.center;
  } else {
    p->pts[0] = sh.capsule.c1;
    p->pts[1] = sh.capsule.c2;
    p->count = 2;
    p->radius = sh.capsule.radius;
    *centroid = lerp(sh.capsule.c1, sh.capsule.c2, 0.5f);
  }
}

// world_runtime.rs:929 make_relative_sweep: from (center0, rotation0) to the current pose
__device__ __forceinline__ Sweep sweep_of(const DSim& s, Pos base) {
  Sweep sw;
  sw.c1 = sub_pos(Pos{s.cx0, s.cy0, s.cz0}, base);
  sw.c2 = sub_pos(Pos{s.cx, s.cy, s.cz}, base);
  sw.q1 = s.q0;
  sw.q2 = s.q;
  sw.local_center = s.local_center;
  return sw;
}

// continuous.rs:337 solve_continuous for one fast (non-bullet) body: each of its shapes that
// is fast on its own (continuous.rs:124) is swept against the static shapes of its sub-world
// whose fat bounds overlap the shape's swept box, in shape order; the earliest hit moves the
// body back along its sweep. Each time of impact is bounded by the best fraction so far, so with
// two hits the visiting order can change the last bits (the reference walks its static tree).
// Fast bodies are independent of one another (they only read static bodies), so one thread per
// fast body gives the reference's serial pass.
__device__ void continuous_finish(const DW& w, const StepParams& p, int i, DSim sim, DState st, const Sweep& sweep,
                                  Pos base, float fraction);

// continuous.rs:262-299: the time of impact of a fast shape (proxy fp on sweep) against shape
// sid on its own sweep, bounded by the best fraction so far; returns the new best fraction.
__device__ float candidate_fraction(const DW& w, int sid, const Proxy& fp, const Sweep& sweep, Pos base,
                                    float fraction) {
  const DShape& ss = w.shapes[sid];
  Proxy sp;
  V3 unused;
  shape_proxy(w, ss, &sp, &unused);
  ToiResult r = time_of_impact(sp, fp, sweep_of(sim_of(w, ss.enc), base), sweep, fraction);
  return (0.0f < r.fraction && r.fraction < fraction) ? r.fraction : fraction;
}

__device__ void continuous_body(const DW& w, const StepParams& p, int i) {
  DSim sim = w.asims[i];
  DState st = w.states[i];
  const Pos base = {sim.cx0, sim.cy0, sim.cz0};
  const Sweep sweep = sweep_of(sim, base);
  const Xf xf1 = xf(sweep.c1 - rotate(sweep.q1, sweep.local_center), sweep.q1);
  const Xf xf2 = xf(sweep.c2 - rotate(sweep.q2, sweep.local_center), sweep.q2);
  const float chord = 2.0f * length(inv_mul_quat(sweep.q1, sweep.q2).v);
  float fraction = 1.0f;
  for (int k = sim.shape_begin; k < sim.shape_end; ++k) {
    const int fid = w.body_shapes[k];
    const DShape& fs = w.shapes[fid];
    const int s0 = w.static_off[fs.world], s1 = w.static_off[fs.world + 1];
    Proxy fp;
    V3 lc;
    shape_proxy(w, fs, &fp, &lc);
    AABB box1 = w.saabb[fid];
    AABB box2 = offset_aabb(shape_box(w, fs, xf2), base);
    w.saabb[fid] = box2;
    // continuous.rs:124 is_shape_fast
    float radius, min_extent;
    if (fs.type == kSphere) {
      radius = fs.sphere.radius;
      min_extent = fs.sphere.radius;
    } else if (fs.type == kCapsule) {
      radius = 0.5f * distance(fs.capsule.c1, fs.capsule.c2) + fs.capsule.radius;
      min_extent = fs.capsule.radius;
    } else {
      const Hull& h = w.hulls[fs.hull];
      V3 far = v3((lc.x - h.bounds.lo.x) > (h.bounds.hi.x - lc.x) ? h.bounds.lo.x : h.bounds.hi.x,
                  (lc.y - h.bounds.lo.y) > (h.bounds.hi.y - lc.y) ? h.bounds.lo.y : h.bounds.hi.y,
                  (lc.z - h.bounds.lo.z) > (h.bounds.hi.z - lc.z) ? h.bounds.lo.z : h.bounds.hi.z);
      radius = distance(far, lc);
      min_extent = h.inner_radius;
    }
    float motion = distance(xf_point(xf1, lc), xf_point(xf2, lc)) + chord * radius;
    if (!(motion > sim.safety_factor * min_extent)) continue;
    AABB swept = aabb(min3(box1.lo, box2.lo), max3(box1.hi, box2.hi));
    for (int t = s0; t < s1; ++t) {
      const int sid = w.static_list[t];
      if (!aabb_overlaps(w.fat[sid], swept) || !should_create_pair(w, sid, fid)) continue;
      fraction = candidate_fraction(w, sid, fp, sweep, base, fraction);
    }
  }
  continuous_finish(w, p, i, sim, st, sweep, base, fraction);
}

// The end of solve_continuous for body i with its earliest fraction (continuous.rs:452-590):
// moved back to the time of impact with the lost gravity, or kept, and its bounds refreshed.
__device__ void continuous_finish(const DW& w, const StepParams& p, int i, DSim sim, DState st, const Sweep& sweep,
                                  Pos base, float fraction) {
  const float spec = speculative_distance();
  if (fraction < 1.0f) {
    // move the body back to the time of impact (continuous.rs:452-470)
    Q q = nlerp(sweep.q1, sweep.q2, fraction);
    V3 c = lerp(sweep.c1, sweep.c2, fraction);
    V3 origin = c - rotate(q, sweep.local_center);
    Pos tp = offset_pos(base, origin);
    Pos center = offset_pos(base, c);
    sim.px = tp.x; sim.py = tp.y; sim.pz = tp.z;
    sim.q = q;
    sim.cx = center.x; sim.cy = center.y; sim.cz = center.z;
    sim.cx0 = center.x; sim.cy0 = center.y; sim.cz0 = center.z;
    sim.q0 = q;
    sim.flags |= kHadToi;
    // the gravity of the time lost (other forces are ignored, as in the reference)
    float time_loss = (1.0f - fraction) * p.dt;
    V3 dv = (-time_loss * sim.gravity_scale) * p.gravity;
    dv.x = (st.flags & kLockLinX) ? 0.0f : dv.x;
    dv.y = (st.flags & kLockLinY) ? 0.0f : dv.y;
    dv.z = (st.flags & kLockLinZ) ? 0.0f : dv.z;
    st.v = st.v + dv;
    for (int k = sim.shape_begin; k < sim.shape_end; ++k) {
      const int sid = w.body_shapes[k];
      const DShape& sh = w.shapes[sid];
      AABB a = offset_aabb(aabb_inflate(shape_box(w, sh, xf(v3(0, 0, 0), q)), spec), tp);
      w.saabb[sid] = a;
      if (!aabb_contains(w.fat[sid], a)) {
        w.fat[sid] = aabb_inflate(a, sh.aabb_margin);
        w.moved[sid] = 1;
        add_converged(&w.ctl->moved_count);
      }
    }
  } else {
    sim.cx0 = sim.cx; sim.cy0 = sim.cy; sim.cz0 = sim.cz;
    sim.q0 = sim.q;
    // the swept end box stands as the shape's bounds (continuous.rs:573-590)
    for (int k = sim.shape_begin; k < sim.shape_end; ++k) {
      const int sid = w.body_shapes[k];
      AABB a = w.saabb[sid];
      if (!aabb_contains(w.fat[sid], a)) {
        w.fat[sid] = aabb_inflate(a, w.shapes[sid].aabb_margin);
        w.moved[sid] = 1;
        add_converged(&w.ctl->moved_count);
      }
    }
  }
  // solver_integration.rs:556-564: the world inverse inertia at the final rotation
  M3 R = matrix_from_quat(sim.q);
  sim.inv_inertia_world = mul_mm(mul_mm(R, sim.inv_inertia_local), transpose(R));
  w.states[i] = st;
  w.asims[i] = sim;
}

// The continuous pass: one thread per fast body queued by k_finalize this step.
__global__ void __launch_bounds__(64) k_continuous(DW w, StepParams p) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w.ctl->fast_count) return;
  continuous_body(w, p, w.fast_list[t]);
}

// solver_integration.rs:949-958, continuous.rs:337 for one fast bullet, one warp each, after
// k_continuous (every other body is final). Every shape of the bullet (no per-shape speed test)
// is swept against its sub-world's static shapes, then against the shapes of its kinematic and
// dynamic non-bullet bodies at their final poses (continuous.rs:429-448: the reference also walks
// its kinematic and dynamic trees for bullets; bullets skip bullets, continuous.rs:253), each
// list in shape order.
// The lanes test 32 candidates' bounds and filters at once; lane 0 runs the times of impact in
// list order, each bounded by the best fraction so far, and finishes the body. Bullets read
// only non-bullet bodies, which no warp here writes, so they are independent of one another.
__global__ void __launch_bounds__(128) k_bullets(DW w, StepParams p) {
  const int q = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31);
  if (q >= w.ctl->bullet_count) return;  // the whole warp leaves together
  const int i = w.bullet_list[q];
  const DSim sim = w.asims[i];
  const Pos base = {sim.cx0, sim.cy0, sim.cz0};
  const Sweep sweep = sweep_of(sim, base);
  const Xf xf2 = xf(sweep.c2 - rotate(sweep.q2, sweep.local_center), sweep.q2);
  float fraction = 1.0f;  // lane 0's
  for (int k = sim.shape_begin; k < sim.shape_end; ++k) {
    const int fid = w.body_shapes[k];
    const DShape& fs = w.shapes[fid];
    Proxy fp;
    V3 lc;
    shape_proxy(w, fs, &fp, &lc);
    const AABB box1 = w.saabb[fid];
    const AABB box2 = offset_aabb(shape_box(w, fs, xf2), base);
    __syncwarp();
    if (lane == 0) w.saabb[fid] = box2;
    const AABB swept = aabb(min3(box1.lo, box2.lo), max3(box1.hi, box2.hi));
    for (int pass = 0; pass < 2; ++pass) {
      const int* list = pass == 0 ? w.static_list : w.dyn_list;
      const int* off = pass == 0 ? w.static_off : w.dyn_off;
      const int t0 = off[fs.world], t1 = off[fs.world + 1];
      for (int tb = t0; tb < t1; tb += 32) {
        const int t = tb + lane;
        int sid = -1;
        bool hit = false;
        if (t < t1) {
          sid = list[t];
          hit = aabb_overlaps(w.fat[sid], swept) && should_create_pair(w, sid, fid) &&
                (pass == 0 || (sim_of(w, w.shapes[sid].enc).flags & kIsBullet) == 0);
        }
        unsigned m = __ballot_sync(0xffffffffu, hit);
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          const int cs = __shfl_sync(0xffffffffu, sid, src);
          if (lane == 0) fraction = candidate_fraction(w, cs, fp, sweep, base, fraction);
        }
      }
    }
  }
  if (lane == 0) continuous_finish(w, p, i, sim, w.states[i], sweep, base, fraction);
}

}  // namespace nsd
