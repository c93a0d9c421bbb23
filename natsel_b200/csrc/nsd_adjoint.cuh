// Adjoint of the step (vector-Jacobian product of a rollout) on the device.
//
// The forward step is replayed from a checkpoint with a tape: the body state at the start of
// the step, the contacts before the narrowphase and after the state pass, the prepared
// constraint planes, per substep three body rows (before integrate-velocities, before and
// after integrate-positions) and the inputs of every push and relax update. The reverse pass
// then walks the step backwards: finalize, impulse store, the substeps (relax colours 22..0,
// integrate positions, push colours 22..0, warm start colours 22..0, integrate velocities),
// prepare, the inverse world inertia and the narrowphase. The solver stages run one thread per
// constraint or body through hand-derived reverse sweeps (nsd_ad.cuh); the barrier-separated
// sweep carries only the bodies' and impulses' cotangents, and the constant planes'
// cotangents of every update are added afterwards by one parallel pass (k_adj_consts).
// Prepare, the inertia and the narrowphase form their vector-Jacobian products with one warp
// each: lane l seeds input directions l, l + 32, ... of the dual-number restatement, evaluates
// it once and contracts the output tangents with the incoming cotangents. Colours keep the
// forward's independence: inside a colour no two constraints share a dynamic body, so their
// body cotangents are written without atomics.
//
// Scope of the adjoint: one world of box bodies (hull shapes) without joints, restitution,
// rolling resistance, continuous collision or overflow constraints; the host rejects other
// worlds.
#pragma once
#include "nsd_solve.cuh"
#include "nsd_ad.cuh"

namespace nsd {

// Device tape of one step.
struct StepTape {
  DSim* sims;        // [n_awake] at the start of the step
  DContact* pre;     // [cap] before the narrowphase (after the pair update)
  DContact* post;    // [cap] after the state pass
  Control* ctl;      // after prepare (colour offsets)
  CPlanes planes;    // after prepare
  DState* body;      // [substep][3][n_awake]: before IV, before IP, after IP
  float4* push;      // [substep][4][cap]: vA|l0, wA|l1, vB|l2, wB|l3 before push
  float4* relax;     // [substep][5][cap]: the same before relax, then fr.x, fr.y, twist
  float4* fin;       // [cap]: friction impulse x, y and twist after the solve
  uint8_t* mode;     // [cap]: narrowphase 0 none/disjoint, 1 recycled, 2 new manifold, 3 no points
  float4* rest;      // [iteration][6][cap]: the inputs of each restitution update (SolveTape::rest)
  DJoint* joints;    // [n_joints] after prepare
  float4* joint;     // [substep][2][6][n_joints]: each joint solve's inputs (SolveTape::joint)
  float4* jwarm;     // [substep][4][n_joints]: the state each relax leaves for the next warm start
  int n_joints;
  int rest_iterations;
  int substeps;
};

// Cotangent buffers of the reverse pass.
enum : int {
  pbInvMass = 0, pbIiw = 1, pbIinv = 10, pbFriction = 19, pbInertia = 20, pbRestitution = 29, kPB = 30,
  // contact manifold cotangent: normal, per point 9 (anchor_a, anchor_b, separation,
  // base separation, normal impulse), friction impulse, twist, cached rotations
  mbN = 0, mbPoint = 3, mbFrictionImpulse = 39, mbTwist = 42, mbRotA = 43, mbRotB = 47, kMB = 51,
};
__host__ __device__ __forceinline__ int mb_point(int q, int f) { return mbPoint + 9 * q + f; }
struct AdjBufs {
  float* bb;   // [n_awake][16]: v|-, w|-, dp|-, dq (cotangents of the solver state)
  float* cq;   // [n_awake][8]: centre|-, rotation (cotangents at the current step boundary)
  float* pb;   // [n_awake][kPB]: parameters
  float* kb;   // [kCVOwn][cap]: constraint entries cvLam.. of each slot
  float* mb;   // [kMB][cap]: manifold state of each contact id
  float* yrec; // [substep][stage][kRelaxOut][cap]: output cotangents each contact update received
  float* totb; // [4][cap]: the points' total normal impulses (what restitution reads of them);
               // null when no shape has restitution
  float* restb;  // [4][cap]: the points' restitution impulses
  float* relb; // [4][cap]: the points' relative normal velocities at prepare
  int* mismatch;  // narrowphase replays that did not reproduce the forward manifold
  float* jb;     // [n_joints][kJState]: the joints' impulses and perp axes
  float* jc;     // [n_joints][kJConst]: the joints' prepared constants (this step)
  const int* joint_list;  // joints by colour (world constant)
  JointRanges jr;
  int cap, n_awake, n_joints;
};

constexpr int kAdjThreads = 256;

__device__ __forceinline__ float& BB(const AdjBufs& a, int i, int f) { return a.bb[(size_t)i * 16 + f]; }
__device__ __forceinline__ float& CQ(const AdjBufs& a, int i, int f) { return a.cq[(size_t)i * 8 + f]; }
__device__ __forceinline__ float& PB(const AdjBufs& a, int i, int f) { return a.pb[(size_t)i * kPB + f]; }
__device__ __forceinline__ float& KB(const AdjBufs& a, int k, int cv) { return a.kb[(size_t)(cv - ad::cvLam) * a.cap + k]; }
__device__ __forceinline__ float& MB(const AdjBufs& a, int c, int f) { return a.mb[(size_t)f * a.cap + c]; }
__device__ __forceinline__ void put3(float* x, int at, V3 v) { x[at] = v.x; x[at + 1] = v.y; x[at + 2] = v.z; }
__device__ __forceinline__ float& JB(const AdjBufs& a, int j, int f) { return a.jb[(size_t)j * ad::kJState + f]; }
__device__ __forceinline__ float& JC(const AdjBufs& a, int j, int f) { return a.jc[(size_t)j * ad::kJConst + f]; }
__device__ __forceinline__ float& TOTB(const AdjBufs& a, int k, int q) { return a.totb[(size_t)q * a.cap + k]; }
__device__ __forceinline__ float& RESTB(const AdjBufs& a, int k, int q) { return a.restb[(size_t)q * a.cap + k]; }
__device__ __forceinline__ float& RELB(const AdjBufs& a, int k, int q) { return a.relb[(size_t)q * a.cap + k]; }

// ---------------------------------------------------------------------------------------------
// Finalize (k_finalize): centre' = centre + dp, q' = normalize(dq q).
__global__ void k_adj_finalize(StepTape t, AdjBufs a, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DSim& s = t.sims[i];
  const DState& last = t.body[((size_t)(t.substeps - 1) * 3 + 2) * n + i];
  float xs[8] = {s.q.v.x, s.q.v.y, s.q.v.z, s.q.s, last.dq.v.x, last.dq.v.y, last.dq.v.z, last.dq.s};
  ad::SeedIn<float, 8> in;
  in.x = xs;
  for (int k = 0; k < 8; ++k) in.dir[k] = k;
  ad::Dual<float, 8> y[4];
  ad::final_rot_fn<ad::Dual<float, 8>>(in, y);
  float qbar[4] = {CQ(a, i, 4), CQ(a, i, 5), CQ(a, i, 6), CQ(a, i, 7)};
  float xb[8];
  for (int k = 0; k < 8; ++k) {
    float acc = 0.0f;
    for (int j = 0; j < 4; ++j) acc += qbar[j] * y[j].d[k];
    xb[k] = acc;
  }
  for (int f = 0; f < 3; ++f) BB(a, i, 8 + f) = CQ(a, i, f);   // dp̄ = centre cotangent
  for (int f = 0; f < 4; ++f) BB(a, i, 12 + f) = xb[4 + f];     // dq̄
  for (int f = 0; f < 4; ++f) CQ(a, i, 4 + f) = xb[f];          // q̄ at the step start
}

// Impulse store (store_constraint): the manifold's impulses after the step are the solver's
// final impulses; their cotangents seed the constraint's own entries.
__global__ void k_adj_store(StepTape t, AdjBufs a, int n_slots) {
  using namespace ad;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_slots) return;
  int4 idx = t.planes.idx[k];
  int cid = idx.z, pc = idx.w & 255;
  for (int cv = cvLam; cv < kCV; ++cv) KB(a, k, cv) = 0.0f;
  // the total normal and restitution impulses start from zero at prepare and nothing after the
  // step reads them: their cotangents start at zero here, as do the relative velocities'
  if (a.totb)
    for (int q = 0; q < 4; ++q) { TOTB(a, k, q) = 0.0f; RESTB(a, k, q) = 0.0f; RELB(a, k, q) = 0.0f; }
  for (int q = 0; q < pc; ++q) {
    KB(a, k, cvLam + q) = MB(a, cid, mb_point(q, 8));
    MB(a, cid, mb_point(q, 8)) = 0.0f;
  }
  V3 F = v3(MB(a, cid, mbFrictionImpulse), MB(a, cid, mbFrictionImpulse + 1), MB(a, cid, mbFrictionImpulse + 2));
  float twist = MB(a, cid, mbTwist);
  for (int f = 0; f < 3; ++f) MB(a, cid, mbFrictionImpulse + f) = 0.0f;
  MB(a, cid, mbTwist) = 0.0f;
  float4 fin = t.fin[k], t1 = t.planes.t1[k], t2 = t.planes.t2[k];
  KB(a, k, cvFr) = F.x * t1.x + F.y * t1.y + F.z * t1.z;
  KB(a, k, cvFr + 1) = F.x * t2.x + F.y * t2.y + F.z * t2.z;
  KB(a, k, cvTwist) = twist;
  KB(a, k, cvT1) = fin.x * F.x; KB(a, k, cvT1 + 1) = fin.x * F.y; KB(a, k, cvT1 + 2) = fin.x * F.z;
  KB(a, k, cvT2) = fin.y * F.x; KB(a, k, cvT2 + 1) = fin.y * F.y; KB(a, k, cvT2 + 2) = fin.y * F.z;
}

// The constraint vector of slot k in stage `stage` of substep `sub`: the values the forward
// update read (body velocities and impulses from the solver tape, dp and dq from the body rows,
// the constants from the prepared planes).
__device__ void gather_cv(const StepTape& t, int n, int cap, int k, int sub, int stage, float* x) {
  using namespace ad;
  const CPlanes& P = t.planes;
  int4 idx = P.idx[k];
  int ia = idx.x, ib = idx.y;
  auto put = [&](int at, float4 v, int cnt) {
    x[at] = v.x; if (cnt > 1) x[at + 1] = v.y; if (cnt > 2) x[at + 2] = v.z; if (cnt > 3) x[at + 3] = v.w;
  };
  const float4* rows = stage == kRelax ? t.relax + (size_t)sub * 5 * cap : t.push + (size_t)sub * 4 * cap;
  for (int r = 0; r < 4; ++r) {
    float4 v = rows[(size_t)r * cap + k];
    if (stage == kWarm) { v.x = 0.0f; v.y = 0.0f; v.z = 0.0f; }  // warm start is affine in them
    put(3 * r, v, 3);
    x[cvLam + r] = v.w;
  }
  {
    float4 v = t.relax[((size_t)sub * 5 + 4) * cap + k];
    x[cvFr] = v.x; x[cvFr + 1] = v.y; x[cvTwist] = v.z;
  }
  int row_sel = stage == kRelax ? 2 : 0;  // the dp, dq the stage sees
  for (int s = 0; s < 2; ++s) {
    int b = s == 0 ? ia : ib;
    float4 dp = make_float4(0, 0, 0, 0), dq = make_float4(0, 0, 0, 1);
    if (b >= 0) {
      const DState& st = t.body[((size_t)sub * 3 + row_sel) * n + b];
      dp = make_float4(st.dp.x, st.dp.y, st.dp.z, 0.0f);
      dq = make_float4(st.dq.v.x, st.dq.v.y, st.dq.v.z, st.dq.s);
    }
    put(s == 0 ? cvDpA : cvDpB, dp, 3);
    put(s == 0 ? cvDqA : cvDqB, dq, 4);
  }
  float4 m = P.mass[k];
  x[cvIma] = m.x; x[cvImb] = m.y; x[cvFriction] = m.z;
  put(cvSa, P.ia0[k], 4);
  float4 v1 = P.ia1[k];
  x[cvSa + 4] = v1.x; x[cvSa + 5] = v1.y; x[cvSb] = v1.z; x[cvSb + 1] = v1.w;
  put(cvSb + 2, P.ib1[k], 4);
  put(cvN, P.n[k], 3);
  float4 t1 = P.t1[k], t2 = P.t2[k], ca = P.ca[k];
  put(cvT1, t1, 3); x[cvTv1] = t1.w;
  put(cvT2, t2, 3); x[cvTv2] = t2.w;
  put(cvCa, ca, 3); x[cvTwistMass] = ca.w;
  put(cvCb, P.cb[k], 3);
  put(cvTm, P.tm[k], 4);
  for (int q = 0; q < 4; ++q) {
    float4 ra = P.pra[(size_t)q * cap + k], rb = P.prb[(size_t)q * cap + k], im = P.pimp[(size_t)q * cap + k];
    put(cv_point(q, 0), ra, 3); x[cv_point(q, 6)] = ra.w;
    put(cv_point(q, 3), rb, 3); x[cv_point(q, 7)] = rb.w;
    x[cv_point(q, 8)] = im.z;
  }
}

__device__ __forceinline__ ad::CParams contact_params(int4 idx, const StepParams& p) {
  ad::CParams cp;
  cp.pc = idx.w & 255;
  cp.is_static = (idx.w & 256) != 0;
  cp.inv_h = p.inv_h;
  cp.contact_speed = p.contact_speed;
  cp.contact_softness = p.contact_softness;
  cp.static_softness = p.static_softness;
  return cp;
}

// Reverse of one contact stage for slot k (one thread), on the reverse solve's critical path:
// the hand-derived reverse sweep of the stage (nsd_ad.cuh) restricted to the two bodies' state
// and the impulses, written back (velocities replace the outputs' for push and relax, dp and
// dq accumulate, impulses replace where the stage updates them and accumulate where it only
// reads them). The output cotangents are recorded for k_adj_consts, which adds the constant
// entries' cotangents of every update afterwards, off the critical path.
template <int Stage>
__device__ void adj_contact(const StepTape& t, const AdjBufs& a, const StepParams& p, int n, int k, int sub) {
  using namespace ad;
  int4 idx = t.planes.idx[k];
  int ia = idx.x, ib = idx.y;
  CParams cp = contact_params(idx, p);
  float x[kCV], xb[cvIma], yb[kRelaxOut];
  gather_cv(t, n, a.cap, k, sub, Stage, x);
  for (int f = 0; f < 12; ++f) {
    int b = f < 6 ? ia : ib;
    int g = f % 6;
    yb[f] = b >= 0 ? BB(a, b, g < 3 ? g : g + 1) : 0.0f;
  }
  for (int q = 0; q < 4; ++q) yb[12 + q] = KB(a, k, cvLam + q);
  // relax adds each point's new normal impulse to its total (imp.y += ni), which restitution
  // reads: the total's cotangent joins the new impulse's and passes on unchanged
  if (Stage == kRelax && a.totb)
    for (int q = 0; q < 4; ++q) yb[12 + q] += TOTB(a, k, q);
  yb[16] = KB(a, k, cvFr); yb[17] = KB(a, k, cvFr + 1); yb[18] = KB(a, k, cvTwist);
  for (int i = 0; i < cvIma; ++i) xb[i] = 0.0f;
  if (Stage == kWarm) warm_vjp<float, false>(x, cp, yb, xb);
  else if (Stage == kPush) push_vjp<float, false>(x, cp, yb, xb);
  else relax_vjp<float, false>(x, cp, yb, xb);
  constexpr int NY = Stage == kWarm ? kWarmOut : Stage == kPush ? kPushOut : kRelaxOut;
  float* rec = a.yrec + ((size_t)(sub * 3 + Stage) * kRelaxOut) * a.cap + k;
  for (int j = 0; j < NY; ++j) rec[(size_t)j * a.cap] = yb[j];
  if (Stage != kWarm) {
    for (int f = 0; f < 12; ++f) {
      int b = f < 6 ? ia : ib;
      int g = f % 6;
      if (b >= 0) BB(a, b, g < 3 ? g : g + 1) = xb[f];
    }
    for (int f = 0; f < 3; ++f) {
      if (ia >= 0) BB(a, ia, 8 + f) += xb[cvDpA + f];
      if (ib >= 0) BB(a, ib, 8 + f) += xb[cvDpB + f];
    }
    for (int f = 0; f < 4; ++f) {
      if (ia >= 0) BB(a, ia, 12 + f) += xb[cvDqA + f];
      if (ib >= 0) BB(a, ib, 12 + f) += xb[cvDqB + f];
    }
  }
  for (int cv = cvLam; cv < cvIma; ++cv) {
    bool updated = Stage == kRelax || (Stage == kPush && cv < cvFr);
    if (updated) KB(a, k, cv) = xb[cv];
    else if (Stage == kWarm) KB(a, k, cv) += xb[cv];
  }
}

// The constant entries' cotangents of every contact update of the step (all substeps and
// stages of slot k, one thread), from the inputs on the tape and the recorded output
// cotangents; summed into the slot's constraint cotangents.
__global__ void k_adj_consts(StepTape t, AdjBufs a, StepParams p, int n_slots) {
  using namespace ad;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_slots) return;
  CParams cp = contact_params(t.planes.idx[k], p);
  float sum[kCV - cvIma];
  for (int i = 0; i < kCV - cvIma; ++i) sum[i] = 0.0f;
  float x[kCV], xb[kCV], yb[kRelaxOut];
  for (int sub = 0; sub < t.substeps; ++sub) {
    for (int stage = kWarm; stage <= kRelax; ++stage) {
      gather_cv(t, a.n_awake, a.cap, k, sub, stage, x);
      const float* rec = a.yrec + ((size_t)(sub * 3 + stage) * kRelaxOut) * a.cap + k;
      int ny = stage == kWarm ? kWarmOut : stage == kPush ? kPushOut : kRelaxOut;
      for (int j = 0; j < kRelaxOut; ++j) yb[j] = j < ny ? rec[(size_t)j * a.cap] : 0.0f;
      for (int i = 0; i < kCV; ++i) xb[i] = 0.0f;
      if (stage == kWarm) warm_vjp(x, cp, yb, xb);
      else if (stage == kPush) push_vjp(x, cp, yb, xb);
      else relax_vjp(x, cp, yb, xb);
      for (int i = 0; i < kCV - cvIma; ++i) sum[i] += xb[cvIma + i];
    }
  }
  for (int i = 0; i < kCV - cvIma; ++i) KB(a, k, cvIma + i) += sum[i];
}

// Reverse of integrate positions for body i (one thread).
__device__ void adj_ip(const StepTape& t, const AdjBufs& a, const StepParams& p, int n, int i, int sub) {
  using namespace ad;
  const DState& st = t.body[((size_t)sub * 3 + 1) * n + i];
  float x[kIP] = {st.v.x, st.v.y, st.v.z, st.w.x, st.w.y, st.w.z, st.dp.x, st.dp.y, st.dp.z,
                  st.dq.v.x, st.dq.v.y, st.dq.v.z, st.dq.s};
  const int map[kIP] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14, 15};
  float yb[kIP], xb[kIP];
  for (int f = 0; f < kIP; ++f) { yb[f] = BB(a, i, map[f]); xb[f] = 0.0f; }
  BParams bp = {};
  bp.h = p.h; bp.inv_dt = p.inv_dt; bp.max_linear_speed = p.max_linear_speed; bp.flags = st.flags;
  ip_vjp(x, bp, yb, xb);
  for (int f = 0; f < kIP; ++f) BB(a, i, map[f]) = xb[f];
}

// Reverse of integrate velocities for body i (one thread): the hand-derived sweep, or for a
// gyroscopic body the dual-number product one input direction at a time.
__device__ void adj_iv(const StepTape& t, const AdjBufs& a, const StepParams& p, int n, int i, int sub) {
  using namespace ad;
  const DState& st = t.body[((size_t)sub * 3 + 0) * n + i];
  const DSim& s = t.sims[i];
  float x[kIVIn];
  x[0] = st.v.x; x[1] = st.v.y; x[2] = st.v.z; x[3] = st.w.x; x[4] = st.w.y; x[5] = st.w.z;
  x[6] = s.inv_mass;
  const float* m = &s.inv_inertia_world.cx.x;
  for (int f = 0; f < 9; ++f) x[7 + f] = m[f];
  x[16] = s.force.x; x[17] = s.force.y; x[18] = s.force.z;
  x[19] = s.torque.x; x[20] = s.torque.y; x[21] = s.torque.z;
  x[22] = s.q.v.x; x[23] = s.q.v.y; x[24] = s.q.v.z; x[25] = s.q.s;
  x[26] = st.dq.v.x; x[27] = st.dq.v.y; x[28] = st.dq.v.z; x[29] = st.dq.s;
  const float* in = &s.inertia.cx.x;
  for (int f = 0; f < 9; ++f) x[30 + f] = in[f];
  const int map[6] = {0, 1, 2, 4, 5, 6};
  float yb[kIVOut], xb[kIVIn];
  for (int f = 0; f < kIVOut; ++f) yb[f] = BB(a, i, map[f]);
  for (int f = 0; f < kIVIn; ++f) xb[f] = 0.0f;
  BParams bp = {};
  bp.h = p.h; bp.lin_damp = s.linear_damping; bp.ang_damp = s.angular_damping; bp.grav_scale = s.gravity_scale;
  bp.gravity = p.gravity;
  bp.flags = s.flags;
  if (s.flags & kGyroscopic) {
    for (int d = 0; d < kIVIn; ++d) {
      if (d >= 16 && d < 22) continue;  // applied force and torque: not returned
      SeedIn<float, 1> sin;
      sin.x = x;
      sin.dir[0] = d;
      Dual<float, 1> y[kIVOut];
      iv_fn(sin, bp, y);
      float acc = 0.0f;
      for (int j = 0; j < kIVOut; ++j) acc += yb[j] * y[j].d[0];
      xb[d] = acc;
    }
  } else {
    iv_vjp_plain(x, bp, yb, xb);
  }
  for (int f = 0; f < 6; ++f) BB(a, i, map[f]) = xb[f];
  PB(a, i, pbInvMass) += xb[6];
  for (int f = 0; f < 9; ++f) PB(a, i, pbIiw + f) += xb[7 + f];
  if (s.flags & kGyroscopic) {
    for (int f = 0; f < 4; ++f) CQ(a, i, 4 + f) += xb[22 + f];      // rotation at the step start
    for (int f = 0; f < 4; ++f) BB(a, i, 12 + f) += xb[26 + f];     // substep rotation dq
    for (int f = 0; f < 9; ++f) PB(a, i, pbInertia + f) += xb[30 + f];
  }
}

// Reverse of one restitution iteration over one colour (the forward runs after the substeps,
// colours 0..22 per iteration; the reverse runs iterations and colours backwards): one warp per
// constraint of colour `colour` evaluates ad::restitution_fn on dual numbers, lane l seeding
// input directions l, l + 32 and l + 64, and contracts the output tangents with the outputs'
// cotangents. Bodies' velocity cotangents, the impulses' and the total and restitution
// impulses' are replaced, position deltas' and constants' accumulated; the restitution
// coefficient's cotangent goes to the shape whose coefficient the contact took
// (max(e_a, e_b), world_runtime.rs mix_restitution), the relative velocities' to k_adj_relvel.
__global__ void __launch_bounds__(kAdjThreads) k_adj_restitution(StepTape t, AdjBufs a, DW w, ad::RParams rp0,
                                                                 int it, int colour) {
  using namespace ad;
  __shared__ float xs_s[kAdjThreads / 32][kRV];
  __shared__ float ys_s[kAdjThreads / 32][kRestOut];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c0 = t.ctl->color_offset[colour], c1 = t.ctl->color_offset[colour + 1];
  const int k = c0 + blockIdx.x * (kAdjThreads / 32) + warp;
  if (k >= c1) return;
  const CPlanes& P = t.planes;
  const float e = P.mass[k].w;
  if (!(e > 0.0f)) return;  // the forward update changed nothing (and recorded no inputs)
  const int4 idx = P.idx[k];
  const int ia = idx.x, ib = idx.y, cid = idx.z, cap = a.cap, n = a.n_awake;
  float* xs = xs_s[warp];
  float* ys = ys_s[warp];
  const float4* rows = t.rest + (size_t)it * 6 * cap;
  if (lane == 0) {
    for (int r = 0; r < 4; ++r) {
      float4 v = rows[(size_t)r * cap + k];
      xs[3 * r] = v.x; xs[3 * r + 1] = v.y; xs[3 * r + 2] = v.z;
      xs[rvLam + r] = v.w;
    }
    float4 tot = rows[4 * (size_t)cap + k], rest = rows[5 * (size_t)cap + k];
    xs[rvTot] = tot.x; xs[rvTot + 1] = tot.y; xs[rvTot + 2] = tot.z; xs[rvTot + 3] = tot.w;
    xs[rvRest] = rest.x; xs[rvRest + 1] = rest.y; xs[rvRest + 2] = rest.z; xs[rvRest + 3] = rest.w;
    // the position deltas restitution sees: after the last substep's integrate positions
    for (int side = 0; side < 2; ++side) {
      int b = side == 0 ? ia : ib;
      V3 dp = v3(0, 0, 0);
      Q dq = qid();
      if (b >= 0) {
        const DState& st = t.body[((size_t)(t.substeps - 1) * 3 + 2) * n + b];
        dp = st.dp;
        dq = st.dq;
      }
      int at = side == 0 ? rvDpA : rvDpB, aq = side == 0 ? rvDqA : rvDqB;
      xs[at] = dp.x; xs[at + 1] = dp.y; xs[at + 2] = dp.z;
      xs[aq] = dq.v.x; xs[aq + 1] = dq.v.y; xs[aq + 2] = dq.v.z; xs[aq + 3] = dq.s;
    }
    float4 m = P.mass[k], a0 = P.ia0[k], a1 = P.ia1[k], b1 = P.ib1[k], nn = P.n[k];
    xs[rvIma] = m.x; xs[rvImb] = m.y; xs[rvE] = m.w;
    xs[rvSa] = a0.x; xs[rvSa + 1] = a0.y; xs[rvSa + 2] = a0.z; xs[rvSa + 3] = a0.w; xs[rvSa + 4] = a1.x;
    xs[rvSa + 5] = a1.y;
    xs[rvSb] = a1.z; xs[rvSb + 1] = a1.w; xs[rvSb + 2] = b1.x; xs[rvSb + 3] = b1.y; xs[rvSb + 4] = b1.z;
    xs[rvSb + 5] = b1.w;
    xs[rvN] = nn.x; xs[rvN + 1] = nn.y; xs[rvN + 2] = nn.z;
    for (int q = 0; q < 4; ++q) {
      float4 ra = P.pra[(size_t)q * cap + k], rbv = P.prb[(size_t)q * cap + k], im = P.pimp[(size_t)q * cap + k];
      xs[rv_point(q, 0)] = ra.x; xs[rv_point(q, 1)] = ra.y; xs[rv_point(q, 2)] = ra.z; xs[rv_point(q, 6)] = ra.w;
      xs[rv_point(q, 3)] = rbv.x; xs[rv_point(q, 4)] = rbv.y; xs[rv_point(q, 5)] = rbv.z; xs[rv_point(q, 7)] = rbv.w;
      xs[rv_point(q, 8)] = im.w;
      xs[rv_point(q, 9)] = 0.0f;
    }
  }
  if (lane < 12) {
    int b = lane < 6 ? ia : ib;
    int g = lane % 6;
    ys[lane] = b >= 0 ? BB(a, b, g < 3 ? g : g + 1) : 0.0f;
  } else if (lane < 16) {
    ys[lane] = KB(a, k, cvLam + lane - 12);
  } else if (lane < 20) {
    ys[lane] = TOTB(a, k, lane - 16);
  } else if (lane < 24) {
    ys[lane] = RESTB(a, k, lane - 20);
  }
  __syncwarp();
  RParams rp = rp0;
  rp.pc = idx.w & 255;
  SeedIn<float, 3> in;
  in.x = xs;
  in.dir[0] = lane;
  in.dir[1] = lane + 32;
  in.dir[2] = lane + 64;
  Dual<float, 3> y[kRestOut];
  restitution_fn(in, rp, y);
  float xb[3];
  for (int kk = 0; kk < 3; ++kk) {
    float acc = 0.0f;
    for (int j = 0; j < kRestOut; ++j) acc += ys[j] * y[j].d[kk];
    xb[kk] = acc;
  }
  __syncwarp();
  for (int kk = 0; kk < 3; ++kk) {
    const int d = in.dir[kk];
    const float v = xb[kk];
    if (d < 12) {
      int b = d < 6 ? ia : ib;
      int g = d % 6;
      if (b >= 0) BB(a, b, g < 3 ? g : g + 1) = v;
    } else if (d < rvDpB) {
      if (ia >= 0) BB(a, ia, 8 + d - rvDpA) += v;
    } else if (d < rvDqA) {
      if (ib >= 0) BB(a, ib, 8 + d - rvDpB) += v;
    } else if (d < rvDqB) {
      if (ia >= 0) BB(a, ia, 12 + d - rvDqA) += v;
    } else if (d < rvLam) {
      if (ib >= 0) BB(a, ib, 12 + d - rvDqB) += v;
    } else if (d < rvTot) {
      KB(a, k, cvLam + d - rvLam) = v;
    } else if (d < rvRest) {
      TOTB(a, k, d - rvTot) = v;
    } else if (d < rvIma) {
      RESTB(a, k, d - rvRest) = v;
    } else if (d == rvIma) {
      KB(a, k, cvIma) += v;
    } else if (d == rvImb) {
      KB(a, k, cvImb) += v;
    } else if (d < rvSb) {
      KB(a, k, cvSa + d - rvSa) += v;
    } else if (d < rvN) {
      KB(a, k, cvSb + d - rvSb) += v;
    } else if (d < rvE) {
      KB(a, k, cvN + d - rvN) += v;
    } else if (d == rvE) {
      // e = max(e_a, e_b): the cotangent goes to the shape that supplied it
      const DContact& c = t.post[cid];
      float ea = w.shapes[c.shape_a].restitution, eb = w.shapes[c.shape_b].restitution;
      int body = ea > eb ? ia : ib;
      if (body >= 0 && v != 0.0f) atomicAdd(&PB(a, body, pbRestitution), v);
    } else {
      int q = (d - rvPoint) / 10, f = (d - rvPoint) % 10;
      // anchors, base separation and normal mass share the constraint layout's point entries
      if (f < 8) KB(a, k, cv_point(q, f)) += v;
      else if (f == 8) RELB(a, k, q) += v;
    }
  }
}

// Reverse of the relative normal velocities prepare records for restitution (one thread per
// slot; ad::relvel_vjp): runs after the reverse solve, when the bodies' velocity cotangents are
// those of the step's start, whose velocities prepare read. The normal's and anchors' cotangents
// go to the contact's manifold, the velocities' to the bodies (atomics: a body has slots in
// every colour).
__global__ void k_adj_relvel(StepTape t, AdjBufs a, int n_slots) {
  using namespace ad;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_slots) return;
  const int4 idx = t.planes.idx[k];
  if (!(t.planes.mass[k].w > 0.0f)) return;  // prepare sampled no velocity
  const int ia = idx.x, ib = idx.y, cid = idx.z, pc = idx.w & 255;
  const Manifold& m = t.post[cid].manifold;
  float x[kRL];
  for (int f = 0; f < 12; ++f) x[f] = 0.0f;
  if (ia >= 0) { const DState& s = t.body[ia]; put3(x, rlVA, s.v); put3(x, rlWA, s.w); }
  if (ib >= 0) { const DState& s = t.body[ib]; put3(x, rlVB, s.v); put3(x, rlWB, s.w); }
  put3(x, rlN, m.normal);
  float acc[kRL];
  for (int f = 0; f < 15; ++f) acc[f] = 0.0f;
  for (int q = 0; q < pc; ++q) {
    float g = RELB(a, k, q);
    if (g == 0.0f) continue;
    put3(x, rlRa, m.points[q].anchor_a);
    put3(x, rlRb, m.points[q].anchor_b);
    float xb[kRL];
    for (int f = 0; f < kRL; ++f) xb[f] = 0.0f;
    relvel_vjp(x, g, xb);
    for (int f = 0; f < 15; ++f) acc[f] += xb[f];
    for (int f = 0; f < 3; ++f) {
      MB(a, cid, mb_point(q, f)) += xb[rlRa + f];
      MB(a, cid, mb_point(q, 3 + f)) += xb[rlRb + f];
    }
  }
  for (int f = 0; f < 3; ++f) {
    MB(a, cid, mbN + f) += acc[rlN + f];
    if (ia >= 0) { atomicAdd(&BB(a, ia, f), acc[rlVA + f]); atomicAdd(&BB(a, ia, 4 + f), acc[rlWA + f]); }
    if (ib >= 0) { atomicAdd(&BB(a, ib, f), acc[rlVB + f]); atomicAdd(&BB(a, ib, 4 + f), acc[rlWB + f]); }
  }
}

// ---------------------------------------------------------------------------------------------
// Revolute joints: one warp per joint evaluates the restatement (nsd_ad.cuh joint_solve_fn,
// joint_warm_fn, joint_prepare_fn) on dual numbers, lane l seeding input directions l, l + 32
// and l + 64, and contracts the output tangents with the outputs' cotangents.

__device__ ad::JParams joint_params(const DJoint& j, const StepParams& p, bool use_bias) {
  ad::JParams jp;
  jp.use_bias = use_bias;
  jp.fixed = j.fixed_rotation != 0;
  jp.spring = j.enable_spring != 0;
  jp.motor = j.enable_motor != 0;
  jp.limit = j.enable_limit != 0;
  jp.cs = j.constraint_softness;
  jp.ss = j.spring_softness;
  jp.target = j.target_angle;
  jp.lower = j.lower_angle;
  jp.upper = j.upper_angle;
  jp.motor_speed = j.motor_speed;
  jp.max_torque_h = j.max_motor_torque * p.h;
  jp.inv_h = p.inv_h;
  return jp;
}
// The prepared constants of the joint vector (jxIma on)
__device__ void joint_consts(const DJoint& j, float* x) {
  using namespace ad;
  x[jxIma] = j.inv_mass_a;
  x[jxImb] = j.inv_mass_b;
  put3(x, jxIA, j.inv_ia.cx); put3(x, jxIA + 3, j.inv_ia.cy); put3(x, jxIA + 6, j.inv_ia.cz);
  put3(x, jxIB, j.inv_ib.cx); put3(x, jxIB + 3, j.inv_ib.cy); put3(x, jxIB + 6, j.inv_ib.cz);
  put3(x, jxFqA, j.frame_a.q.v); x[jxFqA + 3] = j.frame_a.q.s;
  put3(x, jxFqB, j.frame_b.q.v); x[jxFqB + 3] = j.frame_b.q.s;
  put3(x, jxFpA, j.frame_a.p);
  put3(x, jxFpB, j.frame_b.p);
  put3(x, jxAxis, j.rotation_axis_z);
  x[jxAxial] = j.axial_mass;
  put3(x, jxDc, j.delta_center);
}
// A body's position and rotation increments from body row `row` of substep `sub` (identity for
// a static body)
__device__ void joint_body_deltas(const StepTape& t, int n, int sub, int row, int b, float* x, int at_dp, int at_dq) {
  V3 dp = v3(0, 0, 0);
  Q dq = qid();
  if (b >= 0) {
    const DState& st = t.body[((size_t)sub * 3 + row) * n + b];
    dp = st.dp;
    dq = st.dq;
  }
  put3(x, at_dp, dp);
  put3(x, at_dq, dq.v);
  x[at_dq + 3] = dq.s;
}

// Reverse of one joint's push (use_bias) or relax solve at substep sub (one warp). Velocities'
// and impulses' cotangents are replaced (the solve updates them), the perp axes' too (the solve
// recomputes them), position and rotation increments' and the constants' accumulated.
__device__ __noinline__ void adj_joint_solve(const StepTape& t, const AdjBufs& a, const StepParams& p, int stage,
                                             int sub, int ji, int lane, float* xs, float* ys) {
  using namespace ad;
  const DJoint& j = t.joints[ji];
  const int ia = j.index_a, ib = j.index_b, n = a.n_awake;
  const size_t nj = (size_t)a.n_joints;
  if (lane == 0) {
    const float4* rows = t.joint + (size_t)(sub * 2 + (stage == kRelax ? 1 : 0)) * 6 * nj;
    float4 r[6];
    for (int q = 0; q < 6; ++q) r[q] = rows[q * nj + ji];
    xs[jxVA] = r[0].x; xs[jxVA + 1] = r[0].y; xs[jxVA + 2] = r[0].z; xs[jxLin] = r[0].w;
    xs[jxWA] = r[1].x; xs[jxWA + 1] = r[1].y; xs[jxWA + 2] = r[1].z; xs[jxLin + 1] = r[1].w;
    xs[jxVB] = r[2].x; xs[jxVB + 1] = r[2].y; xs[jxVB + 2] = r[2].z; xs[jxLin + 2] = r[2].w;
    xs[jxWB] = r[3].x; xs[jxWB + 1] = r[3].y; xs[jxWB + 2] = r[3].z; xs[jxPerp] = r[3].w;
    xs[jxPerp + 1] = r[4].x; xs[jxSpring] = r[4].y; xs[jxMotor] = r[4].z; xs[jxLower] = r[4].w;
    xs[jxUpper] = r[5].x;
    const int row = stage == kRelax ? 2 : 1;  // push after integrate velocities, relax after positions
    joint_body_deltas(t, n, sub, row, ia, xs, jxDpA, jxDqA);
    joint_body_deltas(t, n, sub, row, ib, xs, jxDpB, jxDqB);
    // the solve recomputes the perp axes (unless the rotation is fixed, when nothing reads them)
    put3(xs, jxPx, j.perp_axis_x);
    put3(xs, jxPy, j.perp_axis_y);
    joint_consts(j, xs);
  }
  if (lane < 12) {
    const int b = lane < 6 ? ia : ib, g = lane % 6;
    ys[lane] = b >= 0 ? BB(a, b, g < 3 ? g : g + 1) : 0.0f;
  } else if (lane < kJSolveOut) {
    ys[lane] = JB(a, ji, lane - 12);
  }
  __syncwarp();
  const JParams jp = joint_params(j, p, stage == kPush);
  SeedIn<float, 3> in;
  in.x = xs;
  for (int kk = 0; kk < 3; ++kk) in.dir[kk] = lane + 32 * kk < kJX ? lane + 32 * kk : -1;
  Dual<float, 3> y[kJSolveOut];
  joint_solve_fn(in, jp, y);
  float xb[3];
  for (int kk = 0; kk < 3; ++kk) {
    float acc = 0.0f;
    for (int q = 0; q < kJSolveOut; ++q) acc += ys[q] * y[q].d[kk];
    xb[kk] = acc;
  }
  __syncwarp();
  for (int kk = 0; kk < 3; ++kk) {
    const int d = in.dir[kk];
    if (d < 0) continue;
    const float v = xb[kk];
    if (d < jxDpA) {
      const int b = d < 6 ? ia : ib, g = d % 6;
      if (b >= 0) BB(a, b, g < 3 ? g : g + 1) = v;
    } else if (d < jxDpB) {
      if (ia >= 0) BB(a, ia, 8 + d - jxDpA) += v;
    } else if (d < jxDqA) {
      if (ib >= 0) BB(a, ib, 8 + d - jxDpB) += v;
    } else if (d < jxDqB) {
      if (ia >= 0) BB(a, ia, 12 + d - jxDqA) += v;
    } else if (d < jxLin) {
      if (ib >= 0) BB(a, ib, 12 + d - jxDqB) += v;
    } else if (d < jxIma) {
      JB(a, ji, d - jxLin) = v;
    } else {
      JC(a, ji, d - jxIma) += v;
    }
  }
}

// Reverse of one joint's part of the warm start of substep sub (one warp): the change it made
// to its bodies' velocities depends on the impulses and perp axes the previous relax left (or
// prepare, for the first substep), the rotation increments and the constants. The bodies'
// velocity cotangents are only read; several joints share a body in this phase, so its rotation
// increments' cotangents are added atomically.
__device__ __noinline__ void adj_joint_warm(const StepTape& t, const AdjBufs& a, int sub, int ji, int lane, float* xs,
                                            float* ys) {
  using namespace ad;
  const DJoint& j = t.joints[ji];
  const int ia = j.index_a, ib = j.index_b, n = a.n_awake;
  const size_t nj = (size_t)a.n_joints;
  if (lane == 0) {
    for (int f = 0; f < jxDpA; ++f) xs[f] = 0.0f;
    if (sub == 0) {
      put3(xs, jxLin, j.linear_impulse);
      xs[jxPerp] = j.perp_impulse.x; xs[jxPerp + 1] = j.perp_impulse.y;
      xs[jxSpring] = j.spring_impulse; xs[jxMotor] = j.motor_impulse;
      xs[jxLower] = j.lower_impulse; xs[jxUpper] = j.upper_impulse;
      put3(xs, jxPx, j.perp_axis_x);
      put3(xs, jxPy, j.perp_axis_y);
    } else {
      const float4* rows = t.jwarm + (size_t)(sub - 1) * 4 * nj;
      float4 r0 = rows[ji], r1 = rows[nj + ji], r2 = rows[2 * nj + ji], r3 = rows[3 * nj + ji];
      xs[jxLin] = r0.x; xs[jxLin + 1] = r0.y; xs[jxLin + 2] = r0.z; xs[jxPerp] = r0.w;
      xs[jxPerp + 1] = r1.x; xs[jxSpring] = r1.y; xs[jxMotor] = r1.z; xs[jxLower] = r1.w;
      xs[jxUpper] = r2.x; xs[jxPx] = r2.y; xs[jxPx + 1] = r2.z; xs[jxPx + 2] = r2.w;
      xs[jxPy] = r3.x; xs[jxPy + 1] = r3.y; xs[jxPy + 2] = r3.z;
    }
    joint_body_deltas(t, n, sub, 0, ia, xs, jxDpA, jxDqA);
    joint_body_deltas(t, n, sub, 0, ib, xs, jxDpB, jxDqB);
    joint_consts(j, xs);
  }
  // body A took v - dva, w - dwa; body B v + dvb, w + dwb (dynamic bodies only)
  if (lane < 12) {
    const int b = lane < 6 ? ia : ib, g = lane % 6;
    const float sgn = lane < 6 ? -1.0f : 1.0f;
    ys[lane] = b >= 0 ? sgn * BB(a, b, g < 3 ? g : g + 1) : 0.0f;
  }
  __syncwarp();
  SeedIn<float, 3> in;
  in.x = xs;
  for (int kk = 0; kk < 3; ++kk) in.dir[kk] = lane + 32 * kk < kJX ? lane + 32 * kk : -1;
  Dual<float, 3> y[12];
  joint_warm_fn(in, y);
  for (int kk = 0; kk < 3; ++kk) {
    const int d = in.dir[kk];
    if (d < jxDqA) continue;  // velocities and position increments: not read
    float v = 0.0f;
    for (int q = 0; q < 12; ++q) v += ys[q] * y[q].d[kk];
    if (d < jxDqB) {
      if (ia >= 0) atomicAdd(&BB(a, ia, 12 + d - jxDqA), v);
    } else if (d < jxLin) {
      if (ib >= 0) atomicAdd(&BB(a, ib, 12 + d - jxDqB), v);
    } else if (d < jxIma) {
      JB(a, ji, d - jxLin) += v;
    } else {
      JC(a, ji, d - jxIma) += v;
    }
  }
  __syncwarp();
}

// Reverse of the solver stages of one step: a persistent launch over the same barriers as the
// forward solver, phases in reverse order, one thread per constraint or body (one warp per
// joint). The joints' reverse is compiled only into the kJoints variant: its dual-number frames
// would otherwise raise every world's stack frame and registers (880 -> 1376 bytes).
template <bool kGrid, bool kJoints>
__global__ void __launch_bounds__(kAdjThreads, 1) k_adj_solve(StepTape t, AdjBufs a, StepParams p, Control* ctl) {
  __shared__ int coff[25];
  __shared__ float jxs[kJoints ? kAdjThreads / 32 : 1][ad::kJX];
  __shared__ float jys[kJoints ? kAdjThreads / 32 : 1][ad::kJSolveOut];
  if (threadIdx.x < 24) coff[threadIdx.x] = t.ctl->color_offset[threadIdx.x];
  if (threadIdx.x == 24) coff[24] = t.ctl->color_offset[23];
  __syncthreads();
  const int n = a.n_awake;
  // items dealt 32 at a time across the blocks, as in the forward solver
  const int g = (((int)threadIdx.x >> 5) * (int)gridDim.x + (int)blockIdx.x) * 32 + ((int)threadIdx.x & 31);
  const int stride = gridDim.x * blockDim.x;
  // joints: one warp each
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int wg = blockIdx.x * (blockDim.x >> 5) + wib, wstride = gridDim.x * (blockDim.x >> 5);
  int bar = 0;
  auto contacts = [&](auto stage_tag, int sub) -> bool {
    constexpr int Stage = decltype(stage_tag)::value;
    for (int c = kOverflowIndex - 1; c >= 0; --c) {
      const int j0 = a.jr.off[c], j1 = a.jr.off[c + 1];
      if (coff[c + 1] == coff[c] && j1 == j0) continue;
      for (int k = coff[c] + g; k < coff[c + 1]; k += stride) adj_contact<Stage>(t, a, p, n, k, sub);
      if (kJoints)
        for (int q = j0 + wg; q < j1; q += wstride)
          adj_joint_solve(t, a, p, Stage, sub, a.joint_list[q], lane, jxs[wib], jys[wib]);
      if (!phase_sync<kGrid>(ctl, bar)) return false;
    }
    return true;
  };
  for (int sub = t.substeps - 1; sub >= 0; --sub) {
    if (!contacts(std::integral_constant<int, kRelax>(), sub)) return;
    for (int i = g; i < n; i += stride) adj_ip(t, a, p, n, i, sub);
    if (!phase_sync<kGrid>(ctl, bar)) return;
    if (!contacts(std::integral_constant<int, kPush>(), sub)) return;
    // Warm start changes a body's velocity by a constant (v - x), so its reverse leaves the body
    // cotangents as they are and only reads them: every colour's warm start reverses in one
    // phase, before integrate-velocities changes those cotangents.
    for (int k = g; k < coff[kOverflowIndex]; k += stride) adj_contact<kWarm>(t, a, p, n, k, sub);
    if (kJoints)
      for (int q = wg; q < a.n_joints; q += wstride) adj_joint_warm(t, a, sub, q, lane, jxs[wib], jys[wib]);
    if (!phase_sync<kGrid>(ctl, bar)) return;
    for (int i = g; i < n; i += stride) adj_iv(t, a, p, n, i, sub);
    if (!phase_sync<kGrid>(ctl, bar)) return;
  }
}

// Reverse of prepare for slot k (one warp): constraint cotangents -> manifold, masses,
// inverse inertia and friction.
__global__ void __launch_bounds__(kAdjThreads) k_adj_prepare(StepTape t, AdjBufs a, DW w, StepParams p, int n_slots) {
  using namespace ad;
  __shared__ float xs_s[kAdjThreads / 32][kPI + 2];
  __shared__ float ys_s[kAdjThreads / 32][kCVOwn];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int k = blockIdx.x * (kAdjThreads / 32) + warp;
  if (k >= n_slots) return;
  float* xs = xs_s[warp];
  float* ys = ys_s[warp];
  int4 idx = t.planes.idx[k];
  int ia = idx.x, ib = idx.y, cid = idx.z;
  const DContact& c = t.post[cid];
  PParams pp;
  pp.pc = idx.w & 255;
  pp.is_static = (idx.w & 256) != 0;
  pp.warm_start = p.warm_start;
  if (lane == 0) {
    const Manifold& m = c.manifold;
    xs[piN] = m.normal.x; xs[piN + 1] = m.normal.y; xs[piN + 2] = m.normal.z;
    for (int q = 0; q < 4; ++q) {
      const ManifoldPoint& mp = m.points[q];
      xs[pi_point(q, 0)] = mp.anchor_a.x; xs[pi_point(q, 1)] = mp.anchor_a.y; xs[pi_point(q, 2)] = mp.anchor_a.z;
      xs[pi_point(q, 3)] = mp.anchor_b.x; xs[pi_point(q, 4)] = mp.anchor_b.y; xs[pi_point(q, 5)] = mp.anchor_b.z;
      xs[pi_point(q, 6)] = mp.separation; xs[pi_point(q, 7)] = mp.normal_impulse;
    }
    xs[piFrictionImpulse] = m.friction_impulse.x; xs[piFrictionImpulse + 1] = m.friction_impulse.y;
    xs[piFrictionImpulse + 2] = m.friction_impulse.z;
    xs[piTwist] = m.twist_impulse;
    xs[piFriction] = c.friction;
  }
  if (lane == 1 || lane == 2) {
    int b = lane == 1 ? ia : ib;
    float im = 0.0f;
    Sym s = sym_zero();
    if (b >= 0) { im = t.sims[b].inv_mass; s = sym_from(t.sims[b].inv_inertia_world); }
    int at = lane == 1 ? piSa : piSb;
    xs[lane == 1 ? piIma : piImb] = im;
    xs[at] = s.xx; xs[at + 1] = s.xy; xs[at + 2] = s.xz; xs[at + 3] = s.yy; xs[at + 4] = s.yz; xs[at + 5] = s.zz;
  }
  for (int j = lane; j < kCVOwn; j += 32) ys[j] = a.kb[(size_t)j * a.cap + k];
  __syncwarp();
  SeedIn<float, 2> in;
  in.x = xs;
  in.dir[0] = lane;
  in.dir[1] = lane + 32 < kPI ? lane + 32 : -1;
  Dual<float, 2> y[kCVOwn];
  prepare_fn(in, pp, y);
  float xb[2];
  for (int kk = 0; kk < 2; ++kk) {
    float acc = 0.0f;
    for (int j = 0; j < kCVOwn; ++j) acc += ys[j] * y[j].d[kk];
    xb[kk] = acc;
  }
  const int sym_to_m3[6] = {0, 1, 2, 4, 5, 8};
  for (int kk = 0; kk < 2; ++kk) {
    int d = in.dir[kk];
    if (d < 0) continue;
    float v = xb[kk];
    if (d < piPoint) MB(a, cid, mbN + d) += v;
    else if (d < piFrictionImpulse) {
      int q = (d - piPoint) / 8, f = (d - piPoint) % 8;
      int mf = f < 7 ? f : 8;  // anchor_a, anchor_b, separation; normal impulse
      MB(a, cid, mb_point(q, mf)) += v;
    } else if (d < piTwist) MB(a, cid, mbFrictionImpulse + d - piFrictionImpulse) += v;
    else if (d == piTwist) MB(a, cid, mbTwist) += v;
    else if (d == piIma) { if (ia >= 0) atomicAdd(&PB(a, ia, pbInvMass), v); }
    else if (d == piImb) { if (ib >= 0) atomicAdd(&PB(a, ib, pbInvMass), v); }
    else if (d < piSb) { if (ia >= 0) atomicAdd(&PB(a, ia, pbIiw + sym_to_m3[d - piSa]), v); }
    else if (d < piFriction) { if (ib >= 0) atomicAdd(&PB(a, ib, pbIiw + sym_to_m3[d - piSb]), v); }
    else {
      // friction = sqrt(fa fb) (world_runtime.rs:1305 mix_friction)
      float fa = w.shapes[c.shape_a].friction, fb = w.shapes[c.shape_b].friction;
      if (c.friction > 0.0f) {
        if (ia >= 0) atomicAdd(&PB(a, ia, pbFriction), v * 0.5f * fb / c.friction);
        if (ib >= 0) atomicAdd(&PB(a, ib, pbFriction), v * 0.5f * fa / c.friction);
      }
    }
  }
}

// Reverse of the joints' prepare (one warp per joint): the constants' and the prepared perp axes'
// cotangents -> the bodies' rotations and centres, inverse masses and world inverse inertias.
// Then the joint's cotangents are made those of the previous step's end: the impulses carry
// over (prepare keeps them, or zeroes them without warm starting), the perp axes and the
// constants start afresh.
__global__ void __launch_bounds__(kAdjThreads) k_adj_joint_prepare(StepTape t, AdjBufs a, DW w, StepParams p) {
  using namespace ad;
  __shared__ float xs_s[kAdjThreads / 32][kJPI];
  __shared__ float ys_s[kAdjThreads / 32][kJPO];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ji = blockIdx.x * (kAdjThreads / 32) + warp;
  if (ji >= a.n_joints) return;
  float* xs = xs_s[warp];
  float* ys = ys_s[warp];
  const DJoint& j = t.joints[ji];
  auto sim_for = [&](int enc) -> const DSim& { return enc >= 0 ? t.sims[enc] : w.ssims[-enc - 2]; };
  const DSim& sa = sim_for(j.enc_a);
  const DSim& sb = sim_for(j.enc_b);
  if (lane == 0) {
    xs[jpQa] = sa.q.v.x; xs[jpQa + 1] = sa.q.v.y; xs[jpQa + 2] = sa.q.v.z; xs[jpQa + 3] = sa.q.s;
    xs[jpQb] = sb.q.v.x; xs[jpQb + 1] = sb.q.v.y; xs[jpQb + 2] = sb.q.v.z; xs[jpQb + 3] = sb.q.s;
    for (int f = 0; f < 6; ++f) xs[jpCa + f] = 0.0f;
    xs[jpIma] = sa.inv_mass;
    xs[jpImb] = sb.inv_mass;
    put3(xs, jpIA, sa.inv_inertia_world.cx); put3(xs, jpIA + 3, sa.inv_inertia_world.cy);
    put3(xs, jpIA + 6, sa.inv_inertia_world.cz);
    put3(xs, jpIB, sb.inv_inertia_world.cx); put3(xs, jpIB + 3, sb.inv_inertia_world.cy);
    put3(xs, jpIB + 6, sb.inv_inertia_world.cz);
  }
  for (int f = lane; f < kJPO; f += 32) ys[f] = f < 6 ? JB(a, ji, jxPx - jxLin + f) : JC(a, ji, f - 6);
  __syncwarp();
  SeedIn<float, 2> in;
  in.x = xs;
  in.dir[0] = lane;
  in.dir[1] = lane + 32 < kJPI ? lane + 32 : -1;
  Dual<float, 2> y[kJPO];
  const Pos ca = {sa.cx, sa.cy, sa.cz}, cb = {sb.cx, sb.cy, sb.cz};
  joint_prepare_fn(in, j.local_frame_a, j.local_frame_b, sa.local_center, sb.local_center, ca, cb, y);
  const int ia = j.enc_a >= 0 ? j.enc_a : -1, ib = j.enc_b >= 0 ? j.enc_b : -1;
  for (int kk = 0; kk < 2; ++kk) {
    const int d = in.dir[kk];
    if (d < 0) continue;
    float v = 0.0f;
    for (int q = 0; q < kJPO; ++q) v += ys[q] * y[q].d[kk];
    if (v == 0.0f) continue;
    if (d < jpQb) { if (ia >= 0) atomicAdd(&CQ(a, ia, 4 + d - jpQa), v); }
    else if (d < jpCa) { if (ib >= 0) atomicAdd(&CQ(a, ib, 4 + d - jpQb), v); }
    else if (d < jpCb) { if (ia >= 0) atomicAdd(&CQ(a, ia, d - jpCa), v); }
    else if (d < jpIma) { if (ib >= 0) atomicAdd(&CQ(a, ib, d - jpCb), v); }
    else if (d == jpIma) { if (ia >= 0) atomicAdd(&PB(a, ia, pbInvMass), v); }
    else if (d == jpImb) { if (ib >= 0) atomicAdd(&PB(a, ib, pbInvMass), v); }
    else if (d < jpIB) { if (ia >= 0) atomicAdd(&PB(a, ia, pbIiw + d - jpIA), v); }
    else { if (ib >= 0) atomicAdd(&PB(a, ib, pbIiw + d - jpIB), v); }
  }
  __syncwarp();
  // the previous step's end: impulses carry over unless prepare zeroed them
  for (int f = lane; f < kJState; f += 32) {
    const bool impulse = f < jxPx - jxLin;
    if (!impulse || p.warm_start == 0.0f) JB(a, ji, f) = 0.0f;
  }
  for (int f = lane; f < kJConst; f += 32) JC(a, ji, f) = 0.0f;
}

// Reverse of the inverse world inertia of finalize (one warp per body, lanes 0..12).
__global__ void __launch_bounds__(kAdjThreads) k_adj_inertia(StepTape t, AdjBufs a) {
  using namespace ad;
  __shared__ float xs_s[kAdjThreads / 32][14];
  __shared__ float ys_s[kAdjThreads / 32][9];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int i = blockIdx.x * (kAdjThreads / 32) + warp;
  if (i >= a.n_awake) return;
  float* xs = xs_s[warp];
  float* ys = ys_s[warp];
  const DSim& s = t.sims[i];
  if (lane == 0) {
    xs[0] = s.q.v.x; xs[1] = s.q.v.y; xs[2] = s.q.v.z; xs[3] = s.q.s;
    const float* m = &s.inv_inertia_local.cx.x;
    for (int f = 0; f < 9; ++f) xs[4 + f] = m[f];
  }
  if (lane < 9) ys[lane] = PB(a, i, pbIiw + lane);
  __syncwarp();
  SeedIn<float, 1> in;
  in.x = xs;
  in.dir[0] = lane < 13 ? lane : -1;
  Dual<float, 1> y[9];
  inv_inertia_fn(in, y);
  float acc = 0.0f;
  for (int j = 0; j < 9; ++j) acc += ys[j] * y[j].d[0];
  __syncwarp();
  if (lane < 4) CQ(a, i, 4 + lane) += acc;
  else if (lane < 13) PB(a, i, pbIinv + lane - 4) += acc;
  if (lane < 9) PB(a, i, pbIiw + lane) = 0.0f;
}

__device__ __forceinline__ const DSim& sim_at(const StepTape& t, const DW& w, int enc) {
  return enc >= 0 ? t.sims[enc] : w.ssims[-enc - 2];
}

// Reverse of the narrowphase for contact cid (one warp): the manifold's cotangent flows to the
// two bodies' poses at the start of the step and to the manifold state the step started from.
__global__ void __launch_bounds__(kAdjThreads) k_adj_narrow(StepTape t, AdjBufs a, DW w) {
  using namespace ad;
  __shared__ float xs_s[kAdjThreads / 32][kRI + 3];
  __shared__ float ys_s[kAdjThreads / 32][kMB + 1];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int cid = blockIdx.x * (kAdjThreads / 32) + warp;
  if (cid >= a.cap) return;
  float* xs = xs_s[warp];
  float* ys = ys_s[warp];
  int mode = t.mode[cid];
  if (mode != 1 && mode != 2) {
    for (int f = lane; f < kMB; f += 32) MB(a, cid, f) = 0.0f;
    return;
  }
  const DContact& post = t.post[cid];
  const DContact& pre = t.pre[cid];
  int ea = post.enc_a, eb = post.enc_b;
  const DSim& sa = sim_at(t, w, ea);
  const DSim& sb = sim_at(t, w, eb);
  int pc = post.manifold.point_count;
  for (int f = lane; f < kMB; f += 32) ys[f] = MB(a, cid, f);
  __syncwarp();
  auto body_bar = [&](int enc, int f, float v) {  // f: centre 0..2, rotation 4..7
    if (enc >= 0) atomicAdd(&CQ(a, enc, f), v);
  };
  if (mode == 2) {
    const DShape& A = w.shapes[post.shape_a];
    const DShape& B = w.shapes[post.shape_b];
    Pos pa = {sa.px, sa.py, sa.pz}, pb = {sb.px, sb.py, sb.pz};
    if (lane == 0) {
      for (int f = 0; f < 3; ++f) { xs[fiCa + f] = 0.0f; xs[fiCb + f] = 0.0f; }
      xs[fiQa] = sa.q.v.x; xs[fiQa + 1] = sa.q.v.y; xs[fiQa + 2] = sa.q.v.z; xs[fiQa + 3] = sa.q.s;
      xs[fiQb] = sb.q.v.x; xs[fiQb + 1] = sb.q.v.y; xs[fiQb + 2] = sb.q.v.z; xs[fiQb + 3] = sb.q.s;
    }
    __syncwarp();
    SeedIn<float, 1> in;
    in.x = xs;
    in.dir[0] = lane < kFI ? lane : -1;
    Dual<float, 1> y[kFO];
    uint32_t ids[4];
    int got;
    if (A.type == kHull && B.type == kHull) {
      NarrowCase nc = {post.sat.type, post.sat.index_a, post.sat.index_b, post.sat.hit};
      got = narrow_box_fn(in, pa, pb, w.hulls[A.hull], w.hulls[B.hull], nc, y, ids);
    } else {
      // the forward's choices from its own poses and GJK cache (every lane alike)
      const Hull* ha = A.type == kHull ? &w.hulls[A.hull] : nullptr;
      WXf wa = {pa, sa.q}, wb = {pb, sb.q};
      RoundCase rc = round_case(A, B, ha, inv_mul_wxf(wa, wb), pre.simplex);
      got = narrow_round_fn(in, pa, pb, A, B, ha, rc, y, ids);
    }
    bool same = got == pc;
    for (int q = 0; same && q < pc; ++q) same = ids[q] == post.manifold.points[q].feature_id;
    if (!same) {
      if (lane == 0) atomicAdd(a.mismatch, 1);
    } else {
      float acc = 0.0f;
      for (int j = 0; j < 3; ++j) acc += ys[mbN + j] * y[j].d[0];
      for (int q = 0; q < pc; ++q) {
        for (int f = 0; f < 6; ++f) acc += ys[mb_point(q, f)] * y[3 + 7 * q + f].d[0];
        acc += (ys[mb_point(q, 6)] + ys[mb_point(q, 7)]) * y[3 + 7 * q + 6].d[0];
      }
      if (lane < 3) body_bar(ea, lane, acc);
      else if (lane < 7) body_bar(ea, 4 + lane - 3, acc + ys[mbRotA + lane - 3]);
      else if (lane < 10) body_bar(eb, lane - 7, acc);
      else if (lane < 14) body_bar(eb, 4 + lane - 10, acc + ys[mbRotB + lane - 10]);
    }
    __syncwarp();
    // the state before the step: matched normal impulses, and the friction and twist
    // impulses a persisting manifold keeps
    if (lane == 0) {
      float out[kMB];
      for (int f = 0; f < kMB; ++f) out[f] = 0.0f;
      int old_count = pre.manifold_count > 0 ? pre.manifold.point_count : 0;
      if (old_count > 0) {
        bool used[4] = {false, false, false, false};
        for (int i = 0; i < pc; ++i) {
          uint32_t fid = post.manifold.points[i].feature_id;
          for (int j = 0; j < old_count; ++j) {
            if (!used[j] && pre.manifold.points[j].feature_id == fid) {
              out[mb_point(j, 8)] += ys[mb_point(i, 8)];
              used[j] = true;
              break;
            }
          }
        }
        for (int f = 0; f < 3; ++f) out[mbFrictionImpulse + f] = ys[mbFrictionImpulse + f];
        out[mbTwist] = ys[mbTwist];
      }
      for (int f = 0; f < kMB; ++f) MB(a, cid, f) = out[f];
    }
  } else {
    // recycled: separations recomputed from the poses and the cached manifold
    Pos ca = {sa.cx, sa.cy, sa.cz}, cb = {sb.cx, sb.cy, sb.cz};
    if (lane == 0) {
      for (int f = 0; f < 6; ++f) xs[riCa + f] = 0.0f;
      xs[riQa] = sa.q.v.x; xs[riQa + 1] = sa.q.v.y; xs[riQa + 2] = sa.q.v.z; xs[riQa + 3] = sa.q.s;
      xs[riQb] = sb.q.v.x; xs[riQb + 1] = sb.q.v.y; xs[riQb + 2] = sb.q.v.z; xs[riQb + 3] = sb.q.s;
      Q ra = post.cached_rot_a, rb = post.cached_rot_b;
      xs[riRotA] = ra.v.x; xs[riRotA + 1] = ra.v.y; xs[riRotA + 2] = ra.v.z; xs[riRotA + 3] = ra.s;
      xs[riRotB] = rb.v.x; xs[riRotB + 1] = rb.v.y; xs[riRotB + 2] = rb.v.z; xs[riRotB + 3] = rb.s;
      const Manifold& m = post.manifold;
      xs[riN] = m.normal.x; xs[riN + 1] = m.normal.y; xs[riN + 2] = m.normal.z;
      for (int q = 0; q < 4; ++q) {
        const ManifoldPoint& mp = m.points[q];
        xs[ri_point(q, 0)] = mp.anchor_a.x; xs[ri_point(q, 1)] = mp.anchor_a.y; xs[ri_point(q, 2)] = mp.anchor_a.z;
        xs[ri_point(q, 3)] = mp.anchor_b.x; xs[ri_point(q, 4)] = mp.anchor_b.y; xs[ri_point(q, 5)] = mp.anchor_b.z;
        xs[ri_point(q, 6)] = mp.base_separation;
      }
    }
    __syncwarp();
    SeedIn<float, 2> in;
    in.x = xs;
    in.dir[0] = lane;
    in.dir[1] = lane + 32 < kRI ? lane + 32 : -1;
    Dual<float, 2> y[4];
    recycle_fn(in, ca, cb, pc, y);
    float xb[2];
    for (int kk = 0; kk < 2; ++kk) {
      float acc = 0.0f;
      for (int q = 0; q < pc; ++q) acc += ys[mb_point(q, 6)] * y[q].d[kk];
      xb[kk] = acc;
    }
    __syncwarp();
    // the state before the step is the manifold itself, except the overwritten separations
    for (int f = lane; f < kMB; f += 32) {
      bool is_sep = f >= mbPoint && f < mbFrictionImpulse && (f - mbPoint) % 9 == 6;
      MB(a, cid, f) = is_sep ? 0.0f : ys[f];
    }
    __syncwarp();
    for (int kk = 0; kk < 2; ++kk) {
      int d = in.dir[kk];
      if (d < 0) continue;
      float v = xb[kk];
      if (d < riCb) body_bar(ea, d - riCa, v);
      else if (d < riQa) body_bar(eb, d - riCb, v);
      else if (d < riQb) body_bar(ea, 4 + d - riQa, v);
      else if (d < riRotA) body_bar(eb, 4 + d - riQb, v);
      else if (d < riRotB) MB(a, cid, mbRotA + d - riRotA) += v;
      else if (d < riN) MB(a, cid, mbRotB + d - riRotB) += v;
      else if (d < riPoint) MB(a, cid, mbN + d - riN) += v;
      else {
        int q = (d - riPoint) / 7, f = (d - riPoint) % 7;
        MB(a, cid, mb_point(q, f < 6 ? f : 7)) += v;  // anchors; base separation
      }
    }
  }
}

// Seeds (cotangents of the final state, body id order) and results.
__global__ void k_adj_seed(AdjBufs a, const int* body_loc, int nb, const float* dpos, const float* drot,
                           const float* dlin, const float* dang) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    int loc = body_loc[i];
    if (loc < 0) continue;
    for (int f = 0; f < 3; ++f) {
      CQ(a, loc, f) = dpos ? dpos[3 * i + f] : 0.0f;
      BB(a, loc, f) = dlin ? dlin[3 * i + f] : 0.0f;
      BB(a, loc, 4 + f) = dang ? dang[3 * i + f] : 0.0f;
    }
    for (int f = 0; f < 4; ++f) CQ(a, loc, 4 + f) = drot ? drot[4 * i + f] : 0.0f;
  }
}
// out per body id: lin 3 | ang 3 | mass | friction | pos 3 | rot 4 | restitution  (16 floats)
__global__ void k_adj_result(AdjBufs a, const DW w, const int* body_loc, int nb, float* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    float* o = out + (size_t)16 * i;
    int loc = body_loc[i];
    if (loc < 0) {
      for (int f = 0; f < 16; ++f) o[f] = 0.0f;
      continue;
    }
    for (int f = 0; f < 3; ++f) { o[f] = BB(a, loc, f); o[3 + f] = BB(a, loc, 4 + f); o[8 + f] = CQ(a, loc, f); }
    for (int f = 0; f < 4; ++f) o[11 + f] = CQ(a, loc, 4 + f);
    o[15] = PB(a, loc, pbRestitution);
    // inv_mass = 1/m and the local inverse inertia scale as 1/m
    const DSim& s = w.asims[loc];
    float im = s.inv_mass;
    const float* il = &s.inv_inertia_local.cx.x;
    float dot_ii = 0.0f;
    for (int f = 0; f < 9; ++f) dot_ii += PB(a, loc, pbIinv + f) * il[f];
    // the local inertia (gyroscopic step) scales as m
    const float* ii = &s.inertia.cx.x;
    float dot_i = 0.0f;
    for (int f = 0; f < 9; ++f) dot_i += PB(a, loc, pbInertia + f) * ii[f];
    o[6] = -PB(a, loc, pbInvMass) * im * im - dot_ii * im + dot_i * im;
    o[7] = PB(a, loc, pbFriction);
  }
}

// Snapshot copies of device buffers: dst[i] <- src[i] for each listed buffer.
struct CopyOp { const char* src; char* dst; size_t bytes; };
__global__ void k_multi_copy(const CopyOp* ops, int n_ops) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (size_t)gridDim.x * blockDim.x;
  for (int o = 0; o < n_ops; ++o) {
    CopyOp op = ops[o];
    size_t n16 = op.bytes / 16;
    const float4* s = (const float4*)op.src;
    float4* d = (float4*)op.dst;
    for (size_t i = tid; i < n16; i += stride) d[i] = s[i];
    for (size_t i = n16 * 16 + tid; i < op.bytes; i += stride) op.dst[i] = op.src[i];
  }
}

// Snapshot of a world's device allocations into one buffer: allocation i lives at base + off.
// save copies the allocations into the buffer, otherwise the buffer back into them.
struct SnapOp { char* dev; size_t off; size_t bytes; };
__global__ void k_snapshot(const SnapOp* ops, int n_ops, char* base, int save) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (size_t)gridDim.x * blockDim.x;
  for (int o = 0; o < n_ops; ++o) {
    SnapOp op = ops[o];
    const char* src = save ? op.dev : base + op.off;
    char* dst = save ? base + op.off : op.dev;
    size_t n16 = op.bytes / 16;
    for (size_t i = tid; i < n16; i += stride) ((float4*)dst)[i] = ((const float4*)src)[i];
    for (size_t i = n16 * 16 + tid; i < op.bytes; i += stride) dst[i] = src[i];
  }
}

}  // namespace nsd
