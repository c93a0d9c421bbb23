// The adjoint's reverse pass on the host in f64 (ns_world_vjp_f64): the same reverse order and
// the same local functions as the device kernels of nsd_adjoint.cuh, evaluated in double from a
// host copy of each step's tape. It is the f64 reference the f32 device adjoint is compared
// with. Differences from the device path, by design: each contact update's reverse sweep runs
// in full (the device splits the constant planes' cotangents into k_adj_consts), and prepare,
// the inverse world inertia and the narrowphase take one input direction at a time.
#pragma once
#include <vector>

#include "nsd_adjoint.cuh"

namespace nsd {
namespace host_adj {

using ad::Dual;
using ad::SeedIn;

struct Bufs {
  int n = 0, cap = 0;
  std::vector<double> bb, cq, pb, kb, mb;
  int64_t mismatch = 0;
  double& BB(int i, int f) { return bb[(size_t)i * 16 + f]; }
  double& CQ(int i, int f) { return cq[(size_t)i * 8 + f]; }
  double& PB(int i, int f) { return pb[(size_t)i * kPB + f]; }
  double& KB(int k, int cv) { return kb[(size_t)(cv - ad::cvLam) * cap + k]; }
  double& MB(int c, int f) { return mb[(size_t)f * cap + c]; }
  void init(int n_, int cap_) {
    n = n_; cap = cap_;
    bb.assign((size_t)n * 16, 0.0); cq.assign((size_t)n * 8, 0.0); pb.assign((size_t)n * kPB, 0.0);
    kb.assign((size_t)ad::kCVOwn * cap, 0.0); mb.assign((size_t)kMB * cap, 0.0);
  }
};

// World constants the reverse pass reads besides the tape.
struct Consts {
  const DShape* shapes;
  const Hull* hulls;
  const DSim* ssims;
};

inline const DSim& sim_at(const StepTape& t, const Consts& c, int enc) { return enc >= 0 ? t.sims[enc] : c.ssims[-enc - 2]; }

// Contraction of the output tangents with their cotangents for one seeded direction.
template <int NY>
double contract(const Dual<double, 1>* y, const double* yb, int ny = NY) {
  double acc = 0.0;
  for (int j = 0; j < ny; ++j) acc += yb[j] * y[j].d[0];
  return acc;
}

inline void finalize(const StepTape& t, Bufs& a) {
  for (int i = 0; i < a.n; ++i) {
    const DSim& s = t.sims[i];
    const DState& last = t.body[((size_t)(t.substeps - 1) * 3 + 2) * a.n + i];
    double xs[8] = {s.q.v.x, s.q.v.y, s.q.v.z, s.q.s, last.dq.v.x, last.dq.v.y, last.dq.v.z, last.dq.s};
    double qbar[4] = {a.CQ(i, 4), a.CQ(i, 5), a.CQ(i, 6), a.CQ(i, 7)};
    double xb[8];
    for (int d = 0; d < 8; ++d) {
      SeedIn<double, 1> in;
      in.x = xs;
      in.dir[0] = d;
      Dual<double, 1> y[4];
      ad::final_rot_fn<Dual<double, 1>>(in, y);
      xb[d] = contract<4>(y, qbar);
    }
    for (int f = 0; f < 3; ++f) a.BB(i, 8 + f) = a.CQ(i, f);
    for (int f = 0; f < 4; ++f) a.BB(i, 12 + f) = xb[4 + f];
    for (int f = 0; f < 4; ++f) a.CQ(i, 4 + f) = xb[f];
  }
}

inline void store(const StepTape& t, Bufs& a, int n_slots) {
  using namespace ad;
  for (int k = 0; k < n_slots; ++k) {
    int4 idx = t.planes.idx[k];
    int cid = idx.z, pc = idx.w & 255;
    for (int cv = cvLam; cv < kCV; ++cv) a.KB(k, cv) = 0.0;
    for (int q = 0; q < pc; ++q) {
      a.KB(k, cvLam + q) = a.MB(cid, mb_point(q, 8));
      a.MB(cid, mb_point(q, 8)) = 0.0;
    }
    double F[3] = {a.MB(cid, mbFrictionImpulse), a.MB(cid, mbFrictionImpulse + 1), a.MB(cid, mbFrictionImpulse + 2)};
    double twist = a.MB(cid, mbTwist);
    for (int f = 0; f < 3; ++f) a.MB(cid, mbFrictionImpulse + f) = 0.0;
    a.MB(cid, mbTwist) = 0.0;
    float4 fin = t.fin[k], t1 = t.planes.t1[k], t2 = t.planes.t2[k];
    a.KB(k, cvFr) = F[0] * t1.x + F[1] * t1.y + F[2] * t1.z;
    a.KB(k, cvFr + 1) = F[0] * t2.x + F[1] * t2.y + F[2] * t2.z;
    a.KB(k, cvTwist) = twist;
    for (int f = 0; f < 3; ++f) { a.KB(k, cvT1 + f) = fin.x * F[f]; a.KB(k, cvT2 + f) = fin.y * F[f]; }
  }
}

// The constraint vector of slot k for stage `stage` of substep `sub` (as nsd_adjoint.cuh gather_cv).
inline void gather(const StepTape& t, int n, int cap, int k, int sub, int stage, double* x) {
  float xf[ad::kCV];
  // gather_cv is a device function; restate its reads here with the same layout
  using namespace ad;
  const CPlanes& P = t.planes;
  int4 idx = P.idx[k];
  int ia = idx.x, ib = idx.y;
  auto put = [&](int at, float4 v, int cnt) {
    xf[at] = v.x; if (cnt > 1) xf[at + 1] = v.y; if (cnt > 2) xf[at + 2] = v.z; if (cnt > 3) xf[at + 3] = v.w;
  };
  const float4* rows = stage == kRelax ? t.relax + (size_t)sub * 5 * cap : t.push + (size_t)sub * 4 * cap;
  for (int r = 0; r < 4; ++r) {
    float4 v = rows[(size_t)r * cap + k];
    if (stage == kWarm) { v.x = 0.0f; v.y = 0.0f; v.z = 0.0f; }
    put(3 * r, v, 3);
    xf[cvLam + r] = v.w;
  }
  float4 fr = t.relax[((size_t)sub * 5 + 4) * cap + k];
  xf[cvFr] = fr.x; xf[cvFr + 1] = fr.y; xf[cvTwist] = fr.z;
  int row_sel = stage == kRelax ? 2 : 0;
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
  xf[cvIma] = m.x; xf[cvImb] = m.y; xf[cvFriction] = m.z;
  put(cvSa, P.ia0[k], 4);
  float4 v1 = P.ia1[k];
  xf[cvSa + 4] = v1.x; xf[cvSa + 5] = v1.y; xf[cvSb] = v1.z; xf[cvSb + 1] = v1.w;
  put(cvSb + 2, P.ib1[k], 4);
  put(cvN, P.n[k], 3);
  float4 t1 = P.t1[k], t2 = P.t2[k], ca = P.ca[k];
  put(cvT1, t1, 3); xf[cvTv1] = t1.w;
  put(cvT2, t2, 3); xf[cvTv2] = t2.w;
  put(cvCa, ca, 3); xf[cvTwistMass] = ca.w;
  put(cvCb, P.cb[k], 3);
  put(cvTm, P.tm[k], 4);
  for (int q = 0; q < 4; ++q) {
    float4 ra = P.pra[(size_t)q * cap + k], rb = P.prb[(size_t)q * cap + k], im = P.pimp[(size_t)q * cap + k];
    put(cv_point(q, 0), ra, 3); xf[cv_point(q, 6)] = ra.w;
    put(cv_point(q, 3), rb, 3); xf[cv_point(q, 7)] = rb.w;
    xf[cv_point(q, 8)] = im.z;
  }
  for (int i = 0; i < kCV; ++i) x[i] = xf[i];
}

inline void contact(const StepTape& t, Bufs& a, const StepParams& p, int k, int sub, int stage) {
  using namespace ad;
  int4 idx = t.planes.idx[k];
  int ia = idx.x, ib = idx.y;
  CParams cp;
  cp.pc = idx.w & 255;
  cp.is_static = (idx.w & 256) != 0;
  cp.inv_h = p.inv_h;
  cp.contact_speed = p.contact_speed;
  cp.contact_softness = p.contact_softness;
  cp.static_softness = p.static_softness;
  double x[kCV], xb[kCV], yb[kRelaxOut];
  gather(t, a.n, a.cap, k, sub, stage, x);
  for (int f = 0; f < 12; ++f) {
    int b = f < 6 ? ia : ib;
    int g = f % 6;
    yb[f] = b >= 0 ? a.BB(b, g < 3 ? g : g + 1) : 0.0;
  }
  for (int q = 0; q < 4; ++q) yb[12 + q] = a.KB(k, cvLam + q);
  yb[16] = a.KB(k, cvFr); yb[17] = a.KB(k, cvFr + 1); yb[18] = a.KB(k, cvTwist);
  for (int i = 0; i < kCV; ++i) xb[i] = 0.0;
  if (stage == kWarm) warm_vjp(x, cp, yb, xb);
  else if (stage == kPush) push_vjp(x, cp, yb, xb);
  else relax_vjp(x, cp, yb, xb);
  if (stage != kWarm) {
    for (int f = 0; f < 12; ++f) {
      int b = f < 6 ? ia : ib;
      int g = f % 6;
      if (b >= 0) a.BB(b, g < 3 ? g : g + 1) = xb[f];
    }
    for (int f = 0; f < 3; ++f) {
      if (ia >= 0) a.BB(ia, 8 + f) += xb[cvDpA + f];
      if (ib >= 0) a.BB(ib, 8 + f) += xb[cvDpB + f];
    }
    for (int f = 0; f < 4; ++f) {
      if (ia >= 0) a.BB(ia, 12 + f) += xb[cvDqA + f];
      if (ib >= 0) a.BB(ib, 12 + f) += xb[cvDqB + f];
    }
  }
  for (int cv = cvLam; cv < cvIma; ++cv) {
    bool updated = stage == kRelax || (stage == kPush && cv < cvFr);
    if (updated) a.KB(k, cv) = xb[cv];
    else if (stage == kWarm) a.KB(k, cv) += xb[cv];
  }
  for (int cv = cvIma; cv < kCV; ++cv) a.KB(k, cv) += xb[cv];
}

inline void ip(const StepTape& t, Bufs& a, const StepParams& p, int i, int sub) {
  using namespace ad;
  const DState& st = t.body[((size_t)sub * 3 + 1) * a.n + i];
  double x[kIP] = {st.v.x, st.v.y, st.v.z, st.w.x, st.w.y, st.w.z, st.dp.x, st.dp.y, st.dp.z,
                   st.dq.v.x, st.dq.v.y, st.dq.v.z, st.dq.s};
  const int map[kIP] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14, 15};
  double yb[kIP], xb[kIP];
  for (int f = 0; f < kIP; ++f) { yb[f] = a.BB(i, map[f]); xb[f] = 0.0; }
  BParams bp = {};
  bp.h = p.h; bp.inv_dt = p.inv_dt; bp.max_linear_speed = p.max_linear_speed; bp.flags = st.flags;
  ip_vjp(x, bp, yb, xb);
  for (int f = 0; f < kIP; ++f) a.BB(i, map[f]) = xb[f];
}

inline void iv(const StepTape& t, Bufs& a, const StepParams& p, int i, int sub) {
  using namespace ad;
  const DState& st = t.body[((size_t)sub * 3 + 0) * a.n + i];
  const DSim& s = t.sims[i];
  double x[kIVIn];
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
  double yb[kIVOut], xb[kIVIn];
  for (int f = 0; f < kIVOut; ++f) yb[f] = a.BB(i, map[f]);
  for (int f = 0; f < kIVIn; ++f) xb[f] = 0.0;
  BParams bp = {};
  bp.h = p.h; bp.lin_damp = s.linear_damping; bp.ang_damp = s.angular_damping; bp.grav_scale = s.gravity_scale;
  bp.gravity = p.gravity;
  bp.flags = s.flags;
  if (s.flags & kGyroscopic) {
    for (int d = 0; d < kIVIn; ++d) {
      if (d >= 16 && d < 22) continue;
      SeedIn<double, 1> sin;
      sin.x = x;
      sin.dir[0] = d;
      Dual<double, 1> y[kIVOut];
      iv_fn(sin, bp, y);
      xb[d] = contract<kIVOut>(y, yb);
    }
  } else {
    iv_vjp_plain(x, bp, yb, xb);
  }
  for (int f = 0; f < 6; ++f) a.BB(i, map[f]) = xb[f];
  a.PB(i, pbInvMass) += xb[6];
  for (int f = 0; f < 9; ++f) a.PB(i, pbIiw + f) += xb[7 + f];
  if (s.flags & kGyroscopic) {
    for (int f = 0; f < 4; ++f) a.CQ(i, 4 + f) += xb[22 + f];
    for (int f = 0; f < 4; ++f) a.BB(i, 12 + f) += xb[26 + f];
    for (int f = 0; f < 9; ++f) a.PB(i, pbInertia + f) += xb[30 + f];
  }
}

inline void solve(const StepTape& t, Bufs& a, const StepParams& p) {
  const int* off = t.ctl->color_offset;
  auto contacts = [&](int stage, int sub) {
    for (int c = kOverflowIndex - 1; c >= 0; --c)
      for (int k = off[c]; k < off[c + 1]; ++k) contact(t, a, p, k, sub, stage);
  };
  for (int sub = t.substeps - 1; sub >= 0; --sub) {
    contacts(kRelax, sub);
    for (int i = 0; i < a.n; ++i) ip(t, a, p, i, sub);
    contacts(kPush, sub);
    contacts(kWarm, sub);
    for (int i = 0; i < a.n; ++i) iv(t, a, p, i, sub);
  }
}

inline void prepare(const StepTape& t, Bufs& a, const Consts& cs, const StepParams& p, int n_slots) {
  using namespace ad;
  const int sym_to_m3[6] = {0, 1, 2, 4, 5, 8};
  for (int k = 0; k < n_slots; ++k) {
    int4 idx = t.planes.idx[k];
    int ia = idx.x, ib = idx.y, cid = idx.z;
    const DContact& c = t.post[cid];
    PParams pp;
    pp.pc = idx.w & 255;
    pp.is_static = (idx.w & 256) != 0;
    pp.warm_start = p.warm_start;
    double xs[kPI], ys[kCVOwn];
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
    for (int side = 0; side < 2; ++side) {
      int b = side == 0 ? ia : ib;
      float im = 0.0f;
      Sym s = sym_zero();
      if (b >= 0) { im = t.sims[b].inv_mass; s = sym_from(t.sims[b].inv_inertia_world); }
      int at = side == 0 ? piSa : piSb;
      xs[side == 0 ? piIma : piImb] = im;
      xs[at] = s.xx; xs[at + 1] = s.xy; xs[at + 2] = s.xz; xs[at + 3] = s.yy; xs[at + 4] = s.yz; xs[at + 5] = s.zz;
    }
    for (int j = 0; j < kCVOwn; ++j) ys[j] = a.kb[(size_t)j * a.cap + k];
    for (int d = 0; d < kPI; ++d) {
      SeedIn<double, 1> in;
      in.x = xs;
      in.dir[0] = d;
      Dual<double, 1> y[kCVOwn];
      prepare_fn(in, pp, y);
      double v = contract<kCVOwn>(y, ys);
      if (d < piPoint) a.MB(cid, mbN + d) += v;
      else if (d < piFrictionImpulse) {
        int q = (d - piPoint) / 8, f = (d - piPoint) % 8;
        a.MB(cid, mb_point(q, f < 7 ? f : 8)) += v;
      } else if (d < piTwist) a.MB(cid, mbFrictionImpulse + d - piFrictionImpulse) += v;
      else if (d == piTwist) a.MB(cid, mbTwist) += v;
      else if (d == piIma) { if (ia >= 0) a.PB(ia, pbInvMass) += v; }
      else if (d == piImb) { if (ib >= 0) a.PB(ib, pbInvMass) += v; }
      else if (d < piSb) { if (ia >= 0) a.PB(ia, pbIiw + sym_to_m3[d - piSa]) += v; }
      else if (d < piFriction) { if (ib >= 0) a.PB(ib, pbIiw + sym_to_m3[d - piSb]) += v; }
      else {
        float fa = cs.shapes[c.shape_a].friction, fb = cs.shapes[c.shape_b].friction;
        if (c.friction > 0.0f) {
          if (ia >= 0) a.PB(ia, pbFriction) += v * 0.5 * fb / c.friction;
          if (ib >= 0) a.PB(ib, pbFriction) += v * 0.5 * fa / c.friction;
        }
      }
    }
  }
}

inline void inertia(const StepTape& t, Bufs& a) {
  for (int i = 0; i < a.n; ++i) {
    const DSim& s = t.sims[i];
    double xs[13] = {s.q.v.x, s.q.v.y, s.q.v.z, s.q.s};
    const float* m = &s.inv_inertia_local.cx.x;
    for (int f = 0; f < 9; ++f) xs[4 + f] = m[f];
    double ys[9];
    for (int f = 0; f < 9; ++f) ys[f] = a.PB(i, pbIiw + f);
    for (int d = 0; d < 13; ++d) {
      SeedIn<double, 1> in;
      in.x = xs;
      in.dir[0] = d;
      Dual<double, 1> y[9];
      ad::inv_inertia_fn(in, y);
      double v = contract<9>(y, ys);
      if (d < 4) a.CQ(i, 4 + d) += v; else a.PB(i, pbIinv + d - 4) += v;
    }
    for (int f = 0; f < 9; ++f) a.PB(i, pbIiw + f) = 0.0;
  }
}

inline void narrow(const StepTape& t, Bufs& a, const Consts& cs) {
  using namespace ad;
  for (int cid = 0; cid < a.cap; ++cid) {
    int mode = t.mode[cid];
    if (mode != 1 && mode != 2) {
      for (int f = 0; f < kMB; ++f) a.MB(cid, f) = 0.0;
      continue;
    }
    const DContact& post = t.post[cid];
    const DContact& pre = t.pre[cid];
    int ea = post.enc_a, eb = post.enc_b;
    const DSim& sa = sim_at(t, cs, ea);
    const DSim& sb = sim_at(t, cs, eb);
    int pc = post.manifold.point_count;
    double ys[kMB];
    for (int f = 0; f < kMB; ++f) ys[f] = a.MB(cid, f);
    auto body_bar = [&](int enc, int f, double v) { if (enc >= 0) a.CQ(enc, f) += v; };
    if (mode == 2) {
      const DShape& A = cs.shapes[post.shape_a];
      const DShape& B = cs.shapes[post.shape_b];
      Pos pa = {sa.px, sa.py, sa.pz}, pb = {sb.px, sb.py, sb.pz};
      double xs[kFI] = {0, 0, 0, sa.q.v.x, sa.q.v.y, sa.q.v.z, sa.q.s, 0, 0, 0, sb.q.v.x, sb.q.v.y, sb.q.v.z, sb.q.s};
      NarrowCase nc = {post.sat.type, post.sat.index_a, post.sat.index_b, post.sat.hit};
      const bool boxes = A.type == kHull && B.type == kHull;
      const Hull* ha = A.type == kHull ? &cs.hulls[A.hull] : nullptr;
      RoundCase rc = {};
      if (!boxes) {
        WXf wa = {pa, sa.q}, wb = {pb, sb.q};
        rc = round_case(A, B, ha, inv_mul_wxf(wa, wb), pre.simplex);
      }
      bool same = true;
      double g[kFI];
      for (int d = 0; d < kFI && same; ++d) {
        SeedIn<double, 1> in;
        in.x = xs;
        in.dir[0] = d;
        Dual<double, 1> y[kFO];
        uint32_t ids[4];
        int got = boxes ? narrow_box_fn(in, pa, pb, cs.hulls[A.hull], cs.hulls[B.hull], nc, y, ids)
                        : narrow_round_fn(in, pa, pb, A, B, ha, rc, y, ids);
        same = got == pc;
        for (int q = 0; same && q < pc; ++q) same = ids[q] == post.manifold.points[q].feature_id;
        double acc = 0.0;
        for (int j = 0; j < 3; ++j) acc += ys[mbN + j] * y[j].d[0];
        for (int q = 0; same && q < pc; ++q) {
          for (int f = 0; f < 6; ++f) acc += ys[mb_point(q, f)] * y[3 + 7 * q + f].d[0];
          acc += (ys[mb_point(q, 6)] + ys[mb_point(q, 7)]) * y[3 + 7 * q + 6].d[0];
        }
        g[d] = acc;
      }
      if (!same) {
        a.mismatch++;
      } else {
        for (int d = 0; d < 3; ++d) body_bar(ea, d, g[d]);
        for (int d = 3; d < 7; ++d) body_bar(ea, 4 + d - 3, g[d] + ys[mbRotA + d - 3]);
        for (int d = 7; d < 10; ++d) body_bar(eb, d - 7, g[d]);
        for (int d = 10; d < 14; ++d) body_bar(eb, 4 + d - 10, g[d] + ys[mbRotB + d - 10]);
      }
      double out[kMB];
      for (int f = 0; f < kMB; ++f) out[f] = 0.0;
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
      for (int f = 0; f < kMB; ++f) a.MB(cid, f) = out[f];
    } else {
      Pos ca = {sa.cx, sa.cy, sa.cz}, cb = {sb.cx, sb.cy, sb.cz};
      double xs[kRI];
      for (int f = 0; f < 6; ++f) xs[riCa + f] = 0.0;
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
      for (int f = 0; f < kMB; ++f) {
        bool is_sep = f >= mbPoint && f < mbFrictionImpulse && (f - mbPoint) % 9 == 6;
        a.MB(cid, f) = is_sep ? 0.0 : ys[f];
      }
      double sepb[4];
      for (int q = 0; q < 4; ++q) sepb[q] = q < pc ? ys[mb_point(q, 6)] : 0.0;
      for (int d = 0; d < kRI; ++d) {
        SeedIn<double, 1> in;
        in.x = xs;
        in.dir[0] = d;
        Dual<double, 1> y[4];
        recycle_fn(in, ca, cb, pc, y);
        double v = contract<4>(y, sepb, pc);
        if (d < riCb) body_bar(ea, d - riCa, v);
        else if (d < riQa) body_bar(eb, d - riCb, v);
        else if (d < riQb) body_bar(ea, 4 + d - riQa, v);
        else if (d < riRotA) body_bar(eb, 4 + d - riQb, v);
        else if (d < riRotB) a.MB(cid, mbRotA + d - riRotA) += v;
        else if (d < riN) a.MB(cid, mbRotB + d - riRotB) += v;
        else if (d < riPoint) a.MB(cid, mbN + d - riN) += v;
        else {
          int q = (d - riPoint) / 7, f = (d - riPoint) % 7;
          a.MB(cid, mb_point(q, f < 6 ? f : 7)) += v;
        }
      }
    }
  }
}

// One step of the reverse pass (the device order: finalize, store, solve, prepare, inertia,
// narrowphase).
inline void step(const StepTape& t, Bufs& a, const Consts& cs, const StepParams& p) {
  int n_slots = t.ctl->color_offset[kOverflowIndex];
  finalize(t, a);
  store(t, a, n_slots);
  solve(t, a, p);
  prepare(t, a, cs, p, n_slots);
  inertia(t, a);
  narrow(t, a, cs);
}

}  // namespace host_adj
}  // namespace nsd
