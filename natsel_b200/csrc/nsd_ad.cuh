// Differentiable restatement of the step's local functions, for the vector-Jacobian product
// of a rollout (the adjoint).
//
// Every function here is a template over its scalar type T and repeats, operation for
// operation, the f32 code of the forward kernels it mirrors (the functions named beside each
// one). Instantiated with a dual number Dual<R, K> it carries K directional derivatives next
// to the value: its value part performs the same IEEE operations in the same order as the
// forward kernel, so for R = float every comparison takes the branch the forward step took,
// and the derivative parts are the exact derivatives of that branch. The adjoint kernels seed
// one input direction per warp lane, evaluate a local function once, and contract the output
// derivatives with the incoming cotangent, which yields one component of the local
// vector-Jacobian product per direction. With R = double the same code is the FP64 check.
#pragma once
#include "nsd_types.cuh"

namespace nsd {
namespace ad {

NSD_HD float rsqrt_(float a) { return sqrtf(a); }
NSD_HD double rsqrt_(double a) { return sqrt(a); }

// ---------------------------------------------------------------------------------------------
// Dual numbers: value v and K tangents d.
template <class R, int K>
struct Dual {
  R v;
  R d[K];
  NSD_HD Dual() {}
  NSD_HD Dual(R x) : v(x) {
#pragma unroll
    for (int k = 0; k < K; ++k) d[k] = R(0);
  }
  friend NSD_HD Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
  }
  friend NSD_HD Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
  }
  friend NSD_HD Dual operator-(const Dual& a) {
    Dual r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
  }
  friend NSD_HD Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
  }
  friend NSD_HD Dual operator/(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v / b.v;
    R ib = R(1) / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
  }
  friend NSD_HD bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
  friend NSD_HD bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
  friend NSD_HD bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
  friend NSD_HD bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
  friend NSD_HD bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
  friend NSD_HD Dual tsqrt(const Dual& a) {
    Dual r;
    r.v = rsqrt_(a.v);
    R s = r.v > R(0) ? R(0.5) / r.v : R(0);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * s;
    return r;
  }
  friend NSD_HD R val(const Dual& a) { return a.v; }
};

NSD_HD float tsqrt(float a) { return sqrtf(a); }
NSD_HD double tsqrt(double a) { return sqrt(a); }
NSD_HD float val(float a) { return a; }
NSD_HD double val(double a) { return a; }

// functions.rs:16-60 semantics: ties return the second operand.
template <class T> NSD_HD T tmin(const T& a, const T& b) { return a < b ? a : b; }
template <class T> NSD_HD T tmax(const T& a, const T& b) { return a > b ? a : b; }
template <class T> NSD_HD T tabs(const T& a) { return a < T(0.0f) ? -a : a; }
template <class T> NSD_HD T tclamp(const T& a, const T& lo, const T& hi) { return a < lo ? lo : (hi < a ? hi : a); }

// ---------------------------------------------------------------------------------------------
// Vectors, quaternions and matrices over T (nsd_math.cuh, same association order).
template <class T> struct TV2 { T x, y; };
template <class T> struct TV3 { T x, y, z; };
template <class T> struct TQ { TV3<T> v; T s; };
template <class T> struct TM3 { TV3<T> cx, cy, cz; };
template <class T> struct TM2 { TV2<T> cx, cy; };
template <class T> struct TSym { T xx, xy, xz, yy, yz, zz; };
template <class T> struct TXf { TV3<T> p; TQ<T> q; };
template <class T> struct TPlane { TV3<T> n; T off; };

template <class T> NSD_HD TV3<T> tv3(const T& x, const T& y, const T& z) { TV3<T> r = {x, y, z}; return r; }
template <class T> NSD_HD TV3<T> tv3(V3 a) { return tv3<T>(T(a.x), T(a.y), T(a.z)); }
template <class T> NSD_HD TV3<T> tzero3() { return tv3<T>(T(0.0f), T(0.0f), T(0.0f)); }
template <class T> NSD_HD TQ<T> tquat(TV3<T> v, const T& s) { TQ<T> r = {v, s}; return r; }
template <class T> NSD_HD TQ<T> tqid() { return tquat<T>(tzero3<T>(), T(1.0f)); }
template <class T> NSD_HD TM3<T> tm3(TV3<T> a, TV3<T> b, TV3<T> c) { TM3<T> r = {a, b, c}; return r; }
template <class T> NSD_HD TM3<T> tm3(const M3& m) { return tm3<T>(tv3<T>(m.cx), tv3<T>(m.cy), tv3<T>(m.cz)); }
template <class T> NSD_HD TPlane<T> tplane(const Plane& p) { TPlane<T> r = {tv3<T>(p.n), T(p.off)}; return r; }

template <class T> NSD_HD TV3<T> operator+(const TV3<T>& a, const TV3<T>& b) { return tv3<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> NSD_HD TV3<T> operator-(const TV3<T>& a, const TV3<T>& b) { return tv3<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> NSD_HD TV3<T> operator-(const TV3<T>& a) { return tv3<T>(-a.x, -a.y, -a.z); }
template <class T> NSD_HD TV3<T> operator*(const T& s, const TV3<T>& a) { return tv3<T>(s * a.x, s * a.y, s * a.z); }

template <class T> NSD_HD T dot(const TV3<T>& a, const TV3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> NSD_HD T length(const TV3<T>& v) { return tsqrt(dot(v, v)); }
template <class T> NSD_HD T length_sq(const TV3<T>& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
template <class T> NSD_HD TV3<T> normalize(const TV3<T>& a) {
  T ls = a.x * a.x + a.y * a.y + a.z * a.z;
  if (ls > T(1000.0f * kMinPositive)) {
    T s = T(1.0f) / tsqrt(ls);
    return tv3<T>(s * a.x, s * a.y, s * a.z);
  }
  return tzero3<T>();
}
template <class T> NSD_HD TV3<T> perp(const TV3<T>& a) {
  TV3<T> p = (a.x < T(-0.5f) || T(0.5f) < a.x) ? tv3<T>(a.y, -a.x, T(0.0f)) : tv3<T>(T(0.0f), a.z, -a.y);
  return normalize(p);
}
template <class T> NSD_HD TV3<T> mul_add(const TV3<T>& a, const T& s, const TV3<T>& b) {
  return tv3<T>(a.x + s * b.x, a.y + s * b.y, a.z + s * b.z);
}
template <class T> NSD_HD TV3<T> mul_sub(const TV3<T>& a, const T& s, const TV3<T>& b) {
  return tv3<T>(a.x - s * b.x, a.y - s * b.y, a.z - s * b.z);
}
template <class T> NSD_HD TV3<T> cross(const TV3<T>& a, const TV3<T>& b) {
  return tv3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class T> NSD_HD TV3<T> lerp(const TV3<T>& a, const TV3<T>& b, const T& t) {
  return tv3<T>((T(1.0f) - t) * a.x + t * b.x, (T(1.0f) - t) * a.y + t * b.y, (T(1.0f) - t) * a.z + t * b.z);
}
template <class T> NSD_HD TV3<T> blend2(const T& s, const TV3<T>& a, const T& t, const TV3<T>& b) {
  return tv3<T>(s * a.x + t * b.x, s * a.y + t * b.y, s * a.z + t * b.z);
}
template <class T> NSD_HD TV3<T> rotate(const TQ<T>& q, const TV3<T>& v) {
  TV3<T> t1 = cross(q.v, v);
  TV3<T> t2 = mul_add(t1, q.s, v);
  TV3<T> t3 = cross(q.v, t2);
  return mul_add(v, T(2.0f), t3);
}
template <class T> NSD_HD TV3<T> inv_rotate(const TQ<T>& q, const TV3<T>& v) {
  TV3<T> t1 = cross(q.v, v);
  TV3<T> t2 = mul_sub(t1, q.s, v);
  TV3<T> t3 = cross(q.v, t2);
  return mul_add(v, T(2.0f), t3);
}
// nsd_types.cuh inv_rotate_wide (contact_solver.rs:291)
template <class T> NSD_HD TV3<T> inv_rotate_wide(const TQ<T>& q, const TV3<T>& a) {
  TV3<T> t0 = cross(q.v, a);
  TV3<T> t = tv3<T>(t0.x + t0.x, t0.y + t0.y, t0.z + t0.z);
  TV3<T> u = cross(q.v, t);
  return tv3<T>((a.x - q.s * t.x) + u.x, (a.y - q.s * t.y) + u.y, (a.z - q.s * t.z) + u.z);
}
template <class T> NSD_HD T dot_quat(const TQ<T>& a, const TQ<T>& b) {
  return a.v.x * b.v.x + a.v.y * b.v.y + a.v.z * b.v.z + a.s * b.s;
}
template <class T> NSD_HD TQ<T> mul_quat(const TQ<T>& q1, const TQ<T>& q2) {
  TV3<T> t1 = cross(q1.v, q2.v);
  TV3<T> t2 = mul_add(t1, q1.s, q2.v);
  TV3<T> t3 = mul_add(t2, q2.s, q1.v);
  return tquat<T>(t3, q1.s * q2.s - dot(q1.v, q2.v));
}
template <class T> NSD_HD TQ<T> inv_mul_quat(const TQ<T>& q1, const TQ<T>& q2) {
  TV3<T> t1 = cross(q2.v, q1.v);
  TV3<T> t2 = mul_add(t1, q1.s, q2.v);
  TV3<T> t3 = mul_sub(t2, q2.s, q1.v);
  return tquat<T>(t3, q1.s * q2.s + dot(q1.v, q2.v));
}
template <class T> NSD_HD TQ<T> conjugate(const TQ<T>& q) { return tquat<T>(tv3<T>(-q.v.x, -q.v.y, -q.v.z), q.s); }
template <class T> NSD_HD TQ<T> normalize_quat(const TQ<T>& q) {
  T ls = dot_quat(q, q);
  if (ls > T(1000.0f * kMinPositive)) {
    T s = T(1.0f) / tsqrt(ls);
    return tquat<T>(tv3<T>(s * q.v.x, s * q.v.y, s * q.v.z), s * q.s);
  }
  return tqid<T>();
}
template <class T> NSD_HD TQ<T> integrate_rotation(const TQ<T>& q1, const TV3<T>& dr) {
  TQ<T> qd = mul_quat(tquat<T>(T(0.5f) * dr, T(0.0f)), q1);
  return normalize_quat(tquat<T>(q1.v + qd.v, qd.s + q1.s));
}
template <class T> NSD_HD TXf<T> invert_xf(const TXf<T>& t) {
  TXf<T> r = {inv_rotate(t.q, -t.p), conjugate(t.q)};
  return r;
}
template <class T> NSD_HD TV3<T> xf_point(const TXf<T>& t, const TV3<T>& v) { return rotate(t.q, v) + t.p; }
template <class T> NSD_HD TM3<T> matrix_from_quat(const TQ<T>& q) {
  T xx = q.v.x * q.v.x, yy = q.v.y * q.v.y, zz = q.v.z * q.v.z;
  T xy = q.v.x * q.v.y, xz = q.v.x * q.v.z, xw = q.v.x * q.s;
  T yz = q.v.y * q.v.z, yw = q.v.y * q.s, zw = q.v.z * q.s;
  const T one(1.0f), two(2.0f);
  return tm3<T>(tv3<T>(one - two * (yy + zz), two * (xy + zw), two * (xz - yw)),
                tv3<T>(two * (xy - zw), one - two * (xx + zz), two * (yz + xw)),
                tv3<T>(two * (xz + yw), two * (yz - xw), one - two * (xx + yy)));
}
template <class T> NSD_HD TV3<T> mul_mv(const TM3<T>& m, const TV3<T>& a) {
  return tv3<T>(m.cx.x * a.x + m.cy.x * a.y + m.cz.x * a.z,
                m.cx.y * a.x + m.cy.y * a.y + m.cz.y * a.z,
                m.cx.z * a.x + m.cy.z * a.y + m.cz.z * a.z);
}
template <class T> NSD_HD TM3<T> mul_mm(const TM3<T>& a, const TM3<T>& b) {
  return tm3<T>(mul_mv(a, b.cx), mul_mv(a, b.cy), mul_mv(a, b.cz));
}
template <class T> NSD_HD TM3<T> transpose(const TM3<T>& m) {
  return tm3<T>(tv3<T>(m.cx.x, m.cy.x, m.cz.x), tv3<T>(m.cx.y, m.cy.y, m.cz.y), tv3<T>(m.cx.z, m.cy.z, m.cz.z));
}
template <class T> NSD_HD TV3<T> sym_mv(const TSym<T>& s, const TV3<T>& a) {
  return tv3<T>(s.xx * a.x + (s.xy * a.y + s.xz * a.z), s.xy * a.x + (s.yy * a.y + s.yz * a.z),
                s.xz * a.x + (s.yz * a.y + s.zz * a.z));
}
template <class T> NSD_HD TSym<T> sym_add(const TSym<T>& a, const TSym<T>& b) {
  TSym<T> s = {a.xx + b.xx, a.xy + b.xy, a.xz + b.xz, a.yy + b.yy, a.yz + b.yz, a.zz + b.zz};
  return s;
}
template <class T> NSD_HD TV2<T> mul_mv2(const TM2<T>& m, const TV2<T>& a) {
  TV2<T> r = {m.cx.x * a.x + m.cy.x * a.y, m.cx.y * a.x + m.cy.y * a.y};
  return r;
}
template <class T> NSD_HD T plane_sep(const TPlane<T>& p, const TV3<T>& x) { return dot(p.n, x) - p.off; }

// A world-space difference of f64 centres, rounded to f32 like sub_pos, plus the difference of
// the two centres' offsets ta - tb. The adjoint passes zero offsets (the value stays sub_pos's
// bits) whose tangents carry the centres' perturbations.
template <class T> NSD_HD TV3<T> sub_pos_t(const Pos& a, const Pos& b, const TV3<T>& ta, const TV3<T>& tb) {
  V3 r = sub_pos(a, b);
  TV3<T> t = ta - tb;
  return tv3<T>(t.x + T(r.x), t.y + T(r.y), t.z + T(r.z));
}

template <class T> NSD_HD V3 real3(const TV3<T>& a) { return v3((float)val(a.x), (float)val(a.y), (float)val(a.z)); }

// ---------------------------------------------------------------------------------------------
// Input access: a local function reads input i as in(i). Plain evaluation returns the stored
// value; a seeded evaluation returns a dual number whose tangent k is 1 when i is the k-th
// direction of this lane.
template <class R>
struct PlainIn {
  const R* x;
  NSD_HD R operator()(int i) const { return x[i]; }
};
template <class R, int K>
struct SeedIn {
  const R* x;
  int dir[K];
  NSD_HD Dual<R, K> operator()(int i) const {
    Dual<R, K> r(x[i]);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = dir[k] == i ? R(1) : R(0);
    return r;
  }
};

// ---------------------------------------------------------------------------------------------
// Constraint vector layout (one contact constraint; shared by warm start, push, relax and the
// output of prepare). Indices below 26 are the two bodies' solver state.
enum CV : int {
  cvVA = 0, cvWA = 3, cvVB = 6, cvWB = 9, cvDpA = 12, cvDpB = 15, cvDqA = 18, cvDqB = 22,
  cvLam = 26, cvFr = 30, cvTwist = 32,
  cvIma = 33, cvImb = 34, cvSa = 35, cvSb = 41, cvN = 47, cvT1 = 50, cvT2 = 53, cvTv1 = 56, cvTv2 = 57,
  cvCa = 58, cvCb = 61, cvTwistMass = 64, cvTm = 65, cvFriction = 69,
  cvPoint = 70,  // + 9 q: ra 0..2, rb 3..5, base separation 6, normal mass 7, lever 8
  kCV = 106,
  kCVOwn = kCV - cvLam,  // the constraint's own entries (impulses and constants)
};
NSD_HD int cv_point(int q, int f) { return cvPoint + 9 * q + f; }

template <class T, class In> NSD_HD TV3<T> in3(const In& x, int i) { return tv3<T>(x(i), x(i + 1), x(i + 2)); }
template <class T, class In> NSD_HD TQ<T> in4(const In& x, int i) { return tquat<T>(tv3<T>(x(i), x(i + 1), x(i + 2)), x(i + 3)); }
template <class T, class In> NSD_HD TSym<T> in_sym(const In& x, int i) {
  TSym<T> s = {x(i), x(i + 1), x(i + 2), x(i + 3), x(i + 4), x(i + 5)};
  return s;
}
template <class T> NSD_HD void out3(T* y, int i, const TV3<T>& a) { y[i] = a.x; y[i + 1] = a.y; y[i + 2] = a.z; }
template <class T> NSD_HD void out4(T* y, int i, const TQ<T>& a) { y[i] = a.v.x; y[i + 1] = a.v.y; y[i + 2] = a.v.z; y[i + 3] = a.s; }

// Parameters of one constraint that are not differentiated.
struct CParams {
  int pc;          // manifold points
  int is_static;   // softness of a static contact
  float inv_h, contact_speed;
  Softness contact_softness, static_softness;
};

// Outputs of warm start: vA wA vB wB (12).
constexpr int kWarmOut = 12;
// nsd_solve.cuh warm_start_constraint (contact_solver.rs:697), rolling resistance zero.
template <class T, class In>
NSD_HD void warm_fn(const In& x, const CParams& cp, T* y) {
  TV3<T> t1 = in3<T>(x, cvT1), t2 = in3<T>(x, cvT2);
  TV3<T> center_a = in3<T>(x, cvCa), center_b = in3<T>(x, cvCb);
  T twist = x(cvTwist);
  TV3<T> li = tzero3<T>(), aia = tzero3<T>(), aib = tzero3<T>();
  T tni = T(0.0f);
  TV3<T> moa = tzero3<T>(), mob = tzero3<T>();
  for (int q = 0; q < cp.pc; ++q) {
    T ni = x(cvLam + q);
    tni = tni + ni;
    moa = mul_add(moa, ni, in3<T>(x, cv_point(q, 0)));
    mob = mul_add(mob, ni, in3<T>(x, cv_point(q, 3)));
  }
  TV3<T> n = in3<T>(x, cvN);
  TV3<T> fi = x(cvFr) * t1;
  fi = mul_add(fi, x(cvFr + 1), t2);
  TV3<T> lin = mul_add(fi, tni, n);
  TV3<T> twi = twist * n;
  TV3<T> anga = cross(moa, n) + cross(center_a, fi) + twi;
  TV3<T> angb = cross(mob, n) + cross(center_b, fi) + twi;
  li = li + lin; aia = aia + anga; aib = aib + angb;
  TSym<T> sa = in_sym<T>(x, cvSa), sb = in_sym<T>(x, cvSb);
  T ima = x(cvIma), imb = x(cvImb);
  out3(y, 3, in3<T>(x, cvWA) - sym_mv(sa, aia));
  out3(y, 0, in3<T>(x, cvVA) - ima * li);
  out3(y, 9, in3<T>(x, cvWB) + sym_mv(sb, aib));
  out3(y, 6, in3<T>(x, cvVB) + imb * li);
}

// Outputs of push: vA wA vB wB (12), normal impulses (4).
constexpr int kPushOut = 16;
// nsd_solve.cuh push_constraint (contact_solver.rs:796)
template <class T, class In>
NSD_HD void push_fn(const In& x, const CParams& cp, T* y) {
  T inv_h = T(cp.inv_h);
  T cs = T(-cp.contact_speed);
  const Softness& so = cp.is_static ? cp.static_softness : cp.contact_softness;
  T br = T(so.mass_scale * so.bias_rate);
  T ms = T(so.mass_scale);
  T is = T(so.impulse_scale);
  TV3<T> va = in3<T>(x, cvVA), wa = in3<T>(x, cvWA), vb = in3<T>(x, cvVB), wb = in3<T>(x, cvWB);
  TQ<T> dqa = in4<T>(x, cvDqA), dqb = in4<T>(x, cvDqB);
  TV3<T> dp = in3<T>(x, cvDpB) - in3<T>(x, cvDpA);
  T ima = x(cvIma), imb = x(cvImb);
  TSym<T> sa = in_sym<T>(x, cvSa), sb = in_sym<T>(x, cvSb);
  T im = ima + imb;
  TV3<T> n = in3<T>(x, cvN);
  T ns = dot(n, dp);
  TV3<T> na = inv_rotate_wide(dqa, n), nb = inv_rotate_wide(dqb, n);
  T lnv = dot(n, vb - va);
  T mi = T(0.0f);
  for (int q = 0; q < 4; ++q) y[12 + q] = x(cvLam + q);
  for (int q = 0; q < cp.pc; ++q) {
    TV3<T> ra = in3<T>(x, cv_point(q, 0)), rb = in3<T>(x, cv_point(q, 3));
    T base_sep = x(cv_point(q, 6)), nmass = x(cv_point(q, 7)), nimp = x(cvLam + q);
    T s = (ns + (dot(nb, rb) - dot(na, ra))) + base_sep;
    bool sep = s > T(0.0f);
    T spec_bias = s * inv_h;
    T ovl = tmax(br * s, cs);
    T vbias = sep ? spec_bias : ovl;
    T pms = sep ? T(1.0f) : ms;
    T pis = sep ? T(0.0f) : is;
    TV3<T> ua = cross(ra, n), ub = cross(rb, n);
    TV3<T> ga = sym_mv(sa, ua), gb = sym_mv(sb, ub);
    T vn = lnv + (dot(ub, wb) - dot(ua, wa));
    T neg = nmass * (pms * vn + vbias) + pis * nimp;
    T impulse = tmax(-neg, -nimp);
    y[12 + q] = nimp + impulse;
    lnv = lnv + im * impulse;
    mi = mi + impulse;
    wa = wa - impulse * ga;
    wb = wb + impulse * gb;
  }
  TV3<T> Pv = mi * n;
  va = va - ima * Pv;
  vb = vb + imb * Pv;
  out3(y, 0, va); out3(y, 3, wa); out3(y, 6, vb); out3(y, 9, wb);
}

// Outputs of relax: vA wA vB wB (12), normal impulses (4), friction impulse (2), twist (1).
constexpr int kRelaxOut = 19;
// nsd_solve.cuh relax_constraint (contact_solver.rs:927), rolling resistance zero.
template <class T, class In>
NSD_HD void relax_fn(const In& x, const CParams& cp, T* y) {
  T inv_h = T(cp.inv_h);
  const T eps(kEps);
  TV3<T> va = in3<T>(x, cvVA), wa = in3<T>(x, cvWA), vb = in3<T>(x, cvVB), wb = in3<T>(x, cvWB);
  TQ<T> dqa = in4<T>(x, cvDqA), dqb = in4<T>(x, cvDqB);
  TV3<T> dp = in3<T>(x, cvDpB) - in3<T>(x, cvDpA);
  T ima = x(cvIma), imb = x(cvImb);
  TSym<T> sa = in_sym<T>(x, cvSa), sb = in_sym<T>(x, cvSb);
  T im = ima + imb;
  TV3<T> n = in3<T>(x, cvN);
  TV3<T> t1 = in3<T>(x, cvT1), t2 = in3<T>(x, cvT2);
  T ns = dot(n, dp);
  TV3<T> na = inv_rotate_wide(dqa, n), nb = inv_rotate_wide(dqb, n);
  TV3<T> dv = vb - va;
  T lnv = dot(n, dv);
  T lt1 = dot(t1, dv) - x(cvTv1);
  T lt2 = dot(t2, dv) - x(cvTv2);
  T mi = T(0.0f), tni = T(0.0f), ttl = T(0.0f);
  for (int q = 0; q < 4; ++q) y[12 + q] = x(cvLam + q);
  for (int q = 0; q < cp.pc; ++q) {
    TV3<T> ra = in3<T>(x, cv_point(q, 0)), rb = in3<T>(x, cv_point(q, 3));
    T s = (ns + (dot(nb, rb) - dot(na, ra))) + x(cv_point(q, 6));
    T vbias = tmax(T(0.0f), s * inv_h);
    TV3<T> ua = cross(ra, n), ub = cross(rb, n);
    TV3<T> ga = sym_mv(sa, ua), gb = sym_mv(sb, ub);
    T vn = lnv + (dot(ub, wb) - dot(ua, wa));
    T neg = x(cv_point(q, 7)) * (vn + vbias);
    T old = x(cvLam + q);
    T impulse = tmax(-neg, -old);
    T ni = old + impulse;
    y[12 + q] = ni;
    tni = tni + ni;
    ttl = ttl + x(cv_point(q, 8)) * ni;
    lnv = lnv + im * impulse;
    mi = mi + impulse;
    wa = wa - impulse * ga;
    wb = wb + impulse * gb;
  }
  T twist_out, frx, fry;
  {
    T ts = dot(n, wb - wa);
    T ml = x(cvFriction) * ttl;
    T old = x(cvTwist);
    T impulse = -(x(cvTwistMass) * ts);
    impulse = tmax(-ml - old, tmin(impulse, ml - old));
    twist_out = old + impulse;
    wa = wa - impulse * sym_mv(sa, n);
    wb = wb + impulse * sym_mv(sb, n);
    TV3<T> ra = in3<T>(x, cvCa), rb = in3<T>(x, cvCb);
    TM2<T> tm;
    tm.cx.x = x(cvTm); tm.cx.y = x(cvTm + 1);
    tm.cy.x = x(cvTm + 2); tm.cy.y = x(cvTm + 3);
    TV3<T> arv = cross(wb, rb) - cross(wa, ra);
    TV2<T> vt = {lt1 + dot(arv, t1), lt2 + dot(arv, t2)};
    TV2<T> di = mul_mv2(tm, vt);
    di.x = -di.x; di.y = -di.y;
    T fx = x(cvFr), fy = x(cvFr + 1);
    TV2<T> ni = {fx + di.x, fy + di.y};
    T mx = x(cvFriction) * tni;
    T lsq = ni.x * ni.x + ni.y * ni.y;
    bool mask = lsq > mx * mx;
    T nrm = mx / (tsqrt(lsq) + eps);
    T sc = mask ? nrm : T(1.0f);
    ni.x = sc * ni.x; ni.y = sc * ni.y;
    di.x = ni.x - fx; di.y = ni.y - fy;
    frx = ni.x; fry = ni.y;
    TV3<T> Pv = di.x * t1;
    Pv = Pv + di.y * t2;
    wa = wa - sym_mv(sa, cross(ra, Pv));
    wb = wb + sym_mv(sb, cross(rb, Pv));
    Pv = Pv + mi * n;
    va = va - ima * Pv;
    vb = vb + imb * Pv;
  }
  out3(y, 0, va); out3(y, 3, wa); out3(y, 6, vb); out3(y, 9, wb);
  y[16] = frx; y[17] = fry; y[18] = twist_out;
}

// ---------------------------------------------------------------------------------------------
// Restitution (nsd_solve.cuh restitution_constraint, contact_solver.rs:1135 apply_restitution_body)
// has its own input vector: the two bodies' velocities and final position deltas, the points'
// normal, total normal and restitution impulses, and the constants the update reads.
enum RV : int {
  rvVA = 0, rvWA = 3, rvVB = 6, rvWB = 9, rvDpA = 12, rvDpB = 15, rvDqA = 18, rvDqB = 22,
  rvLam = 26, rvTot = 30, rvRest = 34, rvIma = 38, rvImb = 39, rvSa = 40, rvSb = 46, rvN = 52, rvE = 55,
  rvPoint = 56,  // + 10 q: ra 0..2, rb 3..5, base separation 6, normal mass 7, relative velocity 8
  kRV = 96,
};
NSD_HD int rv_point(int q, int f) { return rvPoint + 10 * q + f; }
// Outputs: vA wA vB wB (12), normal impulses (4), total normal impulses (4), restitution impulses (4).
constexpr int kRestOut = 24;
struct RParams {
  int pc;
  float inv_h, threshold;
};

// The restitution update of one constraint, restated on a scalar type T (float, double or a dual
// number). With restitution 0 the update does nothing (the outputs are the inputs).
template <class T, class In>
NSD_HD void restitution_fn(const In& x, const RParams& rp, T* y) {
  TV3<T> va = in3<T>(x, rvVA), wa = in3<T>(x, rvWA), vb = in3<T>(x, rvVB), wb = in3<T>(x, rvWB);
  for (int q = 0; q < 4; ++q) {
    y[12 + q] = x(rvLam + q);
    y[16 + q] = x(rvTot + q);
    y[20 + q] = x(rvRest + q);
  }
  T e = x(rvE);
  if (val(e) != 0.0f) {
    T inv_h = T(rp.inv_h);
    T nrt = T(-rp.threshold);
    bool rmask = e > T(0.0f);
    TV3<T> dp = in3<T>(x, rvDpB) - in3<T>(x, rvDpA);
    TV3<T> n = in3<T>(x, rvN);
    T ns = dot(n, dp);
    TQ<T> dqa = in4<T>(x, rvDqA), dqb = in4<T>(x, rvDqB);
    TV3<T> na = inv_rotate_wide(dqa, n), nb = inv_rotate_wide(dqb, n);
    T ima = x(rvIma), imb = x(rvImb);
    TSym<T> sa = in_sym<T>(x, rvSa), sb = in_sym<T>(x, rvSb);
    for (int q = 0; q < rp.pc; ++q) {
      TV3<T> ra = in3<T>(x, rv_point(q, 0)), rb = in3<T>(x, rv_point(q, 3));
      T lam = y[12 + q], tot = y[16 + q], rest = y[20 + q];
      T relvel = x(rv_point(q, 8));
      T s = (ns + (dot(nb, rb) - dot(na, ra))) + x(rv_point(q, 6));
      T nm = rmask ? x(rv_point(q, 7)) : T(0.0f);
      T comp = tot - rest;
      bool armed = rmask && relvel < nrt && comp > T(0.0f);
      T sbias = tmax(T(0.0f), s * inv_h);
      T vbias = armed ? e * relvel : sbias;
      TV3<T> vra = va + cross(wa, ra), vrb = vb + cross(wb, rb);
      T vn = dot(vrb - vra, n);
      T neg = nm * (vn + vbias);
      T ni = tmax(lam - neg, T(0.0f));
      T impulse = ni - lam;
      T app = tmin(tmax(-nm * vn, T(0.0f)), tmax(impulse, T(0.0f)));
      T allow = e * (comp + app) - rest;
      T mx = app + tmax(allow, T(0.0f));
      impulse = armed ? tmin(impulse, mx) : impulse;
      y[12 + q] = lam + impulse;
      y[20 + q] = rest + (impulse - app);
      y[16 + q] = tot + impulse;
      TV3<T> P = impulse * n;
      wa = wa - sym_mv(sa, cross(ra, P));
      va = va - ima * P;
      wb = wb + sym_mv(sb, cross(rb, P));
      vb = vb + imb * P;
    }
  }
  out3(y, 0, va); out3(y, 3, wa); out3(y, 6, vb); out3(y, 9, wb);
}

// The relative normal velocity prepare samples for restitution at one point (nsd_kernels.cuh
// prepare_constraint, contact_solver.rs:626-644): n . ((vB + wB x rB) - (vA + wA x rA)), from
// the bodies' velocities at the step's start, the manifold normal and the point's anchors.
enum RL : int { rlVA = 0, rlWA = 3, rlVB = 6, rlWB = 9, rlN = 12, rlRa = 15, rlRb = 18, kRL = 21 };
template <class T, class In>
NSD_HD void relvel_fn(const In& x, T* y) {
  TV3<T> vra = in3<T>(x, rlVA) + cross(in3<T>(x, rlWA), in3<T>(x, rlRa));
  TV3<T> vrb = in3<T>(x, rlVB) + cross(in3<T>(x, rlWB), in3<T>(x, rlRb));
  y[0] = dot(in3<T>(x, rlN), vrb - vra);
}
// Its reverse: xb += yb * d(relvel)/dx. With d = vrb - vra, the normal takes yb d; vA and vB
// take -/+ yb n; wA and wB take -/+ yb (r x n); rA and rB take -/+ yb (n x w).
template <class R>
NSD_HD void relvel_vjp(const R* x, R yb, R* xb) {
  PlainIn<R> in{x};
  TV3<R> va = in3<R>(in, rlVA), wa = in3<R>(in, rlWA), vb = in3<R>(in, rlVB), wb = in3<R>(in, rlWB);
  TV3<R> n = in3<R>(in, rlN), ra = in3<R>(in, rlRa), rb = in3<R>(in, rlRb);
  TV3<R> d = (vb + cross(wb, rb)) - (va + cross(wa, ra));
  TV3<R> gwa = cross(ra, n), gwb = cross(rb, n), gra = cross(n, wa), grb = cross(n, wb);
  R parts[kRL] = {-n.x, -n.y, -n.z, -gwa.x, -gwa.y, -gwa.z, n.x, n.y, n.z, gwb.x, gwb.y, gwb.z,
                  d.x, d.y, d.z, -gra.x, -gra.y, -gra.z, grb.x, grb.y, grb.z};
  for (int i = 0; i < kRL; ++i) xb[i] += yb * parts[i];
}

// ---------------------------------------------------------------------------------------------
// Hand-derived reverse sweeps of warm start, push and relax (one thread per constraint). Each
// takes the stage's inputs x (constraint vector layout) and the cotangents ybar of its outputs
// and adds the vector-Jacobian product into xbar (kCV entries, zeroed by the caller). They are
// the reverse-mode counterparts of warm_fn, push_fn and relax_fn above, which remain the
// reference they are checked against (ns_adjoint_selfcheck).

// Where a reverse sweep adds its cotangents: all of them, or (kAll false) only the two bodies'
// solver state and the constraint's impulses (entries below cvIma) -- what the next phase of
// the reverse solve needs; the constant entries' terms are then dead code.
template <class R, bool kAll>
struct Sink {
  R* p;
  NSD_HD void add(int i, R v) {
    if (kAll || i < cvIma) p[i] += v;
  }
};

// d(S a) for a symmetric S stored as xx xy xz yy yz zz: Sbar += ybar a^T (symmetrised by
// storage), abar += S ybar.
template <class R, class S>
NSD_HD void sym_mv_vjp(const TSym<R>& s, const TV3<R>& a, const TV3<R>& yb, S& xs, int at, TV3<R>& abar) {
  xs.add(at, yb.x * a.x);
  xs.add(at + 1, yb.x * a.y + yb.y * a.x);
  xs.add(at + 2, yb.x * a.z + yb.z * a.x);
  xs.add(at + 3, yb.y * a.y);
  xs.add(at + 4, yb.y * a.z + yb.z * a.y);
  xs.add(at + 5, yb.z * a.z);
  abar = abar + sym_mv(s, yb);
}
// c = a x b: abar += b x cbar, bbar += cbar x a
template <class R> NSD_HD void cross_vjp(const TV3<R>& a, const TV3<R>& b, const TV3<R>& cb, TV3<R>& abar, TV3<R>& bbar) {
  abar = abar + cross(b, cb);
  bbar = bbar + cross(cb, a);
}
// inv_rotate_wide(q, a) (nsd_types.cuh): out = (a - q.s t) + q.v x t, t = 2 q.v x a
template <class R, class S>
NSD_HD void irw_vjp(const TQ<R>& q, const TV3<R>& a, const TV3<R>& ob, S& xs, int at, TV3<R>& abar) {
  TV3<R> t0 = cross(q.v, a);
  TV3<R> t = tv3<R>(t0.x + t0.x, t0.y + t0.y, t0.z + t0.z);
  abar = abar + ob;
  xs.add(at + 3, -dot(t, ob));
  TV3<R> tb = R(-1) * (q.s * ob);
  TV3<R> qvb = tzero3<R>();
  cross_vjp(q.v, t, ob, qvb, tb);
  TV3<R> t0b = tb + tb;
  cross_vjp(q.v, a, t0b, qvb, abar);
  xs.add(at, qvb.x); xs.add(at + 1, qvb.y); xs.add(at + 2, qvb.z);
}
template <class R, class S> NSD_HD void add3(S& xs, int i, const TV3<R>& v) { xs.add(i, v.x); xs.add(i + 1, v.y); xs.add(i + 2, v.z); }
template <class R> NSD_HD TV3<R> ld3(const R* x, int i) { return tv3<R>(x[i], x[i + 1], x[i + 2]); }
template <class R> NSD_HD TSym<R> ldsym(const R* x, int i) {
  TSym<R> s = {x[i], x[i + 1], x[i + 2], x[i + 3], x[i + 4], x[i + 5]};
  return s;
}

template <class R, bool kAll = true>
NSD_HD void warm_vjp(const R* x, const CParams& cp, const R* yb, R* xbar_) {
  Sink<R, kAll> xbar{xbar_};
  TV3<R> t1 = ld3(x, cvT1), t2 = ld3(x, cvT2), ca = ld3(x, cvCa), cb = ld3(x, cvCb), n = ld3(x, cvN);
  R twist = x[cvTwist], fx = x[cvFr], fy = x[cvFr + 1], ima = x[cvIma], imb = x[cvImb];
  TSym<R> sa = ldsym(x, cvSa), sb = ldsym(x, cvSb);
  R tni = R(0);
  TV3<R> moa = tzero3<R>(), mob = tzero3<R>();
  for (int q = 0; q < cp.pc; ++q) {
    R ni = x[cvLam + q];
    tni = tni + ni;
    moa = mul_add(moa, ni, ld3(x, cv_point(q, 0)));
    mob = mul_add(mob, ni, ld3(x, cv_point(q, 3)));
  }
  TV3<R> fi = mul_add(fx * t1, fy, t2);
  TV3<R> lin = mul_add(fi, tni, n);
  TV3<R> twi = twist * n;
  TV3<R> anga = cross(moa, n) + cross(ca, fi) + twi;
  TV3<R> angb = cross(mob, n) + cross(cb, fi) + twi;
  // reverse (the velocities pass through)
  TV3<R> vab = ld3(yb, 0), wab = ld3(yb, 3), vbb = ld3(yb, 6), wbb = ld3(yb, 9);
  add3(xbar, cvVA, vab); add3(xbar, cvWA, wab); add3(xbar, cvVB, vbb); add3(xbar, cvWB, wbb);
  TV3<R> lib = R(-1) * (ima * vab) + imb * vbb;
  xbar.add(cvIma, -dot(lin, vab));
  xbar.add(cvImb, dot(lin, vbb));
  TV3<R> aiab = tzero3<R>(), aibb = tzero3<R>();
  sym_mv_vjp(sa, anga, R(-1) * wab, xbar, cvSa, aiab);
  sym_mv_vjp(sb, angb, wbb, xbar, cvSb, aibb);
  TV3<R> moab = tzero3<R>(), mobb = tzero3<R>(), nb = tzero3<R>(), cab = tzero3<R>(), cbb = tzero3<R>();
  TV3<R> fib = lib, twib = aiab + aibb;
  cross_vjp(moa, n, aiab, moab, nb);
  cross_vjp(ca, fi, aiab, cab, fib);
  cross_vjp(mob, n, aibb, mobb, nb);
  cross_vjp(cb, fi, aibb, cbb, fib);
  xbar.add(cvTwist, dot(n, twib));
  nb = nb + twist * twib;
  R tnib = dot(n, lib);
  nb = nb + tni * lib;
  xbar.add(cvFr, dot(t1, fib));
  xbar.add(cvFr + 1, dot(t2, fib));
  add3(xbar, cvT1, fx * fib);
  add3(xbar, cvT2, fy * fib);
  for (int q = 0; q < cp.pc; ++q) {
    R ni = x[cvLam + q];
    xbar.add(cvLam + q, dot(ld3(x, cv_point(q, 0)), moab) + dot(ld3(x, cv_point(q, 3)), mobb) + tnib);
    add3(xbar, cv_point(q, 0), ni * moab);
    add3(xbar, cv_point(q, 3), ni * mobb);
  }
  add3(xbar, cvN, nb); add3(xbar, cvCa, cab); add3(xbar, cvCb, cbb);
}

// Shared tail of push and relax: the reverse of the setup (the normal's rotation by the
// substep rotations, the relative displacement).
template <class R, class S>
NSD_HD void contact_setup_vjp(const R* x, const TV3<R>& n, R nsb, const TV3<R>& nab, const TV3<R>& nbb, S& xbar,
                              TV3<R>& nbar) {
  TQ<R> dqa = tquat<R>(ld3(x, cvDqA), x[cvDqA + 3]), dqb = tquat<R>(ld3(x, cvDqB), x[cvDqB + 3]);
  irw_vjp(dqa, n, nab, xbar, cvDqA, nbar);
  irw_vjp(dqb, n, nbb, xbar, cvDqB, nbar);
  TV3<R> dp = ld3(x, cvDpB) - ld3(x, cvDpA);
  nbar = nbar + nsb * dp;
  add3(xbar, cvDpB, nsb * n);
  add3(xbar, cvDpA, R(-1) * (nsb * n));
}

template <class R, bool kAll = true>
NSD_HD void push_vjp(const R* x, const CParams& cp, const R* yb, R* xbar_) {
  Sink<R, kAll> xbar{xbar_};
  const R inv_h = R(cp.inv_h), cs = R(-cp.contact_speed);
  const Softness& so = cp.is_static ? cp.static_softness : cp.contact_softness;
  const R br = R(so.mass_scale * so.bias_rate), ms = R(so.mass_scale), is = R(so.impulse_scale);
  TV3<R> va = ld3(x, cvVA), vb = ld3(x, cvVB), n = ld3(x, cvN);
  TQ<R> dqa = tquat<R>(ld3(x, cvDqA), x[cvDqA + 3]), dqb = tquat<R>(ld3(x, cvDqB), x[cvDqB + 3]);
  R ima = x[cvIma], imb = x[cvImb], im = ima + imb;
  TSym<R> sa = ldsym(x, cvSa), sb = ldsym(x, cvSb);
  TV3<R> dp = ld3(x, cvDpB) - ld3(x, cvDpA);
  R ns = dot(n, dp);
  TV3<R> na = inv_rotate_wide(dqa, n), nbv = inv_rotate_wide(dqb, n);
  // forward, keeping each point's values
  R lnv = dot(n, vb - va), mi = R(0);
  TV3<R> wa = ld3(x, cvWA), wb = ld3(x, cvWB);
  TV3<R> wa_q[4], wb_q[4], ua[4], ub[4], ga[4], gb[4];
  R imp[4], vn[4], vbias[4], pms[4], pis[4];
  bool sepq[4], selq[4], ovlq[4];
  for (int q = 0; q < cp.pc; ++q) {
    TV3<R> ra = ld3(x, cv_point(q, 0)), rb = ld3(x, cv_point(q, 3));
    R nimp = x[cvLam + q];
    R s = (ns + (dot(nbv, rb) - dot(na, ra))) + x[cv_point(q, 6)];
    bool sep = s > R(0);
    R ovl = tmax(br * s, cs);
    ovlq[q] = br * s > cs;
    vbias[q] = sep ? s * inv_h : ovl;
    pms[q] = sep ? R(1) : ms;
    pis[q] = sep ? R(0) : is;
    ua[q] = cross(ra, n); ub[q] = cross(rb, n);
    ga[q] = sym_mv(sa, ua[q]); gb[q] = sym_mv(sb, ub[q]);
    wa_q[q] = wa; wb_q[q] = wb;
    vn[q] = lnv + (dot(ub[q], wb) - dot(ua[q], wa));
    R neg = x[cv_point(q, 7)] * (pms[q] * vn[q] + vbias[q]) + pis[q] * nimp;
    selq[q] = -neg > -nimp;
    imp[q] = tmax(-neg, -nimp);
    lnv = lnv + im * imp[q];
    mi = mi + imp[q];
    wa = wa - imp[q] * ga[q];
    wb = wb + imp[q] * gb[q];
    sepq[q] = sep;
  }
  TV3<R> Pv = mi * n;
  // reverse
  TV3<R> vab = ld3(yb, 0), wab = ld3(yb, 3), vbb = ld3(yb, 6), wbb = ld3(yb, 9);
  add3(xbar, cvVA, vab); add3(xbar, cvVB, vbb);
  TV3<R> Pvb = R(-1) * (ima * vab) + imb * vbb;
  xbar.add(cvIma, -dot(Pv, vab));
  xbar.add(cvImb, dot(Pv, vbb));
  R mib = dot(n, Pvb);
  TV3<R> nbar = mi * Pvb;
  R lnvb = R(0), imb_ = R(0), nsb = R(0);
  TV3<R> nab = tzero3<R>(), nbb = tzero3<R>();
  for (int q = cp.pc - 1; q >= 0; --q) {
    TV3<R> ra = ld3(x, cv_point(q, 0)), rb = ld3(x, cv_point(q, 3));
    R nm = x[cv_point(q, 7)];
    R impb = -dot(ga[q], wab) + dot(gb[q], wbb) + mib + im * lnvb;
    TV3<R> gab = R(-1) * (imp[q] * wab), gbb = imp[q] * wbb;
    imb_ = imb_ + imp[q] * lnvb;
    R lamb = yb[12 + q];
    impb = impb + lamb;
    R nimpb = lamb;
    R negb = R(0);
    if (selq[q]) negb = -impb; else nimpb = nimpb - impb;
    xbar.add(cv_point(q, 7), (pms[q] * vn[q] + vbias[q]) * negb);
    R vnb = nm * pms[q] * negb, vbiasb = nm * negb;
    nimpb = nimpb + pis[q] * negb;
    R sb_ = R(0);
    if (sepq[q]) sb_ = inv_h * vbiasb; else if (ovlq[q]) sb_ = br * vbiasb;
    lnvb = lnvb + vnb;
    TV3<R> uab = R(-1) * (vnb * wa_q[q]), ubb = vnb * wb_q[q];
    wab = wab - vnb * ua[q];
    wbb = wbb + vnb * ub[q];
    sym_mv_vjp(sa, ua[q], gab, xbar, cvSa, uab);
    sym_mv_vjp(sb, ub[q], gbb, xbar, cvSb, ubb);
    TV3<R> rab = tzero3<R>(), rbb = tzero3<R>();
    cross_vjp(ra, n, uab, rab, nbar);
    cross_vjp(rb, n, ubb, rbb, nbar);
    nsb = nsb + sb_;
    nbb = nbb + sb_ * rb;
    rbb = rbb + sb_ * nbv;
    nab = nab - sb_ * ra;
    rab = rab - sb_ * na;
    xbar.add(cv_point(q, 6), sb_);
    add3(xbar, cv_point(q, 0), rab);
    add3(xbar, cv_point(q, 3), rbb);
    xbar.add(cvLam + q, nimpb);
  }
  for (int q = cp.pc; q < 4; ++q) xbar.add(cvLam + q, yb[12 + q]);
  add3(xbar, cvWA, wab); add3(xbar, cvWB, wbb);
  xbar.add(cvIma, imb_); xbar.add(cvImb, imb_);
  nbar = nbar + lnvb * (vb - va);
  add3(xbar, cvVB, lnvb * n);
  add3(xbar, cvVA, R(-1) * (lnvb * n));
  contact_setup_vjp(x, n, nsb, nab, nbb, xbar, nbar);
  add3(xbar, cvN, nbar);
}

template <class R, bool kAll = true>
NSD_HD void relax_vjp(const R* x, const CParams& cp, const R* yb, R* xbar_) {
  Sink<R, kAll> xbar{xbar_};
  const R inv_h = R(cp.inv_h), eps = R(kEps);
  TV3<R> va = ld3(x, cvVA), vb = ld3(x, cvVB), n = ld3(x, cvN), t1 = ld3(x, cvT1), t2 = ld3(x, cvT2);
  TV3<R> ca = ld3(x, cvCa), cb = ld3(x, cvCb);
  TQ<R> dqa = tquat<R>(ld3(x, cvDqA), x[cvDqA + 3]), dqb = tquat<R>(ld3(x, cvDqB), x[cvDqB + 3]);
  R ima = x[cvIma], imb = x[cvImb], im = ima + imb, mu = x[cvFriction];
  TSym<R> sa = ldsym(x, cvSa), sb = ldsym(x, cvSb);
  TV3<R> dp = ld3(x, cvDpB) - ld3(x, cvDpA);
  R ns = dot(n, dp);
  TV3<R> na = inv_rotate_wide(dqa, n), nbv = inv_rotate_wide(dqb, n);
  TV3<R> dv = vb - va;
  R lnv = dot(n, dv);
  R lt1 = dot(t1, dv) - x[cvTv1], lt2 = dot(t2, dv) - x[cvTv2];
  R mi = R(0), tni = R(0), ttl = R(0);
  TV3<R> wa = ld3(x, cvWA), wb = ld3(x, cvWB);
  TV3<R> wa_q[4], wb_q[4], ua[4], ub[4], ga[4], gb[4];
  R imp[4], vn[4], vbias[4], ni[4];
  bool selq[4], actq[4];
  for (int q = 0; q < cp.pc; ++q) {
    TV3<R> ra = ld3(x, cv_point(q, 0)), rb = ld3(x, cv_point(q, 3));
    R s = (ns + (dot(nbv, rb) - dot(na, ra))) + x[cv_point(q, 6)];
    actq[q] = !(R(0) > s * inv_h);
    vbias[q] = tmax(R(0), s * inv_h);
    ua[q] = cross(ra, n); ub[q] = cross(rb, n);
    ga[q] = sym_mv(sa, ua[q]); gb[q] = sym_mv(sb, ub[q]);
    wa_q[q] = wa; wb_q[q] = wb;
    vn[q] = lnv + (dot(ub[q], wb) - dot(ua[q], wa));
    R neg = x[cv_point(q, 7)] * (vn[q] + vbias[q]);
    R old = x[cvLam + q];
    selq[q] = -neg > -old;
    imp[q] = tmax(-neg, -old);
    ni[q] = old + imp[q];
    tni = tni + ni[q];
    ttl = ttl + x[cv_point(q, 8)] * ni[q];
    lnv = lnv + im * imp[q];
    mi = mi + imp[q];
    wa = wa - imp[q] * ga[q];
    wb = wb + imp[q] * gb[q];
  }
  // twist
  TV3<R> wa_p = wa, wb_p = wb;
  R ts = dot(n, wb - wa);
  R ml = mu * ttl, oldt = x[cvTwist], tmw = x[cvTwistMass];
  R it0 = -(tmw * ts);
  bool sel_in = it0 < ml - oldt;
  R inner = sel_in ? it0 : ml - oldt;
  bool sel_out = -ml - oldt > inner;
  R it = sel_out ? -ml - oldt : inner;
  TV3<R> gna = sym_mv(sa, n), gnb = sym_mv(sb, n);
  TV3<R> wa_t = wa_p - it * gna, wb_t = wb_p + it * gnb;
  // friction
  R cxx = x[cvTm], cxy = x[cvTm + 1], cyx = x[cvTm + 2], cyy = x[cvTm + 3];
  TV3<R> arv = cross(wb_t, cb) - cross(wa_t, ca);
  R vtx = lt1 + dot(arv, t1), vty = lt2 + dot(arv, t2);
  R d0x = cxx * vtx + cyx * vty, d0y = cxy * vtx + cyy * vty;
  R fx = x[cvFr], fy = x[cvFr + 1];
  R nx = fx + (-d0x), ny = fy + (-d0y);
  R mx = mu * tni;
  R lsq = nx * nx + ny * ny;
  bool mask = lsq > mx * mx;
  R root = tsqrt(lsq);
  R den = root + eps;
  R nrm = mx / den;
  R sc = mask ? nrm : R(1);
  R nxs = sc * nx, nys = sc * ny;
  R dix = nxs - fx, diy = nys - fy;
  TV3<R> Pv = dix * t1 + diy * t2;
  TV3<R> Pv2 = Pv + mi * n;
  // ---- reverse
  TV3<R> vab = ld3(yb, 0), wab = ld3(yb, 3), vbb = ld3(yb, 6), wbb = ld3(yb, 9);
  R frxb = yb[16], fryb = yb[17], twb = yb[18];
  TV3<R> nbar = tzero3<R>(), t1b = tzero3<R>(), t2b = tzero3<R>(), cab = tzero3<R>(), cbb = tzero3<R>();
  add3(xbar, cvVA, vab); add3(xbar, cvVB, vbb);
  TV3<R> Pv2b = R(-1) * (ima * vab) + imb * vbb;
  xbar.add(cvIma, -dot(Pv2, vab));
  xbar.add(cvImb, dot(Pv2, vbb));
  TV3<R> Pvb = Pv2b;
  R mib = dot(n, Pv2b);
  nbar = nbar + mi * Pv2b;
  {  // wB_F = wB_T + Sb (cb x Pv), wA_F = wA_T - Sa (ca x Pv)
    TV3<R> u = cross(cb, Pv), ubar = tzero3<R>();
    sym_mv_vjp(sb, u, wbb, xbar, cvSb, ubar);
    cross_vjp(cb, Pv, ubar, cbb, Pvb);
    TV3<R> u2 = cross(ca, Pv), u2bar = tzero3<R>();
    sym_mv_vjp(sa, u2, R(-1) * wab, xbar, cvSa, u2bar);
    cross_vjp(ca, Pv, u2bar, cab, Pvb);
  }
  R dixb = dot(t1, Pvb), diyb = dot(t2, Pvb);
  t1b = t1b + dix * Pvb;
  t2b = t2b + diy * Pvb;
  R nxsb = frxb + dixb, nysb = fryb + diyb;
  R fxb = -dixb, fyb = -diyb;
  R scb = nx * nxsb + ny * nysb;
  R nxb = sc * nxsb, nyb = sc * nysb;
  R mxb = R(0), tnib = R(0), ttlb = R(0);
  if (mask) {
    R nrmb = scb;
    mxb = mxb + nrmb / den;
    R denb = -nrmb * mx / (den * den);
    R lsqb = root > R(0) ? denb * R(0.5) / root : R(0);
    nxb = nxb + R(2) * nx * lsqb;
    nyb = nyb + R(2) * ny * lsqb;
  }
  xbar.add(cvFriction, tni * mxb);
  tnib = tnib + mu * mxb;
  fxb = fxb + nxb; fyb = fyb + nyb;
  R d0xb = -nxb, d0yb = -nyb;
  xbar.add(cvTm, d0xb * vtx); xbar.add(cvTm + 2, d0xb * vty);
  xbar.add(cvTm + 1, d0yb * vtx); xbar.add(cvTm + 3, d0yb * vty);
  R vtxb = cxx * d0xb + cxy * d0yb, vtyb = cyx * d0xb + cyy * d0yb;
  R lt1b = vtxb, lt2b = vtyb;
  TV3<R> arvb = vtxb * t1 + vtyb * t2;
  t1b = t1b + vtxb * arv;
  t2b = t2b + vtyb * arv;
  TV3<R> wbtb = wbb, watb = wab;
  cross_vjp(wb_t, cb, arvb, wbtb, cbb);
  cross_vjp(wa_t, ca, R(-1) * arvb, watb, cab);
  // twist: wA_T = wA_P - it gna, wB_T = wB_P + it gnb
  R itb = -dot(gna, watb) + dot(gnb, wbtb) + twb;
  TV3<R> gnab = R(-1) * (it * watb), gnbb = it * wbtb;
  sym_mv_vjp(sa, n, gnab, xbar, cvSa, nbar);
  sym_mv_vjp(sb, n, gnbb, xbar, cvSb, nbar);
  R oldtb = twb, mlb = R(0), innerb = R(0);
  if (sel_out) { mlb = mlb - itb; oldtb = oldtb - itb; } else innerb = itb;
  R it0b = R(0);
  if (sel_in) it0b = innerb; else { mlb = mlb + innerb; oldtb = oldtb - innerb; }
  xbar.add(cvTwistMass, -ts * it0b);
  R tsb = -tmw * it0b;
  xbar.add(cvFriction, ttl * mlb);
  ttlb = ttlb + mu * mlb;
  xbar.add(cvTwist, oldtb);
  nbar = nbar + tsb * (wb_p - wa_p);
  wbb = wbtb + tsb * n;
  wab = watb - tsb * n;
  // points, last to first
  R lnvb = R(0), imb_ = R(0), nsb = R(0);
  TV3<R> nab = tzero3<R>(), nbb = tzero3<R>();
  for (int q = cp.pc - 1; q >= 0; --q) {
    TV3<R> ra = ld3(x, cv_point(q, 0)), rb = ld3(x, cv_point(q, 3));
    R nm = x[cv_point(q, 7)], lev = x[cv_point(q, 8)];
    R impb = -dot(ga[q], wab) + dot(gb[q], wbb) + mib + im * lnvb;
    TV3<R> gab = R(-1) * (imp[q] * wab), gbb = imp[q] * wbb;
    imb_ = imb_ + imp[q] * lnvb;
    xbar.add(cv_point(q, 8), ni[q] * ttlb);
    R nib = lev * ttlb + tnib + yb[12 + q];
    R oldb = nib;
    impb = impb + nib;
    R negb = R(0);
    if (selq[q]) negb = -impb; else oldb = oldb - impb;
    xbar.add(cv_point(q, 7), (vn[q] + vbias[q]) * negb);
    R vnb = nm * negb, vbiasb = nm * negb;
    R sb_ = actq[q] ? inv_h * vbiasb : R(0);
    lnvb = lnvb + vnb;
    TV3<R> uab = R(-1) * (vnb * wa_q[q]), ubb = vnb * wb_q[q];
    wab = wab - vnb * ua[q];
    wbb = wbb + vnb * ub[q];
    sym_mv_vjp(sa, ua[q], gab, xbar, cvSa, uab);
    sym_mv_vjp(sb, ub[q], gbb, xbar, cvSb, ubb);
    TV3<R> rab = tzero3<R>(), rbb = tzero3<R>();
    cross_vjp(ra, n, uab, rab, nbar);
    cross_vjp(rb, n, ubb, rbb, nbar);
    nsb = nsb + sb_;
    nbb = nbb + sb_ * rb;
    rbb = rbb + sb_ * nbv;
    nab = nab - sb_ * ra;
    rab = rab - sb_ * na;
    xbar.add(cv_point(q, 6), sb_);
    add3(xbar, cv_point(q, 0), rab);
    add3(xbar, cv_point(q, 3), rbb);
    xbar.add(cvLam + q, oldb);
  }
  for (int q = cp.pc; q < 4; ++q) xbar.add(cvLam + q, yb[12 + q]);
  add3(xbar, cvWA, wab); add3(xbar, cvWB, wbb);
  xbar.add(cvIma, imb_); xbar.add(cvImb, imb_);
  xbar.add(cvFr, fxb); xbar.add(cvFr + 1, fyb);
  // setup: lnv = n . dv, lt = t . dv - tv, dv = vB - vA
  TV3<R> dvb = lnvb * n + lt1b * t1 + lt2b * t2;
  nbar = nbar + lnvb * dv;
  t1b = t1b + lt1b * dv;
  t2b = t2b + lt2b * dv;
  xbar.add(cvTv1, -lt1b);
  xbar.add(cvTv2, -lt2b);
  add3(xbar, cvVB, dvb);
  add3(xbar, cvVA, R(-1) * dvb);
  contact_setup_vjp(x, n, nsb, nab, nbb, xbar, nbar);
  add3(xbar, cvN, nbar);
  add3(xbar, cvT1, t1b); add3(xbar, cvT2, t2b);
  add3(xbar, cvCa, cab); add3(xbar, cvCb, cbb);
}

// ---------------------------------------------------------------------------------------------
// Prepare (nsd_kernels.cuh prepare_constraint; contact_solver.rs:445): manifold and body mass
// data -> the constraint's own entries of the constraint vector (outputs cvLam..kCV-1).
enum PI : int {
  piN = 0, piPoint = 3,  // + 8 q: anchor_a 0..2, anchor_b 3..5, separation 6, normal impulse 7
  piFrictionImpulse = 35, piTwist = 38, piIma = 39, piImb = 40, piSa = 41, piSb = 47, piFriction = 53,
  kPI = 54,
};
NSD_HD int pi_point(int q, int f) { return piPoint + 8 * q + f; }
struct PParams {
  int pc, is_static;
  float warm_start;
};
template <class T, class In>
NSD_HD void prepare_fn(const In& x, const PParams& pp, T* y /* kCVOwn, index - cvLam */) {
  auto Y = [&](int cv) -> T& { return y[cv - cvLam]; };
  auto Y3 = [&](int cv, const TV3<T>& a) { Y(cv) = a.x; Y(cv + 1) = a.y; Y(cv + 2) = a.z; };
  const T inv_tau = T(1.0f / speculative_distance());
  const T ws = T(pp.warm_start);
  T ima = x(piIma), imb = x(piImb);
  TSym<T> sa = in_sym<T>(x, piSa), sb = in_sym<T>(x, piSb);
  TSym<T> inv_iab = sym_add(sa, sb);
  TV3<T> n = in3<T>(x, piN);
  TV3<T> t1 = perp(n);
  TV3<T> t2 = cross(t1, n);
  TV3<T> tvel = tzero3<T>();
  T tv1 = dot(tvel, t1), tv2 = dot(tvel, t2);
  T twist = ws * x(piTwist);
  TV3<T> fimp = in3<T>(x, piFrictionImpulse);
  T fix = ws * dot(fimp, t1), fiy = ws * dot(fimp, t2);
  TV3<T> ca = tzero3<T>(), cb = tzero3<T>();
  T tw = T(0.0f);
  TV3<T> ra_[4];
  for (int i = 0; i < 4; ++i) {
    for (int f = 0; f < 9; ++f) Y(cv_point(i, f)) = T(0.0f);
    Y(cvLam + i) = T(0.0f);
  }
  for (int i = 0; i < pp.pc; ++i) {
    TV3<T> ra = in3<T>(x, pi_point(i, 0)), rb = in3<T>(x, pi_point(i, 3));
    T sep = x(pi_point(i, 6));
    ra_[i] = ra;
    T base_sep = sep - dot(rb - ra, n);
    T weight = tclamp(T(2.0f) - sep * inv_tau, T(kMinFrictionWeight), T(1.0f));
    ca = ca + weight * ra;
    cb = cb + weight * rb;
    tw = tw + weight;
    TV3<T> rna = cross(ra, n), rnb = cross(rb, n);
    T k = ima + imb;
    k = k + dot(rna, sym_mv(sa, rna));
    k = k + dot(rnb, sym_mv(sb, rnb));
    T nm = k > T(0.0f) ? T(1.0f) / k : T(0.0f);
    Y3(cv_point(i, 0), ra);
    Y(cv_point(i, 6)) = base_sep;
    Y3(cv_point(i, 3), rb);
    Y(cv_point(i, 7)) = nm;
  }
  if (tw > T(0.0f)) {
    ca = (T(1.0f) / tw) * ca;
    cb = (T(1.0f) / tw) * cb;
  } else {
    ca = tzero3<T>(); cb = tzero3<T>();
  }
  for (int i = 0; i < pp.pc; ++i) {
    TV3<T> d = ra_[i] - ca;
    Y(cv_point(i, 8)) = tsqrt(dot(d, d));
    Y(cvLam + i) = ws * x(pi_point(i, 7));
  }
  TV3<T> rta1 = cross(ca, t1), rta2 = cross(ca, t2), rtb1 = cross(cb, t1), rtb2 = cross(cb, t2);
  TV3<T> ia1 = sym_mv(sa, rta1), ia2 = sym_mv(sa, rta2), ib1 = sym_mv(sb, rtb1), ib2 = sym_mv(sb, rtb2);
  T msum = ima + imb;
  T kxx = (msum + dot(rta1, ia1)) + dot(rtb1, ib1);
  T kyy = (msum + dot(rta2, ia2)) + dot(rtb2, ib2);
  T kxy = dot(rta1, ia2) + dot(rtb1, ib2);
  T det2 = kxx * kyy - kxy * kxy;
  bool valid = tabs(det2) > T(1000.0f * kMinPositive) && tw > T(0.0f);
  T inv = valid ? T(1.0f) / det2 : T(0.0f);
  T ktw = dot(n, sym_mv(inv_iab, n));
  T twist_mass = ktw > T(0.0f) ? T(1.0f) / ktw : T(0.0f);
  Y(cvIma) = ima; Y(cvImb) = imb;
  Y(cvSa) = sa.xx; Y(cvSa + 1) = sa.xy; Y(cvSa + 2) = sa.xz; Y(cvSa + 3) = sa.yy; Y(cvSa + 4) = sa.yz; Y(cvSa + 5) = sa.zz;
  Y(cvSb) = sb.xx; Y(cvSb + 1) = sb.xy; Y(cvSb + 2) = sb.xz; Y(cvSb + 3) = sb.yy; Y(cvSb + 4) = sb.yz; Y(cvSb + 5) = sb.zz;
  Y(cvFriction) = x(piFriction);
  Y3(cvN, n);
  Y3(cvT1, t1); Y(cvTv1) = tv1;
  Y3(cvT2, t2); Y(cvTv2) = tv2;
  Y3(cvCa, ca); Y(cvTwistMass) = twist_mass;
  Y3(cvCb, cb); Y(cvTwist) = twist;
  Y(cvTm) = inv * kyy; Y(cvTm + 1) = -(inv * kxy); Y(cvTm + 2) = -(inv * kxy); Y(cvTm + 3) = inv * kxx;
  Y(cvFr) = fix; Y(cvFr + 1) = fiy;
}

// ---------------------------------------------------------------------------------------------
// Body stages.
struct BParams {
  float h, inv_dt, max_linear_speed;
  float lin_damp, ang_damp, grav_scale;
  uint32_t flags;
  V3 gravity;
};
template <class T> NSD_HD T det(const TM3<T>& m) { return dot(m.cx, cross(m.cy, m.cz)); }
template <class T> NSD_HD TV3<T> solve3(const TM3<T>& m, const TV3<T>& a) {
  T d = det(m);
  if (tabs(d) > T(1000.0f * kMinPositive)) {
    T inv_d = T(1.0f) / d;
    TV3<T> sx = cross(m.cy, m.cz), sy = cross(m.cz, m.cx), sz = cross(m.cx, m.cy);
    return tv3<T>(inv_d * dot(sx, a), inv_d * dot(sy, a), inv_d * dot(sz, a));
  }
  return tzero3<T>();
}

// integrate velocities (nsd_solve.cuh apply_iv, solver_integration.rs:263) with the implicit
// gyroscopic step of bodies flagged kGyroscopic.
// Inputs: v 0..2, w 3..5, inv_mass 6, inverse world inertia 7..15 (cx, cy, cz), force 16..18,
// torque 19..21, rotation 22..25, substep rotation dq 26..29, local inertia 30..38 (cx, cy, cz).
// Outputs: v, w.
constexpr int kIVIn = 39, kIVOut = 6;
template <class T, class In>
NSD_HD void iv_fn(const In& x, const BParams& bp, T* y) {
  T h = T(bp.h);
  TV3<T> v = in3<T>(x, 0), wv = in3<T>(x, 3);
  T inv_mass = x(6);
  TM3<T> iiw = tm3<T>(in3<T>(x, 7), in3<T>(x, 10), in3<T>(x, 13));
  TV3<T> force = in3<T>(x, 16), torque = in3<T>(x, 19);
  T ld = T(1.0f) / (T(1.0f) + h * T(bp.lin_damp));
  T ad = T(1.0f) / (T(1.0f) + h * T(bp.ang_damp));
  T gs = inv_mass > T(0.0f) ? T(bp.grav_scale) : T(0.0f);
  TV3<T> lvd = blend2(h * inv_mass, force, h * gs, tv3<T>(bp.gravity));
  v = mul_add(lvd, ld, v);
  TV3<T> avd = h * mul_mv(iiw, torque);
  wv = mul_add(avd, ad, wv);
  if (bp.flags & kGyroscopic) {
    TQ<T> q = mul_quat(in4<T>(x, 26), in4<T>(x, 22));
    TV3<T> om1 = inv_rotate(q, wv);
    TV3<T> om2 = om1;
    T i00 = x(30), i01 = x(33), i02 = x(36);
    T i11 = x(34), i12 = x(37), i22 = x(38);
    T w1 = om2.x, w2 = om2.y, w3 = om2.z;
    T iw1 = i00 * w1 + i01 * w2 + i02 * w3;
    T iw2 = i01 * w1 + i11 * w2 + i12 * w3;
    T iw3 = i02 * w1 + i12 * w2 + i22 * w3;
    TV3<T> dw = om2 - om1;
    TV3<T> b = tv3<T>(i00 * dw.x + i01 * dw.y + i02 * dw.z + h * (w2 * iw3 - w3 * iw2),
                      i01 * dw.x + i11 * dw.y + i12 * dw.z + h * (w3 * iw1 - w1 * iw3),
                      i02 * dw.x + i12 * dw.y + i22 * dw.z + h * (w1 * iw2 - w2 * iw1));
    TM3<T> J = tm3<T>(tv3<T>(i00 + h * (w2 * i02 - w3 * i01), i01 + h * (w3 * i00 - w1 * i02 - iw3),
                             i02 + h * (w1 * i01 - w2 * i00 + iw2)),
                      tv3<T>(i01 + h * (w2 * i12 - w3 * i11 + iw3), i11 + h * (w3 * i01 - w1 * i12),
                             i12 + h * (w1 * i11 - w2 * i01 - iw1)),
                      tv3<T>(i02 + h * (w2 * i22 - w3 * i12 - iw2), i12 + h * (w3 * i02 - w1 * i22 + iw1),
                             i22 + h * (w1 * i12 - w2 * i02)));
    om2 = om2 - solve3(J, b);
    wv = rotate(q, om2);
  }
  out3(y, 0, v); out3(y, 3, wv);
}
// integrate positions (nsd_solve.cuh apply_ip, solver_integration.rs:377).
// Inputs and outputs: v 0..2, w 3..5, dp 6..8, dq 9..12.
constexpr int kIP = 13;
template <class T, class In>
NSD_HD void ip_fn(const In& x, const BParams& bp, T* y) {
  uint32_t flags = bp.flags;
  T maxl = T(bp.max_linear_speed);
  T maxa = T(kMaxRotation * bp.inv_dt);
  T maxl2 = maxl * maxl, maxa2 = maxa * maxa;
  TV3<T> v = in3<T>(x, 0), wv = in3<T>(x, 3);
  v.x = (flags & kLockLinX) ? T(0.0f) : v.x;
  v.y = (flags & kLockLinY) ? T(0.0f) : v.y;
  v.z = (flags & kLockLinZ) ? T(0.0f) : v.z;
  wv.x = (flags & kLockAngX) ? T(0.0f) : wv.x;
  wv.y = (flags & kLockAngY) ? T(0.0f) : wv.y;
  wv.z = (flags & kLockAngZ) ? T(0.0f) : wv.z;
  if (dot(v, v) > maxl2) {
    T ratio = maxl / length(v);
    v = ratio * v;
  }
  if (dot(wv, wv) > maxa2 && (flags & kAllowFastRotation) == 0) {
    T ratio = maxa / length(wv);
    wv = ratio * wv;
  }
  TV3<T> dp = mul_add(in3<T>(x, 6), T(bp.h), v);
  TQ<T> dq = integrate_rotation(in4<T>(x, 9), T(bp.h) * wv);
  out3(y, 0, v); out3(y, 3, wv); out3(y, 6, dp); out4(y, 9, dq);
}
// finalize rotation (nsd_solve.cuh k_finalize, solver_integration.rs:587): q' = normalize(dq q).
// Inputs: q 0..3, dq 4..7. Outputs: q'.
template <class T, class In>
NSD_HD void final_rot_fn(const In& x, T* y) {
  out4(y, 0, normalize_quat(mul_quat(in4<T>(x, 4), in4<T>(x, 0))));
}
// inverse world inertia R I^-1 R^T of finalize. Inputs: q 0..3, local inverse inertia 4..12
// (cx, cy, cz). Outputs: the world matrix (cx, cy, cz).
template <class T, class In>
NSD_HD void inv_inertia_fn(const In& x, T* y) {
  TM3<T> R = matrix_from_quat(in4<T>(x, 0));
  TM3<T> il = tm3<T>(in3<T>(x, 4), in3<T>(x, 7), in3<T>(x, 10));
  TM3<T> m = mul_mm(mul_mm(R, il), transpose(R));
  out3(y, 0, m.cx); out3(y, 3, m.cy); out3(y, 6, m.cz);
}

// Hand-derived reverse of integrate positions (ip_fn): x, ybar and xbar in its 13-entry layout.
template <class R>
NSD_HD void ip_vjp(const R* x, const BParams& bp, const R* yb, R* xbar_) {
  Sink<R, true> xbar{xbar_};
  uint32_t flags = bp.flags;
  const R h = R(bp.h), maxl = R(bp.max_linear_speed), maxa = R(kMaxRotation * bp.inv_dt);
  TV3<R> v = ld3(x, 0), wv = ld3(x, 3);
  v.x = (flags & kLockLinX) ? R(0) : v.x;
  v.y = (flags & kLockLinY) ? R(0) : v.y;
  v.z = (flags & kLockLinZ) ? R(0) : v.z;
  wv.x = (flags & kLockAngX) ? R(0) : wv.x;
  wv.y = (flags & kLockAngY) ? R(0) : wv.y;
  wv.z = (flags & kLockAngZ) ? R(0) : wv.z;
  bool capv = dot(v, v) > maxl * maxl;
  R lv = length(v);
  bool capw = dot(wv, wv) > maxa * maxa && (flags & kAllowFastRotation) == 0;
  R lw = length(wv);
  TV3<R> wc = capw ? (maxa / lw) * wv : wv;
  TQ<R> q1 = tquat<R>(ld3(x, 9), x[12]);
  TV3<R> pv = R(0.5) * (h * wc);
  TQ<R> qd = mul_quat(tquat<R>(pv, R(0)), q1);
  TQ<R> qs = tquat<R>(q1.v + qd.v, qd.s + q1.s);
  // dq' = normalize(qs)
  TQ<R> qsb = tquat<R>(tzero3<R>(), R(0));
  R ls = dot_quat(qs, qs);
  TQ<R> qob = tquat<R>(ld3(yb, 9), yb[12]);
  if (ls > R(1000.0f * kMinPositive)) {
    R inv = R(1) / tsqrt(ls);
    TQ<R> qh = tquat<R>(inv * qs.v, inv * qs.s);
    R d = dot_quat(qh, qob);
    qsb = tquat<R>(inv * (qob.v - d * qh.v), inv * (qob.s - d * qh.s));
  }
  // qd = p (x) q1 with p = (pv, 0): v = pv x q1.v + q1.s pv, s = -pv . q1.v
  TV3<R> pvb = cross(q1.v, qsb.v) + q1.s * qsb.v - qsb.s * q1.v;
  TV3<R> q1vb = qsb.v + cross(qsb.v, pv) - qsb.s * pv;
  R q1sb = qsb.s + dot(pv, qsb.v);
  TV3<R> wcb = ld3(yb, 3) + (R(0.5) * h) * pvb;
  TV3<R> vcb = ld3(yb, 0) + h * ld3(yb, 6);
  add3(xbar, 6, ld3(yb, 6));
  xbar.add(9, q1vb.x); xbar.add(10, q1vb.y); xbar.add(11, q1vb.z); xbar.add(12, q1sb);
  if (capv) {
    TV3<R> vh = (R(1) / lv) * v;
    vcb = (maxl / lv) * (vcb - dot(vh, vcb) * vh);
  }
  if (capw) {
    TV3<R> wh = (R(1) / lw) * wv;
    wcb = (maxa / lw) * (wcb - dot(wh, wcb) * wh);
  }
  xbar.add(0, (flags & kLockLinX) ? R(0) : vcb.x);
  xbar.add(1, (flags & kLockLinY) ? R(0) : vcb.y);
  xbar.add(2, (flags & kLockLinZ) ? R(0) : vcb.z);
  xbar.add(3, (flags & kLockAngX) ? R(0) : wcb.x);
  xbar.add(4, (flags & kLockAngY) ? R(0) : wcb.y);
  xbar.add(5, (flags & kLockAngZ) ? R(0) : wcb.z);
}
// Hand-derived reverse of integrate velocities without the gyroscopic step (iv_fn):
// v' = (h m^-1 F + h gs g) + ld v, w' = h (I^-1 tau) + ad w.
template <class R>
NSD_HD void iv_vjp_plain(const R* x, const BParams& bp, const R* yb, R* xbar_) {
  Sink<R, true> xbar{xbar_};
  const R h = R(bp.h);
  R ld = R(1) / (R(1) + h * R(bp.lin_damp));
  R ad = R(1) / (R(1) + h * R(bp.ang_damp));
  TV3<R> vb = ld3(yb, 0), wb = ld3(yb, 3);
  add3(xbar, 0, ld * vb);
  add3(xbar, 3, ad * wb);
  xbar.add(6, h * dot(ld3(x, 16), vb));
  for (int c = 0; c < 3; ++c) {
    R tau = x[19 + c];
    xbar.add(7 + 3 * c, h * wb.x * tau);
    xbar.add(7 + 3 * c + 1, h * wb.y * tau);
    xbar.add(7 + 3 * c + 2, h * wb.z * tau);
  }
}

// ---------------------------------------------------------------------------------------------
// Contact recycling (nsd_kernels.cuh collide_recycle; collide_pass.rs:606-687): the new
// separations of a recycled manifold. Inputs: tangents of centre A 0..2 and B 3..5 (the
// centres' values are f64 and passed apart), qa 6..9, qb 10..13, cached rotation A 14..17 and
// B 18..21, normal 22..24, per point q: 25 + 7 q + {anchor_a 0..2, anchor_b 3..5, base
// separation 6}. Outputs: the separations (point_count).
enum RI : int { riCa = 0, riCb = 3, riQa = 6, riQb = 10, riRotA = 14, riRotB = 18, riN = 22, riPoint = 25, kRI = 53 };
NSD_HD int ri_point(int q, int f) { return riPoint + 7 * q + f; }
template <class T, class In>
NSD_HD void recycle_fn(const In& x, const Pos& ca, const Pos& cb, int pc, T* y) {
  TQ<T> qa = in4<T>(x, riQa), qb = in4<T>(x, riQb);
  TQ<T> dqa = mul_quat(qa, conjugate(in4<T>(x, riRotA)));
  TQ<T> dqb = mul_quat(qb, conjugate(in4<T>(x, riRotB)));
  TM3<T> ma = matrix_from_quat(dqa), mb = matrix_from_quat(dqb);
  TV3<T> dc = sub_pos_t(cb, ca, in3<T>(x, riCb), in3<T>(x, riCa));
  TV3<T> n = in3<T>(x, riN);
  for (int i = 0; i < pc; ++i) {
    TV3<T> ra = mul_mv(ma, in3<T>(x, ri_point(i, 0)));
    TV3<T> rb = mul_mv(mb, in3<T>(x, ri_point(i, 3)));
    TV3<T> dp = dc + (rb - ra);
    y[i] = x(ri_point(i, 6)) + dot(dp, n);
  }
}

// ---------------------------------------------------------------------------------------------
// Box-box manifolds (nsd_geom.cuh collide_hulls and its builders, convex_manifold.rs), replayed
// along the branch the forward step took: the SAT cache after the narrowphase names the axis
// kind and features, and every comparison inside the builders is taken on the value parts.
template <class T> struct TClipVertex { TV3<T> position; T separation; FeaturePair pair; };
template <class T> struct TLocalPoint { TV3<T> point; T separation; FeaturePair pair; };
template <class T> struct TLocalManifold { TV3<T> normal; TLocalPoint<T> points[4]; int point_count; };

template <class T>
NSD_HD int t_build_polygon(TClipVertex<T>* out, const TXf<T>& t, const Hull& h, int inc_face, const TPlane<T>& ref) {
  int ei = box_face_edge(inc_face);
  int n = 0;
  TM3<T> m = matrix_from_quat(t.q);
  for (;;) {
    HalfEdge e = box_edge(ei);
    int ni = e.next;
    HalfEdge nx = box_edge(ni);
    TClipVertex<T> v;
    v.position = mul_mv(m, tv3<T>(h.points[nx.origin])) + t.p;
    v.separation = plane_sep(ref, v.position);
    v.pair = make_feature_pair(1, ei, 1, ni);
    out[n++] = v;
    ei = ni;
    if (ei == box_face_edge(inc_face) || n >= kClipCap) break;
  }
  return n;
}
template <class T>
NSD_HD int t_clip_polygon(TClipVertex<T>* out, const TClipVertex<T>* poly, int count, const TPlane<T>& clip, int edge,
                          const TPlane<T>& ref) {
  TClipVertex<T> v1 = poly[count - 1];
  T d1 = plane_sep(clip, v1.position);
  int n = 0;
  for (int i = 0; i < count; ++i) {
    TClipVertex<T> v2 = poly[i];
    T d2 = plane_sep(clip, v2.position);
    if (d1 <= T(0.0f) && d2 <= T(0.0f)) {
      if (n < kClipCap) out[n] = v2;
      n++;
    } else if (d1 <= T(0.0f) && d2 > T(0.0f)) {
      T f = d1 / (d1 - d2);
      TV3<T> pos = mul_add(v1.position, f, v2.position - v1.position);
      TClipVertex<T> v;
      v.position = pos; v.separation = plane_sep(ref, pos); v.pair = v2.pair;
      v.pair.owner2 = 0; v.pair.index2 = (uint8_t)edge;
      if (n < kClipCap) out[n] = v;
      n++;
    } else if (d2 <= T(0.0f) && d1 > T(0.0f)) {
      T f = d1 / (d1 - d2);
      TV3<T> pos = mul_add(v1.position, f, v2.position - v1.position);
      TClipVertex<T> v;
      v.position = pos; v.separation = plane_sep(ref, pos); v.pair = v1.pair;
      v.pair.owner1 = 0; v.pair.index1 = (uint8_t)edge;
      if (n < kClipCap) out[n] = v;
      n++;
      if (n < kClipCap) out[n] = v2;
      n++;
    }
    v1 = v2; d1 = d2;
  }
  return n < kClipCap ? n : kClipCap;
}
template <class T>
NSD_HD void t_reduce_manifold_points(TLocalManifold<T>* m, TLocalPoint<T>* pts, int count) {
  if (count <= 4) {
    for (int i = 0; i < count; ++i) m->points[i] = pts[i];
    m->point_count = count;
    return;
  }
  TV3<T> normal = m->normal;
  T spec = T(speculative_distance());
  T tol_sqr = spec * spec;
  const T bias(0.95f);
  int best = kNull;
  T best_score = T(-kFltMax);
  // the normal is the reference face's plane normal, a constant of the hull
  TV3<T> sd = tv3<T>(arbitrary_perp(real3(normal)));
  for (int i = 0; i < count; ++i) {
    if (pts[i].separation > spec) continue;
    T score = -pts[i].separation + dot(sd, pts[i].point);
    if (bias * score > best_score) { best = i; best_score = score; }
  }
  if (best == kNull) { m->point_count = 0; return; }
  m->points[0] = pts[best];
  m->point_count = 1;
  pts[best] = pts[count - 1];
  count--;
  TV3<T> a = m->points[0].point;
  best_score = T(0.0f); best = kNull;
  for (int i = 0; i < count; ++i) {
    TV3<T> d = pts[i].point - a;
    TV3<T> v = mul_sub(d, dot(d, normal), normal);
    T dsq = length_sq(v);
    T sep = tmax(T(0.0f), -pts[i].separation);
    T score = dsq + T(4.0f) * sep * sep;
    if (bias * score > best_score) { best_score = score; best = i; }
  }
  if (best_score < tol_sqr) return;
  m->points[1] = pts[best];
  m->point_count = 2;
  pts[best] = pts[count - 1];
  count--;
  TV3<T> b = m->points[1].point;
  best_score = tol_sqr; best = kNull;
  T best_signed = T(0.0f);
  TV3<T> ba = b - a;
  for (int i = 0; i < count; ++i) {
    TV3<T> p = pts[i].point;
    T signed_area = dot(normal, cross(ba, p - a));
    T score = tabs(signed_area);
    if (bias * score >= best_score) { best_score = score; best = i; best_signed = signed_area; }
  }
  if (best == kNull) return;
  m->points[2] = pts[best];
  m->point_count = 3;
  pts[best] = pts[count - 1];
  count--;
  TV3<T> c = m->points[2].point;
  best_score = tol_sqr; best = kNull;
  T sign = best_signed < T(0.0f) ? T(-1.0f) : T(1.0f);
  for (int i = 0; i < count; ++i) {
    TV3<T> p = pts[i].point;
    T u1 = sign * dot(normal, cross(p - a, ba));
    T u2 = sign * dot(normal, cross(p - b, c - b));
    T u3 = sign * dot(normal, cross(p - c, a - c));
    T score = tmax(u1, tmax(u2, u3));
    if (bias * score > best_score) { best_score = score; best = i; }
  }
  if (best != kNull) {
    m->points[m->point_count] = pts[best];
    m->point_count += 1;
  }
}
// convex_manifold.rs:1150 build_face_a_contact; returns false when the forward step found no
// contact on this axis.
template <class T>
NSD_HD bool t_build_face_a(TLocalManifold<T>* m, const Hull& ha, const Hull& hb, const TXf<T>& xb, int ref_face,
                           int vertex) {
  TClipVertex<T> poly1[kClipCap], poly2[kClipCap];
  TLocalPoint<T> pts[kClipCap];
  TPlane<T> rp = tplane<T>(ha.planes[ref_face]);
  TV3<T> ref_n_in_b = inv_rotate(xb.q, rp.n);
  int inc = find_incident_face(hb, real3(ref_n_in_b), vertex);
  int count = t_build_polygon(poly1, xb, hb, inc, rp);
  int ei = box_face_edge(ref_face);
  bool use1 = true;
  for (;;) {
    HalfEdge e = box_edge(ei);
    int ni = e.next;
    HalfEdge nx = box_edge(ni);
    V3 p1 = ha.points[e.origin], p2 = ha.points[nx.origin];
    V3 tangent = nsd::normalize(p2 - p1);
    V3 binormal = nsd::cross(tangent, ha.planes[ref_face].n);
    TPlane<T> cp = tplane<T>(plane_from_normal_point(binormal, p1));
    if (use1) count = t_clip_polygon(poly2, poly1, count, cp, ei, rp);
    else count = t_clip_polygon(poly1, poly2, count, cp, ei, rp);
    use1 = !use1;
    if (count < 3) return false;
    ei = ni;
    if (ei == box_face_edge(ref_face)) break;
  }
  count = count < kClipCap ? count : kClipCap;
  m->normal = rp.n;
  const TClipVertex<T>* src = use1 ? poly1 : poly2;
  T min_sep = T(kFltMax);
  for (int i = 0; i < count; ++i) {
    TLocalPoint<T> p;
    p.point = mul_sub(src[i].position, T(0.5f) * src[i].separation, rp.n);
    p.separation = src[i].separation;
    p.pair = src[i].pair;
    min_sep = tmin(min_sep, src[i].separation);
    pts[i] = p;
  }
  if (min_sep >= T(speculative_distance())) return false;
  t_reduce_manifold_points(m, pts, count);
  return true;
}
template <class T>
NSD_HD bool t_build_face_b(TLocalManifold<T>* m, const Hull& ha, const Hull& hb, const TXf<T>& xb, int vertex,
                           int ref_face_b) {
  TXf<T> xa = invert_xf(xb);
  if (!t_build_face_a(m, hb, ha, xa, ref_face_b, vertex)) return false;
  TM3<T> mat = matrix_from_quat(xb.q);
  m->normal = -mul_mv(mat, m->normal);
  for (int i = 0; i < m->point_count; ++i) {
    m->points[i].point = mul_mv(mat, m->points[i].point) + xb.p;
    m->points[i].pair = flip_pair(m->points[i].pair);
  }
  return true;
}
template <class T>
NSD_HD bool t_build_edge(TLocalManifold<T>* m, const Hull& ha, const Hull& hb, const TXf<T>& xb, const TV3<T>& normal,
                         int index_a, int index_b) {
  HalfEdge ea = box_edge(index_a);
  HalfEdge ta = box_edge(ea.twin);
  TV3<T> pa = tv3<T>(ha.points[ea.origin]), qa = tv3<T>(ha.points[ta.origin]);
  TV3<T> e_a = qa - pa;
  HalfEdge eb = box_edge(index_b);
  HalfEdge tb = box_edge(eb.twin);
  TV3<T> pb = xf_point(xb, tv3<T>(hb.points[eb.origin]));
  TV3<T> qb = xf_point(xb, tv3<T>(hb.points[tb.origin]));
  TV3<T> e_b = qb - pb;
  // nsd_math.cuh line_distance
  T a11 = dot(e_a, e_a), a12 = -dot(e_a, e_b), a21 = dot(e_b, e_a), a22 = -dot(e_b, e_b);
  TV3<T> wv = pa - pb;
  T b1 = -dot(e_a, wv), b2 = -dot(e_b, wv);
  T d = a11 * a22 - a12 * a21;
  TV3<T> p1, p2;
  T f1, f2;
  if (d * d < T(1000.0f * kMinPositive)) {
    T s1 = dot(pb - pa, e_a) / dot(e_a, e_a);
    p1 = mul_add(pa, s1, e_a); f1 = s1; p2 = pb; f2 = T(0.0f);
  } else {
    T s1 = (a22 * b1 - a12 * b2) / d;
    T s2 = (a11 * b2 - a21 * b1) / d;
    p1 = mul_add(pa, s1, e_a); f1 = s1; p2 = mul_add(pb, s2, e_b); f2 = s2;
  }
  if (!((T(0.0f) <= f1 && f1 <= T(1.0f)) && (T(0.0f) <= f2 && f2 <= T(1.0f)))) return false;
  m->normal = normal;
  m->point_count = 1;
  m->points[0].point = T(0.5f) * (p1 + p2);
  m->points[0].separation = dot(normal, p2 - p1);
  m->points[0].pair = make_feature_pair(0, index_a, 1, index_b);
  return true;
}
// The edge-pair axis as the cached fast path computes it (nsd_geom.cuh collide_hulls).
template <class T>
NSD_HD TV3<T> t_edge_axis_cached(const Hull& ha, const Hull& hb, const TXf<T>& xb, int ia, int ib) {
  HalfEdge e1 = box_edge(ia), t1 = box_edge(ia + 1);
  TV3<T> e_a = tv3<T>(ha.points[t1.origin]) - tv3<T>(ha.points[e1.origin]);
  HalfEdge e2 = box_edge(ib), t2 = box_edge(ib + 1);
  TV3<T> ub = rotate(xb.q, tv3<T>(hb.planes[e2.face].n));
  TV3<T> vb = rotate(xb.q, tv3<T>(hb.planes[t2.face].n));
  T cba = dot(ub, e_a), dba = dot(vb, e_a);
  T t = cba / (cba - dba);
  return -normalize(lerp(ub, vb, t));
}
// The edge-pair axis as the full separating-axis search computes it (nsd_geom.cuh
// compute_separating_axis).
template <class T>
NSD_HD TV3<T> t_edge_axis_sat(const Hull& ha, const Hull& hb, const TXf<T>& xb, int ia, int ib) {
  TM3<T> r = matrix_from_quat(xb.q);
  TV3<T> r0 = tv3<T>(r.cx.x, r.cy.x, r.cz.x), r1 = tv3<T>(r.cx.y, r.cy.y, r.cz.y), r2 = tv3<T>(r.cx.z, r.cy.z, r.cz.z);
  HalfEdge e = box_edge(ib), tw = box_edge(ib + 1);
  auto bface = [&](int f) {
    TV3<T> v = tv3<T>(v3(hb.nx[f], hb.ny[f], hb.nz[f]));
    TV3<T> o = tv3<T>(dot(r0, v), dot(r1, v), dot(r2, v));
    return tv3<T>(-o.x, -o.y, -o.z);
  };
  TV3<T> c = bface(e.face), dn = bface(tw.face);
  HalfEdge ea = box_edge(ia), ta = box_edge(ia + 1);
  int v0 = ea.origin, v1 = ta.origin;
  TV3<T> d = tv3<T>(v3(ha.vx[v1] - ha.vx[v0], ha.vy[v1] - ha.vy[v0], ha.vz[v1] - ha.vz[v0]));
  T cba = dot(c, d), dba = dot(dn, d);
  T t = -cba / (dba - cba);
  TV3<T> n = mul_add(c, t, dn - c);
  T len2 = dot(n, n);
  T inv = T(1.0f) / tsqrt(len2);
  return inv * n;
}

// Narrowphase of a box pair followed by the world transform of update_contact
// (nsd_kernels.cuh update_contact, contact_update.rs:43). Inputs: tangents of centre A 0..2,
// qa 3..6, tangents of centre B 7..9, qb 10..13. Outputs: normal 0..2, per point q:
// 3 + 7 q + {anchor_a 0..2, anchor_b 3..5, separation 6}. Returns the point count, or -1
// when the replay does not reproduce a manifold.
enum FI : int { fiCa = 0, fiQa = 3, fiCb = 7, fiQb = 10, kFI = 14 };
constexpr int kFO = 31;
struct NarrowCase {
  uint8_t type, index_a, index_b, hit;  // SAT cache after the forward narrowphase
};
template <class T, class In>
NSD_HD int narrow_box_fn(const In& x, const Pos& ca, const Pos& cb, const Hull& ha, const Hull& hb, NarrowCase nc,
                         T* y, uint32_t* ids = nullptr) {
  TQ<T> qa = in4<T>(x, fiQa), qb = in4<T>(x, fiQb);
  // inv_mul_wxf(xa, xb): the position of B in A's frame, and the relative rotation
  TV3<T> d = sub_pos_t(cb, ca, in3<T>(x, fiCb), in3<T>(x, fiCa));
  TXf<T> xb;
  xb.p = inv_rotate(qa, d);
  xb.q = inv_mul_quat(qa, qb);
  TLocalManifold<T> lm;
  lm.point_count = 0;
  bool ok = false;
  if (nc.type == kFaceAxisA) {
    int vi = nc.index_b;
    if (nc.hit) {
      V3 sd = -nsd::inv_rotate(Q{real3(xb.q.v), (float)val(xb.q.s)}, ha.planes[nc.index_a].n);
      vi = find_hull_support_vertex(hb, sd);
    }
    ok = t_build_face_a(&lm, ha, hb, xb, nc.index_a, vi);
  } else if (nc.type == kFaceAxisB) {
    int vi = nc.index_a;
    if (nc.hit) {
      V3 sd = -nsd::rotate(Q{real3(xb.q.v), (float)val(xb.q.s)}, hb.planes[nc.index_b].n);
      vi = find_hull_support_vertex(ha, sd);
    }
    ok = t_build_face_b(&lm, ha, hb, xb, vi, nc.index_b);
  } else if (nc.type == kEdgePairAxis) {
    TV3<T> nrm = nc.hit ? t_edge_axis_cached(ha, hb, xb, nc.index_a, nc.index_b)
                        : t_edge_axis_sat(ha, hb, xb, nc.index_a, nc.index_b);
    ok = t_build_edge(&lm, ha, hb, xb, nrm, nc.index_a, nc.index_b);
  }
  if (!ok || lm.point_count == 0) return -1;
  TM3<T> ma = matrix_from_quat(qa);
  TV3<T> dab = sub_pos_t(ca, cb, in3<T>(x, fiCa), in3<T>(x, fiCb));
  out3(y, 0, mul_mv(ma, lm.normal));
  for (int i = 0; i < lm.point_count; ++i) {
    TV3<T> aa = mul_mv(ma, lm.points[i].point);
    out3(y, 3 + 7 * i, aa);
    out3(y, 3 + 7 * i + 3, aa + dab);
    y[3 + 7 * i + 6] = lm.points[i].separation;
    if (ids) ids[i] = make_feature_id(lm.points[i].pair);
  }
  return lm.point_count;
}

// ---------------------------------------------------------------------------------------------
// Manifolds of the pairs with a sphere or a capsule (nsd_geom.cuh collide_spheres,
// collide_capsule_sphere, collide_capsules, collide_hull_sphere, collide_hull_capsule;
// convex_manifold_shapes.rs:21-643), replayed along the branch the forward step took. The box
// pairs make discrete choices the value parts alone cannot repeat (the GJK simplex, the SAT
// face and edge): round_case runs the forward's own f32 routines on the same poses and cache and
// records them, and the restatement follows the record. Inside a branch, GJK's closest points
// are the barycentric projection of the origin onto its final simplex (distance.rs:58-67 and
// :496), whose derivatives are exact; the sphere and capsule pairs take their comparisons on the
// value parts like the box builders.
enum : int {
  kRoundNone = 0,      // no manifold
  kRoundDirect = 1,    // sphere-sphere, capsule-sphere, capsule-capsule
  kRoundGjk = 2,       // box pair, one point from the GJK closest points
  kRoundGjkFace = 3,   // box-capsule, the capsule clipped to the face the GJK normal picks
  kRoundDeepFace = 4,  // box-sphere with the centre inside; box-capsule SAT face
  kRoundDeepEdge = 5,  // box-capsule SAT edge pair
};
struct RoundCase {
  int path, face, edge;
  SimplexCache simplex;  // the GJK simplex after the forward's distance query
};

// The forward's choices for one pair (A the higher shape type), from the f32 routines.
NSD_HD RoundCase round_case(const DShape& A, const DShape& B, const Hull* ha, Xf xb, SimplexCache cache) {
  RoundCase rc;
  rc.path = kRoundNone; rc.face = -1; rc.edge = -1;
  rc.simplex = SimplexCache();
  if (A.type != kHull) { rc.path = kRoundDirect; return rc; }
  const float spec = speculative_distance();
  if (B.type == kSphere) {
    V3 c = xf_point(xb, B.sphere.center);
    DistOut d = shape_distance(ha->points, kHullVertexCount, &c, 1, xf(v3(0, 0, 0), qid()), &cache);
    float r = 0.0f + B.sphere.radius;
    if (d.distance > r + spec) return rc;
    if (d.distance > 100.0f * kEps) { rc.path = kRoundGjk; rc.simplex = cache; return rc; }
    float best_d = -kFltMax;
    for (int i = 0; i < kHullFaceCount; ++i) {
      float dd = plane_sep(ha->planes[i], c);
      if (dd > best_d) { rc.face = i; best_d = dd; }
    }
    rc.path = kRoundDeepFace;
    return rc;
  }
  const Capsule cap = B.capsule;
  V3 cpts[2] = {cap.c1, cap.c2};
  DistOut d = shape_distance(ha->points, kHullVertexCount, cpts, 2, xb, &cache);
  if (d.distance > cap.radius + spec) return rc;
  if (d.distance > 100.0f * kEps) {
    rc.simplex = cache;
    rc.path = kRoundGjk;
    int rf = find_hull_support_face(*ha, d.normal);
    Plane rp = ha->planes[rf];
    if (absf(dot(rp.n, d.normal)) > 0.998f) {
      ClipVertex vb[2];
      vb[0].position = xf_point(xb, cap.c1); vb[0].separation = 0; vb[0].pair = make_feature_pair(0, 0, 0, 0);
      vb[1].position = xf_point(xb, cap.c2); vb[1].separation = 0; vb[1].pair = make_feature_pair(0, 1, 0, 1);
      if (clip_segment_to_hull_face(vb, *ha, rf) == 2) {
        float d1 = plane_sep(rp, vb[0].position), d2 = plane_sep(rp, vb[1].position);
        if (d1 <= cap.radius + spec || d2 <= cap.radius + spec) { rc.path = kRoundGjkFace; rc.face = rf; }
      }
    }
    return rc;
  }
  SepAxis fq = query_face_hull_capsule(*ha, cap, xb);
  if (fq.separation > cap.radius) return rc;
  SepAxis eq = query_edge_hull_capsule(*ha, cap, xb);
  if (eq.separation > cap.radius) return rc;
  LocalManifold lm;
  lm.point_count = 0;
  float face_sep = fq.separation - cap.radius;
  build_hull_face_capsule(&lm, *ha, cap, xb, fq);
  if (lm.point_count == 2) { face_sep = minf(lm.points[0].separation, lm.points[1].separation); rc.path = kRoundDeepFace; }
  rc.face = fq.index_a;
  if (eq.index_a == kNull) return rc;
  float edge_sep = eq.separation - cap.radius;
  if (lm.point_count == 0 || edge_sep > face_sep + linear_slop()) {
    if (build_hull_capsule_edge(&lm, *ha, cap, xb, eq)) { rc.path = kRoundDeepEdge; rc.edge = eq.index_b; }
  }
  return rc;
}

template <class T> struct TSegResult { TV3<T> p1, p2; T f1, f2; };

// nsd_math.cuh point_to_segment (functions.rs:1169)
template <class T>
NSD_HD TV3<T> t_point_to_segment(const TV3<T>& a, const TV3<T>& b, const TV3<T>& q) {
  TV3<T> ab = b - a, aq = q - a;
  T alpha = dot(ab, aq);
  if (alpha <= T(0.0f)) return a;
  T den = dot(ab, ab);
  if (alpha > den) return b;
  alpha = alpha / den;
  return mul_add(a, alpha, ab);
}
// nsd_math.cuh segment_distance (functions.rs:1105)
template <class T>
NSD_HD TSegResult<T> t_segment_distance(const TV3<T>& p1, const TV3<T>& q1, const TV3<T>& p2, const TV3<T>& q2) {
  TSegResult<T> r;
  TV3<T> d1 = q1 - p1, d2 = q2 - p2, rr = p1 - p2;
  T a = dot(d1, d1), b = dot(d1, d2), c = dot(d1, rr), e = dot(d2, d2), f = dot(d2, rr);
  const T small = T(100.0f * kEps), zero = T(0.0f), one = T(1.0f);
  if (a < small && e < small) { r.p1 = p1; r.f1 = zero; r.p2 = p2; r.f2 = zero; return r; }
  if (a < small) {
    T s2 = tclamp(f / e, zero, one);
    r.p1 = p1; r.f1 = zero; r.p2 = mul_add(p2, s2, d2); r.f2 = s2; return r;
  }
  if (e < small) {
    T s1 = tclamp(-c / a, zero, one);
    r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = p2; r.f2 = zero; return r;
  }
  T denom = a * e - b * b;
  T s1 = denom > T(1000.0f * kMinPositive) ? tclamp((b * f - c * e) / denom, zero, one) : zero;
  T s2 = (b * s1 + f) / e;
  if (s2 < zero) {
    s1 = tclamp(-c / a, zero, one);
    s2 = zero;
  } else if (s2 > one) {
    s1 = tclamp((b - c) / a, zero, one);
    s2 = one;
  }
  r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = mul_add(p2, s2, d2); r.f2 = s2;
  return r;
}
// nsd_math.cuh line_distance (functions.rs:1069)
template <class T>
NSD_HD TSegResult<T> t_line_distance(const TV3<T>& p1, const TV3<T>& d1, const TV3<T>& p2, const TV3<T>& d2) {
  TSegResult<T> r;
  T a11 = dot(d1, d1), a12 = -dot(d1, d2), a21 = dot(d2, d1), a22 = -dot(d2, d2);
  TV3<T> w = p1 - p2;
  T b1 = -dot(d1, w), b2 = -dot(d2, w);
  T d = a11 * a22 - a12 * a21;
  if (d * d < T(1000.0f * kMinPositive)) {
    T s1 = dot(p2 - p1, d1) / dot(d1, d1);
    r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = p2; r.f2 = T(0.0f);
    return r;
  }
  T s1 = (a22 * b1 - a12 * b2) / d;
  T s2 = (a11 * b2 - a21 * b1) / d;
  r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = mul_add(p2, s2, d2); r.f2 = s2;
  return r;
}
// nsd_math.cuh get_length_and_normalize (functions.rs:293)
template <class T>
NSD_HD T t_length_and_normalize(const TV3<T>& a, TV3<T>* out) {
  T ls = a.x * a.x + a.y * a.y + a.z * a.z;
  if (ls > T(1000.0f * kMinPositive)) {
    T l = tsqrt(ls);
    T s = T(1.0f) / l;
    *out = tv3<T>(s * a.x, s * a.y, s * a.z);
    return l;
  }
  *out = tzero3<T>();
  return T(0.0f);
}
// nsd_geom.cuh clip_segment (convex_manifold.rs:127) against a constant plane
template <class T>
NSD_HD int t_clip_segment(TClipVertex<T>* seg, const Plane& pf) {
  const TPlane<T> p = tplane<T>(pf);
  int n = 0;
  TClipVertex<T> a = seg[0], b = seg[1];
  T d1 = plane_sep(p, a.position), d2 = plane_sep(p, b.position);
  if (d1 <= T(0.0f)) seg[n++] = a;
  if (d2 <= T(0.0f)) seg[n++] = b;
  if (d1 * d2 < T(0.0f)) {
    T t = d1 / (d1 - d2);
    seg[n].position = (T(1.0f) - t) * a.position + t * b.position;
    seg[n].pair = d1 > T(0.0f) ? a.pair : b.pair;
    n++;
  }
  return n;
}
// nsd_geom.cuh clip_segment_to_hull_face (convex_manifold.rs:163): the side planes are the box's
template <class T>
NSD_HD int t_clip_segment_to_hull_face(TClipVertex<T>* seg, const Hull& h, int ref_face) {
  Plane rp = h.planes[ref_face];
  int start = box_face_edge(ref_face);
  int ei = start;
  for (;;) {
    HalfEdge e = box_edge(ei);
    int ni = e.next;
    HalfEdge nx = box_edge(ni);
    V3 p1 = h.points[e.origin], p2 = h.points[nx.origin];
    V3 tangent = nsd::normalize(p2 - p1);
    V3 binormal = nsd::cross(tangent, rp.n);
    if (t_clip_segment(seg, plane_from_normal_point(binormal, p1)) < 2) return 0;
    ei = ni;
    if (ei == start) break;
  }
  return 2;
}
// The GJK closest points on the final simplex (count 1..3): vertex i pairs point ia[i] of A
// (constant, A's frame) with point ib[i] of B (already in A's frame).
template <class T>
NSD_HD void t_gjk_witness(const SimplexCache& sc, const V3* pa, const TV3<T>* pb, TV3<T>* wa, TV3<T>* wb) {
  TV3<T> A[3], B[3], W[3];
  const int n = sc.count < 3 ? sc.count : 3;
  for (int i = 0; i < n; ++i) {
    A[i] = tv3<T>(pa[sc.ia[i]]);
    B[i] = pb[sc.ib[i]];
    W[i] = B[i] - A[i];
  }
  if (n <= 1) { *wa = A[0]; *wb = B[0]; return; }
  if (n == 2) {
    TV3<T> ab = W[1] - W[0];
    T d = dot(ab, ab), u = dot(W[1], ab), v = -dot(W[0], ab);
    T l0 = u / d, l1 = v / d;
    *wa = blend2(l0, A[0], l1, A[1]);
    *wb = blend2(l0, B[0], l1, B[1]);
    return;
  }
  TV3<T> ab = W[1] - W[0], ac = W[2] - W[0];
  TV3<T> bxc = cross(W[1], W[2]), cxa = cross(W[2], W[0]), axb = cross(W[0], W[1]), n3 = cross(ab, ac);
  T d = dot(n3, n3), u = dot(bxc, n3), v = dot(cxa, n3), w = dot(axb, n3);
  T l0 = u / d, l1 = v / d, l2 = w / d;
  *wa = blend2(l0, A[0], l1, A[1]) + l2 * A[2];
  *wb = blend2(l0, B[0], l1, B[1]) + l2 * B[2];
}

template <class T>
NSD_HD void t_collide_spheres(TLocalManifold<T>* m, Sphere a, Sphere b, const TXf<T>& xb) {
  TV3<T> c1 = tv3<T>(a.center), c2 = xf_point(xb, tv3<T>(b.center));
  float tr = a.radius + b.radius;
  float maxd = tr + speculative_distance();
  TV3<T> off = c2 - c1;
  T dsq = length_sq(off);
  if (dsq > T(maxd * maxd)) return;
  TV3<T> n = tv3<T>(T(0.0f), T(1.0f), T(0.0f));
  T d = tsqrt(dsq);
  if (d * d > T(1000.0f * kMinPositive)) n = (T(1.0f) / d) * off;
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = T(0.5f) * (mul_sub(mul_add(c1, T(a.radius), n) + c2, T(b.radius), n));
  m->points[0].separation = d - T(tr);
  m->points[0].pair = FeaturePair();
}
template <class T>
NSD_HD void t_collide_capsule_sphere(TLocalManifold<T>* m, Capsule a, Sphere b, const TXf<T>& xb) {
  TV3<T> c = xf_point(xb, tv3<T>(b.center));
  float tr = b.radius + a.radius;
  float maxd = tr + speculative_distance();
  TV3<T> cp = t_point_to_segment(tv3<T>(a.c1), tv3<T>(a.c2), c);
  TV3<T> off = c - cp;
  T dsq = length_sq(off);
  if (dsq > T(maxd * maxd)) return;
  TV3<T> n = tv3<T>(T(0.0f), T(1.0f), T(0.0f));
  T d = tsqrt(dsq);
  if (d * d > T(1000.0f * kMinPositive)) n = (T(1.0f) / d) * off;
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = T(0.5f) * mul_add(mul_sub(c, T(b.radius), n) + cp, T(a.radius), n);
  m->points[0].separation = d - T(tr);
  m->points[0].pair = FeaturePair();
}
template <class T>
NSD_HD void t_collide_capsules(TLocalManifold<T>* m, Capsule a, Capsule b, const TXf<T>& xb) {
  TV3<T> a1 = tv3<T>(a.c1), a2 = tv3<T>(a.c2);
  TV3<T> b1 = xf_point(xb, tv3<T>(b.c1)), b2 = xf_point(xb, tv3<T>(b.c2));
  float radius = a.radius + b.radius;
  float maxd = radius + speculative_distance();
  TSegResult<T> res = t_segment_distance(a1, a2, b1, b2);
  TV3<T> off = res.p2 - res.p1;
  T dsq = length_sq(off);
  float mind = 0.01f * linear_slop();
  if (dsq > T(maxd * maxd) || dsq < T(mind * mind)) return;
  V3 ea;
  float la = get_length_and_normalize(a.c2 - a.c1, &ea);
  if (la < min_capsule_length()) return;
  TV3<T> eb;
  T lb = t_length_and_normalize(b2 - b1, &eb);
  if (lb < T(min_capsule_length())) return;
  TV3<T> axis = cross(tv3<T>(ea), eb);
  if (length_sq(axis) < T(0.05f * 0.05f)) {
    Plane pa0 = plane(-ea, -nsd::dot(ea, a.c1));
    Plane pa1 = plane(ea, nsd::dot(ea, a.c2));
    TClipVertex<T> vb[2];
    vb[0].position = b1; vb[0].separation = T(0.0f); vb[0].pair = make_feature_pair(0, 0, 0, 0);
    vb[1].position = b2; vb[1].separation = T(0.0f); vb[1].pair = make_feature_pair(0, 1, 0, 1);
    int pc = t_clip_segment(vb, pa0);
    if (pc == 2) pc = t_clip_segment(vb, pa1);
    if (pc == 2) {
      TV3<T> cp1 = t_point_to_segment(a1, a2, vb[0].position);
      TV3<T> cp2 = t_point_to_segment(a1, a2, vb[1].position);
      T d1 = length(vb[0].position - cp1), d2 = length(vb[1].position - cp2);
      if (d1 <= T(radius) && d2 <= T(radius)) {
        if (d1 < T(mind) || d2 < T(mind)) return;
        TV3<T> n1 = (T(1.0f) / d1) * (vb[0].position - cp1);
        TV3<T> n2 = (T(1.0f) / d2) * (vb[1].position - cp2);
        TV3<T> n = normalize(n1 + n2);
        T ra = T(a.radius), rb = T(b.radius);
        m->normal = n;
        m->point_count = 2;
        m->points[0].point = T(0.5f) * mul_sub(mul_add(vb[0].position, ra, n1) + cp1, rb, n);
        m->points[0].separation = d1 - T(radius);
        m->points[0].pair = vb[0].pair;
        m->points[1].point = T(0.5f) * mul_sub(mul_add(vb[1].position, ra, n2) + cp2, rb, n);
        m->points[1].separation = d2 - T(radius);
        m->points[1].pair = vb[1].pair;
        return;
      }
    }
  }
  TV3<T> n;
  T dv = t_length_and_normalize(off, &n);
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = T(0.5f) * mul_sub(mul_add(res.p1, T(a.radius), n) + res.p2, T(b.radius), n);
  m->points[0].separation = dv - T(radius);
  m->points[0].pair = FeaturePair();
}
template <class T>
NSD_HD void t_hull_sphere(TLocalManifold<T>* m, const Hull& ha, Sphere b, const TXf<T>& xb, const RoundCase& rc) {
  TV3<T> c = xf_point(xb, tv3<T>(b.center));
  const T rb = T(b.radius), r = T(0.0f + b.radius);
  TV3<T> n, pa;
  T sep;
  if (rc.path == kRoundGjk) {
    TV3<T> wb;
    t_gjk_witness(rc.simplex, ha.points, &c, &pa, &wb);
    n = normalize(wb - pa);
    sep = length(wb - pa) - r;
  } else {
    pa = c;  // the centre is inside: GJK's witness points coincide with it
    n = tv3<T>(ha.planes[rc.face].n);
    sep = plane_sep(tplane<T>(ha.planes[rc.face]), c) - r;
  }
  TV3<T> ca = mul_add(c, T(0.0f) - dot(c - pa, n), n);
  TV3<T> cb = mul_sub(c, rb, n);
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = lerp(ca, cb, T(0.5f));
  m->points[0].separation = sep;
  m->points[0].pair = FeaturePair();
}
template <class T>
NSD_HD void t_hull_capsule(TLocalManifold<T>* m, const Hull& ha, Capsule b, const TXf<T>& xb, const RoundCase& rc) {
  const T br = T(b.radius);
  TV3<T> q1 = xf_point(xb, tv3<T>(b.c1)), q2 = xf_point(xb, tv3<T>(b.c2));
  if (rc.path == kRoundGjk) {
    TM3<T> mt = matrix_from_quat(xb.q);
    TV3<T> cpts[2] = {mul_mv(mt, tv3<T>(b.c1)) + xb.p, mul_mv(mt, tv3<T>(b.c2)) + xb.p};
    TV3<T> pa, pb;
    t_gjk_witness(rc.simplex, ha.points, cpts, &pa, &pb);
    TV3<T> delta = normalize(pb - pa);
    m->normal = delta;
    m->point_count = 1;
    m->points[0].point = T(0.5f) * (mul_sub(pa, br, delta) + pb);
    m->points[0].separation = length(pb - pa) - br;
    m->points[0].pair = FeaturePair();
    return;
  }
  if (rc.path == kRoundGjkFace || rc.path == kRoundDeepFace) {
    TClipVertex<T> vb[2];
    vb[0].position = q1; vb[0].separation = T(0.0f); vb[0].pair = make_feature_pair(0, 0, 0, 0);
    vb[1].position = q2; vb[1].separation = T(0.0f); vb[1].pair = make_feature_pair(0, 1, 0, 1);
    if (t_clip_segment_to_hull_face(vb, ha, rc.face) != 2) return;
    TPlane<T> rp = tplane<T>(ha.planes[rc.face]);
    T d1 = plane_sep(rp, vb[0].position), d2 = plane_sep(rp, vb[1].position);
    TV3<T> n = rp.n;
    m->normal = n;
    m->point_count = 2;
    // the two builders sum the half-depths in opposite orders
    T h1 = rc.path == kRoundGjkFace ? T(0.5f) * (br + d1) : T(0.5f) * (d1 + br);
    T h2 = rc.path == kRoundGjkFace ? T(0.5f) * (br + d2) : T(0.5f) * (d2 + br);
    m->points[0].point = mul_sub(vb[0].position, h1, n);
    m->points[0].separation = d1 - br;
    m->points[0].pair = vb[0].pair;
    m->points[1].point = mul_sub(vb[1].position, h2, n);
    m->points[1].separation = d2 - br;
    m->points[1].pair = vb[1].pair;
    return;
  }
  // the SAT edge pair: the capsule's axis against box edge rc.edge (query_edge_hull_capsule)
  TV3<T> ec = q2 - q1;
  HalfEdge e = box_edge(rc.edge), tw = box_edge(rc.edge + 1);
  TV3<T> ub = tv3<T>(ha.planes[e.face].n), vb = tv3<T>(ha.planes[tw.face].n);
  T cba = dot(ub, ec), dba = dot(vb, ec);
  T tt = cba / (cba - dba);
  TV3<T> n = normalize(lerp(ub, vb, tt));
  HalfEdge e2 = box_edge(rc.edge);
  HalfEdge t2 = box_edge(e2.twin);
  TV3<T> ph = tv3<T>(ha.points[e2.origin]), qh = tv3<T>(ha.points[t2.origin]);
  TSegResult<T> r = t_line_distance(ph, qh - ph, q1, ec);
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = T(0.5f) * (mul_sub(r.p1, br, n) + r.p2);
  m->points[0].separation = dot(n, r.p2 - r.p1) - br;
  m->points[0].pair = make_feature_pair(0, 0, 1, rc.edge);
}

// The manifold of a pair with a sphere or a capsule followed by update_contact's world
// transform; same inputs and outputs as narrow_box_fn. Returns the point count, or -1 when the
// replay makes no manifold.
template <class T, class In>
NSD_HD int narrow_round_fn(const In& x, const Pos& ca, const Pos& cb, const DShape& A, const DShape& B, const Hull* ha,
                           const RoundCase& rc, T* y, uint32_t* ids = nullptr) {
  if (rc.path == kRoundNone) return -1;
  TQ<T> qa = in4<T>(x, fiQa), qb = in4<T>(x, fiQb);
  TV3<T> d = sub_pos_t(cb, ca, in3<T>(x, fiCb), in3<T>(x, fiCa));
  TXf<T> xb;
  xb.p = inv_rotate(qa, d);
  xb.q = inv_mul_quat(qa, qb);
  TLocalManifold<T> lm;
  lm.point_count = 0;
  if (A.type == kSphere) t_collide_spheres(&lm, A.sphere, B.sphere, xb);
  else if (A.type == kCapsule && B.type == kSphere) t_collide_capsule_sphere(&lm, A.capsule, B.sphere, xb);
  else if (A.type == kCapsule) t_collide_capsules(&lm, A.capsule, B.capsule, xb);
  else if (B.type == kSphere) t_hull_sphere(&lm, *ha, B.sphere, xb, rc);
  else t_hull_capsule(&lm, *ha, B.capsule, xb, rc);
  if (lm.point_count == 0) return -1;
  TM3<T> ma = matrix_from_quat(qa);
  TV3<T> dab = sub_pos_t(ca, cb, in3<T>(x, fiCa), in3<T>(x, fiCb));
  out3(y, 0, mul_mv(ma, lm.normal));
  for (int i = 0; i < lm.point_count; ++i) {
    TV3<T> aa = mul_mv(ma, lm.points[i].point);
    out3(y, 3 + 7 * i, aa);
    out3(y, 3 + 7 * i + 3, aa + dab);
    y[3 + 7 * i + 6] = lm.points[i].separation;
    if (ids) ids[i] = make_feature_id(lm.points[i].pair);
  }
  return lm.point_count;
}

// ---------------------------------------------------------------------------------------------
// Revolute joints (nsd_solve.cuh solve_joint and joint_warm_delta, nsd_kernels.cuh
// k_prepare_joints; revolute_joint.rs:183-553). The joint vector holds the bodies' velocities,
// position and rotation increments, the joint's impulses and perp axes (the warm start reads the
// axes the last solve wrote; the solve recomputes them) and the prepared constants.
enum JX : int {
  jxVA = 0, jxWA = 3, jxVB = 6, jxWB = 9, jxDpA = 12, jxDpB = 15, jxDqA = 18, jxDqB = 22,
  jxLin = 26, jxPerp = 29, jxSpring = 31, jxMotor = 32, jxLower = 33, jxUpper = 34,
  jxPx = 35, jxPy = 38,
  jxIma = 41, jxImb = 42, jxIA = 43, jxIB = 52, jxFqA = 61, jxFqB = 65, jxFpA = 69, jxFpB = 72,
  jxAxis = 75, jxAxial = 78, jxDc = 79, kJX = 82,
};
// Solve outputs: velocities 0..11, impulses 12..20 (jxLin..jxUpper order), perp axes 21..26.
constexpr int kJSolveOut = 27;
// The joint's carried state (impulses and perp axes: jxLin..jxPy + 2) and its constants
// (jxIma..kJX).
constexpr int kJState = jxIma - jxLin, kJConst = kJX - jxIma;
struct JParams {
  bool use_bias, fixed, spring, motor, limit;
  Softness cs, ss;  // constraint and spring softness
  float target, lower, upper, motor_speed, max_torque_h, inv_h;
};

// nsd_math.cuh atan2_approx (functions.rs:68) and get_twist_angle (:490)
template <class T>
NSD_HD T t_atan2_approx(const T& y, const T& x) {
  if (x == T(0.0f) && y == T(0.0f)) return T(0.0f);
  T ax = tabs(x), ay = tabs(y);
  T mx = tmax(ay, ax), mn = tmin(ay, ax);
  T a = mn / mx;
  T s = a * a, c = s * a, q = s * s;
  T r = T(0.024840285f) * q + T(0.18681418f);
  T t = T(-0.094097948f) * q - T(0.33213072f);
  r = r * s + t;
  r = r * c + a;
  if (ay > ax) r = T(1.57079637f) - r;
  if (x < T(0.0f)) r = T(3.14159274f) - r;
  if (y < T(0.0f)) r = -r;
  return r;
}
template <class T>
NSD_HD T t_twist_angle(const TQ<T>& q) {
  T twist = q.s < T(0.0f) ? t_atan2_approx(-q.v.z, -q.s) : t_atan2_approx(q.v.z, q.s);
  return twist * T(2.0f);
}
// nsd_solve.cuh solve_point_constraint (revolute_joint.rs:95)
template <class T>
NSD_HD TV3<T> t_solve_point_constraint(const T& ma, const T& mb, const TM3<T>& ia, const TM3<T>& ib, const TV3<T>& ra,
                                       const TV3<T>& rb, const TV3<T>& rhs) {
  T axy = ra.z * ia.cy.y - ra.y * ia.cz.y;
  T axz = ra.z * ia.cy.z - ra.y * ia.cz.z;
  TV3<T> ay = ra.x * ia.cz - ra.z * ia.cx;
  TV3<T> az = ra.y * ia.cx - ra.x * ia.cy;
  T bxy = rb.z * ib.cy.y - rb.y * ib.cz.y;
  T bxz = rb.z * ib.cy.z - rb.y * ib.cz.z;
  TV3<T> by = rb.x * ib.cz - rb.z * ib.cx;
  TV3<T> bz = rb.y * ib.cx - rb.x * ib.cy;
  T m = ma + mb;
  T kxx = (axy * ra.z - axz * ra.y) + (bxy * rb.z - bxz * rb.y) + m;
  T kyy = (ay.z * ra.x - ay.x * ra.z) + (by.z * rb.x - by.x * rb.z) + m;
  T kzz = (az.x * ra.y - az.y * ra.x) + (bz.x * rb.y - bz.y * rb.x) + m;
  T kxy = (ay.y * ra.z - ay.z * ra.y) + (by.y * rb.z - by.z * rb.y);
  T kxz = (az.y * ra.z - az.z * ra.y) + (bz.y * rb.z - bz.z * rb.y);
  T kyz = (az.z * ra.x - az.x * ra.z) + (bz.z * rb.x - bz.x * rb.z);
  T cxx = kyy * kzz - kyz * kyz;
  T cyy = kxx * kzz - kxz * kxz;
  T czz = kxx * kyy - kxy * kxy;
  T cxy = kxz * kyz - kxy * kzz;
  T cxz = kxy * kyz - kyy * kxz;
  T cyz = kxy * kxz - kxx * kyz;
  T d = kxx * cxx + kxy * cxy + kxz * cxz;
  if (tabs(d) > T(1000.0f * kMinPositive)) {
    T inv = T(1.0f) / d;
    return tv3<T>(inv * (cxx * rhs.x + cxy * rhs.y + cxz * rhs.z), inv * (cxy * rhs.x + cyy * rhs.y + cyz * rhs.z),
                  inv * (cxz * rhs.x + cyz * rhs.y + czz * rhs.z));
  }
  return tzero3<T>();
}
template <class T, class In> NSD_HD TM3<T> in_m3(const In& x, int i) {
  return tm3<T>(in3<T>(x, i), in3<T>(x, i + 3), in3<T>(x, i + 6));
}
template <class T> NSD_HD TQ<T> tq(const Q& q) { return tquat<T>(tv3<T>(q.v), T(q.s)); }
template <class T> NSD_HD TV3<T> half_perp(const TQ<T>& qa, const TQ<T>& rq, int axis) {
  TV3<T> e = tv3<T>(T(axis == 0 ? 1.0f : 0.0f), T(axis == 1 ? 1.0f : 0.0f), T(0.0f));
  return T(0.5f) * rotate(qa, rq.s * e + cross(rq.v, e));
}

// solve_joint (revolute_joint.rs:316): spring, motor and limits on the axial row, the two
// perpendicular angular rows, then the point constraint.
template <class T, class In>
NSD_HD void joint_solve_fn(const In& x, const JParams& jp, T* y) {
  T mA = x(jxIma), mB = x(jxImb);
  TM3<T> iA = in_m3<T>(x, jxIA), iB = in_m3<T>(x, jxIB);
  TV3<T> va = in3<T>(x, jxVA), wa = in3<T>(x, jxWA), vb = in3<T>(x, jxVB), wb = in3<T>(x, jxWB);
  TQ<T> dqa = in4<T>(x, jxDqA), dqb = in4<T>(x, jxDqB);
  TQ<T> qa = mul_quat(dqa, in4<T>(x, jxFqA));
  TQ<T> qb = mul_quat(dqb, in4<T>(x, jxFqB));
  if (dot_quat(qa, qb) < T(0.0f)) qb = tquat<T>(tv3<T>(-qb.v.x, -qb.v.y, -qb.v.z), -qb.s);
  TQ<T> rq = inv_mul_quat(qa, qb);
  TV3<T> lin = in3<T>(x, jxLin);
  T p0 = x(jxPerp), p1 = x(jxPerp + 1);
  T spring = x(jxSpring), motor = x(jxMotor), lower = x(jxLower), upper = x(jxUpper);
  TV3<T> px = in3<T>(x, jxPx), py = in3<T>(x, jxPy);
  const T zero = T(0.0f), one = T(1.0f);
  if (!jp.fixed && (jp.spring || jp.motor || jp.limit)) {
    TV3<T> axis = in3<T>(x, jxAxis);
    T axial = x(jxAxial);
    TV3<T> ga = mul_mv(iA, axis), gb = mul_mv(iB, axis);
    T k = dot(axis, ga + gb);
    T acd = dot(wb - wa, axis);
    T ai = zero;
    if (jp.spring) {
      T angle = t_twist_angle(rq);
      T c = angle - T(jp.target);
      T bias = T(jp.ss.bias_rate) * c;
      T ms = T(jp.ss.mass_scale), is = T(jp.ss.impulse_scale);
      T di = -ms * axial * (acd + bias) - is * spring;
      spring = spring + di;
      acd = acd + k * di;
      ai = ai + di;
    }
    if (jp.motor) {
      T cdot = acd - T(jp.motor_speed);
      T old = motor;
      T mx = T(jp.max_torque_h);
      T di = tclamp(-axial * cdot, -mx - old, mx - old);
      motor = old + di;
      acd = acd + k * di;
      ai = ai + di;
    }
    if (jp.limit) {
      T angle = t_twist_angle(rq);
      {
        T c = angle - T(jp.lower);
        T bias = zero, ms = one, is = zero;
        if (c > zero) bias = c * T(jp.inv_h);
        else if (jp.use_bias) { bias = T(jp.cs.bias_rate) * c; ms = T(jp.cs.mass_scale); is = T(jp.cs.impulse_scale); }
        T old = lower;
        T di = tmax(-ms * axial * (acd + bias) - is * old, -old);
        lower = old + di;
        acd = acd + k * di;
        ai = ai + di;
      }
      {
        T c = T(jp.upper) - angle;
        T bias = zero, ms = one, is = zero;
        if (c > zero) bias = c * T(jp.inv_h);
        else if (jp.use_bias) { bias = T(jp.cs.bias_rate) * c; ms = T(jp.cs.mass_scale); is = T(jp.cs.impulse_scale); }
        T cdot = -acd;
        T old = upper;
        T di = tmax(-ms * axial * (cdot + bias) - is * old, -old);
        upper = old + di;
        ai = ai - di;
      }
    }
    wa = wa - ai * ga;
    wb = wb + ai * gb;
  }
  if (!jp.fixed) {
    T bx = zero, by = zero, ms = one, is = zero;
    if (jp.use_bias) {
      bx = T(jp.cs.bias_rate) * rq.v.x;
      by = T(jp.cs.bias_rate) * rq.v.y;
      ms = T(jp.cs.mass_scale);
      is = T(jp.cs.impulse_scale);
    }
    px = half_perp(qa, rq, 0);
    py = half_perp(qa, rq, 1);
    TM3<T> sum = tm3<T>(iA.cx + iB.cx, iA.cy + iB.cy, iA.cz + iB.cz);
    T kxx = dot(px, mul_mv(sum, px));
    T kyy = dot(py, mul_mv(sum, py));
    T kxy = dot(px, mul_mv(sum, py));
    TV3<T> wr = wb - wa;
    T rx = dot(wr, px) + bx, ry = dot(wr, py) + by;
    T sx = zero, sy = zero;
    T d = kxx * kyy - kxy * kxy;
    if (d > T(1000.0f * kMinPositive)) {
      T inv = one / d;
      sx = inv * kyy * rx - inv * kxy * ry;
      sy = -inv * kxy * rx + inv * kxx * ry;
    }
    T dix = (-ms) * sx - is * p0, diy = (-ms) * sy - is * p1;
    p0 = p0 + dix;
    p1 = p1 + diy;
    TV3<T> ang = dix * px + diy * py;
    wa = wa - mul_mv(iA, ang);
    wb = wb + mul_mv(iB, ang);
  }
  {
    TV3<T> ra = rotate(dqa, in3<T>(x, jxFpA)), rb = rotate(dqb, in3<T>(x, jxFpB));
    TV3<T> cdot = (vb + cross(wb, rb)) - va - cross(wa, ra);
    TV3<T> bias = tzero3<T>();
    T ms = one, is = zero;
    if (jp.use_bias) {
      TV3<T> sep = ((in3<T>(x, jxDpB) - in3<T>(x, jxDpA)) + (rb - ra)) + in3<T>(x, jxDc);
      bias = T(jp.cs.bias_rate) * sep;
      ms = T(jp.cs.mass_scale);
      is = T(jp.cs.impulse_scale);
    }
    TV3<T> b = t_solve_point_constraint(mA, mB, iA, iB, ra, rb, cdot + bias);
    TV3<T> imp = (-ms) * b - is * lin;
    lin = lin + imp;
    va = va - mA * imp;
    wa = wa - mul_mv(iA, cross(ra, imp));
    vb = vb + mB * imp;
    wb = wb + mul_mv(iB, cross(rb, imp));
  }
  out3(y, 0, va); out3(y, 3, wa); out3(y, 6, vb); out3(y, 9, wb);
  out3(y, 12, lin);
  y[15] = p0; y[16] = p1; y[17] = spring; y[18] = motor; y[19] = lower; y[20] = upper;
  out3(y, 21, px); out3(y, 24, py);
}

// joint_warm_delta (revolute_joint.rs:261): outputs dva 0..2, dwa 3..5, dvb 6..8, dwb 9..11
// (body A takes v - dva, w - dwa; body B v + dvb, w + dwb).
template <class T, class In>
NSD_HD void joint_warm_fn(const In& x, T* y) {
  T mA = x(jxIma), mB = x(jxImb);
  TM3<T> iA = in_m3<T>(x, jxIA), iB = in_m3<T>(x, jxIB);
  TV3<T> ra = rotate(in4<T>(x, jxDqA), in3<T>(x, jxFpA)), rb = rotate(in4<T>(x, jxDqB), in3<T>(x, jxFpB));
  T axial = ((x(jxSpring) + x(jxMotor)) + x(jxLower)) - x(jxUpper);
  TV3<T> ang = x(jxPerp) * in3<T>(x, jxPx) + x(jxPerp + 1) * in3<T>(x, jxPy);
  ang = mul_add(ang, axial, in3<T>(x, jxAxis));
  TV3<T> lin = in3<T>(x, jxLin);
  out3(y, 0, mA * lin);
  out3(y, 3, mul_mv(iA, cross(ra, lin) + ang));
  out3(y, 6, mB * lin);
  out3(y, 9, mul_mv(iB, cross(rb, lin) + ang));
}

// k_prepare_joints (revolute_joint.rs:183, distance_joint_solver.rs:74): the constants and the
// prepare's perp axes from the bodies' poses, inverse masses and world inverse inertias. Inputs:
// qa 0..3, qb 4..7, tangents of centre A 8..10 and B 11..13, inverse masses 14, 15, inverse
// inertias 16..24, 25..33. Outputs: the joint vector from jxPx on (perp axes, then constants).
enum JPI : int { jpQa = 0, jpQb = 4, jpCa = 8, jpCb = 11, jpIma = 14, jpImb = 15, jpIA = 16, jpIB = 25, kJPI = 34 };
constexpr int kJPO = kJX - jxPx;
template <class T, class In>
NSD_HD void joint_prepare_fn(const In& x, const Xf& lfa, const Xf& lfb, V3 lca, V3 lcb, const Pos& ca, const Pos& cb,
                             T* y) {
  TQ<T> qa = in4<T>(x, jpQa), qb = in4<T>(x, jpQb);
  TM3<T> iA = in_m3<T>(x, jpIA), iB = in_m3<T>(x, jpIB);
  TQ<T> fqa = mul_quat(qa, tq<T>(lfa.q)), fqb = mul_quat(qb, tq<T>(lfb.q));
  TV3<T> fpa = rotate(qa, tv3<T>(lfa.p - lca)), fpb = rotate(qb, tv3<T>(lfb.p - lcb));
  TV3<T> dc = sub_pos_t(cb, ca, in3<T>(x, jpCb), in3<T>(x, jpCa));
  TV3<T> axis = rotate(fqa, tv3<T>(T(0.0f), T(0.0f), T(1.0f)));
  TM3<T> sum = tm3<T>(iA.cx + iB.cx, iA.cy + iB.cy, iA.cz + iB.cz);
  T k = dot(axis, mul_mv(sum, axis));
  T axial = k > T(0.0f) ? T(1.0f) / k : T(0.0f);
  TQ<T> rq = inv_mul_quat(fqa, fqb);
  // output i holds joint-vector entry jxPx + i
  out3(y, jxPx - jxPx, half_perp(fqa, rq, 0));
  out3(y, jxPy - jxPx, half_perp(fqa, rq, 1));
  y[jxIma - jxPx] = x(jpIma);
  y[jxImb - jxPx] = x(jpImb);
  for (int i = 0; i < 9; ++i) { y[jxIA - jxPx + i] = x(jpIA + i); y[jxIB - jxPx + i] = x(jpIB + i); }
  out4(y, jxFqA - jxPx, fqa); out4(y, jxFqB - jxPx, fqb);
  out3(y, jxFpA - jxPx, fpa); out3(y, jxFpB - jxPx, fpb);
  out3(y, jxAxis - jxPx, axis);
  y[jxAxial - jxPx] = axial;
  out3(y, jxDc - jxPx, dc);
}

}  // namespace ad
}  // namespace nsd
