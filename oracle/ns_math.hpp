// Oracle math layer. TEST INFRASTRUCTURE ONLY: this directory is the CPU
// restatement of the reference solver used as the parity checker; the
// product library under natsel_b200/ never includes or links it.
//
// Every helper restates one function of the reference (file:line cited)
// with the same operand order. IEEE f32 arithmetic without contraction is
// required: the oracle is compiled with -ffp-contract=off and no fast-math.
#pragma once
#include <cmath>
#include <cstdint>
#include <cfloat>
#include <cstring>
#include <type_traits>

namespace nso {

// The oracle's scalar. The parity build is f32 (the reference's arithmetic, bit for bit); the
// same sources built with NSO_REAL_F64 give the f64 run the trajectory statistics are checked
// against (every operation in double; constants keep their f32 literals' values).
#ifdef NSO_REAL_F64
typedef double real;
static const real kMinPositive = DBL_MIN;
static const real kEps = DBL_EPSILON;
static const real kFltMax = DBL_MAX;
#else
typedef float real;
static const real kMinPositive = FLT_MIN;           // f32::MIN_POSITIVE
static const real kEps = FLT_EPSILON;               // f32::EPSILON
static const real kFltMax = FLT_MAX;
#endif
static const real kPi = 3.14159265359f;             // base/constants.rs:6
static const int kNull = -1;
static const int kGraphColorCount = 24;              // constants.rs:23
static const int kOverflowIndex = kGraphColorCount - 1;      // constraint_graph.rs:20
static const int kDynamicColorCount = kGraphColorCount - 4;  // constraint_graph.rs:23
static const real kMaxRotation = 0.25f * kPi;       // constants.rs:28
static const real kRecycleAngular = 0.99240388f;    // constants.rs:29
static const real kAabbMarginFraction = 0.125f;     // constants.rs:30
static const real kMinFrictionWeight = 1e-10f;      // constants.rs:26
static const real kParallelEdgeTol = 0.005f;        // constants.rs:39

// Length-unit dependent values are computed at run time in the reference
// (constants.rs:79-121), so they are computed the same way here.
inline real length_units() { return 1.0f; }
inline real linear_slop() { return 0.005f * length_units(); }
inline real speculative_distance() { return 4.0f * linear_slop(); }
inline real contact_recycle_distance() { return 10.0f * linear_slop(); }
inline real max_aabb_margin() { return 0.05f * length_units(); }
inline real huge_value() { return 1.0e5f * length_units(); }
inline real min_capsule_length() { return linear_slop(); }

struct V2 { real x, y; };
struct V3 { real x, y, z; };
struct Q { V3 v; real s; };
struct M3 { V3 cx, cy, cz; };
struct M2 { V2 cx, cy; };
struct Pos { double x, y, z; };
struct Xf { V3 p; Q q; };
struct WXf { Pos p; Q q; };
struct AABB { V3 lo, hi; };
struct Plane { V3 n; real off; };

inline V2 v2(real x, real y) { V2 r = {x, y}; return r; }
inline V3 v3(real x, real y, real z) { V3 r = {x, y, z}; return r; }
inline Q quat(V3 v, real s) { Q r = {v, s}; return r; }
inline Q qid() { return quat(v3(0, 0, 0), 1.0f); }
inline M3 m3(V3 a, V3 b, V3 c) { M3 r = {a, b, c}; return r; }
inline M3 m3zero() { return m3(v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0)); }
inline Xf xf(V3 p, Q q) { Xf r = {p, q}; return r; }
inline Plane plane(V3 n, real o) { Plane r = {n, o}; return r; }
inline AABB aabb(V3 lo, V3 hi) { AABB r = {lo, hi}; return r; }

// functions.rs:16-60 -- ties return the second operand.
inline int min_i(int a, int b) { return a < b ? a : b; }
inline int max_i(int a, int b) { return a > b ? a : b; }
inline real absf(real a) { return a < 0.0f ? -a : a; }
inline real minf(real a, real b) { return a < b ? a : b; }
inline real maxf(real a, real b) { return a > b ? a : b; }
inline real clampf(real a, real lo, real hi) { return a < lo ? lo : (hi < a ? hi : a); }

// functions.rs:68 atan2_approx (polynomial, not libm)
inline real atan2_approx(real y, real x) {
  if (x == 0.0f && y == 0.0f) return 0.0f;
  real ax = absf(x), ay = absf(y);
  real mx = maxf(ay, ax), mn = minf(ay, ax);
  real a = mn / mx;
  real s = a * a, c = s * a, q = s * s;
  real r = 0.024840285f * q + 0.18681418f;
  real t = -0.094097948f * q - 0.33213072f;
  r = r * s + t;
  r = r * c + a;
  if (ay > ax) r = 1.57079637f - r;
  if (x < 0.0f) r = 3.14159274f - r;
  if (y < 0.0f) r = -r;
  return r;
}

// functions.rs:147-245 vector operators
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 operator*(real s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }

inline real dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }       // :250
inline real length(V3 v) { return std::sqrt(dot(v, v)); }                        // :256
inline real length_sq(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }      // :262
inline real distance(V3 a, V3 b) { return length(v3(b.x - a.x, b.y - a.y, b.z - a.z)); }
inline real distance_sq(V3 a, V3 b) {                                            // :274
  V3 d = v3(b.x - a.x, b.y - a.y, b.z - a.z);
  return d.x * d.x + d.y * d.y + d.z * d.z;
}
inline V3 normalize(V3 a) {                                                       // :281
  real ls = a.x * a.x + a.y * a.y + a.z * a.z;
  if (ls > 1000.0f * kMinPositive) {
    real s = 1.0f / std::sqrt(ls);
    return v3(s * a.x, s * a.y, s * a.z);
  }
  return v3(0, 0, 0);
}
inline real get_length_and_normalize(V3 a, V3* out) {                            // :293
  real ls = a.x * a.x + a.y * a.y + a.z * a.z;
  if (ls > 1000.0f * kMinPositive) {
    real l = std::sqrt(ls);
    real s = 1.0f / l;
    *out = v3(s * a.x, s * a.y, s * a.z);
    return l;
  }
  *out = v3(0, 0, 0);
  return 0.0f;
}
inline V3 perp(V3 a) {                                                            // :306
  V3 p = (a.x < -0.5f || 0.5f < a.x) ? v3(a.y, -a.x, 0.0f) : v3(0.0f, a.z, -a.y);
  return normalize(p);
}
inline bool is_normalized(V3 a) { return absf(1.0f - dot(a, a)) < 100.0f * kEps; }
inline V3 mul_add(V3 a, real s, V3 b) { return v3(a.x + s * b.x, a.y + s * b.y, a.z + s * b.z); }  // :322
inline V3 mul_sub(V3 a, real s, V3 b) { return v3(a.x - s * b.x, a.y - s * b.y, a.z - s * b.z); }  // :328
inline V3 cross(V3 a, V3 b) {                                                     // :333
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline V3 lerp(V3 a, V3 b, real t) {                                             // :342
  return v3((1.0f - t) * a.x + t * b.x, (1.0f - t) * a.y + t * b.y, (1.0f - t) * a.z + t * b.z);
}
inline V3 blend2(real s, V3 a, real t, V3 b) {                                  // :353
  return v3(s * a.x + t * b.x, s * a.y + t * b.y, s * a.z + t * b.z);
}
inline V3 blend3(real s, V3 a, real t, V3 b, real u, V3 c) {                   // internal_math.rs:249
  return v3(s * a.x + t * b.x + u * c.x, s * a.y + t * b.y + u * c.y, s * a.z + t * b.z + u * c.z);
}
inline V3 abs3(V3 a) { return v3(absf(a.x), absf(a.y), absf(a.z)); }
inline V3 min3(V3 a, V3 b) { return v3(minf(a.x, b.x), minf(a.y, b.y), minf(a.z, b.z)); }
inline V3 max3(V3 a, V3 b) { return v3(maxf(a.x, b.x), maxf(a.y, b.y), maxf(a.z, b.z)); }

// functions.rs:402-450 quaternions
inline V3 rotate(Q q, V3 v) {
  V3 t1 = cross(q.v, v);
  V3 t2 = mul_add(t1, q.s, v);
  V3 t3 = cross(q.v, t2);
  return mul_add(v, 2.0f, t3);
}
inline V3 inv_rotate(Q q, V3 v) {
  V3 t1 = cross(q.v, v);
  V3 t2 = mul_sub(t1, q.s, v);
  V3 t3 = cross(q.v, t2);
  return mul_add(v, 2.0f, t3);
}
inline real dot_quat(Q a, Q b) { return a.v.x * b.v.x + a.v.y * b.v.y + a.v.z * b.v.z + a.s * b.s; }
inline Q mul_quat(Q q1, Q q2) {                                                   // :423
  V3 t1 = cross(q1.v, q2.v);
  V3 t2 = mul_add(t1, q1.s, q2.v);
  V3 t3 = mul_add(t2, q2.s, q1.v);
  return quat(t3, q1.s * q2.s - dot(q1.v, q2.v));
}
inline Q inv_mul_quat(Q q1, Q q2) {                                               // :432
  V3 t1 = cross(q2.v, q1.v);
  V3 t2 = mul_add(t1, q1.s, q2.v);
  V3 t3 = mul_sub(t2, q2.s, q1.v);
  return quat(t3, q1.s * q2.s + dot(q1.v, q2.v));
}
inline Q conjugate(Q q) { return quat(v3(-q.v.x, -q.v.y, -q.v.z), q.s); }
inline Q normalize_quat(Q q) {                                                    // :450
  real ls = dot_quat(q, q);
  if (ls > 1000.0f * kMinPositive) {
    real s = 1.0f / std::sqrt(ls);
    return quat(v3(s * q.v.x, s * q.v.y, s * q.v.z), s * q.s);
  }
  return qid();
}
inline real get_twist_angle(Q q) {                                               // :490
  real twist = q.s < 0.0f ? atan2_approx(-q.v.z, -q.s) : atan2_approx(q.v.z, q.s);
  return twist * 2.0f;
}

// functions.rs:518-560 transforms
inline Xf invert_xf(Xf t) { return xf(inv_rotate(t.q, -t.p), conjugate(t.q)); }
inline V3 xf_point(Xf t, V3 v) { return rotate(t.q, v) + t.p; }
inline V3 inv_xf_point(Xf t, V3 v) { return inv_rotate(t.q, v - t.p); }

// functions.rs:618-660 world positions (f64)
inline V3 sub_pos(Pos a, Pos b) {
  return v3((real)(a.x - b.x), (real)(a.y - b.y), (real)(a.z - b.z));
}
inline Pos offset_pos(Pos p, V3 d) {
  Pos r = {p.x + (double)d.x, p.y + (double)d.y, p.z + (double)d.z};
  return r;
}
inline Pos world_point(WXf t, V3 p) { return offset_pos(t.p, rotate(t.q, p)); }
inline V3 inv_world_point(WXf t, Pos p) { return inv_rotate(t.q, sub_pos(p, t.p)); }
inline Xf inv_mul_wxf(WXf a, WXf b) { return xf(inv_world_point(a, b.p), inv_mul_quat(a.q, b.q)); }

// functions.rs:575-603 directed rounding at the f64->f32 boundary
inline real round_down(double x) {
  real f = (real)x;
  if ((double)f > x) f = std::nextafter(f, -INFINITY);
  return f;
}
inline real round_up(double x) {
  real f = (real)x;
  if ((double)f < x) f = std::nextafter(f, INFINITY);
  return f;
}
inline AABB offset_aabb(AABB b, Pos o) {                                          // :667
  return aabb(v3(round_down(o.x + (double)b.lo.x), round_down(o.y + (double)b.lo.y),
                 round_down(o.z + (double)b.lo.z)),
              v3(round_up(o.x + (double)b.hi.x), round_up(o.y + (double)b.hi.y),
                 round_up(o.z + (double)b.hi.z)));
}

// functions.rs:706-832 matrices
inline real det(M3 m) { return dot(m.cx, cross(m.cy, m.cz)); }
inline V3 mul_mv(M3 m, V3 a) {
  return v3(m.cx.x * a.x + m.cy.x * a.y + m.cz.x * a.z,
            m.cx.y * a.x + m.cy.y * a.y + m.cz.y * a.z,
            m.cx.z * a.x + m.cy.z * a.y + m.cz.z * a.z);
}
inline M3 add_mm(M3 a, M3 b) { return m3(a.cx + b.cx, a.cy + b.cy, a.cz + b.cz); }
inline M3 sub_mm(M3 a, M3 b) { return m3(a.cx - b.cx, a.cy - b.cy, a.cz - b.cz); }
inline M3 mul_sm(real s, M3 a) { return m3(s * a.cx, s * a.cy, s * a.cz); }
inline M3 mul_mm(M3 a, M3 b) { return m3(mul_mv(a, b.cx), mul_mv(a, b.cy), mul_mv(a, b.cz)); }
inline M3 transpose(M3 m) {
  return m3(v3(m.cx.x, m.cy.x, m.cz.x), v3(m.cx.y, m.cy.y, m.cz.y), v3(m.cx.z, m.cy.z, m.cz.z));
}
inline M3 invert_matrix(M3 m) {                                                   // :774
  real d = det(m);
  if (absf(d) > 1000.0f * kMinPositive) {
    real inv_d = 1.0f / d;
    M3 out = m3(inv_d * cross(m.cy, m.cz), inv_d * cross(m.cz, m.cx), inv_d * cross(m.cx, m.cy));
    return transpose(out);
  }
  return m3zero();
}
inline V3 solve3(M3 m, V3 a) {                                                    // :783
  real d = det(m);
  if (absf(d) > 1000.0f * kMinPositive) {
    real inv_d = 1.0f / d;
    V3 sx = cross(m.cy, m.cz), sy = cross(m.cz, m.cx), sz = cross(m.cx, m.cy);
    return v3(inv_d * dot(sx, a), inv_d * dot(sy, a), inv_d * dot(sz, a));
  }
  return v3(0, 0, 0);
}
inline M3 invert_t(M3 m) {                                                        // :800
  real d = det(m);
  if (absf(d) > 1000.0f * kMinPositive) {
    real inv_d = 1.0f / d;
    return m3(inv_d * cross(m.cy, m.cz), inv_d * cross(m.cz, m.cx), inv_d * cross(m.cx, m.cy));
  }
  return m3zero();
}
inline M3 abs_m3(M3 m) { return m3(abs3(m.cx), abs3(m.cy), abs3(m.cz)); }
inline M3 matrix_from_quat(Q q) {                                                 // :821
  real xx = q.v.x * q.v.x, yy = q.v.y * q.v.y, zz = q.v.z * q.v.z;
  real xy = q.v.x * q.v.y, xz = q.v.x * q.v.z, xw = q.v.x * q.s;
  real yz = q.v.y * q.v.z, yw = q.v.y * q.s, zw = q.v.z * q.s;
  return m3(v3(1.0f - 2.0f * (yy + zz), 2.0f * (xy + zw), 2.0f * (xz - yw)),
            v3(2.0f * (xy - zw), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + xw)),
            v3(2.0f * (xz + yw), 2.0f * (yz - xw), 1.0f - 2.0f * (xx + yy)));
}
inline M3 diag(real a, real b, real c) {
  return m3(v3(a, 0, 0), v3(0, b, 0), v3(0, 0, c));
}
inline M3 identity_m3() { return diag(1.0f, 1.0f, 1.0f); }

// functions.rs:855-925 AABB helpers
inline bool aabb_contains(AABB a, AABB b) {
  if (a.lo.x > b.lo.x || b.hi.x > a.hi.x) return false;
  if (a.lo.y > b.lo.y || b.hi.y > a.hi.y) return false;
  if (a.lo.z > b.lo.z || b.hi.z > a.hi.z) return false;
  return true;
}
inline V3 aabb_center(AABB a) { return 0.5f * (a.hi + a.lo); }
inline V3 aabb_extents(AABB a) { return 0.5f * (a.hi - a.lo); }
inline AABB aabb_inflate(AABB a, real e) {
  V3 r = v3(e, e, e);
  return aabb(a.lo - r, a.hi + r);
}
inline bool aabb_overlaps(AABB a, AABB b) {                                       // :903
  if (a.hi.x < b.lo.x || a.lo.x > b.hi.x) return false;
  if (a.hi.y < b.lo.y || a.lo.y > b.hi.y) return false;
  if (a.hi.z < b.lo.z || a.lo.z > b.hi.z) return false;
  return true;
}
inline AABB aabb_transform(Xf t, AABB a) {                                        // :918
  V3 c = xf_point(t, aabb_center(a));
  M3 m = matrix_from_quat(t.q);
  V3 e = mul_mv(abs_m3(m), aabb_extents(a));
  return aabb(c - e, c + e);
}

// functions.rs:993 make_quat_from_matrix; :1029 compute_quat_between_unit_vectors
inline Q quat_between_unit_vectors(V3 v1, V3 v2) {
  Q out = quat(v3(0, 0, 0), 0.0f);
  V3 m = lerp(v1, v2, 0.5f);
  real tol = 100.0f * kEps;
  if (length_sq(m) > tol * tol) {
    out.v = cross(v1, m);
    out.s = dot(v1, m);
  } else {
    if (absf(v1.x) > 0.5f) {
      out.v = v3(v1.y, -v1.x, 0.0f);
    } else {
      out.v = v3(0.0f, v1.z, -v1.y);
    }
    out.s = 0.0f;
  }
  return normalize_quat(out);
}

struct SegResult { V3 p1, p2; real f1, f2; };

inline SegResult line_distance(V3 p1, V3 d1, V3 p2, V3 d2) {                      // :1069
  SegResult r;
  real a11 = dot(d1, d1), a12 = -dot(d1, d2), a21 = dot(d2, d1), a22 = -dot(d2, d2);
  V3 w = p1 - p2;
  real b1 = -dot(d1, w), b2 = -dot(d2, w);
  real d = a11 * a22 - a12 * a21;
  if (d * d < 1000.0f * kMinPositive) {
    real s1 = dot(p2 - p1, d1) / dot(d1, d1);
    r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = p2; r.f2 = 0.0f;
    return r;
  }
  real s1 = (a22 * b1 - a12 * b2) / d;
  real s2 = (a11 * b2 - a21 * b1) / d;
  r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = mul_add(p2, s2, d2); r.f2 = s2;
  return r;
}

inline SegResult segment_distance(V3 p1, V3 q1, V3 p2, V3 q2) {                   // :1105
  SegResult r;
  V3 d1 = q1 - p1, d2 = q2 - p2, rr = p1 - p2;
  real a = dot(d1, d1), b = dot(d1, d2), c = dot(d1, rr), e = dot(d2, d2), f = dot(d2, rr);
  if (a < 100.0f * kEps && e < 100.0f * kEps) {
    r.p1 = p1; r.f1 = 0; r.p2 = p2; r.f2 = 0; return r;
  }
  if (a < 100.0f * kEps) {
    real s2 = clampf(f / e, 0.0f, 1.0f);
    r.p1 = p1; r.f1 = 0; r.p2 = mul_add(p2, s2, d2); r.f2 = s2; return r;
  }
  if (e < 100.0f * kEps) {
    real s1 = clampf(-c / a, 0.0f, 1.0f);
    r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = p2; r.f2 = 0; return r;
  }
  real denom = a * e - b * b;
  real s1 = denom > 1000.0f * kMinPositive ? clampf((b * f - c * e) / denom, 0.0f, 1.0f) : 0.0f;
  real s2 = (b * s1 + f) / e;
  if (s2 < 0.0f) {
    s1 = clampf(-c / a, 0.0f, 1.0f);
    s2 = 0.0f;
  } else if (s2 > 1.0f) {
    s1 = clampf((b - c) / a, 0.0f, 1.0f);
    s2 = 1.0f;
  }
  r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = mul_add(p2, s2, d2); r.f2 = s2;
  return r;
}

inline V3 point_to_segment(V3 a, V3 b, V3 q) {                                    // :1169
  V3 ab = b - a, aq = q - a;
  real alpha = dot(ab, aq);
  if (alpha <= 0.0f) return a;
  real den = dot(ab, ab);
  if (alpha > den) return b;
  alpha /= den;
  return mul_add(a, alpha, ab);
}

inline M3 steiner(real mass, V3 o) {                                             // :1189
  real ixx = mass * (o.y * o.y + o.z * o.z);
  real iyy = mass * (o.x * o.x + o.z * o.z);
  real izz = mass * (o.x * o.x + o.y * o.y);
  real ixy = -mass * o.x * o.y;
  real ixz = -mass * o.x * o.z;
  real iyz = -mass * o.y * o.z;
  return m3(v3(ixx, ixy, ixz), v3(ixy, iyy, iyz), v3(ixz, iyz, izz));
}

// collision/internal_math.rs
inline real dot2(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline V2 mul_mv2(M2 m, V2 a) { return v2(m.cx.x * a.x + m.cy.x * a.y, m.cx.y * a.x + m.cy.y * a.y); }
inline M2 invert2(M2 m) {                                                         // :183
  real d = m.cx.x * m.cy.y - m.cx.y * m.cy.x;
  M2 r;
  if (absf(d) > 1000.0f * kMinPositive) {
    real inv = 1.0f / d;
    r.cx = v2(inv * m.cy.y, -inv * m.cx.y);
    r.cy = v2(-inv * m.cy.x, inv * m.cx.x);
  } else {
    r.cx = v2(0, 0); r.cy = v2(0, 0);
  }
  return r;
}
inline V2 solve2(M2 m, V2 b) {                                                    // :197
  real d = m.cx.x * m.cy.y - m.cx.y * m.cy.x;
  if (d > 1000.0f * kMinPositive) {
    real inv = 1.0f / d;
    return v2(inv * m.cy.y * b.x - inv * m.cy.x * b.y, -inv * m.cx.y * b.x + inv * m.cx.x * b.y);
  }
  return v2(0, 0);
}
inline V3 modified_cross(V3 a, V3 b) {                                            // :258
  return v3(a.y * b.z + a.z * b.y, a.z * b.x + a.x * b.z, a.x * b.y + a.y * b.x);
}
inline V3 arbitrary_perp(V3 v) {                                                  // :278
  V3 p;
  if (v.x < -0.5f || v.x > 0.5f) {
    const real a = 0.67f, b = -0.42f;
    p = v3(a * v.y + b * v.z, -a * v.x, -b * v.x);
  } else if (v.y < -0.5f || v.y > 0.5f) {
    const real a = 0.67f, c = -0.42f;
    p = v3(a * v.y, -a * v.x + c * v.z, -c * v.y);
  } else {
    const real a = 0.67f, b = -0.42f;
    p = v3(a * v.z, b * v.z, -a * v.x - b * v.y);
  }
  return normalize(p);
}
inline real scalar_triple(V3 a, V3 b, V3 c) {                                    // :299
  V3 d = v3(b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x);
  return a.x * d.x + a.y * d.y + a.z * d.z;
}
inline Q integrate_rotation(Q q1, V3 dr) {                                        // :322
  Q qd = mul_quat(quat(0.5f * dr, 0.0f), q1);
  return normalize_quat(quat(q1.v + qd.v, qd.s + q1.s));
}
inline Plane plane_from_normal_point(V3 n, V3 p) { return plane(n, dot(n, p)); }
inline Plane transform_plane(Xf t, Plane p) {                                     // :356
  V3 n = rotate(t.q, p.n);
  return plane(n, p.off + dot(n, t.p));
}
inline real plane_sep(Plane p, V3 x) { return dot(p.n, x) - p.off; }            // :362
inline M3 rotate_inertia(Q q, M3 c) {                                             // :378
  M3 r = matrix_from_quat(q);
  return mul_mm(r, mul_mm(c, transpose(r)));
}

}  // namespace nso
