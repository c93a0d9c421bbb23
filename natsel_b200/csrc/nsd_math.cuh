// Device/host math for the natsel_b200 step kernels. Every helper keeps the
// operand order of the reference solver (simulation and collision math in
// the reference's math/functions.rs and collision/internal_math.rs) so the
// kernels, compiled with --fmad=false and IEEE division/square root, produce
// the reference's f32 bits.
#pragma once
#include <cstdint>
#include <cfloat>
#include <cmath>
#include <cuda_runtime.h>

#define NSD_HD __host__ __device__ __forceinline__

namespace nsd {


constexpr float kPi = 3.14159265359f;             // base/constants.rs:6
constexpr float kMinPositive = FLT_MIN;           // f32::MIN_POSITIVE
constexpr float kEps = FLT_EPSILON;               // f32::EPSILON
constexpr float kFltMax = FLT_MAX;
constexpr int kNull = -1;
constexpr int kGraphColorCount = 24;              // constants.rs:23
constexpr int kOverflowIndex = kGraphColorCount - 1;      // constraint_graph.rs:20
constexpr int kDynamicColorCount = kGraphColorCount - 4;  // constraint_graph.rs:23
constexpr float kMaxRotation = 0.25f * kPi;       // constants.rs:28
constexpr float kRecycleAngular = 0.99240388f;    // constants.rs:29
constexpr float kAabbMarginFraction = 0.125f;     // constants.rs:30
constexpr float kMinFrictionWeight = 1e-10f;      // constants.rs:26
constexpr float kParallelEdgeTol = 0.005f;        // constants.rs:39

// Length-unit dependent values (reference base/constants.rs:79-121) are computed at run time in the reference
// (constants.rs:79-121), so they are computed the same way here.
NSD_HD float length_units() { return 1.0f; }
NSD_HD float linear_slop() { return 0.005f * length_units(); }
NSD_HD float speculative_distance() { return 4.0f * linear_slop(); }
NSD_HD float contact_recycle_distance() { return 10.0f * linear_slop(); }
NSD_HD float max_aabb_margin() { return 0.05f * length_units(); }
NSD_HD float huge_value() { return 1.0e5f * length_units(); }
NSD_HD float min_capsule_length() { return linear_slop(); }

struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct Q { V3 v; float s; };
struct M3 { V3 cx, cy, cz; };
struct M2 { V2 cx, cy; };
struct Pos { double x, y, z; };
struct Xf { V3 p; Q q; };
struct WXf { Pos p; Q q; };
struct AABB { V3 lo, hi; };
struct Plane { V3 n; float off; };

NSD_HD V2 v2(float x, float y) { V2 r = {x, y}; return r; }
NSD_HD V3 v3(float x, float y, float z) { V3 r = {x, y, z}; return r; }
NSD_HD Q quat(V3 v, float s) { Q r = {v, s}; return r; }
NSD_HD Q qid() { return quat(v3(0, 0, 0), 1.0f); }
NSD_HD M3 m3(V3 a, V3 b, V3 c) { M3 r = {a, b, c}; return r; }
NSD_HD M3 m3zero() { return m3(v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0)); }
NSD_HD Xf xf(V3 p, Q q) { Xf r = {p, q}; return r; }
NSD_HD Plane plane(V3 n, float o) { Plane r = {n, o}; return r; }
NSD_HD AABB aabb(V3 lo, V3 hi) { AABB r = {lo, hi}; return r; }

// functions.rs:16-60 -- ties return the second operand.
NSD_HD int min_i(int a, int b) { return a < b ? a : b; }
NSD_HD int max_i(int a, int b) { return a > b ? a : b; }
NSD_HD float absf(float a) { return a < 0.0f ? -a : a; }
NSD_HD float minf(float a, float b) { return a < b ? a : b; }
NSD_HD float maxf(float a, float b) { return a > b ? a : b; }
NSD_HD float clampf(float a, float lo, float hi) { return a < lo ? lo : (hi < a ? hi : a); }

// functions.rs:68 atan2_approx (polynomial, not libm)
NSD_HD float atan2_approx(float y, float x) {
  if (x == 0.0f && y == 0.0f) return 0.0f;
  float ax = absf(x), ay = absf(y);
  float mx = maxf(ay, ax), mn = minf(ay, ax);
  float a = mn / mx;
  float s = a * a, c = s * a, q = s * s;
  float r = 0.024840285f * q + 0.18681418f;
  float t = -0.094097948f * q - 0.33213072f;
  r = r * s + t;
  r = r * c + a;
  if (ay > ax) r = 1.57079637f - r;
  if (x < 0.0f) r = 3.14159274f - r;
  if (y < 0.0f) r = -r;
  return r;
}

// functions.rs:147-245 vector operators
NSD_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
NSD_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
NSD_HD V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
NSD_HD V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
NSD_HD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }

NSD_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }       // :250
NSD_HD float length(V3 v) { return sqrtf(dot(v, v)); }                        // :256
NSD_HD float length_sq(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }      // :262
NSD_HD float distance(V3 a, V3 b) { return length(v3(b.x - a.x, b.y - a.y, b.z - a.z)); }
NSD_HD float distance_sq(V3 a, V3 b) {                                            // :274
  V3 d = v3(b.x - a.x, b.y - a.y, b.z - a.z);
  return d.x * d.x + d.y * d.y + d.z * d.z;
}
NSD_HD V3 normalize(V3 a) {                                                       // :281
  float ls = a.x * a.x + a.y * a.y + a.z * a.z;
  if (ls > 1000.0f * kMinPositive) {
    float s = 1.0f / sqrtf(ls);
    return v3(s * a.x, s * a.y, s * a.z);
  }
  return v3(0, 0, 0);
}
NSD_HD float get_length_and_normalize(V3 a, V3* out) {                            // :293
  float ls = a.x * a.x + a.y * a.y + a.z * a.z;
  if (ls > 1000.0f * kMinPositive) {
    float l = sqrtf(ls);
    float s = 1.0f / l;
    *out = v3(s * a.x, s * a.y, s * a.z);
    return l;
  }
  *out = v3(0, 0, 0);
  return 0.0f;
}
NSD_HD V3 perp(V3 a) {                                                            // :306
  V3 p = (a.x < -0.5f || 0.5f < a.x) ? v3(a.y, -a.x, 0.0f) : v3(0.0f, a.z, -a.y);
  return normalize(p);
}
NSD_HD bool is_normalized(V3 a) { return absf(1.0f - dot(a, a)) < 100.0f * kEps; }
NSD_HD V3 mul_add(V3 a, float s, V3 b) { return v3(a.x + s * b.x, a.y + s * b.y, a.z + s * b.z); }  // :322
NSD_HD V3 mul_sub(V3 a, float s, V3 b) { return v3(a.x - s * b.x, a.y - s * b.y, a.z - s * b.z); }  // :328
NSD_HD V3 cross(V3 a, V3 b) {                                                     // :333
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
NSD_HD V3 lerp(V3 a, V3 b, float t) {                                             // :342
  return v3((1.0f - t) * a.x + t * b.x, (1.0f - t) * a.y + t * b.y, (1.0f - t) * a.z + t * b.z);
}
NSD_HD V3 blend2(float s, V3 a, float t, V3 b) {                                  // :353
  return v3(s * a.x + t * b.x, s * a.y + t * b.y, s * a.z + t * b.z);
}
NSD_HD V3 blend3(float s, V3 a, float t, V3 b, float u, V3 c) {                   // internal_math.rs:249
  return v3(s * a.x + t * b.x + u * c.x, s * a.y + t * b.y + u * c.y, s * a.z + t * b.z + u * c.z);
}
NSD_HD V3 abs3(V3 a) { return v3(absf(a.x), absf(a.y), absf(a.z)); }
NSD_HD V3 min3(V3 a, V3 b) { return v3(minf(a.x, b.x), minf(a.y, b.y), minf(a.z, b.z)); }
NSD_HD V3 max3(V3 a, V3 b) { return v3(maxf(a.x, b.x), maxf(a.y, b.y), maxf(a.z, b.z)); }

// functions.rs:402-450 quaternions
NSD_HD V3 rotate(Q q, V3 v) {
  V3 t1 = cross(q.v, v);
  V3 t2 = mul_add(t1, q.s, v);
  V3 t3 = cross(q.v, t2);
  return mul_add(v, 2.0f, t3);
}
NSD_HD V3 inv_rotate(Q q, V3 v) {
  V3 t1 = cross(q.v, v);
  V3 t2 = mul_sub(t1, q.s, v);
  V3 t3 = cross(q.v, t2);
  return mul_add(v, 2.0f, t3);
}
NSD_HD float dot_quat(Q a, Q b) { return a.v.x * b.v.x + a.v.y * b.v.y + a.v.z * b.v.z + a.s * b.s; }
NSD_HD Q mul_quat(Q q1, Q q2) {                                                   // :423
  V3 t1 = cross(q1.v, q2.v);
  V3 t2 = mul_add(t1, q1.s, q2.v);
  V3 t3 = mul_add(t2, q2.s, q1.v);
  return quat(t3, q1.s * q2.s - dot(q1.v, q2.v));
}
NSD_HD Q inv_mul_quat(Q q1, Q q2) {                                               // :432
  V3 t1 = cross(q2.v, q1.v);
  V3 t2 = mul_add(t1, q1.s, q2.v);
  V3 t3 = mul_sub(t2, q2.s, q1.v);
  return quat(t3, q1.s * q2.s + dot(q1.v, q2.v));
}
NSD_HD Q conjugate(Q q) { return quat(v3(-q.v.x, -q.v.y, -q.v.z), q.s); }
NSD_HD Q normalize_quat(Q q) {                                                    // :450
  float ls = dot_quat(q, q);
  if (ls > 1000.0f * kMinPositive) {
    float s = 1.0f / sqrtf(ls);
    return quat(v3(s * q.v.x, s * q.v.y, s * q.v.z), s * q.s);
  }
  return qid();
}
// internal_math.rs:328 delta_quat_to_rotation
NSD_HD V3 delta_quat_to_rotation(Q q, Q target) {
  Q s = dot_quat(q, target) < 0.0f ? quat(v3(-q.v.x, -q.v.y, -q.v.z), -q.s) : q;
  Q diff = quat(target.v - s.v, target.s - s.s);
  Q product = mul_quat(diff, conjugate(s));
  return 2.0f * product.v;
}
NSD_HD float get_swing_angle(Q q) {                                               // :502
  float x = sqrtf(q.v.z * q.v.z + q.s * q.s);
  float y = sqrtf(q.v.x * q.v.x + q.v.y * q.v.y);
  return 2.0f * atan2_approx(y, x);
}
NSD_HD float get_twist_angle(Q q) {                                               // :490
  float twist = q.s < 0.0f ? atan2_approx(-q.v.z, -q.s) : atan2_approx(q.v.z, q.s);
  return twist * 2.0f;
}

// functions.rs:518-560 transforms
NSD_HD Xf invert_xf(Xf t) { return xf(inv_rotate(t.q, -t.p), conjugate(t.q)); }
NSD_HD V3 xf_point(Xf t, V3 v) { return rotate(t.q, v) + t.p; }
NSD_HD V3 inv_xf_point(Xf t, V3 v) { return inv_rotate(t.q, v - t.p); }

// functions.rs:618-660 world positions (f64)
NSD_HD V3 sub_pos(Pos a, Pos b) {
  return v3((float)(a.x - b.x), (float)(a.y - b.y), (float)(a.z - b.z));
}
NSD_HD Pos offset_pos(Pos p, V3 d) {
  Pos r = {p.x + (double)d.x, p.y + (double)d.y, p.z + (double)d.z};
  return r;
}
NSD_HD Pos world_point(WXf t, V3 p) { return offset_pos(t.p, rotate(t.q, p)); }
NSD_HD V3 inv_world_point(WXf t, Pos p) { return inv_rotate(t.q, sub_pos(p, t.p)); }
NSD_HD Xf inv_mul_wxf(WXf a, WXf b) { return xf(inv_world_point(a, b.p), inv_mul_quat(a.q, b.q)); }

// functions.rs:575-603 directed rounding at the f64->f32 boundary
NSD_HD float round_down(double x) {
  float f = (float)x;
  if ((double)f > x) f = nextafterf(f, -INFINITY);
  return f;
}
NSD_HD float round_up(double x) {
  float f = (float)x;
  if ((double)f < x) f = nextafterf(f, INFINITY);
  return f;
}
NSD_HD AABB offset_aabb(AABB b, Pos o) {                                          // :667
  return aabb(v3(round_down(o.x + (double)b.lo.x), round_down(o.y + (double)b.lo.y),
                 round_down(o.z + (double)b.lo.z)),
              v3(round_up(o.x + (double)b.hi.x), round_up(o.y + (double)b.hi.y),
                 round_up(o.z + (double)b.hi.z)));
}

// functions.rs:706-832 matrices
NSD_HD float det(M3 m) { return dot(m.cx, cross(m.cy, m.cz)); }
NSD_HD V3 mul_mv(M3 m, V3 a) {
  return v3(m.cx.x * a.x + m.cy.x * a.y + m.cz.x * a.z,
            m.cx.y * a.x + m.cy.y * a.y + m.cz.y * a.z,
            m.cx.z * a.x + m.cy.z * a.y + m.cz.z * a.z);
}
NSD_HD M3 add_mm(M3 a, M3 b) { return m3(a.cx + b.cx, a.cy + b.cy, a.cz + b.cz); }
NSD_HD M3 sub_mm(M3 a, M3 b) { return m3(a.cx - b.cx, a.cy - b.cy, a.cz - b.cz); }
NSD_HD M3 mul_sm(float s, M3 a) { return m3(s * a.cx, s * a.cy, s * a.cz); }
NSD_HD M3 mul_mm(M3 a, M3 b) { return m3(mul_mv(a, b.cx), mul_mv(a, b.cy), mul_mv(a, b.cz)); }
NSD_HD M3 transpose(M3 m) {
  return m3(v3(m.cx.x, m.cy.x, m.cz.x), v3(m.cx.y, m.cy.y, m.cz.y), v3(m.cx.z, m.cy.z, m.cz.z));
}
NSD_HD M3 invert_matrix(M3 m) {                                                   // :774
  float d = det(m);
  if (absf(d) > 1000.0f * kMinPositive) {
    float inv_d = 1.0f / d;
    M3 out = m3(inv_d * cross(m.cy, m.cz), inv_d * cross(m.cz, m.cx), inv_d * cross(m.cx, m.cy));
    return transpose(out);
  }
  return m3zero();
}
NSD_HD V3 solve3(M3 m, V3 a) {                                                    // :783
  float d = det(m);
  if (absf(d) > 1000.0f * kMinPositive) {
    float inv_d = 1.0f / d;
    V3 sx = cross(m.cy, m.cz), sy = cross(m.cz, m.cx), sz = cross(m.cx, m.cy);
    return v3(inv_d * dot(sx, a), inv_d * dot(sy, a), inv_d * dot(sz, a));
  }
  return v3(0, 0, 0);
}
NSD_HD M3 invert_t(M3 m) {                                                        // :800
  float d = det(m);
  if (absf(d) > 1000.0f * kMinPositive) {
    float inv_d = 1.0f / d;
    return m3(inv_d * cross(m.cy, m.cz), inv_d * cross(m.cz, m.cx), inv_d * cross(m.cx, m.cy));
  }
  return m3zero();
}
NSD_HD M3 abs_m3(M3 m) { return m3(abs3(m.cx), abs3(m.cy), abs3(m.cz)); }
NSD_HD M3 matrix_from_quat(Q q) {                                                 // :821
  float xx = q.v.x * q.v.x, yy = q.v.y * q.v.y, zz = q.v.z * q.v.z;
  float xy = q.v.x * q.v.y, xz = q.v.x * q.v.z, xw = q.v.x * q.s;
  float yz = q.v.y * q.v.z, yw = q.v.y * q.s, zw = q.v.z * q.s;
  return m3(v3(1.0f - 2.0f * (yy + zz), 2.0f * (xy + zw), 2.0f * (xz - yw)),
            v3(2.0f * (xy - zw), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + xw)),
            v3(2.0f * (xz + yw), 2.0f * (yz - xw), 1.0f - 2.0f * (xx + yy)));
}
NSD_HD M3 diag(float a, float b, float c) {
  return m3(v3(a, 0, 0), v3(0, b, 0), v3(0, 0, c));
}
NSD_HD M3 identity_m3() { return diag(1.0f, 1.0f, 1.0f); }

// functions.rs:855-925 AABB helpers
NSD_HD bool aabb_contains(AABB a, AABB b) {
  if (a.lo.x > b.lo.x || b.hi.x > a.hi.x) return false;
  if (a.lo.y > b.lo.y || b.hi.y > a.hi.y) return false;
  if (a.lo.z > b.lo.z || b.hi.z > a.hi.z) return false;
  return true;
}
NSD_HD V3 aabb_center(AABB a) { return 0.5f * (a.hi + a.lo); }
NSD_HD V3 aabb_extents(AABB a) { return 0.5f * (a.hi - a.lo); }
NSD_HD AABB aabb_inflate(AABB a, float e) {
  V3 r = v3(e, e, e);
  return aabb(a.lo - r, a.hi + r);
}
NSD_HD bool aabb_overlaps(AABB a, AABB b) {                                       // :903
  if (a.hi.x < b.lo.x || a.lo.x > b.hi.x) return false;
  if (a.hi.y < b.lo.y || a.lo.y > b.hi.y) return false;
  if (a.hi.z < b.lo.z || a.lo.z > b.hi.z) return false;
  return true;
}
NSD_HD AABB aabb_transform(Xf t, AABB a) {                                        // :918
  V3 c = xf_point(t, aabb_center(a));
  M3 m = matrix_from_quat(t.q);
  V3 e = mul_mv(abs_m3(m), aabb_extents(a));
  return aabb(c - e, c + e);
}

// functions.rs:993 make_quat_from_matrix; :1029 compute_quat_between_unit_vectors
NSD_HD Q quat_between_unit_vectors(V3 v1, V3 v2) {
  Q out = quat(v3(0, 0, 0), 0.0f);
  V3 m = lerp(v1, v2, 0.5f);
  float tol = 100.0f * kEps;
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

struct SegResult { V3 p1, p2; float f1, f2; };

NSD_HD SegResult line_distance(V3 p1, V3 d1, V3 p2, V3 d2) {                      // :1069
  SegResult r;
  float a11 = dot(d1, d1), a12 = -dot(d1, d2), a21 = dot(d2, d1), a22 = -dot(d2, d2);
  V3 w = p1 - p2;
  float b1 = -dot(d1, w), b2 = -dot(d2, w);
  float d = a11 * a22 - a12 * a21;
  if (d * d < 1000.0f * kMinPositive) {
    float s1 = dot(p2 - p1, d1) / dot(d1, d1);
    r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = p2; r.f2 = 0.0f;
    return r;
  }
  float s1 = (a22 * b1 - a12 * b2) / d;
  float s2 = (a11 * b2 - a21 * b1) / d;
  r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = mul_add(p2, s2, d2); r.f2 = s2;
  return r;
}

NSD_HD SegResult segment_distance(V3 p1, V3 q1, V3 p2, V3 q2) {                   // :1105
  SegResult r;
  V3 d1 = q1 - p1, d2 = q2 - p2, rr = p1 - p2;
  float a = dot(d1, d1), b = dot(d1, d2), c = dot(d1, rr), e = dot(d2, d2), f = dot(d2, rr);
  if (a < 100.0f * kEps && e < 100.0f * kEps) {
    r.p1 = p1; r.f1 = 0; r.p2 = p2; r.f2 = 0; return r;
  }
  if (a < 100.0f * kEps) {
    float s2 = clampf(f / e, 0.0f, 1.0f);
    r.p1 = p1; r.f1 = 0; r.p2 = mul_add(p2, s2, d2); r.f2 = s2; return r;
  }
  if (e < 100.0f * kEps) {
    float s1 = clampf(-c / a, 0.0f, 1.0f);
    r.p1 = mul_add(p1, s1, d1); r.f1 = s1; r.p2 = p2; r.f2 = 0; return r;
  }
  float denom = a * e - b * b;
  float s1 = denom > 1000.0f * kMinPositive ? clampf((b * f - c * e) / denom, 0.0f, 1.0f) : 0.0f;
  float s2 = (b * s1 + f) / e;
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

NSD_HD V3 point_to_segment(V3 a, V3 b, V3 q) {                                    // :1169
  V3 ab = b - a, aq = q - a;
  float alpha = dot(ab, aq);
  if (alpha <= 0.0f) return a;
  float den = dot(ab, ab);
  if (alpha > den) return b;
  alpha /= den;
  return mul_add(a, alpha, ab);
}

NSD_HD M3 steiner(float mass, V3 o) {                                             // :1189
  float ixx = mass * (o.y * o.y + o.z * o.z);
  float iyy = mass * (o.x * o.x + o.z * o.z);
  float izz = mass * (o.x * o.x + o.y * o.y);
  float ixy = -mass * o.x * o.y;
  float ixz = -mass * o.x * o.z;
  float iyz = -mass * o.y * o.z;
  return m3(v3(ixx, ixy, ixz), v3(ixy, iyy, iyz), v3(ixz, iyz, izz));
}

// collision/internal_math.rs
NSD_HD float dot2(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
NSD_HD V2 mul_mv2(M2 m, V2 a) { return v2(m.cx.x * a.x + m.cy.x * a.y, m.cx.y * a.x + m.cy.y * a.y); }
NSD_HD M2 invert2(M2 m) {                                                         // :183
  float d = m.cx.x * m.cy.y - m.cx.y * m.cy.x;
  M2 r;
  if (absf(d) > 1000.0f * kMinPositive) {
    float inv = 1.0f / d;
    r.cx = v2(inv * m.cy.y, -inv * m.cx.y);
    r.cy = v2(-inv * m.cy.x, inv * m.cx.x);
  } else {
    r.cx = v2(0, 0); r.cy = v2(0, 0);
  }
  return r;
}
NSD_HD V2 solve2(M2 m, V2 b) {                                                    // :197
  float d = m.cx.x * m.cy.y - m.cx.y * m.cy.x;
  if (d > 1000.0f * kMinPositive) {
    float inv = 1.0f / d;
    return v2(inv * m.cy.y * b.x - inv * m.cy.x * b.y, -inv * m.cx.y * b.x + inv * m.cx.x * b.y);
  }
  return v2(0, 0);
}
NSD_HD V3 modified_cross(V3 a, V3 b) {                                            // :258
  return v3(a.y * b.z + a.z * b.y, a.z * b.x + a.x * b.z, a.x * b.y + a.y * b.x);
}
NSD_HD V3 arbitrary_perp(V3 v) {                                                  // :278
  V3 p;
  if (v.x < -0.5f || v.x > 0.5f) {
    const float a = 0.67f, b = -0.42f;
    p = v3(a * v.y + b * v.z, -a * v.x, -b * v.x);
  } else if (v.y < -0.5f || v.y > 0.5f) {
    const float a = 0.67f, c = -0.42f;
    p = v3(a * v.y, -a * v.x + c * v.z, -c * v.y);
  } else {
    const float a = 0.67f, b = -0.42f;
    p = v3(a * v.z, b * v.z, -a * v.x - b * v.y);
  }
  return normalize(p);
}
NSD_HD float scalar_triple(V3 a, V3 b, V3 c) {                                    // :299
  V3 d = v3(b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x);
  return a.x * d.x + a.y * d.y + a.z * d.z;
}
NSD_HD Q integrate_rotation(Q q1, V3 dr) {                                        // :322
  Q qd = mul_quat(quat(0.5f * dr, 0.0f), q1);
  return normalize_quat(quat(q1.v + qd.v, qd.s + q1.s));
}
NSD_HD Plane plane_from_normal_point(V3 n, V3 p) { return plane(n, dot(n, p)); }
NSD_HD Plane transform_plane(Xf t, Plane p) {                                     // :356
  V3 n = rotate(t.q, p.n);
  return plane(n, p.off + dot(n, t.p));
}
NSD_HD float plane_sep(Plane p, V3 x) { return dot(p.n, x) - p.off; }            // :362
NSD_HD M3 rotate_inertia(Q q, M3 c) {                                             // :378
  M3 r = matrix_from_quat(q);
  return mul_mm(r, mul_mm(c, transpose(r)));
}

}  // namespace nsd
