// Oracle time of impact. TEST INFRASTRUCTURE ONLY (see ns_math.hpp).
//
// Restates collision/time_of_impact.rs (conservative advancement: a GJK distance at the
// current time, a separation function built from the simplex cache, and a bisection /
// secant root finder on it) and the sweep helpers of collision/distance.rs:817-832, with the
// reference's operation order.
#pragma once
#include "ns_collide.hpp"

namespace nso {

// types/queries.rs:179 Sweep (centres relative to a base position)
struct Sweep { V3 local_center, c1, c2; Q q1, q2; };

// math/functions.rs:511 nlerp
inline Q nlerp(Q q1, Q q2, real alpha) {
  if (dot_quat(q1, q2) < 0.0f) q1 = quat(v3(-q1.v.x, -q1.v.y, -q1.v.z), -q1.s);
  V3 v = lerp(q1.v, q2.v, alpha);
  real s = (1.0f - alpha) * q1.s + alpha * q2.s;
  return normalize_quat(quat(v, s));
}

// math/functions.rs:533 inv_mul_transforms
inline Xf inv_mul_xf(Xf a, Xf b) { return xf(inv_rotate(a.q, b.p - a.p), inv_mul_quat(a.q, b.q)); }

// distance.rs:817 get_sweep_transform / :826 get_final_sweep_transform
inline Xf sweep_xf(const Sweep& s, real t) {
  Q q = nlerp(s.q1, s.q2, t);
  return xf(lerp(s.c1, s.c2, t) - rotate(q, s.local_center), q);
}
inline Xf sweep_final_xf(const Sweep& s) { return xf(s.c2 - rotate(s.q2, s.local_center), s.q2); }

// shape_runtime.rs make_shape_proxy: the shape's points and radius (a box hull's 8 corners)
struct Proxy { V3 pts[8]; int count; real radius; };

struct ToiOut { int state; real fraction, distance; V3 point, normal; int distance_iterations, push_back_iterations, root_iterations; };
enum { kToiUnknown = 0, kToiFailed, kToiOverlapped, kToiHit, kToiSeparated };

enum { kSepUnknown = 0, kSepVertices, kSepEdges, kSepFaceA, kSepFaceB };
struct SepFn { const Proxy* a; const Proxy* b; Sweep sa, sb; V3 w1, w2; int kind; };

// time_of_impact.rs:36 unique_count
inline int unique_count(int n, const int* v) {
  if (n == 1) return 1;
  if (n == 2) return v[0] != v[1] ? 2 : 1;
  if (v[0] != v[1] && v[0] != v[2] && v[1] != v[2]) return 3;
  if (v[0] == v[1] && v[0] == v[2] && v[1] == v[2]) return 1;
  return 2;
}

// time_of_impact.rs:65 check_fast_edges
inline bool check_fast_edges(Xf xa, V3 la, Xf xb, V3 lb, V3 axis0) {
  V3 ea = rotate(xa.q, la), eb = rotate(xb.q, lb);
  return dot(cross(ea, eb), axis0) < 0.0f;
}

// The edge-pair branch shared by the 2- and 3-vertex caches (time_of_impact.rs:121-158,
// :213-253) with its parallel tolerance.
inline void edge_pair_function(SepFn& f, V3 va1, V3 va2, V3 vb1, V3 vb2, Q qa, Q qb, V3 dp, V3 world_normal,
                               real tol_sq) {
  V3 lea = normalize(va2 - va1);
  V3 ea = rotate(qa, lea);
  V3 leb = normalize(vb2 - vb1);
  V3 eb = rotate(qb, leb);
  V3 axis = cross(ea, eb);
  if (length_sq(axis) < tol_sq) {
    f.kind = kSepVertices;
    f.w1 = world_normal;
    return;
  }
  V3 delta = (rotate(qb, vb1) - rotate(qa, va1)) + dp;
  if (dot(delta, axis) < 0.0f) { axis = -axis; leb = -leb; }
  if (check_fast_edges(sweep_final_xf(f.sa), lea, sweep_final_xf(f.sb), leb, axis)) {
    f.kind = kSepVertices;
    f.w1 = normalize(axis);
  } else {
    f.kind = kSepEdges;
    f.w1 = lea;
    f.w2 = leb;
  }
}

// time_of_impact.rs:78 make_separation_function
inline SepFn make_separation_function(const SimplexCache& c, const Proxy& pa, const Sweep& sa, const Proxy& pb,
                                      const Sweep& sb, V3 world_normal, real t1) {
  SepFn f;
  f.a = &pa; f.b = &pb; f.sa = sa; f.sb = sb;
  f.w1 = v3(0, 0, 0); f.w2 = v3(0, 0, 0); f.kind = kSepUnknown;
  int ia[3] = {c.ia[0], c.ia[1], c.ia[2]}, ib[3] = {c.ib[0], c.ib[1], c.ib[2]};
  int ua = unique_count(c.count, ia), ub = unique_count(c.count, ib);
  Xf xa1 = sweep_xf(sa, t1), xb1 = sweep_xf(sb, t1);
  Q qa = xa1.q, qb = xb1.q;
  V3 dp = xb1.p - xa1.p;
  const V3* A = pa.pts;
  const V3* B = pb.pts;
  if (c.count == 1) {
    f.kind = kSepVertices;
    f.w1 = world_normal;
  } else if (c.count == 2) {
    if (ua == 2 && ub == 2) {
      edge_pair_function(f, A[ia[0]], A[ia[1]], B[ib[0]], B[ib[1]], qa, qb, dp, world_normal, 0.05f * 0.05f);
    } else {
      f.kind = kSepVertices;
      f.w1 = world_normal;
    }
  } else {
    if (ua == 3) {
      V3 va1 = A[ia[0]], va2 = A[ia[1]], va3 = A[ia[2]];
      V3 lax = normalize(cross(va2 - va1, va3 - va1));
      V3 ax = rotate(qa, lax);
      V3 lpa = (1.0f / 3.0f) * ((va1 + va2) + va3);
      V3 lpb = B[ib[0]];
      V3 delta = (rotate(qb, lpb) - rotate(qa, lpa)) + dp;
      if (dot(delta, ax) < 0.0f) lax = -lax;
      f.kind = kSepFaceA;
      f.w1 = lax;
      f.w2 = lpa;
    } else if (ub == 3) {
      V3 vb1 = B[ib[0]], vb2 = B[ib[1]], vb3 = B[ib[2]];
      V3 lbx = normalize(cross(vb2 - vb1, vb3 - vb1));
      V3 bx = rotate(qb, lbx);
      V3 lpa = A[ia[0]];
      V3 lpb = (1.0f / 3.0f) * ((vb1 + vb2) + vb3);
      V3 delta = (rotate(qa, lpa) - rotate(qb, lpb)) - dp;
      if (dot(delta, bx) < 0.0f) lbx = -lbx;
      f.kind = kSepFaceB;
      f.w1 = lbx;
      f.w2 = lpb;
    } else {
      if (ia[0] == ia[1]) ia[1] = ia[2];
      if (ib[0] == ib[1]) ib[1] = ib[2];
      edge_pair_function(f, A[ia[0]], A[ia[1]], B[ib[0]], B[ib[1]], qa, qb, dp, world_normal, 0.005f * 0.005f);
    }
  }
  return f;
}

// distance.rs:39 get_point_support is point_support (ns_collide.hpp)

// time_of_impact.rs:266 find_min_separation
inline real find_min_separation(const SepFn& f, int* ia, int* ib, real t) {
  Xf xa = sweep_xf(f.sa, t), xb = sweep_xf(f.sb, t);
  const V3* A = f.a->pts;
  const V3* B = f.b->pts;
  switch (f.kind) {
    case kSepVertices: {
      V3 axis = f.w1;
      *ia = point_support(A, f.a->count, inv_rotate(xa.q, axis));
      *ib = point_support(B, f.b->count, inv_rotate(xb.q, -axis));
      V3 dp = xb.p - xa.p;
      V3 delta = (rotate(xb.q, B[*ib]) - rotate(xa.q, A[*ia])) + dp;
      return dot(delta, axis);
    }
    case kSepEdges: {
      V3 ea = rotate(xa.q, f.w1), eb = rotate(xb.q, f.w2);
      V3 axis = normalize(cross(ea, eb));
      *ia = point_support(A, f.a->count, inv_rotate(xa.q, axis));
      V3 axb = inv_rotate(xb.q, axis);
      *ib = point_support(B, f.b->count, -axb);
      V3 dp = xb.p - xa.p;
      V3 delta = (rotate(xb.q, B[*ib]) - rotate(xa.q, A[*ia])) + dp;
      return dot(delta, axis);
    }
    case kSepFaceA: {
      V3 n = rotate(xa.q, f.w1);
      *ia = -1;
      V3 p_a = xf_point(xa, f.w2);
      V3 axb = inv_rotate(xb.q, n);
      *ib = point_support(B, f.b->count, -axb);
      V3 p_b = xf_point(xb, B[*ib]);
      return dot(p_b - p_a, n);
    }
    case kSepFaceB: {
      V3 n = rotate(xb.q, f.w1);
      V3 axa = inv_rotate(xa.q, n);
      *ia = point_support(A, f.a->count, -axa);
      V3 p_a = xf_point(xa, A[*ia]);
      *ib = -1;
      V3 p_b = xf_point(xb, f.w2);
      return dot(p_a - p_b, n);
    }
  }
  return 0.0f;
}

// time_of_impact.rs:331 evaluate_separation
inline real evaluate_separation(const SepFn& f, int i1, int i2, real beta) {
  Xf x1 = sweep_xf(f.sa, beta), x2 = sweep_xf(f.sb, beta);
  const V3* A = f.a->pts;
  const V3* B = f.b->pts;
  switch (f.kind) {
    case kSepVertices: return dot(xf_point(x2, B[i2]) - xf_point(x1, A[i1]), f.w1);
    case kSepEdges: {
      V3 e1 = rotate(x1.q, f.w1), e2 = rotate(x2.q, f.w2);
      V3 axis = normalize(cross(e1, e2));
      return dot(xf_point(x2, B[i2]) - xf_point(x1, A[i1]), axis);
    }
    case kSepFaceA: {
      V3 axis = rotate(x1.q, f.w1);
      return dot(xf_point(x2, B[i2]) - xf_point(x1, f.w2), axis);
    }
    case kSepFaceB: {
      V3 axis = rotate(x2.q, f.w1);
      return dot(xf_point(x1, A[i1]) - xf_point(x2, f.w2), axis);
    }
  }
  return 0.0f;
}

// time_of_impact.rs:375 force_fixed_axis
inline void force_fixed_axis(SepFn& f, real beta) {
  Xf x1 = sweep_xf(f.sa, beta), x2 = sweep_xf(f.sb, beta);
  V3 e1 = rotate(x1.q, f.w1), e2 = rotate(x2.q, f.w2);
  f.kind = kSepVertices;
  f.w1 = normalize(cross(e1, e2));
  f.w2 = v3(0, 0, 0);
}

// The witness point and normal of a finished query (time_of_impact.rs:459-483, :586-590).
inline void toi_point(ToiOut& o, V3 wpa, V3 wpb, V3 wn, real ra, real rb, V3 origin) {
  V3 pa = mul_add(wpa, ra, wn), pb = mul_add(wpb, -rb, wn);
  o.point = lerp(pa, pb, 0.5f) + origin;
  o.normal = wn;
}

// time_of_impact.rs:391 time_of_impact
inline ToiOut time_of_impact(const Proxy& pa, const Proxy& pb, Sweep sa, Sweep sb, real t_max) {
  ToiOut o;
  o.state = kToiUnknown; o.fraction = -1.0f; o.distance = 0.0f;
  o.point = v3(0, 0, 0); o.normal = v3(0, 0, 0);
  o.distance_iterations = o.push_back_iterations = o.root_iterations = 0;
  V3 origin = sa.c1;
  sa.c1 = v3(0, 0, 0);
  sa.c2 = sa.c2 - origin;
  sb.c1 = sb.c1 - origin;
  sb.c2 = sb.c2 - origin;
  int max_push = pa.count + pb.count;
  real slop = linear_slop();
  real total_radius = pa.radius + pb.radius;
  real target = maxf(slop, total_radius - slop);
  real tol = 0.25f * slop;
  real t1 = 0.0f;
  const int max_iterations = 25;
  int distance_iterations = 0;
  SimplexCache cache;
  for (;;) {
    Xf xa = sweep_xf(sa, t1), xb = sweep_xf(sb, t1);
    DistOut d = shape_distance(pa.pts, pa.count, pb.pts, pb.count, inv_mul_xf(xa, xb), &cache);
    o.distance = d.distance;
    V3 wn = rotate(xa.q, d.normal);
    V3 wpa = xf_point(xa, d.pa);
    V3 wpb = xf_point(xa, d.pb);
    o.distance_iterations += 1;
    distance_iterations += 1;
    if (d.distance <= 0.0f) {
      o.state = kToiOverlapped;
      o.fraction = 0.0f;
      toi_point(o, wpa, wpb, wn, pa.radius, pb.radius, origin);
      break;
    }
    if (d.distance <= target + tol) {
      o.state = kToiHit;
      toi_point(o, wpa, wpb, wn, pa.radius, pb.radius, origin);
      o.fraction = t1;
      break;
    }
    if (distance_iterations == max_iterations) {
      o.state = kToiFailed;
      o.fraction = t1;
      toi_point(o, wpa, wpb, wn, pa.radius, pb.radius, origin);
      break;
    }
    SepFn f = make_separation_function(cache, pa, sa, pb, sb, wn, t1);
    bool done = false;
    real t2 = t_max;
    int push_iterations = 0;
    for (;;) {
      int ia = 0, ib = 0;
      real s2 = find_min_separation(f, &ia, &ib, t2);
      if (s2 - target > tol) {
        o.state = kToiSeparated;
        o.fraction = t_max;
        done = true;
        break;
      }
      if (s2 >= target - tol) {
        t1 = t2;
        break;
      }
      real s1 = evaluate_separation(f, ia, ib, t1);
      if (s1 < target - tol) {
        o.state = kToiFailed;
        o.fraction = t1;
        done = true;
        break;
      }
      if (s1 <= target + tol) {
        o.state = kToiHit;
        o.fraction = t1;
        done = true;
        break;
      }
      int root_iterations = 0;
      const int max_root_iterations = 50;
      real a1 = t1, a2 = t2;
      for (;;) {
        real t = (root_iterations & 1) ? a1 + (target - s1) * (a2 - a1) / (s2 - s1) : 0.5f * (a1 + a2);
        o.root_iterations += 1;
        root_iterations += 1;
        real s = evaluate_separation(f, ia, ib, t);
        if (absf(s - target) <= tol) {
          t2 = t;
          break;
        }
        if (s > target) {
          a1 = t;
          s1 = s;
        } else {
          a2 = t;
          s2 = s;
        }
        if (root_iterations == max_root_iterations) break;
      }
      if (root_iterations == max_root_iterations - 1 && f.kind == kSepEdges) {
        root_iterations = 0;
        t2 = t_max;
        force_fixed_axis(f, t1);
      }
      o.push_back_iterations += 1;
      push_iterations += 1;
      if (push_iterations == max_push) break;
    }
    if (done) {
      toi_point(o, wpa, wpb, wn, pa.radius, pb.radius, origin);
      break;
    }
  }
  return o;
}

}  // namespace nso
