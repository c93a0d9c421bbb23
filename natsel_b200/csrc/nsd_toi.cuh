// Time of impact on the device: conservative advancement of two convex proxies along their
// sweeps (collision/time_of_impact.rs:391 time_of_impact), used by the continuous pass of fast
// bodies against static shapes (continuous.rs:337 solve_continuous).
//
// One thread runs one query. Per iteration it takes the GJK distance at the current time t1
// (shape_distance with a warm simplex cache), and, while the shapes are farther apart than
// the target (linear slop below the summed radii), builds a separation function from the
// cache's support features and advances t1 to the root of that function with a bisection /
// secant alternation. Every loop has the reference's iteration cap (25 distance queries,
// proxy_a.count + proxy_b.count push-backs, 50 root steps), so a query always ends. The f32
// operations follow the reference's order, so the fraction it returns is the reference's.
#pragma once
#include "nsd_geom.cuh"

namespace nsd {

// types/queries.rs:179 Sweep, centres relative to a base position
struct Sweep { V3 local_center, c1, c2; Q q1, q2; };

// A convex proxy: up to 8 points (a box hull's corners) and a radius (shape_runtime.rs:643)
struct Proxy { V3 pts[8]; int count; float radius; };

enum ToiState { kToiUnknown = 0, kToiFailed, kToiOverlapped, kToiHit, kToiSeparated };
struct ToiResult {
  int state;
  float fraction, distance;
  V3 point, normal;
  int distance_iterations, push_back_iterations, root_iterations;
};

// math/functions.rs:511 nlerp: the shorter arc, then a normalised linear blend
NSD_HD Q nlerp(Q a, Q b, float t) {
  if (dot_quat(a, b) < 0.0f) a = quat(v3(-a.v.x, -a.v.y, -a.v.z), -a.s);
  V3 v = lerp(a.v, b.v, t);
  float s = (1.0f - t) * a.s + t * b.s;
  return normalize_quat(quat(v, s));
}

// distance.rs:817 get_sweep_transform and :826 get_final_sweep_transform
NSD_HD Xf sweep_at(const Sweep& s, float t) {
  Q q = nlerp(s.q1, s.q2, t);
  return xf(lerp(s.c1, s.c2, t) - rotate(q, s.local_center), q);
}
NSD_HD Xf sweep_end(const Sweep& s) { return xf(s.c2 - rotate(s.q2, s.local_center), s.q2); }

// Separation function (time_of_impact.rs:25): kind 1 a fixed world axis through two support
// points, 2 the cross product of two body-fixed edges, 3 / 4 a face of A / B with a point on it.
enum SepKind { kSepNone = 0, kSepPoints = 1, kSepEdgePair = 2, kSepFaceOfA = 3, kSepFaceOfB = 4 };
struct SepFunc {
  const Proxy* pa;
  const Proxy* pb;
  Sweep sa, sb;
  V3 axis_or_edge_a, point_or_edge_b;
  int kind;
};

// time_of_impact.rs:36 unique_count for a simplex of n vertices
NSD_HD int distinct_indices(int n, int i0, int i1, int i2) {
  if (n == 1) return 1;
  if (n == 2) return i0 != i1 ? 2 : 1;
  if (i0 != i1 && i0 != i2 && i1 != i2) return 3;
  return (i0 == i1 && i0 == i2 && i1 == i2) ? 1 : 2;
}

// time_of_impact.rs:121-158 / :213-253: an edge pair, unless the edges are parallel within
// the tolerance (a point pair on the GJK normal) or their cross product flips over the sweep
// (a point pair on the fixed axis)
NSD_HD void set_edge_pair(SepFunc& f, V3 a1, V3 a2, V3 b1, V3 b2, Q qa, Q qb, V3 dp, V3 world_normal, float tol_sq) {
  V3 ea_local = normalize(a2 - a1);
  V3 eb_local = normalize(b2 - b1);
  V3 axis = cross(rotate(qa, ea_local), rotate(qb, eb_local));
  if (length_sq(axis) < tol_sq) {
    f.kind = kSepPoints;
    f.axis_or_edge_a = world_normal;
    return;
  }
  V3 gap = (rotate(qb, b1) - rotate(qa, a1)) + dp;
  if (dot(gap, axis) < 0.0f) {
    axis = -axis;
    eb_local = -eb_local;
  }
  // time_of_impact.rs:65 check_fast_edges at the sweeps' ends
  Xf ea_end = sweep_end(f.sa), eb_end = sweep_end(f.sb);
  bool flips = dot(cross(rotate(ea_end.q, ea_local), rotate(eb_end.q, eb_local)), axis) < 0.0f;
  if (flips) {
    f.kind = kSepPoints;
    f.axis_or_edge_a = normalize(axis);
  } else {
    f.kind = kSepEdgePair;
    f.axis_or_edge_a = ea_local;
    f.point_or_edge_b = eb_local;
  }
}

// time_of_impact.rs:78 make_separation_function
NSD_HD void build_separation(SepFunc& f, const SimplexCache& c, V3 world_normal, float t1) {
  f.axis_or_edge_a = v3(0, 0, 0);
  f.point_or_edge_b = v3(0, 0, 0);
  f.kind = kSepNone;
  int a0 = c.ia[0], a1 = c.ia[1], a2 = c.ia[2];
  int b0 = c.ib[0], b1 = c.ib[1], b2 = c.ib[2];
  int na = distinct_indices(c.count, a0, a1, a2), nb = distinct_indices(c.count, b0, b1, b2);
  Xf xa = sweep_at(f.sa, t1), xb = sweep_at(f.sb, t1);
  V3 dp = xb.p - xa.p;
  const V3* A = f.pa->pts;
  const V3* B = f.pb->pts;
  if (c.count == 1 || (c.count == 2 && !(na == 2 && nb == 2))) {
    f.kind = kSepPoints;
    f.axis_or_edge_a = world_normal;
  } else if (c.count == 2) {
    set_edge_pair(f, A[a0], A[a1], B[b0], B[b1], xa.q, xb.q, dp, world_normal, 0.05f * 0.05f);
  } else if (na == 3) {
    V3 n_local = normalize(cross(A[a1] - A[a0], A[a2] - A[a0]));
    V3 on_face = (1.0f / 3.0f) * ((A[a0] + A[a1]) + A[a2]);
    V3 gap = (rotate(xb.q, B[b0]) - rotate(xa.q, on_face)) + dp;
    if (dot(gap, rotate(xa.q, n_local)) < 0.0f) n_local = -n_local;
    f.kind = kSepFaceOfA;
    f.axis_or_edge_a = n_local;
    f.point_or_edge_b = on_face;
  } else if (nb == 3) {
    V3 n_local = normalize(cross(B[b1] - B[b0], B[b2] - B[b0]));
    V3 on_face = (1.0f / 3.0f) * ((B[b0] + B[b1]) + B[b2]);
    V3 gap = (rotate(xa.q, A[a0]) - rotate(xb.q, on_face)) - dp;
    if (dot(gap, rotate(xb.q, n_local)) < 0.0f) n_local = -n_local;
    f.kind = kSepFaceOfB;
    f.axis_or_edge_a = n_local;
    f.point_or_edge_b = on_face;
  } else {
    if (a0 == a1) a1 = a2;
    if (b0 == b1) b1 = b2;
    set_edge_pair(f, A[a0], A[a1], B[b0], B[b1], xa.q, xb.q, dp, world_normal, 0.005f * 0.005f);
  }
}

// time_of_impact.rs:266 find_min_separation (support points found at time t) and :331
// evaluate_separation (support points given), one routine: with find set, *ia / *ib are
// written; otherwise they are read.
NSD_HD float separation_at(const SepFunc& f, bool find, int* ia, int* ib, float t) {
  Xf xa = sweep_at(f.sa, t), xb = sweep_at(f.sb, t);
  const V3* A = f.pa->pts;
  const V3* B = f.pb->pts;
  switch (f.kind) {
    case kSepPoints: {
      V3 axis = f.axis_or_edge_a;
      if (find) {
        *ia = point_support(A, f.pa->count, inv_rotate(xa.q, axis));
        *ib = point_support(B, f.pb->count, inv_rotate(xb.q, -axis));
        V3 gap = (rotate(xb.q, B[*ib]) - rotate(xa.q, A[*ia])) + (xb.p - xa.p);
        return dot(gap, axis);
      }
      return dot(xf_point(xb, B[*ib]) - xf_point(xa, A[*ia]), axis);
    }
    case kSepEdgePair: {
      V3 axis = normalize(cross(rotate(xa.q, f.axis_or_edge_a), rotate(xb.q, f.point_or_edge_b)));
      if (find) {
        *ia = point_support(A, f.pa->count, inv_rotate(xa.q, axis));
        V3 local_b = inv_rotate(xb.q, axis);
        *ib = point_support(B, f.pb->count, -local_b);
        V3 gap = (rotate(xb.q, B[*ib]) - rotate(xa.q, A[*ia])) + (xb.p - xa.p);
        return dot(gap, axis);
      }
      return dot(xf_point(xb, B[*ib]) - xf_point(xa, A[*ia]), axis);
    }
    case kSepFaceOfA: {
      V3 n = rotate(xa.q, f.axis_or_edge_a);
      V3 on_a = xf_point(xa, f.point_or_edge_b);
      if (find) {
        *ia = -1;
        V3 local_b = inv_rotate(xb.q, n);
        *ib = point_support(B, f.pb->count, -local_b);
      }
      return dot(xf_point(xb, B[*ib]) - on_a, n);
    }
    case kSepFaceOfB: {
      V3 n = rotate(xb.q, f.axis_or_edge_a);
      if (find) {
        V3 local_a = inv_rotate(xa.q, n);
        *ia = point_support(A, f.pa->count, -local_a);
        *ib = -1;
      }
      return dot(xf_point(xa, A[*ia]) - xf_point(xb, f.point_or_edge_b), n);
    }
    default: return 0.0f;
  }
}

// time_of_impact.rs:391 time_of_impact. sa and sb are taken by value: the query re-centres
// them on sa.c1.
NSD_HD ToiResult time_of_impact(const Proxy& pa, const Proxy& pb, Sweep sa, Sweep sb, float t_max) {
  ToiResult r;
  r.state = kToiUnknown;
  r.fraction = -1.0f;
  r.distance = 0.0f;
  r.point = v3(0, 0, 0);
  r.normal = v3(0, 0, 0);
  r.distance_iterations = r.push_back_iterations = r.root_iterations = 0;
  const V3 origin = sa.c1;
  sa.c1 = v3(0, 0, 0);
  sa.c2 = sa.c2 - origin;
  sb.c1 = sb.c1 - origin;
  sb.c2 = sb.c2 - origin;
  const int push_cap = pa.count + pb.count;
  const float slop = linear_slop();
  const float target = maxf(slop, (pa.radius + pb.radius) - slop);
  const float tol = 0.25f * slop;
  SimplexCache cache;
  cache.metric = 0.0f;
  cache.count = 0;
  for (int k = 0; k < 4; ++k) { cache.ia[k] = 0; cache.ib[k] = 0; }
  SepFunc f;
  f.pa = &pa;
  f.pb = &pb;
  f.sa = sa;
  f.sb = sb;
  float t1 = 0.0f;
  for (;;) {
    Xf xa = sweep_at(sa, t1), xb = sweep_at(sb, t1);
    Xf b_in_a = xf(inv_rotate(xa.q, xb.p - xa.p), inv_mul_quat(xa.q, xb.q));  // functions.rs:533
    DistOut d = shape_distance(pa.pts, pa.count, pb.pts, pb.count, b_in_a, &cache);
    r.distance = d.distance;
    V3 wn = rotate(xa.q, d.normal);
    V3 wpa = xf_point(xa, d.pa), wpb = xf_point(xa, d.pb);
    r.distance_iterations += 1;
    bool finished = false;
    if (d.distance <= 0.0f) {
      r.state = kToiOverlapped;
      r.fraction = 0.0f;
      finished = true;
    } else if (d.distance <= target + tol) {
      r.state = kToiHit;
      r.fraction = t1;
      finished = true;
    } else if (r.distance_iterations == 25) {
      r.state = kToiFailed;
      r.fraction = t1;
      finished = true;
    } else {
      build_separation(f, cache, wn, t1);
      float t2 = t_max;
      int pushes = 0;
      for (;;) {
        int ia = 0, ib = 0;
        float s2 = separation_at(f, true, &ia, &ib, t2);
        if (s2 - target > tol) {
          r.state = kToiSeparated;
          r.fraction = t_max;
          finished = true;
          break;
        }
        if (s2 >= target - tol) {
          t1 = t2;
          break;
        }
        float s1 = separation_at(f, false, &ia, &ib, t1);
        if (s1 < target - tol) {
          r.state = kToiFailed;
          r.fraction = t1;
          finished = true;
          break;
        }
        if (s1 <= target + tol) {
          r.state = kToiHit;
          r.fraction = t1;
          finished = true;
          break;
        }
        int roots = 0;
        float lo = t1, hi = t2;
        for (;;) {
          // odd steps take the secant through the bracket, even steps bisect it
          float t = (roots & 1) ? lo + (target - s1) * (hi - lo) / (s2 - s1) : 0.5f * (lo + hi);
          r.root_iterations += 1;
          roots += 1;
          float s = separation_at(f, false, &ia, &ib, t);
          if (absf(s - target) <= tol) {
            t2 = t;
            break;
          }
          if (s > target) {
            lo = t;
            s1 = s;
          } else {
            hi = t;
            s2 = s;
          }
          if (roots == 50) break;
        }
        if (roots == 49 && f.kind == kSepEdgePair) {
          // time_of_impact.rs:375 force_fixed_axis: the edge pair becomes a fixed axis
          Xf x1 = sweep_at(f.sa, t1), x2 = sweep_at(f.sb, t1);
          f.axis_or_edge_a = normalize(cross(rotate(x1.q, f.axis_or_edge_a), rotate(x2.q, f.point_or_edge_b)));
          f.point_or_edge_b = v3(0, 0, 0);
          f.kind = kSepPoints;
          t2 = t_max;
        }
        r.push_back_iterations += 1;
        pushes += 1;
        if (pushes == push_cap) break;
      }
    }
    if (finished) {
      float ra = pa.radius, rb = pb.radius;
      V3 p_a = mul_add(wpa, ra, wn), p_b = mul_add(wpb, -rb, wn);
      r.point = lerp(p_a, p_b, 0.5f) + origin;
      r.normal = wn;
      break;
    }
  }
  return r;
}

}  // namespace nsd
