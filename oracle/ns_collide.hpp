// Oracle narrowphase: box hulls, SAT hull manifolds, sphere/capsule
// manifolds and the GJK distance subset they use. TEST INFRASTRUCTURE ONLY
// (the parity checker); the product never includes this file.
#pragma once
#include "ns_math.hpp"

namespace nso {

// ---------------------------------------------------------------------------
// Hull storage (collision/hull.rs). Only box hulls occur in the workloads; the
// layout is the general half-edge structure so the SAT code below follows the
// reference loops unchanged.
struct HalfEdge { uint8_t next, twin, origin, face; };

struct Hull {
  int vertex_count = 0, edge_count = 0, face_count = 0;
  V3 points[8];
  uint8_t vertex_edge[8];
  HalfEdge edges[24];
  uint8_t face_edge[6];
  Plane planes[6];
  // SoA copies padded to a multiple of 8 (hull.rs:231 hull_soa_stride);
  // normals beyond face_count are zero (hull.rs:833-837).
  real vx[8], vy[8], vz[8];
  real nx[8], ny[8], nz[8];
  real edge_cosines[12];  // box hulls never fill these: zero (hull.rs:754)
  AABB bounds;
  real volume = 0, surface_area = 0, inner_radius = 0;
  V3 center;
  M3 central_inertia;
};

// hull.rs:736-748 box template tables (vertex edge, half edge, face edge)
static const uint8_t kBoxVertexEdges[8] = {8, 1, 0, 9, 13, 3, 5, 11};
static const uint8_t kBoxEdgeData[24][4] = {
    {2, 1, 2, 0},   {17, 0, 1, 5}, {4, 3, 1, 0},   {20, 2, 5, 3},  {6, 5, 5, 0},   {23, 4, 6, 4},
    {0, 7, 6, 0},   {18, 6, 2, 2}, {10, 9, 0, 1},  {21, 8, 3, 5},  {12, 11, 3, 1}, {16, 10, 7, 2},
    {14, 13, 7, 1}, {19, 12, 4, 4}, {8, 15, 4, 1}, {22, 14, 0, 3}, {7, 17, 3, 2},  {9, 16, 2, 5},
    {11, 19, 6, 2}, {5, 18, 7, 4},  {15, 21, 1, 3}, {1, 20, 0, 5}, {3, 23, 4, 3},  {13, 22, 5, 4},
};
static const uint8_t kBoxFaceEdges[6] = {0, 8, 16, 20, 19, 21};

// geometry_queries.rs:81
inline M3 box_inertia(real mass, V3 mn, V3 mx) {
  V3 d = mx - mn;
  real ixx = mass * (d.y * d.y + d.z * d.z) / 12.0f;
  real iyy = mass * (d.x * d.x + d.z * d.z) / 12.0f;
  real izz = mass * (d.x * d.x + d.y * d.y) / 12.0f;
  return diag(ixx, iyy, izz);
}

// hull.rs:754 make_transformed_box_hull with the identity transform
inline Hull make_box_hull(real hx, real hy, real hz) {
  Hull h;
  Xf t = xf(v3(0, 0, 0), qid());
  real min_h = 0.2f * linear_slop();
  V3 e = max3(v3(min_h, min_h, min_h), v3(hx, hy, hz));
  h.vertex_count = 8; h.edge_count = 24; h.face_count = 6;
  for (int i = 0; i < 8; ++i) h.vertex_edge[i] = kBoxVertexEdges[i];
  for (int i = 0; i < 24; ++i) {
    h.edges[i].next = kBoxEdgeData[i][0];
    h.edges[i].twin = kBoxEdgeData[i][1];
    h.edges[i].origin = kBoxEdgeData[i][2];
    h.edges[i].face = kBoxEdgeData[i][3];
  }
  for (int i = 0; i < 6; ++i) h.face_edge[i] = kBoxFaceEdges[i];
  h.bounds = aabb_transform(t, aabb(-e, e));
  h.surface_area = 8.0f * (e.x * e.y + e.x * e.z + e.y * e.z);
  h.volume = 8.0f * e.x * e.y * e.z;
  h.inner_radius = minf(e.x, minf(e.y, e.z));
  h.central_inertia = rotate_inertia(t.q, box_inertia(h.volume, -e, e));
  V3 lower = -e, upper = e;
  V3 ax = v3(1, 0, 0), ay = v3(0, 1, 0), az = v3(0, 0, 1);
  h.planes[0] = transform_plane(t, plane_from_normal_point(-ax, lower));
  h.planes[1] = transform_plane(t, plane_from_normal_point(ax, upper));
  h.planes[2] = transform_plane(t, plane_from_normal_point(-ay, lower));
  h.planes[3] = transform_plane(t, plane_from_normal_point(ay, upper));
  h.planes[4] = transform_plane(t, plane_from_normal_point(-az, lower));
  h.planes[5] = transform_plane(t, plane_from_normal_point(az, upper));
  h.points[0] = xf_point(t, v3(e.x, e.y, e.z));
  h.points[1] = xf_point(t, v3(-e.x, e.y, e.z));
  h.points[2] = xf_point(t, v3(-e.x, -e.y, e.z));
  h.points[3] = xf_point(t, v3(e.x, -e.y, e.z));
  h.points[4] = xf_point(t, v3(e.x, e.y, -e.z));
  h.points[5] = xf_point(t, v3(-e.x, e.y, -e.z));
  h.points[6] = xf_point(t, v3(-e.x, -e.y, -e.z));
  h.points[7] = xf_point(t, v3(e.x, -e.y, -e.z));
  h.center = t.p;
  for (int i = 0; i < 8; ++i) {
    h.vx[i] = h.points[i].x; h.vy[i] = h.points[i].y; h.vz[i] = h.points[i].z;
    h.nx[i] = 0.0f; h.ny[i] = 0.0f; h.nz[i] = 0.0f;
  }
  for (int i = 0; i < 6; ++i) {
    h.nx[i] = h.planes[i].n.x; h.ny[i] = h.planes[i].n.y; h.nz[i] = h.planes[i].n.z;
  }
  for (int i = 0; i < 12; ++i) h.edge_cosines[i] = 0.0f;
  return h;
}

// hull.rs:488
inline int find_hull_support_vertex(const Hull& h, V3 d) {
  int best = -1;
  real best_dot = -kFltMax;
  for (int i = 0; i < h.vertex_count; ++i) {
    real p = d.x * h.vx[i] + d.y * h.vy[i] + d.z * h.vz[i];
    if (p > best_dot) { best_dot = p; best = i; }
  }
  return best;
}
// hull.rs:505
inline int find_hull_support_face(const Hull& h, V3 d) {
  int best = -1;
  real best_dot = -kFltMax;
  for (int i = 0; i < h.face_count; ++i) {
    real p = dot(h.planes[i].n, d);
    if (p > best_dot) { best_dot = p; best = i; }
  }
  return best;
}

// ---------------------------------------------------------------------------
// Manifold types (types/collision_types.rs, collision/manifold.rs)
enum SepFeature : uint8_t {
  kInvalidAxis = 0, kBacksideAxis, kFaceAxisA, kFaceAxisB, kEdgePairAxis, kClosestPointsAxis,
  kManualFaceAxisA, kManualFaceAxisB, kManualEdgePairAxis
};
struct SATCache { real separation = 0; uint8_t type = kInvalidAxis, index_a = 0, index_b = 0, hit = 0; };
struct FeaturePair { uint8_t owner1 = 0, index1 = 0, owner2 = 0, index2 = 0; };
struct LocalPoint { V3 point; real separation; FeaturePair pair; };
struct LocalManifold {
  V3 normal = {0, 0, 0};
  LocalPoint points[4];
  int point_count = 0;
};
struct ClipVertex { V3 position = {0, 0, 0}; real separation = 0; FeaturePair pair; };
struct SepAxis { V3 normal; real separation; int index_a, index_b; uint8_t kind; };
struct AxisQuery { SepAxis face_a, face_b, edge; uint8_t separated_feature; };

inline uint32_t make_feature_id(FeaturePair p) {                                   // manifold.rs:58
  return ((uint32_t)p.owner1 << 24) | ((uint32_t)p.index1 << 16) | ((uint32_t)p.owner2 << 8) |
         (uint32_t)p.index2;
}
inline FeaturePair make_feature_pair(int o1, int i1, int o2, int i2) {             // manifold.rs:66
  FeaturePair p;
  p.index1 = (uint8_t)i1; p.owner1 = (uint8_t)o1; p.index2 = (uint8_t)i2; p.owner2 = (uint8_t)o2;
  return p;
}
inline FeaturePair flip_pair(FeaturePair p) {                                      // manifold.rs:84
  FeaturePair r;
  r.owner1 = 1 - p.owner2; r.owner2 = 1 - p.owner1; r.index1 = p.index2; r.index2 = p.index1;
  return r;
}

// manifold.rs:117
inline int find_incident_face(const Hull& h, V3 ref_n, int vertex_index) {
  int min_edge = -1;
  real min_proj = kFltMax;
  int edge_index = h.vertex_edge[vertex_index];
  int start = edge_index;
  V3 origin = h.points[h.edges[edge_index].origin];
  for (;;) {
    HalfEdge e = h.edges[edge_index];
    HalfEdge tw = h.edges[e.twin];
    V3 to = h.points[tw.origin];
    V3 axis = normalize(to - origin);
    real proj = absf(dot(axis, ref_n));
    if (proj < min_proj) { min_edge = edge_index; min_proj = proj; }
    edge_index = tw.next;
    if (edge_index == start) break;
  }
  HalfEdge me = h.edges[min_edge];
  int f1 = me.face;
  int f2 = h.edges[me.twin].face;
  return dot(h.planes[f1].n, ref_n) < dot(h.planes[f2].n, ref_n) ? f1 : f2;
}

// manifold.rs:173
inline int clip_polygon(ClipVertex* out, const ClipVertex* poly, int count, Plane clip, int edge,
                        Plane ref) {
  ClipVertex v1 = poly[count - 1];
  real d1 = plane_sep(clip, v1.position);
  int n = 0;
  for (int i = 0; i < count; ++i) {
    ClipVertex v2 = poly[i];
    real d2 = plane_sep(clip, v2.position);
    if (d1 <= 0.0f && d2 <= 0.0f) {
      out[n++] = v2;
    } else if (d1 <= 0.0f && d2 > 0.0f) {
      real f = d1 / (d1 - d2);
      V3 pos = mul_add(v1.position, f, v2.position - v1.position);
      ClipVertex v;
      v.position = pos; v.separation = plane_sep(ref, pos); v.pair = v2.pair;
      v.pair.owner2 = 0; v.pair.index2 = (uint8_t)edge;
      out[n++] = v;
    } else if (d2 <= 0.0f && d1 > 0.0f) {
      real f = d1 / (d1 - d2);
      V3 pos = mul_add(v1.position, f, v2.position - v1.position);
      ClipVertex v;
      v.position = pos; v.separation = plane_sep(ref, pos); v.pair = v1.pair;
      v.pair.owner1 = 0; v.pair.index1 = (uint8_t)edge;
      out[n++] = v;
      out[n++] = v2;
    }
    v1 = v2; d1 = d2;
  }
  return n;
}

// convex_manifold.rs:127 clip_segment
inline int clip_segment(ClipVertex* seg, Plane p) {
  int n = 0;
  ClipVertex a = seg[0], b = seg[1];
  real d1 = plane_sep(p, a.position), d2 = plane_sep(p, b.position);
  if (d1 <= 0.0f) seg[n++] = a;
  if (d2 <= 0.0f) seg[n++] = b;
  if (d1 * d2 < 0.0f) {
    real t = d1 / (d1 - d2);
    seg[n].position = (1.0f - t) * a.position + t * b.position;
    seg[n].pair = d1 > 0.0f ? a.pair : b.pair;
    n++;
  }
  return n;
}

// convex_manifold.rs:163
inline int clip_segment_to_hull_face(ClipVertex* seg, const Hull& h, int ref_face) {
  Plane rp = h.planes[ref_face];
  int start = h.face_edge[ref_face];
  int ei = start;
  for (;;) {
    HalfEdge e = h.edges[ei];
    int ni = e.next;
    HalfEdge nx = h.edges[ni];
    V3 p1 = h.points[e.origin], p2 = h.points[nx.origin];
    V3 tangent = normalize(p2 - p1);
    V3 binormal = cross(tangent, rp.n);
    int c = clip_segment(seg, plane_from_normal_point(binormal, p1));
    if (c < 2) return 0;
    ei = ni;
    if (ei == start) break;
  }
  return 2;
}

// convex_manifold.rs:198
inline bool test_edge_candidate_sorted(real a1, real a2, real c, real bound) {
  real hi = maxf(a1, a2), lo = minf(a1, a2);
  bool exterior = hi >= bound;
  real u = lo - c * hi;
  bool max_is_interior = u >= 0.0f;
  real s = 1.0f - c * c;
  real bound_term = (bound - hi) * (bound + hi);
  real lhs = u * u;
  real rhs = bound_term * s;
  bool max_beats_bound = lhs >= rhs;
  bool nearly_parallel = s < 1e-4f;
  bool interior = max_is_interior && (max_beats_bound || nearly_parallel);
  return exterior || interior;
}

inline int round_up4(int n) { return (n + 3) & ~3; }

inline void get_face_dots(const Hull& h, V3 d, real* dots) {                     // :227
  for (int i = 0; i < h.face_count; ++i) dots[i] = d.x * h.nx[i] + d.y * h.ny[i] + d.z * h.nz[i];
}
inline void get_face_plane_separations(const Hull& h, V3 c, real* s) {           // :236
  get_face_dots(h, c, s);
  for (int i = 0; i < h.face_count; ++i) s[i] -= h.planes[i].off;
}
inline int filter_edge_candidates(const Hull& h, const real* ps, real bound, int* idx, int count) {
  int kept = 0;
  for (int k = 0; k < count; ++k) {
    int i = idx[k];
    int i1 = h.edges[i].face, i2 = h.edges[i + 1].face;
    real c = h.edge_cosines[i >> 1];
    idx[kept] = i;
    if (test_edge_candidate_sorted(ps[i1], ps[i2], c, bound)) kept++;
  }
  return kept;
}

// convex_manifold.rs:277 -- the vertex index rides in the low 7 mantissa bits
inline real get_support_wide(V3 n, const real* vx, const real* vy, const real* vz, int cnt,
                              real bias, int* vi) {
  // an unsigned integer as wide as the scalar carries its bits
  typedef typename std::conditional<sizeof(real) == 4, uint32_t, uint64_t>::type bits_t;
  const bits_t mask = (bits_t(1) << 7) - 1;
  real min_value = INFINITY;
  for (int i = 0; i < cnt; ++i) {
    real d = n.x * vx[i] + n.y * vy[i] + n.z * vz[i];
    real value = bias - d;
    bits_t bits;
    std::memcpy(&bits, &value, sizeof(real));
    bits = (bits & ~mask) | ((bits_t)i & mask);
    real aug;
    std::memcpy(&aug, &bits, sizeof(real));
    if (aug < min_value) min_value = aug;
  }
  bits_t mb;
  std::memcpy(&mb, &min_value, sizeof(real));
  int v = (int)(mb & mask);
  *vi = v;
  return n.x * vx[v] + n.y * vy[v] + n.z * vz[v];
}

inline real get_face_separation(V3 dir, real plane_sep_v, const real* vx, const real* vy,
                                 const real* vz, int n, V3 center, V3 extents, int* vi) {
  real bias = dot(dir, center) + 1.0625f * dot(abs3(dir), extents);
  real support = get_support_wide(dir, vx, vy, vz, n, bias, vi);
  return plane_sep_v - support;
}

// convex_manifold.rs:392 compute_separating_axis (B in A's frame)
inline AxisQuery compute_separating_axis(const Hull& ha, const Hull& hb, Xf xb, bool early) {
  M3 r = matrix_from_quat(xb.q);
  M3 inv_r = transpose(r);
  real spec = speculative_distance();
  AxisQuery res;
  res.face_a = {v3(0, 0, 0), -INFINITY, kNull, kNull, kFaceAxisA};
  res.face_b = {v3(0, 0, 0), -INFINITY, kNull, kNull, kFaceAxisB};
  res.edge = {v3(0, 0, 0), -INFINITY, kNull, kNull, kEdgePairAxis};
  res.separated_feature = kInvalidAxis;

  real dot_a[8], dot_b[8], pd_a[8], pd_b[8];
  int eia[16], eib[16];

  int wide_vb = round_up4(hb.vertex_count);
  V3 c_b = aabb_center(hb.bounds), h_b = aabb_extents(hb.bounds);
  V3 delta_center = mul_mv(r, hb.center) + xb.p - ha.center;
  real center_distance = length(delta_center);
  real radius = ha.inner_radius + hb.inner_radius;
  real radius_bound = radius - (linear_slop() + 0.001f * (center_distance + radius));

  get_face_dots(ha, delta_center, dot_a);
  int seed_a = 0;
  real max_dot_a = dot_a[0];
  for (int i = 1; i < ha.face_count; ++i)
    if (dot_a[i] > max_dot_a) { max_dot_a = dot_a[i]; seed_a = i; }

  real floor_a = -INFINITY, seed_sep_a = -INFINITY;
  int seed_vb = 0;
  if (early) {
    Plane p = ha.planes[seed_a];
    V3 dir = -mul_mv(inv_r, p.n);
    real ps = dot(p.n, xb.p) - p.off;
    seed_sep_a = get_face_separation(dir, ps, hb.vx, hb.vy, hb.vz, wide_vb, c_b, h_b, &seed_vb);
    floor_a = minf(seed_sep_a, spec);
  }
  for (int i = 0; i < ha.face_count; ++i) {
    if (dot_a[i] - radius_bound < maxf(floor_a, res.face_a.separation)) continue;
    Plane p = ha.planes[i];
    int vi = seed_vb;
    real sep = seed_sep_a;
    if (!early || i != seed_a) {
      V3 dir = -mul_mv(inv_r, p.n);
      real ps = dot(p.n, xb.p) - p.off;
      sep = get_face_separation(dir, ps, hb.vx, hb.vy, hb.vz, wide_vb, c_b, h_b, &vi);
    }
    if (sep > res.face_a.separation) {
      res.face_a.normal = p.n; res.face_a.separation = sep;
      res.face_a.index_a = i; res.face_a.index_b = vi;
      if (sep > spec && early) { res.separated_feature = kFaceAxisA; return res; }
    }
  }

  int wide_va = round_up4(ha.vertex_count);
  V3 c_a = aabb_center(ha.bounds), h_a = aabb_extents(ha.bounds);
  get_face_dots(hb, -mul_mv(inv_r, delta_center), dot_b);
  int seed_b = 0;
  real max_dot_b = dot_b[0];
  for (int i = 1; i < hb.face_count; ++i)
    if (dot_b[i] > max_dot_b) { max_dot_b = dot_b[i]; seed_b = i; }

  real floor_b = -INFINITY, seed_sep_b = -INFINITY;
  int seed_va = 0;
  if (early) {
    Plane p = hb.planes[seed_b];
    V3 dir = -mul_mv(r, p.n);
    real ps = dot(dir, xb.p) - p.off;
    seed_sep_b = get_face_separation(dir, ps, ha.vx, ha.vy, ha.vz, wide_va, c_a, h_a, &seed_va);
    floor_b = maxf(seed_sep_b, res.face_a.separation);
    floor_b = minf(floor_b, spec);
  }
  for (int i = 0; i < hb.face_count; ++i) {
    if (dot_b[i] - radius_bound < maxf(floor_b, res.face_b.separation)) continue;
    Plane p = hb.planes[i];
    V3 dir = -mul_mv(r, p.n);
    int vi = seed_va;
    real sep = seed_sep_b;
    if (!early || i != seed_b) {
      real ps = dot(dir, xb.p) - p.off;
      sep = get_face_separation(dir, ps, ha.vx, ha.vy, ha.vz, wide_va, c_a, h_a, &vi);
    }
    if (sep > res.face_b.separation) {
      res.face_b.normal = dir; res.face_b.separation = sep;
      res.face_b.index_a = vi; res.face_b.index_b = i;
      if (sep > spec && early) { res.separated_feature = kFaceAxisB; return res; }
    }
  }

  int na = 0, nb = 0;
  real max_face_sep = maxf(res.face_a.separation, res.face_b.separation);
  real bound_slack = radius - radius_bound;
  real threshold_a = early ? max_face_sep + hb.inner_radius - bound_slack : -INFINITY;
  real threshold_b = early ? max_face_sep + ha.inner_radius - bound_slack : -INFINITY;
  V3 center_b_in_a = mul_mv(r, hb.center) + xb.p;
  V3 center_a_in_b = mul_mv(inv_r, ha.center - xb.p);
  get_face_plane_separations(ha, center_b_in_a, pd_a);
  get_face_plane_separations(hb, center_a_in_b, pd_b);
  for (int i = 0; i < ha.edge_count; i += 2) {
    int i1 = ha.edges[i].face, i2 = ha.edges[i + 1].face;
    real c = ha.edge_cosines[i >> 1];
    eia[na] = i;
    if (test_edge_candidate_sorted(pd_a[i1], pd_a[i2], c, threshold_a)) na++;
  }
  for (int i = 0; i < hb.edge_count; i += 2) {
    int i1 = hb.edges[i].face, i2 = hb.edges[i + 1].face;
    real c = hb.edge_cosines[i >> 1];
    eib[nb] = i;
    if (test_edge_candidate_sorted(pd_b[i1], pd_b[i2], c, threshold_b)) nb++;
  }

  if (early && nb * ((na + 3) >> 2) >= 10) {
    real probe_bound =
        max_face_sep - (0.1f * linear_slop() + 0.001f * absf(center_distance + radius));
    int vb = res.face_a.index_b != kNull ? res.face_a.index_b : seed_vb;
    V3 probe_b = v3(hb.vx[vb], hb.vy[vb], hb.vz[vb]);
    get_face_plane_separations(ha, mul_mv(r, probe_b) + xb.p, pd_a);
    na = filter_edge_candidates(ha, pd_a, probe_bound, eia, na);
    int va = res.face_b.index_a != kNull ? res.face_b.index_a : seed_va;
    V3 probe_a = v3(ha.vx[va], ha.vy[va], ha.vz[va]);
    get_face_plane_separations(hb, mul_mv(inv_r, probe_a - xb.p), pd_b);
    nb = filter_edge_candidates(hb, pd_b, probe_bound, eib, nb);
  }

  if (na == 0 || nb == 0) return res;

  // negative_transform_from_soa (convex_manifold.rs:340): rows of r dotted with the input
  V3 r0 = v3(r.cx.x, r.cy.x, r.cz.x), r1 = v3(r.cx.y, r.cy.y, r.cz.y), r2 = v3(r.cx.z, r.cy.z, r.cz.z);
  real bfx[8], bfy[8], bfz[8], bwx[8], bwy[8], bwz[8];
  int wide_fb = round_up4(hb.face_count);
  for (int i = 0; i < wide_fb; ++i) {
    V3 v = v3(hb.nx[i], hb.ny[i], hb.nz[i]);
    V3 o = v3(dot(r0, v), dot(r1, v), dot(r2, v));
    bfx[i] = -o.x; bfy[i] = -o.y; bfz[i] = -o.z;
  }
  for (int i = 0; i < wide_vb; ++i) {
    V3 v = v3(hb.vx[i], hb.vy[i], hb.vz[i]);
    V3 o = v3(dot(r0, v), dot(r1, v), dot(r2, v));
    o = o + xb.p;
    bwx[i] = -o.x; bwy[i] = -o.y; bwz[i] = -o.z;
  }
  V3 an0[16], an1[16], ad[16], av0[16];
  real atol[16];
  real sq_tol = kParallelEdgeTol * kParallelEdgeTol;
  for (int k = 0; k < na; ++k) {
    HalfEdge e = ha.edges[eia[k]], tw = ha.edges[eia[k] + 1];
    an0[k] = ha.planes[e.face].n;
    an1[k] = ha.planes[tw.face].n;
    int v0 = e.origin, v1 = tw.origin;
    ad[k] = v3(ha.vx[v1] - ha.vx[v0], ha.vy[v1] - ha.vy[v0], ha.vz[v1] - ha.vz[v0]);
    av0[k] = v3(ha.vx[v0], ha.vy[v0], ha.vz[v0]);
    atol[k] = sq_tol * (ad[k].x * ad[k].x + ad[k].y * ad[k].y + ad[k].z * ad[k].z);
  }
  real ls = linear_slop();
  real eps = -ls * ls;
  for (int j = 0; j < nb; ++j) {
    HalfEdge e = hb.edges[eib[j]], tw = hb.edges[eib[j] + 1];
    int f0 = e.face, f1 = tw.face, v0 = e.origin, v1 = tw.origin;
    V3 c = v3(bfx[f0], bfy[f0], bfz[f0]);
    V3 dn = v3(bfx[f1], bfy[f1], bfz[f1]);
    V3 bv0 = v3(bwx[v0], bwy[v0], bwz[v0]);
    V3 bv1 = v3(bwx[v1], bwy[v1], bwz[v1]);
    V3 dc = bv1 - bv0;
    for (int i = 0; i < na; ++i) {
      V3 d = ad[i];
      real cba = dot(c, d), dba = dot(dn, d);
      if (cba * dba >= eps) continue;
      real adc = dot(an0[i], dc), bdc = dot(an1[i], dc);
      if (adc * bdc >= eps || cba * bdc >= eps) continue;
      real max_cd = maxf(cba * cba, dba * dba);
      if (max_cd <= atol[i]) continue;
      real t = -cba / (dba - cba);
      V3 n = mul_add(c, t, dn - c);
      real len2 = dot(n, n);
      real inv = 1.0f / std::sqrt(len2);
      n = inv * n;
      real sep = -dot(av0[i] + bv0, n);
      if (sep > res.edge.separation) {
        res.edge.normal = n; res.edge.separation = sep;
        res.edge.index_a = eia[i]; res.edge.index_b = eib[j];
        if (sep > spec && early) { res.separated_feature = kEdgePairAxis; return res; }
      }
    }
  }
  return res;
}

// convex_manifold.rs:905
inline void reduce_manifold_points(LocalManifold* m, LocalPoint* pts, int count) {
  if (count <= 4) {
    for (int i = 0; i < count; ++i) m->points[i] = pts[i];
    m->point_count = count;
    return;
  }
  V3 normal = m->normal;
  real spec = speculative_distance();
  real tol_sqr = spec * spec;
  const real bias = 0.95f;
  int best = kNull;
  real best_score = -kFltMax;
  V3 sd = arbitrary_perp(normal);
  for (int i = 0; i < count; ++i) {
    if (pts[i].separation > spec) continue;
    real score = -pts[i].separation + dot(sd, pts[i].point);
    if (bias * score > best_score) { best = i; best_score = score; }
  }
  if (best == kNull) { m->point_count = 0; return; }
  m->points[0] = pts[best];
  m->point_count = 1;
  pts[best] = pts[count - 1];
  count--;
  V3 a = m->points[0].point;

  best_score = 0.0f; best = kNull;
  for (int i = 0; i < count; ++i) {
    V3 d = pts[i].point - a;
    V3 v = mul_sub(d, dot(d, normal), normal);
    real dsq = length_sq(v);
    real sep = maxf(0.0f, -pts[i].separation);
    real score = dsq + 4.0f * sep * sep;
    if (bias * score > best_score) { best_score = score; best = i; }
  }
  if (best_score < tol_sqr) return;
  m->points[1] = pts[best];
  m->point_count = 2;
  pts[best] = pts[count - 1];
  count--;
  V3 b = m->points[1].point;

  best_score = tol_sqr; best = kNull;
  real best_signed = 0.0f;
  V3 ba = b - a;
  for (int i = 0; i < count; ++i) {
    V3 p = pts[i].point;
    real signed_area = dot(normal, cross(ba, p - a));
    real score = absf(signed_area);
    if (bias * score >= best_score) { best_score = score; best = i; best_signed = signed_area; }
  }
  if (best == kNull) return;
  m->points[2] = pts[best];
  m->point_count = 3;
  pts[best] = pts[count - 1];
  count--;
  V3 c = m->points[2].point;

  best_score = tol_sqr; best = kNull;
  real sign = best_signed < 0.0f ? -1.0f : 1.0f;
  for (int i = 0; i < count; ++i) {
    V3 p = pts[i].point;
    real u1 = sign * dot(normal, cross(p - a, ba));
    real u2 = sign * dot(normal, cross(p - b, c - b));
    real u3 = sign * dot(normal, cross(p - c, a - c));
    real score = maxf(u1, maxf(u2, u3));
    if (bias * score > best_score) { best_score = score; best = i; }
  }
  if (best != kNull) {
    m->points[m->point_count] = pts[best];
    m->point_count += 1;
  }
}

// convex_manifold.rs:1071
inline int build_polygon(ClipVertex* out, Xf t, const Hull& h, int inc_face, Plane ref) {
  int ei = h.face_edge[inc_face];
  int n = 0;
  M3 m = matrix_from_quat(t.q);
  for (;;) {
    HalfEdge e = h.edges[ei];
    int ni = e.next;
    HalfEdge nx = h.edges[ni];
    ClipVertex v;
    v.position = mul_mv(m, h.points[nx.origin]) + t.p;
    v.separation = plane_sep(ref, v.position);
    v.pair = make_feature_pair(1, ei, 1, ni);
    out[n++] = v;
    ei = ni;
    if (ei == h.face_edge[inc_face] || n >= 64) break;
  }
  return n;
}

// convex_manifold.rs:1150
inline bool build_face_a_contact(LocalManifold* m, const Hull& ha, const Hull& hb, Xf xb,
                                 SepAxis q, SATCache* cache) {
  ClipVertex poly1[64], poly2[64];
  LocalPoint pts[64];
  int ref_face = q.index_a;
  Plane rp = ha.planes[ref_face];
  V3 ref_n_in_b = inv_rotate(xb.q, rp.n);
  int inc = find_incident_face(hb, ref_n_in_b, q.index_b);
  int count = build_polygon(poly1, xb, hb, inc, rp);
  int ei = ha.face_edge[ref_face];
  bool use1 = true;
  for (;;) {
    HalfEdge e = ha.edges[ei];
    int ni = e.next;
    HalfEdge nx = ha.edges[ni];
    V3 p1 = ha.points[e.origin], p2 = ha.points[nx.origin];
    V3 tangent = normalize(p2 - p1);
    V3 binormal = cross(tangent, rp.n);
    Plane cp = plane_from_normal_point(binormal, p1);
    if (use1) count = clip_polygon(poly2, poly1, count, cp, ei, rp);
    else count = clip_polygon(poly1, poly2, count, cp, ei, rp);
    use1 = !use1;
    if (count < 3) { *cache = SATCache(); return false; }
    ei = ni;
    if (ei == ha.face_edge[ref_face]) break;
  }
  count = min_i(count, 64);
  m->normal = rp.n;
  const ClipVertex* src = use1 ? poly1 : poly2;
  real min_sep = kFltMax;
  for (int i = 0; i < count; ++i) {
    LocalPoint p;
    p.point = mul_sub(src[i].position, 0.5f * src[i].separation, rp.n);
    p.separation = src[i].separation;
    p.pair = src[i].pair;
    min_sep = minf(min_sep, src[i].separation);
    pts[i] = p;
  }
  if (min_sep >= speculative_distance()) { *cache = SATCache(); return false; }
  reduce_manifold_points(m, pts, count);
  cache->separation = min_sep;
  cache->type = kFaceAxisA;
  cache->index_a = (uint8_t)q.index_a;
  cache->index_b = (uint8_t)q.index_b;
  return true;
}

// convex_manifold.rs:1276
inline bool build_face_b_contact(LocalManifold* m, const Hull& ha, const Hull& hb, Xf xb,
                                 SepAxis q, SATCache* cache) {
  Xf xa = invert_xf(xb);
  SepAxis fq = {-q.normal, q.separation, q.index_b, q.index_a, kFaceAxisA};
  bool touching = build_face_a_contact(m, hb, ha, xa, fq, cache);
  if (!touching) { *cache = SATCache(); return false; }
  M3 mat = matrix_from_quat(xb.q);
  m->normal = -mul_mv(mat, m->normal);
  for (int i = 0; i < m->point_count; ++i) {
    m->points[i].point = mul_mv(mat, m->points[i].point) + xb.p;
    m->points[i].pair = flip_pair(m->points[i].pair);
  }
  cache->type = kFaceAxisB;
  cache->index_a = (uint8_t)q.index_a;
  cache->index_b = (uint8_t)q.index_b;
  return true;
}

inline bool within_segments(const SegResult& r) {
  return (0.0f <= r.f1 && r.f1 <= 1.0f) && (0.0f <= r.f2 && r.f2 <= 1.0f);
}

// convex_manifold.rs:1340
inline bool build_edge_contact(LocalManifold* m, const Hull& ha, const Hull& hb, Xf xb, SepAxis q,
                               SATCache* cache) {
  HalfEdge ea = ha.edges[q.index_a];
  HalfEdge ta = ha.edges[ea.twin];
  V3 pa = ha.points[ea.origin], qa = ha.points[ta.origin];
  V3 e_a = qa - pa;
  HalfEdge eb = hb.edges[q.index_b];
  HalfEdge tb = hb.edges[eb.twin];
  V3 pb = xf_point(xb, hb.points[eb.origin]);
  V3 qb = xf_point(xb, hb.points[tb.origin]);
  V3 e_b = qb - pb;
  V3 normal = q.normal;
  SegResult r = line_distance(pa, e_a, pb, e_b);
  if (!within_segments(r)) { *cache = SATCache(); return false; }
  real sep = dot(normal, r.p2 - r.p1);
  V3 point = 0.5f * (r.p1 + r.p2);
  m->normal = normal;
  m->point_count = 1;
  m->points[0].point = point;
  m->points[0].separation = sep;
  m->points[0].pair = make_feature_pair(0, q.index_a, 1, q.index_b);
  cache->separation = sep;
  cache->type = kEdgePairAxis;
  cache->index_a = (uint8_t)q.index_a;
  cache->index_b = (uint8_t)q.index_b;
  return true;
}

// convex_manifold.rs:1445 collide_hulls_with_scratch
inline void collide_hulls(LocalManifold* m, const Hull& ha, const Hull& hb, Xf xb, SATCache* cache,
                          int* sat_calls_out) {
  m->point_count = 0;
  real spec = speculative_distance();
  real ls = linear_slop();
  cache->hit = 0;
  switch (cache->type) {
    case kInvalidAxis: break;
    case kFaceAxisA: {
      Plane p = ha.planes[cache->index_a];
      V3 sd = -inv_rotate(xb.q, p.n);
      int vi = find_hull_support_vertex(hb, sd);
      V3 support = xf_point(xb, hb.points[vi]);
      real sep = plane_sep(p, support);
      if (sep >= spec) { cache->hit = 1; return; }
      SepAxis fq = {p.n, 0.0f, cache->index_a, vi, kFaceAxisA};
      SATCache local;
      bool touching = build_face_a_contact(m, ha, hb, xb, fq, &local);
      if (touching && absf(cache->separation - local.separation) < ls) { cache->hit = 1; return; }
      break;
    }
    case kFaceAxisB: {
      Plane p = hb.planes[cache->index_b];
      V3 sd = -rotate(xb.q, p.n);
      int vi = find_hull_support_vertex(ha, sd);
      V3 support = inv_xf_point(xb, ha.points[vi]);
      real sep = plane_sep(p, support);
      if (sep >= spec) { cache->hit = 1; return; }
      SepAxis fq = {-p.n, 0.0f, vi, cache->index_b, kFaceAxisB};
      SATCache local;
      bool touching = build_face_b_contact(m, ha, hb, xb, fq, &local);
      if (touching && absf(cache->separation - local.separation) < ls) { cache->hit = 1; return; }
      break;
    }
    case kEdgePairAxis: {
      int ia = cache->index_a;
      HalfEdge e1 = ha.edges[ia], t1 = ha.edges[ia + 1];
      V3 pa = ha.points[e1.origin], qa = ha.points[t1.origin];
      V3 e_a = qa - pa;
      V3 ua = ha.planes[e1.face].n, va = ha.planes[t1.face].n;
      int ib = cache->index_b;
      HalfEdge e2 = hb.edges[ib], t2 = hb.edges[ib + 1];
      V3 pb = xf_point(xb, hb.points[e2.origin]);
      V3 qb = xf_point(xb, hb.points[t2.origin]);
      V3 e_b = qb - pb;
      V3 ub = rotate(xb.q, hb.planes[e2.face].n);
      V3 vb = rotate(xb.q, hb.planes[t2.face].n);
      real cba = dot(ub, e_a), dba = dot(vb, e_a);
      real adc = -dot(ua, e_b), bdc = -dot(va, e_b);
      if (cba * dba < 0.0f && adc * bdc < 0.0f && cba * bdc > 0.0f) {
        real sq = kParallelEdgeTol * kParallelEdgeTol;
        if (maxf(cba * cba, dba * dba) >= sq * length_sq(e_a)) {
          real t = cba / (cba - dba);
          V3 axis = normalize(lerp(ub, vb, t));
          real sep = dot(axis, qa - qb);
          if (sep > spec) { cache->hit = 1; return; }
          SepAxis eq = {-axis, 0.0f, cache->index_a, cache->index_b, kEdgePairAxis};
          SATCache local;
          bool touching = build_edge_contact(m, ha, hb, xb, eq, &local);
          if (touching && absf(cache->separation - local.separation) < ls) { cache->hit = 1; return; }
        }
      }
      break;
    }
    default: break;  // manual and backside axes never occur in these workloads
  }
  m->point_count = 0;
  *cache = SATCache();
  if (sat_calls_out) (*sat_calls_out)++;
  AxisQuery aq = compute_separating_axis(ha, hb, xb, true);
  if (aq.separated_feature != kInvalidAxis) {
    cache->type = aq.separated_feature;
    const SepAxis& s = aq.separated_feature == kFaceAxisA ? aq.face_a
                       : aq.separated_feature == kFaceAxisB ? aq.face_b : aq.edge;
    cache->separation = s.separation;
    cache->index_a = (uint8_t)s.index_a;
    cache->index_b = (uint8_t)s.index_b;
    return;
  }
  if (aq.face_a.separation > aq.face_b.separation) {
    build_face_a_contact(m, ha, hb, xb, aq.face_a, cache);
  } else {
    build_face_b_contact(m, ha, hb, xb, aq.face_b, cache);
  }
  SepAxis eq = aq.edge;
  if (eq.index_a == kNull) return;
  real face_sep = maxf(aq.face_a.separation, aq.face_b.separation);
  real clip_sep = cache->separation;
  if ((m->point_count == 0 && eq.separation > face_sep) || eq.separation > clip_sep + ls) {
    LocalManifold em;
    SATCache ec;
    build_edge_contact(&em, ha, hb, xb, eq, &ec);
    if (em.point_count == 1) {
      m->normal = em.normal;
      m->point_count = 1;
      m->points[0] = em.points[0];
      *cache = ec;
    }
  }
}

// ---------------------------------------------------------------------------
// Sphere / capsule pairs (convex_manifold_shapes.rs)
struct Sphere { V3 center; real radius; };
struct Capsule { V3 c1, c2; real radius; };

inline void collide_spheres(LocalManifold* m, Sphere a, Sphere b, Xf xb) {        // :21
  m->point_count = 0;
  V3 c1 = a.center, c2 = xf_point(xb, b.center);
  real tr = a.radius + b.radius;
  real maxd = tr + speculative_distance();
  V3 off = c2 - c1;
  real dsq = length_sq(off);
  if (dsq > maxd * maxd) return;
  V3 n = v3(0.0f, 1.0f, 0.0f);
  real d = std::sqrt(dsq);
  if (d * d > 1000.0f * kMinPositive) n = (1.0f / d) * off;
  V3 point = 0.5f * (mul_sub(mul_add(c1, a.radius, n) + c2, b.radius, n));
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = point;
  m->points[0].separation = d - tr;
  m->points[0].pair = FeaturePair();
}

inline void collide_capsule_sphere(LocalManifold* m, Capsule a, Sphere b, Xf xb) { // :74
  m->point_count = 0;
  V3 c = xf_point(xb, b.center);
  real tr = b.radius + a.radius;
  real maxd = tr + speculative_distance();
  V3 cp = point_to_segment(a.c1, a.c2, c);
  V3 off = c - cp;
  real dsq = length_sq(off);
  if (dsq > maxd * maxd) return;
  V3 n = v3(0.0f, 1.0f, 0.0f);
  real d = std::sqrt(dsq);
  if (d * d > 1000.0f * kMinPositive) n = (1.0f / d) * off;
  V3 point = 0.5f * mul_add(mul_sub(c, b.radius, n) + cp, a.radius, n);
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = point;
  m->points[0].separation = d - tr;
  m->points[0].pair = FeaturePair();
}

// GJK (collision/distance.rs)
struct SimplexCache { real metric = 0; uint16_t count = 0; uint8_t ia[4] = {0, 0, 0, 0}, ib[4] = {0, 0, 0, 0}; };
struct SVert { V3 wa, wb, w; real a; int ia, ib; };
struct Simplex { SVert v[4]; int count = 0; };
struct DistOut { V3 pa, pb, normal; real distance; };

inline int point_support(const V3* pts, int n, V3 axis) {                          // :17/:38
  V3 o = pts[0];
  int mi = 0;
  real mp = 0.0f;
  for (int i = 1; i < n; ++i) {
    real p = dot(axis, pts[i] - o);
    if (p > mp) { mi = i; mp = p; }
  }
  return mi;
}
inline void bary_edge(V3 a, V3 b, real* u, real* v, real* d) {                  // :58
  V3 ab = b - a;
  *d = dot(ab, ab); *u = dot(b, ab); *v = -dot(a, ab);
}
inline void bary_tri(V3 a, V3 b, V3 c, real* u, real* v, real* w, real* d) {   // :67
  V3 ab = b - a, ac = c - a;
  V3 bxc = cross(b, c), cxa = cross(c, a), axb = cross(a, b), abxac = cross(ab, ac);
  *d = dot(abxac, abxac); *u = dot(bxc, abxac); *v = dot(cxa, abxac); *w = dot(axb, abxac);
}
inline void bary_tet(V3 a, V3 b, V3 c, V3 d, real* u, real* v, real* w, real* x, real* dv) {
  V3 ab = b - a, ac = c - a, ad = d - a;
  real divisor = scalar_triple(ab, ac, ad);
  real sign = divisor < 0.0f ? -1.0f : 1.0f;
  *u = sign * scalar_triple(b, c, d);
  *v = sign * scalar_triple(a, d, c);
  *w = sign * scalar_triple(a, b, d);
  *x = sign * scalar_triple(a, c, b);
  *dv = sign * divisor;
}
inline real simplex_metric(const Simplex& s) {                                     // :96
  switch (s.count) {
    case 1: return 0.0f;
    case 2: return distance(s.v[0].w, s.v[1].w);
    case 3: return length(cross(s.v[1].w - s.v[0].w, s.v[2].w - s.v[0].w)) / 2.0f;
    case 4: return scalar_triple(s.v[1].w - s.v[0].w, s.v[2].w - s.v[0].w, s.v[3].w - s.v[0].w) / 6.0f;
  }
  return 0.0f;
}
inline bool solve2(Simplex& s) {                                                   // :130
  V3 a = s.v[0].w, b = s.v[1].w, ab = b - a;
  real divisor = dot(ab, ab), u = dot(b, ab), v = -dot(a, ab);
  if (v <= 0.0f) { s.count = 1; s.v[0].a = 1.0f; return true; }
  if (u <= 0.0f) { s.count = 1; s.v[0] = s.v[1]; s.v[0].a = 1.0f; return true; }
  if (divisor <= 0.0f) return false;
  real den = 1.0f / divisor;
  s.v[0].a = den * u; s.v[1].a = den * v;
  return true;
}
inline bool edge_pick(Simplex& s, SVert a, SVert b, real u, real v, real d) {
  s.count = 2; s.v[0] = a; s.v[1] = b;
  if (d <= 0.0f) return false;
  s.v[0].a = u / d; s.v[1].a = v / d;
  return true;
}
inline bool tri_pick(Simplex& s, SVert a, SVert b, SVert c, real u, real v, real w, real d) {
  s.count = 3; s.v[0] = a; s.v[1] = b; s.v[2] = c;
  if (d <= 0.0f) return false;
  s.v[0].a = u / d; s.v[1].a = v / d; s.v[2].a = w / d;
  return true;
}
inline bool solve3(Simplex& s) {                                                   // :159
  SVert v1 = s.v[0], v2 = s.v[1], v3_ = s.v[2];
  real ab_u, ab_v, ab_d, bc_u, bc_v, bc_d, ca_u, ca_v, ca_d;
  bary_edge(v1.w, v2.w, &ab_u, &ab_v, &ab_d);
  bary_edge(v2.w, v3_.w, &bc_u, &bc_v, &bc_d);
  bary_edge(v3_.w, v1.w, &ca_u, &ca_v, &ca_d);
  if (ab_v <= 0.0f && ca_u <= 0.0f) { s.count = 1; s.v[0] = v1; s.v[0].a = 1.0f; return true; }
  if (bc_v <= 0.0f && ab_u <= 0.0f) { s.count = 1; s.v[0] = v2; s.v[0].a = 1.0f; return true; }
  if (ca_v <= 0.0f && bc_u <= 0.0f) { s.count = 1; s.v[0] = v3_; s.v[0].a = 1.0f; return true; }
  real tu, tv, tw, td;
  bary_tri(v1.w, v2.w, v3_.w, &tu, &tv, &tw, &td);
  if (tw <= 0.0f && ab_u > 0.0f && ab_v > 0.0f) return edge_pick(s, v1, v2, ab_u, ab_v, ab_d);
  if (tu <= 0.0f && bc_u > 0.0f && bc_v > 0.0f) return edge_pick(s, v2, v3_, bc_u, bc_v, bc_d);
  if (tv <= 0.0f && ca_u > 0.0f && ca_v > 0.0f) return edge_pick(s, v3_, v1, ca_u, ca_v, ca_d);
  if (td <= 0.0f) return false;
  s.v[0].a = tu / td; s.v[1].a = tv / td; s.v[2].a = tw / td;
  return true;
}
inline bool solve4(Simplex& s) {                                                   // :249
  SVert A = s.v[0], B = s.v[1], C = s.v[2], D = s.v[3];
  real ab[3], ac[3], ad[3], bc[3], cd[3], db[3];
  bary_edge(A.w, B.w, &ab[0], &ab[1], &ab[2]);
  bary_edge(A.w, C.w, &ac[0], &ac[1], &ac[2]);
  bary_edge(A.w, D.w, &ad[0], &ad[1], &ad[2]);
  bary_edge(B.w, C.w, &bc[0], &bc[1], &bc[2]);
  bary_edge(C.w, D.w, &cd[0], &cd[1], &cd[2]);
  bary_edge(D.w, B.w, &db[0], &db[1], &db[2]);
  if (ab[1] <= 0.0f && ac[1] <= 0.0f && ad[1] <= 0.0f) { s.count = 1; s.v[0] = A; s.v[0].a = 1.0f; return true; }
  if (ab[0] <= 0.0f && db[0] <= 0.0f && bc[1] <= 0.0f) { s.count = 1; s.v[0] = B; s.v[0].a = 1.0f; return true; }
  if (ac[0] <= 0.0f && bc[0] <= 0.0f && cd[1] <= 0.0f) { s.count = 1; s.v[0] = C; s.v[0].a = 1.0f; return true; }
  if (ad[0] <= 0.0f && cd[0] <= 0.0f && db[1] <= 0.0f) { s.count = 1; s.v[0] = D; s.v[0].a = 1.0f; return true; }
  real acb[4], abd[4], adc[4], bcd[4];
  bary_tri(A.w, C.w, B.w, &acb[0], &acb[1], &acb[2], &acb[3]);
  bary_tri(A.w, B.w, D.w, &abd[0], &abd[1], &abd[2], &abd[3]);
  bary_tri(A.w, D.w, C.w, &adc[0], &adc[1], &adc[2], &adc[3]);
  bary_tri(B.w, C.w, D.w, &bcd[0], &bcd[1], &bcd[2], &bcd[3]);
  if (abd[2] <= 0.0f && acb[1] <= 0.0f && ab[0] > 0.0f && ab[1] > 0.0f) return edge_pick(s, A, B, ab[0], ab[1], ab[2]);
  if (acb[2] <= 0.0f && adc[1] <= 0.0f && ac[0] > 0.0f && ac[1] > 0.0f) return edge_pick(s, A, C, ac[0], ac[1], ac[2]);
  if (adc[2] <= 0.0f && abd[1] <= 0.0f && ad[0] > 0.0f && ad[1] > 0.0f) return edge_pick(s, A, D, ad[0], ad[1], ad[2]);
  if (acb[0] <= 0.0f && bcd[2] <= 0.0f && bc[0] > 0.0f && bc[1] > 0.0f) return edge_pick(s, B, C, bc[0], bc[1], bc[2]);
  if (adc[0] <= 0.0f && bcd[0] <= 0.0f && cd[0] > 0.0f && cd[1] > 0.0f) return edge_pick(s, C, D, cd[0], cd[1], cd[2]);
  if (abd[0] <= 0.0f && bcd[1] <= 0.0f && db[0] > 0.0f && db[1] > 0.0f) return edge_pick(s, D, B, db[0], db[1], db[2]);
  real tu, tv, tw, tx, td;
  bary_tet(A.w, B.w, C.w, D.w, &tu, &tv, &tw, &tx, &td);
  if (tx < 0.0f && acb[0] > 0.0f && acb[1] > 0.0f && acb[2] > 0.0f) return tri_pick(s, A, C, B, acb[0], acb[1], acb[2], acb[3]);
  if (tw < 0.0f && abd[0] > 0.0f && abd[1] > 0.0f && abd[2] > 0.0f) return tri_pick(s, A, B, D, abd[0], abd[1], abd[2], abd[3]);
  if (tv < 0.0f && adc[0] > 0.0f && adc[1] > 0.0f && adc[2] > 0.0f) return tri_pick(s, A, D, C, adc[0], adc[1], adc[2], adc[3]);
  if (tu < 0.0f && bcd[0] > 0.0f && bcd[1] > 0.0f && bcd[2] > 0.0f) return tri_pick(s, B, C, D, bcd[0], bcd[1], bcd[2], bcd[3]);
  if (td <= 0.0f) return false;
  s.v[0].a = tu / td; s.v[1].a = tv / td; s.v[2].a = tw / td; s.v[3].a = tx / td;
  return true;
}
inline void witness(const Simplex& s, V3* a, V3* b) {                              // :496
  const SVert* v = s.v;
  switch (s.count) {
    case 1: *a = v[0].wa; *b = v[0].wb; break;
    case 2: *a = blend2(v[0].a, v[0].wa, v[1].a, v[1].wa); *b = blend2(v[0].a, v[0].wb, v[1].a, v[1].wb); break;
    case 3:
      *a = blend3(v[0].a, v[0].wa, v[1].a, v[1].wa, v[2].a, v[2].wa);
      *b = blend3(v[0].a, v[0].wb, v[1].a, v[1].wb, v[2].a, v[2].wb);
      break;
    case 4: {
      V3 sum = blend2(v[0].a, v[0].wa, v[1].a, v[1].wa) + blend2(v[2].a, v[2].wa, v[3].a, v[3].wa);
      *a = sum; *b = sum;
      break;
    }
    default: break;
  }
}
inline V3 closest_on_simplex(const Simplex& s) {                                   // :525
  const SVert* v = s.v;
  switch (s.count) {
    case 1: return v[0].w;
    case 2: return blend2(v[0].a, v[0].w, v[1].a, v[1].w);
    case 3: return blend3(v[0].a, v[0].w, v[1].a, v[1].w, v[2].a, v[2].w);
    case 4: return blend2(v[0].a, v[0].w, v[1].a, v[1].w) + blend2(v[2].a, v[2].w, v[3].a, v[3].w);
  }
  return v3(0, 0, 0);
}

// distance.rs:543 shape_distance with use_radii = false (the only form used here)
inline DistOut shape_distance(const V3* pa, int na, const V3* pb, int nb, Xf x, SimplexCache* cache) {
  M3 m = matrix_from_quat(x.q);
  M3 mt = transpose(m);
  Simplex s;
  s.count = cache->count;
  for (int i = 0; i < cache->count; ++i) {
    int i1 = cache->ia[i], i2 = cache->ib[i];
    V3 w1 = pa[i1];
    V3 w2 = mul_mv(m, pb[i2]) + x.p;
    s.v[i].ia = i1; s.v[i].ib = i2; s.v[i].wa = w1; s.v[i].wb = w2; s.v[i].w = w2 - w1; s.v[i].a = 0.0f;
  }
  if (s.count > 0) {
    real m1 = cache->metric, m2 = simplex_metric(s);
    if (2.0f * m1 < m2 || m2 < 0.5f * m1 || m2 < kEps) s.count = 0;
  }
  if (s.count == 0) {
    V3 w1 = pa[0], w2 = mul_mv(m, pb[0]) + x.p;
    s.count = 1;
    s.v[0].ia = 0; s.v[0].ib = 0; s.v[0].wa = w1; s.v[0].wb = w2; s.v[0].w = w2 - w1; s.v[0].a = 0.0f;
  }
  Simplex backup;
  DistOut out;
  out.pa = out.pb = out.normal = v3(0, 0, 0);
  out.distance = 0;
  real dsq = kFltMax;
  V3 normal = v3(0, 0, 0);
  int it = 0;
  while (it < 32) {
    bool solved;
    switch (s.count) {
      case 1: s.v[0].a = 1.0f; solved = true; break;
      case 2: solved = solve2(s); break;
      case 3: solved = solve3(s); break;
      default: solved = solve4(s); break;
    }
    if (!solved) { s = backup; break; }
    if (s.count == 4) {
      witness(s, &out.pa, &out.pb);
      out.normal = v3(0, 0, 0);
      out.distance = 0.0f;
      return out;
    }
    real old = dsq;
    V3 cp = closest_on_simplex(s);
    dsq = dot(cp, cp);
    if (dsq >= old) { s = backup; break; }
    V3 sd;
    if (s.count == 1) {
      sd = -s.v[0].w;
    } else if (s.count == 2) {
      V3 a = s.v[0].w, b = s.v[1].w, ab = b - a;
      sd = cross(cross(ab, -a), ab);
    } else {
      V3 a = s.v[0].w, b = s.v[1].w, c = s.v[2].w;
      V3 n = cross(b - a, c - a);
      sd = dot(n, a) < 0.0f ? n : -n;
    }
    if (length_sq(sd) < 1000.0f * kMinPositive) {
      witness(s, &out.pa, &out.pb);
      out.normal = v3(0, 0, 0);
      out.distance = 0.0f;
      return out;
    }
    normal = -sd;
    int ia = point_support(pa, na, -sd);
    V3 sa = pa[ia];
    V3 sd2 = mul_mv(mt, sd);
    int ib = point_support(pb, nb, sd2);
    V3 sb = mul_mv(m, pb[ib]) + x.p;
    backup = s;
    bool dup = false;
    for (int i = 0; i < s.count; ++i)
      if (s.v[i].ia == ia && s.v[i].ib == ib) { dup = true; break; }
    if (dup) break;
    int k = s.count;
    s.v[k].ia = ia; s.v[k].ib = ib; s.v[k].wa = sa; s.v[k].wb = sb; s.v[k].w = sb - sa;
    s.count += 1;
    it++;
  }
  witness(s, &out.pa, &out.pb);
  normal = normalize(normal);
  if (!is_normalized(normal)) {
    out.distance = 0.0f;
    out.normal = v3(0, 0, 0);
    return out;
  }
  out.distance = distance(out.pa, out.pb);
  out.normal = normal;
  cache->metric = simplex_metric(s);
  cache->count = (uint16_t)s.count;
  for (int i = 0; i < s.count; ++i) { cache->ia[i] = (uint8_t)s.v[i].ia; cache->ib[i] = (uint8_t)s.v[i].ib; }
  return out;
}

// convex_manifold_shapes.rs:132
inline void collide_hull_sphere(LocalManifold* m, const Hull& ha, Sphere b, Xf xb, SimplexCache* cache) {
  m->point_count = 0;
  V3 c = xf_point(xb, b.center);
  real spec = speculative_distance();
  DistOut d = shape_distance(ha.points, ha.vertex_count, &c, 1, xf(v3(0, 0, 0), qid()), cache);
  real ra = 0.0f, rb = b.radius, r = ra + rb;
  if (d.distance > r + spec) { *cache = SimplexCache(); return; }
  if (d.distance > 100.0f * kEps) {
    V3 n = normalize(d.pb - d.pa);
    V3 ca = mul_add(c, ra - dot(c - d.pa, n), n);
    V3 cb = mul_sub(c, rb, n);
    m->normal = n;
    m->point_count = 1;
    m->points[0].point = lerp(ca, cb, 0.5f);
    m->points[0].separation = d.distance - r;
    m->points[0].pair = FeaturePair();
  } else {
    int best = -1;
    real best_d = -kFltMax;
    for (int i = 0; i < ha.face_count; ++i) {
      real dd = plane_sep(ha.planes[i], c);
      if (dd > best_d) { best = i; best_d = dd; }
    }
    V3 n = ha.planes[best].n;
    V3 ca = mul_add(c, ra - dot(c - d.pa, n), n);
    V3 cb = mul_sub(c, rb, n);
    m->normal = n;
    m->point_count = 1;
    m->points[0].point = lerp(ca, cb, 0.5f);
    m->points[0].separation = best_d - r;
    m->points[0].pair = FeaturePair();
  }
}

// convex_manifold_shapes.rs:245
inline void collide_capsules(LocalManifold* m, Capsule a, Capsule b, Xf xb) {
  m->point_count = 0;
  V3 a1 = a.c1, a2 = a.c2;
  V3 b1 = xf_point(xb, b.c1), b2 = xf_point(xb, b.c2);
  real radius = a.radius + b.radius;
  real maxd = radius + speculative_distance();
  SegResult res = segment_distance(a1, a2, b1, b2);
  V3 off = res.p2 - res.p1;
  real dsq = length_sq(off);
  real ls = linear_slop();
  real mind = 0.01f * ls;
  if (dsq > maxd * maxd || dsq < mind * mind) return;
  V3 ea, eb;
  real la = get_length_and_normalize(a2 - a1, &ea);
  if (la < min_capsule_length()) return;
  real lb = get_length_and_normalize(b2 - b1, &eb);
  if (lb < min_capsule_length()) return;
  const real at = 0.05f;
  real at2 = at * at;
  V3 axis = cross(ea, eb);
  if (length_sq(axis) < at2) {
    Plane pa0 = plane(-ea, -dot(ea, a.c1));
    Plane pa1 = plane(ea, dot(ea, a.c2));
    ClipVertex vb[2];
    vb[0].position = b1; vb[0].separation = 0.0f; vb[0].pair = make_feature_pair(0, 0, 0, 0);
    vb[1].position = b2; vb[1].separation = 0.0f; vb[1].pair = make_feature_pair(0, 1, 0, 1);
    int pc = clip_segment(vb, pa0);
    if (pc == 2) pc = clip_segment(vb, pa1);
    if (pc == 2) {
      V3 cp1 = point_to_segment(a1, a2, vb[0].position);
      V3 cp2 = point_to_segment(a1, a2, vb[1].position);
      real d1 = distance(cp1, vb[0].position);
      real d2 = distance(cp2, vb[1].position);
      if (d1 <= radius && d2 <= radius) {
        if (d1 < mind || d2 < mind) return;
        V3 n1 = (1.0f / d1) * (vb[0].position - cp1);
        V3 n2 = (1.0f / d2) * (vb[1].position - cp2);
        V3 n = normalize(n1 + n2);
        real ra = a.radius, rb = b.radius;
        V3 p1 = 0.5f * mul_sub(mul_add(vb[0].position, ra, n1) + cp1, rb, n);
        V3 p2 = 0.5f * mul_sub(mul_add(vb[1].position, ra, n2) + cp2, rb, n);
        m->normal = n;
        m->point_count = 2;
        m->points[0].point = p1; m->points[0].separation = d1 - radius; m->points[0].pair = vb[0].pair;
        m->points[1].point = p2; m->points[1].separation = d2 - radius; m->points[1].pair = vb[1].pair;
        return;
      }
    }
  }
  V3 n;
  real dv = get_length_and_normalize(off, &n);
  V3 point = 0.5f * mul_sub(mul_add(res.p1, a.radius, n) + res.p2, b.radius, n);
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = point;
  m->points[0].separation = dv - radius;
  m->points[0].pair = FeaturePair();
}

// convex_manifold_shapes.rs:393
inline SepAxis query_face_hull_capsule(const Hull& h, Capsule c, Xf t) {
  int mf = -1, mv = -1;
  real ms = -kFltMax;
  V3 cpts[2] = {xf_point(t, c.c1), xf_point(t, c.c2)};
  for (int f = 0; f < h.face_count; ++f) {
    Plane p = h.planes[f];
    int vi = point_support(cpts, 2, -p.n);
    real sep = plane_sep(p, cpts[vi]);
    if (sep > ms) { mv = vi; mf = f; ms = sep; }
  }
  SepAxis r = {h.planes[mf].n, ms, mf, mv, kFaceAxisA};
  return r;
}
// convex_manifold_shapes.rs:431
inline SepAxis query_edge_hull_capsule(const Hull& h, Capsule c, Xf t) {
  V3 mn = v3(0, 0, 0);
  real ms = -kFltMax;
  int mia = kNull, mib = kNull;
  V3 pa = xf_point(t, c.c1), qa = xf_point(t, c.c2);
  V3 ea = qa - pa;
  real sq = kParallelEdgeTol * kParallelEdgeTol;
  for (int i = 0; i < h.edge_count; i += 2) {
    HalfEdge e = h.edges[i], tw = h.edges[i + 1];
    V3 qb = h.points[tw.origin];
    V3 ub = h.planes[e.face].n, vb = h.planes[tw.face].n;
    real cba = dot(ub, ea), dba = dot(vb, ea);
    if (cba * dba < 0.0f) {
      if (maxf(cba * cba, dba * dba) < sq * length_sq(ea)) continue;
      real tt = cba / (cba - dba);
      V3 axis = normalize(lerp(ub, vb, tt));
      real sep = dot(axis, qa - qb);
      if (sep > ms) { mn = axis; ms = sep; mia = 0; mib = i; }
    }
  }
  SepAxis r = {mn, ms, mia, mib, kEdgePairAxis};
  return r;
}
// convex_manifold_shapes.rs:499
inline bool build_hull_face_capsule(LocalManifold* m, const Hull& ha, Capsule b, Xf xb, SepAxis q) {
  int rf = q.index_a;
  Plane rp = ha.planes[rf];
  ClipVertex sb[2];
  sb[0].position = xf_point(xb, b.c1); sb[0].separation = 0; sb[0].pair = make_feature_pair(0, 0, 0, 0);
  sb[1].position = xf_point(xb, b.c2); sb[1].separation = 0; sb[1].pair = make_feature_pair(0, 1, 0, 1);
  int pc = clip_segment_to_hull_face(sb, ha, rf);
  if (pc < 2) return false;
  real d1 = plane_sep(rp, sb[0].position), d2 = plane_sep(rp, sb[1].position);
  real spec = speculative_distance();
  if (d1 <= spec || d2 <= spec) {
    V3 n = rp.n;
    V3 p1 = mul_sub(sb[0].position, 0.5f * (d1 + b.radius), n);
    V3 p2 = mul_sub(sb[1].position, 0.5f * (d2 + b.radius), n);
    m->normal = n;
    m->point_count = 2;
    m->points[0].point = p1; m->points[0].separation = d1 - b.radius; m->points[0].pair = sb[0].pair;
    m->points[1].point = p2; m->points[1].separation = d2 - b.radius; m->points[1].pair = sb[1].pair;
    return true;
  }
  return false;
}
// convex_manifold_shapes.rs:554
inline bool build_hull_capsule_edge(LocalManifold* m, const Hull& ha, Capsule b, Xf xb, SepAxis q) {
  V3 pc = xf_point(xb, b.c1), qc = xf_point(xb, b.c2);
  V3 ec = qc - pc;
  HalfEdge e2 = ha.edges[q.index_b];
  HalfEdge t2 = ha.edges[e2.twin];
  V3 ph = ha.points[e2.origin], qh = ha.points[t2.origin];
  V3 eh = qh - ph;
  V3 n = q.normal;
  SegResult r = line_distance(ph, eh, pc, ec);
  if (!within_segments(r)) return false;
  V3 point = 0.5f * (mul_sub(r.p1, b.radius, n) + r.p2);
  real sep = dot(n, r.p2 - r.p1);
  m->normal = n;
  m->point_count = 1;
  m->points[0].point = point;
  m->points[0].separation = sep - b.radius;
  m->points[0].pair = make_feature_pair(0, q.index_a, 1, q.index_b);
  return true;
}
// convex_manifold_shapes.rs:643
inline void collide_hull_capsule(LocalManifold* m, const Hull& ha, Capsule b, Xf xb, SimplexCache* cache) {
  m->point_count = 0;
  V3 cpts[2] = {b.c1, b.c2};
  DistOut d = shape_distance(ha.points, ha.vertex_count, cpts, 2, xb, cache);
  real spec = speculative_distance();
  if (d.distance > b.radius + spec) { *cache = SimplexCache(); return; }
  if (d.distance > 100.0f * kEps) {
    V3 delta = d.normal;
    int rf = find_hull_support_face(ha, delta);
    Plane rp = ha.planes[rf];
    const real kt = 0.998f;
    if (absf(dot(rp.n, delta)) > kt) {
      ClipVertex vb[2];
      vb[0].position = xf_point(xb, b.c1); vb[0].separation = 0; vb[0].pair = make_feature_pair(0, 0, 0, 0);
      vb[1].position = xf_point(xb, b.c2); vb[1].separation = 0; vb[1].pair = make_feature_pair(0, 1, 0, 1);
      int pc = clip_segment_to_hull_face(vb, ha, rf);
      if (pc == 2) {
        real d1 = plane_sep(rp, vb[0].position), d2 = plane_sep(rp, vb[1].position);
        if (d1 <= b.radius + spec || d2 <= b.radius + spec) {
          V3 n = rp.n;
          V3 p1 = mul_sub(vb[0].position, 0.5f * (b.radius + d1), n);
          V3 p2 = mul_sub(vb[1].position, 0.5f * (b.radius + d2), n);
          m->normal = n;
          m->point_count = 2;
          m->points[0].point = p1; m->points[0].separation = d1 - b.radius; m->points[0].pair = vb[0].pair;
          m->points[1].point = p2; m->points[1].separation = d2 - b.radius; m->points[1].pair = vb[1].pair;
          return;
        }
      }
    }
    V3 point = 0.5f * (mul_sub(d.pa, b.radius, delta) + d.pb);
    m->normal = delta;
    m->point_count = 1;
    m->points[0].point = point;
    m->points[0].separation = d.distance - b.radius;
    m->points[0].pair = FeaturePair();
    return;
  }
  SepAxis fq = query_face_hull_capsule(ha, b, xb);
  if (fq.separation > b.radius) return;
  SepAxis eq = query_edge_hull_capsule(ha, b, xb);
  if (eq.separation > b.radius) return;
  real face_sep = fq.separation - b.radius;
  build_hull_face_capsule(m, ha, b, xb, fq);
  if (m->point_count == 2) face_sep = minf(m->points[0].separation, m->points[1].separation);
  if (eq.index_a == kNull) return;
  real ls = linear_slop();
  real edge_sep = eq.separation - b.radius;
  if (m->point_count == 0 || edge_sep > face_sep + ls) {
    build_hull_capsule_edge(m, ha, b, xb, eq);
  }
}

}  // namespace nso
