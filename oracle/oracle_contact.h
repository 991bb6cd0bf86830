// TEST INFRASTRUCTURE ONLY — CPU oracle, contact half: restates the
// reference's IPC barrier, distance primitives, CCD and BVH broad phase.
// Never linked into the product.
#pragma once
#include <vector>
#include <cstdint>
#include <cmath>
#include <algorithm>
#include "oracle_math.h"

namespace orc {

// ---------------------------------------------------------------- barrier
// crates/vistio-contact/src/barrier.rs. All d are SQUARED distances. The API
// type is R (f32 in the reference); the internals are f64 as in the reference.
template <class R> R barrier_energy(R d, R d_hat) {  // barrier.rs:18
  if (d >= d_hat || d <= R(0)) return R(0);
  double d64 = d, dh = d_hat, diff = d64 - dh, ratio = d64 / dh;
  return R(-(diff * diff) * std::log(ratio));
}
template <class R> R barrier_gradient(R d, R d_hat) {  // barrier.rs:35
  R d_c = rmin(rmax(d, d_hat * R(1e-3f)), d_hat);
  if (d_c >= d_hat) return R(0);
  double d64 = d_c, dh = d_hat, diff = d64 - dh, ln_ratio = std::log(d64 / dh);
  return R(-(diff) * (2.0 * ln_ratio + diff / d64));
}
template <class R> R barrier_hessian(R d, R d_hat) {  // barrier.rs:53
  if (d >= d_hat || d <= R(0)) return R(0);
  double d64 = d, dh = d_hat, diff = d64 - dh, ln_ratio = std::log(d64 / dh), inv_d = 1.0 / d64;
  return R(-2.0 * ln_ratio - 4.0 * diff * inv_d + diff * diff * inv_d * inv_d);
}
template <class R> R signum(R v) { return std::signbit(v) ? R(-1) : R(1); }
template <class R> R scaled_barrier_gradient(R d, R d_hat, R kappa) {  // barrier.rs:78
  R raw = barrier_gradient(d, d_hat);
  R result = kappa * raw;
  if (std::isfinite(result)) return result;
  return signum(result) * R(1e6f);
}
template <class R> R estimate_initial_kappa(R configured, R avg_mass, R g, R d_hat) {  // barrier.rs:97
  if (configured > R(0)) return configured;
  R d_mid = d_hat * R(0.5);
  R grad_at_mid = std::fabs(barrier_gradient(d_mid, d_hat));
  if (grad_at_mid < R(1e-12f)) return R(1e4f);
  R kappa = avg_mass * g / (R(2) * std::sqrt(d_mid) * grad_at_mid);
  return rclamp(kappa, R(1), R(1e6f));
}
template <class R> R barrier_energy_with_thickness(R d, R d_hat, R t) {  // barrier.rs:126
  R t_sq = t * t, d_eff = d - t_sq;
  if (d_eff <= R(0)) return R(1e6f);
  return barrier_energy(d_eff, d_hat);
}
template <class R> R barrier_gradient_with_thickness(R d, R d_hat, R t) {  // barrier.rs:138
  R t_sq = t * t, d_eff = d - t_sq;
  if (d_eff <= R(0)) return barrier_gradient(R(1e-12f), d_hat);
  return barrier_gradient(d_eff, d_hat);
}
template <class R> R scaled_barrier_gradient_with_thickness(R d, R d_hat, R kappa, R t) {  // barrier.rs:149
  R raw = barrier_gradient_with_thickness(d, d_hat, t);
  R result = kappa * raw;
  if (std::isfinite(result)) return result;
  return signum(result) * R(1e6f);
}

// ---------------------------------------------------- distance primitives
// crates/vistio-contact/src/distance_primitives.rs
enum DistType { DT_FACE = 0, DT_EDGE0 = 1, DT_EDGE1 = 2, DT_EDGE2 = 3, DT_VERT0 = 4, DT_VERT1 = 5,
                DT_VERT2 = 6, DT_EE = 7, DT_DEGEN = 8 };

template <class R> R point_segment_distance_squared(V3<R> p, V3<R> a, V3<R> b) {  // :308
  V3<R> ab = b - a, ap = p - a;
  R ab_sq = ab.length_squared();
  if (ab_sq < R(1e-20f)) return ap.length_squared();
  R t = rclamp(ap.dot(ab) / ab_sq, R(0), R(1));
  V3<R> closest = a + ab * t;
  return (p - closest).length_squared();
}

template <class R>
R point_triangle_distance_squared(V3<R> p, V3<R> a, V3<R> b, V3<R> c, int* dtype) {  // :36
  V3<R> ab = b - a, ac = c - a, ap = p - a, bp = p - b, cp = p - c;
  V3<R> normal = ab.cross(ac);
  R area2_sq = normal.length_squared();
  if (area2_sq < R(1e-20f)) {
    R d_ab = point_segment_distance_squared(p, a, b);
    R d_bc = point_segment_distance_squared(p, b, c);
    R d_ca = point_segment_distance_squared(p, c, a);
    if (d_ab <= d_bc && d_ab <= d_ca) { *dtype = DT_EDGE0; return d_ab; }
    if (d_bc <= d_ca) { *dtype = DT_EDGE1; return d_bc; }
    *dtype = DT_EDGE2; return d_ca;
  }
  R d1 = ab.dot(ap), d2 = ac.dot(ap);
  if (d1 <= R(0) && d2 <= R(0)) { *dtype = DT_VERT0; return ap.length_squared(); }
  R d3 = ab.dot(bp), d4 = ac.dot(bp);
  if (d3 >= R(0) && d4 <= d3) { *dtype = DT_VERT1; return bp.length_squared(); }
  R d5 = ab.dot(cp), d6 = ac.dot(cp);
  if (d6 >= R(0) && d5 <= d6) { *dtype = DT_VERT2; return cp.length_squared(); }
  R vc = d1 * d4 - d3 * d2;
  if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) {
    R v = d1 / (d1 - d3);
    V3<R> closest = a + ab * v;
    *dtype = DT_EDGE0; return (p - closest).length_squared();
  }
  R va = d3 * d6 - d5 * d4;
  if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) {
    R w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    V3<R> closest = b + (c - b) * w;
    *dtype = DT_EDGE1; return (p - closest).length_squared();
  }
  R vb = d5 * d2 - d1 * d6;
  if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) {
    R w = d2 / (d2 - d6);
    V3<R> closest = a + ac * w;
    *dtype = DT_EDGE2; return (p - closest).length_squared();
  }
  R denom = R(1) / (va + vb + vc);
  R v = vb * denom, w = vc * denom;
  V3<R> closest = a + ab * v + ac * w;
  *dtype = DT_FACE;
  return (p - closest).length_squared();
}

template <class R>
void point_triangle_distance_gradient(V3<R> p, V3<R> a, V3<R> b, V3<R> c, V3<R> g[4]) {  // :124
  V3<R> ab = b - a, ac = c - a, normal = ab.cross(ac);
  R area2_sq = normal.length_squared();
  for (int k = 0; k < 4; ++k) g[k] = V3<R>();
  if (area2_sq < R(1e-20f)) return;
  V3<R> n = normal / std::sqrt(area2_sq);
  V3<R> ap = p - a;
  R signed_dist = ap.dot(n);
  V3<R> projected = p - n * signed_dist;
  V3<R> v0 = b - a, v1 = c - a, v2 = projected - a;
  R d00 = v0.dot(v0), d01 = v0.dot(v1), d11 = v1.dot(v1), d20 = v2.dot(v0), d21 = v2.dot(v1);
  R denom = d00 * d11 - d01 * d01;
  if (std::fabs(denom) < R(1e-20f)) return;
  R inv = R(1) / denom;
  R v = (d11 * d20 - d01 * d21) * inv;
  R w = (d00 * d21 - d01 * d20) * inv;
  R u = R(1) - v - w;
  V3<R> closest = a * u + b * v + c * w;
  V3<R> diff = p - closest;
  g[0] = diff * R(2);
  g[1] = -diff * (R(2) * u);
  g[2] = -diff * (R(2) * v);
  g[3] = -diff * (R(2) * w);
}

template <class R>
R edge_edge_distance_squared(V3<R> a0, V3<R> a1, V3<R> b0, V3<R> b1, int* dtype) {  // :185
  V3<R> d1 = a1 - a0, d2 = b1 - b0, r = a0 - b0;
  R a = d1.dot(d1), e = d2.dot(d2), f = d2.dot(r);
  const R eps = R(1e-10f);
  if (a < eps && e < eps) { *dtype = DT_DEGEN; return r.length_squared(); }
  R s, t;
  if (a < eps) {
    t = rclamp(f / e, R(0), R(1)); s = R(0);
  } else {
    R c = d1.dot(r);
    if (e < eps) {
      s = rclamp(-c / a, R(0), R(1)); t = R(0);
    } else {
      R b = d1.dot(d2);
      R denom = a * e - b * b;
      s = std::fabs(denom) > eps ? rclamp((b * f - c * e) / denom, R(0), R(1)) : R(0);
      t = (b * s + f) / e;
      if (t < R(0)) { t = R(0); s = rclamp(-c / a, R(0), R(1)); }
      else if (t > R(1)) { t = R(1); s = rclamp((b - c) / a, R(0), R(1)); }
    }
  }
  V3<R> c1 = a0 + d1 * s, c2 = b0 + d2 * t, diff = c1 - c2;
  *dtype = DT_EE;
  return diff.length_squared();
}

template <class R>
void edge_edge_distance_gradient(V3<R> a0, V3<R> a1, V3<R> b0, V3<R> b1, V3<R> g[4]) {  // :251
  V3<R> d1 = a1 - a0, d2 = b1 - b0, r = a0 - b0;
  R a = d1.dot(d1), e = d2.dot(d2), f = d2.dot(r), c = d1.dot(r), bv = d1.dot(d2);
  const R eps = R(1e-10f);
  R s, t;
  if (a < eps || e < eps) { s = R(0); t = R(0); }
  else {
    R denom = a * e - bv * bv;
    s = std::fabs(denom) > eps ? rclamp((bv * f - c * e) / denom, R(0), R(1)) : R(0);
    t = (bv * s + f) / e;
    if (t < R(0)) { t = R(0); s = rclamp(-c / a, R(0), R(1)); }
    else if (t > R(1)) { t = R(1); s = rclamp((bv - c) / a, R(0), R(1)); }
  }
  V3<R> c1 = a0 + d1 * s, c2 = b0 + d2 * t, diff = c1 - c2;
  g[0] = diff * (R(2) * (R(1) - s));
  g[1] = diff * (R(2) * s);
  g[2] = -diff * (R(2) * (R(1) - t));
  g[3] = -diff * (R(2) * t);
}

// ------------------------------------------------------------------- CCD
// crates/vistio-contact/src/ccd.rs
template <class R> int solve_quadratic_roots(R a, R b, R c, R out[3]) {  // ccd.rs:354
  const R eps = R(1e-8f);
  if (std::fabs(a) < eps) {
    if (std::fabs(b) < eps) return 0;
    out[0] = -c / b; return 1;
  }
  R disc = b * b - R(4) * a * c;
  if (disc < -eps) return 0;
  if (std::fabs(disc) <= eps) { out[0] = -b / (R(2) * a); return 1; }
  R sd = std::sqrt(disc);
  out[0] = (-b + sd) / (R(2) * a);
  out[1] = (-b - sd) / (R(2) * a);
  return 2;
}
template <class R> int solve_cubic_roots(R a, R b, R c, R d, R out[3]) {  // ccd.rs:299
  const R eps = R(1e-8f);
  if (std::fabs(a) < eps) return solve_quadratic_roots(b, c, d, out);
  R p = b / a, q = c / a, r = d / a;
  R a_dep = q - p * p / R(3);
  R b_dep = r - p * q / R(3) + R(2) * p * p * p / R(27);
  R disc = b_dep * b_dep / R(4) + a_dep * a_dep * a_dep / R(27);
  R shift = -p / R(3);
  if (disc > eps) {
    R sd = std::sqrt(disc);
    R u = std::cbrt(-b_dep / R(2) + sd);
    R v = std::cbrt(-b_dep / R(2) - sd);
    out[0] = u + v + shift; return 1;
  } else if (std::fabs(disc) <= eps) {
    if (std::fabs(b_dep) < eps) { out[0] = shift; return 1; }
    R u = std::cbrt(b_dep / R(2));
    out[0] = R(-2) * u + shift; out[1] = u + shift; return 2;
  }
  R r_val = std::sqrt(-a_dep * a_dep * a_dep / R(27));
  if (std::fabs(r_val) < R(1e-12f)) { out[0] = shift; return 1; }
  R cos_val = rclamp(-b_dep / (R(2) * r_val), R(-1), R(1));
  R theta = std::acos(cos_val);
  R m = R(2) * std::cbrt(r_val);
  const R pi = R(3.14159265358979323846);
  out[0] = m * std::cos(theta / R(3)) + shift;
  out[1] = m * std::cos((theta + R(2) * pi) / R(3)) + shift;
  out[2] = m * std::cos((theta + R(4) * pi) / R(3)) + shift;
  return 3;
}

// ccd.rs:32-129 vertex_triangle_ccd; returns true and the safe TOI on a hit.
template <class R>
bool vertex_triangle_ccd(V3<R> p0, V3<R> p1, V3<R> a0, V3<R> a1, V3<R> b0, V3<R> b1,
                         V3<R> c0, V3<R> c1, R* toi_out) {
  const R margin = R(0.9f), min_toi = R(1e-6f);
  V3<R> dp = p1 - p0, da = a1 - a0, db = b1 - b0, dc = c1 - c0;
  V3<R> a_r = a0 - p0, b_r = b0 - p0, c_r = c0 - p0;
  V3<R> a_v = da - dp, b_v = db - dp, c_v = dc - dp;
  V3<R> bv_x_cv = b_v.cross(c_v), br_x_cv = b_r.cross(c_v), bv_x_cr = b_v.cross(c_r),
        br_x_cr = b_r.cross(c_r);
  R ca = a_v.dot(bv_x_cv);
  R cb = a_r.dot(bv_x_cv) + a_v.dot(br_x_cv + bv_x_cr);
  R cc = a_r.dot(br_x_cv + bv_x_cr) + a_v.dot(br_x_cr);
  R cd = a_r.dot(br_x_cr);
  R roots[3];
  int nr = solve_cubic_roots(ca, cb, cc, cd, roots);
  bool hit = false;
  R best = R(0);
  for (int i = 0; i < nr; ++i) {
    R t = roots[i];
    if (t < -min_toi || t > R(1) + min_toi) continue;
    t = rclamp(t, R(0), R(1));
    V3<R> pa = a_r + a_v * t, pb = b_r + b_v * t, pc = c_r + c_v * t;
    V3<R> n = (pb - pa).cross(pc - pa);
    if (n.length_squared() < R(1e-20f)) continue;
    V3<R> v0 = pb - pa, v1 = pc - pa, v2 = V3<R>() - pa;
    R d00 = v0.dot(v0), d01 = v0.dot(v1), d11 = v1.dot(v1), d20 = v2.dot(v0), d21 = v2.dot(v1);
    R denom = d00 * d11 - d01 * d01;
    if (std::fabs(denom) < R(1e-20f)) continue;
    R inv = R(1) / denom;
    R u = (d11 * d20 - d01 * d21) * inv;
    R w = (d00 * d21 - d01 * d20) * inv;
    R v = R(1) - u - w;
    const R tol = R(0.01f);
    if (v >= -tol && u >= -tol && w >= -tol) {
      R safe = rmax(t * margin, min_toi);
      best = hit ? rmin(best, safe) : safe;
      hit = true;
    }
  }
  if (hit) *toi_out = best;
  return hit;
}

// ccd.rs:138-228 edge_edge_ccd (not called by the pipeline; KAT only).
template <class R>
bool edge_edge_ccd(V3<R> a0, V3<R> a1, V3<R> b0, V3<R> b1, V3<R> c0, V3<R> c1, V3<R> d0,
                   V3<R> d1, R* toi_out) {
  const R margin = R(0.9f), min_toi = R(1e-6f);
  V3<R> da = a1 - a0, db = b1 - b0, dc = c1 - c0, dd = d1 - d0;
  V3<R> r0 = c0 - a0, rv = dc - da, e10 = b0 - a0, e1v = db - da, e20 = d0 - c0, e2v = dd - dc;
  V3<R> e1v_x_e2v = e1v.cross(e2v), e10_x_e2v = e10.cross(e2v), e1v_x_e20 = e1v.cross(e20),
        e10_x_e20 = e10.cross(e20);
  R ca = rv.dot(e1v_x_e2v);
  R cb = r0.dot(e1v_x_e2v) + rv.dot(e10_x_e2v + e1v_x_e20);
  R cc = r0.dot(e10_x_e2v + e1v_x_e20) + rv.dot(e10_x_e20);
  R cd = r0.dot(e10_x_e20);
  R roots[3];
  int nr = solve_cubic_roots(ca, cb, cc, cd, roots);
  bool hit = false;
  R best = R(0);
  for (int i = 0; i < nr; ++i) {
    R t = roots[i];
    if (t < -min_toi || t > R(1) + min_toi) continue;
    t = rclamp(t, R(0), R(1));
    V3<R> at = a0 + da * t, bt = b0 + db * t, ct = c0 + dc * t, dt = d0 + dd * t;
    V3<R> e1 = bt - at, e2 = dt - ct, r = ct - at;
    R l1 = e1.dot(e1), l2 = e2.dot(e2);
    if (l1 < R(1e-20f) || l2 < R(1e-20f)) continue;
    R bv = e1.dot(e2), fv = e2.dot(r), cv = e1.dot(r);
    R denom = l1 * l2 - bv * bv;
    if (std::fabs(denom) < R(1e-10f)) continue;
    R s = rclamp((bv * fv - cv * l2) / denom, R(0), R(1));
    R u = rclamp((bv * s + fv) / l2, R(0), R(1));
    const R tol = R(0.05f);
    if (s >= -tol && s <= R(1) + tol && u >= -tol && u <= R(1) + tol) {
      R safe = rmax(t * margin, min_toi);
      best = hit ? rmin(best, safe) : safe;
      hit = true;
    }
  }
  if (hit) *toi_out = best;
  return hit;
}

// ------------------------------------------------------------------- BVH
// crates/vistio-contact/src/bvh.rs
struct Aabb {
  float mn[3], mx[3];
  bool overlaps(const Aabb& o) const {  // bvh.rs:58
    return mn[0] <= o.mx[0] && mx[0] >= o.mn[0] && mn[1] <= o.mx[1] && mx[1] >= o.mn[1] &&
           mn[2] <= o.mx[2] && mx[2] >= o.mn[2];
  }
  static Aabb merge(const Aabb& a, const Aabb& b) {
    Aabb r;
    for (int k = 0; k < 3; ++k) { r.mn[k] = std::fmin(a.mn[k], b.mn[k]); r.mx[k] = std::fmax(a.mx[k], b.mx[k]); }
    return r;
  }
  int longest_axis() const {  // bvh.rs:74
    float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    if (dx >= dy && dx >= dz) return 0;
    if (dy >= dz) return 1;
    return 2;
  }
  float centroid(int k) const { return (mn[k] + mx[k]) * 0.5f; }
};

// bvh.rs:29 Aabb::from_triangle
inline Aabb tri_aabb(const float* px, const float* py, const float* pz, const uint32_t* t, float m) {
  Aabb a;
  const float* P[3] = {px, py, pz};
  for (int k = 0; k < 3; ++k) {
    float v0 = P[k][t[0]], v1 = P[k][t[1]], v2 = P[k][t[2]];
    a.mn[k] = std::fmin(std::fmin(v0, v1), v2) - m;
    a.mx[k] = std::fmax(std::fmax(v0, v1), v2) + m;
  }
  return a;
}

// The reference's median-split tree (bvh.rs:122-275), kept with its
// self-query's `ta < tb` orientation filter (bvh.rs:205-209).
struct RefBvh {
  struct Node { Aabb box; int leaf; int left, right; };
  std::vector<Node> nodes;
  int root = -1;
  int build_rec(const std::vector<Aabb>& leaves, int* idx, int n) {
    if (n == 1) {
      nodes.push_back({leaves[idx[0]], idx[0], -1, -1});
      return int(nodes.size()) - 1;
    }
    Aabb bounds = leaves[idx[0]];
    for (int i = 1; i < n; ++i) bounds = Aabb::merge(bounds, leaves[idx[i]]);
    int axis = bounds.longest_axis();
    std::stable_sort(idx, idx + n, [&](int a, int b) {
      return leaves[a].centroid(axis) < leaves[b].centroid(axis);
    });
    int mid = n / 2;
    int l = build_rec(leaves, idx, mid);
    int r = build_rec(leaves, idx + mid, n - mid);
    Aabb merged = Aabb::merge(nodes[l].box, nodes[r].box);
    nodes.push_back({merged, -1, l, r});
    return int(nodes.size()) - 1;
  }
  void build(const std::vector<Aabb>& leaves) {
    nodes.clear();
    if (leaves.empty()) { root = -1; return; }
    std::vector<int> idx(leaves.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = int(i);
    root = build_rec(leaves, idx.data(), int(idx.size()));
  }
  Aabb refit_rec(int n, const std::vector<Aabb>& leaves) {
    Node& nd = nodes[n];
    if (nd.leaf >= 0) { nd.box = leaves[nd.leaf]; return nd.box; }
    Aabb l = refit_rec(nd.left, leaves), r = refit_rec(nd.right, leaves);
    nodes[n].box = Aabb::merge(l, r);
    return nodes[n].box;
  }
  void refit(const std::vector<Aabb>& leaves) { if (root >= 0) refit_rec(root, leaves); }
  void query_rec(int a, int b, std::vector<std::pair<uint32_t, uint32_t>>& out) const {
    if (!nodes[a].box.overlaps(nodes[b].box)) return;
    const Node& A = nodes[a];
    const Node& B = nodes[b];
    if (A.leaf >= 0 && B.leaf >= 0) {
      if (A.leaf < B.leaf) out.push_back({uint32_t(A.leaf), uint32_t(B.leaf)});
    } else if (A.leaf < 0 && B.leaf >= 0) {
      query_rec(A.left, b, out); query_rec(A.right, b, out);
    } else if (A.leaf >= 0 && B.leaf < 0) {
      query_rec(a, B.left, out); query_rec(a, B.right, out);
    } else if (a == b) {
      query_rec(A.left, A.left, out); query_rec(A.left, A.right, out); query_rec(A.right, A.right, out);
    } else {
      query_rec(A.left, B.left, out); query_rec(A.left, B.right, out);
      query_rec(A.right, B.left, out); query_rec(A.right, B.right, out);
    }
  }
  std::vector<std::pair<uint32_t, uint32_t>> query() const {
    std::vector<std::pair<uint32_t, uint32_t>> out;
    if (root >= 0) query_rec(root, root, out);
    return out;
  }
};

// The tree-independent candidate set {(ta<tb) : inflated AABBs overlap},
// by sort-and-sweep along x; the result is sorted.
inline std::vector<std::pair<uint32_t, uint32_t>> complete_pairs(const std::vector<Aabb>& boxes) {
  std::vector<uint32_t> order(boxes.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = uint32_t(i);
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    if (boxes[a].mn[0] != boxes[b].mn[0]) return boxes[a].mn[0] < boxes[b].mn[0];
    return a < b;
  });
  std::vector<std::pair<uint32_t, uint32_t>> out;
  for (size_t i = 0; i < order.size(); ++i) {
    const Aabb& A = boxes[order[i]];
    for (size_t j = i + 1; j < order.size(); ++j) {
      const Aabb& B = boxes[order[j]];
      if (B.mn[0] > A.mx[0]) break;
      if (A.overlaps(B)) {
        uint32_t a = order[i], b = order[j];
        out.push_back(a < b ? std::make_pair(a, b) : std::make_pair(b, a));
      }
    }
  }
  std::sort(out.begin(), out.end());
  return out;
}

}  // namespace orc
