// TEST INFRASTRUCTURE ONLY — the CPU oracle for the CUDA PD/IPC path.
//
// A restatement of the reference's CPU hot path (Rust, crates/vistio-*),
// written so tests can check the CUDA library on identical inputs. It is
// the checker, never the thing measured or shipped: the product library
// (vistio_b200/) neither includes nor links it. Modes:
//   ref32 — FP32 arithmetic like the reference (f64 only where the reference
//           uses f64: Cholesky, barrier internals, residual sums);
//   fp64  — the same algorithm in double, the "truth" run.
// Hinges are kept in the canonical order sorted by (v0, v1); the reference's
// order follows a Rust HashMap (crates/vistio-mesh/src/topology.rs:73,88) and
// differs from run to run, so only summation order is affected.
// The global solve uses this file's own FP64 sparse LL^T with a geometric
// nested-dissection ordering; the reference calls faer 0.24's supernodal LL^T
// (crates/vistio-math/src/faer_solver.rs:84-88). Any correct FP64 Cholesky
// gives the same solution up to rounding.
#include "oracle.h"
#include "oracle_math.h"
#include "oracle_contact.h"

#include <vector>
#include <map>
#include <set>
#include <memory>
#include <cstring>
#include <cmath>
#include <limits>
#include <numeric>

using namespace orc;

namespace {

// ------------------------------------------------------------- topology
// crates/vistio-mesh/src/topology.rs:58-121 (interior edges, wing vertices)
struct HingeIdx { uint32_t v0, v1, wa, wb; };

uint32_t find_wing(const uint32_t* tris, uint32_t t, uint32_t v0, uint32_t v1) {  // :158
  uint32_t a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
  if (a != v0 && a != v1) return a;
  if (b != v0 && b != v1) return b;
  return c;
}

std::vector<HingeIdx> build_hinges(uint32_t nt, const uint32_t* tris) {
  std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> edge_map;
  for (uint32_t t = 0; t < nt; ++t) {
    uint32_t a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
    uint32_t e[3][2] = {{a, b}, {b, c}, {c, a}};
    for (auto& ed : e) {
      auto key = ed[0] < ed[1] ? std::make_pair(ed[0], ed[1]) : std::make_pair(ed[1], ed[0]);
      edge_map[key].push_back(t);
    }
  }
  std::vector<HingeIdx> out;
  for (auto& kv : edge_map) {
    if (kv.second.size() == 2) {
      uint32_t v0 = kv.first.first, v1 = kv.first.second;
      out.push_back({v0, v1, find_wing(tris, kv.second[0], v0, v1), find_wing(tris, kv.second[1], v0, v1)});
    }
  }
  return out;
}

// ------------------------------------------------------------- elements
template <class R> struct RestTri { uint32_t idx[3]; R dm_inv[4]; R area; R weight; };

// crates/vistio-solver/src/element.rs:228-263
template <class R> void compute_dm_inv(V3<R> e1, V3<R> e2, R out[4]) {
  out[0] = 1; out[1] = 0; out[2] = 0; out[3] = 1;
  R len_e1 = e1.length();
  if (len_e1 < R(1e-10f)) return;
  V3<R> u = e1 / len_e1;
  V3<R> n = e1.cross(e2);
  R n_len = n.length();
  if (n_len < R(1e-10f)) return;
  V3<R> v = n.cross(u).normalize();
  R dm00 = e1.dot(u), dm10 = e1.dot(v), dm01 = e2.dot(u), dm11 = e2.dot(v);
  R det = dm00 * dm11 - dm01 * dm10;
  if (std::fabs(det) < R(1e-10f)) return;
  R inv_det = R(1) / det;
  out[0] = dm11 * inv_det;
  out[1] = -dm10 * inv_det;
  out[2] = -dm01 * inv_det;
  out[3] = dm00 * inv_det;
}

template <class R> struct BendElem {
  uint32_t v[4];  // v0, v1, wing_a, wing_b
  R rest_angle;
  R stencil[4];
  R weight;
};

// crates/vistio-solver/src/bending.rs:56-91
template <class R> R dihedral_angle(V3<R> p0, V3<R> p1, V3<R> pa, V3<R> pb) {
  const R PI = R(3.14159265358979323846);
  V3<R> edge = p1 - p0;
  R len = edge.length();
  if (len < R(1e-10f)) return PI;
  V3<R> ed = edge / len;
  V3<R> to_a = pa - p0, to_b = pb - p0;
  V3<R> perp_a = to_a - ed * to_a.dot(ed);
  V3<R> perp_b = to_b - ed * to_b.dot(ed);
  R la = perp_a.length(), lb = perp_b.length();
  if (la < R(1e-10f) || lb < R(1e-10f)) return PI;
  perp_a = perp_a / la;
  perp_b = perp_b / lb;
  return std::acos(rclamp(perp_a.dot(perp_b), R(-1), R(1)));
}

template <class R> R clamp_rest_angle(R a) {  // bending.rs:122-128
  const R PI = R(3.14159265358979323846);
  if (std::fabs(a - PI) < R(1e-3f)) return PI;
  if (std::fabs(a) < R(1e-3f)) return R(0);
  return a;
}

// bending.rs:231-239
template <class R> V3<R> rotate_around_axis(V3<R> p, V3<R> c, V3<R> axis, R angle) {
  V3<R> v = p - c;
  R ca = std::cos(angle), sa = std::sin(angle);
  R dot = axis.dot(v);
  V3<R> rotated = v * ca + axis.cross(v) * sa + axis * dot * (R(1) - ca);
  return c + rotated;
}

// bending.rs:182-227 (identical in discrete_shells.rs:285-337)
template <class R>
void bend_project(const BendElem<R>& e, const V3<R>* P, V3<R> out[4]) {
  V3<R> p0 = P[e.v[0]], p1 = P[e.v[1]], pa = P[e.v[2]], pb = P[e.v[3]];
  out[0] = p0; out[1] = p1; out[2] = pa; out[3] = pb;
  R cur = dihedral_angle(p0, p1, pa, pb);
  R diff = cur - e.rest_angle;
  if (std::fabs(diff) < R(1e-8f)) return;
  V3<R> edge = p1 - p0;
  R len = edge.length();
  if (len < R(1e-10f)) return;
  V3<R> axis = edge / len;
  V3<R> to_a = pa - p0, to_b = pb - p0;
  V3<R> p_a = to_a - axis * to_a.dot(axis);
  V3<R> p_b = to_b - axis * to_b.dot(axis);
  V3<R> nc = p_a.cross(p_b);
  R sign = nc.dot(axis) >= R(0) ? R(1) : R(-1);
  R half = diff * R(0.5) * sign;
  V3<R> mid = (p0 + p1) * R(0.5);
  out[2] = rotate_around_axis(pa, mid, axis, half);
  out[3] = rotate_around_axis(pb, mid, axis, -half);
}

// --------------------------------------------------------- sparse LL^T
// FP64 up-looking sparse Cholesky on a nested-dissection ordering.
struct SparseChol {
  int n = 0;
  std::vector<int> perm, iperm;   // perm[new] = old
  std::vector<int> Lp, Li;        // CSC, diagonal first in each column
  std::vector<double> Lx;
  bool ok = false;

  // Geometric nested dissection: split the vertex set at the median of its
  // longest coordinate extent; the vertices of the first half that touch the
  // second half form the separator, ordered last.
  static void nd_order(std::vector<int>& verts, const std::vector<std::vector<int>>& adj,
                       const std::vector<double>& xyz, std::vector<char>& side,
                       std::vector<int>& out) {
    if (verts.size() <= 32) { for (int v : verts) out.push_back(v); return; }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int v : verts)
      for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], xyz[3 * v + k]); hi[k] = std::max(hi[k], xyz[3 * v + k]); }
    int ax = 0;
    for (int k = 1; k < 3; ++k) if (hi[k] - lo[k] > hi[ax] - lo[ax]) ax = k;
    std::stable_sort(verts.begin(), verts.end(), [&](int a, int b) { return xyz[3 * a + ax] < xyz[3 * b + ax]; });
    size_t mid = verts.size() / 2;
    std::vector<int> A(verts.begin(), verts.begin() + mid), B(verts.begin() + mid, verts.end());
    for (int v : B) side[v] = 2;
    std::vector<int> A2, S;
    for (int v : A) {
      bool touch = false;
      for (int u : adj[v]) if (side[u] == 2) { touch = true; break; }
      (touch ? S : A2).push_back(v);
    }
    for (int v : B) side[v] = 0;
    nd_order(A2, adj, xyz, side, out);
    nd_order(B, adj, xyz, side, out);
    for (int v : S) out.push_back(v);
  }

  // A given as CSR (full symmetric pattern, summed values).
  bool factor(int n_, const std::vector<int>& Ap, const std::vector<int>& Aj,
              const std::vector<double>& Ax, const std::vector<double>& xyz) {
    n = n_;
    std::vector<std::vector<int>> adj(n);
    for (int i = 0; i < n; ++i)
      for (int p = Ap[i]; p < Ap[i + 1]; ++p) if (Aj[p] != i) adj[i].push_back(Aj[p]);
    std::vector<int> verts(n);
    std::iota(verts.begin(), verts.end(), 0);
    std::vector<char> side(n, 0);
    perm.clear();
    nd_order(verts, adj, xyz, side, perm);
    iperm.assign(n, 0);
    for (int k = 0; k < n; ++k) iperm[perm[k]] = k;
    // Upper triangle of B = P A P^T, by columns, from A's upper triangle in
    // the original numbering: faer factors with Side::Upper
    // (faer_solver.rs:84-88), and A[i][j], A[j][i] of the assembled matrix
    // can differ in the last bit.
    std::vector<std::vector<std::pair<int, double>>> colsB(n);
    for (int i = 0; i < n; ++i)
      for (int p = Ap[i]; p < Ap[i + 1]; ++p) {
        if (Aj[p] < i) continue;
        int r = iperm[i], c = iperm[Aj[p]];
        colsB[std::max(r, c)].push_back({std::min(r, c), Ax[p]});
      }
    // Elimination tree.
    std::vector<int> parent(n, -1), ancestor(n, -1);
    for (int k = 0; k < n; ++k)
      for (auto& e : colsB[k]) {
        int i = e.first;
        while (i != -1 && i < k) {
          int nxt = ancestor[i];
          ancestor[i] = k;
          if (nxt == -1) { parent[i] = k; break; }
          i = nxt;
        }
      }
    // Row patterns via the etree reach; count, then fill.
    std::vector<int> mark(n, -1), stack(n), pattern(n);
    auto ereach = [&](int k) -> int {
      int top = n;
      mark[k] = k;
      for (auto& e : colsB[k]) {
        int i = e.first;
        if (i >= k) continue;
        int len = 0;
        for (; mark[i] != k; i = parent[i]) { stack[len++] = i; mark[i] = k; }
        while (len > 0) pattern[--top] = stack[--len];
      }
      return top;
    };
    std::vector<int> cnt(n, 1);
    for (int k = 0; k < n; ++k) {
      int top = ereach(k);
      for (int p = top; p < n; ++p) cnt[pattern[p]]++;
    }
    Lp.assign(n + 1, 0);
    for (int k = 0; k < n; ++k) Lp[k + 1] = Lp[k] + cnt[k];
    Li.assign(Lp[n], 0);
    Lx.assign(Lp[n], 0.0);
    std::vector<int> cur(Lp.begin(), Lp.end() - 1);
    std::vector<double> x(n, 0.0);
    std::fill(mark.begin(), mark.end(), -1);
    for (int k = 0; k < n; ++k) {
      int top = ereach(k);
      for (auto& e : colsB[k]) x[e.first] += e.second;
      double d = x[k];
      x[k] = 0;
      for (int p = top; p < n; ++p) {
        int i = pattern[p];
        double lki = x[i] / Lx[Lp[i]];
        x[i] = 0;
        for (int q = Lp[i] + 1; q < cur[i]; ++q) x[Li[q]] -= Lx[q] * lki;
        d -= lki * lki;
        int q = cur[i]++;
        Li[q] = k; Lx[q] = lki;
      }
      if (!(d > 0.0)) { ok = false; return false; }
      int q = cur[k]++;
      Li[q] = k; Lx[q] = std::sqrt(d);
    }
    ok = true;
    return true;
  }

  void solve(const double* b, double* xo) const {
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) y[iperm[i]] = b[i];
    for (int j = 0; j < n; ++j) {
      y[j] /= Lx[Lp[j]];
      for (int p = Lp[j] + 1; p < Lp[j + 1]; ++p) y[Li[p]] -= Lx[p] * y[j];
    }
    for (int j = n - 1; j >= 0; --j) {
      double s = y[j];
      for (int p = Lp[j] + 1; p < Lp[j + 1]; ++p) s -= Lx[p] * y[Li[p]];
      y[j] = s / Lx[Lp[j]];
    }
    for (int i = 0; i < n; ++i) xo[i] = y[iperm[i]];
  }
};

// ------------------------------------------------------------ simulation
struct SimBase {
  virtual ~SimBase() {}
  virtual int step(float dt, orc_step_result* res) = 0;
  virtual int step_ipc(float dt, const orc_contact* c, orc_step_result* res) = 0;
  virtual void set_ground(int has, float h) = 0;
  virtual void get_state(float*, float*, float*, float*, float*, float*) = 0;
  virtual void set_state(const float*, const float*, const float*, const float*, const float*, const float*) = 0;
  virtual void get_state64(double*, double*, double*) = 0;
  virtual void assemble_rhs(float dt, float*, float*, float*) = 0;
  virtual void detect(const orc_contact* c, float d_hat, const float*, const float*, const float*,
                      float*, float*, float*, float*, float*, float*, uint8_t*, float*, uint32_t*) = 0;
  virtual void resolve(const orc_contact* c, float* out) = 0;
  uint32_t n = 0, nt = 0;
  std::vector<uint32_t> tris;
  std::vector<HingeIdx> hidx;
  std::vector<int> Ap, Aj;       // summed matrix (CSR)
  std::vector<double> Ax;
  SparseChol chol;
  bool initialized = false;
  std::vector<float> mass_f;      // lumped (matrix) masses as f32
  std::vector<float> hinge_rest, hinge_w, hinge_st;
  std::vector<uint32_t> hinge_v;
};

template <class R> V3<R> v3(const float* a) { return V3<R>(R(a[0]), R(a[1]), R(a[2])); }

template <class R> struct Sim : SimBase {
  orc_params prm;
  orc_config cfg;
  std::vector<RestTri<R>> elems;
  std::vector<BendElem<R>> bend;
  std::vector<R> mass;   // solver lumped masses (pinned = 1e8)
  std::vector<uint8_t> pinned;
  // SimulationState (crates/vistio-solver/src/state.rs:23-64)
  std::vector<V3<R>> pos, vel, prev, pred, lam;
  std::vector<R> inv_mass;
  bool has_ground = false;
  R ground_h = 0;
  // contact state: exclusion sets + broad phase
  std::vector<std::vector<uint32_t>> excl;  // sorted
  RefBvh bvh;
  int frames_since_rebuild = 0;
  bool bvh_built = false;
  std::vector<std::pair<uint32_t, uint32_t>> last_pairs;

  bool init(const float* px, const float* py, const float* pz, const uint8_t* pin,
            const orc_params* p, const orc_config* c) {
    prm = *p;
    cfg = *c;
    pinned.assign(pin, pin + n);
    std::vector<V3<R>> rest(n);
    for (uint32_t i = 0; i < n; ++i) rest[i] = V3<R>(R(px[i]), R(py[i]), R(pz[i]));
    // ElementData::from_mesh (element.rs:54-91)
    elems.resize(nt);
    for (uint32_t t = 0; t < nt; ++t) {
      RestTri<R>& e = elems[t];
      for (int k = 0; k < 3; ++k) e.idx[k] = tris[3 * t + k];
      V3<R> p0 = rest[e.idx[0]], p1 = rest[e.idx[1]], p2 = rest[e.idx[2]];
      V3<R> e1 = p1 - p0, e2 = p2 - p0;
      e.area = R(0.5) * e1.cross(e2).length();
      compute_dm_inv(e1, e2, e.dm_inv);
      e.weight = R(prm.stiffness) * e.area;
    }
    // compute_lumped_masses (pd_solver.rs:1219-1242)
    mass.assign(n, R(0));
    R dens = R(prm.density_gsm) / R(1000);
    for (auto& e : elems) {
      R tri_mass = e.area * dens, third = tri_mass / R(3);
      for (int k = 0; k < 3; ++k) mass[e.idx[k]] += third;
    }
    for (uint32_t i = 0; i < n; ++i) {
      if (pinned[i]) mass[i] = R(1e8f);
      else if (mass[i] < R(1e-8f)) mass[i] = R(1e-8f);
    }
    // Bending data
    hidx = build_hinges(nt, tris.data());
    bend.clear();
    if (prm.bending == ORC_BEND_DIHEDRAL) {  // BendingData::from_topology (bending.rs:98)
      for (auto& h : hidx) {
        BendElem<R> b;
        b.v[0] = h.v0; b.v[1] = h.v1; b.v[2] = h.wa; b.v[3] = h.wb;
        b.rest_angle = clamp_rest_angle(dihedral_angle(rest[h.v0], rest[h.v1], rest[h.wa], rest[h.wb]));
        b.weight = R(prm.bend_stiffness) * (rest[h.v1] - rest[h.v0]).length();
        b.stencil[0] = R(-1); b.stencil[1] = R(-1); b.stencil[2] = R(1); b.stencil[3] = R(1);
        bend.push_back(b);
      }
    } else if (prm.bending == ORC_BEND_DS || prm.bending == ORC_BEND_DS_ANISO) {
      // DiscreteShellsBendingData::from_topology (discrete_shells.rs:106-199)
      for (auto& h : hidx) {
        V3<R> p0 = rest[h.v0], p1 = rest[h.v1], pa = rest[h.wa], pb = rest[h.wb];
        BendElem<R> b;
        b.v[0] = h.v0; b.v[1] = h.v1; b.v[2] = h.wa; b.v[3] = h.wb;
        b.rest_angle = clamp_rest_angle(dihedral_angle(p0, p1, pa, pb));
        R area_a = R(0.5) * (p1 - p0).cross(pa - p0).length();
        R area_b = R(0.5) * (p1 - p0).cross(pb - p0).length();
        V3<R> edge = p1 - p0;
        R len = edge.length();
        if (len < R(1e-10f)) continue;
        R inv_e2 = R(1) / (len * len);
        R c_wa = len / (R(2) * rmax(area_a, R(1e-8f)));
        R c_wb = len / (R(2) * rmax(area_b, R(1e-8f)));
        R dot0_a = (p1 - pa).dot(edge) * inv_e2, dot0_b = (p1 - pb).dot(edge) * inv_e2;
        R c_0 = -dot0_a * c_wa - dot0_b * c_wb;
        R dot1_a = (pa - p0).dot(edge) * inv_e2, dot1_b = (pb - p0).dot(edge) * inv_e2;
        R c_1 = -dot1_a * c_wa - dot1_b * c_wb;
        R raw[4] = {c_0, c_1, c_wa, c_wb};
        R norm = std::sqrt(raw[0] * raw[0] + raw[1] * raw[1] + raw[2] * raw[2] + raw[3] * raw[3]);
        if (norm > R(1e-10f)) for (int k = 0; k < 4; ++k) b.stencil[k] = raw[k] / norm;
        else { b.stencil[0] = b.stencil[1] = R(-0.5); b.stencil[2] = b.stencil[3] = R(0.5); }
        b.weight = R(prm.bend_stiffness) * len;
        bend.push_back(b);
      }
      if (prm.bending == ORC_BEND_DS_ANISO) {  // discrete_shells.rs:219-269
        R k_warp = R(prm.bend_warp), k_weft = R(prm.bend_weft), avg_raw = (k_warp + k_weft) / R(2);
        if (avg_raw > R(1e-8f)) {
          for (auto& b : bend) {
            V3<R> edge = rest[b.v[1]] - rest[b.v[0]];
            R len = edge.length();
            if (len < R(1e-10f)) continue;
            V3<R> ed = edge / len;
            V3<R> hz(ed.x, R(0), ed.z);
            R hl = hz.length();
            if (hl < R(1e-10f)) continue;
            V3<R> hd = hz / hl;
            R cs = std::fabs(hd.x), cos2 = cs * cs, sin2 = R(1) - cos2;
            R k_edge = k_weft * cos2 + k_warp * sin2;
            b.weight *= k_edge / avg_raw;
          }
        }
      }
    }
    // assemble_system_matrix (assembly.rs:44-135): triplets in the
    // reference's order, then duplicates summed in f64 (faer triplets).
    R h = R(prm.matrix_dt);
    R inv_dt2 = R(1) / (h * h);
    std::vector<std::map<int, double>> rows(n);
    for (uint32_t i = 0; i < n; ++i) rows[i][i] += double(mass[i] * inv_dt2);
    for (auto& e : elems) {
      R a = e.dm_inv[0], b = e.dm_inv[1], c = e.dm_inv[2], d = e.dm_inv[3];
      R g[3][2] = {{-(a + b), -(c + d)}, {a, c}, {b, d}};
      for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) {
          R dot = g[x][0] * g[y][0] + g[x][1] * g[y][1];
          if (std::fabs(dot) > R(1e-12f)) rows[e.idx[x]][e.idx[y]] += double(e.weight * dot);
        }
    }
    for (auto& b : bend)
      for (int x = 0; x < 4; ++x)
        for (int y = 0; y < 4; ++y) {
          R val = b.weight * b.stencil[x] * b.stencil[y];
          if (std::fabs(val) > R(1e-12f)) rows[b.v[x]][b.v[y]] += double(val);
        }
    Ap.assign(n + 1, 0); Aj.clear(); Ax.clear();
    for (uint32_t i = 0; i < n; ++i) {
      for (auto& kv : rows[i]) { Aj.push_back(kv.first); Ax.push_back(kv.second); }
      Ap[i + 1] = int(Aj.size());
    }
    std::vector<double> xyz(3 * n);
    for (uint32_t i = 0; i < n; ++i) { xyz[3 * i] = px[i]; xyz[3 * i + 1] = py[i]; xyz[3 * i + 2] = pz[i]; }
    if (!chol.factor(int(n), Ap, Aj, Ax, xyz)) return false;
    // SimulationState::from_mesh_with_masses (state.rs:85-140)
    pos = rest; prev = rest;
    vel.assign(n, V3<R>()); pred.assign(n, V3<R>()); lam.assign(n, V3<R>());
    inv_mass.assign(n, R(0));
    for (uint32_t i = 0; i < n; ++i)
      inv_mass[i] = pinned[i] ? R(0) : (mass[i] > R(1e-12f) ? R(1) / mass[i] : R(0));
    mass_f.resize(n);
    for (uint32_t i = 0; i < n; ++i) mass_f[i] = float(mass[i]);
    hinge_rest.clear(); hinge_w.clear(); hinge_st.clear(); hinge_v.clear();
    for (auto& b : bend) {
      for (int k = 0; k < 4; ++k) hinge_v.push_back(b.v[k]);
      hinge_rest.push_back(float(b.rest_angle)); hinge_w.push_back(float(b.weight));
      for (int k = 0; k < 4; ++k) hinge_st.push_back(float(b.stencil[k]));
    }
    initialized = true;
    return true;
  }

  // ---- local step (element.rs:127-217 and the material models)
  void reconstruct(const M32<R>& tf, const RestTri<R>& e, V3<R> p0, V3<R> p1, V3<R> p2, V3<R> out[3]) const {
    V3<R> centroid = (p0 + p1 + p2) / R(3);
    R det = e.dm_inv[0] * e.dm_inv[3] - e.dm_inv[1] * e.dm_inv[2];
    if (!(std::fabs(det) > R(1e-12f))) { out[0] = p0; out[1] = p1; out[2] = p2; return; }
    R inv_det = R(1) / det;
    R dm00 = e.dm_inv[3] * inv_det, dm01 = -e.dm_inv[2] * inv_det;
    R dm10 = -e.dm_inv[1] * inv_det, dm11 = e.dm_inv[0] * inv_det;
    V3<R> re1 = tf.c0 * dm00 + tf.c1 * dm10;
    V3<R> re2 = tf.c0 * dm01 + tf.c1 * dm11;
    V3<R> rest_c = (re1 + re2) / R(3);
    out[0] = centroid - rest_c;
    out[1] = out[0] + re1;
    out[2] = out[0] + re2;
  }

  M32<R> model_target(const M32<R>& f) const {
    switch (prm.model) {
      case ORC_MODEL_ARAP: return polar_decomposition(f).rot;
      case ORC_MODEL_COROT: {  // corotational.rs:116-137
        Polar<R> pd = polar_decomposition(f);
        R cs[4];
        clamp_stretch(pd, cs);
        return pd.rot.mul2(cs);
      }
      case ORC_MODEL_ORTHO: {  // orthotropic.rs:51-79
        Polar<R> pd = polar_decomposition(f);
        R wk = R(prm.warp), fk = R(prm.weft);
        R max_k = rmax(rmax(wk, fk), R(1e-6f));
        R k_warp = wk / max_k, k_weft = fk / max_k;
        R s0t = pd.s0 + (R(1) - pd.s0) * k_warp;
        R s1t = pd.s1 + (R(1) - pd.s1) * k_weft;
        R t00 = pd.v0.x * pd.v0.x * s0t + pd.v1.x * pd.v1.x * s1t;
        R t01 = pd.v0.x * pd.v0.y * s0t + pd.v1.x * pd.v1.y * s1t;
        R t11 = pd.v0.y * pd.v0.y * s0t + pd.v1.y * pd.v1.y * s1t;
        R ts[4] = {t00, t01, t01, t11};
        return pd.rot.mul2(ts);
      }
      case ORC_MODEL_ANISO: {  // anisotropic.rs:78-143
        Polar<R> pd = polar_decomposition(f);
        R kw = rclamp(R(prm.warp), R(0), R(1)), kf = rclamp(R(prm.weft), R(0), R(1));
        R cos2 = pd.v0.x * pd.v0.x, sin2 = pd.v0.y * pd.v0.y;
        R k0 = kw * cos2 + kf * sin2, k1 = kw * sin2 + kf * cos2;
        R s0t = pd.s0 > R(1) ? R(1) + (pd.s0 - R(1)) * (R(1) - k0) : pd.s0;
        R s1t = pd.s1 > R(1) ? R(1) + (pd.s1 - R(1)) * (R(1) - k1) : pd.s1;
        R t00 = pd.v0.x * pd.v0.x * s0t + pd.v1.x * pd.v1.x * s1t;
        R t01 = pd.v0.x * pd.v0.y * s0t + pd.v1.x * pd.v1.y * s1t;
        R t11 = pd.v0.y * pd.v0.y * s0t + pd.v1.y * pd.v1.y * s1t;
        R ts[4] = {t00, t01, t01, t11};
        return pd.rot.mul2(ts);
      }
      default: return M32<R>::identity();  // isotropic.rs:42-57
    }
  }

  // assemble_rhs (assembly.rs:157-240) for all three axes, after the local step.
  void build_rhs(R dt, std::vector<V3<R>>& rhs) const {
    R inv_dt2 = R(1) / (dt * dt);
    rhs.assign(n, V3<R>());
    for (uint32_t i = 0; i < n; ++i) {
      R c = mass[i] * inv_dt2;
      rhs[i] = V3<R>(c * pred[i].x, c * pred[i].y, c * pred[i].z);
    }
    for (auto& e : elems) {
      V3<R> p0 = pos[e.idx[0]], p1 = pos[e.idx[1]], p2 = pos[e.idx[2]];
      M32<R> f = deformation_gradient(p0, p1, p2, e.dm_inv);
      V3<R> tgt[3];
      reconstruct(model_target(f), e, p0, p1, p2, tgt);
      R a = e.dm_inv[0], b = e.dm_inv[1], c = e.dm_inv[2], d = e.dm_inv[3];
      R g[3][2] = {{-(a + b), -(c + d)}, {a, c}, {b, d}};
      for (int ax = 0; ax < 3; ++ax) {
        R t0 = ax == 0 ? tgt[0].x : ax == 1 ? tgt[0].y : tgt[0].z;
        R t1 = ax == 0 ? tgt[1].x : ax == 1 ? tgt[1].y : tgt[1].z;
        R t2 = ax == 0 ? tgt[2].x : ax == 1 ? tgt[2].y : tgt[2].z;
        R te1 = t1 - t0, te2 = t2 - t0;
        R f0 = te1 * a + te2 * b, f1 = te1 * c + te2 * d;
        for (int k = 0; k < 3; ++k) {
          R contrib = g[k][0] * f0 + g[k][1] * f1;
          R* r = ax == 0 ? &rhs[e.idx[k]].x : ax == 1 ? &rhs[e.idx[k]].y : &rhs[e.idx[k]].z;
          *r += e.weight * contrib;
        }
      }
    }
    for (auto& b : bend) {
      V3<R> tgt[4];
      bend_project(b, pos.data(), tgt);
      for (int ax = 0; ax < 3; ++ax) {
        R l = R(0);
        for (int k = 0; k < 4; ++k) {
          R tk = ax == 0 ? tgt[k].x : ax == 1 ? tgt[k].y : tgt[k].z;
          l += b.stencil[k] * tk;
        }
        for (int k = 0; k < 4; ++k) {
          R* r = ax == 0 ? &rhs[b.v[k]].x : ax == 1 ? &rhs[b.v[k]].y : &rhs[b.v[k]].z;
          *r += b.weight * b.stencil[k] * l;
        }
      }
    }
  }

  // FaerSolver::solve (faer_solver.rs:95-129): R -> f64, LL^T solve, f64 -> R.
  void global_solve(const std::vector<V3<R>>& rhs, std::vector<V3<R>>& sol) const {
    std::vector<double> b(n), x(n);
    sol.resize(n);
    for (int ax = 0; ax < 3; ++ax) {
      for (uint32_t i = 0; i < n; ++i) b[i] = double(ax == 0 ? rhs[i].x : ax == 1 ? rhs[i].y : rhs[i].z);
      chol.solve(b.data(), x.data());
      for (uint32_t i = 0; i < n; ++i) {
        R* s = ax == 0 ? &sol[i].x : ax == 1 ? &sol[i].y : &sol[i].z;
        *s = R(x[i]);
      }
    }
  }

  void predict(R dt) {  // state.rs:145-169
    R dt2 = dt * dt;
    for (uint32_t i = 0; i < n; ++i) {
      if (inv_mass[i] == R(0)) { pred[i] = pos[i]; continue; }
      pred[i].x = pos[i].x + dt * vel[i].x + dt2 * R(cfg.gravity[0]);
      pred[i].y = pos[i].y + dt * vel[i].y + dt2 * R(cfg.gravity[1]);
      pred[i].z = pos[i].z + dt * vel[i].z + dt2 * R(cfg.gravity[2]);
      if (has_ground && pred[i].y < ground_h) pred[i].y = ground_h;
    }
  }
  void enforce_ground() {  // state.rs:180-189
    if (!has_ground) return;
    for (uint32_t i = 0; i < n; ++i)
      if (inv_mass[i] > R(0) && pos[i].y < ground_h) pos[i].y = ground_h;
  }
  void enforce_ground_velocities() {  // state.rs:195-213
    if (!has_ground) return;
    for (uint32_t i = 0; i < n; ++i)
      if (inv_mass[i] > R(0) && pos[i].y <= ground_h) {
        if (vel[i].y < R(0)) vel[i].y = R(0);
        prev[i].y = ground_h;
        vel[i].x *= R(0.5); vel[i].z *= R(0.5);
      }
  }
  void update_velocities(R dt) {  // state.rs:216-223
    R inv_dt = R(1) / dt;
    for (uint32_t i = 0; i < n; ++i) vel[i] = (pos[i] - prev[i]) * inv_dt;
  }
  void damp_velocities(R damping) {  // state.rs:233-240
    R f = R(1) - damping;
    for (uint32_t i = 0; i < n; ++i) vel[i] = vel[i] * f;
  }
  void rayleigh(R dt) {  // pd_solver.rs:456-466
    if (!(cfg.rayleigh_mass_damping > 0.f)) return;
    R factor = R(1) / (R(1) + R(cfg.rayleigh_mass_damping) * dt);
    for (uint32_t i = 0; i < n; ++i) if (inv_mass[i] > R(0)) vel[i] = vel[i] * factor;
  }
  double residual(const std::vector<V3<R>>& sol) const {  // pd_solver.rs:403-421
    double diff_sq = 0, norm_sq = 0;
    for (uint32_t i = 0; i < n; ++i) {
      double dx = double(sol[i].x - pos[i].x), dy = double(sol[i].y - pos[i].y), dz = double(sol[i].z - pos[i].z);
      diff_sq += dx * dx + dy * dy + dz * dz;
      double ox = double(pos[i].x), oy = double(pos[i].y), oz = double(pos[i].z);
      norm_sq += ox * ox + oy * oy + oz * oz;
    }
    return norm_sq > 1e-12 ? std::sqrt(diff_sq / norm_sq) : std::sqrt(diff_sq);
  }

  // SolverStrategy::step for ProjectiveDynamicsSolver (pd_solver.rs:259-476)
  int step(float dtf, orc_step_result* res) override {
    if (!initialized) { if (res) res->status = 3; return 3; }
    R dt = R(dtf);
    prev = pos;
    predict(dt);
    pos = pred;
    std::vector<V3<R>> rhs, sol;
    uint32_t iterations = 0;
    double final_residual = std::numeric_limits<double>::max();
    for (uint32_t it = 0; it < cfg.max_iterations; ++it) {
      build_rhs(dt, rhs);
      global_solve(rhs, sol);
      final_residual = residual(sol);
      pos = sol;
      for (uint32_t i = 0; i < n; ++i) if (inv_mass[i] == R(0)) pos[i] = prev[i];
      enforce_ground();
      iterations = it + 1;
      if (final_residual < cfg.tolerance) break;
    }
    update_velocities(dt);
    enforce_ground_velocities();
    damp_velocities(R(cfg.damping));
    rayleigh(dt);
    if (res) {
      std::memset(res, 0, sizeof(*res));
      res->iterations = iterations;
      res->final_residual = final_residual;
      res->converged = final_residual < cfg.tolerance;
      res->last_alpha = 1.f;
    }
    return 0;
  }

  // ---------------------------------------------------------- contact
  void build_exclusion() {  // exclusion.rs:27-58 with depth 1 (runner.rs:367)
    std::vector<std::set<uint32_t>> ring(n);
    for (uint32_t t = 0; t < nt; ++t) {
      uint32_t v[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
      for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) ring[v[a]].insert(v[b]);
    }
    excl.assign(n, {});
    for (uint32_t i = 0; i < n; ++i) { ring[i].insert(i); excl[i].assign(ring[i].begin(), ring[i].end()); }
  }
  bool should_exclude(uint32_t i, uint32_t j) const {
    return std::binary_search(excl[i].begin(), excl[i].end(), j);
  }

  struct Contact { int type; uint32_t idx[4]; };

  // BvhBroadPhase::update + query_triangle_pairs (bvh.rs:305-392), or the
  // complete candidate set.
  void broad_update(const std::vector<V3<R>>& P, float thickness, bool faithful) {
    std::vector<float> px(n), py(n), pz(n);
    for (uint32_t i = 0; i < n; ++i) { px[i] = float(P[i].x); py[i] = float(P[i].y); pz[i] = float(P[i].z); }
    std::vector<Aabb> leaves(nt);
    for (uint32_t t = 0; t < nt; ++t) leaves[t] = tri_aabb(px.data(), py.data(), pz.data(), &tris[3 * t], thickness);
    if (faithful) {
      frames_since_rebuild += 1;
      if (!bvh_built || frames_since_rebuild >= 10) { bvh.build(leaves); bvh_built = true; frames_since_rebuild = 0; }
      else bvh.refit(leaves);
      last_pairs = bvh.query();
    } else {
      last_pairs = complete_pairs(leaves);
    }
  }

  // CollisionPipeline::detect_ipc_contacts (collision_pipeline.rs:207-352)
  struct Forces {
    std::vector<V3<R>> grad, normal;
    std::vector<uint8_t> in_contact;
    R max_violation = 0;
    uint32_t active = 0;
  };
  Forces detect_forces(const orc_contact& c, R d_hat, const std::vector<V3<R>>& P) {
    Forces F;
    F.grad.assign(n, V3<R>()); F.normal.assign(n, V3<R>()); F.in_contact.assign(n, 0);
    R kappa = R(c.kappa);
    if (c.self_collision) {
      // SelfCollisionSystem::detect_ipc_contacts (self_collision.rs:199-276)
      broad_update(P, c.thickness, c.bvh_faithful != 0);
      std::vector<Contact> contacts;
      auto vt = [&](uint32_t p, uint32_t a, uint32_t b, uint32_t cc) {  // ipc_response.rs:83-114
        int dt;
        R d = point_triangle_distance_squared(P[p], P[a], P[b], P[cc], &dt);
        if (d < d_hat && d > R(0)) contacts.push_back({0, {p, a, b, cc}});
      };
      auto ee = [&](uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1) {  // ipc_response.rs:120-148
        int dt;
        R d = edge_edge_distance_squared(P[a0], P[a1], P[b0], P[b1], &dt);
        if (d < d_hat && d > R(0)) contacts.push_back({1, {a0, a1, b0, b1}});
      };
      for (auto& pr : last_pairs) {
        const uint32_t* A = &tris[3 * pr.first];
        const uint32_t* B = &tris[3 * pr.second];
        for (int k = 0; k < 3; ++k) {
          uint32_t va = A[k];
          if (va == B[0] || va == B[1] || va == B[2]) continue;
          if (should_exclude(va, B[0]) || should_exclude(va, B[1]) || should_exclude(va, B[2])) continue;
          vt(va, B[0], B[1], B[2]);
        }
        for (int k = 0; k < 3; ++k) {
          uint32_t vb = B[k];
          if (vb == A[0] || vb == A[1] || vb == A[2]) continue;
          if (should_exclude(vb, A[0]) || should_exclude(vb, A[1]) || should_exclude(vb, A[2])) continue;
          vt(vb, A[0], A[1], A[2]);
        }
        uint32_t ae[3][2] = {{A[0], A[1]}, {A[1], A[2]}, {A[2], A[0]}};
        uint32_t be[3][2] = {{B[0], B[1]}, {B[1], B[2]}, {B[2], B[0]}};
        for (auto& ea : ae)
          for (auto& eb : be) {
            if (ea[0] == eb[0] || ea[0] == eb[1] || ea[1] == eb[0] || ea[1] == eb[1]) continue;
            if (should_exclude(ea[0], eb[0]) && should_exclude(ea[0], eb[1]) &&
                should_exclude(ea[1], eb[0]) && should_exclude(ea[1], eb[1])) continue;
            ee(ea[0], ea[1], eb[0], eb[1]);
          }
      }
      // compute_barrier_gradient (ipc_response.rs:170-219)
      std::vector<V3<R>> g(n);
      R thick = R(c.thickness);
      R maxv = 0;
      for (auto& ct : contacts) {
        int dt;
        V3<R> dg[4];
        R dsq;
        if (ct.type == 0) {
          dsq = point_triangle_distance_squared(P[ct.idx[0]], P[ct.idx[1]], P[ct.idx[2]], P[ct.idx[3]], &dt);
          point_triangle_distance_gradient(P[ct.idx[0]], P[ct.idx[1]], P[ct.idx[2]], P[ct.idx[3]], dg);
        } else {
          dsq = edge_edge_distance_squared(P[ct.idx[0]], P[ct.idx[1]], P[ct.idx[2]], P[ct.idx[3]], &dt);
          edge_edge_distance_gradient(P[ct.idx[0]], P[ct.idx[1]], P[ct.idx[2]], P[ct.idx[3]], dg);
        }
        R bg = thick > R(0) ? scaled_barrier_gradient_with_thickness(dsq, d_hat, kappa, thick)
                            : scaled_barrier_gradient(dsq, d_hat, kappa);
        for (int k = 0; k < 4; ++k) g[ct.idx[k]] = g[ct.idx[k]] + dg[k] * bg;
        if (dsq <= R(1e-12f)) maxv = rmax(maxv, R(1e-3f));
      }
      for (uint32_t i = 0; i < n; ++i) {
        F.grad[i] = F.grad[i] + g[i];
        R g_sq = g[i].x * g[i].x + g[i].y * g[i].y + g[i].z * g[i].z;
        if (g_sq > R(1e-12f)) {
          R gl = std::sqrt(g_sq);
          F.normal[i] = F.normal[i] + V3<R>(g[i].x / gl, g[i].y / gl, g[i].z / gl);
          F.in_contact[i] = 1;
        }
      }
      F.max_violation = rmax(F.max_violation, maxv);
      F.active += uint32_t(contacts.size());
    }
    if (c.has_ground) {  // ground_plane.rs:68-109 and collision_pipeline.rs:237-258
      R hgt = R(c.ground_height);
      for (uint32_t i = 0; i < n; ++i) {
        R ds = P[i].y - hgt;
        if (ds <= R(0)) {
          F.max_violation = rmax(F.max_violation, -ds);
          R dc = rmax(-ds, R(1e-6f));
          R bg = scaled_barrier_gradient(dc * dc, d_hat, kappa);
          F.active++;
          F.grad[i].y += bg * R(2) * dc;
        } else if (ds * ds < d_hat) {
          F.active++;
          R bg = scaled_barrier_gradient(ds * ds, d_hat, kappa);
          F.grad[i].y += bg * R(2) * ds;
        }
      }
      for (uint32_t i = 0; i < n; ++i) {
        R ds = P[i].y - hgt;
        if (ds * ds < d_hat || ds <= R(0)) { F.normal[i].y += R(1); F.in_contact[i] = 1; }
      }
    }
    if (c.has_sphere) {  // sphere.rs:102-175 and collision_pipeline.rs:261-277
      V3<R> ctr(R(c.sphere_center[0]), R(c.sphere_center[1]), R(c.sphere_center[2]));
      R rad = R(c.sphere_radius);
      for (uint32_t i = 0; i < n; ++i) {
        R dx = P[i].x - ctr.x, dy = P[i].y - ctr.y, dz = P[i].z - ctr.z;
        R r = std::sqrt(dx * dx + dy * dy + dz * dz);
        R ds = r - rad;
        if (ds <= R(0)) {
          F.max_violation = rmax(F.max_violation, -ds);
          R dc = rmax(-ds, R(1e-6f));
          F.active++;
          R bg = scaled_barrier_gradient(dc * dc, d_hat, kappa);
          if (r > R(1e-6f)) {
            R factor = bg * R(2) * dc;
            F.grad[i].x += factor * (dx / r); F.grad[i].y += factor * (dy / r); F.grad[i].z += factor * (dz / r);
          } else {
            F.grad[i].y += bg * R(2) * dc;
          }
        } else if (ds * ds < d_hat) {
          F.active++;
          R bg = scaled_barrier_gradient(ds * ds, d_hat, kappa);
          R factor = bg * R(2) * ds;
          F.grad[i].x += factor * (dx / r); F.grad[i].y += factor * (dy / r); F.grad[i].z += factor * (dz / r);
        }
      }
      for (uint32_t i = 0; i < n; ++i) {
        R dx = P[i].x - ctr.x, dy = P[i].y - ctr.y, dz = P[i].z - ctr.z;
        R r = std::sqrt(dx * dx + dy * dy + dz * dz);
        R ds = r - rad;
        if (ds * ds < d_hat || ds <= R(0)) {
          if (r > R(1e-6f)) { F.normal[i].x += dx / r; F.normal[i].y += dy / r; F.normal[i].z += dz / r; }
          F.in_contact[i] = 1;
        }
      }
    }
    if (c.has_cylinder) {  // cylinder.rs:121-198 (gradient only: collision_pipeline.rs:305-310)
      const R cx = R(c.cylinder_center_x), cz = R(c.cylinder_center_z), top = R(c.cylinder_top_y);
      const R rad = R(c.cylinder_radius);
      for (uint32_t i = 0; i < n; ++i) {
        R dx = P[i].x - cx, dy = P[i].y - top, dz = P[i].z - cz;
        R r = std::sqrt(dx * dx + dz * dz);
        R d_side = r - rad, d_top = dy;
        R gx = 0, gy = 0, gz = 0, dist_sq;
        if (d_top <= R(0) && d_side <= R(0)) {
          F.max_violation = rmax(F.max_violation, -rmax(d_top, d_side));
          if (d_top > d_side) gy = R(1);
          else if (r > R(1e-6f)) { gx = dx / r; gz = dz / r; }
          dist_sq = R(1e-12f);
        } else if (d_top > R(0) && d_side <= R(0)) {
          gy = R(1);
          dist_sq = d_top * d_top;
        } else if (d_top <= R(0) && d_side > R(0)) {
          if (r > R(1e-6f)) { gx = dx / r; gz = dz / r; }
          dist_sq = d_side * d_side;
        } else {
          if (r > R(1e-6f)) {
            R d = std::sqrt(d_side * d_side + d_top * d_top);
            gx = (d_side / d) * (dx / r); gy = d_top / d; gz = (d_side / d) * (dz / r);
          }
          dist_sq = d_side * d_side + d_top * d_top;
        }
        if (dist_sq < d_hat && dist_sq > R(0)) {
          F.active++;
          R factor = scaled_barrier_gradient(dist_sq, d_hat, kappa) * R(2) * std::sqrt(dist_sq);
          F.grad[i].x += factor * gx; F.grad[i].y += factor * gy; F.grad[i].z += factor * gz;
        }
      }
    }
    if (c.has_box) {  // box_collider.rs:107-200 (gradient only: collision_pipeline.rs:312-317)
      R ctr[3], ext[3];
      for (int k = 0; k < 3; ++k) {
        ctr[k] = (R(c.box_min[k]) + R(c.box_max[k])) * R(0.5);
        ext[k] = (R(c.box_max[k]) - R(c.box_min[k])) * R(0.5);
      }
      for (uint32_t i = 0; i < n; ++i) {
        R d[3] = {P[i].x - ctr[0], P[i].y - ctr[1], P[i].z - ctr[2]};
        R q[3], g[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k) q[k] = std::fabs(d[k]) - ext[k];
        R max_q = rmax(rmax(q[0], q[1]), q[2]);
        R dist_sq;
        if (max_q <= R(0)) {
          F.max_violation = rmax(F.max_violation, -max_q);
          int k = max_q == q[0] ? 0 : max_q == q[1] ? 1 : 2;
          g[k] = std::copysign(R(1), d[k]);
          dist_sq = R(1e-12f);
        } else {
          dist_sq = R(0);
          for (int k = 0; k < 3; ++k)
            if (q[k] > R(0)) { dist_sq += q[k] * q[k]; g[k] = q[k] * std::copysign(R(1), d[k]); }
          R dl = std::sqrt(dist_sq);
          if (dl > R(1e-6f)) for (int k = 0; k < 3; ++k) g[k] /= dl;
        }
        if (dist_sq < d_hat && dist_sq > R(0)) {
          F.active++;
          R factor = scaled_barrier_gradient(dist_sq, d_hat, kappa) * R(2) * std::sqrt(dist_sq);
          F.grad[i].x += factor * g[0]; F.grad[i].y += factor * g[1]; F.grad[i].z += factor * g[2];
        }
      }
    }
    for (uint32_t i = 0; i < n; ++i) {  // collision_pipeline.rs:324-337
      if (!F.in_contact[i]) continue;
      V3<R>& nn = F.normal[i];
      R ls = nn.x * nn.x + nn.y * nn.y + nn.z * nn.z;
      if (ls > R(1e-12f)) { R il = R(1) / std::sqrt(ls); nn = nn * il; }
    }
    return F;
  }

  // CollisionPipeline::compute_ccd_step (collision_pipeline.rs:355-400)
  R ccd_step(const orc_contact& c, const std::vector<V3<R>>& P0, const std::vector<V3<R>>& P1) const {
    R min_toi = R(1);
    if (c.self_collision) {  // ccd.rs:238-292
      R mt = R(1);
      for (auto& pr : last_pairs) {
        const uint32_t* A = &tris[3 * pr.first];
        const uint32_t* B = &tris[3 * pr.second];
        for (int side = 0; side < 2; ++side) {
          const uint32_t* X = side == 0 ? A : B;
          const uint32_t* Y = side == 0 ? B : A;
          for (int k = 0; k < 3; ++k) {
            uint32_t vi = X[k];
            if (vi == Y[0] || vi == Y[1] || vi == Y[2]) continue;
            R toi;
            if (vertex_triangle_ccd(P0[vi], P1[vi], P0[Y[0]], P1[Y[0]], P0[Y[1]], P1[Y[1]], P0[Y[2]], P1[Y[2]], &toi))
              mt = rmin(mt, toi);
          }
        }
      }
      min_toi = rmin(min_toi, rmax(mt, R(1e-6f)));
    }
    if (c.has_ground) {  // ground_plane.rs:112-134
      R hgt = R(c.ground_height), mt = R(1);
      for (uint32_t i = 0; i < n; ++i) {
        R y0 = P0[i].y, y1 = P1[i].y;
        if (y0 > hgt && y1 < hgt) {
          R t = (hgt - y0) / (y1 - y0);
          if (t >= R(0) && t <= R(1)) mt = rmin(mt, t * R(0.9f));
        }
      }
      min_toi = rmin(min_toi, rmax(mt, R(1e-6f)));
    }
    if (c.has_sphere) {  // sphere.rs:178-224
      V3<R> ctr(R(c.sphere_center[0]), R(c.sphere_center[1]), R(c.sphere_center[2]));
      R rad = R(c.sphere_radius), r2 = rad * rad, mt = R(1);
      for (uint32_t i = 0; i < n; ++i) {
        R px0 = P0[i].x - ctr.x, py0 = P0[i].y - ctr.y, pz0 = P0[i].z - ctr.z;
        R px1 = P1[i].x - ctr.x, py1 = P1[i].y - ctr.y, pz1 = P1[i].z - ctr.z;
        if (px0 * px0 + py0 * py0 + pz0 * pz0 < r2) continue;
        R vx = px1 - px0, vy = py1 - py0, vz = pz1 - pz0;
        R a = vx * vx + vy * vy + vz * vz;
        R b = R(2) * (px0 * vx + py0 * vy + pz0 * vz);
        R cc = px0 * px0 + py0 * py0 + pz0 * pz0 - r2;
        if (a > R(1e-8f)) {
          R disc = b * b - R(4) * a * cc;
          if (disc >= R(0)) {
            R t = (-b - std::sqrt(disc)) / (R(2) * a);
            if (t >= R(0) && t <= R(1)) mt = rmin(mt, t * R(0.9f));
          }
        }
      }
      min_toi = rmin(min_toi, rmax(mt, R(1e-6f)));
    }
    if (c.has_cylinder) {  // cylinder.rs:201-262
      const R cx = R(c.cylinder_center_x), cz = R(c.cylinder_center_z), top = R(c.cylinder_top_y);
      const R rad = R(c.cylinder_radius), r2 = rad * rad;
      R mt = R(1);
      for (uint32_t i = 0; i < n; ++i) {
        R px0 = P0[i].x - cx, py0 = P0[i].y - top, pz0 = P0[i].z - cz;
        R vx = (P1[i].x - cx) - px0, vy = (P1[i].y - top) - py0, vz = (P1[i].z - cz) - pz0;
        R a = vx * vx + vz * vz, b = R(2) * (px0 * vx + pz0 * vz), cc = px0 * px0 + pz0 * pz0 - r2;
        if (a > R(1e-8f)) {
          R disc = b * b - R(4) * a * cc;
          if (disc >= R(0)) {
            R t = (-b - std::sqrt(disc)) / (R(2) * a);
            if (t >= R(0) && t <= R(1) && py0 + t * vy <= R(0)) mt = rmin(mt, t * R(0.9f));
          }
        }
        if (vy < R(-1e-8f) && py0 > R(0)) {
          R t = -py0 / vy;
          if (t >= R(0) && t <= R(1)) {
            R xh = px0 + t * vx, zh = pz0 + t * vz;
            if (xh * xh + zh * zh <= r2) mt = rmin(mt, t * R(0.9f));
          }
        }
      }
      min_toi = rmin(min_toi, rmax(mt, R(1e-6f)));
    }
    if (c.has_box) {  // box_collider.rs:203-251
      R mt = R(1);
      for (uint32_t i = 0; i < n; ++i) {
        R p0[3] = {P0[i].x, P0[i].y, P0[i].z};
        R v[3] = {P1[i].x - P0[i].x, P1[i].y - P0[i].y, P1[i].z - P0[i].z};
        R t_min = R(0), t_max = R(1);
        bool hit = true;
        for (int k = 0; k < 3 && hit; ++k) {
          R lo = R(c.box_min[k]), hi = R(c.box_max[k]);
          if (std::fabs(v[k]) < R(1e-8f)) {
            hit = p0[k] >= lo && p0[k] <= hi;
          } else {
            R t1 = (lo - p0[k]) / v[k], t2 = (hi - p0[k]) / v[k];
            if (t1 > t2) std::swap(t1, t2);
            t_min = rmax(t_min, t1);
            t_max = rmin(t_max, t2);
            hit = t_min <= t_max && t_max >= R(0);
          }
        }
        if (hit && t_min >= R(0) && t_min <= R(1)) mt = rmin(mt, t_min * R(0.9f));
      }
      min_toi = rmin(min_toi, rmax(mt, R(1e-6f)));
    }
    return rmax(min_toi, R(1e-6f));
  }

  // ProjectiveDynamicsSolver::step_with_ipc (pd_solver.rs:549-1157)
  int step_ipc(float dtf, const orc_contact* cp, orc_step_result* res) override {
    if (!initialized) { if (res) res->status = 3; return 3; }
    const orc_contact& c = *cp;
    if (c.self_collision && excl.empty()) build_exclusion();
    R dt = R(dtf);
    prev = pos;
    R d_hat_cfg = R(cfg.barrier_d_hat);
    R d_hat_eff = cfg.compliant_contact ? d_hat_cfg * R(cfg.compliant_d_hat_scale) : d_hat_cfg;
    {  // velocity clamp (:573-595)
      R max_step = R(0.5) * std::sqrt(d_hat_eff);
      R max_vel = max_step / dt;
      for (uint32_t i = 0; i < n; ++i) {
        if (inv_mass[i] == R(0)) continue;
        R v_sq = vel[i].x * vel[i].x + vel[i].y * vel[i].y + vel[i].z * vel[i].z;
        if (v_sq > max_vel * max_vel) {
          R scale = max_vel / std::sqrt(v_sq);
          vel[i] = vel[i] * scale;
        }
      }
    }
    predict(dt);
    pos = pred;
    std::vector<V3<R>> rhs, sol;
    R mu = R(cfg.al_mu_initial);
    uint32_t total_iterations = 0, al_iters = 0;
    double final_residual = std::numeric_limits<double>::max();
    bool al_converged = false;
    std::vector<uint8_t> ever(n, 0);
    std::vector<V3<R>> fin_n(n);
    Forces updated;
    updated.grad.assign(n, V3<R>()); updated.normal.assign(n, V3<R>()); updated.in_contact.assign(n, 0);
    R alpha = R(1);
    for (uint32_t al = 0; al < cfg.al_max_iterations; ++al) {
      al_iters = al + 1;
      Forces bf = detect_forces(c, d_hat_eff, pos);
      for (uint32_t i = 0; i < n; ++i)
        if (bf.in_contact[i]) { ever[i] = 1; fin_n[i] = bf.normal[i]; }
      for (uint32_t i = 0; i < n; ++i)
        if (!bf.in_contact[i]) lam[i] = V3<R>();
      for (uint32_t it = 0; it < cfg.max_iterations; ++it) {
        build_rhs(dt, rhs);
        for (uint32_t i = 0; i < n; ++i) {  // assemble_barrier_rhs (assembly.rs:272-282)
          rhs[i].x -= mu * bf.grad[i].x + lam[i].x;
          rhs[i].y -= mu * bf.grad[i].y + lam[i].y;
          rhs[i].z -= mu * bf.grad[i].z + lam[i].z;
        }
        global_solve(rhs, sol);
        double diff_sq = 0, norm_sq = 0;
        for (uint32_t i = 0; i < n; ++i) {
          double dx = double(sol[i].x - pos[i].x), dy = double(sol[i].y - pos[i].y), dz = double(sol[i].z - pos[i].z);
          diff_sq += dx * dx + dy * dy + dz * dz;
          double ox = double(pos[i].x), oy = double(pos[i].y), oz = double(pos[i].z);
          norm_sq += ox * ox + oy * oy + oz * oz;
        }
        final_residual = norm_sq > 1e-12 ? std::sqrt(diff_sq / norm_sq) : std::sqrt(diff_sq);
        R max_alpha = ccd_step(c, pos, sol);  // (:896-906)
        if (max_alpha < R(1)) max_alpha *= R(0.8f);
        max_alpha = rmin(max_alpha, R(1));
        alpha = max_alpha;  // backtracking heuristic (:909-932)
        for (int bt = 0; bt < 4; ++bt) {
          if (alpha < R(0.1f)) break;
          double gdd = 0;
          for (uint32_t i = 0; i < n; ++i)
            if (inv_mass[i] > R(0)) {
              R dx = sol[i].x - pos[i].x, dy = sol[i].y - pos[i].y, dz = sol[i].z - pos[i].z;
              gdd += double(bf.grad[i].x * dx + bf.grad[i].y * dy + bf.grad[i].z * dz);
            }
          if (gdd * double(mu) > double(1e-4f) * diff_sq * 100.0) alpha *= R(0.5);
          else break;
        }
        for (uint32_t i = 0; i < n; ++i)
          if (inv_mass[i] > R(0)) pos[i] = pos[i] + (sol[i] - pos[i]) * alpha;
        total_iterations++;
        if (final_residual < cfg.tolerance) break;
      }
      updated = detect_forces(c, d_hat_eff, pos);
      for (uint32_t i = 0; i < n; ++i)
        if (updated.in_contact[i]) { ever[i] = 1; fin_n[i] = updated.normal[i]; }
      if (updated.max_violation < R(cfg.al_tolerance)) { al_converged = true; break; }
      for (uint32_t i = 0; i < n; ++i)
        if (updated.in_contact[i]) lam[i] = lam[i] + updated.grad[i] * mu;
      mu *= R(cfg.al_mu_growth);
    }
    update_velocities(dt);
    // inelastic velocity filter (:1036-1111)
    R muf = R(cfg.friction_coefficient), cd = R(cfg.contact_damping);
    for (uint32_t i = 0; i < n; ++i) {
      if (inv_mass[i] == R(0) || !ever[i]) continue;
      V3<R> nn = fin_n[i];
      if (nn.x * nn.x + nn.y * nn.y + nn.z * nn.z < R(0.5)) continue;
      R vdn = vel[i].x * nn.x + vel[i].y * nn.y + vel[i].z * nn.z;
      vel[i].x -= vdn * nn.x; vel[i].y -= vdn * nn.y; vel[i].z -= vdn * nn.z;
      R vn = std::fabs(vdn);
      V3<R> vt = vel[i];
      R vt_mag = std::sqrt(vt.x * vt.x + vt.y * vt.y + vt.z * vt.z);
      if (vt_mag > R(1e-8f)) {
        R fi = muf * vn;
        if (fi >= vt_mag) vel[i] = V3<R>();
        else { R s = R(1) - fi / vt_mag; vel[i] = vt * s; }
      }
      if (cfg.adaptive_contact_damping) {
        R v_mag = std::sqrt(vel[i].x * vel[i].x + vel[i].y * vel[i].y + vel[i].z * vel[i].z);
        R t = rclamp(R(1) - v_mag / rmax(R(cfg.contact_velocity_threshold), R(1e-6f)), R(0), R(1));
        R ad = cd + t * (R(cfg.contact_damping_max) - cd);
        vel[i] = vel[i] * (R(1) - ad);
      } else {
        vel[i] = vel[i] * (R(1) - cd);
      }
    }
    if (updated.active > 0) damp_velocities(R(0.05f));
    enforce_ground_velocities();
    damp_velocities(R(cfg.damping));
    rayleigh(dt);
    if (res) {
      std::memset(res, 0, sizeof(*res));
      res->iterations = total_iterations;
      res->final_residual = final_residual;
      res->converged = al_converged || final_residual < cfg.tolerance;
      res->al_iterations = al_iters;
      res->active_contacts = updated.active;
      res->last_alpha = float(alpha);
    }
    return 0;
  }

  void set_ground(int has, float h) override { has_ground = has != 0; ground_h = R(h); }
  void get_state(float* px, float* py, float* pz, float* vx, float* vy, float* vz) override {
    for (uint32_t i = 0; i < n; ++i) {
      if (px) px[i] = float(pos[i].x);
      if (py) py[i] = float(pos[i].y);
      if (pz) pz[i] = float(pos[i].z);
      if (vx) vx[i] = float(vel[i].x);
      if (vy) vy[i] = float(vel[i].y);
      if (vz) vz[i] = float(vel[i].z);
    }
  }
  void set_state(const float* px, const float* py, const float* pz, const float* vx, const float* vy,
                 const float* vz) override {
    for (uint32_t i = 0; i < n; ++i) {
      if (px) pos[i].x = R(px[i]);
      if (py) pos[i].y = R(py[i]);
      if (pz) pos[i].z = R(pz[i]);
      if (vx) vel[i].x = R(vx[i]);
      if (vy) vel[i].y = R(vy[i]);
      if (vz) vel[i].z = R(vz[i]);
    }
  }
  void get_state64(double* px, double* py, double* pz) override {
    for (uint32_t i = 0; i < n; ++i) { px[i] = double(pos[i].x); py[i] = double(pos[i].y); pz[i] = double(pos[i].z); }
  }
  void assemble_rhs(float dtf, float* rx, float* ry, float* rz) override {
    std::vector<V3<R>> rhs;
    pred = pos;
    build_rhs(R(dtf), rhs);
    for (uint32_t i = 0; i < n; ++i) { rx[i] = float(rhs[i].x); ry[i] = float(rhs[i].y); rz[i] = float(rhs[i].z); }
  }
  // CollisionPipeline::step with thickness 0 (collision_pipeline.rs:117-199):
  // ground twice, sphere, cylinder, box; out[3c..3c+2] = resolved count,
  // max penetration and depth sum of collider c (ground, sphere, cylinder,
  // box), the first ground pass being the one reported.
  void resolve(const orc_contact* c, float* out) override {
    for (int k = 0; k < 12; ++k) out[k] = 0.f;
    auto note = [&](int col, R depth) {
      out[3 * col] += 1.f;
      out[3 * col + 1] = std::max(out[3 * col + 1], float(depth));
      out[3 * col + 2] += float(depth);
    };
    auto ground = [&](bool report) {  // ground_plane.rs:26-65
      const R h = R(c->ground_height);
      for (uint32_t i = 0; i < n; ++i) {
        if (inv_mass[i] == R(0)) continue;
        R depth = h - pos[i].y;
        if (depth > R(0)) {
          pos[i].y = h;
          prev[i].y = h;
          vel[i].x *= R(0.5);
          vel[i].z *= R(0.5);
          if (vel[i].y < R(0)) vel[i].y = R(0);
          if (report) note(0, depth);
        }
      }
    };
    if (c->has_ground) { ground(true); ground(false); }
    if (c->has_sphere) {  // sphere.rs:29-100
      const V3<R> ctr = v3<R>(c->sphere_center);
      const R rad = R(c->sphere_radius), r2 = rad * rad;
      for (uint32_t i = 0; i < n; ++i) {
        if (inv_mass[i] == R(0)) continue;
        V3<R> d = pos[i] - ctr;
        R dist2 = d.x * d.x + d.y * d.y + d.z * d.z;
        if (dist2 < r2 && dist2 > R(1e-12f)) {
          R dist = std::sqrt(dist2), depth = rad - dist;
          V3<R> nrm(d.x / dist, d.y / dist, d.z / dist);
          pos[i] = pos[i] + nrm * depth;
          R vn = vel[i].x * nrm.x + vel[i].y * nrm.y + vel[i].z * nrm.z;
          if (vn < R(0)) vel[i] = (vel[i] - nrm * vn) * R(0.5);
          note(1, depth);
        } else if (dist2 <= R(1e-12f)) {
          pos[i].y += rad;
          vel[i] = V3<R>();
          note(1, rad);
        }
      }
    }
    if (c->has_cylinder) {  // cylinder.rs:30-118
      const R cx = R(c->cylinder_center_x), cz = R(c->cylinder_center_z), top = R(c->cylinder_top_y);
      const R rad = R(c->cylinder_radius), r2 = rad * rad;
      for (uint32_t i = 0; i < n; ++i) {
        if (inv_mass[i] == R(0) || pos[i].y > top) continue;
        R dx = pos[i].x - cx, dz = pos[i].z - cz;
        R dist2 = dx * dx + dz * dz;
        if (!(dist2 < r2)) continue;
        R dist = std::sqrt(dist2), side = rad - dist, dtop = top - pos[i].y;
        bool up = dtop < side || prev[i].y >= top || dist < R(1e-12f);
        if (up) {
          pos[i].y = top;
          if (vel[i].y < R(0)) vel[i].y = R(0);
          vel[i].x *= R(0.1f);
          vel[i].z *= R(0.1f);
          note(2, dtop);
        } else {
          if (dist > R(1e-12f)) {
            R nx = dx / dist, nz = dz / dist;
            pos[i].x += nx * side;
            pos[i].z += nz * side;
            R vn = vel[i].x * nx + vel[i].z * nz;
            if (vn < R(0)) { vel[i].x -= vn * nx; vel[i].z -= vn * nz; }
            vel[i].y *= R(0.7f);
          }
          note(2, side);
        }
      }
    }
    if (c->has_box) {  // box_collider.rs:26-99
      const V3<R> lo = v3<R>(c->box_min), hi = v3<R>(c->box_max);
      const R fr = R(0.7f);
      for (uint32_t i = 0; i < n; ++i) {
        if (inv_mass[i] == R(0)) continue;
        V3<R>& p = pos[i];
        V3<R>& v = vel[i];
        if (!(p.x >= lo.x && p.x <= hi.x && p.y >= lo.y && p.y <= hi.y && p.z >= lo.z && p.z <= hi.z)) continue;
        const R face[6] = {p.x - lo.x, hi.x - p.x, hi.y - p.y, p.y - lo.y, hi.z - p.z, p.z - lo.z};
        R m = std::min(std::min(std::min(std::min(std::min(face[0], face[1]), face[3]), face[2]), face[5]), face[4]);
        if (prev[i].y >= hi.y) m = face[2];
        // the first face (in the order -x, +x, +y, -y, +z, -z) at the minimum
        int k = 0;
        while (k < 5 && face[k] != m) ++k;
        R* axis[3] = {&v.x, &v.y, &v.z};
        R* coord[3] = {&p.x, &p.y, &p.z};
        const int ax[6] = {0, 0, 1, 1, 2, 2};
        const R to[6] = {lo.x, hi.x, hi.y, lo.y, hi.z, lo.z};
        const int outward[6] = {-1, 1, 1, -1, 1, -1};
        *coord[ax[k]] = to[k];
        R& vn = *axis[ax[k]];
        if (R(outward[k]) * vn < R(0)) vn = R(0);
        for (int a = 0; a < 3; ++a)
          if (a != ax[k]) *axis[a] *= fr;
        note(3, m);
      }
    }
  }

  void detect(const orc_contact* c, float d_hat, const float* px, const float* py, const float* pz,
              float* gx, float* gy, float* gz, float* nx, float* ny, float* nz, uint8_t* inc,
              float* maxv, uint32_t* active) override {
    if (c->self_collision && excl.empty()) build_exclusion();
    std::vector<V3<R>> P(n);
    for (uint32_t i = 0; i < n; ++i) P[i] = V3<R>(R(px[i]), R(py[i]), R(pz[i]));
    Forces F = detect_forces(*c, R(d_hat), P);
    for (uint32_t i = 0; i < n; ++i) {
      gx[i] = float(F.grad[i].x); gy[i] = float(F.grad[i].y); gz[i] = float(F.grad[i].z);
      nx[i] = float(F.normal[i].x); ny[i] = float(F.normal[i].y); nz[i] = float(F.normal[i].z);
      inc[i] = F.in_contact[i];
    }
    *maxv = float(F.max_violation);
    *active = F.active;
  }
};


}  // namespace

// ===================================================================== C API
extern "C" {

void* orc_create(int precision, uint32_t nv, const float* px, const float* py, const float* pz,
                 uint32_t nt, const uint32_t* tris, const uint8_t* pinned,
                 const orc_params* params, const orc_config* cfg, int32_t* status) {
  SimBase* s;
  bool ok;
  if (precision == 1) {
    auto* d = new Sim<double>();
    d->n = nv; d->nt = nt; d->tris.assign(tris, tris + 3 * size_t(nt));
    ok = d->init(px, py, pz, pinned, params, cfg);
    s = d;
  } else {
    auto* f = new Sim<float>();
    f->n = nv; f->nt = nt; f->tris.assign(tris, tris + 3 * size_t(nt));
    ok = f->init(px, py, pz, pinned, params, cfg);
    s = f;
  }
  if (status) *status = ok ? 0 : 3;
  return s;
}
void orc_destroy(void* sim) { delete static_cast<SimBase*>(sim); }
int orc_step(void* sim, float dt, orc_step_result* res) { return static_cast<SimBase*>(sim)->step(dt, res); }
int orc_step_ipc(void* sim, float dt, const orc_contact* c, orc_step_result* res) {
  return static_cast<SimBase*>(sim)->step_ipc(dt, c, res);
}
void orc_resolve(void* sim, const orc_contact* c, float* out) { static_cast<SimBase*>(sim)->resolve(c, out); }

int orc_sparse_solve(uint32_t rows, uint32_t cols, const uint32_t* row_ptr, const uint32_t* col_idx,
                     const float* vals, const float* rhs, float* sol) {
  if (rows != cols) return 1;  // "Matrix must be square"
  if (rows == 0) return 2;     // "Cannot factorize empty matrix"
  const int n = int(rows);
  // upper-triangle entries summed per (row, col) in f64, then mirrored
  std::vector<std::map<int, double>> up(n);
  for (int i = 0; i < n; ++i)
    for (uint32_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
      const int j = int(col_idx[p]);
      if (j >= i) up[i][j] += double(vals[p]);
    }
  std::vector<std::map<int, double>> full(n);
  for (int i = 0; i < n; ++i)
    for (auto& e : up[i]) {
      full[i][e.first] = e.second;
      full[e.first][i] = e.second;
    }
  std::vector<int> Ap(n + 1, 0), Aj;
  std::vector<double> Ax;
  for (int i = 0; i < n; ++i) {
    for (auto& e : full[i]) { Aj.push_back(e.first); Ax.push_back(e.second); }
    Ap[i + 1] = int(Aj.size());
  }
  std::vector<double> xyz(3 * size_t(n), 0.0);
  for (int i = 0; i < n; ++i) xyz[3 * size_t(i)] = double(i);
  SparseChol chol;
  if (!chol.factor(n, Ap, Aj, Ax, xyz)) return 3;
  std::vector<double> b(n), x(n);
  for (int i = 0; i < n; ++i) b[i] = double(rhs[i]);
  chol.solve(b.data(), x.data());
  for (int i = 0; i < n; ++i) sol[i] = float(x[i]);
  return 0;
}
void orc_set_ground(void* sim, int has, float h) { static_cast<SimBase*>(sim)->set_ground(has, h); }
void orc_get_state(void* sim, float* px, float* py, float* pz, float* vx, float* vy, float* vz) {
  static_cast<SimBase*>(sim)->get_state(px, py, pz, vx, vy, vz);
}
void orc_set_state(void* sim, const float* px, const float* py, const float* pz, const float* vx,
                   const float* vy, const float* vz) {
  static_cast<SimBase*>(sim)->set_state(px, py, pz, vx, vy, vz);
}
void orc_get_state64(void* sim, double* px, double* py, double* pz) {
  static_cast<SimBase*>(sim)->get_state64(px, py, pz);
}
uint32_t orc_hinge_count(void* sim) { return uint32_t(static_cast<SimBase*>(sim)->hinge_w.size()); }
void orc_get_hinges(void* sim, uint32_t* v4, float* rest, float* w, float* st) {
  SimBase* s = static_cast<SimBase*>(sim);
  size_t nh = s->hinge_w.size();
  for (size_t h = 0; h < 4 * nh; ++h) v4[h] = s->hinge_v[h];
  for (size_t h = 0; h < nh; ++h) { rest[h] = s->hinge_rest[h]; w[h] = s->hinge_w[h]; }
  for (size_t h = 0; h < 4 * nh; ++h) st[h] = s->hinge_st[h];
}
void orc_get_masses(void* sim, float* mass) {
  SimBase* s = static_cast<SimBase*>(sim);
  std::memcpy(mass, s->mass_f.data(), s->n * sizeof(float));
}
uint32_t orc_matrix_nnz(void* sim) { return uint32_t(static_cast<SimBase*>(sim)->Aj.size()); }
void orc_get_matrix(void* sim, uint32_t* rp, uint32_t* ci, double* v) {
  SimBase* s = static_cast<SimBase*>(sim);
  for (size_t i = 0; i < s->Ap.size(); ++i) rp[i] = uint32_t(s->Ap[i]);
  for (size_t i = 0; i < s->Aj.size(); ++i) { ci[i] = uint32_t(s->Aj[i]); v[i] = s->Ax[i]; }
}
uint64_t orc_factor_nnz(void* sim) { return static_cast<SimBase*>(sim)->chol.Lp.empty() ? 0 : uint64_t(static_cast<SimBase*>(sim)->chol.Lp.back()); }
void orc_assemble_rhs(void* sim, float dt, float* rx, float* ry, float* rz) {
  static_cast<SimBase*>(sim)->assemble_rhs(dt, rx, ry, rz);
}
void orc_solve(void* sim, const float* b, float* x) {
  SimBase* s = static_cast<SimBase*>(sim);
  std::vector<double> bd(s->n), xd(s->n);
  for (uint32_t i = 0; i < s->n; ++i) bd[i] = b[i];
  s->chol.solve(bd.data(), xd.data());
  for (uint32_t i = 0; i < s->n; ++i) x[i] = float(xd[i]);
}

// generators.rs:28-100 quad_grid
void orc_quad_grid(uint32_t cols, uint32_t rows, float width, float height, float* px, float* py,
                   float* pz, uint32_t* tris) {
  uint32_t vx = cols + 1, vy = rows + 1;
  float hw = width / 2.0f, hh = height / 2.0f;
  for (uint32_t j = 0; j < vy; ++j)
    for (uint32_t i = 0; i < vx; ++i) {
      float u = float(i) / float(cols), v = float(j) / float(rows);
      size_t k = size_t(j) * vx + i;
      px[k] = -hw + u * width;
      py[k] = hh - v * height;
      pz[k] = 0.0f;
    }
  size_t t = 0;
  for (uint32_t j = 0; j < rows; ++j)
    for (uint32_t i = 0; i < cols; ++i) {
      uint32_t tl = j * vx + i, tr = tl + 1, bl = tl + vx, br = bl + 1;
      if ((i + j) % 2 == 0) {
        uint32_t a[6] = {tl, bl, tr, tr, bl, br};
        for (int k = 0; k < 6; ++k) tris[t++] = a[k];
      } else {
        uint32_t a[6] = {tl, bl, br, tl, br, tr};
        for (int k = 0; k < 6; ++k) tris[t++] = a[k];
      }
    }
}

float orc_pt_dist2(const float p[3], const float a[3], const float b[3], const float c[3], int* dtype) {
  return point_triangle_distance_squared(v3<float>(p), v3<float>(a), v3<float>(b), v3<float>(c), dtype);
}
float orc_ee_dist2(const float a0[3], const float a1[3], const float b0[3], const float b1[3], int* dtype) {
  return edge_edge_distance_squared(v3<float>(a0), v3<float>(a1), v3<float>(b0), v3<float>(b1), dtype);
}
void orc_pt_grad(const float p[3], const float a[3], const float b[3], const float c[3], float out[12]) {
  V3<float> g[4];
  point_triangle_distance_gradient(v3<float>(p), v3<float>(a), v3<float>(b), v3<float>(c), g);
  for (int k = 0; k < 4; ++k) { out[3 * k] = g[k].x; out[3 * k + 1] = g[k].y; out[3 * k + 2] = g[k].z; }
}
void orc_ee_grad(const float a0[3], const float a1[3], const float b0[3], const float b1[3], float out[12]) {
  V3<float> g[4];
  edge_edge_distance_gradient(v3<float>(a0), v3<float>(a1), v3<float>(b0), v3<float>(b1), g);
  for (int k = 0; k < 4; ++k) { out[3 * k] = g[k].x; out[3 * k + 1] = g[k].y; out[3 * k + 2] = g[k].z; }
}
int orc_vt_ccd(const float* p0, const float* p1, const float* a0, const float* a1, const float* b0,
               const float* b1, const float* c0, const float* c1, float* toi) {
  return vertex_triangle_ccd(v3<float>(p0), v3<float>(p1), v3<float>(a0), v3<float>(a1), v3<float>(b0),
                             v3<float>(b1), v3<float>(c0), v3<float>(c1), toi) ? 1 : 0;
}
int orc_ee_ccd(const float* a0, const float* a1, const float* b0, const float* b1, const float* c0,
               const float* c1, const float* d0, const float* d1, float* toi) {
  return edge_edge_ccd(v3<float>(a0), v3<float>(a1), v3<float>(b0), v3<float>(b1), v3<float>(c0),
                       v3<float>(c1), v3<float>(d0), v3<float>(d1), toi) ? 1 : 0;
}
int orc_cubic_roots(float a, float b, float c, float d, float roots[3]) { return solve_cubic_roots(a, b, c, d, roots); }
float orc_barrier_energy(float d, float dh) { return barrier_energy(d, dh); }
float orc_barrier_gradient(float d, float dh) { return barrier_gradient(d, dh); }
float orc_barrier_hessian(float d, float dh) { return barrier_hessian(d, dh); }
float orc_scaled_barrier_gradient(float d, float dh, float k) { return scaled_barrier_gradient(d, dh, k); }
float orc_barrier_energy_thick(float d, float dh, float t) { return barrier_energy_with_thickness(d, dh, t); }
float orc_barrier_gradient_thick(float d, float dh, float t) { return barrier_gradient_with_thickness(d, dh, t); }
float orc_estimate_kappa(float c, float m, float g, float dh) { return estimate_initial_kappa(c, m, g, dh); }
void orc_polar(const float f[6], float rot[6], float stretch[4], float sv[2]) {
  M32<float> F(V3<float>(f[0], f[1], f[2]), V3<float>(f[3], f[4], f[5]));
  Polar<float> p = polar_decomposition(F);
  rot[0] = p.rot.c0.x; rot[1] = p.rot.c0.y; rot[2] = p.rot.c0.z;
  rot[3] = p.rot.c1.x; rot[4] = p.rot.c1.y; rot[5] = p.rot.c1.z;
  for (int k = 0; k < 4; ++k) stretch[k] = p.stretch[k];
  sv[0] = p.s0; sv[1] = p.s1;
}

uint64_t orc_tri_pairs(uint32_t nv, const float* px, const float* py, const float* pz, uint32_t nt,
                       const uint32_t* tris, float margin, int mode, uint32_t* out, uint64_t cap) {
  (void)nv;
  std::vector<Aabb> leaves(nt);
  for (uint32_t t = 0; t < nt; ++t) leaves[t] = tri_aabb(px, py, pz, tris + 3 * size_t(t), margin);
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  if (mode == 1) {
    RefBvh b;
    b.build(leaves);
    pairs = b.query();
    std::sort(pairs.begin(), pairs.end());
  } else {
    pairs = complete_pairs(leaves);
  }
  for (uint64_t i = 0; i < pairs.size() && i < cap; ++i) { out[2 * i] = pairs[i].first; out[2 * i + 1] = pairs[i].second; }
  return pairs.size();
}

float orc_ccd_hits(uint32_t nv, const float* p0x, const float* p0y, const float* p0z, const float* p1x,
                   const float* p1y, const float* p1z, uint32_t nt, const uint32_t* tris, uint64_t npairs,
                   const uint32_t* pairs, uint32_t* hits, uint64_t cap, uint64_t* nhits) {
  (void)nv; (void)nt;
  std::vector<std::pair<uint32_t, uint32_t>> hv;
  double mt = 1.0;
  auto P0 = [&](uint32_t i) { return V3<double>(p0x[i], p0y[i], p0z[i]); };
  auto P1 = [&](uint32_t i) { return V3<double>(p1x[i], p1y[i], p1z[i]); };
  for (uint64_t k = 0; k < npairs; ++k) {
    uint32_t ta = pairs[2 * k], tb = pairs[2 * k + 1];
    const uint32_t* A = tris + 3 * size_t(ta);
    const uint32_t* B = tris + 3 * size_t(tb);
    for (int side = 0; side < 2; ++side) {
      const uint32_t* X = side == 0 ? A : B;
      const uint32_t* Y = side == 0 ? B : A;
      uint32_t ty = side == 0 ? tb : ta;
      for (int q = 0; q < 3; ++q) {
        uint32_t vi = X[q];
        if (vi == Y[0] || vi == Y[1] || vi == Y[2]) continue;
        double toi;
        if (vertex_triangle_ccd(P0(vi), P1(vi), P0(Y[0]), P1(Y[0]), P0(Y[1]), P1(Y[1]), P0(Y[2]), P1(Y[2]), &toi)) {
          hv.push_back({vi, ty});
          mt = std::min(mt, toi);
        }
      }
    }
  }
  std::sort(hv.begin(), hv.end());
  hv.erase(std::unique(hv.begin(), hv.end()), hv.end());
  for (uint64_t i = 0; i < hv.size() && i < cap; ++i) { hits[2 * i] = hv[i].first; hits[2 * i + 1] = hv[i].second; }
  *nhits = hv.size();
  return float(std::max(mt, 1e-6));
}

void orc_detect(void* sim, const orc_contact* c, float d_hat, const float* px, const float* py,
                const float* pz, float* gx, float* gy, float* gz, float* nx, float* ny, float* nz,
                uint8_t* inc, float* maxv, uint32_t* active) {
  static_cast<SimBase*>(sim)->detect(c, d_hat, px, py, pz, gx, gy, gz, nx, ny, nz, inc, maxv, active);
}

}  // extern "C"
