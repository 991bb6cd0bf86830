// CPU check of the host-side set-up (vistio_b200/csrc/setup.cpp): builds a
// quad-grid instance, then replays the GPU sweep schedule of k_solve (level
// by level: pull-forward through the panel row lists, inverted diagonal
// blocks, panel-transpose backward) on the CPU and reports the relative
// residual of A x = b. Prints one JSON object.
//
// usage: factor_check cols rows width [bending] [pinned_row]
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../../vistio_b200/csrc/setup.h"

using namespace vistio;

template <class T>
static void fwd_sn(const Factor& F, const std::vector<T>& vals, std::vector<T>& Y, std::vector<T>& Tm,
                   std::vector<T>& U, uint32_t k) {
  const Supernode& S = F.sn[k];
  uint32_t s = S.ncols;
  for (uint32_t c = 0; c < s; ++c) {
    uint32_t r = S.first + c;
    T t = Y[r];
    for (uint32_t q = F.fwd_ptr[r]; q < F.fwd_ptr[r + 1]; ++q) t -= U[F.sn[F.fwd_sn[q]].rows_off + F.fwd_pos[q]];
    Tm[r] = t;
  }
  const T* D = vals.data() + S.diag_off;  // column-major inverse
  for (uint32_t c = 0; c < s; ++c) {
    T y = 0;
    for (uint32_t c2 = 0; c2 <= c; ++c2) y += D[uint64_t(c2) * s + c] * Tm[S.first + c2];
    Y[S.first + c] = y;
  }
  const T* Pn = vals.data() + S.panel_off;  // row-major m x s
  for (uint32_t j = 0; j < S.nrows; ++j) {
    T u = 0;
    for (uint32_t c = 0; c < s; ++c) u += Pn[uint64_t(j) * s + c] * Y[S.first + c];
    U[S.rows_off + j] = u;
  }
}

template <class T>
static void bwd_sn(const Factor& F, const std::vector<T>& vals, std::vector<T>& Y, std::vector<T>& Tm, uint32_t k) {
  const Supernode& S = F.sn[k];
  uint32_t s = S.ncols;
  const T* Pn = vals.data() + S.panel_off;
  const uint32_t* rr = F.rows.data() + S.rows_off;
  for (uint32_t c = 0; c < s; ++c) {
    T t = 0;
    for (uint32_t j = 0; j < S.nrows; ++j) t += Pn[uint64_t(j) * s + c] * Y[rr[j]];
    Tm[S.first + c] = Y[S.first + c] - t;
  }
  const T* D = vals.data() + S.diag_off;
  for (uint32_t c = 0; c < s; ++c) {
    T x = 0;
    for (uint32_t c2 = c; c2 < s; ++c2) x += D[uint64_t(c) * s + c2] * Tm[S.first + c2];
    Y[S.first + c] = x;
  }
}

// Replays the GPU schedule: forward = bottom subtrees (postorder), then the
// top levels ascending; backward = top levels descending, then the bottom
// subtrees in reverse postorder.
template <class T>
static void sweep(const Factor& F, const std::vector<T>& vals, std::vector<T>& Y) {
  std::vector<T> Tm(F.n), U(F.rows.size());
  for (size_t q = 0; q < F.sub_first.size(); ++q)
    for (uint32_t k = F.sub_first[q]; k <= F.sub_last[q]; ++k) fwd_sn(F, vals, Y, Tm, U, k);
  for (uint32_t l = 0; l < F.nlevels; ++l)
    for (uint32_t q = F.level_sn_ptr[l]; q < F.level_sn_ptr[l + 1]; ++q) fwd_sn(F, vals, Y, Tm, U, F.level_sn[q]);
  for (int l = int(F.nlevels) - 1; l >= 0; --l)
    for (uint32_t q = F.level_sn_ptr[l]; q < F.level_sn_ptr[l + 1]; ++q) bwd_sn(F, vals, Y, Tm, F.level_sn[q]);
  for (size_t q = 0; q < F.sub_first.size(); ++q)
    for (int k = int(F.sub_last[q]); k >= int(F.sub_first[q]); --k) bwd_sn(F, vals, Y, Tm, uint32_t(k));
}

// Replays the device factorization (k_front in factor_kernels.cuh) on the
// CPU: one dense front per supernode (columns, then rows), assembled from the
// permuted A and the children's update matrices through the map of each
// child row into its parent's front, partial Cholesky of the supernode's
// columns, inv(L_kk) by forward substitution. Returns the largest difference
// to the host factor's values, relative to the largest value.
static double multifrontal_replay(const InstanceSetup& I) {
  const Factor& F = I.factor;
  const uint32_t nsn = uint32_t(F.sn.size());
  std::vector<uint32_t> ap{0}, ac;
  std::vector<double> av;
  append_permuted_matrix(I, 0, ap, ac, av);
  std::vector<std::vector<double>> fronts(nsn);
  std::vector<double> out(F.vals.size(), 0.0);
  auto pos_in = [&](uint32_t k, uint32_t r) -> int64_t {  // position of row r in supernode k's front
    const Supernode& S = F.sn[k];
    if (r >= S.first && r < S.first + S.ncols) return r - S.first;
    const uint32_t* R = F.rows.data() + S.rows_off;
    const uint32_t* it = std::lower_bound(R, R + S.nrows, r);
    if (it == R + S.nrows || *it != r) return -1;
    return S.ncols + (it - R);
  };
  for (uint32_t k = 0; k < nsn; ++k) {  // children precede parents
    const Supernode& S = F.sn[k];
    const uint32_t s = S.ncols, m = S.nrows, nf = s + m, f = S.first;
    std::vector<double>& Fk = fronts[k];
    Fk.assign(size_t(nf) * nf, 0.0);
    for (uint32_t c = 0; c < s; ++c)
      for (uint32_t q = ap[f + c]; q < ap[f + c + 1]; ++q) {
        if (ac[q] < f + c) continue;
        int64_t at = pos_in(k, ac[q]);
        if (at < 0) return 1e30;
        Fk[size_t(c) * nf + at] += av[q];
      }
    for (uint32_t ch = 0; ch < k; ++ch) {
      if (F.sn[ch].parent != k) continue;
      const Supernode& C = F.sn[ch];
      const uint32_t sc = C.ncols, mc = C.nrows, nfc = sc + mc;
      std::vector<int64_t> map(mc);
      for (uint32_t j = 0; j < mc; ++j) {
        map[j] = pos_in(k, F.rows[C.rows_off + j]);
        if (map[j] < 0) return 1e30;
      }
      for (uint32_t j = 0; j < mc; ++j)
        for (uint32_t i = j; i < mc; ++i)
          Fk[size_t(map[j]) * nf + map[i]] += fronts[ch][size_t(sc + j) * nfc + sc + i];
      fronts[ch].clear();
    }
    for (uint32_t j = 0; j < s; ++j) {
      double d = Fk[size_t(j) * nf + j];
      if (!(d > 0.0)) return 1e30;
      d = std::sqrt(d);
      Fk[size_t(j) * nf + j] = d;
      for (uint32_t i = j + 1; i < nf; ++i) Fk[size_t(j) * nf + i] /= d;
      for (uint32_t l = j + 1; l < nf; ++l)
        for (uint32_t i = l; i < nf; ++i) Fk[size_t(l) * nf + i] -= Fk[size_t(j) * nf + i] * Fk[size_t(j) * nf + l];
    }
    double* Dv = out.data() + S.diag_off;
    for (uint32_t c = 0; c < s; ++c) {
      Dv[size_t(c) * s + c] = 1.0 / Fk[size_t(c) * nf + c];
      for (uint32_t i = c + 1; i < s; ++i) {
        double acc = 0.0;
        for (uint32_t q = c; q < i; ++q) acc += Fk[size_t(q) * nf + i] * Dv[size_t(c) * s + q];
        Dv[size_t(c) * s + i] = -acc / Fk[size_t(i) * nf + i];
      }
    }
    double* Pv = out.data() + S.panel_off;
    for (uint32_t r = 0; r < m; ++r)
      for (uint32_t c = 0; c < s; ++c) Pv[size_t(r) * s + c] = Fk[size_t(c) * nf + s + r];
  }
  double big = 0, diff = 0;
  for (size_t e = 0; e < out.size(); ++e) {
    big = std::max(big, std::fabs(F.vals[e]));
    diff = std::max(diff, std::fabs(out[e] - F.vals[e]));
  }
  return diff / big;
}

// The symbolic-only set-up (numeric factorization left to the device) has
// the same ordering, supernodes, rows, schedule and pull lists.
static bool same_structure(const Factor& a, const Factor& b) {
  if (a.perm != b.perm || a.rows != b.rows || a.nlevels != b.nlevels || a.level_sn != b.level_sn ||
      a.level_sn_ptr != b.level_sn_ptr || a.sub_first != b.sub_first || a.sub_last != b.sub_last ||
      a.fwd_ptr != b.fwd_ptr || a.fwd_sn != b.fwd_sn || a.fwd_pos != b.fwd_pos || a.sn.size() != b.sn.size() ||
      a.nnz_stored != b.nnz_stored || b.numeric || !b.vals.empty())
    return false;
  for (size_t k = 0; k < a.sn.size(); ++k) {
    const Supernode &x = a.sn[k], &y = b.sn[k];
    if (x.first != y.first || x.ncols != y.ncols || x.nrows != y.nrows || x.rows_off != y.rows_off ||
        x.panel_off != y.panel_off || x.diag_off != y.diag_off || x.parent != y.parent || x.level != y.level)
      return false;
  }
  return true;
}

int main(int argc, char** argv) {
  uint32_t cols = argc > 1 ? atoi(argv[1]) : 20, rows = argc > 2 ? atoi(argv[2]) : 20;
  float width = argc > 3 ? float(atof(argv[3])) : 1.f;
  int bending = argc > 4 ? atoi(argv[4]) : BEND_DIHEDRAL;
  int pin_row = argc > 5 ? atoi(argv[5]) : 1;
  uint32_t vx = cols + 1, vy = rows + 1, nv = vx * vy;
  std::vector<float> px(nv), py(nv), pz(nv);
  float height = width * float(rows) / float(cols);
  for (uint32_t j = 0; j < vy; ++j)
    for (uint32_t i = 0; i < vx; ++i) {
      uint32_t k = j * vx + i;
      px[k] = -width / 2 + float(i) / float(cols) * width;
      pz[k] = height / 2 - float(j) / float(rows) * height;
      py[k] = 1.0f;
    }
  std::vector<uint32_t> tris;
  for (uint32_t j = 0; j < rows; ++j)
    for (uint32_t i = 0; i < cols; ++i) {
      uint32_t tl = j * vx + i, tr = tl + 1, bl = tl + vx, br = bl + 1;
      if ((i + j) % 2 == 0) tris.insert(tris.end(), {tl, bl, tr, tr, bl, br});
      else tris.insert(tris.end(), {tl, bl, br, tl, br, tr});
    }
  std::vector<uint8_t> pinned(nv, 0);
  if (pin_row)
    for (uint32_t i = 0; i < vx; ++i) pinned[i] = 1;
  SetupParams p;
  p.bending = bending;
  p.stiffness = 1000.f;
  p.bend_stiffness = 1e-4f;
  p.density_gsm = 150.f;
  InstanceSetup I;
  int st = 0;
  std::string err = build_instance(nv, px.data(), py.data(), pz.data(), uint32_t(tris.size() / 3), tris.data(),
                                   pinned.data(), p, I, &st);
  if (!err.empty()) {
    printf("{\"error\": \"%s\", \"status\": %d}\n", err.c_str(), st);
    return 1;
  }
  const Factor& F = I.factor;
  InstanceSetup Isym;
  SetupParams psym = p;
  psym.numeric = false;
  err = build_instance(nv, px.data(), py.data(), pz.data(), uint32_t(tris.size() / 3), tris.data(), pinned.data(),
                       psym, Isym, &st);
  const int symbolic_same = err.empty() && same_structure(F, Isym.factor);
  const double mf_diff = multifrontal_replay(I);
  std::mt19937_64 rng(20261203);
  std::normal_distribution<double> nd;
  std::vector<double> b(nv), yd(nv);
  for (auto& v : b) v = nd(rng);
  for (uint32_t i = 0; i < nv; ++i) yd[F.iperm[i]] = b[i];
  std::vector<float> yf(yd.begin(), yd.end());
  std::vector<float> valsf(F.vals.begin(), F.vals.end());
  sweep<double>(F, F.vals, yd);
  sweep<float>(F, valsf, yf);
  // one FP64 refinement as the GPU does it: W = b - A y with the permuted f64
  // matrix, an FP32 sweep on W, y += W
  std::vector<uint32_t> ap{0}, ac;
  std::vector<double> av;
  append_permuted_matrix(I, 0, ap, ac, av);
  std::vector<float> yr(yf), w(nv);
  for (uint32_t r = 0; r < nv; ++r) {
    double acc = 0;
    for (uint32_t q = ap[r]; q < ap[r + 1]; ++q) acc += av[q] * double(yf[ac[q]]);
    w[r] = float(b[F.perm[r]] - acc);
  }
  sweep<float>(F, valsf, w);
  for (uint32_t r = 0; r < nv; ++r) yr[r] = yf[r] + w[r];
  auto resid = [&](auto& y) {
    double rn = 0, bn = 0;
    for (uint32_t i = 0; i < nv; ++i) {
      double s = b[i];
      for (uint32_t q = I.A_ptr[i]; q < I.A_ptr[i + 1]; ++q) s -= I.A_val[q] * double(y[F.iperm[I.A_col[q]]]);
      rn += s * s;
      bn += b[i] * b[i];
    }
    return std::sqrt(rn / bn);
  };
  auto dist64 = [&](auto& y) {  // relative distance to the FP64 solution
    double e = 0, n2 = 0;
    for (uint32_t r = 0; r < nv; ++r) { double q = double(y[r]) - yd[r]; e += q * q; n2 += yd[r] * yd[r]; }
    return std::sqrt(e / n2);
  };
  uint32_t maxs = 0;
  for (auto& S : F.sn) maxs = std::max(maxs, S.ncols);
  printf("{\"nv\": %u, \"nh\": %u, \"nnz_a\": %zu, \"nnz_l\": %llu, \"stored\": %llu, \"supernodes\": %zu, "
         "\"levels\": %u, \"subtrees\": %zu, \"max_snode\": %u, \"fwd_entries\": %zu, \"resid64\": %.3e, \"resid32\": %.3e, "
         "\"resid32_refined\": %.3e, \"err32\": %.3e, \"err32_refined\": %.3e, \"symbolic_same\": %d, "
         "\"multifrontal_diff\": %.3e}\n",
         nv, I.nh, I.A_col.size(), (unsigned long long)F.nnz_L, (unsigned long long)F.nnz_stored, F.sn.size(),
         F.nlevels, F.sub_first.size(), maxs, F.fwd_sn.size(), resid(yd), resid(yf), resid(yr), dist64(yf), dist64(yr),
         symbolic_same, mf_diff);
  return 0;
}
