// CPU check of the host-side set-up (vistio_b200/csrc/setup.cpp): builds a
// quad-grid instance, then replays the GPU sweep schedule of k_solve (level
// by level: pull-forward through the panel row lists, inverted diagonal
// blocks, panel-transpose backward) on the CPU and reports the relative
// residual of A x = b. Prints one JSON object.
//
// usage: factor_check cols rows width [bending] [pinned_row]
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
         "\"resid32_refined\": %.3e, \"err32\": %.3e, \"err32_refined\": %.3e}\n",
         nv, I.nh, I.A_col.size(), (unsigned long long)F.nnz_L, (unsigned long long)F.nnz_stored, F.sn.size(),
         F.nlevels, F.sub_first.size(), maxs, F.fwd_sn.size(), resid(yd), resid(yf), resid(yr), dist64(yf), dist64(yr));
  return 0;
}
