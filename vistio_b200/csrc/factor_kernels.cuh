// Numeric Cholesky factorization of P A P^T on the GPU in FP64 (multifrontal,
// supernodal), writing the FP32 layout the sweeps read. The host does the
// symbolic analysis (ordering, supernodes, row structures); the numbers are
// computed here once per garment, material and dt, the same arithmetic the
// reference leaves to faer's FP64 LL^T (crates/vistio-solver/src/faer_solver.rs:67-93).
//
// Every supernode k (columns f .. f+s, rows R below, n_f = s + m) has a front:
// an n_f x n_f FP64 matrix, column-major, of which the lower triangle is used.
// Supernodes are processed level by level up the supernodal elimination tree
// (a level = height above the leaves), one block per supernode:
//   assemble  the front = the supernode's columns of A (rows mapped to front
//             positions) + the update matrices of its children (extend-add
//             through the host-computed map of each child's rows into this
//             front), children one after another;
//   factor    right-looking partial Cholesky of the first s columns: the first
//             s columns become [L_kk; L_Rk], the trailing m x m block the
//             update matrix this supernode hands to its parent;
//   invert    inv(L_kk) by forward substitution, one column per thread, kept
//             in the (unused) strict upper triangle;
//   write     D = inv(L_kk) and P = L_Rk in FP32 into the supernode's packed
//             region, leading dimension sn_ld(s) (the row indices after P
//             are written by the host).
#pragma once
#include "pd_kernels.cuh"

namespace vistio {

struct FrontDev {
  const SnDev* sn;
  const uint32_t* rows;       // below-diagonal rows of each supernode (instance-local)
  const uint32_t* a_ptr;      // A in solve order (global rows), f64
  const uint32_t* a_col;
  const double* a_val;
  const uint64_t* front_off;  // doubles: where each supernode's front starts
  const uint32_t* kid_ptr;    // children of each supernode (global ids)
  const uint32_t* kids;
  const uint32_t* relmap;     // per supernode row (indexed like rows): its position in the parent's front
  double* fronts;
  float* vals;
  uint32_t* status;           // bit 5: a pivot <= 0 (not positive definite); bit 6: an entry of A
                              // outside the symbolic structure (an inconsistent set-up)
};

constexpr uint32_t kFrontThreads = 256;

// Position of instance-local row `row` (>= f) in the front of the supernode
// with columns f .. f+s and sorted rows R[0..m); s + m when it is not there.
__device__ __forceinline__ uint32_t front_pos(const uint32_t* R, uint32_t m, uint32_t f, uint32_t s, uint32_t row) {
  if (row < f + s) return row - f;
  uint32_t lo = 0, hi = m;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (R[mid] < row) lo = mid + 1;
    else hi = mid;
  }
  return (lo < m && R[lo] == row) ? s + lo : s + m;
}

__global__ void __launch_bounds__(kFrontThreads) k_front(FrontDev D, const uint32_t* __restrict__ items) {
  __shared__ double s_piv;
  __shared__ uint32_t s_bad;
  const uint32_t k = items[blockIdx.x];
  const SnDev S = D.sn[k];
  const uint32_t s = S.ncols, m = S.nrows, nf = s + m, f = S.first, vb = S.vbase, tid = threadIdx.x;
  double* Fk = D.fronts + D.front_off[k];
  const uint32_t* R = D.rows + S.rows_off;
  if (tid == 0) s_bad = 0;
  for (uint32_t i = tid; i < nf * nf; i += kFrontThreads) Fk[i] = 0.0;
  __syncthreads();
  // the supernode's columns of A: entries on or below the diagonal (row q >= column)
  for (uint32_t c = tid; c < s; c += kFrontThreads) {
    const uint32_t p = vb + f + c;
    for (uint32_t q = D.a_ptr[p], qe = D.a_ptr[p + 1]; q < qe; ++q) {
      const uint32_t row = D.a_col[q] - vb;
      if (row < f + c) continue;
      const uint32_t at = front_pos(R, m, f, s, row);
      if (at < nf) Fk[uint64_t(c) * nf + at] += D.a_val[q];
      else atomicOr(D.status, 64u);
    }
  }
  // extend-add of each child's update matrix (its trailing m_c x m_c block)
  for (uint32_t ci = D.kid_ptr[k], ce = D.kid_ptr[k + 1]; ci < ce; ++ci) {
    __syncthreads();
    const uint32_t ch = D.kids[ci];
    const SnDev C = D.sn[ch];
    const uint32_t sc = C.ncols, mc = C.nrows, nfc = sc + mc;
    const double* Fc = D.fronts + D.front_off[ch];
    const uint32_t* map = D.relmap + C.rows_off;
    for (uint32_t t = tid; t < mc * mc; t += kFrontThreads) {
      const uint32_t j = t / mc, i = t % mc;
      if (i < j) continue;
      Fk[uint64_t(map[j]) * nf + map[i]] += Fc[uint64_t(sc + j) * nfc + sc + i];
    }
  }
  // right-looking partial Cholesky of the first s columns
  for (uint32_t j = 0; j < s; ++j) {
    __syncthreads();
    if (tid == 0) {
      double d = Fk[uint64_t(j) * nf + j];
      if (!(d > 0.0) || !isfinite(d)) {
        s_bad = 1;
        d = 1.0;  // keep going with finite numbers; the host reports the failure
      }
      s_piv = sqrt(d);
      Fk[uint64_t(j) * nf + j] = s_piv;
    }
    __syncthreads();
    const double inv = 1.0 / s_piv;
    double* colj = Fk + uint64_t(j) * nf;
    for (uint32_t i = j + 1 + tid; i < nf; i += kFrontThreads) colj[i] *= inv;
    __syncthreads();
    const uint32_t w = nf - j - 1;
    for (uint32_t t = tid; t < w * w; t += kFrontThreads) {
      const uint32_t l = j + 1 + t / w, i = j + 1 + t % w;
      if (i < l) continue;
      Fk[uint64_t(l) * nf + i] -= colj[i] * colj[l];
    }
  }
  __syncthreads();
  // inv(L_kk): column c of the inverse, x_i for i > c at Fk[i * nf + c]
  for (uint32_t c = tid; c < s; c += kFrontThreads) {
    const double xc = 1.0 / Fk[uint64_t(c) * nf + c];
    for (uint32_t i = c + 1; i < s; ++i) {
      double acc = Fk[uint64_t(c) * nf + i] * xc;
      for (uint32_t q = c + 1; q < i; ++q) acc += Fk[uint64_t(q) * nf + i] * Fk[uint64_t(q) * nf + c];
      Fk[uint64_t(i) * nf + c] = -acc / Fk[uint64_t(i) * nf + i];
    }
  }
  __syncthreads();
  const uint32_t ld = sn_ld(s);
  float* Dv = D.vals + S.d_off;  // Linv[i][c] at c * ld + i
  for (uint32_t t = tid; t < s * s; t += kFrontThreads) {
    const uint32_t c = t / s, i = t % s;
    double v = 0.0;
    if (i == c) v = 1.0 / Fk[uint64_t(c) * nf + c];
    else if (i > c) v = Fk[uint64_t(i) * nf + c];
    Dv[c * ld + i] = float(v);
  }
  float* Pv = D.vals + S.p_off;  // P[r][c] at r * ld + c
  for (uint32_t t = tid; t < m * s; t += kFrontThreads) {
    const uint32_t r = t / s, c = t % s;
    Pv[r * ld + c] = float(Fk[uint64_t(c) * nf + s + r]);
  }
  if (tid == 0 && s_bad) atomicOr(D.status, 32u);
}

}  // namespace vistio
