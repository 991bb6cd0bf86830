// sm_100a self-contact path of the IPC step: triangle broad phase, the
// vertex-triangle / edge-edge barrier gradients and vertex-triangle CCD.
//
// Broad phase. The reference rebuilds a median-split BVH every tenth update
// and refits it otherwise (crates/vistio-contact/src/bvh.rs:122-373). Here
// each garment's triangles, in mesh index order, are the leaves of an
// implicit balanced binary tree: node (l, i) bounds leaves [i 2^l, (i+1) 2^l).
// Mesh order keeps every subtree an intrinsically compact patch of cloth, so
// the tree stays tight when the cloth folds, and a refit is all a detect
// needs. A node's leaf range is known from its position, so the traversal
// for leaf i skips every subtree whose leaves are all <= i and emits exactly
// the pairs (i < j) whose inflated AABBs overlap: the complete candidate set,
// independent of tree shape. Pairs are produced in a count / scan / write
// sequence so their order (and every sum over them) is deterministic.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "contact_kernels.cuh"
#include "../../include/vistio_cuda.h"

struct vistio_solver;
struct vistio_ctx;

namespace vistio {

struct SelfInst {
  uint32_t tbase, nt;      // global triangle range
  uint32_t box_base;       // first box of this garment's tree
  uint32_t nlevels;        // tree levels including the leaf level
  uint32_t lvl_off[28];    // box offset of each level relative to box_base
  uint32_t lvl_cnt[28];    // boxes on each level
};

// Device view of the self-contact buffers: plain pointers, passed to kernels by value.
struct SelfContactView {
  uint32_t ninst;
  uint64_t T;
  uint64_t pair_cap;
  SelfInst* inst;      // per garment
  uint32_t* tri_inst;  // triangle -> garment
  float4* box_min;     // all tree levels
  float4* box_max;
  uint32_t* cnt;       // per triangle pair counts, then exclusive offsets
  uint32_t* block_sums;
  uint2* pairs;        // global (ta, tb)
  uint32_t* npairs;    // [0] pair count, [1] overflow flag
  uint32_t* adj_ptr;   // 1-ring exclusion lists (sorted, include the vertex itself)
  uint32_t* adj;
  uint32_t scan_blocks;
  // LBVH leaf order: triangles sorted by (garment, Morton code of the
  // centroid). leaf_tri[tbase + i] is the global triangle of leaf i (the last
  // sort buffer); null keeps mesh order.
  uint32_t* leaf_tri;
  uint64_t* keys;        // sort keys, ping-pong pair with keys_alt
  uint64_t* keys_alt;
  uint32_t* order;       // sorted triangle ids, ping-pong pair with order_alt
  uint32_t* order_alt;
  uint32_t* sort_hist;   // 256 digit counts per sort block, then their offsets
  uint32_t* sort_sums;   // scan block sums of sort_hist (+1: the total)
  uint32_t sort_blocks, sort_scan_blocks, sort_passes;
  // The self CCD's vertex-triangle tests, each once. A candidate pair (A, B)
  // tests the vertices of A against B and those of B against A, and a vertex
  // v of A meets B again in every other pair (A', B) with v in A': about 2.6
  // times per test on a cloth mesh. The list keeps (v, B) only from the pair
  // whose A is the lowest-numbered triangle around v with a box overlapping
  // B's, which is the first pair the broad phase holds for that test. Built
  // by the detect that opens an AL pass; the pass's CCDs read it.
  uint32_t* leaf_of;     // global triangle -> its leaf in its garment's tree (null: no list)
  uint2* vt;             // (vertex, triangle), global ids
  uint32_t* nvt;         // [0] tests, [1] overflow: the CCD then runs over the pairs
  uint64_t vt_cap;
  int32_t vt_on;         // build and use the list (0: every test of every pair)
};

// Host-side owner of those buffers (never passed to a kernel). They are
// allocated and freed in the order of `stream`, which must outlive them.
struct SelfContactDev : SelfContactView {
  bool ready = false;
  cudaStream_t stream = nullptr;
  SelfContactDev() : SelfContactView{} {}
  SelfContactDev(const SelfContactDev&) = delete;
  SelfContactDev& operator=(const SelfContactDev&) = delete;
  SelfContactView view() const { return static_cast<const SelfContactView&>(*this); }
  void release() {
    for (void* q : {static_cast<void*>(inst), static_cast<void*>(tri_inst), static_cast<void*>(box_min),
                    static_cast<void*>(box_max), static_cast<void*>(cnt), static_cast<void*>(block_sums),
                    static_cast<void*>(pairs), static_cast<void*>(npairs), static_cast<void*>(adj_ptr),
                    static_cast<void*>(adj), static_cast<void*>(keys), static_cast<void*>(keys_alt),
                    static_cast<void*>(order), static_cast<void*>(order_alt), static_cast<void*>(sort_hist),
                    static_cast<void*>(sort_sums), static_cast<void*>(leaf_of), static_cast<void*>(vt),
                    static_cast<void*>(nvt)})
      if (q) cudaFreeAsync(q, stream);
    inst = nullptr; tri_inst = nullptr; box_min = box_max = nullptr; cnt = block_sums = nullptr;
    pairs = nullptr; npairs = nullptr; adj_ptr = adj = nullptr; ready = false;
    keys = keys_alt = nullptr; order = order_alt = leaf_tri = sort_hist = sort_sums = nullptr;
    leaf_of = nullptr; vt = nullptr; nvt = nullptr; vt_cap = 0;
  }
  ~SelfContactDev() { release(); }
};

constexpr int kScanBlock = 1024;
constexpr uint32_t kSortTile = 2048;  // keys per radix-sort block (256 threads x 8)

// ------------------------------------------------------------------ LBVH
// 30-bit Morton code: 10 bits per axis interleaved (x in the lowest bit).
__device__ __forceinline__ uint32_t morton_spread10(uint32_t v) {
  v &= 1023u;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Sort keys of one garment per block: its triangles' centroids, quantized to
// 10 bits per axis within the garment's centroid bounds, as a Morton code
// below the garment index (so each garment stays in its own range).
__global__ void __launch_bounds__(1024) k_self_keys(BatchDev B, SelfContactView S) {
  pdl_begin();
  const SelfInst& I = S.inst[blockIdx.x];
  __shared__ float red[6][32];
  float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
  auto centroid = [&](uint32_t i) {
    const uint4 id = B.tri_idx[I.tbase + i];
    const float4 a = B.pos[id.x], b = B.pos[id.y], c = B.pos[id.z];
    return make_float3((a.x + b.x + c.x) * (1.f / 3.f), (a.y + b.y + c.y) * (1.f / 3.f), (a.z + b.z + c.z) * (1.f / 3.f));
  };
  for (uint32_t i = threadIdx.x; i < I.nt; i += blockDim.x) {
    const float3 c = centroid(i);
    lo[0] = fminf(lo[0], c.x); lo[1] = fminf(lo[1], c.y); lo[2] = fminf(lo[2], c.z);
    hi[0] = fmaxf(hi[0], c.x); hi[1] = fmaxf(hi[1], c.y); hi[2] = fmaxf(hi[2], c.z);
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; ++k) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < 3; ++k) { red[k][w] = lo[k]; red[3 + k][w] = hi[k]; }
  __syncthreads();
  for (int k = 0; k < 3; ++k) {
    lo[k] = red[k][0];
    hi[k] = red[3 + k][0];
    for (uint32_t q = 1; q < (blockDim.x >> 5); ++q) { lo[k] = fminf(lo[k], red[k][q]); hi[k] = fmaxf(hi[k], red[3 + k][q]); }
  }
  float sc[3];
  for (int k = 0; k < 3; ++k) sc[k] = hi[k] > lo[k] ? 1023.f / (hi[k] - lo[k]) : 0.f;
  for (uint32_t i = threadIdx.x; i < I.nt; i += blockDim.x) {
    const float3 c = centroid(i);
    const uint32_t qx = uint32_t(fminf(fmaxf((c.x - lo[0]) * sc[0], 0.f), 1023.f));
    const uint32_t qy = uint32_t(fminf(fmaxf((c.y - lo[1]) * sc[1], 0.f), 1023.f));
    const uint32_t qz = uint32_t(fminf(fmaxf((c.z - lo[2]) * sc[2], 0.f), 1023.f));
    const uint32_t code = morton_spread10(qx) | (morton_spread10(qy) << 1) | (morton_spread10(qz) << 2);
    S.keys[I.tbase + i] = (uint64_t(blockIdx.x) << 30) | code;
    S.order[I.tbase + i] = I.tbase + i;
  }
}

// Stable LSD radix sort of (key, value) pairs, 8-bit digits, over all
// triangles of the batch: per pass a digit histogram per block of kSortTile
// keys (digit-major), an exclusive scan of those counts, and a stable scatter
// (ranks within a block from warp match masks and per-warp digit counts).
__global__ void __launch_bounds__(256) k_rs_hist(const uint64_t* __restrict__ keys, uint32_t n, uint32_t shift,
                                                 uint32_t* __restrict__ hist, uint32_t nblocks) {
  pdl_begin();
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t b0 = blockIdx.x * kSortTile, b1 = min(n, b0 + kSortTile);
  for (uint32_t i = b0 + threadIdx.x; i < b1; i += 256) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  __syncthreads();
  hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(256) k_rs_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                    uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                    uint32_t n, uint32_t shift, const uint32_t* __restrict__ offs,
                                                    uint32_t nblocks) {
  pdl_begin();
  __shared__ uint32_t wcnt[8][256];
  __shared__ uint32_t woff[8][256];
  __shared__ uint32_t run[256];
  const uint32_t t = threadIdx.x, w = t >> 5, lane = t & 31;
  for (uint32_t q = 0; q < 8; ++q) wcnt[q][t] = 0;
  run[t] = offs[t * nblocks + blockIdx.x];
  __syncthreads();
  const uint32_t b0 = blockIdx.x * kSortTile;
  for (uint32_t c0 = b0; c0 < min(n, b0 + kSortTile); c0 += 256) {
    const uint32_t i = c0 + t;
    const bool valid = i < n;
    const uint64_t key = valid ? kin[i] : 0ull;
    const uint32_t d = valid ? uint32_t((key >> shift) & 255u) : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wcnt[w][d] = __popc(peers);
    __syncthreads();
    {  // thread t: digit t's offsets for each warp of this chunk
      uint32_t r = run[t];
      for (uint32_t q = 0; q < 8; ++q) {
        woff[q][t] = r;
        r += wcnt[q][t];
        wcnt[q][t] = 0;
      }
      run[t] = r;
    }
    __syncthreads();
    if (valid) {
      const uint32_t dst = woff[w][d] + rank;
      kout[dst] = key;
      vout[dst] = vin[i];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- trees
// Leaf boxes (bvh.rs:29-43, inflated by the margin) and the level-by-level
// refit, one block per garment.
__global__ void __launch_bounds__(1024) k_self_boxes(BatchDev B, SelfContactView S, float margin_arg) {
  pdl_begin();
  if (blockIdx.x == 0 && threadIdx.x == 0) S.npairs[0] = 0u;  // k_self_pairs counts from zero
  if (blockIdx.x == 0 && threadIdx.x < 2 && S.nvt) S.nvt[threadIdx.x] = 0u;
  const SelfInst& I = S.inst[blockIdx.x];
  if (B.prm->ipc && B.red[blockIdx.x].al_done) return;
  const float margin = margin_arg >= 0.f ? margin_arg : B.prm->thickness;
  float4* mn = S.box_min + I.box_base;
  float4* mx = S.box_max + I.box_base;
  for (uint32_t i = threadIdx.x; i < I.nt; i += blockDim.x) {
    const uint32_t tri = S.leaf_tri ? S.leaf_tri[I.tbase + i] : I.tbase + i;
    if (S.leaf_of) S.leaf_of[tri] = i;
    uint4 id = B.tri_idx[tri];
    float4 a = B.pos[id.x], b = B.pos[id.y], c = B.pos[id.z];
    mn[i] = make_float4(fminf(fminf(a.x, b.x), c.x) - margin, fminf(fminf(a.y, b.y), c.y) - margin,
                        fminf(fminf(a.z, b.z), c.z) - margin, 0.f);
    mx[i] = make_float4(fmaxf(fmaxf(a.x, b.x), c.x) + margin, fmaxf(fmaxf(a.y, b.y), c.y) + margin,
                        fmaxf(fmaxf(a.z, b.z), c.z) + margin, 0.f);
  }
  __syncthreads();
  for (uint32_t l = 1; l < I.nlevels; ++l) {
    uint32_t n = I.lvl_cnt[l], nprev = I.lvl_cnt[l - 1];
    const float4* cmn = mn + I.lvl_off[l - 1];
    const float4* cmx = mx + I.lvl_off[l - 1];
    float4* pmn = mn + I.lvl_off[l];
    float4* pmx = mx + I.lvl_off[l];
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      float4 a0 = cmn[2 * i], a1 = cmx[2 * i];
      if (2 * i + 1 < nprev) {
        float4 b0 = cmn[2 * i + 1], b1 = cmx[2 * i + 1];
        a0 = make_float4(fminf(a0.x, b0.x), fminf(a0.y, b0.y), fminf(a0.z, b0.z), 0.f);
        a1 = make_float4(fmaxf(a1.x, b1.x), fmaxf(a1.y, b1.y), fmaxf(a1.z, b1.z), 0.f);
      }
      pmn[i] = a0;
      pmx[i] = a1;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ bool box_overlap(float4 amn, float4 amx, float4 bmn, float4 bmx) {  // bvh.rs:58
  return amn.x <= bmx.x && amx.x >= bmn.x && amn.y <= bmx.y && amx.y >= bmn.y && amn.z <= bmx.z && amx.z >= bmn.z;
}

// Traversal for leaf i: visits subtrees holding leaves > i whose boxes overlap.
// mode 0 counts, mode 1 writes at the scanned offset.
template <int MODE>
__device__ uint32_t self_traverse(const SelfContactView& S, const SelfInst& I, uint32_t i, uint32_t* count_out,
                                  uint2* out, uint32_t cap) {
  const float4* mn = S.box_min + I.box_base;
  const float4* mx = S.box_max + I.box_base;
  float4 qmn = mn[i], qmx = mx[i];
  uint32_t stack[64];
  int sp = 0;
  stack[sp++] = ((I.nlevels - 1) << 26) | 0u;  // (level, index) packed; index < 2^26
  uint32_t found = 0;
  uint32_t base = MODE == 1 ? *count_out : 0;
  while (sp > 0) {
    uint32_t code = stack[--sp];
    uint32_t l = code >> 26, k = code & ((1u << 26) - 1);
    uint64_t hi = (uint64_t(k) + 1) << l;  // one past the last leaf of the node
    if (hi <= uint64_t(i) + 1) continue;
    uint32_t o = I.lvl_off[l] + k;
    if (!box_overlap(qmn, qmx, mn[o], mx[o])) continue;
    if (l == 0) {
      if (MODE == 1) {
        uint32_t slot = base + found;
        if (slot < cap) {
          uint32_t a = I.tbase + i, b = I.tbase + k;
          if (S.leaf_tri) {
            a = S.leaf_tri[a];
            b = S.leaf_tri[b];
          }
          out[slot] = make_uint2(min(a, b), max(a, b));
        }
      }
      ++found;
      continue;
    }
    // children (l-1, 2k) and (l-1, 2k+1); the right child may not exist.
    // The stack never holds more than two entries per level (< 64).
    if (2 * k + 1 < I.lvl_cnt[l - 1]) stack[sp++] = ((l - 1) << 26) | (2 * k + 1);
    stack[sp++] = ((l - 1) << 26) | (2 * k);
  }
  if (MODE == 0) *count_out = found;
  return found;
}

__global__ void __launch_bounds__(256) k_self_count(BatchDev B, SelfContactView S) {
  pdl_begin();
  int4 ch = B.tri_chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  if (B.prm->ipc && B.red[ch.x].al_done) { S.cnt[ch.y + threadIdx.x] = 0; return; }
  const SelfInst& I = S.inst[ch.x];
  uint32_t t = uint32_t(ch.y) + threadIdx.x;
  uint32_t c = 0;
  self_traverse<0>(S, I, t - I.tbase, &c, nullptr, 0);
  S.cnt[t] = c;
}

// Exclusive scan of the per-triangle counts (three phases).
__global__ void __launch_bounds__(kScanBlock) k_scan_local(uint32_t* v, uint32_t n, uint32_t* block_sums) {
  pdl_begin();
  __shared__ uint32_t sh[kScanBlock];
  uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
  uint32_t x = i < n ? v[i] : 0u;
  sh[threadIdx.x] = x;
  __syncthreads();
  for (int o = 1; o < kScanBlock; o <<= 1) {
    uint32_t y = threadIdx.x >= uint32_t(o) ? sh[threadIdx.x - o] : 0u;
    __syncthreads();
    sh[threadIdx.x] += y;
    __syncthreads();
  }
  if (i < n) v[i] = sh[threadIdx.x] - x;
  if (threadIdx.x == kScanBlock - 1) block_sums[blockIdx.x] = sh[threadIdx.x];
}
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(uint32_t* block_sums, uint32_t nb, uint32_t* total) {
  pdl_begin();
  __shared__ uint32_t sh[kScanBlock];
  uint32_t carry = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += kScanBlock) {
    uint32_t i = b0 + threadIdx.x;
    uint32_t x = i < nb ? block_sums[i] : 0u;
    sh[threadIdx.x] = x;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
      uint32_t y = threadIdx.x >= uint32_t(o) ? sh[threadIdx.x - o] : 0u;
      __syncthreads();
      sh[threadIdx.x] += y;
      __syncthreads();
    }
    if (i < nb) block_sums[i] = carry + sh[threadIdx.x] - x;
    uint32_t last = sh[kScanBlock - 1];
    __syncthreads();
    carry += last;
  }
  if (threadIdx.x == 0) total[0] = carry;
}
__global__ void __launch_bounds__(kScanBlock) k_scan_add(uint32_t* v, uint32_t n, const uint32_t* block_sums) {
  pdl_begin();
  uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) v[i] += block_sums[blockIdx.x];
}

__global__ void __launch_bounds__(256) k_self_write(BatchDev B, SelfContactView S) {
  pdl_begin();
  int4 ch = B.tri_chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  if (B.prm->ipc && B.red[ch.x].al_done) return;
  const SelfInst& I = S.inst[ch.x];
  uint32_t t = uint32_t(ch.y) + threadIdx.x;
  uint32_t off = S.cnt[t];
  self_traverse<1>(S, I, t - I.tbase, &off, S.pairs, uint32_t(S.pair_cap));
  if (threadIdx.x == 0 && S.npairs[0] > S.pair_cap) {
    S.npairs[1] = 1;
    atomicOr(B.status, 2u);  // candidate pairs exceeded the buffer
  }
}

// The candidate pairs in one pass over the tree (the batch detect's form; the
// pair order is not fixed, and nothing downstream depends on it). A thread
// keeps its first kPairBuf pairs in a local buffer while it walks the tree,
// its warp takes slots for all of them with one atomic, and a thread that
// found more walks the tree again to write them all.
constexpr uint32_t kPairBuf = 24;
__global__ void __launch_bounds__(256) k_self_pairs(BatchDev B, SelfContactView S) {
  pdl_begin();
  const int4 ch = B.tri_chunks[blockIdx.x];
  const bool live = (int)threadIdx.x < ch.z && !(B.prm->ipc && B.red[ch.x].al_done);
  const uint32_t lane = threadIdx.x & 31u;
  uint2 buf[kPairBuf];
  uint32_t found = 0, i = 0;
  const SelfInst& I = S.inst[ch.x];  // read in place (cached): the block's threads share it
  if (live) {
    i = uint32_t(ch.y) + threadIdx.x - I.tbase;
    uint32_t zero = 0;
    found = self_traverse<1>(S, I, i, &zero, buf, kPairBuf);
  }
  uint32_t incl = found;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= uint32_t(o)) incl += y;
  }
  uint32_t base = 0;
  if (lane == 31u && incl) base = atomicAdd(S.npairs, incl);
  base = __shfl_sync(0xffffffffu, base, 31) + incl - found;
  if (!live || !found) return;
  const uint64_t cap = S.pair_cap;
  if (uint64_t(base) + found > cap) {
    S.npairs[1] = 1;
    atomicOr(B.status, 2u);  // candidate pairs exceeded the buffer
  }
  if (found <= kPairBuf) {
    for (uint32_t j = 0; j < found; ++j)
      if (uint64_t(base) + j < cap) S.pairs[base + j] = buf[j];
  } else {
    self_traverse<1>(S, I, i, &base, S.pairs, uint32_t(cap));
  }
}

// The deduplicated vertex-triangle CCD tests of this detect's pairs (see
// SelfContactView::vt). A test (v, B) of pair (A, B) is kept unless a
// triangle A' < A around v has a box overlapping B's: the broad phase then
// holds the pair (A', B) too (it lists every pair of overlapping leaf boxes),
// and that pair, or one before it, keeps the test. The CCD's minimum over the
// list is the minimum over every test of every pair, bit for bit.
__global__ void __launch_bounds__(256) k_self_vt(BatchDev B, SelfContactView S) {
  pdl_begin();
  const uint32_t np = min(S.npairs[0], uint32_t(S.pair_cap));
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t k0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); k0 < np; k0 += stride) {
    const uint32_t k = k0 + lane;
    uint2 keep[6];
    uint32_t c = 0;
    if (k < np) {
      const uint2 pr = S.pairs[k];
      const uint32_t inst = S.tri_inst[pr.x];
      const InstDev I = B.inst[inst];
      const uint32_t box_base = S.inst[inst].box_base;
      const uint4 A = B.tri_idx[pr.x], Bt = B.tri_idx[pr.y];
      const uint32_t av[3] = {A.x, A.y, A.z}, bv[3] = {Bt.x, Bt.y, Bt.z};
      const uint32_t* tcode = B.vtri + I.tinc_off;
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const uint32_t* X = side == 0 ? av : bv;
        const uint32_t* Yt = side == 0 ? bv : av;
        const uint32_t xt = side == 0 ? pr.x : pr.y, yt = side == 0 ? pr.y : pr.x;
        const uint32_t yl = box_base + S.leaf_of[yt];
        const float4 ymn = S.box_min[yl], ymx = S.box_max[yl];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const uint32_t v = X[q];
          if (v == Yt[0] || v == Yt[1] || v == Yt[2]) continue;
          bool first = true;
          const uint32_t l = v - I.vbase;
          for (uint32_t e = __ldg(B.vtri_ptr + I.inc_ptr + l), ee = __ldg(B.vtri_ptr + I.inc_ptr + l + 1);
               e < ee && first; ++e) {
            const uint32_t t2 = I.tbase + (__ldg(tcode + e) >> 2);
            if (t2 >= xt) continue;
            const uint32_t o = box_base + S.leaf_of[t2];
            if (box_overlap(S.box_min[o], S.box_max[o], ymn, ymx)) first = false;
          }
          if (first) keep[c++] = make_uint2(v, yt);
        }
      }
    }
    // warp-aggregated slots: one atomic per warp
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= uint32_t(o)) incl += y;
    }
    uint32_t base = 0;
    if (lane == 31u && incl) base = atomicAdd(S.nvt, incl);
    base = __shfl_sync(0xffffffffu, base, 31) + incl - c;
    if (base + c > S.vt_cap) {
      S.nvt[1] = 1u;
    } else {
      for (uint32_t j = 0; j < c; ++j) S.vt[base + j] = keep[j];
    }
  }
}

// ------------------------------------------------- distance primitives
// crates/vistio-contact/src/distance_primitives.rs (FP32 like the reference).
template <class R> struct V3d { R x, y, z; };
template <class R> __device__ __forceinline__ V3d<R> mk(R a, R b, R c) { return {a, b, c}; }
template <class R> __device__ __forceinline__ V3d<R> vsub(V3d<R> a, V3d<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> __device__ __forceinline__ V3d<R> vadd(V3d<R> a, V3d<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> __device__ __forceinline__ V3d<R> vmul(V3d<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> __device__ __forceinline__ R vdot(V3d<R> a, V3d<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> __device__ __forceinline__ V3d<R> vcross(V3d<R> a, V3d<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> __device__ __forceinline__ R rclampd(R v, R lo, R hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ V3d<float> ld3(const float4* p, uint32_t i) { float4 a = p[i]; return {a.x, a.y, a.z}; }

// The primitives are templated on the arithmetic type: FP32 screens every
// candidate, FP64 evaluates those within 10 d_hat of contact (the log barrier
// magnifies the cancellation in these distances there). The thresholds are the
// reference's f32 constants.
template <class R> __device__ __forceinline__ V3d<R> vdiv(V3d<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> __device__ __forceinline__ V3d<R> cvt(V3d<float> a) { return {R(a.x), R(a.y), R(a.z)}; }

template <class R> __device__ R pt_seg_d2(V3d<R> p, V3d<R> a, V3d<R> b) {  // :308-318
  V3d<R> ab = vsub(b, a), ap = vsub(p, a);
  R ab2 = vdot(ab, ab);
  if (ab2 < R(1e-20f)) return vdot(ap, ap);
  R t = rclampd(vdot(ap, ab) / ab2, R(0), R(1));
  V3d<R> c = vadd(a, vmul(ab, t));
  V3d<R> d = vsub(p, c);
  return vdot(d, d);
}

template <class R> __device__ R pt_d2(V3d<R> p, V3d<R> a, V3d<R> b, V3d<R> c) {  // :36-116
  V3d<R> ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a), bp = vsub(p, b), cp = vsub(p, c);
  V3d<R> nrm = vcross(ab, ac);
  if (vdot(nrm, nrm) < R(1e-20f)) {
    R dab = pt_seg_d2(p, a, b), dbc = pt_seg_d2(p, b, c), dca = pt_seg_d2(p, c, a);
    if (dab <= dbc && dab <= dca) return dab;
    if (dbc <= dca) return dbc;
    return dca;
  }
  R d1 = vdot(ab, ap), d2 = vdot(ac, ap);
  if (d1 <= R(0) && d2 <= R(0)) return vdot(ap, ap);
  R d3 = vdot(ab, bp), d4 = vdot(ac, bp);
  if (d3 >= R(0) && d4 <= d3) return vdot(bp, bp);
  R d5 = vdot(ab, cp), d6 = vdot(ac, cp);
  if (d6 >= R(0) && d5 <= d6) return vdot(cp, cp);
  R vc = d1 * d4 - d3 * d2;
  if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) {
    R v = d1 / (d1 - d3);
    V3d<R> q = vsub(p, vadd(a, vmul(ab, v)));
    return vdot(q, q);
  }
  R va = d3 * d6 - d5 * d4;
  if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) {
    R w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    V3d<R> q = vsub(p, vadd(b, vmul(vsub(c, b), w)));
    return vdot(q, q);
  }
  R vb = d5 * d2 - d1 * d6;
  if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) {
    R w = d2 / (d2 - d6);
    V3d<R> q = vsub(p, vadd(a, vmul(ac, w)));
    return vdot(q, q);
  }
  R den = R(1) / (va + vb + vc);
  R v = vb * den, w = vc * den;
  V3d<R> q = vsub(p, vadd(vadd(a, vmul(ab, v)), vmul(ac, w)));
  return vdot(q, q);
}

template <class R> __device__ void pt_grad(V3d<R> p, V3d<R> a, V3d<R> b, V3d<R> c, V3d<R> g[4]) {  // :124-177
  for (int k = 0; k < 4; ++k) g[k] = {R(0), R(0), R(0)};
  V3d<R> ab = vsub(b, a), ac = vsub(c, a), nrm = vcross(ab, ac);
  R a2 = vdot(nrm, nrm);
  if (a2 < R(1e-20f)) return;
  V3d<R> n = vdiv(nrm, R(sqrt(a2)));
  R sd = vdot(vsub(p, a), n);
  V3d<R> pr = vsub(p, vmul(n, sd));
  V3d<R> v2 = vsub(pr, a);
  R d00 = vdot(ab, ab), d01 = vdot(ab, ac), d11 = vdot(ac, ac), d20 = vdot(v2, ab), d21 = vdot(v2, ac);
  R den = d00 * d11 - d01 * d01;
  if (fabs(den) < R(1e-20f)) return;
  R inv = R(1) / den;
  R v = (d11 * d20 - d01 * d21) * inv, w = (d00 * d21 - d01 * d20) * inv, u = R(1) - v - w;
  V3d<R> cl = vadd(vadd(vmul(a, u), vmul(b, v)), vmul(c, w));
  V3d<R> d = vsub(p, cl);
  g[0] = vmul(d, R(2));
  g[1] = vmul(d, R(-2) * u);
  g[2] = vmul(d, R(-2) * v);
  g[3] = vmul(d, R(-2) * w);
}

template <class R>
__device__ void ee_params(V3d<R> d1, V3d<R> d2, V3d<R> r, bool grad_form, R* s_out, R* t_out, bool* degen_both) {
  R a = vdot(d1, d1), e = vdot(d2, d2), f = vdot(d2, r);
  const R eps = R(1e-10f);
  *degen_both = false;
  R s, t;
  if (grad_form) {  // edge_edge_distance_gradient (:251-303)
    if (a < eps || e < eps) { s = R(0); t = R(0); }
    else {
      R c = vdot(d1, r), b = vdot(d1, d2), den = a * e - b * b;
      s = fabs(den) > eps ? rclampd((b * f - c * e) / den, R(0), R(1)) : R(0);
      t = (b * s + f) / e;
      if (t < R(0)) { t = R(0); s = rclampd(-c / a, R(0), R(1)); }
      else if (t > R(1)) { t = R(1); s = rclampd((b - c) / a, R(0), R(1)); }
    }
  } else {  // edge_edge_distance_squared (:185-246)
    if (a < eps && e < eps) { *degen_both = true; s = R(0); t = R(0); }
    else if (a < eps) { t = rclampd(f / e, R(0), R(1)); s = R(0); }
    else {
      R c = vdot(d1, r);
      if (e < eps) { s = rclampd(-c / a, R(0), R(1)); t = R(0); }
      else {
        R b = vdot(d1, d2), den = a * e - b * b;
        s = fabs(den) > eps ? rclampd((b * f - c * e) / den, R(0), R(1)) : R(0);
        t = (b * s + f) / e;
        if (t < R(0)) { t = R(0); s = rclampd(-c / a, R(0), R(1)); }
        else if (t > R(1)) { t = R(1); s = rclampd((b - c) / a, R(0), R(1)); }
      }
    }
  }
  *s_out = s;
  *t_out = t;
}

template <class R> __device__ R ee_d2(V3d<R> a0, V3d<R> a1, V3d<R> b0, V3d<R> b1) {
  V3d<R> d1 = vsub(a1, a0), d2 = vsub(b1, b0), r = vsub(a0, b0);
  R s, t;
  bool dg;
  ee_params(d1, d2, r, false, &s, &t, &dg);
  if (dg) return vdot(r, r);
  V3d<R> q = vsub(vadd(a0, vmul(d1, s)), vadd(b0, vmul(d2, t)));
  return vdot(q, q);
}

template <class R> __device__ void ee_grad(V3d<R> a0, V3d<R> a1, V3d<R> b0, V3d<R> b1, V3d<R> g[4]) {
  V3d<R> d1 = vsub(a1, a0), d2 = vsub(b1, b0), r = vsub(a0, b0);
  R s, t;
  bool dg;
  ee_params(d1, d2, r, true, &s, &t, &dg);
  V3d<R> q = vsub(vadd(a0, vmul(d1, s)), vadd(b0, vmul(d2, t)));
  g[0] = vmul(q, R(2) * (R(1) - s));
  g[1] = vmul(q, R(2) * s);
  g[2] = vmul(q, R(-2) * (R(1) - t));
  g[3] = vmul(q, R(-2) * t);
}

// barrier_gradient_with_thickness (barrier.rs:138-162) in FP64.
__device__ __forceinline__ double scaled_barrier_grad_thick64(double d, double d_hat, double kappa, double th) {
  double tsq = th * th, de = d - tsq;
  double raw = de <= 0.0 ? barrier_grad64(double(1e-12f), d_hat) : barrier_grad64(de, d_hat);
  double r = kappa * raw;
  if (isfinite(r)) return r;
  return signbit(r) ? -1e6 : 1e6;
}

// The two barrier gradients above over an array (the test-only entry point).
__global__ void __launch_bounds__(256) k_barrier_grad(const double* d2, uint32_t n, double d_hat, double kappa,
                                                      double th, double* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = th > 0.0 ? scaled_barrier_grad_thick64(d2[i], d_hat, kappa, th) : scaled_barrier_grad64(d2[i], d_hat, kappa);
}

__device__ __forceinline__ bool excluded(const SelfContactView& S, uint32_t i, uint32_t j) {
  for (uint32_t p = S.adj_ptr[i], e = S.adj_ptr[i + 1]; p < e; ++p) {
    uint32_t a = S.adj[p];
    if (a == j) return true;
    if (a > j) return false;
  }
  return false;
}

// Contributions are summed in FP64: at a vertex between two layers they are
// large and of opposite sign, and an FP32 sum would keep mostly rounding.
// A candidate pair touches at most six vertices (its two triangles'); the
// contributions of its 15 tests are first summed per vertex slot (slots 0-2:
// triangle a's corners, 3-5: triangle b's) in this thread's column of a
// shared-memory array, then added to the accumulator with at most 18 atomics
// instead of up to 180. The column of thread t holds value i at [i][t]:
// consecutive threads, consecutive doubles.
constexpr int kGradThreads = 256;
struct PairGrad {
  double* g;  // this thread's column: value i (slot i / 3, component i % 3) at g[i * kGradThreads]
  __device__ __forceinline__ void clear() const {
#pragma unroll
    for (int i = 0; i < 18; ++i) g[i * kGradThreads] = 0.0;
  }
  __device__ __forceinline__ void add(int slot, V3d<double> v, double bg) const {
    double* q = g + 3 * slot * kGradThreads;
    q[0] += bg * v.x;
    q[kGradThreads] += bg * v.y;
    q[2 * kGradThreads] += bg * v.z;
  }
  __device__ __forceinline__ void flush(double4* G, const uint32_t* av, const uint32_t* bv) const {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const double x = g[(3 * i) * kGradThreads], y = g[(3 * i + 1) * kGradThreads], z = g[(3 * i + 2) * kGradThreads];
      if (x == 0.0 && y == 0.0 && z == 0.0) continue;
      double* p = reinterpret_cast<double*>(G + (i < 3 ? av[i] : bv[i - 3]));
      atomicAdd(p + 0, x);
      atomicAdd(p + 1, y);
      atomicAdd(p + 2, z);
    }
  }
};

// SelfCollisionSystem::detect_ipc_contacts (self_collision.rs:199-276) and
// IpcContactSet::compute_barrier_gradient (ipc_response.rs:170-219), per
// candidate pair: 3+3 vertex-triangle and 9 edge-edge tests. Each test is
// screened in FP32; those with d^2 < 10 d_hat are decided and evaluated in
// FP64 (distance, distance gradient, barrier) and rounded once.
// Compiled for four blocks per SM (64 registers, a few spills in the FP64
// branch) instead of the two that 124 registers allow: contact batch of 64
// sphere drapes 93 -> 86 ms per step (before the per-pair sums).
// Lower bounds of the tests' distances, cheaper than the tests: a
// vertex-triangle distance is at least the vertex's distance to the
// triangle's plane, an edge-edge distance at least the distance between the
// two segments' boxes. A test whose bound reaches the FP32 screen (10 d_hat)
// is skipped without the full test; it could not have been active (d < d_hat)
// in any precision, so the contact set and gradient are unchanged.
__device__ __forceinline__ bool vt_far(V3d<float> p, V3d<float> a, V3d<float> n, float nn, float screen) {
  const float h = vdot(n, vsub(p, a));
  return nn > 1e-30f && h * h >= screen * nn;
}
__device__ __forceinline__ bool ee_far(V3d<float> p0, V3d<float> p1, V3d<float> q0, V3d<float> q1, float screen) {
  auto gap = [](float alo, float ahi, float blo, float bhi) {
    return fmaxf(fmaxf(blo - ahi, alo - bhi), 0.f);
  };
  const float gx = gap(fminf(p0.x, p1.x), fmaxf(p0.x, p1.x), fminf(q0.x, q1.x), fmaxf(q0.x, q1.x));
  const float gy = gap(fminf(p0.y, p1.y), fmaxf(p0.y, p1.y), fminf(q0.y, q1.y), fmaxf(q0.y, q1.y));
  const float gz = gap(fminf(p0.z, p1.z), fmaxf(p0.z, p1.z), fminf(q0.z, q1.z), fmaxf(q0.z, q1.z));
  return gx * gx + gy * gy + gz * gz >= screen;
}

// Three blocks per SM (80 registers, 110 bytes of spill): against four (64
// registers, 174 bytes of spill) the 64-drape contact step 37.25 -> 37.02 ms;
// two (128 registers, no spill) 37.58 ms.
__global__ void __launch_bounds__(kGradThreads, 3) k_self_grad(BatchDev B, SelfContactView S, int mode) {
  pdl_begin();
  __shared__ double acc_s[18 * kGradThreads];  // 36 KB per block
  const StepParams& P = *B.prm;
  uint32_t np = min(S.npairs[0], uint32_t(S.pair_cap));
  double4* G = B.gacc;
  const float screen = 10.f * P.d_hat;
  const double dh = P.d_hat, th = P.thickness;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    uint2 pr = S.pairs[k];
    uint32_t inst = S.tri_inst[pr.x];
    InstRed& R = B.red[inst];
    if (R.al_done) continue;
    const double kap = P.kappa > 0.f ? P.kappa : B.inst[inst].kappa;
    uint4 A = B.tri_idx[pr.x], Bt = B.tri_idx[pr.y];
    uint32_t av[3] = {A.x, A.y, A.z}, bv[3] = {Bt.x, Bt.y, Bt.z};
    uint32_t nact = 0;
    bool viol = false;
    const PairGrad acc{acc_s + threadIdx.x};
    acc.clear();
    for (int side = 0; side < 2; ++side) {
      const uint32_t* X = side == 0 ? av : bv;
      const uint32_t* Yt = side == 0 ? bv : av;
      const int xs = side == 0 ? 0 : 3, ys = side == 0 ? 3 : 0;  // slots of X's and Yt's corners
      const V3d<float> ta = ld3(B.pos, Yt[0]), tb = ld3(B.pos, Yt[1]), tc = ld3(B.pos, Yt[2]);
      const V3d<float> n = vcross(vsub(tb, ta), vsub(tc, ta));
      const float nn = vdot(n, n);
      for (int q = 0; q < 3; ++q) {
        uint32_t v = X[q];
        if (v == Yt[0] || v == Yt[1] || v == Yt[2]) continue;
        const V3d<float> p = ld3(B.pos, v);
        if (vt_far(p, ta, n, nn, screen)) continue;
        // the FP32 screen first: it is cheaper than the exclusion lists, and
        // the two filters commute
        if (!(pt_d2<float>(p, ta, tb, tc) < screen)) continue;
        if (excluded(S, v, Yt[0]) || excluded(S, v, Yt[1]) || excluded(S, v, Yt[2])) continue;
        const V3d<double> p8 = cvt<double>(p), a8 = cvt<double>(ta), b8 = cvt<double>(tb), c8 = cvt<double>(tc);
        double d = pt_d2<double>(p8, a8, b8, c8);
        if (!(d < dh && d > 0.0)) continue;
        ++nact;
        if (d <= double(1e-12f)) viol = true;
        double bg = th > 0.0 ? scaled_barrier_grad_thick64(d, dh, kap, th) : scaled_barrier_grad64(d, dh, kap);
        V3d<double> g[4];
        pt_grad<double>(p8, a8, b8, c8, g);
        acc.add(xs + q, g[0], bg); acc.add(ys + 0, g[1], bg); acc.add(ys + 1, g[2], bg); acc.add(ys + 2, g[3], bg);
      }
    }
    // edges (0,1), (1,2), (2,0) of each triangle, as corner slots
    const int ea[3][2] = {{0, 1}, {1, 2}, {2, 0}};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        uint32_t a0 = av[ea[i][0]], a1 = av[ea[i][1]], b0 = bv[ea[j][0]], b1 = bv[ea[j][1]];
        if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) continue;
        const V3d<float> p0 = ld3(B.pos, a0), p1 = ld3(B.pos, a1), q0 = ld3(B.pos, b0), q1 = ld3(B.pos, b1);
        if (ee_far(p0, p1, q0, q1, screen)) continue;
        if (!(ee_d2<float>(p0, p1, q0, q1) < screen)) continue;
        if (excluded(S, a0, b0) && excluded(S, a0, b1) && excluded(S, a1, b0) && excluded(S, a1, b1)) continue;
        const V3d<double> P0 = cvt<double>(p0), P1 = cvt<double>(p1), Q0 = cvt<double>(q0), Q1 = cvt<double>(q1);
        double d = ee_d2<double>(P0, P1, Q0, Q1);
        if (!(d < dh && d > 0.0)) continue;
        ++nact;
        if (d <= double(1e-12f)) viol = true;
        double bg = th > 0.0 ? scaled_barrier_grad_thick64(d, dh, kap, th) : scaled_barrier_grad64(d, dh, kap);
        V3d<double> g[4];
        ee_grad<double>(P0, P1, Q0, Q1, g);
        acc.add(ea[i][0], g[0], bg); acc.add(ea[i][1], g[1], bg);
        acc.add(3 + ea[j][0], g[2], bg); acc.add(3 + ea[j][1], g[3], bg);
      }
    if (nact) acc.flush(G, av, bv);
    if (mode == 1 && nact) {
      atomicAdd(&R.active, nact);
      if (viol) atomicMax(&R.maxviol_bits, __float_as_uint(1e-3f));
    }
  }
}

// ------------------------------------------------------------------ CCD
// solve_cubic_roots / solve_quadratic_roots (crates/vistio-contact/src/ccd.rs:299-377)
template <class R> __device__ int quad_roots(R a, R b, R c, R* out) {
  const R eps = R(1e-8f);
  if (fabs(a) < eps) {
    if (fabs(b) < eps) return 0;
    out[0] = -c / b;
    return 1;
  }
  R disc = b * b - R(4) * a * c;
  if (disc < -eps) return 0;
  if (fabs(disc) <= eps) { out[0] = -b / (R(2) * a); return 1; }
  R sd = sqrt(disc);
  out[0] = (-b + sd) / (R(2) * a);
  out[1] = (-b - sd) / (R(2) * a);
  return 2;
}
template <class R> __device__ int cubic_roots(R a, R b, R c, R d, R* out) {
  const R eps = R(1e-8f);
  if (fabs(a) < eps) return quad_roots(b, c, d, out);
  R p = b / a, q = c / a, r = d / a;
  R ad = q - p * p / R(3);
  R bd = r - p * q / R(3) + R(2) * p * p * p / R(27);
  R disc = bd * bd / R(4) + ad * ad * ad / R(27);
  R shift = -p / R(3);
  if (disc > eps) {
    R sd = sqrt(disc);
    out[0] = cbrt(-bd / R(2) + sd) + cbrt(-bd / R(2) - sd) + shift;
    return 1;
  } else if (fabs(disc) <= eps) {
    if (fabs(bd) < eps) { out[0] = shift; return 1; }
    R u = cbrt(bd / R(2));
    out[0] = R(-2) * u + shift;
    out[1] = u + shift;
    return 2;
  }
  R rv = sqrt(-ad * ad * ad / R(27));
  if (fabs(rv) < R(1e-12f)) { out[0] = shift; return 1; }
  R cv = rclampd(-bd / (R(2) * rv), R(-1), R(1));
  R th = acos(cv);
  R m = R(2) * cbrt(rv);
  const R pi = R(3.14159265358979323846);
  out[0] = m * cos(th / R(3)) + shift;
  out[1] = m * cos((th + R(2) * pi) / R(3)) + shift;
  out[2] = m * cos((th + R(4) * pi) / R(3)) + shift;
  return 3;
}

// vertex_triangle_ccd (ccd.rs:32-129): returns the safe TOI or a value > 1 for no hit.
template <class R>
__device__ R vt_ccd(V3d<R> p0, V3d<R> p1, V3d<R> a0, V3d<R> a1, V3d<R> b0, V3d<R> b1, V3d<R> c0, V3d<R> c1) {
  const R margin = R(0.9f), min_toi = R(1e-6f);
  V3d<R> dp = vsub(p1, p0);
  V3d<R> ar = vsub(a0, p0), br = vsub(b0, p0), cr = vsub(c0, p0);
  V3d<R> av = vsub(vsub(a1, a0), dp), bvv = vsub(vsub(b1, b0), dp), cv = vsub(vsub(c1, c0), dp);
  V3d<R> bvxcv = vcross(bvv, cv), brxcv = vcross(br, cv), bvxcr = vcross(bvv, cr), brxcr = vcross(br, cr);
  R ca = vdot(av, bvxcv);
  R cb = vdot(ar, bvxcv) + vdot(av, vadd(brxcv, bvxcr));
  R cc = vdot(ar, vadd(brxcv, bvxcr)) + vdot(av, brxcr);
  R cd = vdot(ar, brxcr);
  R roots[3];
  int nr = cubic_roots<R>(ca, cb, cc, cd, roots);
  R best = R(2);
  for (int i = 0; i < nr; ++i) {
    R t = roots[i];
    if (t < -min_toi || t > R(1) + min_toi) continue;
    t = rclampd(t, R(0), R(1));
    V3d<R> pa = vadd(ar, vmul(av, t)), pb = vadd(br, vmul(bvv, t)), pc = vadd(cr, vmul(cv, t));
    V3d<R> v0 = vsub(pb, pa), v1 = vsub(pc, pa);
    V3d<R> n = vcross(v0, v1);
    if (vdot(n, n) < R(1e-20f)) continue;
    V3d<R> v2 = vmul(pa, R(-1));
    R d00 = vdot(v0, v0), d01 = vdot(v0, v1), d11 = vdot(v1, v1), d20 = vdot(v2, v0), d21 = vdot(v2, v1);
    R den = d00 * d11 - d01 * d01;
    if (fabs(den) < R(1e-20f)) continue;
    R inv = R(1) / den;
    R u = (d11 * d20 - d01 * d21) * inv, w = (d00 * d21 - d01 * d20) * inv, v = R(1) - u - w;
    const R tol = R(0.01f);
    if (v >= -tol && u >= -tol && w >= -tol) {
      R safe = fmax(t * margin, min_toi);
      best = fmin(best, safe);
    }
  }
  return best;
}

// compute_max_step_size over the last detect's pairs (ccd.rs:238-292).
// Over the pass's listed tests (SelfContactView::vt), one thread per test; a
// kernel of its own, so that it keeps the registers of one test (six blocks
// per SM). Nothing to do when the list overflowed (k_self_ccd runs then).
__global__ void __launch_bounds__(256, 6) k_self_ccd_list(BatchDev B, SelfContactView S) {
  pdl_begin();
  if (S.nvt[1] != 0u) return;
  const uint32_t nt = min(S.nvt[0], uint32_t(S.vt_cap));
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += gridDim.x * blockDim.x) {
    const uint2 tst = S.vt[k];
    const uint32_t inst = S.tri_inst[tst.y];
    InstRed& R = B.red[inst];
    if (R.al_done) continue;
    const uint32_t vbase = B.inst[inst].vbase;
    const uint4 T = B.tri_idx[tst.y];
    auto P0 = [&](uint32_t v) { return ld3(B.pos, v); };
    auto P1 = [&](uint32_t v) {
      float4 x = B.pos[v], d = B.Y[vbase + B.perm_local[v]];
      return mk<float>(x.x + d.x, x.y + d.y, x.z + d.z);
    };
    const float t = vt_ccd<float>(P0(tst.x), P1(tst.x), P0(T.x), P1(T.x), P0(T.y), P1(T.y), P0(T.z), P1(T.z));
    if (t <= 1.f) atomicMin(&R.toi_bits, __float_as_uint(t));
  }
}

__global__ void __launch_bounds__(256) k_self_ccd(BatchDev B, SelfContactView S) {
  pdl_begin();
  if (S.vt_on && S.nvt[1] == 0u) return;  // k_self_ccd_list has the tests
  uint32_t np = min(S.npairs[0], uint32_t(S.pair_cap));
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    uint2 pr = S.pairs[k];
    uint32_t inst = S.tri_inst[pr.x];
    InstRed& R = B.red[inst];
    if (R.al_done) continue;
    const InstDev I = B.inst[inst];
    uint4 A = B.tri_idx[pr.x], Bt = B.tri_idx[pr.y];
    uint32_t av[3] = {A.x, A.y, A.z}, bv[3] = {Bt.x, Bt.y, Bt.z};
    auto P0 = [&](uint32_t v) { return ld3(B.pos, v); };
    auto P1 = [&](uint32_t v) {
      float4 x = B.pos[v], d = B.Y[I.vbase + B.perm_local[v]];
      return mk<float>(x.x + d.x, x.y + d.y, x.z + d.z);
    };
    float best = 2.f;
    for (int side = 0; side < 2; ++side) {
      const uint32_t* X = side == 0 ? av : bv;
      const uint32_t* Yt = side == 0 ? bv : av;
      for (int q = 0; q < 3; ++q) {
        uint32_t v = X[q];
        if (v == Yt[0] || v == Yt[1] || v == Yt[2]) continue;
        best = fminf(best, vt_ccd<float>(P0(v), P1(v), P0(Yt[0]), P1(Yt[0]), P0(Yt[1]), P1(Yt[1]), P0(Yt[2]), P1(Yt[2])));
      }
    }
    if (best <= 1.f) atomicMin(&R.toi_bits, __float_as_uint(best));
  }
}

// ---------------------------------------------------------------- host side
inline uint32_t self_ccd_launches(const SelfContactView& S) { return S.vt_on ? 2 : 1; }

// The LBVH leaf order: Morton keys, then sort_passes radix passes (5 launches each).
inline uint32_t launch_self_sort(const BatchDev& d, const SelfContactView& S, cudaStream_t st) {
  if (!S.leaf_tri) return 0;
  const uint32_t n = uint32_t(S.T);
  launch_pdl(k_self_keys, S.ninst, 1024, 0, st, d, S);
  uint64_t* k0 = S.keys;
  uint64_t* k1 = S.keys_alt;
  uint32_t* v0 = S.order;
  uint32_t* v1 = S.order_alt;
  const uint32_t L = 256u * S.sort_blocks;
  for (uint32_t p = 0; p < S.sort_passes; ++p) {
    launch_pdl(k_rs_hist, S.sort_blocks, 256, 0, st, k0, n, 8 * p, S.sort_hist, S.sort_blocks);
    launch_pdl(k_scan_local, S.sort_scan_blocks, kScanBlock, 0, st, S.sort_hist, L, S.sort_sums);
    launch_pdl(k_scan_sums, 1, kScanBlock, 0, st, S.sort_sums, S.sort_scan_blocks, S.sort_sums + S.sort_scan_blocks);
    launch_pdl(k_scan_add, S.sort_scan_blocks, kScanBlock, 0, st, S.sort_hist, L, S.sort_sums);
    launch_pdl(k_rs_scatter, S.sort_blocks, 256, 0, st, k0, v0, k1, v1, n, 8 * p, S.sort_hist, S.sort_blocks);
    std::swap(k0, k1);
    std::swap(v0, v1);
  }
  return 1 + 5 * S.sort_passes;
}

// Returns the kernels launched.
inline uint32_t launch_self_detect(const BatchDev& d, const SelfContactView& S, uint32_t n_vtx_chunks,
                                   uint32_t n_tri_chunks, int mode, cudaStream_t st) {
  launch_pdl(k_clear_grad, n_vtx_chunks, 256, 0, st, d);
  const uint32_t ns = launch_self_sort(d, S, st);
  launch_pdl(k_self_boxes, S.ninst, 1024, 0, st, d, S, -1.f);  // margin: StepParams::thickness
  launch_pdl(k_self_pairs, n_tri_chunks, 256, 0, st, d, S);
  uint32_t nl = 4 + ns;
  if (S.vt_on && mode == 0) {  // the pass's CCD tests
    launch_pdl(k_self_vt, 6 * 148, 256, 0, st, d, S);  // 40 registers: six blocks per SM
    ++nl;
  }
  launch_pdl(k_self_grad, 3 * 148, kGradThreads, 0, st, d, S, mode);
  return nl;
}

inline void launch_self_ccd(const BatchDev& d, const SelfContactView& S, cudaStream_t st) {
  if (S.vt_on) launch_pdl(k_self_ccd_list, 6 * 148, 256, 0, st, d, S);
  launch_pdl(k_self_ccd, 4 * 148, 256, 0, st, d, S);
}

vistio_status ensure_self_contact(const BatchDev& d, SelfContactDev& S, const std::vector<vistio_solver*>& solvers,
                                  const std::vector<uint32_t>& vbase, uint64_t T, cudaStream_t st, std::string* err);

vistio_status broadphase_pairs_impl(vistio_ctx* ctx, uint32_t nv, const float* px, const float* py,
                                    const float* pz, uint32_t nt, const uint32_t* tris, float margin, uint32_t* pairs,
                                    uint64_t cap, uint64_t* count);
vistio_status ccd_hits_impl(vistio_ctx* ctx, uint32_t nv, const float* p0, const float* p1,
                            uint32_t nt, const uint32_t* tris, uint64_t npairs, const uint32_t* pairs, uint32_t* hits,
                            uint64_t cap, uint64_t* nhits, float* min_toi);

}  // namespace vistio
