// C ABI of the B200 drape solver (include/vistio_cuda.h).
//
// Ownership: a vistio_solver owns the host-side set-up of one garment (the
// reference's ProjectiveDynamicsSolver after init) and, once stepped, a
// device batch holding just that garment. A vistio_batch packs any number of
// solvers into one set of ragged SoA buffers in HBM and advances them with a
// single CUDA graph per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vistio_cuda.h"
#include "contact_kernels.cuh"
#include "factor_kernels.cuh"
#include "self_contact.cuh"
#include "setup.h"

using namespace vistio;
static_assert(kSubtreeFloats <= kWarpFloats, "a bottom subtree must fit one warp buffer");
static_assert(kSubtreeCols <= kWarpVec, "a bottom subtree's vector slice must fit one warp's vector slots");

struct vistio_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  // Batches free their buffers in the order of this stream, so it lives until
  // the context is destroyed and no batch uses it any more.
  std::mutex mu;
  int refs = 0;
  bool closed = false;
  uint32_t sweep_blocks[3] = {0, 0, 0};  // resident k_sweep blocks on this device: the five- and four-block eight-warp forms, the sixteen-warp form
  uint32_t gsweep_blocks = 0;  // resident k_gsweep blocks
};

namespace {
void ctx_free(vistio_ctx* c) {
  if (c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  delete c;
}
// A batch's hold on its context (declared first in vistio_batch, so released
// after every buffer of the batch has been freed).
struct CtxRef {
  vistio_ctx* c = nullptr;
  void bind(vistio_ctx* x) {
    c = x;
    std::lock_guard<std::mutex> lock(c->mu);
    c->refs++;
  }
  ~CtxRef() {
    if (!c) return;
    bool last;
    {
      std::lock_guard<std::mutex> lock(c->mu);
      last = --c->refs == 0 && c->closed;
    }
    if (last) ctx_free(c);
  }
};
}  // namespace

struct vistio_solver {
  vistio_ctx* ctx = nullptr;
  vistio_solver_config cfg{};
  InstanceSetup setup;
  std::vector<float> host_pos, host_vel;  // SimulationState before the first device step
  int32_t has_ground = 0;
  float ground_h = 0.f;
  vistio_batch* own = nullptr;            // batch of one, created on the first step
};

namespace {

constexpr int kElemThreads = 256;
constexpr int kSolveThreads = 32 * kSolveWarps;
constexpr uint32_t kWideSmem = kWideWarps * (kWarpFloats * 4 + 3 * kWarpVec * 16);

thread_local std::string g_tls_error;

vistio_status fail(vistio_ctx* ctx, vistio_status s, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  g_tls_error = msg;
  return s;
}

#define CU(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? VISTIO_ERR_OOM : VISTIO_ERR_GPU, \
                  std::string(#call) + ": " + cudaGetErrorString(e_));             \
    }                                                                              \
  } while (0)

// Device buffer allocated and freed in the order of one stream (the owning
// context's), so that freeing a retired batch does not synchronise the device
// and stall the work of other streams. The stream must outlive the buffer.
template <class T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  ~DevBuf() { if (p) cudaFreeAsync(p, st); }
  cudaError_t alloc(size_t count, cudaStream_t s) {
    if (p) { cudaFreeAsync(p, st); p = nullptr; }
    st = s;
    n = count;
    if (count == 0) count = 1;
    return cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), s);
  }
  cudaError_t upload(const std::vector<T>& h, cudaStream_t s) {
    cudaError_t e = alloc(h.size(), s);
    if (e != cudaSuccess || h.empty()) return e;
    return cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
  }
  void reset() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    n = 0;
  }
};

}  // namespace

struct vistio_batch {
  CtxRef ctx_ref;  // first member: destroyed last
  vistio_ctx* ctx = nullptr;
  std::vector<vistio_solver*> solvers;
  uint32_t ninst = 0;
  uint64_t V = 0, T = 0, H = 0, NSN = 0;
  std::vector<uint32_t> vbase;
  vistio_solver_config cfg{};
  // device buffers
  DevBuf<InstDev> inst;
  DevBuf<int4> tri_chunks, hinge_chunks, vtx_chunks;
  DevBuf<float4> pos, vel, prev, pred, Y, Tm, hinge_out, grad, grad_up, lam, fin_n;
  DevBuf<float> mass, tri_w, tri_out, vals;
  DevBuf<uint8_t> pinned, in_contact, in_contact_up, ever;
  DevBuf<uint4> tri_idx, hinge_idx;
  DevBuf<float4> tri_dm, hinge_st;
  DevBuf<float2> hinge_wr;
  DevBuf<uint32_t> vtri_ptr, vtri, vhinge_ptr, vhinge, perm_local, rows, lvl_items, fwd_ptr, fwd, status;
  DevBuf<uint2> sub_items;
  uint32_t n_sub = 0;
  uint32_t factor_launches = 0;  // k_front launches of the device factorization
  float factor_ms = 0.f;         // their device time
  // FP64 refinement: permuted f64 CSR of A, kept right-hand side, correction
  DevBuf<uint32_t> a_ptr, a_col;
  DevBuf<double> a_val;
  DevBuf<float4> R0, W;
  uint32_t refine = 0;       // refinement sweeps per refined solve
  BatchDev dev_w{};          // dev with Y = W: the sweeps of a refinement
  // batch levels of the sweeps: offset into lvl_items, block items, warp items
  std::vector<uint32_t> lvl_off, lvl_nb, lvl_nw;
  std::vector<std::pair<uint32_t, uint32_t>> top;  // (level, supernode) of every top-level supernode
  std::vector<SnDev> sn_host;                       // supernode table, for re-scheduling
  // per global supernode: (structure class << 32) | local id. Work units of
  // the per-garment sweeps take equal keys side by side (the same supernode
  // of garments that share a topology: equal work for the block's warps).
  std::vector<uint64_t> sn_key;
  uint32_t warp_limit = kWarpItemLimit;             // s (s + m) limit of a warp item
  uint32_t tri_per = 2, hinge_per = 1;              // elements per thread of k_tri / k_hinge (autotuned)
  uint32_t self_ccd_dedup = 1;                      // self CCD over each vertex-triangle test once
  float tuned_ms = 0.f;                             // sweep time of the tuned schedule (0: not tuned)
  float occ_ms[3] = {-1.f, -1.f, -1.f};  // the autotuner's times of the three forms (ms per solve)
  // k_sweep's compiled form, by blocks per SM: 5 or 4 (eight warps), 2
  // (sixteen warps, units of 2 kUnitItems items); the autotuner's choice
  uint32_t sweep_occ = 4;
  uint32_t unit_items = kUnitItems;  // items per subtree or warp-supernode unit of the schedule
  // sweeps: 0 = one launch per level (k_level), 1 = dependency-driven (k_sweep),
  // 2 = garment groups' tree bottoms by k_gsweep, the rest by k_sweep
  uint32_t sweep_mode = 1;
  std::vector<uint2> units_host;                    // k_sweep work units in forward order
  uint32_t n_units = 0, n_units_fwd = 0;
  std::vector<uint2> units_fwd_host;                // k_sweep forward units: top supernodes deepest first
  std::vector<uint32_t> items_fwd_host;             // their warp supernodes, bundled by depth
  std::vector<uint32_t> sn_depth;                   // ancestors of each supernode in its tree
  DevBuf<uint2> df_units_fwd;
  DevBuf<uint32_t> df_items_fwd;
  DevBuf<uint2> df_units;
  DevBuf<uint32_t> df_parent, df_nkids, df_kid_ptr, df_kids, df_cnt, df_flag, df_queue;
  DevBuf<SnDev> sn;
  DevBuf<float4> U;
  // garment groups (k_gsweep, sweep mode 2): the bottom of the trees of
  // garments that share a symbolic structure, swept one lane per garment
  uint32_t n_groups = 0, n_gitems_fwd = 0, n_gitems_bwd = 0, n_gpack = 0, n_sub_plain = 0;
  std::vector<uint8_t> sn_grouped;  // per global supernode: swept by k_gsweep in mode 2
  DevBuf<GroupDev> grp;
  DevBuf<GsnDev> gsn;
  DevBuf<uint32_t> g_rows, g_fwd_ptr, g_fwd, g_kids, gl_vbase, gl_snbase, gl_inst, g_queue;
  DevBuf<uint2> g_subs, g_items_fwd, g_items_bwd, g_pack;
  DevBuf<float> g_vals;
  uint64_t g_bytes = 0;
  // per topology with groups: what decides which supernodes k_gsweep takes
  struct GTopoHost {
    std::vector<uint8_t> taken, insub;     // laid out for the groups; bottom-subtree supernode
    std::vector<uint32_t> depth, parent, cost;  // cost = s (s + m)
    std::vector<uint64_t> sub_cost;             // factor entries of each bottom subtree
    uint32_t sn_off = 0, sub_base = 0, nsub = 0;
  };
  std::vector<GTopoHost> gtopo_host;
  std::vector<uint32_t> group_topo;                 // per group
  std::vector<std::vector<uint32_t>> group_snbase;  // per group, per lane: the garment's first supernode
  uint32_t group_limit = kWarpItemLimit;            // largest s (s + m) of a supernode above the subtrees in k_gsweep
  DevBuf<InstRed> red;
  DevBuf<StepParams> prm;
  SelfContactDev self;       // self-contact buffers (allocated on first use)
  DevBuf<double4> gacc;      // FP64 self-contact gradient accumulator (first use)
  DevBuf<float> xyz_stage;   // interleaved positions for whole-batch copies (first use)
  DevBuf<uint32_t> res_cnt;  // collider resolve counts and penetrations, 8 per garment (first use)
  DevBuf<double> res_force;  // collider resolve depth sums, 4 per garment (first use)
  uint32_t n_tri_chunks = 0, n_hinge_chunks = 0, n_vtx_chunks = 0;
  uint64_t factor_bytes = 0, device_bytes = 0;
  BatchDev dev{};
  cudaGraphExec_t graph_plain = nullptr, graph_ipc = nullptr;
  int graph_ipc_self = -1;
  uint32_t launches_plain = 0, launches_ipc = 0;
  ~vistio_batch() {
    if (graph_plain) cudaGraphExecDestroy(graph_plain);
    if (graph_ipc) cudaGraphExecDestroy(graph_ipc);
  }
};

struct vistio_factor {
  vistio_ctx* ctx = nullptr;
  uint32_t n = 0;
  std::vector<uint32_t> A_ptr, A_col;
  std::vector<double> A_val;
  Factor f;
  vistio_batch* b = nullptr;  // solve-only device layout
};

namespace {

vistio_status pack_batch(vistio_ctx* ctx, vistio_solver* const* solvers, uint32_t n, vistio_batch* b);

// The level schedule of a batch for a warp-item limit: per level, the
// supernodes for a whole block (heaviest first), then those for one warp
// (heaviest first). Fills lvl_off / lvl_nb / lvl_nw and returns the items.
std::vector<uint32_t> schedule_levels(vistio_batch* b, uint32_t limit) {
  // in sweep mode 2 the garment groups' tree bottoms belong to k_gsweep
  const bool grouped = b->sweep_mode == 2;
  auto skip = [&](uint32_t g) { return grouped && b->sn_grouped[g]; };
  const uint32_t nsub = grouped ? b->n_sub_plain : b->n_sub;
  uint32_t L = 0;
  for (auto& t : b->top) L = std::max(L, t.first + 1);
  std::vector<std::vector<uint32_t>> blk(L), wrp(L);
  for (auto& t : b->top) {
    if (skip(t.second)) continue;
    const SnDev& S = b->sn_host[t.second];
    (warp_item(S.ncols, S.nrows, limit) ? wrp : blk)[t.first].push_back(t.second);
  }
  auto weight = [&](uint32_t q) { return uint64_t(b->sn_host[q].ncols) * (b->sn_host[q].ncols + b->sn_host[q].nrows); };
  // heaviest first; equal supernodes of garments of one topology side by side
  auto heavier = [&](uint32_t a, uint32_t c) {
    const uint64_t wa = weight(a), wc = weight(c);
    if (wa != wc) return wa > wc;
    if (!b->sn_key.empty() && b->sn_key[a] != b->sn_key[c]) return b->sn_key[a] < b->sn_key[c];
    return a < c;
  };
  std::vector<uint32_t> items;
  b->lvl_off.clear(); b->lvl_nb.clear(); b->lvl_nw.clear();
  for (uint32_t l = 0; l < L; ++l) {
    std::stable_sort(blk[l].begin(), blk[l].end(), heavier);
    std::stable_sort(wrp[l].begin(), wrp[l].end(), heavier);
    b->lvl_off.push_back(uint32_t(items.size()));
    b->lvl_nb.push_back(uint32_t(blk[l].size()));
    b->lvl_nw.push_back(uint32_t(wrp[l].size()));
    items.insert(items.end(), blk[l].begin(), blk[l].end());
    items.insert(items.end(), wrp[l].begin(), wrp[l].end());
  }
  b->warp_limit = limit;
  // k_sweep units in forward order: bottom subtrees by eight, then each level's
  // block supernodes one by one and its warp supernodes by eight
  b->units_host.clear();
  const uint32_t UI = b->unit_items;
  for (uint32_t q = 0; q < nsub; q += UI)
    b->units_host.push_back(make_uint2(0u | (std::min(UI, nsub - q) << 2), q));
  for (uint32_t l = 0; l < L; ++l) {
    const uint32_t off = b->lvl_off[l], nb = b->lvl_nb[l], nw = b->lvl_nw[l];
    for (uint32_t i = 0; i < nb; ++i) b->units_host.push_back(make_uint2(1u | (1u << 2), items[off + i]));
    for (uint32_t i = 0; i < nw; i += UI)
      b->units_host.push_back(make_uint2(2u | (std::min(UI, nw - i) << 2), off + nb + i));
  }
  b->n_units = uint32_t(b->units_host.size());
  // The forward sweep's critical path runs from the deepest supernodes of the
  // tallest trees to their roots. Its units: the bottom subtrees as above,
  // then the top supernodes by depth below their root, deepest first (blocks,
  // then warp supernodes by eight of one depth), so the tall trees' chains
  // start while the short trees' supernodes fill the GPU. Children are deeper
  // than their parent: the order stays topological.
  {
    uint32_t D = 0;
    for (auto& t : b->top) D = std::max(D, b->sn_depth[t.second] + 1);
    std::vector<std::vector<uint32_t>> dblk(D), dwrp(D);
    for (auto& t : b->top) {
      if (skip(t.second)) continue;
      const SnDev& S = b->sn_host[t.second];
      (warp_item(S.ncols, S.nrows, limit) ? dwrp : dblk)[b->sn_depth[t.second]].push_back(t.second);
    }
    b->units_fwd_host.clear();
    b->items_fwd_host.clear();
    for (uint32_t q = 0; q < nsub; q += UI)
      b->units_fwd_host.push_back(make_uint2(0u | (std::min(UI, nsub - q) << 2), q));
    for (uint32_t d = D; d-- > 0;) {
      std::stable_sort(dblk[d].begin(), dblk[d].end(), heavier);
      std::stable_sort(dwrp[d].begin(), dwrp[d].end(), heavier);
      for (uint32_t k : dblk[d]) b->units_fwd_host.push_back(make_uint2(1u | (1u << 2), k));
      for (size_t i = 0; i < dwrp[d].size(); i += UI) {
        const uint32_t off = uint32_t(b->items_fwd_host.size());
        const uint32_t cnt = uint32_t(std::min<size_t>(UI, dwrp[d].size() - i));
        b->items_fwd_host.insert(b->items_fwd_host.end(), dwrp[d].begin() + i, dwrp[d].begin() + i + cnt);
        b->units_fwd_host.push_back(make_uint2(2u | (cnt << 2), off));
      }
    }
    b->n_units_fwd = uint32_t(b->units_fwd_host.size());
  }
  return items;
}

// Uploads a schedule from schedule_levels (the unit buffer holds the largest
// possible count, every top supernode its own unit).
cudaError_t upload_schedule(vistio_batch* b, const std::vector<uint32_t>& items, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  if (!items.empty()) e = cudaMemcpyAsync(b->lvl_items.p, items.data(), items.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !b->units_host.empty())
    e = cudaMemcpyAsync(b->df_units.p, b->units_host.data(), b->units_host.size() * sizeof(uint2),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !b->units_fwd_host.empty())
    e = cudaMemcpyAsync(b->df_units_fwd.p, b->units_fwd_host.data(), b->units_fwd_host.size() * sizeof(uint2),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !b->items_fwd_host.empty())
    e = cudaMemcpyAsync(b->df_items_fwd.p, b->items_fwd_host.data(), b->items_fwd_host.size() * 4,
                        cudaMemcpyHostToDevice, st);
  return e;
}
// The supernodes k_gsweep takes at a limit: every bottom-subtree supernode,
// and every laid-out supernode above them whose s (s + m) is at most `limit`
// and all of whose children are taken (closed downwards). Sets the
// per-supernode flags that keep them out of k_sweep's schedule and uploads
// k_gsweep's work items: forward, the subtrees, then the supernodes above them
// deepest first; backward, those shallowest first, then the subtrees. Within
// a depth the same supernode of every group is adjacent (shared row indices).
cudaError_t schedule_groups(vistio_batch* b, uint32_t limit, cudaStream_t st) {
  std::fill(b->sn_grouped.begin(), b->sn_grouped.end(), uint8_t(0));
  std::vector<std::vector<uint8_t>> act(b->gtopo_host.size());
  for (size_t t = 0; t < b->gtopo_host.size(); ++t) {
    const auto& T = b->gtopo_host[t];
    const uint32_t ns = uint32_t(T.taken.size());
    std::vector<uint8_t> kids_ok(ns, 1);
    act[t].assign(ns, 0);
    for (uint32_t q = 0; q < ns; ++q) {  // children precede their parents
      act[t][q] = T.insub[q] || (T.taken[q] && kids_ok[q] && T.cost[q] <= limit);
      if (!act[t][q] && T.parent[q] != UINT32_MAX) kids_ok[T.parent[q]] = 0;
    }
  }
  struct TopItem { uint32_t depth, q, g; };
  std::vector<TopItem> tops;
  std::vector<uint2> fwd, bwd;
  for (uint32_t g = 0; g < b->group_topo.size(); ++g) {
    const uint32_t t = b->group_topo[g];
    const auto& T = b->gtopo_host[t];
    for (uint32_t base : b->group_snbase[g])
      for (uint32_t q = 0; q < act[t].size(); ++q)
        if (act[t][q]) b->sn_grouped[base + q] = 1;
    for (uint32_t q = 0; q < act[t].size(); ++q)
      if (act[t][q] && !T.insub[q]) tops.push_back(TopItem{T.depth[q], q, g});
    for (uint32_t i = 0; i < T.nsub; ++i) fwd.push_back(make_uint2(g, (T.sub_base + i) << 1));
  }
  // the bottom subtrees longest first: each warp runs about two items, so the
  // last ones decide when the launch ends
  std::stable_sort(fwd.begin(), fwd.end(), [&](const uint2& a, const uint2& c) {
    const auto& Ta = b->gtopo_host[b->group_topo[a.x]];
    const auto& Tc = b->gtopo_host[b->group_topo[c.x]];
    return Ta.sub_cost[(a.y >> 1) - Ta.sub_base] > Tc.sub_cost[(c.y >> 1) - Tc.sub_base];
  });
  std::stable_sort(tops.begin(), tops.end(), [](const TopItem& a, const TopItem& c) {
    return a.depth != c.depth ? a.depth > c.depth : a.q != c.q ? a.q < c.q : a.g < c.g;
  });
  const size_t nsub_items = fwd.size();
  for (const TopItem& x : tops) fwd.push_back(make_uint2(x.g, ((b->gtopo_host[b->group_topo[x.g]].sn_off + x.q) << 1) | 1u));
  for (size_t i = tops.size(); i-- > 0;)
    bwd.push_back(make_uint2(tops[i].g, ((b->gtopo_host[b->group_topo[tops[i].g]].sn_off + tops[i].q) << 1) | 1u));
  bwd.insert(bwd.end(), fwd.begin(), fwd.begin() + nsub_items);
  b->n_gitems_fwd = uint32_t(fwd.size());
  b->n_gitems_bwd = uint32_t(bwd.size());
  b->group_limit = limit;
  cudaError_t e = cudaSuccess;
  if (!fwd.empty()) e = cudaMemcpyAsync(b->g_items_fwd.p, fwd.data(), fwd.size() * sizeof(uint2), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !bwd.empty())
    e = cudaMemcpyAsync(b->g_items_bwd.p, bwd.data(), bwd.size() * sizeof(uint2), cudaMemcpyHostToDevice, st);
  return e;
}

inline uint64_t pad4(uint64_t n) { return (n + 3) & ~3ull; }
float estimate_kappa(const vistio_solver_config& c, const InstanceSetup& I);

// Fronts of the device factorization are allocated for groups of garments
// of at most this many bytes (at least one garment per group); one buffer
// serves the groups one after another.
constexpr uint64_t kFrontBudget = 1ull << 30;

// Device bytes one garment occupies in a batch (the sizes pack_batch
// allocates), plus the self-contact buffers when those are used.
uint64_t instance_device_bytes(const InstanceSetup& I, bool refine, bool self_contact) {
  const Factor& F = I.factor;
  uint64_t vals = 0;
  for (const Supernode& X : F.sn) vals += sn_floats(X.ncols, X.nrows);
  const uint64_t V = I.nv, T = I.nt, H = I.nh, R = F.rows.size();
  uint64_t b = vals * 4 + F.sn.size() * sizeof(SnDev) + R * 4 + F.fwd_sn.size() * 4 + (V + 1) * 4 +
               F.sn.size() * 4 + R * 16;
  b += V * (16 * 10 + 4 + 3 + 4 * 3) + T * (16 + 16 + 4 + 36 + 12) + H * (16 + 16 + 8 + 16 + 16) + (V + 1) * 8;
  if (refine || !F.numeric) b += (V + 1) * 4 + I.A_col.size() * 12;
  if (refine) b += V * 32;
  if (!F.numeric) {  // the fronts of the device factorization, freed once it is done (at most kFrontBudget
                     // bytes for a batch of garments that each need less)
    uint64_t fronts = 0;
    for (const Supernode& X : F.sn) fronts += 8 * uint64_t(X.ncols + X.nrows) * (X.ncols + X.nrows);
    b += std::min(fronts, kFrontBudget) + R * 4 + F.sn.size() * 24;
  }
  if (self_contact) b += V * 32 + T * (4 + 2 * 2 * 16 + 4) + 48 * T * 8 + V * 4 + 16 * V * 4;
  return b + 12 * V;  // whole-batch position staging
}


std::vector<int4> make_chunks(const std::vector<uint64_t>& base, const std::vector<uint64_t>& count) {
  std::vector<int4> ch;
  for (size_t k = 0; k < base.size(); ++k)
    for (uint64_t s = 0; s < count[k]; s += kElemThreads)
      ch.push_back(make_int4(int(k), int(base[k] + s), int(std::min<uint64_t>(kElemThreads, count[k] - s)), 0));
  return ch;
}

// Numeric FP64 factorization, on the device, of the garments whose host
// set-up is symbolic only (k_front, one block per supernode, one launch per
// height of the supernodal trees). The batch's supernodes, rows, permuted A
// and (zeroed) factor values are on the device already.
vistio_status factor_on_device(vistio_ctx* ctx, vistio_batch* b, vistio_solver* const* solvers, uint32_t n,
                               const std::vector<InstDev>& hi, const std::vector<SnDev>& sn,
                               const std::vector<uint32_t>& rows) {
  cudaStream_t st = ctx->stream;
  const uint64_t NSN = sn.size();
  std::vector<uint32_t> parent(NSN, UINT32_MAX), height(NSN, 0), kid_ptr(NSN + 1, 0), kids, relmap(rows.size(), 0);
  std::vector<uint64_t> front_off(NSN, 0);
  for (uint32_t k = 0; k < n; ++k) {
    const Factor& F = solvers[k]->setup.factor;
    if (F.numeric) continue;
    const uint32_t base = hi[k].sn_base;
    for (uint32_t q = 0; q < F.sn.size(); ++q) {
      if (F.sn[q].parent == UINT32_MAX) continue;
      const uint32_t g = base + q, p = base + F.sn[q].parent;
      parent[g] = p;
      kid_ptr[p + 1]++;
      height[p] = std::max(height[p], height[g] + 1);  // children precede parents
    }
  }
  for (uint64_t g = 0; g < NSN; ++g) kid_ptr[g + 1] += kid_ptr[g];
  kids.resize(kid_ptr[NSN]);
  {
    std::vector<uint32_t> cur(kid_ptr.begin(), kid_ptr.end() - 1);
    for (uint64_t g = 0; g < NSN; ++g)
      if (parent[g] != UINT32_MAX) kids[cur[parent[g]]++] = uint32_t(g);
  }
  // each child row's position in its parent's front: a column of the parent
  // or one of the parent's rows (the child's rows are a subset of those)
  for (uint64_t g = 0; g < NSN; ++g) {
    if (parent[g] == UINT32_MAX) continue;
    const SnDev &C = sn[g], &P = sn[parent[g]];
    const uint32_t* Rp = rows.data() + P.rows_off;
    for (uint32_t j = 0; j < C.nrows; ++j) {
      const uint32_t r = rows[C.rows_off + j];
      uint32_t at;
      if (r >= P.first && r < P.first + P.ncols) {
        at = r - P.first;
      } else {
        const uint32_t* it = std::lower_bound(Rp, Rp + P.nrows, r);
        if (it == Rp + P.nrows || *it != r)
          return fail(ctx, VISTIO_ERR_INVARIANT, "supernode rows are not contained in the parent's front");
        at = P.ncols + uint32_t(it - Rp);
      }
      relmap[C.rows_off + j] = at;
    }
  }
  // groups of garments, and per group the supernodes by height
  std::vector<uint32_t> items;
  std::vector<uint2> launches;  // (first item, count)
  uint64_t gsize = 0, max_gsize = 0;
  std::vector<uint32_t> group;
  auto flush = [&]() {
    if (group.empty()) return;
    uint32_t hmax = 0;
    for (uint32_t k : group)
      for (uint32_t g = hi[k].sn_base; g < hi[k].sn_base + hi[k].nsn; ++g) hmax = std::max(hmax, height[g]);
    for (uint32_t h = 0; h <= hmax; ++h) {
      const uint32_t first = uint32_t(items.size());
      for (uint32_t k : group)
        for (uint32_t g = hi[k].sn_base; g < hi[k].sn_base + hi[k].nsn; ++g)
          if (height[g] == h) items.push_back(g);
      if (items.size() > first) launches.push_back(make_uint2(first, uint32_t(items.size()) - first));
    }
    max_gsize = std::max(max_gsize, gsize);
    group.clear();
    gsize = 0;
  };
  for (uint32_t k = 0; k < n; ++k) {
    if (solvers[k]->setup.factor.numeric) continue;
    uint64_t fb = 0;
    for (uint32_t g = hi[k].sn_base; g < hi[k].sn_base + hi[k].nsn; ++g) {
      const uint64_t nf = uint64_t(sn[g].ncols) + sn[g].nrows;
      if (nf >= 65536) return fail(ctx, VISTIO_ERR_CAPACITY, "supernode front too large for the device factorization");
      fb += nf * nf;
    }
    if (!group.empty() && (gsize + fb) * 8 > kFrontBudget) flush();
    for (uint32_t g = hi[k].sn_base; g < hi[k].sn_base + hi[k].nsn; ++g) {
      const uint64_t nf = uint64_t(sn[g].ncols) + sn[g].nrows;
      front_off[g] = gsize;
      gsize += nf * nf;
    }
    group.push_back(k);
  }
  flush();
  DevBuf<uint32_t> d_kid_ptr, d_kids, d_relmap, d_items, d_status;
  DevBuf<uint64_t> d_front_off;
  DevBuf<double> d_fronts;
  CU(d_kid_ptr.upload(kid_ptr, st)); CU(d_kids.upload(kids, st)); CU(d_relmap.upload(relmap, st));
  CU(d_items.upload(items, st)); CU(d_front_off.upload(front_off, st));
  CU(d_fronts.alloc(max_gsize, st));
  CU(d_status.alloc(1, st)); CU(cudaMemsetAsync(d_status.p, 0, sizeof(uint32_t), st));
  FrontDev D;
  D.sn = b->sn.p; D.rows = b->rows.p;
  D.a_ptr = b->a_ptr.p; D.a_col = b->a_col.p; D.a_val = b->a_val.p;
  D.front_off = d_front_off.p; D.kid_ptr = d_kid_ptr.p; D.kids = d_kids.p; D.relmap = d_relmap.p;
  D.fronts = d_fronts.p; D.vals = b->vals.p; D.status = d_status.p;
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  CU(cudaEventRecord(e0, st));
  for (const uint2& L : launches) k_front<<<L.y, kFrontThreads, 0, st>>>(D, d_items.p + L.x);
  CU(cudaGetLastError());
  CU(cudaEventRecord(e1, st));
  uint32_t status = 0;
  CU(cudaMemcpyAsync(&status, d_status.p, sizeof(status), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  float ms = 0.f;
  CU(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->factor_ms = ms;
  if (status & 32u) return fail(ctx, VISTIO_ERR_NOT_SPD, "matrix is not symmetric positive definite (device Cholesky pivot)");
  if (status & 64u) return fail(ctx, VISTIO_ERR_INVARIANT, "matrix entry outside the symbolic factor structure");
  b->factor_launches = uint32_t(launches.size());
  return VISTIO_OK;
}

// True if two factors have one symbolic structure: the same ordering
// outcome, supernodes, row structures, elimination tree, bottom subtrees and
// pull lists (only the numbers may differ).
bool same_structure(const Factor& a, const Factor& b) {
  if (a.n != b.n || a.sn.size() != b.sn.size() || a.rows.size() != b.rows.size() || a.nlevels != b.nlevels ||
      a.sub_first.size() != b.sub_first.size() || a.fwd_sn.size() != b.fwd_sn.size())
    return false;
  auto eq = [](const std::vector<uint32_t>& x, const std::vector<uint32_t>& y) {
    return x.size() == y.size() && (x.empty() || std::memcmp(x.data(), y.data(), x.size() * 4) == 0);
  };
  for (size_t q = 0; q < a.sn.size(); ++q) {
    const Supernode &x = a.sn[q], &y = b.sn[q];
    if (x.first != y.first || x.ncols != y.ncols || x.nrows != y.nrows || x.rows_off != y.rows_off ||
        x.parent != y.parent || x.level != y.level)
      return false;
  }
  return eq(a.rows, b.rows) && eq(a.sub_first, b.sub_first) && eq(a.sub_last, b.sub_last) && eq(a.fwd_ptr, b.fwd_ptr) &&
         eq(a.fwd_sn, b.fwd_sn) && eq(a.fwd_pos, b.fwd_pos);
}

// The garment groups of a batch: garments of one symbolic structure (a
// topology), in batch order, kGroupLanes per group; a remainder of fewer
// than kGroupMinLanes garments stays ungrouped. Per topology, the supernodes
// k_gsweep takes: every bottom-subtree supernode, and every supernode of at
// most kWarpVec columns within the default warp-item limit all of whose
// children are taken (so the taken set is closed downwards).
struct GroupPlan {
  struct Topo {
    uint32_t leader = 0;
    std::vector<uint32_t> members;
    std::vector<uint8_t> taken, insub;
    std::vector<uint32_t> depth;  // supernodes above each one
    uint64_t entries = 0;         // interleaved entries of one group's value block
    uint32_t sn_off = 0, row_base = 0, sub_base = 0, rows_base = 0, fwd_base = 0;
  };
  std::vector<Topo> topos;
  std::vector<int32_t> group;  // per garment: its group, or -1
  std::vector<uint32_t> lane;  // per garment: its lane in the group
  std::vector<uint32_t> sclass;  // per garment: its symbolic structure class (any size)
  std::vector<uint32_t> gtopo; // per group: its topology
  std::vector<std::vector<uint32_t>> gmembers;
};

GroupPlan plan_groups(vistio_solver* const* solvers, uint32_t n) {
  GroupPlan G;
  G.group.assign(n, -1);
  G.lane.assign(n, 0);
  G.sclass.assign(n, 0);
  std::vector<GroupPlan::Topo> all;
  for (uint32_t k = 0; k < n; ++k) {
    const Factor& F = solvers[k]->setup.factor;
    size_t t = 0;
    for (; t < all.size(); ++t)
      if (same_structure(solvers[all[t].leader]->setup.factor, F)) break;
    if (t == all.size()) {
      all.emplace_back();
      all.back().leader = k;
    }
    all[t].members.push_back(k);
    G.sclass[k] = uint32_t(t);
  }
  for (auto& T : all) {
    if (T.members.size() < kGroupMinLanes) continue;
    const Factor& F = solvers[T.leader]->setup.factor;
    const uint32_t ns = uint32_t(F.sn.size());
    T.insub.assign(ns, 0);
    for (size_t q = 0; q < F.sub_first.size(); ++q)
      for (uint32_t k = F.sub_first[q]; k <= F.sub_last[q]; ++k) T.insub[k] = 1;
    T.taken.assign(ns, 0);
    std::vector<uint8_t> kids_taken(ns, 1);
    for (uint32_t q = 0; q < ns; ++q) {  // children precede their parents
      const Supernode& X = F.sn[q];
      T.taken[q] = T.insub[q] ||
                   (kids_taken[q] && X.ncols <= kWarpVec && uint64_t(X.ncols) * (X.ncols + X.nrows) <= kWarpItemLimit);
      if (X.parent != UINT32_MAX && !T.taken[q]) kids_taken[X.parent] = 0;
      if (T.taken[q]) T.entries += uint64_t(X.ncols) * (X.ncols + 1) / 2 + uint64_t(X.nrows) * X.ncols;
    }
    T.depth.assign(ns, 0);
    for (uint32_t q = ns; q-- > 0;)
      if (F.sn[q].parent != UINT32_MAX) T.depth[q] = T.depth[F.sn[q].parent] + 1;
    const uint32_t ti = uint32_t(G.topos.size());
    for (size_t i = 0; i < T.members.size(); i += kGroupLanes) {
      const uint32_t cnt = uint32_t(std::min<size_t>(kGroupLanes, T.members.size() - i));
      if (cnt < kGroupMinLanes) break;
      const uint32_t g = uint32_t(G.gmembers.size());
      G.gmembers.emplace_back(T.members.begin() + i, T.members.begin() + i + cnt);
      G.gtopo.push_back(ti);
      for (uint32_t l = 0; l < cnt; ++l) {
        G.group[T.members[i + l]] = int32_t(g);
        G.lane[T.members[i + l]] = l;
      }
    }
    G.topos.push_back(std::move(T));
  }
  return G;
}

vistio_status pack_batch(vistio_ctx* ctx, vistio_solver* const* solvers, uint32_t n, vistio_batch* b) {
  cudaStream_t st = ctx->stream;
  b->ctx = ctx;
  b->ctx_ref.bind(ctx);
  b->solvers.assign(solvers, solvers + n);
  b->ninst = n;
  // untuned: sixteen-warp sweep blocks for a few garments (their solves are
  // one tree's chains), four eight-warp blocks per SM otherwise
  b->sweep_occ = n <= kWideMaxInstances ? 2u : 4u;
  b->unit_items = b->sweep_occ == 2 ? 2 * kUnitItems : kUnitItems;
  b->cfg = solvers[0]->cfg;
  std::vector<InstDev> hi(n);
  std::vector<uint64_t> vb(n), vc(n), tb(n), tc(n), hb(n), hc(n);
  uint64_t V = 0, T = 0, H = 0, NSN = 0, NROWS = 0, NVALS = 0, NLVL = 0, NFWD = 0;
  for (uint32_t k = 0; k < n; ++k) {
    const InstanceSetup& I = solvers[k]->setup;
    vb[k] = V; vc[k] = I.nv; tb[k] = T; tc[k] = I.nt; hb[k] = H; hc[k] = I.nh;
    InstDev& d = hi[k];
    d.vbase = uint32_t(V); d.nv = I.nv;
    d.nlvl = I.factor.nlevels;
    d.model = I.prm.model; d.warp = I.prm.warp; d.weft = I.prm.weft;
    d.inv_hmat2 = 1.f / (I.prm.matrix_dt * I.prm.matrix_dt);
    d.has_ground = solvers[k]->has_ground; d.ground_h = solvers[k]->ground_h;
    d.sn_base = uint32_t(NSN); d.nsn = uint32_t(I.factor.sn.size());
    d.kappa = estimate_kappa(solvers[k]->cfg, I);
    d.unit_stencils = 1;
    for (size_t q = 0; q < I.hinge_st.size() && d.unit_stencils; ++q)
      if (I.hinge_st[q] != ((q & 3u) < 2u ? -1.f : 1.f)) d.unit_stencils = 0;
    V += I.nv; T += I.nt; H += I.nh; NSN += I.factor.sn.size(); NROWS += I.factor.rows.size();
    for (const Supernode& X : I.factor.sn) NVALS += sn_floats(X.ncols, X.nrows);
    NLVL += I.factor.nlevels + 1; NFWD += I.factor.fwd_sn.size();
  }
  if (V >= (1ull << 31) || 3 * T >= (1ull << 30) || 4 * H >= (1ull << 30))
    return fail(ctx, VISTIO_ERR_CAPACITY, "batch too large for 32-bit element indices");
  b->V = V; b->T = T; b->H = H; b->NSN = NSN;
  b->vbase.assign(vb.begin(), vb.end());
  std::vector<float4> pos(V), vel(V);
  std::vector<float> mass(V);
  std::vector<uint8_t> pin(V);
  std::vector<uint4> tri_idx(T);
  std::vector<float4> tri_dm(T);
  std::vector<float> tri_w(T);
  std::vector<uint4> hinge_idx(H);
  std::vector<float4> hinge_st(H);
  std::vector<float2> hinge_wr(H);
  std::vector<uint32_t> vtri_ptr, vhinge_ptr, perm_local(V), fwd_ptr(V + 1, 0), rows;
  std::vector<uint32_t> vtri, vhinge;  // incidence, per connectivity class
  std::vector<SnDev> sn(NSN);
  std::vector<float> vals(NVALS + 4, 0.f);  // +16 bytes: staging windows round up to 16 bytes
  std::vector<uint32_t> fwd(NFWD);
  rows.reserve(NROWS);
  uint32_t LMAX = 0;
  for (uint32_t k = 0; k < n; ++k) LMAX = std::max(LMAX, solvers[k]->setup.factor.nlevels);
  (void)LMAX;
  std::vector<uint2> subs, subs_grouped;
  // Garment groups, and the U slots of every garment: ungrouped garments
  // first, one contiguous run each; then per group 32 slots per local slot,
  // lane-minor (slot i of lane l at u_base + i * 32 + l)
  GroupPlan gp = plan_groups(solvers, n);
  std::vector<uint64_t> ubase(n, 0), g_ubase(gp.gmembers.size(), 0);
  uint64_t NU = 0;
  for (uint32_t k = 0; k < n; ++k)
    if (gp.group[k] < 0) { ubase[k] = NU; NU += solvers[k]->setup.factor.rows.size(); }
  for (size_t g = 0; g < gp.gmembers.size(); ++g) {
    g_ubase[g] = NU;
    NU += uint64_t(kGroupLanes) * solvers[gp.gmembers[g][0]]->setup.factor.rows.size();
  }
  if (NU >= (1ull << 32)) return fail(ctx, VISTIO_ERR_CAPACITY, "batch too large for 32-bit U slot indices");
  uint64_t snb = 0, rowsb = 0, valsb = 0, fwdb = 0;
  for (uint32_t k = 0; k < n; ++k) {
    vistio_solver* S = solvers[k];
    const InstanceSetup& I = S->setup;
    const Factor& F = I.factor;
    uint64_t v0 = vb[k], t0 = tb[k], h0 = hb[k];
    const bool grouped = gp.group[k] >= 0;
    const uint64_t ub = grouped ? g_ubase[gp.group[k]] + gp.lane[k] : ubase[k];
    const uint32_t us = grouped ? kGroupLanes : 1u;  // U slot of local slot i: ub + i * us
    for (uint32_t i = 0; i < I.nv; ++i) {
      pos[v0 + i] = make_float4(S->host_pos[3 * i], S->host_pos[3 * i + 1], S->host_pos[3 * i + 2], 0.f);
      vel[v0 + i] = make_float4(S->host_vel[3 * i], S->host_vel[3 * i + 1], S->host_vel[3 * i + 2], 0.f);
      mass[v0 + i] = I.mass[i];
      pin[v0 + i] = I.pinned[i];
      perm_local[v0 + i] = F.iperm[i];
    }
    for (uint32_t t = 0; t < I.nt; ++t) {
      tri_idx[t0 + t] = make_uint4(uint32_t(v0 + I.tris[3 * t]), uint32_t(v0 + I.tris[3 * t + 1]),
                                   uint32_t(v0 + I.tris[3 * t + 2]), 0u);
      tri_dm[t0 + t] = make_float4(I.dm_inv[4 * t], I.dm_inv[4 * t + 1], I.dm_inv[4 * t + 2], I.dm_inv[4 * t + 3]);
      tri_w[t0 + t] = I.tri_w[t];
    }
    for (uint32_t h = 0; h < I.nh; ++h) {
      hinge_idx[h0 + h] = make_uint4(uint32_t(v0 + I.hinge_v[4 * h]), uint32_t(v0 + I.hinge_v[4 * h + 1]),
                                     uint32_t(v0 + I.hinge_v[4 * h + 2]), uint32_t(v0 + I.hinge_v[4 * h + 3]));
      hinge_st[h0 + h] = make_float4(I.hinge_st[4 * h], I.hinge_st[4 * h + 1], I.hinge_st[4 * h + 2], I.hinge_st[4 * h + 3]);
      hinge_wr[h0 + h] = make_float2(I.hinge_w[h], I.hinge_rest[h]);
    }
    // factor: per supernode one 16-byte aligned region [D | P] (see SnDev)
    for (size_t q = 0; q < F.sn.size(); ++q) {
      const Supernode& X = F.sn[q];
      SnDev& d = sn[snb + q];
      const uint32_t sc = X.ncols, m = X.nrows;
      d.first = X.first; d.ncols = sc; d.nrows = m;
      d.rows_off = uint32_t(rowsb + X.rows_off);
      const uint32_t ld = sn_ld(sc);  // odd leading dimension of D and P (bank-conflict-free reads)
      d.d_off = valsb; valsb += pad4(uint64_t(sc) * ld);
      d.p_off = valsb; valsb += pad4(uint64_t(m) * ld + m);  // panel, then its row indices
      d.vbase = uint32_t(v0);
      d.inst = k;
      d.u_off = uint32_t(ub + uint64_t(X.rows_off) * us);
      d.u_stride = us;
      if (X.level != kBottomLevel) b->top.push_back({X.level, uint32_t(snb + q)});
      if (F.numeric) {  // else the device factorization writes D and P
        const double* Pn = F.vals.data() + X.panel_off;   // row-major m x s
        const double* Dn = F.vals.data() + X.diag_off;    // column-major s x s
        for (uint64_t j = 0; j < m; ++j)
          for (uint32_t c = 0; c < sc; ++c) vals[d.p_off + j * ld + c] = float(Pn[j * sc + c]);
        for (uint64_t c = 0; c < sc; ++c)
          for (uint32_t i = 0; i < sc; ++i) vals[d.d_off + c * ld + i] = float(Dn[c * sc + i]);
      }
      // the panel's row indices (u32 bits), staged with the panel by the sweeps
      std::memcpy(vals.data() + d.p_off + uint64_t(m) * ld, F.rows.data() + X.rows_off, size_t(m) * 4);
    }
    rows.insert(rows.end(), F.rows.begin(), F.rows.end());
    for (size_t q = 0; q < F.sub_first.size(); ++q)
      (grouped ? subs_grouped : subs).push_back(make_uint2(uint32_t(snb + F.sub_first[q]), uint32_t(snb + F.sub_last[q])));
    for (uint32_t r = 0; r < I.nv; ++r) fwd_ptr[v0 + r] = uint32_t(fwdb + F.fwd_ptr[r]);
    for (size_t q = 0; q < F.fwd_sn.size(); ++q)
      fwd[fwdb + q] = uint32_t(ub + uint64_t(F.sn[F.fwd_sn[q]].rows_off + F.fwd_pos[q]) * us);
    snb += F.sn.size(); rowsb += F.rows.size(); fwdb += F.fwd_sn.size();
  }
  fwd_ptr[V] = uint32_t(fwdb);
  // f64 CSR of each instance's A with rows and columns in solve order (global ids)
  std::vector<uint32_t> a_ptr, a_col;
  std::vector<double> a_val;
  bool on_device = false;
  for (uint32_t k = 0; k < n; ++k) on_device = on_device || !solvers[k]->setup.factor.numeric;
  bool have_a = b->cfg.refinement_sweeps > 0 || on_device;
  for (uint32_t k = 0; k < n && have_a; ++k) have_a = !solvers[k]->setup.A_ptr.empty();
  if (on_device && !have_a) return fail(ctx, VISTIO_ERR_INVARIANT, "device factorization without the system matrix");
  if (have_a) {
    uint64_t nnz = 0;
    for (uint32_t k = 0; k < n; ++k) nnz += solvers[k]->setup.A_col.size();
    if (nnz >= (1ull << 32)) return fail(ctx, VISTIO_ERR_CAPACITY, "batch too large for 32-bit matrix offsets");
    a_ptr.reserve(V + 1);
    a_ptr.push_back(0);
    a_col.reserve(nnz);
    a_val.reserve(nnz);
    for (uint32_t k = 0; k < n; ++k) append_permuted_matrix(solvers[k]->setup, uint32_t(vb[k]), a_ptr, a_col, a_val);
    b->refine = b->cfg.refinement_sweeps;
  }
  b->sn_host = sn;
  b->sn_key.assign(NSN, 0);
  for (uint32_t k = 0; k < n; ++k)
    for (uint32_t q = 0; q < hi[k].nsn; ++q) b->sn_key[hi[k].sn_base + q] = (uint64_t(gp.sclass[k]) << 32) | q;
  // subtree units take eight consecutive subtrees: the same subtree of
  // garments of one topology side by side (equal work for the block's warps)
  auto by_key = [&](const uint2& a, const uint2& c) {
    return b->sn_key[a.x] != b->sn_key[c.x] ? b->sn_key[a.x] < b->sn_key[c.x] : a.x < c.x;
  };
  std::sort(subs.begin(), subs.end(), by_key);
  std::sort(subs_grouped.begin(), subs_grouped.end(), by_key);
  b->n_sub_plain = uint32_t(subs.size());
  subs.insert(subs.end(), subs_grouped.begin(), subs_grouped.end());
  b->n_sub = uint32_t(subs.size());
  // the supernodal tree for the dependency-driven sweeps (global ids)
  std::vector<uint32_t> df_parent(NSN, kNoParent), df_nkids(NSN, 0), df_kid_ptr(NSN + 1, 0), df_kids;
  for (uint32_t k = 0; k < n; ++k) {
    const Factor& F = solvers[k]->setup.factor;
    const uint32_t base = hi[k].sn_base;
    for (uint32_t q = 0; q < F.sn.size(); ++q)
      if (F.sn[q].parent != UINT32_MAX) {
        df_parent[base + q] = base + F.sn[q].parent;
        df_nkids[base + F.sn[q].parent]++;
      }
  }
  // depth below the root: parents come after their children (postorder)
  b->sn_depth.assign(NSN, 0);
  for (uint64_t g = NSN; g-- > 0;)
    if (df_parent[g] != kNoParent) b->sn_depth[g] = b->sn_depth[df_parent[g]] + 1;
  std::vector<uint32_t> items = schedule_levels(b, b->warp_limit);
  for (uint64_t g = 0; g < NSN; ++g) df_kid_ptr[g + 1] = df_kid_ptr[g] + df_nkids[g];
  df_kids.resize(df_kid_ptr[NSN]);
  {
    std::vector<uint32_t> cur(df_kid_ptr.begin(), df_kid_ptr.end() - 1);
    for (uint64_t g = 0; g < NSN; ++g)
      if (df_parent[g] != kNoParent) df_kids[cur[df_parent[g]]++] = uint32_t(g);
  }
  // Vertex incidence, once per connectivity class: garments with the same
  // triangles and hinges (the batched workload's garments of one grid side)
  // share one list of (local element << 2 | slot) codes and one array of
  // local offsets per vertex; each garment adds its own element bases.
  {
    std::vector<uint32_t> leader;  // first garment of each class
    for (uint32_t k = 0; k < n; ++k) {
      const InstanceSetup& I = solvers[k]->setup;
      uint32_t c = 0;
      for (; c < leader.size(); ++c) {
        const InstanceSetup& J = solvers[leader[c]]->setup;
        if (J.nv == I.nv && J.nt == I.nt && J.nh == I.nh && J.tris == I.tris && J.hinge_v == I.hinge_v) break;
      }
      if (c == leader.size()) {
        leader.push_back(k);
        const uint32_t pbase = uint32_t(vtri_ptr.size()), tbase = uint32_t(vtri.size()), hbase = uint32_t(vhinge.size());
        std::vector<uint32_t> pt(I.nv + 1, 0), ph(I.nv + 1, 0);
        for (uint32_t t = 0; t < I.nt; ++t)
          for (uint32_t q = 0; q < 3; ++q) pt[I.tris[3 * t + q] + 1]++;
        for (uint32_t h = 0; h < I.nh; ++h)
          for (uint32_t q = 0; q < 4; ++q) ph[I.hinge_v[4 * h + q] + 1]++;
        for (uint32_t i = 0; i < I.nv; ++i) { pt[i + 1] += pt[i]; ph[i + 1] += ph[i]; }
        std::vector<uint32_t> ct(3ull * I.nt), cn(4ull * I.nh);
        std::vector<uint32_t> c1(pt.begin(), pt.end() - 1), c2(ph.begin(), ph.end() - 1);
        for (uint32_t t = 0; t < I.nt; ++t)
          for (uint32_t q = 0; q < 3; ++q) ct[c1[I.tris[3 * t + q]]++] = (t << 2) | q;
        for (uint32_t h = 0; h < I.nh; ++h)
          for (uint32_t q = 0; q < 4; ++q) cn[c2[I.hinge_v[4 * h + q]]++] = (h << 2) | q;
        vtri_ptr.insert(vtri_ptr.end(), pt.begin(), pt.end());
        vhinge_ptr.insert(vhinge_ptr.end(), ph.begin(), ph.end());
        vtri.insert(vtri.end(), ct.begin(), ct.end());
        vhinge.insert(vhinge.end(), cn.begin(), cn.end());
        hi[k].inc_ptr = pbase; hi[k].tinc_off = tbase; hi[k].hinc_off = hbase;
      } else {
        hi[k].inc_ptr = hi[leader[c]].inc_ptr;
        hi[k].tinc_off = hi[leader[c]].tinc_off;
        hi[k].hinc_off = hi[leader[c]].hinc_off;
      }
      hi[k].tbase = uint32_t(tb[k]);
      hi[k].hbase = uint32_t(hb[k]);
    }
  }
  auto tch = make_chunks(tb, tc), hch = make_chunks(hb, hc), vch = make_chunks(vb, vc);
  b->n_tri_chunks = uint32_t(tch.size()); b->n_hinge_chunks = uint32_t(hch.size()); b->n_vtx_chunks = uint32_t(vch.size());
  CU(cudaSetDevice(ctx->device));
  CU(b->inst.upload(hi, st));
  CU(b->tri_chunks.upload(tch, st)); CU(b->hinge_chunks.upload(hch, st)); CU(b->vtx_chunks.upload(vch, st));
  CU(b->pos.upload(pos, st)); CU(b->vel.upload(vel, st));
  CU(b->prev.upload(pos, st)); CU(b->pred.upload(pos, st));
  CU(b->mass.upload(mass, st)); CU(b->pinned.upload(pin, st));
  CU(b->tri_idx.upload(tri_idx, st)); CU(b->tri_dm.upload(tri_dm, st)); CU(b->tri_w.upload(tri_w, st));
  CU(b->tri_out.alloc(9 * T, st));
  CU(b->hinge_idx.upload(hinge_idx, st)); CU(b->hinge_st.upload(hinge_st, st)); CU(b->hinge_wr.upload(hinge_wr, st));
  CU(b->hinge_out.alloc(H, st));
  CU(b->vtri_ptr.upload(vtri_ptr, st)); CU(b->vtri.upload(vtri, st));
  CU(b->vhinge_ptr.upload(vhinge_ptr, st)); CU(b->vhinge.upload(vhinge, st));
  CU(b->perm_local.upload(perm_local, st));
  CU(b->Y.alloc(V, st)); CU(b->Tm.alloc(V, st));
  CU(b->sn.upload(sn, st)); CU(b->rows.upload(rows, st)); CU(b->vals.upload(vals, st));
  CU(b->lvl_items.upload(items, st));
  CU(b->sub_items.upload(subs, st));
  CU(b->df_units.alloc((b->n_sub + kSolveWarps - 1) / kSolveWarps + b->top.size() + 1, st));
  CU(b->df_units_fwd.alloc((b->n_sub + kSolveWarps - 1) / kSolveWarps + b->top.size() + 1, st));
  CU(b->df_items_fwd.alloc(b->top.size() + 1, st));
  CU(upload_schedule(b, items, st));
  CU(b->df_parent.upload(df_parent, st)); CU(b->df_nkids.upload(df_nkids, st));
  CU(b->df_kid_ptr.upload(df_kid_ptr, st)); CU(b->df_kids.upload(df_kids, st));
  CU(b->df_cnt.alloc(NSN, st)); CU(cudaMemsetAsync(b->df_cnt.p, 0, NSN * 4, st));
  CU(b->df_flag.alloc(NSN, st)); CU(cudaMemsetAsync(b->df_flag.p, 0, NSN * 4, st));
  CU(b->df_queue.alloc(2, st)); CU(cudaMemsetAsync(b->df_queue.p, 0, 8, st));
  CU(b->fwd_ptr.upload(fwd_ptr, st)); CU(b->fwd.upload(fwd, st));
  CU(b->U.alloc(NU, st));
  if (have_a) { CU(b->a_ptr.upload(a_ptr, st)); CU(b->a_col.upload(a_col, st)); CU(b->a_val.upload(a_val, st)); }
  if (b->refine) { CU(b->R0.alloc(V, st)); CU(b->W.alloc(V, st)); }
  if (on_device) {
    vistio_status r = factor_on_device(ctx, b, solvers, n, hi, sn, rows);
    if (r != VISTIO_OK) return r;
    if (!b->refine) { b->a_ptr.reset(); b->a_col.reset(); b->a_val.reset(); }
  }
  CU(b->grad.alloc(V, st)); CU(b->grad_up.alloc(V, st)); CU(b->lam.alloc(V, st)); CU(b->fin_n.alloc(V, st));
  CU(cudaMemsetAsync(b->lam.p, 0, V * sizeof(float4), st));
  CU(cudaMemsetAsync(b->grad.p, 0, V * sizeof(float4), st));
  CU(cudaMemsetAsync(b->grad_up.p, 0, V * sizeof(float4), st));
  CU(b->in_contact.alloc(V, st)); CU(b->in_contact_up.alloc(V, st)); CU(b->ever.alloc(V, st));
  CU(b->red.alloc(n, st)); CU(cudaMemsetAsync(b->red.p, 0, n * sizeof(InstRed), st));
  CU(b->prm.alloc(1, st));
  CU(b->status.alloc(1, st)); CU(cudaMemsetAsync(b->status.p, 0, sizeof(uint32_t), st));
  CU(cudaStreamSynchronize(st));
  b->factor_bytes = vals.size() * sizeof(float) + sn.size() * sizeof(SnDev) + rows.size() * 4 + fwd.size() * 4 +
                    fwd_ptr.size() * 4 + items.size() * 4 + rows.size() * 16;
  b->device_bytes = b->factor_bytes + V * (16 * 10 + 4 + 3 + 4 * 3) + T * (16 + 16 + 4 + 36 + 12) +
                    H * (16 + 16 + 8 + 16 + 16) + (V + 1) * 8 + NSN * 28 + b->df_units.n * 8;
  if (b->refine) b->device_bytes += (V + 1) * 4 + a_col.size() * 12 + V * 32;
  BatchDev& d = b->dev;
  d.inst = b->inst.p; d.tri_chunks = b->tri_chunks.p; d.hinge_chunks = b->hinge_chunks.p; d.vtx_chunks = b->vtx_chunks.p;
  d.pos = b->pos.p; d.vel = b->vel.p; d.prev = b->prev.p; d.pred = b->pred.p; d.mass = b->mass.p; d.pinned = b->pinned.p;
  d.tri_idx = b->tri_idx.p; d.tri_dm = b->tri_dm.p; d.tri_w = b->tri_w.p; d.tri_out = b->tri_out.p;
  d.hinge_idx = b->hinge_idx.p; d.hinge_st = b->hinge_st.p; d.hinge_wr = b->hinge_wr.p; d.hinge_out = b->hinge_out.p;
  d.vtri_ptr = b->vtri_ptr.p; d.vtri = b->vtri.p; d.vhinge_ptr = b->vhinge_ptr.p; d.vhinge = b->vhinge.p;
  d.perm_local = b->perm_local.p; d.row_vertex = nullptr; d.Y = b->Y.p; d.T = b->Tm.p;
  d.sn = b->sn.p; d.rows = b->rows.p; d.vals = b->vals.p; d.lvl_items = b->lvl_items.p; d.sub_items = b->sub_items.p;
  d.fwd_ptr = b->fwd_ptr.p; d.fwd = b->fwd.p; d.U = b->U.p;
  d.df_units = b->df_units.p; d.df_parent = b->df_parent.p; d.df_nkids = b->df_nkids.p;
  d.df_units_fwd = b->df_units_fwd.p; d.df_items_fwd = b->df_items_fwd.p;
  d.df_kid_ptr = b->df_kid_ptr.p; d.df_kids = b->df_kids.p; d.df_cnt = b->df_cnt.p; d.df_flag = b->df_flag.p;
  d.df_queue = b->df_queue.p;
  d.a_ptr = b->a_ptr.p; d.a_col = b->a_col.p; d.a_val = b->a_val.p; d.R0 = b->R0.p; d.W = b->W.p;
  d.grad = b->grad.p; d.grad_up = b->grad_up.p; d.lam = b->lam.p; d.fin_n = b->fin_n.p;
  d.in_contact = b->in_contact.p; d.in_contact_up = b->in_contact_up.p; d.ever = b->ever.p;
  d.red = b->red.p; d.prm = b->prm.p; d.status = b->status.p;
  // ---- garment groups: topology tables, lanes, interleaved values, work items
  b->n_groups = uint32_t(gp.gmembers.size());
  b->sn_grouped.assign(NSN, 0);
  if (b->n_groups) {
    std::vector<GsnDev> gsn;
    std::vector<uint32_t> g_rows, g_fwd_ptr, g_fwd, g_kids;
    std::vector<uint2> g_subs;
    for (auto& T : gp.topos) {
      const Factor& F = solvers[T.leader]->setup.factor;
      const uint32_t ns = uint32_t(F.sn.size());
      T.sn_off = uint32_t(gsn.size());
      T.rows_base = uint32_t(g_rows.size());
      T.row_base = uint32_t(g_fwd_ptr.size());
      T.fwd_base = uint32_t(g_fwd.size());
      T.sub_base = uint32_t(g_subs.size());
      std::vector<std::vector<uint32_t>> kids(ns);
      for (uint32_t q = 0; q < ns; ++q)
        if (F.sn[q].parent != UINT32_MAX) kids[F.sn[q].parent].push_back(q);
      uint64_t goff = 0;
      for (uint32_t q = 0; q < ns; ++q) {
        const Supernode& X = F.sn[q];
        GsnDev g{};
        g.first = X.first; g.ncols = X.ncols; g.nrows = X.nrows;
        g.rows_off = T.rows_base + X.rows_off;
        g.u_local = X.rows_off;
        g.parent = X.parent == UINT32_MAX ? kGNone : X.parent;
        g.kid_off = uint32_t(g_kids.size());
        g.nkids = uint32_t(kids[q].size());
        g_kids.insert(g_kids.end(), kids[q].begin(), kids[q].end());
        g.g_off = goff;
        if (T.taken[q]) goff += uint64_t(X.ncols) * (X.ncols + 1) / 2 + uint64_t(X.nrows) * X.ncols;
        gsn.push_back(g);
      }
      g_rows.insert(g_rows.end(), F.rows.begin(), F.rows.end());
      for (uint32_t r = 0; r <= F.n; ++r) g_fwd_ptr.push_back(T.fwd_base + F.fwd_ptr[r]);
      for (size_t q = 0; q < F.fwd_sn.size(); ++q) g_fwd.push_back(F.sn[F.fwd_sn[q]].rows_off + F.fwd_pos[q]);
      for (size_t q = 0; q < F.sub_first.size(); ++q)
        g_subs.push_back(make_uint2(T.sn_off + F.sub_first[q], T.sn_off + F.sub_last[q]));
    }
    const uint32_t NG = b->n_groups;
    std::vector<GroupDev> grp(NG);
    std::vector<uint32_t> gl_vbase(kGroupLanes * NG, 0), gl_snbase(kGroupLanes * NG, 0), gl_inst(kGroupLanes * NG, 0);
    std::vector<uint2> pack;
    uint64_t gbase = 0, max_items = 0;
    for (const auto& T : gp.topos) {
      vistio_batch::GTopoHost h;
      const Factor& F = solvers[T.leader]->setup.factor;
      h.taken = T.taken; h.insub = T.insub; h.depth = T.depth;
      h.sn_off = T.sn_off; h.sub_base = T.sub_base; h.nsub = uint32_t(F.sub_first.size());
      for (const Supernode& X : F.sn) {
        h.parent.push_back(X.parent);
        h.cost.push_back(X.ncols * (X.ncols + X.nrows));
      }
      for (size_t q = 0; q < F.sub_first.size(); ++q) {
        uint64_t c = 0;
        for (uint32_t k = F.sub_first[q]; k <= F.sub_last[q]; ++k)
          c += uint64_t(F.sn[k].ncols) * (F.sn[k].ncols + 1) / 2 + uint64_t(F.sn[k].nrows) * F.sn[k].ncols;
        h.sub_cost.push_back(c);
      }
      b->gtopo_host.push_back(std::move(h));
    }
    for (uint32_t g = 0; g < NG; ++g) {
      const auto& T = gp.topos[gp.gtopo[g]];
      const auto& mem = gp.gmembers[g];
      grp[g] = GroupDev{T.sn_off, uint32_t(mem.size()), gbase, uint32_t(g_ubase[g]), T.row_base};
      gbase += T.entries;
      b->group_topo.push_back(gp.gtopo[g]);
      b->group_snbase.emplace_back();
      for (uint32_t l = 0; l < mem.size(); ++l) {
        const uint32_t k = mem[l];
        gl_vbase[kGroupLanes * g + l] = uint32_t(vb[k]);
        gl_snbase[kGroupLanes * g + l] = hi[k].sn_base;
        gl_inst[kGroupLanes * g + l] = k;
        b->group_snbase.back().push_back(hi[k].sn_base);
      }
      for (uint32_t q = 0; q < T.taken.size(); ++q) {
        if (!T.taken[q]) continue;
        pack.push_back(make_uint2(g, T.sn_off + q));
        ++max_items;  // a supernode above the subtrees, or part of one subtree item
      }
    }
    b->n_gpack = uint32_t(pack.size());
    CU(b->grp.upload(grp, st)); CU(b->gsn.upload(gsn, st));
    CU(b->g_rows.upload(g_rows, st)); CU(b->g_fwd_ptr.upload(g_fwd_ptr, st)); CU(b->g_kids.upload(g_kids, st));
    CU(b->g_fwd.upload(g_fwd, st));
    CU(b->g_subs.upload(g_subs, st));
    CU(b->gl_vbase.upload(gl_vbase, st)); CU(b->gl_snbase.upload(gl_snbase, st)); CU(b->gl_inst.upload(gl_inst, st));
    CU(b->g_items_fwd.alloc(max_items + 1, st)); CU(b->g_items_bwd.alloc(max_items + 1, st));
    CU(b->g_pack.upload(pack, st));
    CU(b->g_queue.alloc(2, st)); CU(cudaMemsetAsync(b->g_queue.p, 0, 8, st));
    CU(b->g_vals.alloc(gbase * kGroupLanes, st));
    d.grp = b->grp.p; d.gsn = b->gsn.p; d.g_rows = b->g_rows.p; d.g_fwd_ptr = b->g_fwd_ptr.p; d.g_fwd = b->g_fwd.p;
    d.g_kids = b->g_kids.p; d.g_subs = b->g_subs.p; d.gl_vbase = b->gl_vbase.p; d.gl_snbase = b->gl_snbase.p;
    d.gl_inst = b->gl_inst.p; d.g_vals = b->g_vals.p; d.g_items_fwd = b->g_items_fwd.p;
    d.g_items_bwd = b->g_items_bwd.p; d.g_queue = b->g_queue.p;
    // the groups' factor values, interleaved from the per-garment regions
    if (!pack.empty()) k_gpack<<<uint32_t(pack.size()), 256, 0, st>>>(d, b->g_vals.p, b->g_pack.p);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(st));
    b->g_bytes = gbase * kGroupLanes * 4 + gsn.size() * sizeof(GsnDev) + (g_rows.size() + g_fwd_ptr.size() +
                 g_fwd.size() + g_kids.size()) * 4 + (2 * max_items + pack.size()) * 8;
    b->device_bytes += b->g_bytes;
    b->g_pack.reset();
    b->sweep_mode = 2;
    CU(schedule_groups(b, b->group_limit, st));
    std::vector<uint32_t> items2 = schedule_levels(b, b->warp_limit);
    CU(upload_schedule(b, items2, st));
    CU(cudaStreamSynchronize(st));
  }
  b->dev_w = d;
  b->dev_w.Y = b->W.p;
  return VISTIO_OK;
}

// estimate_initial_kappa (barrier.rs:97-116) with the runner's inputs (no
// configured kappa, the garment's mean free-vertex lumped mass, |g_y|, the
// configured d_hat). Each garment gets its own, so its result does not depend
// on the garments it is batched with.
float estimate_kappa(const vistio_solver_config& c, const InstanceSetup& I) {
  double sm = 0;
  uint32_t cnt = 0;
  for (uint32_t i = 0; i < I.nv; ++i) if (!I.pinned[i]) { sm += I.mass[i]; ++cnt; }
  const float avg_mass = cnt ? float(sm / cnt) : 1e-3f;
  float dhat = c.barrier_d_hat, dmid = dhat * 0.5f;
  float dcl = std::fmin(std::fmax(dmid, dhat * 1e-3f), dhat);
  double d64 = dcl, dd = dhat, diff = d64 - dd;
  float gm = float(-(diff) * (2.0 * std::log(d64 / dd) + diff / d64));
  gm = std::fabs(gm);
  if (gm < 1e-12f) return 1e4f;
  float kap = avg_mass * std::fabs(c.gravity[1]) / (2.f * std::sqrt(dmid) * gm);
  return std::fmin(std::fmax(kap, 1.f), 1e6f);
}

StepParams make_params(const vistio_solver_config& c, float dt, const vistio_contact_desc* ct) {
  StepParams p{};
  p.dt = dt;
  p.inv_dt2 = 1.f / (dt * dt);
  for (int k = 0; k < 3; ++k) p.gravity[k] = c.gravity[k];
  p.damping = c.damping;
  p.rayleigh = c.rayleigh_mass_damping;
  p.al_tolerance = c.al_tolerance;
  p.al_mu_growth = c.al_mu_growth;
  p.al_mu_initial = c.al_mu_initial;
  p.friction = c.friction_coefficient;
  p.contact_damping = c.contact_damping;
  p.contact_damping_max = c.contact_damping_max;
  p.contact_vthresh = c.contact_velocity_threshold;
  p.adaptive_damping = c.adaptive_contact_damping;
  if (ct) {
    p.ipc = 1;
    float dh = c.compliant_contact ? c.barrier_d_hat * c.compliant_d_hat_scale : c.barrier_d_hat;
    p.d_hat = dh;
    p.max_vel = (0.5f * std::sqrt(dh)) / dt;  // pd_solver.rs:573-595
    p.has_ground = ct->has_ground;
    p.ground_h = ct->ground_height;
    p.has_sphere = ct->has_sphere;
    for (int k = 0; k < 3; ++k) p.sphere_c[k] = ct->sphere_center[k];
    p.sphere_r = ct->sphere_radius;
    p.self_collision = ct->self_collision;
    p.thickness = ct->thickness;
    p.has_cyl = ct->has_cylinder;
    p.cyl[0] = ct->cylinder_center_x; p.cyl[1] = ct->cylinder_center_z;
    p.cyl[2] = ct->cylinder_top_y; p.cyl[3] = ct->cylinder_radius;
    p.has_box = ct->has_box;
    for (int k = 0; k < 3; ++k) { p.box_lo[k] = ct->box_min[k]; p.box_hi[k] = ct->box_max[k]; }
    // explicit stiffness, else 0: each garment uses its own estimate (InstDev::kappa)
    p.kappa = ct->kappa > 0.f ? ct->kappa : (c.barrier_kappa > 0.f ? c.barrier_kappa : 0.f);
  }
  return p;
}

// One k_sweep launch over the batch's units in the chosen compiled form.
void launch_k_sweep(vistio_batch* b, const BatchDev& dv, cudaStream_t st) {
  const uint32_t form = b->sweep_occ == 5 ? 0u : b->sweep_occ == 4 ? 1u : 2u;
  const uint32_t grid = std::min(b->n_units_fwd + b->n_units, b->ctx->sweep_blocks[form]);
  if (form == 0) launch_pdl(k_sweep<5>, grid, kSolveThreads, kSolveSmem, st, dv, b->n_units_fwd, b->n_units);
  else if (form == 1) launch_pdl(k_sweep<4>, grid, kSolveThreads, kSolveSmem, st, dv, b->n_units_fwd, b->n_units);
  else
    launch_pdl(k_sweep<2, kWideWarps>, grid, 32 * kWideWarps, kWideSmem, st, dv, b->n_units_fwd, b->n_units);
}

// Forward then backward sweep, level by level over the whole batch, in place
// on dv.Y (right-hand side in, solution out). Returns the launches.
uint32_t launch_sweeps(vistio_batch* b, const BatchDev& dv, cudaStream_t st) {
  if (b->sweep_mode == 2 && b->n_groups) {
    // the groups' tree bottoms forward, everything above them (and the
    // ungrouped garments) both ways, then the groups' tree bottoms backward
    const uint32_t gf = std::min((b->n_gitems_fwd + kGWarps - 1) / kGWarps, b->ctx->gsweep_blocks);
    const uint32_t gb = std::min((b->n_gitems_bwd + kGWarps - 1) / kGWarps, b->ctx->gsweep_blocks);
    uint32_t n = 0;
    if (gf) { launch_pdl(k_gsweep<0>, gf, kGThreads, kGSmem, st, dv, b->n_gitems_fwd); ++n; }
    if (b->n_units_fwd + b->n_units) {
      launch_k_sweep(b, dv, st);
      ++n;
    }
    if (gb) { launch_pdl(k_gsweep<1>, gb, kGThreads, kGSmem, st, dv, b->n_gitems_bwd); ++n; }
    return n;
  }
  if (b->sweep_mode == 1 && b->n_units) {
    launch_k_sweep(b, dv, st);
    return 1;
  }
  uint32_t L = uint32_t(b->lvl_off.size()), n = 0;
  const uint32_t sub_grid = (b->n_sub + kSolveWarps - 1) / kSolveWarps;
  if (sub_grid) { launch_pdl(k_subtree<0>, sub_grid, kSolveThreads, kSolveSmem, st, dv, b->n_sub); ++n; }
  for (uint32_t l = 0; l < L; ++l) {
    uint32_t grid = b->lvl_nb[l] + (b->lvl_nw[l] + kSolveWarps - 1) / kSolveWarps;
    if (grid) { launch_pdl(k_level<0>, grid, kSolveThreads, kSolveSmem, st, dv, b->lvl_off[l], b->lvl_nb[l], b->lvl_nw[l]); ++n; }
  }
  for (int l = int(L) - 1; l >= 0; --l) {
    uint32_t grid = b->lvl_nb[l] + (b->lvl_nw[l] + kSolveWarps - 1) / kSolveWarps;
    if (grid) { launch_pdl(k_level<1>, grid, kSolveThreads, kSolveSmem, st, dv, b->lvl_off[l], b->lvl_nb[l], b->lvl_nw[l]); ++n; }
  }
  if (sub_grid) { launch_pdl(k_subtree<1>, sub_grid, kSolveThreads, kSolveSmem, st, dv, b->n_sub); ++n; }
  return n;
}

// One FP64 refinement: W = R0 - A d, then the sweeps solve A e = W in place.
uint32_t launch_refinement(vistio_batch* b, cudaStream_t st) {
  launch_pdl(k_refine, b->n_vtx_chunks, kElemThreads, 0, st, b->dev);
  return 1 + launch_sweeps(b, b->dev_w, st);
}

// The global solve: the sweeps, `refine` FP64 refinement sweeps, then the
// residual sums and (plain step) the position update.
uint32_t launch_solve(vistio_batch* b, cudaStream_t st, int do_update, uint32_t refine) {
  uint32_t n = 2;
  launch_pdl(k_red_reset, (b->ninst + 127) / 128, 128, 0, st, b->dev, b->ninst);
  n += launch_sweeps(b, b->dev, st);
  for (uint32_t k = 0; k < refine; ++k) {
    if (k) { launch_pdl(k_accum, b->n_vtx_chunks, kElemThreads, 0, st, b->dev); ++n; }
    n += launch_refinement(b, st);
  }
  launch_pdl(k_update, b->n_vtx_chunks, 128, 0, st, b->dev, do_update, refine > 0);  // two vertices per thread
  return n;
}

// The local steps in the shapes the autotuner chose (elements per thread).
void launch_membrane(vistio_batch* b, cudaStream_t st) {
  if (!b->n_tri_chunks) return;
  if (b->tri_per == 2) launch_pdl(k_tri, b->n_tri_chunks, kTriThreads, 0, st, b->dev);
  else launch_pdl(k_tri1, b->n_tri_chunks, kElemThreads, 0, st, b->dev);
}
void launch_bending(vistio_batch* b, cudaStream_t st) {
  if (!b->n_hinge_chunks) return;
  if (b->hinge_per == 2) launch_pdl(k_hinge2, b->n_hinge_chunks, kElemThreads / 2, 0, st, b->dev);
  else launch_pdl(k_hinge, b->n_hinge_chunks, kElemThreads, 0, st, b->dev);
}

uint32_t launch_plain_iteration(vistio_batch* b, cudaStream_t st, int do_update, uint32_t refine) {
  uint32_t n = 1;
  if (b->n_tri_chunks) { launch_membrane(b, st); ++n; }
  if (b->n_hinge_chunks) { launch_bending(b, st); ++n; }
  launch_pdl(k_gather, b->n_vtx_chunks, kElemThreads, 0, st, b->dev, refine > 0);
  return n + launch_solve(b, st, do_update, refine);
}

vistio_status capture(vistio_batch* b, bool ipc, bool self, cudaGraphExec_t* out, uint32_t* nlaunch) {
  vistio_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  cudaGraph_t g = nullptr;
  uint32_t iters = b->cfg.max_iterations;
  uint32_t small_grid = (b->ninst + 127) / 128;
  CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  launch_pdl(k_predict, b->n_vtx_chunks, kElemThreads, 0, st, b->dev);
  uint32_t L = 2;
  if (!ipc) {
    // Each PD iteration recomputes its residual from x, so a sweep's error is
    // corrected by the next iteration; only the last solve is refined.
    for (uint32_t it = 0; it < iters; ++it) L += launch_plain_iteration(b, st, 1, it + 1 == iters ? b->refine : 0);
  } else {
    for (uint32_t al = 0; al < b->cfg.al_max_iterations; ++al) {
      launch_pdl(k_al_begin, small_grid, 128, 0, st, b->dev, b->ninst);
      if (self) L += launch_self_detect(b->dev, b->self.view(), b->n_vtx_chunks, b->n_tri_chunks, 0, st);
      launch_pdl(k_detect, b->n_vtx_chunks, kElemThreads, 0, st, b->dev, 0);
      for (uint32_t it = 0; it < iters; ++it) {
        // With backtracking (alpha < 1) part of each sweep's error stays in x:
        // every solve is refined.
        L += launch_plain_iteration(b, st, 0, b->refine) + 2;
        if (self) { launch_self_ccd(b->dev, b->self.view(), st); L += self_ccd_launches(b->self.view()); }
        launch_pdl(k_ccd, b->n_vtx_chunks, kElemThreads, 0, st, b->dev);
        launch_pdl(k_ipc_update, b->n_vtx_chunks, kElemThreads, 0, st, b->dev);
      }
      if (self) L += launch_self_detect(b->dev, b->self.view(), b->n_vtx_chunks, b->n_tri_chunks, 1, st);
      launch_pdl(k_detect, b->n_vtx_chunks, kElemThreads, 0, st, b->dev, 1);
      launch_pdl(k_al_end, b->n_vtx_chunks, kElemThreads, 0, st, b->dev);
      launch_pdl(k_al_finish, small_grid, 128, 0, st, b->dev, b->ninst);
      L += 5;
    }
  }
  launch_pdl(k_finalize, b->n_vtx_chunks, kElemThreads, 0, st, b->dev);
  cudaError_t e = cudaStreamEndCapture(st, &g);
  if (e != cudaSuccess) return fail(ctx, VISTIO_ERR_GPU, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(ctx, VISTIO_ERR_GPU, std::string("graph instantiate: ") + cudaGetErrorString(e));
  *nlaunch = L;
  return VISTIO_OK;
}

vistio_status batch_run(vistio_batch* b, float dt, uint32_t nsteps, const vistio_contact_desc* ct) {
  vistio_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  if (!(dt > 0.f) || !std::isfinite(dt)) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "dt must be positive");
  bool ipc = ct != nullptr;
  bool self = ipc && ct->self_collision;
  if (self) {
    if (!b->gacc.p) {
      CU(b->gacc.alloc(b->V, st));
      b->dev.gacc = b->dev_w.gacc = b->gacc.p;
    }
    vistio_status s = ensure_self_contact(b->dev, b->self, b->solvers, b->vbase, b->T, st, &ctx->last_error);
    if (s != VISTIO_OK) return s;
    b->self.vt_on = int32_t(b->self_ccd_dedup);
  }
  StepParams p = make_params(b->cfg, dt, ct);
  CU(cudaMemcpyAsync(b->prm.p, &p, sizeof(p), cudaMemcpyHostToDevice, st));
  cudaGraphExec_t* ge = ipc ? &b->graph_ipc : &b->graph_plain;
  if (ipc && *ge && b->graph_ipc_self != int(self)) { cudaGraphExecDestroy(*ge); *ge = nullptr; }
  if (!*ge) {
    vistio_status s = capture(b, ipc, self, ge, ipc ? &b->launches_ipc : &b->launches_plain);
    if (s != VISTIO_OK) return s;
    if (ipc) b->graph_ipc_self = int(self);
  }
  for (uint32_t k = 0; k < nsteps; ++k) CU(cudaGraphLaunch(*ge, st));
  return VISTIO_OK;
}

vistio_status ensure_own(vistio_solver* s) {
  if (s->own) return VISTIO_OK;
  auto* b = new vistio_batch();
  vistio_solver* arr[1] = {s};
  vistio_status r = pack_batch(s->ctx, arr, 1, b);
  if (r != VISTIO_OK) { delete b; return r; }
  s->own = b;
  return VISTIO_OK;
}

vistio_status read_result(vistio_batch* b, uint32_t k, vistio_step_result* res, bool ipc, double wall) {
  vistio_ctx* ctx = b->ctx;
  InstRed R;
  uint32_t status = 0;
  CU(cudaMemcpyAsync(&R, b->red.p + k, sizeof(R), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(&status, b->status.p, sizeof(status), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  double resid = R.norm_sq > 1e-12 ? std::sqrt(R.diff_sq / R.norm_sq) : std::sqrt(R.diff_sq);
  if (res) {
    std::memset(res, 0, sizeof(*res));
    res->iterations = R.iters;
    res->final_residual = resid;
    res->converged = (ipc && R.al_done) || resid < b->cfg.tolerance;
    res->wall_time = wall;
    res->al_iterations = R.al_iters;
    res->active_contacts = R.last_active;
    res->last_alpha = ipc ? R.alpha : 1.f;
    res->status = (status & 4u) ? VISTIO_ERR_TIMEOUT : (status & 2u) ? VISTIO_ERR_CAPACITY
                : status ? VISTIO_ERR_SOLVER_DIVERGENCE : VISTIO_OK;
  }
  if (status & 4u) return fail(ctx, VISTIO_ERR_TIMEOUT, "a bounded device wait gave up");
  if (status & 2u) return fail(ctx, VISTIO_ERR_CAPACITY, "self-contact candidate pairs exceeded the buffer");
  if (status) return fail(ctx, VISTIO_ERR_SOLVER_DIVERGENCE, "non-finite positions in the global solve");
  return VISTIO_OK;
}

vistio_status init_common(vistio_ctx* ctx, const vistio_mesh_desc* mesh, const vistio_solver_config* cfg,
                          const SetupParams& prm, const uint8_t* pinned, vistio_solver** out) {
  if (!ctx || !mesh || !cfg || !out) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null argument");
  if (!mesh->pos_x || !mesh->pos_y || !mesh->pos_z || !mesh->indices)
    return fail(ctx, VISTIO_ERR_INVALID_MESH, "null mesh array");
  if (cfg->max_iterations == 0) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "max_iterations must be > 0");
  if (cfg->refinement_sweeps > 2) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "refinement_sweeps must be 0, 1 or 2");
  std::vector<uint8_t> pin(mesh->vertex_count, 0);
  if (pinned) std::memcpy(pin.data(), pinned, mesh->vertex_count);
  auto s = std::make_unique<vistio_solver>();
  s->ctx = ctx;
  s->cfg = *cfg;
  int st = 0;
  SetupParams sp = prm;
  sp.numeric = cfg->host_factorization != 0;
  std::string err = build_instance(mesh->vertex_count, mesh->pos_x, mesh->pos_y, mesh->pos_z, mesh->triangle_count,
                                   mesh->indices, pin.data(), sp, s->setup, &st);
  if (!err.empty()) {
    vistio_status code = st == 1 ? VISTIO_ERR_INVALID_MESH : st == 11 ? VISTIO_ERR_NOT_SPD : VISTIO_ERR_INVALID_CONFIG;
    return fail(ctx, code, err);
  }
  s->host_pos = s->setup.rest;
  s->host_vel.assign(s->host_pos.size(), 0.f);
  *out = s.release();
  return VISTIO_OK;
}

}  // namespace

// =================================================================== C ABI
extern "C" {

const char* vistio_status_string(vistio_status s) {
  switch (s) {
    case VISTIO_OK: return "ok";
    case VISTIO_ERR_INVALID_MESH: return "invalid mesh";
    case VISTIO_ERR_INVALID_MATERIAL: return "invalid material parameter";
    case VISTIO_ERR_INVALID_CONFIG: return "invalid configuration";
    case VISTIO_ERR_IO: return "i/o error";
    case VISTIO_ERR_SERIALIZATION: return "serialization error";
    case VISTIO_ERR_GPU: return "gpu error";
    case VISTIO_ERR_SOLVER_DIVERGENCE: return "solver divergence";
    case VISTIO_ERR_INVARIANT: return "invariant violation";
    case VISTIO_ERR_TIMEOUT: return "timeout";
    case VISTIO_ERR_OOM: return "out of device memory";
    case VISTIO_ERR_NOT_SPD: return "matrix not positive definite";
    case VISTIO_ERR_CAPACITY: return "capacity exceeded";
  }
  return "unknown";
}

const char* vistio_last_error(const vistio_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : g_tls_error.c_str();
}

vistio_status vistio_ctx_create(int32_t device, vistio_ctx** out) {
  vistio_ctx* ctx = nullptr;
  if (!out) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null out");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(nullptr, VISTIO_ERR_GPU, "no CUDA device available");
  if (device < 0 || device >= n) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "device index out of range");
  auto c = std::make_unique<vistio_ctx>();
  c->device = device;
  ctx = c.get();
  CU(cudaSetDevice(device));
  CU(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  {  // keep freed batch memory in this process's pool for reuse instead of trimming it at each synchronisation
    cudaMemPool_t pool;
    CU(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    CU(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  CU(cudaFuncSetAttribute(k_level<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolveSmem));
  CU(cudaFuncSetAttribute(k_level<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolveSmem));
  CU(cudaFuncSetAttribute(k_subtree<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolveSmem));
  CU(cudaFuncSetAttribute(k_subtree<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolveSmem));
  CU(cudaFuncSetAttribute(k_sweep<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolveSmem));
  CU(cudaFuncSetAttribute(k_sweep<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSolveSmem));
  CU(cudaFuncSetAttribute(k_sweep<2, kWideWarps>, cudaFuncAttributeMaxDynamicSharedMemorySize, kWideSmem));
  CU(cudaFuncSetAttribute(k_gsweep<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
  CU(cudaFuncSetAttribute(k_gsweep<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
  {
    int per_sm = 0, sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<5>, kSolveThreads, kSolveSmem));
    c->sweep_blocks[0] = uint32_t(std::max(1, per_sm) * std::max(1, sms));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<4>, kSolveThreads, kSolveSmem));
    c->sweep_blocks[1] = uint32_t(std::max(1, per_sm) * std::max(1, sms));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<2, kWideWarps>, 32 * kWideWarps, kWideSmem));
    c->sweep_blocks[2] = uint32_t(std::max(1, per_sm) * std::max(1, sms));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gsweep<0>, kGThreads, kGSmem));
    c->gsweep_blocks = uint32_t(std::max(1, per_sm) * std::max(1, sms));
  }
  *out = c.release();
  return VISTIO_OK;
}

vistio_status vistio_ctx_destroy(vistio_ctx* ctx) {
  if (!ctx) return VISTIO_OK;
  bool now;
  {
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->closed = true;
    now = ctx->refs == 0;
  }
  if (now) ctx_free(ctx);  // else the last batch on it frees it
  return VISTIO_OK;
}

vistio_status vistio_sync(vistio_ctx* ctx) {
  if (!ctx) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null context");
  CU(cudaStreamSynchronize(ctx->stream));
  return VISTIO_OK;
}

vistio_status vistio_solver_init(vistio_ctx* ctx, const vistio_mesh_desc* mesh, const vistio_solver_config* cfg,
                                 const uint8_t* pinned, vistio_solver** out) {
  if (!cfg) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null config");
  SetupParams p;  // pd_solver.rs:228-246
  p.model = MODEL_ARAP;
  p.bending = BEND_DIHEDRAL;
  p.stiffness = cfg->stretch_weight * 1000.0f;
  p.bend_stiffness = cfg->bending_weight * 100.0f;
  p.density_gsm = 200.0f;
  p.matrix_dt = 1.0f / 60.0f;
  return init_common(ctx, mesh, cfg, p, pinned, out);
}

vistio_status vistio_solver_init_with_material(vistio_ctx* ctx, const vistio_mesh_desc* mesh,
                                               const vistio_solver_config* cfg, const vistio_material_desc* m,
                                               const vistio_model_desc* model, int32_t bending_kind,
                                               const uint8_t* pinned, vistio_solver** out) {
  if (!m || !model) return fail(ctx, VISTIO_ERR_INVALID_MATERIAL, "null material or model");
  if (!(m->density > 0.f) || !std::isfinite(m->density))
    return fail(ctx, VISTIO_ERR_INVALID_MATERIAL, "density must be positive");
  if (model->kind < 0 || model->kind > 4) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "unknown model kind");
  if (bending_kind < 0 || bending_kind > 3) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "unknown bending kind");
  SetupParams p;  // pd_solver.rs:115-132, element.rs:106, bending.rs:160, discrete_shells.rs:206
  p.model = model->kind;
  p.bending = bending_kind;
  p.stiffness = ((m->stretch_stiffness_warp + m->stretch_stiffness_weft) / 2.0f) * 10.0f;
  p.bend_stiffness = ((m->bending_stiffness_warp + m->bending_stiffness_weft) / 2.0f) * 100.0f;
  p.density_gsm = m->density;
  p.warp = model->warp_stiffness;
  p.weft = model->weft_stiffness;
  p.bend_warp = m->bending_stiffness_warp;
  p.bend_weft = m->bending_stiffness_weft;
  p.matrix_dt = 1.0f / 60.0f;
  return init_common(ctx, mesh, cfg, p, pinned, out);
}

vistio_status vistio_solver_init_explicit(vistio_ctx* ctx, const vistio_mesh_desc* mesh, const vistio_solver_config* cfg,
                                          const vistio_setup_desc* sd, const uint8_t* pinned, vistio_solver** out) {
  if (!sd) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null setup");
  if (sd->model < 0 || sd->model > 4 || sd->bending < 0 || sd->bending > 3)
    return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "unknown model or bending kind");
  if (!(sd->density_gsm > 0.f)) return fail(ctx, VISTIO_ERR_INVALID_MATERIAL, "density must be positive");
  SetupParams p;
  p.model = sd->model; p.bending = sd->bending; p.stiffness = sd->stiffness; p.bend_stiffness = sd->bend_stiffness;
  p.density_gsm = sd->density_gsm; p.warp = sd->warp_stiffness; p.weft = sd->weft_stiffness;
  p.bend_warp = sd->bend_warp; p.bend_weft = sd->bend_weft; p.matrix_dt = sd->matrix_dt;
  return init_common(ctx, mesh, cfg, p, pinned, out);
}

vistio_status vistio_solver_destroy(vistio_solver* s) {
  if (!s) return VISTIO_OK;
  delete s->own;
  delete s;
  return VISTIO_OK;
}

vistio_status vistio_solver_clone(vistio_solver* s, vistio_ctx* ctx, vistio_solver** out) {
  if (!s || !ctx || !out) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null argument");
  auto c = std::make_unique<vistio_solver>();
  c->ctx = ctx;
  c->cfg = s->cfg;
  c->setup = s->setup;
  c->has_ground = s->has_ground;
  c->ground_h = s->ground_h;
  if (s->own) {  // the source has stepped: copy its current device state
    const uint32_t n = s->setup.nv;
    std::vector<float> a(6 * size_t(n));
    vistio_status r = vistio_solver_get_state(s, a.data(), a.data() + n, a.data() + 2 * n, a.data() + 3 * n,
                                              a.data() + 4 * n, a.data() + 5 * n);
    if (r != VISTIO_OK) return r;
    c->host_pos.resize(3 * size_t(n));
    c->host_vel.resize(3 * size_t(n));
    for (uint32_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) {
        c->host_pos[3 * i + k] = a[size_t(k) * n + i];
        c->host_vel[3 * i + k] = a[size_t(3 + k) * n + i];
      }
  } else {
    c->host_pos = s->host_pos;
    c->host_vel = s->host_vel;
  }
  *out = c.release();
  return VISTIO_OK;
}

vistio_status vistio_solver_device_bytes(const vistio_solver* s, int32_t self_contact, uint64_t* bytes) {
  if (!s || !bytes) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  *bytes = instance_device_bytes(s->setup, s->cfg.refinement_sweeps > 0, self_contact != 0);
  return VISTIO_OK;
}

const char* vistio_solver_name(const vistio_solver*) { return "ProjectiveDynamics"; }

vistio_status vistio_solver_info(const vistio_solver* s, uint32_t* nv, uint32_t* nt, uint32_t* nh, uint64_t* nnz_a,
                                 uint64_t* nnz_l, uint32_t* nsn, uint32_t* nlv) {
  if (!s) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null solver");
  if (nv) *nv = s->setup.nv;
  if (nt) *nt = s->setup.nt;
  if (nh) *nh = s->setup.nh;
  if (nnz_a) *nnz_a = s->setup.A_col.size();
  if (nnz_l) *nnz_l = s->setup.factor.nnz_L;
  if (nsn) *nsn = uint32_t(s->setup.factor.sn.size());
  if (nlv) *nlv = s->setup.factor.nlevels;
  return VISTIO_OK;
}

vistio_status vistio_solver_lumped_masses(const vistio_solver* s, float* out) {
  if (!s || !out) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  std::memcpy(out, s->setup.mass.data(), s->setup.nv * sizeof(float));
  return VISTIO_OK;
}

vistio_status vistio_solver_set_ground(vistio_solver* s, int32_t has, float h) {
  if (!s) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null solver");
  vistio_ctx* ctx = s->ctx;
  s->has_ground = has;
  s->ground_h = h;
  if (s->own) {
    InstDev d;
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaMemcpy(&d, s->own->inst.p, sizeof(d), cudaMemcpyDeviceToHost));
    d.has_ground = has;
    d.ground_h = h;
    CU(cudaMemcpy(s->own->inst.p, &d, sizeof(d), cudaMemcpyHostToDevice));
  }
  return VISTIO_OK;
}

vistio_status vistio_batch_set_state(vistio_batch* b, uint32_t k, const float* px, const float* py, const float* pz,
                                     const float* vx, const float* vy, const float* vz) {
  if (!b || k >= b->ninst) return fail(b ? b->ctx : nullptr, VISTIO_ERR_INVALID_CONFIG, "bad batch index");
  vistio_ctx* ctx = b->ctx;
  uint32_t nv = b->solvers[k]->setup.nv;
  std::vector<float4> p(nv), v(nv);
  CU(cudaStreamSynchronize(ctx->stream));
  CU(cudaMemcpy(p.data(), b->pos.p + b->vbase[k], nv * sizeof(float4), cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(v.data(), b->vel.p + b->vbase[k], nv * sizeof(float4), cudaMemcpyDeviceToHost));
  for (uint32_t i = 0; i < nv; ++i) {
    if (px) p[i].x = px[i];
    if (py) p[i].y = py[i];
    if (pz) p[i].z = pz[i];
    if (vx) v[i].x = vx[i];
    if (vy) v[i].y = vy[i];
    if (vz) v[i].z = vz[i];
  }
  CU(cudaMemcpyAsync(b->pos.p + b->vbase[k], p.data(), nv * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(b->vel.p + b->vbase[k], v.data(), nv * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return VISTIO_OK;
}

vistio_status vistio_batch_get_state(vistio_batch* b, uint32_t k, float* px, float* py, float* pz, float* vx,
                                     float* vy, float* vz) {
  if (!b || k >= b->ninst) return fail(b ? b->ctx : nullptr, VISTIO_ERR_INVALID_CONFIG, "bad batch index");
  vistio_ctx* ctx = b->ctx;
  uint32_t nv = b->solvers[k]->setup.nv;
  std::vector<float4> p(nv), v(nv);
  CU(cudaMemcpyAsync(p.data(), b->pos.p + b->vbase[k], nv * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaMemcpyAsync(v.data(), b->vel.p + b->vbase[k], nv * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  uint32_t status = 0;
  CU(cudaMemcpy(&status, b->status.p, sizeof(status), cudaMemcpyDeviceToHost));
  for (uint32_t i = 0; i < nv; ++i) {
    if (px) px[i] = p[i].x;
    if (py) py[i] = p[i].y;
    if (pz) pz[i] = p[i].z;
    if (vx) vx[i] = v[i].x;
    if (vy) vy[i] = v[i].y;
    if (vz) vz[i] = v[i].z;
  }
  if (status) return fail(ctx, VISTIO_ERR_SOLVER_DIVERGENCE, "non-finite positions in the global solve");
  return VISTIO_OK;
}

vistio_status vistio_solver_set_state(vistio_solver* s, const float* px, const float* py, const float* pz,
                                      const float* vx, const float* vy, const float* vz) {
  if (!s) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null solver");
  for (uint32_t i = 0; i < s->setup.nv; ++i) {
    if (px) s->host_pos[3 * i] = px[i];
    if (py) s->host_pos[3 * i + 1] = py[i];
    if (pz) s->host_pos[3 * i + 2] = pz[i];
    if (vx) s->host_vel[3 * i] = vx[i];
    if (vy) s->host_vel[3 * i + 1] = vy[i];
    if (vz) s->host_vel[3 * i + 2] = vz[i];
  }
  if (s->own) return vistio_batch_set_state(s->own, 0, px, py, pz, vx, vy, vz);
  return VISTIO_OK;
}

vistio_status vistio_solver_get_state(vistio_solver* s, float* px, float* py, float* pz, float* vx, float* vy,
                                      float* vz) {
  if (!s) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null solver");
  if (s->own) return vistio_batch_get_state(s->own, 0, px, py, pz, vx, vy, vz);
  for (uint32_t i = 0; i < s->setup.nv; ++i) {
    if (px) px[i] = s->host_pos[3 * i];
    if (py) py[i] = s->host_pos[3 * i + 1];
    if (pz) pz[i] = s->host_pos[3 * i + 2];
    if (vx) vx[i] = s->host_vel[3 * i];
    if (vy) vy[i] = s->host_vel[3 * i + 1];
    if (vz) vz[i] = s->host_vel[3 * i + 2];
  }
  return VISTIO_OK;
}

vistio_status vistio_solver_contact_force(vistio_solver* s, float* out) {
  if (!s || !out) return fail(s ? s->ctx : nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  const uint32_t nv = s->setup.nv;
  if (!s->own) {
    std::fill(out, out + nv, 0.f);
    return VISTIO_OK;
  }
  vistio_batch* b = s->own;
  vistio_ctx* ctx = b->ctx;
  std::vector<float4> g(nv);
  CU(cudaMemcpyAsync(g.data(), b->grad.p + b->vbase[0], nv * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  for (uint32_t i = 0; i < nv; ++i) out[i] = std::sqrt(g[i].x * g[i].x + g[i].y * g[i].y + g[i].z * g[i].z);
  return VISTIO_OK;
}

vistio_status vistio_step(vistio_solver* s, float dt, vistio_step_result* res) {
  if (!s) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "Solver not initialized. Call init() first.");
  auto t0 = std::chrono::steady_clock::now();
  vistio_status r = ensure_own(s);
  if (r != VISTIO_OK) return r;
  r = batch_run(s->own, dt, 1, nullptr);
  if (r != VISTIO_OK) return r;
  r = read_result(s->own, 0, res, false, 0.0);
  if (res) res->wall_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

vistio_status vistio_step_with_ipc(vistio_solver* s, float dt, const vistio_contact_desc* contact,
                                   vistio_step_result* res) {
  if (!s) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "Solver not initialized. Call init() first.");
  if (!contact) return fail(s->ctx, VISTIO_ERR_INVALID_CONFIG, "null contact description");
  auto t0 = std::chrono::steady_clock::now();
  vistio_status r = ensure_own(s);
  if (r != VISTIO_OK) return r;
  r = batch_run(s->own, dt, 1, contact);
  if (r != VISTIO_OK) return r;
  r = read_result(s->own, 0, res, true, 0.0);
  if (res) res->wall_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

vistio_status vistio_batch_create(vistio_ctx* ctx, vistio_solver* const* solvers, uint32_t n, vistio_batch** out) {
  if (!ctx || !solvers || n == 0 || !out) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "empty batch");
  for (uint32_t k = 0; k < n; ++k)
    if (!solvers[k]) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null solver in batch");
  for (uint32_t k = 1; k < n; ++k)
    if (solvers[k]->cfg.max_iterations != solvers[0]->cfg.max_iterations ||
        solvers[k]->cfg.al_max_iterations != solvers[0]->cfg.al_max_iterations ||
        solvers[k]->cfg.refinement_sweeps != solvers[0]->cfg.refinement_sweeps)
      return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "instances of a batch must share iteration and refinement counts");
  auto* b = new vistio_batch();
  vistio_status r = pack_batch(ctx, solvers, n, b);
  if (r != VISTIO_OK) { delete b; return r; }
  *out = b;
  return VISTIO_OK;
}

vistio_status vistio_batch_destroy(vistio_batch* b) {
  if (!b) return VISTIO_OK;
  cudaStreamSynchronize(b->ctx->stream);
  delete b;
  return VISTIO_OK;
}

vistio_status vistio_batch_step(vistio_batch* b, float dt, uint32_t nsteps, const vistio_contact_desc* contact) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  return batch_run(b, dt, nsteps, contact);
}

vistio_status vistio_batch_resolve_contacts(vistio_batch* b, const vistio_contact_desc* ct,
                                            vistio_collider_results* res) {
  if (!b || !ct) return fail(b ? b->ctx : nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  vistio_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  CU(cudaSetDevice(ctx->device));
  ColliderDev C{};
  C.has_ground = ct->has_ground != 0;
  C.ground_h = ct->ground_height;
  C.has_sphere = ct->has_sphere != 0;
  for (int k = 0; k < 3; ++k) C.sc[k] = ct->sphere_center[k];
  C.sr = ct->sphere_radius;
  C.has_cyl = ct->has_cylinder != 0;
  C.cyl[0] = ct->cylinder_center_x; C.cyl[1] = ct->cylinder_center_z;
  C.cyl[2] = ct->cylinder_top_y; C.cyl[3] = ct->cylinder_radius;
  C.has_box = ct->has_box != 0;
  for (int k = 0; k < 3; ++k) { C.lo[k] = ct->box_min[k]; C.hi[k] = ct->box_max[k]; }
  if (!b->res_cnt.p) {
    CU(b->res_cnt.alloc(8 * size_t(b->ninst), st));
    CU(b->res_force.alloc(4 * size_t(b->ninst), st));
  }
  CU(cudaMemsetAsync(b->res_cnt.p, 0, 32 * size_t(b->ninst), st));
  CU(cudaMemsetAsync(b->res_force.p, 0, 32 * size_t(b->ninst), st));
  if (b->n_vtx_chunks) k_resolve<<<b->n_vtx_chunks, 256, 0, st>>>(b->dev, C, b->res_cnt.p, b->res_force.p);
  CU(cudaGetLastError());
  if (!res) return VISTIO_OK;
  std::vector<uint32_t> cnt(8 * size_t(b->ninst));
  std::vector<double> frc(4 * size_t(b->ninst));
  CU(cudaMemcpyAsync(cnt.data(), b->res_cnt.p, cnt.size() * 4, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(frc.data(), b->res_force.p, frc.size() * 8, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < b->ninst; ++i) {
    vistio_contact_result* r[4] = {&res[i].ground, &res[i].sphere, &res[i].cylinder, &res[i].box};
    for (int c = 0; c < 4; ++c) {
      r[c]->resolved_count = cnt[8 * i + 2 * c];
      std::memcpy(&r[c]->max_residual_penetration, &cnt[8 * i + 2 * c + 1], 4);
      r[c]->total_force_magnitude = float(frc[4 * i + c]);
    }
  }
  return VISTIO_OK;
}

vistio_status vistio_resolve_contacts(vistio_solver* s, const vistio_contact_desc* contact,
                                      vistio_collider_results* res) {
  if (!s) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "Solver not initialized. Call init() first.");
  if (!contact) return fail(s->ctx, VISTIO_ERR_INVALID_CONFIG, "null contact description");
  vistio_status r = ensure_own(s);
  if (r != VISTIO_OK) return r;
  r = vistio_batch_resolve_contacts(s->own, contact, res);
  if (r == VISTIO_OK && !res) {
    vistio_ctx* ctx = s->own->ctx;
    CU(cudaStreamSynchronize(ctx->stream));
  }
  return r;
}

// Whole-batch position copies: one contiguous copy of the interleaved xyz
// through a device staging buffer, packed to / from the float4 rows by a
// kernel (a strided 12-byte-row copy runs at a small fraction of the link).
vistio_status vistio_batch_upload_positions(vistio_batch* b, const float* xyz) {
  if (!b || !xyz) return fail(b ? b->ctx : nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  vistio_ctx* ctx = b->ctx;
  if (!b->xyz_stage.p) CU(b->xyz_stage.alloc(3 * b->V, ctx->stream));
  const uint32_t grid = uint32_t(std::min<uint64_t>((b->V + 255) / 256, 148 * 16));
  CU(cudaMemcpyAsync(b->xyz_stage.p, xyz, 12 * b->V, cudaMemcpyHostToDevice, ctx->stream));
  k_unpack_pos<<<grid, 256, 0, ctx->stream>>>(b->pos.p, b->xyz_stage.p, b->V);
  CU(cudaGetLastError());
  return VISTIO_OK;
}

vistio_status vistio_batch_download_positions(vistio_batch* b, float* xyz) {
  if (!b || !xyz) return fail(b ? b->ctx : nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  vistio_ctx* ctx = b->ctx;
  if (!b->xyz_stage.p) CU(b->xyz_stage.alloc(3 * b->V, ctx->stream));
  const uint32_t grid = uint32_t(std::min<uint64_t>((b->V + 255) / 256, 148 * 16));
  k_pack_pos<<<grid, 256, 0, ctx->stream>>>(b->xyz_stage.p, b->pos.p, b->V);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(xyz, b->xyz_stage.p, 12 * b->V, cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return VISTIO_OK;
}

vistio_status vistio_batch_info(const vistio_batch* b, uint32_t* ni, uint64_t* tv, uint64_t* tt, uint64_t* th,
                                uint64_t* fb, uint64_t* db) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  if (ni) *ni = b->ninst;
  if (tv) *tv = b->V;
  if (tt) *tt = b->T;
  if (th) *th = b->H;
  if (fb) *fb = b->factor_bytes;
  if (db) *db = b->device_bytes;
  return VISTIO_OK;
}

vistio_status vistio_batch_factor_stats(const vistio_batch* b, uint32_t* launches, float* device_ms) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  if (launches) *launches = b->factor_launches;
  if (device_ms) *device_ms = b->factor_ms;
  return VISTIO_OK;
}

vistio_status vistio_batch_launches_per_step(const vistio_batch* b, uint32_t* launches) {
  if (!b || !launches) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  *launches = b->graph_ipc ? b->launches_ipc : b->launches_plain;
  return VISTIO_OK;
}

void* vistio_batch_stream(vistio_batch* b) { return b ? (void*)b->ctx->stream : nullptr; }

// Sweep autotuner. The candidates are the two sweep kinds (one launch per
// level; dependency-driven) times the warp-item limits of s (s + m): 0 (every
// top supernode for a block) ... 2^30 (every one of at most kWarpVec columns
// for a warp).
static const uint32_t kTuneLimits[7] = {0u, 1024u, 2048u, 4096u, 6144u, 12288u, 1u << 30};
// Group limits of the grouped kind's candidates: 0 takes the bottom subtrees only.
static const uint32_t kGroupTuneLimits[7] = {0u, 64u, 128u, 256u, 512u, 1024u, 6144u};

namespace {
vistio_status drop_graphs(vistio_batch* b) {  // captured steps bake the schedule into their launches
  if (b->graph_plain) { cudaGraphExecDestroy(b->graph_plain); b->graph_plain = nullptr; }
  if (b->graph_ipc) { cudaGraphExecDestroy(b->graph_ipc); b->graph_ipc = nullptr; }
  return VISTIO_OK;
}
}  // namespace

vistio_status vistio_batch_tune(vistio_batch* b, uint32_t* chosen_limit, float* candidate_ms) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  vistio_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  StepParams p{};
  p.dt = 1.f / 60.f;
  CU(cudaMemcpyAsync(b->prm.p, &p, sizeof(p), cudaMemcpyHostToDevice, st));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  float best = 0.f, best1 = 0.f;
  uint32_t best_limit = b->warp_limit, best_mode = b->sweep_mode, best_glimit = b->group_limit;
  uint32_t best1_limit = kWarpItemLimit;  // the fastest limit of kind 1: kind 2 runs its rest at it
  b->sweep_occ = 4;
  b->unit_items = kUnitItems;
  for (int c = 0; c < 21; ++c) {
    const uint32_t glimit = c >= 14 ? kGroupTuneLimits[c - 14] : b->group_limit;
    if (c >= 14 && (!b->n_groups || glimit > best1_limit)) {  // no groups, or a limit kind 1's rest could not match
      if (candidate_ms) candidate_ms[c] = -1.f;
      continue;
    }
    b->sweep_mode = uint32_t(c / 7);
    const uint32_t limit = c >= 14 ? best1_limit : kTuneLimits[c % 7];
    if (c >= 14) CU(schedule_groups(b, glimit, st));
    std::vector<uint32_t> items = schedule_levels(b, limit);
    CU(upload_schedule(b, items, st));
    CU(cudaMemsetAsync(b->Y.p, 0, b->V * sizeof(float4), st));
    launch_sweeps(b, b->dev, st);  // warm-up
    CU(cudaEventRecord(e0, st));
    for (int r = 0; r < 3; ++r) launch_sweeps(b, b->dev, st);
    CU(cudaEventRecord(e1, st));
    CU(cudaEventSynchronize(e1));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    ms /= 3.f;
    if (candidate_ms) candidate_ms[c] = ms;
    if (c >= 7 && c < 14 && (c == 7 || ms < best1)) { best1 = ms; best1_limit = limit; }
    if (c == 0 || ms < best) { best = ms; best_limit = limit; best_mode = b->sweep_mode; best_glimit = glimit; }
  }
  uint32_t status = 0;
  CU(cudaMemcpyAsync(&status, b->status.p, sizeof(status), cudaMemcpyDeviceToHost, st));
  b->sweep_mode = best_mode;
  if (b->n_groups) CU(schedule_groups(b, best_glimit, st));
  std::vector<uint32_t> items = schedule_levels(b, best_limit);
  CU(upload_schedule(b, items, st));
  if (best_mode != 0) {
    // the chosen schedule with k_sweep's three compiled forms (five and four
    // eight-warp blocks per SM, two sixteen-warp blocks with units of twice
    // the items): the fastest is kept
    float occ_ms[3] = {0.f, 0.f, 0.f};
    for (int v = 0; v < 3; ++v) {
      b->sweep_occ = v == 0 ? 5u : v == 1 ? 4u : 2u;
      if (v == 2) {
        b->unit_items = 2 * kUnitItems;
        std::vector<uint32_t> wide = schedule_levels(b, best_limit);
        CU(upload_schedule(b, wide, st));
      }
      launch_sweeps(b, b->dev, st);  // warm-up
      CU(cudaEventRecord(e0, st));
      for (int r = 0; r < 3; ++r) launch_sweeps(b, b->dev, st);
      CU(cudaEventRecord(e1, st));
      CU(cudaEventSynchronize(e1));
      CU(cudaEventElapsedTime(&occ_ms[v], e0, e1));
      occ_ms[v] /= 3.f;
    }
    int bv = 0;
    for (int v = 1; v < 3; ++v)
      if (occ_ms[v] < occ_ms[bv]) bv = v;
    b->sweep_occ = bv == 0 ? 5u : bv == 1 ? 4u : 2u;
    if (bv != 2) {  // back to eight-warp units
      b->unit_items = kUnitItems;
      std::vector<uint32_t> narrow = schedule_levels(b, best_limit);
      CU(upload_schedule(b, narrow, st));
    }
    best = occ_ms[bv];
    for (int v = 0; v < 3; ++v) b->occ_ms[v] = occ_ms[v];
  } else {
    b->sweep_occ = 4;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU(cudaStreamSynchronize(st));
  if (status & 4u) return fail(ctx, VISTIO_ERR_TIMEOUT, "a bounded wait of the sweeps gave up while tuning");
  b->tuned_ms = best;
  drop_graphs(b);
  if (chosen_limit) *chosen_limit = best_limit;
  return VISTIO_OK;
}

vistio_status vistio_batch_set_group_limit(vistio_batch* b, uint32_t limit) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  vistio_ctx* ctx = b->ctx;
  if (!b->n_groups) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "the batch has no garment groups");
  CU(schedule_groups(b, std::min(limit, kWarpItemLimit), ctx->stream));
  std::vector<uint32_t> items = schedule_levels(b, b->warp_limit);
  CU(upload_schedule(b, items, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return drop_graphs(b);
}

vistio_status vistio_batch_get_group_limit(const vistio_batch* b, uint32_t* limit) {
  if (!b || !limit) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  *limit = b->group_limit;
  return VISTIO_OK;
}

vistio_status vistio_batch_tune_local(vistio_batch* b, uint32_t* tri_per_thread, uint32_t* hinge_per_thread,
                                      float* candidate_ms) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  vistio_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  StepParams p{};
  p.dt = 1.f / 60.f;
  CU(cudaMemcpyAsync(b->prm.p, &p, sizeof(p), cudaMemcpyHostToDevice, st));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  float ms[4] = {0.f, 0.f, 0.f, 0.f};
  for (int c = 0; c < 4; ++c) {
    const uint32_t per = 1u + uint32_t(c & 1);
    if (c < 2) b->tri_per = per; else b->hinge_per = per;
    for (int r = 0; r < 6; ++r) {  // one warm-up, five timed
      if (r == 1) CU(cudaEventRecord(e0, st));
      if (c < 2) launch_membrane(b, st); else launch_bending(b, st);
    }
    CU(cudaEventRecord(e1, st));
    CU(cudaEventSynchronize(e1));
    CU(cudaEventElapsedTime(&ms[c], e0, e1));
    ms[c] /= 5.f;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU(cudaGetLastError());
  b->tri_per = ms[1] <= ms[0] ? 2u : 1u;
  b->hinge_per = ms[3] < ms[2] ? 2u : 1u;
  if (tri_per_thread) *tri_per_thread = b->tri_per;
  if (hinge_per_thread) *hinge_per_thread = b->hinge_per;
  if (candidate_ms) std::memcpy(candidate_ms, ms, sizeof(ms));
  return drop_graphs(b);
}

vistio_status vistio_batch_set_local_shape(vistio_batch* b, uint32_t tri_per_thread, uint32_t hinge_per_thread) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  if (tri_per_thread < 1 || tri_per_thread > 2 || hinge_per_thread < 1 || hinge_per_thread > 2)
    return fail(b->ctx, VISTIO_ERR_INVALID_CONFIG, "elements per thread must be 1 or 2");
  b->tri_per = tri_per_thread;
  b->hinge_per = hinge_per_thread;
  return drop_graphs(b);
}

vistio_status vistio_batch_set_self_ccd_dedup(vistio_batch* b, uint32_t on) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  if (on > 1) return fail(b->ctx, VISTIO_ERR_INVALID_CONFIG, "on must be 0 or 1");
  b->self_ccd_dedup = on;
  b->self.vt_on = int32_t(on);
  return drop_graphs(b);
}

vistio_status vistio_batch_set_warp_limit(vistio_batch* b, uint32_t limit) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  vistio_ctx* ctx = b->ctx;
  std::vector<uint32_t> items = schedule_levels(b, limit);
  CU(upload_schedule(b, items, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return drop_graphs(b);
}

vistio_status vistio_batch_set_sweep_mode(vistio_batch* b, uint32_t mode) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  if (mode > 2) return fail(b->ctx, VISTIO_ERR_INVALID_CONFIG, "sweep mode must be 0, 1 or 2");
  if (mode == 2 && !b->n_groups)
    return fail(b->ctx, VISTIO_ERR_INVALID_CONFIG, "sweep mode 2 needs garment groups (none in this batch)");
  vistio_ctx* ctx = b->ctx;
  b->sweep_mode = mode;
  std::vector<uint32_t> items = schedule_levels(b, b->warp_limit);  // mode 2 leaves the groups' supernodes out
  CU(upload_schedule(b, items, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return drop_graphs(b);
}

vistio_status vistio_batch_set_sweep_blocks(vistio_batch* b, uint32_t blocks_per_sm) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  if (blocks_per_sm != 2 && blocks_per_sm != 4 && blocks_per_sm != 5)
    return fail(b->ctx, VISTIO_ERR_INVALID_CONFIG, "k_sweep is compiled for 5 or 4 eight-warp blocks or 2 sixteen-warp blocks per SM");
  vistio_ctx* ctx = b->ctx;
  b->sweep_occ = blocks_per_sm;
  const uint32_t ui = blocks_per_sm == 2 ? 2 * kUnitItems : kUnitItems;
  if (ui != b->unit_items) {
    b->unit_items = ui;
    std::vector<uint32_t> items = schedule_levels(b, b->warp_limit);
    CU(upload_schedule(b, items, b->ctx->stream));
    CU(cudaStreamSynchronize(b->ctx->stream));
  }
  return drop_graphs(b);
}

vistio_status vistio_batch_get_sweep_blocks(const vistio_batch* b, uint32_t* blocks_per_sm, float* tuned_ms) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  if (blocks_per_sm) *blocks_per_sm = b->sweep_occ;
  if (tuned_ms) {
    tuned_ms[0] = b->occ_ms[0];
    tuned_ms[1] = b->occ_ms[1];
    tuned_ms[2] = b->occ_ms[2];
  }
  return VISTIO_OK;
}

vistio_status vistio_batch_get_sweep_mode(const vistio_batch* b, uint32_t* mode, uint32_t* warp_limit) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  if (mode) *mode = b->sweep_mode;
  if (warp_limit) *warp_limit = b->warp_limit;
  return VISTIO_OK;
}

vistio_status vistio_batch_launch_phase(vistio_batch* b, int32_t phase) {
  if (!b) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null batch");
  vistio_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  switch (phase) {
    case 0: k_predict<<<b->n_vtx_chunks, kElemThreads, 0, st>>>(b->dev); break;
    case 1: launch_membrane(b, st); break;
    case 2: launch_bending(b, st); break;
    case 3: k_gather<<<b->n_vtx_chunks, kElemThreads, 0, st>>>(b->dev, b->refine > 0); break;
    case 4: launch_solve(b, st, 0, 0); break;
    case 5: k_finalize<<<b->n_vtx_chunks, kElemThreads, 0, st>>>(b->dev); break;
    case 6:
      if (!b->refine) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "the batch has no refinement sweeps");
      launch_refinement(b, st);
      break;
    default: return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "unknown phase");
  }
  CU(cudaGetLastError());
  return VISTIO_OK;
}

vistio_status vistio_batch_phase_bytes(const vistio_batch* b, int32_t phase, uint64_t* bytes) {
  if (!b || !bytes) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null argument");
  uint64_t V = b->V, T = b->T, H = b->H, stored = 0, fwd = 0, rows = 0;
  for (auto* s : b->solvers) {
    stored += s->setup.factor.nnz_stored;
    fwd += s->setup.factor.fwd_sn.size();
    rows += s->setup.factor.rows.size();
  }
  switch (phase) {
    case 0: *bytes = V * (16 * 4 + 16 + 1); break;            // read x, v; write prev, pred, x
    case 1: *bytes = T * (16 + 16 + 4 + 36) + 3 * T * 16; break; // indices, Dm^-1, w, 3 contributions; 3 gathered x
    case 2: *bytes = H * (16 + 16 + 8 + 16) + 4 * H * 16; break; // indices, stencil, (w, theta0), out; 4 gathered x
    case 3: *bytes = V * (4 + 16 + 16 + 16) + (V + 1) * 8 + 3 * T * (4 + 12) + 4 * H * (4 + 16 + 4); break;
    case 4: *bytes = 2 * 4 * stored + fwd * 4 + rows * (4 + 2 * 16) + V * (2 * 16 + 2 * 16) + V * 8; break;
    case 5: *bytes = V * (16 * 3 + 1 + 16); break;
    case 6: {  // refinement: A (f64 value + column), d gathered, R0, W; then one sweep pair
      uint64_t nnz_a = 0;
      for (auto* s : b->solvers) nnz_a += s->setup.A_col.size();
      *bytes = nnz_a * 12 + (V + 1) * 4 + V * (16 + 16 + 16) +
               2 * 4 * stored + fwd * 4 + rows * (4 + 2 * 16) + V * (2 * 16 + 2 * 16);
      break;
    }
    default: return fail(b->ctx, VISTIO_ERR_INVALID_CONFIG, "unknown phase");
  }
  return VISTIO_OK;
}

// ---- SparseSolver mirror (sparse.rs:110-120, faer_solver.rs:67-129) ----
vistio_status vistio_symbolic_cache_info(uint64_t* hits, uint64_t* misses, uint64_t* bytes, uint64_t* entries) {
  symbolic_cache_info(hits, misses, bytes, entries);
  return VISTIO_OK;
}

vistio_status vistio_symbolic_cache_set_limit(uint64_t bytes) {
  symbolic_cache_set_limit(bytes);
  return VISTIO_OK;
}

vistio_status vistio_sparse_factorize(vistio_ctx* ctx, uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                                      const float* values, vistio_factor** out) {
  if (!ctx || !row_ptr || !col_idx || !values || !out) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null argument");
  if (n == 0) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "Cannot factorize empty matrix");
  auto f = std::make_unique<vistio_factor>();
  f->ctx = ctx;
  f->n = n;
  // CSR f32 with possible duplicates -> summed f64 (faer's triplet semantics).
  std::vector<std::pair<uint64_t, double>> tr;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
      if (col_idx[p] >= n) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "column index out of range");
      tr.push_back({(uint64_t(i) << 32) | col_idx[p], double(values[p])});
    }
  std::stable_sort(tr.begin(), tr.end(), [](auto& a, auto& b) { return a.first < b.first; });
  f->A_ptr.assign(n + 1, 0);
  for (size_t k = 0; k < tr.size();) {
    size_t j = k;
    double s = 0;
    while (j < tr.size() && tr[j].first == tr[k].first) s += tr[j++].second;
    uint32_t r = uint32_t(tr[k].first >> 32);
    f->A_col.push_back(uint32_t(tr[k].first & 0xffffffffu));
    f->A_val.push_back(s);
    f->A_ptr[r + 1]++;
    k = j;
  }
  for (uint32_t i = 0; i < n; ++i) f->A_ptr[i + 1] += f->A_ptr[i];
  // faer reads the upper triangle (Side::Upper): the symmetric matrix it defines
  std::vector<uint32_t> sym_ptr = f->A_ptr, sym_col = f->A_col;
  std::vector<double> sym_val = f->A_val;
  mirror_upper(n, sym_ptr, sym_col, sym_val);
  // the host finds the ordering and the symbolic structure; the numeric
  // factorization runs on the device (k_front) when the batch is packed
  int st = 0;
  std::string err = factorize_csr(n, sym_ptr.data(), sym_col.data(), sym_val.data(), nullptr, f->f, &st, false);
  if (!err.empty()) return fail(ctx, st == 11 ? VISTIO_ERR_NOT_SPD : VISTIO_ERR_INVALID_CONFIG, err);
  // Device layout: a one-instance batch with no elements.
  auto* s = new vistio_solver();
  s->ctx = ctx;
  s->cfg.max_iterations = 1;
  s->setup.nv = n;
  s->setup.factor = f->f;
  // the symmetric matrix the upper triangle defines, rows in original order
  s->setup.A_ptr.swap(sym_ptr);
  s->setup.A_col.swap(sym_col);
  s->setup.A_val.swap(sym_val);
  s->setup.mass.assign(n, 0.f);
  s->setup.pinned.assign(n, 0);
  s->setup.prm.matrix_dt = 1.f;
  s->host_pos.assign(3 * size_t(n), 0.f);
  s->host_vel.assign(3 * size_t(n), 0.f);
  f->b = new vistio_batch();
  vistio_solver* arr[1] = {s};
  vistio_status r = pack_batch(ctx, arr, 1, f->b);
  if (r != VISTIO_OK) { delete f->b; f->b = nullptr; delete s; return r; }
  StepParams p{};
  p.dt = 1.f;
  CU(cudaMemcpy(f->b->prm.p, &p, sizeof(p), cudaMemcpyHostToDevice));
  *out = f.release();
  return VISTIO_OK;
}

vistio_status vistio_sparse_solve(vistio_factor* f, const float* rhs, float* solution) {
  if (!f) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "Solver not factorized. Call factorize() first.");
  if (!rhs || !solution) return fail(f->ctx, VISTIO_ERR_INVALID_CONFIG, "null vector");
  vistio_ctx* ctx = f->ctx;
  uint32_t n = f->n;
  vistio_batch* b = f->b;
  // f32 rhs -> device sweeps in FP32 -> two FP64 iterative-refinement passes
  // with the residual b - A x formed on the host in f64.
  std::vector<double> x(n, 0.0), r(n);
  for (uint32_t i = 0; i < n; ++i) r[i] = double(rhs[i]);
  std::vector<float4> y(n);
  for (int pass = 0; pass < 3; ++pass) {
    for (uint32_t i = 0; i < n; ++i) y[f->f.iperm[i]] = make_float4(float(r[i]), 0.f, 0.f, 0.f);
    CU(cudaMemcpyAsync(b->Y.p, y.data(), n * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
    launch_solve(b, ctx->stream, 0, 0);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(y.data(), b->Y.p, n * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (uint32_t i = 0; i < n; ++i) x[i] += double(y[f->f.iperm[i]].x);
    for (uint32_t i = 0; i < n; ++i) {
      double s = double(rhs[i]);
      for (uint32_t p = f->A_ptr[i]; p < f->A_ptr[i + 1]; ++p) s -= f->A_val[p] * x[f->A_col[p]];
      r[i] = s;
    }
  }
  for (uint32_t i = 0; i < n; ++i) solution[i] = float(x[i]);
  return VISTIO_OK;
}

vistio_status vistio_sparse_destroy(vistio_factor* f) {
  if (!f) return VISTIO_OK;
  if (f->b) {
    vistio_solver* s = f->b->solvers.empty() ? nullptr : f->b->solvers[0];
    delete f->b;
    delete s;
  }
  delete f;
  return VISTIO_OK;
}

vistio_status vistio_diag_wait_timeout(vistio_ctx* ctx, uint32_t polls) {
  if (!ctx) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null context");
  if (polls == 0 || polls > kWaitLimit) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "polls must be in 1..2^22");
  DevBuf<uint32_t> st;
  uint32_t bits = 0;
  CU(st.alloc(1, ctx->stream));
  CU(cudaMemsetAsync(st.p, 0, 4, ctx->stream));
  k_diag_wait<<<1, 32, 0, ctx->stream>>>(st.p, polls);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(&bits, st.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  if (bits & 4u)
    return fail(ctx, VISTIO_ERR_TIMEOUT, "bounded device wait gave up after " + std::to_string(polls) + " polls");
  return fail(ctx, VISTIO_ERR_INVARIANT, "the diagnostic wait completed although nothing signalled it");
}

vistio_status vistio_broadphase_pairs(vistio_ctx* ctx, uint32_t nv, const float* px, const float* py, const float* pz,
                                      uint32_t nt, const uint32_t* tris, float margin, uint32_t* pairs, uint64_t cap,
                                      uint64_t* count) {
  return broadphase_pairs_impl(ctx, nv, px, py, pz, nt, tris, margin, pairs, cap, count);
}

vistio_status vistio_ccd_hits(vistio_ctx* ctx, uint32_t nv, const float* p0, const float* p1, uint32_t nt,
                              const uint32_t* tris, uint64_t npairs, const uint32_t* pairs, uint32_t* hits,
                              uint64_t cap, uint64_t* nhits, float* min_toi) {
  return ccd_hits_impl(ctx, nv, p0, p1, nt, tris, npairs, pairs, hits, cap, nhits, min_toi);
}

vistio_status vistio_barrier_grad(vistio_ctx* ctx, uint32_t n, const double* d2, double d_hat, double kappa,
                                  double thickness, double* out) {
  if (!ctx || (n && (!d2 || !out))) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null argument");
  if (n == 0) return VISTIO_OK;
  cudaStream_t st = ctx->stream;
  CU(cudaSetDevice(ctx->device));
  DevBuf<double> din, dout;
  CU(din.alloc(n, st));
  CU(dout.alloc(n, st));
  CU(cudaMemcpyAsync(din.p, d2, 8 * size_t(n), cudaMemcpyHostToDevice, st));
  k_barrier_grad<<<(n + 255) / 256, 256, 0, st>>>(din.p, n, d_hat, kappa, thickness, dout.p);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(out, dout.p, 8 * size_t(n), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  return VISTIO_OK;
}

}  // extern "C"

// ======================================================= self-contact host
namespace vistio {

namespace {
// Builds the per-garment tree layout and the exclusion lists.
vistio_status self_build(SelfContactDev& S, const std::vector<std::pair<const uint32_t*, uint32_t>>& tris,
                         const std::vector<uint32_t>& nverts, const std::vector<uint32_t>& vbase, uint64_t T,
                         cudaStream_t st, std::string* err) {
  auto bad = [&](cudaError_t e, const char* what) {
    if (err) *err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? VISTIO_ERR_OOM : VISTIO_ERR_GPU;
  };
  uint32_t n = uint32_t(tris.size());
  std::vector<SelfInst> si(n);
  std::vector<uint32_t> tri_inst(T);
  uint64_t tb = 0, boxes = 0;
  for (uint32_t k = 0; k < n; ++k) {
    uint32_t nt = tris[k].second;
    if (nt >= (1u << 26)) { if (err) *err = "too many triangles for self contact"; return VISTIO_ERR_CAPACITY; }
    SelfInst& I = si[k];
    std::memset(&I, 0, sizeof(I));
    I.tbase = uint32_t(tb);
    I.nt = nt;
    I.box_base = uint32_t(boxes);
    uint32_t cnt = nt, off = 0, l = 0;
    while (true) {
      I.lvl_off[l] = off;
      I.lvl_cnt[l] = cnt;
      off += cnt;
      ++l;
      if (cnt <= 1) break;
      cnt = (cnt + 1) / 2;
    }
    I.nlevels = l;
    boxes += off;
    for (uint32_t t = 0; t < nt; ++t) tri_inst[tb + t] = k;
    tb += nt;
  }
  // exclusion lists: 1-ring plus the vertex (exclusion.rs:27-58, depth 1), global ids
  uint64_t V = 0;
  for (uint32_t k = 0; k < n; ++k) V = std::max<uint64_t>(V, uint64_t(vbase[k]) + nverts[k]);
  std::vector<std::vector<uint32_t>> ring(V);
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t* t = tris[k].first;
    for (uint32_t i = 0; i < tris[k].second; ++i) {
      uint32_t v[3] = {vbase[k] + t[3 * i], vbase[k] + t[3 * i + 1], vbase[k] + t[3 * i + 2]};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) ring[v[a]].push_back(v[b]);
    }
  }
  std::vector<uint32_t> aptr(V + 1, 0), adj;
  for (uint64_t v = 0; v < V; ++v) {
    auto& r = ring[v];
    r.push_back(uint32_t(v));
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    adj.insert(adj.end(), r.begin(), r.end());
    aptr[v + 1] = uint32_t(adj.size());
  }
  S.release();
  S.stream = st;
  S.ninst = n;
  S.T = T;
  S.pair_cap = std::max<uint64_t>(1024, 48 * T);
  S.scan_blocks = uint32_t((T + kScanBlock - 1) / kScanBlock);
  if (S.scan_blocks == 0) S.scan_blocks = 1;
  cudaError_t e;
#define SA(ptr, bytes) \
  if ((e = cudaMallocAsync(reinterpret_cast<void**>(&ptr), bytes, st)) != cudaSuccess) return bad(e, "cudaMallocAsync")
  SA(S.inst, n * sizeof(SelfInst));
  SA(S.tri_inst, std::max<uint64_t>(T, 1) * 4);
  SA(S.box_min, std::max<uint64_t>(boxes, 1) * sizeof(float4));
  SA(S.box_max, std::max<uint64_t>(boxes, 1) * sizeof(float4));
  SA(S.cnt, std::max<uint64_t>(T, 1) * 4);
  SA(S.block_sums, S.scan_blocks * 4ull);
  SA(S.pairs, S.pair_cap * sizeof(uint2));
  SA(S.npairs, 8);
  SA(S.adj_ptr, (V + 1) * 4);
  SA(S.adj, std::max<size_t>(adj.size(), 1) * 4);
  // LBVH sort buffers: keys carry the garment index above a 30-bit Morton code
  {
    const uint64_t Tn = std::max<uint64_t>(T, 1);
    uint32_t gbits = 0;
    while ((1ull << gbits) < n) ++gbits;
    S.sort_passes = (30 + gbits + 7) / 8;
    S.sort_blocks = uint32_t((Tn + kSortTile - 1) / kSortTile);
    S.sort_scan_blocks = uint32_t((256ull * S.sort_blocks + kScanBlock - 1) / kScanBlock);
    SA(S.keys, Tn * 8);
    SA(S.keys_alt, Tn * 8);
    SA(S.order, Tn * 4);
    SA(S.order_alt, Tn * 4);
    SA(S.sort_hist, 256ull * S.sort_blocks * 4);
    SA(S.sort_sums, (S.sort_scan_blocks + 1ull) * 4);
    S.leaf_tri = S.sort_passes % 2 == 0 ? S.order : S.order_alt;  // where the last pass leaves the order
  }
  // the self CCD's deduplicated tests: as many as the pair capacity (a cloth
  // mesh has about 1.6 per pair); beyond it the CCD runs over the pairs
  S.vt_cap = std::min<uint64_t>(S.pair_cap, 0xffffffffull);
  SA(S.leaf_of, std::max<uint64_t>(T, 1) * 4);
  SA(S.vt, S.vt_cap * sizeof(uint2));
  SA(S.nvt, 8);
#undef SA
  if ((e = cudaMemcpyAsync(S.inst, si.data(), n * sizeof(SelfInst), cudaMemcpyHostToDevice, st)) != cudaSuccess) return bad(e, "copy");
  if (T && (e = cudaMemcpyAsync(S.tri_inst, tri_inst.data(), T * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return bad(e, "copy");
  if ((e = cudaMemcpyAsync(S.adj_ptr, aptr.data(), (V + 1) * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return bad(e, "copy");
  if (!adj.empty() && (e = cudaMemcpyAsync(S.adj, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return bad(e, "copy");
  if ((e = cudaMemsetAsync(S.npairs, 0, 8, st)) != cudaSuccess) return bad(e, "memset");
  if ((e = cudaMemsetAsync(S.nvt, 0, 8, st)) != cudaSuccess) return bad(e, "memset");
  if ((e = cudaMemsetAsync(S.leaf_of, 0, std::max<uint64_t>(T, 1) * 4, st)) != cudaSuccess) return bad(e, "memset");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return bad(e, "sync");
  S.ready = true;
  return VISTIO_OK;
}
}  // namespace

vistio_status ensure_self_contact(const BatchDev&, SelfContactDev& S, const std::vector<vistio_solver*>& solvers,
                                  const std::vector<uint32_t>& vbase, uint64_t T, cudaStream_t st, std::string* err) {
  if (S.ready) return VISTIO_OK;
  std::vector<std::pair<const uint32_t*, uint32_t>> tris;
  std::vector<uint32_t> nverts;
  for (auto* s : solvers) {
    tris.push_back({s->setup.tris.data(), s->setup.nt});
    nverts.push_back(s->setup.nv);
  }
  return self_build(S, tris, nverts, vbase, T, st, err);
}

vistio_status broadphase_pairs_impl(vistio_ctx* ctx, uint32_t nv, const float* px, const float* py,
                                    const float* pz, uint32_t nt, const uint32_t* tris, float margin, uint32_t* pairs,
                                    uint64_t cap, uint64_t* count) {
  if (!ctx) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null context");
  cudaStream_t st = ctx->stream;
  std::string* err = &ctx->last_error;
  if (!px || !py || !pz || !tris || !count) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null argument");
  if (nt == 0) { *count = 0; return VISTIO_OK; }
  for (uint64_t k = 0; k < 3ull * nt; ++k)
    if (tris[k] >= nv) return fail(ctx, VISTIO_ERR_INVALID_MESH, "triangle index out of range");
  std::vector<float4> pos(nv);
  for (uint32_t i = 0; i < nv; ++i) pos[i] = make_float4(px[i], py[i], pz[i], 0.f);
  std::vector<uint4> ti(nt);
  for (uint32_t t = 0; t < nt; ++t) ti[t] = make_uint4(tris[3 * t], tris[3 * t + 1], tris[3 * t + 2], 0u);
  std::vector<uint64_t> b0{0}, c0{nt};
  auto ch = make_chunks(b0, c0);
  DevBuf<float4> dpos; DevBuf<uint4> dti; DevBuf<int4> dch; DevBuf<InstRed> dred; DevBuf<StepParams> dprm;
  DevBuf<uint32_t> dstatus;
  CU(dpos.upload(pos, st)); CU(dti.upload(ti, st)); CU(dch.upload(ch, st));
  CU(dred.alloc(1, st)); CU(cudaMemsetAsync(dred.p, 0, sizeof(InstRed), st));
  StepParams p{};
  std::vector<StepParams> pv{p};
  CU(dprm.upload(pv, st));
  CU(dstatus.alloc(1, st)); CU(cudaMemsetAsync(dstatus.p, 0, 4, st));
  BatchDev d{};
  d.pos = dpos.p; d.tri_idx = dti.p; d.tri_chunks = dch.p; d.red = dred.p; d.prm = dprm.p; d.status = dstatus.p;
  SelfContactDev S;
  std::vector<std::pair<const uint32_t*, uint32_t>> tl{{tris, nt}};
  std::vector<uint32_t> nvs{nv}, vb{0};
  vistio_status r = self_build(S, tl, nvs, vb, nt, st, err);
  if (r != VISTIO_OK) return r;
  launch_self_sort(d, S.view(), st);
  k_self_boxes<<<1, 1024, 0, st>>>(d, S.view(), margin);
  k_self_count<<<uint32_t(ch.size()), 256, 0, st>>>(d, S.view());
  k_scan_local<<<S.scan_blocks, kScanBlock, 0, st>>>(S.cnt, nt, S.block_sums);
  k_scan_sums<<<1, kScanBlock, 0, st>>>(S.block_sums, S.scan_blocks, S.npairs);
  k_scan_add<<<S.scan_blocks, kScanBlock, 0, st>>>(S.cnt, nt, S.block_sums);
  uint32_t total = 0;
  CU(cudaMemcpyAsync(&total, S.npairs, 4, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  if (total > S.pair_cap) {  // grow and recount
    cudaFreeAsync(S.pairs, st);
    S.pairs = nullptr;
    S.pair_cap = total;
    CU(cudaMallocAsync(reinterpret_cast<void**>(&S.pairs), uint64_t(total) * sizeof(uint2), st));
  }
  k_self_write<<<uint32_t(ch.size()), 256, 0, st>>>(d, S.view());
  CU(cudaGetLastError());
  std::vector<uint2> hp(total);
  if (total) CU(cudaMemcpyAsync(hp.data(), S.pairs, uint64_t(total) * sizeof(uint2), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  std::sort(hp.begin(), hp.end(), [](uint2 a, uint2 b) { return a.x != b.x ? a.x < b.x : a.y < b.y; });
  *count = total;
  if (pairs)
    for (uint64_t k = 0; k < total && k < cap; ++k) { pairs[2 * k] = hp[k].x; pairs[2 * k + 1] = hp[k].y; }
  if (pairs && total > cap) return fail(ctx, VISTIO_ERR_CAPACITY, "pair buffer too small");
  return VISTIO_OK;
}

// FP64 vertex-triangle CCD per candidate pair for the hit-set boundary test.
__global__ void k_ccd_hits(const float* p0, const float* p1, const uint32_t* tris, const uint32_t* pairs,
                           uint64_t npairs, uint2* hits, double* tois) {
  uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  uint32_t ta = pairs[2 * k], tb = pairs[2 * k + 1];
  uint32_t A[3] = {tris[3 * ta], tris[3 * ta + 1], tris[3 * ta + 2]};
  uint32_t Bv[3] = {tris[3 * tb], tris[3 * tb + 1], tris[3 * tb + 2]};
  auto L0 = [&](uint32_t v) { return mk<double>(p0[3 * v], p0[3 * v + 1], p0[3 * v + 2]); };
  auto L1 = [&](uint32_t v) { return mk<double>(p1[3 * v], p1[3 * v + 1], p1[3 * v + 2]); };
  for (int side = 0; side < 2; ++side) {
    const uint32_t* X = side == 0 ? A : Bv;
    const uint32_t* Y = side == 0 ? Bv : A;
    uint32_t ty = side == 0 ? tb : ta;
    for (int q = 0; q < 3; ++q) {
      uint32_t v = X[q];
      uint64_t slot = 6 * k + 3 * side + q;
      hits[slot] = make_uint2(0xffffffffu, 0xffffffffu);
      tois[slot] = 2.0;
      if (v == Y[0] || v == Y[1] || v == Y[2]) continue;
      double t = vt_ccd<double>(L0(v), L1(v), L0(Y[0]), L1(Y[0]), L0(Y[1]), L1(Y[1]), L0(Y[2]), L1(Y[2]));
      if (t <= 1.0) { hits[slot] = make_uint2(v, ty); tois[slot] = t; }
    }
  }
}

vistio_status ccd_hits_impl(vistio_ctx* ctx, uint32_t nv, const float* p0, const float* p1,
                            uint32_t nt, const uint32_t* tris, uint64_t npairs, const uint32_t* pairs, uint32_t* hits,
                            uint64_t cap, uint64_t* nhits, float* min_toi) {
  if (!ctx) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null context");
  cudaStream_t st = ctx->stream;
  if (!p0 || !p1 || !tris || (!pairs && npairs) || !nhits) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null argument");
  for (uint64_t k = 0; k < 2 * npairs; ++k)
    if (pairs[k] >= nt) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "pair index out of range");
  for (uint64_t k = 0; k < 3ull * nt; ++k)
    if (tris[k] >= nv) return fail(ctx, VISTIO_ERR_INVALID_MESH, "triangle index out of range");
  std::vector<float> a(p0, p0 + 3ull * nv), b(p1, p1 + 3ull * nv);
  std::vector<uint32_t> tv(tris, tris + 3ull * nt), pv(pairs, pairs + 2 * npairs);
  DevBuf<float> d0, d1; DevBuf<uint32_t> dt, dp; DevBuf<uint2> dh; DevBuf<double> dtoi;
  CU(d0.upload(a, st)); CU(d1.upload(b, st)); CU(dt.upload(tv, st)); CU(dp.upload(pv, st));
  CU(dh.alloc(6 * std::max<uint64_t>(npairs, 1), st)); CU(dtoi.alloc(6 * std::max<uint64_t>(npairs, 1), st));
  if (npairs) k_ccd_hits<<<uint32_t((npairs + 127) / 128), 128, 0, st>>>(d0.p, d1.p, dt.p, dp.p, npairs, dh.p, dtoi.p);
  CU(cudaGetLastError());
  std::vector<uint2> hh(6 * npairs);
  std::vector<double> tt(6 * npairs);
  if (npairs) {
    CU(cudaMemcpyAsync(hh.data(), dh.p, hh.size() * sizeof(uint2), cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(tt.data(), dtoi.p, tt.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CU(cudaStreamSynchronize(st));
  std::vector<std::pair<uint32_t, uint32_t>> out;
  double mt = 1.0;
  for (size_t k = 0; k < hh.size(); ++k)
    if (hh[k].x != 0xffffffffu) { out.push_back({hh[k].x, hh[k].y}); mt = std::min(mt, tt[k]); }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  *nhits = out.size();
  if (min_toi) *min_toi = float(std::max(mt, 1e-6));
  if (hits)
    for (size_t k = 0; k < out.size() && k < cap; ++k) { hits[2 * k] = out[k].first; hits[2 * k + 1] = out[k].second; }
  if (hits && out.size() > cap) return fail(ctx, VISTIO_ERR_CAPACITY, "hit buffer too small");
  return VISTIO_OK;
}

}  // namespace vistio

// ================================================ allocation-free broad phase
// vistio_broadphase_pairs_noalloc finds the same candidate pairs as
// vistio_broadphase_pairs with every device buffer carved out of one fixed
// region that is part of the library image, so the call itself allocates and
// frees no device memory. It is meant for callers that cannot allocate on the
// call: a server whose HBM is fully committed to resident garments and
// factors (a cudaMalloc there can fail, or push out memory it has promised
// elsewhere), and per-frame collision queries on a latency-critical thread,
// where cudaFree's implicit device-wide synchronisation would stall all other
// work on the GPU.
//
// Unlike vistio_broadphase_pairs it does not reorder the triangles by Morton
// code first: the implicit balanced tree is built over the triangles in mesh
// order. The pair set is the same (every overlapping pair is found whatever the
// leaf order); only the traversal cost differs on meshes whose triangles are
// not stored in spatial order.
//
// The region is sized for meshes of up to kNaMaxTris triangles and kNaMaxVerts
// vertices and for up to kNaMaxPairs candidate pairs (about 16 MB); larger
// inputs are rejected with VISTIO_ERR_CAPACITY before any device work. There
// is one region per device, so calls on the same device must not overlap:
// two of them in flight at once (two threads, or two contexts' streams)
// race on it. The call is synchronous (it reads the pair count back) and so
// cannot be captured into a CUDA graph.
namespace vistio_na {
constexpr uint32_t kNaMaxTris = 65536;
constexpr uint32_t kNaMaxVerts = 65536;
constexpr uint32_t kNaMaxPairs = 1u << 20;
constexpr uint32_t kNaMaxBoxes = 2 * kNaMaxTris + 32;  // every tree level of kNaMaxTris leaves
constexpr uint32_t kNaChunks = (kNaMaxTris + kElemThreads - 1) / kElemThreads;
constexpr uint32_t kNaScanBlocks = (kNaMaxTris + vistio::kScanBlock - 1) / vistio::kScanBlock;

constexpr uint64_t na_up(uint64_t x) { return (x + 255) & ~uint64_t(255); }

// Byte offsets of the buffers inside the region, each 256-byte aligned.
struct NaLayout {
  static constexpr uint64_t raw_x = 0;  // caller's SoA positions, as given
  static constexpr uint64_t raw_y = raw_x + na_up(4ull * kNaMaxVerts);
  static constexpr uint64_t raw_z = raw_y + na_up(4ull * kNaMaxVerts);
  static constexpr uint64_t raw_tri = raw_z + na_up(4ull * kNaMaxVerts);
  static constexpr uint64_t pos = raw_tri + na_up(12ull * kNaMaxTris);  // float4 per vertex
  static constexpr uint64_t tri = pos + na_up(16ull * kNaMaxVerts);     // uint4 per triangle
  static constexpr uint64_t chunks = tri + na_up(16ull * kNaMaxTris);
  // red, prm and status must start at zero on every call (cleared together).
  static constexpr uint64_t red = chunks + na_up(16ull * kNaChunks);
  static constexpr uint64_t prm = red + na_up(sizeof(vistio::InstRed));
  static constexpr uint64_t status = prm + na_up(sizeof(vistio::StepParams));
  static constexpr uint64_t zero_end = status + na_up(4);
  static constexpr uint64_t inst = zero_end;
  static constexpr uint64_t tri_inst = inst + na_up(sizeof(vistio::SelfInst));
  static constexpr uint64_t box_min = tri_inst + na_up(4ull * kNaMaxTris);
  static constexpr uint64_t box_max = box_min + na_up(16ull * kNaMaxBoxes);
  static constexpr uint64_t cnt = box_max + na_up(16ull * kNaMaxBoxes);
  static constexpr uint64_t block_sums = cnt + na_up(4ull * kNaMaxTris);
  static constexpr uint64_t npairs = block_sums + na_up(4ull * kNaScanBlocks);  // [count, overflow]: zeroed
  static constexpr uint64_t pairs = npairs + na_up(8);
  static constexpr uint64_t bytes = pairs + na_up(8ull * kNaMaxPairs);
};
}  // namespace vistio_na

using namespace vistio_na;
static __device__ __align__(256) unsigned char g_na_scratch[NaLayout::bytes];

namespace vistio_na {
// Device address of the region on the context's device. Host code cannot use
// g_na_scratch itself (on the host it names a stand-in, not device memory), so
// every call makes the context's device current and asks the runtime for the
// address: a cheap lookup, and never stale after the device's context has been
// reset and the module reloaded.
vistio_status na_region(vistio_ctx* ctx, unsigned char** out) {
  CU(cudaSetDevice(ctx->device));
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
  if (e != cudaSuccess || !p)
    return fail(ctx, VISTIO_ERR_GPU, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  *out = static_cast<unsigned char*>(p);
  return VISTIO_OK;
}

// SoA positions and index triples -> the float4 / uint4 rows the broad-phase
// kernels read; one chunk per 256 triangles, all of garment 0.
__global__ void k_na_pack(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                          uint32_t nv, const uint32_t* __restrict__ t, uint32_t nt, float4* pos, uint4* tri,
                          uint32_t* tri_inst, int4* chunks, uint32_t nchunks) {
  const uint32_t n = nv > nt ? nv : nt;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < nv) pos[i] = make_float4(x[i], y[i], z[i], 0.f);
    if (i < nt) {
      tri[i] = make_uint4(t[3 * i], t[3 * i + 1], t[3 * i + 2], 0u);
      tri_inst[i] = 0u;
    }
    if (i < nchunks) {
      const uint32_t b = i * kElemThreads;
      chunks[i] = make_int4(0, int(b), int(min(uint32_t(kElemThreads), nt - b)), 0);
    }
  }
}

struct NaPair { uint32_t a, b; };
static_assert(sizeof(NaPair) == 8, "pairs are two packed u32");

vistio_status broadphase_pairs_noalloc_impl(vistio_ctx* ctx, uint32_t nv, const float* px, const float* py,
                                            const float* pz, uint32_t nt, const uint32_t* tris, float margin,
                                            uint32_t* pairs, uint64_t cap, uint64_t* count) {
  if (!ctx) return fail(nullptr, VISTIO_ERR_INVALID_CONFIG, "null context");
  if (!px || !py || !pz || !tris || !count) return fail(ctx, VISTIO_ERR_INVALID_CONFIG, "null argument");
  if (nt == 0) { *count = 0; return VISTIO_OK; }
  if (nt > kNaMaxTris || nv > kNaMaxVerts)
    return fail(ctx, VISTIO_ERR_CAPACITY,
                "mesh too large for the allocation-free broad phase (at most 65536 triangles and 65536 vertices); "
                "use vistio_broadphase_pairs");
  for (uint64_t k = 0; k < 3ull * nt; ++k)
    if (tris[k] >= nv) return fail(ctx, VISTIO_ERR_INVALID_MESH, "triangle index out of range");
  unsigned char* base = nullptr;
  vistio_status r = na_region(ctx, &base);
  if (r != VISTIO_OK) return r;
  cudaStream_t st = ctx->stream;
  auto at = [&](uint64_t off) { return base + off; };

  // Tree layout of one garment (host, on the stack).
  SelfInst I;
  std::memset(&I, 0, sizeof(I));
  I.nt = nt;
  for (uint32_t cntl = nt, off = 0, l = 0;; cntl = (cntl + 1) / 2) {
    I.lvl_off[l] = off;
    I.lvl_cnt[l] = cntl;
    off += cntl;
    I.nlevels = ++l;
    if (cntl <= 1) break;
  }
  const uint32_t nchunks = (nt + kElemThreads - 1) / kElemThreads;
  const uint32_t scan_blocks = (nt + kScanBlock - 1) / kScanBlock;

  CU(cudaMemcpyAsync(at(NaLayout::raw_x), px, 4ull * nv, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(at(NaLayout::raw_y), py, 4ull * nv, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(at(NaLayout::raw_z), pz, 4ull * nv, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(at(NaLayout::raw_tri), tris, 12ull * nt, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(at(NaLayout::inst), &I, sizeof(I), cudaMemcpyHostToDevice, st));
  CU(cudaMemsetAsync(at(NaLayout::red), 0, NaLayout::zero_end - NaLayout::red, st));
  CU(cudaMemsetAsync(at(NaLayout::npairs), 0, 8, st));

  BatchDev d{};
  d.pos = reinterpret_cast<float4*>(at(NaLayout::pos));
  d.tri_idx = reinterpret_cast<const uint4*>(at(NaLayout::tri));
  d.tri_chunks = reinterpret_cast<const int4*>(at(NaLayout::chunks));
  d.red = reinterpret_cast<InstRed*>(at(NaLayout::red));
  d.prm = reinterpret_cast<const StepParams*>(at(NaLayout::prm));
  d.status = reinterpret_cast<uint32_t*>(at(NaLayout::status));
  SelfContactView S{};
  S.ninst = 1;
  S.T = nt;
  S.pair_cap = kNaMaxPairs;
  S.inst = reinterpret_cast<SelfInst*>(at(NaLayout::inst));
  S.tri_inst = reinterpret_cast<uint32_t*>(at(NaLayout::tri_inst));
  S.box_min = reinterpret_cast<float4*>(at(NaLayout::box_min));
  S.box_max = reinterpret_cast<float4*>(at(NaLayout::box_max));
  S.cnt = reinterpret_cast<uint32_t*>(at(NaLayout::cnt));
  S.block_sums = reinterpret_cast<uint32_t*>(at(NaLayout::block_sums));
  S.pairs = reinterpret_cast<uint2*>(at(NaLayout::pairs));
  S.npairs = reinterpret_cast<uint32_t*>(at(NaLayout::npairs));
  S.scan_blocks = scan_blocks;

  const uint32_t pack_blocks = std::min<uint32_t>((std::max(nv, nt) + 255) / 256, 148 * 8);
  k_na_pack<<<pack_blocks, 256, 0, st>>>(reinterpret_cast<const float*>(at(NaLayout::raw_x)),
                                         reinterpret_cast<const float*>(at(NaLayout::raw_y)),
                                         reinterpret_cast<const float*>(at(NaLayout::raw_z)), nv,
                                         reinterpret_cast<const uint32_t*>(at(NaLayout::raw_tri)), nt,
                                         d.pos, reinterpret_cast<uint4*>(at(NaLayout::tri)), S.tri_inst,
                                         reinterpret_cast<int4*>(at(NaLayout::chunks)), nchunks);
  k_self_boxes<<<1, 1024, 0, st>>>(d, S, margin);
  k_self_count<<<nchunks, kElemThreads, 0, st>>>(d, S);
  k_scan_local<<<scan_blocks, kScanBlock, 0, st>>>(S.cnt, nt, S.block_sums);
  k_scan_sums<<<1, kScanBlock, 0, st>>>(S.block_sums, scan_blocks, S.npairs);
  k_scan_add<<<scan_blocks, kScanBlock, 0, st>>>(S.cnt, nt, S.block_sums);
  CU(cudaGetLastError());
  uint32_t total = 0;
  CU(cudaMemcpyAsync(&total, S.npairs, 4, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  *count = total;
  if (total > kNaMaxPairs)
    return fail(ctx, VISTIO_ERR_CAPACITY,
                "more than 1048576 candidate pairs: beyond the allocation-free broad phase; use vistio_broadphase_pairs");
  if (!pairs) return VISTIO_OK;  // size query
  if (total > cap) return fail(ctx, VISTIO_ERR_CAPACITY, "pair buffer too small");
  k_self_write<<<nchunks, kElemThreads, 0, st>>>(d, S);
  CU(cudaGetLastError());
  uint32_t status = 0;
  if (total) CU(cudaMemcpyAsync(pairs, S.pairs, 8ull * total, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(&status, d.status, 4, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  if (status & 2u) return fail(ctx, VISTIO_ERR_CAPACITY, "candidate pairs exceeded the scratch");
  NaPair* P = reinterpret_cast<NaPair*>(pairs);
  std::sort(P, P + total, [](const NaPair& u, const NaPair& v) { return u.a != v.a ? u.a < v.a : u.b < v.b; });
  return VISTIO_OK;
}
}  // namespace vistio_na

extern "C" vistio_status vistio_broadphase_pairs_noalloc(vistio_ctx* ctx, uint32_t nv, const float* px,
                                                         const float* py, const float* pz, uint32_t nt,
                                                         const uint32_t* tris, float margin, uint32_t* pairs,
                                                         uint64_t cap, uint64_t* count) {
  return broadphase_pairs_noalloc_impl(ctx, nv, px, py, pz, nt, tris, margin, pairs, cap, count);
}
