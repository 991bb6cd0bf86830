// sm_100a kernels of the Projective Dynamics iteration.
//
// Layout (ragged SoA over every instance of a batch): per-vertex float4
// (x, y, z, -) arrays indexed by a global vertex id; triangles and hinges
// hold global vertex ids; each kernel over elements or vertices runs one
// block per "chunk" (instance, first element, count <= blockDim) so a block
// always sees a single instance and its constants.
//
// The iteration is written in delta form: with A the constant PD matrix
// (M/h^2 + sum w S^T S + sum w_b L^T L) and b the reference's right-hand side
// (assembly.rs:157-240), the solve computes d = A^-1 (b - A x) and sets
// x <- x + d, which equals the reference's x <- A^-1 b in exact arithmetic.
// b - A x collapses per element to w g_k . (F_target - F) for a triangle and
// to w s_k s . (target - x) for a hinge, so the residual is formed from small
// differences and FP32 sweeps lose accuracy relative to |d|, not to |x|.
#pragma once
#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

#include "setup.h"

namespace vistio {

// Programmatic dependent launch. The step's kernels are launched with the
// programmatic stream serialization attribute (launch_pdl on the host), so a
// kernel's blocks may be scheduled while the kernel before it in the stream
// is still running. Each such kernel calls pdl_begin() first: it waits until
// the previous kernel has completed and its memory is visible, which orders
// every earlier kernel too (each of them waited for its own predecessor). A
// grid of at most kPdlEarlyBlocks blocks then lets the next kernel launch
// right away, so that kernel's launch overlaps this one's work; larger grids
// leave the SMs to their own blocks. In a kernel launched without the
// attribute both instructions do nothing.
constexpr uint32_t kPdlEarlyBlocks = 148;
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (gridDim.x * gridDim.y * gridDim.z <= kPdlEarlyBlocks) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches a step kernel with the programmatic stream serialization
// attribute (the kernel calls pdl_begin() first); records errors as a <<<>>>
// launch would.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), uint32_t grid, uint32_t block, size_t smem, cudaStream_t st,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

struct InstDev {
  uint32_t vbase, nv;
  uint32_t nlvl;               // levels of the supernodal elimination tree
  float kappa;                 // barrier stiffness estimated from this garment's own masses
  int32_t model;
  float warp, weft;
  float inv_hmat2;   // 1 / matrix_dt^2
  int32_t has_ground;
  float ground_h;
  uint32_t sn_base, nsn;
  int32_t unit_stencils;       // every hinge stencil is (-1, -1, 1, 1) (dihedral bending): not loaded
  uint32_t tbase, hbase;       // first triangle and hinge of the garment
  uint32_t inc_ptr;            // its connectivity class's per-vertex offsets in vtri_ptr / vhinge_ptr
  uint32_t tinc_off, hinc_off; // its class's codes in vtri / vhinge
};

// One supernode in HBM: one contiguous, 16-byte aligned region holding
//   D  inv(L_kk), s x s column-major with leading dimension ld = sn_ld(s)
//      (odd; Linv[c][c2] at c2*ld + c), then
//   P  the m x s panel below the diagonal block, row-major (P[j][c] at j*ld + c),
//      followed by its m row indices (u32 bits; the same as rows[rows_off..]).
// Both sweeps stage it through shared memory in row chunks.
struct SnDev {
  uint32_t first;    // first column (instance-local permuted row)
  uint32_t ncols;    // s
  uint32_t nrows;    // m
  uint32_t rows_off; // first of the m entries of this supernode in rows / U (global)
  uint64_t d_off;    // D (float offset, multiple of 4)
  uint64_t p_off;    // P (float offset)
  uint32_t vbase;    // first vertex (row) of the owning instance
  uint32_t inst;     // owning instance
  uint32_t u_off;    // U slot of panel row 0; row j's slot is u_off + j * u_stride
  uint32_t u_stride; // 1, or the lanes of a garment group (U interleaved by garment)
};

// Garment groups. Garments of a batch whose factors share one symbolic
// structure (the same mesh topology: the same supernodes, row structures and
// elimination tree; only the numbers differ) are swept together at the bottom
// of their trees, one lane per garment: every lane runs the same loops over
// the same row indices, and a factor entry of the whole group is one 128-byte
// line (the group's values are interleaved, entry-major and garment-minor).
constexpr uint32_t kGroupLanes = 32;
// A group of fewer garments would read less than one 32-byte sector per entry.
constexpr uint32_t kGroupMinLanes = 8;

// One supernode of a group topology. Ids of GsnDev entries are global (every
// topology's supernodes concatenated); parent and kids are local to the
// topology, like the per-garment supernode ids minus the garment's base.
struct GsnDev {
  uint32_t first, ncols, nrows;
  uint32_t rows_off;  // first of its nrows row indices in g_rows
  uint32_t u_local;   // per-garment U slot of panel row 0 (local slot numbering)
  uint32_t parent;    // local parent, or 0xffffffff for a root
  uint32_t kid_off;   // its children in g_kids[kid_off, kid_off + nkids)
  uint32_t nkids;
  uint64_t g_off;     // entries before it in a group's value block: the triangle of
                      // inv(L_kk) (s (s + 1) / 2 entries, row by row), then the
                      // panel (m rows of s entries)
};

struct GroupDev {
  uint32_t sn_off;    // global GsnDev id of the topology's local supernode 0
  uint32_t lanes;     // garments in the group (kGroupMinLanes .. kGroupLanes)
  uint64_t base;      // first entry of the group's value block in g_vals
  uint32_t u_base;    // U slot of local slot 0 of lane 0: slot i of lane l is u_base + i * 32 + l
  uint32_t row_base;  // the topology's rows in g_fwd_ptr start here
};

// Per-step constants read from device memory so a captured graph stays valid
// when dt or the contact set-up change.
struct StepParams {
  float dt, inv_dt2;
  float gravity[3];
  float damping;
  float rayleigh;          // alpha_M
  int32_t ipc;             // step_with_ipc semantics
  // contact
  int32_t has_ground;
  float ground_h;
  int32_t has_sphere;
  float sphere_c[3];
  float sphere_r;
  int32_t self_collision;
  float kappa;
  float thickness;
  int32_t has_cyl;
  float cyl[4];            // center x, center z, top y, radius
  int32_t has_box;
  float box_lo[3], box_hi[3];
  float d_hat;             // effective (compliant) d_hat
  float max_vel;           // velocity clamp (0 = off)
  float al_tolerance, al_mu_growth, al_mu_initial;
  float friction, contact_damping, contact_damping_max, contact_vthresh;
  int32_t adaptive_damping;
};

// Per-instance device scalars of the IPC outer loop and reductions.
struct InstRed {
  double diff_sq, norm_sq;   // residual sums of the last solve
  double gdd;                // sum over free vertices of grad . d
  uint32_t toi_bits;         // min CCD time of impact (float bits, >= 0)
  uint32_t active;           // active contacts of the last detect
  uint32_t maxviol_bits;     // max violation (float bits)
  uint32_t al_done;
  float mu;
  float alpha;
  uint32_t last_active;      // active contacts of the last re-detect
  uint32_t al_iters;
  uint32_t iters;
  uint32_t pad;
};

struct BatchDev {
  const InstDev* inst;
  const int4* tri_chunks;
  const int4* hinge_chunks;
  const int4* vtx_chunks;
  // state
  float4* pos;
  float4* vel;
  float4* prev;
  float4* pred;
  const float* mass;       // solver lumped masses (pinned = 1e8)
  const uint8_t* pinned;
  // elements
  const uint4* tri_idx;    // global vertex ids
  const float4* tri_dm;
  const float* tri_w;
  float* tri_out;          // 9 floats per triangle: the three vertex contributions
  const uint4* hinge_idx;
  const float4* hinge_st;
  const float2* hinge_wr;  // (weight, rest angle)
  float4* hinge_out;       // w * s . (target - x)
  // vertex incidence, one CSR per connectivity class over the garment's local
  // vertex ids (InstDev::inc_ptr, tinc_off, hinc_off)
  const uint32_t* vtri_ptr;
  const uint32_t* vtri;    // (local triangle << 2) | slot
  const uint32_t* vhinge_ptr;
  const uint32_t* vhinge;  // (local hinge << 2) | slot
  // solve
  const uint32_t* perm_local;  // vertex -> instance-local permuted row
  const uint32_t* row_vertex;  // global row -> instance-local vertex
  float4* Y;               // rhs / y / delta, indexed by vbase + row
  float4* T;               // scratch of the sweeps
  const SnDev* sn;
  const uint32_t* rows;        // below-diagonal rows of every supernode (instance-local)
  const float* vals;
  const uint32_t* fwd_ptr;     // global row -> offsets into fwd
  const uint32_t* fwd;         // U slots summed into the row by the forward sweep
  float4* U;                   // forward updates, one per (supernode, panel row)
  const uint32_t* lvl_items;   // supernodes of each batch level (block items first)
  const uint2* sub_items;      // bottom subtrees: (first, last) supernode of each
  // dependency-driven sweeps (k_sweep): work units in forward order (see
  // SweepUnit), the supernodal tree, per-supernode counters (zero between
  // sweeps) and the two work queues
  const uint2* df_units;       // backward sweep, taken from the end
  const uint2* df_units_fwd;   // forward sweep: top supernodes deepest first
  const uint32_t* df_items_fwd;  // warp supernodes of the forward units
  const uint32_t* df_parent;   // parent supernode (global id) or kNoParent
  const uint32_t* df_nkids;
  const uint32_t* df_kid_ptr;
  const uint32_t* df_kids;
  uint32_t* df_cnt;            // forward: children finished
  uint32_t* df_flag;           // backward: parent finished
  uint32_t* df_queue;          // [0] next unit, [1] blocks done (k_sweep resets both)
  // garment-grouped sweeps (k_gsweep)
  const GroupDev* grp;
  const GsnDev* gsn;
  const uint32_t* g_rows;      // topology-local row indices of the panels
  const uint32_t* g_fwd_ptr;   // per topology row (row_base + r): its pull list in g_fwd
  const uint32_t* g_fwd;       // local U slots a row pulls in the forward sweep
  const uint32_t* g_kids;      // local children
  const uint2* g_subs;         // bottom subtrees: (first, last) global GsnDev ids
  const uint32_t* gl_vbase;    // per group lane (group * 32 + lane): the garment's first row
  const uint32_t* gl_snbase;   // ... its first global supernode id
  const uint32_t* gl_inst;     // ... its instance
  const float* g_vals;         // interleaved factor values: entry e of a group at (base + e) * 32 + lane
  const uint2* g_items_fwd;    // work items, forward order: (group, kind | local id << 1)
  const uint2* g_items_bwd;    // backward order
  uint32_t* g_queue;           // [0] next item, [1] warps done (k_gsweep resets both)
  // FP64 refinement: the factored matrix A (f64, rows and columns in each
  // instance's solve order, global row ids), the right-hand side the first
  // sweep solved (R0) and the correction vector the refinement sweeps solve in
  // place (W).
  const uint32_t* a_ptr;
  const uint32_t* a_col;
  const double* a_val;
  float4* R0;
  float4* W;
  // contact / IPC
  float4* grad;            // barrier gradient of the detect at the start of the AL pass
  float4* grad_up;         // gradient of the re-detect
  double4* gacc;           // FP64 accumulator of the self-contact gradient of one detect
  float4* lam;             // AL multipliers
  float4* fin_n;           // final contact normal (ever in contact)
  uint8_t* in_contact;     // of the detect at the start of the AL pass
  uint8_t* in_contact_up;  // of the re-detect
  uint8_t* ever;
  InstRed* red;
  const StepParams* prm;
  uint32_t* status;        // bit 0: non-finite state
};

// ------------------------------------------------------------ math helpers
__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }

// double3 arithmetic for the FP64 local projection.
__device__ __forceinline__ double3 operator+(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 operator-(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 operator*(double3 a, double s) { return make_double3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 d3(float4 a) { return make_double3(a.x, a.y, a.z); }

// 3x2 column-major matrix (mat3x2.rs:16) in FP64.
struct M32 { double3 c0, c1; };

__device__ __forceinline__ M32 mul2(const M32& f, double a, double b, double c, double d) {
  // f * [[a, c], [b, d]] (column-major [a, b, c, d], mat3x2.rs:62)
  M32 r;
  r.c0 = f.c0 * a + f.c1 * b;
  r.c1 = f.c0 * c + f.c1 * d;
  return r;
}

// polar_decomposition_3x2 (crates/vistio-math/src/decomposition.rs:76-138),
// through the eigen-decomposition of F^T F like the reference. It runs in
// FP64: its rounding grows as 1 / sigma_min^2 in compressed triangles, and in
// FP32 that error dominates a step's error wherever the sheet is pressed
// together. The thresholds are the reference's f32 constants.
struct PolarD {
  M32 rot;
  double s0, s1;
  double2 v0, v1;
};
__device__ __forceinline__ PolarD polar_dev(const M32& f) {
  double a = dot3(f.c0, f.c0), b = dot3(f.c0, f.c1), d = dot3(f.c1, f.c1);
  double ht = 0.5 * (a + d), hd = 0.5 * (a - d);
  double disc = sqrt(hd * hd + b * b);
  double l0 = fmax(ht + disc, 0.0), l1 = fmax(ht - disc, 0.0);
  double s0 = sqrt(l0), s1 = sqrt(l1);
  const double eps = double(1.0e-10f);
  PolarD p;
  if (s0 < eps) {
    p.rot.c0 = make_double3(1.0, 0.0, 0.0);
    p.rot.c1 = make_double3(0.0, 1.0, 0.0);
    p.s0 = p.s1 = 0.0;
    p.v0 = make_double2(1.0, 0.0);
    p.v1 = make_double2(0.0, 1.0);
    return p;
  }
  double2 v0, v1;
  if (fabs(b) > eps) {
    double vx = l0 - d, vy = b;
    double r = 1.0 / sqrt(vx * vx + vy * vy);
    v0 = make_double2(vx * r, vy * r);
    v1 = make_double2(-v0.y, v0.x);
  } else if (a >= d) {
    v0 = make_double2(1.0, 0.0); v1 = make_double2(0.0, 1.0);
  } else {
    v0 = make_double2(0.0, 1.0); v1 = make_double2(1.0, 0.0);
  }
  double is0 = 1.0 / s0, is1 = s1 > eps ? 1.0 / s1 : 0.0;
  double si00 = v0.x * v0.x * is0 + v1.x * v1.x * is1;
  double si01 = v0.x * v0.y * is0 + v1.x * v1.y * is1;
  double si11 = v0.y * v0.y * is0 + v1.y * v1.y * is1;
  p.rot = mul2(f, si00, si01, si01, si11);
  p.s0 = s0; p.s1 = s1; p.v0 = v0; p.v1 = v1;
  return p;
}

// Target deformation gradient of the membrane model
// (element.rs:127-174 and crates/vistio-material/src/*.rs).
__device__ __forceinline__ M32 model_target(int model, const M32& F, float warp_f, float weft_f) {
  if (model == 4) {  // IsotropicLinearModel: identity (isotropic.rs:42-57)
    M32 r; r.c0 = make_double3(1.0, 0.0, 0.0); r.c1 = make_double3(0.0, 1.0, 0.0); return r;
  }
  PolarD p = polar_dev(F);
  if (model == 0) return p.rot;  // ARAP: R
  const double warp = warp_f, weft = weft_f;
  double s0t, s1t;
  if (model == 1) {  // co-rotational, tension field: min(sigma, 1) (decomposition.rs:50-66)
    s0t = fmin(p.s0, 1.0); s1t = fmin(p.s1, 1.0);
  } else if (model == 2) {  // orthotropic (orthotropic.rs:51-79)
    double mk = fmax(fmax(warp, weft), double(1e-6f));
    double kw = warp / mk, kf = weft / mk;
    s0t = p.s0 + (1.0 - p.s0) * kw;
    s1t = p.s1 + (1.0 - p.s1) * kf;
  } else {  // anisotropic co-rotational (anisotropic.rs:78-143)
    double kw = fmin(fmax(warp, 0.0), 1.0), kf = fmin(fmax(weft, 0.0), 1.0);
    double cos2 = p.v0.x * p.v0.x, sin2 = p.v0.y * p.v0.y;
    double k0 = kw * cos2 + kf * sin2, k1 = kw * sin2 + kf * cos2;
    s0t = p.s0 > 1.0 ? 1.0 + (p.s0 - 1.0) * (1.0 - k0) : p.s0;
    s1t = p.s1 > 1.0 ? 1.0 + (p.s1 - 1.0) * (1.0 - k1) : p.s1;
  }
  double t00 = p.v0.x * p.v0.x * s0t + p.v1.x * p.v1.x * s1t;
  double t01 = p.v0.x * p.v0.y * s0t + p.v1.x * p.v1.y * s1t;
  double t11 = p.v0.y * p.v0.y * s0t + p.v1.y * p.v1.y * s1t;
  return mul2(p.rot, t00, t01, t01, t11);
}

// ------------------------------------------------------------- kernels
// Local membrane step of one triangle: w * g_k . (F_target - F) for k = 0..2.
// Compiled once (not inlined): the membrane kernels of both shapes run the
// same instructions, so the compiler's multiply-add contraction cannot differ
// between them and their results are bit-identical.
__device__ __noinline__ void tri_project_one(float* __restrict__ tri_out, int32_t model, float warp, float weft,
                                             uint32_t t, float4 dm, float w, float4 q0, float4 q1, float4 q2) {
  // FP64 from the FP32 positions on (the projection is the ill-conditioned
  // part; the outputs are rounded once).
  const double3 p0 = d3(q0), p1 = d3(q1), p2 = d3(q2);
  M32 ds; ds.c0 = p1 - p0; ds.c1 = p2 - p0;
  M32 F = mul2(ds, dm.x, dm.y, dm.z, dm.w);
  float det = dm.x * dm.w - dm.y * dm.z;
  double3 d0 = make_double3(0.0, 0.0, 0.0), d1 = d0;
  if (fabsf(det) > 1e-12f) {  // element.rs:192-202: degenerate rest shape keeps p
    M32 Ft = model_target(model, F, warp, weft);
    d0 = (Ft.c0 - F.c0) * double(w);
    d1 = (Ft.c1 - F.c1) * double(w);
  }
  // g = [[-(a+b), -(c+d)], [a, c], [b, d]] (assembly.rs:77-81)
  const double g00 = -(double(dm.x) + double(dm.y)), g01 = -(double(dm.z) + double(dm.w));
  const double3 c0 = d0 * g00 + d1 * g01;
  const double3 c1 = d0 * double(dm.x) + d1 * double(dm.z);
  const double3 c2 = d0 * double(dm.y) + d1 * double(dm.w);
  float* o = tri_out + 9ull * t;
  o[0] = float(c0.x); o[1] = float(c0.y); o[2] = float(c0.z);
  o[3] = float(c1.x); o[4] = float(c1.y); o[5] = float(c1.z);
  o[6] = float(c2.x); o[7] = float(c2.y); o[8] = float(c2.z);
}
__device__ __forceinline__ void tri_project(const BatchDev& B, const InstDev& I, uint32_t t, float4 dm, float w,
                                            float4 q0, float4 q1, float4 q2) {
  tri_project_one(B.tri_out, I.model, I.warp, I.weft, t, dm, w, q0, q1, q2);
}

// The membrane step over a chunk of up to 256 triangles with 128 threads:
// each thread loads both of its triangles (indices, rest data, the six
// vertex positions) before it projects either, so twice the loads are in
// flight per warp; eight blocks per SM (64 registers). The loads are
// latency-bound: 0.216 -> 0.176 ms per iteration on 7.9 M triangles against
// one triangle per thread at five 256-thread blocks per SM.
constexpr int kTriThreads = 128;
__global__ void __launch_bounds__(kTriThreads, 8) k_tri(BatchDev B) {
  pdl_begin();
  int4 ch = B.tri_chunks[blockIdx.x];
  const uint32_t i0 = threadIdx.x, i1 = threadIdx.x + kTriThreads;
  if ((int)i0 >= ch.z) return;
  if (B.prm->ipc && B.red[ch.x].al_done) return;
  const bool two = (int)i1 < ch.z;
  const uint32_t t0 = uint32_t(ch.y) + i0, t1 = uint32_t(ch.y) + i1;
  const InstDev I = B.inst[ch.x];
  const uint4 a = B.tri_idx[t0], b = two ? B.tri_idx[t1] : a;
  const float4 dma = B.tri_dm[t0], dmb = two ? B.tri_dm[t1] : dma;
  const float wa = B.tri_w[t0], wb = two ? B.tri_w[t1] : wa;
  const float4 qa0 = B.pos[a.x], qa1 = B.pos[a.y], qa2 = B.pos[a.z];
  float4 qb0 = qa0, qb1 = qa1, qb2 = qa2;
  if (two) { qb0 = B.pos[b.x]; qb1 = B.pos[b.y]; qb2 = B.pos[b.z]; }
  tri_project(B, I, t0, dma, wa, qa0, qa1, qa2);
  if (two) tri_project(B, I, t1, dmb, wb, qb0, qb1, qb2);
}

// The same membrane step with one triangle per thread (a chunk of up to 256
// triangles on 256 threads, four blocks per SM): the autotuner's other shape.
__global__ void __launch_bounds__(256, 4) k_tri1(BatchDev B) {
  pdl_begin();
  int4 ch = B.tri_chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  if (B.prm->ipc && B.red[ch.x].al_done) return;
  const uint32_t t = uint32_t(ch.y) + threadIdx.x;
  const InstDev I = B.inst[ch.x];
  const uint4 a = B.tri_idx[t];
  tri_project(B, I, t, B.tri_dm[t], B.tri_w[t], B.pos[a.x], B.pos[a.y], B.pos[a.z]);
}

// Rotation of v = p - centre about `axis` by an angle minus v itself:
// (axis (axis . v) - v)(1 - cos) + (axis x v) sin (bending.rs:231-239), given
// sin and 1 - cos. The two wings turn by +half and -half: the same 1 - cos and
// opposite sines, so one pair of sines serves both.
__device__ __forceinline__ float3 rot_delta(float3 v, float3 axis, float s, float omc) {
  float dt = dot3(axis, v);
  return (axis * dt - v) * omc + cross3(axis, v) * s;
}

// Local bending step of one hinge: w * s . (target - x); only the wings move
// (bending.rs:182-227, discrete_shells.rs:285-337). Compiled once (not
// inlined), so both bending kernels' shapes give bit-identical results.
__device__ __noinline__ float4 hinge_project(float4 st, float2 wr, float3 p0, float3 p1, float3 pa, float3 pb) {
  float3 out = make_float3(0.f, 0.f, 0.f);
  float3 e = p1 - p0;
  float el = len3(e);
  if (el >= 1e-10f) {
    float3 ed = e * (1.f / el);
    float3 ta = pa - p0, tb = pb - p0;
    float3 qa = ta - ed * dot3(ta, ed), qb = tb - ed * dot3(tb, ed);
    float la = len3(qa), lb = len3(qb);
    const float PI = 3.14159265358979323846f;
    float ang = PI;
    if (la >= 1e-10f && lb >= 1e-10f) {
      float c = dot3(qa * (1.f / la), qb * (1.f / lb));
      ang = acosf(fminf(fmaxf(c, -1.f), 1.f));
    }
    float diff = ang - wr.y;
    if (fabsf(diff) >= 1e-8f) {
      float sign = dot3(cross3(qa, qb), ed) >= 0.f ? 1.f : -1.f;
      float half = diff * 0.5f * sign;
      float3 mid = (p0 + p1) * 0.5f;
      const float s = sinf(half), hq = sinf(0.5f * half);
      const float omc = 2.f * hq * hq;  // 1 - cos, without cancellation
      float3 da = rot_delta(pa - mid, ed, s, omc);
      float3 db = rot_delta(pb - mid, ed, -s, omc);
      out = (da * st.z + db * st.w) * wr.x;
    }
  }
  return make_float4(out.x, out.y, out.z, 0.f);
}

// One hinge per thread over a chunk of up to 256 hinges. A garment whose
// stencils are all (-1, -1, 1, 1) skips their load (16 B per hinge), with the
// same products.
__global__ void __launch_bounds__(256) k_hinge(BatchDev B) {
  pdl_begin();
  int4 ch = B.hinge_chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  if (B.prm->ipc && B.red[ch.x].al_done) return;
  uint32_t h = uint32_t(ch.y) + threadIdx.x;
  uint4 id = B.hinge_idx[h];
  const float4 st = B.inst[ch.x].unit_stencils ? make_float4(-1.f, -1.f, 1.f, 1.f) : B.hinge_st[h];
  float2 wr = B.hinge_wr[h];
  B.hinge_out[h] = hinge_project(st, wr, f3(B.pos[id.x]), f3(B.pos[id.y]), f3(B.pos[id.z]), f3(B.pos[id.w]));
}

// Two hinges per thread (128 threads over a chunk of up to 256), both hinges'
// loads issued before either projection: the autotuner's other shape.
__global__ void __launch_bounds__(128, 8) k_hinge2(BatchDev B) {
  pdl_begin();
  int4 ch = B.hinge_chunks[blockIdx.x];
  const uint32_t i0 = threadIdx.x, i1 = threadIdx.x + 128;
  if ((int)i0 >= ch.z) return;
  if (B.prm->ipc && B.red[ch.x].al_done) return;
  const bool two = (int)i1 < ch.z;
  const uint32_t h0 = uint32_t(ch.y) + i0, h1 = two ? uint32_t(ch.y) + i1 : h0;
  const bool unit = B.inst[ch.x].unit_stencils != 0;
  const uint4 a = B.hinge_idx[h0], b = B.hinge_idx[h1];
  const float4 sa = unit ? make_float4(-1.f, -1.f, 1.f, 1.f) : B.hinge_st[h0];
  const float4 sb = unit ? make_float4(-1.f, -1.f, 1.f, 1.f) : B.hinge_st[h1];
  const float2 wa = B.hinge_wr[h0], wb = B.hinge_wr[h1];
  const float3 a0 = f3(B.pos[a.x]), a1 = f3(B.pos[a.y]), a2 = f3(B.pos[a.z]), a3 = f3(B.pos[a.w]);
  const float3 b0 = f3(B.pos[b.x]), b1 = f3(B.pos[b.y]), b2 = f3(B.pos[b.z]), b3 = f3(B.pos[b.w]);
  B.hinge_out[h0] = hinge_project(sa, wa, a0, a1, a2, a3);
  if (two) B.hinge_out[h1] = hinge_project(sb, wb, b0, b1, b2, b3);
}

// Residual gather: r_i = m_i (pred_i / dt^2 - x_i / h^2) + sum of element
// terms [- (mu grad_i + lambda_i)], written in solve (permuted) order.
// keep_rhs also stores r in R0 for a refinement of this iteration's solve.
__global__ void __launch_bounds__(256) k_gather(BatchDev B, int keep_rhs) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  const InstDev I = B.inst[ch.x];
  uint32_t g = uint32_t(ch.y) + threadIdx.x;
  const StepParams& P = *B.prm;
  InstRed& R = B.red[ch.x];
  if (P.ipc && R.al_done) return;
  float m = B.mass[g];
  float3 x = f3(B.pos[g]), q = f3(B.pred[g]);
  float cm = m * I.inv_hmat2, cr = m * P.inv_dt2;
  float3 r = (q - x) * cm + q * (cr - cm);
  // element outputs are read-only here: non-coherent loads, and of a hinge's
  // stencil only this vertex's weight (gather 0.313 -> 0.278 ms per iteration),
  // none where every stencil is (-1, -1, 1, 1): -1 for the edge's ends, 1 for
  // the wings, the same products as the loaded weights
  // the garment's connectivity class's lists (shared by the garments of one
  // mesh topology: read once for all of them, from L2 after the first).
  // Loading the first eight incidences' codes and contributions ahead of the
  // adds was measured slower (62 registers, half the resident warps: 0.264
  // against 0.224 ms per iteration on 512 sheets).
  const uint32_t l = g - I.vbase;
  const uint32_t* tcode = B.vtri + I.tinc_off;
  const uint32_t* hcode = B.vhinge + I.hinc_off;
#pragma unroll 4
  for (uint32_t e = __ldg(B.vtri_ptr + I.inc_ptr + l), ee = __ldg(B.vtri_ptr + I.inc_ptr + l + 1); e < ee; ++e) {
    uint32_t code = __ldg(tcode + e);
    const float* o = B.tri_out + 9ull * (I.tbase + (code >> 2)) + 3 * (code & 3u);
    r.x += __ldg(o); r.y += __ldg(o + 1); r.z += __ldg(o + 2);
  }
#pragma unroll 4
  for (uint32_t e = __ldg(B.vhinge_ptr + I.inc_ptr + l), ee = __ldg(B.vhinge_ptr + I.inc_ptr + l + 1); e < ee; ++e) {
    uint32_t code = __ldg(hcode + e);
    uint32_t h = I.hbase + (code >> 2), k = code & 3u;
    float s = I.unit_stencils ? (k < 2u ? -1.f : 1.f) : __ldg(reinterpret_cast<const float*>(B.hinge_st + h) + k);
    float4 o = __ldg(B.hinge_out + h);
    r.x += s * o.x; r.y += s * o.y; r.z += s * o.z;
  }
  if (P.ipc) {  // assemble_barrier_rhs (assembly.rs:272-282)
    float mu = R.mu;
    float4 gr = B.grad[g], la = B.lam[g];
    r.x -= mu * gr.x + la.x; r.y -= mu * gr.y + la.y; r.z -= mu * gr.z + la.z;
  }
  const uint32_t row = I.vbase + B.perm_local[g];
  B.Y[row] = make_float4(r.x, r.y, r.z, 0.f);
  if (keep_rhs) B.R0[row] = make_float4(r.x, r.y, r.z, 0.f);
}

__device__ __forceinline__ void f4_fma(float4& t, float a, float4 y) {
  t.x += a * y.x; t.y += a * y.y; t.z += a * y.z;
}
__device__ __forceinline__ float4 f4_sub(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, 0.f);
}
__device__ __forceinline__ float4 f4_add(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, 0.f);
}

// Shared-memory sizing of the sweep kernels: each warp owns a staging buffer of
// kWarpFloats floats and kWarpVec float4 vector slots; a narrow level uses
// all of them as one block-wide buffer.
constexpr uint32_t kSolveWarps = 8;
// Sized so that five 256-thread blocks fit an SM (45 KB each): the sweeps
// are bound by the latency of global loads, so warps in flight matter more
// than larger staging buffers.
constexpr uint32_t kWarpFloats = 1024;
constexpr uint32_t kWarpVec = 32;
constexpr uint32_t kSolveSmem = kSolveWarps * (kWarpFloats * 4 + 3 * kWarpVec * 16);
// Blocks per SM the sweep kernels are compiled for (registers of a 256-thread
// block at most 65536 / 5): shared memory admits five.
constexpr int kSolveMinBlocks = 5;
constexpr uint32_t kMaxSupernode = 256;  // enforced by the host set-up
// A supernode is a warp item when its vectors and diagonal block fit a warp's
// slots and its block is small; larger ones get a whole block.
// Default limit of s (s + m) for a warp item; vistio_batch_tune picks one per batch.
constexpr uint32_t kWarpItemLimit = 6144;
__host__ __device__ constexpr bool warp_item(uint32_t s, uint32_t m, uint32_t limit = kWarpItemLimit) {
  return s <= kWarpVec && uint64_t(s) * (s + m) <= limit;
}

// ------------------------------------------------ TMA bulk staging
// A contiguous global range is brought into shared memory with one
// cp.async.bulk (TMA) whose completion is tracked by an mbarrier
// transaction count. Waits are bounded: after kWaitLimit polls the team
// records VISTIO timeout status bit 2 and stops using the data.
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One thread: expect `bytes` on the barrier and start the bulk copy. Callers
// reconverge the issuing warp (__syncwarp) before any lane polls the barrier:
// a warp whose other lanes spin in mbar_wait while the issuing lane sits on
// the other side of a branch was seen to run the spinning side until its poll
// budget ran out, the copy never issued.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kWaitLimit) {
  const uint32_t b = smem_u32(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Diagnostic of the failure path: the sweeps' bounded wait on a barrier that
// nothing completes gives up after `polls` polls and records the timeout
// status bit, as a sweep whose staging copy never lands does.
__global__ void k_diag_wait(uint32_t* status, uint32_t polls) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar);
  mbar_fence_init();
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0u, polls)) atomicOr(status, 4u);
}

// A team is either one warp (a supernode per warp) or the whole block.
struct Team {
  uint32_t rank, size;
  float* buf;      // staging buffer (16-byte aligned)
  uint32_t cap;    // floats in buf
  float4* v0;      // vector slots (s entries each) ...
  float4* v1;
  float4* xg;      // gathered ancestor values, xcap entries
  uint32_t vcap, xcap;
  bool block;
  uint64_t* bar;   // mbarrier of this team's staging buffer
  uint32_t parity; // phase of the next completion
  uint32_t* abort; // shared flag: a bounded wait gave up
  __device__ __forceinline__ void sync() const {
    if (block) __syncthreads();
    else __syncwarp();
  }
};

// Brings floats [src, src + n) into the team buffer with one bulk copy of the
// enclosing 16-byte aligned window (the vals pool is padded so the window
// never leaves the allocation); returns where src[0] landed. Ends with the
// team synchronised and the data visible.
__device__ __forceinline__ const float* stage(Team& tm, const float* __restrict__ src, uint32_t n,
                                              uint32_t* status) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const uintptr_t lo = a & ~uintptr_t(15);
  const uintptr_t hi = (a + uintptr_t(n) * 4 + 15) & ~uintptr_t(15);
  tm.sync();  // previous readers of the buffer are done
  if (tm.rank == 0) bulk_g2s(tm.buf, reinterpret_cast<const void*>(lo), uint32_t(hi - lo), tm.bar);
  __syncwarp();  // the issuing lane first: polling lanes must not starve it
  bool ok = mbar_wait(tm.bar, tm.parity);
  tm.parity ^= 1u;
  if (!ok) {
    atomicOr(status, 4u);
    *tm.abort = 1u;
  }
  return tm.buf + (a - lo) / 4;
}

// The same copy in two halves, so that other work overlaps it: stage_issue
// starts the copy (after the team's previous readers of the buffer are done),
// stage_wait waits for it (bounded) and returns where src[0] landed.
__device__ __forceinline__ void stage_issue(Team& tm, const float* __restrict__ src, uint32_t n) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const uintptr_t lo = a & ~uintptr_t(15);
  const uintptr_t hi = (a + uintptr_t(n) * 4 + 15) & ~uintptr_t(15);
  tm.sync();
  if (tm.rank == 0) bulk_g2s(tm.buf, reinterpret_cast<const void*>(lo), uint32_t(hi - lo), tm.bar);
  __syncwarp();
}
__device__ __forceinline__ const float* stage_wait(Team& tm, const float* __restrict__ src, uint32_t* status) {
  const bool ok = mbar_wait(tm.bar, tm.parity);
  tm.parity ^= 1u;
  if (!ok) {
    atomicOr(status, 4u);
    *tm.abort = 1u;
  }
  return tm.buf + (reinterpret_cast<uintptr_t>(src) & 15) / 4;
}

// Pull for the rows of supernode S: t = r - sum of the updates U that its
// descendants pushed (lanes / threads over columns).
__device__ __forceinline__ void sn_pull(const BatchDev& B, const Team& tm, const SnDev& S, const float4* Y) {
  const uint32_t s = S.ncols, f = S.first, vb = S.vbase;
  for (uint32_t c = tm.rank; c < s; c += tm.size) {
    float4 t = Y[f + c];
    uint32_t q = B.fwd_ptr[vb + f + c], qe = B.fwd_ptr[vb + f + c + 1];
#pragma unroll 4
    for (; q < qe; ++q) t = f4_sub(t, __ldcg(B.U + B.fwd[q]));
    tm.v0[c] = t;
  }
}

// y = inv(L_kk) t with the whole diagonal block in shared memory (Ds, column-major).
__device__ __forceinline__ void sn_diag_fwd_smem(const Team& tm, const SnDev& S, const float* Ds, float4* Y) {
  const uint32_t s = S.ncols, f = S.first, ld = sn_ld(s);
  for (uint32_t c = tm.rank; c < s; c += tm.size) {
    float4 y = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t c2 = 0; c2 <= c; ++c2) f4_fma(y, Ds[c2 * ld + c], tm.v0[c2]);
    tm.v1[c] = y;
    Y[f + c] = y;
  }
}

// U[j] = P[j,:] . y for nr rows staged at Ps (row-major, s columns).
__device__ __forceinline__ void sn_push_rows(const BatchDev& B, const Team& tm, const SnDev& S, const float* Ps,
                                             uint32_t j0, uint32_t nr) {
  const uint32_t s = S.ncols, ld = sn_ld(s);
  for (uint32_t j = tm.rank; j < nr; j += tm.size) {
    float4 u = make_float4(0.f, 0.f, 0.f, 0.f);
    const float* row = Ps + j * ld;
    for (uint32_t c = 0; c < s; ++c) f4_fma(u, row[c], tm.v1[c]);
    B.U[S.u_off + (j0 + j) * S.u_stride] = u;
  }
}

// Forward step of one supernode: pull, y = inv(L_kk) t, push U = P y. The
// diagonal block and the panel are staged through the team buffer (the
// block in column chunks when it does not fit, the panel in row chunks).
__device__ __forceinline__ void sn_forward(const BatchDev& B, Team& tm, const SnDev& S) {
  const uint32_t s = S.ncols, m = S.nrows, f = S.first, ld = sn_ld(s);
  float4* Y = B.Y + S.vbase;
  const float* D = B.vals + S.d_off;
  const float* Pp = B.vals + S.p_off;
  const uint32_t whole = uint32_t(S.p_off - S.d_off) + m * ld + m;  // [D | P | rows] is one contiguous region
  if (whole + 8 <= tm.cap) {
    // the whole supernode in one copy, in flight while the pull gathers
    stage_issue(tm, D, whole);
    sn_pull(B, tm, S, Y);
    const float* Ds = stage_wait(tm, D, B.status);
    tm.sync();
    sn_diag_fwd_smem(tm, S, Ds, Y);
    tm.sync();
    if (m) sn_push_rows(B, tm, S, Ds + (S.p_off - S.d_off), 0, m);
    tm.sync();
    return;
  }
  sn_pull(B, tm, S, Y);
  if (s * ld + 8 <= tm.cap) {
    const float* Ds = stage(tm, D, s * ld, B.status);
    tm.sync();
    sn_diag_fwd_smem(tm, S, Ds, Y);
  } else {
    // column chunks [c0, c1) of D; y accumulates in v1
    for (uint32_t c = tm.rank; c < s; c += tm.size) tm.v1[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t cw = max(1u, (tm.cap - 8) / ld);
    for (uint32_t c0 = 0; c0 < s; c0 += cw) {
      uint32_t c1 = min(s, c0 + cw);
      const float* Dc = stage(tm, D + uint64_t(c0) * ld, (c1 - c0) * ld, B.status);
      for (uint32_t c = c0 + tm.rank; c < s; c += tm.size) {
        float4 y = tm.v1[c];
        uint32_t ce = min(c1, c + 1);
        for (uint32_t c2 = c0; c2 < ce; ++c2) f4_fma(y, Dc[(c2 - c0) * ld + c], tm.v0[c2]);
        tm.v1[c] = y;
      }
    }
    tm.sync();
    for (uint32_t c = tm.rank; c < s; c += tm.size) Y[f + c] = tm.v1[c];
  }
  tm.sync();
  if (m == 0) return;
  const uint32_t rc = max(1u, (tm.cap - 8) / ld);
  for (uint32_t j0 = 0; j0 < m; j0 += rc) {
    uint32_t nr = min(rc, m - j0);
    const float* Ps = stage(tm, Pp + uint64_t(j0) * ld, nr * ld, B.status);
    sn_push_rows(B, tm, S, Ps, j0, nr);
  }
  tm.sync();
}

// Team-wide sums over row slices: thread (cl, part) of a (width x parts)
// split holds acc for column cb + cl; column sums land in out[cb + cl].
__device__ __forceinline__ void team_column_sum(const Team& tm, float4 acc, uint32_t width, uint32_t parts,
                                                uint32_t cb, uint32_t s, const float4* base, float4* out,
                                                bool subtract) {
  const uint32_t cl = tm.rank % width, part = tm.rank / width;
  if (!tm.block) {
    for (uint32_t o = width; o < 32; o <<= 1) {
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
      acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
    }
    if (part == 0 && cb + cl < s) out[cb + cl] = subtract ? f4_sub(base[cb + cl], acc) : acc;
  } else {
    float4* red = tm.xg;  // xcap >= block size
    tm.sync();
    red[tm.rank] = acc;
    tm.sync();
    if (tm.rank < width && cb + tm.rank < s) {
      float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
      for (uint32_t q = 0; q < parts; ++q) a = f4_add(a, red[q * width + tm.rank]);
      out[cb + tm.rank] = subtract ? f4_sub(base[cb + tm.rank], a) : a;
    }
  }
  tm.sync();
}

__device__ __forceinline__ uint32_t team_width(const Team& tm, uint32_t s) {
  uint32_t width = 1;
  while (width < s && width < tm.size) width <<= 1;
  return width;
}

// x = inv(L_kk)^T t with the whole diagonal block in shared memory (Ds).
__device__ __forceinline__ void sn_diag_bwd_smem(const Team& tm, const SnDev& S, const float* Ds, float4* Y) {
  const uint32_t s = S.ncols, f = S.first, ld = sn_ld(s);
  for (uint32_t c = tm.rank; c < s; c += tm.size) {
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t c2 = c; c2 < s; ++c2) f4_fma(x, Ds[c * ld + c2], tm.v0[c2]);
    Y[f + c] = x;
  }
}

// Backward step of one supernode with a warp team: t = y - P^T x[R];
// x = inv(L_kk)^T t. Lane c < s owns column c and forms its sum over the panel
// rows j in ascending order (one FMA chain from zero), then x_c = sum over
// c2 = c .. s-1 of inv(L_kk)(c2, c) t_c2, again ascending: the same order the
// garment-grouped sweep (one lane per garment) uses, so the two give the same
// bits. Rows arrive in chunks (their x gathered into xg, the panel staged
// whole or by row chunks); the order of the sums does not depend on the chunks.
__device__ __forceinline__ void sn_backward_warp(const BatchDev& B, Team& tm, const SnDev& S) {
  const uint32_t s = S.ncols, m = S.nrows, f = S.first, ld = sn_ld(s);
  float4* Y = B.Y + S.vbase;
  const float* D = B.vals + S.d_off;
  const float* Pp = B.vals + S.p_off;
  const uint32_t* Rr = B.rows + S.rows_off;
  const uint32_t c = tm.rank;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  // own columns through L2: the forward sweep may have written them in this
  // launch, on another SM
  const float4 yc = c < s ? __ldcg(Y + f + c) : acc;
  const uint32_t whole = uint32_t(S.p_off - S.d_off) + m * ld + m;  // [D | P | rows] is one contiguous region
  const float* Ds = nullptr;
  if (whole + 8 <= tm.cap) {
    // the whole supernode in one copy, in flight while the first chunk of
    // x[R] is gathered
    stage_issue(tm, D, whole);
    for (uint32_t j0 = 0; j0 < m; j0 += tm.xcap) {
      const uint32_t nr = min(tm.xcap, m - j0);
      __syncwarp();
      for (uint32_t j = tm.rank; j < nr; j += tm.size) tm.xg[j] = __ldcg(Y + Rr[j0 + j]);
      if (!Ds) Ds = stage_wait(tm, D, B.status);
      __syncwarp();
      if (c < s) {
        const float* P0 = Ds + (S.p_off - S.d_off) + size_t(j0) * ld + c;
        for (uint32_t j = 0; j < nr; ++j) f4_fma(acc, P0[j * ld], tm.xg[j]);
      }
    }
    if (!Ds) Ds = stage_wait(tm, D, B.status);
    __syncwarp();
    if (c < s) tm.v0[c] = f4_sub(yc, acc);
    __syncwarp();
    sn_diag_bwd_smem(tm, S, Ds, Y);
    __syncwarp();
    return;
  }
  const uint32_t rc = max(1u, min((tm.cap - 8) / ld, tm.xcap));
  for (uint32_t j0 = 0; j0 < m; j0 += rc) {
    const uint32_t nr = min(rc, m - j0);
    __syncwarp();  // previous readers of xg are done
    for (uint32_t j = tm.rank; j < nr; j += tm.size) tm.xg[j] = __ldcg(Y + Rr[j0 + j]);
    const float* Ps = stage(tm, Pp + uint64_t(j0) * ld, nr * ld, B.status);
    __syncwarp();
    if (c < s)
      for (uint32_t j = 0; j < nr; ++j) f4_fma(acc, Ps[j * ld + c], tm.xg[j]);
  }
  __syncwarp();
  if (c < s) tm.v0[c] = f4_sub(yc, acc);
  __syncwarp();
  if (s * ld + 8 <= tm.cap) {
    Ds = stage(tm, D, s * ld, B.status);
    __syncwarp();
    sn_diag_bwd_smem(tm, S, Ds, Y);
  } else {
    // column chunks of D: x_c needs only column c (rows c .. s-1)
    const uint32_t cw = max(1u, (tm.cap - 8) / ld);
    for (uint32_t c0 = 0; c0 < s; c0 += cw) {
      const uint32_t c1 = min(s, c0 + cw);
      const float* Dc = stage(tm, D + uint64_t(c0) * ld, (c1 - c0) * ld, B.status);
      if (c >= c0 && c < c1) {
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        for (uint32_t c2 = c; c2 < s; ++c2) f4_fma(x, Dc[(c - c0) * ld + c2], tm.v0[c2]);
        Y[f + c] = x;
      }
    }
  }
  __syncwarp();
}

// Backward step of one supernode: t = y - P^T x[R]; x = inv(L_kk)^T t. A
// block team splits each column's sum over parts of the rows and adds the
// parts in a fixed order.
__device__ __forceinline__ void sn_backward(const BatchDev& B, Team& tm, const SnDev& S) {
  if (!tm.block) {
    sn_backward_warp(B, tm, S);
    return;
  }
  const uint32_t s = S.ncols, m = S.nrows, f = S.first, ld = sn_ld(s);
  float4* Y = B.Y + S.vbase;
  const float* D = B.vals + S.d_off;
  const float* Pp = B.vals + S.p_off;
  const uint32_t* Rr = B.rows + S.rows_off;
  const uint32_t whole = uint32_t(S.p_off - S.d_off) + m * ld + m;
  if (whole + 8 <= tm.cap) {
    // the whole supernode in one copy, in flight while y and the first
    // chunk of x[R] are gathered; columns in at most two rounds of the team
    // width (warp items have s <= kWarpVec, block items s <= 256 <= the block width)
    stage_issue(tm, D, whole);
    // own columns through L2: the forward sweep may have written them in
    // this launch, on another SM
    for (uint32_t c = tm.rank; c < s; c += tm.size) tm.v1[c] = __ldcg(Y + f + c);
    const uint32_t width = team_width(tm, s), parts = tm.size / width;
    const uint32_t cl = tm.rank % width, part = tm.rank / width;
    float4 sum0 = make_float4(0.f, 0.f, 0.f, 0.f), sum1 = sum0;
    const float* Ds = nullptr;
    for (uint32_t j0 = 0; j0 < m; j0 += tm.xcap) {
      const uint32_t nr = min(tm.xcap, m - j0);
      tm.sync();
      for (uint32_t j = tm.rank; j < nr; j += tm.size) tm.xg[j] = __ldcg(Y + Rr[j0 + j]);
      if (!Ds) Ds = stage_wait(tm, D, B.status);
      tm.sync();
      if (part < parts) {
        const float* P0 = Ds + (S.p_off - S.d_off) + size_t(j0) * ld;
        if (cl < s)
          for (uint32_t j = part; j < nr; j += parts) f4_fma(sum0, P0[j * ld + cl], tm.xg[j]);
        if (width + cl < s)
          for (uint32_t j = part; j < nr; j += parts) f4_fma(sum1, P0[j * ld + width + cl], tm.xg[j]);
      }
    }
    if (!Ds) Ds = stage_wait(tm, D, B.status);
    tm.sync();
    team_column_sum(tm, sum0, width, parts, 0, s, tm.v1, tm.v0, true);
    if (width < s) team_column_sum(tm, sum1, width, parts, width, s, tm.v1, tm.v0, true);
    sn_diag_bwd_smem(tm, S, Ds, Y);
    tm.sync();
    return;
  }
  for (uint32_t c = tm.rank; c < s; c += tm.size) tm.v1[c] = __ldcg(Y + f + c);
  const uint32_t width = team_width(tm, s);
  const uint32_t parts = tm.size / width;
  const uint32_t cl = tm.rank % width, part = tm.rank / width;
  const uint32_t rc = max(1u, min((tm.cap - 8) / ld, tm.xcap));
  for (uint32_t cb = 0; cb < s; cb += width) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t c = cb + cl;
    for (uint32_t j0 = 0; j0 < m; j0 += rc) {
      uint32_t nr = min(rc, m - j0);
      tm.sync();  // previous readers of xg are done
      for (uint32_t j = tm.rank; j < nr; j += tm.size) tm.xg[j] = __ldcg(Y + Rr[j0 + j]);
      const float* Ps = stage(tm, Pp + uint64_t(j0) * ld, nr * ld, B.status);
      tm.sync();
      if (c < s && part < parts)
        for (uint32_t j = part; j < nr; j += parts) f4_fma(acc, Ps[j * ld + c], tm.xg[j]);
    }
    tm.sync();
    team_column_sum(tm, acc, width, parts, cb, s, tm.v1, tm.v0, true);
  }
  if (s * ld + 8 <= tm.cap) {
    const float* Ds = stage(tm, D, s * ld, B.status);
    tm.sync();
    sn_diag_bwd_smem(tm, S, Ds, Y);
  } else {
    // column chunks of D: x_c needs column c (rows c..s-1)
    const uint32_t cw = max(1u, (tm.cap - 8) / ld);
    for (uint32_t c0 = 0; c0 < s; c0 += cw) {
      uint32_t c1 = min(s, c0 + cw);
      const float* Dc = stage(tm, D + uint64_t(c0) * ld, (c1 - c0) * ld, B.status);
      // a chunk can be wider than the team: columns in rounds of the team width
      const uint32_t w = team_width(tm, c1 - c0), np = tm.size / w;
      const uint32_t ccl = tm.rank % w, pp = tm.rank / w;
      for (uint32_t cb = c0; cb < c1; cb += w) {
        const uint32_t cc = cb + ccl;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        if (cc < c1 && pp < np)
          for (uint32_t r = cc + pp; r < s; r += np) f4_fma(acc, Dc[(cc - c0) * ld + r], tm.v0[r]);
        team_column_sum(tm, acc, w, np, cb, c1, nullptr, Y + f, false);
      }
    }
  }
  tm.sync();
}

// The supernodes [first, last] of one bottom subtree, swept by one warp in
// postorder (forward) or reverse postorder (backward). The subtree's columns
// [c0, c1) are contiguous and every update to them comes from inside the
// subtree, so its slice of the vector stays in shared memory (acc) for the
// whole sweep: the forward sweep pulls nothing from global memory and pushes
// only the updates bound for rows above the subtree (U slots that the top
// levels pull); the backward sweep reads global memory only for the final
// values of those rows. The factor data arrives with one bulk copy, issued
// before the vector slice is loaded so that the two overlap.
template <int DIR>
__device__ __forceinline__ void subtree_sweep(const BatchDev& B, Team& tm, uint32_t first, uint32_t last) {
  const SnDev F = B.sn[first], Lz = B.sn[last];
  const uint64_t end = Lz.p_off + ((uint64_t(Lz.nrows) * sn_ld(Lz.ncols) + Lz.nrows + 3) & ~3ull);
  const float* src = B.vals + F.d_off;  // 16-byte aligned: d_off is a multiple of 4
  const uint32_t bytes = uint32_t(end - F.d_off) * 4u;
  tm.sync();  // previous readers of the buffer are done
  if (tm.rank == 0) bulk_g2s(tm.buf, src, bytes, tm.bar);
  __syncwarp();
  const uint32_t c0 = F.first, c1 = Lz.first + Lz.ncols, nc = c1 - c0;
  float4* Yg = B.Y + F.vbase;
  float4* acc = tm.v1;  // rows c0 .. c1 of this instance (nc <= vcap, enforced by the set-up)
  for (uint32_t c = tm.rank; c < nc; c += tm.size) acc[c] = __ldcg(Yg + c0 + c);  // possibly written this launch
  const bool ok = mbar_wait(tm.bar, tm.parity);
  tm.parity ^= 1u;
  if (!ok) {
    atomicOr(B.status, 4u);
    *tm.abort = 1u;
  }
  tm.sync();
  const float* base = tm.buf;
  for (uint32_t i = 0; i <= last - first; ++i) {
    const uint32_t k = DIR == 0 ? first + i : last - i;
    const SnDev S = B.sn[k];
    const float* Ds = base + (S.d_off - F.d_off);
    const float* Ps = base + (S.p_off - F.d_off);
    const uint32_t s = S.ncols, m = S.nrows, f = S.first - c0, ld = sn_ld(s);
    const uint32_t* Rr = reinterpret_cast<const uint32_t*>(Ps + m * ld);  // staged with the panel
    if (DIR == 0) {
      // t = acc (all descendant updates are in); y = inv(L_kk) t into acc
      for (uint32_t c = tm.rank; c < s; c += tm.size) tm.v0[c] = acc[f + c];
      tm.sync();
      for (uint32_t c = tm.rank; c < s; c += tm.size) {
        float4 y = make_float4(0.f, 0.f, 0.f, 0.f);
        for (uint32_t c2 = 0; c2 <= c; ++c2) f4_fma(y, Ds[c2 * ld + c], tm.v0[c2]);
        acc[f + c] = y;
      }
      tm.sync();
      // u_j = P[j,:] . y: into acc for rows of the subtree (distinct rows per
      // j, all below this supernode's block), else into the row's U slot
      for (uint32_t j = tm.rank; j < m; j += tm.size) {
        const uint32_t r = Rr[j];
        float4 u = make_float4(0.f, 0.f, 0.f, 0.f);
        const float* row = Ps + j * ld;
        for (uint32_t c = 0; c < s; ++c) f4_fma(u, row[c], acc[f + c]);
        if (r < c1) acc[r - c0] = f4_sub(acc[r - c0], u);
        else B.U[S.u_off + j * S.u_stride] = u;
      }
      tm.sync();
    } else {
      // t = y - P^T x[R] (x of rows in the subtree from acc, above it from Y),
      // the gathered x in chunks of xcap rows; lane c < s sums column c over
      // the rows in ascending order
      float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
      const uint32_t c = tm.rank;
      for (uint32_t j0 = 0; j0 < m; j0 += tm.xcap) {
        const uint32_t nr = min(tm.xcap, m - j0);
        tm.sync();
        for (uint32_t j = tm.rank; j < nr; j += tm.size) {
          const uint32_t r = Rr[j0 + j];
          tm.xg[j] = r < c1 ? acc[r - c0] : __ldcg(Yg + r);
        }
        tm.sync();
        if (c < s) {
          const float* P0 = Ps + size_t(j0) * ld + c;
          for (uint32_t j = 0; j < nr; ++j) f4_fma(sum, P0[j * ld], tm.xg[j]);
        }
      }
      tm.sync();
      if (c < s) tm.v0[c] = f4_sub(acc[f + c], sum);
      tm.sync();
      // x = inv(L_kk)^T t into acc
      for (uint32_t c = tm.rank; c < s; c += tm.size) {
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        for (uint32_t c2 = c; c2 < s; ++c2) f4_fma(x, Ds[c * ld + c2], tm.v0[c2]);
        acc[f + c] = x;
      }
      tm.sync();
    }
  }
  for (uint32_t c = tm.rank; c < nc; c += tm.size) Yg[c0 + c] = acc[c];
}

// Shared-memory teams of one sweep kernel block: one team per warp and, over
// the same memory, the block team, and bn: the block supernodes' backward
// team, the first eight warps' worth of threads and buffer (in an eight-warp
// block the same as bt, on its own mbarrier). The backward step of a block
// supernode splits each column's sum over parts of the rows, and how depends
// on the team's width and buffer; with bn it is the same in every compiled
// form of k_sweep, and the results stay bit-identical. (The forward step's
// sums do not depend on the team.)
struct SweepTeams {
  Team wt, bt, bn;
};
template <uint32_t NW = kSolveWarps>
__device__ __forceinline__ SweepTeams make_teams(float4* smem4, uint64_t* s_bar, uint32_t* s_abort) {
  constexpr uint32_t NT = 32 * NW;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float* fbuf = reinterpret_cast<float*>(smem4);
  float4* vbuf = smem4 + NW * kWarpFloats / 4;
  if (tid <= NW + 1) mbar_init(&s_bar[tid]);
  if (tid == 0) *s_abort = 0u;
  mbar_fence_init();
  __syncthreads();
  SweepTeams t;
  t.wt = Team{lane, 32, fbuf + warp * kWarpFloats, kWarpFloats, vbuf + warp * 3 * kWarpVec,
              vbuf + warp * 3 * kWarpVec + kWarpVec, vbuf + warp * 3 * kWarpVec + 2 * kWarpVec, kWarpVec, kWarpVec,
              false, &s_bar[warp], 0u, s_abort};
  // block team: all warps' buffers; the vector slots split kMaxSupernode /
  // kMaxSupernode / NT (xg doubles as the NT-entry reduction buffer).
  static_assert(3 * kWarpVec * NW >= 2 * kMaxSupernode + NT, "block-team vector slots");
  t.bt = Team{tid, NT, fbuf, NW * kWarpFloats, vbuf, vbuf + kMaxSupernode, vbuf + 2 * kMaxSupernode, kMaxSupernode, NT,
              true, &s_bar[NW], 0u, s_abort};
  // threads beyond the first eight warps take no part in bn's loops (their
  // rank is beyond its size) but keep its barriers
  constexpr uint32_t NR = 32 * kSolveWarps;
  t.bn = Team{tid, NR, fbuf, kSolveWarps * kWarpFloats, vbuf, vbuf + kMaxSupernode, vbuf + 2 * kMaxSupernode,
              kMaxSupernode, NR, true, &s_bar[NW + 1], 0u, s_abort};
  return t;
}

// One level of the forward (DIR = 0) or backward (DIR = 1) sweep over every
// instance of the batch. The level's supernodes (across instances) are listed
// with those too large for a warp first: blocks [0, nblock) take one of those
// each with the whole block; the remaining blocks take eight of the rest, one
// per warp. Supernodes of a level are independent; levels are ordered by
// kernel boundaries.
template <int DIR>
__global__ void __launch_bounds__(32 * kSolveWarps, kSolveMinBlocks) k_level(BatchDev B, uint32_t off, uint32_t nblock, uint32_t nwarp) {
  pdl_begin();
  extern __shared__ float4 smem4[];
  __shared__ uint64_t s_bar[kSolveWarps + 2];
  __shared__ uint32_t s_abort;
  SweepTeams t = make_teams(smem4, s_bar, &s_abort);
  const bool ipc = B.prm->ipc != 0;
  if (blockIdx.x < nblock) {
    SnDev S = B.sn[B.lvl_items[off + blockIdx.x]];
    if (ipc && B.red[S.inst].al_done) return;
    if (DIR == 0) sn_forward(B, t.bt, S);
    else sn_backward(B, t.bt, S);
  } else {
    uint32_t q = (blockIdx.x - nblock) * kSolveWarps + (threadIdx.x >> 5);
    if (q >= nwarp) return;
    SnDev S = B.sn[B.lvl_items[off + nblock + q]];
    if (ipc && B.red[S.inst].al_done) return;
    if (DIR == 0) sn_forward(B, t.wt, S);
    else sn_backward(B, t.wt, S);
  }
}

// Bottom subtrees of every instance, one per warp.
template <int DIR>
__global__ void __launch_bounds__(32 * kSolveWarps, kSolveMinBlocks) k_subtree(BatchDev B, uint32_t nitems) {
  pdl_begin();
  extern __shared__ float4 smem4[];
  __shared__ uint64_t s_bar[kSolveWarps + 2];
  __shared__ uint32_t s_abort;
  SweepTeams t = make_teams(smem4, s_bar, &s_abort);
  uint32_t q = blockIdx.x * kSolveWarps + (threadIdx.x >> 5);
  if (q >= nitems) return;
  uint2 it = B.sub_items[q];
  if (B.prm->ipc && B.red[B.sn[it.x].inst].al_done) return;
  subtree_sweep<DIR>(B, t.wt, it.x, it.y);
}

// Clears the per-instance residual sums before a sweep.
// ---------------------------------------------- dependency-driven sweeps
// One launch per direction instead of one per level. Blocks stay resident and
// take work units from a global queue in a topological order of the
// supernodal tree (forward: bottom subtrees, then the top levels upwards;
// backward: the reverse), so a unit only waits for units handed out before
// it, whose blocks are running: no deadlock whatever the number of resident
// blocks. A unit waits for its own inputs only, not for the whole level
// below it:
//   forward   a top supernode waits until all its children have pushed their
//             updates (df_cnt counts them), then counts itself in at its parent;
//   backward  a supernode or bottom subtree waits until its parent has its
//             final values (df_flag), then flags its own children.
// A waiting supernode resets its counter once the wait is over (no one
// writes it again in this sweep), so the counters are zero between sweeps.
// Writers fence before they signal; readers of data produced in the same
// launch (U, ancestors' Y) load it through L2 (__ldcg). Every wait is
// bounded; a wait that gives up sets status bit 4, and every later wait
// returns at once, so a failing sweep ends quickly with the error recorded.
//
// Items per unit of bottom subtrees or warp supernodes: the block's eight
// warps take them one at a time, each its next item as soon as it is done
// with the last, so a unit lasts about two items rather than the slowest of
// eight.
constexpr uint32_t kUnitItems = 16;
// The sixteen-warp form of k_sweep: its units hold twice as many items, and
// untuned batches of at most this many garments use it.
constexpr uint32_t kWideWarps = 16;
constexpr uint32_t kWideMaxInstances = 8;
// SweepUnit (uint2): x = kind | count << 2; kind 0: `count` bottom subtrees
// from sub_items[y]; kind 1: the top supernode y with the whole block; kind
// 2: `count` top supernodes, one per warp, from lvl_items[y].
constexpr uint32_t kNoParent = 0xffffffffu;
constexpr uint32_t kDepPolls = 1u << 21;

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits (bounded) until *word >= target; false if it gave up or an earlier
// wait of the batch did.
__device__ __forceinline__ bool dep_wait(const BatchDev& B, const uint32_t* word, uint32_t target) {
  for (uint32_t it = 0; it < kDepPolls; ++it) {
    if (ld_acquire_u32(word) >= target) return true;
    if ((it & 31u) == 31u && (*reinterpret_cast<volatile uint32_t*>(B.status) & 4u)) return false;
    __nanosleep(64);
  }
  atomicOr(B.status, 4u);
  return false;
}

// Forward: wait for the children of supernode k; backward: for its parent's
// backward, or for a root its own forward (both sweeps share one launch).
template <int DIR>
__device__ __forceinline__ void dep_enter(const BatchDev& B, uint32_t k) {
  if (DIR == 0) {
    const uint32_t need = B.df_nkids[k];
    if (need && dep_wait(B, B.df_cnt + k, need)) B.df_cnt[k] = 0u;
  } else if (dep_wait(B, B.df_flag + k, 1u)) {
    B.df_flag[k] = 0u;
  }
}

// Forward: count k in at its parent (a root releases its own backward);
// backward: release k's children (lanes `rank` of `size` share the children).
template <int DIR>
__device__ __forceinline__ void dep_leave(const BatchDev& B, uint32_t k, uint32_t rank, uint32_t size) {
  if (DIR == 0) {
    const uint32_t p = B.df_parent[k];
    if (rank == 0) {
      if (p != kNoParent) atomicAdd(B.df_cnt + p, 1u);
      else atomicExch(B.df_flag + k, 1u);
    }
  } else {
    for (uint32_t q = B.df_kid_ptr[k] + rank, qe = B.df_kid_ptr[k + 1]; q < qe; q += size)
      atomicExch(B.df_flag + B.df_kids[q], 1u);
  }
}

// One work unit of the dependency-driven sweeps (the whole block runs it).
template <int DIR>
__device__ __forceinline__ void sweep_unit(const BatchDev& B, SweepTeams& t, uint2 u, bool ipc, uint32_t* next) {
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t kind = u.x & 3u, count = u.x >> 2;
  if (kind == 1) {
    const uint32_t k = u.y;
    const SnDev S = B.sn[k];
    if (ipc && B.red[S.inst].al_done) return;
    if (tid == 0) dep_enter<DIR>(B, k);
    __syncthreads();
    if (DIR == 0) sn_forward(B, t.bt, S);
    else sn_backward(B, t.bn, S);
    // one fence after the barrier covers the whole block's writes (the fence
    // is cumulative over what the barrier ordered before it); then signal
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      dep_leave<DIR>(B, k, 0, 1);
    }
  } else {
    // warp w takes item w, then the unit's next free item until none is left
    for (uint32_t i = warp; i < count;) {
      if (kind == 0) {
        const uint2 it = B.sub_items[u.y + i];
        if (!(ipc && B.red[B.sn[it.x].inst].al_done)) {
          if (DIR == 1 && lane == 0) dep_enter<1>(B, it.y);
          __syncwarp();
          subtree_sweep<DIR>(B, t.wt, it.x, it.y);
          __syncwarp();
          if (DIR == 0 && lane == 0) {
            __threadfence();
            dep_leave<0>(B, it.y, 0, 1);
          }
        }
      } else {
        const uint32_t k = (DIR == 0 ? B.df_items_fwd : B.lvl_items)[u.y + i];
        const SnDev S = B.sn[k];
        if (!(ipc && B.red[S.inst].al_done)) {
          if (lane == 0) dep_enter<DIR>(B, k);
          __syncwarp();
          if (DIR == 0) sn_forward(B, t.wt, S);
          else sn_backward(B, t.wt, S);
          __syncwarp();
          if (lane == 0) {
            __threadfence();
            dep_leave<DIR>(B, k, 0, 1);
          }
        }
      }
      uint32_t nxt = 0;
      if (lane == 0) nxt = atomicAdd(next, 1u);
      i = __shfl_sync(0xffffffffu, nxt, 0);
    }
  }
}

// Both dependency-driven sweeps in one launch: resident blocks take the
// forward units (top supernodes deepest first), then the backward units (the
// level order from the top). A unit waits only for units handed out before
// it: in the forward sweep for its children, in the backward sweep for its
// parent's backward or, at a root, for its own forward. So a garment's
// backward sweep starts as soon as its own forward sweep ends, beside the
// forward tail of the others. The last block out resets the queue.
//
// Compiled in three forms, NW warps per block and MINB resident blocks per
// SM: eight warps at five blocks (48 registers, 68 bytes per thread spilled)
// or four (64 registers, 28 bytes), and sixteen warps at two blocks (64
// registers; units of twice as many items). With four eight-warp blocks each
// unit is shorter than with five; with five, more units are in flight; with
// sixteen warps a block supernode has twice the threads and staging buffer,
// which shortens the chains of a single garment's tree. The autotuner times
// the forms on the batch: on 512 sheets of 8 topologies the eight-warp forms
// tie and sixteen warps are 14% slower; on 64 contact drapes four eight-warp
// blocks are 6% faster than five; on single garments sixteen warps shorten
// the step by 4-12%. Untuned batches take sixteen warps for at most
// kWideMaxInstances garments, else four eight-warp blocks.
template <int MINB, uint32_t NW = kSolveWarps>
__global__ void __launch_bounds__(32 * NW, MINB) k_sweep(BatchDev B, uint32_t nfwd, uint32_t nbwd) {
  pdl_begin();
  extern __shared__ float4 smem4[];
  __shared__ uint64_t s_bar[NW + 2];
  __shared__ uint32_t s_abort, s_unit[2], s_next[2];
  SweepTeams t = make_teams<NW>(smem4, s_bar, &s_abort);
  const uint32_t tid = threadIdx.x;
  const bool ipc = B.prm->ipc != 0;
  // Thread 0 takes the next unit from the queue while the block works on the
  // current one (the atomic's latency hides behind the unit). A block then
  // holds one unit it has not started, which cannot deadlock: the smallest
  // unfinished unit is always one that a block is working on (a block takes
  // its next unit after its current one), and it waits only for smaller ones.
  if (tid == 0) {
    s_unit[0] = atomicAdd(B.df_queue, 1u);
    s_next[0] = NW;  // the first item a warp takes after its own
  }
  for (uint32_t it = 0;; ++it) {
    __syncthreads();  // every warp is done with the previous unit; s_unit[it & 1] is written
    const uint32_t q = s_unit[it & 1];
    if (q >= nfwd + nbwd) break;
    uint32_t next = 0;
    if (tid == 0) next = atomicAdd(B.df_queue, 1u);
    if (tid == 0) s_next[(it + 1) & 1] = NW;  // the next unit's counter (unused until the barrier)
    if (q < nfwd) sweep_unit<0>(B, t, B.df_units_fwd[q], ipc, &s_next[it & 1]);
    else sweep_unit<1>(B, t, B.df_units[nbwd - 1 - (q - nfwd)], ipc, &s_next[it & 1]);
    if (tid == 0) s_unit[(it + 1) & 1] = next;  // read by all after the next barrier
  }
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(B.df_queue + 1, 1u) == gridDim.x - 1) {  // every block has taken its last unit
      B.df_queue[0] = 0u;
      B.df_queue[1] = 0u;
    }
  }
}

// ------------------------------------------------ garment-grouped sweeps
// k_gsweep sweeps the bottom of the supernodal trees of every garment group:
// the bottom subtrees, then the supernodes above them that a warp would take
// (at most 32 columns, s (s + m) within the default warp-item limit) as long
// as all their descendants are swept here too. Each warp takes work items from
// a queue (no block-wide barrier): one bottom subtree or one such supernode of
// a topology, for every garment of one group at once, lane l for the group's
// garment l. The lanes never exchange data: each runs, for its own garment,
// the per-garment warp sweep's arithmetic in the same order
//   forward   t = y - the pulled U slots in list order; y_c = sum over
//             c2 <= c ascending of inv(L_kk)(c, c2) t_c2; u_j = sum over c
//             ascending of P(j, c) y_c;
//   backward  each column's sum over the panel rows ascending, t_c = y_c -
//             that sum; x_c = sum over c2 >= c ascending of inv(L_kk)(c2, c) t_c2,
// so a garment's solution is bit-identical to the per-garment sweeps'. Each
// lane keeps its vector (a supernode's columns, or a subtree's slice of at
// most 32 columns) in shared memory, component k of column c of lane l at
// [(3 c + k) * 32 + l]: a warp's accesses hit 32 banks. Factor entries come
// straight from HBM: one entry of a whole group is one coalesced 128-byte
// line, and a topology's row indices and pull lists are read once for all
// its garments. Dependencies are per garment, as in k_sweep: each lane waits
// on, and signals, its own garment's counters. Waits are bounded (status bit 4).
constexpr uint32_t kGWarps = 8;
constexpr uint32_t kGThreads = 32 * kGWarps;
constexpr uint32_t kGCols = 32;
constexpr uint32_t kGSmem = kGWarps * kGCols * 3 * 32 * 4;  // 96 KB: two blocks per SM
constexpr uint32_t kGColBlock = 8;                          // backward: columns summed side by side
constexpr uint32_t kGNone = 0xffffffffu;

struct GLane {
  float* v;  // component x of column 0 of this lane
  __device__ __forceinline__ float4 get(uint32_t c) const {
    return make_float4(v[(3 * c) * 32], v[(3 * c + 1) * 32], v[(3 * c + 2) * 32], 0.f);
  }
  __device__ __forceinline__ void set(uint32_t c, float4 a) const {
    v[(3 * c) * 32] = a.x;
    v[(3 * c + 1) * 32] = a.y;
    v[(3 * c + 2) * 32] = a.z;
  }
};

// Streamed factor entry (read once per sweep).
__device__ __forceinline__ float gval(const float* p) { return __ldcs(p); }

// Brings [p, p + bytes) into L2 ahead of its use (a bulk prefetch, no
// shared memory involved); p 16-byte aligned, bytes rounded down to 16.
__device__ __forceinline__ void l2_prefetch(const void* p, uint64_t bytes) {
  for (uint64_t o = 0; o + 16 <= bytes; o += 32768) {
    const uint64_t left = bytes - o;
    const uint32_t n = uint32_t(left < 32768 ? left : 32768) & ~15u;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(static_cast<const char*>(p) + o), "r"(n)
                 : "memory");
  }
}

// y = inv(L_kk) t in place on columns f .. f + s of L, the triangle's rows at
// D (entry (c, c2) at D[(c (c + 1) / 2 + c2) * 32]); descending c, two rows
// per pass (each y_c reads only t values, so the rows are independent and
// their loads overlap), each row summed over c2 ascending.
__device__ __forceinline__ void g_diag_fwd(const GLane& L, uint32_t f, uint32_t s, const float* D) {
  int c = int(s) - 1;
  for (; c >= 1; c -= 2) {
    float4 y0 = make_float4(0.f, 0.f, 0.f, 0.f), y1 = y0;
    const float* r0 = D + size_t(uint32_t(c) * uint32_t(c + 1) / 2) * 32;
    const float* r1 = D + size_t(uint32_t(c - 1) * uint32_t(c) / 2) * 32;
#pragma unroll 8
    for (uint32_t c2 = 0; c2 < uint32_t(c); ++c2) {
      const float4 t = L.get(f + c2);
      f4_fma(y0, gval(r0 + c2 * 32), t);
      f4_fma(y1, gval(r1 + c2 * 32), t);
    }
    f4_fma(y0, gval(r0 + uint32_t(c) * 32), L.get(f + uint32_t(c)));
    L.set(f + uint32_t(c), y0);
    L.set(f + uint32_t(c) - 1, y1);
  }
  if (c == 0) {
    float4 y = make_float4(0.f, 0.f, 0.f, 0.f);
    f4_fma(y, gval(D), L.get(f));
    L.set(f, y);
  }
}

// x = inv(L_kk)^T t in place on columns f .. f + s of L; ascending c, two
// rows per pass (each x_c reads only t values), each summed over c2 ascending.
__device__ __forceinline__ void g_diag_bwd(const GLane& L, uint32_t f, uint32_t s, const float* D) {
  uint32_t c = 0;
  for (; c + 1 < s; c += 2) {
    float4 x0 = make_float4(0.f, 0.f, 0.f, 0.f), x1 = x0;
    f4_fma(x0, gval(D + size_t(c * (c + 1) / 2 + c) * 32), L.get(f + c));
#pragma unroll 8
    for (uint32_t c2 = c + 1; c2 < s; ++c2) {
      const float4 t = L.get(f + c2);
      const float* row = D + size_t(c2 * (c2 + 1) / 2 + c) * 32;
      f4_fma(x0, gval(row), t);
      f4_fma(x1, gval(row + 32), t);
    }
    L.set(f + c, x0);
    L.set(f + c + 1, x1);
  }
  if (c < s) {
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
    f4_fma(x, gval(D + size_t(c * (c + 1) / 2 + c) * 32), L.get(f + c));
    L.set(f + c, x);
  }
}

// u_j = P(j, :) . y for the m panel rows (P row-major, y in columns f .. f + s
// of L), eight rows at a time so that each y_c is read once per eight rows and
// the rows' loads overlap; emit(j, u) takes each row's update.
constexpr uint32_t kGPushRows = 8;
template <class Emit>
__device__ __forceinline__ void g_push(const GLane& L, uint32_t f, uint32_t s, uint32_t m, const float* P, Emit emit) {
  for (uint32_t j0 = 0; j0 < m; j0 += kGPushRows) {
    const uint32_t nr = min(kGPushRows, m - j0);
    float4 u[kGPushRows];
#pragma unroll
    for (uint32_t r = 0; r < kGPushRows; ++r) u[r] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float* P0 = P + size_t(j0) * s * 32;
#pragma unroll 4
    for (uint32_t c = 0; c < s; ++c) {
      const float4 y = L.get(f + c);
#pragma unroll
      for (uint32_t r = 0; r < kGPushRows; ++r)
        if (r < nr) f4_fma(u[r], gval(P0 + size_t(r * s + c) * 32), y);
    }
#pragma unroll
    for (uint32_t r = 0; r < kGPushRows; ++r)
      if (r < nr) emit(j0 + r, u[r]);
  }
}

// t_c = L_c - sum over panel rows j of P(j, c) x(R_j) for the s columns at f,
// kGColBlock columns side by side, each column's sum in ascending j; xget(r)
// gives x of row r.
template <class XGet>
__device__ __forceinline__ void g_bwd_panel(const GLane& L, uint32_t f, uint32_t s, uint32_t m, const float* P,
                                            const uint32_t* R, XGet xget) {
  for (uint32_t cb = 0; cb < s; cb += kGColBlock) {
    float4 acc[kGColBlock];
#pragma unroll
    for (uint32_t k = 0; k < kGColBlock; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 4
    for (uint32_t j = 0; j < m; ++j) {
      const float4 x = xget(__ldg(R + j));
      const float* Pj = P + (size_t(j) * s + cb) * 32;
#pragma unroll
      for (uint32_t k = 0; k < kGColBlock; ++k)
        if (cb + k < s) f4_fma(acc[k], gval(Pj + k * 32), x);
    }
#pragma unroll
    for (uint32_t k = 0; k < kGColBlock; ++k)
      if (cb + k < s) L.set(f + cb + k, f4_sub(L.get(f + cb + k), acc[k]));
  }
}

// One work item for one lane (its group's garment `lane`).
template <int DIR>
__device__ __forceinline__ void g_item(const BatchDev& B, uint2 it, const GLane& L, uint32_t lane, bool ipc) {
  const GroupDev G = B.grp[it.x];
  if (lane >= G.lanes) return;
  const uint32_t gl = it.x * kGroupLanes + lane;
  if (ipc && B.red[B.gl_inst[gl]].al_done) return;
  const uint32_t snb = B.gl_snbase[gl];
  float4* Y = B.Y + B.gl_vbase[gl];
  const float* vals = B.g_vals + G.base * 32 + lane;
  float4* U = B.U + G.u_base + lane;  // the garment's U slot i at U[i * 32]
  const uint32_t id = it.y >> 1;
  if ((it.y & 1u) == 0) {
    // one bottom subtree: the warp keeps its slice of the vector (columns
    // c0 .. c1) for the whole sweep, as the per-garment subtree sweep does
    const uint2 st = B.g_subs[id];
    const GsnDev A = B.gsn[st.x], Z = B.gsn[st.y];
    const uint32_t c0 = A.first, c1 = Z.first + Z.ncols, nc = c1 - c0;
    const uint32_t root = snb + (st.y - G.sn_off);
    const GsnDev Zn = B.gsn[st.y];  // the item's data: [A.g_off, end of Z) is contiguous
    if (lane == 0) {
      const uint64_t e0 = A.g_off, e1 = Zn.g_off + uint64_t(Zn.ncols) * (Zn.ncols + 1) / 2 + uint64_t(Zn.nrows) * Zn.ncols;
      const uint64_t nb = (e1 - e0) * 128;
      l2_prefetch(B.g_vals + (G.base + e0) * 32, nb < 65536 ? nb : 65536);
    }
    if (DIR == 1 && dep_wait(B, B.df_flag + root, 1u)) B.df_flag[root] = 0u;
    for (uint32_t c = 0; c < nc; ++c) L.set(c, __ldcg(Y + c0 + c));
    if (DIR == 0) {
      for (uint32_t q = st.x; q <= st.y; ++q) {
        const GsnDev S = B.gsn[q];
        const uint32_t s = S.ncols, m = S.nrows, f = S.first - c0;
        const float* D = vals + S.g_off * 32;
        g_diag_fwd(L, f, s, D);
        const uint32_t* R = B.g_rows + S.rows_off;
        g_push(L, f, s, m, D + size_t(s * (s + 1) / 2) * 32, [&](uint32_t j, float4 u) {
          const uint32_t r = __ldg(R + j);
          if (r < c1) L.set(r - c0, f4_sub(L.get(r - c0), u));
          else U[size_t(S.u_local + j) * 32] = u;
        });
      }
    } else {
      for (uint32_t q = st.y + 1; q-- > st.x;) {
        const GsnDev S = B.gsn[q];
        const uint32_t s = S.ncols, m = S.nrows, f = S.first - c0;
        const float* D = vals + S.g_off * 32;
        g_bwd_panel(L, f, s, m, D + size_t(s * (s + 1) / 2) * 32, B.g_rows + S.rows_off,
                    [&](uint32_t r) { return r < c1 ? L.get(r - c0) : __ldcg(Y + r); });
        g_diag_bwd(L, f, s, D);
      }
    }
    for (uint32_t c = 0; c < nc; ++c) Y[c0 + c] = L.get(c);
    __threadfence();
    if (DIR == 0) {
      if (Z.parent != kGNone) atomicAdd(B.df_cnt + snb + Z.parent, 1u);
      else atomicExch(B.df_flag + root, 1u);
    }
    return;
  }
  // one supernode above the subtrees
  const GsnDev S = B.gsn[id];
  const uint32_t s = S.ncols, m = S.nrows, f = S.first;
  const uint32_t me = snb + (id - G.sn_off);
  const float* D = vals + S.g_off * 32;
  const float* P = D + size_t(s * (s + 1) / 2) * 32;
  if (lane == 0)  // in flight while the dependency wait runs
    l2_prefetch(B.g_vals + (G.base + S.g_off) * 32, (uint64_t(s) * (s + 1) / 2 + uint64_t(m) * s) * 128);
  if (DIR == 0) {
    if (S.nkids && dep_wait(B, B.df_cnt + me, S.nkids)) B.df_cnt[me] = 0u;
    const uint32_t* fp = B.g_fwd_ptr + G.row_base + f;
    for (uint32_t c = 0; c < s; ++c) {
      float4 t = Y[f + c];
      for (uint32_t q = __ldg(fp + c), qe = __ldg(fp + c + 1); q < qe; ++q)
        t = f4_sub(t, __ldcg(U + size_t(__ldg(B.g_fwd + q)) * 32));
      L.set(c, t);
    }
    g_diag_fwd(L, 0, s, D);
    for (uint32_t c = 0; c < s; ++c) Y[f + c] = L.get(c);
    g_push(L, 0, s, m, P, [&](uint32_t j, float4 u) { U[size_t(S.u_local + j) * 32] = u; });
    __threadfence();
    if (S.parent != kGNone) atomicAdd(B.df_cnt + snb + S.parent, 1u);
    else atomicExch(B.df_flag + me, 1u);
  } else {
    if (dep_wait(B, B.df_flag + me, 1u)) B.df_flag[me] = 0u;
    for (uint32_t c = 0; c < s; ++c) L.set(c, __ldcg(Y + f + c));
    g_bwd_panel(L, 0, s, m, P, B.g_rows + S.rows_off, [&](uint32_t r) { return __ldcg(Y + r); });
    g_diag_bwd(L, 0, s, D);
    for (uint32_t c = 0; c < s; ++c) Y[f + c] = L.get(c);
    __threadfence();
    for (uint32_t k = 0; k < S.nkids; ++k) atomicExch(B.df_flag + snb + __ldg(B.g_kids + S.kid_off + k), 1u);
  }
}

// The forward (DIR = 0) or backward (DIR = 1) grouped sweep over `nitems`
// work items in topological order. Each warp takes items until the queue is
// empty; an item only waits for items handed out before it, whose warps are
// running, so there is no deadlock whatever the number of resident warps. The
// last warp out resets the queue.
template <int DIR>
__global__ void __launch_bounds__(kGThreads, 2) k_gsweep(BatchDev B, uint32_t nitems) {
  pdl_begin();
  extern __shared__ float gsm[];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const GLane L{gsm + warp * (kGCols * 3 * 32) + lane};
  const bool ipc = B.prm->ipc != 0;
  const uint2* items = DIR == 0 ? B.g_items_fwd : B.g_items_bwd;
  // An item is taken when the warp is free: with few long items per warp,
  // taking the next one ahead would hand the tail items to busy warps.
  for (;;) {
    uint32_t q = 0;
    if (lane == 0) q = atomicAdd(B.g_queue, 1u);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= nitems) break;
    g_item<DIR>(B, items[q], L, lane, ipc);
    __syncwarp();
  }
  if (lane == 0) {
    __threadfence();
    if (atomicAdd(B.g_queue + 1, 1u) == gridDim.x * kGWarps - 1) {
      B.g_queue[0] = 0u;
      B.g_queue[1] = 0u;
    }
  }
}

// Largest c with c (c + 1) / 2 <= e.
__device__ __forceinline__ uint32_t tri_row(uint32_t e) {
  uint32_t c = uint32_t((sqrtf(8.f * float(e) + 1.f) - 1.f) * 0.5f);
  while ((c + 1) * (c + 2) / 2 <= e) ++c;
  while (c * (c + 1) / 2 > e) --c;
  return c;
}

// Copies the grouped supernodes' factor values from the per-garment regions
// (D column-major, P row-major, leading dimension sn_ld(s)) into the groups'
// interleaved blocks; one block per (group, global GsnDev id) of `work`.
// Lanes beyond a group's garments get zeros.
__global__ void __launch_bounds__(256) k_gpack(BatchDev B, float* g_vals, const uint2* work) {
  const uint2 w = work[blockIdx.x];
  const GroupDev G = B.grp[w.x];
  const GsnDev S = B.gsn[w.y];
  const uint32_t lane = threadIdx.x & 31, row = threadIdx.x >> 5, rows = blockDim.x >> 5;
  const uint32_t s = S.ncols, m = S.nrows, nd = s * (s + 1) / 2, ne = nd + m * s;
  float* out = g_vals + (G.base + S.g_off) * 32 + lane;
  if (lane >= G.lanes) {
    for (uint32_t e = row; e < ne; e += rows) out[size_t(e) * 32] = 0.f;
    return;
  }
  const SnDev P = B.sn[B.gl_snbase[w.x * kGroupLanes + lane] + (w.y - G.sn_off)];
  const uint32_t ld = sn_ld(s);
  for (uint32_t e = row; e < ne; e += rows) {
    float v;
    if (e < nd) {
      const uint32_t c = tri_row(e), c2 = e - c * (c + 1) / 2;
      v = B.vals[P.d_off + uint64_t(c2) * ld + c];
    } else {
      const uint32_t j = (e - nd) / s, c = (e - nd) % s;
      v = B.vals[P.p_off + uint64_t(j) * ld + c];
    }
    out[size_t(e) * 32] = v;
  }
}

__global__ void k_red_reset(BatchDev B, uint32_t ninst) {
  pdl_begin();
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ninst) return;
  InstRed& R = B.red[k];
  if (B.prm->ipc && R.al_done) return;
  R.diff_sq = 0.0;
  R.norm_sq = 0.0;
  R.toi_bits = __float_as_uint(1.0f);
  R.gdd = 0.0;
}

// Iterative refinement of the global solve: W = R0 - A d in FP64, with d the
// sweeps' FP32 solution in Y and A the f64 matrix that was factored. Each
// instance's rows are numbered like its vertices, so the vertex chunks cover
// them. The sweeps then solve A e = W in place and d + e replaces d.
__global__ void __launch_bounds__(256) k_refine(BatchDev B) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  if (B.prm->ipc && B.red[ch.x].al_done) return;
  const uint32_t p = uint32_t(ch.y) + threadIdx.x;
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (uint32_t q = B.a_ptr[p], qe = B.a_ptr[p + 1]; q < qe; ++q) {
    const double a = B.a_val[q];
    const float4 d = B.Y[B.a_col[q]];
    ax += a * d.x; ay += a * d.y; az += a * d.z;
  }
  const float4 r = B.R0[p];
  B.W[p] = make_float4(float(double(r.x) - ax), float(double(r.y) - ay), float(double(r.z) - az), 0.f);
}

// d <- d + e between two refinement sweeps.
__global__ void __launch_bounds__(256) k_accum(BatchDev B) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  if (B.prm->ipc && B.red[ch.x].al_done) return;
  const uint32_t p = uint32_t(ch.y) + threadIdx.x;
  B.Y[p] = f4_add(B.Y[p], B.W[p]);
}

// After the sweeps: residual sums (pd_solver.rs:403-421) and, for the plain
// step, x <- x + d, the pin reset (:429-435) and the ground clamp (:438).
// add_w folds the last refinement correction into d (and into Y, where the
// IPC kernels read d).
__device__ __forceinline__ void update_one(const BatchDev& B, const InstDev& I, uint32_t g, float4 d, float4 x,
                                           int do_update, int add_w, uint32_t row, double& dsq, double& nsq,
                                           bool& bad) {
  if (add_w) {
    d = f4_add(d, B.W[row]);
    B.Y[row] = d;
  }
  dsq += double(d.x) * d.x + double(d.y) * d.y + double(d.z) * d.z;
  nsq += double(x.x) * x.x + double(x.y) * x.y + double(x.z) * x.z;
  bad = bad || !(isfinite(d.x) && isfinite(d.y) && isfinite(d.z));
  if (do_update) {
    float4 nx;
    if (B.pinned[g]) nx = B.prev[g];
    else {
      nx = make_float4(x.x + d.x, x.y + d.y, x.z + d.z, 0.f);
      if (I.has_ground && nx.y < I.ground_h) nx.y = I.ground_h;  // state.rs:180-189
    }
    B.pos[g] = nx;
  }
}

// Two vertices per thread (128 threads over a chunk of up to 256), both
// vertices' loads issued before either update: 0.063 -> about 0.043 ms per
// iteration on 4.05 M vertices (the solve phase 1.315 -> 1.295 ms).
__global__ void __launch_bounds__(128) k_update(BatchDev B, int do_update, int add_w) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  const InstDev I = B.inst[ch.x];
  InstRed& R = B.red[ch.x];
  if (B.prm->ipc && R.al_done) return;
  double dsq = 0.0, nsq = 0.0;
  bool bad = false;
  const uint32_t i0 = threadIdx.x, i1 = threadIdx.x + 128;
  if ((int)i0 < ch.z) {
    const bool two = (int)i1 < ch.z;
    const uint32_t g0 = uint32_t(ch.y) + i0, g1 = uint32_t(ch.y) + i1;
    const uint32_t r0 = I.vbase + B.perm_local[g0], r1 = two ? I.vbase + B.perm_local[g1] : r0;
    const float4 d0 = B.Y[r0], d1 = two ? B.Y[r1] : d0;
    const float4 x0 = B.pos[g0], x1 = two ? B.pos[g1] : x0;
    update_one(B, I, g0, d0, x0, do_update, add_w, r0, dsq, nsq, bad);
    if (two) update_one(B, I, g1, d1, x1, do_update, add_w, r1, dsq, nsq, bad);
  }
  for (int o = 16; o > 0; o >>= 1) {
    dsq += __shfl_down_sync(0xffffffffu, dsq, o);
    nsq += __shfl_down_sync(0xffffffffu, nsq, o);
  }
  if (bad) atomicOr(B.status, 1u);
  if ((threadIdx.x & 31) == 0 && (dsq != 0.0 || nsq != 0.0)) {
    atomicAdd(&R.diff_sq, dsq);
    atomicAdd(&R.norm_sq, nsq);
  }
  if (threadIdx.x == 0 && ch.y == int(I.vbase)) R.iters += 1;
}

// Whole-batch positions between interleaved xyz (the host layout, one
// contiguous copy) and the float4 state rows.
__global__ void __launch_bounds__(256) k_unpack_pos(float4* pos, const float* __restrict__ xyz, uint64_t n) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    float4 p = pos[i];
    p.x = xyz[3 * i]; p.y = xyz[3 * i + 1]; p.z = xyz[3 * i + 2];
    pos[i] = p;
  }
}
__global__ void __launch_bounds__(256) k_pack_pos(float* __restrict__ xyz, const float4* pos, uint64_t n) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const float4 p = pos[i];
    xyz[3 * i] = p.x; xyz[3 * i + 1] = p.y; xyz[3 * i + 2] = p.z;
  }
}

// save_previous + (IPC) velocity clamp + predict + x <- pred (state.rs:145-169,
// pd_solver.rs:273-283 and 566-603).
__global__ void __launch_bounds__(256) k_predict(BatchDev B) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  const InstDev I = B.inst[ch.x];
  const StepParams& P = *B.prm;
  if (threadIdx.x == 0 && ch.y == int(I.vbase)) {
    InstRed& R = B.red[ch.x];
    R.iters = 0;
    R.al_iters = 0;
    R.al_done = 0;
    R.mu = P.al_mu_initial;
    R.last_active = 0;
    R.alpha = 1.f;
  }
  if ((int)threadIdx.x >= ch.z) return;
  uint32_t g = uint32_t(ch.y) + threadIdx.x;
  float4 x = B.pos[g];
  float4 v = B.vel[g];
  B.prev[g] = x;
  bool pin = B.pinned[g] != 0;
  bool ground = P.ipc ? P.has_ground : I.has_ground;
  float gh = P.ipc ? P.ground_h : I.ground_h;
  if (P.ipc) {
    if (!pin && P.max_vel > 0.f) {
      float vsq = v.x * v.x + v.y * v.y + v.z * v.z;
      if (vsq > P.max_vel * P.max_vel) {
        float sc = P.max_vel / sqrtf(vsq);
        v.x *= sc; v.y *= sc; v.z *= sc;
        B.vel[g] = v;
      }
    }
    B.ever[g] = 0;
    B.fin_n[g] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  float4 q = x;
  if (!pin) {
    float dt = P.dt, dt2 = dt * dt;
    q.x = x.x + dt * v.x + dt2 * P.gravity[0];
    q.y = x.y + dt * v.y + dt2 * P.gravity[1];
    q.z = x.z + dt * v.z + dt2 * P.gravity[2];
    if (ground && q.y < gh) q.y = gh;
  }
  B.pred[g] = q;
  B.pos[g] = q;
}

// update_velocities, (IPC) inelastic velocity filter, ground velocities,
// damping and Rayleigh damping (pd_solver.rs:447-466 and 1027-1147).
__global__ void __launch_bounds__(256) k_finalize(BatchDev B) {
  pdl_begin();
  int4 ch = B.vtx_chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  const InstDev I = B.inst[ch.x];
  const StepParams& P = *B.prm;
  uint32_t g = uint32_t(ch.y) + threadIdx.x;
  float4 x = B.pos[g], pv = B.prev[g];
  float inv_dt = 1.f / P.dt;
  float3 v = make_float3((x.x - pv.x) * inv_dt, (x.y - pv.y) * inv_dt, (x.z - pv.z) * inv_dt);
  bool pin = B.pinned[g] != 0;
  bool ground = P.ipc ? P.has_ground : I.has_ground;
  float gh = P.ipc ? P.ground_h : I.ground_h;
  if (P.ipc) {
    const InstRed& R = B.red[ch.x];
    if (!pin && B.ever[g]) {
      float4 n4 = B.fin_n[g];
      float3 n = f3(n4);
      if (dot3(n, n) >= 0.5f) {
        float vdn = dot3(v, n);
        v = v - n * vdn;
        float vn = fabsf(vdn);
        float vt = len3(v);
        if (vt > 1e-8f) {
          float fi = P.friction * vn;
          if (fi >= vt) v = make_float3(0.f, 0.f, 0.f);
          else v = v * (1.f - fi / vt);
        }
        float cd = P.contact_damping;
        if (P.adaptive_damping) {
          float vm = len3(v);
          float tt = fminf(fmaxf(1.f - vm / fmaxf(P.contact_vthresh, 1e-6f), 0.f), 1.f);
          float ad = cd + tt * (P.contact_damping_max - cd);
          v = v * (1.f - ad);
        } else {
          v = v * (1.f - cd);
        }
      }
    }
    if (R.last_active > 0) v = v * (1.f - 0.05f);
  }
  if (ground && !pin && x.y <= gh) {  // state.rs:195-213
    if (v.y < 0.f) v.y = 0.f;
    pv.y = gh;
    B.prev[g] = pv;
    v.x *= 0.5f; v.z *= 0.5f;
  }
  v = v * (1.f - P.damping);
  if (P.rayleigh > 0.f && !pin) v = v * (1.f / (1.f + P.rayleigh * P.dt));
  B.vel[g] = make_float4(v.x, v.y, v.z, 0.f);
}

}  // namespace vistio
