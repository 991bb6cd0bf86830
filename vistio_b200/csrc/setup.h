// Host-side set-up for one drape instance: rest-state element data, hinge
// (bending) data, lumped masses, the constant PD system matrix and its
// supernodal FP64 Cholesky factor laid out for the GPU triangular sweeps.
//
// This is the part of ProjectiveDynamicsSolver::init* that runs once per
// (topology, material, dt) in the reference (crates/vistio-solver/src/
// pd_solver.rs:106-257); it stays on the host and produces the flat arrays
// the batch packer uploads to HBM.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace vistio {

enum ModelKind : int32_t { MODEL_ARAP = 0, MODEL_COROT = 1, MODEL_ORTHO = 2, MODEL_ANISO = 3, MODEL_ISO_LINEAR = 4 };
enum BendKind : int32_t { BEND_NONE = 0, BEND_DIHEDRAL = 1, BEND_DS = 2, BEND_DS_ANISO = 3 };

struct SetupParams {
  int32_t model = MODEL_ARAP;
  int32_t bending = BEND_DIHEDRAL;
  float stiffness = 1000.f;       // element weight = stiffness * rest area
  float bend_stiffness = 1e-4f;   // hinge weight = bend_stiffness * edge length
  float density_gsm = 200.f;
  float warp = 0.f, weft = 0.f;   // membrane model warp/weft
  float bend_warp = 0.f, bend_weft = 0.f;
  float matrix_dt = 1.0f / 60.0f; // dt used in A (the reference always assembles with 1/60)
  bool numeric = true;            // false: symbolic factorization only (the numbers on the GPU)
};

// Largest supernode (columns); the GPU sweeps size their shared-memory vectors for it.
constexpr uint32_t kMaxSupernodeCols = 256;
// Bottom subtrees of the supernodal elimination tree whose factor data (in
// floats, as packed for the GPU: sn_floats per supernode) fits this budget
// are swept as one unit by one warp.
constexpr uint32_t kSubtreeFloats = 1024;
// ... and whose columns (contiguous in postorder) number at most this: the
// warp keeps the subtree's slice of the vector in shared memory.
constexpr uint32_t kSubtreeCols = 32;
constexpr uint32_t kBottomLevel = 0xffffffffu;
#if defined(__CUDACC__)
#define VISTIO_HD __host__ __device__
#else
#define VISTIO_HD
#endif
// Leading dimension of a supernode's diagonal block (column-major) and panel
// (row-major) as packed for the GPU: s rounded up to an odd number, so that
// 32 lanes reading one column of 32 consecutive panel rows, or one row of 32
// consecutive diagonal-block columns, hit 32 different shared-memory banks.
VISTIO_HD constexpr uint32_t sn_ld(uint32_t s) { return s | 1u; }
// Floats of one supernode's packed region: inv(L_kk) (s columns of sn_ld(s)),
// then the panel (m rows of sn_ld(s)) followed by its m row indices, each
// part padded to 4 floats.
inline uint64_t sn_floats(uint32_t s, uint32_t m) {
  return ((uint64_t(s) * sn_ld(s) + 3) & ~3ull) + ((uint64_t(m) * sn_ld(s) + m + 3) & ~3ull);
}

// Supernodal factor of P A P^T = L L^T in the layout the GPU sweeps read.
// Columns are in the permuted (elimination) order.
struct Supernode {
  uint32_t first;     // first column
  uint32_t ncols;     // s
  uint32_t nrows;     // |R|: rows strictly below the diagonal block
  uint32_t rows_off;  // offset of R (sorted row indices) in Factor::rows
  uint64_t panel_off; // offset of the |R| x s row-major panel in Factor::vals
  uint64_t diag_off;  // offset of inv(L_kk), s x s column-major, in Factor::vals
  uint32_t parent;    // parent supernode, or UINT32_MAX for a root
  uint32_t level;     // sweep level above the bottom subtrees (kBottomLevel inside one)
};

struct Factor {
  uint32_t n = 0;
  std::vector<uint32_t> perm;   // perm[new] = old vertex
  std::vector<uint32_t> iperm;  // iperm[old] = new
  std::vector<Supernode> sn;
  std::vector<uint32_t> rows;   // below-diagonal row structures
  std::vector<double> vals;     // panels and inverted diagonal blocks (FP64)
  std::vector<uint32_t> row_sn; // supernode owning each column
  // Level schedule: supernodes grouped by level; rows of those supernodes.
  uint32_t nlevels = 0;
  std::vector<uint32_t> level_ptr;  // nlevels+1 offsets into level_rows
  std::vector<uint32_t> level_rows; // rows (columns) of the level's supernodes, grouped by supernode
  std::vector<uint32_t> level_sn_ptr; // nlevels+1 offsets into level_sn
  std::vector<uint32_t> level_sn;     // supernodes of each level, largest first
  // Bottom subtrees: supernode ranges [first, last] in postorder (last = root).
  std::vector<uint32_t> sub_first, sub_last;
  // Forward-sweep pull lists: for each row r, the (supernode, panel row) pairs
  // of the descendants whose panels hold row r.
  std::vector<uint32_t> fwd_ptr;    // n+1
  std::vector<uint32_t> fwd_sn;     // supernode id
  std::vector<uint32_t> fwd_pos;    // row position inside that supernode's panel
  uint64_t nnz_L = 0;               // nonzeros of the simplicial factor (incl. diagonal)
  bool numeric = true;              // vals holds the factor (else symbolic only)
  uint64_t nnz_stored = 0;          // entries stored in panels + diagonal blocks
};

struct InstanceSetup {
  uint32_t nv = 0, nt = 0, nh = 0;
  SetupParams prm;
  std::vector<float> rest;          // 3*nv rest positions
  std::vector<uint32_t> tris;       // 3*nt
  std::vector<float> dm_inv;        // 4*nt (column-major Dm^-1)
  std::vector<float> area;          // nt
  std::vector<float> tri_w;         // nt
  std::vector<uint32_t> hinge_v;    // 4*nh (v0, v1, wing_a, wing_b)
  std::vector<float> hinge_st;      // 4*nh stencil
  std::vector<float> hinge_w;       // nh
  std::vector<float> hinge_rest;    // nh rest dihedral angle
  std::vector<float> mass;          // solver lumped masses (pinned = 1e8)
  std::vector<uint8_t> pinned;
  // Constant system matrix A (CSR, f64 sums of the f32 triplets).
  std::vector<uint32_t> A_ptr, A_col;
  std::vector<double> A_val;
  Factor factor;
};

// Builds everything; returns an empty string on success or an error text.
// `status` receives the status code (0 ok, 1 invalid mesh, 3 invalid config, 11 not SPD).
std::string build_instance(uint32_t nv, const float* px, const float* py, const float* pz,
                           uint32_t nt, const uint32_t* tris, const uint8_t* pinned,
                           const SetupParams& prm, InstanceSetup& out, int* status);

// The process-wide cache of symbolic factors (factorize_csr with numeric ==
// false), keyed by the exact adjacency and dissection order: counters, bytes
// held and entries; and its byte bound (default 1 GiB; 0 disables it and
// empties it).
void symbolic_cache_info(uint64_t* hits, uint64_t* misses, uint64_t* bytes, uint64_t* entries);
void symbolic_cache_set_limit(uint64_t limit_bytes);

// Replaces a CSR matrix (rows sorted) by the symmetric matrix its upper
// triangle (column >= row) defines, rows sorted: what faer factors with
// Side::Upper (crates/vistio-math/src/faer_solver.rs:84-88). Mirrored pairs of
// a PD system matrix can differ in the last bit (w s_a s_b against w s_b s_a).
void mirror_upper(uint32_t n, std::vector<uint32_t>& ptr, std::vector<uint32_t>& col, std::vector<double>& val);

// Appends I's system matrix with rows and columns in solve (permuted) order:
// for each permuted row r the end offset to ptr, and its entries (column
// base + iperm[col], f64 value) to col / val. ptr starts as {0} (or the end of
// the previous instance).
void append_permuted_matrix(const InstanceSetup& I, uint32_t base, std::vector<uint32_t>& ptr,
                            std::vector<uint32_t>& col, std::vector<double>& val);

// Factorizes a general SPD matrix (CSR, either triangle or both) into the GPU layout.
// coords (3*n) steer the nested dissection; may be null (a BFS-based split is used).
// With numeric == false only the symbolic analysis is done (ordering,
// supernodes, row structures, schedules; vals stays empty): the GPU computes
// the numbers (multifrontal, FP64) when the garment is packed into a batch.
std::string factorize_csr(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                          const double* vals, const float* coords, Factor& f, int* status, bool numeric = true);

}  // namespace vistio
