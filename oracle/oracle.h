// TEST INFRASTRUCTURE ONLY — the CPU oracle's C interface (ctypes-bound by
// tests/oracle_api.py). The product never includes or links this.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// Membrane projection used in the local step.
enum { ORC_MODEL_ARAP = 0,        // ElementData::project (element.rs:127), `init` path
       ORC_MODEL_COROT = 1,       // CoRotationalModel (corotational.rs:50)
       ORC_MODEL_ORTHO = 2,       // OrthotropicLinearModel (orthotropic.rs:50)
       ORC_MODEL_ANISO = 3,       // AnisotropicCoRotationalModel (anisotropic.rs:77)
       ORC_MODEL_ISO_LINEAR = 4 };// IsotropicLinearModel (isotropic.rs:41)
enum { ORC_BEND_NONE = 0, ORC_BEND_DIHEDRAL = 1, ORC_BEND_DS = 2, ORC_BEND_DS_ANISO = 3 };

// Set-up parameters. `init` (pd_solver.rs:221) maps to stiffness =
// stretch_weight*1000, bend_stiffness = bending_weight*100, density 200 g/m^2;
// `init_with_material` maps to stiffness = avg_stretch*10 (element.rs:106),
// bend_stiffness = avg_bending*100, density = material density.
typedef struct orc_params {
  int32_t model;
  int32_t bending;
  float stiffness;       // element stiffness k: weight = k * rest_area
  float bend_stiffness;  // k_b: hinge weight = k_b * edge_len
  float density_gsm;     // area density (g/m^2) for lumped masses
  float warp, weft;      // model warp/weft stiffness (ORTHO / ANISO)
  float bend_warp, bend_weft;  // material bending warp/weft (DS_ANISO)
  float matrix_dt;       // dt used when assembling A (reference hardcodes 1/60)
} orc_params;

// Live fields of SolverConfig (crates/vistio-solver/src/config.rs:10-129).
typedef struct orc_config {
  uint32_t max_iterations;
  uint32_t al_max_iterations;
  double tolerance;
  float gravity[3];
  float damping;
  float rayleigh_mass_damping;
  float barrier_d_hat;
  float al_mu_initial;
  float al_mu_growth;
  float al_tolerance;
  float friction_coefficient;
  float contact_damping;
  float compliant_d_hat_scale;
  float contact_damping_max;
  float contact_velocity_threshold;
  int32_t compliant_contact;
  int32_t adaptive_contact_damping;
} orc_config;

// What the reference's RunnerIpcHandler / CollisionPipeline is wired with
// (crates/vistio-bench/src/runner.rs:48-99, 190-204).
typedef struct orc_contact {
  int32_t has_ground;
  float ground_height;
  int32_t has_sphere;
  float sphere_center[3];
  float sphere_radius;
  int32_t self_collision;   // BVH self contact (exclusion depth 1)
  int32_t bvh_faithful;     // 1: reference median-split BVH incl. its pair drop; 0: complete set
  float kappa;              // barrier stiffness (already estimated)
  float thickness;          // C-IPC thickness for self contacts (1.5 * d_hat in the runner)
  int32_t has_cylinder;     // CylinderCollider (cylinder.rs:11-21), endless downwards
  float cylinder_center_x, cylinder_center_z, cylinder_top_y, cylinder_radius;
  int32_t has_box;          // BoxCollider (box_collider.rs)
  float box_min[3], box_max[3];
} orc_contact;

typedef struct orc_step_result {
  uint32_t iterations;
  int32_t converged;
  double final_residual;
  int32_t status;  // 0 ok, 3 invalid config (not SPD / not initialised)
  uint32_t al_iterations;
  uint32_t active_contacts;
  float last_alpha;
} orc_step_result;

// precision: 0 = ref32 (FP32 like the reference), 1 = fp64 truth run.
void* orc_create(int precision, uint32_t nv, const float* px, const float* py, const float* pz,
                 uint32_t nt, const uint32_t* tris, const uint8_t* pinned,
                 const orc_params* params, const orc_config* cfg, int32_t* status);
void orc_destroy(void* sim);
int orc_step(void* sim, float dt, orc_step_result* res);
int orc_step_ipc(void* sim, float dt, const orc_contact* contact, orc_step_result* res);
// The colliders' resolve() after a plain step (CollisionPipeline::step with
// thickness 0, collision_pipeline.rs:117-199). out[12]: per collider (ground,
// sphere, cylinder, box) the resolved count, max penetration and depth sum.
void orc_resolve(void* sim, const orc_contact* contact, float* out);
void orc_set_ground(void* sim, int has_ground, float height);
// Read/write state (SoA float arrays of length nv; NULL skips).
void orc_get_state(void* sim, float* px, float* py, float* pz, float* vx, float* vy, float* vz);
void orc_set_state(void* sim, const float* px, const float* py, const float* pz,
                   const float* vx, const float* vy, const float* vz);
void orc_get_state64(void* sim, double* px, double* py, double* pz);
uint32_t orc_hinge_count(void* sim);
void orc_get_hinges(void* sim, uint32_t* v4, float* rest_angle, float* weight, float* stencil4);
void orc_get_masses(void* sim, float* mass);
// System matrix A: the reference's f32 triplets (assembly.rs:44-135) with
// duplicates summed in f64 as faer's try_new_from_triplets does; CSR, sorted.
uint32_t orc_matrix_nnz(void* sim);
void orc_get_matrix(void* sim, uint32_t* row_ptr, uint32_t* col_idx, double* values);
uint64_t orc_factor_nnz(void* sim);
// One local step + RHS assembly at the current positions (per axis), for boundary tests.
void orc_assemble_rhs(void* sim, float dt, float* rx, float* ry, float* rz);
// SparseSolver mirror: solve A x = b with the oracle's FP64 factor.
void orc_solve(void* sim, const float* b, float* x);

// ---- mesh generation (crates/vistio-mesh/src/generators.rs:28) ----
void orc_quad_grid(uint32_t cols, uint32_t rows, float width, float height,
                   float* px, float* py, float* pz, uint32_t* tris);

// ---- known-answer kernels for the contact primitives ----
// SparseSolver::factorize + solve (crates/vistio-math/src/faer_solver.rs:67-125)
// on a general CSR with f32 values: duplicates summed in f64, the upper
// triangle read (Side::Upper), the oracle's FP64 LL^T. Returns 0 ok, 1 not
// square, 2 empty, 3 not SPD.
int orc_sparse_solve(uint32_t rows, uint32_t cols, const uint32_t* row_ptr, const uint32_t* col_idx,
                     const float* vals, const float* rhs, float* sol);
float orc_pt_dist2(const float p[3], const float a[3], const float b[3], const float c[3], int* dtype);
float orc_ee_dist2(const float a0[3], const float a1[3], const float b0[3], const float b1[3], int* dtype);
void orc_pt_grad(const float p[3], const float a[3], const float b[3], const float c[3], float out[12]);
void orc_ee_grad(const float a0[3], const float a1[3], const float b0[3], const float b1[3], float out[12]);
int orc_vt_ccd(const float* p0, const float* p1, const float* a0, const float* a1,
               const float* b0, const float* b1, const float* c0, const float* c1, float* toi);
int orc_ee_ccd(const float* a0, const float* a1, const float* b0, const float* b1,
               const float* c0, const float* c1, const float* d0, const float* d1, float* toi);
int orc_cubic_roots(float a, float b, float c, float d, float roots[3]);
float orc_barrier_energy(float d, float d_hat);
float orc_barrier_gradient(float d, float d_hat);
float orc_barrier_hessian(float d, float d_hat);
float orc_scaled_barrier_gradient(float d, float d_hat, float kappa);
float orc_barrier_energy_thick(float d, float d_hat, float t);
float orc_barrier_gradient_thick(float d, float d_hat, float t);
float orc_estimate_kappa(float configured, float avg_mass, float g, float d_hat);
void orc_polar(const float f[6], float rot[6], float stretch[4], float sv[2]);

// ---- contact queries on explicit positions (for pair-set parity) ----
// Candidate triangle pairs (ta<tb) whose AABBs, inflated by `margin`, overlap.
// mode 0: complete set; mode 1: the reference's freshly built median-split BVH.
// Returns the count; writes at most `cap` pairs (2 u32 each), sorted.
uint64_t orc_tri_pairs(uint32_t nv, const float* px, const float* py, const float* pz,
                       uint32_t nt, const uint32_t* tris, float margin, int mode,
                       uint32_t* out, uint64_t cap);
// Vertex-triangle CCD hits over candidate pairs (reference ccd.rs:238-292),
// evaluated in FP64; writes (vertex, triangle) hits sorted; returns min TOI.
float orc_ccd_hits(uint32_t nv, const float* p0x, const float* p0y, const float* p0z,
                   const float* p1x, const float* p1y, const float* p1z,
                   uint32_t nt, const uint32_t* tris, uint64_t npairs, const uint32_t* pairs,
                   uint32_t* hits, uint64_t cap, uint64_t* nhits);
// Full IPC detect at explicit positions (CollisionPipeline::detect_ipc_contacts,
// collision_pipeline.rs:207-352). Outputs per-vertex gradient / normal / flag.
void orc_detect(void* sim, const orc_contact* contact, float d_hat,
                const float* px, const float* py, const float* pz,
                float* gx, float* gy, float* gz, float* nx, float* ny, float* nz,
                uint8_t* in_contact, float* max_violation, uint32_t* active);

#ifdef __cplusplus
}
#endif
