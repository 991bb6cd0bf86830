/*
 * vistio_cuda.h — C ABI of the B200 (sm_100a) Projective Dynamics + IPC drape
 * solver. Plain C types only; every call returns a vistio_status.
 *
 * Each group of entry points replaces one interface of the reference
 * (Rust, MTawhid7/Vistio). Paths cite files inside that project:
 *
 *   vistio_solver_init*        SolverStrategy::init            crates/vistio-solver/src/strategy.rs:42-56
 *                              ProjectiveDynamicsSolver::init  crates/vistio-solver/src/pd_solver.rs:221-257
 *                              ::init_with_material            pd_solver.rs:106-143
 *                              ::init_with_material_tier3/4    pd_solver.rs:152-211
 *   vistio_solver_lumped_masses  ::lumped_masses               pd_solver.rs:95-97
 *   vistio_solver_set/get_state  SimulationState fields        crates/vistio-solver/src/state.rs:23-140
 *   vistio_step                SolverStrategy::step            strategy.rs:57-64, pd_solver.rs:259-476
 *   vistio_step_with_ipc       ::step_with_ipc                 pd_solver.rs:549-1157, with the handler
 *                              IpcCollisionHandler             pd_solver.rs:483-489 implemented inside
 *                              the library as CollisionPipeline::detect_ipc_contacts / compute_ccd_step
 *                              crates/vistio-contact/src/collision_pipeline.rs:207-400
 *   vistio_sparse_factorize/solve  SparseSolver                crates/vistio-math/src/sparse.rs:110-120,
 *                              FaerSolver                      crates/vistio-math/src/faer_solver.rs:25-129
 *   vistio_broadphase_pairs    BroadPhase::update + query_triangle_pairs  crates/vistio-contact/src/broad.rs:39-56
 *   vistio_ccd_hits            compute_max_step_size           crates/vistio-contact/src/ccd.rs:238-292
 *   vistio_batch_*             (no counterpart: the reference steps one garment at a time)
 *
 * Threading: a context is used from one host thread at a time. Device work
 * runs on the context's stream; the calls that return host data synchronise.
 */
#ifndef VISTIO_CUDA_H
#define VISTIO_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: VistioError variants (crates/vistio-types/src/error.rs:9-44)
 * plus the device-side conditions. */
typedef enum vistio_status {
  VISTIO_OK = 0,
  VISTIO_ERR_INVALID_MESH = 1,      /* VistioError::InvalidMesh */
  VISTIO_ERR_INVALID_MATERIAL = 2,  /* VistioError::InvalidMaterial */
  VISTIO_ERR_INVALID_CONFIG = 3,    /* VistioError::InvalidConfig (also: not initialised) */
  VISTIO_ERR_IO = 4,                /* VistioError::Io */
  VISTIO_ERR_SERIALIZATION = 5,     /* VistioError::Serialization */
  VISTIO_ERR_GPU = 6,               /* VistioError::Gpu: a CUDA call failed */
  VISTIO_ERR_SOLVER_DIVERGENCE = 7, /* VistioError::SolverDivergence: non-finite state */
  VISTIO_ERR_INVARIANT = 8,         /* VistioError::InvariantViolation */
  VISTIO_ERR_TIMEOUT = 9,           /* a bounded device wait gave up */
  VISTIO_ERR_OOM = 10,              /* device allocation failed / over the memory budget */
  VISTIO_ERR_NOT_SPD = 11,          /* Cholesky pivot <= 0 (reported by the reference as InvalidConfig) */
  VISTIO_ERR_CAPACITY = 12          /* an output buffer is too small */
} vistio_status;

typedef struct vistio_ctx vistio_ctx;
typedef struct vistio_solver vistio_solver;
typedef struct vistio_batch vistio_batch;
typedef struct vistio_factor vistio_factor;

/* TriangleMesh (crates/vistio-mesh/src/mesh.rs): SoA positions + u32 indices. */
typedef struct vistio_mesh_desc {
  uint32_t vertex_count;
  uint32_t triangle_count;
  const float* pos_x;
  const float* pos_y;
  const float* pos_z;
  const uint32_t* indices; /* 3 * triangle_count */
} vistio_mesh_desc;

/* Live fields of SolverConfig (crates/vistio-solver/src/config.rs:10-129).
 * Fields the reference declares but never reads on this path
 * (contact_weight, chebyshev_acceleration, spectral_radius,
 * self_collision_d_hat, cloth_thickness, ccd_enabled, material_name) are
 * not carried. */
typedef struct vistio_solver_config {
  uint32_t max_iterations;
  uint32_t al_max_iterations;
  double tolerance;
  float gravity[3];
  float damping;
  float stretch_weight;
  float bending_weight;
  float rayleigh_mass_damping;
  float barrier_d_hat;   /* squared-distance activation threshold */
  float barrier_kappa;   /* 0 = estimate (barrier.rs:97) */
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
  /* FP64 iterative refinement of the global solve (no counterpart in the
   * reference, whose solve runs in FP64): after the FP32 sweeps, the residual
   * b - A d is formed in FP64 from the factored matrix and the sweeps solve for
   * the correction, this many times (0, 1 or 2). step_with_ipc refines every
   * solve; the plain step refines its last iteration's solve (each earlier
   * iteration's error is corrected by the next iteration's residual). */
  uint32_t refinement_sweeps;
  /* Where the numeric FP64 Cholesky factorization of the system matrix runs
   * (faer's LL^T in the reference, faer_solver.rs:67-93). 0: on the GPU,
   * multifrontal, when the garment is first packed into a batch; the host
   * computes the ordering and the symbolic structure. 1: on the host. */
  uint32_t host_factorization;
  uint32_t reserved0; /* must be 0 */
} vistio_solver_config;

/* FabricProperties (crates/vistio-material/src/properties.rs:23-58). */
typedef struct vistio_material_desc {
  float density;                 /* g/m^2 */
  float stretch_stiffness_warp;
  float stretch_stiffness_weft;
  float shear_stiffness;         /* carried, unused by the reference's PD path */
  float bending_stiffness_warp;
  float bending_stiffness_weft;
  float thickness;
  float friction;
  float damping;
} vistio_material_desc;

/* ConstitutiveModel implementations (crates/vistio-material/src/traits.rs:36-56). */
typedef enum vistio_model_kind {
  VISTIO_MODEL_ARAP = 0,         /* ElementData::project, the `init` path (element.rs:127) */
  VISTIO_MODEL_COROTATIONAL = 1, /* CoRotationalModel (corotational.rs:50) */
  VISTIO_MODEL_ORTHOTROPIC = 2,  /* OrthotropicLinearModel (orthotropic.rs:50) */
  VISTIO_MODEL_ANISOTROPIC = 3,  /* AnisotropicCoRotationalModel (anisotropic.rs:77) */
  VISTIO_MODEL_ISOTROPIC_LINEAR = 4 /* IsotropicLinearModel (isotropic.rs:41) */
} vistio_model_kind;

typedef struct vistio_model_desc {
  int32_t kind;          /* vistio_model_kind */
  float warp_stiffness;  /* ORTHOTROPIC / ANISOTROPIC */
  float weft_stiffness;
} vistio_model_desc;

typedef enum vistio_bending_kind {
  VISTIO_BENDING_NONE = 0,
  VISTIO_BENDING_DIHEDRAL = 1,       /* BendingData (bending.rs:44) */
  VISTIO_BENDING_DISCRETE_SHELLS = 2,/* DiscreteShellsBendingData (discrete_shells.rs:81) */
  VISTIO_BENDING_DISCRETE_SHELLS_ANISOTROPIC = 3
} vistio_bending_kind;

/* The explicit form every init path reduces to. */
typedef struct vistio_setup_desc {
  int32_t model;          /* vistio_model_kind */
  int32_t bending;        /* vistio_bending_kind */
  float stiffness;        /* element weight = stiffness * rest area */
  float bend_stiffness;   /* hinge weight = bend_stiffness * rest edge length */
  float density_gsm;      /* lumped-mass area density, g/m^2 */
  float warp_stiffness, weft_stiffness;
  float bend_warp, bend_weft;
  float matrix_dt;        /* dt of the system matrix; the reference always uses 1/60 */
} vistio_setup_desc;

/* What the reference's RunnerIpcHandler wires into the CollisionPipeline
 * (crates/vistio-bench/src/runner.rs:48-99,190-204). */
typedef struct vistio_contact_desc {
  int32_t has_ground;
  float ground_height;       /* y of the ground plane (Y-up) */
  int32_t has_sphere;
  float sphere_center[3];
  float sphere_radius;
  int32_t self_collision;    /* triangle self contact, 1-ring exclusion */
  float kappa;               /* barrier stiffness; <= 0 estimates it from avg vertex mass */
  float thickness;           /* C-IPC thickness for self contacts (runner: 1.5 * d_hat) */
  /* CylinderCollider (crates/vistio-contact/src/cylinder.rs:11-21): a vertical
   * cylinder of the given radius around (center_x, center_z) with its top face
   * at top_y, reaching down without end (the Cusick drape pedestal). */
  int32_t has_cylinder;
  float cylinder_center_x, cylinder_center_z, cylinder_top_y, cylinder_radius;
  /* BoxCollider (crates/vistio-contact/src/box_collider.rs): an axis-aligned
   * box [box_min, box_max] (the cantilever shelf). */
  int32_t has_box;
  float box_min[3], box_max[3];
} vistio_contact_desc;

/* StepResult (strategy.rs:15-24) plus contact diagnostics. */
typedef struct vistio_step_result {
  uint32_t iterations;
  int32_t converged;
  double final_residual;
  double wall_time;          /* seconds, host clock around the call */
  uint32_t al_iterations;
  uint32_t active_contacts;
  float last_alpha;
  int32_t status;
} vistio_step_result;

/* ContactResult (crates/vistio-contact/src/response.rs:13-20). */
typedef struct vistio_contact_result {
  uint32_t resolved_count;
  float max_residual_penetration;
  float total_force_magnitude;   /* the sum of the depths resolved */
} vistio_contact_result;

/* The collider rows of CollisionStepResult (collision_pipeline.rs:405-420). */
typedef struct vistio_collider_results {
  vistio_contact_result ground, sphere, cylinder, box;
} vistio_collider_results;

/* ---- context ---- */
vistio_status vistio_ctx_create(int32_t device, vistio_ctx** out);
vistio_status vistio_ctx_destroy(vistio_ctx* ctx);
const char* vistio_status_string(vistio_status s);
const char* vistio_last_error(const vistio_ctx* ctx);
vistio_status vistio_sync(vistio_ctx* ctx);

/* ---- solver (one garment) ---- */
vistio_status vistio_solver_init(vistio_ctx* ctx, const vistio_mesh_desc* mesh, const vistio_solver_config* cfg,
                                 const uint8_t* pinned, vistio_solver** out);
vistio_status vistio_solver_init_with_material(vistio_ctx* ctx, const vistio_mesh_desc* mesh,
                                               const vistio_solver_config* cfg, const vistio_material_desc* material,
                                               const vistio_model_desc* model, int32_t bending_kind,
                                               const uint8_t* pinned, vistio_solver** out);
vistio_status vistio_solver_init_explicit(vistio_ctx* ctx, const vistio_mesh_desc* mesh,
                                          const vistio_solver_config* cfg, const vistio_setup_desc* setup,
                                          const uint8_t* pinned, vistio_solver** out);
vistio_status vistio_solver_destroy(vistio_solver* s);
const char* vistio_solver_name(const vistio_solver* s); /* "ProjectiveDynamics" */
/* A new solver with the same set-up (mesh data, factor, configuration) and
 * the source's current state, bound to `ctx`; it saves the set-up cost when
 * the same garment, material and dt are simulated again. */
vistio_status vistio_solver_clone(vistio_solver* s, vistio_ctx* ctx, vistio_solver** out);
/* Device bytes the garment occupies inside a batch (with the self-contact
 * buffers when self_contact != 0): the admission estimate of a server. */
vistio_status vistio_solver_device_bytes(const vistio_solver* s, int32_t self_contact, uint64_t* bytes);
vistio_status vistio_solver_info(const vistio_solver* s, uint32_t* nv, uint32_t* nt, uint32_t* nh,
                                 uint64_t* nnz_a, uint64_t* nnz_l, uint32_t* nsupernodes, uint32_t* nlevels);
vistio_status vistio_solver_lumped_masses(const vistio_solver* s, float* out);
vistio_status vistio_solver_set_ground(vistio_solver* s, int32_t has_ground, float height);
vistio_status vistio_solver_set_state(vistio_solver* s, const float* px, const float* py, const float* pz,
                                      const float* vx, const float* vy, const float* vz);
vistio_status vistio_solver_get_state(vistio_solver* s, float* px, float* py, float* pz, float* vx, float* vy,
                                      float* vz);
/* Per vertex, the magnitude of the contact barrier gradient (colliders and
 * self contact) of the last detect of the last step_with_ipc; zeros before
 * any contact step. No counterpart in the reference's solver API: it fills
 * the I/O contract's VertexMetadata::contact_force (crates/vistio-io/src/
 * contract.rs:79-88). */
vistio_status vistio_solver_contact_force(vistio_solver* s, float* out);
vistio_status vistio_step(vistio_solver* s, float dt, vistio_step_result* res);
vistio_status vistio_step_with_ipc(vistio_solver* s, float dt, const vistio_contact_desc* contact,
                                   vistio_step_result* res);
/* The runner's non-IPC branch after vistio_step (runner.rs:209-215 calling
 * CollisionPipeline::step, collision_pipeline.rs:117-199, with the runner's
 * thickness and stiffness of 0, which leave out the mesh contacts):
 * GroundPlane::resolve twice, then SphereCollider, CylinderCollider and
 * BoxCollider ::resolve, each on the colliders `contact` enables; the self
 * collision and kappa fields are not read. Positions and velocities of the
 * vertices inside a collider are projected onto its surface; `res` may be
 * NULL. */
vistio_status vistio_resolve_contacts(vistio_solver* s, const vistio_contact_desc* contact,
                                      vistio_collider_results* res);

/* ---- batches: many garments advanced together from HBM-resident ragged SoA ---- */
vistio_status vistio_batch_create(vistio_ctx* ctx, vistio_solver* const* solvers, uint32_t n, vistio_batch** out);
vistio_status vistio_batch_destroy(vistio_batch* b);
/* Advances every instance `nsteps` steps of size dt; contact may be NULL. Asynchronous. */
vistio_status vistio_batch_step(vistio_batch* b, float dt, uint32_t nsteps, const vistio_contact_desc* contact);
/* vistio_resolve_contacts on every garment of the batch with the same
 * colliders; res, when not NULL, holds one entry per garment. */
vistio_status vistio_batch_resolve_contacts(vistio_batch* b, const vistio_contact_desc* contact,
                                            vistio_collider_results* res);
vistio_status vistio_batch_set_state(vistio_batch* b, uint32_t k, const float* px, const float* py, const float* pz,
                                     const float* vx, const float* vy, const float* vz);
vistio_status vistio_batch_get_state(vistio_batch* b, uint32_t k, float* px, float* py, float* pz, float* vx,
                                     float* vy, float* vz);
/* Whole-batch positions in instance order (3 * total vertices, interleaved xyz), one copy each way. */
vistio_status vistio_batch_upload_positions(vistio_batch* b, const float* xyz);
vistio_status vistio_batch_download_positions(vistio_batch* b, float* xyz);
vistio_status vistio_batch_info(const vistio_batch* b, uint32_t* n_instances, uint64_t* total_vertices,
                                uint64_t* total_triangles, uint64_t* total_hinges, uint64_t* factor_bytes,
                                uint64_t* device_bytes);
/* Autotuner of the sweeps (no counterpart in the reference). Two things are
 * chosen by timing this batch's forward and backward sweeps:
 * - the sweep kind: 0 = one kernel launch per level of the supernodal trees;
 *   1 = one dependency-driven launch for both directions, in which each
 *   supernode waits only for its own children (forward) or parent (backward);
 *   2 (batches with garment groups: at least 8 garments of one mesh topology)
 *   = the bottom of the groups' trees swept one lane per garment, before and
 *   after kind 1 sweeps the rest; the same results, bit for bit, as kind 1 at
 *   the limit 6144;
 * - which top-level supernodes a single warp takes and which a whole block,
 *   by a limit on s (s + m): 0, 1024, 2048, 4096, 6144, 12288 and 2^30.
 * candidate_ms (21 entries, may be NULL) receives the time of each limit for
 * kind 0 (entries 0-6) and kind 1 (entries 7-13); entries 14-20 time kind 2 at
 * kind 1's fastest limit with the group limits 0, 64, 128, 256, 512, 1024 and
 * 6144 (the largest s (s + m) of a supernode above the bottom subtrees that
 * the groups sweep one lane per garment; -1 without garment groups or above
 * that warp-item limit). The fastest candidate is kept (*chosen_limit; the
 * kind from vistio_batch_get_sweep_mode, the group limit from
 * vistio_batch_get_group_limit). Without tuning: kind 2 if the batch has
 * garment groups, else kind 1, with the limits 6144. For kinds 1 and 2 the
 * chosen schedule is then timed with both compiled forms of the dependency-
 * driven kernel (vistio_batch_get_sweep_blocks). Captured step graphs are
 * rebuilt on the next step. Synchronises the batch's stream. */
vistio_status vistio_batch_tune(vistio_batch* b, uint32_t* chosen_limit, float* candidate_ms);
/* Autotunes the shapes of the local steps on this batch (no reference
 * counterpart): triangles per thread of the membrane step (1: 256 threads
 * per chunk of 256 triangles; 2: 128 threads, both triangles' loads issued
 * first) and hinges per thread of the bending step (the same two shapes),
 * each timed over five launches; the faster of each pair is kept. The shapes
 * compute the same arithmetic per element: results are bit-identical.
 * candidate_ms (4 entries, may be NULL): membrane 1, 2, bending 1, 2. Without
 * tuning: 2 triangles and 1 hinge per thread. Synchronises the stream. */
vistio_status vistio_batch_tune_local(vistio_batch* b, uint32_t* tri_per_thread, uint32_t* hinge_per_thread,
                                      float* candidate_ms);
/* Sets the local steps' elements per thread directly (1 or 2 each). */
vistio_status vistio_batch_set_local_shape(vistio_batch* b, uint32_t tri_per_thread, uint32_t hinge_per_thread);
/* How the self-contact CCD step bound (compute_max_step_size,
 * crates/vistio-contact/src/ccd.rs:238-292) visits its vertex-triangle tests.
 * on = 1 (default): the detect that opens each AL pass lists every test of
 * its candidate pairs once (a vertex of A meets triangle B again in each
 * other pair (A', B) with the vertex in A', about 2.6 times per test on a
 * cloth mesh) and the pass's CCDs run over that list; 0: every test of every
 * pair, as the reference does. The minimum, and so every step, is
 * bit-identical either way. No reference counterpart. */
vistio_status vistio_batch_set_self_ccd_dedup(vistio_batch* b, uint32_t on);
/* Sets / reads the group limit of sweep kind 2 (see vistio_batch_tune; at
 * most 6144; the batch must have garment groups). No reference counterpart. */
vistio_status vistio_batch_set_group_limit(vistio_batch* b, uint32_t limit);
vistio_status vistio_batch_get_group_limit(const vistio_batch* b, uint32_t* limit);
/* Sets the warp-item limit directly (any value; see vistio_batch_tune). */
vistio_status vistio_batch_set_warp_limit(vistio_batch* b, uint32_t limit);
/* Sets the sweep kind (0, 1, or 2 for a batch with garment groups; see
 * vistio_batch_tune). */
vistio_status vistio_batch_set_sweep_mode(vistio_batch* b, uint32_t mode);
/* The sweep kind and warp-item limit in use. */
vistio_status vistio_batch_get_sweep_mode(const vistio_batch* b, uint32_t* mode, uint32_t* warp_limit);
/* The dependency-driven sweep kernel (kinds 1 and 2) is compiled in three
 * forms, named by resident blocks per SM: 5 and 4 (eight-warp blocks, 48 and
 * 64 registers per thread) and 2 (sixteen-warp blocks, whose units hold twice
 * as many items); no reference counterpart. vistio_batch_tune times the three
 * with the schedule it chose and keeps the fastest; without tuning, 2 for a
 * batch of at most 8 garments, else 4. All give the same results, bit for
 * bit. get: the form in use and, in tuned_ms (3 entries, may be NULL), the
 * tuner's times of the forms 5, 4 and 2 (-1 before tuning or for kind 0). */
vistio_status vistio_batch_set_sweep_blocks(vistio_batch* b, uint32_t blocks_per_sm);
vistio_status vistio_batch_get_sweep_blocks(const vistio_batch* b, uint32_t* blocks_per_sm, float* tuned_ms);
/* The device factorization done when the batch was created (the garments
 * whose solver config has host_factorization = 0): its kernel launches (one
 * per height of the supernodal trees per group of garments) and their device
 * time in milliseconds; 0 and 0 when every garment was factorized on the host. */
vistio_status vistio_batch_factor_stats(const vistio_batch* b, uint32_t* launches, float* device_ms);
/* Kernel launches in one batch step (graph nodes), for launch accounting. */
vistio_status vistio_batch_launches_per_step(const vistio_batch* b, uint32_t* launches);
/* The stream the batch runs on (cudaStream_t as void*), for event timing. */
void* vistio_batch_stream(vistio_batch* b);
/* Launches one kernel phase of a plain PD iteration on the batch stream, for
 * per-kernel timing: 0 predict, 1 local membrane, 2 local bending, 3 residual
 * gather, 4 forward + back substitution (no position update), 5 finalize.
 * Uses the step constants of the last vistio_batch_step call. Asynchronous. */
vistio_status vistio_batch_launch_phase(vistio_batch* b, int32_t phase);
/* Algorithmic bytes of one launch of a phase over the whole batch (see
 * vistio_batch_launch_phase), from the batch's element counts and factor sizes:
 * stored factor entries are counted at 4 bytes each. */
vistio_status vistio_batch_phase_bytes(const vistio_batch* b, int32_t phase, uint64_t* bytes);

/* ---- serving: continuous batching of drape requests ----
 * No counterpart in the reference, whose runner simulates one scenario at a
 * time. Requests are submitted with their own mesh, material, contact set-up,
 * dt and step count. Host threads build each request's set-up (cached by
 * topology, material, configuration and dt). At every vistio_server_tick the
 * ready requests that share a step configuration are packed into a new cohort
 * (one batch, on its own stream) when the device-memory budget allows, so
 * requests arriving while others run are admitted at once and their work
 * overlaps on the GPU. A finished cohort hands back its states and frees its
 * memory without synchronising the device. One host thread calls
 * submit / tick / query / result; the set-up threads are internal. */
typedef struct vistio_server vistio_server;

typedef struct vistio_server_config {
  int32_t device;
  uint64_t hbm_budget_bytes;  /* admission budget for resident cohorts */
  uint32_t max_cohort;        /* most requests packed into one cohort */
  uint32_t setup_threads;     /* host threads building set-ups (>= 1) */
  uint32_t steps_per_slice;   /* steps queued per cohort ahead of the GPU (>= 1) */
  uint64_t cache_bytes;       /* host memory for cached set-ups (0: no cache) */
  /* 0: the set-up threads compute each request's numeric factorization on the
   * host, in parallel with the GPU's work (each request's host_factorization
   * is overridden); 1: each request's own setting (0 = its cohort factorizes
   * on the GPU when it starts, on the thread that calls vistio_server_tick). */
  uint32_t gpu_factorization;
  /* Sweep kind of every cohort (vistio_batch_set_sweep_mode): 0 = one launch
   * per level, 1 = dependency-driven. Cohorts run side by side on their own
   * streams, and the dependency-driven sweeps keep blocks resident that wait
   * for one another, so 0 suits a busy server. */
  uint32_t sweep_mode;
  /* Admission window: while any cohort is running, ready requests of one step
   * configuration wait up to this long (from the first one's readiness) for
   * others to form a larger cohort, unless max_cohort of them are ready.
   * Fewer, larger cohorts keep the GPU's work in fewer, wider launches. 0:
   * every tick starts a cohort with whatever is ready. */
  uint32_t admit_wait_ms;
} vistio_server_config;

typedef struct vistio_request {
  vistio_mesh_desc mesh;
  const uint8_t* pinned;          /* may be NULL */
  vistio_solver_config config;
  vistio_setup_desc setup;
  int32_t has_contact;            /* 0: SolverStrategy::step, 1: step_with_ipc */
  vistio_contact_desc contact;    /* with has_contact 0 only has_ground / ground_height are used */
  float dt;
  uint32_t steps;
} vistio_request;

typedef enum vistio_request_state {
  VISTIO_REQ_QUEUED = 0,   /* waiting for a set-up thread */
  VISTIO_REQ_SETUP = 1,    /* set-up being built */
  VISTIO_REQ_READY = 2,    /* waiting for admission */
  VISTIO_REQ_RUNNING = 3,  /* in a cohort on the GPU */
  VISTIO_REQ_DONE = 4,
  VISTIO_REQ_FAILED = 5
} vistio_request_state;

typedef struct vistio_request_info {
  int32_t state;            /* vistio_request_state */
  int32_t status;           /* vistio_status of a failed request */
  uint32_t vertex_count;
  uint32_t cohort;          /* cohort id (0 before admission) */
  int32_t cache_hit;        /* set-up taken from the cache */
  double submit_s, ready_s, start_s, done_s;  /* server clock, seconds */
} vistio_request_info;

typedef struct vistio_server_stats {
  uint64_t submitted, completed, failed;
  uint64_t cohorts_started, cohorts_active, max_cohorts_active;
  uint64_t bytes_in_use, max_bytes_in_use;
  uint64_t cache_hits, cache_misses;
  uint64_t instance_steps;  /* steps of completed requests */
  double p50_latency_s, p99_latency_s, mean_latency_s;  /* submit -> done, completed requests */
  double throughput;        /* instance_steps / (last completion - first submission) */
} vistio_server_stats;

vistio_status vistio_server_create(const vistio_server_config* cfg, vistio_server** out);
vistio_status vistio_server_destroy(vistio_server* s);
const char* vistio_server_last_error(const vistio_server* s);
vistio_status vistio_server_submit(vistio_server* s, const vistio_request* r, uint64_t* id);
/* One scheduling round: retire finished cohorts, queue the next slice of
 * running ones, admit ready requests. *unfinished (may be NULL) = requests not
 * yet done or failed. Does not wait for the GPU. */
vistio_status vistio_server_tick(vistio_server* s, uint32_t* unfinished);
/* Ticks until every submitted request is done or failed, or timeout_s passes
 * (VISTIO_ERR_TIMEOUT). */
vistio_status vistio_server_drain(vistio_server* s, double timeout_s);
vistio_status vistio_server_query(vistio_server* s, uint64_t id, vistio_request_info* info);
/* Final state of a done request (vertex_count entries each). */
vistio_status vistio_server_result(vistio_server* s, uint64_t id, float* px, float* py, float* pz, float* vx,
                                   float* vy, float* vz);
/* Forgets a done or failed request (its result memory). */
vistio_status vistio_server_release(vistio_server* s, uint64_t id);
vistio_status vistio_server_get_stats(vistio_server* s, vistio_server_stats* st);

/* ---- diagnostics (no counterpart in the reference) ---- */
/* Runs the bounded barrier wait the sweep kernels use on a barrier nothing
 * completes. The wait gives up after `polls` polls (1..2^22) and the call
 * returns VISTIO_ERR_TIMEOUT, as a step whose staging copy never landed would;
 * the context stays usable. Exercises the device-side failure path without a
 * fault. */
vistio_status vistio_diag_wait_timeout(vistio_ctx* ctx, uint32_t polls);

/* ---- symbolic analysis cache ---- */
/* The host keeps the symbolic factorizations it computes (ordering,
 * supernodes, row structures, sweep schedules) in a process-wide cache keyed
 * by the exact matrix pattern and dissection order; a hit returns what a new
 * analysis would compute. Garments that share a mesh topology, at any uniform
 * scale, then pay for the analysis once. It serves the set-ups whose numbers
 * are factorized on the GPU (host_factorization = 0, the default) and
 * vistio_sparse_factorize. No counterpart in the reference. */
vistio_status vistio_symbolic_cache_info(uint64_t* hits, uint64_t* misses, uint64_t* bytes, uint64_t* entries);
/* Bound on the bytes it holds (default 1 GiB), least recently used out
 * first; 0 empties and disables it. */
vistio_status vistio_symbolic_cache_set_limit(uint64_t bytes);

/* ---- SparseSolver mirror ---- */
vistio_status vistio_sparse_factorize(vistio_ctx* ctx, uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                                      const float* values, vistio_factor** out);
vistio_status vistio_sparse_solve(vistio_factor* f, const float* rhs, float* solution);
vistio_status vistio_sparse_destroy(vistio_factor* f);

/* ---- contact boundary queries ---- */
/* Candidate triangle pairs (ta < tb) whose AABBs inflated by `margin` overlap,
 * computed on the GPU (balanced tree over mesh-order triangles, count / scan /
 * write). Writes up to `cap` pairs sorted; *count = total. */
vistio_status vistio_broadphase_pairs(vistio_ctx* ctx, uint32_t nv, const float* px, const float* py, const float* pz,
                                      uint32_t nt, const uint32_t* tris, float margin, uint32_t* pairs, uint64_t cap,
                                      uint64_t* count);
/* Allocation-free variant of vistio_broadphase_pairs (no counterpart in the
 * reference). Same inputs and the same sorted pair list, but the call allocates
 * and frees no device memory: every buffer it uses lives in one fixed region
 * (about 16 MB) built into the library. For callers that cannot allocate on
 * the call: a server whose device memory is fully committed to resident
 * garments (a cudaMalloc could fail there), or a per-frame collision query on
 * a latency-critical thread, where cudaFree would synchronise the whole device.
 * Limits: at most VISTIO_NOALLOC_MAX_TRIANGLES triangles and
 * VISTIO_NOALLOC_MAX_VERTICES vertices (else VISTIO_ERR_CAPACITY before any
 * device work), and at most VISTIO_NOALLOC_MAX_PAIRS candidate pairs (else
 * VISTIO_ERR_CAPACITY with *count set). pairs == NULL queries the count;
 * cap < *count returns VISTIO_ERR_CAPACITY and writes nothing.
 * The call makes the context's device current, looks up the region's address
 * (cudaGetSymbolAddress) and is synchronous: it returns with the pairs on the
 * host, so it cannot be captured into a CUDA graph. The triangles are not
 * reordered by Morton code first (vistio_broadphase_pairs does that): the tree
 * is built over mesh order, which finds the same pairs at a traversal cost that
 * depends on how spatially ordered the mesh is. The region is shared by every
 * call on the device: calls on one device must not overlap (two threads or two
 * contexts with calls in flight at once race on it). Each call clears the
 * counters it needs; nothing has to be zeroed by the caller. */
#define VISTIO_NOALLOC_MAX_TRIANGLES 65536u
#define VISTIO_NOALLOC_MAX_VERTICES 65536u
#define VISTIO_NOALLOC_MAX_PAIRS 1048576u
vistio_status vistio_broadphase_pairs_noalloc(vistio_ctx* ctx, uint32_t nv, const float* px, const float* py,
                                              const float* pz, uint32_t nt, const uint32_t* tris, float margin,
                                              uint32_t* pairs, uint64_t cap, uint64_t* count);
/* Vertex-triangle CCD over candidate pairs on the GPU: sorted unique
 * (vertex, triangle) hits and the minimum safe TOI. */
vistio_status vistio_ccd_hits(vistio_ctx* ctx, uint32_t nv, const float* p0, const float* p1, uint32_t nt,
                              const uint32_t* tris, uint64_t npairs, const uint32_t* pairs, uint32_t* hits,
                              uint64_t cap, uint64_t* nhits, float* min_toi);
/* The device's barrier gradient for n squared distances d2: kappa b'(d2)
 * (crates/vistio-contact/src/barrier.rs:35-46 and the scaled form's clamp of
 * non-finite values, :78-87), or with thickness > 0 the C-IPC form
 * b'(d2 - thickness^2) (:138-163), in FP64 as the contact kernels evaluate
 * it. Test-only. */
vistio_status vistio_barrier_grad(vistio_ctx* ctx, uint32_t n, const double* d2, double d_hat, double kappa,
                                  double thickness, double* out);

#ifdef __cplusplus
}
#endif
#endif /* VISTIO_CUDA_H */
