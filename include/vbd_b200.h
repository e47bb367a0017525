/*
 * vbd_b200.h -- C ABI of the B200 (sm_100a) Vertex Block Descent cloth library.
 *
 * This is the drop-in boundary for Newton's particle VBD cloth step.  Every entry point is
 * plain C: integers, floats, and host or device pointers.  No torch, Warp or CUDA types
 * appear in a signature; a CUDA stream is passed as `void*` (a `cudaStream_t`, NULL for the
 * legacy default stream).
 *
 * Reference interfaces that each entry point replaces (paths inside the Newton source tree):
 *
 *   vbd_model_create      ModelBuilder.finalize -> Model particle/tri/edge/adjacency/coloring
 *                         arrays (newton/_src/sim/builder.py:10962, :11033-11070, :11796-11832)
 *                         and MeshAdjacency.init_vertex_adjacency (newton/_src/utils/mesh.py:595)
 *   vbd_collide           CollisionPipeline.collide soft-contact branch
 *                         (newton/_src/sim/collide.py:1553-1590) -> create_soft_contacts
 *                         (newton/_src/geometry/kernels.py:1020-1184)
 *   vbd_solver_create     SolverVBD.__init__ particle part
 *                         (newton/_src/solvers/vbd/solver_vbd.py:221-618)
 *   vbd_step              SolverVBD.step (newton/_src/solvers/vbd/solver_vbd.py:1774-1825),
 *                         i.e. SolverBase.step(state_in, state_out, control, contacts, dt)
 *                         (newton/_src/solvers/solver.py:358-373)
 *   vbd_forward           SolverVBD._initialize_particles (solver_vbd.py:2065-2100):
 *                         forward_step + apply_truncation_ts
 *   vbd_sweep_color       one color of SolverVBD._solve_particle_iteration (solver_vbd.py:2552-2702):
 *                         accumulate_particle_body_contact_force_and_hessian +
 *                         solve_elasticity(_tile) + apply_truncation_ts
 *   vbd_finalize          end of _solve_particle_iteration (copy, solver_vbd.py:2704) +
 *                         SolverVBD._finalize_particles / update_velocity (solver_vbd.py:3158-3169)
 *   vbd_residual          no reference counterpart: the per-vertex force residual used to gate
 *                         iterations (Jacobi evaluation of the same force the sweep solves)
 *   vbd_color_graph       ModelBuilder.color -> color_graph (newton/_src/sim/graph_coloring.py:243-311),
 *                         whose assignment in the reference is done by Warp's native
 *                         graph_coloring_assign / graph_coloring_balance
 *
 * Status: every function returns 0 (VBD_OK) on success or a VBD_ERR_* code; the message of
 * the last failure on the calling thread is returned by vbd_last_error().
 *
 * Memory: vbd_model_create and vbd_solver_create allocate all device memory the solver will
 * ever use.  vbd_step, vbd_forward, vbd_sweep_color, vbd_finalize, vbd_residual and
 * vbd_collide allocate nothing.
 *
 * Threading: a solver is not thread-safe (its scratch is mutable), exactly like the reference.
 */
#ifndef VBD_B200_H
#define VBD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------- */
#define VBD_OK 0
#define VBD_ERR_INVALID_ARGUMENT 1
#define VBD_ERR_CUDA 2
#define VBD_ERR_OUT_OF_MEMORY 3
#define VBD_ERR_TIMEOUT 4
#define VBD_ERR_UNSUPPORTED 5

/* ---- reference enumerations (values kept identical) ---------------------------------- */
/* ParticleFlags (newton/_src/geometry/flags.py:8) */
#define VBD_PARTICLE_ACTIVE 1
/* ShapeFlags.COLLIDE_PARTICLES (newton/_src/geometry/flags.py:38) */
#define VBD_SHAPE_COLLIDE_PARTICLES 4
/* GeoType (newton/_src/geometry/types.py:70) -- the static primitives this path supports */
#define VBD_GEO_PLANE 1
#define VBD_GEO_SPHERE 3
#define VBD_GEO_BOX 7

/* A static collision shape (Model.shape_* arrays with shape_body == -1). */
typedef struct VbdShape {
    int32_t geo_type;      /* VBD_GEO_* */
    int32_t flags;         /* ShapeFlags bits; VBD_SHAPE_COLLIDE_PARTICLES enables particle contact */
    int32_t world;         /* shape_world, -1 = global */
    int32_t reserved;
    float xform[7];        /* shape_transform: position xyz, quaternion xyzw */
    float scale[3];        /* shape_scale: plane (width, length, 0); sphere (r, -, -); box (hx, hy, hz) */
    float margin;          /* shape_margin [m] */
    float material_ke;     /* shape_material_ke */
    float material_kd;     /* shape_material_kd */
    float material_mu;     /* shape_material_mu */
} VbdShape;

/* Finalized cloth model.  All pointers are HOST pointers, read only during vbd_model_create.
 * Array layouts are those of newton.Model. */
typedef struct VbdModelDesc {
    int32_t particle_count;
    int32_t tri_count;
    int32_t edge_count;
    int32_t shape_count;
    int32_t color_count;
    int32_t reserved;
    const float* particle_mass;            /* [V] */
    const float* particle_inv_mass;        /* [V] */
    const float* particle_radius;          /* [V] */
    const int32_t* particle_flags;         /* [V] */
    const int32_t* particle_world;         /* [V] or NULL (all global) */
    const int32_t* tri_indices;            /* [T,3] */
    const float* tri_poses;                /* [T,2,2] row-major DmInv */
    const float* tri_materials;            /* [T,5] (ke=mu, ka=lambda, kd, drag, lift) */
    const float* tri_areas;                /* [T] */
    const int32_t* edge_indices;           /* [E,4] (o0, o1, v0, v1) */
    const float* edge_rest_angle;          /* [E] */
    const float* edge_rest_length;         /* [E] */
    const float* edge_bending_properties;  /* [E,2] (ke, kd) */
    const int32_t* v_adj_tris_offsets;     /* [V+1], counts int32 values (2 per record) */
    const int32_t* v_adj_tris;             /* (tri, slot) pairs */
    const int32_t* v_adj_edges_offsets;    /* [V+1] */
    const int32_t* v_adj_edges;            /* (edge, slot) pairs */
    const int32_t* color_group_offsets;    /* [C+1] offsets into color_group_particles */
    const int32_t* color_group_particles;  /* concatenated Model.particle_color_groups */
    float gravity[3];                      /* Model.gravity[0] (the reference applies world 0's) */
    float soft_contact_ke;                 /* Model.soft_contact_ke */
    float soft_contact_kd;                 /* Model.soft_contact_kd */
    float soft_contact_mu;                 /* Model.soft_contact_mu */
    const VbdShape* shapes;                /* [S] */
    const float* particle_q;               /* [V,3] rest/initial positions or NULL; used to cut the model
                                              into compact patches for the resident step kernel and, with
                                              self-contact, as the rest shape (grid cell size, rest
                                              exclusion radius); required for self-contact */
} VbdModelDesc;

/* Solver options (SolverVBD keyword arguments that touch the particle path, plus launch shape). */
typedef struct VbdSolverOptions {
    int32_t iterations;           /* default VBD iterations per step (reference default 10) */
    float friction_epsilon;       /* reference default 1e-2 */
    int32_t lanes_per_vertex;     /* 1,2,4,8,16 = that many lanes cooperate on one vertex; 0 = default (4);
                                     -1 = record-parallel sweep (one thread per element record) */
    int32_t block_size;           /* threads per block of the sweep, 0 = default 128 (64/128/256 when
                                     lanes_per_vertex is 0) */
    int32_t contacts_per_vertex;  /* capacity of the per-vertex contact table, 0 = default 4 */
    int32_t use_graph;            /* 1: replay vbd_step from a cached CUDA graph */
    int32_t step_kernel;          /* 0 = one launch per color (default); 1 = one persistent
                                     shared-memory-resident kernel per step when the model fits the
                                     GPU's shared memory (else one launch per color) */
    /* particle self-contact (SolverVBD particle_* keywords, solver_vbd.py:231-241) */
    int32_t self_contact;                  /* particle_enable_self_contact (0/1) */
    float self_contact_radius;             /* particle_self_contact_radius (reference default 0.2) */
    float self_contact_margin;             /* particle_self_contact_margin (0.2), must be >= radius */
    float conservative_bound_relaxation;   /* particle_conservative_bound_relaxation (0.85) */
    int32_t vertex_contact_buffer_size;    /* particle_vertex_contact_buffer_size (32) */
    int32_t edge_contact_buffer_size;      /* particle_edge_contact_buffer_size (64) */
    int32_t collision_detection_interval;  /* particle_collision_detection_interval (0) */
    float edge_parallel_epsilon;           /* particle_edge_parallel_epsilon (1e-5) */
    int32_t topological_filter_threshold;  /* particle_topological_contact_filter_threshold (2) */
    float rest_exclusion_radius;           /* particle_rest_shape_contact_exclusion_radius (0) */
    /* particle_external_vertex_contact_filtering_map / ..._edge_... as HOST CSR arrays (may be NULL):
       vertex v never collides with triangles vertex_filter_triangles[offsets[v] .. offsets[v+1]),
       edge e never with edges edge_filter_edges[offsets[e] .. offsets[e+1]); each list ascending.
       Copied at vbd_solver_create. */
    const int32_t* vertex_filter_offsets;  /* [V+1] */
    const int32_t* vertex_filter_triangles;
    const int32_t* edge_filter_offsets;    /* [E+1] */
    const int32_t* edge_filter_edges;
} VbdSolverOptions;

/* Soft-contact records in the reference layout (newton.Contacts soft_contact_*; DEVICE pointers). */
typedef struct VbdContacts {
    int32_t soft_contact_max;
    int32_t reserved;
    int32_t* soft_contact_count;        /* [1] */
    int32_t* soft_contact_particle;     /* [max] */
    int32_t* soft_contact_indices;      /* [max,3]  (p, -1, -1) */
    float* soft_contact_barycentric;    /* [max,3]  (1, 0, 0) */
    int32_t* soft_contact_shape;        /* [max] */
    float* soft_contact_body_pos;       /* [max,3] */
    float* soft_contact_body_vel;       /* [max,3] */
    float* soft_contact_normal;         /* [max,3] */
} VbdContacts;

/* Device status counters since the solver was created (or last reset). */
typedef struct VbdStatus {
    int64_t steps;
    int32_t nonfinite_updates;    /* vertex updates whose displacement was NaN/Inf (update skipped) */
    int32_t singular_blocks;      /* |det H| <= 1e-8: update skipped, as in the reference */
    int32_t contact_overflow;     /* contacts dropped because a vertex had more than the table holds */
    int32_t timeouts;             /* bounded grid-barrier waits that gave up */
    int32_t self_contact_overflow;  /* self-contact candidates dropped because a fixed-size list was
                                       full (the reference sets a resize flag in the same case) */
    int32_t reserved;
} VbdStatus;

/* Statistics of residual-gated steps (vbd_set_residual_gate), since the gate was first enabled
 * or last reset.  Residuals are in the gate's norm (max or mean of |f_i| / (m_i |g|)). */
typedef struct VbdGateStats {
    int64_t steps;                  /* gated steps finished */
    int64_t iterations;             /* iterations summed over those steps */
    int64_t capped_steps;           /* steps that stopped at max_iterations above the tolerance */
    int32_t last_iterations;        /* iterations of the last step */
    int32_t body_kernels;           /* kernel launches of one loop round (last capture; -1 unknown) */
    float last_residual;            /* final residual norm of the last step */
    float last_start_residual;      /* residual where the last step's iterations started */
    float last_reference_residual;  /* relative mode: residual at the inertia target y */
    int32_t body_programmatic_edges; /* programmatic-dependent-launch edges of one loop body (last
                                        capture; 0 after the step fell back to plain launches) */
    int64_t body_passes;            /* passes of the device-side loop body summed over the steps */
} VbdGateStats;

typedef struct VbdModel VbdModel;
typedef struct VbdSolver VbdSolver;

/* Message of the last error on this thread ("" if none). */
const char* vbd_last_error(void);

/* Library version string. */
const char* vbd_version(void);

/* Build the device-resident model on the current CUDA device (copies and re-lays-out all arrays).
 * Replaces ModelBuilder.finalize's uploads (builder.py:11033-11070, :11796-11832). */
int vbd_model_create(const VbdModelDesc* desc, VbdModel** out);
int vbd_model_destroy(VbdModel* model);

/* Particle-vs-static-shape contact generation: CollisionPipeline.collide soft branch
 * (collide.py:1553-1590) / create_soft_contacts (geometry/kernels.py:1020-1184).
 * particle_q: DEVICE [V,3] float32.  Resets and fills `contacts` (count included). */
int vbd_collide(const VbdModel* model, const float* particle_q, float soft_contact_margin,
                const VbdContacts* contacts, void* stream);

/* SolverVBD(model, iterations=..., friction_epsilon=...) particle part (solver_vbd.py:221-618). */
int vbd_solver_create(const VbdModel* model, const VbdSolverOptions* options, VbdSolver** out);
int vbd_solver_destroy(VbdSolver* solver);

/* SolverVBD.step(state_in, state_out, control, contacts, dt) (solver_vbd.py:1774-1825).
 * All arrays DEVICE [V,3] float32 in the model's particle order.
 *   q_in   : state_in.particle_q   -- read, then OVERWRITTEN with the solved positions
 *            (the reference keeps its Gauss-Seidel iterate in state_in.particle_q)
 *   qd_in  : state_in.particle_qd  -- read
 *   f_ext  : state_in.particle_f   -- read (may be NULL = zero external force)
 *   q_out  : state_out.particle_q  -- written
 *   qd_out : state_out.particle_qd -- written
 * contacts may be NULL (no particle-shape contact).  iterations < 0 uses the solver default. */
int vbd_step(VbdSolver* solver, float* q_in, const float* qd_in, const float* f_ext, float* q_out,
             float* qd_out, const VbdContacts* contacts, float dt, int32_t iterations, void* stream);

/* Batched step of `count` independent solvers (each with its own model and state) in one call:
 * element b of every array is solver b's argument to vbd_step, and the steps are enqueued in
 * order on `stream`, so the results are those of `count` vbd_step calls.  f_ext and contacts may
 * be NULL as a whole (no external force / no contacts for every solver) or hold NULL entries;
 * iterations may be NULL (every solver's default) or hold one count per solver (< 0: default).
 * The reference batches by putting several worlds in one Model (ModelBuilder.add_world), which
 * vbd_model_create supports directly and which is the faster layout for many small cloths (one
 * launch per color for all worlds); this entry point is for models that cannot be merged.
 * On an error no further solver is enqueued and the message names the failing index. */
int vbd_batch_step(VbdSolver* const* solvers, int32_t count, float* const* q_in, const float* const* qd_in,
                   const float* const* f_ext, float* const* q_out, float* const* qd_out,
                   const VbdContacts* const* contacts, float dt, const int32_t* iterations, void* stream);

/* Allocation-free variant of vbd_step (no counterpart in the reference, whose solver always
 * allocates its scratch).  For callers that cannot call cudaMalloc -- code running during CUDA
 * stream capture, host callbacks or real-time loops where an allocation could block or
 * synchronize the device, and embedders whose device memory belongs to a framework allocator --
 * and therefore cannot create a VbdSolver.  The step's scratch lives in a static device array of
 * the library sized for at most 16384 particles (about 5.3 MiB, held on every GPU that loads the
 * library until the process exits); larger models are rejected with VBD_ERR_INVALID_ARGUMENT.
 * Allocates nothing and takes no solver: same arrays, aliasing and bit-identical results as
 * vbd_step of a solver with the default options (lanes_per_vertex 4, block_size 128, 4 contacts
 * per vertex, no self-contact, no warm start).  Call it with the model's device current (another
 * current device is rejected).  The first call on a device looks up the array's device address;
 * make that first call before any stream capture.  Every call shares the one array (it clears
 * the parts that must start at zero), so calls that overlap on the GPU -- concurrent streams or
 * threads -- race; serialize them. */
int vbd_step_static(const VbdModel* model, float* q_in, const float* qd_in, const float* f_ext, float* q_out,
                    float* qd_out, const VbdContacts* contacts, float dt, int32_t iterations,
                    float friction_epsilon, void* stream);
/* Diagnostics of the last vbd_step_static on the current device (the counters vbd_status reports
 * for vbd_step: non-finite updates, singular blocks, contacts beyond 4 per vertex, timeouts;
 * `steps` and `self_contact_overflow` are 0).  Copies from the static array without allocating;
 * synchronize the stream of the step first.  The next vbd_step_static clears the counters. */
int vbd_step_static_status(VbdStatus* out);

/* Residual-gated iteration count (no counterpart in the reference, whose step runs the fixed
 * `for iter_num in range(self.iterations)` loop of solver_vbd.py:1817-1819).  With tolerance > 0,
 * vbd_step evaluates the Jacobi force residual r_i = |f_i| / (m_i |g|) of every solved vertex at
 * the iterate the iterations start from and after every `check_every` iterations (the same
 * evaluation as vbd_residual: inertia + elastic + contact force at the current positions), and
 * keeps iterating while the residual norm exceeds the tolerance and fewer than max_iterations (at
 * most 100000) have run.  The norm is max_i r_i, or with VBD_GATE_MEAN the mean of r_i over the
 * solved vertices (summed in fixed point, 1/256 m|g| resolution, so the sum is deterministic).
 * VBD_GATE_SWEEP replaces the Jacobi evaluations by the Gauss-Seidel residual the sweeps form
 * anyway: each vertex's force norm when its color is solved, accumulated by the last iteration
 * before a check (no extra launch; the first check follows the first iteration, whose residual is
 * that of the start iterate as each color meets it; at least one iteration runs unless
 * max_iterations is 0).  VBD_GATE_RELATIVE makes the tolerance relative to the norm of the
 * Jacobi residual at the inertia target y, the plain start (one evaluation per step where the
 * gate does not evaluate it anyway; with a warm start it is still taken at y, so that both starts
 * are held to the same absolute residual).  The iteration count is a multiple of
 * check_every (the cap is rounded up to one).  The
 * loop runs on the device as a conditional (while) node of the step's CUDA graph: no host round
 * trip; a gated vbd_step always runs from a graph (use_graph is implied), and inside a caller's
 * stream capture it adds the loop to the caller's graph.  tolerance <= 0 turns the gate off (the
 * vbd_step `iterations` argument applies again); while it is on, `iterations` is ignored.  Not
 * available with self-contact (VBD_ERR_UNSUPPORTED).  The iteration count of each step is
 * reported by vbd_gate_stats.  In VBD_GATE_SWEEP mode one pass of the loop body holds R check
 * rounds (R * check_every iterations, a decision after each round; the sweeps of the rounds after
 * the decision return at once), because every pass of the body costs a pipeline drain between
 * its last and first sweep; R is (mode >> VBD_GATE_ROUNDS_SHIFT) & 15, 0 = 4. */
#define VBD_GATE_RELATIVE 1
#define VBD_GATE_MEAN 2
#define VBD_GATE_SWEEP 4
#define VBD_GATE_ROUNDS_SHIFT 8
#define VBD_GATE_ROUNDS_MASK 0xF00
int vbd_set_residual_gate(VbdSolver* solver, float tolerance, int32_t max_iterations, int32_t check_every,
                          int32_t mode);
/* Gate statistics (synchronizes the device); reset != 0 zeroes the step / iteration sums. */
int vbd_gate_stats(VbdSolver* solver, VbdGateStats* out, int32_t reset);

/* Staged pieces of vbd_step, for parity tests against a staged oracle. */
int vbd_forward(VbdSolver* solver, const float* q_in, const float* qd_in, const float* f_ext,
                const VbdContacts* contacts, float dt, void* stream);
int vbd_sweep_color(VbdSolver* solver, int32_t color, const VbdContacts* contacts, float dt, void* stream);
/* Start of iteration `iteration` of a staged step: with self-contact, the detection that
 * particle_collision_detection_interval schedules there (solver_vbd.py:2540-2545); otherwise a
 * no-op. */
int vbd_begin_iteration(VbdSolver* solver, int32_t iteration, void* stream);

/* Self-contact detection alone at particle_q (DEVICE [V,3], model order): the vertex-triangle
 * and edge-edge queries of TriMeshCollisionDetector (solvers/vbd/tri_mesh_collision.py:645-730)
 * with the solver's margin and filters.  vbd_self_contact_lists copies the result to HOST
 * arrays (any may be NULL): per vertex the colliding triangle ids and per edge the colliding
 * edge ids, ascending, -1 padded to the buffer sizes (vertex_contact_buffer_size,
 * edge_contact_buffer_size); synchronizes the device. */
int vbd_self_contact_detect(VbdSolver* solver, const float* particle_q, void* stream);
int vbd_self_contact_lists(VbdSolver* solver, int32_t* vt_counts, int32_t* vt_lists, int32_t* ee_counts,
                           int32_t* ee_lists);
int vbd_finalize(VbdSolver* solver, float* q_in, float* q_out, float* qd_out, float dt, void* stream);

/* Warm start (no reference counterpart): after vbd_forward, move the initial Gauss-Seidel iterate
 * from the inertia target y to y + delta for every vertex the sweep solves.  delta: DEVICE [V,3]
 * in model particle order (e.g. the learned per-vertex correction). */
int vbd_warm_start(VbdSolver* solver, const float* delta, void* stream);

/* ---- learned warm start (no reference counterpart) -----------------------------------------
 * A per-vertex MLP 64 -> 128 -> 128 -> 3 (SiLU), trained on BF16 tensor-core tiles and run on
 * FP16 ones (FP32 accumulation in both), predicts the coming step's correction x_solved - y, in
 * units of the vertex's
 * characteristic element length L; the warm start is y + prediction * L (a zero network leaves
 * the start at y, plain VBD).  Parameters: an FP32 blob of vbd_mlp_sizes()->params floats
 * (W1 [64][128], b1, W2 [128][128], b2, W3 [128][8] with columns 3..7 zero, b3 [8]) and its BF16
 * copy of the three weight matrices (vbd_mlp_sizes()->weights16 values, refreshed by
 * vbd_mlp_adam or vbd_mlp_pack_weights).  All pointers are DEVICE pointers. */
int vbd_mlp_sizes(int32_t* params, int32_t* weights16, int32_t* in_features, int32_t* hidden, int32_t* out_features);
/* Feature sets of the network's input (vbd_set_feature_set).
 * VBD_FEATURES_CORRECTIONS (default): inertia offset (y - x) / L, the previous step's correction
 *   corr_prev of the vertex and of 8 one-ring neighbours / L, the 8 one-ring edge vectors / L,
 *   log-stiffnesses, log10 mass, contact flag, one-ring size, solvable flag.
 * VBD_FEATURES_KINEMATIC: the vertex's motion only -- previous step's displacement v dt / L,
 *   velocity v (m/s), inertia offset (y - x) / L -- with the same one-ring edge vectors,
 *   log-stiffnesses, mass and flags; corr_prev is not read. */
#define VBD_FEATURES_CORRECTIONS 0
#define VBD_FEATURES_KINEMATIC 1
/* Select the feature set of vbd_mlp_features, vbd_mlp_warm_start and the warm-start step mode
 * (a network is trained on one set and must run with it). */
int vbd_set_feature_set(VbdSolver* solver, int32_t feature_set);
/* Per-vertex features [V][64] (model particle order) of the step prepared by vbd_forward, in the
 * solver's feature set; corr_prev [V][3] (the previous step's correction, model order) may be
 * NULL.  mean / inv_std [64] standardise them (both NULL = raw).  out must be 16-byte aligned. */
int vbd_mlp_features(VbdSolver* solver, const float* corr_prev, const float* mean, const float* inv_std, float* out,
                     void* stream);
/* Y [n][3] = MLP(X [n][64]) on the 5th-generation tensor cores (tcgen05.mma: the FP32 weights of
 * params and the inputs rounded to FP16 in shared memory, FP32 accumulators in tensor memory;
 * bias + SiLU in f16x2 arithmetic with the hardware tanh approximation).  w16 is not read (it is
 * the BF16 copy the training kernels use).  X must be 16-byte aligned.  A wait that gives up is
 * counted (vbd_mlp_timeouts). */
int vbd_mlp_forward(const float* params, const uint16_t* w16, const float* X, int32_t n, float* Y, void* stream);
/* The same inference on the previous tensor-core path (mma.sync m16n8k16 fragments, exact SiLU),
 * kept to cross-check the tcgen05 kernel. */
int vbd_mlp_forward_mma_sync(const float* params, const uint16_t* w16, const float* X, int32_t n, float* Y,
                             void* stream);
/* Waits of the tcgen05 inference kernel that gave up since the last reset (0 in normal operation);
 * reset != 0 zeroes the counter.  Synchronizes with the device. */
int vbd_mlp_timeouts(uint32_t* count, int32_t reset);
/* Workspace bytes vbd_mlp_backward needs for n samples. */
int vbd_mlp_workspace_bytes(int32_t n, int64_t* bytes);
/* Gradients of L = grad_scale * sum |MLP(X) - T|^2 into grads (FP32 blob layout); loss (device
 * scalar, may be NULL) accumulates the unscaled sum of squared errors. */
int vbd_mlp_backward(const float* params, const uint16_t* w16, const float* X, const float* T, int32_t n,
                     float grad_scale, float* grads, float* loss, void* workspace, int64_t workspace_bytes,
                     void* stream);
/* One Adam step (bias-corrected, step >= 1) on the FP32 parameters; refreshes the BF16 weights. */
int vbd_mlp_adam(float* params, const float* grads, float* m1, float* m2, uint16_t* w16, int32_t step, float lr,
                 float beta1, float beta2, float eps, void* stream);
/* BF16 weights from the FP32 parameters. */
int vbd_mlp_pack_weights(const float* params, uint16_t* w16, void* stream);
/* After vbd_forward: features (corr_prev, the previous step's correction x_solved - y in model
 * order, is an input feature; may be NULL) -> MLP -> start the iterations from y + prediction * L,
 * L the vertex's mean rest edge length.  A network whose output is zero leaves the start at y
 * exactly.  workspace holds V * 70 floats. */
int vbd_mlp_warm_start(VbdSolver* solver, const float* params, const uint16_t* w16, const float* corr_prev,
                       const float* mean, const float* inv_std, float* workspace, int64_t workspace_floats,
                       void* stream);

/* Learned warm start as a mode of vbd_step: every step becomes forward -> features -> MLP ->
 * start from y + prediction -> `iterations` colour sweeps (or the residual gate's loop) ->
 * finalize, and the step's correction x_solved - y is kept (solver-owned) as the next step's
 * feature.  Features, inference and the start run as one tcgen05 kernel (no feature rows in
 * memory); the results equal vbd_mlp_features -> vbd_mlp_forward -> vbd_mlp_warm_start's bit for
 * bit.  params / w16 / mean / inv_std are caller-owned device buffers that must outlive the
 * solver's use of them; params == NULL turns the mode off.  Allocates the solver's correction
 * buffer on first use. */
int vbd_set_warm_start(VbdSolver* solver, const float* params, const uint16_t* w16, const float* mean,
                       const float* inv_std, int32_t iterations);

/* The previous step's correction x_solved - y that the warm-start step mode feeds to the next
 * step's features (model order, DEVICE [V,3]); replaces the one the last step left.  For
 * stepping the learned solver from states of another trajectory with that trajectory's history
 * (the equal-residual A/B).  The warm start must be on. */
int vbd_set_warm_start_correction(VbdSolver* solver, const float* corr, void* stream);

/* Copy the solver's current Gauss-Seidel iterate (model particle order) into q_out [V,3] (DEVICE). */
int vbd_get_positions(const VbdSolver* solver, float* q_out, void* stream);

/* Force residual at the current iterate, evaluated for every vertex at the same positions
 * (Jacobi): r_i = |m_i (y_i - x_i)/dt^2 + f_i^elastic + f_i^contact| / (m_i |g|) for active
 * vertices with m_i > 0, 0 otherwise.  per_vertex_out [V] (DEVICE, may be NULL) and
 * max_out [1] (DEVICE, may be NULL). */
int vbd_residual(VbdSolver* solver, const VbdContacts* contacts, float dt, float* per_vertex_out,
                 float* max_out, void* stream);

/* Read (synchronously) and optionally reset the device status counters. */
int vbd_status(VbdSolver* solver, VbdStatus* out, int32_t reset);

/* Number of colors and vertex count of each color as laid out on the device (host out arrays). */
int vbd_solver_info(const VbdSolver* solver, int32_t* color_count, int32_t* lanes_per_vertex,
                    int32_t* block_size);

/* Staged sweep (no reference counterpart; the north_star's "adjacency staged into shared memory
 * per color block"): on != 0 makes every color sweep load, per block, the positions its vertices'
 * element records read (the block's one-ring "patch", built on the host for the current launch
 * shape and rebuilt by vbd_set_launch) into shared memory once, and read them from there; the
 * records carry 16-bit indices into the patch.  Same math in the same order: results are
 * bit-identical to the unstaged sweep.  Not used with self-contact, for the record-parallel
 * shape, or when a block's patch would exceed 1,536 positions (the sweep then stays unstaged).
 * Allocates the patch tables when turned on.  vbd_staged_sweep_info: whether the sweeps of the
 * next step are staged, the largest patch and the patch entries in total (out pointers may be
 * NULL). */
int vbd_set_staged_sweep(VbdSolver* solver, int32_t on);
int vbd_staged_sweep_info(const VbdSolver* solver, int32_t* active, int32_t* max_patch, int64_t* patch_entries);

/* How vbd_step runs the colors: resident = 1 when one persistent shared-memory-resident kernel
 * (cooperative launch, one CTA per patch, neighbour-only synchronisation) runs all colors of all
 * iterations; 0 when each color is its own launch.  patches / smem_bytes describe the resident
 * kernel (0 otherwise). */
int vbd_solver_step_kernel(const VbdSolver* solver, int32_t* resident, int32_t* patches, int32_t* smem_bytes);

/* Kernel launches of the most recent vbd_step: the kernel nodes of the CUDA graph it replayed
 * (memset nodes excluded), or -1 when that step ran as plain launches (use_cuda_graph = 0, or
 * inside the caller's own stream capture).  Diagnostics; no reference counterpart. */
int vbd_step_kernel_count(const VbdSolver* solver, int32_t* kernels);

/* Bound (in polling iterations) of every wait of the resident kernel; a wait that runs out counts
 * in VbdStatus.timeouts and the kernel returns early instead of hanging.  Default 4,194,304. */
int vbd_set_spin_limit(VbdSolver* solver, uint32_t spins);

/* Override the sweep launch shape (used by the autotuner): lanes_per_vertex 0 with block_size
 * 64/128/256 (record-parallel), or lanes_per_vertex in {1,2,4,8,16} with a block_size multiple of 32. */
int vbd_set_launch(VbdSolver* solver, int32_t lanes_per_vertex, int32_t block_size);

/* Graph coloring of an undirected graph (host arrays): ModelBuilder.color -> color_graph
 * (graph_coloring.py:243-311).  algorithm 0 = maximum cardinality search (MCS), 1 = degree-ordered
 * greedy.  edges: [num_edges,2].  colors_out: [num_nodes].  With balance != 0, vertices are moved
 * out of the largest color until max/min color size <= target_ratio or no move is possible. */
int vbd_color_graph(int32_t num_nodes, int64_t num_edges, const int32_t* edges, int32_t algorithm,
                    int32_t balance, float target_ratio, int32_t* colors_out, int32_t* num_colors_out);

/* The conflict graph's edge list from raw vertex pairs (host arrays): the canonicalisation step of
 * construct_trimesh_graph_edges (graph_coloring.py:99-197).  pairs: [num_pairs,2], any order,
 * duplicates and self-pairs allowed.  edges_out ([num_pairs,2] capacity) receives the unique
 * (min, max) pairs in lexicographic order; num_edges_out their count. */
int vbd_coloring_graph_edges(int32_t num_nodes, int64_t num_pairs, const int32_t* pairs, int32_t* edges_out,
                             int64_t* num_edges_out);

/* The conflict graph of construct_trimesh_graph_edges (graph_coloring.py:99-197) straight from the
 * element arrays (host, already filtered by the active masks): each triangle [nt,3] adds its 3
 * vertex pairs, each bending hinge [nb,4] (may be NULL when nb = 0) all 6 pairs of its vertices,
 * pairs with a negative id skipped; edges_out ([3 nt + 6 nb, 2] capacity) receives the unique
 * (min, max) pairs in lexicographic order, num_edges_out their count. */
int vbd_trimesh_graph_edges(int32_t num_nodes, const int32_t* tris, int64_t nt, const int32_t* bend, int64_t nb,
                            int32_t* edges_out, int64_t* num_edges_out);

/* Bending-edge table of a triangle mesh (host arrays): MeshAdjacency._compute_edge_adjacency
 * (utils/mesh.py:465-531).  tris [nt,3].  Undirected edges are numbered in first-occurrence order
 * of the traversal (triangle t, local edge k = (tris[t][k], tris[t][k+1]), opposite tris[t][k+2]);
 * edge_indices rows are [o0, o1, v0, v1] (o1 = -1 on a boundary), edge_tri the two triangles,
 * tri_edge [nt,3] each triangle's edges.  Outputs sized for 3 nt edges; num_edges receives the
 * count, nonmanifold (may be NULL) the number of triangle sides beyond the second on an edge. */
int vbd_mesh_edge_adjacency(const int32_t* tris, int32_t nt, int32_t* edge_indices, int32_t* edge_tri,
                            int32_t* tri_edge, int32_t* num_edges, int32_t* nonmanifold);

/* Per-vertex CSR of (element id, local slot) records (host arrays): init_vertex_adjacency and its
 * count / fill kernels (utils/mesh.py:595-655, :675-772).  entries [n_elements, per_element] are
 * vertex ids (-1 skipped) and slot_of[per_element] the slot each position records; records are in
 * element order.  values receives 2 ints per record; offsets [particle_count + 1] counts ints. */
int vbd_mesh_vertex_csr(const int32_t* entries, int32_t n_elements, int32_t per_element, const int32_t* slot_of,
                        int32_t particle_count, int32_t* values, int32_t* offsets);

/* The three set-up tables above on the GPU: the same rules and the same tables, element for
 * element, from DEVICE arrays (inputs and outputs, same layouts and capacities as the host
 * versions) on `stream`; counts are returned to host variables (the call synchronizes the
 * stream).  Temporary memory is allocated (cudaMalloc) and freed within the call.
 * vbd_mesh_vertex_csr_device: slot_of is a HOST array; n_elements * per_element <= 2^30; values
 * needs 2 ints per record; num_records (may be NULL) receives the record count. */
int vbd_mesh_edge_adjacency_device(const int32_t* tris, int32_t nt, int32_t* edge_indices, int32_t* edge_tri,
                                   int32_t* tri_edge, int32_t* num_edges, int32_t* nonmanifold, void* stream);
int vbd_mesh_vertex_csr_device(const int32_t* entries, int32_t n_elements, int32_t per_element,
                               const int32_t* slot_of, int32_t particle_count, int32_t* values, int32_t* offsets,
                               int32_t* num_records, void* stream);
int vbd_trimesh_graph_edges_device(int32_t num_nodes, const int32_t* tris, int64_t nt, const int32_t* bend,
                                   int64_t nb, int32_t* edges_out, int64_t* num_edges_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VBD_B200_H */
