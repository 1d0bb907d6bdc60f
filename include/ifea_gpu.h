/*
 * ifea_gpu.h — C ABI of the B200 (sm_100a) forging hot path.
 *
 * The per-Newton-iteration path of ImpressionFEA.Core's rigid-viscoplastic forging solvers runs on the GPU:
 * element stiffness and residual (linear tets with averaged-nodal-pressure penalty; 4-node axisymmetric /
 * plane-strain quads with reduced-integration penalty), rigid-die contact frames and m*k friction, deterministic
 * gather-assembly into the reference's fixed sparse pattern, and the Newton / line-search / PCG update around a
 * sparse Cholesky factorisation. The host keeps the increment loop, exactly as Forging3DSolver / ForgingSolver.
 *
 * Conventions: plain C types only; host arrays are borrowed for the duration of the call (copied to the device);
 * device state is owned by the context and released by *_destroy. Every call returns an ifea_status; on failure
 * *_last_error() returns the message the reference would have put in its exception.
 * Contexts are independent: one per solver instance, each with its own CUDA stream and library handles.
 */
#ifndef IFEA_GPU_H
#define IFEA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; the mapping to the reference's exception types (Solver/SolverExceptions.cs:4-43). */
typedef enum ifea_status {
    IFEA_OK = 0,
    IFEA_INPUT_INVALID = 1,     /* InputValidationException                         */
    IFEA_DIVERGED = 2,          /* SolverDivergenceException                        */
    IFEA_MESH_DISTORTED = 3,    /* MeshDistortionException                          */
    IFEA_NOT_SPD = 4,           /* MatrixNotPositiveDefiniteException               */
    IFEA_BAD_STATE = 5,         /* InvalidOperationException (e.g. stepping after closure) */
    IFEA_CUDA_ERROR = 6,        /* EngineUnavailableException (device or library failure) */
    IFEA_CANCELLED = 7          /* OperationCanceledException                       */
} ifea_status;

/* NodeContact (Simulation/SimulationResult.cs:17-22). */
enum { IFEA_FREE = 0, IFEA_BOTTOM_DIE = 1, IFEA_TOP_DIE = 2 };

/* ------------------------------------------------------------------ 3D (Forging3DSolver) */

/* SimulationConfig3D fields and the Forging3DSolver statics the path reads
 * (ThreeD/SimulationConfig3D.cs:19-76; ThreeD/Forging3DSolver.cs:27-50, :1048). */
typedef struct ifea3d_params {
    double C, N, M, eps0;         /* FlowStressLaw (Materials/FlowStressLaw.cs:6)          */
    double friction;              /* FrictionFactor m                                      */
    double ram;                   /* RamSpeed, mm/s                                        */
    double h;                     /* ElementSize, mm                                       */
    double ds;                    /* StrokeIncrement, mm                                   */
    double tol;                   /* Tolerance on |dv|/|v|                                 */
    int32_t max_iter;             /* MaxIterations                                         */
    int32_t auto_step;            /* AutoStep                                              */
    int32_t max_cutbacks;         /* MaxCutbacks                                           */
    double remesh_quality;        /* RemeshQuality                                         */
    double size;                  /* rateRef = ram / size (Forging3DSolver.cs:145-146)     */
    int32_t sym_x, sym_y, sym_factor;
    double penalty_factor;        /* PenaltyFactor (1e4)                                   */
    double newton_blend;          /* NewtonBlend (0.6)                                     */
    int32_t quadratic_ls;         /* QuadraticLineSearch                                   */
    int32_t extrapolate_start;    /* ExtrapolateStart                                      */
    int32_t adaptive_newton;      /* AdaptiveNewton                                        */
    int32_t sticky_secant;        /* StickySecant                                          */
    int32_t pcg_budget;           /* PcgBudget (15)                                        */
} ifea3d_params;

/* Per-increment telemetry (ForgingSnapshot fields the solver fills, Simulation/SimulationResult.cs:25-84). */
typedef struct ifea_step_info {
    int32_t step;                 /* StepIndex                                             */
    int32_t iterations;           /* Newton iterations of the accepted pass                */
    double load;                  /* LoadNewton = power / ram * symmetry factor            */
    double reaction;              /* top-die reaction, symmetry-scaled                     */
    double stroke;                /* gap0 - gap                                            */
    double gap;                   /* remaining die gap                                     */
    double time;                  /* process time                                          */
    double dt;                    /* time increment used                                   */
    double volume_change_pct;     /* VolumeChangePercent                                   */
    double last_rel;              /* |dv|/|v| of the last iteration                        */
    int32_t n_factor;             /* factorisations so far                                 */
    int32_t n_pcg;                /* PCG solves so far                                     */
    int32_t remesh_requests;      /* increments where the reference would have remeshed    */
    int32_t cutbacks;             /* cutbacks used in this increment                       */
} ifea_step_info;

typedef struct ifea3d ifea3d;

/* new Forging3DSolver(config) minus the internal mesher (Forging3DSolver.cs:125-187). */
ifea_status ifea3d_create(const ifea3d_params *params, ifea3d **out);
void ifea3d_destroy(ifea3d *ctx);
const char *ifea3d_last_error(const ifea3d *ctx);

/* Mesh handed over by the host mesher (IsosurfaceStuffing result, Forging3DSolver.cs:153-155 / BuildMesh :205-206):
 * x = nn*3 coordinates, tets = ne*4 positively oriented node ids, symmetry-plane flags per node.
 * Builds TetMesh topology, the two-ring pattern (BuildPattern :469-521) and the slot maps (:1248-1261). */
ifea_status ifea3d_set_mesh(ifea3d *ctx, int32_t nn, int32_t ne, const double *x, const int32_t *tets,
                            const uint8_t *on_x0, const uint8_t *on_y0);

/* Height-field die (ThreeD/HeightFieldDie.cs:15-26): side 0 = bottom, 1 = top (closed position);
 * samples h[(ny+1)*(nx+1)], row-major in y. */
ifea_status ifea3d_set_die(ifea3d *ctx, int32_t side, int32_t nx, int32_t ny, double x0, double y0, double dx,
                           const double *h);

/* Constructor tail (Forging3DSolver.cs:156-184): initial gap, initial contact and placement, initial velocity
 * from the billet bounds (min_x, min_y, min_z, max_x, max_y), reference volume. */
/* A die given as a closed triangulated solid instead of a height field (TriMeshDie over TriMeshSolid,
 * ThreeD/TriMeshSolid.cs:248-297): nv vertices (3 doubles each), nt triangles (3 vertex indices each, outward normals
 * by winding), the top die in its closed position. Its clearance, projection and surface height follow the
 * reference's bucket grids and ring search. */
ifea_status ifea3d_set_trimesh_die(ifea3d *ctx, int32_t side, int32_t nv, const double *v, int32_t nt, const int32_t *tri);
/* Clearance (IRigidDie.Clearance), Project (closest point, normal out of the die) and SurfaceZ of one die, moved by
 * `offset` along z, at n points (3 doubles each), evaluated on the device: clearance[n], projected[3n], normal[3n],
 * surface_z[n] (NaN where a triangulated die has no surface above or below the point). */
ifea_status ifea3d_die_query(ifea3d *ctx, int32_t side, int32_t n, const double *p, double offset, double *clearance,
                             double *projected, double *normal, double *surface_z);
ifea_status ifea3d_init(ifea3d *ctx, double gap0, double min_x, double min_y, double min_z, double max_x,
                        double max_y);

/* One increment: Forging3DSolver.Step (:540-638). Remeshing is host-side and out of this library's scope;
 * where the reference would remesh, the increment continues as if the remesh had been rejected and the
 * request is counted in info->remesh_requests. cancel (may be NULL) is polled between Newton iterations. */
ifea_status ifea3d_step(ifea3d *ctx, ifea_step_info *info, const volatile int32_t *cancel);

/* Pattern of the assembled system: full symmetric CSC in 3x3 node blocks (BuildPattern :496-515). */
ifea_status ifea3d_pattern_size(ifea3d *ctx, int64_t *nnz, int32_t *ndof);
ifea_status ifea3d_get_pattern(ifea3d *ctx, int32_t *col_ptr, int32_t *row_idx);

/* Lower-level steps of one increment, for teacher-forced parity (each mirrors a private method). */
ifea_status ifea3d_prepare_step(ifea3d *ctx);                                       /* PrepareStep :660-758   */
ifea_status ifea3d_assemble(ifea3d *ctx, int32_t matrix, int32_t newton, const double *v_host,
                            double *energy, double *power);                         /* Assemble :1115-1217    */
ifea_status ifea3d_apply_bc(ifea3d *ctx, double *max_diag);                         /* SolveVelocity :892-913 */
ifea_status ifea3d_solve_velocity(ifea3d *ctx, int32_t *iterations, int32_t *converged,
                                  const volatile int32_t *cancel);                  /* SolveVelocity :875-948 */
ifea_status ifea3d_final_evaluation(ifea3d *ctx, double *power, double *reaction); /* FinalEvaluation        */
ifea_status ifea3d_try_update(ifea3d *ctx, double dt, int32_t *ok);                 /* TryUpdate :1455-1537   */
ifea_status ifea3d_set_warm(ifea3d *ctx, int32_t warm);
/* Issue all further work of this context on the caller's CUDA stream (a cudaStream_t; the caller keeps it alive
 * for the context's lifetime). Lets a host time the context with events on its own stream. */
ifea_status ifea3d_set_stream(ifea3d *ctx, void *cuda_stream);

/* Copy a named state array to host memory (count elements of the named array's type):
 * "x","vg","v","r","dv" (double), "eps","dmg","el_sig","el_rate","el_mean","el_dev","grad","vol","ax",
 * "fixed_val","k_fric","a_fric","v_node","kvol","val","h_local" (double), "contact","release","fixed"
 * (uint8), "n_fix","die_axis","e_nbr","nbr_start","nbr" (int32). Returns IFEA_INPUT_INVALID on unknown names. */
ifea_status ifea3d_get_array(ifea3d *ctx, const char *name, void *dst, int64_t count);
ifea_status ifea3d_array_size(ifea3d *ctx, const char *name, int64_t *count, int32_t *elem_bytes);
/* Replace a named state array ("x","vg","eps","el_sig","contact","v","dmg") with host data. */
ifea_status ifea3d_set_array(ifea3d *ctx, const char *name, const void *src, int64_t count);
ifea_status ifea3d_get_scalar(ifea3d *ctx, const char *name, double *value);
ifea_status ifea3d_set_scalar(ifea3d *ctx, const char *name, double value);

/* ------------------------------------------------------------------ ISpdSolver (Solver/Linear/ISpdSolver.cs:24-41)
 * Sparse SPD direct solver over a full symmetric CSC pattern, for the reference's pluggable factorisation seam
 * (replaces CudssSolver.cs:105-145 behind ISpdSolver). Host buffers, like the reference's backends. */
typedef struct ifea_spd ifea_spd;
ifea_status ifea_spd_create(ifea_spd **out);
void ifea_spd_destroy(ifea_spd *s);
const char *ifea_spd_last_error(const ifea_spd *s);
ifea_status ifea_spd_analyze(ifea_spd *s, int32_t n, const int32_t *col_ptr, const int32_t *row_idx);
ifea_status ifea_spd_factorize(ifea_spd *s, const double *values);
ifea_status ifea_spd_solve(ifea_spd *s, const double *b, double *x);
int64_t ifea_spd_factor_nonzeros(const ifea_spd *s);
const char *ifea_spd_name(const ifea_spd *s);

/* Snapshot telemetry: FillPercent (ThreeD/Forging3DSolver.cs:2174-2185) on the device. The cavity samples
 * (BuildCavitySamples, :2157-2172: columns over the impression between the closed dies; 3 per point) are given once;
 * each call counts the ones inside the current mesh. The volume change is ifea3d_get_scalar(ctx, "volume"). */
ifea_status ifea3d_set_cavity(ifea3d *ctx, int32_t n, const double *xyz);
ifea_status ifea3d_fill_percent(ifea3d *ctx, double *pct);

/* ------------------------------------------------------------------ many cases at once
 *
 * Independent cases (the reference: Parallel.For over the levels of a mesh study, ThreeD/MeshConvergence.cs:117)
 * stepped together: each context keeps its own streams and graphs, a pool of host threads (threads <= 0: one per
 * case, at most the host's hardware threads) steps them, so their kernels share the GPU. The contexts must not be
 * used elsewhere while ifea_batch_step runs. infos: (n3 + n2) x increments, case-major (3D cases first);
 * status: one per case (the first failure of that case; its later increments are skipped). */
typedef struct ifea_batch ifea_batch;
typedef struct ifea2d ifea2d;
ifea_status ifea_batch_create(int32_t n3, ifea3d *const *ctx3, int32_t n2, ifea2d *const *ctx2, int32_t threads,
                              ifea_batch **out);
ifea_status ifea_batch_step(ifea_batch *b, int32_t increments, ifea_step_info *infos, int32_t *status);
void ifea_batch_destroy(ifea_batch *b);
/* Launch-parameter tuner: times one factorisation + solve of the next increment's first matrix for every pair of
 * (tensor-core trailing update from 512 / 1024 / 2048 rows / never) x (multi-CTA solves from 96 / 192 / 384 rows)
 * and keeps the fastest; with use_cache, a pair found before for the same size class (log2 of the equation count)
 * is applied without measuring. Call after choosing the precision (factor_fp32). */
ifea_status ifea3d_autotune(ifea3d *ctx, int32_t use_cache, double *tc_rows, double *wide_rows, double *best_ms);
/* one factorisation of the current matrix and one solve, device milliseconds (what the tuner compares) */
ifea_status ifea3d_time_factor_solve(ifea3d *ctx, double *ms);

/* ------------------------------------------------------------------ remeshing (3D, host side)
 *
 * With ifea3d_set_scalar(ctx, "remesh", 1) the stepper remeshes where the reference does (RemeshTrigger at the
 * start of an increment, a stalled velocity solution, a fold during the update: ThreeD/Forging3DSolver.cs:544-611)
 * by RemeshCore (:1958-2101) on the host and continues on the new mesh with the remapped state; off by default
 * (the requests are only counted). "refinement_levels" (0-3, default 1) and "max_nodes" bound the local
 * refinement around failures. The two building blocks are exported as the reference's public statics: */
typedef int32_t (*ifea_inside_fn)(double x, double y, double z, void *user);
typedef double (*ifea_size_fn)(double x, double y, double z, void *user);
typedef struct ifea_tetmesh ifea_tetmesh;
/* IsosurfaceStuffing.Stuff (ThreeD/IsosurfaceStuffing.cs:19-84): body-centred-cubic lattice of spacing h over
 * [lo, hi], cut, warped and clipped to the body; sym_x / sym_y keep x >= 0 / y >= 0 with flat symmetry planes */
ifea_status ifea_tetmesh_stuff(ifea_inside_fn inside, void *user, const double *lo3, const double *hi3, double h,
                               int32_t sym_x, int32_t sym_y, ifea_tetmesh **out);
/* TetRefiner.Refine (ThreeD/TetRefiner.cs:14-158): longest-edge bisection to the target size, within max_nodes */
ifea_status ifea_tetmesh_refine(ifea_tetmesh *m, ifea_size_fn size, void *user, int32_t max_nodes, int32_t *splits);
int32_t ifea_tetmesh_node_count(const ifea_tetmesh *m);
int32_t ifea_tetmesh_tet_count(const ifea_tetmesh *m);
ifea_status ifea_tetmesh_get(const ifea_tetmesh *m, double *x, int32_t *tets);
void ifea_tetmesh_destroy(ifea_tetmesh *m);
/* why the last remesh of the context was rejected, or what the last accepted one made */
const char *ifea3d_last_remesh(const ifea3d *ctx);
/* RemeshCore itself on host arrays, for a host that steps the increments elsewhere (the C# solver's Remesh, or a
 * CPU solver): the deformed mesh and its state in, the new mesh and the remapped state out. Returns IFEA_OK when
 * the new mesh is accepted, IFEA_MESH_DISTORTED when rejected (ifea_remesh_why says why). */
typedef struct ifea_die_grid {
    int32_t nx, ny;
    double x0, y0, dx;
    const double *h;              /* (nx + 1) * (ny + 1) heights, row-major in y; the top die at its closed place */
} ifea_die_grid;
typedef struct ifea_remesh_args {
    int32_t nn, ne;
    const double *x;              /* 3 per node */
    const int32_t *tets;          /* 4 per tet */
    const double *vg;             /* global velocity, 3 per node */
    const double *eps, *dmg, *sig, *rate, *mean;   /* per tet */
    ifea_die_grid bottom, top;
    double gap, h, vol_target;    /* die gap, element size, initial volume of the modelled part */
    int32_t sym_x, sym_y, recovery_pass, refinement_levels, max_nodes;
    double sig_ref;               /* flow stress where no old element is found */
    int32_t n_hot;
    const double *hot;            /* 4 per failure place: x, y, z, refinement level */
} ifea_remesh_args;
typedef struct ifea_remesh_result ifea_remesh_result;
ifea_status ifea_remesh_workpiece(const ifea_remesh_args *args, ifea_remesh_result **out);
int32_t ifea_remesh_node_count(const ifea_remesh_result *r);
int32_t ifea_remesh_tet_count(const ifea_remesh_result *r);
const char *ifea_remesh_why(const ifea_remesh_result *r);
/* any output pointer may be NULL */
ifea_status ifea_remesh_get(const ifea_remesh_result *r, double *x, int32_t *tets, uint8_t *on_x0, uint8_t *on_y0,
                            uint8_t *contact, double *vg, double *eps, double *dmg, double *sig, double *rate,
                            double *mean);
void ifea_remesh_destroy(ifea_remesh_result *r);

/* ------------------------------------------------------------------ learned warm start (3D)
 *
 * Replaces the initial velocity guess of each increment, LoadVelocityGuess (ThreeD/Forging3DSolver.cs:854-869:
 * the previous increment's velocity in the nodal frames; ExtrapolateStart, :43-44 and :861-866, adds its trend).
 * A per-node MLP, 16 inputs -> 3 hidden layers of 128 (GELU) -> 3 outputs, predicts the change of each node's
 * global velocity over the coming increment from the node's state (previous velocity and its trend, mean
 * effective strain and strain rate, contact state, die clearances, stroke increment, position). BF16 weights and
 * activations, FP32 accumulation on the tensor cores; FP32 master weights trained by Adam on samples the solver
 * records from its own converged increments. The reference has no counterpart beyond the guess it replaces. */
typedef struct ifea_mlp ifea_mlp;
ifea_status ifea_mlp_create(uint64_t seed, ifea_mlp **out);   /* seeded He-uniform weights, zero biases */
void ifea_mlp_destroy(ifea_mlp *m);
const char *ifea_mlp_last_error(const ifea_mlp *m);
int64_t ifea_mlp_param_count(void);                              /* FP32 parameters: W1 b1 W2 b2 W3 b3 W4 b4 */
ifea_status ifea_mlp_get_params(ifea_mlp *m, float *params, int64_t count);
ifea_status ifea_mlp_set_params(ifea_mlp *m, const float *params, int64_t count);   /* resets Adam's moments */
/* input mean[16], input std[16], output mean[3], output std[3] */
ifea_status ifea_mlp_get_normalisation(ifea_mlp *m, float *norm38);
ifea_status ifea_mlp_set_normalisation(ifea_mlp *m, const float *norm38);
/* training set: raw inputs [n][16] and raw targets [n][3] (host arrays) */
ifea_status ifea_mlp_add_samples(ifea_mlp *m, const float *inputs, const float *targets, int64_t n);
int64_t ifea_mlp_samples(const ifea_mlp *m);
ifea_status ifea_mlp_clear_samples(ifea_mlp *m);
ifea_status ifea_mlp_fit_normalisation(ifea_mlp *m);             /* mean / std of the training set */
/* raw outputs [n][3] for raw inputs [n][16] (host arrays) */
ifea_status ifea_mlp_forward(ifea_mlp *m, const float *inputs, int64_t n, float *outputs);
/* gradient of the mean squared error over the normalised targets at the current parameters, n rows (a multiple
 * of 128, at most 8192); grad gets ifea_mlp_param_count() values */
ifea_status ifea_mlp_gradients(ifea_mlp *m, const float *inputs, const float *targets, int64_t n, float *grad,
                               float *loss);
/* Adam (beta 0.9 / 0.999) over seeded random batches of the training set; *final_loss = mean loss of the last
 * tenth of the steps, *gpu_ms = device time of the training */
ifea_status ifea_mlp_train(ifea_mlp *m, int32_t steps, int32_t batch, float lr, uint64_t seed, float *final_loss,
                           double *gpu_ms);
/* mode 0 off; bit 1: record (inputs, target) of every accepted increment into m's training set; bit 2: start
 * each increment from the network's prediction when the functional is lower there than at the reference's start
 * (which is kept otherwise). m must outlive the context's use of it. */
ifea_status ifea3d_set_warm_start(ifea3d *ctx, ifea_mlp *m, int32_t mode);

/* ------------------------------------------------------------------ 2D (ForgingSolver) */

/* SimulationConfig + DieSet fields the 2D path reads (Simulation/SimulationConfig.cs:14-45, Geometry/DieSet.cs). */
typedef struct ifea2d_params {
    double C, N, M, eps0;
    double friction;
    double ram;
    double ds;                    /* StrokeIncrement                                       */
    double tol;
    int32_t max_iter;
    int32_t axisymmetric;         /* Symmetry.Axisymmetric (1) / PlaneStrain (0)           */
    double length;                /* BilletLength (plane strain)                           */
    double radius, height;        /* billet                                                */
    int32_t nx, nz;               /* ElementsX, ElementsZ                                  */
} ifea2d_params;

typedef struct ifea2d ifea2d;
/* new ForgingSolver(config) (Solver/ForgingSolver.cs:104-145): structured mesh, RCM numbering, dies as
 * piecewise-linear profiles (x strictly increasing, closed position). */
ifea_status ifea2d_create(const ifea2d_params *params, int32_t n_bottom, const double *bottom_xy, int32_t n_top,
                          const double *top_xy, ifea2d **out);
void ifea2d_destroy(ifea2d *ctx);
const char *ifea2d_last_error(const ifea2d *ctx);
ifea_status ifea2d_step(ifea2d *ctx, ifea_step_info *info, const volatile int32_t *cancel); /* Advance :215-290 */
ifea_status ifea2d_prepare(ifea2d *ctx);                      /* PrepareConstraints + LoadVelocityGuess */
ifea_status ifea2d_assemble(ifea2d *ctx, int32_t matrix, int32_t newton, const double *v_host, double *energy,
                            double *power);                   /* Assemble :471-538 */
ifea_status ifea2d_solve_velocity(ifea2d *ctx, int32_t picard_fallback, int32_t *iterations, int32_t *converged);
ifea_status ifea2d_get_array(ifea2d *ctx, const char *name, void *dst, int64_t count);
ifea_status ifea2d_array_size(ifea2d *ctx, const char *name, int64_t *count, int32_t *elem_bytes);
ifea_status ifea2d_get_scalar(ifea2d *ctx, const char *name, double *value);

/* SymmetricBandMatrix (Solver/SymmetricBandMatrix.cs:7-111) factorised on the GPU: lower band stored row-wise,
 * a[i*(b+1) + (j-i+b)]. Host buffers. On a non-positive pivot returns IFEA_NOT_SPD with *bad_row = the row. */
ifea_status ifea_band_factor_solve(int32_t n, int32_t half_bandwidth, double *band, double *rhs, int32_t *bad_row,
                                   double *pivot);

/* No counterpart in the reference. SymmetricBandMatrix.Factorize + Solve on buffers the caller already owns on the
 * device, for callers that cannot allocate device memory at that point (their GPU memory belongs to their own
 * pooling allocator, or the solve sits in a loop that must not call cudaMalloc/cudaFree). d_band (n*(b+1) doubles,
 * the same row-wise lower band as ifea_band_factor_solve) is overwritten by L, d_rhs (n doubles, may be NULL) by x;
 * work is issued on cuda_stream (a cudaStream_t, NULL = default stream) and the call returns after it finished.
 * The factorisation's working rows live in the kernel's shared memory, or, for a band too wide for that window,
 * in d_band itself; the only other working memory is a fixed 16-byte device array inside the library holding the
 * two status words, present on every GPU that loads it until the process exits. Every call looks up that array's
 * device address in the current device's context, launches one kernel, copies the status words back and waits
 * for cuda_stream to finish (so it cannot be called while cuda_stream is being captured into a CUDA graph). All
 * calls on a device share the status words; each call re-initialises them, but
 * calls that overlap on the same GPU race on them and must be serialised by the caller.
 * Returns IFEA_NOT_SPD with *bad_row / *pivot on a non-positive pivot. Allocates nothing. */
ifea_status ifea_band_factor_solve_noalloc(int32_t n, int32_t half_bandwidth, double *d_band, double *d_rhs,
                                           int32_t *bad_row, double *pivot, void *cuda_stream);

/* Library build / device description for the log. */
const char *ifea_version(void);

#ifdef __cplusplus
}
#endif
#endif
