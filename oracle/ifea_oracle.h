/*
 * ifea_oracle.h — CPU FP64 restatement of ImpressionFEA.Core's per-Newton-iteration forging path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker the CUDA path is compared against. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity pin: the reference (C# .NET 10) cannot be built or run here, and it ships no golden field vectors.
 * The restatement is pinned by the reference's own analytic known-answer tests (frictionless upset loads,
 * band Cholesky vs dense, non-SPD detection, die projection values), re-run against this code in tests/.
 * Field-level (velocity, strain) parity against the reference's binaries is therefore unpinned.
 *
 * Every function cites the reference file:line it restates (paths relative to the reference project).
 * Compiled with -ffp-contract=off: the .NET JIT does not contract a*b+c into FMAs.
 */
#ifndef IFEA_ORACLE_H
#define IFEA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ 3D solver (Forging3DSolver) */
typedef struct o3d_params {
    double C, N, M, eps0;         /* FlowStressLaw(C, N, M, Eps0)                          */
    double friction;              /* SimulationConfig3D.FrictionFactor                     */
    double ram;                   /* RamSpeed, mm/s                                        */
    double h;                     /* ElementSize, mm                                       */
    double ds;                    /* StrokeIncrement, mm                                   */
    double tol;                   /* Tolerance                                             */
    int max_iter;                 /* MaxIterations                                         */
    int auto_step;                /* AutoStep                                              */
    int max_cutbacks;             /* MaxCutbacks                                           */
    double remesh_quality;        /* RemeshQuality                                         */
    double size;                  /* billet size that sets rateRef = ram / size            */
    int sym_x, sym_y, sym_factor; /* DieSet3D symmetry                                     */
    double penalty_factor;        /* Forging3DSolver.PenaltyFactor (1e4)                   */
    double newton_blend;          /* NewtonBlend (0.6)                                     */
    int quadratic_ls;             /* QuadraticLineSearch (true)                            */
    int extrapolate_start;        /* ExtrapolateStart (false)                              */
    int adaptive_newton;          /* AdaptiveNewton (true)                                 */
    int sticky_secant;            /* StickySecant (false)                                  */
    int pcg_budget;               /* PcgBudget (15)                                        */
} o3d_params;

typedef struct o3d o3d;

o3d *o3d_create(const o3d_params *p);
void o3d_destroy(o3d *s);
const char *o3d_error(const o3d *s);
/* Mesh: nn nodes (xyz interleaved), ne positively oriented tets, symmetry-plane flags. */
int o3d_set_mesh(o3d *s, int nn, int ne, const double *x, const int32_t *tets, const uint8_t *on_x0,
                 const uint8_t *on_y0);
/* Height-field die (side 0 = bottom, 1 = top in the closed position). */
int o3d_set_die(o3d *s, int side, int nx, int ny, double x0, double y0, double dx, const double *h);
/* Constructor tail (Forging3DSolver.cs:156-184): initial contact, placement, initial velocity, volume. */
int o3d_init(o3d *s, double gap0, double min_x, double min_y, double min_z, double max_x, double max_y);
/* One increment (Forging3DSolver.Step). */
int o3d_step(o3d *s);
/* remeshing through the host's remesher: fn(user, s) reads the state (o3d_array / o3d_scalar), installs the new
 * mesh with o3d_replace_mesh and returns 1, or returns 0 when it rejects the new mesh */
typedef int (*o3d_remesh_fn)(void *user, o3d *s);
void o3d_set_remesher(o3d *s, o3d_remesh_fn fn, void *user);
int o3d_replace_mesh(o3d *s, int nn, int ne, const double *x, const int32_t *tets, const uint8_t *on_x0,
                     const uint8_t *on_y0, const uint8_t *contact, const double *vg, const double *eps,
                     const double *dmg, const double *sig, const double *rate, const double *mean);

/* Lower-level entry points for teacher-forced parity. */
int o3d_prepare_step(o3d *s);
double o3d_assemble(o3d *s, int matrix, int newton, const double *v, double *power);
int o3d_apply_bc(o3d *s, double *max_diag);
int o3d_solve_velocity(o3d *s, int *converged);
double o3d_final_evaluation(o3d *s, double *reaction);
int o3d_try_update(o3d *s, double dt, int *ok);
void o3d_set_warm(o3d *s, int warm);

/* Array access: returns a pointer to internal storage and its element count. */
void *o3d_array(o3d *s, const char *name, int64_t *count);
double o3d_scalar(o3d *s, const char *name);
int o3d_set_scalar(o3d *s, const char *name, double v);

/* ------------------------------------------------------------------ sparse SPD factorisation (ISpdSolver) */
typedef struct ospd ospd;
ospd *ospd_create(void);
void ospd_destroy(ospd *f);
/* optional: node coordinates (3 equations per node) for a coordinate nested-dissection order */
void ospd_set_geometry(ospd *f, int nnodes, const double *xyz);
int ospd_analyze(ospd *f, int n, const int32_t *col_ptr, const int32_t *row_idx);
int ospd_factorize(ospd *f, const double *values);
int ospd_solve(ospd *f, const double *b, double *x);
int64_t ospd_factor_nonzeros(const ospd *f);
int ospd_bad_pivot(const ospd *f);
double ospd_factor_flops(const ospd *f);  /* multiply-adds of one factorisation */
int ospd_supernodes(const ospd *f);

/* ------------------------------------------------------------------ band Cholesky (SymmetricBandMatrix) */
typedef struct oband oband;
oband *oband_create(int n, int half_bandwidth);
void oband_destroy(oband *b);
int oband_bandwidth(const oband *b);
int oband_add(oband *b, int i, int j, double v);
double oband_get(const oband *b, int i, int j);
void oband_constrain(oband *b, int i);
void oband_clear(oband *b);
int oband_factorize(oband *b, double *pivot); /* returns -1 ok, else failing row */
int oband_solve(oband *b, double *rhs);
double *oband_data(oband *b, int64_t *count);

/* ------------------------------------------------------------------ 2D solver (ForgingSolver) */
typedef struct o2d_params {
    double C, N, M, eps0;
    double friction;
    double ram;
    double ds;             /* StrokeIncrement */
    double tol;
    int max_iter;
    int axisymmetric;      /* Symmetry.Axisymmetric (1) or PlaneStrain (0) */
    double length;         /* BilletLength (plane strain) */
    double radius, height; /* billet */
    int nx, nz;            /* ElementsX, ElementsZ */
} o2d_params;

typedef struct o2d o2d;
o2d *o2d_create(const o2d_params *p, int n_bottom, const double *bottom_xy, int n_top, const double *top_xy);
void o2d_destroy(o2d *s);
const char *o2d_error(const o2d *s);
int o2d_step(o2d *s);
int o2d_prepare(o2d *s);                   /* PrepareConstraints + LoadVelocityGuess */
double o2d_assemble(o2d *s, int matrix, int newton, const double *v, double *power);
int o2d_solve_velocity(o2d *s, int picard_fallback, int *converged);
double o2d_final_evaluation(o2d *s, double *reaction);
void *o2d_array(o2d *s, const char *name, int64_t *count);
double o2d_scalar(o2d *s, const char *name);

/* 2D die surface queries (DieSurface) and 3D height-field / triangle helpers for the geometry KATs. */
double o2d_die_project(const double *pts, int npts, int side, double px, double py, double offset,
                       double *qx, double *qy, double *nx, double *ny);
double o2d_die_height(const double *pts, int npts, double x);
int o3d_set_trimesh_die(o3d *s, int side, int nv, const double *v, int nt, const int *tri);
double o3d_die_height(o3d *s, int side, double x, double y);
double o3d_die_project(o3d *s, int side, const double *p, double offset, double *q, double *nrm);
double o3d_die_clearance(o3d *s, int side, const double *p, double offset);
double o3d_tet_quality(const double *a, const double *b, const double *c, const double *d);
double o_flow_stress(double C, double N, double M, double eps0, double strain, double rate);
double o_principal_max3(double xx, double yy, double zz, double xy, double yz, double zx);

#ifdef __cplusplus
}
#endif
#endif
