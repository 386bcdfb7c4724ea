/*
 * ffr_oracle.h — CPU restatement of ff-room's per-timestep solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load it.  The product (ff-room_b200/) never links or calls it.
 *
 * It restates, in plain C, the algorithm of the reference files
 *   cpp/src/core/Grid.{hpp,cpp}, BoundaryManager.cpp, FluidSolver.cpp,
 *   PoissonSolver.cpp (CG part), LBMSolver.cpp
 * with every quirk kept (see the per-function citations in ffr_oracle.c).
 * It is pinned against the compiled reference (oracle/_ref) through the
 * golden fixtures in tests/golden/.
 */
#ifndef FFR_ORACLE_H
#define FFR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { int i_min, i_max, j_min, j_max, k_min, k_max; double vel[3]; } ffro_fan;
typedef struct { int axis, side, a_min, a_max, b_min, b_max; } ffro_patch;
typedef struct { ffro_patch patch; double T_outside; } ffro_opening;
typedef struct { int i_min, i_max, j_min, j_max, k_min, k_max; double T; } ffro_heat;

typedef struct {
    int nx, ny, nz;
    double dx;                /* Lx/Nx, the LBM reference length */
    const double *dxv, *dyv, *dzv;
    const uint8_t *cell_type; /* 0 FLUID, 1 SOLID, 2 INFLOW, 3 OUTFLOW */
    int nfans;  const ffro_fan *fans;
    int nout;   const ffro_patch *outflows;   /* outflows + openings, insertion order */
    int nopen;  const ffro_opening *openings;
    int nheat;  const ffro_heat *heats;       /* fixed-T patches (extension) */
} ffro_room;

typedef struct {
    double rho, nu, dt;
    double convergence_tol;
    int    poisson_max_iter;
    double poisson_tol;
    int    advection;        /* 0 upwind1, 1 QUICK, 2 Lax-Wendroff */
    int    thermal;
    double T_initial, T_target;
    int    buoyancy;
    double g_accel, beta, k_thermal, cp;
} ffro_params;

typedef struct {
    int    step;
    double velocity_change, pressure_residual, divergence_max;
    int    converged;
    double T_mean;
    int    cg_iterations;
} ffro_result;

/* Fields of one room, caller-owned, reference layout (k fastest). */
typedef struct {
    double *u, *v, *w, *p, *T;
} ffro_fields;

/* FluidSolver ctor side effects: T := T_initial; opening T if thermal. */
void ffro_fluid_init(const ffro_room *r, const ffro_params *prm, ffro_fields *f);
/* Runs up to nsteps projection steps; stops early on convergence when
 * stop_on_converge != 0.  Returns the number of steps taken. */
int  ffro_fluid_run(const ffro_room *r, const ffro_params *prm, ffro_fields *f,
                    int step0, int nsteps, int stop_on_converge, ffro_result *out);

/* Building blocks, exported for unit tests. */
void   ffro_apply_noslip(const ffro_room *r, double *u, double *v, double *w);
void   ffro_apply_inflow(const ffro_room *r, double *u, double *v, double *w);
void   ffro_apply_outflow(const ffro_room *r, double *u, double *v, double *w);
void   ffro_apply_opening_T(const ffro_room *r, const double *u, const double *v,
                            const double *w, double *T);
void   ffro_laplacian(const ffro_room *r, const double *x, double *Ax);
double ffro_cg_solve(const ffro_room *r, const double *rhs, double *x,
                     int max_iter, double tol, int *iters);
double ffro_divergence_max(const ffro_room *r, const double *u, const double *v,
                           const double *w);

/* D3Q19 LBM.  f and ftmp hold 19*N doubles each. */
void ffro_lbm_init(const ffro_room *r, double tau, double dt, double *f);
int  ffro_lbm_run(const ffro_room *r, double tau, double dt, double tol,
                  double *f, double *ftmp, ffro_fields *fl, int step0, int nsteps,
                  int stop_on_converge, ffro_result *out);

#ifdef __cplusplus
}
#endif
#endif
