// ref_driver.cpp — a thin C driver around the reference solver, compiled
// together with the reference's own cpp/src/core/*.cpp by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY.  It exists because the reference binds no CG
// iteration count (PoissonSolver::last_iterations, PoissonSolver.hpp:27,
// is not exported by module.cpp), and because the host cores of a GPU box
// have no Python copy of the reference: bench.py's reference arm and the
// golden-fixture generator drive the reference through this C ABI.
//
// The room is assembled through the reference BoundaryManager in the same
// order Scene._build uses (scene.py:91-106): solid boxes, fans, openings,
// then outflows.
#include <vector>
#include <functional>
#include <array>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <chrono>

// Read access to FluidSolver::poisson_ (a private member) for the iteration
// count; the reference sources themselves are compiled unchanged.
#define private public
#include "core/FluidSolver.hpp"
#include "core/LBMSolver.hpp"
#undef private

using namespace ffroom;

extern "C" {

struct ffref_room {
    int nx, ny, nz;
    double lx, ly, lz;
    const double *xs, *ys, *zs;          // face coordinates or null (uniform)
    int nsolid; const int *solids;       // 6 ints per box
    int nfans;  const int *fan_box;      // 6 ints per fan
    const double *fan_vel;               // 3 doubles per fan
    int nopen;  const int *open_patch;   // 6 ints per opening (axis, side, a0, a1, b0, b1)
    const double *open_T;
    int nout;   const int *out_patch;    // 6 ints per outflow
    int nheat;  const int *heat_box;     // 6 ints per fixed-T patch (extension)
    const double *heat_T;
};

struct ffref_params {
    double rho, nu, dt;
    int max_steps;
    double convergence_tol;
    int poisson_max_iter;
    double poisson_tol;
    int advection;
    int use_openmp;
    int thermal;
    double T_initial, T_target;
    int buoyancy;
    double g_accel, beta, k_thermal, cp;
    double time_budget;   // seconds of stepping after which a run stops (0 = none)
};

struct ffref_result {
    int step;
    double velocity_change, pressure_residual, divergence_max;
    int converged;
    double T_mean;
    int cg_iterations;
    double seconds;       // wall time of the solver's step() call
};

static void build(const ffref_room *d, Grid &g, BoundaryManager &bm)
{
    if (d->xs) {
        g.set_face_coords(std::vector<double>(d->xs, d->xs + d->nx + 1),
                          std::vector<double>(d->ys, d->ys + d->ny + 1),
                          std::vector<double>(d->zs, d->zs + d->nz + 1));
    }
    for (int s = 0; s < d->nsolid; s++) {
        const int *b = d->solids + 6 * s;
        bm.add_solid_box(g, b[0], b[1], b[2], b[3], b[4], b[5]);
    }
    for (int f = 0; f < d->nfans; f++) {
        const int *b = d->fan_box + 6 * f;
        FanBC fan;
        fan.i_min = b[0]; fan.i_max = b[1]; fan.j_min = b[2];
        fan.j_max = b[3]; fan.k_min = b[4]; fan.k_max = b[5];
        fan.vel = {d->fan_vel[3 * f], d->fan_vel[3 * f + 1], d->fan_vel[3 * f + 2]};
        bm.add_fan(g, fan);
    }
    for (int o = 0; o < d->nopen; o++) {
        const int *b = d->open_patch + 6 * o;
        OpeningBC ob;
        ob.axis = b[0]; ob.side = b[1]; ob.a_min = b[2]; ob.a_max = b[3];
        ob.b_min = b[4]; ob.b_max = b[5]; ob.T_outside = d->open_T[o];
        bm.add_opening(g, ob);
    }
    for (int o = 0; o < d->nout; o++) {
        const int *b = d->out_patch + 6 * o;
        OutflowBC ob;
        ob.axis = b[0]; ob.side = b[1]; ob.a_min = b[2]; ob.a_max = b[3];
        ob.b_min = b[4]; ob.b_max = b[5];
        bm.add_outflow(g, ob);
    }
}

static void heat(const ffref_room *d, Grid &g)
{
    for (int h = 0; h < d->nheat; h++) {
        const int *b = d->heat_box + 6 * h;
        for (int i = std::max(0, b[0]); i <= std::min(g.Nx - 1, b[1]); i++)
            for (int j = std::max(0, b[2]); j <= std::min(g.Ny - 1, b[3]); j++)
                for (int k = std::max(0, b[4]); k <= std::min(g.Nz - 1, b[5]); k++)
                    g.T[g.c_idx(i, j, k)] = d->heat_T[h];
    }
}

static void put(const std::vector<double> &v, double *o)
{
    if (o) std::memcpy(o, v.data(), v.size() * sizeof(double));
}

// Runs up to nsteps projection steps.  init_u/v/w (may be null) seed the
// velocity before the solver is built.  Returns the steps taken.
int ffref_fluid_run(const ffref_room *d, const ffref_params *p, int nsteps,
                    int stop_on_converge, const double *init_u, const double *init_v,
                    const double *init_w, uint8_t *cell_type_out, double *u, double *v,
                    double *w, double *pr, double *T, ffref_result *res)
{
    Grid g(d->nx, d->ny, d->nz, d->lx, d->ly, d->lz);
    BoundaryManager bm;
    build(d, g, bm);
    if (init_u) std::memcpy(g.u.data(), init_u, g.u.size() * sizeof(double));
    if (init_v) std::memcpy(g.v.data(), init_v, g.v.size() * sizeof(double));
    if (init_w) std::memcpy(g.w.data(), init_w, g.w.size() * sizeof(double));
    FluidSolverParams fp;
    fp.rho = p->rho; fp.nu = p->nu; fp.dt = p->dt; fp.max_steps = p->max_steps;
    fp.convergence_tol = p->convergence_tol;
    fp.poisson.max_iter = p->poisson_max_iter; fp.poisson.tol = p->poisson_tol;
    fp.advection = static_cast<AdvectionScheme>(p->advection);
    fp.use_openmp = p->use_openmp != 0;
    fp.thermal = p->thermal != 0; fp.T_initial = p->T_initial; fp.T_target = p->T_target;
    fp.buoyancy = p->buoyancy != 0; fp.g_accel = p->g_accel; fp.beta = p->beta;
    fp.k_thermal = p->k_thermal; fp.cp = p->cp;
    FluidSolver s(g, bm, fp);
    int done = 0;
    double spent = 0.0;
    for (; done < nsteps; done++) {
        if (p->time_budget > 0 && spent >= p->time_budget) break;
        const auto t0 = std::chrono::steady_clock::now();
        StepResult r = s.step();
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        spent += sec;
        if (res) {
            res[done].seconds = sec;
            res[done].step = r.step;
            res[done].velocity_change = r.velocity_change;
            res[done].pressure_residual = r.pressure_residual;
            res[done].divergence_max = r.divergence_max;
            res[done].converged = r.converged ? 1 : 0;
            res[done].T_mean = r.T_mean;
            res[done].cg_iterations = s.poisson_.last_iterations();
        }
        heat(d, g);
        if (r.converged && stop_on_converge) { done++; break; }
    }
    if (cell_type_out)
        for (size_t c = 0; c < g.cell_type.size(); c++)
            cell_type_out[c] = static_cast<uint8_t>(g.cell_type[c]);
    put(g.u, u); put(g.v, v); put(g.w, w); put(g.p, pr); put(g.T, T);
    return done;
}

int ffref_lbm_run(const ffref_room *d, double tau, double dt, double tol, int nsteps,
                  int stop_on_converge, double *u, double *v, double *w, double *pr,
                  ffref_result *res)
{
    Grid g(d->nx, d->ny, d->nz, d->lx, d->ly, d->lz);
    BoundaryManager bm;
    build(d, g, bm);
    LBMSolver s(g, bm, tau, nsteps, tol, dt);
    int done = 0;
    for (; done < nsteps; done++) {
        const auto t0 = std::chrono::steady_clock::now();
        StepResult r = s.step();
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (res) {
            res[done].seconds = sec;
            res[done].step = r.step;
            res[done].velocity_change = r.velocity_change;
            res[done].pressure_residual = r.pressure_residual;
            res[done].divergence_max = r.divergence_max;
            res[done].converged = r.converged ? 1 : 0;
            res[done].T_mean = r.T_mean;
            res[done].cg_iterations = 0;
        }
        if (r.converged && stop_on_converge) { done++; break; }
    }
    put(g.u, u); put(g.v, v); put(g.w, w); put(g.p, pr);
    return done;
}

// PoissonSolver::solve (PoissonSolver.cpp:93-158) on a grid whose cell
// types are given cell by cell, as the reference's own Poisson test sets
// them (a room no BoundaryManager call can build).  Writes the pressure and
// the iteration count; returns the relative residual.
double ffref_poisson_solve(int nx, int ny, int nz, double lx, double ly, double lz,
                           const uint8_t *cell_type, const double *rhs, int max_iter, double tol,
                           double *p, int *iterations)
{
    Grid g(nx, ny, nz, lx, ly, lz);
    for (size_t c = 0; c < g.cell_type.size(); c++) g.cell_type[c] = static_cast<CellType>(cell_type[c]);
    PoissonSolverParams prm;
    prm.max_iter = max_iter;
    prm.tol = tol;
    PoissonSolver s(prm);
    const double res = s.solve(g, std::vector<double>(rhs, rhs + g.p.size()));
    put(g.p, p);
    if (iterations) *iterations = s.last_iterations();
    return res;
}

}  // extern "C"
