/*
 * ffr_oracle.c — CPU restatement of ff-room's per-timestep solver.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  Every
 * function cites the reference file:line whose behaviour it restates;
 * paths are relative to the ff-room project root.  Quirks of the
 * reference are reproduced on purpose, because parity is measured
 * against it:
 *   - QUICK uses phi_mm on the right face for negative velocity
 *     (FluidSolver.cpp:64-68) and never uses phi_pp;
 *   - the u-QUICK j-2 / k-2 neighbours are formed by flat index
 *     arithmetic, so at j=1 (k=1) they read the previous j-row (k-row)
 *     of the flat array (FluidSolver.cpp:139,141);
 *   - the v/w QUICK "far" neighbours are the near ones (FluidSolver.cpp:
 *     208,211,275,276);
 *   - boundary-adjacent neighbour faces read as zero (FluidSolver.cpp:
 *     110-111,120-121,194-195,268-269);
 *   - max-reductions ignore NaN like std::max(acc, x) (FluidSolver.cpp:
 *     527-534).
 */
#include "ffr_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { CT_FLUID = 0, CT_SOLID = 1, CT_INFLOW = 2, CT_OUTFLOW = 3 };

/* Flat layout, k fastest (Grid.hpp:59-65). */
#define UI(i, j, k) ((long)(i) * (long)(r->ny * r->nz) + (long)(j) * r->nz + (k))
#define VI(i, j, k) ((long)(i) * (long)((r->ny + 1) * r->nz) + (long)(j) * r->nz + (k))
#define WI(i, j, k) ((long)(i) * (long)(r->ny * (r->nz + 1)) + (long)(j) * (r->nz + 1) + (k))
#define CI(i, j, k) ((long)(i) * (long)(r->ny * r->nz) + (long)(j) * r->nz + (k))

static long n_u(const ffro_room *r) { return (long)(r->nx + 1) * r->ny * r->nz; }
static long n_v(const ffro_room *r) { return (long)r->nx * (r->ny + 1) * r->nz; }
static long n_w(const ffro_room *r) { return (long)r->nx * r->ny * (r->nz + 1); }
static long n_c(const ffro_room *r) { return (long)r->nx * r->ny * r->nz; }

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

/* std::max(acc, x): returns acc unless acc < x (NaN x is ignored). */
static double keep_max(double acc, double x) { return (acc < x) ? x : acc; }

/* ---------------------------------------------------------------- BCs */

/* BoundaryManager::apply_noslip, BoundaryManager.cpp:60-109. */
void ffro_apply_noslip(const ffro_room *r, double *u, double *v, double *w)
{
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    const uint8_t *ct = r->cell_type;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
            if (ct[CI(0, j, k)] != CT_OUTFLOW) u[UI(0, j, k)] = 0.0;
            if (ct[CI(nx - 1, j, k)] != CT_OUTFLOW) u[UI(nx, j, k)] = 0.0;
        }
    for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++) {
            if (ct[CI(i, 0, k)] != CT_OUTFLOW) v[VI(i, 0, k)] = 0.0;
            if (ct[CI(i, ny - 1, k)] != CT_OUTFLOW) v[VI(i, ny, k)] = 0.0;
        }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            if (ct[CI(i, j, 0)] != CT_OUTFLOW) w[WI(i, j, 0)] = 0.0;
            if (ct[CI(i, j, nz - 1)] != CT_OUTFLOW) w[WI(i, j, nz)] = 0.0;
        }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                if (ct[CI(i, j, k)] != CT_SOLID) continue;
                u[UI(i, j, k)] = 0.0; u[UI(i + 1, j, k)] = 0.0;
                v[VI(i, j, k)] = 0.0; v[VI(i, j + 1, k)] = 0.0;
                w[WI(i, j, k)] = 0.0; w[WI(i, j, k + 1)] = 0.0;
            }
}

/* BoundaryManager::apply_inflow, BoundaryManager.cpp:111-130: every cell of
 * each fan box (clamped, not filtered by cell type), later fans win, only
 * components that are exactly non-zero. */
void ffro_apply_inflow(const ffro_room *r, double *u, double *v, double *w)
{
    for (int f = 0; f < r->nfans; f++) {
        const ffro_fan *fn = &r->fans[f];
        for (int i = imax(0, fn->i_min); i <= imin(r->nx - 1, fn->i_max); i++)
            for (int j = imax(0, fn->j_min); j <= imin(r->ny - 1, fn->j_max); j++)
                for (int k = imax(0, fn->k_min); k <= imin(r->nz - 1, fn->k_max); k++) {
                    if (fn->vel[0] != 0.0) { u[UI(i, j, k)] = fn->vel[0]; u[UI(i + 1, j, k)] = fn->vel[0]; }
                    if (fn->vel[1] != 0.0) { v[VI(i, j, k)] = fn->vel[1]; v[VI(i, j + 1, k)] = fn->vel[1]; }
                    if (fn->vel[2] != 0.0) { w[WI(i, j, k)] = fn->vel[2]; w[WI(i, j, k + 1)] = fn->vel[2]; }
                }
    }
}

/* BoundaryManager::apply_outflow, BoundaryManager.cpp:180-220: zero-gradient
 * copy of the adjacent interior face, patch by patch in insertion order. */
void ffro_apply_outflow(const ffro_room *r, double *u, double *v, double *w)
{
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int o = 0; o < r->nout; o++) {
        const ffro_patch *pt = &r->outflows[o];
        for (int a = pt->a_min; a <= pt->a_max; a++)
            for (int b = pt->b_min; b <= pt->b_max; b++) {
                if (pt->axis == 0) {
                    if (pt->side == 1) u[UI(nx, a, b)] = u[UI(nx - 1, a, b)];
                    else               u[UI(0, a, b)]  = u[UI(1, a, b)];
                } else if (pt->axis == 1) {
                    if (pt->side == 1) v[VI(a, ny, b)] = v[VI(a, ny - 1, b)];
                    else               v[VI(a, 0, b)]  = v[VI(a, 1, b)];
                } else {
                    if (pt->side == 1) w[WI(a, b, nz)] = w[WI(a, b, nz - 1)];
                    else               w[WI(a, b, 0)]  = w[WI(a, b, 1)];
                }
            }
    }
}

/* BoundaryManager::apply_opening_temperature, BoundaryManager.cpp:137-178. */
void ffro_apply_opening_T(const ffro_room *r, const double *u, const double *v,
                          const double *w, double *T)
{
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int o = 0; o < r->nopen; o++) {
        const ffro_patch *pt = &r->openings[o].patch;
        const double Tout = r->openings[o].T_outside;
        const int sd = pt->side;
        for (int a = pt->a_min; a <= pt->a_max; a++)
            for (int b = pt->b_min; b <= pt->b_max; b++) {
                double vf; long cw, cin;
                if (pt->axis == 0) {
                    vf  = u[UI(sd ? nx : 0, a, b)];
                    cw  = CI(sd ? nx - 1 : 0, a, b);
                    cin = CI(sd ? nx - 2 : 1, a, b);
                } else if (pt->axis == 1) {
                    vf  = v[VI(a, sd ? ny : 0, b)];
                    cw  = CI(a, sd ? ny - 1 : 0, b);
                    cin = CI(a, sd ? ny - 2 : 1, b);
                } else {
                    vf  = w[WI(a, b, sd ? nz : 0)];
                    cw  = CI(a, b, sd ? nz - 1 : 0);
                    cin = CI(a, b, sd ? nz - 2 : 1);
                }
                int incoming = sd ? (vf <= 0.0) : (vf >= 0.0);
                T[cw] = incoming ? Tout : T[cin];
            }
    }
}

/* --------------------------------------------------- advection kernels */

/* upwind1, FluidSolver.cpp:47-50 (strict > 0). */
static double adv_upwind(double pm, double pc, double pp, double a, double h)
{
    if (a > 0.0) return a * (pc - pm) / h;
    return a * (pp - pc) / h;
}

/* quick_adv, FluidSolver.cpp:56-72 (>= 0; phi_mm on the negative branch). */
static double adv_quick(double pmm, double pm, double pc, double pp, double a, double h)
{
    double fr, fl;
    if (a >= 0.0) {
        fr = (6.0 * pc + 3.0 * pp - pm) / 8.0;
        fl = (6.0 * pm + 3.0 * pc - pmm) / 8.0;
    } else {
        fr = (6.0 * pp + 3.0 * pc - pmm) / 8.0;
        fl = (6.0 * pc + 3.0 * pp - pm) / 8.0;
    }
    return a * (fr - fl) / h;
}

/* lax_wendroff_adv, FluidSolver.cpp:75-81. */
static double adv_lw(double pm, double pc, double pp, double a, double dt, double h)
{
    double cr = a * dt / h;
    double flr = a * (0.5 * (pc + pp) - 0.5 * cr * (pp - pc));
    double fll = a * (0.5 * (pm + pc) - 0.5 * cr * (pc - pm));
    return (flr - fll) / h;
}

/* FluidSolver::compute_intermediate, FluidSolver.cpp:83-309.
 * Reads (u,v,w), writes the predicted faces into (us,vs,ws). */
static void predict(const ffro_room *r, const ffro_params *prm,
                    const double *u, const double *v, const double *w,
                    double *us, double *vs, double *ws)
{
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    const double dt = prm->dt, nu = prm->nu;
    const int quick = prm->advection == 1, lw = prm->advection == 2;

    /* u faces, FluidSolver.cpp:94-169 */
    for (int i = 0; i <= nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const long c = UI(i, j, k);
                if (i == 0 || i == nx) { us[c] = u[c]; continue; }
                const double hx = r->dxv[i], hy = r->dyv[j], hz = r->dzv[k];
                const double cx = 1.0 / (hx * hx), cy = 1.0 / (hy * hy), cz = 1.0 / (hz * hz);
                const double uc = u[c];
                const double xm = (i > 1) ? u[UI(i - 1, j, k)] : 0.0;
                const double xp = (i < nx - 1) ? u[UI(i + 1, j, k)] : 0.0;
                const double av = (j > 0 && j < ny) ? 0.5 * (v[VI(i - 1, j, k)] + v[VI(i, j, k)]) : 0.0;
                const double ym = (j > 0) ? u[UI(i, j - 1, k)] : 0.0;
                const double yp = (j < ny - 1) ? u[UI(i, j + 1, k)] : 0.0;
                const double aw = (k > 0 && k < nz) ? 0.5 * (w[WI(i - 1, j, k)] + w[WI(i, j, k)]) : 0.0;
                const double zm = (k > 0) ? u[UI(i, j, k - 1)] : 0.0;
                const double zp = (k < nz - 1) ? u[UI(i, j, k + 1)] : 0.0;
                double adv;
                if (quick && i >= 2 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
                    /* flat-index far neighbours: may wrap into the previous row */
                    const double xmm = u[UI(i - 2, j, k)];
                    const double ymm = u[UI(i, j - 2, k)];
                    const double zmm = u[UI(i, j, k - 2)];
                    adv = adv_quick(xmm, xm, uc, xp, uc, hx)
                        + adv_quick(ymm, ym, uc, yp, av, hy)
                        + adv_quick(zmm, zm, uc, zp, aw, hz);
                } else if (lw) {
                    adv = adv_lw(xm, uc, xp, uc, dt, hx)
                        + adv_lw(ym, uc, yp, av, dt, hy)
                        + adv_lw(zm, uc, zp, aw, dt, hz);
                } else {
                    adv = adv_upwind(xm, uc, xp, uc, hx)
                        + adv_upwind(ym, uc, yp, av, hy)
                        + adv_upwind(zm, uc, zp, aw, hz);
                }
                const double dif = nu * (cx * (xm - 2 * uc + xp) + cy * (ym - 2 * uc + yp)
                                         + cz * (zm - 2 * uc + zp));
                us[c] = uc + dt * (-adv + dif);
            }

    /* v faces, FluidSolver.cpp:175-236 */
    for (int i = 0; i < nx; i++)
        for (int j = 0; j <= ny; j++)
            for (int k = 0; k < nz; k++) {
                const long c = VI(i, j, k);
                if (j == 0 || j == ny) { vs[c] = v[c]; continue; }
                const double hx = r->dxv[i], hy = r->dyv[j], hz = r->dzv[k];
                const double cx = 1.0 / (hx * hx), cy = 1.0 / (hy * hy), cz = 1.0 / (hz * hz);
                const double vc = v[c];
                const double au = (i > 0 && i < nx) ? 0.5 * (u[UI(i, j - 1, k)] + u[UI(i, j, k)]) : 0.0;
                const double xm = (i > 0) ? v[VI(i - 1, j, k)] : 0.0;
                const double xp = (i < nx - 1) ? v[VI(i + 1, j, k)] : 0.0;
                const double ym = (j > 1) ? v[VI(i, j - 1, k)] : 0.0;
                const double yp = (j < ny - 1) ? v[VI(i, j + 1, k)] : 0.0;
                const double aw = (k > 0 && k < nz) ? 0.5 * (w[WI(i, j - 1, k)] + w[WI(i, j, k)]) : 0.0;
                const double zm = (k > 0) ? v[VI(i, j, k - 1)] : 0.0;
                const double zp = (k < nz - 1) ? v[VI(i, j, k + 1)] : 0.0;
                double adv;
                if (quick && i >= 1 && i <= nx - 2 && j >= 2 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
                    const double xmm = v[VI(i - 1, j, k)];
                    const double ymm = v[VI(i, j - 2, k)];
                    const double zmm = v[VI(i, j, k - 1)];
                    adv = adv_quick(xmm, xm, vc, xp, au, hx)
                        + adv_quick(ymm, ym, vc, yp, vc, hy)
                        + adv_quick(zmm, zm, vc, zp, aw, hz);
                } else if (lw) {
                    adv = adv_lw(xm, vc, xp, au, dt, hx)
                        + adv_lw(ym, vc, yp, vc, dt, hy)
                        + adv_lw(zm, vc, zp, aw, dt, hz);
                } else {
                    adv = adv_upwind(xm, vc, xp, au, hx)
                        + adv_upwind(ym, vc, yp, vc, hy)
                        + adv_upwind(zm, vc, zp, aw, hz);
                }
                const double dif = nu * (cx * (xm - 2 * vc + xp) + cy * (ym - 2 * vc + yp)
                                         + cz * (zm - 2 * vc + zp));
                vs[c] = vc + dt * (-adv + dif);
            }

    /* w faces, FluidSolver.cpp:242-303 */
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k <= nz; k++) {
                const long c = WI(i, j, k);
                if (k == 0 || k == nz) { ws[c] = w[c]; continue; }
                const double hx = r->dxv[i], hy = r->dyv[j], hz = r->dzv[k];
                const double cx = 1.0 / (hx * hx), cy = 1.0 / (hy * hy), cz = 1.0 / (hz * hz);
                const double wc = w[c];
                const double au = (i > 0 && i < nx) ? 0.5 * (u[UI(i, j, k - 1)] + u[UI(i, j, k)]) : 0.0;
                const double xm = (i > 0) ? w[WI(i - 1, j, k)] : 0.0;
                const double xp = (i < nx - 1) ? w[WI(i + 1, j, k)] : 0.0;
                const double av = (j > 0 && j < ny) ? 0.5 * (v[VI(i, j, k - 1)] + v[VI(i, j, k)]) : 0.0;
                const double ym = (j > 0) ? w[WI(i, j - 1, k)] : 0.0;
                const double yp = (j < ny - 1) ? w[WI(i, j + 1, k)] : 0.0;
                const double zm = (k > 1) ? w[WI(i, j, k - 1)] : 0.0;
                const double zp = (k < nz - 1) ? w[WI(i, j, k + 1)] : 0.0;
                double adv;
                if (quick && i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 2 && k <= nz - 2) {
                    const double xmm = w[WI(i - 1, j, k)];
                    const double ymm = w[WI(i, j - 1, k)];
                    const double zmm = w[WI(i, j, k - 2)];
                    adv = adv_quick(xmm, xm, wc, xp, au, hx)
                        + adv_quick(ymm, ym, wc, yp, av, hy)
                        + adv_quick(zmm, zm, wc, zp, wc, hz);
                } else if (lw) {
                    adv = adv_lw(xm, wc, xp, au, dt, hx)
                        + adv_lw(ym, wc, yp, av, dt, hy)
                        + adv_lw(zm, wc, zp, wc, dt, hz);
                } else {
                    adv = adv_upwind(xm, wc, xp, au, hx)
                        + adv_upwind(ym, wc, yp, av, hy)
                        + adv_upwind(zm, wc, zp, wc, hz);
                }
                const double dif = nu * (cx * (xm - 2 * wc + xp) + cy * (ym - 2 * wc + yp)
                                         + cz * (zm - 2 * wc + zp));
                ws[c] = wc + dt * (-adv + dif);
            }
}

/* FluidSolver::apply_buoyancy, FluidSolver.cpp:373-386: interior z-faces of
 * every cell, SOLID and INFLOW included (the BCs override afterwards). */
static void buoyancy(const ffro_room *r, const ffro_params *prm, double *w, const double *T)
{
    const double coeff = prm->g_accel * prm->beta * prm->dt;
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 1; k < r->nz; k++)
                w[WI(i, j, k)] += coeff * (0.5 * (T[CI(i, j, k - 1)] + T[CI(i, j, k)]) - prm->T_initial);
}

/* FluidSolver::build_poisson_rhs, FluidSolver.cpp:311-330. */
static void poisson_rhs(const ffro_room *r, const ffro_params *prm, const double *u,
                        const double *v, const double *w, double *rhs)
{
    const double factor = -(prm->rho / prm->dt);
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                const long c = CI(i, j, k);
                if (r->cell_type[c] == CT_SOLID) { rhs[c] = 0.0; continue; }
                double div = (u[UI(i + 1, j, k)] - u[UI(i, j, k)]) / r->dxv[i]
                           + (v[VI(i, j + 1, k)] - v[VI(i, j, k)]) / r->dyv[j]
                           + (w[WI(i, j, k + 1)] - w[WI(i, j, k)]) / r->dzv[k];
                rhs[c] = factor * div;
            }
}

/* ---------------------------------------------------------- pressure */

/* One neighbour term of PoissonSolver::apply_laplacian (PoissonSolver.cpp:
 * 61-77): outside the domain or SOLID -> nothing; OUTFLOW -> Dirichlet
 * ghost (2*scale on the diagonal); otherwise the interior coupling. */
static void lap_term(const ffro_room *r, int ni, int nj, int nk, double s,
                     const double *x, double *diag, double *off)
{
    if (ni < 0 || ni >= r->nx || nj < 0 || nj >= r->ny || nk < 0 || nk >= r->nz) return;
    const long nc = CI(ni, nj, nk);
    const uint8_t t = r->cell_type[nc];
    if (t == CT_OUTFLOW) *diag += 2.0 * s;
    else if (t != CT_SOLID) { *diag += s; *off += s * x[nc]; }
}

/* PoissonSolver::apply_laplacian, PoissonSolver.cpp:22-91 (L = -lap). */
void ffro_laplacian(const ffro_room *r, const double *x, double *Ax)
{
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int i = 0; i < nx; i++) {
        const double hl = (i > 0) ? 0.5 * (r->dxv[i - 1] + r->dxv[i]) : r->dxv[i];
        const double hr = (i < nx - 1) ? 0.5 * (r->dxv[i] + r->dxv[i + 1]) : r->dxv[i];
        const double sxl = 1.0 / (hl * r->dxv[i]), sxr = 1.0 / (hr * r->dxv[i]);
        for (int j = 0; j < ny; j++) {
            const double gl = (j > 0) ? 0.5 * (r->dyv[j - 1] + r->dyv[j]) : r->dyv[j];
            const double gr = (j < ny - 1) ? 0.5 * (r->dyv[j] + r->dyv[j + 1]) : r->dyv[j];
            const double syl = 1.0 / (gl * r->dyv[j]), syr = 1.0 / (gr * r->dyv[j]);
            for (int k = 0; k < nz; k++) {
                const long c = CI(i, j, k);
                if (r->cell_type[c] == CT_SOLID) { Ax[c] = x[c]; continue; }
                const double el = (k > 0) ? 0.5 * (r->dzv[k - 1] + r->dzv[k]) : r->dzv[k];
                const double er = (k < nz - 1) ? 0.5 * (r->dzv[k] + r->dzv[k + 1]) : r->dzv[k];
                const double szl = 1.0 / (el * r->dzv[k]), szr = 1.0 / (er * r->dzv[k]);
                double diag = 0.0, off = 0.0;
                lap_term(r, i - 1, j, k, sxl, x, &diag, &off);
                lap_term(r, i + 1, j, k, sxr, x, &diag, &off);
                lap_term(r, i, j - 1, k, syl, x, &diag, &off);
                lap_term(r, i, j + 1, k, syr, x, &diag, &off);
                lap_term(r, i, j, k - 1, szl, x, &diag, &off);
                lap_term(r, i, j, k + 1, szr, x, &diag, &off);
                if (diag < 1e-30) diag = 1.0;
                Ax[c] = diag * x[c] - off;
            }
        }
    }
}

/* PoissonSolver::solve, PoissonSolver.cpp:93-158: unpreconditioned CG from
 * x0 = 0, stop on the recurrence residual ||r||/||rhs|| < tol checked
 * before the direction update, silent break when |d.Ad| < 1e-30, and on
 * running out of iterations the residual of the last accepted rr. */
double ffro_cg_solve(const ffro_room *r, const double *rhs, double *x,
                     int max_iter, double tol, int *iters)
{
    const long n = n_c(r);
    double *res = malloc(sizeof(double) * n), *dir = malloc(sizeof(double) * n);
    double *adir = malloc(sizeof(double) * n);
    double rr = 0.0, out;
    for (long c = 0; c < n; c++) {
        x[c] = 0.0;
        res[c] = (r->cell_type[c] == CT_SOLID) ? 0.0 : rhs[c];
        dir[c] = res[c];
    }
    for (long c = 0; c < n; c++) rr += res[c] * res[c];
    const double bnorm = sqrt(rr);
    if (bnorm < 1e-15) { *iters = 0; out = 0.0; goto done; }
    for (int it = 0; it < max_iter; it++) {
        ffro_laplacian(r, dir, adir);
        double dad = 0.0;
        for (long c = 0; c < n; c++) dad += dir[c] * adir[c];
        if (fabs(dad) < 1e-30) break;
        const double alpha = rr / dad;
        double rr1 = 0.0;
        for (long c = 0; c < n; c++) {
            x[c] += alpha * dir[c];
            res[c] -= alpha * adir[c];
            rr1 += res[c] * res[c];
        }
        const double rel = sqrt(rr1) / bnorm;
        if (rel < tol) { *iters = it + 1; out = rel; goto done; }
        const double beta = rr1 / rr;
        for (long c = 0; c < n; c++) dir[c] = res[c] + beta * dir[c];
        rr = rr1;
    }
    *iters = max_iter;
    out = sqrt(rr) / bnorm;
done:
    free(res); free(dir); free(adir);
    return out;
}

/* FluidSolver::apply_correction, FluidSolver.cpp:332-371. */
static void correct(const ffro_room *r, const ffro_params *prm, const double *p,
                    double *u, double *v, double *w)
{
    const double c0 = prm->dt / prm->rho;
    for (int i = 1; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                const double h = 0.5 * (r->dxv[i - 1] + r->dxv[i]);
                u[UI(i, j, k)] -= c0 * ((p[CI(i, j, k)] - p[CI(i - 1, j, k)]) / h);
            }
    for (int i = 0; i < r->nx; i++)
        for (int j = 1; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                const double h = 0.5 * (r->dyv[j - 1] + r->dyv[j]);
                v[VI(i, j, k)] -= c0 * ((p[CI(i, j, k)] - p[CI(i, j - 1, k)]) / h);
            }
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 1; k < r->nz; k++) {
                const double h = 0.5 * (r->dzv[k - 1] + r->dzv[k]);
                w[WI(i, j, k)] -= c0 * ((p[CI(i, j, k)] - p[CI(i, j, k - 1)]) / h);
            }
}

/* ------------------------------------------------------------ thermal */

/* get_T lambda of FluidSolver::advect_temperature, FluidSolver.cpp:417-422:
 * Neumann (the centre value) outside the domain and at SOLID cells. */
static double t_at(const ffro_room *r, const double *T, int i, int j, int k, double tc)
{
    if (i < 0 || i >= r->nx || j < 0 || j >= r->ny || k < 0 || k >= r->nz) return tc;
    const long c = CI(i, j, k);
    return (r->cell_type[c] == CT_SOLID) ? tc : T[c];
}

/* FluidSolver::advect_temperature, FluidSolver.cpp:388-456. */
static void advect_T(const ffro_room *r, const ffro_params *prm, const double *u,
                     const double *v, const double *w, const double *T, double *Tn)
{
    const double dt = prm->dt;
    const double alpha = prm->k_thermal / (prm->rho * prm->cp);
    const int quick = prm->advection == 1, lw = prm->advection == 2;
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                const long c = CI(i, j, k);
                if (r->cell_type[c] != CT_FLUID) { Tn[c] = T[c]; continue; }
                const double hx = r->dxv[i], hy = r->dyv[j], hz = r->dzv[k];
                const double tc = T[c];
                const double ac = 0.5 * (u[UI(i, j, k)] + u[UI(i + 1, j, k)]);
                const double bc = 0.5 * (v[VI(i, j, k)] + v[VI(i, j + 1, k)]);
                const double cc = 0.5 * (w[WI(i, j, k)] + w[WI(i, j, k + 1)]);
                const double xm = t_at(r, T, i - 1, j, k, tc), xp = t_at(r, T, i + 1, j, k, tc);
                const double ym = t_at(r, T, i, j - 1, k, tc), yp = t_at(r, T, i, j + 1, k, tc);
                const double zm = t_at(r, T, i, j, k - 1, tc), zp = t_at(r, T, i, j, k + 1, tc);
                double adv;
                if (quick && i >= 1 && i <= r->nx - 2 && j >= 1 && j <= r->ny - 2 && k >= 1 && k <= r->nz - 2) {
                    const double xmm = t_at(r, T, i - 2, j, k, tc);
                    const double ymm = t_at(r, T, i, j - 2, k, tc);
                    const double zmm = t_at(r, T, i, j, k - 2, tc);
                    adv = adv_quick(xmm, xm, tc, xp, ac, hx)
                        + adv_quick(ymm, ym, tc, yp, bc, hy)
                        + adv_quick(zmm, zm, tc, zp, cc, hz);
                } else if (lw) {
                    adv = adv_lw(xm, tc, xp, ac, dt, hx)
                        + adv_lw(ym, tc, yp, bc, dt, hy)
                        + adv_lw(zm, tc, zp, cc, dt, hz);
                } else {
                    adv = adv_upwind(xm, tc, xp, ac, hx)
                        + adv_upwind(ym, tc, yp, bc, hy)
                        + adv_upwind(zm, tc, zp, cc, hz);
                }
                const double dif = alpha * ((xm - 2 * tc + xp) / (hx * hx)
                                            + (ym - 2 * tc + yp) / (hy * hy)
                                            + (zm - 2 * tc + zp) / (hz * hz));
                Tn[c] = tc + dt * (-adv + dif);
            }
}

/* FluidSolver::compute_T_mean, FluidSolver.cpp:458-468. */
static double t_mean(const ffro_room *r, const ffro_params *prm, const double *T)
{
    double sum = 0.0;
    long n = 0;
    for (long c = 0; c < n_c(r); c++)
        if (r->cell_type[c] == CT_FLUID) { sum += T[c]; n++; }
    return n > 0 ? sum / (double)n : prm->T_initial;
}

/* FluidSolver::compute_divergence_max, FluidSolver.cpp:470-484 (FLUID only). */
double ffro_divergence_max(const ffro_room *r, const double *u, const double *v,
                           const double *w)
{
    double m = 0.0;
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                if (r->cell_type[CI(i, j, k)] != CT_FLUID) continue;
                double d = fabs((u[UI(i + 1, j, k)] - u[UI(i, j, k)]) / r->dxv[i]
                              + (v[VI(i, j + 1, k)] - v[VI(i, j, k)]) / r->dyv[j]
                              + (w[WI(i, j, k + 1)] - w[WI(i, j, k)]) / r->dzv[k]);
                m = keep_max(m, d);
            }
    return m;
}

/* Fixed-temperature patches: the floor/ceiling heat extension, applied after
 * the step exactly as a per-step callback writing Grid.T_shaped() would. */
static void apply_heat(const ffro_room *r, double *T)
{
    for (int h = 0; h < r->nheat; h++) {
        const ffro_heat *hp = &r->heats[h];
        for (int i = imax(0, hp->i_min); i <= imin(r->nx - 1, hp->i_max); i++)
            for (int j = imax(0, hp->j_min); j <= imin(r->ny - 1, hp->j_max); j++)
                for (int k = imax(0, hp->k_min); k <= imin(r->nz - 1, hp->k_max); k++)
                    T[CI(i, j, k)] = hp->T;
    }
}

/* FluidSolver ctor, FluidSolver.cpp:18-32. */
void ffro_fluid_init(const ffro_room *r, const ffro_params *prm, ffro_fields *f)
{
    for (long c = 0; c < n_c(r); c++) f->T[c] = prm->T_initial;
    if (prm->thermal) ffro_apply_opening_T(r, f->u, f->v, f->w, f->T);
}

/* FluidSolver::step / run, FluidSolver.cpp:486-560. */
int ffro_fluid_run(const ffro_room *r, const ffro_params *prm, ffro_fields *f,
                   int step0, int nsteps, int stop_on_converge, ffro_result *out)
{
    const long nu_ = n_u(r), nv_ = n_v(r), nw_ = n_w(r), nc_ = n_c(r);
    double *u0 = malloc(sizeof(double) * nu_), *v0 = malloc(sizeof(double) * nv_);
    double *w0 = malloc(sizeof(double) * nw_), *rhs = malloc(sizeof(double) * nc_);
    double *Tn = malloc(sizeof(double) * nc_);
    int s;
    for (s = 0; s < nsteps; s++) {
        memcpy(u0, f->u, sizeof(double) * nu_);
        memcpy(v0, f->v, sizeof(double) * nv_);
        memcpy(w0, f->w, sizeof(double) * nw_);
        predict(r, prm, u0, v0, w0, f->u, f->v, f->w);
        if (prm->buoyancy) buoyancy(r, prm, f->w, f->T);
        ffro_apply_noslip(r, f->u, f->v, f->w);
        ffro_apply_inflow(r, f->u, f->v, f->w);
        poisson_rhs(r, prm, f->u, f->v, f->w, rhs);
        int iters = 0;
        const double pres = ffro_cg_solve(r, rhs, f->p, prm->poisson_max_iter, prm->poisson_tol, &iters);
        correct(r, prm, f->p, f->u, f->v, f->w);
        ffro_apply_noslip(r, f->u, f->v, f->w);
        ffro_apply_inflow(r, f->u, f->v, f->w);
        ffro_apply_outflow(r, f->u, f->v, f->w);
        double tm = prm->T_initial;
        if (prm->thermal) {
            ffro_apply_opening_T(r, f->u, f->v, f->w, f->T);
            advect_T(r, prm, f->u, f->v, f->w, f->T, Tn);
            memcpy(f->T, Tn, sizeof(double) * nc_);
            ffro_apply_opening_T(r, f->u, f->v, f->w, f->T);
            tm = t_mean(r, prm, f->T);
        }
        double dmax = 0.0;
        for (long c = 0; c < nu_; c++) dmax = keep_max(dmax, fabs(f->u[c] - u0[c]));
        for (long c = 0; c < nv_; c++) dmax = keep_max(dmax, fabs(f->v[c] - v0[c]));
        for (long c = 0; c < nw_; c++) dmax = keep_max(dmax, fabs(f->w[c] - w0[c]));
        dmax /= prm->dt;
        int conv;
        if (prm->thermal && prm->T_target < 1e29)
            conv = (prm->T_target >= prm->T_initial) ? (tm >= prm->T_target) : (tm <= prm->T_target);
        else
            conv = dmax < prm->convergence_tol;
        ffro_result *o = &out[s];
        o->step = step0 + s + 1;
        o->velocity_change = dmax;
        o->pressure_residual = pres;
        o->divergence_max = ffro_divergence_max(r, f->u, f->v, f->w);
        o->converged = conv;
        o->T_mean = tm;
        o->cg_iterations = iters;
        apply_heat(r, f->T);
        if (conv && stop_on_converge) { s++; break; }
    }
    free(u0); free(v0); free(w0); free(rhs); free(Tn);
    return s;
}

/* ---------------------------------------------------------------- LBM */

/* D3Q19 tables, LBMSolver.cpp:13-27. */
static const int LX[19] = { 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0 };
static const int LY[19] = { 0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1 };
static const int LZ[19] = { 0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1 };
static const int LOPP[19] = { 0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17 };
static double lw_(int q)
{
    return q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
}

/* LBMSolver::feq, LBMSolver.hpp:89-93 (cs2 = 1/3). */
static double feq(int q, double rho, double ux, double uy, double uz)
{
    const double cs2 = 1.0 / 3.0;
    const double eu = LX[q] * ux + LY[q] * uy + LZ[q] * uz;
    const double usq = ux * ux + uy * uy + uz * uz;
    return lw_(q) * rho * (1.0 + eu / cs2 + eu * eu / (2.0 * cs2 * cs2) - usq / (2.0 * cs2));
}

/* LBMSolver::apply_inflow_bc, LBMSolver.cpp:80-99. */
static void lbm_inflow(const ffro_room *r, double p2l, double *f)
{
    const long n = n_c(r);
    for (int a = 0; a < r->nfans; a++) {
        const ffro_fan *fn = &r->fans[a];
        const double vx = fn->vel[0] * p2l, vy = fn->vel[1] * p2l, vz = fn->vel[2] * p2l;
        for (int i = fn->i_min; i <= fn->i_max; i++)
            for (int j = fn->j_min; j <= fn->j_max; j++)
                for (int k = fn->k_min; k <= fn->k_max; k++) {
                    if (i < 0 || i >= r->nx || j < 0 || j >= r->ny || k < 0 || k >= r->nz) continue;
                    const long c = CI(i, j, k);
                    if (r->cell_type[c] != CT_INFLOW) continue;
                    for (int q = 0; q < 19; q++) f[q * n + c] = feq(q, 1.0, vx, vy, vz);
                }
    }
}

/* LBMSolver ctor / initialize_f, LBMSolver.cpp:33-74. */
void ffro_lbm_init(const ffro_room *r, double tau, double dt, double *f)
{
    (void)tau;
    const long n = n_c(r);
    for (int q = 0; q < 19; q++)
        for (long c = 0; c < n; c++) f[q * n + c] = lw_(q);
    lbm_inflow(r, dt / r->dx, f);
}

/* moments of one cell (LBMSolver.cpp:116-128, 306-318). */
static void moments(const double *f, long n, long c, double *rho, double *ux, double *uy, double *uz)
{
    double m0 = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
    for (int q = 0; q < 19; q++) {
        const double fq = f[q * n + c];
        m0 += fq; mx += fq * LX[q]; my += fq * LY[q]; mz += fq * LZ[q];
    }
    if (m0 > 1e-14) { mx /= m0; my /= m0; mz /= m0; }
    *rho = m0; *ux = mx; *uy = my; *uz = mz;
}

/* LBMSolver::collision, LBMSolver.cpp:106-144. */
static void lbm_collide(const ffro_room *r, double tau, double *f)
{
    const long n = n_c(r);
    const double itau = 1.0 / tau;
    for (long c = 0; c < n; c++) {
        const uint8_t t = r->cell_type[c];
        if (t == CT_SOLID || t == CT_INFLOW) continue;
        double rho, ux, uy, uz;
        moments(f, n, c, &rho, &ux, &uy, &uz);
        for (int q = 0; q < 19; q++) {
            const double fe = feq(q, rho, ux, uy, uz);
            f[q * n + c] += itau * (fe - f[q * n + c]);
        }
    }
}

/* LBMSolver::streaming, LBMSolver.cpp:151-190 (push with halfway
 * bounce-back into a zeroed buffer). */
static void lbm_stream(const ffro_room *r, const double *f, double *g)
{
    const long n = n_c(r);
    memset(g, 0, sizeof(double) * 19 * n);
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                const long c = CI(i, j, k);
                if (r->cell_type[c] == CT_SOLID) continue;
                for (int q = 0; q < 19; q++) {
                    const int a = i + LX[q], b = j + LY[q], e = k + LZ[q];
                    const int oob = a < 0 || a >= r->nx || b < 0 || b >= r->ny || e < 0 || e >= r->nz;
                    if (oob || r->cell_type[CI(a, b, e)] == CT_SOLID)
                        g[LOPP[q] * n + c] += f[q * n + c];
                    else
                        g[q * n + CI(a, b, e)] += f[q * n + c];
                }
            }
}

/* LBMSolver::apply_outflow_bc, LBMSolver.cpp:196-282: the outflow list
 * (which already holds the openings, BoundaryManager.cpp:132-135) and then
 * the opening list again. */
static void lbm_outflow_list(const ffro_room *r, const ffro_patch *pts, int np, long stride, double *f)
{
    const long n = n_c(r);
    for (int o = 0; o < np; o++) {
        const ffro_patch *pt = (const ffro_patch *)((const char *)pts + o * stride);
        const int lim_a = pt->axis == 0 ? r->ny : r->nx;
        const int lim_b = pt->axis == 2 ? r->ny : r->nz;
        const int nax = pt->axis == 0 ? r->nx : (pt->axis == 1 ? r->ny : r->nz);
        const int wall = pt->side == 0 ? 0 : nax - 1;
        const int src = pt->side == 0 ? 1 : nax - 2;
        if (src < 0 || src >= nax) continue;
        for (int a = pt->a_min; a <= pt->a_max; a++)
            for (int b = pt->b_min; b <= pt->b_max; b++) {
                if (a < 0 || a >= lim_a || b < 0 || b >= lim_b) continue;
                long cd, cs;
                if (pt->axis == 0)      { cd = CI(wall, a, b); cs = CI(src, a, b); }
                else if (pt->axis == 1) { cd = CI(a, wall, b); cs = CI(a, src, b); }
                else                    { cd = CI(a, b, wall); cs = CI(a, b, src); }
                if (r->cell_type[cd] != CT_OUTFLOW) continue;
                for (int q = 0; q < 19; q++) f[q * n + cd] = f[q * n + cs];
            }
    }
}

/* LBMSolver::extract_macroscopic, LBMSolver.cpp:288-376. */
static void lbm_macro(const ffro_room *r, double l2p, const double *f, ffro_fields *fl,
                      double *cx, double *cy, double *cz)
{
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    const long n = n_c(r);
    for (long c = 0; c < n; c++) {
        if (r->cell_type[c] == CT_SOLID) { cx[c] = cy[c] = cz[c] = 0.0; continue; }
        double rho, ux, uy, uz;
        moments(f, n, c, &rho, &ux, &uy, &uz);
        cx[c] = ux * l2p; cy[c] = uy * l2p; cz[c] = uz * l2p;
        fl->p[c] = rho * (1.0 / 3.0);
    }
    for (int i = 0; i <= nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++)
                fl->u[UI(i, j, k)] = i == 0 ? cx[CI(0, j, k)]
                                   : i == nx ? cx[CI(nx - 1, j, k)]
                                   : 0.5 * (cx[CI(i - 1, j, k)] + cx[CI(i, j, k)]);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j <= ny; j++)
            for (int k = 0; k < nz; k++)
                fl->v[VI(i, j, k)] = j == 0 ? cy[CI(i, 0, k)]
                                   : j == ny ? cy[CI(i, ny - 1, k)]
                                   : 0.5 * (cy[CI(i, j - 1, k)] + cy[CI(i, j, k)]);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k <= nz; k++)
                fl->w[WI(i, j, k)] = k == 0 ? cz[CI(i, j, 0)]
                                   : k == nz ? cz[CI(i, j, nz - 1)]
                                   : 0.5 * (cz[CI(i, j, k - 1)] + cz[CI(i, j, k)]);
}

/* LBMSolver::step / run, LBMSolver.cpp:402-454. */
int ffro_lbm_run(const ffro_room *r, double tau, double dt, double tol,
                 double *f, double *ftmp, ffro_fields *fl, int step0, int nsteps,
                 int stop_on_converge, ffro_result *out)
{
    const long nu_ = n_u(r), nv_ = n_v(r), nw_ = n_w(r), n = n_c(r);
    const double p2l = dt / r->dx, l2p = r->dx / dt;
    double *u0 = malloc(sizeof(double) * nu_), *v0 = malloc(sizeof(double) * nv_);
    double *w0 = malloc(sizeof(double) * nw_);
    double *cx = malloc(sizeof(double) * n), *cy = malloc(sizeof(double) * n), *cz = malloc(sizeof(double) * n);
    double *cur = f, *nxt = ftmp;
    int s;
    for (s = 0; s < nsteps; s++) {
        memcpy(u0, fl->u, sizeof(double) * nu_);
        memcpy(v0, fl->v, sizeof(double) * nv_);
        memcpy(w0, fl->w, sizeof(double) * nw_);
        lbm_inflow(r, p2l, cur);
        lbm_collide(r, tau, cur);
        lbm_stream(r, cur, nxt);
        { double *t = cur; cur = nxt; nxt = t; }
        lbm_outflow_list(r, r->outflows, r->nout, sizeof(ffro_patch), cur);
        if (r->nopen > 0)
            lbm_outflow_list(r, &r->openings[0].patch, r->nopen, sizeof(ffro_opening), cur);
        lbm_macro(r, l2p, cur, fl, cx, cy, cz);
        double dmax = 0.0;
        for (long c = 0; c < nu_; c++) dmax = keep_max(dmax, fabs(fl->u[c] - u0[c]));
        for (long c = 0; c < nv_; c++) dmax = keep_max(dmax, fabs(fl->v[c] - v0[c]));
        for (long c = 0; c < nw_; c++) dmax = keep_max(dmax, fabs(fl->w[c] - w0[c]));
        dmax /= dt;
        ffro_result *o = &out[s];
        o->step = step0 + s + 1;
        o->velocity_change = dmax;
        o->pressure_residual = 0.0;
        o->divergence_max = ffro_divergence_max(r, fl->u, fl->v, fl->w);
        o->converged = dmax < tol;
        o->T_mean = 0.0;
        o->cg_iterations = 0;
        if (o->converged && stop_on_converge) { s++; break; }
    }
    /* The live populations must end up in the caller's f buffer. */
    if (cur != f) memcpy(f, cur, sizeof(double) * 19 * n);
    free(u0); free(v0); free(w0); free(cx); free(cy); free(cz);
    return s;
}
