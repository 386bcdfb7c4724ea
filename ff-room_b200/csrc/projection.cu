// projection.cu — Chorin projection step on the MAC grid, FP64 (sm_100a).
//
// One step (FluidSolver::step, cpp/src/core/FluidSolver.cpp:486-550) is
//   k_predict        advection + diffusion + buoyancy + no-slip/inflow codes
//   k_cg             persistent cooperative CG: rhs, x0 = 0, iterations
//   k_correct        pressure correction + BC codes + outflow copy,
//                    max |du| and max |div| in the same pass (cell-centric)
//   k_opening_T,     thermal: opening BC, advection-diffusion of T with the
//   k_advect_T,      block partial sums of T over FLUID cells, opening BC,
//   k_heat           fixed-T patches
//   k_finalize       StepResult, convergence, halt flag, T buffer swap
// All kernels return at once when the room's halt flag is set, so a run of
// queued steps can stop on convergence without a host round trip.
#include "projection.cuh"
#include "mgpcg.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

namespace ffr {

#define UIX(i, j, k) (((i) * ny + (j)) * nz + (k))
#define VIX(i, j, k) (((i) * (ny + 1) + (j)) * nz + (k))
#define WIX(i, j, k) (((i) * ny + (j)) * (nz + 1) + (k))

// ------------------------------------------------- advection formulas

// upwind1, FluidSolver.cpp:47-50.
template <class F>
__device__ __forceinline__ F adv_up(F pm, F pc, F pp, F a, F h)
{
    return (a > F(0)) ? a * (pc - pm) / h : a * (pp - pc) / h;
}

// quick_adv, FluidSolver.cpp:56-72 (phi_mm on the negative branch, >= 0).
template <class F>
__device__ __forceinline__ F adv_quick(F pmm, F pm, F pc, F pp, F a, F h)
{
    F fr, fl;
    if (a >= F(0)) {
        fr = (F(6) * pc + F(3) * pp - pm) / F(8);
        fl = (F(6) * pm + F(3) * pc - pmm) / F(8);
    } else {
        fr = (F(6) * pp + F(3) * pc - pmm) / F(8);
        fl = (F(6) * pc + F(3) * pp - pm) / F(8);
    }
    return a * (fr - fl) / h;
}

// lax_wendroff_adv, FluidSolver.cpp:75-81.
template <class F>
__device__ __forceinline__ F adv_lw(F pm, F pc, F pp, F a, F dt, F h)
{
    const F cr = a * dt / h;
    const F flr = a * (F(0.5) * (pc + pp) - F(0.5) * cr * (pp - pc));
    const F fll = a * (F(0.5) * (pm + pc) - F(0.5) * cr * (pc - pm));
    return (flr - fll) / h;
}

// The three schemes with the reciprocal spacing ih = 1/h (mixed precision).
template <class F>
__device__ __forceinline__ F adv_up_r(F pm, F pc, F pp, F a, F ih)
{
    return (a > F(0)) ? a * (pc - pm) * ih : a * (pp - pc) * ih;
}

template <class F>
__device__ __forceinline__ F adv_quick_r(F pmm, F pm, F pc, F pp, F a, F ih)
{
    F fr, fl;
    if (a >= F(0)) {
        fr = (F(6) * pc + F(3) * pp - pm) * F(0.125);
        fl = (F(6) * pm + F(3) * pc - pmm) * F(0.125);
    } else {
        fr = (F(6) * pp + F(3) * pc - pmm) * F(0.125);
        fl = (F(6) * pc + F(3) * pp - pm) * F(0.125);
    }
    return a * (fr - fl) * ih;
}

template <class F>
__device__ __forceinline__ F adv_lw_r(F pm, F pc, F pp, F a, F dt, F ih)
{
    const F cr = a * dt * ih;
    const F flr = a * (F(0.5) * (pc + pp) - F(0.5) * cr * (pp - pc));
    const F fll = a * (F(0.5) * (pm + pc) - F(0.5) * cr * (pc - pm));
    return (flr - fll) * ih;
}

// The spacing argument of face_increment along one axis: the cell width
// for FP64 arithmetic, its correctly rounded FP32 reciprocal (a table of
// the room) for the mixed-precision mode.
template <class F>
__device__ __forceinline__ F axis_spacing(const double *width, const float *rwidth, int i)
{
    if constexpr (sizeof(F) == 4) return rwidth[i];
    else return width[i];
}

// The predicted increment dt*(-adv + dif) of one face from its stencil
// values (FluidSolver.cpp:132-162), in arithmetic F.  ax is the advecting
// velocity along x for this face, etc.; hx, hy, hz are axis_spacing<F>
// values (widths in FP64, reciprocal widths in FP32); scheme 1 = QUICK (the caller has
// checked its activation range and passes the far neighbours), 2 = LW.
template <class F>
__device__ __forceinline__ F face_increment(int use_quick, int lw, F c, F xmm, F xm, F xp, F ymm, F ym, F yp,
                                            F zmm, F zm, F zp, F ax, F ay, F az, F hx, F hy, F hz, F nu, F dt)
{
    if constexpr (sizeof(F) == 4) {
        // mixed precision: products with the correctly rounded reciprocal
        // widths in place of the six divisions (well inside the mixed bound)
        const F ix = hx, iy = hy, iz = hz;
        F adv;
        if (use_quick) {
            adv = adv_quick_r(xmm, xm, c, xp, ax, ix) + adv_quick_r(ymm, ym, c, yp, ay, iy) +
                  adv_quick_r(zmm, zm, c, zp, az, iz);
        } else if (lw) {
            adv = adv_lw_r(xm, c, xp, ax, dt, ix) + adv_lw_r(ym, c, yp, ay, dt, iy) + adv_lw_r(zm, c, zp, az, dt, iz);
        } else {
            adv = adv_up_r(xm, c, xp, ax, ix) + adv_up_r(ym, c, yp, ay, iy) + adv_up_r(zm, c, zp, az, iz);
        }
        const F dif = nu * ((ix * ix) * (xm - F(2) * c + xp) + (iy * iy) * (ym - F(2) * c + yp) +
                            (iz * iz) * (zm - F(2) * c + zp));
        return dt * (-adv + dif);
    }
    F adv;
    if (use_quick) {
        adv = adv_quick(xmm, xm, c, xp, ax, hx) + adv_quick(ymm, ym, c, yp, ay, hy) + adv_quick(zmm, zm, c, zp, az, hz);
    } else if (lw) {
        adv = adv_lw(xm, c, xp, ax, dt, hx) + adv_lw(ym, c, yp, ay, dt, hy) + adv_lw(zm, c, zp, az, dt, hz);
    } else {
        adv = adv_up(xm, c, xp, ax, hx) + adv_up(ym, c, yp, ay, hy) + adv_up(zm, c, zp, az, hz);
    }
    const F cx = F(1) / (hx * hx), cy = F(1) / (hy * hy), cz = F(1) / (hz * hz);
    const F dif = nu * (cx * (xm - F(2) * c + xp) + cy * (ym - F(2) * c + yp) + cz * (zm - F(2) * c + zp));
    return dt * (-adv + dif);
}

__device__ __forceinline__ double face_code(uint8_t code, double val, const double *fanvel, int comp)
{
    const int c = code & 0x7f;
    if (c == FC_KEEP) return val;
    if (c == FC_ZERO) return 0.0;
    return fanvel[(c - FC_FAN0) * 3 + comp];
}

struct PredArgs {
    double dt, nu;
    int scheme;          // 0 upwind, 1 QUICK, 2 Lax-Wendroff
    int buoyancy;
    double bcoeff;       // g * beta * dt
    double T_ref;
};

// The predicted value of one interior face from its loaded neighbourhood
// (compute_intermediate, FluidSolver.cpp:83-309): the boundary selects (a
// neighbour outside reads as 0, as in the reference), the far-neighbour
// selection of QUICK, then the increment in arithmetic F.  c is the face's
// own value, xm0 .. zp0 its six neighbours, xmm0 .. zmm0 the far ones (read
// only under QUICK), a0/a1 and b0/b1 the two pairs of the other components
// averaged into the advecting velocities.
template <class F>
__device__ __forceinline__ double pred_u(int quick, int lw, int nx, int ny, int nz, int i, int j, int k, double c,
                                         double xmm0, double xm0, double xp0, double ymm0, double ym0, double yp0,
                                         double zmm0, double zm0, double zp0, double v0, double v1, double w0,
                                         double w1, F hx, F hy, F hz, F nu, F dt)
{
    const int q = quick && i >= 2 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2;
    // flat-index far neighbours (FluidSolver.cpp:137-141): at j=1 (k=1)
    // they fall into the previous row of the flat array
    const double xmm = q ? xmm0 : 0.0, ymm = q ? ymm0 : 0.0, zmm = q ? zmm0 : 0.0;
    const double xm = (i > 1) ? xm0 : 0.0, xp = (i < nx - 1) ? xp0 : 0.0;
    const double av = (j > 0 && j < ny) ? 0.5 * (v0 + v1) : 0.0;
    const double ym = (j > 0) ? ym0 : 0.0, yp = (j < ny - 1) ? yp0 : 0.0;
    const double aw = (k > 0 && k < nz) ? 0.5 * (w0 + w1) : 0.0;
    const double zm = (k > 0) ? zm0 : 0.0, zp = (k < nz - 1) ? zp0 : 0.0;
    return c + (double)face_increment<F>(q, lw, F(c), F(xmm), F(xm), F(xp), F(ymm), F(ym), F(yp), F(zmm), F(zm),
                                         F(zp), F(c), F(av), F(aw), hx, hy, hz, nu, dt);
}

template <class F>
__device__ __forceinline__ double pred_v(int quick, int lw, int nx, int ny, int nz, int i, int j, int k, double c,
                                         double xm0, double xp0, double ymm0, double ym0, double yp0, double zm0,
                                         double zp0, double u0, double u1, double w0, double w1, F hx, F hy, F hz,
                                         F nu, F dt)
{
    const int q = quick && i >= 1 && i <= nx - 2 && j >= 2 && j <= ny - 2 && k >= 1 && k <= nz - 2;
    // v's x and z "far" neighbours are the near ones (FluidSolver.cpp:208,211)
    const double ymm = q ? ymm0 : 0.0;
    const double au = (i > 0) ? 0.5 * (u0 + u1) : 0.0;
    const double xm = (i > 0) ? xm0 : 0.0, xp = (i < nx - 1) ? xp0 : 0.0;
    const double ym = (j > 1) ? ym0 : 0.0, yp = (j < ny - 1) ? yp0 : 0.0;
    const double aw = (k > 0 && k < nz) ? 0.5 * (w0 + w1) : 0.0;
    const double zm = (k > 0) ? zm0 : 0.0, zp = (k < nz - 1) ? zp0 : 0.0;
    return c + (double)face_increment<F>(q, lw, F(c), F(xm), F(xm), F(xp), F(ymm), F(ym), F(yp), F(zm), F(zm),
                                         F(zp), F(au), F(c), F(aw), hx, hy, hz, nu, dt);
}

// w additionally takes apply_buoyancy (FluidSolver.cpp:373-386) from the
// temperatures tb, tc of the cells below and above the face.
template <class F>
__device__ __forceinline__ double pred_w(const PredArgs &A, int quick, int lw, int nx, int ny, int nz, int i, int j,
                                         int k, double c, double xm0, double xp0, double ym0, double yp0,
                                         double zmm0, double zm0, double zp0, double u0, double u1, double v0,
                                         double v1, double tb, double tc, F hx, F hy, F hz, F nu, F dt)
{
    const int q = quick && i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 2 && k <= nz - 2;
    // w's x and y "far" neighbours are the near ones (FluidSolver.cpp:275-276)
    const double zmm = q ? zmm0 : 0.0;
    const double au = (i > 0) ? 0.5 * (u0 + u1) : 0.0;
    const double xm = (i > 0) ? xm0 : 0.0, xp = (i < nx - 1) ? xp0 : 0.0;
    const double av = (j > 0) ? 0.5 * (v0 + v1) : 0.0;
    const double ym = (j > 0) ? ym0 : 0.0, yp = (j < ny - 1) ? yp0 : 0.0;
    const double zm = (k > 1) ? zm0 : 0.0, zp = (k < nz - 1) ? zp0 : 0.0;
    double val = c + (double)face_increment<F>(q, lw, F(c), F(xm), F(xm), F(xp), F(ym), F(ym), F(yp), F(zmm),
                                               F(zm), F(zp), F(au), F(av), F(c), hx, hy, hz, nu, dt);
    if (A.buoyancy) val += (double)(F(A.bcoeff) * (F(0.5) * (F(tb) + F(tc)) - F(A.T_ref)));
    return val;
}

// Predictor for every face of u, v and w: FluidSolver::compute_intermediate
// (FluidSolver.cpp:83-309), then apply_buoyancy on interior w faces
// (FluidSolver.cpp:373-386), then the no-slip / inflow codes
// (BoundaryManager.cpp:60-130).  F is the arithmetic of the increment:
// double reproduces the reference; float is the mixed-precision mode (FP32
// increment added to the FP64 state).  The body over work items start,
// start + stride, ... (all blocks of one room).
//
// One pass over the corners (i, j, k) of the extended grid
// (nx+1)(ny+1)(nz+1): the u, v and w faces with that lower corner, so the
// three components are streamed once between them (three passes, one per
// component, each re-read the other two after L2 had dropped them).
// Neighbour loads go through indices clamped into their array and are
// issued before the boundary tests select them.
template <class F>
__device__ __forceinline__ void predict_body(const RoomDev &R, const PredArgs &A, const double *__restrict__ u,
                                             const double *__restrict__ v, const double *__restrict__ w,
                                             const double *__restrict__ T0, const double *__restrict__ T1,
                                             double *__restrict__ us, double *__restrict__ vs,
                                             double *__restrict__ ws, const StepState *st, int start, int stride)
{
    const int nx = R.nx, ny = R.ny, nz = R.nz;
    const int quick = A.scheme == 1, lw = A.scheme == 2;
    const F dt = F(A.dt), nu = F(A.nu);
    const double *T = st->tpar ? T1 : T0;
    const int pu = ny * nz, lastu = R.nu - 1;
    const int pv = (ny + 1) * nz, lastv = R.nv - 1;
    const int pw = ny * (nz + 1), lastw = R.nw - 1;
    const InvSpacing I(R);
    for (Walk wk(start, stride, ny + 1, nz + 1, (nx + 1) * (ny + 1) * (nz + 1)); wk.ok(); wk.next()) {
        const int i = wk.i, j = wk.j, k = wk.k;
        // spacings of the corner's cell (entries past the last cell of an
        // axis are read only by faces that take no increment)
        const F hx = axis_spacing<F>(R.dxv, I.fx, min(i, nx - 1));
        const F hy = axis_spacing<F>(R.dyv, I.fy, min(j, ny - 1));
        const F hz = axis_spacing<F>(R.dzv, I.fz, min(k, nz - 1));
        if (j < ny && k < nz) {
            const int t = UIX(i, j, k);
            const uint8_t code = R.fcu[t];
            double val = u[t];
            if (i > 0 && i < nx) {
                const double xm0 = u[max(t - pu, 0)], xp0 = u[min(t + pu, lastu)];
                const double ym0 = u[max(t - nz, 0)], yp0 = u[min(t + nz, lastu)];
                const double zm0 = u[max(t - 1, 0)], zp0 = u[min(t + 1, lastu)];
                const double v0 = v[VIX(i - 1, j, k)], v1 = v[VIX(i, j, k)];
                const double w0 = w[WIX(i - 1, j, k)], w1 = w[WIX(i, j, k)];
                double xmm = 0.0, ymm = 0.0, zmm = 0.0;
                if (quick) {
                    xmm = u[max(t - 2 * pu, 0)];
                    ymm = u[max(t - 2 * nz, 0)];
                    zmm = u[max(t - 2, 0)];
                }
                val = pred_u<F>(quick, lw, nx, ny, nz, i, j, k, val, xmm, xm0, xp0, ymm, ym0, yp0, zmm, zm0, zp0,
                                v0, v1, w0, w1, hx, hy, hz, nu, dt);
            }
            us[t] = face_code(code, val, R.fanvel, 0);
        }
        if (i < nx && k < nz) {
            const int f = VIX(i, j, k);
            const uint8_t code = R.fcv[f];
            double val = v[f];
            if (j > 0 && j < ny) {
                const double u0 = u[UIX(i, j - 1, k)], u1 = u[UIX(i, j, k)];
                const double xm0 = v[max(f - pv, 0)], xp0 = v[min(f + pv, lastv)];
                const double ym0 = v[max(f - nz, 0)], yp0 = v[min(f + nz, lastv)];
                const double w0 = w[WIX(i, j - 1, k)], w1 = w[WIX(i, j, k)];
                const double zm0 = v[max(f - 1, 0)], zp0 = v[min(f + 1, lastv)];
                const double ymm = quick ? v[max(f - 2 * nz, 0)] : 0.0;
                val = pred_v<F>(quick, lw, nx, ny, nz, i, j, k, val, xm0, xp0, ymm, ym0, yp0, zm0, zp0, u0, u1, w0,
                                w1, hx, hy, hz, nu, dt);
            }
            vs[f] = face_code(code, val, R.fanvel, 1);
        }
        if (i < nx && j < ny) {
            const int f = WIX(i, j, k);
            const uint8_t code = R.fcw[f];
            double val = w[f];
            if (k > 0 && k < nz) {
                const double u0 = u[UIX(i, j, k - 1)], u1 = u[UIX(i, j, k)];
                const double xm0 = w[max(f - pw, 0)], xp0 = w[min(f + pw, lastw)];
                const double v0 = v[VIX(i, j, k - 1)], v1 = v[VIX(i, j, k)];
                const double ym0 = w[max(f - (nz + 1), 0)], yp0 = w[min(f + (nz + 1), lastw)];
                const double zm0 = w[max(f - 1, 0)], zp0 = w[min(f + 1, lastw)];
                double tb = 0.0, tc = 0.0;
                if (A.buoyancy) {
                    const int c = UIX(i, j, k);
                    tb = T[c - 1];
                    tc = T[c];
                }
                const double zmm = quick ? w[max(f - 2, 0)] : 0.0;
                val = pred_w<F>(A, quick, lw, nx, ny, nz, i, j, k, val, xm0, xp0, ym0, yp0, zmm, zm0, zp0, u0, u1,
                                v0, v1, tb, tc, hx, hy, hz, nu, dt);
            }
            ws[f] = face_code(code, val, R.fanvel, 2);
        }
    }
}

template <class F>
__global__ void __launch_bounds__(256) k_predict(RoomDev R, PredArgs A, const double *__restrict__ u,
                                                 const double *__restrict__ v,
                                                 const double *__restrict__ w,
                                                 const double *__restrict__ T0,
                                                 const double *__restrict__ T1,
                                                 double *__restrict__ us, double *__restrict__ vs,
                                                 double *__restrict__ ws, const StepState *st)
{
    if (st->halt) return;
    predict_body<F>(R, A, u, v, w, T0, T1, us, vs, ws, st, blockIdx.x * blockDim.x + threadIdx.x,
                    gridDim.x * blockDim.x);
}

// ------------------------------------------------------------ pressure

__device__ __forceinline__ void stencil_term(unsigned cls, double s, double xn, double &diag,
                                             double &off)
{
    if (cls == SC_IN) {
        diag += s;
        off += s * xn;
    } else if (cls == SC_DIR) {
        diag += 2.0 * s;
    }
}

// PoissonSolver::solve (PoissonSolver.cpp:93-158) as one cooperative launch.
// Per iteration: phase A forms the direction d = r + beta*d_old (the first
// iteration uses d = r), applies the deferred x += alpha_old*d_old, computes
// Ad with the mask stencil of apply_laplacian (PoissonSolver.cpp:22-91) and
// the block partials of d.Ad; phase B does r -= alpha*Ad and ||r||^2.  Each
// phase ends in a deterministic grid-wide sum.  Stopping rules, the
// |d.Ad| < 1e-30 break and the returned residual follow the reference.
__global__ void __launch_bounds__(256, 4) k_cg(CGArgs A)
{
    __shared__ double sh[32];
    if (A.st && A.st->halt) return;
    const RoomDev &R = A.R;
    const int nx = R.nx, ny = R.ny, nz = R.nz, n = R.n, plane = ny * nz;
    const double *sxl = R.scale, *sxr = sxl + nx, *syl = sxr + nx, *syr = syl + ny, *szl = syr + ny,
                 *szr = szl + nz;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    double *x = A.x, *r = A.r, *ad = A.ad;

    // Phase 0: r = rhs (0 in SOLID rows), d = r, x = 0, ||r||^2.
    double acc[1] = {0.0};
    for (int c = t0; c < n; c += nth) {
        double rv = 0.0;
        if (!(R.sc[c] & SC_SOLID)) {
            if (A.from_faces) {
                const int i = c / plane, rem = c - i * plane, j = rem / nz, k = rem - j * nz;
                const double div = (A.us[UIX(i + 1, j, k)] - A.us[UIX(i, j, k)]) / R.dxv[i]
                                 + (A.vs[VIX(i, j + 1, k)] - A.vs[VIX(i, j, k)]) / R.dyv[j]
                                 + (A.ws[WIX(i, j, k + 1)] - A.ws[WIX(i, j, k)]) / R.dzv[k];
                rv = A.rhs_factor * div;
            } else {
                rv = A.rhs[c];
            }
        }
        r[c] = rv;
        A.da[c] = rv;
        x[c] = 0.0;
        acc[0] += rv * rv;
    }
    bool ok = grid_allreduce<1>(A.gs, A.partials, A.sc->red, acc, sh);
    double rr = acc[0];
    const double bnorm = sqrt(rr);
    int flags = 0, iters = 0;
    double res = 0.0;
    if (!ok) { flags = FFR_FLAG_TIMEOUT; goto finish; }
    if (bnorm < 1e-15) goto finish;
    {
        double *dold = A.da, *dnew = A.db;
        double beta = 0.0, alpha_prev = 0.0, alpha = 0.0;
        bool first = true, pending = false;
        int it = 0;
        for (; it < A.max_iter; it++) {
            double dacc[1] = {0.0};
            // the cells of this thread in the same order as before (so every
            // partial sum is unchanged); coordinates carried by the walk, and
            // every load issued before the stencil code is tested (neighbour
            // indices clamped into the array; a clamped value is only ever
            // used for a neighbour that is an unknown, i.e. inside the room)
            for (Walk w(t0, nth, ny, nz, n); w.ok(); w.next()) {
                const int c = w.c, i = w.i, j = w.j, k = w.k;
                const unsigned code = R.sc[c];
                const int nb[6] = {max(c - plane, 0), min(c + plane, n - 1), max(c - nz, 0), min(c + nz, n - 1),
                                   max(c - 1, 0), min(c + 1, n - 1)};
                const double dp = dold[c];
                double dc, dn[6];
                if (first) {
                    dc = dp;
#pragma unroll
                    for (int q = 0; q < 6; q++) dn[q] = dold[nb[q]];
                } else {
                    dc = fma(beta, dp, r[c]);
#pragma unroll
                    for (int q = 0; q < 6; q++) dn[q] = fma(beta, dold[nb[q]], r[nb[q]]);
                    x[c] = fma(alpha_prev, dp, x[c]);
                    dnew[c] = dc;
                }
                double a;
                if (code & SC_SOLID) {
                    a = dc;
                } else {
                    const double sc6[6] = {sxl[i], sxr[i], syl[j], syr[j], szl[k], szr[k]};
                    double diag = 0.0, off = 0.0;
#pragma unroll
                    for (int q = 0; q < 6; q++) {
                        const unsigned cls = (code >> (2 * q)) & 3u;
                        if (cls) stencil_term(cls, sc6[q], cls == SC_IN ? dn[q] : 0.0, diag, off);
                    }
                    if (diag < 1e-30) diag = 1.0;
                    a = diag * dc - off;
                }
                ad[c] = a;
                dacc[0] += dc * a;
            }
            if (!grid_allreduce<1>(A.gs, A.partials, A.sc->red, dacc, sh)) {
                flags = FFR_FLAG_TIMEOUT;
                goto finish;
            }
            const double dad = dacc[0];
            if (!first) {
                double *tmp = dold; dold = dnew; dnew = tmp;
            }
            first = false;
            pending = false;
            if (fabs(dad) < 1e-30) {
                flags |= FFR_FLAG_CG_BREAKDOWN;
                break;
            }
            alpha = rr / dad;
            double racc[1] = {0.0};
            for (int c = t0; c < n; c += nth) {
                const double rv = r[c] - alpha * ad[c];
                r[c] = rv;
                racc[0] += rv * rv;
            }
            if (!grid_allreduce<1>(A.gs, A.partials, A.sc->red, racc, sh)) {
                flags = FFR_FLAG_TIMEOUT;
                goto finish;
            }
            pending = true;
            const double rr1 = racc[0];
            res = sqrt(rr1) / bnorm;
            if (res < A.tol) {
                iters = it + 1;
                break;
            }
            beta = rr1 / rr;
            rr = rr1;
            alpha_prev = alpha;
        }
        if (it >= A.max_iter || (flags & FFR_FLAG_CG_BREAKDOWN)) {
            iters = A.max_iter;
            res = sqrt(rr) / bnorm;
            if (!(flags & FFR_FLAG_CG_BREAKDOWN)) flags |= FFR_FLAG_CG_MAXITER;
        }
        // dold now holds the direction of the last completed iteration.
        if (pending) {
            const double a_last = (iters == A.max_iter && !(flags & FFR_FLAG_CG_BREAKDOWN) && res >= A.tol)
                                      ? alpha_prev : alpha;
            for (int c = t0; c < n; c += nth) x[c] = fma(a_last, dold[c], x[c]);
        }
    }
finish:
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (A.out_res) *A.out_res = res;
        if (A.out_iters) *A.out_iters = iters;
        if (A.out_flags) *A.out_flags = flags;
        if (A.st) {
            A.st->pres = res;
            A.st->iters = iters;
            atomicOr(&A.st->flags, flags);
        }
    }
}

// --------------------------------------------------------- correction

struct CorrArgs {
    double c0;        // dt / rho
};

// Cell-centric pressure correction (FluidSolver::apply_correction,
// FluidSolver.cpp:332-371) followed by the BC appliers (FluidSolver.cpp:
// 512-515) expressed through the face codes.  A thread owns the three low
// faces of its cell (and the high boundary faces of the last cells) and
// recomputes the three high faces, so it can also fold max |u_new - u_old|
// (FluidSolver.cpp:527-534) and, for FLUID cells, |div u|
// (compute_divergence_max, FluidSolver.cpp:470-484) in the same pass.
template <bool PAIRS>
__device__ __forceinline__ void correct_body(const RoomDev &R, const CorrArgs &A, double *__restrict__ u,
                                             double *__restrict__ v, double *__restrict__ w,
                                             const double *__restrict__ us, const double *__restrict__ vs,
                                             const double *__restrict__ ws, const double *__restrict__ p,
                                             StepState *st, int start, int stride)
{
    __shared__ double sh[32];
    const int nx = R.nx, ny = R.ny, nz = R.nz, plane = ny * nz;
    const double c0 = A.c0;
    double dmax = 0.0, divmax = 0.0;
    int nan = 0;
    const int last = R.n - 1;
    const InvSpacing I(R);
    // One face along an axis: the correction where the face is interior
    // (lo/hi flags), then its code.  The same arithmetic for every face
    // whichever cell forms it, so a face two cells share comes out the same.
    auto xface = [&](double f, bool interior, double pd, double rc) {
        return interior ? f - c0 * (pd * rc) : f;
    };
    if constexpr (PAIRS) {
        // Even rows (PAIRS needs nz even): the cells (i, j, k0) and
        // (i, j, k0 + 1) of a pair.  The
        // pressure, the x and y face arrays and the codes hold both at an
        // even index, so each pair of values moves with one 16-byte (2-byte
        // for codes) load or store; the z face between the two cells is
        // formed once (an interior face carries no outflow copy, so both
        // cells would form it alike).  A neighbour pair outside the grid is
        // clamped to a pair inside it and not used, as in the general loop.
        const int pk = nz >> 1;
        for (Walk wk(start, stride, ny, pk, nx * ny * pk); wk.ok(); wk.next()) {
            const int i = wk.i, j = wk.j, k0 = 2 * wk.k;
            const int c = (i * ny + j) * nz + k0;
            const double2 pc = *reinterpret_cast<const double2 *>(p + c);
            const double2 pxm = *reinterpret_cast<const double2 *>(p + max(c - plane, 0));
            const double2 pxp = *reinterpret_cast<const double2 *>(p + min(c + plane, last - 1));
            const double2 pym = *reinterpret_cast<const double2 *>(p + max(c - nz, 0));
            const double2 pyp = *reinterpret_cast<const double2 *>(p + min(c + nz, last - 1));
            const double pzm = p[max(c - 1, 0)], pzp = p[min(c + 2, last)];
            const int vl = VIX(i, j, k0), wl = WIX(i, j, k0);
            const double2 usl = *reinterpret_cast<const double2 *>(us + c);
            const double2 ush = *reinterpret_cast<const double2 *>(us + c + plane);
            const double2 vsl = *reinterpret_cast<const double2 *>(vs + vl);
            const double2 vsh = *reinterpret_cast<const double2 *>(vs + vl + nz);
            const double ws0 = ws[wl], ws1 = ws[wl + 1], ws2 = ws[wl + 2];
            const uchar2 cul = *reinterpret_cast<const uchar2 *>(R.fcu + c);
            const uchar2 cuh = *reinterpret_cast<const uchar2 *>(R.fcu + c + plane);
            const uchar2 cvl = *reinterpret_cast<const uchar2 *>(R.fcv + vl);
            const uchar2 cvh = *reinterpret_cast<const uchar2 *>(R.fcv + vl + nz);
            const uint8_t cw0 = R.fcw[wl], cw1 = R.fcw[wl + 1], cw2 = R.fcw[wl + 2];
            const double2 uo = *reinterpret_cast<const double2 *>(u + c);
            const double2 vo = *reinterpret_cast<const double2 *>(v + vl);
            const double wo0 = w[wl], wo1 = w[wl + 1];
            const uchar2 ctp = *reinterpret_cast<const uchar2 *>(R.ct + c);
            const double rxl = I.cx[i], rxh = I.cx[min(i + 1, nx - 1)];
            const double ryl = I.cy[j], ryh = I.cy[min(j + 1, ny - 1)];
            const bool xl = i >= 1, xh = i + 1 <= nx - 1, yl = j >= 1, yh = j + 1 <= ny - 1;
            // faces of one cell along x or y: corrected, coded, outflow copies
            auto pair_faces = [&](double lo, double hi, uint8_t cl, uint8_t ch, bool il, bool ih, double pdl,
                                  double pdh, double rl, double rh, int comp, double &flo, double &fhi) {
                lo = face_code(cl, xface(lo, il, pdl, rl), R.fanvel, comp);
                hi = face_code(ch, xface(hi, ih, pdh, rh), R.fanvel, comp);
                if (cl & FC_OUTCOPY) lo = hi;
                if (ch & FC_OUTCOPY) hi = lo;
                flo = lo;
                fhi = hi;
            };
            double ulo0, uhi0, ulo1, uhi1, vlo0, vhi0, vlo1, vhi1;
            pair_faces(usl.x, ush.x, cul.x, cuh.x, xl, xh, pc.x - pxm.x, pxp.x - pc.x, rxl, rxh, 0, ulo0, uhi0);
            pair_faces(usl.y, ush.y, cul.y, cuh.y, xl, xh, pc.y - pxm.y, pxp.y - pc.y, rxl, rxh, 0, ulo1, uhi1);
            pair_faces(vsl.x, vsh.x, cvl.x, cvh.x, yl, yh, pc.x - pym.x, pyp.x - pc.x, ryl, ryh, 1, vlo0, vhi0);
            pair_faces(vsl.y, vsh.y, cvl.y, cvh.y, yl, yh, pc.y - pym.y, pyp.y - pc.y, ryl, ryh, 1, vlo1, vhi1);
            // z faces k0, k0 + 1 (shared, always interior), k0 + 2
            const double f0 = face_code(cw0, xface(ws0, k0 >= 1, pc.x - pzm, I.cz[k0]), R.fanvel, 2);
            const double f1 = face_code(cw1, xface(ws1, true, pc.y - pc.x, I.cz[k0 + 1]), R.fanvel, 2);
            const double f2 = face_code(cw2, xface(ws2, k0 + 2 <= nz - 1, pzp - pc.y, I.cz[min(k0 + 2, nz - 1)]),
                                        R.fanvel, 2);
            double wlo0 = f0, whi0 = f1, wlo1 = f1, whi1 = f2;
            if (cw0 & FC_OUTCOPY) wlo0 = whi0;
            if (cw1 & FC_OUTCOPY) whi0 = wlo0;
            if (cw1 & FC_OUTCOPY) wlo1 = whi1;
            if (cw2 & FC_OUTCOPY) whi1 = wlo1;
            dmax = fmax(dmax, fmax(fabs(ulo0 - uo.x), fabs(ulo1 - uo.y)));
            dmax = fmax(dmax, fmax(fabs(vlo0 - vo.x), fabs(vlo1 - vo.y)));
            dmax = fmax(dmax, fmax(fabs(wlo0 - wo0), fabs(wlo1 - wo1)));
            *reinterpret_cast<double2 *>(u + c) = make_double2(ulo0, ulo1);
            *reinterpret_cast<double2 *>(v + vl) = make_double2(vlo0, vlo1);
            w[wl] = wlo0;
            w[wl + 1] = wlo1;
            if (i == nx - 1) {
                const double2 o = *reinterpret_cast<const double2 *>(u + c + plane);
                dmax = fmax(dmax, fmax(fabs(uhi0 - o.x), fabs(uhi1 - o.y)));
                *reinterpret_cast<double2 *>(u + c + plane) = make_double2(uhi0, uhi1);
            }
            if (j == ny - 1) {
                const double2 o = *reinterpret_cast<const double2 *>(v + vl + nz);
                dmax = fmax(dmax, fmax(fabs(vhi0 - o.x), fabs(vhi1 - o.y)));
                *reinterpret_cast<double2 *>(v + vl + nz) = make_double2(vhi0, vhi1);
            }
            if (k0 + 2 == nz) {
                dmax = fmax(dmax, fabs(whi1 - w[wl + 2]));
                w[wl + 2] = whi1;
            }
            if (isnan(ulo0) || isnan(uhi0) || isnan(vlo0) || isnan(vhi0) || isnan(wlo0) || isnan(whi0) ||
                isnan(ulo1) || isnan(uhi1) || isnan(vlo1) || isnan(vhi1) || isnan(wlo1) || isnan(whi1))
                nan = 1;
            const double rwx = I.wx[i], rwy = I.wy[j];
            if (ctp.x == CT_FLUID)
                divmax = fmax(divmax, fabs((uhi0 - ulo0) * rwx + (vhi0 - vlo0) * rwy + (whi0 - wlo0) * I.wz[k0]));
            if (ctp.y == CT_FLUID)
                divmax = fmax(divmax, fabs((uhi1 - ulo1) * rwx + (vhi1 - vlo1) * rwy + (whi1 - wlo1) * I.wz[k0 + 1]));
        }
    } else {
        // Any row length: one cell per work item.  The spacing factors are
        // formed by division as the reference forms them (the reciprocal
        // tables measured several times slower in this loop).
        for (Walk wk(start, stride, ny, nz, R.n); wk.ok(); wk.next()) {
            const int c = wk.c, i = wk.i, j = wk.j, k = wk.k;
            // the pressure stencil and the old low faces, loaded before any test
            const double pc = p[c];
            const double pxm = p[max(c - plane, 0)], pxp = p[min(c + plane, last)];
            const double pym = p[max(c - nz, 0)], pyp = p[min(c + nz, last)];
            const double pzm = p[max(c - 1, 0)], pzp = p[min(c + 1, last)];
            // x faces
            const int ul = c, uh = c + plane;
            double lo = us[ul], hi = us[uh];
            if (i >= 1) lo = lo - c0 * ((pc - pxm) / (0.5 * (R.dxv[i - 1] + R.dxv[i])));
            if (i + 1 <= nx - 1) hi = hi - c0 * ((pxp - pc) / (0.5 * (R.dxv[i] + R.dxv[i + 1])));
            uint8_t cl = R.fcu[ul], ch = R.fcu[uh];
            lo = face_code(cl, lo, R.fanvel, 0);
            hi = face_code(ch, hi, R.fanvel, 0);
            if (cl & FC_OUTCOPY) lo = hi;
            if (ch & FC_OUTCOPY) hi = lo;
            const double ulo = lo, uhi = hi;
            dmax = fmax(dmax, fabs(lo - u[ul]));
            u[ul] = lo;
            if (i == nx - 1) {
                dmax = fmax(dmax, fabs(hi - u[uh]));
                u[uh] = hi;
            }
            // y faces
            const int vl = VIX(i, j, k), vh = vl + nz;
            lo = vs[vl]; hi = vs[vh];
            if (j >= 1) lo = lo - c0 * ((pc - pym) / (0.5 * (R.dyv[j - 1] + R.dyv[j])));
            if (j + 1 <= ny - 1) hi = hi - c0 * ((pyp - pc) / (0.5 * (R.dyv[j] + R.dyv[j + 1])));
            cl = R.fcv[vl]; ch = R.fcv[vh];
            lo = face_code(cl, lo, R.fanvel, 1);
            hi = face_code(ch, hi, R.fanvel, 1);
            if (cl & FC_OUTCOPY) lo = hi;
            if (ch & FC_OUTCOPY) hi = lo;
            const double vlo = lo, vhi = hi;
            dmax = fmax(dmax, fabs(lo - v[vl]));
            v[vl] = lo;
            if (j == ny - 1) {
                dmax = fmax(dmax, fabs(hi - v[vh]));
                v[vh] = hi;
            }
            // z faces
            const int wl = WIX(i, j, k), wh = wl + 1;
            lo = ws[wl]; hi = ws[wh];
            if (k >= 1) lo = lo - c0 * ((pc - pzm) / (0.5 * (R.dzv[k - 1] + R.dzv[k])));
            if (k + 1 <= nz - 1) hi = hi - c0 * ((pzp - pc) / (0.5 * (R.dzv[k] + R.dzv[k + 1])));
            cl = R.fcw[wl]; ch = R.fcw[wh];
            lo = face_code(cl, lo, R.fanvel, 2);
            hi = face_code(ch, hi, R.fanvel, 2);
            if (cl & FC_OUTCOPY) lo = hi;
            if (ch & FC_OUTCOPY) hi = lo;
            const double wlo = lo, whi = hi;
            dmax = fmax(dmax, fabs(lo - w[wl]));
            w[wl] = lo;
            if (k == nz - 1) {
                dmax = fmax(dmax, fabs(hi - w[wh]));
                w[wh] = hi;
            }
            if (isnan(ulo) || isnan(uhi) || isnan(vlo) || isnan(vhi) || isnan(wlo) || isnan(whi)) nan = 1;
            if (R.ct[c] == CT_FLUID) {
                const double d = fabs((uhi - ulo) / R.dxv[i] + (vhi - vlo) / R.dyv[j] + (whi - wlo) / R.dzv[k]);
                divmax = fmax(divmax, d);
            }
        }
    }
    dmax = block_max(dmax, sh);
    divmax = block_max(divmax, sh);
    nan = __syncthreads_or(nan);
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&st->dmax_bits, dmax);
        atomic_max_nonneg(&st->div_bits, divmax);
        if (nan) atomicOr(&st->flags, FFR_FLAG_NAN);
    }
}

template <bool PAIRS>
__global__ void __launch_bounds__(256) k_correct(RoomDev R, CorrArgs A, double *__restrict__ u,
                                                 double *__restrict__ v, double *__restrict__ w,
                                                 const double *__restrict__ us,
                                                 const double *__restrict__ vs,
                                                 const double *__restrict__ ws,
                                                 const double *__restrict__ p, StepState *st)
{
    if (st->halt) return;
    correct_body<PAIRS>(R, A, u, v, w, us, vs, ws, p, st, blockIdx.x * blockDim.x + threadIdx.x,
                        gridDim.x * blockDim.x);
}

// compute_divergence_max (FluidSolver.cpp:470-484) on demand.
__global__ void k_divergence(RoomDev R, const double *u, const double *v, const double *w,
                             unsigned long long *out)
{
    __shared__ double sh[32];
    const int nx = R.nx, ny = R.ny, nz = R.nz, plane = ny * nz;
    (void)nx;
    double m = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < R.n; c += gridDim.x * blockDim.x) {
        if (R.ct[c] != CT_FLUID) continue;
        const int i = c / plane, rem = c - i * plane, j = rem / nz, k = rem - j * nz;
        const double d = fabs((u[c + plane] - u[c]) / R.dxv[i]
                              + (v[VIX(i, j + 1, k)] - v[VIX(i, j, k)]) / R.dyv[j]
                              + (w[WIX(i, j, k + 1)] - w[WIX(i, j, k)]) / R.dzv[k]);
        m = fmax(m, d);
    }
    m = block_max(m, sh);
    if (threadIdx.x == 0) atomic_max_nonneg(out, m);
}

// ------------------------------------------------------------ thermal

// BoundaryManager::apply_opening_temperature (BoundaryManager.cpp:137-178)
// for one opening patch; `next` picks the T buffer the step is writing.
__device__ __forceinline__ void opening_body(const RoomDev &R, const ffr_patch &P, const double *u,
                                             const double *v, const double *w, double *T0, double *T1,
                                             const StepState *st, int next, int start, int stride)
{
    const int nx = R.nx, ny = R.ny, nz = R.nz;
    double *T = ((st ? st->tpar : 0) ^ next) ? T1 : T0;
    const int na = P.a_max - P.a_min + 1, nb = P.b_max - P.b_min + 1;
    const int sd = P.side;
    for (int t = start; t < na * nb; t += stride) {
        const int a = P.a_min + t / nb, b = P.b_min + t % nb;
        double vf;
        int cw, cin;
        if (P.axis == 0) {
            vf = u[UIX(sd ? nx : 0, a, b)];
            cw = UIX(sd ? nx - 1 : 0, a, b);
            cin = UIX(sd ? nx - 2 : 1, a, b);
        } else if (P.axis == 1) {
            vf = v[VIX(a, sd ? ny : 0, b)];
            cw = UIX(a, sd ? ny - 1 : 0, b);
            cin = UIX(a, sd ? ny - 2 : 1, b);
        } else {
            vf = w[WIX(a, b, sd ? nz : 0)];
            cw = UIX(a, b, sd ? nz - 1 : 0);
            cin = UIX(a, b, sd ? nz - 2 : 1);
        }
        const bool incoming = sd ? (vf <= 0.0) : (vf >= 0.0);
        T[cw] = incoming ? P.T_outside : T[cin];
    }
}

__global__ void k_opening_T(RoomDev R, ffr_patch P, const double *u, const double *v,
                            const double *w, double *T0, double *T1, const StepState *st, int next)
{
    if (st && st->halt) return;
    opening_body(R, P, u, v, w, T0, T1, st, next, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

struct ThermArgs {
    double dt, alpha;
    int scheme;
};

// The new temperature of one FLUID cell (FluidSolver::advect_temperature,
// FluidSolver.cpp:388-456) from its value tc, its six neighbours' types and
// values in the order x-, x+, y-, y+, z-, z+ and its six face velocities.
// F as for k_predict.
template <class F>
__device__ __forceinline__ double temp_cell(const RoomDev &R, const ThermArgs &A, const InvSpacing &I,
                                            const double *T, int i, int j, int k, double tc, const uint8_t (&nct)[6],
                                            const double (&nT)[6], double u0, double u1, double v0, double v1,
                                            double w0, double w1)
{
    const int nx = R.nx, ny = R.ny, nz = R.nz;
    const int quick = A.scheme == 1, lw = A.scheme == 2;
    const double ac = 0.5 * (u0 + u1);
    const double bc = 0.5 * (v0 + v1);
    const double cc = 0.5 * (w0 + w1);
    // Neumann at the domain edge and at SOLID cells (FluidSolver.cpp:417-422)
    const bool inside[6] = {i > 0, i < nx - 1, j > 0, j < ny - 1, k > 0, k < nz - 1};
    double tn6[6];
#pragma unroll
    for (int a = 0; a < 6; a++) tn6[a] = (inside[a] && nct[a] != CT_SOLID) ? nT[a] : tc;
    auto tat = [&](int ii, int jj, int kk) -> double {
        if (ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) return tc;
        const int qq = UIX(ii, jj, kk);
        return R.ct[qq] == CT_SOLID ? tc : T[qq];
    };
    const double xm = tn6[0], xp = tn6[1];
    const double ym = tn6[2], yp = tn6[3];
    const double zm = tn6[4], zp = tn6[5];
    const int q = quick && i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2;
    const double xmm = q ? tat(i - 2, j, k) : 0.0, ymm = q ? tat(i, j - 2, k) : 0.0,
                 zmm = q ? tat(i, j, k - 2) : 0.0;
    const F hx = axis_spacing<F>(R.dxv, I.fx, i), hy = axis_spacing<F>(R.dyv, I.fy, j),
            hz = axis_spacing<F>(R.dzv, I.fz, k), dt = F(A.dt);
    F adv, dif;
    const F ftc = F(tc);
    if constexpr (sizeof(F) == 4) {
        // mixed precision: reciprocal spacings in place of the divisions
        const F ix = hx, iy = hy, iz = hz;
        if (q) {
            adv = adv_quick_r(F(xmm), F(xm), ftc, F(xp), F(ac), ix) +
                  adv_quick_r(F(ymm), F(ym), ftc, F(yp), F(bc), iy) +
                  adv_quick_r(F(zmm), F(zm), ftc, F(zp), F(cc), iz);
        } else if (lw) {
            adv = adv_lw_r(F(xm), ftc, F(xp), F(ac), dt, ix) + adv_lw_r(F(ym), ftc, F(yp), F(bc), dt, iy) +
                  adv_lw_r(F(zm), ftc, F(zp), F(cc), dt, iz);
        } else {
            adv = adv_up_r(F(xm), ftc, F(xp), F(ac), ix) + adv_up_r(F(ym), ftc, F(yp), F(bc), iy) +
                  adv_up_r(F(zm), ftc, F(zp), F(cc), iz);
        }
        dif = F(A.alpha) * ((F(xm) - F(2) * ftc + F(xp)) * (ix * ix) + (F(ym) - F(2) * ftc + F(yp)) * (iy * iy) +
                            (F(zm) - F(2) * ftc + F(zp)) * (iz * iz));
    } else {
        if (q) {
            adv = adv_quick(F(xmm), F(xm), F(tc), F(xp), F(ac), hx) +
                  adv_quick(F(ymm), F(ym), F(tc), F(yp), F(bc), hy) +
                  adv_quick(F(zmm), F(zm), F(tc), F(zp), F(cc), hz);
        } else if (lw) {
            adv = adv_lw(F(xm), F(tc), F(xp), F(ac), dt, hx) + adv_lw(F(ym), F(tc), F(yp), F(bc), dt, hy) +
                  adv_lw(F(zm), F(tc), F(zp), F(cc), dt, hz);
        } else {
            adv = adv_up(F(xm), F(tc), F(xp), F(ac), hx) + adv_up(F(ym), F(tc), F(yp), F(bc), hy) +
                  adv_up(F(zm), F(tc), F(zp), F(cc), hz);
        }
        dif = F(A.alpha) * ((F(xm) - F(2) * ftc + F(xp)) / (hx * hx) + (F(ym) - F(2) * ftc + F(yp)) / (hy * hy) +
                            (F(zm) - F(2) * ftc + F(zp)) / (hz * hz));
    }
    return tc + (double)(dt * (-adv + dif));
}

// FluidSolver::advect_temperature (FluidSolver.cpp:388-456) with the block
// partial sums of the new T over FLUID cells for compute_T_mean
// (FluidSolver.cpp:458-468).  F as for k_predict.
// tpart[lblock] receives this block's partial sum.
template <class F>
__device__ __forceinline__ void advect_T_body(const RoomDev &R, const ThermArgs &A, const double *__restrict__ u,
                                              const double *__restrict__ v, const double *__restrict__ w,
                                              double *T0, double *T1, double *tpart, const StepState *st,
                                              int start, int stride, int lblock)
{
    __shared__ double sh[32];
    const int ny = R.ny, nz = R.nz, plane = ny * nz;
    const double *T = st->tpar ? T1 : T0;
    double *Tn = st->tpar ? T0 : T1;
    double sum = 0.0;
    const int last = R.n - 1;
    const InvSpacing I(R);
    for (Walk wk(start, stride, ny, nz, R.n); wk.ok(); wk.next()) {
        const int c = wk.c, i = wk.i, j = wk.j, k = wk.k;
        const uint8_t tcell = R.ct[c];
        const double tc = T[c];
        // the six neighbours' types and temperatures and the face velocities,
        // loaded before any test (indices clamped into the arrays)
        const int nb[6] = {max(c - plane, 0), min(c + plane, last), max(c - nz, 0),
                           min(c + nz, last), max(c - 1, 0), min(c + 1, last)};
        uint8_t nct[6];
        double nT[6];
#pragma unroll
        for (int a = 0; a < 6; a++) {
            nct[a] = R.ct[nb[a]];
            nT[a] = T[nb[a]];
        }
        const double u0 = u[c], u1 = u[c + plane];
        const double v0 = v[VIX(i, j, k)], v1 = v[VIX(i, j + 1, k)];
        const double w0 = w[WIX(i, j, k)], w1 = w[WIX(i, j, k + 1)];
        if (tcell != CT_FLUID) {
            Tn[c] = tc;
            continue;
        }
        const double tn = temp_cell<F>(R, A, I, T, i, j, k, tc, nct, nT, u0, u1, v0, v1, w0, w1);
        Tn[c] = tn;
        sum += tn;
    }
    sum = block_sum(sum, sh);
    if (threadIdx.x == 0) tpart[lblock] = sum;
}

template <class F>
__global__ void __launch_bounds__(256) k_advect_T(RoomDev R, ThermArgs A, const double *__restrict__ u,
                                                  const double *__restrict__ v,
                                                  const double *__restrict__ w, double *T0,
                                                  double *T1, double *tpart, const StepState *st)
{
    if (st->halt) return;
    advect_T_body<F>(R, A, u, v, w, T0, T1, tpart, st, blockIdx.x * blockDim.x + threadIdx.x,
                     gridDim.x * blockDim.x, blockIdx.x);
}

// Fixed-temperature box (heat-patch extension) on the buffer that is
// current once the step completes.
__device__ __forceinline__ void heat_body(const RoomDev &R, const ffr_heat_patch &H, double *T0, double *T1,
                                          const StepState *st, int next, int start, int stride)
{
    const int ny = R.ny, nz = R.nz;
    double *T = (st->tpar ^ next) ? T1 : T0;
    const int i0 = max(0, H.i_min), i1 = min(R.nx - 1, H.i_max);
    const int j0 = max(0, H.j_min), j1 = min(ny - 1, H.j_max);
    const int k0 = max(0, H.k_min), k1 = min(nz - 1, H.k_max);
    if (i0 > i1 || j0 > j1 || k0 > k1) return;
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
    for (int t = start; t < ni * nj * nk; t += stride) {
        const int a = t / (nj * nk), rem = t - a * nj * nk, b = rem / nk, e = rem - b * nk;
        T[UIX(i0 + a, j0 + b, k0 + e)] = H.T;
    }
}

__global__ void k_heat(RoomDev R, ffr_heat_patch H, double *T0, double *T1, const StepState *st,
                       int next)
{
    if (st->halt) return;
    heat_body(R, H, T0, T1, st, next, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// T := T_initial on every cell (FluidSolver ctor, FluidSolver.cpp:28).
__global__ void k_fill(double *x, int n, double val)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) x[c] = val;
}

struct FinArgs {
    double dt, convergence_tol, T_initial, T_target;
    int thermal;
    long long n_fluid;
    int tblocks;
};

// StepResult and convergence test of FluidSolver::step (FluidSolver.cpp:
// 526-549); the velocity change max and divergence max were folded by
// k_correct, the pressure residual by k_cg, the T partials by k_advect_T.
__device__ __forceinline__ void finalize_body(const FinArgs &A, const double *tpart, StepState *st,
                                              ffr_step_result *ring)
{
    __shared__ double sh[32];
    double tmean = A.T_initial;
    if (A.thermal) {
        double s = 0.0;
        for (int b = threadIdx.x; b < A.tblocks; b += blockDim.x) s += tpart[b];
        s = block_sum(s, sh);
        tmean = A.n_fluid > 0 ? s / (double)A.n_fluid : A.T_initial;
    }
    if (threadIdx.x != 0) return;
    const double vc = __longlong_as_double((long long)st->dmax_bits) / A.dt;
    const double dv = __longlong_as_double((long long)st->div_bits);
    int conv;
    if (A.thermal && A.T_target < 1e29)
        conv = (A.T_target >= A.T_initial) ? (tmean >= A.T_target) : (tmean <= A.T_target);
    else
        conv = vc < A.convergence_tol;
    ffr_step_result r;
    r.step = st->step + 1;
    r.velocity_change = vc;
    r.pressure_residual = st->pres;
    r.divergence_max = dv;
    r.converged = conv;
    r.T_mean = tmean;
    r.cg_iterations = st->iters;
    r.flags = st->flags;
    ring[st->ring_slot] = r;
    st->ring_slot += 1;
    st->step += 1;
    if (A.thermal) st->tpar ^= 1;
    st->dmax_bits = 0;
    st->div_bits = 0;
    st->flags = 0;
    if (conv && st->stop_on_converge) st->halt = 1;
}

__global__ void k_finalize(FinArgs A, const double *tpart, StepState *st, ffr_step_result *ring)
{
    if (st->halt) return;
    finalize_body(A, tpart, st, ring);
}

// Start of a queued chunk of steps: results go to slot 0 on, the halt
// flag of an earlier converged chunk is cleared.
__global__ void k_begin_chunk(StepState *st, int stop_on_converge)
{
    st->ring_slot = 0;
    st->halt = 0;
    st->stop_on_converge = stop_on_converge;
}

// Cell-centred velocity (face averages) and speed, the snapshot of
// SolverBridge.run_animated (solver_bridge.py:222-238), on the device.
__global__ void __launch_bounds__(256) k_snapshot(RoomDev R, const double *__restrict__ u,
                                                  const double *__restrict__ v, const double *__restrict__ w,
                                                  double *__restrict__ uc, double *__restrict__ vc,
                                                  double *__restrict__ wc, double *__restrict__ speed)
{
    const int ny = R.ny, nz = R.nz, plane = ny * nz;
    for (Walk wk(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, ny, nz, R.n); wk.ok(); wk.next()) {
        const int c = wk.c, i = wk.i, j = wk.j, k = wk.k;
        const double a = 0.5 * (u[c] + u[c + plane]);
        const double b = 0.5 * (v[VIX(i, j, k)] + v[VIX(i, j + 1, k)]);
        const double e = 0.5 * (w[WIX(i, j, k)] + w[WIX(i, j, k + 1)]);
        uc[c] = a;
        vc[c] = b;
        wc[c] = e;
        speed[c] = sqrt(a * a + b * b + e * e);
    }
}

// ---------------------------------------------------------- batched rooms
//
// One launch per stage advances every room of a batch.  Block b works on
// room m.room[b] with the position it would have in that room's own launch
// (the same block count per room), so each room's arithmetic, including
// the order of every partial sum, is the one its own launches perform.

// Everything the step kernels need about one room (a device array, one
// entry per room of the batch).
struct BRoom {
    RoomDev R;
    PredArgs pa;
    CorrArgs co;
    ThermArgs ta;
    FinArgs fa;
    double *u, *v, *w, *us, *vs, *ws, *p, *T0, *T1, *tpart;
    StepState *st;
    ffr_step_result *ring;
    int mixed, thermal;
};

// An opening or heat patch of one room (one launch item).
struct OpenItem {
    int room, pad;
    ffr_patch P;
};
struct HeatItem {
    int room, pad;
    ffr_heat_patch H;
};

template <class T>
__device__ __forceinline__ void load_shared(T &dst, const T *src)
{
    static_assert(sizeof(T) % 8 == 0, "8-byte words");
    const unsigned long long *a = reinterpret_cast<const unsigned long long *>(src);
    unsigned long long *d = reinterpret_cast<unsigned long long *>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(T) / 8); i += blockDim.x) d[i] = a[i];
    __syncthreads();
}

__global__ void k_b_begin(const BRoom *rooms, int n, int stop_on_converge)
{
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        StepState *st = rooms[r].st;
        st->ring_slot = 0;
        st->halt = 0;
        st->stop_on_converge = stop_on_converge;
    }
}

__global__ void __launch_bounds__(256) k_b_predict(const BRoom *rooms, BMap m)
{
    __shared__ __align__(16) BRoom B;
    BPos P;
    const int r = bmap(m, P);
    load_shared(B, rooms + r);
    if (B.st->halt) return;
    const int start = P.lb * blockDim.x + threadIdx.x, stride = P.nb * blockDim.x;
    if (B.mixed)
        predict_body<float>(B.R, B.pa, B.u, B.v, B.w, B.T0, B.T1, B.us, B.vs, B.ws, B.st, start, stride);
    else
        predict_body<double>(B.R, B.pa, B.u, B.v, B.w, B.T0, B.T1, B.us, B.vs, B.ws, B.st, start, stride);
}

__global__ void __launch_bounds__(256, 2) k_b_correct(const BRoom *rooms, BMap m)
{
    __shared__ __align__(16) BRoom B;
    BPos P;
    const int r = bmap(m, P);
    load_shared(B, rooms + r);
    if (B.st->halt) return;
    // the form the room's own launch takes (bit-identical results)
    if ((B.R.nz & 1) == 0)
        correct_body<true>(B.R, B.co, B.u, B.v, B.w, B.us, B.vs, B.ws, B.p, B.st, P.lb * blockDim.x + threadIdx.x,
                           P.nb * blockDim.x);
    else
        correct_body<false>(B.R, B.co, B.u, B.v, B.w, B.us, B.vs, B.ws, B.p, B.st, P.lb * blockDim.x + threadIdx.x,
                            P.nb * blockDim.x);
}

__global__ void k_b_opening(const BRoom *rooms, const OpenItem *items, BMap m, int next)
{
    __shared__ __align__(16) BRoom B;
    BPos P;
    const int it = bmap(m, P);
    const OpenItem I = items[it];
    load_shared(B, rooms + I.room);
    if (B.st->halt) return;
    opening_body(B.R, I.P, B.u, B.v, B.w, B.T0, B.T1, B.st, next, P.lb * blockDim.x + threadIdx.x,
                 P.nb * blockDim.x);
}

__global__ void __launch_bounds__(256) k_b_advect_T(const BRoom *rooms, BMap m)
{
    __shared__ __align__(16) BRoom B;
    BPos P;
    const int r = bmap(m, P);
    load_shared(B, rooms + r);
    if (B.st->halt || !B.thermal) return;
    const int start = P.lb * blockDim.x + threadIdx.x, stride = P.nb * blockDim.x;
    if (B.mixed)
        advect_T_body<float>(B.R, B.ta, B.u, B.v, B.w, B.T0, B.T1, B.tpart, B.st, start, stride, P.lb);
    else
        advect_T_body<double>(B.R, B.ta, B.u, B.v, B.w, B.T0, B.T1, B.tpart, B.st, start, stride, P.lb);
}

__global__ void k_b_heat(const BRoom *rooms, const HeatItem *items, BMap m)
{
    __shared__ __align__(16) BRoom B;
    BPos P;
    const int it = bmap(m, P);
    const HeatItem I = items[it];
    load_shared(B, rooms + I.room);
    if (B.st->halt) return;
    heat_body(B.R, I.H, B.T0, B.T1, B.st, B.thermal, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x);
}

// one block per room
__global__ void k_b_finalize(const BRoom *rooms)
{
    __shared__ __align__(16) BRoom B;
    load_shared(B, rooms + blockIdx.x);
    if (B.st->halt) return;
    finalize_body(B.fa, B.tpart, B.st, B.ring);
}

#undef UIX
#undef VIX
#undef WIX

// Self-test of the bounded device waits: every block but block 0 enters the
// library's grid reduction, which block 0 never joins, so nothing releases
// it; each waiting block gives up after the wait limit, records
// FFR_FLAG_TIMEOUT and returns.  No wait is unbounded and no access leaves
// the buffers (partials holds gridDim.x values).
__global__ void k_wait_selftest(GridSync *gs, double *partials, double *out, int *flags)
{
    __shared__ double sh[32];
    if (blockIdx.x == 0) return;
    double v[1] = {1.0};
    if (!grid_allreduce<1>(gs, partials, out, v, sh) && threadIdx.x == 0) atomicOr(flags, FFR_FLAG_TIMEOUT);
}

FFR_DEFINE_WAIT_LIMIT_SETTER(set_wait_limit_projection)

}  // namespace ffr

// =================================================================== host

using namespace ffr;

extern "C" int ffr_set_device_wait_limit(double seconds)
{
    if (!(seconds >= 0.0) || seconds > 60.0) return fail(FFR_EINVAL, "wait limit must be in [0, 60] s");
    const unsigned long long ns =
        seconds == 0.0 ? kBarrierTimeoutNs : (unsigned long long)(seconds * 1e9 + 0.5);
    int rc = set_wait_limit_projection(ns);
    if (!rc) rc = set_wait_limit_mgpcg(ns);
    return rc;
}

extern "C" int ffr_selftest_device_wait(int blocks, double *elapsed_ms)
{
    if (blocks < 2 || blocks > 64) return fail(FFR_EINVAL, "blocks must be in [2, 64]");
    cudaStream_t st = nullptr;
    FFR_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const size_t bytes = 256 + 8 * 64 + 256 + 256;
    unsigned char *buf = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&buf, bytes, st);
    if (e != cudaSuccess) { cudaStreamDestroy(st); return cuda_fail(e, "cudaMallocAsync(self-test)"); }
    GridSync *gs = reinterpret_cast<GridSync *>(buf);
    double *partials = reinterpret_cast<double *>(buf + 256);
    double *out = reinterpret_cast<double *>(buf + 256 + 8 * 64);
    int *flags = reinterpret_cast<int *>(buf + 256 + 8 * 64 + 256);
    int host_flags = 0;
    cudaEvent_t ev[2];
    cudaEventCreate(&ev[0]);
    cudaEventCreate(&ev[1]);
    e = cudaMemsetAsync(buf, 0, bytes, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], st);
    if (e == cudaSuccess) {
        k_wait_selftest<<<blocks, 128, 0, st>>>(gs, partials, out, flags);
        e = cudaGetLastError();
        count_launch(1);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev[1], st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host_flags, flags, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float ms = 0.0f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, ev[0], ev[1]);
    cudaFreeAsync(buf, st);
    cudaStreamSynchronize(st);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return cuda_fail(e, "device wait self-test");
    if (elapsed_ms) *elapsed_ms = ms;
    if (host_flags & FFR_FLAG_TIMEOUT) return fail(FFR_ETIMEDOUT, "self-test wait gave up at the wait limit");
    return FFR_OK;
}

namespace {

constexpr int kRing = 1024;
constexpr int kThreads = 256;

int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// Grid of a streaming kernel: four items per thread, at most 8 blocks per
// SM (many rooms in one batched launch fill the GPU by their number).
unsigned stream_blocks(long long work)
{
    const long long cap = (long long)sm_count() * 8;
    return (unsigned)std::max<long long>(1, std::min<long long>(cap, (work + 4 * kThreads - 1) / (4 * kThreads)));
}

// Device copy of the room-derived tables shared by a solver and its CG.
struct RoomTables {
    double *dxv, *dyv, *dzv, *scale, *fanvel, *inv;
    uint8_t *ct, *fcu, *fcv, *fcw;
    uint16_t *sc;
};

size_t tables_bytes(const HostRoom &h)
{
    const RoomGeom &g = h.g;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    return al(8 * g.nx) + al(8 * g.ny) + al(8 * g.nz) + al(8 * 2 * (g.nx + g.ny + g.nz)) +
           al(8 * 3 * kMaxFans) + al(g.n) + al(g.nu) + al(g.nv) + al(g.nw) + al(2 * g.n) +
           al(20 * (size_t)(g.nx + g.ny + g.nz) + 8);
}

// Carves the tables from the arena and points R at them (no device work).
int carve_tables(const HostRoom &h, Arena &ar, RoomTables &t, RoomDev &R)
{
    const RoomGeom &g = h.g;
    t.dxv = ar.take<double>(g.nx);
    t.dyv = ar.take<double>(g.ny);
    t.dzv = ar.take<double>(g.nz);
    t.scale = ar.take<double>(2 * (size_t)(g.nx + g.ny + g.nz));
    t.fanvel = ar.take<double>(3 * kMaxFans);
    t.ct = ar.take<uint8_t>(g.n);
    t.fcu = ar.take<uint8_t>(g.nu);
    t.fcv = ar.take<uint8_t>(g.nv);
    t.fcw = ar.take<uint8_t>(g.nw);
    t.sc = ar.take<uint16_t>(g.n);
    t.inv = ar.take<double>((size_t)(5 * (g.nx + g.ny + g.nz) + 1) / 2);
    if (!t.inv) return fail(FFR_ENOMEM, "arena exhausted (tables)");
    R.nx = g.nx; R.ny = g.ny; R.nz = g.nz;
    R.n = (int)g.n; R.nu = (int)g.nu; R.nv = (int)g.nv; R.nw = (int)g.nw;
    R.dxv = t.dxv; R.dyv = t.dyv; R.dzv = t.dzv;
    R.ct = t.ct; R.fcu = t.fcu; R.fcv = t.fcv; R.fcw = t.fcw;
    R.sc = t.sc; R.scale = t.scale; R.fanvel = t.fanvel; R.inv = t.inv;
    return FFR_OK;
}

// Staging bytes queue_tables needs.
size_t tables_stage_bytes(const HostRoom &h)
{
    const RoomGeom &g = h.g;
    return 8 * 3 * (size_t)(g.nx + g.ny + g.nz) + 8 * 3 * kMaxFans + 5 * 16 +
           20 * (size_t)(g.nx + g.ny + g.nz) + 32;
}

// The cell types, by a synchronous staged copy.  Made before any kernel is
// queued on s, it waits for nothing but the link.
int upload_cell_types(const HostRoom &h, const RoomTables &t, cudaStream_t s)
{
    return staged_copy(t.ct, h.ct.data(), h.g.n, false, s);
}

// Queues the rest of the tables on s without waiting: spacings, stencil
// scales and fan velocities through the staging block, the stencil and
// face codes by kernels from the uploaded cell types.
int queue_tables(const HostRoom &h, const RoomTables &t, HostStage &hs, cudaStream_t s)
{
    const RoomGeom &g = h.g;
    std::vector<double> scale;
    stencil_scales(h, scale);
    std::vector<double> fan(3 * kMaxFans, 0.0);
    for (size_t f = 0; f < h.fans.size(); f++)
        for (int c = 0; c < 3; c++) fan[3 * f + c] = h.fans[f].vel[c];
    // Reciprocal spacings (RoomDev::inv): the centre distance is formed as
    // the kernels formed it, 0.5 * (d[i-1] + d[i]); the FP32 entry is the
    // correctly rounded reciprocal of the rounded width, the value
    // __frcp_rn((float)d[i]) gives on the device.
    const int S = g.nx + g.ny + g.nz;
    std::vector<double> inv((5 * (size_t)S + 1) / 2, 0.0);
    float *finv = reinterpret_cast<float *>(inv.data() + 2 * S);
    const std::vector<double> *d3[3] = {&h.dxv, &h.dyv, &h.dzv};
    for (int a = 0, off = 0; a < 3; off += (int)d3[a]->size(), a++) {
        const std::vector<double> &d = *d3[a];
        for (size_t i = 0; i < d.size(); i++) {
            if (i > 0) inv[off + i] = 1.0 / (0.5 * (d[i - 1] + d[i]));
            inv[S + off + i] = 1.0 / d[i];
            finv[off + i] = 1.0f / (float)d[i];
        }
    }
    int rc;
    if ((rc = hs.put(t.dxv, h.dxv.data(), 8 * g.nx, s)) || (rc = hs.put(t.dyv, h.dyv.data(), 8 * g.ny, s)) ||
        (rc = hs.put(t.dzv, h.dzv.data(), 8 * g.nz, s)) || (rc = hs.put(t.scale, scale.data(), 8 * scale.size(), s)) ||
        (rc = hs.put(t.fanvel, fan.data(), 8 * fan.size(), s)) || (rc = hs.put(t.inv, inv.data(), 8 * inv.size(), s)))
        return rc;
    return build_codes(h, t.ct, t.sc, t.fcu, t.fcv, t.fcw, s);
}

// CG launch geometry: as many co-resident blocks as the room can use.
struct CGLaunch {
    unsigned blocks;
    double *partials;
    GridSync *gs;
    CGScalars *sc;
};

unsigned cg_max_blocks()
{
    static unsigned cap = 0;
    if (!cap) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg, kThreads, 0);
        if (per_sm <= 0) per_sm = 1;
        cap = (unsigned)(per_sm * sm_count());
    }
    return cap;
}

}  // namespace

unsigned ffr::cg_block_cap() { return cg_max_blocks(); }

namespace {

int launch_cg(const CGArgs &a, unsigned blocks, cudaStream_t s)
{
    FFR_CUDA(cudaMemsetAsync(a.gs, 0, sizeof(GridSync), s));
    void *args[] = {(void *)&a};
    FFR_CUDA(cudaLaunchCooperativeKernel((void *)k_cg, dim3(blocks), dim3(kThreads), args, 0, s));
    count_launch(1);
    return FFR_OK;
}

}  // namespace

// ------------------------------------------------------- fluid handle

// Pressure-solve grid of a room: as many co-resident blocks as it can use.
// Blocks of the persistent CG launch: co-resident (a cooperative launch).
unsigned fluid_cg_blocks(const RoomGeom &g)
{
    return std::max(1u, std::min(cg_max_blocks(), (unsigned)((g.n + kThreads - 1) / kThreads)));
}

// Block partials both persistent solves may write (four per block).
size_t fluid_partials(const RoomGeom &g)
{
    const unsigned want = (unsigned)((g.n + kThreads - 1) / kThreads);
    const unsigned most = std::max(1u, std::min(std::max(cg_max_blocks(), pcg_max_blocks()), want));
    return std::max<size_t>((size_t)most * 4, 2 * 2368);
}

// Device bytes of one projection handle (its single arena).
size_t fluid_arena_bytes(const HostRoom &room, bool mg, const MGHost &mgh)
{
    const RoomGeom &g = room.g;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    return tables_bytes(room) + 2 * (al(8 * g.nu) + al(8 * g.nv) + al(8 * g.nw)) + (mg ? 9 : 7) * al(8 * g.n) +
           al(8 * fluid_partials(g)) + al(8 * stream_blocks(g.n)) + al(256) +
           al(sizeof(GridSync)) + al(sizeof(CGScalars)) + al(sizeof(StepState)) +
           al(sizeof(ffr_step_result) * kRing) + 4 * 256 + (mg ? mg_bytes(room, mgh) : 0);
}

// Removes a room that is being destroyed from every batch it belongs to
// (defined with the batch below).
void fluid_leave_batches(ffr_fluid *s);

struct ffr_fluid {
    HostRoom room;
    ffr_fluid_params prm;
    std::vector<ffr_batch *> batches;   // the batches this room is a member of
    cudaStream_t stream = nullptr;
    Arena arena;
    RoomTables tab;
    RoomDev R;
    double *u, *v, *w, *us, *vs, *ws, *p, *T0, *T1;
    double *r, *da, *db, *ad, *partials, *tpart, *cg_res;
    int *cg_iters, *cg_flags;
    GridSync *gs;
    CGScalars *sc;
    StepState *st;
    ffr_step_result *ring;
    ffr_step_result *ring_host;
    StepState *st_host;
    unsigned long long *div_slot;
    unsigned cg_blocks, blocks_faces, blocks_cells;
    GroupTimer prof;
    bool mg = false, mixed = false;
    MGDev M;
    MGHost mgh;
    unsigned block_override = 0;   // pressure-solve grid size chosen by the caller (0: automatic)
    int cluster_ctas = 0;          // >0: the multigrid solve runs in one cluster of that many blocks
    int pending = 0;               // steps queued by ffr_fluid_enqueue and not yet polled
    cudaEvent_t done_ev = nullptr;
    cudaGraph_t graph = nullptr;   // one captured step, replayed per step when use_graph
    cudaGraphExec_t graph_exec = nullptr;
    bool use_graph = false;
    unsigned graph_launches = 0;   // kernels in the captured step
    unsigned split_body = 0;       // kernels per PCG iteration of a captured split solve
    bool capturing_split = false;  // the multigrid solve is being recorded in its split form
    void *split_state = nullptr;   // device SplitState of the split solve
    cudaStream_t body_stream = nullptr;
    int split_mode = -1;           // multigrid schedule: -1 split in graphs only, 0 never, 1 always
    SplitHost split_host;          // host pacing of the eager split solve
    HostStage stage;               // page-locked source of the set-up copies
    bool warm_start = true;        // multigrid solve starts from the previous step's pressure
    double *p0 = nullptr;          // multigrid: the pressure the last solve started from
    double *pprev = nullptr;       // multigrid: the solution of the step before the last
    bool p0_valid = false;         // p0 belongs to the last step (taken by this handle's own launches)
};

namespace {

// Pressure solve of the current step on stream st.  capture: 2 = the stream
// is being captured and the multigrid solve is recorded in its split form
// (WHILE node); 1 = the stream is being captured (no host-paced launches);
// 0 = eager launch.
int enqueue_pressure(ffr_fluid *s, cudaStream_t st, int capture, unsigned *body_kernels, bool restore = false)
{
    const ffr_fluid_params &P = s->prm;
    if (s->mg) {
        PCGArgs pa2{};
        pa2.R = s->R; pa2.M = s->M;
        pa2.us = s->us; pa2.vs = s->vs; pa2.ws = s->ws;
        pa2.rhs_factor = -(P.rho / P.dt);
        pa2.from_faces = 1;
        pa2.warm = s->warm_start ? 1 : 0;
        pa2.x = s->p; pa2.r = s->r; pa2.da = s->da; pa2.db = s->db; pa2.q = s->ad;
        pa2.xprev = s->pprev; pa2.x0 = s->p0;
        pa2.partials = s->partials; pa2.gs = s->gs; pa2.sc = s->sc;
        pa2.max_iter = P.poisson_max_iter; pa2.tol = P.poisson_tol;
        pa2.st = s->st;
        if (s->warm_start) {
            // the start of this solve; a re-solve of the same system
            // (restore: ffr_fluid_time_pressure) starts from the kept copy
            if (restore)
                FFR_CUDA(cudaMemcpyAsync(s->p, s->p0, 8 * (size_t)s->room.g.n, cudaMemcpyDeviceToDevice, st));
            else if (int rc = launch_extrapolate(pa2, st))
                return rc;
        }
        const bool plain_grid = s->cluster_ctas == 0 && s->block_override == 0;
        if (capture == 2) return capture_split_pcg(pa2, s->split_state, st, s->body_stream, body_kernels);
        if (capture == 0 && plain_grid && s->split_mode == 1)
            return launch_split_pcg(pa2, s->split_state, st, s->split_host);
        return s->cluster_ctas > 0 ? launch_pcg_cluster(pa2, st, s->cluster_ctas)
                                   : launch_pcg(pa2, st, nullptr, s->block_override);
    }
    CGArgs ca{};
    ca.R = s->R;
    ca.us = s->us; ca.vs = s->vs; ca.ws = s->ws;
    ca.rhs_factor = -(P.rho / P.dt);
    ca.from_faces = 1;
    ca.x = s->p; ca.r = s->r; ca.da = s->da; ca.db = s->db; ca.ad = s->ad;
    ca.partials = s->partials; ca.gs = s->gs; ca.sc = s->sc;
    ca.max_iter = P.poisson_max_iter; ca.tol = P.poisson_tol;
    ca.st = s->st;
    return launch_cg(ca, s->block_override ? std::min(s->block_override, s->cg_blocks) : s->cg_blocks, st);
}

int fluid_enqueue_step(ffr_fluid *s)
{
    const ffr_fluid_params &P = s->prm;
    cudaStream_t st = s->stream;
    const RoomGeom &g = s->room.g;
    PredArgs pa{P.dt, P.nu, P.advection, P.buoyancy ? 1 : 0, P.g_accel * P.beta * P.dt, P.T_initial};
    s->prof.begin(FFR_PROF_PREDICT, st);
    if (s->mixed)
        k_predict<float><<<s->blocks_faces, kThreads, 0, st>>>(s->R, pa, s->u, s->v, s->w, s->T0, s->T1, s->us,
                                                                s->vs, s->ws, s->st);
    else
        k_predict<double><<<s->blocks_faces, kThreads, 0, st>>>(s->R, pa, s->u, s->v, s->w, s->T0, s->T1, s->us,
                                                                 s->vs, s->ws, s->st);
    FFR_LAUNCHED(1);
    s->prof.end(st, 1);
    s->prof.begin(FFR_PROF_PRESSURE, st);
    int rc = enqueue_pressure(s, st, s->capturing_split ? 2 : 0, &s->split_body);
    if (rc) return rc;
    s->p0_valid = true;
    s->prof.end(st, 1);
    CorrArgs co{P.dt / P.rho};
    s->prof.begin(FFR_PROF_CORRECT, st);
    // rows of even length take the paired form (16-byte loads of two cells)
    if ((s->R.nz & 1) == 0)
        k_correct<true><<<s->blocks_cells, kThreads, 0, st>>>(s->R, co, s->u, s->v, s->w, s->us, s->vs, s->ws,
                                                              s->p, s->st);
    else
        k_correct<false><<<s->blocks_cells, kThreads, 0, st>>>(s->R, co, s->u, s->v, s->w, s->us, s->vs, s->ws,
                                                               s->p, s->st);
    FFR_LAUNCHED(1);
    s->prof.end(st, 1);
    int nthermal = 1;
    s->prof.begin(FFR_PROF_THERMAL, st);
    if (P.thermal) {
        for (const ffr_patch &op : s->room.patches) {
            if (!op.is_opening) continue;
            k_opening_T<<<stream_blocks((long long)(op.a_max - op.a_min + 1) * (op.b_max - op.b_min + 1)),
                          kThreads, 0, st>>>(s->R, op, s->u, s->v, s->w, s->T0, s->T1, s->st, 0);
            FFR_LAUNCHED(1);
            nthermal++;
        }
        ThermArgs ta{P.dt, P.k_thermal / (P.rho * P.cp), P.advection};
        if (s->mixed)
            k_advect_T<float><<<s->blocks_cells, kThreads, 0, st>>>(s->R, ta, s->u, s->v, s->w, s->T0, s->T1,
                                                                     s->tpart, s->st);
        else
            k_advect_T<double><<<s->blocks_cells, kThreads, 0, st>>>(s->R, ta, s->u, s->v, s->w, s->T0, s->T1,
                                                                      s->tpart, s->st);
        FFR_LAUNCHED(1);
        nthermal++;
        for (const ffr_patch &op : s->room.patches) {
            if (!op.is_opening) continue;
            k_opening_T<<<stream_blocks((long long)(op.a_max - op.a_min + 1) * (op.b_max - op.b_min + 1)),
                          kThreads, 0, st>>>(s->R, op, s->u, s->v, s->w, s->T0, s->T1, s->st, 1);
            FFR_LAUNCHED(1);
            nthermal++;
        }
    }
    for (const ffr_heat_patch &h : s->room.heats) {
        k_heat<<<stream_blocks((long long)(h.i_max - h.i_min + 1) * (h.j_max - h.j_min + 1) *
                               (h.k_max - h.k_min + 1)),
                 kThreads, 0, st>>>(s->R, h, s->T0, s->T1, s->st, P.thermal ? 1 : 0);
        FFR_LAUNCHED(1);
        nthermal++;
    }
    FinArgs fa{P.dt, P.convergence_tol, P.T_initial, P.T_target, P.thermal ? 1 : 0,
               s->room.n_fluid, (int)s->blocks_cells};
    k_finalize<<<1, kThreads, 0, st>>>(fa, s->tpart, s->st, s->ring);
    FFR_LAUNCHED(1);
    s->prof.end(st, nthermal);
    (void)g;
    return FFR_OK;
}

double *field_ptr(ffr_fluid *s, int field)
{
    switch (field) {
    case FFR_FIELD_U: return s->u;
    case FFR_FIELD_V: return s->v;
    case FFR_FIELD_W: return s->w;
    case FFR_FIELD_P: return s->p;
    case FFR_FIELD_T: return s->st_host->tpar ? s->T1 : s->T0;
    default: return nullptr;
    }
}

long long field_len(const ffr_fluid *s, int field)
{
    const RoomGeom &g = s->room.g;
    switch (field) {
    case FFR_FIELD_U: return g.nu;
    case FFR_FIELD_V: return g.nv;
    case FFR_FIELD_W: return g.nw;
    default: return g.n;
    }
}

int pull_state(ffr_fluid *s)
{
    if (s->pending) {
        // a queued chunk: wait for it; its results stay available to poll
        FFR_CUDA(cudaEventSynchronize(s->done_ev));
    }
    FFR_CUDA(cudaMemcpyAsync(s->st_host, s->st, sizeof(StepState), cudaMemcpyDeviceToHost, s->stream));
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    s->prof.collect();
    return FFR_OK;
}

}  // namespace

extern "C" {

int ffr_fluid_create(const ffr_room_desc *room, const ffr_fluid_params *params,
                     const ffr_fields *init, ffr_fluid **out)
{
    if (!params || !out) return fail(FFR_EINVAL, "NULL params or out");
    *out = nullptr;
    if (params->precision != FFR_PREC_FP64 && params->precision != FFR_PREC_MIXED)
        return fail(FFR_EINVAL, "bad precision");
    if (params->poisson != FFR_POISSON_CG && params->poisson != FFR_POISSON_MGPCG)
        return fail(FFR_EINVAL, "bad pressure solver");
    if (!(params->dt > 0) || !(params->rho > 0)) return fail(FFR_EINVAL, "dt and rho must be positive");
    if (params->advection < 0 || params->advection > 2) return fail(FFR_EINVAL, "bad advection scheme");
    if (params->poisson_max_iter < 0) return fail(FFR_EINVAL, "negative poisson_max_iter");
    ffr_fluid *s = new (std::nothrow) ffr_fluid();
    if (!s) return fail(FFR_ENOMEM, "host allocation");
    int rc = load_room(room, s->room);
    if (rc) { delete s; return rc; }
    s->prm = *params;
    s->mixed = params->precision == FFR_PREC_MIXED;
    s->mg = params->poisson == FFR_POISSON_MGPCG || params->use_multigrid;
    if (s->mg) build_mg_levels(s->room, s->mgh);
    const RoomGeom &g = s->room.g;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return fail(FFR_ECUDA, "cudaStreamCreate");
    }
    s->cg_blocks = fluid_cg_blocks(g);
    s->blocks_faces = stream_blocks(g.nu + g.nv + g.nw);
    s->blocks_cells = stream_blocks(g.n);
    rc = s->arena.alloc(fluid_arena_bytes(s->room, s->mg, s->mgh), s->stream);
    if (rc) { cudaStreamDestroy(s->stream); delete s; return rc; }
    rc = carve_tables(s->room, s->arena, s->tab, s->R);
    Arena &a = s->arena;
    s->u = a.take<double>(g.nu); s->v = a.take<double>(g.nv); s->w = a.take<double>(g.nw);
    s->us = a.take<double>(g.nu); s->vs = a.take<double>(g.nv); s->ws = a.take<double>(g.nw);
    s->p = a.take<double>(g.n); s->T0 = a.take<double>(g.n); s->T1 = a.take<double>(g.n);
    s->r = a.take<double>(g.n); s->da = a.take<double>(g.n); s->db = a.take<double>(g.n);
    s->ad = a.take<double>(g.n);
    if (s->mg) {
        s->p0 = a.take<double>(g.n);
        s->pprev = a.take<double>(g.n);
    }
    s->partials = a.take<double>(fluid_partials(g));
    s->tpart = a.take<double>(s->blocks_cells);
    s->split_state = a.take<char>(256);
    s->gs = a.take<GridSync>(1);
    s->sc = a.take<CGScalars>(1);
    s->st = a.take<StepState>(1);
    s->ring = a.take<ffr_step_result>(kRing);
    s->cg_res = a.take<double>(1);
    s->cg_iters = a.take<int>(1);
    s->cg_flags = a.take<int>(1);
    s->div_slot = a.take<unsigned long long>(1);
    if (rc || !s->div_slot || s->arena.failed) {
        if (!rc) rc = fail(FFR_ENOMEM, "arena exhausted");
        ffr_fluid_destroy(s);
        return rc;
    }
    s->ring_host = static_cast<ffr_step_result *>(pinned_get(sizeof(ffr_step_result) * kRing));
    s->st_host = static_cast<StepState *>(pinned_get(sizeof(StepState)));
    if (!s->ring_host || !s->st_host) {
        ffr_fluid_destroy(s);
        return fail(FFR_ENOMEM, "pinned host allocation");
    }
    memset(s->st_host, 0, sizeof(StepState));
    s->prof.reset(FFR_PROF_N);
    if (cudaEventCreateWithFlags(&s->done_ev, cudaEventDisableTiming) != cudaSuccess) {
        ffr_fluid_destroy(s);
        return fail(FFR_ECUDA, "cudaEventCreate");
    }
    cudaStream_t st = s->stream;
    // Synchronous copies first, while nothing is queued on the stream (so
    // they wait for the link only, not for other rooms' kernels); then the
    // rest of the set-up is queued and create returns without waiting.
    rc = upload_cell_types(s->room, s->tab, st);
    if (rc) { ffr_fluid_destroy(s); return rc; }
    if (init) {
        const double *src[4] = {init->u, init->v, init->w, init->p};
        double *dst[4] = {s->u, s->v, s->w, s->p};
        const long long cnt[4] = {g.nu, g.nv, g.nw, g.n};
        for (int f = 0; f < 4; f++)
            if (src[f] && (rc = staged_copy(dst[f], src[f], 8 * cnt[f], false, st))) {
                ffr_fluid_destroy(s);
                return rc;
            }
    }
    {
        const double *src[4] = {init ? init->u : nullptr, init ? init->v : nullptr, init ? init->w : nullptr,
                                init ? init->p : nullptr};
        double *dst[4] = {s->u, s->v, s->w, s->p};
        const long long cnt[4] = {g.nu, g.nv, g.nw, g.n};
        for (int f = 0; f < 4; f++)
            if (!src[f]) FFR_CUDA(cudaMemsetAsync(dst[f], 0, 8 * cnt[f], st));
    }
    rc = s->stage.reserve(tables_stage_bytes(s->room) + (s->mg ? mg_stage_bytes(s->room) : 0));
    if (!rc) rc = queue_tables(s->room, s->tab, s->stage, st);
    if (!rc && s->mg) {
        rc = mg_upload(s->room, s->mgh, s->R, s->arena, s->stage, st, s->M);
        s->M.vol_x = s->R.dxv; s->M.vol_y = s->R.dyv; s->M.vol_z = s->R.dzv;
    }
    if (rc) { ffr_fluid_destroy(s); return rc; }
    FFR_CUDA(cudaMemsetAsync(s->st, 0, sizeof(StepState), st));
    FFR_CUDA(cudaMemsetAsync(s->split_state, 0, 256, st));
    if (s->mg) FFR_CUDA(cudaMemsetAsync(s->pprev, 0, 8 * g.n, st));
    k_fill<<<stream_blocks(g.n), kThreads, 0, st>>>(s->T0, (int)g.n, params->T_initial);
    FFR_LAUNCHED(1);
    if (params->thermal) {
        for (const ffr_patch &op : s->room.patches) {
            if (!op.is_opening) continue;
            k_opening_T<<<stream_blocks((long long)(op.a_max - op.a_min + 1) * (op.b_max - op.b_min + 1)),
                          kThreads, 0, st>>>(s->R, op, s->u, s->v, s->w, s->T0, s->T1, s->st, 0);
            FFR_LAUNCHED(1);
        }
    }
    *out = s;
    return FFR_OK;
}

int ffr_fluid_destroy(ffr_fluid *s)
{
    if (!s) return FFR_OK;
    fluid_leave_batches(s);
    if (s->stream) cudaStreamSynchronize(s->stream);
    s->prof.destroy();
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    if (s->body_stream) cudaStreamDestroy(s->body_stream);
    s->split_host.release();
    if (s->done_ev) cudaEventDestroy(s->done_ev);
    s->stage.release();
    s->arena.release();
    pinned_put(s->ring_host, sizeof(ffr_step_result) * kRing);
    pinned_put(s->st_host, sizeof(StepState));
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FFR_OK;
}

int ffr_fluid_enqueue(ffr_fluid *s, int nsteps, int stop_on_converge)
{
    if (!s || nsteps < 0 || nsteps > kRing) return fail(FFR_EINVAL, "bad handle or nsteps (0..1024)");
    if (s->pending) return fail(FFR_EINVAL, "a queued chunk has not been polled yet");
    k_begin_chunk<<<1, 1, 0, s->stream>>>(s->st, stop_on_converge ? 1 : 0);
    FFR_LAUNCHED(1);
    for (int k = 0; k < nsteps; k++) {
        if (s->use_graph) {
            FFR_CUDA(cudaGraphLaunch(s->graph_exec, s->stream));
            count_launch(s->graph_launches);
            continue;
        }
        int rc = fluid_enqueue_step(s);
        if (rc) return rc;
    }
    if (nsteps > 0)
        FFR_CUDA(cudaMemcpyAsync(s->ring_host, s->ring, sizeof(ffr_step_result) * nsteps, cudaMemcpyDeviceToHost,
                                 s->stream));
    FFR_CUDA(cudaMemcpyAsync(s->st_host, s->st, sizeof(StepState), cudaMemcpyDeviceToHost, s->stream));
    FFR_CUDA(cudaEventRecord(s->done_ev, s->stream));
    s->pending = nsteps > 0 ? nsteps : -1;
    return FFR_OK;
}

int ffr_fluid_poll(ffr_fluid *s, ffr_step_result *results, int max_results, int *nresults, int *ready)
{
    if (!s || !ready) return fail(FFR_EINVAL, "NULL argument");
    if (nresults) *nresults = 0;
    if (!s->pending) { *ready = 1; return FFR_OK; }
    cudaError_t e = cudaEventQuery(s->done_ev);
    if (e == cudaErrorNotReady) { *ready = 0; return FFR_OK; }
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventQuery");
    *ready = 1;
    s->pending = 0;
    s->prof.collect();
    const int got = s->st_host->ring_slot;
    // the graph launch counted the loop body once; it ran once per iteration
    if (s->use_graph && s->split_body)
        for (int k = 0; k < got; k++)
            count_launch(s->split_body * (unsigned)std::max(0, s->ring_host[k].cg_iterations - 1));
    const int n = std::min(got, std::max(0, max_results));
    if (results && n > 0) memcpy(results, s->ring_host, sizeof(ffr_step_result) * n);
    if (nresults) *nresults = n;
    for (int k = 0; k < got; k++)
        if (s->ring_host[k].flags & FFR_FLAG_TIMEOUT)
            return fail(FFR_ETIMEDOUT, "pressure-solve grid barrier timed out");
    return FFR_OK;
}

int ffr_fluid_advance(ffr_fluid *s, int nsteps, int stop_on_converge, ffr_step_result *results,
                      int *steps_done)
{
    if (!s || nsteps < 0) return fail(FFR_EINVAL, "bad handle or nsteps");
    if (s->pending) return fail(FFR_EINVAL, "a queued chunk has not been polled yet");
    int done_total = 0;
    while (done_total < nsteps) {
        const int chunk = std::min(kRing, nsteps - done_total);
        int rc = ffr_fluid_enqueue(s, chunk, stop_on_converge);
        if (rc) return rc;
        FFR_CUDA(cudaEventSynchronize(s->done_ev));
        int got = 0, ready = 0;
        rc = ffr_fluid_poll(s, results ? results + done_total : nullptr, chunk, &got, &ready);
        if (!results) got = s->st_host->ring_slot;
        done_total += got;
        if (rc) {
            if (steps_done) *steps_done = done_total;
            return rc;
        }
        if (got < chunk) break;   // halted on convergence
    }
    if (steps_done) *steps_done = done_total;
    return FFR_OK;
}

int ffr_fluid_set_blocks(ffr_fluid *s, int blocks)
{
    if (!s || blocks < 0) return fail(FFR_EINVAL, "bad handle or blocks");
    if (s->use_graph) return fail(FFR_EINVAL, "set the grid size before capturing the step graph");
    s->block_override = (unsigned)std::min<long long>(blocks, s->cg_blocks);
    return FFR_OK;
}

int ffr_fluid_set_cluster(ffr_fluid *s, int ctas)
{
    if (!s || ctas < 0 || ctas > 16) return fail(FFR_EINVAL, "bad handle or cluster size (0..16)");
    if (ctas > 0 && !s->mg) return fail(FFR_ENOTSUP, "cluster schedule is built for the multigrid solve only");
    if (s->use_graph) return fail(FFR_EINVAL, "set the schedule before capturing the step graph");
    s->cluster_ctas = ctas;
    return FFR_OK;
}

int ffr_fluid_time_pressure(ffr_fluid *s, int nrep, double *ms_per_solve, int *iterations)
{
    if (!s || nrep <= 0 || !ms_per_solve) return fail(FFR_EINVAL, "bad arguments");
    if (s->pending) return fail(FFR_EINVAL, "a queued chunk has not been polled yet");
    if (s->mg && s->warm_start && !s->p0_valid)
        return fail(FFR_EINVAL, "no step of this handle's own launches to re-solve (warm-started solve)");
    cudaStream_t st = s->stream;
    FFR_CUDA(cudaStreamSynchronize(st));
    // the solve reads the predicted faces and halt flag of the last step
    StepState hs;
    FFR_CUDA(cudaMemcpy(&hs, s->st, sizeof(StepState), cudaMemcpyDeviceToHost));
    const int halt = hs.halt;
    hs.halt = 0;
    FFR_CUDA(cudaMemcpy(s->st, &hs, sizeof(StepState), cudaMemcpyHostToDevice));
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    unsigned body = 0;
    const unsigned long long l0 = ffr_launch_count();
    unsigned captured = 0;
    int rc = FFR_OK;
    if (s->use_graph) {
        // the same form the step graph holds
        const bool split = s->mg && s->cluster_ctas == 0 && s->block_override == 0 && s->split_mode != 0;
        if (split && !s->body_stream) FFR_CUDA(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
        FFR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        rc = enqueue_pressure(s, st, split ? 2 : 1, &body, true);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(pressure)");
        e = cudaGraphInstantiate(&ge, g, 0);
        if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(e, "cudaGraphInstantiate(pressure)"); }
        captured = (unsigned)(ffr_launch_count() - l0);
    }
    cudaEvent_t a, b;
    FFR_CUDA(cudaEventCreate(&a));
    FFR_CUDA(cudaEventCreate(&b));
    for (int r = 0; r <= nrep && rc == FFR_OK; r++) {   // r = 0 is the warm-up
        if (r == 1) FFR_CUDA(cudaEventRecord(a, st));
        if (ge) {
            FFR_CUDA(cudaGraphLaunch(ge, st));
        } else {
            rc = enqueue_pressure(s, st, 0, nullptr, true);
        }
    }
    FFR_CUDA(cudaEventRecord(b, st));
    FFR_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    FFR_CUDA(cudaEventElapsedTime(&ms, a, b));
    *ms_per_solve = ms / nrep;
    FFR_CUDA(cudaMemcpy(&hs, s->st, sizeof(StepState), cudaMemcpyDeviceToHost));
    if (iterations) *iterations = hs.iters;
    hs.halt = halt;
    FFR_CUDA(cudaMemcpy(s->st, &hs, sizeof(StepState), cudaMemcpyHostToDevice));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ge) {
        cudaGraphExecDestroy(ge);
        cudaGraphDestroy(g);
        // replays ran the loop body once per iteration; the capture counted it once
        const unsigned per_solve = captured + body * (unsigned)std::max(0, hs.iters - 1);
        count_launch(per_solve * (unsigned)(nrep + 1) - captured);
    }
    return rc;
}

int ffr_fluid_set_warm_start(ffr_fluid *s, int enable)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    if (s->pending) return fail(FFR_EINVAL, "a queued chunk has not been polled yet");
    if (s->use_graph || s->graph_exec) return fail(FFR_EINVAL, "choose the start before capturing the step graph");
    s->warm_start = enable != 0;
    s->p0_valid = false;
    return FFR_OK;
}

int ffr_fluid_set_split(ffr_fluid *s, int mode)
{
    if (!s || mode < -1 || mode > 1) return fail(FFR_EINVAL, "bad handle or mode (-1, 0, 1)");
    if (s->use_graph || s->graph_exec) return fail(FFR_EINVAL, "choose the schedule before capturing the step graph");
    s->split_mode = mode;
    return FFR_OK;
}

int ffr_fluid_use_graph(ffr_fluid *s, int enable)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    if (s->pending) return fail(FFR_EINVAL, "a queued chunk has not been polled yet");
    if (!enable) {
        s->use_graph = false;
        return FFR_OK;
    }
    if (s->graph_exec) {
        s->use_graph = true;
        return FFR_OK;
    }
    if (s->prof.on) return fail(FFR_EINVAL, "disable kernel-group timing before capturing the step graph");
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    const unsigned long long l0 = ffr_launch_count();
    s->capturing_split = s->mg && s->cluster_ctas == 0 && s->block_override == 0 && s->split_mode != 0;
    if (s->capturing_split && !s->body_stream)
        FFR_CUDA(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
    FFR_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeRelaxed));
    int rc = fluid_enqueue_step(s);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    s->capturing_split = false;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(step)");
    e = cudaGraphInstantiate(&s->graph_exec, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(e, "cudaGraphInstantiate(step)");
    }
    s->graph = g;
    s->graph_launches = (unsigned)(ffr_launch_count() - l0);
    s->use_graph = true;
    return FFR_OK;
}

int ffr_fluid_estimate_bytes(const ffr_room_desc *room, const ffr_fluid_params *params, size_t *bytes)
{
    if (!params || !bytes) return fail(FFR_EINVAL, "NULL params or bytes");
    HostRoom r;
    int rc = load_room(room, r);
    if (rc) return rc;
    MGHost mgh;
    const bool mg = params->poisson == FFR_POISSON_MGPCG || params->use_multigrid;
    if (mg) build_mg_levels(r, mgh);
    // the arena plus the transient scratch of the multigrid coefficient build
    size_t scratch = 0;
    if (mg && mgh.nx.size() > 1) {
        const size_t m1 = (size_t)mgh.nx[1] * mgh.ny[1] * mgh.nz[1];
        scratch = 2 * (48 * m1 + ((m1 + 255) & ~size_t(255)));
    }
    *bytes = fluid_arena_bytes(r, mg, mgh) + scratch;
    return FFR_OK;
}

int ffr_fluid_device_bytes(ffr_fluid *s, size_t *bytes)
{
    if (!s || !bytes) return fail(FFR_EINVAL, "NULL argument");
    *bytes = s->arena.size;
    return FFR_OK;
}

int ffr_fluid_step(ffr_fluid *s, ffr_step_result *out)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    ffr_step_result tmp;
    if (!out) out = &tmp;
    int done = 0;
    int rc = ffr_fluid_advance(s, 1, 0, out, &done);
    if (rc) return rc;
    return done == 1 ? FFR_OK : fail(FFR_ECUDA, "step did not execute");
}

int ffr_fluid_divergence_max(ffr_fluid *s, double *out)
{
    if (!s || !out) return fail(FFR_EINVAL, "NULL argument");
    FFR_CUDA(cudaMemsetAsync(s->div_slot, 0, 8, s->stream));
    k_divergence<<<s->blocks_cells, kThreads, 0, s->stream>>>(s->R, s->u, s->v, s->w, s->div_slot);
    FFR_LAUNCHED(1);
    unsigned long long bits = 0;
    FFR_CUDA(cudaMemcpyAsync(&bits, s->div_slot, 8, cudaMemcpyDeviceToHost, s->stream));
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    memcpy(out, &bits, 8);
    return FFR_OK;
}

int ffr_fluid_snapshot(ffr_fluid *s, double *uc, double *vc, double *wc, double *speed)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    int rc = pull_state(s);
    if (rc) return rc;
    // the CG work vectors are free between steps: they hold the snapshot
    k_snapshot<<<s->blocks_cells, kThreads, 0, s->stream>>>(s->R, s->u, s->v, s->w, s->r, s->da, s->db, s->ad);
    FFR_LAUNCHED(1);
    const size_t bytes = 8 * (size_t)s->room.g.n;
    if (uc) FFR_CUDA(cudaMemcpyAsync(uc, s->r, bytes, cudaMemcpyDeviceToHost, s->stream));
    if (vc) FFR_CUDA(cudaMemcpyAsync(vc, s->da, bytes, cudaMemcpyDeviceToHost, s->stream));
    if (wc) FFR_CUDA(cudaMemcpyAsync(wc, s->db, bytes, cudaMemcpyDeviceToHost, s->stream));
    if (speed) FFR_CUDA(cudaMemcpyAsync(speed, s->ad, bytes, cudaMemcpyDeviceToHost, s->stream));
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    return FFR_OK;
}

int ffr_fluid_current_step(ffr_fluid *s, int *out)
{
    if (!s || !out) return fail(FFR_EINVAL, "NULL argument");
    int rc = pull_state(s);
    if (rc) return rc;
    *out = s->st_host->step;
    return FFR_OK;
}

int ffr_fluid_get_field(ffr_fluid *s, int field, double *host)
{
    if (!s || !host || field < 0 || field > 4) return fail(FFR_EINVAL, "bad get_field arguments");
    int rc = pull_state(s);
    if (rc) return rc;
    return staged_copy(host, field_ptr(s, field), 8 * field_len(s, field), true, s->stream);
}

int ffr_fluid_set_field(ffr_fluid *s, int field, const double *host)
{
    if (!s || !host || field < 0 || field > 4) return fail(FFR_EINVAL, "bad set_field arguments");
    int rc = pull_state(s);
    if (rc) return rc;
    return staged_copy(field_ptr(s, field), host, 8 * field_len(s, field), false, s->stream);
}

int ffr_fluid_field_dev(ffr_fluid *s, int field, double **dev)
{
    if (!s || !dev || field < 0 || field > 4) return fail(FFR_EINVAL, "bad field_dev arguments");
    int rc = pull_state(s);
    if (rc) return rc;
    *dev = field_ptr(s, field);
    return FFR_OK;
}

int ffr_fluid_synchronize(ffr_fluid *s)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    s->prof.collect();
    return FFR_OK;
}

int ffr_fluid_stream(ffr_fluid *s, void **stream)
{
    if (!s || !stream) return fail(FFR_EINVAL, "NULL argument");
    *stream = (void *)s->stream;
    return FFR_OK;
}

int ffr_fluid_profile(ffr_fluid *s, int enable)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    s->prof.collect();
    s->prof.reset(FFR_PROF_N);
    s->prof.on = enable != 0;
    return FFR_OK;
}

int ffr_fluid_profile_read(ffr_fluid *s, double *ms, long long *launches)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    s->prof.collect();
    for (int g = 0; g < FFR_PROF_N; g++) {
        if (ms) ms[g] = s->prof.ms[g];
        if (launches) launches[g] = s->prof.launches[g];
    }
    return FFR_OK;
}

}  // extern "C"

// ------------------------------------------------------- batched rooms

struct ffr_batch {
    std::vector<ffr_fluid *> rooms;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    BatchSplit split;
    void *dev = nullptr;          // BRoom array, launch tables, patch items
    size_t cap = 0;               // its size (reused while large enough)
    const BRoom *broom = nullptr;
    BMap faces{}, cells{}, openm{}, heatm{};
    unsigned nb_faces = 0, nb_cells = 0, nb_open = 0, nb_heat = 0;
    const OpenItem *open = nullptr;
    const HeatItem *heat = nullptr;
    bool any_thermal = false;
    int max_iter = 0;
    int cluster_ctas = 0;         // > 0: every room's whole solve on one cluster of this size
    // one captured batched step (predictor, the solve's WHILE node,
    // correction, thermal, finalize), replayed per step when use_graph;
    // recaptured after a membership change
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t body_stream = nullptr;
    unsigned graph_launches = 0;
    // a member was destroyed (its pointers are still in the device tables)
    // or setting the members failed part-way: nothing is queued until the
    // members are set again
    bool stale = false;
};

// A destroyed room leaves every batch: the batch's queued launches may
// still read the room, and the batch queues nothing more until its members
// are set again.
void fluid_leave_batches(ffr_fluid *s)
{
    for (ffr_batch *b : s->batches) {
        if (b->stream) cudaStreamSynchronize(b->stream);
        b->rooms.erase(std::remove(b->rooms.begin(), b->rooms.end(), s), b->rooms.end());
        b->stale = true;
    }
    s->batches.clear();
}

namespace {

// Drops b from the membership lists of its rooms.
void batch_detach_all(ffr_batch *b)
{
    for (ffr_fluid *s : b->rooms) {
        auto &v = s->batches;
        v.erase(std::remove(v.begin(), v.end(), b), v.end());
    }
}

void batch_free(ffr_batch *b)
{
    if (!b) return;
    batch_detach_all(b);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->body_stream) cudaStreamDestroy(b->body_stream);
    batch_split_release(b->split);
    if (b->split.active_host) cudaFreeHost(b->split.active_host);
    for (int k = 0; k < 2; k++)
        if (b->split.ev[k]) cudaEventDestroy(b->split.ev[k]);
    if (b->dev) cudaFree(b->dev);
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

PCGArgs room_pcg_args(ffr_fluid *s)
{
    const ffr_fluid_params &P = s->prm;
    PCGArgs a{};
    a.R = s->R; a.M = s->M;
    a.us = s->us; a.vs = s->vs; a.ws = s->ws;
    a.rhs_factor = -(P.rho / P.dt);
    a.from_faces = 1;
    a.warm = s->warm_start ? 1 : 0;
    a.x = s->p; a.r = s->r; a.da = s->da; a.db = s->db; a.q = s->ad;
    a.xprev = s->pprev; a.x0 = s->p0;
    a.partials = s->partials; a.gs = s->gs; a.sc = s->sc;
    a.max_iter = P.poisson_max_iter; a.tol = P.poisson_tol;
    a.st = s->st;
    return a;
}

BRoom room_step_args(ffr_fluid *s)
{
    const ffr_fluid_params &P = s->prm;
    BRoom b{};
    b.R = s->R;
    b.pa = PredArgs{P.dt, P.nu, P.advection, P.buoyancy ? 1 : 0, P.g_accel * P.beta * P.dt, P.T_initial};
    b.co = CorrArgs{P.dt / P.rho};
    b.ta = ThermArgs{P.dt, P.k_thermal / (P.rho * P.cp), P.advection};
    b.fa = FinArgs{P.dt, P.convergence_tol, P.T_initial, P.T_target, P.thermal ? 1 : 0, s->room.n_fluid,
                   (int)s->blocks_cells};
    b.u = s->u; b.v = s->v; b.w = s->w; b.us = s->us; b.vs = s->vs; b.ws = s->ws;
    b.p = s->p; b.T0 = s->T0; b.T1 = s->T1; b.tpart = s->tpart;
    b.st = s->st;
    b.ring = s->ring;
    b.mixed = s->mixed ? 1 : 0;
    b.thermal = P.thermal ? 1 : 0;
    return b;
}

}  // namespace

extern "C" {

int ffr_batch_set_rooms(ffr_batch *b, ffr_fluid *const *rooms, int nrooms)
{
    if (!b || nrooms <= 0 || !rooms) return fail(FFR_EINVAL, "bad arguments");
    for (int r = 0; r < nrooms; r++) {
        ffr_fluid *s = rooms[r];
        if (!s) return fail(FFR_EINVAL, "NULL room handle");
        if (!s->mg) return fail(FFR_EINVAL, "a batch takes rooms with the multigrid pressure solve");
        if (s->pending) return fail(FFR_EINVAL, "a room has a queued chunk that was not polled");
        if (s->block_override) return fail(FFR_EINVAL, "a batched room keeps the default grid");
        if (s->cluster_ctas != rooms[0]->cluster_ctas)
            return fail(FFR_EINVAL, "the rooms of a batch share one schedule (all split, or one cluster size)");
        for (int q = 0; q < r; q++)
            if (rooms[q] == s) return fail(FFR_EINVAL, "a room appears twice in the batch");
    }
    // the tables of the previous membership may still be read by its launches
    FFR_CUDA(cudaStreamSynchronize(b->stream));
    // a captured step holds the previous tables' addresses
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
    batch_detach_all(b);
    b->rooms.assign(rooms, rooms + nrooms);
    for (ffr_fluid *s : b->rooms) s->batches.push_back(b);
    b->stale = true;   // until the tables below are built
    b->cluster_ctas = rooms[0]->cluster_ctas;
    b->any_thermal = false;
    b->max_iter = 0;
    // per-room arguments, block tables of the step kernels, patch items
    std::vector<BRoom> br(nrooms);
    std::vector<PCGArgs> pa(nrooms);
    std::vector<void *> ss(nrooms);
    std::vector<int> froom, ffirst{0}, croom, cfirst{0}, oroom, ofirst{0}, hroom, hfirst{0};
    std::vector<OpenItem> oitems;
    std::vector<HeatItem> hitems;
    for (int r = 0; r < nrooms; r++) {
        ffr_fluid *s = rooms[r];
        br[r] = room_step_args(s);
        pa[r] = room_pcg_args(s);
        ss[r] = s->split_state;
        b->any_thermal |= s->prm.thermal != 0;
        b->max_iter = std::max(b->max_iter, s->prm.poisson_max_iter);
        for (unsigned k = 0; k < s->blocks_faces; k++) froom.push_back(r);
        ffirst.push_back((int)froom.size());
        for (unsigned k = 0; k < s->blocks_cells; k++) croom.push_back(r);
        cfirst.push_back((int)croom.size());
        if (s->prm.thermal) {
            for (const ffr_patch &op : s->room.patches) {
                if (!op.is_opening) continue;
                const int it = (int)oitems.size();
                oitems.push_back(OpenItem{r, 0, op});
                const unsigned nb = stream_blocks((long long)(op.a_max - op.a_min + 1) * (op.b_max - op.b_min + 1));
                for (unsigned k = 0; k < nb; k++) oroom.push_back(it);
                ofirst.push_back((int)oroom.size());
            }
        }
        for (const ffr_heat_patch &h : s->room.heats) {
            const int it = (int)hitems.size();
            hitems.push_back(HeatItem{r, 0, h});
            const unsigned nb = stream_blocks((long long)(h.i_max - h.i_min + 1) * (h.j_max - h.j_min + 1) *
                                              (h.k_max - h.k_min + 1));
            for (unsigned k = 0; k < nb; k++) hroom.push_back(it);
            hfirst.push_back((int)hroom.size());
        }
    }
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t bytes = al(sizeof(BRoom) * nrooms) + al(4 * (froom.size() + ffirst.size())) +
                         al(4 * (croom.size() + cfirst.size())) + al(4 * (oroom.size() + ofirst.size())) +
                         al(4 * (hroom.size() + hfirst.size())) + al(sizeof(OpenItem) * (oitems.size() + 1)) +
                         al(sizeof(HeatItem) * (hitems.size() + 1));
    std::vector<unsigned char> host(bytes, 0);
    if (bytes > b->cap) {
        if (b->dev) cudaFree(b->dev);
        b->dev = nullptr;
        b->cap = 0;
        if (cudaMalloc(&b->dev, bytes + bytes / 2) != cudaSuccess) return fail(FFR_ENOMEM, "batch tables");
        b->cap = bytes + bytes / 2;
    }
    unsigned char *d = static_cast<unsigned char *>(b->dev);
    size_t off = 0;
    auto put = [&](const void *src, size_t len) -> unsigned char * {
        if (len) std::memcpy(host.data() + off, src, len);
        unsigned char *p = d + off;
        off += al(len);
        return p;
    };
    auto put_map = [&](const std::vector<int> &room, const std::vector<int> &first, BMap &m) {
        std::vector<int> both(room);
        both.insert(both.end(), first.begin(), first.end());
        const int *p = reinterpret_cast<const int *>(put(both.data(), 4 * both.size()));
        m.room = p;
        m.first = p + room.size();
        return (unsigned)room.size();
    };
    b->broom = reinterpret_cast<const BRoom *>(put(br.data(), sizeof(BRoom) * nrooms));
    b->nb_faces = put_map(froom, ffirst, b->faces);
    b->nb_cells = put_map(croom, cfirst, b->cells);
    b->nb_open = put_map(oroom, ofirst, b->openm);
    b->nb_heat = put_map(hroom, hfirst, b->heatm);
    oitems.push_back(OpenItem{});
    hitems.push_back(HeatItem{});
    b->open = reinterpret_cast<const OpenItem *>(put(oitems.data(), sizeof(OpenItem) * oitems.size()));
    b->heat = reinterpret_cast<const HeatItem *>(put(hitems.data(), sizeof(HeatItem) * hitems.size()));
    FFR_CUDA(cudaMemcpy(b->dev, host.data(), bytes, cudaMemcpyHostToDevice));
    const int rc = batch_split_build(b->split, pa, ss);
    if (rc == FFR_OK) b->stale = false;
    return rc;
}

int ffr_batch_create(ffr_fluid *const *rooms, int nrooms, ffr_batch **out)
{
    if (!out || nrooms <= 0 || !rooms) return fail(FFR_EINVAL, "bad arguments");
    *out = nullptr;
    ffr_batch *b = new (std::nothrow) ffr_batch();
    if (!b) return fail(FFR_ENOMEM, "host allocation");
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess) {
        batch_free(b);
        return fail(FFR_ECUDA, "batch stream");
    }
    int rc = ffr_batch_set_rooms(b, rooms, nrooms);
    if (rc) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return FFR_OK;
}

int ffr_batch_destroy(ffr_batch *b)
{
    batch_free(b);
    return FFR_OK;
}

int ffr_batch_size(const ffr_batch *b, int *nrooms)
{
    if (!b || !nrooms) return fail(FFR_EINVAL, "NULL argument");
    *nrooms = (int)b->rooms.size();
    return FFR_OK;
}

}  // extern "C"

namespace {

// One batched step: every stage one launch for all rooms.  capturing: the
// pressure solve is recorded as a WHILE node (the batch stream is being
// captured), else it is paced by the host.
int batch_enqueue_step(ffr_batch *b, bool capturing)
{
    cudaStream_t st = b->stream;
    const int n = (int)b->rooms.size();
    k_b_predict<<<b->nb_faces, kThreads, 0, st>>>(b->broom, b->faces);
    FFR_LAUNCHED(1);
    int rc = b->cluster_ctas > 0 ? launch_batch_cluster(b->split, st, b->cluster_ctas)
             : capturing           ? capture_batch_split(b->split, st, b->body_stream)
                                   : batch_split_solve(b->split, st, b->max_iter);
    if (rc) return rc;
    k_b_correct<<<b->nb_cells, kThreads, 0, st>>>(b->broom, b->cells);
    FFR_LAUNCHED(1);
    if (b->any_thermal) {
        if (b->nb_open) {
            k_b_opening<<<b->nb_open, kThreads, 0, st>>>(b->broom, b->open, b->openm, 0);
            FFR_LAUNCHED(1);
        }
        k_b_advect_T<<<b->nb_cells, kThreads, 0, st>>>(b->broom, b->cells);
        FFR_LAUNCHED(1);
        if (b->nb_open) {
            k_b_opening<<<b->nb_open, kThreads, 0, st>>>(b->broom, b->open, b->openm, 1);
            FFR_LAUNCHED(1);
        }
    }
    if (b->nb_heat) {
        k_b_heat<<<b->nb_heat, kThreads, 0, st>>>(b->broom, b->heat, b->heatm);
        FFR_LAUNCHED(1);
    }
    k_b_finalize<<<n, kThreads, 0, st>>>(b->broom);
    FFR_LAUNCHED(1);
    return FFR_OK;
}

int batch_capture(ffr_batch *b)
{
    if (!b->body_stream) FFR_CUDA(cudaStreamCreateWithFlags(&b->body_stream, cudaStreamNonBlocking));
    const unsigned long long l0 = ffr_launch_count();
    FFR_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
    int rc = batch_enqueue_step(b, true);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(batched step)");
    e = cudaGraphInstantiate(&b->graph_exec, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(e, "cudaGraphInstantiate(batched step)");
    }
    b->graph = g;
    b->graph_launches = (unsigned)(ffr_launch_count() - l0);
    return FFR_OK;
}

}  // namespace

extern "C" {

int ffr_batch_use_graph(ffr_batch *b, int enable)
{
    if (!b) return fail(FFR_EINVAL, "NULL batch");
    b->use_graph = enable != 0;
    return FFR_OK;
}

int ffr_batch_enqueue(ffr_batch *b, int nsteps, int stop_on_converge)
{
    if (!b || nsteps < 0 || nsteps > kRing) return fail(FFR_EINVAL, "bad handle or nsteps (0..1024)");
    if (b->stale)
        return fail(FFR_EINVAL, "the batch has no valid members (a member was destroyed, or setting the "
                                "members failed): set the batch's rooms again");
    cudaStream_t st = b->stream;
    for (ffr_fluid *s : b->rooms) {
        if (s->pending) return fail(FFR_EINVAL, "a room has a queued chunk that was not polled");
        // the batch stream follows everything queued on the room's own stream
        FFR_CUDA(cudaEventRecord(b->ev, s->stream));
        FFR_CUDA(cudaStreamWaitEvent(st, b->ev, 0));
        s->p0_valid = false;      // batched steps keep no starting pressure
    }
    const int n = (int)b->rooms.size();
    if (b->use_graph && nsteps > 0 && !b->graph_exec) {
        int rc = batch_capture(b);
        if (rc) return rc;
    }
    k_b_begin<<<1, 256, 0, st>>>(b->broom, n, stop_on_converge ? 1 : 0);
    FFR_LAUNCHED(1);
    for (int k = 0; k < nsteps; k++) {
        if (b->use_graph) {
            FFR_CUDA(cudaGraphLaunch(b->graph_exec, st));
            count_launch(b->graph_launches);
            continue;
        }
        int rc = batch_enqueue_step(b, false);
        if (rc) return rc;
    }
    // each room's results as ffr_fluid_enqueue leaves them, for ffr_fluid_poll
    for (ffr_fluid *s : b->rooms) {
        if (nsteps > 0)
            FFR_CUDA(cudaMemcpyAsync(s->ring_host, s->ring, sizeof(ffr_step_result) * nsteps,
                                     cudaMemcpyDeviceToHost, st));
        FFR_CUDA(cudaMemcpyAsync(s->st_host, s->st, sizeof(StepState), cudaMemcpyDeviceToHost, st));
        FFR_CUDA(cudaEventRecord(s->done_ev, st));
        FFR_CUDA(cudaStreamWaitEvent(s->stream, s->done_ev, 0));
        s->pending = nsteps > 0 ? nsteps : -1;
    }
    return FFR_OK;
}

}  // extern "C"

// ----------------------------------------------------- poisson handle

struct ffr_poisson {
    HostRoom room;
    cudaStream_t stream = nullptr;
    Arena arena;
    RoomTables tab;
    RoomDev R;
    int max_iter;
    double tol;
    double *r, *da, *db, *ad, *partials, *res, *x_tmp, *b_tmp;
    int *iters, *flags;
    GridSync *gs;
    CGScalars *sc;
    unsigned blocks;
    HostStage stage;
};

extern "C" {

int ffr_poisson_create(const ffr_room_desc *room, int max_iter, double tol, ffr_poisson **out)
{
    if (!out) return fail(FFR_EINVAL, "NULL out");
    *out = nullptr;
    if (max_iter < 0) return fail(FFR_EINVAL, "negative max_iter");
    ffr_poisson *s = new (std::nothrow) ffr_poisson();
    if (!s) return fail(FFR_ENOMEM, "host allocation");
    int rc = load_room(room, s->room);
    if (rc) { delete s; return rc; }
    s->max_iter = max_iter;
    s->tol = tol;
    const RoomGeom &g = s->room.g;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return fail(FFR_ECUDA, "cudaStreamCreate");
    }
    s->blocks = std::max(1u, std::min(cg_max_blocks(), (unsigned)((g.n + kThreads - 1) / kThreads)));
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t bytes = tables_bytes(s->room) + 6 * al(8 * g.n) + al(8 * s->blocks * 4) +
                         al(sizeof(GridSync)) + al(sizeof(CGScalars)) + 4 * 256;
    rc = s->arena.alloc(bytes);
    if (rc) { cudaStreamDestroy(s->stream); delete s; return rc; }
    rc = carve_tables(s->room, s->arena, s->tab, s->R);
    if (!rc) rc = upload_cell_types(s->room, s->tab, s->stream);
    if (!rc) rc = s->stage.reserve(tables_stage_bytes(s->room));
    if (!rc) rc = queue_tables(s->room, s->tab, s->stage, s->stream);
    Arena &a = s->arena;
    s->r = a.take<double>(g.n); s->da = a.take<double>(g.n); s->db = a.take<double>(g.n);
    s->ad = a.take<double>(g.n); s->x_tmp = a.take<double>(g.n); s->b_tmp = a.take<double>(g.n);
    s->partials = a.take<double>(s->blocks * 4);
    s->gs = a.take<GridSync>(1);
    s->sc = a.take<CGScalars>(1);
    s->res = a.take<double>(1);
    s->iters = a.take<int>(1);
    s->flags = a.take<int>(1);
    if (rc || !s->flags || s->arena.failed) {
        if (!rc) rc = fail(FFR_ENOMEM, "arena exhausted");
        ffr_poisson_destroy(s);
        return rc;
    }
    // a solve may run on the caller's stream: the set-up must be complete
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
        ffr_poisson_destroy(s);
        return fail(FFR_ECUDA, "poisson set-up");
    }
    *out = s;
    return FFR_OK;
}

int ffr_poisson_destroy(ffr_poisson *s)
{
    if (!s) return FFR_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    s->stage.release();
    s->arena.release();
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FFR_OK;
}

int ffr_poisson_solve_dev(ffr_poisson *s, const double *rhs_dev, double *p_dev, void *stream,
                          double *residual, int *iterations)
{
    if (!s || !rhs_dev || !p_dev) return fail(FFR_EINVAL, "NULL argument");
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    CGArgs ca{};
    ca.R = s->R;
    ca.from_faces = 0;
    ca.rhs = rhs_dev;
    ca.x = p_dev; ca.r = s->r; ca.da = s->da; ca.db = s->db; ca.ad = s->ad;
    ca.partials = s->partials; ca.gs = s->gs; ca.sc = s->sc;
    ca.max_iter = s->max_iter; ca.tol = s->tol;
    ca.st = nullptr;
    ca.out_res = s->res; ca.out_iters = s->iters; ca.out_flags = s->flags;
    int rc = launch_cg(ca, s->blocks, st);
    if (rc) return rc;
    double res = 0.0;
    int it = 0, fl = 0;
    FFR_CUDA(cudaMemcpyAsync(&res, s->res, 8, cudaMemcpyDeviceToHost, st));
    FFR_CUDA(cudaMemcpyAsync(&it, s->iters, 4, cudaMemcpyDeviceToHost, st));
    FFR_CUDA(cudaMemcpyAsync(&fl, s->flags, 4, cudaMemcpyDeviceToHost, st));
    FFR_CUDA(cudaStreamSynchronize(st));
    if (residual) *residual = res;
    if (iterations) *iterations = it;
    if (fl & FFR_FLAG_TIMEOUT) return fail(FFR_ETIMEDOUT, "pressure-solve grid barrier timed out");
    return FFR_OK;
}

int ffr_poisson_solve(ffr_poisson *s, const double *rhs, double *p, double *residual,
                      int *iterations)
{
    if (!s || !rhs || !p) return fail(FFR_EINVAL, "NULL argument");
    const long long n = s->room.g.n;
    FFR_CUDA(cudaMemcpyAsync(s->b_tmp, rhs, 8 * n, cudaMemcpyHostToDevice, s->stream));
    int rc = ffr_poisson_solve_dev(s, s->b_tmp, s->x_tmp, nullptr, residual, iterations);
    if (rc) return rc;
    FFR_CUDA(cudaMemcpyAsync(p, s->x_tmp, 8 * n, cudaMemcpyDeviceToHost, s->stream));
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    return FFR_OK;
}

}  // extern "C"

namespace ffr {
// y = L x with the CG stencil (used by ffr_poisson_apply).
__global__ void k_apply_stencil(RoomDev R, const double *x, double *y)
{
    const int nx = R.nx, ny = R.ny, nz = R.nz, plane = ny * nz;
    const double *sxl = R.scale, *sxr = sxl + nx, *syl = sxr + nx, *syr = syl + ny, *szl = syr + ny,
                 *szr = szl + nz;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < R.n; c += gridDim.x * blockDim.x) {
        const unsigned code = R.sc[c];
        if (code & SC_SOLID) { y[c] = x[c]; continue; }
        const int i = c / plane, rem = c - i * plane, j = rem / nz, k = rem - j * nz;
        double diag = 0.0, off = 0.0;
        if ((code >> 0) & 3) stencil_term((code >> 0) & 3, sxl[i], ((code >> 0) & 3) == SC_IN ? x[c - plane] : 0.0, diag, off);
        if ((code >> 2) & 3) stencil_term((code >> 2) & 3, sxr[i], ((code >> 2) & 3) == SC_IN ? x[c + plane] : 0.0, diag, off);
        if ((code >> 4) & 3) stencil_term((code >> 4) & 3, syl[j], ((code >> 4) & 3) == SC_IN ? x[c - nz] : 0.0, diag, off);
        if ((code >> 6) & 3) stencil_term((code >> 6) & 3, syr[j], ((code >> 6) & 3) == SC_IN ? x[c + nz] : 0.0, diag, off);
        if ((code >> 8) & 3) stencil_term((code >> 8) & 3, szl[k], ((code >> 8) & 3) == SC_IN ? x[c - 1] : 0.0, diag, off);
        if ((code >> 10) & 3) stencil_term((code >> 10) & 3, szr[k], ((code >> 10) & 3) == SC_IN ? x[c + 1] : 0.0, diag, off);
        if (diag < 1e-30) diag = 1.0;
        y[c] = diag * x[c] - off;
    }
}
}  // namespace ffr

extern "C" int ffr_poisson_apply(ffr_poisson *s, const double *x, double *ax)
{
    if (!s || !x || !ax) return fail(FFR_EINVAL, "NULL argument");
    const long long n = s->room.g.n;
    FFR_CUDA(cudaMemcpyAsync(s->b_tmp, x, 8 * n, cudaMemcpyHostToDevice, s->stream));
    k_apply_stencil<<<stream_blocks(n), kThreads, 0, s->stream>>>(s->R, s->b_tmp, s->x_tmp);
    FFR_LAUNCHED(1);
    FFR_CUDA(cudaMemcpyAsync(ax, s->x_tmp, 8 * n, cudaMemcpyDeviceToHost, s->stream));
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    return FFR_OK;
}
