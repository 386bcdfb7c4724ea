// lbm.cu — D3Q19 BGK lattice Boltzmann, fused pull-stream/collide (sm_100a).
//
// The reference step (LBMSolver::step, cpp/src/core/LBMSolver.cpp:402-440)
// is inflow BC -> collision -> push streaming with halfway bounce-back into
// a zeroed buffer -> outflow copy -> macroscopic extraction.  Here the state
// kept between steps is the post-collision population f* of every cell, in
// two A/B buffers.  One kernel per step
//   1. pulls, for every non-SOLID cell x and direction q, what the
//      reference's push delivers into slot q of x: f*_q(x - e_q) when that
//      cell is in the domain and not SOLID, plus f*_OPP[q](x) when x's own
//      direction OPP[q] is blocked (outside the domain or SOLID);
//   2. for OUTFLOW cells first redirects x to the cell whose post-stream
//      populations the reference's outflow copies leave there (the chain of
//      copies is resolved on the host, in the reference's patch order);
//   3. takes the moments (the reference's extract_macroscopic input) and
//      writes the cell velocity and p = rho*cs^2;
//   4. applies the next step's inflow BC / BGK collision and stores f*.
// A second kernel forms the face velocities, max |du| and max |div|.
//
// Storage modes: FP64 (the reference arithmetic), FP32 and FP16.  The
// narrow modes store the shifted populations g_q = f_q - w_q (the "DDF
// shifting" of Lehmann, Krause, Amati, Sega, Harting & Gekle, Phys. Rev. E
// 106, 015308 (2022)) and collide in FP32.
#include "common.cuh"

#include <cuda_fp16.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <unordered_map>
#include <type_traits>

namespace ffr {

// D3Q19 velocities and opposites (LBMSolver.cpp:11-27) as compile-time
// functions: in the unrolled q loops every e_q folds into the arithmetic
// (an add, a subtract or nothing) instead of a load and a conversion.
//   e_x = +1 for q in {1,7,9,11,13}, -1 for {2,8,10,12,14}
//   e_y = +1 for q in {3,7,8,15,17}, -1 for {4,9,10,16,18}
//   e_z = +1 for q in {5,11,12,15,16}, -1 for {6,13,14,17,18}
__host__ __device__ constexpr int lbm_sign(unsigned plus, unsigned minus, int q)
{
    return (int)((plus >> q) & 1u) - (int)((minus >> q) & 1u);
}
__host__ __device__ constexpr int c_ex(int q) { return lbm_sign(0x2A82u, 0x5504u, q); }
__host__ __device__ constexpr int c_ey(int q) { return lbm_sign(0x28188u, 0x50610u, q); }
__host__ __device__ constexpr int c_ez(int q) { return lbm_sign(0x19820u, 0x66040u, q); }
// OPP pairs q with q+1 for odd q (1<->2, 3<->4, ..., 17<->18)
__host__ __device__ constexpr int c_opp(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }
// the direction -e_q (not OPP[q] for the diagonals)
__host__ __device__ constexpr int c_rev(int q)
{
    int r = 0;
    for (int p = 0; p < 19; p++)
        if (c_ex(p) == -c_ex(q) && c_ey(p) == -c_ey(q) && c_ez(p) == -c_ez(q)) r = p;
    return r;
}
static_assert(c_rev(7) == 10 && c_rev(8) == 9 && c_rev(11) == 14 && c_rev(12) == 13 && c_rev(15) == 18 &&
                  c_rev(16) == 17 && c_rev(1) == 2 && c_rev(0) == 0,
              "D3Q19 reverse directions");

// e_q . (ux, uy, uz) over the non-zero components, in the order x, y, z
// (the zero terms of the reference's sum add a signed zero only).
template <class F>
__device__ __forceinline__ F edot(int q, F ux, F uy, F uz)
{
    F s = F(0);
    bool any = false;
    if (c_ex(q)) { s = c_ex(q) > 0 ? ux : -ux; any = true; }
    if (c_ey(q)) { s = any ? (c_ey(q) > 0 ? s + uy : s - uy) : (c_ey(q) > 0 ? uy : -uy); any = true; }
    if (c_ez(q)) { s = any ? (c_ez(q) > 0 ? s + uz : s - uz) : (c_ez(q) > 0 ? uz : -uz); }
    return s;
}

// rho, j += f_q (1, e_q) without the zero products
template <class F>
__device__ __forceinline__ void add_moments(int q, F f, F &rho, F &jx, F &jy, F &jz)
{
    rho += f;
    if (c_ex(q) > 0) jx += f; else if (c_ex(q) < 0) jx -= f;
    if (c_ey(q) > 0) jy += f; else if (c_ey(q) < 0) jy -= f;
    if (c_ez(q) > 0) jz += f; else if (c_ez(q) < 0) jz -= f;
}

// D3Q19 weights (LBMSolver.cpp:19-25).
__host__ __device__ __forceinline__ double lbm_w(int q)
{
    return q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
}

// LBMSolver::feq (LBMSolver.hpp:89-93), cs2 = 1/3, in the reference's
// operation order, except that the divisions by cs2, 2 cs2^2 and 2 cs2 are
// multiplications by their FP64 reciprocals (each term within one rounding
// of the reference's quotient).
__device__ __forceinline__ double feq64(int q, double rho, double ux, double uy, double uz)
{
    const double cs2 = 1.0 / 3.0;
    const double r1 = 1.0 / cs2, r2 = 1.0 / (2.0 * cs2 * cs2), r3 = 1.0 / (2.0 * cs2);
    const double eu = edot<double>(q, ux, uy, uz);
    const double usq = ux * ux + uy * uy + uz * uz;
    return lbm_w(q) * rho * (1.0 + eu * r1 + eu * eu * r2 - usq * r3);
}

// Shifted equilibrium feq_q - w_q in FP32 for rho = 1 + drho.
__device__ __forceinline__ float geq32(int q, float drho, float ux, float uy, float uz)
{
    const float eu = edot<float>(q, ux, uy, uz);
    const float usq = ux * ux + uy * uy + uz * uz;
    const float rho = 1.0f + drho;
    return (float)lbm_w(q) * (drho + rho * (3.0f * eu + 4.5f * eu * eu - 1.5f * usq));
}

template <int MODE> struct Store;
template <> struct Store<0> {
    using T = double;
    __device__ static double ld(const double *p) { return *p; }
    __device__ static void st(double *p, double v) { *p = v; }
};
template <> struct Store<1> {
    using T = float;
    __device__ static float ld(const float *p) { return *p; }
    __device__ static void st(float *p, float v) { *p = v; }
};
template <> struct Store<2> {
    using T = __half;
    __device__ static float ld(const __half *p) { return __half2float(*p); }
    __device__ static void st(__half *p, float v) { *p = __float2half_rn(v); }
};

// Per-cell flags of the step kernel (besides the cell type in bits 0-1).
enum : uint8_t { LF_OPEN = 4,    // all 18 neighbours in the domain and not SOLID
                 LF_REMAP = 8 }; // OUTFLOW cell whose populations come from another cell

struct LbmDev {
    int nx, ny, nz, n, nu, nv, nw;
    const uint8_t *ct;          // cell types
    const uint8_t *fl;          // cell type | LF_* flags
    const uint32_t *blk;        // bit q: x + e_q outside the room or SOLID (non-open cells)
    const uint8_t *fan_of;      // fan index of each INFLOW cell (255: none)
    const double *fan_lat;      // lattice fan velocity, 3 per fan
    const int *remap_dst;       // sorted OUTFLOW destinations
    const int *remap_src;       // their resolved source cells
    int nremap;
    const double *dxv, *dyv, *dzv;
    const double *idxv, *idyv, *idzv;   // 1 / spacing (the per-step divergence)
    double tau, l2p;
};

struct LbmState {
    int step, halt, stop_on_converge, par;
    unsigned long long dmax_bits, div_bits;
    int ring_slot, flags;
};

__device__ __forceinline__ int find_src(const LbmDev &L, int c)
{
    int lo = 0, hi = L.nremap - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int d = L.remap_dst[mid];
        if (d == c) return L.remap_src[mid];
        if (d < c) lo = mid + 1; else hi = mid - 1;
    }
    return c;
}

// Cell-centred velocity between the step and face kernels: FP64 with FP64
// populations, FP32 with the narrow storage modes (their collision is FP32).
template <int MODE> using CellVel = typename std::conditional<MODE == 0, double, float>::type;

// One fused step; see the file comment.  fa = f* of this step, fb = f* of
// the next, cu/cv/cw = cell-centred velocity (m/s), p = rho*cs^2.
template <int MODE>
__global__ void __launch_bounds__(256, MODE == 0 ? 3 : 4)
    k_lbm_step(LbmDev L, const typename Store<MODE>::T *f0, typename Store<MODE>::T *f1,
               CellVel<MODE> *__restrict__ cu, CellVel<MODE> *__restrict__ cv, CellVel<MODE> *__restrict__ cw,
               double *__restrict__ p, const LbmState *st)
{
    using S = Store<MODE>;
    using T = typename S::T;
    if (st->halt) return;
    const T *__restrict__ fa = st->par ? f1 : f0;
    T *__restrict__ fb = st->par ? (T *)f0 : f1;
    const int ny = L.ny, nz = L.nz, n = L.n, plane = ny * nz;
    // The flags and blocked-direction mask of the next cell are loaded while
    // this cell's populations are in flight, so each cell waits for one
    // round trip to memory only.
    const int c0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    uint8_t fl = 0, fln = 0;
    unsigned Bc = 0, Bn = 0;
    // (interior cells have no blocked direction and skip the mask load)
    if (c0 < n) { fl = L.fl[c0]; Bc = (fl & LF_OPEN) ? 0u : L.blk[c0]; }
    for (int c = c0; c < n; c += stride, fl = fln, Bc = Bn) {
        if (c + stride < n) {
            fln = L.fl[c + stride];
            Bn = (fln & LF_OPEN) ? 0u : L.blk[c + stride];
        }
        const uint8_t t = fl & 3;
        if (t == CT_SOLID) {
            cu[c] = 0; cv[c] = 0; cw[c] = 0;
            continue;
        }
        using C = typename std::conditional<MODE == 0, double, float>::type;
        C fq[19];
        // x: the cell whose post-stream populations this cell ends with
        const int o = (fl & LF_REMAP) ? find_src(L, c) : c;
        if ((fl & LF_REMAP) && L.ct[o] == CT_SOLID) {
#pragma unroll
            for (int q = 0; q < 19; q++) fq[q] = MODE == 0 ? C(0) : C(-lbm_w(q));
        } else {
            // blocked directions of x (bit q: x + e_q outside the room or
            // SOLID; 0 for an interior cell).  Slot q receives
            //  (a) f*_q(x - e_q) when x - e_q = x + e_{-q} is not blocked;
            //  (b) f*_OPP[q](x) when x's own direction OPP[q] is blocked.
            // OPP of LBMSolver.cpp:27 pairs the diagonals as mirror images
            // (7 <-> 8 is (1,1,0) <-> (-1,1,0)), so (a) and (b) are
            // independent and a slot gets 0, 1 or 2 values.
            const unsigned B = (fl & LF_REMAP) ? L.blk[o] : Bc;
            // (a) for every slot, unconditionally: a blocked source reads the
            // cell's own slot instead (a valid address) and is replaced below
#pragma unroll
            for (int q = 0; q < 19; q++) {
                const int s = o - (c_ex(q) * plane + c_ey(q) * nz + c_ez(q));
                fq[q] = C(S::ld(fa + (q * n + (((B >> c_rev(q)) & 1u) ? o : s))));
            }
            if (B) {
                // cells next to a wall or SOLID: drop blocked sources, add (b)
#pragma unroll
                for (int q = 0; q < 19; q++) {
                    const int qq = c_opp(q);
                    const bool ina = !((B >> c_rev(q)) & 1u);
                    const bool inb = (B >> qq) & 1u;
                    const C va = fq[q];
                    const C vb = inb ? C(S::ld(fa + (qq * n + o))) : C(0);
                    if (MODE == 0) {
                        // the reference's zeroed slot plus what arrives
                        fq[q] = ina ? (inb ? va + vb : va) : vb;
                    } else {
                        // shifted storage g = f - w (w_q == w_OPP[q]): two
                        // arrivals give g_a + g_b + w, none gives -w
                        fq[q] = ina ? (inb ? va + vb + C(lbm_w(q)) : va) : (inb ? vb : C(-lbm_w(q)));
                    }
                }
            }
        }
        // moments (LBMSolver.cpp:306-318) and next-step collision
        if (MODE == 0) {
            double rho = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
#pragma unroll
            for (int q = 0; q < 19; q++) add_moments<double>(q, fq[q], rho, ux, uy, uz);
            if (rho > 1e-14) { ux /= rho; uy /= rho; uz /= rho; }
            cu[c] = ux * L.l2p; cv[c] = uy * L.l2p; cw[c] = uz * L.l2p;
            p[c] = rho * (1.0 / 3.0);
            if (t == CT_INFLOW && L.fan_of[c] != 255) {
                const double *fv = L.fan_lat + 3 * L.fan_of[c];
#pragma unroll
                for (int q = 0; q < 19; q++) S::st(fb + (q * n + c), feq64(q, 1.0, fv[0], fv[1], fv[2]));
            } else if (t == CT_INFLOW) {
#pragma unroll
                for (int q = 0; q < 19; q++) S::st(fb + (q * n + c), fq[q]);
            } else {
                const double itau = 1.0 / L.tau;
#pragma unroll
                for (int q = 0; q < 19; q++) {
                    const double fe = feq64(q, rho, ux, uy, uz);
                    S::st(fb + (q * n + c), fq[q] + itau * (fe - fq[q]));
                }
            }
        } else {
            float drho = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
#pragma unroll
            for (int q = 0; q < 19; q++) add_moments<float>(q, fq[q], drho, jx, jy, jz);
            const float rho = 1.0f + drho;
            float ux = jx, uy = jy, uz = jz;
            if (rho > 1e-14f) { ux /= rho; uy /= rho; uz /= rho; }
            cu[c] = (float)((double)ux * L.l2p);
            cv[c] = (float)((double)uy * L.l2p);
            cw[c] = (float)((double)uz * L.l2p);
            p[c] = (double)rho * (1.0 / 3.0);
            if (t == CT_INFLOW && L.fan_of[c] != 255) {
                const double *fv = L.fan_lat + 3 * L.fan_of[c];
#pragma unroll
                for (int q = 0; q < 19; q++)
                    S::st(fb + (q * n + c), geq32(q, 0.0f, (float)fv[0], (float)fv[1], (float)fv[2]));
            } else if (t == CT_INFLOW) {
#pragma unroll
                for (int q = 0; q < 19; q++) S::st(fb + (q * n + c), fq[q]);
            } else {
                const float itau = (float)(1.0 / L.tau);
#pragma unroll
                for (int q = 0; q < 19; q++) {
                    const float ge = geq32(q, drho, ux, uy, uz);
                    S::st(fb + (q * n + c), fq[q] + itau * (ge - fq[q]));
                }
            }
        }
    }
}

// Initial f* : f = w_q (LBMSolver.cpp:65-74), INFLOW cells feq(1, u_fan)
// (apply_inflow_bc, LBMSolver.cpp:80-99), then the first collision.
template <int MODE>
__global__ void k_lbm_init(LbmDev L, typename Store<MODE>::T *f)
{
    using S = Store<MODE>;
    const int n = L.n;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const uint8_t t = L.ct[c];
        if (MODE == 0) {
            double fq[19];
            const bool fan = t == CT_INFLOW && L.fan_of[c] != 255;
            const double *fv = fan ? L.fan_lat + 3 * L.fan_of[c] : nullptr;
#pragma unroll
            for (int q = 0; q < 19; q++) fq[q] = fan ? feq64(q, 1.0, fv[0], fv[1], fv[2]) : lbm_w(q);
            if (t == CT_FLUID || t == CT_OUTFLOW) {
                double rho = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
                for (int q = 0; q < 19; q++) {
                    rho += fq[q]; ux += fq[q] * c_ex(q); uy += fq[q] * c_ey(q); uz += fq[q] * c_ez(q);
                }
                if (rho > 1e-14) { ux /= rho; uy /= rho; uz /= rho; }
                const double itau = 1.0 / L.tau;
                for (int q = 0; q < 19; q++) fq[q] += itau * (feq64(q, rho, ux, uy, uz) - fq[q]);
            }
#pragma unroll
            for (int q = 0; q < 19; q++) S::st(f + (size_t)q * n + c, fq[q]);
        } else {
            float g[19];
            const bool fan = t == CT_INFLOW && L.fan_of[c] != 255;
            const double *fv = fan ? L.fan_lat + 3 * L.fan_of[c] : nullptr;
#pragma unroll
            for (int q = 0; q < 19; q++)
                g[q] = fan ? geq32(q, 0.0f, (float)fv[0], (float)fv[1], (float)fv[2]) : 0.0f;
            if (t == CT_FLUID || t == CT_OUTFLOW) {
                float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
                for (int q = 0; q < 19; q++) {
                    drho += g[q]; jx += g[q] * c_ex(q); jy += g[q] * c_ey(q); jz += g[q] * c_ez(q);
                }
                const float rho = 1.0f + drho;
                const float itau = (float)(1.0 / L.tau);
                for (int q = 0; q < 19; q++) g[q] += itau * (geq32(q, drho, jx / rho, jy / rho, jz / rho) - g[q]);
            }
#pragma unroll
            for (int q = 0; q < 19; q++) S::st(f + (size_t)q * n + c, g[q]);
        }
    }
}

// Face velocities of extract_macroscopic (LBMSolver.cpp:333-375), max
// |du| against the previous faces (LBMSolver.cpp:423-433) and max |div|
// over FLUID cells (LBMSolver.cpp:382-396), cell-centric like k_correct.
template <class V>
__global__ void __launch_bounds__(256) k_lbm_faces(LbmDev L, const V *__restrict__ cu,
                                                   const V *__restrict__ cv,
                                                   const V *__restrict__ cw, double *__restrict__ u,
                                                   double *__restrict__ v, double *__restrict__ w,
                                                   LbmState *st)
{
    __shared__ double sh[32];
    if (st->halt) return;
    const int nx = L.nx, ny = L.ny, nz = L.nz, plane = ny * nz;
    double dmax = 0.0, divmax = 0.0;
    for (Walk wk(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, ny, nz, L.n); wk.ok(); wk.next()) {
        const int c = wk.c, i = wk.i, j = wk.j, k = wk.k;
        const int uf = c, vf = (i * (ny + 1) + j) * nz + k, wf = (i * ny + j) * (nz + 1) + k;
        // every load first, then the arithmetic, then the stores
        const double cuc = cu[c], cvc = cv[c], cwc = cw[c];
        // neighbours through indices clamped into the arrays (the value is
        // only used when the neighbour exists)
        const int last = L.n - 1;
        const double cum = cu[max(c - plane, 0)], cup = cu[min(c + plane, last)];
        const double cvm = cv[max(c - nz, 0)], cvp = cv[min(c + nz, last)];
        const double cwm = cw[max(c - 1, 0)], cwp = cw[min(c + 1, last)];
        const double uo = u[uf], vo = v[vf], wo = w[wf];
        const double uho = (i == nx - 1) ? u[uf + plane] : 0.0;
        const double vho = (j == ny - 1) ? v[vf + nz] : 0.0;
        const double who = (k == nz - 1) ? w[wf + 1] : 0.0;
        const bool fluid = L.ct[c] == CT_FLUID;
        const double ulo = (i == 0) ? cuc : 0.5 * (cum + cuc);
        const double uhi = (i == nx - 1) ? cuc : 0.5 * (cuc + cup);
        const double vlo = (j == 0) ? cvc : 0.5 * (cvm + cvc);
        const double vhi = (j == ny - 1) ? cvc : 0.5 * (cvc + cvp);
        const double wlo = (k == 0) ? cwc : 0.5 * (cwm + cwc);
        const double whi = (k == nz - 1) ? cwc : 0.5 * (cwc + cwp);
        dmax = fmax(dmax, fabs(ulo - uo));
        dmax = fmax(dmax, fabs(vlo - vo));
        dmax = fmax(dmax, fabs(wlo - wo));
        if (i == nx - 1) dmax = fmax(dmax, fabs(uhi - uho));
        if (j == ny - 1) dmax = fmax(dmax, fabs(vhi - vho));
        if (k == nz - 1) dmax = fmax(dmax, fabs(whi - who));
        if (fluid)
            divmax = fmax(divmax, fabs((uhi - ulo) * L.idxv[i] + (vhi - vlo) * L.idyv[j] + (whi - wlo) * L.idzv[k]));
        u[uf] = ulo;
        v[vf] = vlo;
        w[wf] = wlo;
        if (i == nx - 1) u[uf + plane] = uhi;
        if (j == ny - 1) v[vf + nz] = vhi;
        if (k == nz - 1) w[wf + 1] = whi;
    }
    dmax = block_max(dmax, sh);
    divmax = block_max(divmax, sh);
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&st->dmax_bits, dmax);
        atomic_max_nonneg(&st->div_bits, divmax);
    }
}

__global__ void k_lbm_finalize(double dt, double tol, LbmState *st, ffr_step_result *ring)
{
    if (st->halt || threadIdx.x != 0) return;
    const double vc = __longlong_as_double((long long)st->dmax_bits) / dt;
    ffr_step_result r;
    r.step = st->step + 1;
    r.velocity_change = vc;
    r.pressure_residual = 0.0;
    r.divergence_max = __longlong_as_double((long long)st->div_bits);
    r.converged = vc < tol;
    r.T_mean = 0.0;
    r.cg_iterations = 0;
    r.flags = st->flags;
    ring[st->ring_slot] = r;
    st->ring_slot += 1;
    st->step += 1;
    st->par ^= 1;
    st->dmax_bits = 0;
    st->div_bits = 0;
    st->flags = 0;
    if (r.converged && st->stop_on_converge) st->halt = 1;
}

__global__ void k_lbm_divergence(LbmDev L, const double *u, const double *v, const double *w,
                                 unsigned long long *out)
{
    __shared__ double sh[32];
    const int ny = L.ny, nz = L.nz, plane = ny * nz;
    double m = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < L.n; c += gridDim.x * blockDim.x) {
        if (L.ct[c] != CT_FLUID) continue;
        const int i = c / plane, rem = c - i * plane, j = rem / nz, k = rem - j * nz;
        const int vf = (i * (ny + 1) + j) * nz + k, wf = (i * ny + j) * (nz + 1) + k;
        m = fmax(m, fabs((u[c + plane] - u[c]) / L.dxv[i] + (v[vf + nz] - v[vf]) / L.dyv[j] +
                         (w[wf + 1] - w[wf]) / L.dzv[k]));
    }
    m = block_max(m, sh);
    if (threadIdx.x == 0) atomic_max_nonneg(out, m);
}

// ------------------------------------------------------- set-up kernels

// Step-kernel flags and blocked-direction masks from the cell types: bit q
// of blocked[c] is set when x + e_q is outside the grid or SOLID (halfway
// bounce-back, LBMSolver.cpp:151-190); LF_OPEN marks a non-SOLID cell with
// no blocked direction.  Re-mapped OUTFLOW cells are flagged afterwards
// (k_lbm_remap_flags).
__global__ void k_lbm_flags(const uint8_t *__restrict__ ct, int nx, int ny, int nz, uint8_t *__restrict__ flags,
                            uint32_t *__restrict__ blocked)
{
    const int n = nx * ny * nz, plane = ny * nz;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c / plane, rem = c - i * plane, j = rem / nz, k = rem - j * nz;
        uint32_t bl = 0;
#pragma unroll
        for (int q = 1; q < 19; q++) {
            const int a = i + c_ex(q), b = j + c_ey(q), e = k + c_ez(q);
            const bool ok = a >= 0 && a < nx && b >= 0 && b < ny && e >= 0 && e < nz &&
                            ct[(a * ny + b) * nz + e] != CT_SOLID;
            if (!ok) bl |= 1u << q;
        }
        blocked[c] = bl;
        const uint8_t t = ct[c];
        flags[c] = (uint8_t)(t | ((t != CT_SOLID && bl == 0) ? LF_OPEN : 0));
    }
}

// OUTFLOW cells that take their populations from another cell: the cell
// type plus LF_REMAP, never LF_OPEN.
__global__ void k_lbm_remap_flags(const uint8_t *__restrict__ ct, const int *__restrict__ dst, int m,
                                  uint8_t *__restrict__ flags)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x)
        flags[dst[t]] = (uint8_t)(ct[dst[t]] | LF_REMAP);
}

// Fan index of the INFLOW cells of one fan's box; fans are applied in
// order, so the last fan whose box holds a cell wins.
__global__ void k_lbm_fan_of(const uint8_t *__restrict__ ct, int nx, int ny, int nz, ffr_fan fn, uint8_t f,
                             uint8_t *__restrict__ fan_of)
{
    const int i0 = max(0, fn.i_min), j0 = max(0, fn.j_min), k0 = max(0, fn.k_min);
    const int bi = min(nx - 1, fn.i_max) - i0 + 1, bj = min(ny - 1, fn.j_max) - j0 + 1,
              bk = min(nz - 1, fn.k_max) - k0 + 1;
    const long long cells = (long long)bi * bj * bk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = i0 + (int)(t / ((long long)bj * bk)), rem = (int)(t % ((long long)bj * bk));
        const int c = (i * ny + j0 + rem / bk) * nz + k0 + rem % bk;
        if (ct[c] == CT_INFLOW) fan_of[c] = f;
    }
}

// Checkpoint conversion between the stored populations and FP64 f in the
// reference's layout f[q*N + c] (LBMSolver.hpp:77-82): FP64 storage holds f
// itself, the narrow modes the shifted g = f - w_q.  SOLID cells stream
// nothing and their slots of the second buffer are never written; they are
// exported as 0, the value the reference's push streaming leaves in them
// (LBMSolver.cpp:151-190), and never read by a step.
template <int MODE>
__global__ void k_lbm_export(int n, const uint8_t *__restrict__ ct, const typename Store<MODE>::T *__restrict__ f,
                             double *__restrict__ out)
{
    const long long total = 19ll * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(t / n);
        const int c = (int)(t - (long long)q * n);
        double v = 0.0;
        if (ct[c] != CT_SOLID) {
            v = (double)Store<MODE>::ld(f + t);
            if (MODE != 0) v += lbm_w(q);
        }
        out[t] = v;
    }
}

template <int MODE>
__global__ void k_lbm_import(int n, const double *__restrict__ in, typename Store<MODE>::T *__restrict__ f)
{
    const long long total = 19ll * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(t / n);
        const double v = in[t];
        if (MODE == 0) Store<0>::st(reinterpret_cast<double *>(f) + t, v);
        else if (MODE == 1) reinterpret_cast<float *>(f)[t] = (float)(v - lbm_w(q));
        else reinterpret_cast<__half *>(f)[t] = __double2half(v - lbm_w(q));
    }
}

}  // namespace ffr

using namespace ffr;

namespace {
constexpr int kRingL = 1024;
constexpr int kThr = 256;

unsigned blocks_for(long long n)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return (unsigned)std::max<long long>(1, std::min<long long>((long long)sms * 8, (n + kThr - 1) / kThr));
}
}  // namespace

struct ffr_lbm {
    HostRoom room;
    int storage;
    double tau, dt, tol;
    int max_steps;
    cudaStream_t stream = nullptr;
    Arena arena;
    LbmDev L;
    void *f0, *f1;
    double *cu, *cv, *cw, *u, *v, *w, *p;
    LbmState *st, *st_host;
    ffr_step_result *ring, *ring_host;
    unsigned long long *div_slot;
    unsigned blocks;
    GroupTimer prof;
};

namespace {

int lbm_enqueue(ffr_lbm *s)
{
    cudaStream_t st = s->stream;
    s->prof.begin(FFR_LPROF_STREAM_COLLIDE, st);
    switch (s->storage) {
    case FFR_LBM_FP64:
        k_lbm_step<0><<<s->blocks, kThr, 0, st>>>(s->L, (const double *)s->f0, (double *)s->f1,
                                                    (CellVel<0> *)s->cu, (CellVel<0> *)s->cv,
                                                    (CellVel<0> *)s->cw, s->p, s->st);
        break;
    case FFR_LBM_FP32:
        k_lbm_step<1><<<s->blocks, kThr, 0, st>>>(s->L, (const float *)s->f0, (float *)s->f1,
                                                    (CellVel<1> *)s->cu, (CellVel<1> *)s->cv,
                                                    (CellVel<1> *)s->cw, s->p, s->st);
        break;
    default:
        k_lbm_step<2><<<s->blocks, kThr, 0, st>>>(s->L, (const __half *)s->f0, (__half *)s->f1,
                                                    (CellVel<2> *)s->cu, (CellVel<2> *)s->cv,
                                                    (CellVel<2> *)s->cw, s->p, s->st);
    }
    FFR_LAUNCHED(1);
    s->prof.end(st, 1);
    s->prof.begin(FFR_LPROF_FACES, st);
    if (s->storage == FFR_LBM_FP64)
        k_lbm_faces<double><<<s->blocks, kThr, 0, st>>>(s->L, s->cu, s->cv, s->cw, s->u, s->v, s->w, s->st);
    else
        k_lbm_faces<float><<<s->blocks, kThr, 0, st>>>(s->L, (const float *)s->cu, (const float *)s->cv,
                                                       (const float *)s->cw, s->u, s->v, s->w, s->st);
    FFR_LAUNCHED(1);
    k_lbm_finalize<<<1, 32, 0, st>>>(s->dt, s->tol, s->st, s->ring);
    FFR_LAUNCHED(1);
    s->prof.end(st, 2);
    return FFR_OK;
}

int lbm_pull(ffr_lbm *s)
{
    FFR_CUDA(cudaMemcpyAsync(s->st_host, s->st, sizeof(LbmState), cudaMemcpyDeviceToHost, s->stream));
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    s->prof.collect();
    return FFR_OK;
}

// Sequential outflow copies of LBMSolver::apply_outflow_bc (LBMSolver.cpp:
// 196-282) resolved to one source per destination: the outflow list (which
// holds the openings too) and then the opening list again.
void resolve_remap(const HostRoom &h, std::vector<int> &dst, std::vector<int> &src)
{
    const int nx = h.g.nx, ny = h.g.ny, nz = h.g.nz;
    // source of each cell that differs from itself (patch cells only)
    std::unordered_map<int, int> map;
    auto get = [&](int c) {
        auto it = map.find(c);
        return it == map.end() ? c : it->second;
    };
    auto CI = [&](int i, int j, int k) { return (i * ny + j) * nz + k; };
    auto pass = [&](const ffr_patch &p) {
        const int N[3] = {nx, ny, nz};
        const int wall = p.side == 0 ? 0 : N[p.axis] - 1, s = p.side == 0 ? 1 : N[p.axis] - 2;
        if (s < 0 || s >= N[p.axis]) return;
        const int la = p.axis == 0 ? ny : nx, lb = p.axis == 2 ? ny : nz;
        for (int a = p.a_min; a <= p.a_max; a++)
            for (int b = p.b_min; b <= p.b_max; b++) {
                if (a < 0 || a >= la || b < 0 || b >= lb) continue;
                int cd, cs;
                if (p.axis == 0) { cd = CI(wall, a, b); cs = CI(s, a, b); }
                else if (p.axis == 1) { cd = CI(a, wall, b); cs = CI(a, s, b); }
                else { cd = CI(a, b, wall); cs = CI(a, b, s); }
                if (h.ct[cd] != CT_OUTFLOW) continue;
                map[cd] = get(cs);
            }
    };
    for (const ffr_patch &p : h.patches) pass(p);
    for (const ffr_patch &p : h.patches) if (p.is_opening) pass(p);
    std::vector<std::pair<int, int>> moved;
    for (const auto &kv : map)
        if (kv.second != kv.first) moved.push_back(kv);
    std::sort(moved.begin(), moved.end());
    dst.clear(); src.clear();
    for (const auto &kv : moved) { dst.push_back(kv.first); src.push_back(kv.second); }
}

}  // namespace

extern "C" {

int ffr_lbm_create(const ffr_room_desc *room, double tau, int max_steps, double convergence_tol,
                   double dt, int storage, const ffr_fields *init, ffr_lbm **out)
{
    if (!out) return fail(FFR_EINVAL, "NULL out");
    *out = nullptr;
    if (storage < FFR_LBM_FP64 || storage > FFR_LBM_FP16) return fail(FFR_EINVAL, "bad LBM storage mode");
    if (!(dt > 0) || !(tau > 0)) return fail(FFR_EINVAL, "tau and dt must be positive");
    ffr_lbm *s = new (std::nothrow) ffr_lbm();
    if (!s) return fail(FFR_ENOMEM, "host allocation");
    int rc = load_room(room, s->room);
    if (rc) { delete s; return rc; }
    const RoomGeom &g = s->room.g;
    if (19ll * g.n >= (1ll << 31)) { delete s; return fail(FFR_ERANGE, "lattice too large (19*N >= 2^31)"); }
    s->storage = storage; s->tau = tau; s->dt = dt; s->tol = convergence_tol; s->max_steps = max_steps;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return fail(FFR_ECUDA, "cudaStreamCreate");
    }
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const double p2l = dt / (g.lx / g.nx);   // phys_to_lat = dt / grid.dx (LBMSolver.cpp:42-44)
    std::vector<double> fan_lat(3 * std::max<size_t>(1, s->room.fans.size()), 0.0);
    for (size_t f = 0; f < s->room.fans.size(); f++)
        for (int c = 0; c < 3; c++) fan_lat[3 * f + c] = s->room.fans[f].vel[c] * p2l;
    std::vector<int> rd, rs;
    resolve_remap(s->room, rd, rs);
    const size_t es = storage == FFR_LBM_FP64 ? 8 : (storage == FFR_LBM_FP32 ? 4 : 2);
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t bytes = 2 * al(es * 19 * g.n) + 4 * al(8 * g.n) + al(8 * g.nu) + al(8 * g.nv) +
                         al(8 * g.nw) + 3 * al(g.n) + al(4 * g.n) + al(8 * fan_lat.size()) + 2 * al(4 * (rd.size() + 1)) +
                         2 * (al(8 * g.nx) + al(8 * g.ny) + al(8 * g.nz)) + al(sizeof(LbmState)) +
                         al(sizeof(ffr_step_result) * kRingL) + al(8);
    rc = s->arena.alloc(bytes, s->stream);
    if (rc) { cudaStreamDestroy(s->stream); delete s; return rc; }
    Arena &a = s->arena;
    s->f0 = a.take<char>(es * 19 * g.n);
    s->f1 = a.take<char>(es * 19 * g.n);
    s->cu = a.take<double>(g.n); s->cv = a.take<double>(g.n); s->cw = a.take<double>(g.n);
    s->p = a.take<double>(g.n);
    s->u = a.take<double>(g.nu); s->v = a.take<double>(g.nv); s->w = a.take<double>(g.nw);
    uint8_t *ct = a.take<uint8_t>(g.n), *fo = a.take<uint8_t>(g.n), *fld = a.take<uint8_t>(g.n);
    uint32_t *blk = a.take<uint32_t>(g.n);
    double *fl = a.take<double>(fan_lat.size());
    int *rdd = a.take<int>(rd.size() + 1), *rsd = a.take<int>(rd.size() + 1);
    double *dxv = a.take<double>(g.nx), *dyv = a.take<double>(g.ny), *dzv = a.take<double>(g.nz);
    double *idxv = a.take<double>(g.nx), *idyv = a.take<double>(g.ny), *idzv = a.take<double>(g.nz);
    s->st = a.take<LbmState>(1);
    s->ring = a.take<ffr_step_result>(kRingL);
    s->div_slot = a.take<unsigned long long>(1);
    s->st_host = static_cast<LbmState *>(pinned_get(sizeof(LbmState)));
    s->ring_host = static_cast<ffr_step_result *>(pinned_get(sizeof(ffr_step_result) * kRingL));
    if (!s->div_slot || a.failed || !s->st_host || !s->ring_host) {
        ffr_lbm_destroy(s);
        return fail(FFR_ENOMEM, "LBM allocation");
    }
    cudaStream_t st = s->stream;
    rc = staged_copy(ct, s->room.ct.data(), g.n, false, st);
    if (rc) { ffr_lbm_destroy(s); return rc; }
    FFR_CUDA(cudaMemcpyAsync(fl, fan_lat.data(), 8 * fan_lat.size(), cudaMemcpyHostToDevice, st));
    if (!rd.empty()) {
        FFR_CUDA(cudaMemcpyAsync(rdd, rd.data(), 4 * rd.size(), cudaMemcpyHostToDevice, st));
        FFR_CUDA(cudaMemcpyAsync(rsd, rs.data(), 4 * rs.size(), cudaMemcpyHostToDevice, st));
    }
    // per-cell fan index (255: none), step flags and blocked directions,
    // formed on the device from the cell types
    FFR_CUDA(cudaMemsetAsync(fo, 255, g.n, st));
    for (size_t f = 0; f < s->room.fans.size(); f++) {
        const ffr_fan &fn = s->room.fans[f];
        const long long bi = std::min(nx - 1, fn.i_max) - std::max(0, fn.i_min) + 1,
                        bj = std::min(ny - 1, fn.j_max) - std::max(0, fn.j_min) + 1,
                        bk = std::min(nz - 1, fn.k_max) - std::max(0, fn.k_min) + 1;
        if (bi <= 0 || bj <= 0 || bk <= 0) continue;
        k_lbm_fan_of<<<blocks_for(bi * bj * bk), kThr, 0, st>>>(ct, nx, ny, nz, fn, (uint8_t)f, fo);
        FFR_LAUNCHED(1);
    }
    k_lbm_flags<<<blocks_for(g.n), kThr, 0, st>>>(ct, nx, ny, nz, fld, blk);
    FFR_LAUNCHED(1);
    if (!rd.empty()) {
        k_lbm_remap_flags<<<blocks_for((long long)rd.size()), kThr, 0, st>>>(ct, rdd, (int)rd.size(), fld);
        FFR_LAUNCHED(1);
    }
    FFR_CUDA(cudaMemcpyAsync(dxv, s->room.dxv.data(), 8 * g.nx, cudaMemcpyHostToDevice, st));
    std::vector<double> inv(g.nx + g.ny + g.nz);
    for (int i = 0; i < g.nx; i++) inv[i] = 1.0 / s->room.dxv[i];
    for (int j = 0; j < g.ny; j++) inv[g.nx + j] = 1.0 / s->room.dyv[j];
    for (int k = 0; k < g.nz; k++) inv[g.nx + g.ny + k] = 1.0 / s->room.dzv[k];
    FFR_CUDA(cudaMemcpyAsync(idxv, inv.data(), 8 * g.nx, cudaMemcpyHostToDevice, st));
    FFR_CUDA(cudaMemcpyAsync(idyv, inv.data() + g.nx, 8 * g.ny, cudaMemcpyHostToDevice, st));
    FFR_CUDA(cudaMemcpyAsync(idzv, inv.data() + g.nx + g.ny, 8 * g.nz, cudaMemcpyHostToDevice, st));
    FFR_CUDA(cudaMemcpyAsync(dyv, s->room.dyv.data(), 8 * g.ny, cudaMemcpyHostToDevice, st));
    FFR_CUDA(cudaMemcpyAsync(dzv, s->room.dzv.data(), 8 * g.nz, cudaMemcpyHostToDevice, st));
    auto up = [&](double *d, const double *h, long long cnt) -> int {
        if (h) return staged_copy(d, h, 8 * cnt, false, st);
        else FFR_CUDA(cudaMemsetAsync(d, 0, 8 * cnt, st));
        return FFR_OK;
    };
    if ((rc = up(s->u, init ? init->u : nullptr, g.nu)) || (rc = up(s->v, init ? init->v : nullptr, g.nv)) ||
        (rc = up(s->w, init ? init->w : nullptr, g.nw)) || (rc = up(s->p, init ? init->p : nullptr, g.n))) {
        ffr_lbm_destroy(s);
        return rc;
    }
    FFR_CUDA(cudaMemsetAsync(s->st, 0, sizeof(LbmState), st));
    s->L = LbmDev{nx, ny, nz, (int)g.n, (int)g.nu, (int)g.nv, (int)g.nw, ct, fld, blk, fo, fl, rdd, rsd,
                  (int)rd.size(), dxv, dyv, dzv, idxv, idyv, idzv, tau, (g.lx / g.nx) / dt};
    s->blocks = blocks_for(g.n);
    switch (storage) {
    case FFR_LBM_FP64: k_lbm_init<0><<<s->blocks, kThr, 0, st>>>(s->L, (double *)s->f0); break;
    case FFR_LBM_FP32: k_lbm_init<1><<<s->blocks, kThr, 0, st>>>(s->L, (float *)s->f0); break;
    default: k_lbm_init<2><<<s->blocks, kThr, 0, st>>>(s->L, (__half *)s->f0);
    }
    FFR_LAUNCHED(1);
    FFR_CUDA(cudaStreamSynchronize(st));
    memset(s->st_host, 0, sizeof(LbmState));
    s->prof.reset(FFR_LPROF_N);
    *out = s;
    return FFR_OK;
}

int ffr_lbm_destroy(ffr_lbm *s)
{
    if (!s) return FFR_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    s->prof.destroy();
    s->arena.release();
    pinned_put(s->st_host, sizeof(LbmState));
    pinned_put(s->ring_host, sizeof(ffr_step_result) * kRingL);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FFR_OK;
}

int ffr_lbm_advance(ffr_lbm *s, int nsteps, int stop_on_converge, ffr_step_result *results, int *steps_done)
{
    if (!s || nsteps < 0) return fail(FFR_EINVAL, "bad handle or nsteps");
    int total = 0;
    while (total < nsteps) {
        const int chunk = std::min(kRingL, nsteps - total);
        int rc = lbm_pull(s);
        if (rc) return rc;
        LbmState hs = *s->st_host;
        hs.ring_slot = 0;
        hs.halt = 0;
        hs.stop_on_converge = stop_on_converge ? 1 : 0;
        FFR_CUDA(cudaMemcpyAsync(s->st, &hs, sizeof(LbmState), cudaMemcpyHostToDevice, s->stream));
        for (int k = 0; k < chunk; k++)
            if ((rc = lbm_enqueue(s))) return rc;
        FFR_CUDA(cudaMemcpyAsync(s->ring_host, s->ring, sizeof(ffr_step_result) * chunk, cudaMemcpyDeviceToHost,
                                 s->stream));
        if ((rc = lbm_pull(s))) return rc;
        const int got = s->st_host->ring_slot;
        if (results) memcpy(results + total, s->ring_host, sizeof(ffr_step_result) * got);
        total += got;
        if (got < chunk) break;
    }
    if (steps_done) *steps_done = total;
    return FFR_OK;
}

int ffr_lbm_step(ffr_lbm *s, ffr_step_result *out)
{
    ffr_step_result tmp;
    int done = 0;
    int rc = ffr_lbm_advance(s, 1, 0, out ? out : &tmp, &done);
    if (rc) return rc;
    return done == 1 ? FFR_OK : fail(FFR_ECUDA, "step did not execute");
}

int ffr_lbm_divergence_max(ffr_lbm *s, double *out)
{
    if (!s || !out) return fail(FFR_EINVAL, "NULL argument");
    FFR_CUDA(cudaMemsetAsync(s->div_slot, 0, 8, s->stream));
    k_lbm_divergence<<<s->blocks, kThr, 0, s->stream>>>(s->L, s->u, s->v, s->w, s->div_slot);
    FFR_LAUNCHED(1);
    unsigned long long bits = 0;
    FFR_CUDA(cudaMemcpyAsync(&bits, s->div_slot, 8, cudaMemcpyDeviceToHost, s->stream));
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    memcpy(out, &bits, 8);
    return FFR_OK;
}

int ffr_lbm_current_step(ffr_lbm *s, int *out)
{
    if (!s || !out) return fail(FFR_EINVAL, "NULL argument");
    int rc = lbm_pull(s);
    if (rc) return rc;
    *out = s->st_host->step;
    return FFR_OK;
}

static double *lbm_field(ffr_lbm *s, int field, long long *len)
{
    const RoomGeom &g = s->room.g;
    switch (field) {
    case FFR_FIELD_U: *len = g.nu; return s->u;
    case FFR_FIELD_V: *len = g.nv; return s->v;
    case FFR_FIELD_W: *len = g.nw; return s->w;
    case FFR_FIELD_P: *len = g.n; return s->p;
    default: return nullptr;
    }
}

int ffr_lbm_get_field(ffr_lbm *s, int field, double *host)
{
    long long len = 0;
    double *d = s && host ? lbm_field(s, field, &len) : nullptr;
    if (!d) return fail(FFR_EINVAL, "bad LBM get_field arguments");
    return staged_copy(host, d, 8 * len, true, s->stream);
}

int ffr_lbm_field_dev(ffr_lbm *s, int field, double **dev)
{
    long long len = 0;
    double *d = s && dev ? lbm_field(s, field, &len) : nullptr;
    if (!d) return fail(FFR_EINVAL, "bad LBM field_dev arguments");
    *dev = d;
    return FFR_OK;
}

int ffr_lbm_set_field(ffr_lbm *s, int field, const double *host)
{
    long long len = 0;
    double *d = s && host ? lbm_field(s, field, &len) : nullptr;
    if (!d) return fail(FFR_EINVAL, "bad LBM set_field arguments");
    return staged_copy(d, host, 8 * len, false, s->stream);
}

// Populations of the current buffer (the post-collision state the step
// keeps) through a device staging array of 19*N doubles and the staged
// host copy.
static int lbm_state_io(ffr_lbm *s, double *host_out, const double *host_in, int *step_io)
{
    const long long total = 19ll * s->room.g.n;
    int rc = lbm_pull(s);
    if (rc) return rc;
    LbmState hs = *s->st_host;
    void *cur = hs.par ? s->f1 : s->f0;
    double *tmp = nullptr;
    FFR_CUDA(cudaMallocAsync((void **)&tmp, 8 * total, s->stream));
    const unsigned nb = blocks_for(total);
    const int n = (int)s->room.g.n;
    if (host_out) {
        switch (s->storage) {
        case FFR_LBM_FP64: k_lbm_export<0><<<nb, kThr, 0, s->stream>>>(n, s->L.ct, (const double *)cur, tmp); break;
        case FFR_LBM_FP32: k_lbm_export<1><<<nb, kThr, 0, s->stream>>>(n, s->L.ct, (const float *)cur, tmp); break;
        default: k_lbm_export<2><<<nb, kThr, 0, s->stream>>>(n, s->L.ct, (const __half *)cur, tmp);
        }
        FFR_LAUNCHED(1);
        rc = staged_copy(host_out, tmp, 8 * total, true, s->stream);
        if (step_io) *step_io = hs.step;
    } else {
        rc = staged_copy(tmp, host_in, 8 * total, false, s->stream);
        if (!rc) {
            switch (s->storage) {
            case FFR_LBM_FP64: k_lbm_import<0><<<nb, kThr, 0, s->stream>>>(n, tmp, (double *)cur); break;
            case FFR_LBM_FP32: k_lbm_import<1><<<nb, kThr, 0, s->stream>>>(n, tmp, (float *)cur); break;
            default: k_lbm_import<2><<<nb, kThr, 0, s->stream>>>(n, tmp, (__half *)cur);
            }
            FFR_LAUNCHED(1);
            if (step_io) {
                hs.step = *step_io;
                FFR_CUDA(cudaMemcpyAsync(s->st, &hs, sizeof(LbmState), cudaMemcpyHostToDevice, s->stream));
            }
        }
    }
    cudaFreeAsync(tmp, s->stream);
    if (!rc) FFR_CUDA(cudaStreamSynchronize(s->stream));
    if (!rc) rc = lbm_pull(s);
    return rc;
}

int ffr_lbm_get_populations(ffr_lbm *s, double *f_host, int *step)
{
    if (!s || !f_host) return fail(FFR_EINVAL, "NULL handle or buffer");
    return lbm_state_io(s, f_host, nullptr, step);
}

int ffr_lbm_set_populations(ffr_lbm *s, const double *f_host, int step)
{
    if (!s || !f_host) return fail(FFR_EINVAL, "NULL handle or buffer");
    if (step < 0) return fail(FFR_EINVAL, "negative step");
    return lbm_state_io(s, nullptr, f_host, &step);
}

int ffr_lbm_synchronize(ffr_lbm *s)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    s->prof.collect();
    return FFR_OK;
}

int ffr_lbm_stream(ffr_lbm *s, void **stream)
{
    if (!s || !stream) return fail(FFR_EINVAL, "NULL argument");
    *stream = (void *)s->stream;
    return FFR_OK;
}

int ffr_lbm_profile(ffr_lbm *s, int enable)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    s->prof.collect();
    s->prof.reset(FFR_LPROF_N);
    s->prof.on = enable != 0;
    return FFR_OK;
}

int ffr_lbm_profile_read(ffr_lbm *s, double *ms, long long *launches)
{
    if (!s) return fail(FFR_EINVAL, "NULL handle");
    FFR_CUDA(cudaStreamSynchronize(s->stream));
    s->prof.collect();
    for (int g = 0; g < FFR_LPROF_N; g++) {
        if (ms) ms[g] = s->prof.ms[g];
        if (launches) launches[g] = s->prof.launches[g];
    }
    return FFR_OK;
}

}  // extern "C"
