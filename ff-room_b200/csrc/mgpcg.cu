// mgpcg.cu — mixed-precision multigrid-preconditioned CG (sm_100a).
//
// The pressure system of PoissonSolver::solve (PoissonSolver.cpp:22-91,
// 93-158) restricted to its FLUID/INFLOW rows is closed: those rows see
// OUTFLOW neighbours only as Dirichlet ghosts (diag += 2s).  Scaled by the
// cell volume V = dx*dy*dz it is symmetric positive definite, also on
// stretched grids (V*s across a face is area/distance).  So:
//   1. FP64 preconditioned CG on M = V*A_ff with right-hand side V*b,
//      stopping on the reference's measure ||b - A x||_2 / ||b||_2 (all
//      non-SOLID rows; the OUTFLOW rows are satisfied exactly by step 2);
//   2. the OUTFLOW unknowns by one back-substitution of their own rows,
//      x_o = (b_o + sum_fluid s x_nb) / diag_o;
//   3. preconditioner: one V-cycle in FP32 on 2x2x2 cell aggregates, down to
//      a level of at most kCoarsestCells cells.  Coarse face coefficients
//      are half the sum of the fine ones across the coarse face (the
//      rediscretised volume-scaled Laplacian), restriction sums the
//      children's residuals, prolongation injects.  Smoothing is red-black
//      Gauss-Seidel, kSmoothSweeps sweeps red then black before the coarse
//      correction and black then red after it, so the V-cycle is a
//      symmetric operator and CG applies.
// The whole solve is one cooperative launch; levels larger than
// kBlockLevelCells are swept by the whole grid between grid barriers, the
// remaining small levels by block 0 alone.
#include "mgpcg.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <thread>
#include <cmath>

namespace ffr {

// ---------------------------------------------------------------- host

// Coarsening.  Each level halves the axes whose spacing is within a factor
// two of the level's smallest spacing (semi-coarsening of anisotropic
// cells: the strongly coupled directions first), so that the coarse cells
// approach cubes; isotropic cells halve every axis.  The coarse operator is
// the fine one re-discretised on the coarse cells: a coarse face couples
// with the sum of the fine couplings it covers divided by the coarsening
// factor along its normal (area summed, distance scaled), and likewise
// for the Dirichlet (outflow) part of the diagonal, kept per axis.
//
// The host plans the level sizes (they depend on the dimensions and room
// size only); the coefficients are gathered on the device, one thread per
// coarse cell, from the uploaded cell types and spacings (level 1) or the
// previous level's couplings (mg_upload).
void build_mg_levels(const HostRoom &r, MGHost &out)
{
    out.nx.clear(); out.ny.clear(); out.nz.clear();
    out.sx.clear(); out.sy.clear(); out.sz.clear();
    int nx = r.g.nx, ny = r.g.ny, nz = r.g.nz;
    out.nx.push_back(nx); out.ny.push_back(ny); out.nz.push_back(nz);
    const double lx = r.g.lx, ly = r.g.ly, lz = r.g.lz;
    while ((size_t)nx * ny * nz > (size_t)kCoarsestCells && (int)out.nx.size() < kMaxLevels) {
        // axes to halve at this level
        const double hx = lx / nx, hy = ly / ny, hz = lz / nz;
        const double hmin = std::min(hx, std::min(hy, hz));
        const int sx = (nx > 1 && hx < 2.0 * hmin) ? 1 : 0;
        const int sy = (ny > 1 && hy < 2.0 * hmin) ? 1 : 0;
        const int sz = (nz > 1 && hz < 2.0 * hmin) ? 1 : 0;
        if (!sx && !sy && !sz) break;
        const int mx = sx ? (nx + 1) / 2 : nx, my = sy ? (ny + 1) / 2 : ny, mz = sz ? (nz + 1) / 2 : nz;
        out.sx.push_back(sx); out.sy.push_back(sy); out.sz.push_back(sz);
        out.nx.push_back(mx); out.ny.push_back(my); out.nz.push_back(mz);
        nx = mx; ny = my; nz = mz;
    }
    // the coarsest level has no next level
    out.sx.push_back(0); out.sy.push_back(0); out.sz.push_back(0);
}

namespace {

// Per cell of a level: couplings to the +x, +y, +z neighbour (t0..t2) and
// the Dirichlet diagonal parts along x, y, z (t3..t5); act = the cell has
// a FLUID/INFLOW child.  Device scratch of the coefficient build.
struct LevelOps {
    double *t[6];
    uint8_t *act;
};

__device__ __forceinline__ bool ct_active(uint8_t t) { return t == CT_FLUID || t == CT_INFLOW; }

// Fine-level (FP64) couplings of cell (i, j, k): T to the + neighbour (0
// unless both are unknowns) and the Dirichlet part of the diagonal per
// axis, from the reference's centre distances (PoissonSolver.cpp:33-49).
// The additions are explicit round-to-nearest operations, so the values do
// not depend on how the compiler contracts them.
__device__ __forceinline__ bool fine_ops(const uint8_t *__restrict__ ct, const double *__restrict__ dxv,
                                         const double *__restrict__ dyv, const double *__restrict__ dzv, int nx,
                                         int ny, int nz, int i, int j, int k, double (&t)[6])
{
    for (int d = 0; d < 6; d++) t[d] = 0.0;
    auto C0 = [&](int a, int b, int c) { return ((size_t)a * ny + b) * nz + c; };
    if (!ct_active(ct[C0(i, j, k)])) return false;
    auto hc = [](const double *h, int a, int b) { return 0.5 * __dadd_rn(h[a], h[b]); };
    const double ax = __dmul_rn(dyv[j], dzv[k]), ay = __dmul_rn(dxv[i], dzv[k]), az = __dmul_rn(dxv[i], dyv[j]);
    if (i + 1 < nx) {
        const double v = ax / hc(dxv, i, i + 1);
        const uint8_t nt = ct[C0(i + 1, j, k)];
        if (ct_active(nt)) t[0] = v; else if (nt == CT_OUTFLOW) t[3] = __dadd_rn(t[3], 2 * v);
    }
    if (j + 1 < ny) {
        const double v = ay / hc(dyv, j, j + 1);
        const uint8_t nt = ct[C0(i, j + 1, k)];
        if (ct_active(nt)) t[1] = v; else if (nt == CT_OUTFLOW) t[4] = __dadd_rn(t[4], 2 * v);
    }
    if (k + 1 < nz) {
        const double v = az / hc(dzv, k, k + 1);
        const uint8_t nt = ct[C0(i, j, k + 1)];
        if (ct_active(nt)) t[2] = v; else if (nt == CT_OUTFLOW) t[5] = __dadd_rn(t[5], 2 * v);
    }
    // - neighbours that are Dirichlet ghosts
    if (i > 0 && ct[C0(i - 1, j, k)] == CT_OUTFLOW) t[3] = __dadd_rn(t[3], 2 * ax / hc(dxv, i - 1, i));
    if (j > 0 && ct[C0(i, j - 1, k)] == CT_OUTFLOW) t[4] = __dadd_rn(t[4], 2 * ay / hc(dyv, j - 1, j));
    if (k > 0 && ct[C0(i, j, k - 1)] == CT_OUTFLOW) t[5] = __dadd_rn(t[5], 2 * az / hc(dzv, k - 1, k));
    return true;
}

struct CoarsenArgs {
    // level 1 from the fine cells (cur.act == nullptr) or level l+1 from
    // level l's couplings
    const uint8_t *ct;
    const double *dxv, *dyv, *dzv;
    LevelOps cur, next;
    int nx, ny, nz;       // the finer level
    int sx, sy, sz;       // axes halved
    int mx, my, mz;       // the coarser level
};

// One thread per coarse cell: sums its children's couplings (only those
// across the parent's + faces for t0..t2, every child's Dirichlet parts),
// then scales by the coarsening factor along each normal.
__global__ void k_mg_coarsen(CoarsenArgs a)
{
    const long long m = (long long)a.mx * a.my * a.mz;
    const double f[3] = {a.sx ? 0.5 : 1.0, a.sy ? 0.5 : 1.0, a.sz ? 0.5 : 1.0};
    const bool from_fine = a.cur.act == nullptr;
    for (long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x; P < m;
         P += (long long)gridDim.x * blockDim.x) {
        const int I = (int)(P / ((long long)a.my * a.mz)), rem = (int)(P - (long long)I * a.my * a.mz);
        const int J = rem / a.mz, K = rem - J * a.mz;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        bool any = false;
        for (int x = 0; x <= a.sx; x++) {
            const int i = (I << a.sx) + x;
            if (i >= a.nx) break;
            for (int y = 0; y <= a.sy; y++) {
                const int j = (J << a.sy) + y;
                if (j >= a.ny) break;
                for (int z = 0; z <= a.sz; z++) {
                    const int k = (K << a.sz) + z;
                    if (k >= a.nz) break;
                    double t[6];
                    bool act;
                    if (from_fine) {
                        act = fine_ops(a.ct, a.dxv, a.dyv, a.dzv, a.nx, a.ny, a.nz, i, j, k, t);
                    } else {
                        const size_t c = ((size_t)i * a.ny + j) * a.nz + k;
                        for (int d = 0; d < 6; d++) t[d] = a.cur.t[d][c];
                        act = a.cur.act[c] != 0;
                    }
                    if (!act) continue;
                    any = true;
                    for (int d = 3; d < 6; d++) acc[d] = __dadd_rn(acc[d], t[d]);
                    // couplings across the parent's + faces only
                    if (t[0] > 0 && ((i + 1) >> a.sx) != (i >> a.sx)) acc[0] = __dadd_rn(acc[0], t[0]);
                    if (t[1] > 0 && ((j + 1) >> a.sy) != (j >> a.sy)) acc[1] = __dadd_rn(acc[1], t[1]);
                    if (t[2] > 0 && ((k + 1) >> a.sz) != (k >> a.sz)) acc[2] = __dadd_rn(acc[2], t[2]);
                }
            }
        }
        a.next.act[P] = any;
        for (int d = 0; d < 6; d++) a.next.t[d][P] = __dmul_rn(acc[d], f[d % 3]);
    }
}

// FP32 coefficients of a coarse level: (T x+, T y+, T z+, diagonal), the
// diagonal summed in the order t0..t5, then the - neighbours' + couplings;
// inactive cells get diagonal 0, an active cell without couplings 1.
__global__ void k_mg_coef(LevelOps L, int mx, int my, int mz, float4 *__restrict__ coef)
{
    const long long m = (long long)mx * my * mz;
    for (long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x; P < m;
         P += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(P / ((long long)my * mz)), rem = (int)(P - (long long)i * my * mz);
        const int j = rem / mz, k = rem - j * mz;
        double D = 0.0;
        if (L.act[P]) {
            D = L.t[0][P];
            for (int d = 1; d < 6; d++) D = __dadd_rn(D, L.t[d][P]);
            if (i > 0) D = __dadd_rn(D, L.t[0][P - (long long)my * mz]);
            if (j > 0) D = __dadd_rn(D, L.t[1][P - mz]);
            if (k > 0) D = __dadd_rn(D, L.t[2][P - 1]);
            if (!(D > 0)) D = 1.0;
        }
        coef[P] = make_float4((float)L.t[0][P], (float)L.t[1][P], (float)L.t[2][P], (float)D);
    }
}

unsigned coarse_blocks(long long m)
{
    return (unsigned)std::max<long long>(1, std::min<long long>(8 * 148, (m + 255) / 256));
}

}  // namespace

// -------------------------------------------------------------- device

// FLUID or INFLOW from the stencil code alone (no cell-type load)
__device__ __forceinline__ bool active_code(unsigned code) { return !(code & (SC_SOLID | SC_OUTF)); }

// Grid barrier without a reduction (same protocol as grid_allreduce).
__device__ bool grid_barrier(GridSync *gs)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned g = ld_acquire(&gs->gen);
        const unsigned arrived = atomicAdd(&gs->count, 1u);
        s_ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(&gs->count, 0u);
            __threadfence();
            atomicAdd(&gs->gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            while (ld_acquire(&gs->gen) == g) {
                __nanosleep(32);
                if (global_ns() - t0 > g_wait_limit_ns || *(volatile int *)&gs->err) {
                    atomicExch(&gs->err, 1);
                    s_ok = 0;
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return s_ok;
}

// Level-0 (fine) FP32 coefficients of cell (i,j,k) from its stencil code:
// t[6] in the order x-, x+, y-, y+, z-, z+ (0 unless the neighbour is an
// unknown) and the diagonal (Dirichlet ghosts count twice).
__device__ __forceinline__ void fine_coefs(const MGDev &M, unsigned code, int i, int j, int k, float (&t)[6],
                                           float &D)
{
    float tt[6];
    float vol;
    if (M.uniform) {
        tt[0] = tt[1] = M.tx;
        tt[2] = tt[3] = M.ty;
        tt[4] = tt[5] = M.tz;
        vol = M.vol;
    } else {
        const float dx = M.dx[i], dy = M.dy[j], dz = M.dz[k];
        tt[0] = dy * dz * M.ixl[i]; tt[1] = dy * dz * M.ixr[i];
        tt[2] = dx * dz * M.iyl[j]; tt[3] = dx * dz * M.iyr[j];
        tt[4] = dx * dy * M.izl[k]; tt[5] = dx * dy * M.izr[k];
        vol = dx * dy * dz;
    }
    if ((code & 0xFFFu) == SC_ALLIN) {
        // the general sum below with every class SC_IN, same order
        D = 0.0f;
#pragma unroll
        for (int a = 0; a < 6; a++) {
            t[a] = tt[a];
            D += tt[a];
        }
    } else {
        D = 0.0f;
#pragma unroll
        for (int a = 0; a < 6; a++) {
            const unsigned cls = (code >> (2 * a)) & 3u;
            t[a] = cls == SC_IN ? tt[a] : 0.0f;
            D += cls == SC_IN ? tt[a] : (cls == SC_DIR ? 2.0f * tt[a] : 0.0f);
        }
    }
    if (!(D > 0.0f)) D = vol;
}

// The six neighbour indices of cell c (x-, x+, y-, y+, z-, z+), clamped into
// [0, n): loads through them are always in bounds, so a pass can issue them
// before it has read the cell's stencil code; a neighbour that is not an
// unknown gets weight 0 and its value is never used.
__device__ __forceinline__ void nb_index(int c, int plane, int nz, int n, int (&idx)[6])
{
    idx[0] = max(c - plane, 0);
    idx[1] = min(c + plane, n - 1);
    idx[2] = max(c - nz, 0);
    idx[3] = min(c + nz, n - 1);
    idx[4] = max(c - 1, 0);
    idx[5] = min(c + 1, n - 1);
}

// v[a] += the level-(l+1) correction at the parent of neighbour a of cell
// (i, j, k) of level L: the parent of a neighbour is the cell's own parent
// or the one next to it along the neighbour's axis (when that axis is
// halved, by the parity of the coordinate).  Indices are clamped into the
// parent array (a clamped index is only read for a weight-0 neighbour
// outside the room).
__device__ __forceinline__ void add_parents(const MGLevel &L, const MGLevel &Lc, int i, int j, int k, float (&v)[6])
{
    const int pl = Lc.ny * Lc.nz, pz = Lc.nz, last = Lc.n - 1;
    const int P0 = ((i >> L.sx) * Lc.ny + (j >> L.sy)) * pz + (k >> L.sz);
    const bool ox = L.sx && (i & 1), oy = L.sy && (j & 1), oz = L.sz && (k & 1);
    const bool ex = L.sx && !(i & 1), ey = L.sy && !(j & 1), ez = L.sz && !(k & 1);
    const int p[6] = {ox ? P0 : P0 - pl, ex ? P0 : P0 + pl, oy ? P0 : P0 - pz,
                      ey ? P0 : P0 + pz, oz ? P0 : P0 - 1, ez ? P0 : P0 + 1};
#pragma unroll
    for (int a = 0; a < 6; a++) v[a] += Lc.x[min(max(p[a], 0), last)];
}

// sum_nb T_nb * (x_nb [+ e_parent(nb)]) and the diagonal of cell c on
// level L (L >= 1: explicit coefficients).  Every load is issued before any
// coefficient is tested; the sums are taken in the order x-, x+, y-, y+,
// z-, z+ over the non-zero couplings.
template <bool CORR>
__device__ __forceinline__ float coarse_nbsum(const MGLevel &L, const MGLevel &Lc, int c, int i, int j, int k,
                                              float &D)
{
    const int plane = L.ny * L.nz, nz = L.nz;
    int idx[6];
    nb_index(c, plane, nz, L.n, idx);
    const float4 cf = L.coef[c];
    const float txm = L.coef[idx[0]].x, tym = L.coef[idx[2]].y, tzm = L.coef[idx[4]].z;
    float v[6];
#pragma unroll
    for (int a = 0; a < 6; a++) v[a] = L.x[idx[a]];
    if (CORR) add_parents(L, Lc, i, j, k, v);
    D = cf.w;
    const float t[6] = {i > 0 ? txm : 0.0f, i < L.nx - 1 ? cf.x : 0.0f, j > 0 ? tym : 0.0f,
                        j < L.ny - 1 ? cf.y : 0.0f, k > 0 ? tzm : 0.0f, k < L.nz - 1 ? cf.z : 0.0f};
    float s = 0.0f;
#pragma unroll
    for (int a = 0; a < 6; a++)
        if (t[a] != 0.0f) s += t[a] * v[a];
    return s;
}

template <bool CORR>
__device__ __forceinline__ float fine_nbsum(const RoomDev &R, const MGDev &M, const MGLevel &L0, const MGLevel &L1,
                                            unsigned code, int c, int i, int j, int k, float &D)
{
    const int plane = R.ny * R.nz, nz = R.nz;
    int idx[6];
    nb_index(c, plane, nz, R.n, idx);
    float v[6];
#pragma unroll
    for (int a = 0; a < 6; a++) v[a] = L0.x[idx[a]];
    if (CORR) add_parents(L0, L1, i, j, k, v);
    float t[6];
    fine_coefs(M, code, i, j, k, t, D);
    float s = 0.0f;
#pragma unroll
    for (int a = 0; a < 6; a++)
        if (t[a] != 0.0f) s += t[a] * v[a];
    return s;
}

// One Gauss-Seidel half sweep on `color` of level l of the hierarchy lv.
// CORR adds the coarse correction of level l+1 to the neighbour values (the
// post-smoothing pass right after prolongation).
template <bool CORR>
__device__ void smooth_color(const PCGArgs &A, const MGLevel *lv, int nlev, int l, int color, int start,
                             int stride)
{
    const MGDev &M = A.M;
    const MGLevel &L = lv[l];
    const MGLevel &Lc = lv[l + 1 < nlev ? l + 1 : l];
    // one thread per pair (k, k+1) of a row: exactly one of the two has the colour
    const int pk = (L.nz + 1) >> 1;
    for (Walk w(start, stride, L.ny, pk, L.nx * L.ny * pk); w.ok(); w.next()) {
        const int i = w.i, j = w.j, k = 2 * w.k + ((w.i + w.j + color) & 1);
        if (k >= L.nz) continue;
        const int c = (i * L.ny + j) * L.nz + k;
        float D, s;
        const float bc = L.b[c];
        if (l == 0) {
            const unsigned code = A.R.sc[c];
            s = fine_nbsum<CORR>(A.R, M, L, Lc, code, c, i, j, k, D);
            if (!active_code(code)) continue;
        } else {
            s = coarse_nbsum<CORR>(L, Lc, c, i, j, k, D);
            if (D == 0.0f) continue;
        }
        L.x[c] = (bc + s) / D;
    }
}

// Residual of the red cells of level l (the black ones are exact after a
// black sweep), summed into the parent rhs on level l+1, and the red-only
// first sweep of level l+1 from a zero guess.
__device__ void restrict_level(const PCGArgs &A, const MGLevel *lv, int l, int start, int stride)
{
    const MGDev &M = A.M;
    const MGLevel &L = lv[l];
    const MGLevel &C = lv[l + 1];
    for (Walk w(start, stride, C.ny, C.nz, C.n); w.ok(); w.next()) {
        const int P = w.c, I = w.i, J = w.j, K = w.k;
        const float DP = C.coef[P].w;
        float sum = 0.0f;
#pragma unroll
        for (int a = 0; a < 2; a++) {
#pragma unroll
            for (int b = 0; b < 2; b++) {
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    // children of P along the halved axes
                    if ((a && !L.sx) || (b && !L.sy) || (e && !L.sz)) continue;
                    const int i = (I << L.sx) + a, j = (J << L.sy) + b, k = (K << L.sz) + e;
                    // red children inside the level (the same order as a
                    // nested a, b, e loop that skips the rest)
                    if (i >= L.nx || j >= L.ny || k >= L.nz || ((i + j + k) & 1) != 0) continue;
                    const int c = (i * L.ny + j) * L.nz + k;
                    const float bc = L.b[c], xc = L.x[c];
                    float D, s;
                    bool act;
                    if (l == 0) {
                        const unsigned code = A.R.sc[c];
                        s = fine_nbsum<false>(A.R, M, L, L, code, c, i, j, k, D);
                        act = active_code(code);
                    } else {
                        s = coarse_nbsum<false>(L, L, c, i, j, k, D);
                        act = D != 0.0f;
                    }
                    if (act) sum += bc - (D * xc - s);
                }
            }
        }
        C.b[P] = sum;
        C.x[P] = (((I + J + K) & 1) == 0 && DP != 0.0f) ? sum / DP : 0.0f;
    }
}

// Levels lo .. nlev-1 inside one block (__syncthreads only).  When they fit,
// they run in shared memory: level lo's coefficients, rhs and first guess
// are copied in, the V-cycle below lo runs there, and level lo's solution
// is copied back.
constexpr int kBlockSmemCells = 1536;

__device__ void block_vcycle(const PCGArgs &A, int lo)
{
    __shared__ float4 s_coef[kBlockSmemCells];
    __shared__ float s_x[kBlockSmemCells], s_b[kBlockSmemCells];
    const MGDev &M = A.M;
    const int t = threadIdx.x, nt = blockDim.x;
    const int nlev = M.nlev;
    MGLevel lv[kMaxLevels];
    int total = 0;
    for (int l = 0; l < nlev; l++) {
        lv[l] = M.lv[l];
        if (l >= lo) total += M.lv[l].n;
    }
    const bool smem = total <= kBlockSmemCells;
    if (smem) {
        int off = 0;
        for (int l = lo; l < nlev; l++) {
            const MGLevel &G = M.lv[l];
            for (int c = t; c < G.n; c += nt) {
                s_coef[off + c] = G.coef[c];
                if (l == lo) {
                    s_x[off + c] = G.x[c];
                    s_b[off + c] = G.b[c];
                }
            }
            lv[l].coef = s_coef + off;
            lv[l].x = s_x + off;
            lv[l].b = s_b + off;
            off += G.n;
        }
        __syncthreads();
    }
    for (int l = lo; l < nlev - 1; l++) {
        smooth_color<false>(A, lv, nlev, l, 1, t, nt);
        __syncthreads();
        for (int sw = 1; sw < level_sweeps(l); sw++) {
            smooth_color<false>(A, lv, nlev, l, 0, t, nt);
            __syncthreads();
            smooth_color<false>(A, lv, nlev, l, 1, t, nt);
            __syncthreads();
        }
        restrict_level(A, lv, l, t, nt);
        __syncthreads();
    }
    const int last = nlev - 1;
    for (int sweep = 0; sweep < kCoarsestSweeps; sweep++) {
        smooth_color<false>(A, lv, nlev, last, 1, t, nt);
        __syncthreads();
        smooth_color<false>(A, lv, nlev, last, 0, t, nt);
        __syncthreads();
    }
    for (int l = nlev - 2; l >= lo; l--) {
        smooth_color<true>(A, lv, nlev, l, 1, t, nt);
        __syncthreads();
        smooth_color<false>(A, lv, nlev, l, 0, t, nt);
        __syncthreads();
        for (int sw = 1; sw < level_sweeps(l); sw++) {
            smooth_color<false>(A, lv, nlev, l, 1, t, nt);
            __syncthreads();
            smooth_color<false>(A, lv, nlev, l, 0, t, nt);
            __syncthreads();
        }
    }
    if (smem) {
        const MGLevel &G = M.lv[lo];
        for (int c = t; c < G.n; c += nt) G.x[c] = lv[lo].x[c];
        __syncthreads();
    }
}

// The reference's FP64 operator row (PoissonSolver.cpp:22-91) of cell c
// applied to a direction given by dir(offset).  On a uniform grid every
// scale 1/(h_face h) equals 1/h^2 (M.s64); a cell with six unknown
// neighbours takes the same sums in the same order without the class tests.
template <class F>
__device__ __forceinline__ double ref_row(const RoomDev &R, const MGDev &M, unsigned code, int i, int j, int k,
                                          double xc, F dir)
{
    const int nx = R.nx, ny = R.ny, nz = R.nz, plane = ny * nz;
    double s[6];
    if (M.uniform) {
        s[0] = s[1] = M.s64x;
        s[2] = s[3] = M.s64y;
        s[4] = s[5] = M.s64z;
    } else {
        const double *sxl = R.scale, *sxr = sxl + nx, *syl = sxr + nx, *syr = syl + ny, *szl = syr + ny,
                     *szr = szl + nz;
        s[0] = sxl[i]; s[1] = sxr[i]; s[2] = syl[j]; s[3] = syr[j]; s[4] = szl[k]; s[5] = szr[k];
    }
    const int off[6] = {-plane, plane, -nz, nz, -1, 1};
    double diag = 0.0, o = 0.0;
    if ((code & 0xFFFu) == SC_ALLIN) {
#pragma unroll
        for (int a = 0; a < 6; a++) {
            diag += s[a];
            o += s[a] * dir(off[a]);
        }
    } else {
#pragma unroll
        for (int a = 0; a < 6; a++) {
            const unsigned cls = (code >> (2 * a)) & 3u;
            if (cls == SC_IN) {
                diag += s[a];
                o += s[a] * dir(off[a]);
            } else if (cls == SC_DIR) {
                diag += 2.0 * s[a];
            }
        }
    }
    if (diag < 1e-30) diag = 1.0;
    return diag * xc - o;
}

// Cell volume dx*dy*dz in FP64 (the product order of the general case).
__device__ __forceinline__ double cell_vol(const MGDev &M, int i, int j, int k)
{
    return M.uniform ? M.vol64 : M.vol_x[i] * M.vol_y[j] * M.vol_z[k];
}

// FP64 weights of the reference row: w[a] = scale if neighbour a is an
// unknown, else 0; diag = sum of scale (unknown) and 2*scale (Dirichlet
// ghost) in the order a = 0..5, as ref_row accumulates it.
__device__ __forceinline__ void ref_weights(const RoomDev &R, const MGDev &M, unsigned code, int i, int j, int k,
                                            double (&w)[6], double &diag)
{
    const bool allin = (code & 0xFFFu) == SC_ALLIN;
    if (M.uniform) {
        if (allin) {
            // six unknown neighbours: the sums below, precomputed in the same order
            w[0] = w[1] = M.s64x;
            w[2] = w[3] = M.s64y;
            w[4] = w[5] = M.s64z;
            diag = M.diag64;
            return;
        }
    }
    double s[6];
    if (M.uniform) {
        s[0] = s[1] = M.s64x;
        s[2] = s[3] = M.s64y;
        s[4] = s[5] = M.s64z;
    } else {
        const int nx = R.nx, ny = R.ny, nz = R.nz;
        const double *sxl = R.scale, *sxr = sxl + nx, *syl = sxr + nx, *syr = syl + ny, *szl = syr + ny,
                     *szr = szl + nz;
        s[0] = sxl[i]; s[1] = sxr[i]; s[2] = syl[j]; s[3] = syr[j]; s[4] = szl[k]; s[5] = szr[k];
    }
    diag = 0.0;
    if (allin) {
#pragma unroll
        for (int a = 0; a < 6; a++) {
            w[a] = s[a];
            diag += s[a];
        }
    } else {
#pragma unroll
        for (int a = 0; a < 6; a++) {
            const unsigned cls = (code >> (2 * a)) & 3u;
            w[a] = cls == SC_IN ? s[a] : 0.0;
            diag += cls == SC_IN ? s[a] : (cls == SC_DIR ? 2.0 * s[a] : 0.0);
        }
    }
    if (diag < 1e-30) diag = 1.0;
}

__device__ __forceinline__ double face_rhs(const PCGArgs &A, int c, int i, int j, int k)
{
    const RoomDev &R = A.R;
    if (!A.from_faces) return A.rhs[c];
    const int ny = R.ny, nz = R.nz;
    const int u0 = c, u1 = c + ny * nz;
    const int v0 = (i * (ny + 1) + j) * nz + k, w0 = (i * ny + j) * (nz + 1) + k;
    const double div = (A.us[u1] - A.us[u0]) / R.dxv[i] + (A.vs[v0 + nz] - A.vs[v0]) / R.dyv[j]
                     + (A.ws[w0 + 1] - A.ws[w0]) / R.dzv[k];
    return A.rhs_factor * div;
}

// Synchronisation groups of the preconditioned solve.
//  GridGroup    - every block of a cooperative launch (one room on the whole GPU)
//  ClusterGroup - the blocks of one thread-block cluster (one room on 1-16 SMs;
//                 hardware cluster barrier, reductions through distributed
//                 shared memory), so that many small rooms run side by side.
struct GridGroup {
    __device__ static int rank() { return blockIdx.x; }
    __device__ static int size() { return gridDim.x; }
    __device__ static void init() {}
    __device__ static bool sync(const PCGArgs &A) { return grid_barrier(A.gs); }
    template <int NV>
    __device__ static bool allreduce(const PCGArgs &A, double (&v)[NV], double *sh)
    {
        return grid_allreduce<NV>(A.gs, A.partials, A.sc->red, v, sh);
    }
    __device__ static void finish() {}
};

struct ClusterGroup {
    __device__ static int rank() { return (int)cooperative_groups::this_cluster().block_rank(); }
    __device__ static int size() { return (int)cooperative_groups::this_cluster().num_blocks(); }
    __device__ static double (&slots())[2][4]
    {
        __shared__ double s_slot[2][4];
        return s_slot;
    }
    __device__ static int &parity()
    {
        __shared__ int s_par;
        return s_par;
    }
    __device__ static void init()
    {
        if (threadIdx.x == 0) parity() = 0;
        __syncthreads();
    }
    __device__ static bool sync(const PCGArgs &)
    {
        __threadfence();
        cooperative_groups::this_cluster().sync();
        return true;
    }
    // Deterministic: every block adds the blocks' partials in rank order.
    // Two slot buffers alternate, so a block never overwrites a slot another
    // block may still be reading (a cluster barrier separates the reuse).
    template <int NV>
    __device__ static bool allreduce(const PCGArgs &, double (&v)[NV], double *sh)
    {
        auto cl = cooperative_groups::this_cluster();
        const int p = parity();
        for (int a = 0; a < NV; a++) {
            const double t = block_sum(v[a], sh);
            if (threadIdx.x == 0) slots()[p][a] = t;
        }
        __threadfence();
        cl.sync();
        const int nb = (int)cl.num_blocks();
        for (int a = 0; a < NV; a++) {
            double tot = 0.0;
            for (int r = 0; r < nb; r++) tot += *cl.map_shared_rank(&slots()[p][a], r);
            v[a] = tot;
        }
        __syncthreads();
        if (threadIdx.x == 0) parity() = p ^ 1;
        __syncthreads();
        return true;
    }
    // no block may leave while another can still read its shared memory
    __device__ static void finish() { cooperative_groups::this_cluster().sync(); }
};

// ---- the passes of one preconditioned-CG solve, each over the cells
// start, start + stride, ... (a persistent group or one item per thread)

// rhs, r = V*rhs on the unknowns, x = 0, d = 0, z = red sweep from 0;
// acc = {||b||^2 over non-SOLID rows, ||b||^2 over unknowns}.  Warm start
// (A.warm): x keeps its values (the previous step's pressure) and
// r = V*(rhs - A x) on the unknowns, A the reference's row (the operator
// of the direction pass); OUTFLOW values of x do not enter these rows.
__device__ __forceinline__ void pass_init(const PCGArgs &A, int start, int stride, double (&acc)[2])
{
    const RoomDev &R = A.R;
    const MGDev &M = A.M;
    float *z = M.lv[0].x;
    const int n = R.n, plane = R.ny * R.nz, nz = R.nz;
    for (Walk wk(start, stride, R.ny, R.nz, R.n); wk.ok(); wk.next()) {
        const int c = wk.c, i = wk.i, j = wk.j, k = wk.k;
        const unsigned code = R.sc[c];
        if (!A.warm) A.x[c] = 0.0;
        A.da[c] = 0.0;
        A.db[c] = 0.0;
        double rv = 0.0;
        float zv = 0.0f;
        if (!(code & SC_SOLID)) {
            const double b = face_rhs(A, c, i, j, k);
            acc[0] += b * b;
            if (active_code(code)) {
                acc[1] += b * b;
                rv = b * cell_vol(M, i, j, k);
                if (A.warm) {
                    int idx[6];
                    nb_index(c, plane, nz, n, idx);
                    double wt[6], diag, o = 0.0;
                    ref_weights(R, M, code, i, j, k, wt, diag);
#pragma unroll
                    for (int a = 0; a < 6; a++) o += wt[a] * A.x[idx[a]];
                    rv -= cell_vol(M, i, j, k) * (diag * A.x[c] - o);
                }
                if (((i + j + k) & 1) == 0) {
                    float tt[6], D;
                    fine_coefs(M, code, i, j, k, tt, D);
                    zv = (float)rv / D;
                }
            }
        }
        A.r[c] = rv;
        M.r32[c] = (float)rv;
        z[c] = zv;
    }
}

// The level-0 passes below visit the cells in pairs (k, k+1) of a row: one
// thread per pair, so exactly one cell of each thread is red and the red-only
// work does not diverge, and both cells' loads are in flight together.  A row
// of odd length ends in a single cell (c1 == c0, nothing stored for it).
struct CellPair {
    int i, j, k0, c0, c1;
    bool two, red0;   // a second cell; cell 0 is red ((i + j + k) even)
    __device__ __forceinline__ CellPair(const Walk &w, int ny, int nz)
    {
        i = w.i;
        j = w.j;
        k0 = 2 * w.k;
        two = k0 + 1 < nz;
        c0 = (i * ny + j) * nz + k0;
        c1 = two ? c0 + 1 : c0;
        red0 = ((i + j + k0) & 1) == 0;
    }
    __device__ __forceinline__ int kred(int nz) const { return red0 ? k0 : min(k0 + 1, nz - 1); }
    __device__ __forceinline__ int cred() const { return red0 ? c0 : c1; }
};

// Warm-start extrapolation (see launch_extrapolate): elementwise, so every
// launch shape gives the same values.  The state of a halted room is kept.
// Half a step of linear extrapolation through a room's first ten steps (the
// early transient, where it starts several times closer to the solution
// than the previous pressure and than a full step), a full step after that
// (closer than half a step once the flow evolves smoothly).
__device__ __forceinline__ void pass_extrapolate(const PCGArgs &A, int start, int stride)
{
    if (!A.warm || (A.st && A.st->halt)) return;
    const int step = A.st ? A.st->step : 0;
    const double theta = step >= 10 ? 1.0 : (step >= 2 ? 0.5 : 0.0);
    for (int c = start; c < A.R.n; c += stride) {
        const double a = __ldcs(A.x + c), b = __ldcs(A.xprev + c);
        const double x0 = a + theta * (a - b);
        __stcs(A.x + c, x0);
        __stcs(A.xprev + c, a);
        __stcs(A.x0 + c, x0);
    }
}

// the last red sweep of level 0 fused with r.z
__device__ __forceinline__ void pass_redpost_dot(const PCGArgs &A, int start, int stride, double &acc)
{
    const RoomDev &R = A.R;
    const MGDev &M = A.M;
    float *z = M.lv[0].x;
    const bool sweep = M.nlev_grid >= 1;
    const int n = R.n, ny = R.ny, nz = R.nz, plane = ny * nz, pk = (nz + 1) >> 1;
    if ((nz & 1) == 0) {
        // even rows: pair loads (see pass_direction); the red cell's x and y
        // neighbours are one half of the neighbouring pairs, its z neighbours
        // the other cell of the pair and one single load
        for (Walk w(start, stride, ny, pk, R.nx * ny * pk); w.ok(); w.next()) {
            const int i = w.i, j = w.j, k0 = 2 * w.k;
            const int c0 = (i * ny + j) * nz + k0;
            const bool red0 = ((i + j + k0) & 1) == 0;
            const ushort2 cd = *reinterpret_cast<const ushort2 *>(R.sc + c0);
            const double2 r = __ldcs(reinterpret_cast<const double2 *>(A.r + c0));
            const float2 zc = *reinterpret_cast<const float2 *>(z + c0);
            float z0 = zc.x, z1 = zc.y;
            const int cr = red0 ? c0 : c0 + 1;
            const float br = M.r32[cr];
            const int ox[4] = {max(c0 - plane, 0), min(c0 + plane, n - 2), max(c0 - nz, 0), min(c0 + nz, n - 2)};
            float zn[6];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                const float2 zv = *reinterpret_cast<const float2 *>(z + ox[a]);
                zn[a] = red0 ? zv.x : zv.y;
            }
            const float zo = z[red0 ? max(c0 - 1, 0) : min(c0 + 2, n - 1)];
            zn[4] = red0 ? zo : zc.x;
            zn[5] = red0 ? zc.y : zo;
            const unsigned coder = red0 ? cd.x : cd.y;
            if (sweep && active_code(coder)) {
                float t[6], D;
                fine_coefs(M, coder, i, j, red0 ? k0 : k0 + 1, t, D);
                float sum = 0.0f;
#pragma unroll
                for (int a = 0; a < 6; a++)
                    if (t[a] != 0.0f) sum += t[a] * zn[a];
                const float zr = (br + sum) / D;
                z[cr] = zr;
                if (red0) z0 = zr; else z1 = zr;
            }
            if (active_code(cd.x)) acc += r.x * (double)z0;
            if (active_code(cd.y)) acc += r.y * (double)z1;
        }
        return;
    }
    for (Walk w(start, stride, ny, pk, R.nx * ny * pk); w.ok(); w.next()) {
        const CellPair P(w, ny, nz);
        const unsigned code0 = R.sc[P.c0], code1 = R.sc[P.c1];
        const double r0 = A.r[P.c0], r1 = A.r[P.c1];
        float z0 = z[P.c0], z1 = z[P.c1];
        const int cr = P.cred();
        const float br = M.r32[cr];
        int idx[6];
        nb_index(cr, plane, nz, n, idx);
        float zn[6];
#pragma unroll
        for (int a = 0; a < 6; a++) zn[a] = z[idx[a]];
        const unsigned coder = P.red0 ? code0 : code1;
        if (sweep && active_code(coder) && (P.red0 || P.two)) {
            float t[6], D;
            fine_coefs(M, coder, P.i, P.j, P.kred(nz), t, D);
            float sum = 0.0f;
#pragma unroll
            for (int a = 0; a < 6; a++)
                if (t[a] != 0.0f) sum += t[a] * zn[a];
            const float zr = (br + sum) / D;
            z[cr] = zr;
            if (P.red0) z0 = zr; else z1 = zr;
        }
        if (active_code(code0)) acc += r0 * (double)z0;
        if (P.two && active_code(code1)) acc += r1 * (double)z1;
    }
}

// d = z + beta d_old, the deferred x += alpha_prev d_old, q = M d; acc = d.q
__device__ __forceinline__ void pass_direction(const PCGArgs &A, int start, int stride, double beta,
                                               double alpha_prev, bool update_x, const double *__restrict__ dold,
                                               double *__restrict__ dnew, double &acc)
{
    const RoomDev &R = A.R;
    const MGDev &M = A.M;
    const float *z = M.lv[0].x;
    const int n = R.n, ny = R.ny, nz = R.nz, plane = ny * nz, pk = (nz + 1) >> 1;
    if ((nz & 1) == 0) {
        // Even rows: both cells of every pair, and the pairs of its x and y
        // neighbours, sit at even indices, so each pair moves with one
        // 16-byte (8-byte for FP32, 4-byte for codes) load or store.  A
        // neighbour pair outside the grid is clamped to a pair inside it;
        // its values get weight 0, exactly as the clamped single loads of
        // the general loop below.
        for (Walk w(start, stride, ny, pk, R.nx * ny * pk); w.ok(); w.next()) {
            const int i = w.i, j = w.j, k0 = 2 * w.k;
            const int c0 = (i * ny + j) * nz + k0;
            const ushort2 cd = *reinterpret_cast<const ushort2 *>(R.sc + c0);
            const double2 dp = *reinterpret_cast<const double2 *>(dold + c0);
            const float2 zc = *reinterpret_cast<const float2 *>(z + c0);
            const double2 xo = update_x ? __ldcs(reinterpret_cast<const double2 *>(A.x + c0)) : make_double2(0.0, 0.0);
            const int ox[4] = {max(c0 - plane, 0), min(c0 + plane, n - 2), max(c0 - nz, 0), min(c0 + nz, n - 2)};
            double n0[6], n1[6];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                const double2 dv = *reinterpret_cast<const double2 *>(dold + ox[a]);
                const float2 zv = *reinterpret_cast<const float2 *>(z + ox[a]);
                n0[a] = fma(beta, dv.x, (double)zv.x);
                n1[a] = fma(beta, dv.y, (double)zv.y);
            }
            const int zm = max(c0 - 1, 0), zp = min(c0 + 2, n - 1);
            n0[4] = fma(beta, dold[zm], (double)z[zm]);
            n1[5] = fma(beta, dold[zp], (double)z[zp]);
            const double d0 = fma(beta, dp.x, (double)zc.x), d1 = fma(beta, dp.y, (double)zc.y);
            n0[5] = d1;
            n1[4] = d0;
            auto cell = [&](unsigned code, int k, double dp_, double dc, double xo_, const double (&dn)[6],
                            double &dout, double &qout, double &xout) {
                xout = xo_;
                if (!active_code(code)) {
                    dout = 0.0;
                    qout = 0.0;
                    return;
                }
                if (update_x) xout = fma(alpha_prev, dp_, xo_);
                dout = dc;
                double wt[6], diag;
                ref_weights(R, M, code, i, j, k, wt, diag);
                double o = 0.0;
#pragma unroll
                for (int a = 0; a < 6; a++) o += wt[a] * dn[a];
                const double qc = cell_vol(M, i, j, k) * (diag * dc - o);
                qout = qc;
                acc += dc * qc;
            };
            double2 dn2, q2, xn2;
            cell(cd.x, k0, dp.x, d0, xo.x, n0, dn2.x, q2.x, xn2.x);
            cell(cd.y, k0 + 1, dp.y, d1, xo.y, n1, dn2.y, q2.y, xn2.y);
            *reinterpret_cast<double2 *>(dnew + c0) = dn2;
            __stcs(reinterpret_cast<double2 *>(A.q + c0), q2);
            if (update_x) __stcs(reinterpret_cast<double2 *>(A.x + c0), xn2);
        }
        return;
    }
    for (Walk w(start, stride, ny, pk, R.nx * ny * pk); w.ok(); w.next()) {
        const CellPair P(w, ny, nz);
        const int c0 = P.c0, c1 = P.c1;
        const unsigned code0 = R.sc[c0], code1 = R.sc[c1];
        const double dp0 = dold[c0], dp1 = dold[c1];
        const float z0 = z[c0], z1 = z[c1];
        const double x0 = update_x ? A.x[c0] : 0.0, x1 = update_x ? A.x[c1] : 0.0;
        // new direction values of the neighbours: x-, x+, y-, y+ of each cell,
        // the row neighbours outside the pair; inside the pair each cell is
        // the other's z neighbour
        const int o0[5] = {max(c0 - plane, 0), min(c0 + plane, n - 1), max(c0 - nz, 0), min(c0 + nz, n - 1),
                           max(c0 - 1, 0)};
        const int o1[5] = {max(c1 - plane, 0), min(c1 + plane, n - 1), max(c1 - nz, 0), min(c1 + nz, n - 1),
                           min(c1 + 1, n - 1)};
        double n0[6], n1[6];
#pragma unroll
        for (int a = 0; a < 4; a++) {
            n0[a] = fma(beta, dold[o0[a]], (double)z[o0[a]]);
            n1[a] = fma(beta, dold[o1[a]], (double)z[o1[a]]);
        }
        n0[4] = fma(beta, dold[o0[4]], (double)z[o0[4]]);
        n1[5] = fma(beta, dold[o1[4]], (double)z[o1[4]]);
        const double d0 = fma(beta, dp0, (double)z0), d1 = fma(beta, dp1, (double)z1);
        n0[5] = P.two ? d1 : n1[5];
        n1[4] = d0;
        auto cell = [&](int c, unsigned code, int k, double dp, double dc, double xo, const double (&dn)[6]) {
            if (!active_code(code)) {
                dnew[c] = 0.0;
                A.q[c] = 0.0;
                return;
            }
            if (update_x) A.x[c] = fma(alpha_prev, dp, xo);
            dnew[c] = dc;
            double wt[6], diag;
            ref_weights(R, M, code, P.i, P.j, k, wt, diag);
            double o = 0.0;
#pragma unroll
            for (int a = 0; a < 6; a++) o += wt[a] * dn[a];
            const double qc = cell_vol(M, P.i, P.j, k) * (diag * dc - o);
            A.q[c] = qc;
            acc += dc * qc;
        };
        cell(c0, code0, P.k0, dp0, d0, x0, n0);
        if (P.two) cell(c1, code1, P.k0 + 1, dp1, d1, x1, n1);
    }
}

// r -= alpha q, acc = ||b - A x||^2 (unscaled), the red sweep of the next z
__device__ __forceinline__ void pass_residual(const PCGArgs &A, int start, int stride, double alpha, double &acc)
{
    const RoomDev &R = A.R;
    const MGDev &M = A.M;
    float *z = M.lv[0].x;
    const int ny = R.ny, nz = R.nz, pk = (nz + 1) >> 1;
    if ((nz & 1) == 0) {
        // even rows: pair loads and stores (see pass_direction).  A cell
        // that is not an unknown keeps r (stored back unchanged) and its
        // r32 and z, which the solve's set-up pass made 0.
        for (Walk w(start, stride, ny, pk, R.nx * ny * pk); w.ok(); w.next()) {
            const int i = w.i, j = w.j, k0 = 2 * w.k;
            const int c0 = (i * ny + j) * nz + k0;
            const bool red0 = ((i + j + k0) & 1) == 0;
            const ushort2 cd = *reinterpret_cast<const ushort2 *>(R.sc + c0);
            const double2 rq = __ldcs(reinterpret_cast<const double2 *>(A.r + c0));
            const double2 qq = __ldcs(reinterpret_cast<const double2 *>(A.q + c0));
            float tt[6], D;
            fine_coefs(M, red0 ? cd.x : cd.y, i, j, red0 ? k0 : k0 + 1, tt, D);
            double2 rn = rq;
            float2 r32v = make_float2(0.0f, 0.0f), zv = make_float2(0.0f, 0.0f);
            auto cell = [&](unsigned code, int k, double r0, double q0, bool red, double &rout, float &r32out,
                            float &zout) {
                if (!active_code(code)) return;
                const double rv = r0 - alpha * q0;
                rout = rv;
                const double ru = rv / cell_vol(M, i, j, k);
                acc += ru * ru;
                const float r32 = (float)rv;
                r32out = r32;
                zout = red ? r32 / D : 0.0f;
            };
            cell(cd.x, k0, rq.x, qq.x, red0, rn.x, r32v.x, zv.x);
            cell(cd.y, k0 + 1, rq.y, qq.y, !red0, rn.y, r32v.y, zv.y);
            __stcs(reinterpret_cast<double2 *>(A.r + c0), rn);
            *reinterpret_cast<float2 *>(M.r32 + c0) = r32v;
            *reinterpret_cast<float2 *>(z + c0) = zv;
        }
        return;
    }
    for (Walk w(start, stride, ny, pk, R.nx * ny * pk); w.ok(); w.next()) {
        const CellPair P(w, ny, nz);
        const unsigned code0 = R.sc[P.c0], code1 = R.sc[P.c1];
        const double ra = A.r[P.c0], qa = A.q[P.c0], rb = A.r[P.c1], qb = A.q[P.c1];
        float tt[6], D;
        fine_coefs(M, P.red0 ? code0 : code1, P.i, P.j, P.kred(nz), tt, D);
        auto cell = [&](int c, unsigned code, int k, double r0, double q0, bool red) {
            if (!active_code(code)) return;
            const double rv = r0 - alpha * q0;
            A.r[c] = rv;
            const double ru = rv / cell_vol(M, P.i, P.j, k);
            acc += ru * ru;
            const float r32 = (float)rv;
            M.r32[c] = r32;
            z[c] = red ? r32 / D : 0.0f;
        };
        cell(P.c0, code0, P.k0, ra, qa, P.red0);
        if (P.two) cell(P.c1, code1, P.k0 + 1, rb, qb, !P.red0);
    }
}

__device__ __forceinline__ void pass_final_x(const PCGArgs &A, int start, int stride, double alpha,
                                             const double *__restrict__ d)
{
    for (int c = start; c < A.R.n; c += stride)
        if (active_code(A.R.sc[c])) A.x[c] = fma(alpha, d[c], A.x[c]);
}

// OUTFLOW rows by back-substitution in the reference's own row form:
// diag*x_o - sum_in s*x_nb = b  ->  x_o = (b + sum) / diag
__device__ __forceinline__ void pass_backsub(const PCGArgs &A, int start, int stride)
{
    const RoomDev &R = A.R;
    double *x = A.x;
    for (Walk wk(start, stride, R.ny, R.nz, R.n); wk.ok(); wk.next()) {
        const int c = wk.c, i = wk.i, j = wk.j, k = wk.k;
        const unsigned code = R.sc[c];
        if (!(code & SC_OUTF)) continue;
        const double b = face_rhs(A, c, i, j, k);
        const double row0 = ref_row(R, A.M, code, i, j, k, 0.0, [&](int o) { return x[c + o]; });
        const double diag = ref_row(R, A.M, code, i, j, k, 1.0, [&](int) { return 0.0; });
        x[c] = (b - row0) / diag;
    }
}

// Threads per block of the one-cluster schedule: a cluster of at most 16
// blocks must still hold enough warps per SM to hide memory latency.
constexpr int kClusterThreads = 512;

// The whole solve on the blocks of group G (a cooperative grid or one
// thread-block cluster).
template <class G>
__device__ __forceinline__ void pcg_body(const PCGArgs &A)
{
    __shared__ double sh[32];
    if (A.st && A.st->halt) return;
    const MGDev &M = A.M;
    G::init();
    const int t0 = G::rank() * blockDim.x + threadIdx.x, nth = G::size() * blockDim.x;
    int flags = 0, iters = 0;
    double res = 0.0;
    {
        double acc[2] = {0.0, 0.0};
        pass_init(A, t0, nth, acc);
        if (!G::template allreduce<2>(A, acc, sh)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
        const double bnorm = sqrt(acc[0]);
        if (bnorm < 1e-15) goto finish;

        double *dold = A.da, *dnew = A.db;
        double rz_old = 0.0, alpha = 0.0, alpha_prev = 0.0;
        bool pending = false;
        for (int it = 0;; it++) {
            // ---- preconditioner: V-cycle from the red sweep already in z
            for (int l = 0; l < M.nlev_grid && l < M.nlev - 1; l++) {
                smooth_color<false>(A, M.lv, M.nlev, l, 1, t0, nth);
                if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                for (int sw = 1; sw < level_sweeps(l); sw++) {
                    smooth_color<false>(A, M.lv, M.nlev, l, 0, t0, nth);
                    if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                    smooth_color<false>(A, M.lv, M.nlev, l, 1, t0, nth);
                    if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                }
                restrict_level(A, M.lv, l, t0, nth);
                if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
            }
            if (M.nlev_grid < M.nlev) {
                if (G::rank() == 0) block_vcycle(A, M.nlev_grid);
                if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
            }
            for (int l = min(M.nlev_grid, M.nlev - 1) - 1; l >= 1; l--) {
                smooth_color<true>(A, M.lv, M.nlev, l, 1, t0, nth);
                if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                smooth_color<false>(A, M.lv, M.nlev, l, 0, t0, nth);
                if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                for (int sw = 1; sw < level_sweeps(l); sw++) {
                    smooth_color<false>(A, M.lv, M.nlev, l, 1, t0, nth);
                    if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                    smooth_color<false>(A, M.lv, M.nlev, l, 0, t0, nth);
                    if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                }
            }
            if (M.nlev_grid >= 1 && M.nlev > 1) {
                smooth_color<true>(A, M.lv, M.nlev, 0, 1, t0, nth);
                if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                // the further sweeps; the last red half is the r.z pass's
                for (int sw = 1; sw < level_sweeps(0); sw++) {
                    smooth_color<false>(A, M.lv, M.nlev, 0, 0, t0, nth);
                    if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                    smooth_color<false>(A, M.lv, M.nlev, 0, 1, t0, nth);
                    if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
                }
            }
            double acc1[1] = {0.0};
            pass_redpost_dot(A, t0, nth, acc1[0]);
            if (!G::template allreduce<1>(A, acc1, sh)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
            const double rz = acc1[0];
            const double beta = it == 0 ? 0.0 : rz / rz_old;
            rz_old = rz;

            double acc2[1] = {0.0};
            pass_direction(A, t0, nth, beta, alpha_prev, it > 0, dold, dnew, acc2[0]);
            if (!G::template allreduce<1>(A, acc2, sh)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
            { double *tmp = dold; dold = dnew; dnew = tmp; }   // dold = current direction
            pending = false;
            const double dq = acc2[0];
            if (fabs(dq) < 1e-30) {
                flags |= FFR_FLAG_CG_BREAKDOWN;
                iters = it;
                break;
            }
            alpha = rz / dq;

            double acc3[1] = {0.0};
            pass_residual(A, t0, nth, alpha, acc3[0]);
            if (!G::template allreduce<1>(A, acc3, sh)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
            pending = true;
            res = sqrt(acc3[0]) / bnorm;
            iters = it + 1;
            if (res < A.tol) break;
            if (iters >= A.max_iter) { flags |= FFR_FLAG_CG_MAXITER; break; }
            alpha_prev = alpha;
        }
        if (pending) pass_final_x(A, t0, nth, alpha, dold);
        if (!G::sync(A)) { flags = FFR_FLAG_TIMEOUT; goto finish; }
        pass_backsub(A, t0, nth);
    }
finish:
    G::finish();
    if (G::rank() == 0 && threadIdx.x == 0) {
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

template <class G, int NT = 256>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : 1) k_pcg(PCGArgs A)
{
    pcg_body<G>(A);
}

// Batched rooms, one thread-block cluster per room: cluster c (blocks
// c*ctas .. c*ctas + ctas - 1) runs the whole solve of room order[c], exactly as
// that room's own one-cluster launch (k_pcg<ClusterGroup>) does, so many
// rooms' solves run side by side in one launch with no host pacing.
__global__ void __launch_bounds__(kClusterThreads, 1) k_bpcg_cluster(BatchDev D, const int *order, int ctas)
{
    __shared__ __align__(16) PCGArgs A;
    const int r = order[blockIdx.x / (unsigned)ctas];
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(D.args + r);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(&A);
    for (int i = threadIdx.x; i < (int)(sizeof(PCGArgs) / 8); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    pcg_body<ClusterGroup>(A);
}

// ================================================================ split
//
// The same solve as k_pcg, one plain kernel per pass (one item per thread,
// full occupancy), for replay inside a CUDA graph.  Loop control lives on the
// device: the scalars sit in SplitState, every reducing kernel's last block
// (ticket counter) adds the block partials in block order and updates them,
// and the residual kernel sets the conditional handle of the graph's WHILE
// node to 0 once the solve is over.

#ifndef FFR_L0_BLOCKS
#define FFR_L0_BLOCKS 1184
#endif
constexpr int kSplitMaxBlocks = FFR_L0_BLOCKS;   // level-0 pass grid cap (a multiple of the 148 SMs)

struct SplitState {
    double bnorm, rz_old, beta, alpha, alpha_prev, res;
    int it, done, pending, flags, dpar, pad;
    unsigned ticket;
    unsigned pad2;
};


// Block partials -> partials[lb]; true in the one block of the room that
// arrives last, which then holds the room total (summed in block order) in v.
template <int NV>
__device__ bool last_block_total(double (&v)[NV], double *partials, unsigned *ticket, double *sh, BPos P)
{
    __shared__ int s_last;
    for (int a = 0; a < NV; a++) {
        const double t = block_sum(v[a], sh);
        if (threadIdx.x == 0) partials[(size_t)P.lb * NV + a] = t;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == (unsigned)P.nb - 1;
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    for (int a = 0; a < NV; a++) {
        double t = 0.0;
        for (int b = threadIdx.x; b < P.nb; b += blockDim.x) t += __ldcg(&partials[(size_t)b * NV + a]);
        v[a] = block_sum(t, sh);
    }
    if (threadIdx.x == 0) *ticket = 0;
    return true;
}

// ---- bodies of the split solve's kernels, for one room, given the block's
// position among that room's blocks.  `active` (batched solves only) counts
// the rooms still iterating: +1 when a room starts, -1 when it finishes.

__device__ __forceinline__ void sp_init_body(const PCGArgs &A, SplitState *ss, BPos P, int *active,
                                             cudaGraphConditionalHandle cond, int use_cond)
{
    __shared__ double sh[32];
    if (A.st && A.st->halt) {
        if (P.lb == 0 && threadIdx.x == 0) {
            ss->done = 1;
            if (use_cond) cudaGraphSetConditional(cond, 0);
        }
        return;
    }
    double acc[2] = {0.0, 0.0};
    pass_init(A, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x, acc);
    if (last_block_total<2>(acc, A.partials, &ss->ticket, sh, P) && threadIdx.x == 0) {
        ss->bnorm = sqrt(acc[0]);
        ss->it = 0;
        ss->pending = 0;
        ss->flags = 0;
        ss->dpar = 0;
        ss->res = 0.0;
        ss->alpha = ss->alpha_prev = ss->rz_old = ss->beta = 0.0;
        ss->done = ss->bnorm < 1e-15;
        if (!ss->done && active) atomicAdd(active, 1);
        if (use_cond) cudaGraphSetConditional(cond, ss->done ? 0u : 1u);
    }
}

__device__ __forceinline__ void sp_redpost_body(const PCGArgs &A, SplitState *ss, BPos P)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    pass_redpost_dot(A, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x, acc[0]);
    if (last_block_total<1>(acc, A.partials, &ss->ticket, sh, P) && threadIdx.x == 0) {
        ss->beta = ss->it == 0 ? 0.0 : acc[0] / ss->rz_old;
        ss->rz_old = acc[0];
    }
}

__device__ __forceinline__ void sp_direction_body(const PCGArgs &A, SplitState *ss, BPos P, int *active)
{
    __shared__ double sh[32];
    const double *dold = ss->dpar ? A.db : A.da;
    double *dnew = ss->dpar ? A.da : A.db;
    double acc[1] = {0.0};
    pass_direction(A, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x, ss->beta, ss->alpha_prev, ss->it > 0,
                   dold, dnew, acc[0]);
    if (last_block_total<1>(acc, A.partials, &ss->ticket, sh, P) && threadIdx.x == 0) {
        ss->dpar ^= 1;            // the new direction is current from here on
        ss->pending = 0;
        if (fabs(acc[0]) < 1e-30) {
            ss->flags |= FFR_FLAG_CG_BREAKDOWN;
            ss->done = 1;
            if (active) atomicSub(active, 1);
        } else {
            ss->alpha = ss->rz_old / acc[0];
        }
    }
}

__device__ __forceinline__ void sp_residual_body(const PCGArgs &A, SplitState *ss, BPos P, int *active,
                                                 cudaGraphConditionalHandle cond, int use_cond)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    pass_residual(A, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x, ss->alpha, acc[0]);
    if (last_block_total<1>(acc, A.partials, &ss->ticket, sh, P) && threadIdx.x == 0) {
        ss->pending = 1;
        ss->res = sqrt(acc[0]) / ss->bnorm;
        ss->it += 1;
        if (ss->res < A.tol) {
            ss->done = 1;
        } else if (ss->it >= A.max_iter) {
            ss->flags |= FFR_FLAG_CG_MAXITER;
            ss->done = 1;
        } else {
            ss->alpha_prev = ss->alpha;
        }
        if (ss->done && active) atomicSub(active, 1);
        if (use_cond) cudaGraphSetConditional(cond, ss->done ? 0u : 1u);
    }
}

__device__ __forceinline__ void sp_final_body(const PCGArgs &A, const SplitState *ss, BPos P)
{
    if (ss->pending)
        pass_final_x(A, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x, ss->alpha, ss->dpar ? A.db : A.da);
}

__device__ __forceinline__ void sp_backsub_body(const PCGArgs &A, const SplitState *ss, BPos P)
{
    pass_backsub(A, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x);
    if (P.lb == 0 && threadIdx.x == 0) {
        const int iters = ss->bnorm < 1e-15 ? 0 : ss->it;
        if (A.out_res) *A.out_res = ss->res;
        if (A.out_iters) *A.out_iters = iters;
        if (A.out_flags) *A.out_flags = ss->flags;
        if (A.st) {
            A.st->pres = ss->res;
            A.st->iters = iters;
            atomicOr(&A.st->flags, ss->flags);
        }
    }
}

// Levels mid .. nlev-1 of the V-cycle in one thread-block cluster: the
// grid-sized levels from mid on (pre-smooth + restriction going down,
// post-smooth coming up) with the hardware cluster barrier between passes,
// and the levels of at most kBlockLevelCells cells in block 0.  Every cell
// update is the one the one-kernel-per-pass form makes (the colours are
// Jacobi sweeps), so the result does not depend on this grouping.
__device__ __forceinline__ void sp_mid_body(const PCGArgs &A, int mid)
{
    auto cl = cooperative_groups::this_cluster();
    const MGDev &M = A.M;
    const int t0 = (int)cl.block_rank() * blockDim.x + threadIdx.x, nth = (int)cl.num_blocks() * blockDim.x;
    auto csync = [&]() {
        __threadfence();
        cl.sync();
    };
    const int top = min(M.nlev_grid, M.nlev - 1);
    for (int l = mid; l < top; l++) {
        smooth_color<false>(A, M.lv, M.nlev, l, 1, t0, nth);
        csync();
        for (int sw = 1; sw < level_sweeps(l); sw++) {
            smooth_color<false>(A, M.lv, M.nlev, l, 0, t0, nth);
            csync();
            smooth_color<false>(A, M.lv, M.nlev, l, 1, t0, nth);
            csync();
        }
        restrict_level(A, M.lv, l, t0, nth);
        csync();
    }
    if (M.nlev_grid < M.nlev) {
        if (cl.block_rank() == 0) block_vcycle(A, M.nlev_grid);
        csync();
    }
    for (int l = top - 1; l >= mid; l--) {
        smooth_color<true>(A, M.lv, M.nlev, l, 1, t0, nth);
        csync();
        smooth_color<false>(A, M.lv, M.nlev, l, 0, t0, nth);
        for (int sw = 1; sw < level_sweeps(l); sw++) {
            csync();
            smooth_color<false>(A, M.lv, M.nlev, l, 1, t0, nth);
            csync();
            smooth_color<false>(A, M.lv, M.nlev, l, 0, t0, nth);
        }
        if (l > mid) csync();
    }
}

// ---- one-room kernels (the grid is the room's)


__device__ __forceinline__ int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int gthreads() { return gridDim.x * blockDim.x; }

// use_cond: the kernel runs inside a graph with a WHILE node on `cond`
// (otherwise the host paces the iterations and reads ss->done).
__global__ void __launch_bounds__(256) k_sp_init(PCGArgs A, SplitState *ss, cudaGraphConditionalHandle cond,
                                                 int use_cond)
{
    sp_init_body(A, ss, grid_pos(), nullptr, cond, use_cond);
}

template <bool CORR>
__global__ void __launch_bounds__(256) k_sp_smooth(PCGArgs A, const SplitState *ss, int l, int color)
{
    if (ss->done) return;
    smooth_color<CORR>(A, A.M.lv, A.M.nlev, l, color, gtid(), gthreads());
}

__global__ void __launch_bounds__(256) k_sp_restrict(PCGArgs A, const SplitState *ss, int l)
{
    if (ss->done) return;
    restrict_level(A, A.M.lv, l, gtid(), gthreads());
}

__global__ void __launch_bounds__(1024) k_sp_coarse(PCGArgs A, const SplitState *ss, int lo)
{
    if (ss->done) return;
    block_vcycle(A, lo);
}

__global__ void __launch_bounds__(kMidThreads, 1) k_sp_mid(PCGArgs A, const SplitState *ss, int mid)
{
    if (ss->done) return;   // the same value in every block of the cluster
    sp_mid_body(A, mid);
}

__global__ void __launch_bounds__(256) k_sp_redpost(PCGArgs A, SplitState *ss)
{
    if (ss->done) return;
    sp_redpost_body(A, ss, grid_pos());
}

__global__ void __launch_bounds__(256, 3) k_sp_direction(PCGArgs A, SplitState *ss)
{
    if (ss->done) return;
    sp_direction_body(A, ss, grid_pos(), nullptr);
}

__global__ void __launch_bounds__(256) k_sp_residual(PCGArgs A, SplitState *ss, cudaGraphConditionalHandle cond,
                                                     int use_cond)
{
    if (ss->done) {
        if (use_cond && gtid() == 0) cudaGraphSetConditional(cond, 0);
        return;
    }
    sp_residual_body(A, ss, grid_pos(), nullptr, cond, use_cond);
}

__global__ void __launch_bounds__(256) k_sp_extrapolate(PCGArgs A)
{
    pass_extrapolate(A, gtid(), gthreads());
}

__global__ void __launch_bounds__(256) k_sp_final(PCGArgs A, const SplitState *ss)
{
    if (A.st && A.st->halt) return;
    sp_final_body(A, ss, grid_pos());
}

__global__ void __launch_bounds__(256) k_sp_backsub(PCGArgs A, const SplitState *ss)
{
    if (A.st && A.st->halt) return;
    sp_backsub_body(A, ss, grid_pos());
}

// ---- batched kernels: one launch works on every room of a batch.  Block b
// belongs to room m.room[b]; the room's blocks are m.first[r] ..
// m.first[r + 1] - 1, as many as its one-room launch has, so every room
// computes exactly what its own launch would.  Each block copies its room's
// arguments to shared memory first.

__device__ __forceinline__ void load_args(PCGArgs &dst, const PCGArgs *src)
{
    static_assert(sizeof(PCGArgs) % 8 == 0, "PCGArgs copy in 8-byte words");
    const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
    unsigned long long *d = reinterpret_cast<unsigned long long *>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(PCGArgs) / 8); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_bsp_extrapolate(BatchDev D, BMap m)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    load_args(A, D.args + r);
    pass_extrapolate(A, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x);
}

__global__ void __launch_bounds__(256) k_bsp_init(BatchDev D, BMap m)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    load_args(A, D.args + r);
    sp_init_body(A, D.ss[r], P, D.active, cudaGraphConditionalHandle{}, 0);
}

template <bool CORR>
__global__ void __launch_bounds__(256) k_bsp_smooth(BatchDev D, BMap m, int l, int color)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    if (D.ss[r]->done) return;
    load_args(A, D.args + r);
    smooth_color<CORR>(A, A.M.lv, A.M.nlev, l, color, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x);
}

__global__ void __launch_bounds__(256) k_bsp_restrict(BatchDev D, BMap m, int l)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    if (D.ss[r]->done) return;
    load_args(A, D.args + r);
    restrict_level(A, A.M.lv, l, P.lb * blockDim.x + threadIdx.x, P.nb * blockDim.x);
}

// one block per room of the list: the levels from nlev_grid on
__global__ void __launch_bounds__(1024) k_bsp_coarse(BatchDev D, const int *rooms)
{
    __shared__ __align__(16) PCGArgs A;
    const int r = rooms[blockIdx.x];
    if (D.ss[r]->done) return;
    load_args(A, D.args + r);
    block_vcycle(A, A.M.nlev_grid);
}

__global__ void __launch_bounds__(256) k_bsp_redpost(BatchDev D, BMap m)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    if (D.ss[r]->done) return;
    load_args(A, D.args + r);
    sp_redpost_body(A, D.ss[r], P);
}

__global__ void __launch_bounds__(256, 3) k_bsp_direction(BatchDev D, BMap m)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    if (D.ss[r]->done) return;
    load_args(A, D.args + r);
    sp_direction_body(A, D.ss[r], P, D.active);
}

__global__ void __launch_bounds__(256) k_bsp_residual(BatchDev D, BMap m)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    if (D.ss[r]->done) return;
    load_args(A, D.args + r);
    sp_residual_body(A, D.ss[r], P, D.active, cudaGraphConditionalHandle{}, 0);
}

// Condition of the batched solve's WHILE node: iterate while any room of
// the batch is still iterating (the count its init and residual passes keep).
__global__ void k_bsp_cond(const int *active, cudaGraphConditionalHandle cond)
{
    if (threadIdx.x == 0) cudaGraphSetConditional(cond, *(volatile const int *)active > 0 ? 1u : 0u);
}

__global__ void __launch_bounds__(256) k_bsp_final(BatchDev D, BMap m)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    load_args(A, D.args + r);
    if (A.st && A.st->halt) return;
    sp_final_body(A, D.ss[r], P);
}

__global__ void __launch_bounds__(256) k_bsp_backsub(BatchDev D, BMap m)
{
    __shared__ __align__(16) PCGArgs A;
    BPos P;
    const int r = bmap(m, P);
    load_args(A, D.args + r);
    if (A.st && A.st->halt) return;
    sp_backsub_body(A, D.ss[r], P);
}

}  // namespace ffr

// ---------------------------------------------------------------- host

namespace ffr {

size_t mg_bytes(const HostRoom &r, const MGHost &h)
{
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const RoomGeom &g = r.g;
    size_t b = 2 * al(4 * g.n) + 9 * al(4 * std::max(g.nx, std::max(g.ny, g.nz)));
    for (size_t l = 1; l < h.nx.size(); l++) {
        const size_t m = (size_t)h.nx[l] * h.ny[l] * h.nz[l];
        b += al(16 * m) + 2 * al(4 * m);
    }
    return b + 256;
}

size_t mg_stage_bytes(const HostRoom &r)
{
    return 4 * 3 * (size_t)(r.g.nx + r.g.ny + r.g.nz) + 9 * 16;
}

int mg_upload(const HostRoom &r, const MGHost &h, const RoomDev &R, Arena &ar, HostStage &hs, cudaStream_t s,
              MGDev &M)
{
    const RoomGeom &g = r.g;
    M.nlev = (int)h.nx.size();
    M.nlev_grid = 0;
    for (int l = 0; l < M.nlev; l++)
        if ((long long)h.nx[l] * h.ny[l] * h.nz[l] > kBlockLevelCells) M.nlev_grid = l + 1;
    // first level (>= 1) small enough for the one-cluster part of the split solve
    M.nlev_mid = 1;
    for (int l = 1; l < M.nlev; l++)
        if ((long long)h.nx[l] * h.ny[l] * h.nz[l] > kMidLevelCells) M.nlev_mid = l + 1;
    M.nlev_mid = std::min(M.nlev_mid, std::max(1, M.nlev_grid));
    // fine-level factors in FP32 (PoissonSolver.cpp:33-49 centre distances)
    auto axis = [](const std::vector<double> &hh, std::vector<float> &d, std::vector<float> &il,
                   std::vector<float> &ir) {
        const int m = (int)hh.size();
        d.resize(m); il.resize(m); ir.resize(m);
        for (int i = 0; i < m; i++) {
            d[i] = (float)hh[i];
            const double hl = (i > 0) ? 0.5 * (hh[i - 1] + hh[i]) : hh[i];
            const double hr = (i < m - 1) ? 0.5 * (hh[i] + hh[i + 1]) : hh[i];
            il[i] = (float)(1.0 / hl);
            ir[i] = (float)(1.0 / hr);
        }
    };
    std::vector<float> dx, ixl, ixr, dy, iyl, iyr, dz, izl, izr;
    axis(r.dxv, dx, ixl, ixr);
    axis(r.dyv, dy, iyl, iyr);
    axis(r.dzv, dz, izl, izr);
    float *fx = ar.take<float>(g.nx), *fxl = ar.take<float>(g.nx), *fxr = ar.take<float>(g.nx);
    float *fy = ar.take<float>(g.ny), *fyl = ar.take<float>(g.ny), *fyr = ar.take<float>(g.ny);
    float *fz = ar.take<float>(g.nz), *fzl = ar.take<float>(g.nz), *fzr = ar.take<float>(g.nz);
    // (6 arrays were budgeted per axis set; dx/dy/dz reuse the same slots)
    M.lv[0].nx = g.nx; M.lv[0].ny = g.ny; M.lv[0].nz = g.nz; M.lv[0].n = (int)g.n;
    M.lv[0].sx = h.sx[0]; M.lv[0].sy = h.sy[0]; M.lv[0].sz = h.sz[0];
    M.lv[0].coef = nullptr;
    M.lv[0].x = ar.take<float>(g.n);
    M.r32 = ar.take<float>(g.n);
    M.lv[0].b = M.r32;
    if (!M.r32 || !fzr) return fail(FFR_ENOMEM, "arena exhausted (multigrid)");
    {
        float *dev[9] = {fx, fxl, fxr, fy, fyl, fyr, fz, fzl, fzr};
        const std::vector<float> *src[9] = {&dx, &ixl, &ixr, &dy, &iyl, &iyr, &dz, &izl, &izr};
        for (int q = 0; q < 9; q++) {
            const int rc = hs.put(dev[q], src[q]->data(), 4 * src[q]->size(), s);
            if (rc) return rc;
        }
    }
    FFR_CUDA(cudaMemsetAsync(M.lv[0].x, 0, 4 * g.n, s));
    FFR_CUDA(cudaMemsetAsync(M.r32, 0, 4 * g.n, s));
    M.dx = fx; M.dy = fy; M.dz = fz;
    auto flat = [](const std::vector<double> &hh) {
        for (double v : hh) if (v != hh[0]) return false;
        return true;
    };
    M.uniform = flat(r.dxv) && flat(r.dyv) && flat(r.dzv);
    M.tx = (float)(r.dyv[0] * r.dzv[0] / r.dxv[0]);
    M.ty = (float)(r.dxv[0] * r.dzv[0] / r.dyv[0]);
    M.tz = (float)(r.dxv[0] * r.dyv[0] / r.dzv[0]);
    M.vol = (float)(r.dxv[0] * r.dyv[0] * r.dzv[0]);
    // the reference's scales 1/(h_face h) with h_face = h (uniform axis)
    M.s64x = 1.0 / (r.dxv[0] * r.dxv[0]);
    M.s64y = 1.0 / (r.dyv[0] * r.dyv[0]);
    M.s64z = 1.0 / (r.dzv[0] * r.dzv[0]);
    M.vol64 = r.dxv[0] * r.dyv[0] * r.dzv[0];
    {
        // diagonal of a row with six unknown neighbours, summed in the row's order
        double d = 0.0;
        const double sx[6] = {M.s64x, M.s64x, M.s64y, M.s64y, M.s64z, M.s64z};
        for (double v : sx) d += v;
        M.diag64 = d;
    }
    M.ixl = fxl; M.ixr = fxr; M.iyl = fyl; M.iyr = fyr; M.izl = fzl; M.izr = fzr;
    for (int l = 1; l < M.nlev; l++) {
        const size_t m = (size_t)h.nx[l] * h.ny[l] * h.nz[l];
        MGLevel &L = M.lv[l];
        L.nx = h.nx[l]; L.ny = h.ny[l]; L.nz = h.nz[l]; L.n = (int)m;
        L.sx = h.sx[l]; L.sy = h.sy[l]; L.sz = h.sz[l];
        L.coef = ar.take<float4>(m);
        L.x = ar.take<float>(m);
        L.b = ar.take<float>(m);
        if (!L.b) return fail(FFR_ENOMEM, "arena exhausted (multigrid levels)");
        FFR_CUDA(cudaMemsetAsync(L.x, 0, 4 * m, s));
        FFR_CUDA(cudaMemsetAsync(L.b, 0, 4 * m, s));
    }
    if (M.nlev > 1) {
        // couplings of two consecutive levels in stream-ordered scratch
        // (level 1 is the largest coarse level)
        const size_t m1 = (size_t)h.nx[1] * h.ny[1] * h.nz[1];
        const size_t per = 6 * 8 * m1 + ((m1 + 255) & ~size_t(255));
        char *scratch = nullptr;
        FFR_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&scratch), 2 * per, s));
        LevelOps ops[2];
        for (int b = 0; b < 2; b++) {
            char *p = scratch + b * per;
            for (int d = 0; d < 6; d++) ops[b].t[d] = reinterpret_cast<double *>(p + (size_t)d * 8 * m1);
            ops[b].act = reinterpret_cast<uint8_t *>(p + 6 * 8 * m1);
        }
        int rc = FFR_OK;
        for (int l = 1; l < M.nlev && !rc; l++) {
            CoarsenArgs c{};
            c.ct = R.ct; c.dxv = R.dxv; c.dyv = R.dyv; c.dzv = R.dzv;
            c.cur = ops[l & 1];
            if (l == 1) c.cur.act = nullptr;     // gather from the fine cells
            c.next = ops[(l + 1) & 1];
            c.nx = h.nx[l - 1]; c.ny = h.ny[l - 1]; c.nz = h.nz[l - 1];
            c.sx = h.sx[l - 1]; c.sy = h.sy[l - 1]; c.sz = h.sz[l - 1];
            c.mx = h.nx[l]; c.my = h.ny[l]; c.mz = h.nz[l];
            const long long m = (long long)c.mx * c.my * c.mz;
            k_mg_coarsen<<<coarse_blocks(m), 256, 0, s>>>(c);
            k_mg_coef<<<coarse_blocks(m), 256, 0, s>>>(c.next, c.mx, c.my, c.mz,
                                                       const_cast<float4 *>(M.lv[l].coef));
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = cuda_fail(e, "multigrid coefficient kernels");
            count_launch(2);
        }
        cudaFreeAsync(scratch, s);
        if (rc) return rc;
    }
    return FFR_OK;
}

unsigned pcg_max_blocks()
{
    static unsigned cap = 0;
    if (!cap) {
        int per_sm = 0, dev = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<GridGroup>, 256, 0);
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (per_sm <= 0) per_sm = 1;
        if (sms <= 0) sms = 148;
        cap = (unsigned)(per_sm * sms);
    }
    return cap;
}

int launch_pcg_cluster(const PCGArgs &a, cudaStream_t s, int ctas)
{
    static bool attr_set = false;
    if (!attr_set) {
        FFR_CUDA(cudaFuncSetAttribute(k_pcg<ClusterGroup, kClusterThreads>,
                                      cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        attr_set = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FFR_CUDA(cudaLaunchKernelEx(&cfg, k_pcg<ClusterGroup, kClusterThreads>, a));
    count_launch(1);
    return FFR_OK;
}

int launch_pcg(const PCGArgs &a, cudaStream_t s, unsigned *blocks_used, unsigned override_blocks)
{
    const unsigned want = (unsigned)std::max<long long>(1, (a.R.n + 255) / 256);
    unsigned blocks = std::max(1u, std::min(pcg_max_blocks(), want));
    if (override_blocks) blocks = std::min(blocks, override_blocks);
    if (blocks_used) *blocks_used = blocks;
    FFR_CUDA(cudaMemsetAsync(a.gs, 0, sizeof(GridSync), s));
    void *args[] = {(void *)&a};
    FFR_CUDA(cudaLaunchCooperativeKernel((void *)k_pcg<GridGroup>, dim3(blocks), dim3(256), args, 0, s));
    count_launch(1);
    return FFR_OK;
}

}  // namespace ffr

namespace ffr {

namespace {

// Level-0 passes (over cells or cell pairs): four cells per thread, at most
// kSplitMaxBlocks blocks.
unsigned split_blocks_level0(long long n)
{
    return (unsigned)std::max<long long>(1, std::min<long long>((n + 1023) / 1024, kSplitMaxBlocks));
}

// Grid sizes of the split solve's launches: two items (pairs or coarse
// cells) per thread, so each block amortises its start-up over more work
// (many rooms in one batched launch fill the GPU by their number).
unsigned split_blocks_pairs(const MGDev &M, int l)
{
    const MGLevel &L = M.lv[l];
    const long long w = (long long)L.nx * L.ny * ((L.nz + 1) / 2);
    return (unsigned)std::max<long long>(1, (w + 511) / 512);
}

unsigned split_blocks_cells(const MGDev &M, int l)
{
    return (unsigned)std::max<long long>(1, ((long long)M.lv[l].n + 511) / 512);
}

// Cluster size of k_sp_mid: the largest of 16 and 8 blocks that the device
// can co-schedule (16 needs the non-portable cluster-size attribute).
int mid_cluster_ctas()
{
    static int ctas = 0;
    if (ctas) return ctas;
    cudaFuncSetAttribute(k_sp_mid, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    for (int want : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)want);
        cfg.blockDim = dim3(kMidThreads);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)want;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, k_sp_mid, &cfg) == cudaSuccess && nclusters > 0) {
            ctas = want;
            return ctas;
        }
        cudaGetLastError();
    }
    ctas = 1;
    return ctas;
}

// Kernels one PCG iteration of the split solve runs (the body below).
unsigned split_body_kernels(const MGDev &M)
{
    if (M.nlev <= 1) return 3;
    const int top = std::min(M.nlev_grid, M.nlev - 1);
    const int gdown = std::min(M.nlev_mid, top);
    unsigned k = 2u * (unsigned)gdown;                        // grid levels: smooth + restrict
    for (int l = 0; l < gdown; l++) k += 2u * (level_sweeps(l) - 1);   // their further pre-sweeps
    if (M.nlev_mid < top || M.nlev_grid < M.nlev) k += 1;     // k_sp_mid
    for (int l = 1; l < gdown; l++) k += 2u * level_sweeps(l);         // post-smoothing, levels gdown-1 .. 1
    if (M.nlev_grid >= 1) k += 2u * level_sweeps(0) - 1;      // level-0 post-smoothing before the r.z pass
    return k + 3;                                             // red post + r.z, direction, residual
}

// Launches one PCG iteration of the split solve on stream bs.
int split_iteration(const PCGArgs &a, SplitState *ss, cudaStream_t bs, cudaGraphConditionalHandle cond,
                    int use_cond)
{
    const MGDev &M = a.M;
    const unsigned cb = split_blocks_level0(a.R.n);
    int rc = FFR_OK;
    auto chk = [&]() {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess && rc == FFR_OK) rc = cuda_fail(e, "split kernel launch");
        count_launch(1);
    };
    if (M.nlev > 1) {
        const int top = std::min(M.nlev_grid, M.nlev - 1);
        const int gdown = std::min(M.nlev_mid, top);
        for (int l = 0; l < gdown; l++) {
            k_sp_smooth<false><<<split_blocks_pairs(M, l), 256, 0, bs>>>(a, ss, l, 1);
            chk();
            for (int sw = 1; sw < level_sweeps(l); sw++) {
                k_sp_smooth<false><<<split_blocks_pairs(M, l), 256, 0, bs>>>(a, ss, l, 0);
                chk();
                k_sp_smooth<false><<<split_blocks_pairs(M, l), 256, 0, bs>>>(a, ss, l, 1);
                chk();
            }
            k_sp_restrict<<<split_blocks_cells(M, l + 1), 256, 0, bs>>>(a, ss, l);
            chk();
        }
        if (M.nlev_mid < top || M.nlev_grid < M.nlev) {
            const int ctas = mid_cluster_ctas();
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)ctas);
            cfg.blockDim = dim3(kMidThreads);
            cfg.stream = bs;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = (unsigned)ctas;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            cudaError_t e = cudaLaunchKernelEx(&cfg, k_sp_mid, a, (const SplitState *)ss, M.nlev_mid);
            if (e != cudaSuccess && rc == FFR_OK) rc = cuda_fail(e, "cudaLaunchKernelEx(k_sp_mid)");
            chk();
        }
        for (int l = gdown - 1; l >= 1; l--) {
            k_sp_smooth<true><<<split_blocks_pairs(M, l), 256, 0, bs>>>(a, ss, l, 1);
            chk();
            k_sp_smooth<false><<<split_blocks_pairs(M, l), 256, 0, bs>>>(a, ss, l, 0);
            chk();
            for (int sw = 1; sw < level_sweeps(l); sw++) {
                k_sp_smooth<false><<<split_blocks_pairs(M, l), 256, 0, bs>>>(a, ss, l, 1);
                chk();
                k_sp_smooth<false><<<split_blocks_pairs(M, l), 256, 0, bs>>>(a, ss, l, 0);
                chk();
            }
        }
        if (M.nlev_grid >= 1) {
            k_sp_smooth<true><<<split_blocks_pairs(M, 0), 256, 0, bs>>>(a, ss, 0, 1);
            chk();
            // the further sweeps; the last red half is k_sp_redpost's
            for (int sw = 1; sw < level_sweeps(0); sw++) {
                k_sp_smooth<false><<<split_blocks_pairs(M, 0), 256, 0, bs>>>(a, ss, 0, 0);
                chk();
                k_sp_smooth<false><<<split_blocks_pairs(M, 0), 256, 0, bs>>>(a, ss, 0, 1);
                chk();
            }
        }
    }
    k_sp_redpost<<<cb, 256, 0, bs>>>(a, ss);
    chk();
    k_sp_direction<<<cb, 256, 0, bs>>>(a, ss);
    chk();
    k_sp_residual<<<cb, 256, 0, bs>>>(a, ss, cond, use_cond);
    chk();
    return rc;
}

}  // namespace

size_t split_state_bytes() { return sizeof(SplitState); }

int launch_extrapolate(const PCGArgs &a, cudaStream_t s)
{
    k_sp_extrapolate<<<split_blocks_level0(a.R.n), 256, 0, s>>>(a);
    FFR_LAUNCHED(1);
    return FFR_OK;
}

int capture_split_pcg(const PCGArgs &a, void *ss_dev, cudaStream_t s, cudaStream_t bs, unsigned *body_kernels)
{
    SplitState *ss = static_cast<SplitState *>(ss_dev);
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    FFR_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(FFR_EINVAL, "split solve must be captured");
    cudaGraphConditionalHandle cond;
    FFR_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
    const unsigned cb = split_blocks_level0(a.R.n);
    k_sp_init<<<cb, 256, 0, s>>>(a, ss, cond, 1);
    FFR_LAUNCHED(1);
    FFR_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    FFR_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    FFR_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));

    // one PCG iteration, replayed while the residual kernel keeps the condition set
    FFR_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int rc = split_iteration(a, ss, bs, cond, 1);
    if (body_kernels) *body_kernels = split_body_kernels(a.M);
    cudaGraph_t body_out = nullptr;
    cudaError_t e = cudaStreamEndCapture(bs, &body_out);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(PCG iteration)");

    k_sp_final<<<cb, 256, 0, s>>>(a, ss);
    FFR_LAUNCHED(1);
    k_sp_backsub<<<cb, 256, 0, s>>>(a, ss);
    FFR_LAUNCHED(1);
    return FFR_OK;
}


int SplitHost::init()
{
    if (flags) return FFR_OK;
    flags = static_cast<int *>(pinned_get(4 * sizeof(int)));
    if (!flags) return fail(FFR_ENOMEM, "pinned host memory");
    for (int k = 0; k < 2; k++) FFR_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
    return FFR_OK;
}

void SplitHost::release()
{
    pinned_put(flags, 4 * sizeof(int));
    for (int k = 0; k < 2; k++)
        if (ev[k]) cudaEventDestroy(ev[k]);
    flags = nullptr;
    ev[0] = ev[1] = nullptr;
}

int launch_split_pcg(const PCGArgs &a, void *ss_dev, cudaStream_t s, SplitHost &h)
{
    int rc = h.init();
    if (rc) return rc;
    SplitState *ss = static_cast<SplitState *>(ss_dev);
    const unsigned cb = split_blocks_level0(a.R.n);
    k_sp_init<<<cb, 256, 0, s>>>(a, ss, cudaGraphConditionalHandle{}, 0);
    FFR_LAUNCHED(1);
    const int max_iter = std::max(0, a.max_iter);
    int launched = 0;
    // queue `nb` iterations, then a copy of (it, done) into slot `slot`
    auto batch = [&](int nb, int slot) -> int {
        for (int k = 0; k < nb; k++) {
            int r = split_iteration(a, ss, s, cudaGraphConditionalHandle{}, 0);
            if (r) return r;
        }
        launched += nb;
        FFR_CUDA(cudaMemcpyAsync(h.flags + 2 * slot, &ss->it, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        FFR_CUDA(cudaEventRecord(h.ev[slot], s));
        return FFR_OK;
    };
    // the first batch is the previous solve's count less two; then batches of
    // two, each queued before the host waits on the one before it, so the
    // stream never drains while the host decides
    int slot = 0;
    if (max_iter > 0) {
        rc = batch(std::min(max_iter, std::max(1, h.last_iters - 2)), slot);
        if (rc) return rc;
        while (true) {
            const int prev = slot;
            const bool more = launched < max_iter;
            if (more) {
                slot ^= 1;
                rc = batch(std::min(2, max_iter - launched), slot);
                if (rc) return rc;
            }
            FFR_CUDA(cudaEventSynchronize(h.ev[prev]));
            if (h.flags[2 * prev + 1]) {
                h.last_iters = h.flags[2 * prev];
                break;
            }
            if (!more) break;
        }
    }
    k_sp_final<<<cb, 256, 0, s>>>(a, ss);
    FFR_LAUNCHED(1);
    k_sp_backsub<<<cb, 256, 0, s>>>(a, ss);
    FFR_LAUNCHED(1);
    return FFR_OK;
}


// ---------------------------------------------------------- batched solve

namespace {

// Room -> (grid size) of each launch shape, from the one-room launch sizes.
struct RoomShape {
    unsigned cb;                  // level-0 passes
    int gdown;                    // grid levels smoothed and restricted on the way down
    unsigned pairs[kMaxLevels], coarse[kMaxLevels];
    bool mid;                     // has levels small enough for one block
};

RoomShape room_shape(const PCGArgs &a)
{
    RoomShape r{};
    const MGDev &M = a.M;
    r.cb = split_blocks_level0(a.R.n);
    if (M.nlev > 1) {
        // every grid-sized level in batched launches (many rooms fill the
        // GPU there), the levels of at most kBlockLevelCells cells in one
        // block per room; the cell updates are those of the one-room split
        // solve, which runs the levels from nlev_mid on in one cluster
        const int top = std::min(M.nlev_grid, M.nlev - 1);
        r.gdown = top;
        for (int l = 0; l < r.gdown; l++) {
            r.pairs[l] = split_blocks_pairs(M, l);
            r.coarse[l] = split_blocks_cells(M, l + 1);
        }
        r.mid = M.nlev_grid < M.nlev;
    }
    return r;
}

// Appends the table of one launch shape: room[] over all blocks, first[]
// per room (nrooms + 1 entries; rooms without blocks get an empty range).
unsigned build_map(std::vector<int> &room, std::vector<int> &first, const std::vector<unsigned> &nb)
{
    first.push_back(0);
    unsigned total = 0;
    for (size_t r = 0; r < nb.size(); r++) {
        for (unsigned b = 0; b < nb[r]; b++) room.push_back((int)r);
        total += nb[r];
        first.push_back((int)total);
    }
    return total;
}

}  // namespace

int batch_split_build(BatchSplit &B, const std::vector<PCGArgs> &args, const std::vector<void *> &ss)
{
    const int n = (int)args.size();
    B.nrooms = n;
    if (n == 0) return FFR_OK;
    std::vector<RoomShape> sh(n);
    int nlev = 0;
    for (int r = 0; r < n; r++) {
        sh[r] = room_shape(args[r]);
        nlev = std::max(nlev, sh[r].gdown);
    }
    B.nlev = nlev;
    // host images of every table, then one device allocation
    struct Tab {
        std::vector<int> room, first;
        unsigned total = 0;
    };
    Tab t_cells0, t_pairs[kMaxLevels], t_coarse[kMaxLevels];
    std::vector<unsigned> nb(n);
    for (int r = 0; r < n; r++) nb[r] = sh[r].cb;
    t_cells0.total = build_map(t_cells0.room, t_cells0.first, nb);
    for (int l = 0; l < nlev; l++) {
        for (int r = 0; r < n; r++) nb[r] = l < sh[r].gdown ? sh[r].pairs[l] : 0;
        t_pairs[l].total = build_map(t_pairs[l].room, t_pairs[l].first, nb);
        for (int r = 0; r < n; r++) nb[r] = l < sh[r].gdown ? sh[r].coarse[l] : 0;
        t_coarse[l].total = build_map(t_coarse[l].room, t_coarse[l].first, nb);
    }
    std::vector<int> mids;
    for (int r = 0; r < n; r++)
        if (sh[r].mid) mids.push_back(r);
    // the one-cluster-per-room launch takes the rooms largest first, so the
    // last clusters to start are the shortest (less tail at the stage end)
    std::vector<int> order(n);
    for (int r = 0; r < n; r++) order[r] = r;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return args[a].R.n > args[b].R.n; });
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t bytes = al(sizeof(PCGArgs) * n) + al(sizeof(void *) * n) + al(sizeof(int)) +
                   al(4 * (t_cells0.room.size() + t_cells0.first.size())) + al(4 * (mids.size() + 1)) +
                   al(4 * n);
    for (int l = 0; l < nlev; l++)
        bytes += al(4 * (t_pairs[l].room.size() + t_pairs[l].first.size())) +
                 al(4 * (t_coarse[l].room.size() + t_coarse[l].first.size()));
    std::vector<unsigned char> host(bytes, 0);
    if (bytes > B.cap) {
        if (B.dev) cudaFree(B.dev);
        B.dev = nullptr;
        B.cap = 0;
        FFR_CUDA(cudaMalloc(&B.dev, bytes + bytes / 2));
        B.cap = bytes + bytes / 2;
    }
    if (!B.active_host) FFR_CUDA(cudaHostAlloc(&B.active_host, 2 * sizeof(int), cudaHostAllocDefault));
    for (int k = 0; k < 2; k++)
        if (!B.ev[k]) FFR_CUDA(cudaEventCreateWithFlags(&B.ev[k], cudaEventDisableTiming));
    unsigned char *dbase = static_cast<unsigned char *>(B.dev);
    size_t off = 0;
    auto put = [&](const void *src, size_t len) -> unsigned char * {
        if (len) std::memcpy(host.data() + off, src, len);
        unsigned char *d = dbase + off;
        off += al(len);
        return d;
    };
    B.D.args = reinterpret_cast<const PCGArgs *>(put(args.data(), sizeof(PCGArgs) * n));
    B.D.ss = reinterpret_cast<SplitState *const *>(put(ss.data(), sizeof(void *) * n));
    int zero = 0;
    B.D.active = reinterpret_cast<int *>(put(&zero, sizeof(int)));
    auto put_map = [&](const Tab &t, BMap &m) {
        std::vector<int> both(t.room);
        both.insert(both.end(), t.first.begin(), t.first.end());
        const int *d = reinterpret_cast<const int *>(put(both.data(), 4 * both.size()));
        m.room = d;
        m.first = d + t.room.size();
    };
    put_map(t_cells0, B.cells0);
    B.nb_cells0 = t_cells0.total;
    for (int l = 0; l < nlev; l++) {
        put_map(t_pairs[l], B.pairs[l]);
        B.nb_pairs[l] = t_pairs[l].total;
        put_map(t_coarse[l], B.coarse[l]);
        B.nb_coarse[l] = t_coarse[l].total;
    }
    mids.push_back(0);
    B.mid_rooms = reinterpret_cast<const int *>(put(mids.data(), 4 * mids.size()));
    B.nmid = (int)mids.size() - 1;
    B.cluster_order = reinterpret_cast<const int *>(put(order.data(), 4 * order.size()));
    FFR_CUDA(cudaMemcpy(B.dev, host.data(), bytes, cudaMemcpyHostToDevice));
    return FFR_OK;
}

void batch_split_release(BatchSplit &B)
{
    if (B.dev) cudaFree(B.dev);
    B.dev = nullptr;
    B.cap = 0;
    B.nrooms = 0;
    B.nlev = 0;
    B.nmid = 0;
}

namespace {

int batch_iteration(BatchSplit &B, cudaStream_t s)
{
    int rc = FFR_OK;
    auto chk = [&](const char *what) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess && rc == FFR_OK) rc = cuda_fail(e, what);
        count_launch(1);
    };
    for (int l = 0; l < B.nlev; l++) {
        if (!B.nb_pairs[l]) continue;
        k_bsp_smooth<false><<<B.nb_pairs[l], 256, 0, s>>>(B.D, B.pairs[l], l, 1);
        chk("k_bsp_smooth");
        for (int sw = 1; sw < level_sweeps(l); sw++) {
            k_bsp_smooth<false><<<B.nb_pairs[l], 256, 0, s>>>(B.D, B.pairs[l], l, 0);
            chk("k_bsp_smooth");
            k_bsp_smooth<false><<<B.nb_pairs[l], 256, 0, s>>>(B.D, B.pairs[l], l, 1);
            chk("k_bsp_smooth");
        }
        k_bsp_restrict<<<B.nb_coarse[l], 256, 0, s>>>(B.D, B.coarse[l], l);
        chk("k_bsp_restrict");
    }
    if (B.nmid) {
        k_bsp_coarse<<<B.nmid, 1024, 0, s>>>(B.D, B.mid_rooms);
        chk("k_bsp_coarse");
    }
    for (int l = B.nlev - 1; l >= 1; l--) {
        if (!B.nb_pairs[l]) continue;
        k_bsp_smooth<true><<<B.nb_pairs[l], 256, 0, s>>>(B.D, B.pairs[l], l, 1);
        chk("k_bsp_smooth");
        k_bsp_smooth<false><<<B.nb_pairs[l], 256, 0, s>>>(B.D, B.pairs[l], l, 0);
        chk("k_bsp_smooth");
        for (int sw = 1; sw < level_sweeps(l); sw++) {
            k_bsp_smooth<false><<<B.nb_pairs[l], 256, 0, s>>>(B.D, B.pairs[l], l, 1);
            chk("k_bsp_smooth");
            k_bsp_smooth<false><<<B.nb_pairs[l], 256, 0, s>>>(B.D, B.pairs[l], l, 0);
            chk("k_bsp_smooth");
        }
    }
    if (B.nlev >= 1 && B.nb_pairs[0]) {
        k_bsp_smooth<true><<<B.nb_pairs[0], 256, 0, s>>>(B.D, B.pairs[0], 0, 1);
        chk("k_bsp_smooth");
        // the further sweeps; the last red half is k_bsp_redpost's
        for (int sw = 1; sw < level_sweeps(0); sw++) {
            k_bsp_smooth<false><<<B.nb_pairs[0], 256, 0, s>>>(B.D, B.pairs[0], 0, 0);
            chk("k_bsp_smooth");
            k_bsp_smooth<false><<<B.nb_pairs[0], 256, 0, s>>>(B.D, B.pairs[0], 0, 1);
            chk("k_bsp_smooth");
        }
    }
    k_bsp_redpost<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    chk("k_bsp_redpost");
    k_bsp_direction<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    chk("k_bsp_direction");
    k_bsp_residual<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    chk("k_bsp_residual");
    return rc;
}

}  // namespace

int batch_split_solve(BatchSplit &B, cudaStream_t s, int max_iter)
{
    if (B.nrooms == 0) return FFR_OK;
    FFR_CUDA(cudaMemsetAsync(B.D.active, 0, sizeof(int), s));
    k_bsp_extrapolate<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    k_bsp_init<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    int launched = 0, rc = FFR_OK;
    auto batch = [&](int nb, int slot) -> int {
        for (int k = 0; k < nb; k++) {
            int r = batch_iteration(B, s);
            if (r) return r;
        }
        launched += nb;
        FFR_CUDA(cudaMemcpyAsync(B.active_host + slot, B.D.active, sizeof(int), cudaMemcpyDeviceToHost, s));
        FFR_CUDA(cudaEventRecord(B.ev[slot], s));
        return FFR_OK;
    };
    // paced as launch_split_pcg: a first batch of the previous solve's
    // count less two, then batches of two queued ahead of the host's wait
    int slot = 0;
    if (max_iter > 0) {
        rc = batch(std::min(max_iter, std::max(1, B.last_iters - 2)), slot);
        if (rc) return rc;
        while (true) {
            const int prev = slot;
            const bool more = launched < max_iter;
            if (more) {
                slot ^= 1;
                rc = batch(std::min(2, max_iter - launched), slot);
                if (rc) return rc;
            }
            FFR_CUDA(cudaEventSynchronize(B.ev[prev]));
            if (B.active_host[prev] <= 0) {
                B.last_iters = launched - (more ? 2 : 0);
                break;
            }
            if (!more) break;
        }
    }
    k_bsp_final<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    k_bsp_backsub<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    return FFR_OK;
}

int launch_batch_cluster(BatchSplit &B, cudaStream_t s, int ctas)
{
    if (B.nrooms == 0) return FFR_OK;
    static bool attr_set = false;
    if (!attr_set) {
        FFR_CUDA(cudaFuncSetAttribute(k_bpcg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        attr_set = true;
    }
    k_bsp_extrapolate<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(B.nrooms * ctas));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FFR_CUDA(cudaLaunchKernelEx(&cfg, k_bpcg_cluster, B.D, B.cluster_order, ctas));
    count_launch(1);
    return FFR_OK;
}

int capture_batch_split(BatchSplit &B, cudaStream_t s, cudaStream_t bs)
{
    if (B.nrooms == 0) return FFR_OK;
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    FFR_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(FFR_EINVAL, "batched solve must be captured");
    FFR_CUDA(cudaMemsetAsync(B.D.active, 0, sizeof(int), s));
    k_bsp_extrapolate<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    k_bsp_init<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    FFR_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphConditionalHandle cond;
    FFR_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    k_bsp_cond<<<1, 32, 0, s>>>(B.D.active, cond);
    FFR_LAUNCHED(1);
    FFR_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    FFR_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    FFR_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    // one iteration of every room still iterating, then the condition; a
    // room that finished returns at once from every pass, and each room
    // stops itself at its own poisson_max_iter, so the loop ends
    FFR_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int rc = batch_iteration(B, bs);
    if (!rc) {
        k_bsp_cond<<<1, 32, 0, bs>>>(B.D.active, cond);
        FFR_LAUNCHED(1);
    }
    cudaGraph_t body_out = nullptr;
    cudaError_t e = cudaStreamEndCapture(bs, &body_out);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(batched PCG iteration)");
    k_bsp_final<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    k_bsp_backsub<<<B.nb_cells0, 256, 0, s>>>(B.D, B.cells0);
    FFR_LAUNCHED(1);
    return FFR_OK;
}

FFR_DEFINE_WAIT_LIMIT_SETTER(set_wait_limit_mgpcg)

}  // namespace ffr
