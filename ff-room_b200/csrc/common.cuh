// common.cuh — shared device/host helpers of libffroom_cuda.so (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "ffroom.h"

#include <algorithm>
#include <thread>
#include <vector>

namespace ffr {

// ------------------------------------------------------------ errors

void set_error(const std::string &msg);
int fail(int status, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
void count_launch(unsigned n = 1);

#define FFR_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return ::ffr::cuda_fail(e_, #call);            \
    } while (0)

#define FFR_LAUNCHED(n)                                                       \
    do {                                                                      \
        cudaError_t e_ = cudaGetLastError();                                  \
        if (e_ != cudaSuccess) return ::ffr::cuda_fail(e_, "kernel launch");  \
        ::ffr::count_launch(n);                                               \
    } while (0)

// Cell types (Grid.hpp:9-14).
enum : uint8_t { CT_FLUID = 0, CT_SOLID = 1, CT_INFLOW = 2, CT_OUTFLOW = 3 };

// Face override codes, one byte per face: the low 7 bits say what the
// no-slip + inflow appliers leave on the face (0 keep, 1 zero, 2+f the
// velocity of fan f); bit 7 marks a zero-gradient outflow destination.
enum : uint8_t { FC_KEEP = 0, FC_ZERO = 1, FC_FAN0 = 2, FC_OUTCOPY = 0x80 };
constexpr int kMaxFans = 120;

// Pressure-stencil code, one uint16 per cell: 2 bits per neighbour in the
// order x-, x+, y-, y+, z-, z+ (0 no term, 1 interior, 2 Dirichlet ghost of
// an OUTFLOW neighbour) and bit 12 for a SOLID (identity) row.
// SC_OUTF marks an OUTFLOW cell (a Dirichlet row of the pressure system);
// SC_ALLIN is the code of a cell whose six neighbours are all unknowns.
enum : uint16_t { SC_NONE = 0, SC_IN = 1, SC_DIR = 2, SC_SOLID = 1u << 12, SC_OUTF = 1u << 13, SC_ALLIN = 0x555 };

// --------------------------------------------------------- room setup

struct RoomGeom {
    int nx, ny, nz;
    long long n, nu, nv, nw;
    double lx, ly, lz;
};

// Host-side, fully validated copy of an ffr_room_desc.
struct HostRoom {
    RoomGeom g;
    std::vector<double> dxv, dyv, dzv;
    std::vector<uint8_t> ct;
    std::vector<ffr_fan> fans;
    std::vector<ffr_patch> patches;
    std::vector<ffr_heat_patch> heats;
    long long n_fluid = 0;
};

int load_room(const ffr_room_desc *d, HostRoom &out);

// On the device, from the cell types already there (ct): the pressure
// stencil codes (sc, one per cell) and the face codes (fu/fv/fw) that
// replay the reference's BC appliers.  Kernels queued on `s`.
int build_codes(const HostRoom &r, const uint8_t *ct, uint16_t *sc, uint8_t *fu, uint8_t *fv, uint8_t *fw,
                cudaStream_t s);
int launch_stencil_codes(const uint8_t *ct, int nx, int ny, int nz, uint16_t *sc, cudaStream_t s);
// Per-axis stencil scales (PoissonSolver.cpp:33-49): 2*(nx+ny+nz), l,r per index.
void stencil_scales(const HostRoom &r, std::vector<double> &scale);

// ------------------------------------------------------ device memory

// One cudaMalloc per handle, carved into 256-byte aligned slices.
// Exhaustion is sticky: once a take() fails every later take() fails too,
// so checking the last slice of a carve (before any copy or launch) covers
// every slice taken before it.
// One device allocation per handle, carved into 256-byte aligned slices.
// With a stream it comes from the device's stream-ordered memory pool
// (cudaMallocAsync / cudaFreeAsync, memory kept cached in the pool), so
// creating and destroying handles while other rooms run does not
// synchronise the device the way cudaMalloc / cudaFree do.
struct Arena {
    char *base = nullptr;
    size_t size = 0, used = 0;
    bool failed = false;
    cudaStream_t stream = nullptr;   // set: pool allocation ordered on this stream
    int alloc(size_t bytes, cudaStream_t s = nullptr);
    template <class T> T *take(size_t count) {
        size_t b = (count * sizeof(T) + 255) & ~size_t(255);
        if (failed || used + b > size) {
            failed = true;
            return nullptr;
        }
        T *p = reinterpret_cast<T *>(base + used);
        used += b;
        return p;
    }
    void release();
};

// Host loop over [0, n) split into contiguous slabs, one per host thread:
// f(begin, end).  For set-up work over cells or planes of a room.
template <class F>
void parallel_slabs(int n, F f)
{
    const unsigned hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    const int nt = (int)std::min<unsigned>(hw, (unsigned)std::max(1, n / 2));
    if (nt <= 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    const int chunk = (n + nt - 1) / nt;
    for (int t = 0; t < nt; t++) {
        const int b = t * chunk, e = std::min(n, b + chunk);
        if (b < e) th.emplace_back(f, b, e);
    }
    for (auto &x : th) x.join();
}

// Page-locked staging of a handle's small set-up arrays (spacings, scales,
// fan velocities, multigrid factors): each array is copied into the block
// and sent with an asynchronous copy, so queuing a handle's set-up never
// waits on its stream.  The block lives as long as the handle.
struct HostStage {
    char *base = nullptr;
    size_t size = 0, used = 0;
    int reserve(size_t bytes);
    int put(void *dev, const void *src, size_t bytes, cudaStream_t s);
    void release();
};

// Synchronous copy between pageable host memory and the device, ordered
// after the work queued on `st`: large copies run on up to 16 host threads,
// each staging its slice through two page-locked bounce buffers on its own
// stream (the DMA of one chunk overlaps the host copy of the other).  Small
// copies go direct.
int staged_copy(void *dst, const void *src, size_t bytes, bool to_host, cudaStream_t st);

// Page-locked host buffers from a process-wide cache (cudaFreeHost may
// synchronise the device; returned buffers are kept for the next handle).
void *pinned_get(size_t bytes);
void pinned_put(void *p, size_t bytes);

// ------------------------------------------------ grid-wide barrier

// Counter barrier for a cooperative launch (all blocks co-resident).  Every
// wait is bounded by the wait limit below; a block that gives up sets `err`
// and returns false so that the kernel can unwind.
struct GridSync {
    unsigned int count;
    unsigned int gen;
    int err;
    int pad;
};
constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;  // 4 s, the default wait limit

// The bound of every device-side wait of this translation unit's kernels
// (one copy per .cu file and device).  ffr_set_device_wait_limit sets every
// copy on the current device; a test shortens it to make a wait run out.
static __device__ unsigned long long g_wait_limit_ns = kBarrierTimeoutNs;

// Host side: sets this translation unit's copy on the current device.  Each
// .cu file with device waits exports one wrapper (set_wait_limit_<file>).
#define FFR_DEFINE_WAIT_LIMIT_SETTER(NAME)                                                 \
    int NAME(unsigned long long ns)                                                        \
    {                                                                                      \
        const cudaError_t e = cudaMemcpyToSymbol(g_wait_limit_ns, &ns, sizeof(ns));        \
        return e == cudaSuccess ? FFR_OK : cuda_fail(e, "cudaMemcpyToSymbol(wait limit)"); \
    }
int set_wait_limit_projection(unsigned long long ns);
int set_wait_limit_mgpcg(unsigned long long ns);

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Deterministic block sum (fixed shuffle tree, fixed warp order).  All
// threads get the total.  `sh` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
    if (wid == 0) t = warp_sum(t);
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    t = sh[0];
    __syncthreads();
    return t;
}

__device__ __forceinline__ double block_max(double v, double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
    if (wid == 0) t = warp_max(t);
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    t = sh[0];
    __syncthreads();
    return t;
}

// Grid-wide sum of NV values: block partials go to partials[b*NV+v]; the
// last block to arrive adds them in block order (so the result does not
// depend on arrival order), publishes out[v] and releases the others.
// Returns false when the wait timed out.
template <int NV>
__device__ bool grid_allreduce(GridSync *gs, double *partials, double *out, double (&vals)[NV],
                               double *sh)
{
    __shared__ int s_last, s_ok;
    for (int v = 0; v < NV; v++) {
        double t = block_sum(vals[v], sh);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * NV + v] = t;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned g = ld_acquire(&gs->gen);
        const unsigned arrived = atomicAdd(&gs->count, 1u);
        s_last = (arrived == gridDim.x - 1);
        s_ok = 1;
        if (!s_last) {
            const unsigned long long t0 = global_ns();
            while (ld_acquire(&gs->gen) == g) {
                __nanosleep(64);
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
    if (s_last) {
        for (int v = 0; v < NV; v++) {
            double t = 0.0;
            for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
                t += __ldcg(&partials[(size_t)b * NV + v]);
            t = block_sum(t, sh);
            if (threadIdx.x == 0) __stcg(&out[v], t);
        }
        if (threadIdx.x == 0) {
            __threadfence();
            atomicExch(&gs->count, 0u);
            __threadfence();
            atomicAdd(&gs->gen, 1u);
        }
    }
    __syncthreads();
    const bool ok = s_ok;
    for (int v = 0; v < NV; v++) vals[v] = __ldcg(&out[v]);
    __syncthreads();
    return ok;
}

// Max of non-negative doubles through their bit patterns (monotone for
// x >= 0).  NaN never reaches it: callers fold with fmax, which drops NaN
// the way std::max(acc, x) does (FluidSolver.cpp:527-534).
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *slot, double v)
{
    if (v > 0.0) atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// Event-pair timing of kernel groups on one stream (host side).
struct GroupTimer {
    bool on = false;
    int ngroups = 0;
    std::vector<cudaEvent_t> pool;
    struct Pending { int group; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<double> ms;
    std::vector<long long> launches;
    cudaEvent_t open_ev = nullptr;
    int open_group = -1;

    void reset(int groups)
    {
        ngroups = groups;
        ms.assign(groups, 0.0);
        launches.assign(groups, 0);
    }
    cudaEvent_t take()
    {
        if (pool.empty()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    // Opens group g at the current point of stream s.
    void begin(int g, cudaStream_t s)
    {
        if (!on) return;
        open_ev = take();
        open_group = g;
        cudaEventRecord(open_ev, s);
    }
    void end(cudaStream_t s, int nlaunch)
    {
        if (!on || open_group < 0) return;
        cudaEvent_t b = take();
        cudaEventRecord(b, s);
        pending.push_back({open_group, open_ev, b});
        launches[open_group] += nlaunch;
        open_group = -1;
    }
    // Call after the stream has been synchronised.
    void collect()
    {
        for (const Pending &p : pending) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) ms[p.group] += t;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void destroy()
    {
        collect();
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
        pool.clear();
    }
};

__device__ __forceinline__ void decode(int c, int ny, int nz, int &i, int &j, int &k)
{
    const int plane = ny * nz;
    i = c / plane;
    const int rem = c - i * plane;
    j = rem / nz;
    k = rem - j * nz;
}

// Visits the flat indices start, start + stride, ... < n of a (., ny, nz)
// grid and keeps (i, j, k) up to date with carries instead of dividing for
// every cell.
struct Walk {
    int c, i, j, k, si, sj, sk, stride, ny, nz, n;
    __device__ __forceinline__ Walk(int start, int stride_, int ny_, int nz_, int n_)
        : c(start), stride(stride_), ny(ny_), nz(nz_), n(n_)
    {
        decode(start, ny, nz, i, j, k);
        decode(stride, ny, nz, si, sj, sk);
    }
    __device__ __forceinline__ bool ok() const { return c < n; }
    __device__ __forceinline__ void next()
    {
        c += stride;
        k += sk;
        j += sj;
        i += si;
        if (k >= nz) { k -= nz; j++; }
        if (j >= ny) { j -= ny; i++; }
    }
};

}  // namespace ffr
