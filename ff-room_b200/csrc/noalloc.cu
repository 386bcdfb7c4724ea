// noalloc.cu — the pressure solve without any device allocation.
//
// Some callers of this library cannot allocate device memory at solve time:
// a process whose GPU memory has been handed to another allocator up front
// (a framework that pre-reserves the device), or a latency-critical control
// loop that must not take the implicit device synchronisation a
// cudaMalloc / cudaFree can cause.  ffr_poisson_solve_noalloc serves them:
// every buffer it needs lives in one file-scope __device__ array of fixed
// size, reserved when the library is loaded and kept on every GPU that
// loads it until the process exits.
//
// The array is shared by all calls on a device and keeps the contents of
// the last call; calls that overlap on the GPU (different streams, or
// different host threads on one device) race on it and must be serialised
// by the caller.  Every call looks the array's device address up on the
// current device (cudaGetSymbolAddress; no allocation), so a device reset
// between calls is harmless.  Each call is synchronous: it copies the
// spacings in, waits for its stream to finish the solve and copies the
// residual and the iteration count back, so it cannot be captured into a
// CUDA graph.  The stream must belong to the current device.
#include "projection.cuh"

#include <cstring>
#include <vector>

namespace ffr {

constexpr long long kNoAllocMaxCells = FFR_NOALLOC_MAX_CELLS;
constexpr int kNoAllocMaxDim = FFR_NOALLOC_MAX_DIM;
constexpr int kNoAllocMaxBlocks = 2048;

// Layout of the scratch array (offsets in bytes, each 256-aligned).
constexpr size_t al256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kOffCodes = 0;
constexpr size_t kOffR = kOffCodes + al256(2 * kNoAllocMaxCells);
constexpr size_t kOffDa = kOffR + al256(8 * kNoAllocMaxCells);
constexpr size_t kOffDb = kOffDa + al256(8 * kNoAllocMaxCells);
constexpr size_t kOffAd = kOffDb + al256(8 * kNoAllocMaxCells);
constexpr size_t kOffScale = kOffAd + al256(8 * kNoAllocMaxCells);
constexpr size_t kOffPart = kOffScale + al256(8 * 6 * (size_t)kNoAllocMaxDim);
constexpr size_t kOffSync = kOffPart + al256(8 * kNoAllocMaxBlocks);
constexpr size_t kOffScal = kOffSync + al256(sizeof(GridSync));
constexpr size_t kOffOut = kOffScal + al256(sizeof(CGScalars));
constexpr size_t kScratchBytes = kOffOut + al256(64);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

}  // namespace ffr

using namespace ffr;

extern "C" int ffr_poisson_solve_noalloc(int nx, int ny, int nz, const double *dxv, const double *dyv,
                                         const double *dzv, const uint8_t *cell_type_dev, const double *rhs_dev,
                                         double *p_dev, int max_iter, double tol, void *stream,
                                         double *residual, int *iterations)
{
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(FFR_EINVAL, "Grid dimensions must be positive");
    if (!dxv || !dyv || !dzv || !cell_type_dev || !rhs_dev || !p_dev) return fail(FFR_EINVAL, "NULL argument");
    if (max_iter < 0) return fail(FFR_EINVAL, "negative max_iter");
    const long long n = (long long)nx * ny * nz;
    if (n > kNoAllocMaxCells || nx > kNoAllocMaxDim || ny > kNoAllocMaxDim || nz > kNoAllocMaxDim)
        return fail(FFR_ERANGE, "room exceeds the no-allocation capacity (FFR_NOALLOC_MAX_CELLS cells, "
                                "FFR_NOALLOC_MAX_DIM per axis)");
    void *ptr = nullptr;
    {
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
    }
    unsigned char *base = static_cast<unsigned char *>(ptr);
    cudaStream_t st = (cudaStream_t)stream;
    // per-axis stencil scales (PoissonSolver.cpp:33-49), computed on the host
    // exactly as stencil_scales does, copied into the scratch array
    std::vector<double> scale(6 * (size_t)kNoAllocMaxDim);
    auto axis = [](const double *h, int m, double *sl, double *sr) {
        for (int i = 0; i < m; i++) {
            const double hl = (i > 0) ? 0.5 * (h[i - 1] + h[i]) : h[i];
            const double hr = (i < m - 1) ? 0.5 * (h[i] + h[i + 1]) : h[i];
            sl[i] = 1.0 / (hl * h[i]);
            sr[i] = 1.0 / (hr * h[i]);
        }
    };
    for (int i = 0; i < nx; i++) if (!(dxv[i] > 0)) return fail(FFR_EINVAL, "non-positive x spacing");
    for (int j = 0; j < ny; j++) if (!(dyv[j] > 0)) return fail(FFR_EINVAL, "non-positive y spacing");
    for (int k = 0; k < nz; k++) if (!(dzv[k] > 0)) return fail(FFR_EINVAL, "non-positive z spacing");
    double *sp = scale.data();
    axis(dxv, nx, sp, sp + nx);
    axis(dyv, ny, sp + 2 * nx, sp + 2 * nx + ny);
    axis(dzv, nz, sp + 2 * nx + 2 * ny, sp + 2 * nx + 2 * ny + nz);
    const size_t nscale = 2 * (size_t)(nx + ny + nz);
    FFR_CUDA(cudaMemcpyAsync(base + kOffScale, sp, 8 * nscale, cudaMemcpyHostToDevice, st));
    // the barrier state must start at zero on every call
    FFR_CUDA(cudaMemsetAsync(base + kOffSync, 0, sizeof(GridSync), st));
    uint16_t *codes = reinterpret_cast<uint16_t *>(base + kOffCodes);
    int rc = launch_stencil_codes(cell_type_dev, nx, ny, nz, codes, st);
    if (rc) return rc;

    CGArgs a{};
    a.R.nx = nx; a.R.ny = ny; a.R.nz = nz; a.R.n = (int)n;
    a.R.sc = codes;
    a.R.ct = cell_type_dev;
    a.R.scale = reinterpret_cast<const double *>(base + kOffScale);
    a.from_faces = 0;
    a.rhs = rhs_dev;
    a.x = p_dev;
    a.r = reinterpret_cast<double *>(base + kOffR);
    a.da = reinterpret_cast<double *>(base + kOffDa);
    a.db = reinterpret_cast<double *>(base + kOffDb);
    a.ad = reinterpret_cast<double *>(base + kOffAd);
    a.partials = reinterpret_cast<double *>(base + kOffPart);
    a.gs = reinterpret_cast<GridSync *>(base + kOffSync);
    a.sc = reinterpret_cast<CGScalars *>(base + kOffScal);
    a.max_iter = max_iter;
    a.tol = tol;
    a.st = nullptr;
    double *out_res = reinterpret_cast<double *>(base + kOffOut);
    int *out_it = reinterpret_cast<int *>(base + kOffOut + 8);
    int *out_fl = reinterpret_cast<int *>(base + kOffOut + 12);
    a.out_res = out_res; a.out_iters = out_it; a.out_flags = out_fl;
    const unsigned blocks = (unsigned)std::max<long long>(
        1, std::min<long long>(std::min<long long>(cg_block_cap(), kNoAllocMaxBlocks), (n + 255) / 256));
    void *args[] = {(void *)&a};
    FFR_CUDA(cudaLaunchCooperativeKernel((void *)k_cg, dim3(blocks), dim3(256), args, 0, st));
    count_launch(1);
    double res = 0.0;
    int it = 0, fl = 0;
    FFR_CUDA(cudaMemcpyAsync(&res, out_res, 8, cudaMemcpyDeviceToHost, st));
    FFR_CUDA(cudaMemcpyAsync(&it, out_it, 4, cudaMemcpyDeviceToHost, st));
    FFR_CUDA(cudaMemcpyAsync(&fl, out_fl, 4, cudaMemcpyDeviceToHost, st));
    FFR_CUDA(cudaStreamSynchronize(st));
    if (residual) *residual = res;
    if (iterations) *iterations = it;
    if (fl & FFR_FLAG_TIMEOUT) return fail(FFR_ETIMEDOUT, "pressure-solve grid barrier timed out");
    return FFR_OK;
}
