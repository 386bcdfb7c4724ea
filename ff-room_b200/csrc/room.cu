// room.cu — room validation, mask-derived codes, arena, error plumbing.
#include "common.cuh"

#include <mutex>
#include <unordered_map>
#include <vector>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>

namespace ffr {

static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int status, const std::string &msg)
{
    set_error(msg);
    return status;
}

int cuda_fail(cudaError_t e, const char *what)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    set_error(buf);
    return e == cudaErrorMemoryAllocation ? FFR_ENOMEM : FFR_ECUDA;
}

void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
// Keep freed pool memory cached (the default release threshold returns it
// to the system at every synchronisation), once per device.
void keep_pool_cached()
{
    static std::mutex mu;
    static bool done[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        unsigned long long thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done[dev] = true;
}
}  // namespace

int Arena::alloc(size_t bytes, cudaStream_t s)
{
    size = (bytes + 255) & ~size_t(255);
    used = 0;
    failed = false;
    stream = s;
    cudaError_t e;
    if (s) {
        keep_pool_cached();
        e = cudaMallocAsync(reinterpret_cast<void **>(&base), size, s);
    } else {
        e = cudaMalloc(&base, size);
    }
    if (e != cudaSuccess) {
        base = nullptr;
        return cuda_fail(e, s ? "cudaMallocAsync(arena)" : "cudaMalloc(arena)");
    }
    return FFR_OK;
}

void Arena::release()
{
    if (base) {
        if (stream) cudaFreeAsync(base, stream);
        else cudaFree(base);
    }
    base = nullptr;
    size = used = 0;
}

namespace {
std::mutex g_pinned_mu;
std::unordered_map<size_t, std::vector<void *>> g_pinned;
}  // namespace

void *pinned_get(size_t bytes)
{
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        auto it = g_pinned.find(bytes);
        if (it != g_pinned.end() && !it->second.empty()) {
            void *p = it->second.back();
            it->second.pop_back();
            return p;
        }
    }
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    return p;
}

void pinned_put(void *p, size_t bytes)
{
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned[bytes].push_back(p);
}

int HostStage::reserve(size_t bytes)
{
    size_t sz = 64u << 10;           // power-of-two sizes keep the pinned cache reusable
    while (sz < bytes) sz <<= 1;
    base = static_cast<char *>(pinned_get(sz));
    if (!base) return fail(FFR_ENOMEM, "pinned staging block");
    size = sz;
    used = 0;
    return FFR_OK;
}

int HostStage::put(void *dev, const void *src, size_t bytes, cudaStream_t s)
{
    const size_t b = (bytes + 15) & ~size_t(15);
    if (!base || used + b > size) return fail(FFR_ENOMEM, "set-up staging block exhausted");
    std::memcpy(base + used, src, bytes);
    FFR_CUDA(cudaMemcpyAsync(dev, base + used, bytes, cudaMemcpyHostToDevice, s));
    used += b;
    return FFR_OK;
}

void HostStage::release()
{
    pinned_put(base, size);
    base = nullptr;
    size = used = 0;
}

namespace {
// One host thread's slice of a staged copy: chunks through two page-locked
// bounce buffers on the thread's own stream, so the DMA of one chunk
// overlaps the host copy of the other.  `start` orders the first DMA after
// the work queued on the caller's stream before the copy.
cudaError_t staged_slice(char *d, const char *s, size_t bytes, bool to_host, cudaEvent_t start, int dev)
{
    constexpr size_t kChunk = 2u << 20;
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return e;
    cudaStream_t ws = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    char *buf[2] = {static_cast<char *>(pinned_get(kChunk)), static_cast<char *>(pinned_get(kChunk))};
    if (!buf[0] || !buf[1]) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking);
    for (cudaEvent_t &x : ev)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ws, start, 0);
    const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice;
    const size_t nch = (bytes + kChunk - 1) / kChunk;
    auto len = [&](size_t c) { return std::min(kChunk, bytes - c * kChunk); };
    for (size_t c = 0; c < nch && e == cudaSuccess; c++) {
        const int b = (int)(c & 1);
        if (to_host) {
            // chunk c into buf[b] (its previous contents, chunk c-2, were
            // copied out in the last iteration), then chunk c-1 to the host
            e = cudaMemcpyAsync(buf[b], s + c * kChunk, len(c), kind, ws);
            if (e == cudaSuccess) e = cudaEventRecord(ev[b], ws);
            if (e == cudaSuccess && c > 0) {
                e = cudaEventSynchronize(ev[b ^ 1]);
                if (e == cudaSuccess) std::memcpy(d + (c - 1) * kChunk, buf[b ^ 1], len(c - 1));
            }
        } else {
            // buf[b] is free once the DMA of chunk c-2 has finished
            if (c > 1) e = cudaEventSynchronize(ev[b]);
            if (e == cudaSuccess) {
                std::memcpy(buf[b], s + c * kChunk, len(c));
                e = cudaMemcpyAsync(d + c * kChunk, buf[b], len(c), kind, ws);
            }
            if (e == cudaSuccess) e = cudaEventRecord(ev[b], ws);
        }
    }
    if (e == cudaSuccess && to_host && nch > 0) {
        const int b = (int)((nch - 1) & 1);
        e = cudaEventSynchronize(ev[b]);
        if (e == cudaSuccess) std::memcpy(d + (nch - 1) * kChunk, buf[b], len(nch - 1));
    }
    // the bounce buffers go back to the cache only after their last DMA
    if (ws) {
        const cudaError_t e2 = cudaStreamSynchronize(ws);
        if (e == cudaSuccess) e = e2;
        cudaStreamDestroy(ws);
    }
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    pinned_put(buf[0], kChunk);
    pinned_put(buf[1], kChunk);
    return e;
}
}  // namespace

// Synchronous copy between pageable host memory and the device.  Large
// copies are cut into page-aligned slices, one per host thread (up to 16,
// at least 4 MB each), each staged through its own bounce buffers and
// stream, so the host-side copies (and the page faults of a freshly
// allocated destination) run in parallel while the DMAs share the link.
int staged_copy(void *dst, const void *src, size_t bytes, bool to_host, cudaStream_t st)
{
    constexpr size_t kSlice = 4u << 20;
    const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice;
    if (bytes < 2 * kSlice) {
        FFR_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, st));
        FFR_CUDA(cudaStreamSynchronize(st));
        return FFR_OK;
    }
    const unsigned hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
    const int nt = (int)std::min<size_t>(hw, bytes / kSlice);
    const size_t piece = ((bytes + nt - 1) / nt + 4095) & ~size_t(4095);
    int dev = 0;
    FFR_CUDA(cudaGetDevice(&dev));
    cudaEvent_t start = nullptr;
    FFR_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(start, st);
    if (e == cudaSuccess) {
        std::vector<cudaError_t> err(nt, cudaSuccess);
        std::vector<std::thread> th;
        char *d = static_cast<char *>(dst);
        const char *s = static_cast<const char *>(src);
        auto one = [&](int q) {
            const size_t o = (size_t)q * piece;
            if (o < bytes) err[q] = staged_slice(d + o, s + o, std::min(piece, bytes - o), to_host, start, dev);
        };
        for (int q = 1; q < nt; q++) th.emplace_back(one, q);
        one(0);
        for (auto &t : th) t.join();
        for (cudaError_t x : err)
            if (x != cudaSuccess && e == cudaSuccess) e = x;
    }
    cudaEventDestroy(start);
    if (e != cudaSuccess) return cuda_fail(e, "staged copy");
    return FFR_OK;
}

// Validates a room descriptor and copies it.  The reference accepts some of
// the rejected inputs silently (an outflow patch outside the grid writes out
// of bounds in BoundaryManager::add_outflow, BoundaryManager.cpp:24-44); a
// bad Grid size throws std::invalid_argument there (Grid.cpp:10-11).
int load_room(const ffr_room_desc *d, HostRoom &r)
{
    if (!d) return fail(FFR_EINVAL, "room descriptor is NULL");
    if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0)
        return fail(FFR_EINVAL, "Grid dimensions must be positive");
    const long long n = (long long)d->nx * d->ny * d->nz;
    if (n > (1ll << 31) - 1 - 4ll * d->nx * d->ny ||
        (long long)(d->nx + 1) * (d->ny + 1) * (d->nz + 1) > (1ll << 31) - 1)
        return fail(FFR_ERANGE, "grid too large for 32-bit face indexing");
    if (!d->dxv || !d->dyv || !d->dzv || !d->cell_type)
        return fail(FFR_EINVAL, "room spacing or cell_type pointer is NULL");
    r.g.nx = d->nx; r.g.ny = d->ny; r.g.nz = d->nz;
    r.g.n = n;
    r.g.nu = (long long)(d->nx + 1) * d->ny * d->nz;
    r.g.nv = (long long)d->nx * (d->ny + 1) * d->nz;
    r.g.nw = (long long)d->nx * d->ny * (d->nz + 1);
    r.g.lx = d->lx; r.g.ly = d->ly; r.g.lz = d->lz;
    r.dxv.assign(d->dxv, d->dxv + d->nx);
    r.dyv.assign(d->dyv, d->dyv + d->ny);
    r.dzv.assign(d->dzv, d->dzv + d->nz);
    for (double h : r.dxv) if (!(h > 0)) return fail(FFR_EINVAL, "non-positive x spacing");
    for (double h : r.dyv) if (!(h > 0)) return fail(FFR_EINVAL, "non-positive y spacing");
    for (double h : r.dzv) if (!(h > 0)) return fail(FFR_EINVAL, "non-positive z spacing");
    // copy, range check and FLUID count in 256 k-cell pieces on all host threads
    r.ct.resize(n);
    const int pieces = (int)((n + (1 << 18) - 1) >> 18);
    std::vector<long long> fluid(pieces, 0);
    std::vector<char> bad(pieces, 0);
    parallel_slabs(pieces, [&](int p0, int p1) {
        for (int p = p0; p < p1; p++) {
            const long long b = (long long)p << 18, e = std::min(n, b + (1ll << 18));
            std::memcpy(r.ct.data() + b, d->cell_type + b, (size_t)(e - b));
            long long f = 0;
            uint8_t mx = 0;
            for (long long c = b; c < e; c++) {
                const uint8_t t = r.ct[c];
                f += (t == CT_FLUID);
                mx = std::max(mx, t);
            }
            fluid[p] = f;
            bad[p] = mx > CT_OUTFLOW;
        }
    });
    r.n_fluid = 0;
    for (int p = 0; p < pieces; p++) {
        if (bad[p]) return fail(FFR_EINVAL, "cell_type value out of range");
        r.n_fluid += fluid[p];
    }
    if (d->nfans < 0 || d->npatches < 0 || d->nheat < 0) return fail(FFR_EINVAL, "negative count");
    if (d->nfans > kMaxFans) return fail(FFR_ERANGE, "more than 120 fans");
    r.fans.assign(d->fans, d->fans + d->nfans);
    r.patches.assign(d->patches, d->patches + d->npatches);
    r.heats.assign(d->heats, d->heats + d->nheat);
    const int N[3] = {d->nx, d->ny, d->nz};
    for (const ffr_patch &p : r.patches) {
        if (p.axis < 0 || p.axis > 2 || (p.side != 0 && p.side != 1))
            return fail(FFR_EINVAL, "patch axis/side out of range");
        const int ta = p.axis == 0 ? 1 : 0, tb = p.axis == 2 ? 1 : 2;
        if (p.a_min < 0 || p.b_min < 0 || p.a_max >= N[ta] || p.b_max >= N[tb])
            return fail(FFR_EINVAL, "outflow patch outside the grid");
        if (N[p.axis] < 2)
            return fail(FFR_ENOTSUP, "outflow on an axis with fewer than 2 cells");
    }
    return FFR_OK;
}

// ------------------------------------------------ codes built on the device
//
// The per-cell and per-face codes are pure functions of the cell types, the
// fan boxes and the outflow patches, so they are formed on the GPU from the
// uploaded cell types (one thread per cell or face) instead of on the host.

// Pressure-stencil code of each cell: the neighbour classes of
// PoissonSolver::apply_laplacian (PoissonSolver.cpp:61-77) — outside the
// grid or SOLID: no term; OUTFLOW: Dirichlet ghost; otherwise an unknown —
// plus SC_SOLID for a SOLID row and SC_OUTF for an OUTFLOW row.
__global__ void k_stencil_codes(const uint8_t *__restrict__ ct, int nx, int ny, int nz, uint16_t *__restrict__ sc)
{
    const int n = nx * ny * nz, plane = ny * nz;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const uint8_t t = ct[c];
        if (t == CT_SOLID) { sc[c] = SC_SOLID; continue; }
        const int i = c / plane, rem = c - i * plane, j = rem / nz, k = rem - j * nz;
        auto cls = [&](bool inside, int o) -> unsigned {
            if (!inside) return SC_NONE;
            const uint8_t u = ct[c + o];
            return u == CT_OUTFLOW ? SC_DIR : (u == CT_SOLID ? SC_NONE : SC_IN);
        };
        sc[c] = (uint16_t)(cls(i > 0, -plane) | cls(i < nx - 1, plane) << 2 | cls(j > 0, -nz) << 4 |
                           cls(j < ny - 1, nz) << 6 | cls(k > 0, -1) << 8 | cls(k < nz - 1, 1) << 10 |
                           (t == CT_OUTFLOW ? SC_OUTF : 0));
    }
}

// What BoundaryManager::apply_noslip leaves on each face (BoundaryManager.cpp:
// 60-109): a domain-wall face is zeroed unless its cell is OUTFLOW, and all
// six faces of a SOLID cell are zeroed.  One thread per face of u, v, w.
__global__ void k_face_codes(const uint8_t *__restrict__ ct, int nx, int ny, int nz, uint8_t *__restrict__ fu,
                             uint8_t *__restrict__ fv, uint8_t *__restrict__ fw)
{
    const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)nx * (ny + 1) * nz,
                    nw = (long long)nx * ny * (nz + 1);
    auto CI = [&](int i, int j, int k) { return ((long long)i * ny + j) * nz + k; };
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nu + nv + nw;
         f += (long long)gridDim.x * blockDim.x) {
        if (f < nu) {
            const int i = (int)(f / ((long long)ny * nz)), rem = (int)(f - (long long)i * ny * nz);
            const int j = rem / nz, k = rem - j * nz;
            const bool zero = (i == 0 && ct[CI(0, j, k)] != CT_OUTFLOW) ||
                              (i == nx && ct[CI(nx - 1, j, k)] != CT_OUTFLOW) ||
                              (i < nx && ct[CI(i, j, k)] == CT_SOLID) || (i > 0 && ct[CI(i - 1, j, k)] == CT_SOLID);
            fu[f] = zero ? FC_ZERO : FC_KEEP;
        } else if (f < nu + nv) {
            const long long g = f - nu;
            const int i = (int)(g / ((long long)(ny + 1) * nz)), rem = (int)(g - (long long)i * (ny + 1) * nz);
            const int j = rem / nz, k = rem - j * nz;
            const bool zero = (j == 0 && ct[CI(i, 0, k)] != CT_OUTFLOW) ||
                              (j == ny && ct[CI(i, ny - 1, k)] != CT_OUTFLOW) ||
                              (j < ny && ct[CI(i, j, k)] == CT_SOLID) || (j > 0 && ct[CI(i, j - 1, k)] == CT_SOLID);
            fv[g] = zero ? FC_ZERO : FC_KEEP;
        } else {
            const long long g = f - nu - nv;
            const int i = (int)(g / ((long long)ny * (nz + 1))), rem = (int)(g - (long long)i * ny * (nz + 1));
            const int j = rem / (nz + 1), k = rem - j * (nz + 1);
            const bool zero = (k == 0 && ct[CI(i, j, 0)] != CT_OUTFLOW) ||
                              (k == nz && ct[CI(i, j, nz - 1)] != CT_OUTFLOW) ||
                              (k < nz && ct[CI(i, j, k)] == CT_SOLID) || (k > 0 && ct[CI(i, j, k - 1)] == CT_SOLID);
            fw[g] = zero ? FC_ZERO : FC_KEEP;
        }
    }
}

// BoundaryManager::apply_inflow (BoundaryManager.cpp:111-130) for one fan:
// both faces of each cell of its (clamped) box, per non-zero component,
// take the fan's code.  Fans are applied in order, so a later fan's box
// overrides an earlier one's, as the reference's loop does.
__global__ void k_face_fan(int nx, int ny, int nz, ffr_fan fn, uint8_t code, uint8_t *__restrict__ fu,
                           uint8_t *__restrict__ fv, uint8_t *__restrict__ fw)
{
    const int i0 = max(0, fn.i_min), j0 = max(0, fn.j_min), k0 = max(0, fn.k_min);
    const int bi = min(nx - 1, fn.i_max) - i0 + 1, bj = min(ny - 1, fn.j_max) - j0 + 1,
              bk = min(nz - 1, fn.k_max) - k0 + 1;
    const long long cells = (long long)bi * bj * bk;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = i0 + (int)(c / ((long long)bj * bk)), rem = (int)(c % ((long long)bj * bk));
        const int j = j0 + rem / bk, k = k0 + rem % bk;
        if (fn.vel[0] != 0.0) {
            const long long u = ((long long)i * ny + j) * nz + k;
            fu[u] = fu[u + (long long)ny * nz] = code;
        }
        if (fn.vel[1] != 0.0) {
            const long long v = ((long long)i * (ny + 1) + j) * nz + k;
            fv[v] = fv[v + nz] = code;
        }
        if (fn.vel[2] != 0.0) {
            const long long w = ((long long)i * ny + j) * (nz + 1) + k;
            fw[w] = fw[w + 1] = code;
        }
    }
}

// The faces BoundaryManager::apply_outflow overwrites (BoundaryManager.cpp:
// 180-220) for one patch: its wall faces get the FC_OUTCOPY bit.
__global__ void k_face_patch(int nx, int ny, int nz, ffr_patch p, uint8_t *__restrict__ fu,
                             uint8_t *__restrict__ fv, uint8_t *__restrict__ fw)
{
    const int na = p.a_max - p.a_min + 1, nb = p.b_max - p.b_min + 1;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < na * nb; c += gridDim.x * blockDim.x) {
        const int a = p.a_min + c / nb, b = p.b_min + c % nb;
        if (p.axis == 0) fu[((long long)(p.side ? nx : 0) * ny + a) * nz + b] |= FC_OUTCOPY;
        else if (p.axis == 1) fv[((long long)a * (ny + 1) + (p.side ? ny : 0)) * nz + b] |= FC_OUTCOPY;
        else fw[((long long)a * ny + b) * (nz + 1) + (p.side ? nz : 0)] |= FC_OUTCOPY;
    }
}

namespace {
unsigned setup_blocks(long long work)
{
    return (unsigned)std::max<long long>(1, std::min<long long>(4 * 148, (work + 255) / 256));
}
}  // namespace

int launch_stencil_codes(const uint8_t *ct, int nx, int ny, int nz, uint16_t *sc, cudaStream_t s)
{
    k_stencil_codes<<<setup_blocks((long long)nx * ny * nz), 256, 0, s>>>(ct, nx, ny, nz, sc);
    FFR_LAUNCHED(1);
    return FFR_OK;
}

int build_codes(const HostRoom &r, const uint8_t *ct, uint16_t *sc, uint8_t *fu, uint8_t *fv, uint8_t *fw,
                cudaStream_t s)
{
    const int nx = r.g.nx, ny = r.g.ny, nz = r.g.nz;
    int rc = launch_stencil_codes(ct, nx, ny, nz, sc, s);
    if (rc) return rc;
    k_face_codes<<<setup_blocks(r.g.nu + r.g.nv + r.g.nw), 256, 0, s>>>(ct, nx, ny, nz, fu, fv, fw);
    FFR_LAUNCHED(1);
    for (size_t f = 0; f < r.fans.size(); f++) {
        const ffr_fan &fn = r.fans[f];
        const long long bi = std::min(nx - 1, fn.i_max) - std::max(0, fn.i_min) + 1,
                        bj = std::min(ny - 1, fn.j_max) - std::max(0, fn.j_min) + 1,
                        bk = std::min(nz - 1, fn.k_max) - std::max(0, fn.k_min) + 1;
        if (bi <= 0 || bj <= 0 || bk <= 0) continue;
        k_face_fan<<<setup_blocks(bi * bj * bk), 256, 0, s>>>(nx, ny, nz, fn, (uint8_t)(FC_FAN0 + f), fu, fv, fw);
        FFR_LAUNCHED(1);
    }
    for (const ffr_patch &p : r.patches) {
        k_face_patch<<<setup_blocks((long long)(p.a_max - p.a_min + 1) * (p.b_max - p.b_min + 1)), 256, 0, s>>>(
            nx, ny, nz, p, fu, fv, fw);
        FFR_LAUNCHED(1);
    }
    return FFR_OK;
}

// Per-axis scales of PoissonSolver::apply_laplacian (PoissonSolver.cpp:
// 33-49), computed with the same double expressions so that the device
// stencil uses identical coefficients.  Layout: [sxl(nx) sxr(nx) syl(ny)
// syr(ny) szl(nz) szr(nz)].
void stencil_scales(const HostRoom &r, std::vector<double> &scale)
{
    const int nx = r.g.nx, ny = r.g.ny, nz = r.g.nz;
    scale.assign(2 * (size_t)(nx + ny + nz), 0.0);
    auto axis = [&](const std::vector<double> &h, int m, double *sl, double *sr) {
        for (int i = 0; i < m; i++) {
            const double hl = (i > 0) ? 0.5 * (h[i - 1] + h[i]) : h[i];
            const double hr = (i < m - 1) ? 0.5 * (h[i] + h[i + 1]) : h[i];
            sl[i] = 1.0 / (hl * h[i]);
            sr[i] = 1.0 / (hr * h[i]);
        }
    };
    double *sp = scale.data();
    axis(r.dxv, nx, sp, sp + nx);
    axis(r.dyv, ny, sp + 2 * nx, sp + 2 * nx + ny);
    axis(r.dzv, nz, sp + 2 * nx + 2 * ny, sp + 2 * nx + 2 * ny + nz);
}

}  // namespace ffr

extern "C" {

const char *ffr_status_string(int s)
{
    switch (s) {
    case FFR_OK: return "ok";
    case FFR_EINVAL: return "invalid argument";
    case FFR_ENOMEM: return "out of memory";
    case FFR_ECUDA: return "CUDA error";
    case FFR_ETIMEDOUT: return "device wait timed out";
    case FFR_ENOTSUP: return "not supported";
    case FFR_ERANGE: return "size out of range";
    default: return "unknown status";
    }
}

const char *ffr_last_error(void) { return ffr::g_last_error.c_str(); }

const char *ffr_version(void) { return "0.1.0 sm_100a"; }

unsigned long long ffr_launch_count(void) { return ffr::g_launches.load(); }

}  // extern "C"
