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

namespace {
// memcpy of n bytes on up to four host threads (pieces of at least 1 MB)
void host_copy(char *d, const char *s, size_t n)
{
    const int parts = (int)std::min<size_t>(4, std::max<size_t>(1, n >> 20));
    const size_t piece = (n + parts - 1) / parts;
    auto one = [&](int q) {
        const size_t o = (size_t)q * piece;
        if (o < n) std::memcpy(d + o, s + o, std::min(piece, n - o));
    };
    std::vector<std::thread> th;
    for (int q = 1; q < parts; q++) th.emplace_back(one, q);
    one(0);
    for (auto &t : th) t.join();
}
}  // namespace

int staged_copy(void *dst, const void *src, size_t bytes, bool to_host, cudaStream_t st)
{
    constexpr size_t kChunk = 8u << 20;
    const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice;
    char *buf[2] = {nullptr, nullptr};
    if (bytes > 2 * kChunk) {
        buf[0] = static_cast<char *>(pinned_get(kChunk));
        buf[1] = static_cast<char *>(pinned_get(kChunk));
    }
    if (!buf[0] || !buf[1]) {
        pinned_put(buf[0], kChunk);
        pinned_put(buf[1], kChunk);
        FFR_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, st));
        FFR_CUDA(cudaStreamSynchronize(st));
        return FFR_OK;
    }
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int rc = FFR_OK;
    auto done = [&]() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        pinned_put(buf[0], kChunk);
        pinned_put(buf[1], kChunk);
        return rc;
    };
    for (cudaEvent_t &e : ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            rc = fail(FFR_ECUDA, "cudaEventCreate");
            return done();
        }
    char *d = static_cast<char *>(dst);
    const char *s = static_cast<const char *>(src);
    const size_t nch = (bytes + kChunk - 1) / kChunk;
    auto len = [&](size_t c) { return std::min(kChunk, bytes - c * kChunk); };
    cudaError_t e = cudaSuccess;
    for (size_t c = 0; c < nch && e == cudaSuccess; c++) {
        const int b = (int)(c & 1);
        if (to_host) {
            // chunk c into buf[b] (its previous contents, chunk c-2, were
            // copied out in the last iteration), then chunk c-1 to the host
            e = cudaMemcpyAsync(buf[b], s + c * kChunk, len(c), kind, st);
            if (e == cudaSuccess) e = cudaEventRecord(ev[b], st);
            if (e == cudaSuccess && c > 0) {
                e = cudaEventSynchronize(ev[b ^ 1]);
                if (e == cudaSuccess) host_copy(d + (c - 1) * kChunk, buf[b ^ 1], len(c - 1));
            }
        } else {
            // buf[b] is free once the DMA of chunk c-2 has finished
            if (c > 1) e = cudaEventSynchronize(ev[b]);
            if (e == cudaSuccess) {
                host_copy(buf[b], s + c * kChunk, len(c));
                e = cudaMemcpyAsync(d + c * kChunk, buf[b], len(c), kind, st);
            }
            if (e == cudaSuccess) e = cudaEventRecord(ev[b], st);
        }
    }
    if (e == cudaSuccess && to_host) {
        const int b = (int)((nch - 1) & 1);
        e = cudaEventSynchronize(ev[b]);
        if (e == cudaSuccess) host_copy(d + (nch - 1) * kChunk, buf[b], len(nch - 1));
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_fail(e, "staged copy");
    return done();
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
    if (n > (1ll << 31) - 1 - 4ll * d->nx * d->ny)
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
    r.ct.assign(d->cell_type, d->cell_type + n);
    r.n_fluid = 0;
    for (uint8_t t : r.ct) {
        if (t > CT_OUTFLOW) return fail(FFR_EINVAL, "cell_type value out of range");
        r.n_fluid += (t == CT_FLUID);
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

// Replays BoundaryManager::apply_noslip then apply_inflow
// (BoundaryManager.cpp:60-130) on per-face codes, then marks the faces that
// apply_outflow (BoundaryManager.cpp:180-220) overwrites.  The result is a
// per-face statement of what the reference leaves on each face after those
// appliers, whatever the face held before.
void build_face_codes(const HostRoom &r, std::vector<uint8_t> &fu, std::vector<uint8_t> &fv,
                      std::vector<uint8_t> &fw)
{
    const int nx = r.g.nx, ny = r.g.ny, nz = r.g.nz;
    auto UI = [&](int i, int j, int k) { return (size_t)i * ny * nz + (size_t)j * nz + k; };
    auto VI = [&](int i, int j, int k) { return (size_t)i * (ny + 1) * nz + (size_t)j * nz + k; };
    auto WI = [&](int i, int j, int k) { return (size_t)i * ny * (nz + 1) + (size_t)j * (nz + 1) + k; };
    auto CI = [&](int i, int j, int k) { return (size_t)i * ny * nz + (size_t)j * nz + k; };
    fu.assign(r.g.nu, FC_KEEP);
    fv.assign(r.g.nv, FC_KEEP);
    fw.assign(r.g.nw, FC_KEEP);
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
            if (r.ct[CI(0, j, k)] != CT_OUTFLOW) fu[UI(0, j, k)] = FC_ZERO;
            if (r.ct[CI(nx - 1, j, k)] != CT_OUTFLOW) fu[UI(nx, j, k)] = FC_ZERO;
        }
    for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++) {
            if (r.ct[CI(i, 0, k)] != CT_OUTFLOW) fv[VI(i, 0, k)] = FC_ZERO;
            if (r.ct[CI(i, ny - 1, k)] != CT_OUTFLOW) fv[VI(i, ny, k)] = FC_ZERO;
        }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            if (r.ct[CI(i, j, 0)] != CT_OUTFLOW) fw[WI(i, j, 0)] = FC_ZERO;
            if (r.ct[CI(i, j, nz - 1)] != CT_OUTFLOW) fw[WI(i, j, nz)] = FC_ZERO;
        }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                if (r.ct[CI(i, j, k)] != CT_SOLID) continue;
                fu[UI(i, j, k)] = fu[UI(i + 1, j, k)] = FC_ZERO;
                fv[VI(i, j, k)] = fv[VI(i, j + 1, k)] = FC_ZERO;
                fw[WI(i, j, k)] = fw[WI(i, j, k + 1)] = FC_ZERO;
            }
    for (size_t f = 0; f < r.fans.size(); f++) {
        const ffr_fan &fn = r.fans[f];
        const uint8_t code = (uint8_t)(FC_FAN0 + f);
        for (int i = std::max(0, fn.i_min); i <= std::min(nx - 1, fn.i_max); i++)
            for (int j = std::max(0, fn.j_min); j <= std::min(ny - 1, fn.j_max); j++)
                for (int k = std::max(0, fn.k_min); k <= std::min(nz - 1, fn.k_max); k++) {
                    if (fn.vel[0] != 0.0) fu[UI(i, j, k)] = fu[UI(i + 1, j, k)] = code;
                    if (fn.vel[1] != 0.0) fv[VI(i, j, k)] = fv[VI(i, j + 1, k)] = code;
                    if (fn.vel[2] != 0.0) fw[WI(i, j, k)] = fw[WI(i, j, k + 1)] = code;
                }
    }
    for (const ffr_patch &p : r.patches)
        for (int a = p.a_min; a <= p.a_max; a++)
            for (int b = p.b_min; b <= p.b_max; b++) {
                if (p.axis == 0) fu[UI(p.side ? nx : 0, a, b)] |= FC_OUTCOPY;
                else if (p.axis == 1) fv[VI(a, p.side ? ny : 0, b)] |= FC_OUTCOPY;
                else fw[WI(a, b, p.side ? nz : 0)] |= FC_OUTCOPY;
            }
}

// Neighbour classes of PoissonSolver::apply_laplacian (PoissonSolver.cpp:
// 61-77) and its per-axis scales (PoissonSolver.cpp:33-49), computed with
// the same double expressions so that the device stencil uses identical
// coefficients.
void build_stencil(const HostRoom &r, std::vector<uint16_t> &sc, std::vector<double> &scale)
{
    const int nx = r.g.nx, ny = r.g.ny, nz = r.g.nz;
    sc.assign(r.g.n, 0);
    auto CI = [&](int i, int j, int k) { return (size_t)i * ny * nz + (size_t)j * nz + k; };
    auto cls = [&](int i, int j, int k) -> uint16_t {
        if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) return SC_NONE;
        const uint8_t t = r.ct[CI(i, j, k)];
        return t == CT_OUTFLOW ? SC_DIR : (t == CT_SOLID ? SC_NONE : SC_IN);
    };
    parallel_slabs(nx, [&](int i0, int i1) {
    for (int i = i0; i < i1; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                uint16_t c = 0;
                if (r.ct[CI(i, j, k)] == CT_SOLID) {
                    c = SC_SOLID;
                } else {
                    c |= cls(i - 1, j, k) << 0;
                    c |= cls(i + 1, j, k) << 2;
                    c |= cls(i, j - 1, k) << 4;
                    c |= cls(i, j + 1, k) << 6;
                    c |= cls(i, j, k - 1) << 8;
                    c |= cls(i, j, k + 1) << 10;
                    if (r.ct[CI(i, j, k)] == CT_OUTFLOW) c |= SC_OUTF;
                }
                sc[CI(i, j, k)] = c;
            }
    });
    // layout: [sxl(nx) sxr(nx) syl(ny) syr(ny) szl(nz) szr(nz)]
    scale.assign(2 * (size_t)(nx + ny + nz), 0.0);
    auto axis = [&](const std::vector<double> &h, int m, double *sl, double *sr) {
        for (int i = 0; i < m; i++) {
            const double hl = (i > 0) ? 0.5 * (h[i - 1] + h[i]) : h[i];
            const double hr = (i < m - 1) ? 0.5 * (h[i] + h[i + 1]) : h[i];
            sl[i] = 1.0 / (hl * h[i]);
            sr[i] = 1.0 / (hr * h[i]);
        }
    };
    double *s = scale.data();
    axis(r.dxv, nx, s, s + nx);
    axis(r.dyv, ny, s + 2 * nx, s + 2 * nx + ny);
    axis(r.dzv, nz, s + 2 * nx + 2 * ny, s + 2 * nx + 2 * ny + nz);
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
