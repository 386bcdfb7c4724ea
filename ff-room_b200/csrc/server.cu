// server.cu — continuous-batching server over one GPU (host code only).
//
// Requests wait in arrival order; a request is admitted while fewer than
// max_active rooms are in flight and its device bytes (ffr_fluid_estimate_
// bytes) fit the budget next to the rooms in flight.  A request that does
// not fit does not block the ones behind it: later, smaller requests that
// fit are admitted past it, but each waiting request can be passed at most
// kMaxPassed times; once the oldest blocked request reaches that bound no
// one passes it any more, so the rooms in flight drain until it fits
// (bounded waiting for large rooms).  An admitted room gets
// its own ffr_fluid handle (own stream, CUDA-graph steps, the size-class
// schedule below) and advances in chunks: ffr_fluid_enqueue queues a chunk,
// ffr_fluid_poll collects it without blocking, and the next chunk is queued
// at once.  A room leaves when a chunk ends early (the room converged, with
// stop_on_converge) or at its step cap; its memory then admits the next
// request.  No thread is started: the caller's progress/drain calls drive
// everything, so the C ABI stays single-threaded per server.
#include "common.cuh"

#include <chrono>
#include <deque>
#include <new>
#include <thread>
#include <vector>

namespace ffr {
namespace {

constexpr long long kClusterMaxCells = 1ll << 20;   // one 16-block cluster per room up to this size
constexpr int kClusterCtas = 16;
constexpr int kMaxPassed = 16;      // admissions past one waiting request before it blocks the queue
constexpr size_t kScanDepth = 256;  // queued requests looked at per admission round

double now_s(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// A room descriptor with its own copies of every array.
struct RoomCopy {
    std::vector<double> dxv, dyv, dzv;
    std::vector<uint8_t> ct;
    std::vector<ffr_fan> fans;
    std::vector<ffr_patch> patches;
    std::vector<ffr_heat_patch> heats;
    ffr_room_desc desc{};

    void take(const ffr_room_desc &d)
    {
        const size_t n = (size_t)d.nx * d.ny * d.nz;
        dxv.assign(d.dxv, d.dxv + d.nx);
        dyv.assign(d.dyv, d.dyv + d.ny);
        dzv.assign(d.dzv, d.dzv + d.nz);
        ct.assign(d.cell_type, d.cell_type + n);
        fans.assign(d.fans, d.fans + (d.fans ? d.nfans : 0));
        patches.assign(d.patches, d.patches + (d.patches ? d.npatches : 0));
        heats.assign(d.heats, d.heats + (d.heats ? d.nheat : 0));
        desc = d;
        desc.dxv = dxv.data(); desc.dyv = dyv.data(); desc.dzv = dzv.data();
        desc.cell_type = ct.data();
        desc.fans = fans.data(); desc.nfans = (int)fans.size();
        desc.patches = patches.data(); desc.npatches = (int)patches.size();
        desc.heats = heats.data(); desc.nheat = (int)heats.size();
    }
};

struct Request {
    long long id = 0;
    RoomCopy room;
    ffr_fluid_params prm{};
    int max_steps = 0;
    size_t bytes = 0;
    double t_submit = 0.0;
    int passed = 0;     // later requests admitted while this one waited
};

struct Active {
    Request *req = nullptr;
    ffr_fluid *h = nullptr;
    int steps = 0, queued = 0;
    ffr_step_result last{};
    bool has_last = false;
    double t_admit = 0.0;
};

}  // namespace
}  // namespace ffr

using namespace ffr;

struct ffr_server {
    size_t budget = 0, used = 0;
    int max_active = 1, chunk = 1;
    std::chrono::steady_clock::time_point t0;
    std::deque<Request *> queue;
    std::vector<Active> active;
    std::deque<ffr_outcome> done;
    std::vector<ffr_step_result> buf;
};

namespace {

ffr_outcome finish(ffr_server *s, Active &a, int status)
{
    ffr_outcome o{};
    o.id = a.req->id;
    o.cells = (long long)a.req->room.desc.nx * a.req->room.desc.ny * a.req->room.desc.nz;
    o.status = status;
    o.steps = a.steps;
    o.converged = a.has_last ? a.last.converged : 0;
    o.velocity_change = a.has_last ? a.last.velocity_change : 0.0;
    o.divergence_max = a.has_last ? a.last.divergence_max : 0.0;
    o.T_mean = a.has_last ? a.last.T_mean : 0.0;
    o.t_submit = a.req->t_submit;
    o.t_admit = a.t_admit;
    o.t_done = now_s(s->t0);
    if (a.h) ffr_fluid_destroy(a.h);
    a.h = nullptr;
    s->used -= a.req->bytes;
    delete a.req;
    a.req = nullptr;
    return o;
}

int launch_chunk(ffr_server *s, Active &a)
{
    a.queued = std::min(s->chunk, a.req->max_steps - a.steps);
    return ffr_fluid_enqueue(a.h, a.queued, 1);
}

// Creates the room's handle with its size-class schedule and queues its
// first chunk; a failure ends the request with that status.
int admit(ffr_server *s, Request *r, Active &a)
{
    a = Active{};
    a.req = r;
    a.t_admit = now_s(s->t0);
    int rc = ffr_fluid_create(&r->room.desc, &r->prm, nullptr, &a.h);
    if (rc) return rc;
    const long long cells = (long long)r->room.desc.nx * r->room.desc.ny * r->room.desc.nz;
    const bool mg = r->prm.poisson == FFR_POISSON_MGPCG || r->prm.use_multigrid;
    if (mg && cells <= kClusterMaxCells) rc = ffr_fluid_set_cluster(a.h, kClusterCtas);
    if (!rc) rc = ffr_fluid_use_graph(a.h, 1);
    if (!rc && r->max_steps > 0) rc = launch_chunk(s, a);
    return rc;
}

}  // namespace

extern "C" {

int ffr_server_create(size_t mem_budget, int max_active, int chunk, ffr_server **out)
{
    if (!out) return fail(FFR_EINVAL, "NULL out");
    *out = nullptr;
    if (mem_budget == 0 || max_active <= 0 || chunk <= 0 || chunk > 1024)
        return fail(FFR_EINVAL, "budget, max_active and chunk (1..1024) must be positive");
    ffr_server *s = new (std::nothrow) ffr_server();
    if (!s) return fail(FFR_ENOMEM, "host allocation");
    s->budget = mem_budget;
    s->max_active = max_active;
    s->chunk = chunk;
    s->t0 = std::chrono::steady_clock::now();
    s->buf.resize(1024);
    *out = s;
    return FFR_OK;
}

int ffr_server_destroy(ffr_server *s)
{
    if (!s) return FFR_OK;
    for (Active &a : s->active) {
        if (a.h) ffr_fluid_destroy(a.h);
        delete a.req;
    }
    for (Request *r : s->queue) delete r;
    delete s;
    return FFR_OK;
}

int ffr_server_submit(ffr_server *s, long long id, const ffr_room_desc *room, const ffr_fluid_params *params,
                      int max_steps)
{
    if (!s || !room || !params) return fail(FFR_EINVAL, "NULL server, room or params");
    if (max_steps < 0) return fail(FFR_EINVAL, "negative max_steps");
    size_t bytes = 0;
    int rc = ffr_fluid_estimate_bytes(room, params, &bytes);   // also validates the room
    if (rc) return rc;
    if (bytes > s->budget) return fail(FFR_ERANGE, "the room alone exceeds the server's memory budget");
    Request *r = new (std::nothrow) Request();
    if (!r) return fail(FFR_ENOMEM, "host allocation");
    r->id = id;
    r->room.take(*room);
    r->prm = *params;
    r->max_steps = max_steps;
    r->bytes = bytes;
    r->t_submit = now_s(s->t0);
    s->queue.push_back(r);
    return FFR_OK;
}

int ffr_server_progress(ffr_server *s, ffr_outcome *out, int max_out, int *nout, int *pending)
{
    if (!s || (max_out > 0 && !out) || max_out < 0) return fail(FFR_EINVAL, "bad server progress arguments");
    // admission: arrival order, a free slot and room in the budget (the
    // first room is always admitted when nothing runs); requests that fit
    // may pass ones that do not, up to kMaxPassed times each
    size_t qi = 0;
    while (qi < s->queue.size() && qi < kScanDepth && (int)s->active.size() < s->max_active) {
        Request *r = s->queue[qi];
        if (!s->active.empty() && s->used + r->bytes > s->budget) {
            if (r->passed >= kMaxPassed) break;   // this one waits longest: let the GPU drain for it
            qi++;
            continue;
        }
        for (size_t b = 0; b < qi; b++) s->queue[b]->passed++;
        s->queue.erase(s->queue.begin() + (long)qi);
        s->used += r->bytes;
        s->active.emplace_back();
        Active &a = s->active.back();
        const int rc = admit(s, r, a);
        if (rc || r->max_steps == 0) {
            s->done.push_back(finish(s, a, rc));
            s->active.pop_back();
        }
    }
    // completion of queued chunks; the next chunk goes out at once
    std::vector<Active> still;
    still.reserve(s->active.size());
    for (Active &a : s->active) {
        int got = 0, ready = 0;
        int rc = ffr_fluid_poll(a.h, s->buf.data(), (int)s->buf.size(), &got, &ready);
        if (rc) {
            s->done.push_back(finish(s, a, rc));
            continue;
        }
        if (!ready) {
            still.push_back(a);
            continue;
        }
        a.steps += got;
        if (got > 0) {
            a.last = s->buf[got - 1];
            a.has_last = true;
        }
        const bool halted = got < a.queued;
        if (halted || a.steps >= a.req->max_steps || (a.has_last && a.last.converged)) {
            s->done.push_back(finish(s, a, FFR_OK));
            continue;
        }
        rc = launch_chunk(s, a);
        if (rc) {
            s->done.push_back(finish(s, a, rc));
            continue;
        }
        still.push_back(a);
    }
    s->active.swap(still);
    int n = 0;
    while (n < max_out && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    if (nout) *nout = n;
    if (pending) *pending = (int)(s->queue.size() + s->active.size() + s->done.size());
    return FFR_OK;
}

int ffr_server_drain(ffr_server *s, ffr_outcome *out, int max_out, int *nout)
{
    if (!s) return fail(FFR_EINVAL, "NULL server");
    int total = 0;
    while (true) {
        int got = 0, pending = 0;
        const int rc = ffr_server_progress(s, out ? out + total : nullptr, max_out - total, &got, &pending);
        if (rc) return rc;
        total += got;
        if (s->queue.empty() && s->active.empty()) break;
        if (got == 0) std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    if (nout) *nout = total;
    return FFR_OK;
}

}  // extern "C"
