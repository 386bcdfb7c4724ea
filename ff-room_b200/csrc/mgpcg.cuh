// mgpcg.cuh — multigrid-preconditioned CG for the pressure Poisson problem.
#pragma once
#include "projection.cuh"

#include <vector>

namespace ffr {

constexpr int kMaxLevels = 12;
// Levels with at most this many cells run inside one CTA (no grid barrier).
constexpr int kBlockLevelCells = 640;
// Levels (>= 1) with at most this many cells run, in the split solve, inside
// one thread-block cluster of kMidThreads-thread blocks.
constexpr int kMidLevelCells = 32 * 1024;
constexpr int kMidThreads = 512;
// Red-black Gauss-Seidel sweeps per visit of a level in the V-cycle, before
// and after its coarse-grid correction (symmetric, as CG needs).  On level
// 0 the first sweep's red half before the correction is fused into the
// residual pass and the last sweep's red half after it into the r.z pass.
// Measured on the 320x256x96 thermal room: one sweep everywhere 17.2 PCG
// iterations per step at 388 us each (7.13 ms per step), two on the coarse
// levels 13.75 at 444 us (6.56 ms), two on every level 9.7 at 571 us
// (6.01 ms), three on the coarse levels no better than two.
constexpr int kSmoothSweeps = 2;
__host__ __device__ constexpr int level_sweeps(int) { return kSmoothSweeps; }
// The hierarchy coarsens until a level has at most kCoarsestCells cells,
// which kCoarsestSweeps red-black sweeps then solve all but exactly.  The
// coarse solve was the preconditioner's weak point: with levels down to 512
// cells and 8 sweeps the room above took 9.7 iterations per step, with 16
// sweeps 8.75, with levels down to 16 cells and 16 sweeps 6.8 (6.01 -> 4.65
// ms per step); 32 sweeps or levels down to 8 cells gave no fewer.
constexpr int kCoarsestCells = 16;
constexpr int kCoarsestSweeps = 16;

// One coarse level: per cell (T to the x+, y+, z+ neighbour, diagonal), FP32.
// Inactive cells (no FLUID/INFLOW child) have diagonal 0.
struct MGLevel {
    int nx, ny, nz, n;
    int sx, sy, sz, pad;  // 1 where the next coarser level halves the axis
    const float4 *coef;   // level >= 1
    float *x, *b;
};

struct MGDev {
    int nlev;             // levels including the fine one
    int nlev_grid;        // levels 0 .. nlev_grid-1 use grid-wide passes
    int nlev_mid;         // split solve: levels nlev_mid .. nlev_grid-1 run in one cluster
    MGLevel lv[kMaxLevels];
    // fine-level face transmissibility factors (FP32): T_x-(i,j,k) =
    // dy[j]*dz[k]*ix_l[i] and so on; vol = dx*dy*dz
    const float *dx, *dy, *dz, *ixl, *ixr, *iyl, *iyr, *izl, *izr;
    const double *vol_x, *vol_y, *vol_z;   // FP64 spacings for the cell volume
    int uniform;          // all spacings equal per axis: tx, ty, tz, vol hold the constants
    float tx, ty, tz, vol;
    double s64x, s64y, s64z, vol64;   // uniform: FP64 stencil scales 1/h^2 and cell volume
    double diag64;                    // uniform: FP64 diagonal of an all-interior row
    float *r32;           // FP32 copy of the scaled CG residual (level-0 rhs)
};

// Host side: the level sizes of a room's hierarchy.
struct MGHost {
    std::vector<int> nx, ny, nz;
    std::vector<int> sx, sy, sz;             // axes halved towards the next level
};
void build_mg_levels(const HostRoom &r, MGHost &out);
// Device bytes the hierarchy needs (FP32 z, r32, coarse levels, factors).
size_t mg_bytes(const HostRoom &r, const MGHost &h);
// Carves the hierarchy from `ar`, fills `M` and queues on s, without
// waiting: the fine-level factors (through the staging block hs) and the
// coarse coefficients, built by kernels from the room's uploaded cell
// types and spacings (R).
int mg_upload(const HostRoom &r, const MGHost &h, const RoomDev &R, Arena &ar, HostStage &hs, cudaStream_t s,
              MGDev &M);
// Staging bytes mg_upload needs.
size_t mg_stage_bytes(const HostRoom &r);

struct PCGArgs {
    RoomDev R;
    MGDev M;
    const double *us, *vs, *ws;    // rhs from predicted faces when from_faces
    double rhs_factor;
    int from_faces;
    int warm;                      // start from x as it is (else from x = 0)
    const double *rhs;
    double *x, *r, *da, *db, *q;
    double *xprev, *x0;            // warm start: the previous solution, the start kept
    double *partials;
    GridSync *gs;
    CGScalars *sc;
    int max_iter;
    double tol;
    StepState *st;
    double *out_res;
    int *out_iters;
    int *out_flags;
};
// Warm start of the next solve, queued before it: x0 = x + theta (x - xprev)
// (x the previous step's solution, xprev the one before; theta 0 on a
// room's first two steps, 1/2 up to its tenth, 1 after); xprev = x; the
// start is also kept in a.x0.
int launch_extrapolate(const PCGArgs &a, cudaStream_t s);
// Cooperative launch of the whole preconditioned solve.
int launch_pcg(const PCGArgs &a, cudaStream_t s, unsigned *blocks_used, unsigned override_blocks = 0);
unsigned pcg_max_blocks();
// One thread-block cluster of `ctas` blocks (1..16) solves the room.
int launch_pcg_cluster(const PCGArgs &a, cudaStream_t s, int ctas);
// The same solve as one plain kernel per pass, recorded into the graph being
// captured on `s` with a conditional WHILE node around one iteration (the
// iteration body is captured on `bs`).  ss_dev holds split_state_bytes()
// of zeroed device memory; the partials array needs 2 * 2368 doubles.
size_t split_state_bytes();
// Records the split solve into the stream capture in progress on `s`; the
// loop body (one PCG iteration) is captured on `bs`.  *body_kernels receives
// the number of kernels one iteration runs.
int capture_split_pcg(const PCGArgs &a, void *ss_dev, cudaStream_t s, cudaStream_t bs,
                      unsigned *body_kernels = nullptr);
// Host-side state of the eagerly launched split solve: a pinned copy of the
// device iteration count and done flag per batch, and the iteration count of
// the previous solve (the size of the first batch).
struct SplitHost {
    int *flags = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int last_iters = 8;
    int init();
    void release();
};
// ---- batched split solve: one launch per pass over every room of a batch.
struct SplitState;
// Block -> room table of one launch shape: room[b] for every block b of the
// launch; the blocks of room r are first[r] .. first[r + 1] - 1.
struct BMap {
    const int *room;
    const int *first;
};
// Position of a block among the blocks that work on one room: its index
// lb and their number nb (the whole grid for a one-room launch).
struct BPos {
    int lb, nb;
};
__device__ __forceinline__ BPos grid_pos() { return BPos{(int)blockIdx.x, (int)gridDim.x}; }
// The room of this block in a batched launch, and its position there.
__device__ __forceinline__ int bmap(const BMap &m, BPos &P)
{
    const int r = m.room[blockIdx.x];
    const int f = m.first[r];
    P.lb = (int)blockIdx.x - f;
    P.nb = m.first[r + 1] - f;
    return r;
}
// Device view of a batch: per-room arguments and split states, and the
// count of rooms still iterating.
struct BatchDev {
    const PCGArgs *args;
    SplitState *const *ss;
    int *active;
};
// Host side: the launch shapes of a batch (device tables built by
// batch_split_build) and the pacing state.
struct BatchSplit {
    BatchDev D{};
    int nrooms = 0;
    // level-0 passes (init, red post-smooth, direction, residual, final,
    // back-substitution): the one-room grid of each room
    BMap cells0{};
    unsigned nb_cells0 = 0;
    // per grid level l: smoothing (pairs of level l) and restriction (cells
    // of level l + 1), for the rooms that smooth level l on the grid
    int nlev = 0;
    BMap pairs[kMaxLevels]{}, coarse[kMaxLevels]{};
    unsigned nb_pairs[kMaxLevels]{}, nb_coarse[kMaxLevels]{};
    BMap post[kMaxLevels]{};          // up-sweep smoothing of level l >= 1
    unsigned nb_post[kMaxLevels]{};
    BMap post0{};                     // level-0 black post-smoothing
    unsigned nb_post0 = 0;
    const int *mid_rooms = nullptr;   // rooms with levels small enough for one block
    const int *cluster_order = nullptr;   // rooms largest first (one-cluster-per-room launch)
    int nmid = 0;
    void *dev = nullptr;              // device allocation holding all tables
    size_t cap = 0;                   // its size (reused while large enough)
    int *active_host = nullptr;       // pinned copy of the active count
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int last_iters = 8;
};
// Builds the tables for rooms with the given per-room arguments (host
// copies; device pointers inside) and device split states.  The device
// buffer of an earlier build is reused when large enough; no launch of an
// earlier build may still be running.
int batch_split_build(BatchSplit &B, const std::vector<PCGArgs> &args, const std::vector<void *> &ss);
void batch_split_release(BatchSplit &B);
// The split solve of every room of the batch, host-paced like
// launch_split_pcg: iterations are queued in batches until no room is
// still iterating.
// max_iter bounds the batches queued (the largest poisson_max_iter of the
// rooms; every room also stops itself at its own).
int batch_split_solve(BatchSplit &B, cudaStream_t s, int max_iter);
// The same solve recorded into the graph being captured on s: a WHILE node
// whose body (captured on bs) is one iteration of every room, repeated while
// any room is still iterating, so a batched step replays with no host
// involvement.
int capture_batch_split(BatchSplit &B, cudaStream_t s, cudaStream_t bs);
// Every room's whole solve in one launch, one thread-block cluster of `ctas`
// blocks per room (each room's own one-cluster schedule, ffr_fluid_set_
// cluster), after the batched warm-start extrapolation.  No host pacing and
// nothing to capture specially.
int launch_batch_cluster(BatchSplit &B, cudaStream_t s, int ctas);

// The split solve launched kernel by kernel outside any graph.  The host
// queues iterations in batches and stops at the first batch whose copy of
// the done flag reads set; kernels queued past convergence return at once.
// Blocks the calling thread until the solve's last batch has been queued.
int launch_split_pcg(const PCGArgs &a, void *ss_dev, cudaStream_t s, SplitHost &h);

}  // namespace ffr
