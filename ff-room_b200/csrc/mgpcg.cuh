// mgpcg.cuh — multigrid-preconditioned CG for the pressure Poisson problem.
#pragma once
#include "projection.cuh"

#include <vector>

namespace ffr {

constexpr int kMaxLevels = 12;
// Levels with at most this many cells run inside one CTA (no grid barrier).
constexpr int kBlockLevelCells = 640;

// One coarse level: per cell (T to the x+, y+, z+ neighbour, diagonal), FP32.
// Inactive cells (no FLUID/INFLOW child) have diagonal 0.
struct MGLevel {
    int nx, ny, nz, n;
    const float4 *coef;   // level >= 1
    float *x, *b;
};

struct MGDev {
    int nlev;             // levels including the fine one
    int nlev_grid;        // levels 0 .. nlev_grid-1 use grid-wide passes
    MGLevel lv[kMaxLevels];
    // fine-level face transmissibility factors (FP32): T_x-(i,j,k) =
    // dy[j]*dz[k]*ix_l[i] and so on; vol = dx*dy*dz
    const float *dx, *dy, *dz, *ixl, *ixr, *iyl, *iyr, *izl, *izr;
    const double *vol_x, *vol_y, *vol_z;   // FP64 spacings for the cell volume
    int uniform;          // all spacings equal per axis: tx, ty, tz, vol hold the constants
    float tx, ty, tz, vol;
    float *r32;           // FP32 copy of the scaled CG residual (level-0 rhs)
};

// Host side: builds the coarse levels of a room and uploads them.
struct MGHost {
    std::vector<int> nx, ny, nz;
    std::vector<std::vector<float4>> coef;   // index 0 unused
};
void build_mg_levels(const HostRoom &r, MGHost &out);
// Device bytes the hierarchy needs (FP32 z, r32, coarse levels, factors).
size_t mg_bytes(const HostRoom &r, const MGHost &h);
// Carves the hierarchy from `ar`, uploads it and fills `M`.
int mg_upload(const HostRoom &r, const MGHost &h, Arena &ar, cudaStream_t s, MGDev &M);

struct PCGArgs {
    RoomDev R;
    MGDev M;
    const double *us, *vs, *ws;    // rhs from predicted faces when from_faces
    double rhs_factor;
    int from_faces;
    const double *rhs;
    double *x, *r, *da, *db, *q;
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
// Cooperative launch of the whole preconditioned solve.
int launch_pcg(const PCGArgs &a, cudaStream_t s, unsigned *blocks_used, unsigned override_blocks = 0);
unsigned pcg_max_blocks();
// One thread-block cluster of `ctas` blocks (1..16) solves the room.
int launch_pcg_cluster(const PCGArgs &a, cudaStream_t s, int ctas);

}  // namespace ffr
