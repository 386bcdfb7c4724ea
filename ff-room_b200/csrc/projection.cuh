// projection.cuh — device view of one room for the projection kernels.
#pragma once
#include "common.cuh"

namespace ffr {

// Per-step device state.  Kernels of a step return immediately when `halt`
// is set (a converged room whose remaining queued steps must do nothing).
struct StepState {
    int step;            // steps executed so far
    int halt;            // 1 after a converged step when stop-on-converge
    int stop_on_converge;
    int tpar;            // which T buffer is current
    unsigned long long dmax_bits;   // max |u_new - u_old| (bit pattern)
    unsigned long long div_bits;    // max |div| over FLUID cells
    double pres;         // pressure-solve relative residual
    int iters;           // pressure-solve iterations
    int flags;           // FFR_FLAG_* of the running step
    int ring_slot;       // next result slot
    int pad;
};

// Scalars a CG solve publishes between its grid-wide phases.
struct CGScalars {
    double red[4];       // grid_allreduce outputs
};

struct RoomDev {
    int nx, ny, nz;
    int n, nu, nv, nw;
    const double *dxv, *dyv, *dzv;
    const uint8_t *ct;
    const uint8_t *fcu, *fcv, *fcw;
    const uint16_t *sc;
    const double *scale;   // sxl sxr syl syr szl szr
    const double *fanvel;  // 3 per fan
    // Reciprocal spacings, S = nx + ny + nz entries per table, axes in
    // turn: [0, S) 1/(cell-centre distance below the cell) (entry 0 of an
    // axis unused), [S, 2S) 1/(cell width) in FP64, then S floats holding
    // the correctly rounded FP32 reciprocal of the FP32 cell width.
    const double *inv;
};

// The reciprocal-spacing tables of a room (RoomDev::inv).
struct InvSpacing {
    const double *cx, *cy, *cz, *wx, *wy, *wz;
    const float *fx, *fy, *fz;
    __device__ __forceinline__ InvSpacing(const RoomDev &R)
    {
        const int S = R.nx + R.ny + R.nz;
        cx = R.inv; cy = cx + R.nx; cz = cy + R.ny;
        wx = R.inv + S; wy = wx + R.nx; wz = wy + R.ny;
        fx = reinterpret_cast<const float *>(R.inv + 2 * S); fy = fx + R.nx; fz = fy + R.ny;
    }
};

struct CGArgs {
    RoomDev R;
    const double *us, *vs, *ws;    // rhs from predicted faces when from_faces
    double rhs_factor;             // -(rho / dt), FluidSolver.cpp:315
    int from_faces;
    const double *rhs;             // explicit right-hand side otherwise
    double *x;
    double *r, *da, *db, *ad;
    double *partials;
    GridSync *gs;
    CGScalars *sc;
    int max_iter;
    double tol;
    StepState *st;                 // may be null
    double *out_res;
    int *out_iters;
    int *out_flags;
};

// The reference's unpreconditioned CG as one cooperative launch
// (projection.cu).
__global__ void __launch_bounds__(256) k_cg(CGArgs A);
unsigned cg_block_cap();

}  // namespace ffr
