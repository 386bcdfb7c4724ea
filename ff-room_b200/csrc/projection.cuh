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
};

}  // namespace ffr
