/*
 * ffroom.h — C ABI of the B200 (sm_100a) room solver, libffroom_cuda.so.
 *
 * This is the drop-in boundary for ff-room's per-timestep solver: the
 * pybind11 module `_ffroom_core` shipped next to the library (the same class
 * surface as the reference's cpp/src/bindings/module.cpp) calls only these
 * functions, and a C, ctypes or cgo caller can bind them directly.  Every
 * entry point returns an ffr_status; no C++ exception crosses the ABI.
 * Field arrays use the reference layout (cpp/src/core/Grid.hpp:59-65):
 * flat, k fastest; u is (nx+1)*ny*nz, v nx*(ny+1)*nz, w nx*ny*(nz+1),
 * p / T / cell_type nx*ny*nz.  Host pointers are plain `double *`; device
 * pointers are marked `_dev`.
 *
 * Thread safety: a handle may be used by one host thread at a time; distinct
 * handles are independent (each owns its CUDA stream and memory).
 */
#ifndef FFROOM_H
#define FFROOM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status */
typedef enum ffr_status {
    FFR_OK = 0,
    FFR_EINVAL = 1,      /* bad argument (the reference would throw or misbehave) */
    FFR_ENOMEM = 2,      /* device or pinned-host allocation failed */
    FFR_ECUDA = 3,       /* a CUDA runtime call failed */
    FFR_ETIMEDOUT = 4,   /* a bounded device-side wait gave up */
    FFR_ENOTSUP = 5,     /* valid for the reference, not supported here */
    FFR_ERANGE = 6       /* a size exceeds a fixed capacity */
} ffr_status;

/* Step-result status bits (ffr_step_result.flags). */
#define FFR_FLAG_NAN          1  /* a NaN reached the velocity field */
#define FFR_FLAG_CG_MAXITER   2  /* the pressure solve hit poisson_max_iter */
#define FFR_FLAG_CG_BREAKDOWN 4  /* |d.Ad| < 1e-30 ended the pressure solve */
#define FFR_FLAG_TIMEOUT      8  /* a device barrier timed out */

/* Static text for a status code.  Status codes and the message below take
 * the place of the reference's C++ exceptions (e.g. Grid.cpp:10-11 throws
 * std::invalid_argument), which cannot cross a C ABI. */
const char *ffr_status_string(int status);
/* Detail of the most recent failure on the calling thread ("" if none). */
const char *ffr_last_error(void);
/* Upper bound of every bounded device-side wait (the grid barriers of the
 * persistent solves), in seconds on the current device; 0 restores the
 * default of 4 s.  For tests of the failure path; no counterpart in the
 * reference. */
int ffr_set_device_wait_limit(double seconds);
/* Self-test of that bound: a kernel whose blocks wait at a grid barrier
 * that one block never reaches.  Every wait gives up at the limit, the
 * kernel returns and this returns FFR_ETIMEDOUT with the kernel's duration
 * in *elapsed_ms; the CUDA context stays usable.  No counterpart in the
 * reference. */
int ffr_selftest_device_wait(int blocks, double *elapsed_ms);
/* Library version, e.g. "0.1.0 sm_100a" (no counterpart in the reference). */
const char *ffr_version(void);
/* Kernels this library has launched since load (all handles; no
 * counterpart in the reference). */
unsigned long long ffr_launch_count(void);

/* ------------------------------------------------------------- rooms */

/* Cell types, cpp/src/core/Grid.hpp:9-14. */
enum { FFR_FLUID = 0, FFR_SOLID = 1, FFR_INFLOW = 2, FFR_OUTFLOW = 3 };
/* Advection schemes, cpp/src/core/FluidSolver.hpp:9. */
enum { FFR_UPWIND1 = 0, FFR_QUICK = 1, FFR_LAX_WENDROFF = 2 };
/* Field selectors. */
enum { FFR_FIELD_U = 0, FFR_FIELD_V = 1, FFR_FIELD_W = 2, FFR_FIELD_P = 3, FFR_FIELD_T = 4 };
/* Arithmetic of the projection step. */
enum { FFR_PREC_FP64 = 0,   /* the reference method, FP64 throughout */
       FFR_PREC_MIXED = 1 };/* FP32 predictor/thermal, FP64 Krylov outer loop */
/* Pressure solver. */
enum { FFR_POISSON_CG = 0,    /* the reference's unpreconditioned CG */
       FFR_POISSON_MGPCG = 1 };/* multigrid-preconditioned CG */
/* LBM population storage. */
enum { FFR_LBM_FP64 = 0, FFR_LBM_FP32 = 1, FFR_LBM_FP16 = 2 };

/* FanBC, cpp/src/core/BoundaryManager.hpp:8-13: an inclusive cell box
 * (clamped to the grid) and the face velocity it imposes. */
typedef struct ffr_fan {
    int i_min, i_max, j_min, j_max, k_min, k_max;
    double vel[3];
} ffr_fan;

/* OutflowBC / OpeningBC, cpp/src/core/BoundaryManager.hpp:15-29: a patch of
 * boundary cells on wall (axis, side); openings also carry T_outside. */
typedef struct ffr_patch {
    int axis, side, a_min, a_max, b_min, b_max;
    int is_opening;
    double T_outside;
} ffr_patch;

/* Fixed-temperature cell box (no counterpart in the reference: the heated
 * floor / cooled ceiling extension, re-imposed after every step). */
typedef struct ffr_heat_patch {
    int i_min, i_max, j_min, j_max, k_min, k_max;
    double T;
} ffr_heat_patch;

/* One room: the state a reference Grid + BoundaryManager pair carries
 * (Grid.hpp:26-69, BoundaryManager.hpp:31-72).  `patches` is the
 * BoundaryManager outflow list in insertion order with openings included,
 * exactly as add_outflow/add_opening build it (BoundaryManager.cpp:24-44,
 * 132-135). */
typedef struct ffr_room_desc {
    int nx, ny, nz;
    double lx, ly, lz;
    const double *dxv, *dyv, *dzv;     /* cell spacings, sizes nx, ny, nz */
    const uint8_t *cell_type;          /* nx*ny*nz */
    int nfans;    const ffr_fan *fans;
    int npatches; const ffr_patch *patches;
    int nheat;    const ffr_heat_patch *heats;
} ffr_room_desc;

/* FluidSolverParams + PoissonSolverParams, cpp/src/core/FluidSolver.hpp:
 * 11-38 and PoissonSolver.hpp:14-18, plus precision / poisson selectors. */
typedef struct ffr_fluid_params {
    double rho, nu, dt;
    int max_steps;
    double convergence_tol;
    int poisson_max_iter;
    double poisson_tol;
    int advection;
    int use_multigrid;     /* reference flag; selects FFR_POISSON_MGPCG here */
    int thermal;
    double T_initial, T_target;
    int buoyancy;
    double g_accel, beta, k_thermal, cp;
    int precision;         /* FFR_PREC_* */
    int poisson;           /* FFR_POISSON_* */
} ffr_fluid_params;

/* StepResult, cpp/src/core/FluidSolver.hpp:40-47, plus the pressure-solve
 * iteration count and status flags (FFR_FLAG_*). */
typedef struct ffr_step_result {
    int step;
    double velocity_change;
    double pressure_residual;
    double divergence_max;
    int converged;
    double T_mean;
    int cg_iterations;
    int flags;
} ffr_step_result;

/* Initial fields for a new solver; any pointer may be NULL (zeros). */
typedef struct ffr_fields {
    const double *u, *v, *w, *p;
} ffr_fields;

/* --------------------------------------------------- projection solver */
typedef struct ffr_fluid ffr_fluid;

/* FluidSolver::FluidSolver (cpp/src/core/FluidSolver.cpp:18-32): uploads the
 * room and the initial fields, sets T := T_initial and, when thermal,
 * applies the opening temperature BC.  The cell types and fields are copied
 * before it returns; the tables derived from them (stencil and face codes,
 * multigrid coefficients) are built by kernels queued on the handle's
 * stream, which every later call on the handle follows, so a server
 * creating rooms never waits for a busy GPU here. */
int ffr_fluid_create(const ffr_room_desc *room, const ffr_fluid_params *params,
                     const ffr_fields *init, ffr_fluid **out);
/* Frees the handle (the reference's FluidSolver destructor); waits for its
 * queued work and leaves every batch it belongs to. */
int ffr_fluid_destroy(ffr_fluid *s);

/* FluidSolver::step (FluidSolver.cpp:486-550): one projection step; `out`
 * may be NULL (then no host synchronisation happens). */
int ffr_fluid_step(ffr_fluid *s, ffr_step_result *out);

/* FluidSolver::run (FluidSolver.cpp:552-560) without the per-step callback:
 * up to `nsteps` steps queued on the device with no host synchronisation in
 * between; with stop_on_converge the steps after the first converged one do
 * no work.  `results` (nsteps entries, may be NULL) receives every executed
 * step; `steps_done` the count. */
int ffr_fluid_advance(ffr_fluid *s, int nsteps, int stop_on_converge,
                      ffr_step_result *results, int *steps_done);

/* Asynchronous form of ffr_fluid_advance for serving many rooms at once
 * (no counterpart in the reference): queues up to 1024 steps on the handle's
 * stream and returns at once.  One chunk may be pending per handle. */
int ffr_fluid_enqueue(ffr_fluid *s, int nsteps, int stop_on_converge);
/* Non-blocking completion check of the pending chunk: *ready = 0 while it
 * runs; once done, copies up to max_results step results (the executed
 * steps only) and sets *ready = 1.  With nothing pending, *ready = 1 and no
 * results. */
int ffr_fluid_poll(ffr_fluid *s, ffr_step_result *results, int max_results, int *nresults,
                   int *ready);
/* Schedules and sizes below have no counterpart in the reference.
 * Grid size of the cooperative pressure solve (0 = as large as the room can
 * use).  Smaller grids let several rooms run side by side. */
int ffr_fluid_set_blocks(ffr_fluid *s, int blocks);
/* Runs the multigrid-preconditioned pressure solve of this room in one
 * thread-block cluster of `ctas` blocks (1..16; 0 = the whole GPU through a
 * cooperative launch).  Many small rooms then advance side by side, each on
 * its own SMs, synchronising through the hardware cluster barrier. */
int ffr_fluid_set_cluster(ffr_fluid *s, int ctas);
/* Device memory the handle holds (one allocation, made at create). */
int ffr_fluid_device_bytes(ffr_fluid *s, size_t *bytes);
/* Device memory ffr_fluid_create would take for this room and parameters
 * (its allocation plus the transient scratch of the multigrid set-up),
 * without creating anything: admission control for servers. */
int ffr_fluid_estimate_bytes(const ffr_room_desc *room, const ffr_fluid_params *params, size_t *bytes);
/* Captures one step (all its kernels) as a CUDA graph and replays it for
 * every later step of ffr_fluid_enqueue/advance/step (enable = 1), or goes
 * back to direct launches (0).  The kernels read their per-step state from
 * device memory, so one captured step is valid for every step. */
int ffr_fluid_use_graph(ffr_fluid *s, int enable);
/* Benchmark aid (no counterpart in the reference): solves the pressure
 * system of the last step again `nrep` times from a pressure-only CUDA graph
 * (the same kernels the step runs, from the same starting pressure, the
 * same result each time) and returns the mean milliseconds per solve and its
 * iteration count.  With a warm-started multigrid solve the last step must
 * have been taken by this handle's own launches (not by a batch). */
int ffr_fluid_time_pressure(ffr_fluid *s, int nrep, double *ms_per_solve, int *iterations);
/* Starting pressure of the multigrid-PCG solve: 1 (default) = linear
 * extrapolation of the last two pressures (half a step through a room's
 * first ten steps, a full step after; the previous pressure on its first
 * two steps), 0 = zero, as PoissonSolver::solve starts
 * (PoissonSolver.cpp:93-158).  Either way the solve stops on the
 * reference's ||b - A x|| / ||b|| < tol, so the solution lies within the same
 * tolerance of the exact one; the warm start needs fewer iterations.  The
 * plain FP64 CG always starts from zero.  Set before ffr_fluid_use_graph. */
int ffr_fluid_set_warm_start(ffr_fluid *s, int enable);
/* Multigrid-PCG schedule (no counterpart in the reference): 1 = one kernel
 * per multigrid pass, also outside graphs (the host paces the iterations and
 * ffr_fluid_enqueue returns only after the last step's solve is queued);
 * 0 = one persistent cooperative kernel per solve, also in graphs; -1
 * (default) = split inside captured step graphs, persistent otherwise.
 * Set before ffr_fluid_use_graph. */
int ffr_fluid_set_split(ffr_fluid *s, int mode);

/* Batched rooms (no counterpart in the reference, which solves one room at a
 * time): one kernel launch per stage advances every room of a batch, each
 * room's blocks doing what its own launch would (results identical to the
 * room solved alone with the one-kernel-per-pass multigrid schedule).  The
 * rooms stay ordinary handles: after ffr_batch_enqueue each room's results
 * are collected with ffr_fluid_poll, and fields are read as usual.  Rooms
 * must use the multigrid pressure solve and one common schedule: either the
 * default grid (the solve runs one batched kernel per pass, paced by the
 * host or by a WHILE node of the step graph) or one cluster size set with
 * ffr_fluid_set_cluster (every room's whole solve runs on its own cluster of
 * that size, all rooms in one launch; results identical to the room solved
 * alone with that cluster size); a room may
 * belong to several batches but only one may run at a time.  Destroying a
 * member waits for the batch's queued work and removes the room from the
 * batch; ffr_batch_enqueue then fails with FFR_EINVAL (queueing nothing)
 * until ffr_batch_set_rooms replaces the members, since the batch's device
 * tables still name the destroyed room.  The same holds after an
 * ffr_batch_set_rooms that failed. */
typedef struct ffr_batch ffr_batch;
int ffr_batch_create(ffr_fluid *const *rooms, int nrooms, ffr_batch **out);
/* Replaces the member rooms (the batch's device tables are rebuilt in
 * place, reusing their memory while it is large enough). */
int ffr_batch_set_rooms(ffr_batch *b, ffr_fluid *const *rooms, int nrooms);
int ffr_batch_destroy(ffr_batch *b);
int ffr_batch_size(const ffr_batch *b, int *nrooms);
/* Queues nsteps (0..1024) steps of every room; returns once the last
 * step's pressure solve is queued (the solves are paced by the host, or,
 * with ffr_batch_use_graph, replayed from the captured step graph). */
int ffr_batch_enqueue(ffr_batch *b, int nsteps, int stop_on_converge);
/* enable != 0: the next ffr_batch_enqueue captures one batched step as a
 * CUDA graph (every stage one launch for all rooms; the pressure solve a
 * WHILE node that iterates while any room is still iterating) and each step
 * replays it, so the host queues one graph launch per step and never waits
 * inside a chunk.  Results are identical to the host-paced form.  A
 * membership change (ffr_batch_set_rooms) recaptures it. */
int ffr_batch_use_graph(ffr_batch *b, int enable);

/* FluidSolver::compute_divergence_max (FluidSolver.cpp:470-484). */
int ffr_fluid_divergence_max(ffr_fluid *s, double *out);
/* Snapshot of SolverBridge.run_animated (python/ff_room/solver_bridge.py:
 * 222-238) computed on the device: cell-centred velocity components (face
 * averages) and speed, each nx*ny*nz doubles in the field layout; any
 * output may be NULL.  Only the requested arrays cross PCIe. */
int ffr_fluid_snapshot(ffr_fluid *s, double *uc, double *vc, double *wc, double *speed);
/* FluidSolver::current_step (FluidSolver.hpp:63). */
int ffr_fluid_current_step(ffr_fluid *s, int *out);

/* Host <-> device copies of one field (FFR_FIELD_*), reference layout.  They
 * back the Grid's numpy views (module.cpp:45-80). */
int ffr_fluid_get_field(ffr_fluid *s, int field, double *host);
int ffr_fluid_set_field(ffr_fluid *s, int field, const double *host);
/* Device pointer of one field (valid until destroy; the solver swaps its
 * buffers between steps, so re-query after every step).  This and the two
 * calls below have no counterpart in the reference, whose fields live in
 * host memory. */
int ffr_fluid_field_dev(ffr_fluid *s, int field, double **dev);
/* Blocks until all queued work of the handle is done. */
int ffr_fluid_synchronize(ffr_fluid *s);
/* The cudaStream_t all work of the handle runs on. */
int ffr_fluid_stream(ffr_fluid *s, void **stream);

/* Kernel-group timing: while enabled, every queued step records CUDA events
 * on the handle's stream around each group (no counterpart in the
 * reference; it backs the benchmark's per-kernel roofline).  _read returns
 * the milliseconds and the launch count accumulated per group since the
 * last enable. */
enum { FFR_PROF_PREDICT = 0, FFR_PROF_PRESSURE = 1, FFR_PROF_CORRECT = 2, FFR_PROF_THERMAL = 3,
       FFR_PROF_N = 4 };
int ffr_fluid_profile(ffr_fluid *s, int enable);
int ffr_fluid_profile_read(ffr_fluid *s, double *ms, long long *launches);

/* ------------------------------------------------------------ server */
/* Continuous-batching server over one GPU (no counterpart in the
 * reference, which solves one room per call): rooms are submitted as
 * requests, admitted while a slot and the device-memory budget allow
 * (each charged ffr_fluid_estimate_bytes), advanced on their own streams in
 * chunks of steps (ffr_fluid_enqueue / ffr_fluid_poll, no host wait between
 * chunks), and leave on convergence (stop_on_converge) or at their step
 * cap, when the next queued room is admitted.  Admission goes in arrival
 * order, except that a request which does not fit the budget lets later
 * requests that do fit pass it, at most 16 of them; then it blocks the
 * queue until the rooms in flight leave room for it.  The budget is charged
 * with each room's arena bytes (ffr_fluid_estimate_bytes); the CUDA-graph
 * executables, streams and events of a handle come on top of it, so leave
 * a margin of device memory beyond the budget.  A room's schedule follows
 * its size: up to 2^20 cells the multigrid solve runs in one 16-block
 * thread-block cluster (many rooms side by side), above that on the whole
 * GPU; every step replays a captured CUDA graph.  The server lives on the
 * calling thread: it advances only inside ffr_server_progress/drain. */
typedef struct ffr_server ffr_server;

/* One finished request.  Times are seconds since ffr_server_create. */
typedef struct ffr_outcome {
    long long id;
    long long cells;
    int status;            /* FFR_OK, or the error that ended the request */
    int steps;
    int converged;
    double velocity_change, divergence_max, T_mean;
    double t_submit, t_admit, t_done;
} ffr_outcome;

/* max_active: rooms in flight at once; chunk: steps per queued chunk. */
int ffr_server_create(size_t mem_budget, int max_active, int chunk, ffr_server **out);
int ffr_server_destroy(ffr_server *s);
/* Queues one room (its arrays are copied); it runs up to max_steps steps.
 * FFR_ERANGE when the room alone exceeds the memory budget. */
int ffr_server_submit(ffr_server *s, long long id, const ffr_room_desc *room, const ffr_fluid_params *params,
                      int max_steps);
/* One non-blocking round: admits queued rooms, collects finished chunks,
 * queues the next ones; copies up to max_out finished requests to `out`
 * (*nout of them; the rest wait for the next call) and sets *pending to the
 * requests not yet returned. */
int ffr_server_progress(ffr_server *s, ffr_outcome *out, int max_out, int *nout, int *pending);
/* Rounds until every submitted request has finished; returns up to max_out
 * of them as ffr_server_progress does. */
int ffr_server_drain(ffr_server *s, ffr_outcome *out, int max_out, int *nout);

/* ------------------------------------------------------ pressure solve */
typedef struct ffr_poisson ffr_poisson;

/* A PoissonSolver bound to one room's mask and spacing
 * (cpp/src/core/PoissonSolver.hpp:20-38); allocates its CG scratch. */
int ffr_poisson_create(const ffr_room_desc *room, int max_iter, double tol,
                       ffr_poisson **out);
/* Frees the handle and its CG scratch. */
int ffr_poisson_destroy(ffr_poisson *s);

/* PoissonSolver::solve (PoissonSolver.cpp:93-158) on device buffers: CG
 * from x0 = 0 on L = -lap with the mask-dependent stencil
 * (PoissonSolver.cpp:22-91).  `stream` is a cudaStream_t (NULL = the
 * handle's own stream).  Synchronises and returns the relative residual and
 * the iteration count. */
int ffr_poisson_solve_dev(ffr_poisson *s, const double *rhs_dev, double *p_dev,
                          void *stream, double *residual, int *iterations);

/* The same on host buffers (uploads rhs, downloads p). */
int ffr_poisson_solve(ffr_poisson *s, const double *rhs, double *p,
                      double *residual, int *iterations);

/* PoissonSolver::apply_laplacian (PoissonSolver.cpp:22-91) on host buffers. */
int ffr_poisson_apply(ffr_poisson *s, const double *x, double *ax);

/* The same pressure solve as ffr_poisson_solve_dev, for callers that cannot
 * allocate device memory when they solve: a process whose GPU memory was
 * handed to another allocator up front, or a latency-critical loop that
 * must not take the implicit device synchronisation of cudaMalloc/cudaFree.
 * No counterpart in the reference.  It allocates nothing: its scratch is one
 * fixed __device__ array (about 9 MB, held on every GPU that loads the
 * library until exit) sized for at most FFR_NOALLOC_MAX_CELLS cells and
 * FFR_NOALLOC_MAX_DIM cells per axis; larger rooms get FFR_ERANGE.  The
 * caller passes the spacings on the host and the cell types, rhs and
 * pressure on the device; the stream must belong to the current device.
 * The call is synchronous: it returns only after the solve has finished
 * on that stream (it reads the residual and iteration count back), so it
 * cannot be captured into a CUDA graph.  All calls on a device share that
 * array, so calls that overlap on the GPU race.  Every call looks the
 * array's address up on the current device, so a device reset between
 * calls needs no reload. */
#define FFR_NOALLOC_MAX_CELLS (64 * 64 * 64)
#define FFR_NOALLOC_MAX_DIM 4096
int ffr_poisson_solve_noalloc(int nx, int ny, int nz, const double *dxv, const double *dyv,
                              const double *dzv, const uint8_t *cell_type_dev,
                              const double *rhs_dev, double *p_dev, int max_iter, double tol,
                              void *stream, double *residual, int *iterations);

/* ------------------------------------------------------------------ LBM */
typedef struct ffr_lbm ffr_lbm;

/* LBMSolver::LBMSolver (cpp/src/core/LBMSolver.cpp:33-74): f := W_q, INFLOW
 * cells := feq(1, u_fan*dt/dx).  `init` seeds the face velocities that the
 * first step's velocity change is measured against (NULL = zeros). */
int ffr_lbm_create(const ffr_room_desc *room, double tau, int max_steps,
                   double convergence_tol, double dt, int storage,
                   const ffr_fields *init, ffr_lbm **out);
/* Frees the handle (the reference's LBMSolver destructor). */
int ffr_lbm_destroy(ffr_lbm *s);
/* LBMSolver::step (LBMSolver.cpp:402-440). */
int ffr_lbm_step(ffr_lbm *s, ffr_step_result *out);
/* LBMSolver::run (LBMSolver.cpp:446-454) without the callback. */
int ffr_lbm_advance(ffr_lbm *s, int nsteps, int stop_on_converge,
                    ffr_step_result *results, int *steps_done);
/* LBMSolver::compute_divergence_max (LBMSolver.cpp:382-396). */
int ffr_lbm_divergence_max(ffr_lbm *s, double *out);
/* LBMSolver::current_step (LBMSolver.hpp:38). */
int ffr_lbm_current_step(ffr_lbm *s, int *out);
/* Fields as the reference writes them into the Grid each step
 * (extract_macroscopic, LBMSolver.cpp:288-376): u, v, w faces and p. */
int ffr_lbm_get_field(ffr_lbm *s, int field, double *host);
int ffr_lbm_set_field(ffr_lbm *s, int field, const double *host);
/* Device pointer of the u, v, w or p field (valid until destroy; written in
 * place by every step, so read it in stream order), a wait for the handle's
 * queued work, and its cudaStream_t; no counterpart in the reference. */
int ffr_lbm_field_dev(ffr_lbm *s, int field, double **dev);
int ffr_lbm_synchronize(ffr_lbm *s);
int ffr_lbm_stream(ffr_lbm *s, void **stream);
/* Checkpoint and resume of an LBM room (the reference keeps its populations
 * private: LBMSolver.hpp:77-82 f_, laid out f[q*N + c]).  get copies the
 * populations the handle keeps between steps (post-collision, ready to
 * stream) into f_host as 19*N FP64 values in that layout, with the step
 * counter; set loads them (narrow storage rounds them to its type) and sets
 * the counter.  Together with the u, v, w, p fields (ffr_lbm_get_field /
 * ffr_lbm_set_field) they are the whole state of a room: a handle created
 * for the same room and parameters and loaded this way continues exactly
 * as the saved one would (bit-identically in FP64 storage). */
int ffr_lbm_get_populations(ffr_lbm *s, double *f_host, int *step);
int ffr_lbm_set_populations(ffr_lbm *s, const double *f_host, int step);
/* Kernel-group timing as for ffr_fluid_profile; groups FFR_LPROF_*. */
enum { FFR_LPROF_STREAM_COLLIDE = 0, FFR_LPROF_FACES = 1, FFR_LPROF_N = 2 };
int ffr_lbm_profile(ffr_lbm *s, int enable);
int ffr_lbm_profile_read(ffr_lbm *s, double *ms, long long *launches);

#ifdef __cplusplus
}
#endif
#endif /* FFROOM_H */
