// module.cpp — `_ffroom_core`, the drop-in pybind11 module.
//
// It exports the class surface of ff-room's binding module
// (cpp/src/bindings/module.cpp:15-210) with the same names, argument names,
// defaults, fields and StepResult repr, and runs the solvers on the B200
// through the C ABI of libffroom_cuda.so (include/ffroom.h).  Host code only:
// no CUDA header is included here.
//
// Field ownership.  A Grid owns host vectors as the reference's does
// (Grid.hpp:43-53); a solver keeps the live copy of u, v, w, p and T in
// device memory.  The Grid tracks, per field, whether the host or the
// device copy is current and how many numpy views alias the host vector:
//   * a property or *_shaped() call first brings the host copy up to date;
//   * while a view of a field is alive, the solver uploads that field before
//     each step and downloads it after, so a held view behaves like the
//     reference's aliasing view (module.cpp:45-80);
//   * BoundaryManager::apply_* run on the host copy and mark it newer.
// When the mask, the spacing or the boundary lists change after a solver was
// built, the solver rebuilds its device room from the host state.
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>

#include "ffroom.h"

namespace py = pybind11;

namespace b200 {

enum class CellType : uint8_t { FLUID = 0, SOLID = 1, INFLOW = 2, OUTFLOW = 3 };
enum class AdvectionScheme : int { UPWIND1 = 0, QUICK = 1, LAX_WENDROFF = 2 };

[[noreturn]] void raise_status(int st)
{
    std::string msg = std::string(ffr_status_string(st)) + ": " + ffr_last_error();
    if (st == FFR_EINVAL) throw py::value_error(msg);
    throw std::runtime_error(msg);
}

inline void check(int st)
{
    if (st != FFR_OK) raise_status(st);
}

constexpr int kFields = 5;   // u v w p T

struct FieldOwner {
    virtual void pull(int field, double *host) = 0;
    virtual void push(int field, const double *host) = 0;
    virtual ~FieldOwner() = default;
};

struct Grid {
    int Nx, Ny, Nz;
    double dx, dy, dz;
    std::vector<double> dxv, dyv, dzv, xs, ys, zs;
    std::vector<double> u, v, w, p, T;
    std::vector<uint8_t> cell_type;
    // device mirror bookkeeping
    FieldOwner *owner = nullptr;
    std::array<bool, kFields> host_valid{{true, true, true, true, true}};
    std::array<bool, kFields> dev_valid{{true, true, true, true, true}};
    std::array<int, kFields> views{{0, 0, 0, 0, 0}};
    unsigned long long geom_gen = 0, mask_gen = 0;

    // Grid::Grid (Grid.cpp:6-37).
    Grid(int nx, int ny, int nz, double lx, double ly, double lz)
        : Nx(nx), Ny(ny), Nz(nz), dx(lx / nx), dy(ly / ny), dz(lz / nz)
    {
        if (nx <= 0 || ny <= 0 || nz <= 0) throw py::value_error("Grid dimensions must be positive");
        u.assign((size_t)(nx + 1) * ny * nz, 0.0);
        v.assign((size_t)nx * (ny + 1) * nz, 0.0);
        w.assign((size_t)nx * ny * (nz + 1), 0.0);
        p.assign((size_t)nx * ny * nz, 0.0);
        T.assign((size_t)nx * ny * nz, 0.0);
        cell_type.assign((size_t)nx * ny * nz, 0);
        xs.resize(nx + 1); ys.resize(ny + 1); zs.resize(nz + 1);
        for (int i = 0; i <= nx; i++) xs[i] = i * dx;
        for (int j = 0; j <= ny; j++) ys[j] = j * dy;
        for (int k = 0; k <= nz; k++) zs[k] = k * dz;
        dxv.assign(nx, dx); dyv.assign(ny, dy); dzv.assign(nz, dz);
    }
    ~Grid();

    std::vector<double> &field(int f)
    {
        switch (f) {
        case 0: return u;
        case 1: return v;
        case 2: return w;
        case 3: return p;
        default: return T;
        }
    }

    void ensure_host(int f)
    {
        if (owner && !host_valid[f]) {
            owner->pull(f, field(f).data());
            host_valid[f] = true;
        }
    }
    void ensure_host_all()
    {
        for (int f = 0; f < kFields; f++) ensure_host(f);
    }
    void host_written(int f) { dev_valid[f] = false; }

    // Grid::set_face_coords (Grid.cpp:39-47).
    void set_face_coords(std::vector<double> xs_, std::vector<double> ys_, std::vector<double> zs_)
    {
        if ((int)xs_.size() < Nx + 1 || (int)ys_.size() < Ny + 1 || (int)zs_.size() < Nz + 1)
            throw py::value_error("face coordinate arrays are too short");
        xs = std::move(xs_); ys = std::move(ys_); zs = std::move(zs_);
        for (int i = 0; i < Nx; i++) dxv[i] = xs[i + 1] - xs[i];
        for (int j = 0; j < Ny; j++) dyv[j] = ys[j + 1] - ys[j];
        for (int k = 0; k < Nz; k++) dzv[k] = zs[k + 1] - zs[k];
        geom_gen++;
    }
    // Grid::zero_velocity / zero_pressure (Grid.cpp:49-58).
    void zero_velocity()
    {
        for (int f = 0; f < 3; f++) {
            std::fill(field(f).begin(), field(f).end(), 0.0);
            host_valid[f] = true;
            host_written(f);
        }
    }
    void zero_pressure()
    {
        std::fill(p.begin(), p.end(), 0.0);
        host_valid[3] = true;
        host_written(3);
    }
};

struct FanBC {
    int i_min = 0, i_max = 0, j_min = 0, j_max = 0, k_min = 0, k_max = 0;
    std::array<double, 3> vel{{0.0, 0.0, 0.0}};
};
struct OutflowBC {
    int axis = 0, side = 0, a_min = 0, a_max = 0, b_min = 0, b_max = 0;
};
struct OpeningBC : OutflowBC {
    double T_outside = 20.0;
};
struct HeatPatch {
    int i_min, i_max, j_min, j_max, k_min, k_max;
    double T;
};

// BoundaryManager (BoundaryManager.hpp:31-72).  The mask writers change the
// Grid's host cell_type; the per-step appliers run on the host copy of the
// fields (the solvers apply the same rules on the device inside a step).
struct BoundaryManager {
    std::vector<FanBC> fans;
    std::vector<ffr_patch> patches;      // outflows_ incl. openings, in order
    std::vector<OpeningBC> openings;
    std::vector<HeatPatch> heats;
    unsigned long long gen = 0;

    static int c_idx(const Grid &g, int i, int j, int k) { return (i * g.Ny + j) * g.Nz + k; }

    void add_solid_box(Grid &g, int i0, int i1, int j0, int j1, int k0, int k1)
    {
        for (int i = std::max(0, i0); i <= std::min(g.Nx - 1, i1); i++)
            for (int j = std::max(0, j0); j <= std::min(g.Ny - 1, j1); j++)
                for (int k = std::max(0, k0); k <= std::min(g.Nz - 1, k1); k++)
                    g.cell_type[c_idx(g, i, j, k)] = (uint8_t)CellType::SOLID;
        g.mask_gen++;
    }
    void add_fan(Grid &g, const FanBC &f)
    {
        fans.push_back(f);
        for (int i = std::max(0, f.i_min); i <= std::min(g.Nx - 1, f.i_max); i++)
            for (int j = std::max(0, f.j_min); j <= std::min(g.Ny - 1, f.j_max); j++)
                for (int k = std::max(0, f.k_min); k <= std::min(g.Nz - 1, f.k_max); k++)
                    g.cell_type[c_idx(g, i, j, k)] = (uint8_t)CellType::INFLOW;
        g.mask_gen++;
        gen++;
    }
    void mark_patch(Grid &g, const OutflowBC &o)
    {
        const int N[3] = {g.Nx, g.Ny, g.Nz};
        const int la = o.axis == 0 ? g.Ny : g.Nx, lb = o.axis == 2 ? g.Ny : g.Nz;
        if (o.axis < 0 || o.axis > 2 || o.a_min < 0 || o.b_min < 0 || o.a_max >= la || o.b_max >= lb)
            throw py::value_error("outflow patch outside the grid");
        const int wall = o.side == 0 ? 0 : N[o.axis] - 1;
        for (int a = o.a_min; a <= o.a_max; a++)
            for (int b = o.b_min; b <= o.b_max; b++) {
                int c = o.axis == 0 ? c_idx(g, wall, a, b)
                      : o.axis == 1 ? c_idx(g, a, wall, b) : c_idx(g, a, b, wall);
                g.cell_type[c] = (uint8_t)CellType::OUTFLOW;
            }
        g.mask_gen++;
        gen++;
    }
    void add_outflow(Grid &g, const OutflowBC &o)
    {
        mark_patch(g, o);
        patches.push_back(ffr_patch{o.axis, o.side, o.a_min, o.a_max, o.b_min, o.b_max, 0, 0.0});
    }
    void add_opening(Grid &g, const OpeningBC &o)
    {
        mark_patch(g, o);
        openings.push_back(o);
        patches.push_back(ffr_patch{o.axis, o.side, o.a_min, o.a_max, o.b_min, o.b_max, 1, o.T_outside});
    }
    void add_heat_patch(Grid &, int i0, int i1, int j0, int j1, int k0, int k1, double T)
    {
        heats.push_back(HeatPatch{i0, i1, j0, j1, k0, k1, T});
        gen++;
    }

    // BoundaryManager::apply_noslip (BoundaryManager.cpp:60-109).
    void apply_noslip(Grid &g)
    {
        for (int f = 0; f < 3; f++) g.ensure_host(f);
        const int nx = g.Nx, ny = g.Ny, nz = g.Nz;
        auto out = [&](int i, int j, int k) { return g.cell_type[c_idx(g, i, j, k)] == (uint8_t)CellType::OUTFLOW; };
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                if (!out(0, j, k)) g.u[(size_t)(0 * ny + j) * nz + k] = 0.0;
                if (!out(nx - 1, j, k)) g.u[(size_t)(nx * ny + j) * nz + k] = 0.0;
            }
        for (int i = 0; i < nx; i++)
            for (int k = 0; k < nz; k++) {
                if (!out(i, 0, k)) g.v[(size_t)(i * (ny + 1) + 0) * nz + k] = 0.0;
                if (!out(i, ny - 1, k)) g.v[(size_t)(i * (ny + 1) + ny) * nz + k] = 0.0;
            }
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) {
                if (!out(i, j, 0)) g.w[(size_t)(i * ny + j) * (nz + 1) + 0] = 0.0;
                if (!out(i, j, nz - 1)) g.w[(size_t)(i * ny + j) * (nz + 1) + nz] = 0.0;
            }
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++)
                for (int k = 0; k < nz; k++) {
                    if (g.cell_type[c_idx(g, i, j, k)] != (uint8_t)CellType::SOLID) continue;
                    g.u[(size_t)(i * ny + j) * nz + k] = 0.0;
                    g.u[(size_t)((i + 1) * ny + j) * nz + k] = 0.0;
                    g.v[(size_t)(i * (ny + 1) + j) * nz + k] = 0.0;
                    g.v[(size_t)(i * (ny + 1) + j + 1) * nz + k] = 0.0;
                    g.w[(size_t)(i * ny + j) * (nz + 1) + k] = 0.0;
                    g.w[(size_t)(i * ny + j) * (nz + 1) + k + 1] = 0.0;
                }
        for (int f = 0; f < 3; f++) g.host_written(f);
    }
    // BoundaryManager::apply_inflow (BoundaryManager.cpp:111-130).
    void apply_inflow(Grid &g)
    {
        for (int f = 0; f < 3; f++) g.ensure_host(f);
        const int ny = g.Ny, nz = g.Nz;
        for (const FanBC &f : fans)
            for (int i = std::max(0, f.i_min); i <= std::min(g.Nx - 1, f.i_max); i++)
                for (int j = std::max(0, f.j_min); j <= std::min(g.Ny - 1, f.j_max); j++)
                    for (int k = std::max(0, f.k_min); k <= std::min(g.Nz - 1, f.k_max); k++) {
                        if (f.vel[0] != 0.0) {
                            g.u[(size_t)(i * ny + j) * nz + k] = f.vel[0];
                            g.u[(size_t)((i + 1) * ny + j) * nz + k] = f.vel[0];
                        }
                        if (f.vel[1] != 0.0) {
                            g.v[(size_t)(i * (ny + 1) + j) * nz + k] = f.vel[1];
                            g.v[(size_t)(i * (ny + 1) + j + 1) * nz + k] = f.vel[1];
                        }
                        if (f.vel[2] != 0.0) {
                            g.w[(size_t)(i * ny + j) * (nz + 1) + k] = f.vel[2];
                            g.w[(size_t)(i * ny + j) * (nz + 1) + k + 1] = f.vel[2];
                        }
                    }
        for (int f = 0; f < 3; f++) g.host_written(f);
    }
    // BoundaryManager::apply_outflow (BoundaryManager.cpp:180-220).
    void apply_outflow(Grid &g)
    {
        for (int f = 0; f < 3; f++) g.ensure_host(f);
        const int nx = g.Nx, ny = g.Ny, nz = g.Nz;
        for (const ffr_patch &o : patches)
            for (int a = o.a_min; a <= o.a_max; a++)
                for (int b = o.b_min; b <= o.b_max; b++) {
                    if (o.axis == 0) {
                        if (o.side) g.u[(size_t)(nx * ny + a) * nz + b] = g.u[(size_t)((nx - 1) * ny + a) * nz + b];
                        else g.u[(size_t)a * nz + b] = g.u[(size_t)(ny + a) * nz + b];
                    } else if (o.axis == 1) {
                        if (o.side) g.v[(size_t)(a * (ny + 1) + ny) * nz + b] = g.v[(size_t)(a * (ny + 1) + ny - 1) * nz + b];
                        else g.v[(size_t)(a * (ny + 1)) * nz + b] = g.v[(size_t)(a * (ny + 1) + 1) * nz + b];
                    } else {
                        if (o.side) g.w[(size_t)(a * ny + b) * (nz + 1) + nz] = g.w[(size_t)(a * ny + b) * (nz + 1) + nz - 1];
                        else g.w[(size_t)(a * ny + b) * (nz + 1)] = g.w[(size_t)(a * ny + b) * (nz + 1) + 1];
                    }
                }
        for (int f = 0; f < 3; f++) g.host_written(f);
    }
    // BoundaryManager::apply_opening_temperature (BoundaryManager.cpp:137-178).
    void apply_opening_temperature(Grid &g)
    {
        g.ensure_host_all();
        const int nx = g.Nx, ny = g.Ny, nz = g.Nz;
        for (const OpeningBC &o : openings) {
            const int sd = o.side;
            for (int a = o.a_min; a <= o.a_max; a++)
                for (int b = o.b_min; b <= o.b_max; b++) {
                    double vf;
                    int cw, cin;
                    if (o.axis == 0) {
                        vf = g.u[(size_t)((sd ? nx : 0) * ny + a) * nz + b];
                        cw = c_idx(g, sd ? nx - 1 : 0, a, b); cin = c_idx(g, sd ? nx - 2 : 1, a, b);
                    } else if (o.axis == 1) {
                        vf = g.v[(size_t)(a * (ny + 1) + (sd ? ny : 0)) * nz + b];
                        cw = c_idx(g, a, sd ? ny - 1 : 0, b); cin = c_idx(g, a, sd ? ny - 2 : 1, b);
                    } else {
                        vf = g.w[(size_t)(a * ny + b) * (nz + 1) + (sd ? nz : 0)];
                        cw = c_idx(g, a, b, sd ? nz - 1 : 0); cin = c_idx(g, a, b, sd ? nz - 2 : 1);
                    }
                    const bool in = sd ? (vf <= 0.0) : (vf >= 0.0);
                    g.T[cw] = in ? o.T_outside : g.T[cin];
                }
        }
        g.host_written(4);
    }
};

struct PoissonSolverParams {
    int max_iter = 1000;
    double tol = 1e-6;
};

// FluidSolverParams (FluidSolver.hpp:11-38) + precision / poisson_method.
struct FluidSolverParams {
    double rho = 1.2, nu = 1.5e-5, dt = 0.01;
    int max_steps = 500;
    double convergence_tol = 1.0;
    PoissonSolverParams poisson;
    AdvectionScheme advection = AdvectionScheme::UPWIND1;
    bool use_openmp = false;
    bool use_multigrid = false;
    bool thermal = false;
    double T_initial = 20.0, T_target = 1e30;
    bool buoyancy = false;
    double g_accel = 9.81, beta = 1.0 / 293.0, k_thermal = 0.026, cp = 1005.0;
    std::string precision = "fp64";
    std::string poisson_method = "cg";
};

struct StepResult {
    int step = 0;
    double velocity_change = 0.0, pressure_residual = 0.0, divergence_max = 0.0;
    bool converged = false;
    double T_mean = 0.0;
    int cg_iterations = 0;
    int flags = 0;
};

StepResult from_abi(const ffr_step_result &r, int offset)
{
    StepResult s;
    s.step = r.step + offset;
    s.velocity_change = r.velocity_change;
    s.pressure_residual = r.pressure_residual;
    s.divergence_max = r.divergence_max;
    s.converged = r.converged != 0;
    s.T_mean = r.T_mean;
    s.cg_iterations = r.cg_iterations;
    s.flags = r.flags;
    return s;
}

Grid::~Grid() = default;

// Shared plumbing of the two solvers: owning the Grid's fields on the device.
struct DeviceSolver : FieldOwner {
    Grid &grid;
    BoundaryManager &bm;
    unsigned long long seen_geom = ~0ull, seen_mask = ~0ull, seen_bm = ~0ull;
    int step_offset = 0;
    std::vector<int> fields;   // fields this solver owns on the device

    DeviceSolver(Grid &g, BoundaryManager &b, std::vector<int> f) : grid(g), bm(b), fields(std::move(f)) {}

    ffr_room_desc desc(std::vector<ffr_fan> &fans, std::vector<ffr_heat_patch> &heats)
    {
        fans.clear();
        for (const FanBC &f : bm.fans)
            fans.push_back(ffr_fan{f.i_min, f.i_max, f.j_min, f.j_max, f.k_min, f.k_max,
                                   {f.vel[0], f.vel[1], f.vel[2]}});
        heats.clear();
        for (const HeatPatch &h : bm.heats)
            heats.push_back(ffr_heat_patch{h.i_min, h.i_max, h.j_min, h.j_max, h.k_min, h.k_max, h.T});
        ffr_room_desc d{};
        d.nx = grid.Nx; d.ny = grid.Ny; d.nz = grid.Nz;
        d.lx = grid.dx * grid.Nx; d.ly = grid.dy * grid.Ny; d.lz = grid.dz * grid.Nz;
        d.dxv = grid.dxv.data(); d.dyv = grid.dyv.data(); d.dzv = grid.dzv.data();
        d.cell_type = grid.cell_type.data();
        d.nfans = (int)fans.size(); d.fans = fans.data();
        d.npatches = (int)bm.patches.size(); d.patches = bm.patches.data();
        d.nheat = (int)heats.size(); d.heats = heats.data();
        return d;
    }
    bool stale() const
    {
        return seen_geom != grid.geom_gen || seen_mask != grid.mask_gen || seen_bm != bm.gen;
    }
    void mark_seen()
    {
        seen_geom = grid.geom_gen; seen_mask = grid.mask_gen; seen_bm = bm.gen;
    }
    // Takes the Grid's fields onto this solver's device state.
    void acquire()
    {
        if (grid.owner != this) {
            if (grid.owner) grid.ensure_host_all();
            grid.owner = this;
            for (int f : fields) grid.dev_valid[f] = false;
        }
        if (stale()) rebuild();
        for (int f : fields)
            if (!grid.dev_valid[f] || grid.views[f] > 0) {
                push(f, grid.field(f).data());
                grid.dev_valid[f] = true;
            }
    }
    // After device work: host copies are stale, live views are refreshed.
    void release_after_step()
    {
        for (int f : fields) {
            grid.host_valid[f] = false;
            if (grid.views[f] > 0) grid.ensure_host(f);
        }
    }
    virtual void rebuild() = 0;
    void detach()
    {
        if (grid.owner == this) {
            grid.ensure_host_all();
            grid.owner = nullptr;
        }
    }
};

struct FluidSolver : DeviceSolver {
    FluidSolverParams params;
    ffr_fluid *h = nullptr;

    ffr_fluid_params abi_params() const
    {
        ffr_fluid_params p{};
        p.rho = params.rho; p.nu = params.nu; p.dt = params.dt;
        p.max_steps = params.max_steps; p.convergence_tol = params.convergence_tol;
        p.poisson_max_iter = params.poisson.max_iter; p.poisson_tol = params.poisson.tol;
        p.advection = (int)params.advection;
        p.use_multigrid = params.use_multigrid ? 1 : 0;
        p.thermal = params.thermal ? 1 : 0;
        p.T_initial = params.T_initial; p.T_target = params.T_target;
        p.buoyancy = params.buoyancy ? 1 : 0;
        p.g_accel = params.g_accel; p.beta = params.beta; p.k_thermal = params.k_thermal; p.cp = params.cp;
        p.precision = params.precision == "mixed" ? FFR_PREC_MIXED : FFR_PREC_FP64;
        p.poisson = (params.use_multigrid || params.poisson_method == "mgpcg") ? FFR_POISSON_MGPCG : FFR_POISSON_CG;
        return p;
    }

    // FluidSolver::FluidSolver (FluidSolver.cpp:18-32).
    FluidSolver(Grid &g, BoundaryManager &b, FluidSolverParams p)
        : DeviceSolver(g, b, {0, 1, 2, 3, 4}), params(std::move(p))
    {
        if (grid.owner) grid.ensure_host_all();
        for (int f = 0; f < 3; f++) grid.ensure_host(f);
        std::vector<ffr_fan> fans;
        std::vector<ffr_heat_patch> heats;
        ffr_room_desc d = desc(fans, heats);
        ffr_fluid_params ap = abi_params();
        ffr_fields init{grid.u.data(), grid.v.data(), grid.w.data(), grid.p.data()};
        check(ffr_fluid_create(&d, &ap, &init, &h));
        mark_seen();
        if (grid.owner && grid.owner != this) grid.owner = nullptr;
        grid.owner = this;
        for (int f = 0; f < kFields; f++) grid.dev_valid[f] = true;
        grid.host_valid[4] = false;   // T was filled on the device
    }
    ~FluidSolver() override
    {
        try { detach(); } catch (...) {}
        if (h) ffr_fluid_destroy(h);
    }
    void pull(int f, double *host) override { check(ffr_fluid_get_field(h, f, host)); }
    void push(int f, const double *host) override { check(ffr_fluid_set_field(h, f, host)); }

    void rebuild() override
    {
        int cur = 0;
        check(ffr_fluid_current_step(h, &cur));
        grid.ensure_host_all();
        ffr_fluid_destroy(h);
        h = nullptr;
        std::vector<ffr_fan> fans;
        std::vector<ffr_heat_patch> heats;
        ffr_room_desc d = desc(fans, heats);
        ffr_fluid_params ap = abi_params();
        ffr_fields init{grid.u.data(), grid.v.data(), grid.w.data(), grid.p.data()};
        check(ffr_fluid_create(&d, &ap, &init, &h));
        step_offset += cur;
        for (int f : fields) grid.dev_valid[f] = false;   // T must come from the host, not the ctor fill
        mark_seen();
    }

    StepResult step()
    {
        acquire();
        ffr_step_result r{};
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = ffr_fluid_step(h, &r);
        }
        check(rc);
        release_after_step();
        return from_abi(r, step_offset);
    }

    // FluidSolver::run (FluidSolver.cpp:552-560).  Without a callback the
    // whole run is queued on the device and stops there on convergence.
    StepResult run(py::object callback)
    {
        StepResult last;
        if (callback.is_none()) {
            acquire();
            std::vector<ffr_step_result> res(std::max(1, params.max_steps));
            int done = 0, rc;
            {
                py::gil_scoped_release nogil;
                rc = ffr_fluid_advance(h, params.max_steps, 1, res.data(), &done);
            }
            check(rc);
            release_after_step();
            if (done > 0) last = from_abi(res[done - 1], step_offset);
            return last;
        }
        for (int s = 0; s < params.max_steps; s++) {
            last = step();
            callback(last);
            if (last.converged) break;
        }
        return last;
    }

    double compute_divergence_max()
    {
        acquire();
        double d = 0.0;
        check(ffr_fluid_divergence_max(h, &d));
        return d;
    }

    // The cell-centred velocity and speed of SolverBridge.run_animated's
    // snapshots (python/ff_room/solver_bridge.py:222-238), formed on the
    // device: {"speed": (Nx, Ny, Nz), "vel": (Nx, Ny, Nz, 3)}.  No
    // counterpart in the reference module; run_animated may call it in place
    // of reading the three face arrays back (the fields stay on the GPU).
    py::dict snapshot()
    {
        acquire();
        const size_t n = (size_t)grid.Nx * grid.Ny * grid.Nz;
        std::vector<double> uc(n), vc(n), wc(n);
        py::array_t<double> speed({(py::ssize_t)grid.Nx, (py::ssize_t)grid.Ny, (py::ssize_t)grid.Nz});
        py::array_t<double> vel({(py::ssize_t)grid.Nx, (py::ssize_t)grid.Ny, (py::ssize_t)grid.Nz, (py::ssize_t)3});
        double *sp = speed.mutable_data();
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = ffr_fluid_snapshot(h, uc.data(), vc.data(), wc.data(), sp);
        }
        check(rc);
        double *vp = vel.mutable_data();
        for (size_t c = 0; c < n; c++) {
            vp[3 * c] = uc[c];
            vp[3 * c + 1] = vc[c];
            vp[3 * c + 2] = wc[c];
        }
        py::dict d;
        d["speed"] = speed;
        d["vel"] = vel;
        return d;
    }
    int current_step()
    {
        int c = 0;
        check(ffr_fluid_current_step(h, &c));
        return c + step_offset;
    }
};

struct LBMSolver : DeviceSolver {
    double tau, tol, dt;
    int max_steps;
    int storage;
    ffr_lbm *h = nullptr;

    // LBMSolver::LBMSolver (LBMSolver.cpp:33-59).
    LBMSolver(Grid &g, BoundaryManager &b, double tau_, int max_steps_, double tol_, double dt_,
              const std::string &storage_)
        : DeviceSolver(g, b, {0, 1, 2, 3}), tau(tau_), tol(tol_), dt(dt_), max_steps(max_steps_)
    {
        storage = storage_ == "fp32" ? FFR_LBM_FP32 : storage_ == "fp16" ? FFR_LBM_FP16 : FFR_LBM_FP64;
        create();
    }
    void create()
    {
        grid.ensure_host_all();
        std::vector<ffr_fan> fans;
        std::vector<ffr_heat_patch> heats;
        ffr_room_desc d = desc(fans, heats);
        ffr_fields init{grid.u.data(), grid.v.data(), grid.w.data(), grid.p.data()};
        check(ffr_lbm_create(&d, tau, max_steps, tol, dt, storage, &init, &h));
        mark_seen();
        grid.owner = this;
        for (int f : fields) grid.dev_valid[f] = true;
    }
    ~LBMSolver() override
    {
        try { detach(); } catch (...) {}
        if (h) ffr_lbm_destroy(h);
    }
    // T is not an LBM field: the host copy stays authoritative.
    void pull(int f, double *host) override
    {
        if (f < 4) check(ffr_lbm_get_field(h, f, host));
    }
    void push(int f, const double *host) override
    {
        if (f < 4) check(ffr_lbm_set_field(h, f, host));
    }
    void rebuild() override
    {
        // The reference LBM re-reads the masks and lists each step; the
        // populations here are tied to the mask they were built with, so a
        // change restarts from the Grid's current fields.
        int cur = 0;
        check(ffr_lbm_current_step(h, &cur));
        grid.ensure_host_all();
        ffr_lbm_destroy(h);
        h = nullptr;
        step_offset += cur;
        create();
    }
    StepResult step()
    {
        acquire();
        ffr_step_result r{};
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = ffr_lbm_step(h, &r);
        }
        check(rc);
        release_after_step();
        return from_abi(r, step_offset);
    }
    StepResult run(py::object callback)
    {
        StepResult last;
        if (callback.is_none()) {
            acquire();
            std::vector<ffr_step_result> res(std::max(1, max_steps));
            int done = 0, rc;
            {
                py::gil_scoped_release nogil;
                rc = ffr_lbm_advance(h, max_steps, 1, res.data(), &done);
            }
            check(rc);
            release_after_step();
            if (done > 0) last = from_abi(res[done - 1], step_offset);
            return last;
        }
        for (int s = 0; s < max_steps; s++) {
            last = step();
            callback(last);
            if (last.converged) break;
        }
        return last;
    }
    double compute_divergence_max()
    {
        acquire();
        double d = 0.0;
        check(ffr_lbm_divergence_max(h, &d));
        return d;
    }
    int current_step()
    {
        int c = 0;
        check(ffr_lbm_current_step(h, &c));
        return c + step_offset;
    }
};

// A numpy view aliasing one Grid field.  Its base capsule keeps the Grid
// alive (as the reference's base=Grid does) and counts the view, so that the
// owning solver keeps the field in sync while the view exists.
py::array field_view(Grid &g, int f, std::vector<py::ssize_t> shape)
{
    g.ensure_host(f);
    g.views[f]++;
    g.host_written(f);
    struct Hold {
        py::object grid;
        Grid *g;
        int f;
    };
    Hold *hold = new Hold{py::cast(&g, py::return_value_policy::reference), &g, f};
    py::capsule cap(hold, [](void *p) {
        Hold *h = static_cast<Hold *>(p);
        h->g->views[h->f]--;
        delete h;
    });
    return py::array_t<double>(shape, g.field(f).data(), cap);
}

}  // namespace b200

PYBIND11_MODULE(_ffroom_core, m)
{
    using namespace b200;
    m.doc() = "ff-room CFD core (projection method on MAC grid) — B200 sm_100a backend";
    m.attr("__backend__") = py::str(std::string("b200 ") + ffr_version());

    py::enum_<AdvectionScheme>(m, "AdvectionScheme")
        .value("UPWIND1", AdvectionScheme::UPWIND1)
        .value("QUICK", AdvectionScheme::QUICK)
        .value("LAX_WENDROFF", AdvectionScheme::LAX_WENDROFF)
        .export_values();

    py::enum_<CellType>(m, "CellType")
        .value("FLUID", CellType::FLUID)
        .value("SOLID", CellType::SOLID)
        .value("INFLOW", CellType::INFLOW)
        .value("OUTFLOW", CellType::OUTFLOW)
        .export_values();

    py::class_<Grid>(m, "Grid")
        .def(py::init<int, int, int, double, double, double>(), py::arg("nx"), py::arg("ny"), py::arg("nz"),
             py::arg("lx"), py::arg("ly"), py::arg("lz"))
        .def_readonly("Nx", &Grid::Nx)
        .def_readonly("Ny", &Grid::Ny)
        .def_readonly("Nz", &Grid::Nz)
        .def_readonly("dx", &Grid::dx)
        .def_readonly("dy", &Grid::dy)
        .def_readonly("dz", &Grid::dz)
        .def_property_readonly("u", [](Grid &g) { return field_view(g, 0, {(py::ssize_t)g.u.size()}); })
        .def_property_readonly("v", [](Grid &g) { return field_view(g, 1, {(py::ssize_t)g.v.size()}); })
        .def_property_readonly("w", [](Grid &g) { return field_view(g, 2, {(py::ssize_t)g.w.size()}); })
        .def_property_readonly("p", [](Grid &g) { return field_view(g, 3, {(py::ssize_t)g.p.size()}); })
        .def("u_shaped", [](Grid &g) { return field_view(g, 0, {g.Nx + 1, g.Ny, g.Nz}); })
        .def("v_shaped", [](Grid &g) { return field_view(g, 1, {g.Nx, g.Ny + 1, g.Nz}); })
        .def("w_shaped", [](Grid &g) { return field_view(g, 2, {g.Nx, g.Ny, g.Nz + 1}); })
        .def("p_shaped", [](Grid &g) { return field_view(g, 3, {g.Nx, g.Ny, g.Nz}); })
        .def("T_shaped", [](Grid &g) { return field_view(g, 4, {g.Nx, g.Ny, g.Nz}); })
        .def("cell_type_shaped", [](Grid &g) {
            auto arr = py::array_t<uint8_t>({g.Nx, g.Ny, g.Nz});
            std::memcpy(arr.mutable_data(), g.cell_type.data(), g.cell_type.size());
            return arr;
        })
        .def("xs", [](Grid &g) { return py::array_t<double>({g.Nx + 1}, g.xs.data(), py::cast(&g, py::return_value_policy::reference)); })
        .def("ys", [](Grid &g) { return py::array_t<double>({g.Ny + 1}, g.ys.data(), py::cast(&g, py::return_value_policy::reference)); })
        .def("zs", [](Grid &g) { return py::array_t<double>({g.Nz + 1}, g.zs.data(), py::cast(&g, py::return_value_policy::reference)); })
        .def("set_face_coords", &Grid::set_face_coords, py::arg("xs"), py::arg("ys"), py::arg("zs"))
        .def("zero_velocity", &Grid::zero_velocity)
        .def("zero_pressure", &Grid::zero_pressure);

    py::class_<FanBC>(m, "FanBC")
        .def(py::init<>())
        .def_readwrite("i_min", &FanBC::i_min)
        .def_readwrite("i_max", &FanBC::i_max)
        .def_readwrite("j_min", &FanBC::j_min)
        .def_readwrite("j_max", &FanBC::j_max)
        .def_readwrite("k_min", &FanBC::k_min)
        .def_readwrite("k_max", &FanBC::k_max)
        .def_readwrite("vel", &FanBC::vel);

    py::class_<OutflowBC>(m, "OutflowBC")
        .def(py::init<>())
        .def_readwrite("axis", &OutflowBC::axis)
        .def_readwrite("side", &OutflowBC::side)
        .def_readwrite("a_min", &OutflowBC::a_min)
        .def_readwrite("a_max", &OutflowBC::a_max)
        .def_readwrite("b_min", &OutflowBC::b_min)
        .def_readwrite("b_max", &OutflowBC::b_max);

    py::class_<OpeningBC, OutflowBC>(m, "OpeningBC")
        .def(py::init<>())
        .def_readwrite("axis", &OpeningBC::axis)
        .def_readwrite("side", &OpeningBC::side)
        .def_readwrite("a_min", &OpeningBC::a_min)
        .def_readwrite("a_max", &OpeningBC::a_max)
        .def_readwrite("b_min", &OpeningBC::b_min)
        .def_readwrite("b_max", &OpeningBC::b_max)
        .def_readwrite("T_outside", &OpeningBC::T_outside);

    py::class_<BoundaryManager>(m, "BoundaryManager")
        .def(py::init<>())
        .def("add_solid_box", &BoundaryManager::add_solid_box)
        .def("add_fan", &BoundaryManager::add_fan)
        .def("add_outflow", &BoundaryManager::add_outflow)
        .def("add_opening", &BoundaryManager::add_opening)
        .def("add_heat_patch", &BoundaryManager::add_heat_patch)
        .def("apply_noslip", &BoundaryManager::apply_noslip)
        .def("apply_inflow", &BoundaryManager::apply_inflow)
        .def("apply_outflow", &BoundaryManager::apply_outflow)
        .def("apply_opening_temperature", &BoundaryManager::apply_opening_temperature);

    py::class_<PoissonSolverParams>(m, "PoissonSolverParams")
        .def(py::init<>())
        .def_readwrite("max_iter", &PoissonSolverParams::max_iter)
        .def_readwrite("tol", &PoissonSolverParams::tol);

    py::class_<FluidSolverParams>(m, "FluidSolverParams")
        .def(py::init<>())
        .def_readwrite("rho", &FluidSolverParams::rho)
        .def_readwrite("nu", &FluidSolverParams::nu)
        .def_readwrite("dt", &FluidSolverParams::dt)
        .def_readwrite("max_steps", &FluidSolverParams::max_steps)
        .def_readwrite("convergence_tol", &FluidSolverParams::convergence_tol)
        .def_readwrite("poisson", &FluidSolverParams::poisson)
        .def_readwrite("advection", &FluidSolverParams::advection)
        .def_readwrite("use_openmp", &FluidSolverParams::use_openmp)
        .def_readwrite("use_multigrid", &FluidSolverParams::use_multigrid)
        .def_readwrite("thermal", &FluidSolverParams::thermal)
        .def_readwrite("T_initial", &FluidSolverParams::T_initial)
        .def_readwrite("T_target", &FluidSolverParams::T_target)
        .def_readwrite("buoyancy", &FluidSolverParams::buoyancy)
        .def_readwrite("g_accel", &FluidSolverParams::g_accel)
        .def_readwrite("beta", &FluidSolverParams::beta)
        .def_readwrite("k_thermal", &FluidSolverParams::k_thermal)
        .def_readwrite("cp", &FluidSolverParams::cp)
        .def_readwrite("precision", &FluidSolverParams::precision)
        .def_readwrite("poisson_method", &FluidSolverParams::poisson_method);

    py::class_<StepResult>(m, "StepResult")
        .def_readonly("step", &StepResult::step)
        .def_readonly("velocity_change", &StepResult::velocity_change)
        .def_readonly("pressure_residual", &StepResult::pressure_residual)
        .def_readonly("divergence_max", &StepResult::divergence_max)
        .def_readonly("converged", &StepResult::converged)
        .def_readonly("T_mean", &StepResult::T_mean)
        .def_readonly("cg_iterations", &StepResult::cg_iterations)
        .def_readonly("flags", &StepResult::flags)
        .def("__repr__", [](const StepResult &r) {
            return "StepResult(step=" + std::to_string(r.step) + ", vel_change=" + std::to_string(r.velocity_change) +
                   ", p_res=" + std::to_string(r.pressure_residual) + ", div_max=" + std::to_string(r.divergence_max) +
                   ", T_mean=" + std::to_string(r.T_mean) + ", converged=" + (r.converged ? "True" : "False") + ")";
        });

    py::class_<FluidSolver>(m, "FluidSolver")
        .def(py::init<Grid &, BoundaryManager &, FluidSolverParams>(), py::arg("grid"), py::arg("bm"),
             py::arg("params") = FluidSolverParams{}, py::keep_alive<1, 2>(), py::keep_alive<1, 3>())
        .def("step", &FluidSolver::step)
        .def("run", &FluidSolver::run, py::arg("callback") = py::none())
        .def("compute_divergence_max", &FluidSolver::compute_divergence_max)
        .def("snapshot", &FluidSolver::snapshot)
        .def_property_readonly("current_step", &FluidSolver::current_step);

    py::class_<LBMSolver>(m, "LBMSolver")
        .def(py::init<Grid &, BoundaryManager &, double, int, double, double, const std::string &>(),
             py::arg("grid"), py::arg("bm"), py::arg("tau"), py::arg("max_steps"), py::arg("convergence_tol"),
             py::arg("dt") = 0.01, py::arg("storage") = "fp64", py::keep_alive<1, 2>(), py::keep_alive<1, 3>())
        .def("step", &LBMSolver::step)
        .def("run", &LBMSolver::run, py::arg("callback") = py::none())
        .def("compute_divergence_max", &LBMSolver::compute_divergence_max)
        .def_property_readonly("current_step", &LBMSolver::current_step);
}
