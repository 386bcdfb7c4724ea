"""The pressure solve alone (ffr_poisson_*) against the oracle's CG
(PoissonSolver.cpp:93-158 restated) on seeded right-hand sides.
Tolerance: same iteration count; solution within 1e-9 max-norm relative."""
import numpy as np
import pytest

from conftest import Golden, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1_upwind_10", "edge_odd_quick_10", "summer_cooling_10",
                                  "oblique_stretch_10", "updraft_laxw_10"])
def test_poisson_matches_oracle(name, oracle):
    from ffrb import capi
    g = Golden(name)
    rng = np.random.default_rng(1)
    rhs = rng.standard_normal(g.room.n_cells)
    rhs[g.room.cell_type == 1] = 0.0
    h = capi.PoissonHandle(g.room, 3000, 1e-8)
    x, res, it = h.solve(rhs)
    xo, reso, ito = oracle.cg_solve(g.room, rhs, 3000, 1e-8)
    assert it == ito and rel_err(x, xo) <= 1e-9 and abs(res - reso) <= 1e-9 * max(reso, 1e-30) + 1e-12
    # the operator itself
    y = h.apply(rhs)
    assert rel_err(y, oracle.laplacian(g.room, rhs)) <= 1e-14


def test_poisson_edge_cases(oracle):
    from ffrb import capi
    from ffrb.scene import empty_room
    room = empty_room(5, 4, 3, 1.0, 1.0, 1.0)
    h = capi.PoissonHandle(room, 100, 1e-10)
    x, res, it = h.solve(np.zeros(room.n_cells))          # ||rhs|| < 1e-15: x = 0, no iteration
    assert it == 0 and res == 0.0 and not np.any(x)
    room.cell_type[:] = 1                                  # all SOLID: identity rows, r = 0
    h = capi.PoissonHandle(room, 100, 1e-10)
    x, res, it = h.solve(np.ones(room.n_cells))
    assert it == 0 and not np.any(x)
    room = empty_room(6, 5, 4, 1.0, 1.0, 1.0)
    h = capi.PoissonHandle(room, 3, 1e-14)                 # max_iter exhausted
    rhs = np.random.default_rng(2).standard_normal(room.n_cells)
    x, res, it = h.solve(rhs)
    xo, reso, ito = oracle.cg_solve(room, rhs, 3, 1e-14)
    assert it == ito == 3 and rel_err(x, xo) <= 1e-12 and abs(res - reso) <= 1e-12


def test_poisson_device_pointers(oracle):
    """ffr_poisson_solve_dev on torch-allocated device buffers."""
    import torch
    from ffrb import capi
    g = Golden("c1_upwind_10")
    rhs = np.random.default_rng(3).standard_normal(g.room.n_cells)
    b = torch.tensor(rhs, device="cuda", dtype=torch.float64)
    x = torch.empty_like(b)
    h = capi.PoissonHandle(g.room, 2000, 1e-8)
    res, it = h.solve_dev(b.data_ptr(), x.data_ptr(), torch.cuda.current_stream().cuda_stream)
    xo, reso, ito = oracle.cg_solve(g.room, rhs, 2000, 1e-8)
    assert it == ito and rel_err(x.cpu().numpy(), xo) <= 1e-9
