"""The allocation-free pressure solve (ffr_poisson_solve_noalloc).

It exists for callers that cannot allocate device memory at solve time;
here it must give the same pressure as the allocating entry point
(ffr_poisson_solve_dev) within the tolerance the other pressure tests use
(same iteration count, solution within 1e-9 max-norm relative), on two
calls in a row, so that what the shared scratch keeps from one call cannot
leak into the next.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from conftest import Golden, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1_upwind_10", "edge_odd_quick_10", "summer_cooling_10",
                                  "oblique_stretch_10"])
def test_noalloc_matches_allocating_solve(name):
    import torch
    from ffrb import capi
    g = Golden(name)
    stream = torch.cuda.current_stream().cuda_stream
    ct = torch.tensor(g.room.cell_type, device="cuda", dtype=torch.uint8)
    h = capi.PoissonHandle(g.room, 3000, 1e-8)
    rng = np.random.default_rng(7)
    for call in range(2):
        rhs = rng.standard_normal(g.room.n_cells)
        rhs[g.room.cell_type == 1] = 0.0
        b = torch.tensor(rhs, device="cuda", dtype=torch.float64)
        x_ref = torch.empty_like(b)
        x_na = torch.full_like(b, float("nan"))
        res_ref, it_ref = h.solve_dev(b.data_ptr(), x_ref.data_ptr(), stream)
        res_na, it_na = capi.poisson_solve_noalloc(g.room, ct.data_ptr(), b.data_ptr(), x_na.data_ptr(),
                                                   3000, 1e-8, stream)
        torch.cuda.synchronize()
        assert it_na == it_ref, (call, it_na, it_ref)
        assert rel_err(x_na.cpu().numpy(), x_ref.cpu().numpy()) <= 1e-9
        assert abs(res_na - res_ref) <= 1e-9 * max(res_ref, 1e-30) + 1e-15
    h.close()


def test_noalloc_takes_no_device_memory():
    """A solve through the allocation-free entry point must not take device
    memory: after a first call (which may do its one-time set-up), a second
    call leaves the free device memory no lower and torch's pool unchanged.
    Every tensor is made before the first call."""
    import torch
    from ffrb import capi
    g = Golden("c1_upwind_10")
    stream = torch.cuda.current_stream().cuda_stream
    ct = torch.tensor(g.room.cell_type, device="cuda", dtype=torch.uint8)
    rhs = np.random.default_rng(3).standard_normal(g.room.n_cells)
    rhs[g.room.cell_type == 1] = 0.0
    b = torch.tensor(rhs, device="cuda", dtype=torch.float64)
    x = torch.zeros_like(b)
    capi.poisson_solve_noalloc(g.room, ct.data_ptr(), b.data_ptr(), x.data_ptr(), 3000, 1e-8, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0, allocated0 = torch.cuda.memory_reserved(), torch.cuda.memory_allocated()
    capi.poisson_solve_noalloc(g.room, ct.data_ptr(), b.data_ptr(), x.data_ptr(), 3000, 1e-8, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0, (free0, free1)
    assert torch.cuda.memory_reserved() == reserved0
    assert torch.cuda.memory_allocated() == allocated0


def test_noalloc_rejects_rooms_beyond_its_capacity():
    import torch
    from ffrb import capi
    from ffrb.scene import empty_room
    room = empty_room(128, 64, 64, 4.0, 2.0, 2.0)     # 524288 cells > 64^3
    buf = torch.zeros(8, device="cuda", dtype=torch.float64)
    ct = torch.zeros(8, device="cuda", dtype=torch.uint8)
    with pytest.raises(capi.FfrError) as e:
        capi.poisson_solve_noalloc(room, ct.data_ptr(), buf.data_ptr(), buf.data_ptr(), 10, 1e-8)
    assert e.value.status == capi.FFR_ERANGE
