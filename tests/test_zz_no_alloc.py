"""pl_pcg_solve_device_noalloc against pl_pcg_solve_device, through the C ABI (needs a GPU).

Both run the same MIC(0) FP64 kernels in the same order; the allocation-free call only takes its
scratch from the library's fixed static device array. Tolerance: relative max difference 1e-12
of the solution (the two are expected to agree bit for bit), equal iteration counts and residuals.
"""
import numpy as np
import pytest

from teapotfluidsimulation_b200 import abi

pytestmark = pytest.mark.gpu

TOL = 1e-12


def free_surface_system(nx, ny, nz, seed):
    """A liquid pool in the lower part of a walled box, an air gap above it, and a random rhs."""
    rng = np.random.default_rng(seed)
    cell = np.full((nz, ny, nx), abi.SOLID, np.uint8)
    cell[1:-1, 1:-1, 1:-1] = abi.AIR
    level = max(2, (2 * (nz - 2)) // 3)
    cell[1:1 + level, 1:-1, 1:-1] = abi.FLUID
    cell = cell.reshape(-1)
    b = np.where(cell == abi.FLUID, rng.standard_normal(cell.size), 0.0)
    return cell, b


@pytest.mark.parametrize("shape", [(9, 7, 5), (40, 32, 24), (64, 64, 64)])
def test_noalloc_solve_matches_allocating_solve(engine, shape):
    import torch

    nx, ny, nz = shape
    assert nx * ny * nz <= engine.engine.NOALLOC_MAX_CELLS
    cell, b = free_surface_system(nx, ny, nz, seed=nx)
    dc = torch.tensor(cell, device="cuda")
    db = torch.tensor(b, device="cuda")
    q_ref = torch.zeros(cell.size, dtype=torch.float64, device="cuda")
    ref = engine.pcg_solve_device(dc.data_ptr(), db.data_ptr(), q_ref.data_ptr(), nx, ny, nz, 1e-10, 400)
    assert ref[1], ref
    want = q_ref.cpu().numpy()
    scale = max(np.abs(want).max(), 1e-300)
    for _ in range(2):  # two calls in a row reuse the same scratch
        q = torch.full((cell.size,), float("nan"), dtype=torch.float64, device="cuda")
        got = engine.pcg_solve_device_noalloc(dc.data_ptr(), db.data_ptr(), q.data_ptr(), nx, ny, nz, 1e-10, 400)
        assert got[0] == ref[0] and got[1] == ref[1]
        assert abs(got[2] - ref[2]) <= TOL * max(abs(ref[2]), 1e-300)
        qn = q.cpu().numpy()
        assert np.isfinite(qn).all()
        assert np.abs(qn - want).max() <= TOL * scale


def test_noalloc_solve_rejects_grids_beyond_its_scratch(engine):
    import torch

    nx, ny, nz = 65, 64, 64  # 266,240 cells > 262,144
    assert nx * ny * nz > engine.engine.NOALLOC_MAX_CELLS
    dc = torch.zeros(nx * ny * nz, dtype=torch.uint8, device="cuda")
    db = torch.zeros(nx * ny * nz, dtype=torch.float64, device="cuda")
    dq = torch.zeros_like(db)
    with pytest.raises(engine.EngineError, match="PL_NOALLOC_MAX_CELLS"):
        engine.pcg_solve_device_noalloc(dc.data_ptr(), db.data_ptr(), dq.data_ptr(), nx, ny, nz, 1e-10, 10)
    # the rejection launched nothing; a valid call right after still works
    cell, b = free_surface_system(9, 7, 5, seed=1)
    dc, db = torch.tensor(cell, device="cuda"), torch.tensor(b, device="cuda")
    dq = torch.zeros(cell.size, dtype=torch.float64, device="cuda")
    _, conv, _ = engine.pcg_solve_device_noalloc(dc.data_ptr(), db.data_ptr(), dq.data_ptr(), 9, 7, 5, 1e-10, 200)
    assert conv
