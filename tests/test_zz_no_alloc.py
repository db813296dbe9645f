"""pl_pcg_solve_device_noalloc against pl_pcg_solve_device, through the C ABI (needs a GPU).

The allocation-free entry point is for hosts that own all device memory and cannot let a library
call cudaMalloc. Both calls run the same MIC(0) FP64 kernels in the same order; the allocation-free
call only takes its scratch from the library's fixed static device array. Tolerance: relative max
difference 1e-12 of the solution (the two are expected to agree bit for bit), equal iteration
counts and residuals. This file is collected last, so a run that stops at the first failure has
run every other test before it; it also passes alone in a fresh process.
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


def solve_both(engine, nx, ny, nz, seed, tol=1e-10, max_iter=400):
    """One system solved by the allocating call and by the allocation-free call."""
    import torch

    cell, b = free_surface_system(nx, ny, nz, seed)
    dc, db = torch.tensor(cell, device="cuda"), torch.tensor(b, device="cuda")
    q_ref = torch.zeros(cell.size, dtype=torch.float64, device="cuda")
    ref = engine.pcg_solve_device(dc.data_ptr(), db.data_ptr(), q_ref.data_ptr(), nx, ny, nz, tol, max_iter)
    q = torch.full((cell.size,), float("nan"), dtype=torch.float64, device="cuda")
    got = engine.pcg_solve_device_noalloc(dc.data_ptr(), db.data_ptr(), q.data_ptr(), nx, ny, nz, tol, max_iter)
    return ref, q_ref.cpu().numpy(), got, q.cpu().numpy()


def test_small_call_after_a_large_call_matches(engine):
    # the scratch keeps the large call's contents; the small call that follows must not read any of it
    for shape, seed in (((64, 64, 64), 5), ((9, 7, 5), 6), ((40, 32, 24), 7), ((11, 9, 6), 8)):
        ref, want, got, qn = solve_both(engine, *shape, seed)
        assert ref[1] and got[0] == ref[0] and got[1] == ref[1], (shape, ref, got)
        assert abs(got[2] - ref[2]) <= TOL * max(abs(ref[2]), 1e-300)
        assert np.isfinite(qn).all()
        assert np.abs(qn - want).max() <= TOL * max(np.abs(want).max(), 1e-300), shape


def test_noalloc_solve_rejects_grids_beyond_its_scratch(engine):
    import torch

    nx, ny, nz = 65, 64, 64  # 266,240 cells > 262,144
    assert nx * ny * nz > engine.engine.NOALLOC_MAX_CELLS
    dc = torch.zeros(nx * ny * nz, dtype=torch.uint8, device="cuda")
    db = torch.zeros(nx * ny * nz, dtype=torch.float64, device="cuda")
    dq = torch.zeros_like(db)
    with pytest.raises(engine.EngineError, match="PL_NOALLOC_MAX_CELLS"):
        engine.pcg_solve_device_noalloc(dc.data_ptr(), db.data_ptr(), dq.data_ptr(), nx, ny, nz, 1e-10, 10)
    # the rejection launched nothing; a valid call right after still works and matches
    ref, want, got, qn = solve_both(engine, 9, 7, 5, seed=1)
    assert got[1] and got[0] == ref[0]
    assert np.abs(qn - want).max() <= TOL * max(np.abs(want).max(), 1e-300)
