"""Poisson batch on the GPU against the FP64 oracle (Pcg3D.solve, src/sim3d/solver3d.ts:858-973).

MIC0 is the reference's preconditioner, level-scheduled, so in FP64 it follows the oracle's iterations;
MG is the 3D multigrid V-cycle (src/sim/multigrid.ts in 3D); MIXED keeps FP32 vectors with FP64 inner
products and true-residual refinement and must still meet the requested max-norm tolerance.
"""
import numpy as np
import pytest
import torch

from poisson_util import FLUID, SOLID, AIR, apply_a
from teapotfluidsimulation_b200 import abi

pytestmark = pytest.mark.gpu


def solve(engine, cell, b, n, method, precision, tol, max_iter=3000):
    E = engine.engine
    count = cell.shape[0]
    dc = torch.from_numpy(np.ascontiguousarray(cell)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    dx = torch.zeros((count, n ** 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    pb = E.PoissonBatch(n, count, method, precision)
    it, res, conv = pb.solve(dc.data_ptr(), db.data_ptr(), dx.data_ptr(), tol, max_iter)
    x = dx.cpu().numpy()
    pb.destroy()
    return x, it, res, conv


def oracle_solutions(oracle_mod, cell, b, n, tol):
    out = []
    for s in range(cell.shape[0]):
        q, it, conv, res = oracle_mod.poisson_solve(cell[s], b[s].astype(np.float64), n, tol=tol, max_iter=5000)
        assert conv
        out.append((q, it))
    return out


@pytest.mark.parametrize("n", [8, 16, 32])
def test_mic0_f64_follows_the_oracle(engine, oracle_mod, n):
    E = engine.engine
    cell, b = E.poisson_generate(n, 0, 2)
    x, it, res, conv = solve(engine, cell, b, n, E.POISSON_MIC0, engine.abi.SOLVE_F64, 1e-10)
    ref = oracle_solutions(oracle_mod, cell, b, n, 1e-10)
    for s, (q, oit) in enumerate(ref):
        assert conv[s]
        assert abs(int(it[s]) - oit) <= 1, (it[s], oit)
        assert np.abs(x[s] - q).max() <= 1e-8 * max(np.abs(q).max(), 1e-30)


@pytest.mark.parametrize("n", [8, 16, 32])
def test_mg_f64_reaches_the_oracle_solution(engine, oracle_mod, n):
    E = engine.engine
    cell, b = E.poisson_generate(n, 4, 3)
    x, it, res, conv = solve(engine, cell, b, n, E.POISSON_MG, engine.abi.SOLVE_F64, 1e-12)
    ref = oracle_solutions(oracle_mod, cell, b, n, 1e-12)
    for s, (q, oit) in enumerate(ref):
        assert conv[s]
        assert np.abs(x[s] - q).max() <= 1e-9 * np.abs(q).max()
        r = b[s].astype(np.float64) - apply_a(cell[s], x[s], n)
        assert np.abs(r).max() <= 1e-12 * np.abs(b[s]).max() * 1.0001
        if n >= 32:
            assert it[s] < oit  # the V-cycle preconditions better than MIC(0) at this size


@pytest.mark.parametrize("method", [0, 1])
def test_mixed_meets_tolerance_and_is_close_to_fp64(engine, oracle_mod, method):
    E = engine.engine
    n = 32
    cell, b = E.poisson_generate(n, 9, 3)
    x, it, res, conv = solve(engine, cell, b, n, method, engine.abi.SOLVE_MIXED, 1e-6)
    ref = oracle_solutions(oracle_mod, cell, b, n, 1e-12)
    for s, (q, _) in enumerate(ref):
        assert conv[s]
        r = b[s].astype(np.float64) - apply_a(cell[s], x[s], n)
        assert np.abs(r).max() <= 1e-6 * np.abs(b[s]).max() * 1.0001  # true residual, max norm
        assert np.abs(x[s] - q).max() <= 1e-3 * np.abs(q).max()


def test_batch_equals_single_snapshots(engine):
    E = engine.engine
    n = 16
    cell, b = E.poisson_generate(n, 20, 3)
    xb, itb, _, _ = solve(engine, cell, b, n, E.POISSON_MG, engine.abi.SOLVE_MIXED, 1e-6)
    for s in range(3):
        xs, its, _, _ = solve(engine, cell[s:s + 1], b[s:s + 1], n, E.POISSON_MG, engine.abi.SOLVE_MIXED, 1e-6)
        assert its[0] == itb[s]
        assert np.array_equal(xs[0], xb[s])


@pytest.mark.parametrize("method", [0, 1])
def test_enclosed_component_with_gauge_fix(engine, oracle_mod, method):
    E = engine.engine
    n = 16
    cell = np.full((1, n ** 3), SOLID, np.uint8)
    c3 = cell.reshape(n, n, n)
    c3[2:7, 2:7, 2:7] = FLUID                    # enclosed by solid: all-Neumann without the fix
    c3[9:14, 3:8, 8:13] = FLUID
    c3[9:14, 8:12, 8:13] = AIR                   # free surface above the second pool
    b = np.random.default_rng(7).standard_normal((1, n ** 3)).astype(np.float32)
    b[(cell & 3) != FLUID] = 0
    assert E.poisson_gauge_fix(n, cell, b).tolist() == [1]
    x, it, res, conv = solve(engine, cell, b, n, method, engine.abi.SOLVE_F64, 1e-10)
    q = oracle_solutions(oracle_mod, cell, b, n, 1e-10)[0][0]
    assert conv[0]
    assert np.abs(x[0] - q).max() <= 1e-7 * np.abs(q).max()


def test_empty_and_zero_rhs(engine):
    E = engine.engine
    n = 16
    cell = np.full((2, n ** 3), AIR, np.uint8)
    cell.reshape(2, n, n, n)[:, 4:8, 4:8, 4:8] = FLUID
    b = np.zeros((2, n ** 3), np.float32)     # zero rhs: converged with 0 iterations (solver3d.ts:901)
    cell[1] = SOLID                           # no unknowns at all
    x, it, res, conv = solve(engine, cell, b, n, E.POISSON_MG, engine.abi.SOLVE_MIXED, 1e-6)
    assert it.tolist() == [0, 0] and conv.all() and (x == 0).all()


def pour_box(oracle_mod, box, mm=10, steps=5):
    """A pressure system of the reference pour (the oracle after a few substeps) in a SOLID-padded box:
    the cells, and b = A q for the oracle's pressure q (so the exact solution is known)."""
    sim = oracle_mod.OracleSim(abi.gentle_pour(mm, 1.0))
    for _ in range(steps):
        sim.step(-1)
    nx, ny, nz = sim.nx, sim.ny, sim.nz
    cell = sim.field(abi.FIELD_CELL).reshape(nz, ny, nx)
    q = sim.field(abi.FIELD_PRESSURE).reshape(nz, ny, nx)
    X, Y, Z = box
    bc = np.full((Z, Y, X), SOLID, np.uint8)
    bc[:nz, :ny, :nx] = cell
    bq = np.zeros((Z, Y, X))
    bq[:nz, :ny, :nx] = np.where(cell == FLUID, q, 0)
    bc = bc.reshape(1, -1)
    b = apply_a(bc[0], bq.reshape(-1), box).astype(np.float32)
    return bc, b.reshape(1, -1)


@pytest.mark.parametrize("method", [0, 1])
def test_box_of_a_pour_system(engine, oracle_mod, method):
    E = engine.engine
    box = (64, 64, 16)
    cell, b = pour_box(oracle_mod, box)
    E2 = engine.engine
    dc, db = torch.from_numpy(cell).cuda(), torch.from_numpy(b).cuda()
    dx = torch.zeros((1, int(np.prod(box))), dtype=torch.float64, device="cuda")
    pb = E2.PoissonBatch(box, 1, method, engine.abi.SOLVE_F64)
    it, res, conv = pb.solve(dc.data_ptr(), db.data_ptr(), dx.data_ptr(), 1e-10, 2000)
    pb.destroy()
    x = dx.cpu().numpy()[0]
    q, oit, oconv, _ = oracle_mod.poisson_solve(cell[0], b[0].astype(np.float64), box, tol=1e-10)
    assert conv[0] and oconv
    assert np.abs(x - q).max() <= 1e-8 * np.abs(q).max()
    if method == 0:
        assert abs(int(it[0]) - oit) <= 1


@pytest.mark.parametrize("method", [0, 1])
def test_reused_solver_object_repeats_itself(engine, method):
    # one solver object: snapshots A, then other cells B in the same buffers, then A again, then A
    # once more (the recorded solve graph is reused when nothing it depends on changed): every solve of
    # A gives the same iterations and bitwise the same solution
    E = engine.engine
    n, count = 32, 3
    ca, ba = E.poisson_generate(n, 10, count)
    cb, bb = E.poisson_generate(n, 20, count)
    dc = torch.from_numpy(ca.copy()).cuda()
    db = torch.from_numpy(ba.copy()).cuda()
    dx = torch.zeros((count, n ** 3), dtype=torch.float64, device="cuda")
    pb = E.PoissonBatch(n, count, method, abi.SOLVE_MIXED)
    runs = []
    for cells, rhs in ((ca, ba), (cb, bb), (ca, ba), (ca, ba)):
        dc.copy_(torch.from_numpy(cells))
        db.copy_(torch.from_numpy(rhs))
        it, res, conv = pb.solve(dc.data_ptr(), db.data_ptr(), dx.data_ptr(), 1e-6, 3000)
        assert conv.all()
        runs.append((it.copy(), dx.cpu().numpy()))
    pb.destroy()
    for k in (2, 3):
        assert np.array_equal(runs[k][0], runs[0][0]) and np.array_equal(runs[k][1], runs[0][1]), k
    assert not np.array_equal(runs[1][1], runs[0][1])
