"""Poisson batch on the CPU: the synthetic workload generator, the gauge fix and the oracle's pinned solve.

No counterpart in the reference as a batch; the operator and stopping rule are Pcg3D's
(src/sim3d/solver3d.ts:858-973) and the gauge fix is fixEnclosedGauges (src/sim/pressure.ts:232-268).
"""
import numpy as np
import pytest

from poisson_util import AIR, FLUID, PIN, SOLID, apply_a, unknowns


def test_generator_is_deterministic_and_offset_consistent(engine):
    c0, b0 = engine.engine.poisson_generate(16, 0, 3, threads=2)
    c1, b1 = engine.engine.poisson_generate(16, 0, 3, threads=1)
    c2, b2 = engine.engine.poisson_generate(16, 2, 1)
    assert np.array_equal(c0, c1) and np.array_equal(b0, b1)
    assert np.array_equal(c0[2], c2[0]) and np.array_equal(b0[2], b2[0])


def test_generator_masks(engine):
    n = 32
    cell, b = engine.engine.poisson_generate(n, 5, 2)
    for s in range(2):
        c = cell[s].reshape(n, n, n)  # (k, j, i)
        t = c & 3
        assert (t[0] == SOLID).all() and (t[-1] == SOLID).all() and (t[:, 0] == SOLID).all()
        assert (t[:, :, 0] == SOLID).all() and (t[:, :, -1] == SOLID).all() and (t[:, -1] == SOLID).all()
        k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        outside = (i + 0.5 - n / 2) ** 2 + (k + 0.5 - n / 2) ** 2 > (60 / 128 * n) ** 2
        assert (t[outside] == SOLID).all()
        slab = max(2, int(16 * n / 128))
        inner = ~outside & (i > 0) & (j > 0) & (k > 0) & (i < n - 1) & (k < n - 1) & (j < slab)
        assert (t[inner] == FLUID).all()
        assert set(np.unique(t)) <= {AIR, FLUID, SOLID}
        u = unknowns(cell[s], n).reshape(-1)
        assert (b[s][~u] == 0).all() and np.abs(b[s][u]).max() > 0


def test_gauge_fix_pins_enclosed_components_and_removes_their_mean(engine):
    n = 16
    cell = np.full((1, n ** 3), SOLID, np.uint8)
    c3 = cell.reshape(n, n, n)
    c3[4:8, 4:8, 4:8] = FLUID                     # enclosed by solid
    c3[10:14, 3:6, 9:12] = FLUID
    c3[12, 5, 10] = AIR                           # touches air: not enclosed
    b = np.random.default_rng(0).standard_normal((1, n ** 3)).astype(np.float32)
    b[cell != FLUID] = 0
    before = b.copy()
    enc = engine.engine.poisson_gauge_fix(n, cell, b)
    assert enc.tolist() == [1]
    assert np.flatnonzero(cell[0] & PIN).tolist() == [4 * n * n + 4 * n + 4]  # first cell in index order
    box = np.zeros((n, n, n), bool)
    box[4:8, 4:8, 4:8] = True
    box = box.reshape(-1)
    assert abs(float(b[0][box].astype(np.float64).sum())) < 1e-5
    other = (cell[0] & 3 == FLUID) & ~box
    assert np.array_equal(b[0][other], before[0][other])


def test_oracle_pinned_solve_converges(oracle_mod, engine):
    n = 16
    cell = np.full(n ** 3, SOLID, np.uint8)
    cell.reshape(n, n, n)[3:9, 3:9, 3:9] = FLUID
    b = np.random.default_rng(1).standard_normal(n ** 3).astype(np.float32)
    b[cell != FLUID] = 0
    cell2, b2 = cell[None].copy(), b[None].copy()
    engine.engine.poisson_gauge_fix(n, cell2, b2)
    q, it, conv, res = oracle_mod.poisson_solve(cell2[0], b2[0].astype(np.float64), n, tol=1e-12)
    assert conv and it > 0
    r = b2[0].astype(np.float64) - apply_a(cell2[0], q, n)
    assert np.abs(r).max() <= 1e-12 * np.abs(b2[0]).max() * 10


def test_oracle_matches_pcg3d_on_unpinned_cells(oracle_mod, engine):
    # without pins the snapshot solve is Pcg3D.solve on the same cells (solver3d.ts:858-937)
    n = 16
    cell, b = engine.engine.poisson_generate(n, 3, 1)
    assert not (cell & PIN).any()
    q1, it1, c1, _ = oracle_mod.poisson_solve(cell[0], b[0].astype(np.float64), n, tol=1e-10, max_iter=400)
    q2, it2, c2, _ = oracle_mod.pcg_solve(cell[0], b[0].astype(np.float64), n, n, n, 1e-10, 400)
    assert it1 == it2 and np.array_equal(q1, q2)
