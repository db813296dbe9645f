"""Training data and training loop of the learned pressure preconditioner (pl_unet_*, pl_poisson LEARNED).

The pairs come from the pour itself: the engine runs a gentle pour and, every few substeps, its pressure
system (cell types and the solved pressure q of Simulation3D.project, src/sim3d/solver3d.ts:530-543) is
read back, embedded in a SOLID-padded power-of-two box, and turned into an exact pair (r = A q, e = q) with
the Pcg3D operator (solver3d.ts:939-953). Training runs on the GPU with the network's own kernels.
"""
from __future__ import annotations

import numpy as np

from . import abi
from . import engine as E

AIR, FLUID, SOLID = abi.AIR, abi.FLUID, abi.SOLID


def box_for(nx: int, ny: int, nz: int) -> tuple[int, int, int]:
    """Smallest power-of-two box (each side >= 8) that holds an nx x ny x nz grid."""
    p = lambda v: max(8, 1 << (int(v) - 1).bit_length())
    return p(nx), p(ny), p(nz)


def apply_a(cell: np.ndarray, x: np.ndarray) -> np.ndarray:
    """A x of the Pcg3D operator on a (nz, ny, nx) box (FP64): non-SOLID neighbours count on the
    diagonal (+1 on a pinned cell), FLUID neighbours couple with -1; non-liquid and border cells are
    not unknowns."""
    typ = cell & 3
    u = typ == FLUID
    u[0, :, :] = u[-1, :, :] = u[:, 0, :] = u[:, -1, :] = u[:, :, 0] = u[:, :, -1] = False
    xu = np.where(u, x, 0.0)
    diag = ((cell & 4) != 0).astype(np.float64)  # the gauge pin (pl_poisson_gauge_fix)
    nsum = np.zeros(cell.shape)
    for axis in range(3):
        for sh in (1, -1):
            diag += np.roll(typ, sh, axis=axis) != SOLID
            nsum += np.roll(xu, sh, axis=axis)
    return np.where(u, diag * xu - nsum, 0.0)


def harvest_pour_systems(cell_mm: float = 5.0, count: int = 32, every: int = 12, seconds: float = 12.0,
                         preconditioner: int = abi.PRECOND_CHEB, box: tuple | None = None, **over):
    """Run the gentle pour on the engine and collect `count` pressure systems, one every `every` substeps
    (keyword overrides of the config by field name, e.g. domain, transfer, solve_precision).

    Returns (box (nx, ny, nz), cells u8 (count, cells), r f32, e f32): r = A e with e the engine's
    pressure on the liquid cells."""
    cfg = abi.gentle_pour(cell_mm, seconds, **over)
    cfg.preconditioner = preconditioner
    if "solve_precision" not in over:
        cfg.solve_precision = abi.SOLVE_MIXED if preconditioner == abi.PRECOND_BOX_MG else abi.SOLVE_F64
    sim = E.Simulation3D(cfg)
    box = box or box_for(sim.nx, sim.ny, sim.nz)
    X, Y, Z = box
    cells, rs, es = [], [], []
    k = 0
    while len(cells) < count and not sim.finished:
        sim.step(-1.0)
        k += 1
        if k % every:
            continue
        c = sim.field(abi.FIELD_CELL).reshape(sim.nz, sim.ny, sim.nx)
        q = sim.field(abi.FIELD_PRESSURE).reshape(sim.nz, sim.ny, sim.nx)
        bc = np.full((Z, Y, X), SOLID, np.uint8)
        bc[:sim.nz, :sim.ny, :sim.nx] = c
        bq = np.zeros((Z, Y, X))
        bq[:sim.nz, :sim.ny, :sim.nx] = np.where(c == FLUID, q, 0.0)
        cells.append(bc.reshape(-1))
        rs.append(apply_a(bc, bq).astype(np.float32).reshape(-1))
        es.append(bq.astype(np.float32).reshape(-1))
    sim.destroy()
    return box, np.stack(cells), np.stack(rs), np.stack(es)


def residual_pairs(box, cells: np.ndarray, r: np.ndarray, e: np.ndarray, iters=(1, 2, 3)):
    """Residual/correction pairs of the plain multigrid PCG: for each system and each k in `iters`,
    x_k after k iterations from zero, r_k = r - A x_k and e_k = e - x_k (so A e_k = r_k exactly, up to
    FP32 rounding of the stored vectors). Together with the systems' own (r, e) they cover the
    residuals the flexible CG hands the network in its later iterations. Returns (cells, r, e) with
    the systems' pairs first, then those of each k."""
    X, Y, Z = box
    cs, rs, es = [cells], [r], [e]
    for k in iters:
        x, _, _, _ = solve(box, cells, r, E.POISSON_MG, tol=1e-30, max_iter=int(k))
        rk = np.empty_like(r)
        for i in range(cells.shape[0]):
            ax = apply_a(cells[i].reshape(Z, Y, X), x[i].reshape(Z, Y, X)).reshape(-1)
            rk[i] = (r[i].astype(np.float64) - ax).astype(np.float32)
        cs.append(cells)
        rs.append(rk)
        es.append((e.astype(np.float64) - x).astype(np.float32))
    return np.concatenate(cs), np.concatenate(rs), np.concatenate(es)


def train(net: E.UNet, box, cells: np.ndarray, r: np.ndarray, e: np.ndarray, steps: int, batch: int = 4,
          lr: float = 1e-3, seed: int = 0, time_limit: float | None = None):
    """Adam steps on random batches of the pairs (device copies made once). Returns the loss history."""
    import time

    import torch

    X, Y, Z = box
    dc = torch.from_numpy(np.ascontiguousarray(cells)).cuda()
    dr = torch.from_numpy(np.ascontiguousarray(r)).cuda()
    de = torch.from_numpy(np.ascontiguousarray(e)).cuda()
    rng = np.random.default_rng(seed)
    n = cells.shape[0]
    hist = []
    t0 = time.perf_counter()
    for _ in range(steps):
        idx = torch.from_numpy(rng.choice(n, size=min(batch, n), replace=False)).cuda()
        bc, br, be = dc[idx].contiguous(), dr[idx].contiguous(), de[idx].contiguous()
        hist.append(net.train_step(bc.data_ptr(), br.data_ptr(), be.data_ptr(), X, Y, Z, bc.shape[0], lr))
        if time_limit is not None and time.perf_counter() - t0 > time_limit:
            break
    torch.cuda.synchronize()
    return hist


def solve(box, cells: np.ndarray, r: np.ndarray, method: int, tol: float = 1e-6, max_iter: int = 1000,
          net: E.UNet | None = None, reps: int = 1, history: list | None = None):
    """pl_poisson_solve of the systems (FP32 vectors, FP64 refinement); returns (x, iterations,
    converged, ms of the fastest repetition). A list passed as `history` receives, per system, the
    max-norm residual after each iteration and the iterations taken with the network."""
    import torch

    count = cells.shape[0]
    dc = torch.from_numpy(np.ascontiguousarray(cells)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(r)).cuda()
    dx = torch.zeros((count, int(np.prod(box))), dtype=torch.float64, device="cuda")
    pb = E.PoissonBatch(box, count, method, abi.SOLVE_MIXED)
    if net is not None:
        E._check(E.lib().pl_poisson_set_unet(pb._h, net._h))
    best = None
    for _ in range(reps):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        it, res, conv = pb.solve(dc.data_ptr(), db.data_ptr(), dx.data_ptr(), tol, max_iter)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
    if history is not None:
        history.extend(pb.history(s) for s in range(count))
    pb.destroy()
    return dx.cpu().numpy(), it, conv, best
