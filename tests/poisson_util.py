"""Shared numpy helpers for the Poisson-batch tests: the dense operator of Pcg3D (solver3d.ts:858-953)
with the gauge-fix pin (src/sim/pressure.ts:265)."""
import numpy as np

AIR, FLUID, SOLID, PIN = 0, 1, 2, 4


def unknowns(cell: np.ndarray, n: int) -> np.ndarray:
    t = (cell.reshape(n, n, n) & 3) == FLUID
    t[0, :, :] = t[-1, :, :] = t[:, 0, :] = t[:, -1, :] = t[:, :, 0] = t[:, :, -1] = False
    return t


def apply_a(cell: np.ndarray, x: np.ndarray, n: int) -> np.ndarray:
    """A x on the unknowns of one snapshot (FP64), zero elsewhere."""
    c = cell.reshape(n, n, n)
    u = unknowns(cell, n)
    typ = c & 3
    x3 = np.where(u, x.reshape(n, n, n).astype(np.float64), 0.0)
    diag = np.zeros((n, n, n))
    nsum = np.zeros((n, n, n))
    for axis in range(3):
        for sh in (1, -1):
            tn = np.roll(typ, sh, axis=axis)
            diag += tn != SOLID
            nsum += np.roll(x3, sh, axis=axis)
    diag += (c & PIN) != 0
    return np.where(u, diag * x3 - nsum, 0.0).reshape(-1)
