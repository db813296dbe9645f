"""Shared numpy helpers for the Poisson-batch tests: the dense operator of Pcg3D (solver3d.ts:858-953)
with the gauge-fix pin (src/sim/pressure.ts:265)."""
import numpy as np

AIR, FLUID, SOLID, PIN = 0, 1, 2, 4


def shape3(n):
    """(nz, ny, nx) of a cube edge n or an (nx, ny, nz) box."""
    return (n, n, n) if isinstance(n, int) else (n[2], n[1], n[0])


def unknowns(cell: np.ndarray, n) -> np.ndarray:
    t = (cell.reshape(shape3(n)) & 3) == FLUID
    t[0, :, :] = t[-1, :, :] = t[:, 0, :] = t[:, -1, :] = t[:, :, 0] = t[:, :, -1] = False
    return t


def apply_a(cell: np.ndarray, x: np.ndarray, n) -> np.ndarray:
    """A x on the unknowns of one snapshot (FP64), zero elsewhere; n is the cube's edge or (nx, ny, nz)."""
    sh = shape3(n)
    c = cell.reshape(sh)
    u = unknowns(cell, n)
    typ = c & 3
    x3 = np.where(u, x.reshape(sh).astype(np.float64), 0.0)
    diag = np.zeros(sh)
    nsum = np.zeros(sh)
    for axis in range(3):
        for sh in (1, -1):
            tn = np.roll(typ, sh, axis=axis)
            diag += tn != SOLID
            nsum += np.roll(x3, sh, axis=axis)
    diag += (c & PIN) != 0
    return np.where(u, diag * x3 - nsum, 0.0).reshape(-1)
