"""Host side of the learned preconditioner: the operator used to build training pairs, the box rule,
and the FP64 restatement's energy-norm loss against a direct evaluation."""
import numpy as np
import torch

import unet_ref
from teapotfluidsimulation_b200 import learned as Lr


def random_box(seed, shape=(6, 8, 10)):
    rng = np.random.default_rng(seed)
    cell = rng.choice(np.array([0, 1, 1, 1, 2], np.uint8), size=shape)
    cell[rng.random(shape) < 0.03] |= 4  # a few gauge pins on any type; only liquid ones matter
    return cell, rng.standard_normal(shape)


def dense_a(cell):
    """The operator as a dense matrix over the unknowns, written out cell by cell."""
    Z, Y, X = cell.shape
    unk = [(k, j, i) for k in range(1, Z - 1) for j in range(1, Y - 1) for i in range(1, X - 1)
           if cell[k, j, i] & 3 == 1]
    pos = {c: n for n, c in enumerate(unk)}
    A = np.zeros((len(unk), len(unk)))
    for (k, j, i), n in pos.items():
        A[n, n] = 1.0 if cell[k, j, i] & 4 else 0.0
        for dk, dj, di in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            q = (k + dk, j + dj, i + di)
            if cell[q] & 3 != 2:
                A[n, n] += 1
            if q in pos:
                A[n, pos[q]] = -1
    return A, unk


def test_apply_a_matches_the_dense_operator():
    for seed in range(3):
        cell, x = random_box(seed)
        A, unk = dense_a(cell)
        xv = np.array([x[c] for c in unk])
        ax = Lr.apply_a(cell, x)
        assert np.allclose([ax[c] for c in unk], A @ xv, atol=1e-12)
        mask = np.ones(cell.shape, bool)
        for c in unk:
            mask[c] = False
        assert np.all(ax[mask] == 0)
        assert np.allclose(A, A.T)


def test_restatement_operator_matches_numpy():
    cell, x = random_box(5)
    ax, _ = unet_ref.apply_a(cell[None], torch.tensor(x[None]))
    assert np.allclose(ax.numpy()[0], Lr.apply_a(cell, x), atol=1e-12)


def test_energy_norm_error_matches_the_dense_formula():
    # the restatement's energy-norm error (z - e).A(z - e) / e.Ae against the dense matrix
    cell, e = random_box(7, (8, 8, 8))
    A, unk = dense_a(cell)
    ev = np.array([e[c] for c in unk])
    d = 0.1 * np.random.default_rng(1).standard_normal(len(unk))
    ref = d @ A @ d / (ev @ A @ ev)
    z = np.zeros_like(e)
    for n, c in enumerate(unk):
        z[c] = ev[n] + d[n]
    _, ut = unet_ref.apply_a(cell[None], torch.zeros((1,) + e.shape, dtype=torch.float64))
    dd = torch.tensor(z - e)[None] * ut
    ad, _ = unet_ref.apply_a(cell[None], dd)
    ae, _ = unet_ref.apply_a(cell[None], torch.tensor(e[None]))
    got = float((dd * ad).sum() / (torch.tensor(e[None]) * ut * ae).sum())
    assert abs(got - ref) <= 1e-10 * abs(ref)


def test_box_for_rounds_up_to_powers_of_two():
    assert Lr.box_for(33, 33, 9) == (64, 64, 16)
    assert Lr.box_for(3, 8, 9) == (8, 8, 16)
