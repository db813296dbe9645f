"""The learned preconditioner end to end: pairs harvested from the engine's own pour, training on the GPU
with the network's kernels, and flexible CG with the network inside the Poisson batch, multigrid as the
fallback and every system held to the same max-norm tolerance."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained(engine):
    from teapotfluidsimulation_b200 import learned as Lr

    box, cells, r, e = Lr.harvest_pour_systems(cell_mm=10, count=24, every=8, seconds=6.0)
    net = engine.engine.UNet(seed=2)
    hist = Lr.train(net, box, cells[:20], r[:20], e[:20], steps=300, batch=4, lr=1e-3)
    return Lr, box, cells, r, e, net, hist


def test_training_fits_the_harvested_pairs(trained):
    Lr, box, cells, r, e, net, hist = trained
    assert box == (64, 64, 16) and cells.shape[0] == 24
    assert np.mean(hist[-10:]) < 0.1 * hist[0]


def test_trained_network_gains_over_the_untrained_one(trained, engine):
    # what training buys: on held-out systems of the same pour the network's correction is far closer
    # to A^-1 r than the same network at its initial weights
    Lr, box, cells, r, e, net, hist = trained
    X, Y, Z = box
    ev = slice(20, 24)

    def rel_err(nt):
        dc = torch.from_numpy(cells[ev].copy()).cuda()
        dr = torch.from_numpy(r[ev].copy()).cuda()
        dz = torch.zeros_like(dr)
        nt.apply(dc.data_ptr(), dr.data_ptr(), dz.data_ptr(), X, Y, Z, dc.shape[0])
        torch.cuda.synchronize()
        z = dz.cpu().numpy()
        return np.linalg.norm(z - e[ev], axis=1) / np.linalg.norm(e[ev], axis=1)

    untrained = engine.engine.UNet(seed=2)
    assert rel_err(net).max() < 0.4 < 0.9 < rel_err(untrained).min()


@pytest.mark.parametrize("which", ["trained", "untrained"])
def test_learned_cg_meets_the_tolerance(trained, engine, which):
    # with either network the flexible CG (and, when the network stalls, its multigrid fallback) ends on
    # the max-norm rule, confirmed by the FP64 true residual
    Lr, box, cells, r, e, net, hist = trained
    X, Y, Z = box
    use = net if which == "trained" else engine.engine.UNet(seed=2)
    ev = slice(20, 24)
    x, it, conv, ms = Lr.solve(box, cells[ev], r[ev], engine.engine.POISSON_LEARNED, net=use)
    assert conv.all()
    for i in range(x.shape[0]):
        res = r[ev][i].astype(np.float64) - Lr.apply_a(cells[ev][i].reshape(Z, Y, X), x[i].reshape(Z, Y, X)).reshape(-1)
        assert np.abs(res).max() <= 1e-6 * np.abs(r[ev][i]).max() * 1.0001
        assert np.abs(x[i] - e[ev][i]).max() <= 1e-3 * np.abs(e[ev][i]).max()
