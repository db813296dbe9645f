"""The learned preconditioner end to end: residual/correction pairs harvested from the engine's own pour
and its multigrid PCG, training on the GPU with the network's kernels (energy-norm loss), and flexible CG
with the network inside the Poisson batch, multigrid as the fallback and every system held to the same
max-norm tolerance."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TRAIN = 20  # systems for training; the rest are held out


@pytest.fixture(scope="module")
def trained(engine):
    from teapotfluidsimulation_b200 import learned as Lr

    E = engine.engine
    box, cells, r, e = Lr.harvest_pour_systems(cell_mm=10, count=24, every=10, seconds=8.0)
    tc, tr, te = Lr.residual_pairs(box, cells[:TRAIN], r[:TRAIN], e[:TRAIN], iters=(1, 2, 3, 5, 8))
    net = E.UNet(seed=2)
    net.set_loss(E.UNET_LOSS_ENERGY)
    hist = Lr.train(net, box, tc, tr, te, steps=1000, batch=4, lr=1e-3)
    return Lr, box, cells, r, e, net, hist


def one_step_ratio(Lr, box, cells, r, net):
    """||r - alpha A z|| / ||r|| with z = net(r) and the best alpha, per system."""
    X, Y, Z = box
    dc, dr = torch.from_numpy(cells.copy()).cuda(), torch.from_numpy(r.copy()).cuda()
    dz = torch.zeros_like(dr)
    net.apply(dc.data_ptr(), dr.data_ptr(), dz.data_ptr(), X, Y, Z, dc.shape[0])
    torch.cuda.synchronize()
    z = dz.cpu().numpy().astype(np.float64)
    out = []
    for i in range(cells.shape[0]):
        az = Lr.apply_a(cells[i].reshape(Z, Y, X), z[i].reshape(Z, Y, X)).reshape(-1)
        ri = r[i].astype(np.float64)
        a = ri @ z[i] / (z[i] @ az) if z[i] @ az > 0 else 0.0
        out.append(np.linalg.norm(ri - a * az) / np.linalg.norm(ri))
    return np.array(out)


def test_harvest_and_training(trained):
    Lr, box, cells, r, e, net, hist = trained
    assert box == (64, 64, 16) and cells.shape[0] == 24
    # r = A e on the unknowns by construction
    X, Y, Z = box
    ae = Lr.apply_a(cells[0].reshape(Z, Y, X), e[0].reshape(Z, Y, X).astype(np.float64)).reshape(-1)
    assert np.abs(ae - r[0]).max() <= 1e-5 * np.abs(r[0]).max()
    assert np.mean(hist[-20:]) < 0.2 * hist[0]


def test_trained_network_is_a_preconditioner_and_the_untrained_one_is_not(trained, engine):
    # on held-out systems one network step with the best step length removes a large part of the
    # residual; the same network at its initial weights makes the residual larger
    Lr, box, cells, r, e, net, hist = trained
    ho = slice(TRAIN, None)
    assert one_step_ratio(Lr, box, cells[ho], r[ho], net).max() < 0.75
    assert one_step_ratio(Lr, box, cells[ho], r[ho], engine.engine.UNet(seed=2)).min() > 1.0


def test_learned_cg_converges_on_the_network_alone(trained, engine):
    # the trained network preconditions every iteration to the tolerance (no fall-back); the untrained
    # one stalls and the multigrid fall-back finishes; both end on the max-norm rule, confirmed by the
    # FP64 true residual
    Lr, box, cells, r, e, net, hist = trained
    E = engine.engine
    X, Y, Z = box
    ho = slice(TRAIN, None)
    for name, use in (("trained", net), ("untrained", E.UNet(seed=2))):
        h = []
        x, it, conv, ms = Lr.solve(box, cells[ho], r[ho], E.POISSON_LEARNED, net=use, history=h)
        assert conv.all(), name
        learned_it = np.array([q[1] for q in h])
        if name == "trained":
            assert np.all(learned_it == it), (it, learned_it)
        else:
            assert np.all(learned_it < it), (it, learned_it)
        for i in range(x.shape[0]):
            res = r[ho][i].astype(np.float64) - Lr.apply_a(cells[ho][i].reshape(Z, Y, X), x[i].reshape(Z, Y, X)).reshape(-1)
            assert np.abs(res).max() <= 1e-6 * np.abs(r[ho][i]).max() * 1.0001
            assert np.abs(x[i] - e[ho][i]).max() <= 1e-3 * np.abs(e[ho][i]).max()


def test_history_records_the_residuals(trained, engine):
    Lr, box, cells, r, e, net, hist = trained
    h = []
    x, it, conv, ms = Lr.solve(box, cells[:2], r[:2], engine.engine.POISSON_MG, history=h)
    for i, (q, n) in enumerate(zip(h, it)):
        assert q[0].size == n and q[1] == 0
        assert q[0][-1] <= 1e-6 * np.abs(r[i]).max() * 10


def test_reused_solver_matches_a_fresh_one(trained, engine):
    # a solver object that first solved other systems (another active-tile footprint) gives the same
    # iterations and bitwise the same solution as a fresh one: no per-tile state survives a solve
    Lr, box, cells, r, e, net, hist = trained
    E = engine.engine
    X, Y, Z = box
    n = X * Y * Z

    def run(pb, c, b):
        dc, db = torch.from_numpy(c.copy()).cuda(), torch.from_numpy(b.copy()).cuda()
        dx = torch.zeros((c.shape[0], n), dtype=torch.float64, device="cuda")
        it, res, conv = pb.solve(dc.data_ptr(), db.data_ptr(), dx.data_ptr(), 1e-6, 400)
        return it, dx.cpu().numpy()

    reduced = cells[:2].copy()  # the lower half's liquid turned to air: tiles active before are inactive now
    low = reduced[:, : n // 2]
    low[(low & 3) == 1] = 0
    pb = E.PoissonBatch(box, 2, E.POISSON_LEARNED, 1)
    E._check(E.lib().pl_poisson_set_unet(pb._h, net._h))
    run(pb, cells[:2], r[:2])
    it_a, x_a = run(pb, reduced, r[:2])
    pb.destroy()
    pb = E.PoissonBatch(box, 2, E.POISSON_LEARNED, 1)
    E._check(E.lib().pl_poisson_set_unet(pb._h, net._h))
    it_b, x_b = run(pb, reduced, r[:2])
    pb.destroy()
    assert np.array_equal(it_a, it_b) and np.array_equal(x_a, x_b)


def test_learned_cg_against_multigrid_pcg_in_wall_time(trained, engine):
    # What the trained network gains over the method without it, in device time: flexible CG with the
    # network against multigrid PCG, the same held-out systems, the same max-norm 1e-6 rule, the fastest
    # of three solves each. The north star asks for at most 0.5x; measured at these 64x64x16 boxes the
    # learned solve takes more time than multigrid PCG although the network alone converges (fewer than
    # 2x the iterations): one application of the network costs far more than one V-cycle. The bound
    # below holds the measured state (about 20x) against regressions; the ratio is printed.
    Lr, box, cells, r, e, net, hist = trained
    E = engine.engine
    ho = slice(TRAIN, None)
    _, it_mg, conv_mg, ms_mg = Lr.solve(box, cells[ho], r[ho], E.POISSON_MG, reps=3)
    _, it_ln, conv_ln, ms_ln = Lr.solve(box, cells[ho], r[ho], E.POISSON_LEARNED, net=net, reps=3)
    ratio = ms_ln / ms_mg
    print(f"\nlearned FCG {ms_ln:.2f} ms ({it_ln.mean():.1f} iterations) vs multigrid PCG {ms_mg:.2f} ms "
          f"({it_mg.mean():.1f} iterations) on {cells[ho].shape[0]} held-out systems: {ratio:.1f}x")
    assert conv_mg.all() and conv_ln.all()
    assert it_ln.max() < 2 * it_mg.max() + 8  # the network preconditions nearly as well per iteration
    assert 0 < ratio < 60
