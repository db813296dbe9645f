"""The learned preconditioner's U-Net kernels (BF16 tensor-core convolutions, FP32 accumulation) against
the CPU FP64 restatement in unet_ref.py: the forward output, the loss and every layer's gradient."""
import numpy as np
import pytest
import torch

import unet_ref

pytestmark = pytest.mark.gpu

NX, NY, NZ, N = 16, 12, 8, 2


def case(seed=3):
    rng = np.random.default_rng(seed)
    cell = np.full((N, NZ, NY, NX), 2, np.uint8)
    cell[:, 1:-1, 1:-1, 1:-1] = 0
    cell[:, 1:-1, 1:7, 1:-1] = 1                      # a liquid slab under air
    cell[1, 2:5, 7:10, 3:9] = 1                       # and a blob in the second box
    r = (rng.standard_normal(cell.shape) * (cell == 1)).astype(np.float32)
    e = (rng.standard_normal(cell.shape) * (cell == 1)).astype(np.float32)
    return cell, r, e


def exact_corrections(cell, r):
    """e = A^-1 r on each box's unknowns (liquid cells off the border; dense FP64 solve), 0 elsewhere."""
    from teapotfluidsimulation_b200 import learned as Lr

    e = np.zeros(r.shape, np.float32)
    for s in range(cell.shape[0]):
        c = cell[s]
        u = (c & 3) == 1
        u[0] = u[-1] = u[:, 0] = u[:, -1] = u[:, :, 0] = u[:, :, -1] = False
        unk = np.flatnonzero(u)
        A = np.empty((unk.size, unk.size))
        for n, i in enumerate(unk):
            A[:, n] = Lr.apply_a(c, np.eye(1, c.size, i).reshape(c.shape)).reshape(-1)[unk]
        es = np.zeros(c.size)
        es[unk] = np.linalg.solve(A, r[s].reshape(-1)[unk].astype(np.float64))
        e[s] = es.reshape(c.shape)
    return e


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_forward_matches_fp64_restatement(engine):
    cell, r, e = case()
    net = engine.engine.UNet(seed=5)
    p = net.params()
    dc, dr = dev(cell), dev(r)
    dz = torch.zeros_like(dr)
    net.apply(dc.data_ptr(), dr.data_ptr(), dz.data_ptr(), NX, NY, NZ, N)
    torch.cuda.synchronize()
    z = dz.cpu().numpy().astype(np.float64)
    zr, _ = unet_ref.forward(unet_ref.unpack(p), cell, r)
    zr = zr.detach().numpy()
    assert np.all(z[cell != 1] == 0)
    rel = np.linalg.norm(z - zr) / np.linalg.norm(zr)
    assert rel < 3e-2, rel  # BF16 weights and activations through 11 layers


@pytest.mark.parametrize("energy", [False, True])
def test_gradient_matches_fp64_restatement(engine, energy):
    cell, r, e = case()
    if energy:  # the pairs the energy loss is meant for: e solves A e = r
        e = exact_corrections(cell, r)
    net = engine.engine.UNet(seed=5)
    if energy:
        net.set_loss(engine.engine.UNET_LOSS_ENERGY)
    p = net.params()
    dc, dr, de = dev(cell), dev(r), dev(e)
    loss, g = net.gradient(dc.data_ptr(), dr.data_ptr(), de.data_ptr(), NX, NY, NZ, N)
    loss_ref, g_ref, _ = unet_ref.loss_and_grad(p.astype(np.float64), cell, r, e, energy=energy)
    assert abs(loss - loss_ref) < 2e-2 * abs(loss_ref)
    cos = float(g @ g_ref / (np.linalg.norm(g) * np.linalg.norm(g_ref)))
    assert cos > 0.995, cos
    o = 0
    for li, (ci, co) in enumerate(unet_ref.LAYERS):
        n = 27 * ci * co + co
        a, b = g[o:o + n], g_ref[o:o + n]
        o += n
        if np.linalg.norm(b) > 0:
            # the energy loss's output gradient 2 s A d is rough (the stencil of a difference), so its BF16
            # copy loses more through the 11 layers to the first one
            tol = 0.25 if energy else 0.1
            assert np.linalg.norm(a - b) <= tol * np.linalg.norm(b), (li, np.linalg.norm(a - b) / np.linalg.norm(b))


def test_training_lowers_the_loss(engine):
    cell, r, e = case(7)
    net = engine.engine.UNet(seed=9)
    dc, dr, de = dev(cell), dev(r), dev(e)
    first = net.train_step(dc.data_ptr(), dr.data_ptr(), de.data_ptr(), NX, NY, NZ, N, 1e-3)
    last = first
    for _ in range(60):
        last = net.train_step(dc.data_ptr(), dr.data_ptr(), de.data_ptr(), NX, NY, NZ, N, 1e-3)
    assert last < 0.7 * first, (first, last)


@pytest.mark.parametrize("shape", [(16, 12, 8, 2), (32, 16, 12, 3), (128, 8, 12, 2), (256, 4, 8, 1)])
def test_tcgen05_and_mma_sync_kernels_agree(engine, shape):
    # the two convolution kernels compute the same BF16 products with FP32 accumulation in different
    # orders: the network's output agrees to BF16 rounding, the loss and gradient closely (x extents
    # of 128 and 256 take the row-tile tcgen05 kernel at full resolution, the others the gather kernel)
    X, Y, Z, n = shape
    rng = np.random.default_rng(1)
    cell = np.full((n, Z, Y, X), 2, np.uint8)
    cell[:, 1:-1, 1:-1, 1:-1] = rng.choice(np.array([0, 1, 1], np.uint8), size=(n, Z - 2, Y - 2, X - 2))
    r = (rng.standard_normal(cell.shape) * (cell == 1)).astype(np.float32)
    e = (rng.standard_normal(cell.shape) * (cell == 1)).astype(np.float32)
    dc, dr, de = dev(cell), dev(r), dev(e)
    out = {}
    for kind in (engine.engine.UNET_CONV_TCGEN05, engine.engine.UNET_CONV_MMA_SYNC):
        net = engine.engine.UNet(seed=5)
        net.set_conv_kernel(kind)
        dz = torch.zeros_like(dr)
        net.apply(dc.data_ptr(), dr.data_ptr(), dz.data_ptr(), X, Y, Z, n)
        torch.cuda.synchronize()
        loss, g = net.gradient(dc.data_ptr(), dr.data_ptr(), de.data_ptr(), X, Y, Z, n)
        assert net.error() == 0
        out[kind] = (dz.cpu().numpy().astype(np.float64), loss, g.astype(np.float64))
    (z0, l0, g0), (z1, l1, g1) = out.values()
    assert np.linalg.norm(z0 - z1) <= 1e-2 * np.linalg.norm(z1)
    assert abs(l0 - l1) <= 1e-3 * abs(l1)
    assert float(g0 @ g1 / (np.linalg.norm(g0) * np.linalg.norm(g1))) > 0.999
