"""CPU FP64 restatement of the learned preconditioner's U-Net (the network of the engine's pl_unet_*):
the same layers, taps, padding, pooling, upsampling, concatenation, input packing, output scaling and
loss, written with torch on the CPU in float64 so autograd gives the exact gradient of this restatement."""
import numpy as np
import torch

LAYERS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16), (16, 16)]
AIR, FLUID = 0, 1


def unpack(params: np.ndarray):
    """Flat parameters -> [(W[27][cin][cout], b[cout])] as float64 tensors that require gradients."""
    out, o = [], 0
    for ci, co in LAYERS:
        w = torch.tensor(params[o:o + 27 * ci * co].reshape(27, ci, co), dtype=torch.float64, requires_grad=True)
        o += 27 * ci * co
        b = torch.tensor(params[o:o + co], dtype=torch.float64, requires_grad=True)
        o += co
        out.append((w, b))
    return out


def conv(x, w, b):
    """x: (N, C, Z, Y, X); tap t = dz*9 + dy*3 + dx reads the input at offset (dx-1, dy-1, dz-1)."""
    ci, co = w.shape[1], w.shape[2]
    wt = w.reshape(3, 3, 3, ci, co).permute(4, 3, 0, 1, 2)  # (co, ci, kz, ky, kx)
    return torch.nn.functional.conv3d(x, wt, b, padding=1)


def forward(layers, cell, r):
    """cell, r: (N, Z, Y, X) numpy; returns z (N, Z, Y, X) torch float64 and the scales."""
    liq = torch.tensor(cell == FLUID, dtype=torch.float64)
    air = torch.tensor(cell == AIR, dtype=torch.float64)
    rt = torch.tensor(r, dtype=torch.float64)
    s = torch.stack([torch.where(liq[i] > 0, rt[i].abs(), torch.zeros_like(rt[i])).max() for i in range(r.shape[0])])
    s = torch.where(s > 0, s, torch.ones_like(s))
    x = torch.zeros((r.shape[0], 16) + r.shape[1:], dtype=torch.float64)
    x[:, 0] = rt / s[:, None, None, None] * liq
    x[:, 1] = liq
    x[:, 2] = air
    relu = torch.relu
    pool = lambda t: torch.nn.functional.avg_pool3d(t, 2)
    up = lambda t: t.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)
    a0 = relu(conv(x, *layers[0]))
    s1 = relu(conv(a0, *layers[1]))
    a2 = relu(conv(pool(s1), *layers[2]))
    s2 = relu(conv(a2, *layers[3]))
    a4 = relu(conv(pool(s2), *layers[4]))
    a5 = relu(conv(a4, *layers[5]))
    a6 = relu(conv(torch.cat([up(a5), s2], 1), *layers[6]))
    a7 = relu(conv(a6, *layers[7]))
    a8 = relu(conv(torch.cat([up(a7), s1], 1), *layers[8]))
    a9 = relu(conv(a8, *layers[9]))
    o = conv(a9, *layers[10])
    z = s[:, None, None, None] * o[:, 0] * liq
    return z, s


def apply_a(cell, x):
    """The 7-point pressure operator on (N, Z, Y, X) boxes: unknowns are liquid cells off the border;
    diagonal = non-SOLID neighbours (+1 on pinned cells), -1 between neighbouring unknowns."""
    typ = cell & 3
    u = typ == FLUID
    u[:, 0] = u[:, -1] = u[:, :, 0] = u[:, :, -1] = u[:, :, :, 0] = u[:, :, :, -1] = False
    ut = torch.tensor(u, dtype=torch.float64)
    diag = torch.tensor((cell & 4) != 0, dtype=torch.float64)
    ns = torch.tensor(typ != 2, dtype=torch.float64)
    xu = x * ut
    nsum = torch.zeros_like(x)
    for axis in (1, 2, 3):
        for sh in (1, -1):
            diag = diag + torch.roll(ns, sh, axis)
            nsum = nsum + torch.roll(xu, sh, axis)
    return (diag * xu - nsum) * ut, ut


def loss_and_grad(params, cell, r, e, energy=False):
    """Loss of the network on (r, e) pairs and its gradient: the relative squared error over the liquid
    cells, or (energy=True) the relative error in the operator's energy norm over the unknowns."""
    layers = unpack(params)
    z, _ = forward(layers, cell, r)
    liq = torch.tensor(cell == FLUID, dtype=torch.float64)
    n = r.shape[0]
    if energy:
        e64 = torch.tensor(e, dtype=torch.float64)
        ae, ut = apply_a(cell, e64)
        d = (z - e64) * ut
        ad, _ = apply_a(cell, d)
        en = (e64 * ut * ae).sum(dim=(1, 2, 3))
        en = torch.where(en > 0, en, torch.ones_like(en))
        loss = ((d * ad).sum(dim=(1, 2, 3)) / en).sum() / n
    else:
        et = torch.tensor(e, dtype=torch.float64) * liq
        en = (et ** 2).sum(dim=(1, 2, 3))
        en = torch.where(en > 0, en, torch.ones_like(en))
        loss = (((z - et) ** 2).sum(dim=(1, 2, 3)) / en).sum() / n
    loss.backward()
    g = np.concatenate([np.concatenate([w.grad.numpy().reshape(-1), b.grad.numpy()]) for w, b in layers])
    return float(loss.detach()), g, z.detach().numpy()
