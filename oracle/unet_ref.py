"""FP64 numpy restatement of the pressure-solve U-Net (forward and backward).

TEST INFRASTRUCTURE ONLY: the checker of the network kernels in csrc/nn.cu (layer order,
parameter layout, pooling, upsampling, concatenation, ReLU, head, squared-error loss).  The
network has no counterpart in the reference; this file pins the CUDA kernels to the
mathematics they claim to compute, in FP64 with hand-written backpropagation.

Layout: volumes are numpy arrays (nz, ny, nx, C) — channels last, x fastest, as on the GPU.
Parameters: per conv layer W[27][Cout][Cin] (tap = dx + 3 dy + 9 dz, offsets d - 1) then
bias[Cout]; the head is w[16] then b.
"""
from __future__ import annotations

import numpy as np

LAYERS = [  # (cin, cout, level)
    (16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 96, 3),
    (96, 96, 3), (160, 64, 2), (64, 64, 2), (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0),
]


def num_params():
    return sum(27 * co * ci + co for ci, co, _ in LAYERS) + 17


def unpack(theta):
    out, o = [], 0
    for ci, co, _ in LAYERS:
        W = theta[o:o + 27 * co * ci].reshape(27, co, ci)
        o += 27 * co * ci
        b = theta[o:o + co]
        o += co
        out.append((W, b))
    head = (theta[o:o + 16], theta[o + 16])
    return out, head


def conv3(x, W, b):
    """3x3x3, zero padding: out[z,y,x,co] = sum_tap sum_ci xpad[...] W[tap,co,ci] + b."""
    nz, ny, nx, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((nz, ny, nx, W.shape[1]))
    for t in range(27):
        dx, dy, dz = t % 3, (t // 3) % 3, t // 9
        out += xp[dz:dz + nz, dy:dy + ny, dx:dx + nx, :] @ W[t].T
    return out + b


def conv3_dx(dz_, W, shape):
    """input gradient of conv3"""
    nz, ny, nx, _ = shape
    gp = np.zeros((nz + 2, ny + 2, nx + 2, W.shape[2]))
    for t in range(27):
        dx, dy, dzz = t % 3, (t // 3) % 3, t // 9
        gp[dzz:dzz + nz, dy:dy + ny, dx:dx + nx, :] += dz_ @ W[t]
    return gp[1:-1, 1:-1, 1:-1, :]


def conv3_dw(x, dz_):
    nz, ny, nx, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    dW = np.zeros((27, dz_.shape[3], x.shape[3]))
    for t in range(27):
        dx, dy, dzz = t % 3, (t // 3) % 3, t // 9
        xs = xp[dzz:dzz + nz, dy:dy + ny, dx:dx + nx, :].reshape(-1, x.shape[3])
        dW[t] = dz_.reshape(-1, dz_.shape[3]).T @ xs
    return dW, dz_.reshape(-1, dz_.shape[3]).sum(axis=0)


def pool(x):
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).mean(axis=(1, 3, 5))


def up(x):
    return x.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)


def forward(theta, x3):
    """x3: (nz, ny, nx, 3) -> prediction (nz, ny, nx), and the cache for backward."""
    convs, (hw, hb) = unpack(theta)
    x = np.zeros(x3.shape[:3] + (16,))
    x[..., :3] = x3
    a, pools, ins = [None] * 14, [None] * 3, [None] * 14

    def layer(l, inp):
        ins[l] = inp
        a[l] = np.maximum(conv3(inp, *convs[l]), 0.0)
        return a[l]

    layer(0, x); layer(1, a[0]); pools[0] = pool(a[1])
    layer(2, pools[0]); layer(3, a[2]); pools[1] = pool(a[3])
    layer(4, pools[1]); layer(5, a[4]); pools[2] = pool(a[5])
    layer(6, pools[2]); layer(7, a[6])
    layer(8, np.concatenate([up(a[7]), a[5]], axis=3)); layer(9, a[8])
    layer(10, np.concatenate([up(a[9]), a[3]], axis=3)); layer(11, a[10])
    layer(12, np.concatenate([up(a[11]), a[1]], axis=3)); layer(13, a[12])
    out = a[13] @ hw + hb
    return out, (a, ins)


def loss_grad(theta, x3, target):
    """mean squared error and its gradient w.r.t. theta (FP64 backpropagation)."""
    convs, (hw, hb) = unpack(theta)
    out, (a, ins) = forward(theta, x3)
    V = out.size
    e = out - target
    loss = float((e ** 2).mean())
    dout = 2.0 / V * e
    grads = [None] * 14
    gact = [np.zeros_like(t) for t in a]
    g_head = np.concatenate([(a[13] * dout[..., None]).reshape(-1, 16).sum(axis=0), [dout.sum()]])
    gact[13] = dout[..., None] * hw
    for l in range(13, -1, -1):
        dz = gact[l] * (a[l] > 0)
        dW, db = conv3_dw(ins[l], dz)
        grads[l] = (dW, db)
        if l == 0:
            break
        dx = conv3_dx(dz, convs[l][0], ins[l].shape)
        if l in (8, 10, 12):
            coarse, skip = {8: (7, 5), 10: (9, 3), 12: (11, 1)}[l]
            ca = a[coarse].shape[3]
            d_up = dx[..., :ca]
            nz, ny, nx, _ = d_up.shape
            gact[coarse] = d_up.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, ca).sum(axis=(1, 3, 5))
            gact[skip] = gact[skip] + dx[..., ca:]
        elif l in (2, 4, 6):
            gact[l - 1] = gact[l - 1] + up(dx) / 8.0
        else:
            gact[l - 1] = dx
    flat = []
    for dW, db in grads:
        flat += [dW.ravel(), db]
    flat.append(g_head)
    return loss, np.concatenate(flat)


def init_params(seed=0):
    """He-normal weights for the ReLU layers (zero for the padded input channels), zero biases,
    a small head."""
    rng = np.random.default_rng(seed)
    theta = []
    for l, (ci, co, _) in enumerate(LAYERS):
        real = 3 if l == 0 else ci
        W = rng.standard_normal((27, co, ci)) * np.sqrt(2.0 / (27 * real))
        if l == 0:
            W[:, :, 3:] = 0.0
        theta += [W.ravel(), np.zeros(co)]
    theta += [rng.standard_normal(16) * 0.1, np.zeros(1)]
    return np.concatenate(theta)
