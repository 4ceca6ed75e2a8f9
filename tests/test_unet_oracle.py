"""CPU: the FP64 network oracle (oracle/unet_ref.py) and the package's parameter layout.

The oracle's hand-written backpropagation is pinned by central finite differences of its
own loss; the GPU tests then hold the CUDA forward/backward kernels to this oracle.
"""
import numpy as np
import pytest

import unet_ref


def test_layout_matches_package(pkg):
    assert unet_ref.LAYERS == pkg.learned.LAYERS
    assert unet_ref.num_params() == pkg.learned.num_params()
    w = pkg.learned.init_params(3)
    assert w.dtype == np.float32 and w.size == unet_ref.num_params()
    convs, (hw, hb) = unet_ref.unpack(w.astype(np.float64))
    assert convs[0][0].shape == (27, 16, 16)
    assert np.all(convs[0][0][:, :, 3:] == 0)        # padded input channels carry no weight
    assert convs[8][0].shape == (27, 64, 160)
    assert hw.shape == (16,)


def test_library_param_count(pkg):
    lib = pkg.load_library()
    assert lib.suli_nn_num_params() == unet_ref.num_params()


def _problem(n=8, seed=0):
    rng = np.random.default_rng(seed)
    theta = unet_ref.init_params(seed)
    # non-zero biases and a unit-scale head exercise every gradient path
    convs, _ = unet_ref.unpack(theta)
    o = 0
    for ci, co, _ in unet_ref.LAYERS:
        o += 27 * co * ci
        theta[o:o + co] = 0.05 * rng.standard_normal(co)
        o += co
    theta[o:o + 16] = rng.standard_normal(16)
    theta[o + 16] = 0.3
    x3 = rng.standard_normal((n, n, n, 3))
    tgt = rng.standard_normal((n, n, n))
    return theta, x3, tgt


def test_oracle_gradient_finite_differences():
    theta, x3, tgt = _problem()
    loss, g = unet_ref.loss_grad(theta, x3, tgt)
    assert np.isfinite(loss) and g.shape == theta.shape
    rng = np.random.default_rng(1)
    # coordinates in every layer's weights, every bias block and the head
    offs = [0]
    for ci, co, _ in unet_ref.LAYERS:
        offs.append(offs[-1] + 27 * co * ci + co)
    picks = []
    for l in range(len(unet_ref.LAYERS)):
        ci, co, _ = unet_ref.LAYERS[l]
        w_lo, b_lo = offs[l], offs[l] + 27 * co * ci
        real_ci = 3 if l == 0 else ci
        tap, c_o, c_i = rng.integers(27), rng.integers(co), rng.integers(real_ci)
        picks.append(w_lo + (tap * co + c_o) * ci + c_i)
        picks.append(b_lo + rng.integers(co))
    picks += [offs[-1] + 3, offs[-1] + 16]
    h = 1e-6
    bad = []
    for q in picks:
        tp = theta.copy(); tp[q] += h
        tm = theta.copy(); tm[q] -= h
        fd = (unet_ref.loss_grad(tp, x3, tgt)[0] - unet_ref.loss_grad(tm, x3, tgt)[0]) / (2 * h)
        if abs(fd - g[q]) > 1e-5 * max(abs(fd), abs(g[q])) + 1e-9:
            bad.append((q, fd, g[q]))
    # a ReLU kink inside [-h, h] can spoil one difference; more means a wrong gradient
    assert len(bad) <= 1, bad
