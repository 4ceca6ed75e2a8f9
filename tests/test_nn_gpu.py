"""GPU: the network kernels (csrc/nn.cu, nn_conv.cuh) against references.

* the three tensor-core convolutions (the persistent tcgen05 pipeline with TMA loads, tcgen05
  with one tile per CTA, and mma.sync) against an FP64 convolution of the same BF16 inputs,
  including the decoder's input (half-resolution tensor upsampled and concatenated with a
  full-resolution skip);
* forward, loss and parameter gradient of the whole U-Net against the FP64 oracle
  (oracle/unet_ref.py, itself pinned by finite differences), with the conv weights and the
  input rounded to BF16 as the GPU reads them.  The GPU keeps activations and activation
  gradients in BF16, so the tolerances are those of BF16 storage (2^-8 relative per value),
  stated per check below;
* Adam steps lower the loss; forward passes are deterministic.
"""
import numpy as np
import pytest

import unet_ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available()
    return T


def _bf16(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16)


@pytest.mark.parametrize("kernel", [0, 1, 2], ids=["tcgen05_pipe", "mma_sync", "tcgen05_tile"])
@pytest.mark.parametrize("shape,cin,cout,relu", [
    ((12, 10, 9), 16, 16, True),
    ((8, 8, 8), 32, 48, False),
    ((9, 5, 7), 160, 64, True),
    ((16, 8, 4), 96, 96, False),
    ((6, 6, 6), 64, 160, False),
    ((10, 4, 12), 16, 32, True),
    ((8, 33, 3), 48, 16, True),
])
def test_conv3d_matches_fp64(pkg, torch, shape, cin, cout, relu, kernel):
    nx, ny, nz = shape
    rng = np.random.default_rng(cin * 1000 + cout)
    x = _bf16(torch, rng.standard_normal((nz, ny, nx, cin)))
    w = _bf16(torch, rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
    b = torch.from_numpy(rng.standard_normal(cout).astype(np.float32))
    out = torch.empty((nz, ny, nx, cout), dtype=torch.bfloat16, device="cuda:0")
    xd, wd, bd = x.to("cuda:0"), w.to("cuda:0"), b.to("cuda:0")
    pkg.learned.conv3d(xd, wd, bd, out, shape, cin, cout, relu, kernel=kernel)
    torch.cuda.synchronize()
    # FP64 reference: cross-correlation with zero padding, tap = dx + 3 dy + 9 dz
    xin = x.double().permute(3, 0, 1, 2).unsqueeze(0)              # (1, cin, nz, ny, nx)
    wt = w.double().reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2)   # (cout, cin, dz, dy, dx)
    ref = torch.nn.functional.conv3d(xin, wt, b.double(), padding=1)[0].permute(1, 2, 3, 0)
    if relu:
        ref = ref.clamp_min(0.0)
    got = out.double().cpu()
    err = (got - ref).abs()
    # BF16 rounding of the output (<= 2^-9 relative) plus FP32 accumulation order
    tol = 2.0 ** -8 * ref.abs() + 1e-5 * ref.abs().max()
    assert bool((err <= tol).all()), float((err - tol).max())


@pytest.mark.parametrize("shape,cin,cout", [
    ((64, 64, 64), 16, 16),      # 512+ tiles: several per CTA, resident weights, x taps folded into N
    ((128, 64, 48), 32, 32),     # the ring of halo slots wraps around
    ((64, 64, 32), 96, 32),      # six chunks per tile
    ((40, 48, 22), 32, 64),      # 8 x 16 tiles, two planes per tile, ragged in every direction
    ((24, 32, 13), 64, 96),      # weights streamed with each chunk, one plane per tile
    ((16, 16, 9), 64, 160),      # the widest input-gradient shape: 512 TMEM columns, one slot
])
def test_pipeline_kernel_at_scale(pkg, torch, shape, cin, cout):
    """The pipelined kernel where every CTA walks many tiles, against an FP64 convolution of the
    same BF16 inputs (BF16 output rounding).  Where it keeps the one-tile kernel's 8 x 16 tile
    (Cout >= 48) it issues the same MMAs in the same order, so the two agree bit for bit."""
    nx, ny, nz = shape
    g = torch.Generator(device="cuda:0").manual_seed(cin + cout)
    x = torch.randn((nz, ny, nx, cin), generator=g, device="cuda:0").to(torch.bfloat16)
    w = (torch.randn((27, cout, cin), generator=g, device="cuda:0") / (27 * cin) ** 0.5).to(torch.bfloat16)
    b = torch.randn(cout, generator=g, device="cuda:0")
    outs = []
    for kernel in (0, 2):
        out = torch.full((nz, ny, nx, cout), float("nan"), dtype=torch.bfloat16, device="cuda:0")
        pkg.learned.conv3d(x, w, b, out, shape, cin, cout, True, kernel=kernel)
        outs.append(out)
    torch.cuda.synchronize()
    xin = x.double().permute(3, 0, 1, 2).unsqueeze(0)
    wt = w.double().reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2)
    ref = torch.nn.functional.conv3d(xin, wt, b.double(), padding=1)[0].permute(1, 2, 3, 0).clamp_min(0.0)
    err = (outs[0].double() - ref).abs()
    tol = 2.0 ** -8 * ref.abs() + 1e-5 * ref.abs().max()
    assert bool((err <= tol).all()), float((err - tol).max())
    if cout >= 48:
        assert torch.equal(outs[0], outs[1])


def _pool_ref(torch, out):
    """k_pool's arithmetic on a BF16 [nz][ny][nx][C] tensor: FP32 sum of the 8 children in the
    order (x, y, z) = (0,0,0), (1,0,0), (0,1,0), (1,1,0), then z = 1, times 1/8, rounded to BF16."""
    f = out.float()
    s = torch.zeros_like(f[::2, ::2, ::2])
    for d in range(8):
        dx, dy, dz = d & 1, (d >> 1) & 1, d >> 2
        s = s + f[dz::2, dy::2, dx::2]
    return (0.125 * s).to(torch.bfloat16)


@pytest.mark.parametrize("kernel", [0, 2], ids=["tcgen05_pipe", "tcgen05_tile"])
@pytest.mark.parametrize("shape,cin,cout,head", [
    ((64, 48, 32), 16, 16, True),    # x taps folded, 4 planes a tile: pooling and head in the epilogue
    ((32, 32, 16), 32, 32, False),   # x taps folded, 2 planes a tile
    ((16, 32, 16), 32, 64, False),   # 8 x 16 tile, 2 planes
])
def test_fused_pool_and_head(pkg, torch, shape, cin, cout, head, kernel):
    """The pooling and the head the network fuses into its convolutions: the pooled tensor equals
    k_pool's arithmetic on the convolution's own BF16 output bit for bit, the head equals
    w . x + b of that output to FP32 rounding."""
    nx, ny, nz = shape
    g = torch.Generator(device="cuda:0").manual_seed(cin * 7 + cout)
    x = torch.randn((nz, ny, nx, cin), generator=g, device="cuda:0").to(torch.bfloat16)
    w = (torch.randn((27, cout, cin), generator=g, device="cuda:0") / (27 * cin) ** 0.5).to(torch.bfloat16)
    b = torch.randn(cout, generator=g, device="cuda:0") * 0.1
    out = torch.empty((nz, ny, nx, cout), dtype=torch.bfloat16, device="cuda:0")
    pool = torch.full((nz // 2, ny // 2, nx // 2, cout), float("nan"), dtype=torch.bfloat16, device="cuda:0")
    hw = torch.randn(17, generator=g, device="cuda:0") if head else None
    ho = torch.full((nz, ny, nx), float("nan"), device="cuda:0") if head else None
    pkg.learned.conv3d(x, w, b, out, shape, cin, cout, True, kernel=kernel, pool=pool, head_w=hw, head_out=ho)
    torch.cuda.synchronize()
    assert torch.equal(pool, _pool_ref(torch, out))
    if head:
        ref = (out.double() * hw[:16].double()).sum(-1) + float(hw[16])
        scale = (out.double().abs() * hw[:16].double().abs()).sum(-1) + abs(float(hw[16]))
        assert bool(((ho.double() - ref).abs() <= 1e-6 * scale).all())


def test_network_forward_pipeline_matches_tile_kernel(pkg, torch):
    """Whole network at 128 x 128 x 64 (many tiles per CTA on every level), including the
    decoder's upsampled half-resolution inputs gathered with cp.async: the pipelined kernel and
    the one-tile kernel agree to BF16 activation rounding (the folded layers sum the three x
    taps in another order)."""
    nx, ny, nz = 128, 128, 64
    net = pkg.learned.Net.load(nx, ny, nz)
    g = torch.Generator(device="cuda:0").manual_seed(3)
    d_in = torch.randn(nx * ny * nz * 3, generator=g, device="cuda:0")
    outs = []
    for kernel in (0, 2):
        net.set_kernel(kernel)
        y = torch.empty(nx * ny * nz, device="cuda:0")
        net.forward(d_in, y)
        outs.append(y)
    assert torch.isfinite(outs[0]).all() and outs[0].abs().max() > 0
    rel = float((outs[0] - outs[1]).norm() / outs[1].norm())
    assert rel < 1e-2, rel
    net.close()


def _setup(torch, n, seed):
    rng = np.random.default_rng(seed)
    theta = unet_ref.init_params(seed)
    o = 0
    for ci, co, _ in unet_ref.LAYERS:
        o += 27 * co * ci
        theta[o:o + co] = 0.05 * rng.standard_normal(co)
        o += co
    theta[o:o + 16] = rng.standard_normal(16)
    theta[o + 16] = 0.3
    theta32 = theta.astype(np.float32)
    x3 = rng.standard_normal((n, n, n, 3)).astype(np.float32)
    tgt = rng.standard_normal((n, n, n)).astype(np.float32)
    # what the GPU computes with: BF16 conv weights and input, FP32 biases and head
    theta_ref = theta32.astype(np.float64)
    o = 0
    for ci, co, _ in unet_ref.LAYERS:
        nw = 27 * co * ci
        theta_ref[o:o + nw] = _bf16(torch, theta32[o:o + nw]).double().numpy()
        o += nw + co
    x3_ref = _bf16(torch, x3).double().numpy()
    return theta32, theta_ref, x3, x3_ref, tgt


def _layer_slices():
    out, o = [], 0
    for l, (ci, co, _) in enumerate(unet_ref.LAYERS):
        out.append((f"W{l}", slice(o, o + 27 * co * ci)))
        o += 27 * co * ci
        out.append((f"b{l}", slice(o, o + co)))
        o += co
    out.append(("head", slice(o, o + 17)))
    return out


@pytest.mark.parametrize("kernel", [0, 1, 2], ids=["tcgen05_pipe", "mma_sync", "tcgen05_tile"])
def test_forward_matches_oracle(pkg, torch, kernel):
    n = 16
    theta32, theta_ref, x3, x3_ref, _ = _setup(torch, n, 5)
    net = pkg.learned.Net(n, n, n, params=theta32)
    net.set_kernel(kernel)
    d_in = torch.from_numpy(x3).to("cuda:0")
    d_out = torch.empty(n ** 3, dtype=torch.float32, device="cuda:0")
    net.forward(d_in, d_out)
    got = d_out.cpu().numpy().reshape(n, n, n)
    ref, _ = unet_ref.forward(theta_ref, x3_ref)
    rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    # 14 layers of BF16 activations: a few 2^-8 roundings per value, far below 5%
    assert rel < 0.03, rel
    # deterministic: a second pass gives the same bits
    d_out2 = torch.empty_like(d_out)
    net.forward(d_in, d_out2)
    assert torch.equal(d_out, d_out2)
    net.close()


@pytest.mark.parametrize("kernel", [0, 1, 2], ids=["tcgen05_pipe", "mma_sync", "tcgen05_tile"])
def test_loss_and_gradient_match_oracle(pkg, torch, kernel):
    n = 16
    theta32, theta_ref, x3, x3_ref, tgt = _setup(torch, n, 7)
    net = pkg.learned.Net(n, n, n, params=theta32)
    net.set_kernel(kernel)
    d_in = torch.from_numpy(x3).to("cuda:0")
    d_t = torch.from_numpy(tgt.ravel()).to("cuda:0")
    loss, g = net.loss_grad(d_in, d_t)
    loss_ref, g_ref = unet_ref.loss_grad(theta_ref, x3_ref, tgt.astype(np.float64))
    assert abs(loss - loss_ref) <= 0.03 * loss_ref, (loss, loss_ref)
    g = g.astype(np.float64)
    cos = float(g @ g_ref / (np.linalg.norm(g) * np.linalg.norm(g_ref)))
    assert cos > 0.995, cos
    worst = {}
    for name, sl in _layer_slices():
        if name == "W0":    # weights of the zero-padded input channels: compare the real ones
            a = g[sl].reshape(27, 16, 16)[:, :, :3]
            b = g_ref[sl].reshape(27, 16, 16)[:, :, :3]
        else:
            a, b = g[sl], g_ref[sl]
        worst[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    # BF16 activation gradients through up to 14 layers: per-block relative error under 10%
    assert max(worst.values()) < 0.10, worst
    # reproducible: per-block partial sums added in a fixed order, no float atomics
    _, g2 = net.loss_grad(d_in, d_t)
    assert np.array_equal(g.astype(np.float32), g2), "gradient differs between two identical calls"
    net.close()


@pytest.mark.parametrize("n", [16, 32])
def test_tensor_core_weight_gradient_matches_cuda_cores(pkg, torch, monkeypatch, n):
    """The weight gradients on the tensor cores (k_wgrad_tc, mma.sync BF16 -> FP32, default)
    against the CUDA-core kernel (SULI_WGRAD_CUDA_CORES=1): the same BF16 products summed in FP32
    in another order, so every parameter block agrees to 1e-3 of its norm; at 32^3 the CTAs'
    voxel chunks and the row sums are exercised (8 chunks of 4096 voxels).  Both reproducible."""
    theta32, _, x3, _, tgt = _setup(torch, n, 5)
    d_in = torch.from_numpy(x3).to("cuda:0")
    d_t = torch.from_numpy(tgt.ravel()).to("cuda:0")
    grads = {}
    for cc in ("1", "0"):
        monkeypatch.setenv("SULI_WGRAD_CUDA_CORES", cc)
        net = pkg.learned.Net(n, n, n, params=theta32)
        loss, g = net.loss_grad(d_in, d_t)
        _, g2 = net.loss_grad(d_in, d_t)
        assert np.array_equal(g, g2)
        grads[cc] = (loss, g.astype(np.float64))
        net.close()
    (l1, g1), (l0, g0) = grads["1"], grads["0"]
    assert l1 == l0
    for name, sl in _layer_slices():
        a, b = g0[sl], g1[sl]
        assert np.linalg.norm(a - b) <= 1e-3 * max(np.linalg.norm(b), 1e-30), name


def test_adam_lowers_loss_and_params_roundtrip(pkg, torch):
    n = 16
    theta32, _, x3, _, tgt = _setup(torch, n, 11)
    net = pkg.learned.Net(n, n, n, params=theta32)
    assert np.array_equal(net.get_params(), theta32)
    d_in = torch.from_numpy(x3).to("cuda:0")
    d_t = torch.from_numpy(tgt.ravel()).to("cuda:0")
    losses = [net.train_step(d_in, d_t, 1e-3) for _ in range(40)]
    assert losses[-1] < 0.7 * losses[0], losses[::8]
    w = net.get_params()
    assert not np.array_equal(w, theta32) and np.all(np.isfinite(w))
    net.close()


def test_bad_grid_refused(pkg):
    with pytest.raises(pkg.learned.NetError):
        pkg.learned.Net(12, 16, 16)
