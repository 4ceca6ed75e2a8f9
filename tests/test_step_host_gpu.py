"""suli_step_host: a time step whose state comes from and goes back to host arrays.

The entry point must give exactly what suli_upload of each input, suli_step and suli_download
of each output give: the same kernels run in the same order, only the copies move to their own
streams.  The tests run both on the same host arrays, which are changed between steps so that
every step really reads what was copied in, and compare every result bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import pkg

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "prd1", "ls"]


def _pinned(shape):
    torch = pytest.importorskip("torch")
    t = torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True)
    return t, t.numpy().reshape(shape, order="F")


def _perturb(host, k):
    # what a host-side driver might do between steps: rescale the pressure, nudge a velocity
    host["prd1"] *= 0.5
    host["u"] += 1e-4 * np.sin(0.3 * k + np.arange(host["u"].size).reshape(host["u"].shape, order="F") * 1e-3)


def _run_pair(p, init, steps, pinned, extra_out=()):
    a, b = pkg.Solver(p), pkg.Solver(p)
    init(a)
    init(b)
    keep = []
    host_a, host_b = {}, {}
    for f in STATE:
        arr = a.download(f)
        if pinned:
            t, v = _pinned(arr.shape)
            keep.append(t)
            v[...] = arr
            host_b[f] = v
        else:
            host_b[f] = np.asfortranarray(arr.copy())
        host_a[f] = np.asfortranarray(arr.copy())
    outs_b = {f: host_b[f] for f in STATE}
    for f in extra_out:
        outs_b[f] = np.empty(b.shape(f), dtype=np.float64, order="F")
    for k in range(1, steps + 1):
        _perturb(host_a, k)
        _perturb(host_b, k)
        for f in STATE:
            a.upload(f, host_a[f])
        sa = a.step(k)
        for f in STATE:
            a.download(f, out=host_a[f])
        sb = b.step_host(k, {f: host_b[f] for f in STATE}, outs_b)
        assert sa == sb, (k, sa, sb)
        for f in STATE:
            assert np.array_equal(host_a[f], host_b[f]), (k, f)
        for f in extra_out:
            assert np.array_equal(a.download(f), outs_b[f]), (k, f)
    # the fields that never crossed to the host agree as well
    for f in ("rho", "hs", "kurv", "prd", "prd0", "nut"):
        assert np.array_equal(a.download(f), b.download(f)), f
    a.close()
    b.close()
    del keep


@pytest.mark.parametrize("pinned", [True, False])
def test_step_host_equals_upload_step_download(pinned):
    """Dam break, FP64 path, three steps: prd1 copied in during the level-set stage, ls copied
    out during the RK stages; pinned and pageable host memory."""
    p, init = pkg.cases.dam_break(nx=32, ny=16, nz=24, dx=0.02, cg_tol=1e-12)
    _run_pair(p, init, 3, pinned, extra_out=("rho",))


def test_step_host_mixed_path():
    """The mixed-precision solve (precision 1) behind the same copies."""
    p, init = pkg.cases.dam_break(nx=32, ny=16, nz=24, dx=0.02, cg_tol=1e-10)
    p.precision, p.inner_tol, p.refine_maxit = 1, 1e-3, 30
    _run_pair(p, init, 2, True)


def test_step_host_with_wave_inflow():
    """With wave inflow the level set is rounded in every RK stage, so ls goes out after the
    step; the inflow planes are copied synchronously when listed."""
    p, init = pkg.cases.wave_channel(wave_t=2, cg_tol=1e-12, outflow_fix=1)
    _run_pair(p, init, 2, True, extra_out=("bxx1",))


def test_step_host_rejects_bad_lists():
    p, init = pkg.cases.dam_break(nx=16, ny=8, nz=12, dx=0.04)
    s = pkg.Solver(p)
    init(s)
    u = s.download("u")
    lib = s.lib
    two = (C.c_int * 2)(pkg._abi.FIELD["u"], pkg._abi.FIELD["u"])   # a field listed twice
    ptrs2 = (C.c_void_p * 2)(u.ctypes.data, u.ctypes.data)
    assert lib.suli_step_host(s._h, 1, 2, two, ptrs2, 0, None, None, None) == pkg._abi.ERR_ARG
    assert lib.suli_step_host(s._h, 1, 0, None, None, 2, two, ptrs2, None) == pkg._abi.ERR_ARG
    n = pkg._abi.STEP_HOST_MAX_FIELDS + 1
    ids = (C.c_int * n)(*range(n))
    ptrs = (C.c_void_p * n)(*([u.ctypes.data] * n))
    assert lib.suli_step_host(s._h, 1, n, ids, ptrs, 0, None, None, None) == pkg._abi.ERR_ARG
    bad = (C.c_int * 1)(-1)
    assert lib.suli_step_host(s._h, 1, 1, bad, ptrs, 0, None, None, None) == pkg._abi.ERR_ARG
    with pytest.raises(ValueError):
        s.step_host(1, {"u": np.zeros((3, 3, 3))}, {})
    s.close()
