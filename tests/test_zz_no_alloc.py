"""suli_est_static: the divergence check for callers that may not let the library allocate.

Some drivers keep u, v, w on the GPU under another runtime (OpenACC or CUDA Fortran device
arrays, or a framework that has reserved the device memory for its own caching allocator).
They can hand the library device pointers, but a cudaMalloc inside the library could fail for
lack of unreserved memory and cudaMalloc/cudaFree would stall their other work.  This entry
point takes its reduction scratch from a fixed array built into the library instead.

The test holds the velocity fields in device memory that the test (the caller) allocated,
calls the entry point through the C-ABI twice in a row, and checks each result against the
context-based suli_est on the same fields.  It is collected last and needs nothing from the
other test files.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import load_state, seeded_state, small_params

pytestmark = pytest.mark.gpu


def _device_copy(torch, a):
    # Fortran-ordered host array -> contiguous device buffer with the same element order
    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to("cuda:0")


def _est_static(pkg, torch, p, u, v, w):
    lib = pkg.load_library()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    rc = lib.suli_est_static(C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()), C.c_void_p(w.data_ptr()),
                             p.nx, p.ny, p.nz, p.dx, p.dy, p.dz, C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert rc == 0, rc
    torch.cuda.synchronize(0)
    return float(out.item())


def test_est_static_matches_est_twice(pkg):
    torch = pytest.importorskip("torch")
    p = small_params(nx=40, ny=24, nz=20)
    s = pkg.Solver(p)
    load_state(s, seeded_state(p, 21))
    s.contorno(1)
    for call in range(2):
        if call == 1:   # different fields for the second call: the shared scratch must not leak
            u = s.download("u")
            u[:, :, :] *= -2.5
            s.upload("u", u)
        ref = s.est()
        du, dv, dw = (_device_copy(torch, s.download(f)) for f in ("u", "v", "w"))
        got = _est_static(pkg, torch, p, du, dv, dw)
        assert ref > 0.0
        assert abs(got - ref) <= 1e-13 * ref, (call, got, ref)


def test_est_static_refuses_grids_beyond_its_scratch(pkg):
    torch = pytest.importorskip("torch")
    lib = pkg.load_library()
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    ptr = C.c_void_p(dummy.data_ptr())
    # 512 x 256 x 256 needs exactly the 8192 block partials the library holds; one more row of
    # tiles in y does not fit.  The size check happens before any device access.
    rc = lib.suli_est_static(ptr, ptr, ptr, 512, 264, 256, 0.01, 0.01, 0.01, ptr, None)
    assert rc == pkg._abi.ERR_SIZE
    assert pkg._abi.EST_STATIC_MAX_BLOCKS == 8192
