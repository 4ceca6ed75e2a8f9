"""CPU tests of the drop-in boundary: the C-ABI library loads, exports every entry point the
header declares, agrees with the Python binding on struct layout, defaults and extents, and
refuses to run without a GPU instead of falling back to the CPU."""
import ctypes as C
import pathlib
import re

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "suli_gpu.h"


def header_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(suli_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol(pkg):
    lib = pkg.load_library()
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared in suli_gpu.h but not exported: {missing}"
    assert sorted(pkg._abi.HEADER_SYMBOLS) == names


def test_struct_sizes_match_binding(pkg):
    lib = pkg.load_library()
    pb, sb = C.c_int(), C.c_int()
    assert lib.suli_abi_sizes(C.byref(pb), C.byref(sb)) == 0
    assert pb.value == C.sizeof(pkg.SuliParams)
    assert sb.value == C.sizeof(pkg.SuliStepStats)


def test_defaults_match_reference_modules(pkg):
    """suli_params_default = 0_modules.f90 + 14_level_set.f90:25-31, same as the binding."""
    lib = pkg.load_library()
    p = pkg.SuliParams()
    assert lib.suli_params_default(C.byref(p)) == 0
    q = pkg.default_params()
    for k, v in q.as_dict().items():
        assert getattr(p, k) == pytest.approx(v, rel=0, abs=0), k
    assert (p.nx, p.ny, p.nz) == (25, 50, 45)       # int(.5/dx), int(1/dy), int(.9/dz)
    assert p.cg_tol == 0.0001 and p.cg_maxit == 10000


def test_field_extents_match_binding(pkg):
    lib = pkg.load_library()
    p = pkg.default_params()
    p.nx, p.ny, p.nz = 7, 5, 6
    lo, hi = (C.c_int * 3)(), (C.c_int * 3)()
    for name, fid in pkg.FIELD.items():
        assert lib.suli_field_extent(C.byref(p), fid, lo, hi) == 0
        ext = pkg.field_extent(p, name)
        assert tuple((lo[d], hi[d]) for d in range(3)) == ext, name
    assert lib.suli_field_extent(C.byref(p), 999, lo, hi) < 0


def test_create_without_gpu_fails_loudly(pkg):
    """No CUDA device -> SULI_ERR_NODEVICE; the library has no CPU path."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = pkg.load_library()
    p = pkg.default_params()
    h = C.c_void_p()
    rc = lib.suli_create(C.byref(p), 0, C.byref(h))
    assert rc == pkg._abi.ERR_NODEVICE
    assert not h.value


def test_step_host_without_context_is_refused(pkg):
    """suli_step_host checks its context before touching a device or a host pointer."""
    lib = pkg.load_library()
    ids = (C.c_int * 1)(pkg._abi.FIELD["u"])
    ptrs = (C.c_void_p * 1)(None)
    assert lib.suli_step_host(None, 1, 1, ids, ptrs, 1, ids, ptrs, None) == pkg._abi.ERR_ARG
    assert pkg._abi.STEP_HOST_MAX_FIELDS == 8


def test_invalid_parameters_rejected(pkg):
    lib = pkg.load_library()
    h = C.c_void_p()
    p = pkg.default_params()
    p.ccx0, p.ccxf = 0, 2           # periodic on one side only (0_modules.f90:56)
    assert lib.suli_create(C.byref(p), 0, C.byref(h)) == pkg._abi.ERR_ARG
    p = pkg.default_params()
    p.nx, p.ny, p.nz = 15, 13, 11   # the mixed path's multigrid needs a grid that halves
    p.precision, p.cg_stop = 1, 1
    assert lib.suli_create(C.byref(p), 0, C.byref(h)) == pkg._abi.ERR_UNSUPPORTED
    p = pkg.default_params()
    p.t_hs = 2                      # the reference defines t_hs 0 and 1 (14_level_set.f90:696-703)
    assert lib.suli_create(C.byref(p), 0, C.byref(h)) == pkg._abi.ERR_ARG
    p = pkg.default_params()
    p.obst_t = 11                   # obstaculo has presets 1..10
    assert lib.suli_create(C.byref(p), 0, C.byref(h)) == pkg._abi.ERR_ARG
    p = pkg.default_params()
    p.nx = 3                        # WENO needs 4 cells per direction
    assert lib.suli_create(C.byref(p), 0, C.byref(h)) == pkg._abi.ERR_ARG
    # the reference defines der 1-3, adv_type 1-3 and m_turb 0-2 (0_modules.f90:26-31)
    for field, bad in (("der", 0), ("der", 4), ("m_turb", -1), ("m_turb", 3), ("adv_type", 0), ("adv_type", 4)):
        p = pkg.default_params()
        setattr(p, field, bad)
        assert lib.suli_create(C.byref(p), 0, C.byref(h)) == pkg._abi.ERR_ARG, (field, bad)
    for adv in (2, 3):              # rotacional and antissim stop for any scheme but upwind
        p = pkg.default_params()
        p.adv_type, p.der = adv, 2
        assert lib.suli_create(C.byref(p), 0, C.byref(h)) == pkg._abi.ERR_ARG, adv


def test_no_oracle_in_product(pkg):
    """The product package and library never reference the oracle."""
    for path in list((ROOT / "suli-openmp_b200").rglob("*.py")) + list((ROOT / "suli-openmp_b200" / "csrc").glob("*.cu*")):
        text = path.read_text()
        assert "oracle" not in text.lower(), path
    lib = pkg.load_library()
    assert not hasattr(lib, "orc_create")


def test_step_host_binding_checks_arrays_before_the_call(pkg):
    """Solver.step_host refuses arrays of the wrong shape, order or type, and more fields than
    the library takes, before it calls the library (no context or GPU needed to reach them)."""
    import numpy as np
    s = object.__new__(pkg.Solver)   # the checks need only the parameters
    s.params = pkg.default_params()
    s.params.nx, s.params.ny, s.params.nz = 6, 5, 4
    s.lib, s._h = None, None
    good = np.zeros(s.shape("u"), order="F")
    with pytest.raises(ValueError):
        s.step_host(1, {"u": np.zeros((3, 3, 3), order="F")}, {})
    with pytest.raises(ValueError):
        s.step_host(1, {}, {"u": np.ascontiguousarray(good)})     # C order
    with pytest.raises(ValueError):
        s.step_host(1, {"u": good.astype(np.float32)}, {})
    names = ["u", "v", "w", "prd1", "prd0", "prd", "rho", "ls", "hs"]
    many = {n: np.zeros(s.shape(n), order="F") for n in names}
    assert len(many) > pkg._abi.STEP_HOST_MAX_FIELDS
    with pytest.raises(ValueError):
        s.step_host(1, many, {})
