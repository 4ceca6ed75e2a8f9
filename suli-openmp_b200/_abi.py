"""ctypes mirror of include/suli_gpu.h and the loader of libsuli_gpu.so.

The structures and enumerations here must match the header field for field; the
`test_abi.py` CPU test checks the sizes against the compiled library.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libsuli_gpu.so"


class SuliParams(C.Structure):
    """`suli_params` — the reference's compile-time parameters (0_modules.f90) at run time."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("dt", C.c_double),
        ("ccx0", C.c_int), ("ccxf", C.c_int),
        ("ccy0", C.c_int), ("ccyf", C.c_int),
        ("ccz0", C.c_int), ("cczf", C.c_int),
        ("t_tempo", C.c_int), ("der", C.c_int), ("adv_type", C.c_int),
        ("m_turb", C.c_int), ("obst_t", C.c_int), ("t_hs", C.c_int),
        ("csmag", C.c_double),
        ("gx", C.c_double), ("gz", C.c_double),
        ("chezy", C.c_double),
        ("rho_f1", C.c_double), ("mi_f1", C.c_double),
        ("rho_f2", C.c_double), ("mi_f2", C.c_double),
        ("sigma", C.c_double),
        ("alpha1", C.c_double),
        ("dt1", C.c_double),
        ("reinit_maxit", C.c_int),
        ("vol_tol", C.c_double),
        ("cg_stop", C.c_int),
        ("cg_tol", C.c_double),
        ("cg_maxit", C.c_int),
        ("precision", C.c_int),
        ("refine_maxit", C.c_int),
        ("inner_tol", C.c_double),
        ("mg_omega", C.c_double),
        ("mg_alpha", C.c_double),
        ("mg_kernels", C.c_int),
        ("wave_t", C.c_int),
        ("outflow_fix", C.c_int),
        ("periodic_faces", C.c_int),
        ("mg_omega2", C.c_double),
        ("div_tol", C.c_double),
    ]

    def copy(self) -> "SuliParams":
        out = SuliParams()
        C.pointer(out)[0] = self
        return out

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SuliStepStats(C.Structure):
    _fields_ = [
        ("cg_iters", C.c_int * 3),
        ("cg_resid", C.c_double * 3),
        ("vol_ins", C.c_double),
        ("max_div", C.c_double),
        ("status", C.c_int),
    ]


# --- status codes -------------------------------------------------------------------------
OK = 0
WARN_CG_MAXIT = 1
ERR_ARG = -1
ERR_CUDA = -2
ERR_NAN = -3
ERR_UNSUPPORTED = -4
ERR_NOMEM = -5
ERR_NODEVICE = -6
ERR_SIZE = -7

# --- field identifiers (enum suli_field) ------------------------------------------------------
FIELD_NAMES = [
    "u", "v", "w", "prd1", "prd0", "prd", "rho", "ls_nu",
    "Fu", "u0", "fu0", "fu1", "Fv", "v0", "fv0", "fv1", "Fw", "w0", "fw0", "fw1",
    "nut", "xnut", "ynut", "znut",
    "ls", "mod_ls", "kurv", "hs", "ddlsdx", "ddlsdy", "ddlsdz", "hsx", "hsy", "hsz",
    "ub", "vb", "wb", "tf_u", "tf_v", "tf_w",
    "bxx0", "bxx1", "bxy0", "bxz0", "bxxf", "bxxf1", "bxyf", "bxzf",
    "byx0", "byy0", "byy1", "byz0", "byxf", "byyf", "byyf1", "byzf",
    "bzx0", "bzy0", "bzz0", "bzz1", "bzxf", "bzyf", "bzzf", "bzzf1",
]
FIELD = {n: i for i, n in enumerate(FIELD_NAMES)}
FIELD_COUNT = len(FIELD_NAMES)

SCALAR_NAMES = ["dt", "vol_ini", "vol_ins", "dt1", "t", "ntt", "a_dt1", "a_dt2", "a_dt3", "fallbacks"]
SCALAR = {n: i for i, n in enumerate(SCALAR_NAMES)}


def field_extent(p: SuliParams, name: str):
    """Inclusive Fortran ranges ((lo0,hi0),(lo1,hi1),(lo2,hi2)) of a module array."""
    nx, ny, nz = p.nx, p.ny, p.nz
    if name in ("u", "ub"):
        return (0, nx + 2), (0, ny + 1), (0, nz + 1)
    if name in ("v", "vb"):
        return (0, nx + 1), (0, ny + 2), (0, nz + 1)
    if name in ("w", "wb"):
        return (0, nx + 1), (0, ny + 1), (0, nz + 2)
    if name in ("prd1", "prd0", "prd"):
        return (0, nx + 1), (0, ny + 1), (0, nz + 1)
    if name in ("rho", "ls_nu", "nut", "ls", "mod_ls", "kurv", "hs", "ddlsdx", "ddlsdy",
                "ddlsdz", "hsx", "hsy", "hsz"):
        return (1, nx), (1, ny), (1, nz)
    if name in ("Fu", "u0", "fu0", "fu1", "xnut", "tf_u"):
        return (1, nx + 1), (1, ny), (1, nz)
    if name in ("Fv", "v0", "fv0", "fv1", "ynut", "tf_v"):
        return (1, nx), (1, ny + 1), (1, nz)
    if name in ("Fw", "w0", "fw0", "fw1", "znut", "tf_w"):
        return (1, nx), (1, ny), (1, nz + 1)
    if name in ("bxx0", "bxx1", "bxxf", "bxxf1"):
        return (0, ny + 1), (0, nz + 1), (0, 0)
    if name in ("bxy0", "bxyf"):
        return (0, ny + 2), (0, nz + 1), (0, 0)
    if name in ("bxz0", "bxzf"):
        return (0, ny + 1), (0, nz + 2), (0, 0)
    if name in ("byx0", "byxf"):
        return (0, nx + 2), (0, nz + 1), (0, 0)
    if name in ("byy0", "byy1", "byyf", "byyf1"):
        return (0, nx + 1), (0, nz + 1), (0, 0)
    if name in ("byz0", "byzf"):
        return (0, nx + 1), (0, nz + 2), (0, 0)
    if name in ("bzx0", "bzxf"):
        return (0, nx + 2), (0, ny + 1), (0, 0)
    if name in ("bzy0", "bzyf"):
        return (0, nx + 1), (0, ny + 2), (0, 0)
    if name in ("bzz0", "bzz1", "bzzf", "bzzf1"):
        return (0, nx + 1), (0, ny + 1), (0, 0)
    raise KeyError(name)


def mask_shapes(p: SuliParams):
    """numpy shapes of the obstacle masks ku(0:nx+2, 0:ny+1), kv(0:nx+1, 0:ny+2),
    kw(0:nx+1, 0:ny+1) (0_modules.f90:76-79)."""
    return (p.nx + 3, p.ny + 2), (p.nx + 2, p.ny + 3), (p.nx + 2, p.ny + 2)


def field_shape(p: SuliParams, name: str):
    """numpy shape (Fortran order: pass order='F') of a module array."""
    return tuple(h - l + 1 for l, h in field_extent(p, name))


def default_params() -> SuliParams:
    """The reference's compiled defaults (0_modules.f90, 14_level_set.f90:25-31)."""
    import math

    p = SuliParams()
    p.dx = p.dy = p.dz = 0.02
    p.nx, p.ny, p.nz = int(0.5 / p.dx), int(1.0 / p.dy), int(0.9 / p.dz)
    p.dt = 0.001
    p.ccx0 = p.ccxf = 0
    p.ccy0 = p.ccyf = 2
    p.ccz0, p.cczf = 2, 1
    p.t_tempo, p.der, p.adv_type, p.m_turb, p.obst_t, p.t_hs = 1, 1, 1, 0, 0, 0
    p.csmag = 0.13
    decliv = 0.0002
    p.gx = 9.80665 * math.sin(math.atan(decliv))
    p.gz = 9.80665 * math.cos(math.atan(decliv))
    p.chezy = 44.5
    p.rho_f1, p.mi_f1 = 1.204, 0.000018253
    p.rho_f2, p.mi_f2 = 998.0, 0.00100798
    p.sigma = 0.0728
    p.alpha1 = 1.5
    p.dt1 = 0.1 * max(p.dx, p.dy, p.dz)
    p.reinit_maxit = 3
    p.vol_tol = 0.1
    p.cg_stop, p.cg_tol, p.cg_maxit = 0, 0.0001, 10000
    p.precision, p.refine_maxit, p.inner_tol = 0, 20, 1e-4
    p.mg_omega, p.mg_alpha = 0.9, 1.8
    return p


_LIB = None


def load_library(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load libsuli_gpu.so (built in-tree by csrc/Makefile).  Fails loudly if absent."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    lib_path = pathlib.Path(path) if path else LIB_PATH
    if not lib_path.exists():
        raise RuntimeError(
            f"libsuli_gpu.so not found at {lib_path}; build it with "
            "`make -C suli-openmp_b200/csrc` (there is no CPU fallback)")
    lib = C.CDLL(str(lib_path))
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "suli_params_default": (C.c_int, [P(SuliParams)]),
        "suli_abi_sizes": (C.c_int, [P(C.c_int), P(C.c_int)]),
        "suli_field_extent": (C.c_int, [P(SuliParams), C.c_int, P(C.c_int), P(C.c_int)]),
        "suli_create": (C.c_int, [P(SuliParams), C.c_int, P(vp)]),
        "suli_destroy": (C.c_int, [vp]),
        "suli_last_error": (C.c_char_p, [vp]),
        "suli_synchronize": (C.c_int, [vp]),
        "suli_upload": (C.c_int, [vp, C.c_int, P(C.c_double)]),
        "suli_download": (C.c_int, [vp, C.c_int, P(C.c_double)]),
        "suli_set_scalar": (C.c_int, [vp, C.c_int, C.c_double]),
        "suli_get_scalar": (C.c_int, [vp, C.c_int, P(C.c_double)]),
        "suli_iniciais": (C.c_int, [vp, C.c_double]),
        "suli_level_set_ini": (C.c_int, [vp]),
        "suli_level_set": (C.c_int, [vp, P(C.c_double)]),
        "suli_heaviside": (C.c_int, [vp]),
        "suli_mod_ls1": (C.c_int, [vp]),
        "suli_visco": (C.c_int, [vp]),
        "suli_convdiff": (C.c_int, [vp]),
        "suli_tempo": (C.c_int, [vp, C.c_int, C.c_int]),
        "suli_contorno": (C.c_int, [vp, C.c_int]),
        "suli_graddin": (C.c_int, [vp, P(C.c_int), P(C.c_double)]),
        "suli_posdin": (C.c_int, [vp]),
        "suli_est": (C.c_int, [vp, P(C.c_double)]),
        "suli_set_dt": (C.c_int, [vp, C.c_double]),
        "suli_set_obstacle": (C.c_int, [vp, P(C.c_int), P(C.c_int), P(C.c_int)]),
        "suli_boundary_waves": (C.c_int, [vp]),
        "suli_step": (C.c_int, [vp, C.c_int, P(SuliStepStats)]),
        "suli_step_host": (C.c_int, [vp, C.c_int, C.c_int, P(C.c_int), P(vp), C.c_int, P(C.c_int), P(vp),
                                     P(SuliStepStats)]),
        "suli_stream": (C.c_int, [vp, P(vp)]),
        "suli_profile_enable": (C.c_int, [vp, C.c_int]),
        "suli_profile_read": (C.c_int, [vp, P(C.c_double), P(C.c_longlong), P(C.c_longlong)]),
        "suli_est_static": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                      C.c_double, vp, vp]),
        "suli_nn_num_params": (C.c_longlong, []),
        "suli_nn_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P(vp)]),
        "suli_nn_destroy": (C.c_int, [vp]),
        "suli_nn_last_error": (C.c_char_p, [vp]),
        "suli_nn_set_params": (C.c_int, [vp, P(C.c_float), C.c_longlong]),
        "suli_nn_get_params": (C.c_int, [vp, P(C.c_float), C.c_longlong]),
        "suli_nn_forward": (C.c_int, [vp, vp, vp]),
        "suli_nn_loss_grad": (C.c_int, [vp, vp, vp, P(C.c_double), P(C.c_float)]),
        "suli_nn_train_step": (C.c_int, [vp, vp, vp, C.c_float, P(C.c_double)]),
        "suli_nn_conv3d": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, vp, C.c_int, C.c_int, vp, C.c_int]),
        "suli_nn_conv3d_ex": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, vp, C.c_int, C.c_int, vp, vp, vp,
                                        vp, C.c_int]),
        "suli_nn_set_kernel": (C.c_int, [vp, C.c_int]),
        "suli_attach_nn": (C.c_int, [vp, vp, C.c_int]),
        "suli_graddin_record": (C.c_int, [vp, vp, vp, P(C.c_int), P(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


# Exported C symbols of include/suli_gpu.h (checked by the CPU test suite).
HEADER_SYMBOLS = [
    "suli_field_extent", "suli_params_default", "suli_abi_sizes", "suli_create", "suli_destroy",
    "suli_last_error", "suli_synchronize", "suli_upload", "suli_download",
    "suli_set_scalar", "suli_get_scalar", "suli_iniciais", "suli_level_set_ini",
    "suli_level_set", "suli_heaviside", "suli_mod_ls1", "suli_visco", "suli_convdiff",
    "suli_tempo", "suli_contorno", "suli_graddin", "suli_posdin", "suli_est",
    "suli_set_dt", "suli_set_obstacle", "suli_boundary_waves", "suli_step", "suli_step_host", "suli_stream", "suli_profile_enable", "suli_profile_read",
    "suli_est_static",
    "suli_nn_num_params", "suli_nn_create", "suli_nn_destroy", "suli_nn_last_error",
    "suli_nn_set_params", "suli_nn_get_params", "suli_nn_forward", "suli_nn_loss_grad",
    "suli_nn_train_step", "suli_nn_conv3d", "suli_nn_conv3d_ex", "suli_nn_set_kernel", "suli_attach_nn", "suli_graddin_record",
]
EST_STATIC_MAX_BLOCKS = 8192   # SULI_EST_STATIC_MAX_BLOCKS
STEP_HOST_MAX_FIELDS = 8       # SULI_STEP_HOST_MAX_FIELDS

# enum suli_kernel: kernel classes of the tracing counters
KERNEL_NAMES = [
    "ls_advect", "reinit", "lsprops", "curv", "volfix", "visco", "convdiff", "tempo", "contorno",
    "cg_setup", "cg_spmv", "cg_update", "cg_final", "posdin", "est", "mg", "refine", "nn",
]
