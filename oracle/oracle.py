"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle*.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline as the checker.  `Oracle` exposes the same methods as suli_b200.Solver so a test
can drive both with one script.  Parity is unpinned (see suli_oracle.cpp).
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import os
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent


def _pkg():
    if "suli_b200" not in sys.modules:
        d = ROOT / "suli-openmp_b200"
        spec = importlib.util.spec_from_file_location("suli_b200", d / "__init__.py",
                                                      submodule_search_locations=[str(d)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["suli_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["suli_b200"]


def build(quiet: bool = True) -> None:
    """Compile the oracle libraries with its Makefile (gcc)."""
    subprocess.run(["make", "-C", str(HERE)], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib_path(openmp: bool = False) -> pathlib.Path:
    return HERE / "_build" / ("liboracle_omp.so" if openmp else "liboracle.so")


_LIBS = {}


def load(openmp: bool = False) -> C.CDLL:
    if openmp in _LIBS:
        return _LIBS[openmp]
    path = lib_path(openmp)
    if not path.exists():
        build()
    abi = _pkg()._abi
    lib = C.CDLL(str(path))
    vp, P, d, i = C.c_void_p, C.POINTER, C.c_double, C.c_int
    sig = {
        "orc_create": (vp, [P(abi.SuliParams)]),
        "orc_destroy": (None, [vp]),
        "orc_upload": (i, [vp, i, P(d)]),
        "orc_download": (i, [vp, i, P(d)]),
        "orc_set_scalar": (i, [vp, i, d]),
        "orc_get_scalar": (i, [vp, i, P(d)]),
        "orc_iniciais": (i, [vp, d]),
        "orc_level_set_ini": (i, [vp]),
        "orc_level_set": (i, [vp, P(d)]),
        "orc_heaviside": (i, [vp]),
        "orc_mod_ls1": (i, [vp]),
        "orc_volume": (i, [vp, P(d)]),
        "orc_der_weno": (i, [vp, i, P(d)]),
        "orc_reinic_weno": (i, [vp, P(i)]),
        "orc_visco": (i, [vp]),
        "orc_convdiff": (i, [vp]),
        "orc_tempo": (i, [vp, i, i]),
        "orc_contorno": (i, [vp, i]),
        "orc_graddin": (i, [vp, P(i), P(d)]),
        "orc_posdin": (i, [vp]),
        "orc_est": (i, [vp, P(d)]),
        "orc_set_dt": (i, [vp, d]),
        "orc_step": (i, [vp, i, P(abi.SuliStepStats)]),
        "orc_last_reinit_iters": (i, [vp]),
        "orc_num_threads": (i, []),
        "orc_set_obstacle": (i, [vp, P(i), P(i), P(i)]),
        "orc_boundary_waves": (i, [vp]),
        "orc_field_extent": (i, [P(abi.SuliParams), i, P(i), P(i)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIBS[openmp] = lib
    return lib


class Oracle:
    """CPU restatement with the Solver surface."""

    def __init__(self, params, openmp: bool = False):
        abi = _pkg()._abi
        self._abi = abi
        self.lib = load(openmp)
        self.params = params.copy()
        self._h = self.lib.orc_create(C.byref(self.params))
        if not self._h:
            raise ValueError("oracle: bad parameters")

    def close(self):
        if getattr(self, "_h", None):
            self.lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, name):
        return self._abi.field_shape(self.params, name)

    def upload(self, name, arr):
        a = np.asfortranarray(np.broadcast_to(np.asarray(arr, dtype=np.float64), self.shape(name)),
                              dtype=np.float64)
        rc = self.lib.orc_upload(self._h, self._abi.FIELD[name], a.ctypes.data_as(C.POINTER(C.c_double)))
        assert rc == 0

    def download(self, name):
        out = np.empty(self.shape(name), dtype=np.float64, order="F")
        rc = self.lib.orc_download(self._h, self._abi.FIELD[name], out.ctypes.data_as(C.POINTER(C.c_double)))
        assert rc == 0
        return out

    def set_scalar(self, name, v):
        assert self.lib.orc_set_scalar(self._h, self._abi.SCALAR[name], float(v)) == 0

    def get_scalar(self, name):
        v = C.c_double()
        assert self.lib.orc_get_scalar(self._h, self._abi.SCALAR[name], C.byref(v)) == 0
        return v.value

    @property
    def ntt(self):
        return int(self.get_scalar("ntt"))

    @property
    def a_dt(self):
        return [self.get_scalar("a_dt1"), self.get_scalar("a_dt2"), self.get_scalar("a_dt3")]

    def synchronize(self):
        pass

    def set_obstacle(self, ku, kv, kw):
        """Obstacle masks (integer arrays in Fortran layout, see suli_set_obstacle)."""
        m = [np.asfortranarray(a, dtype=np.int32) for a in (ku, kv, kw)]
        for a, s in zip(m, self._abi.mask_shapes(self.params)):
            if a.shape != s:
                raise ValueError(f"mask shape {a.shape} != {s}")
        rc = self.lib.orc_set_obstacle(self._h, *[a.ctypes.data_as(C.POINTER(C.c_int)) for a in m])
        if rc != 0:
            raise ValueError("oracle: mask values out of range")
        self.obstacle = tuple(a.copy() for a in m)

    def boundary_waves(self):
        assert self.lib.orc_boundary_waves(self._h) == 0

    def iniciais(self, u_init=0.0):
        self.lib.orc_iniciais(self._h, float(u_init))

    def level_set_ini(self):
        self.lib.orc_level_set_ini(self._h)

    def level_set(self):
        v = C.c_double()
        self.lib.orc_level_set(self._h, C.byref(v))
        return v.value

    def heaviside(self):
        self.lib.orc_heaviside(self._h)

    def mod_ls1(self):
        self.lib.orc_mod_ls1(self._h)

    def volume(self):
        v = C.c_double()
        self.lib.orc_volume(self._h, C.byref(v))
        return v.value

    def der_weno(self, name="ls"):
        n = int(np.prod(self.shape("ls")))
        out = np.empty(6 * n, dtype=np.float64)
        assert self.lib.orc_der_weno(self._h, self._abi.FIELD[name], out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        return [out[m * n:(m + 1) * n].reshape(self.shape("ls"), order="F") for m in range(6)]

    def reinic_weno(self):
        it = C.c_int()
        self.lib.orc_reinic_weno(self._h, C.byref(it))
        return it.value

    def visco(self):
        self.lib.orc_visco(self._h)

    def convdiff(self):
        self.lib.orc_convdiff(self._h)

    def tempo(self, tt, it):
        self.lib.orc_tempo(self._h, int(tt), int(it))

    def contorno(self, nlock):
        self.lib.orc_contorno(self._h, int(nlock))

    def graddin(self):
        n, r = C.c_int(), C.c_double()
        self.lib.orc_graddin(self._h, C.byref(n), C.byref(r))
        return n.value, r.value

    def posdin(self):
        self.lib.orc_posdin(self._h)

    def est(self):
        v = C.c_double()
        self.lib.orc_est(self._h, C.byref(v))
        return v.value

    def set_dt(self, dt):
        self.lib.orc_set_dt(self._h, float(dt))

    def step(self, it):
        st = self._abi.SuliStepStats()
        self.lib.orc_step(self._h, int(it), C.byref(st))
        return {"cg_iters": list(st.cg_iters), "cg_resid": list(st.cg_resid),
                "vol_ins": st.vol_ins, "max_div": st.max_div, "status": st.status}

    @property
    def last_reinit_iters(self):
        return self.lib.orc_last_reinit_iters(self._h)


def num_threads(openmp: bool = True) -> int:
    return load(openmp).orc_num_threads()
