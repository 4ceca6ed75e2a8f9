"""Host-side mirror of the reference's subroutine surface over libsuli_gpu.so.

`Solver` keeps the names and call order of SuLi-IC (1_principal.f90:36-108): a driver
written against the Fortran program reads the same here —

    s = Solver(params)
    s.iniciais(u_init); s.upload("ls", ls0); s.level_set_ini()
    s.contorno(1); s.contorno(3)
    for it in range(1, ts + 1):
        s.level_set(); s.contorno(3)
        for tt in range(1, s.ntt + 1):
            s.set_dt(s.a_dt[tt - 1])
            s.visco(); s.convdiff(); s.tempo(tt, it); s.contorno(2)
            s.graddin(); s.posdin(); s.contorno(1)

or simply `s.step(it)`.  Every call goes through the C-ABI (include/suli_gpu.h); the fields
stay on the GPU and only the arrays a caller asks for are copied.  A missing library or
device raises; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import FIELD, SCALAR, SuliParams, SuliStepStats


class SuliError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Solver:
    """One solver context (one CUDA stream, all fields resident in HBM)."""

    def __init__(self, params: SuliParams, device: int = 0, lib_path=None):
        self.lib = _abi.load_library(lib_path)
        self.params = params.copy()
        h = C.c_void_p()
        rc = self.lib.suli_create(C.byref(self.params), int(device), C.byref(h))
        if rc != 0:
            raise SuliError(rc, "suli_create failed (see stderr)")
        self._h = h
        self.last_status = 0

    # ---------------------------------------------------------------- plumbing
    def close(self):
        if getattr(self, "_h", None):
            self.lib.suli_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str) -> int:
        if rc < 0:
            msg = self.lib.suli_last_error(self._h)
            raise SuliError(rc, f"{what}: {msg.decode() if msg else ''}")
        self.last_status = rc
        return rc

    def shape(self, name: str):
        return _abi.field_shape(self.params, name)

    def upload(self, name: str, arr) -> None:
        a = np.asfortranarray(arr, dtype=np.float64)
        if a.shape != self.shape(name):
            a = np.asfortranarray(np.broadcast_to(a, self.shape(name)), dtype=np.float64)
        ptr = a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.suli_upload(self._h, FIELD[name], ptr), f"upload {name}")

    def upload_device(self, name: str, t) -> None:
        """Copy a field from device memory: `t` is a contiguous float64 torch tensor whose
        shape is the field's Fortran shape reversed (so its memory order is Fortran order)."""
        want = tuple(reversed(self.shape(name)))
        if tuple(t.shape) != want or str(t.dtype) != "torch.float64" or not t.is_contiguous():
            raise ValueError(f"upload_device {name}: need contiguous float64 of shape {want}")
        import torch
        torch.cuda.synchronize(t.device)   # the library copies on its own stream
        ptr = C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))
        self._check(self.lib.suli_upload(self._h, FIELD[name], ptr), f"upload {name}")

    def download(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """Copy a field to the host (into `out` if given: Fortran-ordered float64, e.g. a
        view of pinned memory)."""
        if out is None:
            out = np.empty(self.shape(name), dtype=np.float64, order="F")
        elif out.shape != self.shape(name) or out.dtype != np.float64 or not out.flags.f_contiguous:
            raise ValueError(f"download {name}: out must be float64, Fortran-ordered, {self.shape(name)}")
        ptr = out.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.suli_download(self._h, FIELD[name], ptr), f"download {name}")
        return out

    def set_scalar(self, name: str, v: float) -> None:
        self._check(self.lib.suli_set_scalar(self._h, SCALAR[name], float(v)), f"set {name}")

    def get_scalar(self, name: str) -> float:
        v = C.c_double()
        self._check(self.lib.suli_get_scalar(self._h, SCALAR[name], C.byref(v)), f"get {name}")
        return v.value

    @property
    def ntt(self) -> int:
        return int(self.get_scalar("ntt"))

    @property
    def a_dt(self):
        return [self.get_scalar("a_dt1"), self.get_scalar("a_dt2"), self.get_scalar("a_dt3")]

    def synchronize(self) -> None:
        self._check(self.lib.suli_synchronize(self._h), "synchronize")

    @property
    def stream_ptr(self) -> int:
        """cudaStream_t of this context (e.g. for torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        self._check(self.lib.suli_stream(self._h, C.byref(s)), "stream")
        return int(s.value or 0)

    def profile_enable(self, on: bool = True) -> None:
        self._check(self.lib.suli_profile_enable(self._h, int(bool(on))), "profile_enable")

    def profile_read(self) -> dict:
        """Per kernel class: {'ms': device milliseconds, 'launches': n}; plus 'cg_iterations'."""
        n = len(_abi.KERNEL_NAMES)
        ms = (C.c_double * n)()
        la = (C.c_longlong * n)()
        it = C.c_longlong()
        self._check(self.lib.suli_profile_read(self._h, ms, la, C.byref(it)), "profile_read")
        out = {k: {"ms": ms[i], "launches": la[i]} for i, k in enumerate(_abi.KERNEL_NAMES)}
        out["cg_iterations"] = it.value
        return out

    # ---------------------------------------------------------------- reference surface
    def set_obstacle(self, ku, kv, kw) -> None:
        """Bottom-obstacle masks (integer arrays in Fortran layout, shapes _abi.mask_shapes);
        needs obst_t != 0, before iniciais.  See cases.obstaculo for the reference's presets."""
        m = [np.asfortranarray(a, dtype=np.int32) for a in (ku, kv, kw)]
        for a, s in zip(m, _abi.mask_shapes(self.params)):
            if a.shape != s:
                raise ValueError(f"mask shape {a.shape} != {s}")
        P = C.POINTER(C.c_int)
        self._check(self.lib.suli_set_obstacle(self._h, *[a.ctypes.data_as(P) for a in m]), "set_obstacle")
        self.obstacle = tuple(a.copy() for a in m)

    def boundary_waves(self) -> None:
        self._check(self.lib.suli_boundary_waves(self._h), "boundary_waves")

    def iniciais(self, u_init: float = 0.0) -> None:
        self._check(self.lib.suli_iniciais(self._h, float(u_init)), "iniciais")

    def level_set_ini(self) -> None:
        self._check(self.lib.suli_level_set_ini(self._h), "level_set_ini")

    def level_set(self) -> float:
        v = C.c_double()
        self._check(self.lib.suli_level_set(self._h, C.byref(v)), "level_set")
        return v.value

    def heaviside(self) -> None:
        self._check(self.lib.suli_heaviside(self._h), "heaviside")

    def mod_ls1(self) -> None:
        self._check(self.lib.suli_mod_ls1(self._h), "mod_ls1")

    def visco(self) -> None:
        self._check(self.lib.suli_visco(self._h), "visco")

    def convdiff(self) -> None:
        self._check(self.lib.suli_convdiff(self._h), "convdiff")

    def tempo(self, tt: int, it: int) -> None:
        self._check(self.lib.suli_tempo(self._h, int(tt), int(it)), "tempo")

    def contorno(self, nlock: int) -> None:
        self._check(self.lib.suli_contorno(self._h, int(nlock)), "contorno")

    def graddin(self):
        n = C.c_int()
        r = C.c_double()
        self._check(self.lib.suli_graddin(self._h, C.byref(n), C.byref(r)), "graddin")
        return n.value, r.value

    def graddin_record(self, in3_ptr: int, target_ptr: int):
        """graddin() that also writes the network's training pair for this solve into device
        buffers: in3 [V][3] FP32 (input features) and target [V] FP32 (scaled correction)."""
        import torch
        torch.cuda.synchronize()   # buffers from torch's allocator: its pending work first
        n = C.c_int()
        r = C.c_double()
        self._check(self.lib.suli_graddin_record(self._h, C.c_void_p(in3_ptr), C.c_void_p(target_ptr),
                                                 C.byref(n), C.byref(r)), "graddin_record")
        return n.value, r.value

    def attach_nn(self, net, mode: int = 1) -> None:
        """Use `net` (a `learned.Net` of the same grid) as the pressure solve's initial guess
        (mode 1, precision 1), also as the preconditioner of the outer refinement iteration
        (mode 2), or detach it (mode 0 / net None)."""
        if net is None or mode == 0:
            self._check(self.lib.suli_attach_nn(self._h, None, 0), "attach_nn")
            self._net = None
            return
        self._check(self.lib.suli_attach_nn(self._h, net.handle, int(mode)), "attach_nn")
        self._net = net   # keep the network alive while attached

    def posdin(self) -> None:
        self._check(self.lib.suli_posdin(self._h), "posdin")

    def est(self) -> float:
        v = C.c_double()
        self._check(self.lib.suli_est(self._h, C.byref(v)), "est")
        return v.value

    def set_dt(self, dt: float) -> None:
        self._check(self.lib.suli_set_dt(self._h, float(dt)), "set_dt")

    @staticmethod
    def _stats(st) -> dict:
        return {
            "cg_iters": list(st.cg_iters),
            "cg_resid": list(st.cg_resid),
            "vol_ins": st.vol_ins,
            "max_div": st.max_div,
            "status": st.status,
        }

    def step(self, it: int) -> dict:
        st = SuliStepStats()
        self._check(self.lib.suli_step(self._h, int(it), C.byref(st)), "step")
        return self._stats(st)

    def step_host(self, it: int, inputs: dict, outputs: dict) -> dict:
        """One time step with the state in host arrays (suli_step_host): every array of
        `inputs` is copied in before the fields it feeds are read, every array of `outputs`
        receives its field after the step; the copies overlap the step where its order allows.
        Arrays are float64, Fortran-ordered, of the field's shape (pinned memory, e.g. a
        numpy view of a pinned torch tensor, lets the copies overlap)."""
        def lists(d, what):
            if len(d) > _abi.STEP_HOST_MAX_FIELDS:
                raise ValueError(f"step_host: at most {_abi.STEP_HOST_MAX_FIELDS} {what} fields")
            ids, ptrs = [], []
            for name, a in d.items():
                if a.shape != self.shape(name) or a.dtype != np.float64 or not a.flags.f_contiguous:
                    raise ValueError(f"step_host {name}: need float64, Fortran-ordered, {self.shape(name)}")
                ids.append(FIELD[name])
                ptrs.append(a.ctypes.data)
            n = len(ids)
            return n, (C.c_int * max(n, 1))(*ids), (C.c_void_p * max(n, 1))(*ptrs)
        n_in, f_in, p_in = lists(inputs, "input")
        n_out, f_out, p_out = lists(outputs, "output")
        st = SuliStepStats()
        self._check(self.lib.suli_step_host(self._h, int(it), n_in, f_in, p_in, n_out, f_out, p_out, C.byref(st)),
                    "step_host")
        return self._stats(st)
