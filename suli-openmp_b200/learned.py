"""The learned initial guess of the pressure solve: a 3-D U-Net run by libsuli_gpu.so.

`Net` wraps the library's `suli_nn` object (include/suli_gpu.h): forward passes, the loss
and its gradient, Adam steps, all on the GPU through the project's own kernels (BF16
implicit-GEMM convolutions on the tensor cores, FP32 accumulation and master weights).
`Solver.attach_nn(net)` makes a mixed-precision solver start each pressure solve from
e0 + alpha * s * net(features) instead of e0 (the previous pressure); the solve still stops on
the same FP64 residual test.

Architecture (conv layers in order, 3x3x3, ReLU; 2x2x2 average pooling between encoder
levels; nearest upsampling and skip concatenation in the decoder; a 1x1x1 head):
level channels 16/32/64/96, input 3 channels padded to 16.  Parameter vector layout: per
layer W[27][Cout][Cin] (tap = dx + 3 dy + 9 dz) then bias[Cout]; head w[16], b.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

from . import _abi

LAYERS = [  # (cin, cout, level)
    (16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 96, 3),
    (96, 96, 3), (160, 64, 2), (64, 64, 2), (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0),
]
IN_CHANNELS = 3
WEIGHTS_PATH = pathlib.Path(__file__).resolve().parent / "weights" / "unet_pressure.npy"


def num_params() -> int:
    return sum(27 * co * ci + co for ci, co, _ in LAYERS) + 17


def init_params(seed: int = 0, head_scale: float = 0.1) -> np.ndarray:
    """He-normal conv weights (fan-in of the real input channels), zero biases, a small head."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (ci, co, _) in enumerate(LAYERS):
        fan = 27 * (IN_CHANNELS if l == 0 else ci)
        W = rng.standard_normal((27, co, ci)).astype(np.float32) * np.float32(np.sqrt(2.0 / fan))
        if l == 0:
            W[:, :, IN_CHANNELS:] = 0.0
        parts += [W.ravel(), np.zeros(co, np.float32)]
    parts += [rng.standard_normal(16).astype(np.float32) * np.float32(head_scale), np.zeros(1, np.float32)]
    out = np.concatenate(parts)
    assert out.size == num_params()
    return out


def _ptr(x) -> int:
    """Device address of a torch tensor, or an integer address as given."""
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    return int(x)


class NetError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Net:
    """One network for an nx x ny x nz grid (multiples of 8) on `device`."""

    def __init__(self, nx: int, ny: int, nz: int, device: int = 0, params: np.ndarray | None = None,
                 lib_path=None):
        self.lib = _abi.load_library(lib_path)
        self.shape = (nx, ny, nz)
        h = C.c_void_p()
        rc = self.lib.suli_nn_create(int(nx), int(ny), int(nz), int(device), C.byref(h))
        if rc != 0:
            raise NetError(rc, f"suli_nn_create({nx}, {ny}, {nz}) failed")
        self._h = h
        self.n = int(self.lib.suli_nn_num_params())
        if params is not None:
            self.set_params(params)

    @classmethod
    def load(cls, nx: int, ny: int, nz: int, device: int = 0, path=None) -> "Net":
        """A network with the trained weights shipped in the package (or `path`)."""
        w = np.load(pathlib.Path(path) if path else WEIGHTS_PATH)
        return cls(nx, ny, nz, device, params=w)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.suli_nn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            msg = self.lib.suli_nn_last_error(self._h)
            raise NetError(rc, f"{what}: {msg.decode() if msg else ''}")

    def set_params(self, w: np.ndarray) -> None:
        a = np.ascontiguousarray(w, dtype=np.float32)
        if a.size != self.n:
            raise ValueError(f"expected {self.n} parameters, got {a.size}")
        self._check(self.lib.suli_nn_set_params(self._h, a.ctypes.data_as(C.POINTER(C.c_float)), self.n),
                    "set_params")

    def get_params(self) -> np.ndarray:
        a = np.empty(self.n, np.float32)
        self._check(self.lib.suli_nn_get_params(self._h, a.ctypes.data_as(C.POINTER(C.c_float)), self.n),
                    "get_params")
        return a

    def save(self, path) -> None:
        p = pathlib.Path(path)
        p.parent.mkdir(parents=True, exist_ok=True)
        np.save(p, self.get_params())

    def forward(self, in3, out) -> None:
        """out[V] = net(in3[V][3]) on device buffers (FP32, x fastest)."""
        self._check(self.lib.suli_nn_forward(self._h, C.c_void_p(_ptr(in3)), C.c_void_p(_ptr(out))), "forward")

    def loss_grad(self, in3, target, grad: bool = True):
        """Mean squared error against `target` and (if asked) its parameter gradient."""
        loss = C.c_double()
        g = np.empty(self.n, np.float32) if grad else None
        gp = g.ctypes.data_as(C.POINTER(C.c_float)) if grad else None
        self._check(self.lib.suli_nn_loss_grad(self._h, C.c_void_p(_ptr(in3)), C.c_void_p(_ptr(target)),
                                               C.byref(loss), gp), "loss_grad")
        return loss.value, g

    def set_kernel(self, kernel: int) -> None:
        """Convolution kernel: 0 = the pipelined tcgen05 kernel (TMA loads, accumulators in TMEM,
        the default), 1 = mma.sync, 2 = tcgen05 with one tile per CTA."""
        self._check(self.lib.suli_nn_set_kernel(self._h, int(kernel)), "set_kernel")

    def train_step(self, in3, target, lr: float) -> float:
        """One Adam step; returns the loss before the step."""
        loss = C.c_double()
        self._check(self.lib.suli_nn_train_step(self._h, C.c_void_p(_ptr(in3)), C.c_void_p(_ptr(target)),
                                                float(lr), C.byref(loss)), "train_step")
        return loss.value


def conv3d(x, w, bias, out, shape, cin: int, cout: int, relu: bool = False, kernel: int = 0,
           lib_path=None, pool=None, head_w=None, head_out=None) -> None:
    """The convolution primitive on device buffers (channels-last BF16, see suli_nn_conv3d_ex);
    kernel 0 = pipelined tcgen05, 1 = mma.sync, 2 = tcgen05 one tile per CTA.  `pool` (BF16
    [V/8][cout]) receives the 2x2x2 average of the output, `head_w` (17 FP32) / `head_out` (FP32
    [V]) the 1x1x1 head, as the network fuses them into its convolutions."""
    lib = _abi.load_library(lib_path)
    nx, ny, nz = shape
    opt = lambda a: C.c_void_p(_ptr(a)) if a is not None else None
    rc = lib.suli_nn_conv3d_ex(int(nx), int(ny), int(nz), C.c_void_p(_ptr(x)), int(cin), C.c_void_p(_ptr(w)),
                               opt(bias), int(cout), int(relu), C.c_void_p(_ptr(out)), opt(pool), opt(head_w),
                               opt(head_out), int(kernel))
    if rc != 0:
        raise NetError(rc, "suli_nn_conv3d_ex failed")
