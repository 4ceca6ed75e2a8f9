"""Random two-phase pressure problems: the training data of the learned initial guess.

Each snapshot is a closed tank of n^3 cells holding water (rho 1000) under air (rho 1.2):
a flat or sinusoidal free surface plus 1-4 ellipsoidal water bodies with semi-axes uniform
in 0.1-0.4 of the domain, and a velocity field of Gaussian-smoothed white noise (sigma = 3
cells, zero normal velocity on the walls) whose divergence is the Poisson right-hand side.
A pair of solves per snapshot mimics a time step: the first starts from zero pressure, the
second from the first one's converged pressure with a correlated velocity field.  Every
solve goes through `Solver.graddin_record`, so the network sees exactly the features the
solver computes, and the targets are the solver's own converged FP64 solutions.

The fields are generated on the GPU (torch tensors) and handed to the solver by device
pointer; nothing here is on the time-step path.
"""
from __future__ import annotations

import math

from ._abi import field_shape
from .cases import _two_phase
from ._abi import default_params


def tank_params(n: int = 128, dx: float = 0.005, cg_tol: float = 1e-8, precision: int = 1, ny: int | None = None,
                nz: int | None = None):
    """Closed tank, no-slip walls and a free-slip lid, as the sloshing case (n^3 cells, or
    n x ny x nz)."""
    p = default_params()
    p.nx = n
    p.ny = ny if ny else n
    p.nz = nz if nz else n
    p.dx = p.dy = p.dz = dx
    p.ccx0 = p.ccxf = 2
    p.ccy0 = p.ccyf = 2
    p.ccz0, p.cczf = 2, 1
    _two_phase(p, cs=0.1)
    p.cg_tol = cg_tol
    p.dt = 0.25 * dx / math.sqrt(9.81 * 0.32)
    p.precision = precision
    return p


class SnapshotGenerator:
    """Draws snapshots for one solver (`Solver` of `tank_params`) with a torch generator."""

    def __init__(self, solver, seed: int, device: str = "cuda:0"):
        import torch
        self.torch = torch
        self.s = solver
        self.p = solver.params
        self.dev = device
        self.g = torch.Generator(device=device)
        self.g.manual_seed(int(seed))
        n0, n1, n2 = self.p.nx, self.p.ny, self.p.nz
        self.V = n0 * n1 * n2
        T = torch
        dx = self.p.dx
        # cell centres, array order (z, y, x) = Fortran order of (x, y, z)
        z = (T.arange(n2, device=device, dtype=T.float64) + 0.5) * dx
        y = (T.arange(n1, device=device, dtype=T.float64) + 0.5) * dx
        x = (T.arange(n0, device=device, dtype=T.float64) + 0.5) * dx
        self.Z, self.Y, self.X = T.meshgrid(z, y, x, indexing="ij")
        self.L = (n0 * dx, n1 * dx, n2 * dx)

    def _u(self, lo, hi):
        return float(lo + (hi - lo) * self.torch.rand((), generator=self.g, device=self.dev, dtype=self.torch.float64))

    def level_set(self):
        """Signed-distance-like level set, positive in water."""
        T = self.torch
        Lx, Ly, Lz = self.L
        depth = self._u(0.15, 0.6) * Lz
        ls = depth - self.Z
        if self._u(0, 1) < 0.5:   # sinusoidal surface
            amp = self._u(0.01, 0.08) * Lz
            kx, ky = int(self._u(1, 3.999)), int(self._u(0, 2.999))
            ph = self._u(0, 2 * math.pi)
            ls = ls + amp * T.cos(kx * math.pi * self.X / Lx + ph) * T.cos(ky * math.pi * self.Y / Ly)
        for _ in range(int(self._u(1, 4.999))):
            a = [self._u(0.1, 0.4) * L for L in self.L]
            c = [self._u(0, 1) * L for L in self.L]
            r = T.sqrt(((self.X - c[0]) / a[0]) ** 2 + ((self.Y - c[1]) / a[1]) ** 2 + ((self.Z - c[2]) / a[2]) ** 2)
            ls = T.maximum(ls, (1.0 - r) * min(a))
        return ls

    def _smooth_noise(self, shape, sigma=3.0):
        T = self.torch
        w = T.randn(shape, generator=self.g, device=self.dev, dtype=T.float64)
        f = T.fft.rfftn(w)
        k = [T.fft.fftfreq(shape[0], device=self.dev, dtype=T.float64),
             T.fft.fftfreq(shape[1], device=self.dev, dtype=T.float64),
             T.fft.rfftfreq(shape[2], device=self.dev, dtype=T.float64)]
        K2 = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
        f = f * T.exp(-2.0 * (math.pi * sigma) ** 2 * K2)
        out = T.fft.irfftn(f, s=shape)
        return out / out.std()

    def velocity(self):
        """u, v, w in Fortran layout (torch arrays in reversed index order), walls closed."""
        out = {}
        for name, axis in (("u", 0), ("v", 1), ("w", 2)):
            sh = field_shape(self.p, name)           # Fortran (n0, n1, n2)
            a = self._smooth_noise((sh[2], sh[1], sh[0]))
            # normal velocity on the wall faces (index 1 and n + 1 of the face axis) is zero
            n = (self.p.nx, self.p.ny, self.p.nz)[axis]
            dim = 2 - axis
            a.index_fill_(dim, self.torch.tensor([1, n + 1], device=self.dev), 0.0)
            out[name] = a.contiguous()
        return out

    def draw(self, mix: float = 0.5):
        """One snapshot: level set and the velocity fields of its two solves."""
        ls = self.level_set()
        v1 = self.velocity()
        v2 = self.velocity()
        c = 1.0 / math.sqrt(1.0 + mix * mix)
        v2 = {k: ((v1[k] + mix * v2[k]) * c).contiguous() for k in v1}
        return ls.contiguous(), v1, v2

    def load_density(self, ls):
        """Level set -> Heaviside density; previous pressure zero."""
        self.s.upload_device("ls", ls)
        self.s.heaviside()
        self.s.upload("prd1", 0.0)

    def load_velocity(self, vel):
        for name, a in vel.items():
            self.s.upload_device(name, a)

    def solve_pair(self, snap, solve):
        """Run `solve(k)` (k = 0, 1) on the two solves of a snapshot: the first from zero
        pressure, the second from the first one's converged pressure."""
        ls, v1, v2 = snap
        self.load_density(ls)
        self.load_velocity(v1)
        out = [solve(0)]
        self.load_velocity(v2)
        out.append(solve(1))
        return out

    def pair(self, in3, target):
        """Record the two training pairs of a fresh snapshot into in3[k], target[k] (device
        tensors).  Returns [(iterations, relative residual)] of the two solves."""
        return self.solve_pair(self.draw(),
                               lambda k: self.s.graddin_record(in3[k].data_ptr(), target[k].data_ptr()))
