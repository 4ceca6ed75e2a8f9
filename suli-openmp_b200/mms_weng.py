"""The reference's manufactured-solution harness, 13_mms.f90 (Weng 2009): mms_t = 1 steady,
mms_t = 2 unsteady.

Host side only, as in the reference, where it is driver code around the hot path:
  * `fields(t)`      the manufactured u, v, w, p and free surface h at the staggered points
                     (mms_i, 13_mms.f90:12-212, and the exact fields of mms, :218-338);
  * `planes(t)`      the prescribed boundary planes of mms_bc (:468-816): the exact velocity at
                     each plane's staggered position;
  * `sources(t)`     the momentum sources tf_u, tf_v, tf_w of termo_fonte1 (:819-1064) and
                     termo_fonte2 (:1070-1322), added by convdiff (6_convdiff.f90:156, 168, 183);
  * `errors(model)`  the RMS errors of mms (:392-452) over the faces (cells) whose interpolated
                     level set is positive (water), with the reference's pressure-error array
                     that is never cleared between calls;
  * `init(model)` and `step(model, it)`: the driver of 1_principal.f90:46-99 with mms_t > 0: the
                     sources at it = 1 (steady) or every step (unsteady), level_set, contorno(3),
                     and per RK stage visco, convdiff, tempo and contorno(2) only (graddin and
                     posdin are skipped when mms_t > 0, 1_principal.f90:89).

`model` is a suli_b200.Solver, or any object with the same subroutine surface (the tests pass the
CPU restatement used as their checker), driven by one sequence.

The case: the reference's fluids (14_level_set.f90:25-31) and schemes, the domain
[0, 2 pi]^2 x [0, lz] (mms_t = 1) or [-pi, pi]^2 x [0, lz] (mms_t = 2, the fields' own offsets),
free surface at h0 + a(...) with the module constants a = 0, h0 = 2, coef = 0 by default
(0_modules.f90:208-212), every wall prescribed (cc = 3) from mms_bc's planes, and no gravity
or surface tension: the sources carry neither, so the reference's own MMS check only holds with
them off.  The unsteady case leaves out the volume correction of level_set, as the reference
does for mms_t = 2 (14_level_set.f90:257).
"""
from __future__ import annotations

import math

import numpy as np

from ._abi import default_params, field_shape

PI = math.acos(-1.0)
VISC = 0.00100798 / 998.0      # the sources' kinematic viscosity (13_mms.f90:845, 1098)


def _coords(n, h, lo, hi, stag, off):
    """Coordinates (index - 1 for a staggered axis, index - 0.5 otherwise) * h - off over the
    Fortran index range lo..hi."""
    idx = np.arange(lo, hi + 1, dtype=np.float64)
    return (idx - (1.0 if stag else 0.5)) * h - off


class WengMMS:
    """One manufactured-solution case (mms_t 1 or 2) on an nx x ny x nz grid."""

    def __init__(self, mms_t: int, nx: int = 32, ny: int = 32, nz: int = 24, lz: float = 3.0, a: float = 0.0,
                 h0: float = 2.0, coef: float = 0.0, dt: float = 1e-3, t_tempo: int = 1, precision: int = 0):
        if mms_t not in (1, 2):
            raise ValueError("mms_t must be 1 (steady) or 2 (unsteady)")
        self.mms_t, self.a, self.h0, self.coef = mms_t, a, h0, coef
        p = default_params()
        p.nx, p.ny, p.nz = nx, ny, nz
        p.dx, p.dy, p.dz = 2.0 * PI / nx, 2.0 * PI / ny, lz / nz
        p.dt = dt
        p.dt1 = 0.1 * max(p.dx, p.dy, p.dz)
        p.ccx0 = p.ccxf = p.ccy0 = p.ccyf = p.ccz0 = p.cczf = 3
        p.gx = p.gz = 0.0
        p.sigma = 0.0
        p.t_tempo = t_tempo
        p.precision = precision
        if mms_t == 2:
            p.vol_tol = 1e300        # no volume correction (14_level_set.f90:257)
        self.p = p
        self.off = PI if mms_t == 2 else 0.0
        self.erro_p = np.zeros((nx, ny, nz))
        self.erro_t = 0.0
        self.history = []

    # ------------------------------------------------------------------ exact fields
    def surface(self, x, y, t):
        a, h0 = self.a, self.h0
        if self.mms_t == 1:
            return a * np.sin(x) * np.sin(y) + h0
        return a * np.cos(x * 0.5) * np.cos(y * 0.5) * math.cos(t) + h0

    def u_m(self, x, y, z, t):
        h = self.surface(x, y, t)
        if self.mms_t == 1:
            return np.sin(x) * np.cos(y) * np.sin(PI * 0.5 * z / h) - np.cos(x) * np.sin(y) * (np.cos(PI * 2. * z / h) - 1.)
        return np.sin(y) * np.cos(x * 0.5) * np.cos(x * 0.5) * np.cos(0.5 * PI * (1. - z / h)) * math.sin(t)

    def v_m(self, x, y, z, t):
        h = self.surface(x, y, t)
        if self.mms_t == 1:
            return -np.cos(x) * np.sin(y) * np.sin(PI * 0.5 * z / h) + np.sin(x) * np.cos(y) * (np.cos(PI * 2. * z / h) - 1.)
        return -np.sin(x) * np.cos(y * 0.5) * np.cos(y * 0.5) * np.cos(0.5 * PI * (1. - z / h)) * math.sin(t)

    def w_m(self, x, y, z, t):
        h = self.surface(x, y, t)
        a = self.a
        if self.mms_t == 1:
            return (-a * (np.sin(x) ** 2. * np.cos(y) ** 2. - np.cos(x) ** 2. * np.sin(y) ** 2.)
                    * (np.sin(2. * PI * z / h) - 2. * PI * z / h * np.cos(2. * PI * z / h) + 2. * PI) / (2. * PI))
        return -a * np.cos(x * 0.5) * np.cos(y * 0.5) * np.cos(0.5 * PI * (1. - z / h)) * math.sin(t)

    def p_m(self, x, y, z, t):
        """The unsteady pressure (:202, :327); the steady case never sets p_m in the reference."""
        h = self.surface(x, y, t)
        return -self.coef * np.cos(x) * np.cos(y) * np.cos(0.5 * PI * z / h)

    def _grid(self, name, lo, hi):
        """Mesh of the staggered coordinates of a field over Fortran index ranges lo..hi."""
        p = self.p
        stag = {"u": (1, 0, 0), "v": (0, 1, 0), "w": (0, 0, 1), "p": (0, 0, 0)}[name]
        x = _coords(p.nx, p.dx, lo[0], hi[0], stag[0], self.off)
        y = _coords(p.ny, p.dy, lo[1], hi[1], stag[1], self.off)
        z = _coords(p.nz, p.dz, lo[2], hi[2], stag[2], 0.0)
        return np.meshgrid(x, y, z, indexing="ij")

    def fields(self, t):
        """Exact u(1:nx1,1:ny,1:nz), v(1:nx,1:ny1,1:nz), w(1:nx,1:ny,1:nz1), p(1:nx,1:ny,1:nz)."""
        p = self.p
        nx, ny, nz = p.nx, p.ny, p.nz
        return {"u": self.u_m(*self._grid("u", (1, 1, 1), (nx + 1, ny, nz)), t),
                "v": self.v_m(*self._grid("v", (1, 1, 1), (nx, ny + 1, nz)), t),
                "w": self.w_m(*self._grid("w", (1, 1, 1), (nx, ny, nz + 1)), t),
                "p": self.p_m(*self._grid("p", (1, 1, 1), (nx, ny, nz)), t)}

    def level_set(self, t):
        """mms_i's level set h(x, y, t) - z at the cell centres."""
        X, Y, Z = self._grid("p", (1, 1, 1), (self.p.nx, self.p.ny, self.p.nz))
        return self.surface(X, Y, t) - Z

    # ------------------------------------------------------------------ mms_bc
    def planes(self, t):
        """The boundary planes of mms_bc: each plane holds the exact component at the staggered
        position of its index (bxx0 at i = 0, bxx1 at i = 1, bxxf at nx+1, bxxf1 at nx+2; the
        tangential planes at the ghost layers i = 0 and nx + 1; likewise in y and z).  As in the
        reference, the loops cover 0..n+1 of each plane's two axes, so a plane's last row along
        a staggered axis (bxy0 at j = ny+2, for one) stays 0; and in the unsteady case bzy0 and
        bzyf take the w expression at v's position (13_mms.f90:797, 809)."""
        p = self.p
        nx, ny, nz = p.nx, p.ny, p.nz
        ev = {"u": self.u_m, "v": self.v_m, "w": self.w_m}
        out = {}

        def plane(name, comp, axis, idx, lo, hi, expr=None):
            lo, hi = list(lo), list(hi)
            lo[axis] = hi[axis] = idx
            X, Y, Z = self._grid(comp, tuple(lo), tuple(hi))
            val = np.squeeze(ev[expr or comp](X, Y, Z, t), axis=axis)
            # the reference loops run over 0..n+1 on both plane axes (13_mms.f90:486-487, ...)
            ax = [d for d in range(3) if d != axis]
            lim = [(nx, ny, nz)[d] + 1 for d in ax]
            val[lim[0] + 1:, :] = 0.0
            val[:, lim[1] + 1:] = 0.0
            out[name] = val

        # x planes: (j, k) over 0..ny+1 (v: 0..ny+2), 0..nz+1 (w: 0..nz+2)
        for nm, idx in (("bxx0", 0), ("bxx1", 1), ("bxxf", nx + 1), ("bxxf1", nx + 2)):
            plane(nm, "u", 0, idx, (0, 0, 0), (0, ny + 1, nz + 1))
        plane("bxy0", "v", 0, 0, (0, 0, 0), (0, ny + 2, nz + 1))
        plane("bxz0", "w", 0, 0, (0, 0, 0), (0, ny + 1, nz + 2))
        plane("bxyf", "v", 0, nx + 1, (0, 0, 0), (0, ny + 2, nz + 1))
        plane("bxzf", "w", 0, nx + 1, (0, 0, 0), (0, ny + 1, nz + 2))
        # y planes: (i, k)
        for nm, idx in (("byy0", 0), ("byy1", 1), ("byyf", ny + 1), ("byyf1", ny + 2)):
            plane(nm, "v", 1, idx, (0, 0, 0), (nx + 1, 0, nz + 1))
        plane("byx0", "u", 1, 0, (0, 0, 0), (nx + 2, 0, nz + 1))
        plane("byz0", "w", 1, 0, (0, 0, 0), (nx + 1, 0, nz + 2))
        plane("byxf", "u", 1, ny + 1, (0, 0, 0), (nx + 2, 0, nz + 1))
        plane("byzf", "w", 1, ny + 1, (0, 0, 0), (nx + 1, 0, nz + 2))
        # z planes: (i, j)
        for nm, idx in (("bzz0", 0), ("bzz1", 1), ("bzzf", nz + 1), ("bzzf1", nz + 2)):
            plane(nm, "w", 2, idx, (0, 0, 0), (nx + 1, ny + 1, 0))
        quirk = "w" if self.mms_t == 2 else None
        plane("bzx0", "u", 2, 0, (0, 0, 0), (nx + 2, ny + 1, 0))
        plane("bzy0", "v", 2, 0, (0, 0, 0), (nx + 1, ny + 2, 0), expr=quirk)
        plane("bzxf", "u", 2, nz + 1, (0, 0, 0), (nx + 2, ny + 1, 0))
        plane("bzyf", "v", 2, nz + 1, (0, 0, 0), (nx + 1, ny + 2, 0), expr=quirk)
        return {k: v[..., None] for k, v in out.items()}

    # ------------------------------------------------------------------ termo_fonte1/2
    def sources(self, t):
        """tf_u(1:nx1,1:ny,1:nz), tf_v(1:nx,1:ny1,1:nz), tf_w(1:nx,1:ny,1:nz1)."""
        p = self.p
        nx, ny, nz = p.nx, p.ny, p.nz
        XU = self._grid("u", (1, 1, 1), (nx + 1, ny, nz))
        XV = self._grid("v", (1, 1, 1), (nx, ny + 1, nz))
        XW = self._grid("w", (1, 1, 1), (nx, ny, nz + 1))
        if self.mms_t == 1:
            return {"tf_u": self._fonte1_u(*XU), "tf_v": self._fonte1_v(*XV), "tf_w": self._fonte1_w(*XW)}
        return {"tf_u": self._fonte2_u(*XU, t), "tf_v": self._fonte2_v(*XV, t), "tf_w": self._fonte2_w(*XW, t)}

    # steady case (termo_fonte1): no time derivative
    def _h1(self, x, y):
        a, h0 = self.a, self.h0
        dhdx, dhdy = a * np.cos(x) * np.sin(y), a * np.sin(x) * np.cos(y)
        d2hdx2 = d2hdy2 = -a * np.sin(x) * np.sin(y)
        d2hdxy = a * np.cos(x) * np.cos(y)
        h1 = a * np.sin(x) * np.sin(y) + h0
        return dhdx, dhdy, d2hdx2, d2hdy2, d2hdxy, h1

    def _vel1(self, x, y, z, h1):
        a, hpi, dpi = self.a, 0.5 * PI, 2.0 * PI
        zh1 = z / h1
        u = np.sin(x) * np.cos(y) * np.sin(hpi * zh1) - np.cos(x) * np.sin(y) * (np.cos(dpi * zh1) - 1.)
        v = -np.cos(x) * np.sin(y) * np.sin(hpi * zh1) + np.sin(x) * np.cos(y) * (np.cos(dpi * zh1) - 1.)
        w = (-a * (np.sin(x) ** 2. * np.cos(y) ** 2. - np.cos(x) ** 2. * np.sin(y) ** 2.)
             * (np.sin(dpi * zh1) - dpi * zh1 * np.cos(dpi * zh1) + dpi) / dpi)
        return u, v, w

    def _fonte1_u(self, x, y, z):
        a, hpi, dpi, pi = self.a, 0.5 * PI, 2.0 * PI, PI
        sin, cos = np.sin, np.cos
        dhdx, dhdy, d2hdx2, d2hdy2, d2hdxy, h1 = self._h1(x, y)
        h2 = h1 * h1; h3 = h2 * h1; h4 = h3 * h1
        zh1 = z / h1
        ux, vx, wx = self._vel1(x, y, z, h1)
        dudx = (cos(x) * cos(y) * sin(hpi * zh1) + sin(x) * sin(y) * (cos(dpi * zh1) - 1.)
                - sin(x) * cos(y) * (hpi * z / h2) * cos(hpi * zh1) * dhdx
                - cos(x) * sin(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdx)
        dudy = (-sin(x) * sin(y) * sin(hpi * zh1) - cos(x) * cos(y) * (cos(dpi * zh1) - 1.)
                + sin(x) * cos(y) * (-hpi * z / h2) * cos(hpi * zh1) * dhdy
                + cos(x) * sin(y) * (-dpi * z / h2) * sin(dpi * zh1) * dhdy)
        dudz = (hpi / h1) * sin(x) * cos(y) * cos(hpi * zh1) + (dpi / h1) * cos(x) * sin(y) * sin(dpi * zh1)
        d2udx2 = (-ux
                  + 2. * cos(x) * cos(y) * (-hpi * z / h2) * cos(hpi * zh1) * dhdx
                  + 2. * sin(x) * sin(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdx
                  + sin(x) * cos(y) * (-(hpi * z / h2) ** 2 * sin(hpi * zh1) + (pi * z / h3) * cos(hpi * zh1)) * dhdx ** 2
                  + cos(x) * sin(y) * ((dpi * z / h2) ** 2 * cos(dpi * zh1) + 4. * pi * z / h3 * sin(dpi * zh1)) * dhdx ** 2
                  - (sin(x) * cos(y) * hpi * z / h2 * cos(hpi * zh1) + cos(x) * sin(y) * (dpi * z / h2) * sin(dpi * zh1))
                  * d2hdx2)
        d2udy2 = (-ux
                  - 2. * sin(x) * sin(y) * (-hpi * z / h2) * cos(hpi * zh1) * dhdy
                  - 2. * cos(x) * cos(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdy
                  + sin(x) * cos(y) * (-(hpi * z / h2) ** 2 * sin(hpi * zh1) + (pi * z / h3) * cos(hpi * zh1)) * dhdy ** 2
                  + cos(x) * sin(y) * ((dpi * z / h2) ** 2 * cos(dpi * zh1) + 4. * pi * z / h3 * sin(dpi * zh1)) * dhdy ** 2
                  - (sin(x) * cos(y) * hpi * z / h2 * cos(hpi * zh1) - cos(x) * sin(y) * (dpi * z / h2) * sin(dpi * zh1))
                  * d2hdy2)
        d2udz2 = (-(hpi / h1) ** 2. * sin(x) * cos(y) * sin(hpi * zh1)
                  + (dpi / h1) ** 2. * cos(x) * sin(y) * cos(dpi * zh1))
        d2vdxy = (sin(x) * cos(y) * sin(hpi * zh1) - cos(x) * sin(y) * (cos(dpi * zh1) - 1.0)
                  + sin(x) * sin(y) * (-hpi * z / h2) * cos(hpi * zh1) * dhdy
                  + cos(x) * cos(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdy
                  + cos(x) * cos(y) * (hpi * z / h2) * cos(hpi * zh1) * dhdx
                  - sin(x) * sin(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdx
                  + cos(x) * sin(y) * ((hpi * z / h2) ** 2 * sin(hpi * zh1) - (pi * z / h3) * cos(hpi * zh1)) * dhdx * dhdy
                  + sin(x) * cos(y) * (-(dpi * z / h2) ** 2 * cos(dpi * zh1) - (4. * pi * z / h3) * sin(dpi * zh1))
                  * dhdx * dhdy
                  + (cos(x) * sin(y) * (hpi * z / h2) * cos(hpi * zh1) + sin(x) * cos(y) * dpi * z / h2 * sin(dpi * zh1))
                  * d2hdxy)
        d2wdxz = (-a / dpi * sin(2. * x) * (dpi * dpi * z / h2) * sin(dpi * zh1)
                  + a / dpi * (sin(x) ** 2 * cos(y) ** 2 - cos(x) ** 2 * sin(y) ** 2)
                  * ((8. * pi * pi * z / h3) * sin(dpi * zh1) + (8. * pi * pi * pi * z * z / h4) * cos(dpi * zh1)) * dhdx)
        return (ux * dudx + vx * dudy + wx * dudz
                - VISC * (d2udx2 + d2udy2 + d2udz2 + d2udx2 + d2vdxy + d2wdxz))

    def _fonte1_v(self, x, y, z):
        a, hpi, dpi, pi = self.a, 0.5 * PI, 2.0 * PI, PI
        sin, cos = np.sin, np.cos
        dhdx, dhdy, d2hdx2, d2hdy2, d2hdxy, h1 = self._h1(x, y)
        h2 = h1 * h1; h3 = h2 * h1; h4 = h3 * h1
        zh1 = z / h1
        uy, vy, wy = self._vel1(x, y, z, h1)
        dvdx = (sin(x) * sin(y) * sin(hpi * zh1) + cos(x) * cos(y) * (cos(dpi * zh1) - 1.0)
                + cos(x) * sin(y) * (hpi * z / h2) * cos(hpi * zh1) * dhdx
                + sin(x) * cos(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdx)
        dvdy = (-cos(x) * cos(y) * sin(hpi * zh1) - sin(x) * sin(y) * (cos(dpi * zh1) - 1.0)
                + cos(x) * sin(y) * (hpi * z / h2) * cos(hpi * zh1) * dhdy
                + sin(x) * cos(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdy)
        dvdz = -(hpi / h1) * cos(x) * sin(y) * cos(hpi * zh1) - sin(x) * cos(y) * (dpi / h1) * sin(dpi * zh1)
        d2vdx2 = (-vy
                  + 2. * sin(x) * sin(y) * (-hpi * z / h2) * cos(hpi * zh1) * dhdx
                  + 2. * cos(x) * cos(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdx
                  - cos(x) * sin(y) * (-(hpi * z / h2) ** 2 * sin(hpi * zh1) + pi * z / h3 * cos(hpi * zh1)) * dhdx ** 2
                  - sin(x) * cos(y) * ((dpi * z / h2) ** 2 * cos(dpi * zh1) + 4. * pi * z / h3 * sin(dpi * zh1)) * dhdx ** 2
                  + (cos(x) * sin(y) * hpi * z / h2 * cos(hpi * zh1) + sin(x) * cos(y) * dpi * z / h2 * sin(dpi * zh1))
                  * d2hdx2)
        d2vdy2 = (-vy
                  - 2. * cos(x) * cos(y) * (-hpi * z / h2) * cos(hpi * zh1) * dhdy
                  - 2. * sin(x) * sin(y) * (dpi * z / h2) * sin(dpi * zh1) * dhdy
                  + (cos(x) * sin(y) * hpi * z / h2 * cos(hpi * zh1) + sin(x) * cos(y) * (dpi * z / h2) * sin(dpi * zh1))
                  * d2hdy2
                  + cos(x) * sin(y) * ((hpi * z / h2) ** 2 * sin(hpi * zh1) - pi * z / h3 * cos(hpi * zh1)) * dhdy * dhdy
                  - sin(x) * cos(y) * ((dpi * z / h2) ** 2 * cos(dpi * zh1) + 4. * pi * z / h3 * sin(dpi * zh1))
                  * dhdy * dhdy)
        d2vdz2 = (hpi / h1) ** 2 * cos(x) * sin(y) * sin(hpi * zh1) - sin(x) * cos(y) * (dpi / h1) ** 2 * cos(dpi * zh1)
        d2udxy = (-cos(x) * sin(y) * sin(hpi * zh1) + sin(x) * cos(y) * (cos(dpi * zh1) - 1.0)
                  + (sin(x) * sin(y) * dhdx - cos(x) * cos(y) * dhdy) * (hpi * z / h2) * cos(hpi * zh1)
                  + (sin(x) * sin(y) * dhdy - cos(x) * cos(y) * dhdx) * (dpi * z / h2) * sin(dpi * zh1)
                  - (sin(x) * cos(y) * (hpi * z / h2) * cos(hpi * zh1) + cos(x) * sin(y) * (dpi * z / h2) * sin(dpi * zh1))
                  * d2hdxy
                  + sin(x) * cos(y) * (-(hpi * z / h2) ** 2 * sin(hpi * zh1) + pi * z / h3 * cos(hpi * zh1)) * dhdx * dhdy
                  + cos(x) * sin(y) * ((dpi * z / h2) ** 2 * cos(dpi * zh1) + 4. * pi * z / h3 * sin(dpi * zh1))
                  * dhdx * dhdy)
        d2wdyz = (a / dpi * sin(2. * y) * (dpi * dpi * z / h2) * sin(dpi * zh1)
                  + a / dpi * (sin(x) ** 2 * cos(y) ** 2 - cos(x) ** 2 * sin(y) ** 2)
                  * ((8. * pi * pi * z / h3) * sin(dpi * zh1) + (8. * pi * pi * pi * z * z / h4) * cos(dpi * zh1)) * dhdy)
        return (uy * dvdx + vy * dvdy + wy * dvdz
                - VISC * (d2vdx2 + d2vdy2 + d2vdz2 + d2udxy + d2vdy2 + d2wdyz))

    def _fonte1_w(self, x, y, z):
        a, hpi, dpi, pi = self.a, 0.5 * PI, 2.0 * PI, PI
        sin, cos = np.sin, np.cos
        dhdx, dhdy, d2hdx2, d2hdy2, d2hdxy, h1 = self._h1(x, y)
        h2 = h1 * h1; h3 = h2 * h1; h4 = h3 * h1; h5 = h4 * h1
        zh1 = z / h1
        uz, vz, wz = self._vel1(x, y, z, h1)
        q = sin(x) ** 2 * cos(y) ** 2 - cos(x) ** 2 * sin(y) ** 2
        dwdx = (-a / dpi * sin(2. * x) * (sin(dpi * zh1) - (dpi * zh1) * cos(dpi * zh1) + dpi)
                + a / dpi * q * (dpi * dpi * z * z / h3) * sin(dpi * zh1) * dhdx)
        dwdy = (a / dpi * sin(2. * y) * (sin(dpi * zh1) - (dpi * zh1) * cos(dpi * zh1) + dpi)
                + a / dpi * q * (dpi * dpi * z * z / h3) * sin(dpi * zh1) * dhdy)
        dwdz = -a * dpi * z / h2 * q * sin(dpi * zh1)
        d2wdx2 = (-a / pi * cos(2. * x) * (sin(dpi * zh1) - (dpi * zh1) * cos(dpi * zh1) + dpi)
                  + a / pi * sin(2. * x) * (dpi * dpi * z * z / h3) * sin(dpi * zh1) * dhdx
                  + a / dpi * q * (-(dpi ** 3. * z ** 3. / h5) * cos(dpi * zh1) - (12. * pi * pi * z * z / h4) * sin(dpi * zh1))
                  * dhdx * dhdx
                  + a / dpi * q * (4. * pi * pi * z * z / h3) * sin(dpi * zh1) * d2hdx2)
        d2wdy2 = (a / pi * cos(2. * y) * (sin(dpi * zh1) - (dpi * zh1) * cos(dpi * zh1) + dpi)
                  - a / pi * sin(2. * y) * (dpi * dpi * z * z / h3) * sin(dpi * zh1) * dhdy
                  + a / dpi * q * (-(dpi ** 3. * z ** 3. / h5) * cos(dpi * zh1) - (12. * pi * pi * z * z / h4) * sin(dpi * zh1))
                  * dhdy * dhdy
                  + a / dpi * q * (dpi * dpi * z * z / h3) * sin(dpi * zh1) * d2hdy2)
        d2wdz2 = -a * q * (dpi * dpi * z / h3 * cos(dpi * zh1) + (dpi / h2) * sin(dpi * zh1))
        d2vdyz = (-cos(x) * cos(y) * (hpi / h1) * cos(hpi * zh1) + sin(x) * sin(y) * (dpi / h1) * sin(dpi * zh1)
                  + cos(x) * sin(y) * (-pi * pi * z / 4. / h3 * sin(hpi * zh1) + hpi / h2 * cos(hpi * zh1)) * dhdy
                  + sin(x) * cos(y) * (4. * pi * pi * z / h3 * cos(dpi * zh1) + dpi / h2 * sin(dpi * zh1)) * dhdy)
        d2udxz = (cos(x) * cos(y) * (hpi / h1) * cos(hpi * zh1) - sin(x) * sin(y) * (dpi / h1) * sin(dpi * zh1)
                  + sin(x) * cos(y) * (pi * pi * z / 4. / h3 * sin(hpi * zh1) - hpi / h2 * cos(hpi * zh1)) * dhdx
                  - cos(x) * sin(y) * (4. * pi * pi * z / h3 * cos(dpi * zh1) + dpi / h2 * sin(dpi * zh1)) * dhdx)
        return (uz * dwdx + vz * dwdy + wz * dwdz
                - VISC * (d2wdx2 + d2wdy2 + d2wdz2 + d2udxz + d2vdyz + d2wdz2))

    # unsteady case (termo_fonte2): c = cos(pi/2 (1 - z/h)) and its derivatives
    def _h2(self, x, y, z, t):
        a, h0, hpi, pi = self.a, self.h0, 0.5 * PI, PI
        sin, cos = np.sin, np.cos
        ct = math.cos(t)
        dhdx = -a * 0.5 * sin(x * 0.5) * cos(y * 0.5) * ct
        dhdy = -a * 0.5 * cos(x * 0.5) * sin(y * 0.5) * ct
        d2hdx2 = d2hdy2 = -a * 0.25 * cos(x * 0.5) * cos(y * 0.5) * ct
        d2hdxy = -a * 0.25 * sin(x * 0.5) * sin(y * 0.5) * ct
        h1 = a * cos(x * 0.5) * cos(y * 0.5) * ct + h0
        h2 = h1 * h1
        h3 = h2 * h1
        zh1 = z / h1
        c = cos(hpi * (1.0 - zh1))
        s = sin(hpi * (1.0 - zh1))
        d = {"c": c, "s": s, "h1": h1, "zh1": zh1}
        d["dcdx"] = -hpi * z / h2 * s * dhdx
        d["dcdy"] = -hpi * z / h2 * s * dhdy
        d["dcdz"] = hpi / h1 * s
        dsdx = hpi * z / h2 * c * dhdx
        dsdy = hpi * z / h2 * c * dhdy
        d["d2cdx2"] = -hpi * z / h2 * dsdx * dhdx + pi * z / h3 * s * dhdx * dhdx - hpi * z / h2 * s * d2hdx2
        d["d2cdy2"] = -hpi * z / h2 * dsdy * dhdy + pi * z / h3 * s * dhdy * dhdy - hpi * z / h2 * s * d2hdy2
        d["d2cdz2"] = -(hpi / h1) ** 2. * c
        d["d2cdxy"] = -hpi * z / h2 * dsdy * dhdx + pi * z / h3 * s * dhdx * dhdy - hpi * z / h2 * s * d2hdxy
        d["d2cdxz"] = hpi * z / h2 * hpi / h1 * c * dhdx - hpi / h2 * s * dhdx
        d["d2cdyz"] = hpi * z / h2 * hpi / h1 * c * dhdy - hpi / h2 * s * dhdy
        return d

    def _vel2(self, x, y, zh1, t):
        a, hpi = self.a, 0.5 * PI
        sin, cos = np.sin, np.cos
        st = math.sin(t)
        u = sin(y) * cos(x * 0.5) * cos(x * 0.5) * cos(hpi * (1. - zh1)) * st
        v = -sin(x) * cos(y * 0.5) * cos(y * 0.5) * cos(hpi * (1. - zh1)) * st
        w = -a * cos(x * 0.5) * cos(y * 0.5) * cos(hpi * (1. - zh1)) * st
        return u, v, w

    def _fonte2_u(self, x, y, z, t):
        a = self.a
        sin, cos = np.sin, np.cos
        st, ct = math.sin(t), math.cos(t)
        D = self._h2(x, y, z, t)
        c, dcdx, dcdy, dcdz = D["c"], D["dcdx"], D["dcdy"], D["dcdz"]
        ux, vx, wx = self._vel2(x, y, D["zh1"], t)
        dudt = sin(y) * cos(0.5 * x) * cos(0.5 * x) * c * ct
        dudx = -0.5 * sin(x) * sin(y) * c * st + sin(y) * cos(0.5 * x) * cos(0.5 * x) * dcdx * st
        dudy = cos(0.5 * x) * cos(0.5 * x) * cos(y) * c * st + sin(y) * cos(0.5 * x) * cos(0.5 * x) * dcdy * st
        dudz = cos(0.5 * x) * cos(0.5 * x) * sin(y) * dcdz * st
        d2udx2 = (-0.5 * cos(x) * sin(y) * c * st - sin(x) * sin(y) * dcdx * st
                  + sin(y) * cos(0.5 * x) * cos(0.5 * x) * D["d2cdx2"] * st)
        d2udy2 = (-cos(0.5 * x) * cos(0.5 * x) * sin(y) * c * st + 2.0 * cos(y) * cos(0.5 * x) * cos(0.5 * x) * dcdy * st
                  + sin(y) * cos(0.5 * x) * cos(0.5 * x) * D["d2cdy2"] * st)
        d2udz2 = cos(0.5 * x) * cos(0.5 * x) * sin(y) * D["d2cdz2"] * st
        d2vdxy = (0.5 * sin(y) * cos(x) * c * st + 0.5 * sin(x) * sin(y) * dcdx * st
                  - cos(0.5 * y) * cos(0.5 * y) * cos(x) * dcdy * st - sin(x) * cos(0.5 * y) * cos(0.5 * y) * D["d2cdxy"] * st)
        d2wdxz = 0.5 * a * sin(0.5 * x) * cos(0.5 * y) * dcdz * st - a * cos(0.5 * x) * cos(0.5 * y) * D["d2cdxz"] * st
        return (dudt + ux * dudx + vx * dudy + wx * dudz
                - VISC * (d2udx2 + d2udy2 + d2udz2 + d2udx2 + d2vdxy + d2wdxz))

    def _fonte2_v(self, x, y, z, t):
        a = self.a
        sin, cos = np.sin, np.cos
        st, ct = math.sin(t), math.cos(t)
        D = self._h2(x, y, z, t)
        c, dcdx, dcdy, dcdz = D["c"], D["dcdx"], D["dcdy"], D["dcdz"]
        uy, vy, wy = self._vel2(x, y, D["zh1"], t)
        dvdt = -sin(x) * cos(0.5 * y) * cos(0.5 * y) * c * ct
        dvdx = -cos(x) * cos(0.5 * y) * cos(0.5 * y) * c * st - sin(x) * cos(0.5 * y) * cos(0.5 * y) * dcdx * st
        dvdy = 0.5 * sin(x) * sin(y) * c * st - sin(x) * cos(0.5 * y) * cos(0.5 * y) * dcdy * st
        dvdz = -cos(0.5 * y) * cos(0.5 * y) * sin(x) * dcdz * st
        d2vdx2 = (sin(x) * cos(0.5 * y) * cos(0.5 * y) * c * st - 2.0 * cos(x) * cos(0.5 * y) * cos(0.5 * y) * dcdx * st
                  - sin(x) * cos(0.5 * y) * cos(0.5 * y) * D["d2cdx2"] * st)
        d2vdy2 = (0.5 * sin(x) * cos(y) * c * st + sin(x) * sin(y) * dcdy * st
                  - sin(x) * cos(0.5 * y) * cos(0.5 * y) * D["d2cdy2"] * st)
        d2vdz2 = -sin(x) * cos(0.5 * y) * cos(0.5 * y) * D["d2cdz2"] * st
        d2udxy = (-0.5 * sin(x) * cos(y) * c * st - 0.5 * sin(x) * sin(y) * dcdy * st
                  + cos(0.5 * x) * cos(0.5 * x) * cos(y) * dcdx * st + sin(y) * cos(0.5 * x) * cos(0.5 * x) * D["d2cdxy"] * st)
        d2wdyz = 0.5 * a * cos(0.5 * x) * sin(0.5 * y) * dcdz * st - a * cos(0.5 * x) * cos(0.5 * y) * D["d2cdyz"] * st
        return (dvdt + uy * dvdx + vy * dvdy + wy * dvdz
                - VISC * (d2vdx2 + d2vdy2 + d2vdz2 + d2udxy + d2vdy2 + d2wdyz))

    def _fonte2_w(self, x, y, z, t):
        a = self.a
        sin, cos = np.sin, np.cos
        st, ct = math.sin(t), math.cos(t)
        D = self._h2(x, y, z, t)
        c, dcdx, dcdy, dcdz = D["c"], D["dcdx"], D["dcdy"], D["dcdz"]
        uz, vz, wz = self._vel2(x, y, D["zh1"], t)
        dwdt = -a * cos(0.5 * x) * cos(0.5 * y) * c * ct
        dwdx = 0.5 * a * sin(0.5 * x) * cos(0.5 * y) * c * st - a * cos(0.5 * x) * cos(0.5 * y) * dcdx * st
        dwdy = 0.5 * a * cos(0.5 * x) * sin(0.5 * y) * c * st - a * cos(0.5 * x) * cos(0.5 * y) * dcdy * st
        dwdz = -a * cos(0.5 * x) * cos(0.5 * y) * dcdz * st
        d2wdx2 = (0.25 * a * cos(0.5 * x) * cos(0.5 * y) * c * st + a * sin(0.5 * x) * cos(0.5 * y) * dcdx * st
                  - a * cos(0.5 * x) * cos(0.5 * y) * D["d2cdx2"] * st)
        d2wdy2 = (0.25 * a * cos(0.5 * x) * cos(0.5 * y) * c * st + a * cos(0.5 * x) * sin(0.5 * y) * dcdy * st
                  - a * cos(0.5 * x) * cos(0.5 * y) * D["d2cdy2"] * st)
        d2wdz2 = -a * cos(0.5 * x) * cos(0.5 * y) * D["d2cdz2"] * st
        d2vdyz = 0.5 * sin(x) * sin(y) * dcdz * st - sin(x) * cos(0.5 * y) * cos(0.5 * y) * D["d2cdyz"] * st
        d2udxz = -0.5 * sin(x) * sin(y) * dcdz * st + sin(y) * cos(0.5 * x) * cos(0.5 * x) * D["d2cdxz"] * st
        return (dwdt + uz * dwdx + vz * dwdy + wz * dwdz
                - VISC * (d2wdx2 + d2wdy2 + d2wdz2 + d2udxz + d2vdyz + d2wdz2))

    # ------------------------------------------------------------------ driver
    def _upload_planes(self, model, t):
        for k, v in self.planes(t).items():
            model.upload(k, v)

    def _upload_sources(self, model, t):
        for k, v in self.sources(t).items():
            model.upload(k, v)

    def init(self, model):
        """iniciais with level_set_ini's tipo 6 (mms_i), contorno(1), contorno(3), the first
        mms() (1_principal.f90:46-51)."""
        p = self.p
        model.iniciais(0.0)
        ex = self.fields(0.0)
        for name in ("u", "v", "w"):
            full = np.zeros(field_shape(p, name))
            full[1:1 + ex[name].shape[0], 1:1 + ex[name].shape[1], 1:1 + ex[name].shape[2]] = ex[name]
            model.upload(name, full)
        if self.mms_t == 2:
            pr = np.zeros(field_shape(p, "prd1"))
            pr[1:-1, 1:-1, 1:-1] = ex["p"]
            model.upload("prd1", pr)
        model.upload("ls", self.level_set(0.0))
        model.level_set_ini()
        self._upload_planes(model, 0.0)
        model.contorno(1)
        model.contorno(3)
        return self.errors(model, 0.0)

    def step(self, model, it: int):
        """One time step of 1_principal.f90:64-99 with mms_t > 0; returns the errors of mms()."""
        p = self.p
        t = it * p.dt
        model.set_scalar("t", t)
        if self.mms_t == 1 and it == 1:
            self._upload_sources(model, t)
        if self.mms_t == 2:
            self._upload_sources(model, t)
            self._upload_planes(model, t)
        model.level_set()
        model.contorno(3)
        a_dt = model.a_dt
        for tt in range(1, model.ntt + 1):
            model.set_dt(a_dt[tt - 1])
            model.visco()
            model.convdiff()
            model.tempo(tt, it)
            model.contorno(2)
        return self.errors(model, t)

    def errors(self, model, t):
        """mms() (13_mms.f90:218-465): RMS of exact - computed over the faces whose interpolated
        level set is positive, and over the cells with ls > 0 for the pressure (its squared-error
        array keeps values from earlier calls where the cell is no longer water, as erro_p is
        never cleared); erro_t accumulates the mean velocity error."""
        p = self.p
        nx, ny, nz = p.nx, p.ny, p.nz
        ex = self.fields(t)
        ls = model.download("ls")
        # interp?_cf with the end faces copied from their neighbours (8_derivadas.f90:304-434)
        lsx = np.empty((nx + 1, ny, nz)); lsx[1:nx] = (ls[1:] + ls[:-1]) * 0.5; lsx[0] = lsx[1]; lsx[nx] = lsx[nx - 1]
        lsy = np.empty((nx, ny + 1, nz)); lsy[:, 1:ny] = (ls[:, 1:] + ls[:, :-1]) * 0.5
        lsy[:, 0] = lsy[:, 1]; lsy[:, ny] = lsy[:, ny - 1]
        lsz = np.empty((nx, ny, nz + 1)); lsz[:, :, 1:nz] = (ls[:, :, 1:] + ls[:, :, :-1]) * 0.5
        lsz[:, :, 0] = lsz[:, :, 1]; lsz[:, :, nz] = lsz[:, :, nz - 1]
        u = model.download("u")[1:nx + 2, 1:ny + 1, 1:nz + 1]
        v = model.download("v")[1:nx + 1, 1:ny + 2, 1:nz + 1]
        w = model.download("w")[1:nx + 1, 1:ny + 1, 1:nz + 2]
        out = {}
        for nm, comp, m in (("u", u, lsx > 0.), ("v", v, lsy > 0.), ("w", w, lsz > 0.)):
            e2 = np.where(m, (ex[nm] - comp) ** 2., 0.0)
            out[nm] = math.sqrt(float(e2.sum()) / max(int(m.sum()), 1))
        prd = model.download("prd1")[1:nx + 1, 1:ny + 1, 1:nz + 1]
        wet = ls > 0.
        self.erro_p[wet] = (ex["p"][wet] - prd[wet]) ** 2.
        out["p"] = math.sqrt(float(self.erro_p.sum()) / max(int(wet.sum()), 1))
        self.erro_t += (out["u"] + out["v"] + out["w"]) / 3.
        out["t"] = t
        self.history.append(out)
        return out
