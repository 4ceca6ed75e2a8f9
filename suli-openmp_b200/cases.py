"""Synthetic cases: parameters and initial state of the workloads this library is run on.

The reference sets its cases at compile time (0_modules.f90, level_set_ini presets at
14_level_set.f90:75-195).  Here each case is a function returning a `SuliParams` and an
`init(model)` that writes the initial state through the same calls the Fortran program makes
(iniciais, level_set_ini, contorno(1), contorno(3); 1_principal.f90:36-47).  `model` is any
object with the Solver surface.
All inputs are seeded and synthetic; no external dataset is involved.
"""
from __future__ import annotations

import math

import numpy as np

from ._abi import SuliParams, default_params


def _centres(p: SuliParams):
    x = (np.arange(1, p.nx + 1) - 0.5) * p.dx
    y = (np.arange(1, p.ny + 1) - 0.5) * p.dy
    z = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    return np.meshgrid(x, y, z, indexing="ij")


def _two_phase(p: SuliParams, *, cs=0.1, cfl_dt=None):
    """Water/air as the benchmark cases state them: rho 1000/1.2, mu 1e-3/1.8e-5."""
    p.rho_f1, p.mi_f1 = 1.2, 1.8e-5
    p.rho_f2, p.mi_f2 = 1000.0, 1e-3
    p.gx, p.gz = 0.0, 9.81
    p.m_turb, p.csmag = 1, cs
    p.t_tempo = 2                      # RK3
    p.cg_stop, p.cg_maxit = 1, 20000   # relative residual test
    p.dt1 = 0.1 * max(p.dx, p.dy, p.dz)
    return p


def standard_init(model, ls0: np.ndarray, u_init: float = 0.0):
    """iniciais + level-set preset + level_set_ini + contorno(1), contorno(3)."""
    model.iniciais(u_init)
    model.upload("ls", ls0)
    model.level_set_ini()
    model.contorno(1)
    model.contorno(3)


def dam_break(nx=64, ny=32, nz=48, dx=0.01, cg_tol=1e-10):
    """Plain FP64 3-D dam break: water box 0.25 x 0.32 x 0.30 m against the x = 0 wall.

    ls is the signed distance to the water region (positive in water, the reference's
    convention, 14_level_set.f90:26-29), counting only its free faces x = 0.25, z = 0.30.
    No-slip walls, free-slip top, RK3; dt from CFL 0.2 with the shallow-water speed
    sqrt(g H) of the column, fixed over the run.
    """
    p = default_params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dx = p.dy = p.dz = dx
    p.ccx0 = p.ccxf = 2
    p.ccy0 = p.ccyf = 2
    p.ccz0, p.cczf = 2, 1
    _two_phase(p, cs=0.1)
    p.cg_tol = cg_tol
    umax = math.sqrt(9.81 * 0.30)
    p.dt = 0.2 * dx / umax
    a, h = 0.25 * (nx * dx / 0.64), 0.30 * (nz * dx / 0.48)
    X, Y, Z = _centres(p)
    inside = (X <= a) & (Z <= h)
    d_in = np.minimum(a - X, h - Z)
    dxo, dzo = np.maximum(X - a, 0.0), np.maximum(Z - h, 0.0)
    d_out = -np.sqrt(dxo ** 2 + dzo ** 2)
    ls0 = np.where(inside, d_in, d_out)

    def init(model):
        standard_init(model, ls0)

    return p, init


def sloshing(nx=256, ny=128, nz=128, dx=0.005, cg_tol=1e-8, cfl=0.25, amp=0.02, depth=0.32):
    """Sloshing tank: free surface z = depth + amp cos(pi x/Lx) cos(pi y/Ly).

    L = (nx, ny, nz) * dx (1.28 x 0.64 x 0.64 m at the metric size), closed no-slip tank with
    a free-slip lid, Smagorinsky Cs = 0.1, RK3.  The time step follows CFL `cfl` with the
    linear gravity-wave speed sqrt(g*depth) and stays fixed over the run.
    """
    p = default_params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dx = p.dy = p.dz = dx
    p.ccx0 = p.ccxf = 2
    p.ccy0 = p.ccyf = 2
    p.ccz0, p.cczf = 2, 1
    _two_phase(p, cs=0.1)
    p.cg_tol = cg_tol
    p.dt = cfl * dx / math.sqrt(9.81 * depth)
    lx, ly = nx * dx, ny * dx
    depth = depth * (nz * dx / 0.64)
    X, Y, Z = _centres(p)
    ls0 = depth + amp * np.cos(math.pi * X / lx) * np.cos(math.pi * Y / ly) - Z

    def init(model):
        standard_init(model, ls0)

    return p, init


def reference_default(nx=None, ny=None, nz=None):
    """The reference's compiled case: flat surface at z = 0.5, u = 0.31, x periodic, RK2."""
    p = default_params()
    if nx:
        p.nx = nx
    if ny:
        p.ny = ny
    if nz:
        p.nz = nz
    X, Y, Z = _centres(p)
    ls0 = 0.5 - Z        # tipo = 1 with ampl = 0 (14_level_set.f90:77-114)

    def init(model):
        standard_init(model, ls0, u_init=0.31)

    return p, init


def random_state(p: SuliParams, seed: int = 0, *, vel=0.2, wave=0.03):
    """Seeded random-but-smooth state for kernel-level parity tests."""
    rng = np.random.default_rng(seed)
    X, Y, Z = _centres(p)
    lz = p.nz * p.dz
    lx, ly = p.nx * p.dx, p.ny * p.dy
    ph = rng.uniform(0, 2 * math.pi, 4)
    ls = (0.5 * lz + wave * lz * np.sin(2 * math.pi * X / lx + ph[0]) * np.cos(2 * math.pi * Y / ly + ph[1]) - Z
          + 0.002 * rng.standard_normal(X.shape))
    out = {"ls": ls}
    from ._abi import field_shape
    for name in ("u", "v", "w"):
        sh = field_shape(p, name)
        out[name] = vel * rng.standard_normal(sh)
    out["prd1"] = 0.01 * rng.standard_normal(field_shape(p, "prd1"))
    return out
