"""Helpers shared by the tests: small parameter sets and field comparison."""
from __future__ import annotations

import numpy as np

import conftest

pkg = conftest.load_pkg()

# every field a kernel may write, by subroutine
OUT_FIELDS = {
    "visco": ["nut", "xnut", "ynut", "znut"],
    "convdiff": ["Fu", "Fv", "Fw", "prd0"],
    "tempo": ["u", "v", "w", "u0", "v0", "w0", "fu0", "fv0", "fw0", "fu1", "fv1", "fw1"],
    "contorno": ["u", "v", "w", "prd1", "ub", "vb", "wb"],
    "heaviside": ["hs", "hsx", "hsy", "hsz", "rho", "ls_nu"],
    "mod_ls1": ["mod_ls", "kurv", "ddlsdx", "ddlsdy", "ddlsdz"],
    "level_set": ["ls", "mod_ls", "kurv", "hs", "hsx", "hsy", "hsz", "rho", "ls_nu"],
    "posdin": ["u", "v", "w", "prd"],
}

STATE_FIELDS = ["u", "v", "w", "prd1", "ls", "rho", "ls_nu", "hs", "hsx", "hsy", "hsz", "kurv", "mod_ls",
                "nut", "xnut", "ynut", "znut", "ub", "vb", "wb"]


def small_params(nx=12, ny=10, nz=9, bc=(2, 2, 2, 2, 2, 1), m_turb=1, t_tempo=2, dx=0.02):
    p = pkg.default_params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dx = p.dy = p.dz = dx
    p.ccx0, p.ccxf, p.ccy0, p.ccyf, p.ccz0, p.cczf = bc
    p.m_turb, p.csmag = m_turb, 0.1
    p.t_tempo = t_tempo
    p.rho_f1, p.mi_f1, p.rho_f2, p.mi_f2 = 1.2, 1.8e-5, 1000.0, 1e-3
    p.gx, p.gz = 0.0, 9.81
    p.dt = 2e-3
    p.dt1 = 0.1 * dx
    return p


def seeded_state(p, seed=0):
    """A random-but-smooth state with interfaces crossing the domain."""
    return pkg.cases.random_state(p, seed)


def load_state(model, st: dict):
    for k, v in st.items():
        model.upload(k, v)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale
