"""Wave inflow (wave_t = 1 Stokes I, 2 Stokes II, 5 Stokes V): waves_coef and boundary_waves
(3_contorno.f90:952-1205), called after tempo in every stage (1_principal.f90:84).

CPU tests pin the oracle to linear wave theory written out here (dispersion relation,
elevation and the Stokes I velocity profile) and to the reference's handling of the level set
(a single-precision round trip) and of the planes it does not set.  GPU tests compare the
library with the oracle."""
import math

import numpy as np
import pytest

from helpers import load_state, pkg, rel_err

cases = pkg.cases


def wave_state(orc, wave_t, t=0.37):
    p, init = cases.wave_channel(wave_t=wave_t)
    o = orc.Oracle(p)
    init(o)
    rng = np.random.default_rng(wave_t)
    ls = o.download("ls") + 1e-3 * rng.standard_normal(o.shape("ls"))
    o.upload("ls", ls)
    o.set_scalar("t", t)
    return p, o, ls


def linear_wave(gz):
    """Stokes I constants of waves_coef: a = 0.03, T = 2.5, h = 1, wavelength from
    L = g T^2/(2 pi) tanh(2 pi h/L) by the same 1000 fixed-point sweeps."""
    T, h = 2.5, 1.0
    L = gz * T * T / (2. * math.pi)
    for _ in range(1000):
        L = gz * T * T / (2. * math.pi) * math.tanh(2. * math.pi * h / L)
    return 0.03, 2. * math.pi / T, 2. * math.pi / L, h, L


def test_stokes_i_against_linear_theory(orc):
    p, o, ls0 = wave_state(orc, 1)
    a, f, n, h, L = linear_wave(p.gz)
    assert abs(L - p.gz * 2.5 ** 2 / (2 * math.pi) * math.tanh(2 * math.pi * h / L)) < 1e-12 * L
    t = 0.37
    o.boundary_waves()
    ls = o.download("ls")
    kp = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    eta1 = h + a * math.cos(n * p.dx * 0.5 - f * t)            # elevation over column i = 1
    assert np.array_equal(ls[0, :, :], np.broadcast_to((eta1 - kp).astype(np.float32).astype(np.float64), ls[0].shape))
    # u at the inflow face (i = 1 of u; the ghost face i = 0 is bxx0) below the surface
    bxx0, bxx1 = o.download("bxx0")[:, :, 0], o.download("bxx1")[:, :, 0]
    kpp = (np.arange(0, p.nz + 2) - 0.5) * p.dz
    eta0 = h + a * math.cos(n * p.dx * (-0.5) - f * t)
    u0 = a * f * np.cosh(n * kpp) / math.sinh(n * h) * math.cos(n * p.dx * (-1.) - f * t)
    u0[np.float32(eta0 - kpp) < 0] = 0.
    np.testing.assert_allclose(bxx0, np.broadcast_to(u0, bxx0.shape), rtol=1e-13, atol=1e-16)
    assert (bxx1[:, np.float32(eta1 - kpp) < 0] == 0).all() and (bxx1[:, 3] != 0).all()


def test_level_set_round_trip_and_unset_planes(orc):
    """Every cell but the inflow column keeps ls rounded to float32 (the reference's real(4)
    copy); bxy0 and the top row of bxz0, never set by the reference, are 0."""
    p, o, ls0 = wave_state(orc, 2)
    o.upload("bxy0", np.full(o.shape("bxy0"), 5.0))
    o.upload("bxz0", np.full(o.shape("bxz0"), 5.0))
    o.boundary_waves()
    ls = o.download("ls")
    assert np.array_equal(ls[1:], ls0[1:].astype(np.float32).astype(np.float64))
    assert (o.download("bxy0") == 0).all()
    assert (o.download("bxz0")[:, p.nz + 2, 0] == 0).all()


def test_stokes_v_elevation(orc):
    """Stokes V (Fenton's coefficients, 3_contorno.f90:1118-1196): the crest of the elevation
    over the cycle is close to the linear amplitude 0.03 above the still depth, sharper than
    the trough."""
    p, init = cases.wave_channel(wave_t=5, nx=8, ny=4, nz=12)
    o = orc.Oracle(p)
    init(o)
    crest, trough = -1., 1.
    kp = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    for t in np.linspace(0.0, 2.5, 26):
        o.set_scalar("t", t)
        o.boundary_waves()
        eta = o.download("ls")[0, 0, 0] + kp[0] - 1.0            # h_f(1) - h0, to float precision
        crest, trough = max(crest, eta), min(trough, eta)
    assert 0.025 < crest < 0.04 and -0.03 < trough < -0.02 and crest > -trough


def test_wave_step_runs(orc):
    p, init = cases.wave_channel(wave_t=1)
    o = orc.Oracle(p)
    init(o)
    st = o.step(1)
    assert st["status"] == 0
    assert (o.download("bxy0") == 0).all()


# ------------------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("wave_t", [1, 2])
def test_boundary_waves_gpu(orc, wave_t):
    """The planes within 1e-12 of their scale (cos, cosh, sinh of the device and of the host
    differ in the last bits); the level set within one float32 rounding step (a double that
    differs in its last bit can round to the neighbouring float)."""
    p, init = cases.wave_channel(wave_t=wave_t)
    g = pkg.Solver(p)
    o = orc.Oracle(p)
    init(g)
    init(o)
    for m in (g, o):
        m.set_scalar("t", 0.61)
        m.boundary_waves()
    for f in ("bxx0", "bxx1", "bxz0", "bxy0"):
        assert rel_err(g.download(f), o.download(f)) <= 1e-12, f
    assert rel_err(g.download("ls"), o.download("ls")) <= 2.0 ** -23
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("wave_t", [1, 2, 5])
def test_step_parity_waves(orc, wave_t):
    """One step of the wave flume (three stages, each with boundary_waves): velocities within
    1e-6 of the velocity scale, other fields within 1e-6 of their scale (the level set passes
    through single precision at every stage).  The wave's inflow flux is not matched by the
    reference's outflow copy, which leaves graddin's all-Neumann system inconsistent and its
    CG iterates at the mercy of rounding; outflow_fix = 1 balances the flux so that the two
    solves converge to the same field."""
    p, init = cases.wave_channel(wave_t=wave_t, cg_tol=1e-12, outflow_fix=1)
    g = pkg.Solver(p)
    o = orc.Oracle(p)
    init(g)
    init(o)
    sg, so = g.step(1), o.step(1)
    assert sg["status"] == 0 and so["status"] == 0
    vel = {f: (g.download(f), o.download(f)) for f in ("u", "v", "w")}
    vs = max(float(np.abs(b).max()) for _, b in vel.values())
    worst = {f: float(np.abs(a - b).max()) / vs for f, (a, b) in vel.items()}
    worst.update({f: rel_err(g.download(f), o.download(f)) for f in ("ls", "rho", "bxx1")})
    assert max(worst.values()) <= 1e-6, worst
    g.close()
