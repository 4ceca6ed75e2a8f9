"""The reference's manufactured-solution harness (13_mms.f90, Weng 2009), restated in
suli_b200.mms_weng and run on the oracle and on the GPU.

CPU:
* the restated momentum sources (termo_fonte1/2) against a symbolic derivation of the same
  momentum equation, u_t + u.grad u - nu div(grad u + grad u^T), from the manufactured fields:
  equal for the module's a = 0; with a != 0 the unsteady sources differentiate in time with the
  surface h held fixed (a simplification of the reference), and a few viscous second
  derivatives of the steady u source carry a sign of their own (a relative effect below 1e-6);
* mms_bc's planes: the exact components at the planes' staggered positions, the reference's
  loop ranges and the unsteady case's bzy0 / bzyf, which take the w expression;
* on the oracle: the RMS errors of mms() fall as the grid is refined.
GPU: the GPU's error norms equal the oracle's after ten steps of each case, and so do the
fields (graddin and posdin are skipped when mms_t > 0, 1_principal.f90:89, so this checks the
predictor: level set, viscosity, convection-diffusion with the sources, RK stages, boundaries).
"""
import numpy as np
import pytest

from helpers import pkg, rel_err

W = pkg.mms_weng


def _residual_sources(mt, a, freeze_h_in_time):
    sp = pytest.importorskip("sympy")
    x, y, z, t = sp.symbols("x y z t", real=True)
    hs = sp.Symbol("hs")
    A, h0, pi, nu = sp.Float(a), sp.Float(2.0), sp.pi, sp.Float(W.VISC)

    def fields(h):
        if mt == 1:
            u = sp.sin(x) * sp.cos(y) * sp.sin(pi / 2 * z / h) - sp.cos(x) * sp.sin(y) * (sp.cos(2 * pi * z / h) - 1)
            v = -sp.cos(x) * sp.sin(y) * sp.sin(pi / 2 * z / h) + sp.sin(x) * sp.cos(y) * (sp.cos(2 * pi * z / h) - 1)
            w = (-A * (sp.sin(x) ** 2 * sp.cos(y) ** 2 - sp.cos(x) ** 2 * sp.sin(y) ** 2)
                 * (sp.sin(2 * pi * z / h) - 2 * pi * z / h * sp.cos(2 * pi * z / h) + 2 * pi) / (2 * pi))
            return u, v, w
        c = sp.cos(pi / 2 * (1 - z / h))
        return (sp.sin(y) * sp.cos(x / 2) ** 2 * c * sp.sin(t), -sp.sin(x) * sp.cos(y / 2) ** 2 * c * sp.sin(t),
                -A * sp.cos(x / 2) * sp.cos(y / 2) * c * sp.sin(t))

    h = A * sp.sin(x) * sp.sin(y) + h0 if mt == 1 else A * sp.cos(x / 2) * sp.cos(y / 2) * sp.cos(t) + h0
    u, v, w = fields(h)
    d = sp.diff
    if mt == 1:
        dt = [0, 0, 0]
    elif freeze_h_in_time:
        uf, vf, wf = fields(hs)
        dt = [d(f, t).subs(hs, h) for f in (uf, vf, wf)]
    else:
        dt = [d(f, t) for f in (u, v, w)]
    su = dt[0] + u * d(u, x) + v * d(u, y) + w * d(u, z) - nu * (2 * d(u, x, 2) + d(u, y, 2) + d(u, z, 2) + d(v, x, y) + d(w, x, z))
    sv = dt[1] + u * d(v, x) + v * d(v, y) + w * d(v, z) - nu * (d(v, x, 2) + 2 * d(v, y, 2) + d(v, z, 2) + d(u, x, y) + d(w, y, z))
    sw = dt[2] + u * d(w, x) + v * d(w, y) + w * d(w, z) - nu * (d(w, x, 2) + d(w, y, 2) + 2 * d(w, z, 2) + d(u, x, z) + d(v, y, z))
    return [sp.lambdify((x, y, z, t), s, "numpy") for s in (su, sv, sw)]


def _restated(m):
    if m.mms_t == 1:
        return [lambda X, Y, Z, T, f=f: f(X, Y, Z) for f in (m._fonte1_u, m._fonte1_v, m._fonte1_w)]
    return [m._fonte2_u, m._fonte2_v, m._fonte2_w]


def _max_rel(f_ref, f_got, pts, T):
    X, Y, Z = pts
    ref = np.broadcast_to(np.asarray(f_ref(X, Y, Z, T), dtype=float), X.shape)
    got = f_got(X, Y, Z, T)
    return float(np.abs(got - ref).max()) / max(float(np.abs(ref).max()), 1e-300), float(np.abs(got - ref).max())


@pytest.fixture(scope="module")
def pts():
    rng = np.random.default_rng(0)
    return rng.uniform(-3, 3, 300), rng.uniform(-3, 3, 300), rng.uniform(0.1, 1.9, 300)


@pytest.mark.parametrize("mt", [1, 2])
def test_sources_equal_the_momentum_residual(mt, pts):
    """a = 0 (0_modules.f90:208): every source equals the symbolic residual to rounding."""
    m = W.WengMMS(mt, a=0.0)
    for f_ref, f_got in zip(_residual_sources(mt, 0.0, False), _restated(m)):
        rel, ab = _max_rel(f_ref, f_got, pts, 0.7)
        assert rel <= 1e-12 or ab <= 1e-15


def test_sources_with_a_moving_surface(pts):
    """a = 0.3: the unsteady sources equal the residual whose time derivative holds the surface
    h fixed (the reference's dudt, dvdt, dwdt, 13_mms.f90:1146, 1219, 1289) to 1e-7, and differ
    from the full residual by more than 1 %; the steady sources match to 1e-6 (the steady u
    source's viscous terms, 13_mms.f90:868-886)."""
    m2 = W.WengMMS(2, a=0.3)
    for f_ref, f_got in zip(_residual_sources(2, 0.3, True), _restated(m2)):
        assert _max_rel(f_ref, f_got, pts, 0.7)[0] <= 1e-7
    worst = max(_max_rel(f_ref, f_got, pts, 0.7)[0] for f_ref, f_got in zip(_residual_sources(2, 0.3, False), _restated(m2)))
    assert worst > 1e-2
    m1 = W.WengMMS(1, a=0.3)
    for f_ref, f_got in zip(_residual_sources(1, 0.3, False), _restated(m1)):
        assert _max_rel(f_ref, f_got, pts, 0.0)[0] <= 1e-6


@pytest.mark.parametrize("mt", [1, 2])
def test_planes(mt):
    m = W.WengMMS(mt, nx=8, ny=6, nz=5, a=0.2)
    t = 0.37
    pl = m.planes(t)
    p = m.p
    for name, arr in pl.items():
        assert arr.shape == pkg.field_shape(p, name), name
    dx, dy, dz, off = p.dx, p.dy, p.dz, m.off
    # bxx0 at i = 0: u at x = -dx (- pi), y = (j - 0.5) dy, z = (k - 0.5) dz
    j, k = 3, 2
    want = m.u_m(np.array(-dx - off), np.array((j - 0.5) * dy - off), np.array((k - 0.5) * dz), t)
    assert pl["bxx0"][j, k, 0] == pytest.approx(float(want), rel=1e-14, abs=1e-300)
    # rows beyond the reference's loops (j = ny + 2 of bxy0, k = nz + 2 of bxz0) stay 0
    assert (pl["bxy0"][p.ny + 2] == 0).all() and (pl["bxz0"][:, p.nz + 2] == 0).all()
    # bzy0 at k = 0: v's position; the unsteady case evaluates w's expression there
    i, j = 4, 2
    X, Y, Z = np.array((i - 0.5) * dx - off), np.array((j - 1.0) * dy - off), np.array(-0.5 * dz)
    want = (m.w_m if mt == 2 else m.v_m)(X, Y, Z, t)
    assert pl["bzy0"][i, j, 0] == pytest.approx(float(want), rel=1e-14, abs=1e-300)


def test_errors_fall_under_refinement(orc):
    """The steady case on the oracle: after 20 steps the u error (upwind advection, first order)
    is about halved by halving the cells."""
    errs = []
    for n in (16, 32):
        m = W.WengMMS(1, nx=n, ny=n, nz=3 * n // 4, dt=2e-3)
        o = orc.Oracle(m.p)
        m.init(o)
        for it in range(1, 21):
            e = m.step(o, it)
        errs.append(e)
        assert e["w"] < 1e-8 and e["p"] == 0.0
    assert 1.6 < errs[0]["u"] / errs[1]["u"] < 2.4
    assert errs[1]["u"] == pytest.approx(errs[1]["v"], rel=1e-6)   # the field is symmetric in x, y


@pytest.mark.gpu
@pytest.mark.parametrize("mt", [1, 2])
def test_error_norms_gpu(orc, mt):
    """Ten steps of each case on the GPU and on the oracle: every error norm of mms() within
    1e-9 of the largest one (w is 0 in the exact field for a = 0, so its error is rounding noise
    of order 1e-11 on both sides), the velocities within 1e-10 of the velocity scale and the
    level set of its own."""
    mg = W.WengMMS(mt, nx=32, ny=32, nz=24, dt=2e-3)
    mo = W.WengMMS(mt, nx=32, ny=32, nz=24, dt=2e-3)
    g = pkg.Solver(mg.p)
    o = orc.Oracle(mo.p)
    mg.init(g)
    mo.init(o)
    for it in range(1, 11):
        eg, eo = mg.step(g, it), mo.step(o, it)
        scale = max(eo["u"], eo["v"], eo["w"], 1e-300)
        for k in ("u", "v", "w", "p"):
            assert abs(eg[k] - eo[k]) <= 1e-9 * scale, (it, k, eg[k], eo[k])
    assert mg.erro_t == pytest.approx(mo.erro_t, rel=1e-9)
    vel = {f: (g.download(f), o.download(f)) for f in ("u", "v", "w")}
    vs = max(float(np.abs(b).max()) for _, b in vel.values())
    for f, (a, b) in vel.items():
        assert float(np.abs(a - b).max()) <= 1e-10 * vs, f
    assert rel_err(g.download("ls"), o.download("ls")) <= 1e-10
    g.close()
