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


def standard_init(model, ls0: np.ndarray, u_init: float = 0.0, masks=None):
    """[obstacle masks +] iniciais + level-set preset + level_set_ini + contorno(1), contorno(3)."""
    if masks is not None:
        model.set_obstacle(*masks)
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


def sloshing(nx=256, ny=128, nz=128, dx=0.005, cg_tol=1e-8, cfl=0.25, amp=0.02, depth=0.32, div_tol=0.0):
    """Sloshing tank: free surface z = depth + amp cos(pi x/Lx) cos(pi y/Ly).

    L = (nx, ny, nz) * dx (1.28 x 0.64 x 0.64 m at the metric size), closed no-slip tank with
    a free-slip lid, Smagorinsky Cs = 0.1, RK3.  The time step follows CFL `cfl` with the
    linear gravity-wave speed sqrt(g*depth) and stays fixed over the run.  div_tol > 0 adds
    the Poisson solve's divergence test (max |div u| after the projection within div_tol).
    """
    p = default_params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dx = p.dy = p.dz = dx
    p.ccx0 = p.ccxf = 2
    p.ccy0 = p.ccyf = 2
    p.ccz0, p.cczf = 2, 1
    _two_phase(p, cs=0.1)
    p.cg_tol = cg_tol
    p.div_tol = div_tol
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


def _nint(v: np.ndarray) -> np.ndarray:
    """Fortran NINT: nearest integer, halves away from zero."""
    a = np.abs(v)
    r = np.floor(a)
    r = r + (a - r >= 0.5)
    return (np.sign(v) * r).astype(np.int64)


def obstacle_masks(p: SuliParams, height) -> tuple:
    """ku, kv, kw from a bottom height on the half-cell grid (3_contorno.f90:741-760).

    `height(i, j)` takes integer arrays of half-cell indices i = -1 .. 2(nx+1)+2,
    j = -1 .. 2(ny+1)+2 and returns the height there; then
    ku(i,j) = nint(h(2i-1, 2j)/dz + 0.5) and kv(i,j) = nint(h(2i, 2j-1)/dz + 0.5), at most nz,
    kw(i,j) = floor(h(2i, 2j)/dz + 1), at most nz+1; Fortran order, shapes _abi.mask_shapes."""
    nx, ny, nz, dz = p.nx, p.ny, p.nz, p.dz
    I = np.arange(-1, 2 * (nx + 1) + 3)
    J = np.arange(-1, 2 * (ny + 1) + 3)
    aux = np.asarray(height(I[:, None], J[None, :]), dtype=np.float64) * np.ones((I.size, J.size))
    A = lambda i, j: aux[i + 1, j + 1]                         # auxx(i, j), i, j from -1
    iu, ju = np.meshgrid(np.arange(0, nx + 3), np.arange(0, ny + 2), indexing="ij")
    ku = np.minimum(_nint(A(iu * 2 - 1, ju * 2) / dz + 0.5), nz)
    iv, jv = np.meshgrid(np.arange(0, nx + 2), np.arange(0, ny + 3), indexing="ij")
    kv = np.minimum(_nint(A(iv * 2, jv * 2 - 1) / dz + 0.5), nz)
    iw, jw = np.meshgrid(np.arange(0, nx + 2), np.arange(0, ny + 2), indexing="ij")
    kw = np.minimum(np.floor(A(iw * 2, jw * 2) / dz + 1.).astype(np.int64), nz + 1)
    return tuple(np.asfortranarray(m, dtype=np.int32) for m in (ku, kv, kw))


def obstaculo(p: SuliParams, obst_t: int) -> tuple:
    """The masks of the reference's bottom presets 1..10 (obstaculo, 3_contorno.f90:494-740).

    Heights at x = (i-1) dx/2, y = (j-1) dy/2 on the half-cell grid (preset 5: x = (i-2) dx/2).
    Presets 2, 8 and 9 read values the reference leaves unset: preset 2's running offsets
    before the first segment that sets them are 0 here, and presets 8 and 9 are -dz (no
    obstacle) outside the wall, as preset 10 sets explicitly."""
    dx, dy, dz, ny, nz = p.dx, p.dy, p.dz, p.ny, p.nz
    pi = math.pi

    def xs(i, shift=1.0):
        return (i - shift) * (dx * 0.5)

    def ys(j):
        return (j - 1.) * (dy * 0.5)

    if obst_t == 1:      # dunes (:524-533): elev is an integer parameter, int(50 dz) (0_modules.f90:80)
        elev, amp, comp, fase = int(50. * dz), 0.50, .5, -pi / 2.
        return obstacle_masks(p, lambda i, j: elev + amp * (1. + np.sin(fase + 2. * pi * xs(i) / comp)) + 0. * j)
    if obst_t == 2:      # Yue et al. (2003) dune (:534-568), evaluated in the reference's loop order
        def h2(i, j):
            out = np.empty((i.size, j.size))
            aux1 = aux2 = 0.0
            for jj in range(j.size):
                for ii in range(i.size):
                    x = xs(float(i[ii, 0]))
                    if x <= 0.01:
                        v = 0.02
                    elif x <= 0.05:
                        v = -math.tan(26. * pi / 180.) * x + 0.02
                    elif x <= 0.075:
                        v = 0.0005
                    elif x <= 0.1375:
                        v = math.tan(1.8 * pi / 180.) * x + 0.0005
                        aux1 = v
                    elif x <= 0.325:
                        v = math.tan(5. * pi / 180.) * x + aux1
                        aux2 = v
                    elif x <= 0.39:
                        v = math.tan(1.8 * pi / 180.) * x + aux2
                    else:
                        v = 0.02
                    out[ii, jj] = v
            return out
        return obstacle_masks(p, h2)
    if obst_t == 3:      # 3-D Gaussian bump (:570-591)
        d, x0, y0, a, sigx, sigy = 0.2, 3., ny / 2. * dy, 2.0, 0.5, 0.5
        def h3(i, j):
            aux1 = (ys(j) - y0) * (ys(j) - y0) / (2. * sigy * sigy)
            aux2 = (xs(i) - x0) * (xs(i) - x0) / (2. * sigx * sigx)
            return np.exp(-aux2 - aux1) * a + d
        return obstacle_masks(p, h3)
    if obst_t == 4:      # Beji and Battjes (1994) bar (:593-618)
        def h4(i, j):
            x = xs(i) + 0. * j
            return np.select([x < 6., x < 12., x < 14., x < 17.],
                             [0. * x, math.tan(1. / 20.) * (x - 6.), 0.30 + 0. * x, -math.tan(1. / 10.) * (x - 14.) + 0.30],
                             0. * x)
        return obstacle_masks(p, h4)
    if obst_t == 5:      # Delft 1980 channel 0 (:620-633)
        return obstacle_masks(p, lambda i, j: np.where(xs(i, 2.0) + 0. * j <= 1.0, 0.2, 0.))
    if obst_t == 6:      # Delft 1980 channel 1_2 (:635-659)
        def h6(i, j):
            x = xs(i) + 0. * j
            return np.select([x < 1., x < 1.4, x < 2.4, x < 2.8],
                             [0.2 + 0. * x, -1. / 2. * (x - 1.) + 0.2, 0. * x, 1. / 2. * (x - 2.4)], 0.2 + 0. * x)
        return obstacle_masks(p, h6)
    if obst_t == 7:      # holes and bumps (:661-681)
        raio = 0.12
        def h7(i, j):
            x = xs(i) + 0. * j
            inner = np.sqrt(np.maximum(-(x - 1.) ** 2. + raio ** 2., 0.))
            return np.select([x < (1. - raio), x < 1.], [0. * x, inner], raio + 0. * x)
        return obstacle_masks(p, h7)
    if obst_t in (8, 9, 10):   # walls with an opening (:683-740)
        lo, hi, wall, ylo, yhi = {8: (90., 100., (nz + 1) * dz, 95., 170.),
                                  9: (0.8, 0.825, (nz + 1) * dz, 0.45, 0.75),
                                  10: (0.75 - 0.16 * 0.5, 0.75 + 0.16 * 0.5, 0.16, 0.5 - 0.4 * 0.5, 0.5 + 0.4 * 0.5)}[obst_t]
        def h8(i, j):
            x, y = xs(i) + 0. * j, ys(j) + 0. * i
            h = np.full(x.shape, -dz)
            h = np.where((x >= lo) & (x <= hi), wall, h)
            return np.where((y > ylo) & (y < yhi), -dz, h)
        return obstacle_masks(p, h8)
    raise ValueError(f"obst_t {obst_t}: the reference defines presets 1..10")


def bump_channel(nx=32, ny=16, nz=24, dx=0.02, cg_tol=1e-10, u_init=0.1, outflow_fix=0):
    """A small two-phase channel over a Gaussian bottom bump (the obst_t = 3 shape scaled to the
    box): water 0.6 of the depth, inflow u_init at x = 0 (ccx0 = 3), outflow at x = xf
    (ccxf = 4), periodic y, free-slip top.

    With the reference's outflow copy (outflow_fix = 0) the outflow plane carries a different
    flux than the inflow once the flow passes the bump, graddin's all-Neumann system is
    inconsistent and its CG reports convergence on a recurrence residual that has left the true
    one (a second solve from the result takes as many iterations again).  outflow_fix = 1 makes
    the system consistent."""
    p = default_params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dx = p.dy = p.dz = dx
    p.ccx0, p.ccxf = 3, 4
    p.ccy0 = p.ccyf = 0
    p.ccz0, p.cczf = 2, 1
    _two_phase(p, cs=0.1)
    p.cg_tol = cg_tol
    p.obst_t = 3
    p.outflow_fix = outflow_fix
    p.dt = 0.2 * dx / (u_init + math.sqrt(9.81 * 0.6 * nz * dx))
    Lx, Ly, H = nx * dx, ny * dx, nz * dx

    def height(i, j):
        x, y = (i - 1.) * (dx * 0.5), (j - 1.) * (dx * 0.5)
        return 0.25 * H * np.exp(-((x - 0.5 * Lx) ** 2 + (y - 0.5 * Ly) ** 2) / (2. * (0.15 * Lx) ** 2)) + 0.1 * H

    masks = obstacle_masks(p, height)
    X, Y, Z = _centres(p)
    ls0 = 0.6 * H - Z

    def init(model):
        standard_init(model, ls0, u_init, masks=masks)

    return p, init, masks


def les_channel(nx=512, ny=256, nz=256, cg_tol=1e-8, seed=0, x0=3.0, outflow_fix=1, periodic_faces=1):
    """The LES channel over a bottom bump: 6 x 3 x 3 m (dx = dy = dz = 6/nx at the default
    size, 0.01171875), water 2 m deep, the obst_t = 3 Gaussian bump with height 0.3 m, no flat
    base (d = 0), sigma 0.5 m, centred at (x0, Ly/2); inflow u = 1 + 0.05 U(-1, 1) (seeded,
    per inflow-plane point) at x = 0, outflow at x = xf, periodic y, no-slip bottom, free-slip
    top, Smagorinsky Cs = 0.12, RK3, dt from CFL 0.3 with the inflow speed plus sqrt(g h).
    Smaller nx, ny, nz keep the 6 x 3 x 3 m box at the coarser spacing.

    The reference's pressure solve has Neumann conditions on every face and no correction of
    the net flux (9_grad.f90:96-116): with this fluctuating inflow and the boundary layer the
    outflow copy carries, the problem is inconsistent and its CG diverges within the first
    steps (in this library and in the CPU restatement of the tests alike), as it does for the
    wave flume; a uniform flow through the same faces stays exactly steady.  The case therefore
    turns on outflow_fix (the outflow plane shifted to balance the inflow) unless told not to.
    Once the surface moves, the density also varies across the periodic y boundary, where the
    reference's clamped end faces make the scaled Poisson operator non-symmetric and the CG
    breaks down after a few steps; periodic_faces (the wrap average at both end faces) is on
    for the same reason."""
    p = default_params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dx, p.dy, p.dz = 6.0 / nx, 3.0 / ny, 3.0 / nz
    p.ccx0, p.ccxf = 3, 4
    p.ccy0 = p.ccyf = 0
    p.ccz0, p.cczf = 2, 1
    _two_phase(p, cs=0.12)
    p.cg_tol = cg_tol
    p.obst_t = 3
    p.outflow_fix = outflow_fix
    p.periodic_faces = periodic_faces
    p.dt = 0.3 * min(p.dx, p.dy, p.dz) / (1.05 + math.sqrt(9.81 * 2.0))
    ly = ny * p.dy

    def height(i, j):
        x, y = (i - 1.) * (p.dx * 0.5), (j - 1.) * (p.dy * 0.5)
        return np.exp(-((x - x0) * (x - x0) / (2. * 0.5 * 0.5)) - (y - ly / 2.) * (y - ly / 2.) / (2. * 0.5 * 0.5)) * 0.3

    masks = obstacle_masks(p, height)
    X, Y, Z = _centres(p)
    ls0 = 2.0 - Z
    rng = np.random.default_rng(seed)
    from ._abi import field_shape
    inflow = 1.0 + 0.05 * rng.uniform(-1.0, 1.0, field_shape(p, "bxx0"))

    def init(model):
        standard_init(model, ls0, 1.0, masks=masks)
        # the inflow planes with the seeded fluctuation, zero inside the bump as iniciais makes
        # them (2_iniciais.f90:60-65)
        for name in ("bxx0", "bxx1"):
            plane = model.download(name)
            model.upload(name, np.where(plane == 0.0, 0.0, inflow))
        model.contorno(1)

    return p, init, masks


def wave_channel(wave_t=1, nx=32, ny=8, nz=12, dx=0.1, dz=0.1, cg_tol=1e-10, outflow_fix=0):
    """A wave flume for the wave inflow of boundary_waves (3_contorno.f90:952-1082): still water
    1 m deep (h0_f of waves_coef), the wave entering at x = 0 (ccx0 = 3), outflow at x = xf
    (ccxf = 4), periodic y, no-slip bottom, free-slip top; dt from CFL 0.2 with sqrt(g h).
    The wave's inflow flux varies in time and the outflow copy does not follow it, so with the
    reference's outflow (outflow_fix = 0) the all-Neumann Poisson system (9_grad.f90) is
    inconsistent: its CG stops on a recurrence residual that no longer matches the true one.
    outflow_fix = 1 balances the flux and makes the solve well posed."""
    p = default_params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dx = p.dy = dx
    p.dz = dz
    p.ccx0, p.ccxf = 3, 4
    p.ccy0 = p.ccyf = 0
    p.ccz0, p.cczf = 2, 1
    _two_phase(p, cs=0.1)
    p.cg_tol = cg_tol
    p.wave_t = wave_t
    p.outflow_fix = outflow_fix
    p.dt = 0.2 * min(dx, dz) / math.sqrt(9.81 * 1.0)
    X, Y, Z = _centres(p)
    ls0 = 1.0 - Z

    def init(model):
        standard_init(model, ls0)

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


class TaylorGreenMMS:
    """Manufactured solution on the periodic box [0, 2 pi]^3, single phase (rho 1, nu):

        u = sin x cos y cos z e^-t,  v = -cos x sin y cos z e^-t,  w = 0,
        p = (cos 2x + cos 2y) e^-2t / 4.

    The velocity is divergence-free; the source that makes it an exact solution of the
    incompressible Navier-Stokes equations (d_t u + u.grad u = -grad p + nu lap u + f) is

        f_u = (3 nu - 1) u - sin 2x sin^2 z e^-2t / 2,
        f_v = (3 nu - 1) v - sin 2y sin^2 z e^-2t / 2,   f_w = 0,

    added through the reference's source-term arrays tf_u/v/w (6_convdiff.f90:156,168,183),
    refreshed once per step at t = it dt as the reference's MMS driver does
    (1_principal.f90:69-71).  Unlike that driver, the projection runs (graddin, posdin), so the
    solver's own pressure is checked too.  x, y, z periodic; RK3; the level set is constant
    (one phase), so the interface terms vanish.
    """

    def __init__(self, n=128, nu=0.01, dt=1e-3, precision=0, cg_tol=1e-10):
        p = default_params()
        p.nx = p.ny = p.nz = n
        p.dx = p.dy = p.dz = 2.0 * math.pi / n
        p.dt = dt
        p.ccx0 = p.ccxf = p.ccy0 = p.ccyf = p.ccz0 = p.cczf = 0
        p.t_tempo = 2
        p.m_turb = 0
        p.rho_f1 = p.rho_f2 = 1.0
        p.mi_f1 = p.mi_f2 = nu
        p.sigma = 0.0
        p.gx = p.gz = 0.0
        p.cg_stop, p.cg_tol, p.cg_maxit = 1, cg_tol, 20000
        p.precision = precision
        p.dt1 = 0.1 * p.dx
        self.p, self.nu = p, nu

    def _grid(self, name):
        """Coordinates of a field's points over its Fortran extents."""
        from ._abi import field_extent
        p = self.p
        (i0, i1), (j0, j1), (k0, k1) = field_extent(p, name)
        fx, fy, fz = {"u": (1, 0, 0), "tf_u": (1, 0, 0), "v": (0, 1, 0), "tf_v": (0, 1, 0),
                      "w": (0, 0, 1), "tf_w": (0, 0, 1)}.get(name, (0, 0, 0))
        x = (np.arange(i0, i1 + 1) - (1.0 if fx else 0.5)) * p.dx
        y = (np.arange(j0, j1 + 1) - (1.0 if fy else 0.5)) * p.dy
        z = (np.arange(k0, k1 + 1) - (1.0 if fz else 0.5)) * p.dz
        return np.meshgrid(x, y, z, indexing="ij")

    def exact(self, name, t):
        X, Y, Z = self._grid(name)
        e = math.exp(-t)
        if name == "u":
            return np.sin(X) * np.cos(Y) * np.cos(Z) * e
        if name == "v":
            return -np.cos(X) * np.sin(Y) * np.cos(Z) * e
        if name == "w":
            return np.zeros_like(X)
        if name == "prd1":
            return 0.25 * (np.cos(2 * X) + np.cos(2 * Y)) * e * e
        raise KeyError(name)

    def source(self, name, t):
        # f = (3 nu - 1) e^-t A(x) - e^-2t B(x) / 2: the spatial factors are computed once
        if not hasattr(self, "_src"):
            self._src = {}
        if name not in self._src:
            X, Y, Z = self._grid(name)
            if name == "tf_u":
                self._src[name] = (np.sin(X) * np.cos(Y) * np.cos(Z), np.sin(2 * X) * np.sin(Z) ** 2)
            elif name == "tf_v":
                self._src[name] = (-np.cos(X) * np.sin(Y) * np.cos(Z), np.sin(2 * Y) * np.sin(Z) ** 2)
            elif name == "tf_w":
                self._src[name] = (np.zeros_like(X), np.zeros_like(X))
            else:
                raise KeyError(name)
        a, b = self._src[name]
        e = math.exp(-t)
        return (3.0 * self.nu - 1.0) * e * a - 0.5 * e * e * b

    def init(self, model):
        model.iniciais(0.0)
        model.upload("ls", 1.0)
        model.level_set_ini()
        for name in ("u", "v", "w", "prd1"):
            model.upload(name, self.exact(name, 0.0))
        model.contorno(1)
        model.contorno(3)

    def step(self, model, it):
        t = it * self.p.dt
        for name in ("tf_u", "tf_v", "tf_w"):
            model.upload(name, self.source(name, t))
        return model.step(it)

    def errors(self, model, t):
        """L2 (rms) and Linf errors of u, v, w (interior faces) and of the mean-free pressure
        (cells) against the exact solution at time t."""
        n = self.p.nx
        out = {}
        for name in ("u", "v", "w", "prd1"):
            got = model.download(name)
            ref = self.exact(name, t)
            if name == "prd1":
                g = got[1:n + 1, 1:n + 1, 1:n + 1]
                r = ref[1:n + 1, 1:n + 1, 1:n + 1]
                g, r = g - g.mean(), r - r.mean()
            else:
                sl = {"u": np.s_[1:n + 1, 1:n + 1, 1:n + 1], "v": np.s_[1:n + 1, 1:n + 1, 1:n + 1],
                      "w": np.s_[1:n + 1, 1:n + 1, 1:n + 1]}[name]
                g, r = got[sl], ref[sl]
            d = g - r
            out[name] = {"l2": float(np.sqrt(np.mean(d * d))), "linf": float(np.abs(d).max())}
        return out
