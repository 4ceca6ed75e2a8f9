"""Bottom obstacles (obst_t != 0): the masks of obstaculo, the obstacle columns of contorno(1/2),
the level set inside the obstacle of contorno(3) and the masked inflow planes of iniciais
(3_contorno.f90:266-294, 445-487, 494-762; 2_iniciais.f90:60-65).

CPU tests pin the oracle to the reference's rules, restated here per column and per cell; GPU
tests compare the library with the oracle through the C-ABI."""
import numpy as np
import pytest

from helpers import load_state, pkg, rel_err, seeded_state, small_params

cases = pkg.cases


def random_masks(p, seed):
    """Masks over the whole range suli_set_obstacle accepts, neighbours of different heights."""
    rng = np.random.default_rng(seed)
    shapes = pkg._abi.mask_shapes(p)
    return [np.asfortranarray(rng.integers(-1, p.nz + 1 + (m == 2), size=s), dtype=np.int32)
            for m, s in enumerate(shapes)]


def obstacle_params(bc=(1, 1, 1, 1, 1, 1)):
    p = small_params(nx=9, ny=7, nz=8, bc=bc)
    q = p.copy()
    q.obst_t = 3
    return p, q


def state_with_ghosts(p, seed):
    rng = np.random.default_rng(seed)
    st = seeded_state(p, seed)
    for f in ("ub", "vb", "wb"):
        st[f] = rng.standard_normal(pkg.field_shape(p, f))
    st["ls"] = rng.standard_normal(pkg.field_shape(p, "ls"))
    return st


# ------------------------------------------------------------------------------- CPU
def test_nint_and_floor_of_the_masks():
    """A flat bottom h: ku = nint(h/dz + 1/2) rounds halves away from zero, kw = floor(h/dz + 1)."""
    p = small_params(nx=6, ny=5, nz=10)
    p.dz = 0.05
    for h, ku, kw in ((0.2, 5, 5), (0.21, 5, 5), (0.0, 1, 1), (-0.05, -1, 0), (0.024, 1, 1)):
        m = cases.obstacle_masks(p, lambda i, j: np.full(np.broadcast_shapes(i.shape, j.shape), h))
        assert (m[0] == ku).all() and (m[1] == ku).all() and (m[2] == kw).all(), (h, m[0].min(), m[2].min())
    m = cases.obstacle_masks(p, lambda i, j: np.full(np.broadcast_shapes(i.shape, j.shape), 9.0))
    assert (m[0] == p.nz).all() and (m[2] == p.nz + 1).all()      # clamped to nz and nz+1


def test_presets():
    """obstaculo presets: the Gaussian bump's peak column and the walls of preset 10."""
    p = small_params(nx=60, ny=30, nz=60)
    p.dx = p.dy = p.dz = 0.1
    ku, kv, kw = cases.obstaculo(p, 3)
    # h = 2 exp(-(x-3)^2/0.5 - (y-1.5)^2/0.5) + 0.2, kw sampled at x = (2i-1) dx/2, y = (2j-1) dy/2,
    # ku at x = (2i-2) dx/2, y = (2j-1) dy/2
    h = lambda x, y: np.exp(-((x - 3.) * (x - 3.) / 0.5) - (y - 1.5) * (y - 1.5) / 0.5) * 2.0 + 0.2
    for i, j in ((30, 15), (31, 16), (25, 10), (0, 0)):
        assert kw[i, j] == int(np.floor(h((2 * i - 1) * 0.05, (2 * j - 1) * 0.05) / p.dz + 1.)), (i, j)
        assert ku[i, j] == int(cases._nint(np.array([h((2 * i - 2) * 0.05, (2 * j - 1) * 0.05) / p.dz + 0.5]))[0])
    assert kw.max() == 22 and kw.min() == 3
    q = small_params(nx=40, ny=20, nz=10)
    q.dx = q.dy = q.dz = 0.05
    ku, kv, kw = cases.obstaculo(q, 10)
    x_w = (2 * np.arange(q.nx + 2) - 1) * q.dx * 0.5
    wall = (x_w >= 0.67) & (x_w <= 0.83)
    y_w = (2 * np.arange(q.ny + 2) - 1) * q.dy * 0.5
    opening = (y_w > 0.3) & (y_w < 0.7)
    for i in range(q.nx + 2):
        for j in range(q.ny + 2):
            assert kw[i, j] == (int(np.floor(0.16 / q.dz + 1.)) if wall[i] and not opening[j] else 0)
    for t in range(1, 11):
        m = cases.obstaculo(q, t)
        assert [a.shape for a in m] == list(pkg._abi.mask_shapes(q))


def test_obstacle_columns(orc):
    """contorno(1) with masks = contorno(1) without, then per column: velocities zeroed for
    k <= mask, the first value above captured into ub, vb, wb; u at i = nx+2 and v at
    j = ny+2 only zeroed (3_contorno.f90:266-294)."""
    p, q = obstacle_params()
    masks = random_masks(p, 1)
    st = state_with_ghosts(p, 2)
    a = orc.Oracle(p); load_state(a, st); a.contorno(1)
    b = orc.Oracle(q); load_state(b, st); b.set_obstacle(*masks); b.contorno(1)
    ku, kv, kw = masks
    for name, nb, m, (ni, nj) in (("u", "ub", ku, (p.nx + 3, p.ny + 2)), ("v", "vb", kv, (p.nx + 2, p.ny + 3)),
                                  ("w", "wb", kw, (p.nx + 2, p.ny + 2))):
        want, want_b = a.download(name), st[nb].copy()
        for i in range(ni):
            for j in range(nj):
                want[i, j, :m[i, j] + 1] = 0.
                main = i <= p.nx + 1 and j <= p.ny + 1
                if main:
                    want_b[i, j, m[i, j] + 1] = want[i, j, m[i, j] + 1]
        assert np.array_equal(b.download(name), want), name
        assert np.array_equal(b.download(nb), want_b), nb


def ls_extension_py(ls, kw, nx, ny, nz):
    """contorno(3)'s branch table (3_contorno.f90:446-481) per cell; neighbours outside the
    domain count as not fluid."""
    out = ls.copy()
    L = lambda i, j, k: ls[i - 1, j - 1, k - 1]
    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            for k in range(1, kw[i, j]):
                fl = lambda a, b: 1 <= a <= nx and 1 <= b <= ny and kw[a, b] < k
                so = lambda a, b: kw[a, b] >= k
                if fl(i - 1, j) and fl(i, j - 1):
                    v = (L(i - 1, j, k) + L(i, j - 1, k)) * 0.5
                elif fl(i + 1, j) and fl(i, j - 1):
                    v = (L(i + 1, j, k) + L(i, j - 1, k)) * 0.5
                elif fl(i + 1, j) and fl(i, j + 1):
                    v = (L(i + 1, j, k) + L(i, j + 1, k)) * 0.5
                elif fl(i - 1, j) and fl(i, j + 1):
                    v = (L(i - 1, j, k) + L(i, j + 1, k)) * 0.5
                elif fl(i - 1, j) and so(i, j - 1) and so(i, j + 1):
                    v = L(i - 1, j, k)
                elif fl(i, j - 1) and so(i - 1, j) and so(i + 1, j):
                    v = L(i, j - 1, k)
                elif fl(i + 1, j) and so(i, j - 1) and so(i, j + 1):
                    v = L(i + 1, j, k)
                elif fl(i, j + 1) and so(i - 1, j) and so(i + 1, j):
                    v = L(i, j + 1, k)
                elif k == kw[i, j] - 1 and k < nz:
                    v = L(i, j, k + 1)
                else:
                    continue
                out[i - 1, j - 1, k - 1] = v
    return out


@pytest.mark.parametrize("seed", [3, 4, 5])
def test_level_set_extension(orc, seed):
    """contorno(3): the level set inside the obstacle, then heaviside."""
    p, q = obstacle_params()
    masks = random_masks(p, seed)
    st = state_with_ghosts(p, seed)
    o = orc.Oracle(q); load_state(o, st); o.set_obstacle(*masks)
    o.contorno(3)
    want = ls_extension_py(st["ls"], masks[2], p.nx, p.ny, p.nz)
    assert np.array_equal(o.download("ls"), want)
    assert not np.array_equal(want, st["ls"])             # cells were extended
    r = orc.Oracle(p); load_state(r, st); r.upload("ls", want); r.heaviside()
    assert np.array_equal(o.download("rho"), r.download("rho"))


def test_iniciais_masks_inflow_planes(orc):
    """bxx1(:,0:ku(1,j)) = 0 for every j: whole rows up to the highest ku(1,j); bxx0 with
    ku(0,j) (2_iniciais.f90:60-65)."""
    p, q = obstacle_params()
    masks = random_masks(p, 6)
    o = orc.Oracle(q)
    o.set_obstacle(*masks)
    o.iniciais(0.7)
    for name, col in (("bxx1", 1), ("bxx0", 0)):
        kmax = masks[0][col, :].max()
        plane = o.download(name)[:, :, 0]
        assert (plane[:, :kmax + 1] == 0).all() and (plane[:, kmax + 1:] == 0.7).all(), name


def test_masks_out_of_range_refused(orc):
    p, q = obstacle_params()
    masks = random_masks(p, 7)
    masks[0][2, 3] = p.nz + 1
    with pytest.raises(ValueError):
        orc.Oracle(q).set_obstacle(*masks)


def test_bump_channel_steps(orc):
    """The obstacle case steps (oracle): columns stay zero, volume within the reference's
    trigger."""
    p, init, masks = cases.bump_channel(nx=32, ny=16, nz=24, dx=0.02)
    o = orc.Oracle(p)
    init(o)
    v0 = o.get_scalar("vol_ini")
    for it in range(1, 3):
        assert o.step(it)["status"] == 0
    u = o.download("u")
    ku = masks[0]
    assert all((u[i, j, :ku[i, j] + 1] == 0).all() for i in range(p.nx + 3) for j in range(p.ny + 2))
    assert abs(o.get_scalar("vol_ins") - v0) / v0 < 0.1


# ------------------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("bc", [(1, 1, 1, 1, 1, 1), (0, 0, 0, 0, 2, 1), (3, 4, 0, 0, 2, 1)])
def test_contorno_obstacle_gpu(orc, bc):
    """contorno(1), contorno(2) and contorno(3) with random masks: the GPU equals the oracle
    (exact for the copies and zeros; heaviside's fields within 1e-13)."""
    p, q = obstacle_params(bc)
    masks = random_masks(p, 11)
    st = state_with_ghosts(p, 12)
    g = pkg.Solver(q)
    o = orc.Oracle(q)
    for m in (g, o):
        load_state(m, st)
        m.set_obstacle(*masks)
    for nlock in (1, 2):
        for m in (g, o):
            m.contorno(nlock)
        for f in ("u", "v", "w", "ub", "vb", "wb", "prd1"):
            assert np.array_equal(g.download(f), o.download(f)), (nlock, f)
    for m in (g, o):
        m.contorno(3)
    assert np.array_equal(g.download("ls"), o.download("ls"))
    for f in ("hs", "rho", "ls_nu"):
        assert rel_err(g.download(f), o.download(f)) <= 1e-13, f
    g.close()


def _div_sum(m, p):
    """Sum over the cells of div u (the sum of graddin's right-hand side, 9_grad.f90:80-87)."""
    u, v, w = m.download("u"), m.download("v"), m.download("w")
    nx, ny, nz = p.nx, p.ny, p.nz
    d = ((u[2:nx + 2, 1:ny + 1, 1:nz + 1] - u[1:nx + 1, 1:ny + 1, 1:nz + 1]) / p.dx
         + (v[1:nx + 1, 2:ny + 2, 1:nz + 1] - v[1:nx + 1, 1:ny + 1, 1:nz + 1]) / p.dy
         + (w[1:nx + 1, 1:ny + 1, 2:nz + 2] - w[1:nx + 1, 1:ny + 1, 1:nz + 1]) / p.dz)
    return float(d.sum()), float(np.abs(d).sum())


def _stage_to_graddin(m, it, tt):
    m.set_dt(m.a_dt[tt - 1])
    m.visco()
    m.convdiff()
    m.tempo(tt, it)
    m.contorno(2)


def test_outflow_fix_restated(orc):
    """outflow_fix = 1: contorno(2) as with 0, then u(nx+1, j, k) above ku(nx+1, j) shifted by
    -(net boundary flux) / (open faces * dy * dz); the other fields untouched."""
    p, init, masks = cases.bump_channel(nx=32, ny=16, nz=24, dx=0.02)
    q = p.copy()
    q.outflow_fix = 1
    a, b = orc.Oracle(p), orc.Oracle(q)
    for m in (a, b):
        init(m)
        m.level_set()
        m.contorno(3)
        _stage_to_graddin(m, 1, 1)
    u = a.download("u")
    nx, ny, nz = p.nx, p.ny, p.nz
    v, w = a.download("v"), a.download("w")
    fx = (u[nx + 1, 1:ny + 1, 1:nz + 1] - u[1, 1:ny + 1, 1:nz + 1]).sum()
    fy = (v[1:nx + 1, ny + 1, 1:nz + 1] - v[1:nx + 1, 1, 1:nz + 1]).sum()
    fz = (w[1:nx + 1, 1:ny + 1, nz + 1] - w[1:nx + 1, 1:ny + 1, 1]).sum()
    net = fx * p.dy * p.dz + fy * p.dx * p.dz + fz * p.dx * p.dy
    ku = masks[0]
    kk = np.arange(1, nz + 1)[None, :]
    open_ = kk > ku[nx + 1, 1:ny + 1][:, None]
    want = u.copy()
    want[nx + 1, 1:ny + 1, 1:nz + 1] += np.where(open_, -net / (open_.sum() * p.dy * p.dz), 0.0)
    got = b.download("u")
    assert abs(net) > 1e-9                       # the reference's copy leaves a net flux here
    assert np.allclose(got, want, rtol=0, atol=1e-15)
    for f in ("v", "w", "prd1", "ls"):
        assert np.array_equal(a.download(f), b.download(f)), f
    s, sabs = _div_sum(b, p)
    assert abs(s) <= 1e-13 * sabs


def test_outflow_fix_makes_the_solve_consistent(orc):
    """With the reference's outflow the Poisson system of the bump channel is inconsistent: the
    CG reaches its relative tolerance on the recurrence residual, yet a second solve from that
    result needs many iterations again.  With outflow_fix = 1 the second solve needs none."""
    for fix, again in ((0, lambda n: n > 100), (1, lambda n: n == 0)):
        p, init, masks = cases.bump_channel(nx=32, ny=16, nz=24, dx=0.02, cg_tol=1e-12, outflow_fix=fix)
        o = orc.Oracle(p)
        init(o)
        for it in (1, 2):
            o.level_set()
            o.contorno(3)
            for tt in range(1, o.ntt + 1):
                _stage_to_graddin(o, it, tt)
                n1, r1 = o.graddin()
                n2, r2 = o.graddin()
                assert r1 <= 1e-12 and r2 <= 1e-12
                if it == 2:
                    assert again(n2), (fix, tt, n1, n2)
                o.posdin()
                o.contorno(1)


@pytest.mark.gpu
@pytest.mark.parametrize("bc", [(3, 4, 0, 0, 2, 1), (3, 4, 2, 2, 2, 2)])
def test_outflow_fix_gpu(orc, bc):
    """contorno(2) with outflow_fix = 1 and random obstacle masks: the GPU equals the oracle
    (the shift differs only by the order of its sums)."""
    p, q = obstacle_params(bc)
    q.outflow_fix = 1
    masks = random_masks(p, 13)
    st = state_with_ghosts(p, 14)
    g = pkg.Solver(q)
    o = orc.Oracle(q)
    for m in (g, o):
        load_state(m, st)
        m.set_obstacle(*masks)
        m.contorno(2)
    for f in ("v", "w", "ub", "vb", "wb", "prd1"):
        assert np.array_equal(g.download(f), o.download(f)), f
    assert rel_err(g.download("u"), o.download("u")) <= 1e-14
    g.close()


@pytest.mark.gpu
def test_step_parity_obstacle(orc):
    """Three steps of the channel over a bottom bump (inflow, outflow with outflow_fix, periodic
    y): iteration counts close, every state field within 1e-10 of its scale, the velocities
    within 1e-10 of the velocity scale.  The reference's own outflow makes this Poisson system
    inconsistent (test_outflow_fix_makes_the_solve_consistent), and the iterates of an
    inconsistent CG depend on rounding, so the comparison is made on the consistent system."""
    p, init, masks = cases.bump_channel(nx=32, ny=16, nz=24, dx=0.02, cg_tol=1e-12, outflow_fix=1)
    g = pkg.Solver(p)
    o = orc.Oracle(p)
    init(g)
    init(o)
    for it in range(1, 4):
        sg, so = g.step(it), o.step(it)
        assert sg["status"] == 0 and so["status"] == 0
        assert all(abs(a - b) <= max(3, 0.02 * b) for a, b in zip(sg["cg_iters"], so["cg_iters"]))
    vel = {f: (g.download(f), o.download(f)) for f in ("u", "v", "w")}
    vs = max(float(np.abs(b).max()) for _, b in vel.values())
    worst = {f: float(np.abs(a - b).max()) / vs for f, (a, b) in vel.items()}
    worst.update({f: rel_err(g.download(f), o.download(f)) for f in ("ls", "rho", "ub", "wb")})
    pg, po = g.download("prd1"), o.download("prd1")
    worst["prd1(mean-free)"] = rel_err(pg - pg.mean(), po - po.mean())
    assert max(worst.values()) <= 1e-10, worst
    g.close()


def test_restart_and_campos_carry_the_masks(orc, tmp_path):
    """A restart of an obstacle run carries ku, kv, kw and restores them; the campos record's
    obstacle field is 1 at the cells k < kw (4_plot.f90:285-296)."""
    p, init, masks = cases.bump_channel(nx=32, ny=16, nz=24, dx=0.02)
    o = orc.Oracle(p)
    init(o)
    assert o.step(1)["status"] == 0
    f = tmp_path / "arquivorestart"
    pkg.fileio.write_restart(o, f)
    r = orc.Oracle(p)
    pkg.fileio.read_restart(r, f)
    for a, b in zip(r.obstacle, masks):
        assert np.array_equal(a, b)
    assert o.step(2)["cg_iters"] == r.step(2)["cg_iters"]
    assert np.array_equal(o.download("u"), r.download("u"))
    wr = pkg.fileio.FieldWriter(tmp_path, p, t_plot=0)
    wr.snapshot(o)
    wr.close()
    kaux = pkg.fileio.read_campos(tmp_path / "campos_00010", p, 0)[7]
    kw = masks[2]
    for i, j in ((1, 1), (16, 8), (20, 3)):
        assert (kaux[i - 1, j - 1, :] == (np.arange(1, p.nz + 1) < kw[i, j])).all()


def test_les_channel_steps(orc):
    """The LES channel at 64 x 32 x 32 runs 12 steps on the oracle with both consistency options
    (every solve converged, the level-set volume within 1e-4); with the reference's end faces
    across the periodic y boundary its CG breaks down within those steps."""
    for pf in (1, 0):
        p, init, masks = cases.les_channel(nx=64, ny=32, nz=32, periodic_faces=pf)
        p.cg_maxit = 3000
        o = orc.Oracle(p, openmp=True)
        init(o)
        v0 = o.get_scalar("vol_ini")
        ok = True
        for it in range(1, 13):
            st = o.step(it)
            ok = ok and st["status"] == 0 and max(st["cg_resid"]) <= 1e-8
            if not ok:
                break
        if pf == 1:
            assert ok and abs(o.get_scalar("vol_ins") - v0) / v0 < 1e-4
        else:
            assert not ok


def test_les_channel_case():
    """Config C5 built at a small size: the 6 x 3 x 3 m box, the 0.3 m bump's masks, the seeded
    inflow 1 +- 0.05."""
    p, init, masks = cases.les_channel(nx=48, ny=24, nz=24)
    assert (p.nx * p.dx, p.ny * p.dy, p.nz * p.dz) == (6.0, 3.0, 3.0) and p.obst_t == 3
    kw = masks[2]
    assert kw.max() == int(np.floor(0.3 * np.exp(-(((2 * 24 - 1) * p.dx / 2 - 3.0) ** 2 / 0.5)
                                                   - ((2 * 12 - 1) * p.dy / 2 - 1.5) ** 2 / 0.5) / p.dz + 1.))
    assert kw.min() == 1
