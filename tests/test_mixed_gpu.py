"""GPU tests of the mixed-precision path (precision = 1): FP32 stencil arithmetic over the FP64
fields, and the pressure solve as FP32 multigrid-preconditioned CG inside FP64 iterative
refinement, stopping on the same FP64 relative residual as the plain path.  Each result is checked against the FP64 CPU oracle solved to a
tighter tolerance; the error bars are stated per test."""
import numpy as np
import pytest

from helpers import STATE_FIELDS, load_state, rel_err, seeded_state, small_params

pytestmark = pytest.mark.gpu


def _prepared(pkg, orc, p, seed):
    """Oracle-derived state (rho, viscosities, ghosts) uploaded to a GPU context."""
    o = orc.Oracle(p)
    st = seeded_state(p, seed)
    load_state(o, st)
    o.heaviside(); o.mod_ls1(); o.visco(); o.contorno(1)
    full = {f: o.download(f) for f in STATE_FIELDS}
    return o, full


@pytest.mark.parametrize("shape", [(16, 12, 8), (14, 12, 10), (32, 16, 24)])
def test_mixed_poisson_reaches_fp64_tolerance(pkg, orc, shape):
    """Relative FP64 residual <= 1e-10 (the solver's own test), and the projected velocity
    within 1e-7 of the oracle's FP64 CG at 1e-13 (both solutions are within the tolerance of
    the exact discrete one)."""
    p = small_params(nx=shape[0], ny=shape[1], nz=shape[2])
    p.cg_stop, p.cg_maxit = 1, 20000
    q = p.copy()
    q.precision, q.cg_tol, q.inner_tol, q.refine_maxit = 1, 1e-10, 1e-3, 30
    p.cg_tol = 1e-13
    o, st = _prepared(pkg, orc, p, 31)
    g = pkg.Solver(q)
    load_state(g, st)
    for m in (g, o):
        m.set_dt(1e-3)
        m.contorno(2)
    ng, rg = g.graddin()
    no, ro = o.graddin()
    assert rg <= 1e-10, rg
    assert ng < no, (ng, no)            # the preconditioned inner solve needs fewer iterations
    for m in (g, o):
        m.posdin()
        m.contorno(1)
    for f in ("u", "v", "w"):
        assert rel_err(g.download(f), o.download(f)) <= 1e-7, f
    assert g.est() <= 1e-6


def test_mixed_steps_track_fp64(pkg, orc):
    """Three dam-break steps of the mixed path (FP32 stencil arithmetic, FP32 inner solves,
    FP64 refinement to 1e-10) against the FP64 oracle at 1e-12: every field within 1e-6 of its
    own scale, the velocity components within 1e-6 of the velocity scale (v, across the tank,
    is about 1e-6 of u in this nearly two-dimensional flow, so its own maximum is no scale)."""
    p, init = pkg.cases.dam_break(nx=32, ny=16, nz=24, dx=0.02, cg_tol=1e-12)
    q = p.copy()
    q.precision, q.cg_tol, q.inner_tol, q.refine_maxit = 1, 1e-10, 1e-3, 30
    g = pkg.Solver(q)
    o = orc.Oracle(p)
    init(g)
    init(o)
    for it in range(1, 4):
        sg, so = g.step(it), o.step(it)
        assert sg["status"] == 0
        assert max(sg["cg_resid"]) <= 1e-10
    vel = {f: (g.download(f), o.download(f)) for f in ("u", "v", "w")}
    vs = max(float(np.abs(b).max()) for _, b in vel.values())
    for f, (a, b) in vel.items():
        assert float(np.abs(a - b).max()) <= 1e-6 * vs, f
    for f in ("ls", "rho"):
        assert rel_err(g.download(f), o.download(f)) <= 1e-6, f


@pytest.mark.parametrize("case", ["dam_break", "periodic"])
def test_cluster_levels_match_per_level_kernels(pkg, monkeypatch, case):
    """The three coarsest levels in one 16-CTA cluster launch (mg_kernels = 2) against the same
    levels as kernels per level (mg_kernels = 0): the same stages and per-cell arithmetic (only
    the restriction to the coarsest grid adds its children in two halves), so the inner solves
    follow the same course.  Walls (dam break 128x64x64, cluster levels 64x32x32 .. 16x8x8) and a
    box periodic in every direction (64^3, so the z wrap crosses from the last CTA to the first),
    two steps each: iteration counts within 2 per step, velocities within 1e-9 of their scale, and
    the tracer shows the cluster path's launch count (7 kernels an inner iteration, not 15).
    The per-level side keeps four kernels a coarse level (SULI_MG_FUSED=0)."""
    monkeypatch.setenv("SULI_MG_FUSED", "0")
    res = {}
    for mk in (0, 2):
        if case == "dam_break":
            p, init = pkg.cases.dam_break(nx=128, ny=64, nz=64, dx=0.005, cg_tol=1e-10)
            p.precision, p.inner_tol, p.refine_maxit = 1, 1e-4, 30
            p.mg_kernels = mk
            s = pkg.Solver(p)
            init(s)
            s.profile_enable(True)
            steps = [s.step(it) for it in (1, 2)]
        else:
            m = pkg.cases.TaylorGreenMMS(64, precision=1)
            m.p.mg_kernels = mk
            s = pkg.Solver(m.p)
            m.init(s)
            s.profile_enable(True)
            steps = [m.step(s, it) for it in (1, 2)]
        prof = s.profile_read()
        s.profile_enable(False)
        assert all(st["status"] == 0 for st in steps)
        iters = [sum(st["cg_iters"]) if isinstance(st["cg_iters"], list) else st["cg_iters"] for st in steps]
        res[mk] = (iters, {f: s.download(f) for f in ("u", "v", "w")}, prof)
        s.close()
    (it0, v0, p0), (it2, v2, p2) = res[0], res[2]
    assert all(abs(a - b) <= 2 for a, b in zip(it0, it2)), (it0, it2)
    vs = max(float(np.abs(b).max()) for b in v0.values())
    for f in v0:
        assert float(np.abs(v0[f] - v2[f]).max()) <= 1e-9 * vs, f
    per_it = lambda pr: pr["mg"]["launches"] / max(pr["cg_iterations"], 1)
    assert per_it(p2) < 0.6 * per_it(p0), (per_it(p2), per_it(p0))


def test_column_depths_agree(pkg, monkeypatch):
    """The vectorised kernels with 4 cells along z a thread (SULI_MG_KZ=4) against 2 (default):
    the same per-cell arithmetic, the FP64 dot products grouped differently; dam break
    128x64x64, two steps: iteration counts within 2, velocities within 1e-9 of their scale."""
    res = {}
    for kz in ("4", "2"):
        monkeypatch.setenv("SULI_MG_KZ", kz)
        p, init = pkg.cases.dam_break(nx=128, ny=64, nz=64, dx=0.005, cg_tol=1e-10)
        p.precision, p.inner_tol, p.refine_maxit = 1, 1e-4, 30
        s = pkg.Solver(p)
        init(s)
        steps = [s.step(it) for it in (1, 2)]
        assert all(st["status"] == 0 for st in steps)
        res[kz] = ([sum(st["cg_iters"]) for st in steps], {f: s.download(f) for f in ("u", "v", "w")})
        s.close()
    (i4, v4), (i2, v2) = res["4"], res["2"]
    assert all(abs(a - b) <= 2 for a, b in zip(i4, i2)), (i4, i2)
    vs = max(float(np.abs(b).max()) for b in v4.values())
    for f in v4:
        assert float(np.abs(v4[f] - v2[f]).max()) <= 1e-9 * vs, f


@pytest.mark.parametrize("shape,chunk", [((128, 64, 64), None), ((64, 36, 24), None), ((128, 64, 64), "7")])
def test_streaming_kernels_match_vectorised(pkg, monkeypatch, shape, chunk):
    """The level-0 kernels that stream z-planes through shared memory with TMA (default where
    they apply) against the vectorised level-0 kernels (SULI_NO_STREAM=1): per cell the same
    arithmetic, the FP64 dot products grouped differently.  Dam break at 128x64x64 (2 planes a
    CTA), at 64x36x24 (rows not a multiple of the 8-row tile, 1 plane a CTA) and at 128x64x64
    with 7 planes a CTA (SULI_STREAM_CHUNK: the slot ring wraps, the last CTA of a column has 1
    plane); two steps: iteration counts within 2, velocities within 1e-9 of their scale."""
    res = {}
    if chunk:
        monkeypatch.setenv("SULI_STREAM_CHUNK", chunk)
    for ns in ("1", "0"):
        monkeypatch.setenv("SULI_NO_STREAM", ns)
        nx, ny, nz = shape
        p, init = pkg.cases.dam_break(nx=nx, ny=ny, nz=nz, dx=0.005, cg_tol=1e-10)
        p.precision, p.inner_tol, p.refine_maxit = 1, 1e-4, 30
        s = pkg.Solver(p)
        init(s)
        steps = [s.step(it) for it in (1, 2)]
        assert all(st["status"] == 0 for st in steps)
        res[ns] = ([sum(st["cg_iters"]) for st in steps], {f: s.download(f) for f in ("u", "v", "w")})
        s.close()
    (i1, v1), (i0, v0) = res["1"], res["0"]
    assert all(abs(a - b) <= 2 for a, b in zip(i1, i0)), (i1, i0)
    vs = max(float(np.abs(b).max()) for b in v1.values())
    for f in v1:
        assert float(np.abs(v1[f] - v0[f]).max()) <= 1e-9 * vs, f


@pytest.mark.parametrize("case", ["dam_break", "periodic"])
def test_tail_kernel_matches_per_level_kernels(pkg, monkeypatch, case):
    """The last level above the coarsest and the coarsest solve in one CTA (k_mg_tail,
    SULI_TAIL=1) against their per-level kernels (default): the same per-cell
    arithmetic.  Walls (dam break 128x64x64: 32x16x16 and 16x8x8 in the CTA) and a box periodic
    in every direction (64^3: 16^3 and 8^3, wrapped neighbours); two steps: iteration counts
    within 2, velocities within 1e-9 of their scale."""
    res = {}
    for nt in ("0", "1"):
        monkeypatch.setenv("SULI_TAIL", nt)
        if case == "dam_break":
            p, init = pkg.cases.dam_break(nx=128, ny=64, nz=64, dx=0.005, cg_tol=1e-10)
            p.precision, p.inner_tol, p.refine_maxit = 1, 1e-4, 30
            s = pkg.Solver(p)
            init(s)
            steps = [s.step(it) for it in (1, 2)]
        else:
            m = pkg.cases.TaylorGreenMMS(64, precision=1)
            s = pkg.Solver(m.p)
            m.init(s)
            steps = [m.step(s, it) for it in (1, 2)]
        assert all(st["status"] == 0 for st in steps)
        iters = [sum(st["cg_iters"]) if isinstance(st["cg_iters"], list) else st["cg_iters"] for st in steps]
        res[nt] = (iters, {f: s.download(f) for f in ("u", "v", "w")})
        s.close()
    (i1, v1), (i0, v0) = res["1"], res["0"]
    assert all(abs(a - b) <= 2 for a, b in zip(i1, i0)), (i1, i0)
    vs = max(float(np.abs(b).max()) for b in v1.values())
    for f in v1:
        assert float(np.abs(v1[f] - v0[f]).max()) <= 1e-9 * vs, f


@pytest.mark.parametrize("case", ["dam_break", "periodic"])
def test_fused_coarse_legs_match_per_level_kernels(pkg, monkeypatch, case):
    """Each leg of the V-cycle on the coarse levels as one kernel (k_mgf_down, k_mgf_up;
    SULI_MG_FUSED=1) against the four per-level kernels (default): the same per-cell
    expressions, the cells around a tile recomputed under the operator's ghost map.  Walls
    (dam break 128x64x64) and a box periodic in every direction (64^3, wrapped neighbours around
    the tiles); two steps: iteration counts within 2, velocities within 1e-9 of their scale."""
    res = {}
    for fu in ("0", "1"):
        monkeypatch.setenv("SULI_MG_FUSED", fu)
        if case == "dam_break":
            p, init = pkg.cases.dam_break(nx=128, ny=64, nz=64, dx=0.005, cg_tol=1e-10)
            p.precision, p.inner_tol, p.refine_maxit = 1, 1e-4, 30
            s = pkg.Solver(p)
            init(s)
            steps = [s.step(it) for it in (1, 2)]
        else:
            m = pkg.cases.TaylorGreenMMS(64, precision=1)
            s = pkg.Solver(m.p)
            m.init(s)
            steps = [m.step(s, it) for it in (1, 2)]
        assert all(st["status"] == 0 for st in steps)
        iters = [sum(st["cg_iters"]) if isinstance(st["cg_iters"], list) else st["cg_iters"] for st in steps]
        res[fu] = (iters, {f: s.download(f) for f in ("u", "v", "w")})
        s.close()
    (i1, v1), (i0, v0) = res["1"], res["0"]
    assert all(abs(a - b) <= 2 for a, b in zip(i1, i0)), (i1, i0)
    vs = max(float(np.abs(b).max()) for b in v0.values())
    for f in v0:
        assert float(np.abs(v1[f] - v0[f]).max()) <= 1e-9 * vs, f


def test_chebyshev_coarsest_solve(pkg, monkeypatch):
    """The coarsest solve as the Chebyshev polynomial over [lo, 2] of the Jacobi-scaled operator
    (SULI_COARSE_CHEB=lo) against the damped Jacobi sweeps (SULI_COARSE_CHEB=0): another fixed
    symmetric positive preconditioner, so PCG still converges to the same FP64 tolerance; dam
    break 128x64x64 (levels down to 16x8x8), two steps: no more iterations than the Jacobi
    sweeps, velocities within 1e-7 of their scale (both solves stop at relative residual 1e-10)."""
    res = {}
    for lo in ("0", "0.02"):
        monkeypatch.setenv("SULI_COARSE_CHEB", lo)
        p, init = pkg.cases.dam_break(nx=128, ny=64, nz=64, dx=0.005, cg_tol=1e-10)
        p.precision, p.inner_tol, p.refine_maxit = 1, 1e-4, 30
        s = pkg.Solver(p)
        init(s)
        steps = [s.step(it) for it in (1, 2)]
        assert all(st["status"] == 0 for st in steps)
        res[lo] = (sum(sum(st["cg_iters"]) for st in steps), {f: s.download(f) for f in ("u", "v", "w")})
        s.close()
    (ic, vc), (ij, vj) = res["0.02"], res["0"]
    assert ic <= ij, (ic, ij)
    vs = max(float(np.abs(b).max()) for b in vj.values())
    for f in vj:
        assert float(np.abs(vc[f] - vj[f]).max()) <= 1e-7 * vs, f


def test_fused_update_matches_separate_update(pkg, monkeypatch):
    """The inner PCG update inside the level-0 pre-smoothing kernel (SULI_FUSED_UPDATE=1)
    against the separate update kernel (default): the same residual values, r.r summed in
    another grouping; dam break 128x64x64, two steps: iteration counts within 2, velocities
    within 1e-9 of their scale."""
    res = {}
    for fu in ("1", "0"):
        monkeypatch.setenv("SULI_FUSED_UPDATE", fu)
        p, init = pkg.cases.dam_break(nx=128, ny=64, nz=64, dx=0.005, cg_tol=1e-10)
        p.precision, p.inner_tol, p.refine_maxit = 1, 1e-4, 30
        s = pkg.Solver(p)
        init(s)
        steps = [s.step(it) for it in (1, 2)]
        assert all(st["status"] == 0 for st in steps)
        res[fu] = ([sum(st["cg_iters"]) for st in steps], {f: s.download(f) for f in ("u", "v", "w")})
        s.close()
    (i1, v1), (i0, v0) = res["1"], res["0"]
    assert all(abs(a - b) <= 2 for a, b in zip(i1, i0)), (i1, i0)
    vs = max(float(np.abs(b).max()) for b in v0.values())
    for f in v0:
        assert float(np.abs(v1[f] - v0[f]).max()) <= 1e-9 * vs, f


@pytest.mark.parametrize("case", ["dam_break", "periodic"])
def test_vector_kernels_match_one_cell_kernels(pkg, case):
    """The 4-cells-a-thread multigrid/PCG kernels (mg_kernels = 0) against the one-cell kernels
    (mg_kernels = 1): per cell the same arithmetic, only the FP64 dot products sum in another
    order, so the inner solves follow the same course.  Walls (dam break 64x32x32) and a box
    periodic in every direction (the manufactured-solution case, 32^3), two steps each: the
    iteration counts agree within 2 per step and the velocities within 1e-9 of their scale."""
    res = {}
    for mk in (0, 1):
        if case == "dam_break":
            p, init = pkg.cases.dam_break(nx=64, ny=32, nz=32, dx=0.01, cg_tol=1e-10)
            p.precision, p.inner_tol, p.refine_maxit = 1, 1e-4, 30
            p.mg_kernels = mk
            s = pkg.Solver(p)
            init(s)
            steps = [s.step(it) for it in (1, 2)]
        else:
            m = pkg.cases.TaylorGreenMMS(32, precision=1)
            m.p.mg_kernels = mk
            s = pkg.Solver(m.p)
            m.init(s)
            steps = [m.step(s, it) for it in (1, 2)]
        assert all(st["status"] == 0 for st in steps)
        res[mk] = ([sum(st["cg_iters"]) if isinstance(st["cg_iters"], list) else st["cg_iters"] for st in steps],
                   {f: s.download(f) for f in ("u", "v", "w")})
        s.close()
    (it0, v0), (it1, v1) = res[0], res[1]
    assert all(abs(a - b) <= 2 for a, b in zip(it0, it1)), (it0, it1)
    vs = max(float(np.abs(b).max()) for b in v1.values())
    for f in v0:
        assert float(np.abs(v0[f] - v1[f]).max()) <= 1e-9 * vs, f


@pytest.mark.parametrize("der, adv, m_turb", [(1, 1, 1), (2, 1, 2), (3, 1, 2), (1, 2, 1), (1, 3, 2)])
def test_mixed_stencils_track_fp64(pkg, orc, der, adv, m_turb):
    """visco and convdiff in FP32 arithmetic (precision 1), every advective form and scheme
    and both Smagorinsky models, against the FP64 oracle on the same state: face viscosities
    and forces within 1e-5 of each field's scale (FP32 rounding of terms no larger than the
    field's scale)."""
    p = small_params(nx=16, ny=12, nz=8, m_turb=m_turb)
    p.der, p.adv_type = der, adv
    q = p.copy()
    q.precision, q.cg_stop = 1, 1
    o, st = _prepared(pkg, orc, p, 41)
    g = pkg.Solver(q)
    load_state(g, st)
    for m in (g, o):
        m.visco()
        m.convdiff()
    for f in ("xnut", "ynut", "znut", "Fu", "Fv", "Fw"):
        assert rel_err(g.download(f), o.download(f)) <= 1e-5, f


@pytest.mark.parametrize("precision", [0, 1])
def test_divergence_stopping_test_gpu(pkg, orc, precision):
    """div_tol = 1e-8 on the sloshing tank: the FP64 CG (precision 0, threshold lowered and the
    device loop resumed) and the mixed solve (precision 1, more refinement passes) leave
    max |div u| <= 1e-8 after every step, with the relative residual <= 1e-8; the FP64 path
    stops where the oracle's does (iteration counts within 3 + 2 %)."""
    p, init = pkg.cases.sloshing(nx=32, ny=16, nz=16, dx=0.04, cg_tol=1e-8, div_tol=1e-8)
    q = p.copy()
    if precision == 1:
        q.precision, q.refine_maxit, q.inner_tol = 1, 30, 1e-4
    g = pkg.Solver(q)
    o = orc.Oracle(p)
    init(g)
    init(o)
    for it in (1, 2, 3):
        sg, so = g.step(it), o.step(it)
        assert sg["status"] == 0 and so["status"] == 0
        assert sg["max_div"] <= 1e-8 and max(sg["cg_resid"]) <= 1e-8, sg
        if precision == 0:
            assert all(abs(a - b) <= max(3, 0.02 * b) for a, b in zip(sg["cg_iters"], so["cg_iters"])), (sg, so)
    g.close()


def test_stalled_refinement_falls_back_to_fp64_cg(pkg):
    """The sloshing tank at 256x128x128 with inner solves to 1e-4 and the divergence test: later
    refinement passes stop converging (the FP32 inner solve hits its cap on the small, rough
    residuals), and the plain FP64 CG finishes those solves from the better iterate.  Every step
    still meets both stopping tests, and the fallback count says it happened."""
    p, init = pkg.cases.sloshing(cg_tol=1e-8, div_tol=1e-8)
    p.precision, p.refine_maxit, p.inner_tol = 1, 30, 1e-4
    s = pkg.Solver(p)
    init(s)
    for it in (1, 2, 3):
        st = s.step(it)
        assert st["status"] == 0 and max(st["cg_resid"]) <= 1e-8 and st["max_div"] <= 1e-8, st
    assert s.get_scalar("fallbacks") >= 1
    s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_eager_loops_match_graph_loops(pkg, precision, monkeypatch):
    """SULI_EAGER_LOOPS=1 (a profiling aid: iterations launched from the host instead of the
    device-side graph loop) runs the same kernels in the same order: bit-identical pressure,
    velocities and iteration counts over two steps."""
    p, init = pkg.cases.sloshing(nx=32, ny=16, nz=16, dx=0.04, cg_tol=1e-8, div_tol=1e-8)
    if precision == 1:
        p.precision, p.refine_maxit, p.inner_tol = 1, 30, 1e-4
    out = []
    for eager in ("0", "1"):
        monkeypatch.setenv("SULI_EAGER_LOOPS", eager)
        s = pkg.Solver(p)
        init(s)
        its = [s.step(it)["cg_iters"] for it in (1, 2)]
        out.append((its, {f: s.download(f) for f in ("u", "v", "w", "prd1")}))
        s.close()
    assert out[0][0] == out[1][0]
    for f in ("u", "v", "w", "prd1"):
        assert np.array_equal(out[0][1][f], out[1][1][f]), f


def test_mixed_rejects_unsupported(pkg):
    p = small_params(nx=15, ny=13, nz=11)   # cannot halve to <= 1024 cells
    p.precision, p.cg_stop = 1, 1
    with pytest.raises(pkg.SuliError):
        pkg.Solver(p)
