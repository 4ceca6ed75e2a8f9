"""GPU: manufactured-solution verification on the periodic box (cases.TaylorGreenMMS).

The exact solution is known, so the checks are absolute as well as relative:
* the FP64 GPU run equals the oracle's run of the same steps to 1e-10 per field, and its
  errors against the exact fields equal the oracle's;
* the mixed-precision run (FP32 inner solves, FP64 refinement to the same tolerance)
  follows the FP64 GPU run to 1e-7 in velocity and 1e-6 in (mean-free) pressure, and so
  has the same errors against the exact fields;
* max |div u| after every step stays below 1e-8.
"""
import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu

N, STEPS = 32, 10


def _run(pkg, model, m):
    m.init(model)
    divs = []
    for it in range(1, STEPS + 1):
        st = m.step(model, it)
        assert st["status"] == 0, st
        divs.append(st["max_div"])
    return divs


def _fields(model):
    out = {k: model.download(k) for k in ("u", "v", "w")}
    p = model.download("prd1")[1:-1, 1:-1, 1:-1]
    out["prd1"] = p - p.mean()
    return out


def test_mms_fp64_matches_oracle_and_exact(pkg, orc):
    m = pkg.cases.TaylorGreenMMS(N, precision=0)
    g = pkg.Solver(m.p)
    o = orc.Oracle(m.p)
    dg = _run(pkg, g, m)
    _run(pkg, o, m)
    assert max(dg) <= 1e-8
    fg, fo = _fields(g), _fields(o)
    # velocity components relative to the velocity scale (w is ~1e-5 of it), pressure to its own
    vs = max(float(np.abs(fo[k]).max()) for k in ("u", "v", "w"))
    for k in ("u", "v", "w"):
        assert float(np.abs(fg[k] - fo[k]).max()) <= 1e-10 * vs, k
    assert rel_err(fg["prd1"], fo["prd1"]) <= 1e-10
    t = STEPS * m.p.dt
    eg, eo = m.errors(g, t), m.errors(o, t)
    for k in eg:
        assert abs(eg[k]["l2"] - eo[k]["l2"]) <= 1e-8 * max(eo[k]["l2"], 1e-12), k
    # first-order upwind advection at 32^3: velocity error ~2e-4 after 10 steps
    assert eg["u"]["l2"] < 5e-4 and eg["prd1"]["l2"] < 3e-3, eg
    g.close()


def test_mms_mixed_tracks_fp64(pkg):
    res = {}
    for prec in (0, 1):
        m = pkg.cases.TaylorGreenMMS(N, precision=prec)
        s = pkg.Solver(m.p)
        divs = _run(pkg, s, m)
        assert max(divs) <= 1e-8, (prec, max(divs))
        res[prec] = (_fields(s), m.errors(s, STEPS * m.p.dt))
        s.close()
    (f0, e0), (f1, e1) = res[0], res[1]
    for k in ("u", "v"):
        assert rel_err(f1[k], f0[k]) <= 1e-7, k
    assert rel_err(f1["prd1"], f0["prd1"]) <= 1e-6
    for k in e0:
        assert abs(e1[k]["l2"] - e0[k]["l2"]) <= 1e-3 * e0[k]["l2"] + 1e-9, (k, e0[k], e1[k])
