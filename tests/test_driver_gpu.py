"""suli_run on the GPU: the reference's loop body as one entry point per subroutine
(mode=loop), suli_step (mode=step) and suli_step_host (mode=host) give the same state bit for
bit, and the state matches the Python driver's (Solver.step) on the same dam break.
"""
import os
import pathlib
import shutil
import subprocess

import numpy as np
import pytest

from helpers import pkg

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parent.parent
SRC = ROOT / "suli-openmp_b200" / "csrc" / "suli_run.cpp"
LIB = ROOT / "suli-openmp_b200" / "lib"
FIELDS = ["u", "v", "w", "prd1", "ls"]
CASE = ["case=dam_break", "nx=32", "ny=16", "nz=24", "dx=0.02", "cg_tol=1e-12", "steps=3"]


@pytest.fixture(scope="module")
def suli_run(tmp_path_factory):
    pkg.load_library()
    cxx = os.environ.get("CXX") or shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = tmp_path_factory.mktemp("driver_gpu") / "suli_run"
    subprocess.run([cxx, "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(SRC), f"-L{LIB}", "-lsuli_gpu",
                    f"-Wl,-rpath,{LIB}", "-o", str(exe)], check=True)
    return exe


def test_modes_agree_and_match_python_driver(suli_run, tmp_path):
    outs, states = {}, {}
    p, init = pkg.cases.dam_break(nx=32, ny=16, nz=24, dx=0.02, cg_tol=1e-12)
    shapes = {f: pkg.field_shape(p, f) for f in FIELDS}
    for mode in ("loop", "step", "host"):
        r = subprocess.run([str(suli_run), *CASE, f"mode={mode}", f"dump={tmp_path / mode}"], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("it ")]
        assert len(lines) == 3
        outs[mode] = lines
        states[mode] = {f: np.fromfile(tmp_path / f"{mode}_{f}.bin", dtype=np.float64).reshape(shapes[f], order="F")
                        for f in FIELDS}
    assert outs["loop"] == outs["step"] == outs["host"]
    for f in FIELDS:
        assert np.array_equal(states["loop"][f], states["step"][f]), f
        assert np.array_equal(states["loop"][f], states["host"][f]), f
    for ln in outs["loop"]:
        assert float(ln.split("max|div u|")[1].split()[0]) <= 1e-10, ln
    # the Python driver on the same case and steps
    s = pkg.Solver(p)
    init(s)
    for it in range(1, 4):
        assert s.step(it)["status"] == 0
    vs = max(float(np.abs(s.download(f)).max()) for f in ("u", "v", "w"))
    for f in FIELDS:
        a, b = states["loop"][f], s.download(f)
        scale = vs if f in ("u", "v", "w") else max(float(np.abs(b).max()), 1e-300)
        assert float(np.abs(a - b).max()) <= 1e-12 * scale, f
    s.close()
