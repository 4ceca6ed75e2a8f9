"""suli_run, the native host program that runs the reference's time loop through the C-ABI.

On the CPU the tests build it from suli-openmp_b200/csrc/suli_run.cpp against
include/suli_gpu.h and libsuli_gpu.so (so the header compiles as C++ and every entry point
it uses links), then check its argument handling, that its presets (time step and level set)
are the Python cases', and that, with no GPU, it stops at suli_create with SULI_ERR_NODEVICE
instead of running anything on the host.
"""
import os
import pathlib
import shutil
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
SRC = ROOT / "suli-openmp_b200" / "csrc" / "suli_run.cpp"
LIB = ROOT / "suli-openmp_b200" / "lib"


@pytest.fixture(scope="module")
def suli_run(tmp_path_factory, pkg):
    pkg.load_library()   # fails loudly if the library was not built
    cxx = os.environ.get("CXX") or shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = tmp_path_factory.mktemp("driver") / "suli_run"
    subprocess.run([cxx, "-O1", "-std=c++17", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", str(SRC),
                    f"-L{LIB}", "-lsuli_gpu", f"-Wl,-rpath,{LIB}", "-o", str(exe)], check=True)
    return exe


def _run(exe, *args):
    return subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("args", [("bogus",), ("mode=fast",), ("case=cavity",), ("nx=0",), ("steps",),
                                  ("precision=2",)])
def test_usage_errors(suli_run, args):
    r = _run(suli_run, *args)
    assert r.returncode == 1
    assert "usage: suli_run" in r.stderr


@pytest.mark.parametrize("mode", ["loop", "step", "host"])
def test_no_gpu_stops_at_create(suli_run, mode):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    r = _run(suli_run, f"mode={mode}", "steps=2", "nx=16", "ny=8", "nz=12", "dx=0.04")
    assert r.returncode == 2
    assert "SULI_ERR_NODEVICE" in r.stderr
    assert "it " not in r.stdout   # no step ran


class _Recorder:
    """Stands in for a solver in a case's init closure and keeps the level-set preset."""

    def __init__(self):
        self.ls = None

    def upload(self, name, a):
        if name == "ls":
            self.ls = np.asfortranarray(a, dtype=np.float64)

    def __getattr__(self, name):   # iniciais, level_set_ini, contorno, set_obstacle
        return lambda *a, **k: None


@pytest.mark.parametrize("case,shape,dx", [("dam_break", (24, 8, 16), 0.02), ("sloshing", (32, 16, 16), 0.02)])
def test_presets_match_python_cases(suli_run, pkg, tmp_path, case, shape, dx):
    """The program's time step and level-set preset are the Python cases' (bit for bit for the
    dam break; the sloshing surface's cosines may differ in the last bits between the C library
    and numpy)."""
    nx, ny, nz = shape
    out = tmp_path / "preset.bin"
    r = _run(suli_run, f"case={case}", f"nx={nx}", f"ny={ny}", f"nz={nz}", f"dx={dx}", f"preset={out}")
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, dtype=np.float64)
    dt, ls = raw[0], raw[1:].reshape(shape, order="F")
    p, init = getattr(pkg.cases, case)(nx=nx, ny=ny, nz=nz, dx=dx)
    rec = _Recorder()
    init(rec)
    assert dt == p.dt
    if case == "dam_break":
        assert np.array_equal(ls, rec.ls)
    else:
        assert float(np.abs(ls - rec.ls).max()) <= 4 * np.finfo(np.float64).eps * float(np.abs(rec.ls).max())
