"""CPU: the benchmark's accounting, without a GPU.

* the algorithmic byte and FLOP counts the rooflines divide by (CG kernel A, the inner PCG
  iteration, the U-Net forward) against hand counts;
* the committed ncu summaries the benchmark reads (DRAM bytes per launch, kernel shares) exist
  and parse, so a bench line always carries its `traffic` and kernel-A duration split;
* the plain-path roofline from a synthetic tracer record: the iteration time apportioned by the
  committed launch-list share.
"""
import importlib.util
import pathlib

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_unet_flops_hand_count(bench, pkg):
    p = pkg.snapshots.tank_params(n=16, precision=1)
    p.nx, p.ny, p.nz = 256, 128, 128
    V = 256 * 128 * 128
    per_level = {0: 0, 1: 0, 2: 0, 3: 0}
    for ci, co, lv in pkg.learned.LAYERS:
        per_level[lv] += ci * co
    want = sum(2 * 27 * s * V // 8 ** lv for lv, s in per_level.items()) + 2 * 16 * V
    assert bench.unet_flops(pkg, p) == want
    assert abs(want - 586.75e9) < 0.01e9   # 586.7 GFLOP per forward at 256x128x128


def test_inner_iteration_bytes(bench, pkg):
    p = pkg.snapshots.tank_params(n=16, precision=1)
    p.nx, p.ny, p.nz = 256, 128, 128
    b = bench.mg_iteration_bytes(p)
    N = 256 * 128 * 128
    # 28.25 fine passes plus 25.25 passes of each coarser level down to the coarsest grid of
    # 1024 cells (1/8, 1/64, 1/512, 1/4096 of N), 4-byte values
    want = 4 * N * (28.25 + 25.25 * (1 / 8 + 1 / 64 + 1 / 512 + 1 / 4096))
    assert abs(b - want) <= 1e-6 * want


def test_committed_profiles_parse(bench):
    N = 256 * 128 * 128
    t = bench.profiled_traffic("cg_spmv2_256x128x128", N)
    assert t is not None and 1e8 < t < 5e8
    t = bench.profiled_traffic("unet_forward_256x128x128", N)
    assert t is not None and 5e8 < t < 5e9
    s = bench.launch_share("launches_sloshing_256x128x128_fp64", "k_cg_spmv2", ("k_cg_spmv2", "k_cg_update"))
    assert s is not None and 0.3 < s < 0.8


def test_plain_roofline_from_tracer(bench, pkg):
    p = pkg.snapshots.tank_params(n=16, precision=0)
    p.nx, p.ny, p.nz = 256, 128, 128
    it = 1000
    prof = {"cg_iterations": it, "cg_spmv": {"ms": 100.0}, "cg_update": {"ms": 5.0}}
    r = bench.cg_roofline(p, prof)
    t_it = 105.0 / it / 1e3
    share = bench.launch_share("launches_sloshing_256x128x128_fp64", "k_cg_spmv2", ("k_cg_spmv2", "k_cg_update"))
    assert abs(r["cg_iteration"]["us"] - t_it * 1e6) < 1e-9
    assert abs(r["avg_launch_us"] - t_it * share * 1e6) < 1e-9
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12


@pytest.mark.parametrize("openmp", [False, True])
def test_cpu_steps_are_whole_timed_steps(bench, pkg, openmp):
    """The CPU baseline times whole steps: one untimed step, then the timed ones, every Poisson
    solve to the same stopping tests as the GPU (both met), no iteration cap; the serial build
    runs on one thread."""
    p, init = pkg.cases.sloshing(nx=16, ny=8, nz=8, dx=0.04, cg_tol=1e-8, div_tol=1e-8)
    s = bench.cpu_steps(pkg, p, init, 2, openmp=openmp)
    assert len(s["t_step_s"]) == 2 and all(t > 0 for t in s["t_step_s"])
    assert s["steps_timed"] == [2, 3]
    assert s["max_div"] <= 1e-8 and s["cg_resid_max"] <= 1e-8
    assert all(n > 0 for n in s["poisson_iters_per_step"])
    assert s["t_step_s_median"] == sorted(s["t_step_s"])[0] + (sorted(s["t_step_s"])[1] - sorted(s["t_step_s"])[0]) / 2
    if not openmp:
        assert s["cores"] == 1
    assert "no iteration cap" in bench.cpu_desc(s, openmp)


def test_field_errors(bench):
    """Velocity errors over the velocity scale, level set and pressure over their own scale."""
    import numpy as np
    ref = {"u": np.array([2.0, -1.0]), "v": np.array([0.5, 0.0]), "w": np.array([0.1, 0.0]),
           "ls": np.array([4.0, -4.0]), "prd1": np.array([10.0, -10.0])}
    a = {k: v.copy() for k, v in ref.items()}
    a["v"][1] += 1e-3
    a["ls"][0] += 4e-3
    e = bench.field_errors(a, ref)
    assert e["u"] == 0.0 and abs(e["v"] - 5e-4) < 1e-15 and abs(e["ls"] - 1e-3) < 1e-15 and e["prd1"] == 0.0
