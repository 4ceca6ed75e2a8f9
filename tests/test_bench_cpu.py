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
def test_cpu_sample_scaling(bench, pkg, openmp):
    """The CPU baseline's step estimate: the capped step's non-Poisson time plus three solve
    set-ups plus the measured iteration count times the per-iteration cost; the serial build
    runs on one thread."""
    p, init = pkg.cases.sloshing(nx=16, ny=8, nz=8, dx=0.04, cg_tol=1e-8)
    s = bench.cpu_sample(pkg, p, init, 3, 40.0, openmp=openmp)
    assert s["t_noncg_s"] > 0 and s["t_iter_s"] > 0 and s["iters_per_step"] == 40.0
    want = s["t_noncg_s"] + 3 * s["t_setup_s"] + 40.0 * s["t_iter_s"]
    assert abs(s["t_step_s"] - want) <= 1e-12 * want
    if not openmp:
        assert s["cores"] == 1
