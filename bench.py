#!/usr/bin/env python
"""bench.py — time-steps/s of the SuLi-IC hot path on B200.

Workload (one "step" = one time step of 1_principal.f90:64-108 plus est()): the sloshing
tank at 256 x 128 x 128 cells (dx = 0.005 m, water/air 1000/1.2, Smagorinsky Cs = 0.1, RK3,
fixed dt from CFL 0.25), every Poisson solve stopped by two tests on every path: relative FP64
residual <= 1e-8 and max |div u| after the projection <= 1e-8 (div_tol).  Seeded synthetic
initial state; the fields (~2.6 GB) exceed the 126 MB L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  `value` is device-timed (CUDA events on the library's stream,
max over ranks); `e2e` times the same steps through the C-ABI (suli_step_host) with the state
copied from and to pinned host memory every step, the copies overlapping the step where its
order allows.  Multi-GPU runs are independent replicas (the path is one
domain on one GPU), so `value` sums the replicas' time steps over the slowest replica's time.
The reference arm (--impl reference) times the CPU restatement of the same path (OpenMP, all
host cores): a bounded number of real, whole steps of the same workload (no iteration cap).
"""
from __future__ import annotations

import argparse
import csv
import importlib.util
import io
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
PKG_DIR = ROOT / "suli-openmp_b200"
METRIC = "time-steps/s at 256x128x128, learned+FP32 vs plain FP64 GPU @ resid<=1e-8"
UNIT = "time-steps/s"
FALLBACK_HBM_GBS = 6650.0


def load_pkg():
    if "suli_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("suli_b200", PKG_DIR / "__init__.py",
                                                      submodule_search_locations=[str(PKG_DIR)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["suli_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["suli_b200"]


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=128)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--dx", type=float, default=0.005)
    ap.add_argument("--cg-tol", type=float, default=1e-8)
    ap.add_argument("--div-tol", type=float, default=1e-8,
                    help="second stopping test of every Poisson solve: max |div u| after the projection")
    ap.add_argument("--inner-tol", type=float, default=1e-3, help="relative tolerance of each FP32 inner solve")
    ap.add_argument("--mg-omega", type=float, default=0.56, help="damping of the multigrid Jacobi sweeps")
    ap.add_argument("--mg-alpha", type=float, default=1.8, help="scale of the multigrid coarse-grid correction")
    ap.add_argument("--mg-kernels", type=int, default=0,
                    help="multigrid kernels: 0 vectorised per level, 1 one cell a thread, 2 with the cluster coarse levels")
    ap.add_argument("--mg-omega2", type=float, default=1.39,
                    help="weight of the second pre-smoothing (first post-smoothing) sweep; 0: --mg-omega")
    ap.add_argument("--path", choices=["all", "plain", "mixed", "learned"], default="all",
                    help="time every solver path (headline = learned + mixed precision) or one of them")
    ap.add_argument("--weights", default=None, help="network weights (.npy); default: the shipped ones")
    ap.add_argument("--mms-n", type=int, default=128, help="grid of the manufactured-solution check (0: skip)")
    ap.add_argument("--mms-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=3, help="whole steps timed on the host cores (after one warm-up step)")
    ap.add_argument("--cpu-serial-steps", type=int, default=1,
                    help="whole steps timed on one thread, as the reference runs (0: skip)")
    ap.add_argument("--long-steps", type=int, default=500,
                    help="steps of the long-window block (C3's 500; 0: skip)")
    ap.add_argument("--long-paths", default="learned,plain",
                    help="paths timed over the long window (comma list of plain, mixed, learned)")
    ap.add_argument("--c5-steps", type=int, default=4,
                    help="timed steps of the LES channel over a bump at 512x256x256 (0: skip)")
    ap.add_argument("--c5-n", default="512,256,256", help="grid of the LES channel block")
    ap.add_argument("--c4-snapshots", type=int, default=3,
                    help="held-out random tanks (two solves each) of the per-solve comparison at the bench grid (0: skip)")
    return ap.parse_args()


# ------------------------------------------------------------------------------ plumbing
class Dist:
    """Rank bookkeeping; replicas only, torch.distributed just for barrier and max."""

    def __init__(self, backend):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.pg.get_backend() == "nccl":
                import torch
                self.pg.barrier(device_ids=[self.local])
            else:
                self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        dev = f"cuda:{self.local}" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = vis.split(",")[self.dev] if vis else str(self.dev)
            self.path = pathlib.Path(os.environ.get("TMPDIR", "/tmp")) / f"suli_clocks_{os.getpid()}.csv"
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", idx, f"--query-gpu={self.Q}", "--format=csv",
                                          "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = list(csv.reader(io.StringIO(self.path.read_text())))
        self.path.unlink(missing_ok=True)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows[1:]:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1].split()[0]))
                smax.append(float(r[2].split()[0]))
                power.append(float(r[3].split()[0]))
            except ValueError:
                continue
            for nm, val in zip(names, r[5:9]):
                if "Active" in val and "Not" not in val:
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            d = json.loads(f.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel: str, ncell: int):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/), scaled to
    `ncell` cells when the capture ran on a smaller grid."""
    f = ROOT / "profiles" / f"{kernel}.txt"
    if not f.exists():
        return None
    vals = {}
    for line in f.read_text().splitlines():
        if ":" in line and line.split(":")[0].strip() in ("dram_bytes_per_launch", "cells"):
            k, v = line.split(":", 1)
            try:
                vals[k.strip()] = float(v.split()[0])
            except ValueError:
                pass
    if "dram_bytes_per_launch" not in vals:
        return None
    scale = ncell / vals.get("cells", ncell)
    return vals["dram_bytes_per_launch"] * scale


# ------------------------------------------------------------------------------ CPU steps
def cpu_steps(pkg, p, init, timed: int, openmp: bool = True, warm: int = 1):
    """Whole time steps of the CPU restatement (oracle/, FP64): the OpenMP build on every host
    core it may use, or the serial build on one thread (as the reference's own program runs).
    `warm` untimed steps from the initial state, then `timed` steps, each timed by the wall
    clock; every Poisson solve runs to the same two stopping tests as the GPU paths."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    t_init = time.perf_counter()
    o = oracle.Oracle(p, openmp=openmp)
    init(o)
    t_init = time.perf_counter() - t_init
    it = 0
    for _ in range(warm):
        it += 1
        o.step(it)
    times, iters, divs, res = [], [], [], []
    for _ in range(timed):
        it += 1
        t0 = time.perf_counter()
        st = o.step(it)
        times.append(time.perf_counter() - t0)
        iters.append(sum(st["cg_iters"]))
        divs.append(st["max_div"])
        res.append(max(st["cg_resid"]))
    o.close()
    return {"t_step_s_median": statistics.median(times), "t_step_s": times, "steps_timed": list(range(it - timed + 1, it + 1)),
            "poisson_iters_per_step": iters, "max_div": max(divs), "cg_resid_max": max(res),
            "cores": oracle.num_threads(openmp), "init_s": t_init}


def cpu_desc(cs, openmp):
    who = "OpenMP build of the FP64 CPU restatement on every host core" if openmp else \
        "serial build of the FP64 CPU restatement on one thread (as the reference runs)"
    return (f"{who}: median of {len(cs['t_step_s'])} whole steps (steps {cs['steps_timed'][0]}-"
            f"{cs['steps_timed'][-1]} from the seeded state, after {cs['steps_timed'][0] - 1} untimed), "
            f"Poisson solves to the same two stopping tests, no iteration cap "
            f"({statistics.mean(cs['poisson_iters_per_step']):.0f} CG iterations per step)")


# ------------------------------------------------------------------------------ C5
# Algorithmic N-sized FP64 passes (8 bytes a cell) per launch of each stencil kernel class:
# reads and writes of whole fields, halos not counted twice.
CLASS_PASSES = {
    "ls_advect": 6,    # ls, stage start, u, v, w in; ls out
    "reinit": 4,       # mean of S(phi0) (2), stage (5) and band error (2) launches
    "lsprops": 11,     # ls in; mod_ls, 3 normals, hs, hsx..z, rho, ls_nu out
    "curv": 7,         # 3 normals in; ddlsdx..z, kurv out
    "visco": 5,        # nut: u, v, w, rho in, nut out; faces: nut, ls_nu in, xnut..znut out
    "convdiff": 20,    # u, v, w, rho, hsx..z, kurv, nut, xnut..znut in, Fu..Fw out; prd0 = prd1 copy
    "tempo": 15,       # per component: velocity, F in; velocity and two stage stores out
    "posdin": 10,      # u, v, w, prd1, rho in; u, v, w out; the prd = prd1 copy timed with it
    "est": 3,          # u, v, w in
}


def class_bandwidth(p, kernels):
    """GB/s of the stencil kernel classes from the tracer's device time and launches per step."""
    n8 = 8.0 * p.nx * p.ny * p.nz
    out = {}
    for k, passes in CLASS_PASSES.items():
        v = kernels.get(k)
        if not v or v["ms_per_step"] <= 0:
            continue
        b = passes * n8 * v["launches_per_step"]
        out[k] = {"ms_per_step": round(v["ms_per_step"], 4), "launches_per_step": v["launches_per_step"],
                  "gbs": round(b / (v["ms_per_step"] / 1e3) / 1e9, 1)}
    return out


def c5_block(args, dist, pkg, dev):
    """The LES channel over a Gaussian bump (6 x 3 x 3 m, water 2 m deep, inflow 1 m/s + 5 %
    seeded noise, outflow, periodic y, Cs = 0.12, CFL 0.3): the plain FP64 path and the
    learned + mixed path, each timed over --c5-steps steps after 2 warm-up steps from the same
    state; time-steps/s, GB/s per stencil kernel class, level-set volume drift, the divergence
    and the learned path's error per field against the plain run."""
    import torch
    nx, ny, nz = (int(v) for v in args.c5_n.split(","))
    p, init, _ = pkg.cases.les_channel(nx=nx, ny=ny, nz=nz, cg_tol=args.cg_tol)
    q = mixed_params(p, args)
    q.div_tol = 0.0
    out = {"grid": f"{nx}x{ny}x{nz}", "dx": p.dx, "dt": p.dt, "steps": args.c5_steps, "warmup": 2,
           "options": "outflow_fix = 1, periodic_faces = 1 (the reference's outflow copy and periodic end faces "
                      "make this Poisson system inconsistent and non-symmetric)",
           "max_div_note": "max|div u| includes the cells beside the bump, where contorno zeroes the velocities "
                           "after the projection (3_contorno.f90:266-294)"}
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup = args.c5_steps, 2
    net = None
    states = {}
    for key, prm in (("plain_fp64", p), ("learned", q)):
        if key == "learned":
            net, src = load_net(pkg, q, args, dev)
            if net is None:
                out[key] = {"skipped": src}
                continue
        r = time_path(sub, dist, pkg, prm, init, dev, net=net)
        s = r["solver"]
        v0, v1 = s.get_scalar("vol_ini"), s.get_scalar("vol_ins")
        states[key] = state_of(s)
        s.close()
        out[key] = {"value": r["value"], "ms_per_step": r["ms"] / sub.steps, "poisson_iters_per_step": r["iters_per_step"],
                    "volume_drift": (v1 - v0) / v0, "max_div": max(st["max_div"] for st in r["stats"]),
                    "cg_resid_max": max(max(st["cg_resid"]) for st in r["stats"]),
                    "kernel_gbs": class_bandwidth(prm, r["kernels"]),
                    "clocks": {k: r["clocks"].get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons")}}
    if net is not None:
        net.close()
    if "plain_fp64" in states and "learned" in states:
        out["learned"]["error_vs_plain_fp64"] = field_errors(states["learned"], states["plain_fp64"])
        out["learned"]["speedup_vs_plain_fp64"] = out["learned"]["value"] / out["plain_fp64"]["value"]
    return out


# ------------------------------------------------------------------------------ C4
def c4_block(args, pkg, dev):
    """Iterations and device time per pressure solve at the bench grid, to the same FP64
    relative residual, on held-out random tanks (snapshots.SnapshotGenerator with seeds the
    network was not trained on; each tank is solved from zero pressure and then again from that
    solution with a correlated velocity field): the plain FP64 Jacobi-scaled CG of the reference,
    the mixed FP32 multigrid-preconditioned solve, and the same with the learned initial guess."""
    import torch
    out = {"grid": f"{args.nx}x{args.ny}x{args.nz}", "cg_tol": args.cg_tol, "snapshots": args.c4_snapshots,
           "seeds": [9001 + q for q in range(args.c4_snapshots)]}
    net = None
    for key, prec, learned in (("plain_jacobi_pcg_fp64", 0, False), ("mixed_multigrid_pcg", 1, False),
                               ("mixed_multigrid_pcg_learned_guess", 1, True)):
        q = pkg.snapshots.tank_params(n=args.nx, ny=args.ny, nz=args.nz, dx=args.dx, cg_tol=args.cg_tol, precision=prec)
        if prec == 1:
            q.refine_maxit, q.inner_tol = 30, args.inner_tol
            q.mg_omega, q.mg_alpha = args.mg_omega, args.mg_alpha
            q.mg_omega2 = args.mg_omega2
        s = pkg.Solver(q, device=dev)
        if learned:
            net, src = load_net(pkg, q, args, dev)
            if net is None:
                out[key] = {"skipped": src}
                s.close()
                continue
            s.attach_nn(net)
        ext = torch.cuda.ExternalStream(s.stream_ptr, device=dev)
        its, ms, res = [], [], []
        for seed in out["seeds"]:
            gen = pkg.snapshots.SnapshotGenerator(s, seed)

            def solve(k):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.synchronize()
                e0.record(ext)
                n, r = s.graddin()
                e1.record(ext)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
                return n, r
            for n, r in gen.solve_pair(gen.draw(), solve):
                its.append(n)
                res.append(r)
        s.close()
        out[key] = {"iters_per_solve": statistics.mean(its), "ms_per_solve": statistics.mean(ms),
                    "iters": its, "resid_max": max(res),
                    "iterations": "FP64 CG iterations" if prec == 0 else "inner FP32 PCG iterations"}
    if net is not None:
        net.close()
    base = out.get("plain_jacobi_pcg_fp64", {}).get("ms_per_solve")
    for k in ("mixed_multigrid_pcg", "mixed_multigrid_pcg_learned_guess"):
        if base and "ms_per_solve" in out.get(k, {}):
            out[k]["speedup_vs_plain_jacobi_pcg"] = base / out[k]["ms_per_solve"]
    return out


# ------------------------------------------------------------------------------ arms
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        # torchrun starts every rank with OMP_NUM_THREADS=1; the other ranks exit without
        # work, so rank 0 takes every host core it may run on (read when the OpenMP oracle
        # library loads, below)
        os.environ["OMP_NUM_THREADS"] = str(len(os.sched_getaffinity(0)))
    pkg = load_pkg()
    p, init = pkg.cases.sloshing(nx=args.nx, ny=args.ny, nz=args.nz, dx=args.dx, cg_tol=args.cg_tol,
                                 div_tol=args.div_tol)
    # a bounded sample: --steps whole steps would take minutes each on the host cores
    timed = max(1, min(args.steps, args.cpu_steps))
    t0 = time.perf_counter()
    cs = cpu_steps(pkg, p, init, timed, openmp=True)
    wall = time.perf_counter() - t0
    t = sum(cs["t_step_s"])
    value = timed / t
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": timed,
        "steps_requested": args.steps, "warmup": 1, "ms_per_step": 1e3 * t / timed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cs["cores"], "kind": "port",
                         "sample": cpu_desc(cs, True)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0, "max_div": cs["max_div"], "cg_resid_max": cs["cg_resid_max"],
        "poisson_iters_per_step": cs["poisson_iters_per_step"], "t_step_s": cs["t_step_s"],
        "wall_s_incl_init": wall,
        "config": workload_config(p, args, "cpu-openmp-fp64"),
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(p, args, path):
    return {
        "workload": (f"sloshing tank {p.nx}x{p.ny}x{p.nz} dx={p.dx} RK3 Smagorinsky, Poisson rel. residual "
                     f"{p.cg_tol:g} and max|div u| {p.div_tol:g}"),
        "nx": p.nx, "ny": p.ny, "nz": p.nz, "dt": p.dt, "cg_tol": p.cg_tol, "div_tol": p.div_tol, "path": path,
        "l2": "state of ~2.6 GB per replica exceeds the 126 MB L2; no flush",
        "parallelism": f"replicas{args.gpus}",
    }


def time_path(args, dist, pkg, p, init, dev, it0=0, net=None, nn_mode=1):
    """Warm up, then time K steps of one solver path with CUDA events on its own stream
    (with `net` attached as the pressure solve's initial guess, if given)."""
    import torch

    s = pkg.Solver(p, device=dev)
    init(s)
    if net is not None:
        s.attach_nn(net, nn_mode)
    ext = torch.cuda.ExternalStream(s.stream_ptr, device=dev)
    it = it0
    for _ in range(args.warmup):
        it += 1
        s.step(it)
    s.synchronize()
    s.profile_enable(True)
    clocks = ClockSampler(dev)
    dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    stats = []
    for _ in range(args.steps):
        it += 1
        stats.append(s.step(it))
    e1.record(ext)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    dist.barrier()
    ms_local = e0.elapsed_time(e1)
    prof = s.profile_read()
    s.profile_enable(False)
    ms = dist.max(ms_local)
    return {"solver": s, "it": it, "ms": ms, "value": dist.world * args.steps / (ms / 1e3), "prof": prof,
            "stats": stats, "clocks": clk,
            "iters_per_step": prof["cg_iterations"] / args.steps,
            "launches": sum(v["launches"] for k, v in prof.items() if isinstance(v, dict)),
            "kernels": {k: {"ms_per_step": v["ms"] / args.steps, "launches_per_step": v["launches"] / args.steps}
                        for k, v in prof.items() if isinstance(v, dict)}}


def launch_share(profile: str, kernel: str, among: tuple):
    """`kernel`'s share of the device time of the kernels `among` in a committed ncu launch list
    (profiles/<profile>.txt), or None."""
    f = ROOT / "profiles" / f"{profile}.txt"
    if not f.exists():
        return None
    tot = {}
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] in among:
            try:
                tot[parts[0]] = float(parts[2])
            except ValueError:
                pass
    if kernel not in tot or sum(tot.values()) <= 0:
        return None
    return tot[kernel] / sum(tot.values())


def cg_roofline(p, prof):
    """Roofline of the plain path's dominant kernel (CG kernel A) and of a whole CG iteration.
    Both CG kernels run inside one device-side graph loop, so CUDA events time the iteration;
    kernel A's duration is that time times its share of the two kernels in the committed ncu
    launch list of this workload."""
    N = p.nx * p.ny * p.nz
    faces = (p.nx + 1) * p.ny * p.nz + p.nx * (p.ny + 1) * p.nz + p.nx * p.ny * (p.nz + 1)
    bytes_spmv = 8 * (4 * N + faces)
    bytes_upd = 8 * 6 * N
    n_it = max(prof["cg_iterations"], 1)
    t_it = (prof["cg_spmv"]["ms"] + prof["cg_update"]["ms"]) / n_it / 1e3
    share = launch_share("launches_sloshing_256x128x128_fp64", "k_cg_spmv2", ("k_cg_spmv2", "k_cg_update"))
    peak, peak_kind = measured_peaks()
    it = {"kernels": "k_cg_spmv2 + k_cg_update (one graph loop)", "bytes": bytes_spmv + bytes_upd, "us": t_it * 1e6,
          "achieved_gbs": (bytes_spmv + bytes_upd) / t_it / 1e9,
          "frac": (bytes_spmv + bytes_upd) / t_it / 1e9 / peak}
    t_spmv = t_it * (share if share else 1.0)
    ach = bytes_spmv / t_spmv / 1e9
    return {
        "kernel": "k_cg_spmv2 (FP64 CG kernel A, two cells a thread: p = r + beta p, q = A p, p.q)",
        "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s",
        "traffic": profiled_traffic("cg_spmv2_256x128x128", N), "algorithmic_bytes_per_launch": bytes_spmv,
        "avg_launch_us": t_spmv * 1e6,
        "duration": ("CUDA-event time of a CG iteration x k_cg_spmv2's share of the two CG kernels in "
                     "profiles/launches_sloshing_256x128x128_fp64.txt" if share else
                     "CUDA-event time of a whole CG iteration (no launch list to apportion it)"),
        "cg_iteration": it,
    }


def unet_flops(pkg, p):
    """Algorithmic FLOPs of one U-Net forward: 2 * 27 * Cin * Cout per voxel of each layer's
    level, plus the 1x1x1 head."""
    V0 = p.nx * p.ny * p.nz
    f = sum(2 * 27 * ci * co * V0 // (8 ** lv) for ci, co, lv in pkg.learned.LAYERS)
    return f + 2 * 16 * V0


def mg_iteration_bytes(p):
    """Algorithmic HBM bytes of one inner FP32 PCG iteration (4-byte values, N-sized passes):
    level 0 forms its faces from the density, so SpMV 5, update 6, pre-smoothing 4, restriction
    3 1/8, prolongation + smoothing 5 1/8, last smoothing sweep 5 passes; each coarser level
    (stored faces) 25 1/4 passes of its own size."""
    N = p.nx * p.ny * p.nz
    fine = 5 + 6 + 4 + 3.125 + 5.125 + 5
    coarse, n = 0.0, N
    nx, ny, nz = p.nx, p.ny, p.nz
    while nx * ny * nz > 1024 and nx % 2 == 0 and ny % 2 == 0 and nz % 2 == 0:
        nx, ny, nz = nx // 2, ny // 2, nz // 2
        coarse += 25.25 * (nx * ny * nz) / N
    return 4 * N * (fine + coarse)


def headline_rooflines(pkg, p, head, peaks):
    """Rooflines of the two kernel classes that dominate the learned + mixed step."""
    peak_hbm, kind = peaks
    out = {}
    k = head["kernels"]
    it = max(head["iters_per_step"], 1e-9)
    if k.get("mg", {}).get("ms_per_step", 0) > 0:
        t = k["mg"]["ms_per_step"] / it / 1e3
        b = mg_iteration_bytes(p)
        out["inner_pcg_iteration"] = {
            "kernel": "one FP32 inner PCG iteration (CUDA graph: SpMV, update, multigrid V-cycle)",
            "bound": "hbm", "achieved": b / t / 1e9, "peak": peak_hbm, "unit": "GB/s", "frac": b / t / 1e9 / peak_hbm,
            "algorithmic_bytes": b, "us": t * 1e6,
            "traffic": profiled_traffic("inner_pcg_iteration_256x128x128", p.nx * p.ny * p.nz)}
    if k.get("nn", {}).get("launches_per_step", 0) > 0:
        # one forward per Poisson solve; every solve ends with one k_cg_final
        fwd = k.get("cg_final", {}).get("launches_per_step", 0)
        t = k["nn"]["ms_per_step"] / max(fwd, 1e-9) / 1e3
        fl = unet_flops(pkg, p)
        pk = measured_tensor_peak()
        out["unet_forward"] = {
            "kernel": "U-Net forward with its input features and guess (k_nn_stats, k_nn_features16, 14 x k_conv3_tp: "
                      "TMA + tcgen05 pipeline with pooling and head in the epilogues, k_nn_dots, k_nn_apply)",
            "bound": "tensor", "achieved": fl / t / 1e12, "peak": pk, "unit": "TFLOP/s", "frac": fl / t / 1e12 / pk,
            "peak_source": "measured bf16_tflops_sustained (MEASURED_PEAKS.json)",
            "algorithmic_flops": fl, "ms": t * 1e3,
            "traffic": profiled_traffic("unet_forward_256x128x128", p.nx * p.ny * p.nz)}
    return out


def measured_tensor_peak():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["bf16_tflops_sustained"])
        except (KeyError, ValueError):
            pass
    return 1400.0


def mixed_params(p, args):
    q = p.copy()
    q.precision, q.cg_stop, q.cg_tol = 1, 1, args.cg_tol
    q.inner_tol, q.refine_maxit = args.inner_tol, 30
    q.mg_omega, q.mg_alpha = args.mg_omega, args.mg_alpha
    q.mg_omega2 = args.mg_omega2
    q.mg_kernels = args.mg_kernels
    return q


def load_net(pkg, p, args, dev):
    """The trained network for this grid, or None when no weights are available."""
    import pathlib as _pl
    path = _pl.Path(args.weights) if args.weights else pkg.learned.WEIGHTS_PATH
    if not path.exists():
        return None, f"no weights at {path}"
    name = str(path.relative_to(ROOT)) if path.is_relative_to(ROOT) else str(path)
    return pkg.learned.Net.load(p.nx, p.ny, p.nz, device=dev, path=path), name


def mms_check(pkg, args, dev):
    """Manufactured solution on the periodic box (cases.TaylorGreenMMS): errors of the FP64
    and the mixed path against the exact fields, and of the mixed path against FP64."""
    import numpy as np
    out = {"grid": f"{args.mms_n}^3 periodic [0,2pi]^3, nu=0.01, dt=1e-3, RK3", "steps": args.mms_steps}
    fields = {}
    for prec, tag in ((0, "fp64"), (1, "mixed")):
        m = pkg.cases.TaylorGreenMMS(args.mms_n, precision=prec, cg_tol=1e-10)
        s = pkg.Solver(m.p, device=dev)
        m.init(s)
        divs = []
        t0 = time.perf_counter()
        for it in range(1, args.mms_steps + 1):
            divs.append(m.step(s, it)["max_div"])
        wall = time.perf_counter() - t0
        out[tag] = {"vs_exact": m.errors(s, args.mms_steps * m.p.dt), "max_div": max(divs),
                    "wall_s_incl_host_source_upload": wall}
        f = {k: s.download(k) for k in ("u", "v", "w")}
        pr = s.download("prd1")[1:-1, 1:-1, 1:-1]
        f["prd1"] = pr - pr.mean()
        fields[tag] = f
        s.close()
    out["mixed_vs_fp64_rel_max"] = {
        k: float(np.abs(fields["mixed"][k] - fields["fp64"][k]).max() / max(np.abs(fields["fp64"][k]).max(), 1e-300))
        for k in ("u", "v", "w", "prd1")}
    return out


STATE = ("u", "v", "w", "ls", "prd1")


def state_of(s):
    """The fields compared between paths: velocities, level set and the mean-free pressure."""
    out = {f: s.download(f) for f in STATE if f != "prd1"}
    pr = s.download("prd1")[1:-1, 1:-1, 1:-1]
    out["prd1"] = pr - pr.mean()
    return out


def field_errors(a, ref):
    """Max |a - ref| per field: the velocity components over the velocity scale (the largest
    |u|, |v|, |w| of the reference state), the level set and the pressure over their own."""
    import numpy as np
    vs = max(float(np.abs(ref[f]).max()) for f in ("u", "v", "w"))
    e = {f: float(np.abs(a[f] - ref[f]).max()) / vs for f in ("u", "v", "w")}
    for f in ("ls", "prd1"):
        e[f] = float(np.abs(a[f] - ref[f]).max()) / max(float(np.abs(ref[f]).max()), 1e-300)
    return e


def long_window(args, dist, pkg, p, init, dev, net=None):
    """A fresh run of `--long-steps` steps from the seeded state, timed as one CUDA-event window:
    steps/s, Poisson iterations per step in blocks of 50 steps, the worst max|div u| and residual,
    and the clocks sampled over the window."""
    import torch
    s = pkg.Solver(p, device=dev)
    init(s)
    if net is not None:
        s.attach_nn(net)
    ext = torch.cuda.ExternalStream(s.stream_ptr, device=dev)
    dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    iters, divs, res = [], [], []
    for it in range(1, args.long_steps + 1):
        st = s.step(it)
        iters.append(sum(st["cg_iters"]))
        divs.append(st["max_div"])
        res.append(max(st["cg_resid"]))
    e1.record(ext)
    e1.synchronize()
    clk = clocks.stop()
    ms = dist.max(e0.elapsed_time(e1))
    vol0, vol1 = s.get_scalar("vol_ini"), s.get_scalar("vol_ins")
    s.close()
    blk = 50
    return {"steps": args.long_steps, "value": dist.world * args.long_steps / (ms / 1e3), "ms_per_step": ms / args.long_steps,
            "poisson_iters_per_step_by_50": [round(statistics.mean(iters[q:q + blk]), 1) for q in range(0, len(iters), blk)],
            "max_div": max(divs), "cg_resid_max": max(res), "volume_drift": (vol1 - vol0) / vol0,
            "clocks": {k: clk.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons", "samples")}}


def run_ours(args):
    import numpy as np
    import torch

    dist = Dist("nccl")
    dev = dist.local
    torch.cuda.set_device(dev)
    pkg = load_pkg()
    p, init = pkg.cases.sloshing(nx=args.nx, ny=args.ny, nz=args.nz, dx=args.dx, cg_tol=args.cg_tol,
                                 div_tol=args.div_tol)
    q = mixed_params(p, args)
    runs = {}
    # plain FP64 path (the reference's Jacobi-scaled CG): the comparison
    if args.path in ("all", "plain"):
        runs["plain"] = time_path(args, dist, pkg, p, init, dev)
    # mixed precision: FP32 multigrid-preconditioned inner CG inside FP64 refinement
    if args.path in ("all", "mixed"):
        runs["mixed"] = time_path(args, dist, pkg, q, init, dev)
    # learned + mixed: the network's guess starts every pressure solve
    net, net_src = None, None
    if args.path in ("all", "learned"):
        net, net_src = load_net(pkg, q, args, dev)
        if net is not None:
            runs["learned"] = time_path(args, dist, pkg, q, init, dev, net=net)
        elif args.path == "learned":
            raise SystemExit(f"--path learned: {net_src}")
    # the network also as the preconditioner of the outer refinement iteration (measured beside)
    if net is not None and args.path == "all":
        q2 = q.copy()
        runs["learned_precond"] = time_path(args, dist, pkg, q2, init, dev, net=net, nn_mode=2)
    head_key = "learned" if "learned" in runs else ("mixed" if "mixed" in runs else "plain")
    head = runs[head_key]
    # every path ran the same warm-up + timed steps from the same state: per-field error of the
    # mixed-precision paths against the plain FP64 run
    states = {k: state_of(r["solver"]) for k, r in runs.items()}
    errors = {k: field_errors(states[k], states["plain"]) for k in runs if k != "plain" and "plain" in states}
    del states
    for k, r in runs.items():
        if k != head_key:
            r["solver"].close()
    s = head["solver"]
    it = head["it"]
    value, ms, prof, stats, clk = head["value"], head["ms"], head["prof"], head["stats"], head["clocks"]
    roof_plain = cg_roofline(p, runs["plain"]["prof"]) if "plain" in runs else None
    roof_head = headline_rooflines(pkg, p, head, measured_peaks()) if head_key != "plain" else {}
    # the dominant kernel of the headline path: the class with the most device time
    if roof_head:
        dom = max(roof_head, key=lambda k: {"inner_pcg_iteration": head["kernels"].get("mg", {}).get("ms_per_step", 0),
                                            "unet_forward": head["kernels"].get("nn", {}).get("ms_per_step", 0)}[k])
        roofline = dict(roof_head[dom], name=dom)
    else:
        roofline = roof_plain
    # ---- end to end through the C-ABI: pinned host state in and out every step
    e2e = None
    if not args.no_e2e:
        names = ["u", "v", "w", "prd1", "ls"]
        pinned = {}
        for nm in names:
            shape = s.shape(nm)
            t = torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True)
            a = t.numpy().reshape(shape, order="F")
            s.download(nm, out=a)
            pinned[nm] = (t, a)
        h2d = sum(a.nbytes for _, a in pinned.values())
        s.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        state = {nm: pinned[nm][1] for nm in names}
        for _ in range(args.steps):
            it += 1
            s.step_host(it, state, state)   # in from and back to the same pinned arrays
        s.synchronize()
        t_e2e = dist.max(time.perf_counter() - t0)
        e2e = {"value": dist.world * args.steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": h2d, "fields": names, "path": head_key, "api": "suli_step_host"}
    s.close()
    # ---- the long window (C3's 500 steps) of the headline and the plain path
    long = {}
    if args.long_steps > 0:
        for k in [x.strip() for x in args.long_paths.split(",") if x.strip()]:
            if k == "plain":
                long[k] = long_window(args, dist, pkg, p, init, dev)
            elif k == "mixed":
                long[k] = long_window(args, dist, pkg, q, init, dev)
            elif k == "learned" and net is not None:
                long[k] = long_window(args, dist, pkg, q, init, dev, net=net)
        if "plain" in long:
            for k in long:
                if k != "plain":
                    long[k]["speedup_vs_plain_fp64"] = long[k]["value"] / long["plain"]["value"]
    if net is not None:
        net.close()
    # ---- CPU baseline (rank 0, N = 1 only): whole steps, no cap
    cpu = None
    if dist.world == 1 and not args.no_cpu_baseline:
        cs = cpu_steps(pkg, p, init, args.cpu_steps, openmp=True)
        cpu = {"value": 1.0 / cs["t_step_s_median"], "unit": UNIT, "cores": cs["cores"], "kind": "port",
               "sample": cpu_desc(cs, True), "t_step_s": cs["t_step_s"],
               "poisson_iters_per_step": cs["poisson_iters_per_step"], "max_div": cs["max_div"]}
        if args.cpu_serial_steps > 0:
            ss = cpu_steps(pkg, p, init, args.cpu_serial_steps, openmp=False)
            cpu["one_thread"] = {"value": 1.0 / ss["t_step_s_median"], "unit": UNIT, "cores": ss["cores"],
                                 "kind": "port", "sample": cpu_desc(ss, False), "t_step_s": ss["t_step_s"]}
    mms = None
    if dist.world == 1 and args.mms_n > 0:
        mms = mms_check(pkg, args, dev)
    c5 = c5_block(args, dist, pkg, dev) if args.c5_steps > 0 else None
    c4 = c4_block(args, pkg, dev) if (args.c4_snapshots > 0 and dist.world == 1) else None
    if dist.rank == 0:
        desc = {"plain": "plain FP64: the reference's Jacobi-scaled CG",
                "mixed": "mixed: FP32 stencils, FP32 multigrid-preconditioned inner CG inside FP64 iterative "
                         "refinement to the same FP64 stopping tests",
                "learned": "learned + mixed: the U-Net's guess (energy-optimal FP64 step) starts every pressure "
                           "solve of the mixed path, which then runs to the same FP64 stopping tests"}
        cfg = workload_config(q if head_key != "plain" else p, args, desc[head_key])
        cfg["inner_tol"] = args.inner_tol
        cfg["mg_omega"], cfg["mg_alpha"] = args.mg_omega, args.mg_alpha
        cfg["mg_omega2"] = args.mg_omega2 or args.mg_omega
        cfg["mg_kernels"] = args.mg_kernels
        lo = os.environ.get("SULI_COARSE_CHEB", "0.02")
        steps = os.environ.get("SULI_COARSE_SWEEPS", "20" if float(lo) > 0 else "40")
        cfg["coarse_solve"] = (f"Chebyshev over [{lo}, 2] of D^-1 A, {steps} steps" if float(lo) > 0
                               else f"damped Jacobi, {steps} sweeps")
        if net_src:
            cfg["weights"] = net_src
        arm_acc = {k: {"max_div": max(st["max_div"] for st in r["stats"]),
                       "cg_resid_max": max(max(st["cg_resid"]) for st in r["stats"])} for k, r in runs.items()}
        ok = all(a["max_div"] <= args.div_tol and a["cg_resid_max"] <= args.cg_tol for a in arm_acc.values())
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32+bf16" if head_key == "learned" else "f64+f32", "data": "synthetic",
            "accuracy_ok": ok,
            "accuracy": {"bound": {"cg_resid": args.cg_tol, "max_div": args.div_tol}, **arm_acc},
            "error_vs_plain_fp64": errors,
            "e2e": e2e, "gpu_launches": head["launches"],
            "cpu_baseline": cpu,
            "roofline": roofline,
            "clocks": clk,
            "poisson_iters_per_step": head["iters_per_step"],
            "config": cfg,
        }
        for k, r in runs.items():
            if k == head_key:
                continue
            line[{"plain": "plain_fp64", "mixed": "mixed_no_net", "learned": "learned",
                  "learned_precond": "learned_preconditioner"}[k]] = {
                "value": r["value"], "ms_per_step": r["ms"] / args.steps,
                "poisson_iters_per_step": r["iters_per_step"], "gpu_launches": r["launches"],
                "clocks": {kk: r["clocks"].get(kk) for kk in ("sm_mhz", "sm_max_mhz", "reasons")}}
        if "plain" in runs and head_key != "plain":
            line["speedup_vs_plain_fp64"] = value / runs["plain"]["value"]
        if "mixed" in runs and head_key == "learned":
            line["learned_vs_mixed"] = {"speedup": value / runs["mixed"]["value"],
                                        "poisson_iters_saved_per_step":
                                            runs["mixed"]["iters_per_step"] - head["iters_per_step"]}
        if "mixed" in runs and "learned_precond" in runs:
            line["learned_preconditioner_vs_mixed"] = {
                "speedup": runs["learned_precond"]["value"] / runs["mixed"]["value"],
                "poisson_iters_saved_per_step": runs["mixed"]["iters_per_step"] - runs["learned_precond"]["iters_per_step"]}
        if long:
            line["long_window"] = long
        line["roofline_classes"] = roof_head
        line["roofline_plain_fp64"] = roof_plain
        if mms is not None:
            line["mms"] = mms
        if c5 is not None:
            line["c5_les_channel"] = c5
        if c4 is not None:
            line["c4_per_solve"] = c4
        line["kernel_gbs"] = class_bandwidth(p, head["kernels"])
        if "plain" in runs:
            line["kernel_gbs_plain_fp64"] = class_bandwidth(p, runs["plain"]["kernels"])
        line["kernels"] = {k: {kk: round(vv, 4) for kk, vv in v.items()} for k, v in head["kernels"].items()}
        line["config"]["path"] = head_key
        print(json.dumps(line), flush=True)
    dist.close()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
