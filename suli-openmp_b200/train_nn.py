"""Train the learned initial guess of the pressure solve on a GPU.

    python suli-openmp_b200/train_nn.py --n 128 --snapshots 2000 --steps 6000 \\
        --out suli-openmp_b200/weights/unet_pressure.npy

Training pairs come from the solver itself: for every random two-phase snapshot
(snapshots.py) the mixed-precision solver runs two pressure solves to the FP64 tolerance
through `Solver.graddin_record`, which writes the network's input features and the
converged scaled correction.  Pairs go to a ring of `--pool` pairs in HBM; Adam steps
(learned.Net.train_step: the project's forward/backward kernels) draw random pairs from it
while it fills and refreshes.  Targets are divided by one fixed scale (the rms of the first
pairs' targets): the solver uses the output as a search direction whose length it picks
itself (alpha), so that scale does not matter at inference.

After training, the solver is run on held-out snapshots with and without the network and
the iterations and milliseconds per solve are written with the weights (`<out>.json`).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import pathlib
import sys
import time


def _package():
    here = pathlib.Path(__file__).resolve().parent
    if "suli_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("suli_b200", here / "__init__.py",
                                                      submodule_search_locations=[str(here)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["suli_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["suli_b200"]


def lr_at(step: int, total: int, lr: float, warmup: int) -> float:
    if step < warmup:
        return lr * (step + 1) / warmup
    q = (step - warmup) / max(1, total - warmup)
    return lr * (0.02 + 0.98 * 0.5 * (1.0 + math.cos(math.pi * min(q, 1.0))))


def evaluate(pkg, solver, net, seed: int, count: int):
    """Iterations and ms per solve with and without the network on `count` held-out
    snapshots (two solves each: from zero pressure, then from the previous pressure)."""
    import torch
    gen = pkg.snapshots.SnapshotGenerator(solver, seed)
    rows = []
    for _ in range(count):
        snap = gen.draw()
        row = {}
        for tag, n in (("plain", None), ("learned", net)):
            solver.attach_nn(n)

            def solve(k):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                it, res = solver.graddin()
                return it, res, 1e3 * (time.perf_counter() - t0)
            row[tag] = gen.solve_pair(snap, solve)
        solver.attach_nn(None)
        rows.append(row)
    out = {}
    for tag in ("plain", "learned"):
        for k, name in ((0, "from_zero"), (1, "from_previous")):
            its = [r[tag][k][0] for r in rows]
            ms = [r[tag][k][2] for r in rows]
            res = [r[tag][k][1] for r in rows]
            out[f"{tag}_{name}"] = {"iters": sum(its) / len(its), "ms": sum(ms) / len(ms), "max_resid": max(res)}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--snapshots", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--pool", type=int, default=384)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--eval", type=int, default=16)
    ap.add_argument("--init", default=None, help="start from these weights (.npy)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)

    import numpy as np
    import torch
    pkg = _package()
    n = args.n
    V = n ** 3
    p = pkg.snapshots.tank_params(n=n, precision=1, cg_tol=1e-8)
    solver = pkg.Solver(p)
    gen = pkg.snapshots.SnapshotGenerator(solver, args.seed)
    w0 = np.load(args.init) if args.init else pkg.learned.init_params(args.seed)
    net = pkg.learned.Net(n, n, n, params=w0)
    P = args.pool
    pool_in = torch.empty((P, V * 3), dtype=torch.float32, device="cuda:0")
    pool_t = torch.empty((P, V), dtype=torch.float32, device="cuda:0")
    rng = np.random.default_rng(args.seed)
    filled, wptr, step = 0, 0, 0
    t_scale = None
    min_fill = min(P, 64)
    ema, hist, solve_iters = None, [], []
    t0 = time.time()
    for k in range(args.snapshots):
        i0, i1 = wptr, (wptr + 1) % P
        stats = gen.pair([pool_in[i0], pool_in[i1]], [pool_t[i0], pool_t[i1]])
        solve_iters += [s[0] for s in stats]
        if max(s[1] for s in stats) > 1e-8:
            raise RuntimeError(f"snapshot {k}: solve did not converge: {stats}")
        wptr = (wptr + 2) % P
        filled = min(P, filled + 2)
        if t_scale is None:
            if filled < min_fill:
                continue
            t_scale = float(pool_t[:filled].double().pow(2).mean().sqrt())
            pool_t[:filled] /= t_scale
        else:
            pool_t[i0] /= t_scale
            pool_t[i1] /= t_scale
        goal = int(round((k + 1) * args.steps / args.snapshots))
        while step < goal:
            j = int(rng.integers(filled))
            lr = lr_at(step, args.steps, args.lr, args.warmup)
            loss = net.train_step(pool_in[j], pool_t[j], lr)
            if not math.isfinite(loss):
                raise RuntimeError(f"step {step}: loss {loss}")
            ema = loss if ema is None else 0.98 * ema + 0.02 * loss
            step += 1
            if step % 100 == 0:
                hist.append({"step": step, "loss_ema": ema, "lr": lr, "snapshots": k + 1,
                             "seconds": time.time() - t0})
                print(json.dumps(hist[-1]), flush=True)
    train_s = time.time() - t0
    summary = {"n": n, "snapshots": args.snapshots, "pairs": 2 * args.snapshots, "steps": step,
               "pool": P, "lr": args.lr, "target_scale": t_scale, "train_seconds": train_s,
               "mean_solve_iters_recorded": float(np.mean(solve_iters)),
               "final_loss_ema": ema, "history": hist}
    summary["eval"] = evaluate(pkg, solver, net, args.seed + 10_000, args.eval)
    print(json.dumps(summary["eval"], indent=1), flush=True)
    if args.out:
        net.save(args.out)
        with open(str(args.out) + ".json", "w") as f:
            json.dump(summary, f, indent=1)
    net.close()
    solver.close()
    return summary


if __name__ == "__main__":
    main()
