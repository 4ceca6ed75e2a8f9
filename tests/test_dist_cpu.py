"""CPU, two processes over gloo: the N > 1 plumbing of bench.py.

The path runs as independent replicas (no collective in the data path), so what crosses ranks
is the plumbing: the barrier around the timed region and the maximum of the per-rank times;
and the reference arm, which rank 0 alone runs while the other ranks exit 0 without work.
Both are launched the way the benchmark is, with torch.distributed.run on 127.0.0.1."""
import json
import os
import pathlib
import socket
import subprocess
import sys

ROOT = pathlib.Path(__file__).resolve().parent.parent

WORKER = """
import importlib.util, json, pathlib, sys
spec = importlib.util.spec_from_file_location("bench_mod", sys.argv[1])
bench = importlib.util.module_from_spec(spec)
spec.loader.exec_module(bench)
d = bench.Dist("gloo")
d.barrier()
m = d.max(0.5 + d.rank)
d.barrier()
out = pathlib.Path(sys.argv[2]) / f"rank{d.rank}.json"
out.write_text(json.dumps({"rank": d.rank, "world": d.world, "max": m}))
d.close()
"""


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun(*args, timeout=300):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), *args]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "OMP_NUM_THREADS")}
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    return r, lines


def test_barrier_and_max_over_ranks(tmp_path):
    """Every rank gets the slowest rank's time (the benchmark's max over ranks)."""
    w = tmp_path / "worker.py"
    w.write_text(WORKER)
    r, _ = torchrun(str(w), str(ROOT / "bench.py"), str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{n}.json").read_text()) for n in (0, 1)]
    assert [l["rank"] for l in lines] == [0, 1]
    assert all(l["world"] == 2 and l["max"] == 1.5 for l in lines), lines


def test_reference_arm_runs_on_rank0_only():
    """Two ranks, a small tank: one JSON line (rank 0's), exit code 0, the CPU restatement
    timed on every host core rank 0 may use, no host-device traffic and no GPU launches."""
    r, lines = torchrun("bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
                        "--nx", "16", "--ny", "8", "--nz", "8", "--dx", "0.04")
    assert r.returncode == 0, r.stderr[-2000:]
    assert len(lines) == 1, lines
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["cores"] == len(os.sched_getaffinity(0))
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["gpu_launches"] == 0
