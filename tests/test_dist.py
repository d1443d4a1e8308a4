"""The multi-GPU path on CPU: bench.py runs one replica per rank and the only
collective is the max over ranks of the timings.  World size 2 over gloo:
the max reduction, and the reference arm's rule (rank 0 alone runs the CPU
reference and prints one line, the other ranks exit without work)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, port: int, q):
    import importlib.util
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    ws, r, local, pg = bench.dist_init(backend="gloo")
    # every rank reports its own step time; the job's is the slowest
    got = bench.barrier_max(pg, 1.5 + 2.0 * r, "cpu")
    pg.barrier()
    pg.destroy_process_group()
    q.put((r, ws, got))


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 3.5), (1, 2, 3.5)]


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    env = dict(os.environ, SBG_CPU_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--workload", "mul16k", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
    # the contract's keys, in the metric and unit of our own line for this workload
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["metric"] == "product Mlimb/s" and d["unit"] == "Mlimb/s" and d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["parity"]["golden_match"] is True       # the reference's product is the committed digest


def _rank_dies(rank: int, port: int, q):
    import importlib.util
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    ws, r, local, pg = bench.dist_init(backend="gloo", timeout_s=20)
    if r == 1:
        os._exit(3)                 # a rank that dies between steps, with nothing in flight
    try:
        bench.barrier_max(pg, 1.0, "cpu")
        q.put((r, "no error"))
    except Exception as e:          # the survivor learns of it at its next collective
        q.put((r, type(e).__name__))


def test_a_dead_rank_ends_the_next_collective_with_an_error():
    """Failure detection on the host: rank 1 exits between steps; rank 0's
    next collective (the max over ranks of the timings) ends with an error
    instead of waiting for ever."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_dies, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    r, what = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
    assert r == 0 and what != "no error"
    assert ps[1].exitcode == 3
