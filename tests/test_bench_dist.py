"""bench.py's multi-rank plumbing on CPU (gloo, world size 2): the barrier
and the max / sum over ranks that the timing uses, and the reference arm
launched as the driver launches it (torchrun, two ranks: rank 0 alone
prints one JSON line, the other exits 0 without work)."""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, str(ROOT))
    import bench

    d = bench.Dist(world)
    d.barrier()
    q.put((rank, d.max(1.5 * (rank + 1)), d.sum(float(rank + 1)), d.device))
    d.close()


def test_max_and_sum_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 3.0, 3.0, "cpu"), (1, 3.0, 3.0, "cpu")]


def test_reference_arm_under_torchrun_prints_once():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--size", "400", "--steps", "2", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    res = json.loads(lines[0])
    assert res["impl"] == "reference"
    if "unavailable" not in res:
        assert res["n_gpus"] == 2 and res["value"] > 0 and res["cpu_baseline"]["kind"] == "reference"
        assert res["e2e"]["h2d_bytes_per_step"] == 0
