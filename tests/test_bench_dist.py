"""The multi-rank plumbing of bench.py on CPU: world_size-2 gloo process groups.

Ranks shard the frames (each rank maps its own agent into its own map; no collective on the
data path).  What is shared is the timing and aggregation: a barrier around the timed region,
the maximum of the per-rank times, the sum of the per-rank work, and one JSON line from rank 0.
"""
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


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    r, w, local = bench.dist_init()
    assert (r, w, local) == (rank, world, rank)
    bench.barrier()
    mx = bench.allreduce_max(1.0 + rank)      # per-rank times 1.0 and 2.0 -> 2.0
    sm = bench.allreduce_sum(10.0 * (rank + 1))  # per-rank work 10 and 20 -> 30
    out.put((rank, mx, sm))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_rank_aggregation_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2.0, 30.0), (1, 2.0, 30.0)]


def test_reference_arm_under_torchrun_prints_one_line():
    """`--impl reference` at N=2: rank 0 times the CPU path and prints the only line; rank 1
    exits 0 without work."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    proc = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [l for l in proc.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, proc.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["steps"] == 1
    assert rec["value"] > 0 and rec["unit"] == "voxel updates/s"
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["kind"] == "port"
