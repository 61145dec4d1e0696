"""The benchmark's multi-rank path on the CPU, world size 2 over gloo (no GPU): replicas only, so the one collective is
the timing's max over ranks (bench.reduce_max), and the reference arm under torchrun runs on rank 0 alone and prints
one JSON line while the other rank exits cleanly."""

import json
import os
import subprocess
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _rank_main(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out.put((rank, bench.reduce_max(1.5 + rank, dist, "cpu"), bench.reduce_max(10.0 - rank, dist, "cpu")))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_the_timing_is_the_slowest_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2.5, 10.0), (1, 2.5, 10.0)]


def test_the_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "2", "--warmup", "3", "--partition-worlds", "200"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT),
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
