"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): ranks are
independent replicas (no data-path collective); the only collective is the
element-wise maximum of the timings, and under torchrun the reference arm
prints one line from rank 0 while the other rank exits cleanly."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
ROOT = Path(__file__).resolve().parents[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    vals = bench.max_over_ranks([float(rank), -float(rank), 10.0 + rank], dist, torch.device("cpu"))
    out.put((rank, vals))
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == got[1] == [1.0, 0.0, 11.0]


def test_max_over_ranks_single_process():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks([3.0, 4.0], None, None) == [3.0, 4.0]


def test_reference_arm_under_torchrun():
    port = 30500 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "1", "--frames", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
