"""Multi-rank plumbing of bench.py on CPU: ranks are independent replicas
(no data-path collective); the timed region's length is the maximum over
ranks, and under torchrun only rank 0 prints its JSON line."""
import json
import os
import subprocess
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    got = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist)
    out[rank] = got
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, 29517, out), nprocs=2, join=True)
        assert out[0] == [2.0, 10.0] and out[1] == [2.0, 10.0]


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 4.0], None) == [3.0, 4.0]


def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", "29519", os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--cpu-sample-steps", "8"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
