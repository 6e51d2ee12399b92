"""The multi-GPU path of bench.py on the CPU: replicas over a world-size-2 gloo group (the
aggregation the NCCL run performs), and the reference arm's rank rule."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        boards = 1000 * (rank + 1)
        dev_ms = 10.0 + rank
        e2e = (500 * (rank + 1), 2.0 + rank)
        out.put((rank, bench.aggregate_ranks(dist, boards, dev_ms, e2e, "cpu"),
                 bench.aggregate_ranks(dist, boards, dev_ms, None, "cpu")))
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, (boards, dev_ms, rate), (b2, d2, r2) in res:
        assert boards == 3000 and dev_ms == 11.0      # sum of boards, slowest rank
        assert rate == pytest.approx(1500 / 3.0)       # all boards over the slowest wall time
        assert (b2, d2, r2) == (3000, 11.0, None)


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
