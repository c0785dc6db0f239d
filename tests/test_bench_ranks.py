"""The multi-GPU replica path of bench.py on the CPU: two gloo ranks reduce
their device times (max) and scanned edges (sum) as the NCCL ranks do, and
the reference arm prints nothing on ranks other than 0."""
from __future__ import annotations

import os
import subprocess
import sys

import torch.multiprocessing as mp

from tests.conftest import ROOT


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms, edges = bench.reduce_over_ranks(dist, 100.0 + 50.0 * rank, 1_000 * (rank + 1), "cpu")
        out.put((rank, ms, edges))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_times_and_edges_reduce_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, edges in got:
        assert ms == 150.0  # the slowest rank's time
        assert edges == 3_000.0  # all ranks' edges


def test_single_process_reduction_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.reduce_over_ranks(None, 12.5, 40, "cpu") == (12.5, 40.0)


def test_reference_arm_is_silent_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, env=env, cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
