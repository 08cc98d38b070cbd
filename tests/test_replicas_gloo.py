"""The multi-GPU form of the benchmark is replicas only: N independent
renderers, each on its own sample stream, whose timed regions are reduced
(max over ranks) and whose paths are summed.  This checks that host logic
with two gloo ranks on CPU."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, paths = bench.replica_reduce(10.0 + 5.0 * rank, 1000 * (rank + 1), dist, "cpu")
        q.put((rank, ms, paths, bench.rank_frame_offset(rank, 64, 4)))
    finally:
        dist.destroy_process_group()


def test_replica_reduction_two_ranks():
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, paths, f0 in res:
        assert ms == pytest.approx(15.0)  # the slower rank's time
        assert paths == 3000  # both ranks' paths
        assert f0 == rank * 68  # disjoint sample streams
