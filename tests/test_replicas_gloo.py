"""The replica plumbing of bench.py on two CPU ranks (gloo): barrier,
max-over-ranks timing and the whole-job value.  No data-path collective
exists: every rank runs its own propagation."""

import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), PQ_DIST_BACKEND="gloo")
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    w, r, _ = bench.dist_setup()
    bench.barrier(w)
    slowest = bench.max_over_ranks(w, 1.0 + r)  # rank r "took" 1 + r seconds
    out.put((r, slowest, bench.replica_value(w, 100.0, slowest)))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_replicas_time_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2.0, 100.0), (1, 2.0, 100.0)]
