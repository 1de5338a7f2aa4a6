"""The multi-GPU path of bench.py is replicas only: every rank runs its own
walk + train and the ranks meet only for the barrier and the max / sum over
ranks of the timing and the counts.  This runs that plumbing as two gloo
ranks on the CPU (no GPU, no data-path collective)."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup(None)
    assert (w, r, local) == (world, rank, rank) and pg is not None
    pg.barrier()
    mx = bench.max_over_ranks(pg, 10.0 + rank)      # per-rank device time: the job takes the slowest
    sm = bench.sum_over_ranks(pg, 1000.0 * (rank + 1))  # per-rank tokens: the job processes all of them
    # the reference arm runs on rank 0 only; other ranks leave without output
    buf = io.StringIO()
    with redirect_stdout(buf):
        if rank != 0:
            bench.bench_reference(type("A", (), {"config": "c1"})())
    pg.barrier()
    pg.destroy_process_group()
    out.put((rank, mx, sm, buf.getvalue()))


def test_two_gloo_ranks_reduce_like_the_bench():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(world))
    for rank, mx, sm, printed in res:
        assert mx == 11.0 and sm == 3000.0
        if rank != 0:
            assert printed == ""
    json.dumps(res)
