"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (127.0.0.1).

The hot path runs as independent replicas (one per GPU, no collective on the
data path); what crosses ranks is the timing: a barrier on both sides of the
timed region and the maximum over ranks.  The reference arm prints on rank 0
only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench._barrier(world, None)
        mx = bench._max_over_ranks(10.0 + rank, world, None)
        bench._barrier(world, None)
        # The reference arm: ranks other than 0 return without work or output.
        out = io.StringIO()
        if rank != 0:
            with redirect_stdout(out):
                bench.run_reference(bench_args())
        q.put((rank, mx, out.getvalue()))
    finally:
        dist.destroy_process_group()


def bench_args():
    import argparse
    return argparse.Namespace(steps=1, warmup=3, gpus=2)


def test_two_gloo_ranks_barrier_and_max():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[1] for r in res] == [11.0, 11.0]
    assert res[1][2] == ""
