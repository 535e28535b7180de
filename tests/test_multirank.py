"""The N > 1 host logic of bench.py on CPU: two gloo ranks, as torchrun launches them.

Each rank reads RANK / WORLD_SIZE / LOCAL_RANK, encodes its own clip (distinct seeds: replicas,
weak scaling, no collective on the data path), and every reported time is the maximum over ranks;
the reference arm runs on rank 0 alone and the other ranks return without output.
"""
import datetime
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import io
    import contextlib
    import torch.distributed as dist
    import bench
    r, w, local = bench.dist_env()
    dist.init_process_group("gloo", rank=r, world_size=w, timeout=datetime.timedelta(seconds=60))
    slowest = bench.max_over_ranks(10.0 + 5.0 * r, dist, "cpu")
    out = io.StringIO()

    class Args:
        gpus, steps, warmup = w, 1, 0
    with contextlib.redirect_stdout(out):
        if r != 0:
            bench.run_reference(Args, r, w)  # returns at once on ranks other than 0
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, local, slowest, bench.clip_seed(r), out.getvalue()))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[:3] for r in results] == [(0, 2, 0), (1, 2, 1)]
    assert all(r[3] == 15.0 for r in results), "max over ranks"
    assert results[0][4] != results[1][4], "each rank encodes its own clip"
    assert results[1][5] == "", "reference arm prints on rank 0 only"
