"""The multi-rank path on CPU: two gloo ranks (world size 2) shard the units, reduce the step time to the slowest
rank and sum the processed units, as bench.py does over NCCL with one process per GPU."""
import multiprocessing as mp
import os
import socket

import pytest

from xclean_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ws, rk, _ = D.env()
        a, b = D.shard(500, rk, ws)
        ms = 10.0 + 5.0 * rk                  # this rank's (fake) step time
        q.put((rk, a, b, D.max_over_ranks(ms), D.sum_over_ranks(b - a)))
    finally:
        dist.destroy_process_group()


def test_shards_partition_the_units():
    for n in (0, 1, 7, 500, 1001):
        for world in (1, 2, 3, 8):
            parts = [D.shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def test_single_process_reductions_are_identity():
    assert D.max_over_ranks(3.5) == 3.5 and D.sum_over_ranks(2.0) == 2.0


@pytest.mark.timeout(120)
def test_two_gloo_ranks_reduce_time_and_units():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [(a, b) for _, a, b, _, _ in out] == [(0, 250), (250, 500)]
    assert all(m == 15.0 for _, _, _, m, _ in out)
    assert all(s == 500.0 for _, _, _, _, s in out)
