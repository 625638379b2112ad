"""CPU, world_size 2 (gloo): the multi-rank plumbing bench.py uses for `--gpus N` -- rendezvous
on 127.0.0.1, barrier, and the max-over-ranks reduction of the timed region.  Multiplications
are independent (replicas only), so there is no data-path collective to test."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, REPO)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init()
    assert (w, r) == (world, rank)
    bench.barrier(w)
    # each rank reports a different elapsed time; every rank must see the maximum
    got = bench.max_over_ranks(10.0 + rank, w)
    q.put((rank, got))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    results = dict(q.get(timeout=5) for _ in range(2))
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert results == {0: 11.0, 1: 11.0}
