"""Replica runs of bench.py on several ranks: the two scalar reductions (max of the times, sum of the
pairs) over a gloo process group of two CPU ranks, as torchrun starts them."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(world)
    out = (d.max(1.0 + rank), d.sum(10.0 * (rank + 1)))
    d.close()
    q.put((rank, out))


def test_replica_reductions_over_two_gloo_ranks():
    pytest.importorskip("torch.distributed")
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == (2.0, 30.0)
