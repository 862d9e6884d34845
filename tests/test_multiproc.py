"""bench.py's multi-GPU host logic (replicas, barrier, max over ranks) run as
two gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    ws, r, local, pg = bench.dist_setup()
    bench.barrier(pg)
    m = bench.max_over_ranks(pg, 10.0 * (r + 1))
    q.put((r, ws, local, m))
    pg.destroy_process_group()


def test_two_ranks_gloo():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [x[0] for x in res] == [0, 1]
    assert all(x[1] == 2 for x in res)
    assert all(x[3] == 20.0 for x in res)   # max over ranks
