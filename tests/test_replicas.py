"""The multi-GPU plumbing (discoeb_b200.replicas) with two gloo ranks on the CPU: start-up from
the torchrun environment, the max-over-ranks timing reduction, barriers, tear-down, and the
round-robin mode split."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "disco-eb_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      LOCAL_RANK=str(rank))
    from discoeb_b200 import replicas
    r, w, dist = replicas.init("gloo", timeout_s=60)
    assert (r, w) == (rank, world) and dist is not None
    replicas.barrier(dist)
    m = replicas.max_over_ranks(1.5 + rank, dist)
    ks = np.geomspace(1e-4, 10.0, 11)
    mine = replicas.shard(ks, r, w)
    # every rank gets all rows back in the caller's order; partial sums add up
    rows = np.stack([mine * 1.0, np.sqrt(mine + 1.0)], axis=1)[:, :, None]
    full = replicas.gather_rows(rows, mine, ks.size, dist)
    total = replicas.sum_over_ranks(np.array([rank + 1.0, 0.5]), dist)
    replicas.finish(dist)
    out.put((rank, m, mine.tolist(), full.tolist(), total.tolist()))


def test_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]
    want = np.stack([np.arange(11.0), np.sqrt(np.arange(11.0) + 1.0)], axis=1)[:, :, None]
    for r in res:
        np.testing.assert_array_equal(np.array(r[3]), want)
        assert r[4] == [3.0, 1.0]
    parts = [set(r[2]) for r in res]
    assert parts[0].isdisjoint(parts[1]) and parts[0] | parts[1] == set(range(11))
    assert abs(len(parts[0]) - len(parts[1])) <= 1


def test_single_process_needs_no_process_group(monkeypatch):
    from discoeb_b200 import replicas
    monkeypatch.setenv("WORLD_SIZE", "1")
    rank, world, dist = replicas.init("gloo")
    assert world == 1 and dist is None
    assert replicas.max_over_ranks(3.0, dist) == 3.0
    replicas.finish(dist)
    np.testing.assert_array_equal(replicas.shard(np.array([0.1, 1.0, 0.01]), 0, 1), [0, 1, 2])
    np.testing.assert_array_equal(replicas.gather_rows(np.array([[1.0], [2.0]]), [1, 0], 2, dist), [[2.0], [1.0]])
    np.testing.assert_array_equal(replicas.sum_over_ranks([1.0, 2.0], dist), [1.0, 2.0])
