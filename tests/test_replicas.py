"""CPU tests (gloo, world size 2) of the replica host logic that bench.py and a
multi-GPU serving driver use: max-over-ranks timing, whole-job rate, per-rank
seeds and request dispatch."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from kg_b200 import replicas
    w, r, _ = replicas.rank_env()
    replicas.init(w, backend="gloo", timeout_s=30)
    ms = 10.0 + 5.0 * r                      # rank 1 is the slower one
    m = replicas.max_over_ranks(ms, w)
    mine = replicas.dispatch(range(11), w, r)
    out[r] = (m, replicas.job_rate(1000, w, m), replicas.replica_seed(7, r), mine)
    replicas.finish(w)


def test_two_rank_replica_logic():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    (m0, rate0, s0, d0), (m1, rate1, s1, d1) = out[0], out[1]
    assert m0 == m1 == 15.0                  # every rank sees the slowest rank's time
    assert rate0 == rate1 == pytest.approx(2 * 1000 / 0.015)
    assert s0 != s1
    assert sorted(d0 + d1) == list(range(11)) and not set(d0) & set(d1)


def test_single_process_defaults():
    from kg_b200 import replicas
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.job_rate(10, 1, 1000.0) == 10.0
    assert replicas.dispatch([1, 2, 3], 1, 0) == [1, 2, 3]
