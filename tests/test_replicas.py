"""The multi-GPU layout of the benchmark (independent replicas, one per
process) on the host: two gloo ranks take the max-over-ranks of their times
and compute the whole-job rate the same way bench.py does."""
import os
import socket

import torch.multiprocessing as mp

from rsdft_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    r, w, local = replicas.rank_info()
    pg = replicas.init(w, "gloo", timeout_s=60)
    try:
        ms = 10.0 + 5.0 * r  # rank 1 is the slow one
        worst = replicas.max_over_ranks(ms, pg)
        out[r] = (r, w, local, worst, replicas.whole_job_rate(1000.0, w, worst))
    finally:
        pg.destroy_process_group()


def test_two_replicas_max_over_ranks():
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
    assert sorted(out.keys()) == [0, 1]
    for r in (0, 1):
        rank, world, local, worst, rate = out[r]
        assert (rank, world, local) == (r, 2, r)
        assert worst == 15.0
        assert abs(rate - 2 * 1000.0 / 15.0) < 1e-12


def test_single_process_needs_no_group():
    assert replicas.rank_info({}) == (0, 1, 0)
    assert replicas.init(1) is None
    assert replicas.max_over_ranks(3.5, None) == 3.5
