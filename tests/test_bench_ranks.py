"""The multi-rank path of bench.py on CPU: two gloo ranks take the largest
step time over ranks and report all ranks' points over it (replicas; the
evaluation itself runs on one GPU per rank)."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=__import__("datetime").timedelta(seconds=60))
    import bench
    t = bench.max_over_ranks(10.0 + 5.0 * rank, ws)   # rank 1 is slower
    out[rank] = (t, bench.whole_job_rate(1000, ws, t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_step():
    import torch.multiprocessing as mp
    ws = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
    for r in range(ws):
        t, rate = out[r]
        assert t == 15.0
        assert rate == pytest.approx(2 * 1000 / 15e-3)


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.whole_job_rate(100, 1, 2.0) == pytest.approx(5e4)
