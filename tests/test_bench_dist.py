"""The N-GPU bench path without GPUs: two gloo ranks on the CPU run the
bench's max-over-ranks reduction and its whole-job aggregation (every rank
solves its own replica; the slowest rank sets the time)."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        times = [10.0 + rank, 20.0 - 5.0 * rank]          # per-rank ms of two timed regions
        got = bench.max_over_ranks(times, ws, "cpu")
        out[rank] = (got, bench.aggregate(ws, 4, got[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_aggregate():
    import torch.multiprocessing as mp
    ws = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(ws, _free_port(), out), nprocs=ws, join=True)
    for r in range(ws):
        got, sps = out[r]
        assert got == [11.0, 20.0]                        # the max over ranks, on every rank
        assert sps == pytest.approx(ws * 4 / 0.011)       # 2 ranks x 4 solves in the slowest 11 ms


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks([3.0, 4.0], 1, "cpu") == [3.0, 4.0]
    assert bench.aggregate(1, 10, 500.0) == pytest.approx(20.0)
