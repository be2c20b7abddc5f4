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


def test_reference_arm_small_grid():
    """`bench.py --impl reference` on a 24^3 grid: independent single-core oracle
    processes solve the whole problem (no size extrapolation); the line's steps
    times ms_per_step is the timed region, and the solves reach rerr 1e-10."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--n", "24",
                        "--steps", "4", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 4 and line["config"]["n"] == 24
    cb = line["cpu_baseline"]
    nsolves = sum(len(s) for s in cb["solve_s"])
    assert nsolves == 4 and 4 % cb["cores"] == 0
    assert line["value"] == pytest.approx(1e3 / line["ms_per_step"])
    assert max(max(s) for s in cb["solve_s"]) <= line["ms_per_step"] * 4 / 1e3 * (1 + 1e-9)
    assert all(it > 0 for its in cb["iterations"] for it in its)
