"""The replica (N > 1) host logic of bench.py on two CPU ranks over gloo: the max-over-ranks timing
reduction every workload uses, the dealing of serving requests and batch systems to ranks, and the
whole-job rate.  No GPU: the ranks are two processes on 127.0.0.1."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import argparse

        import bench
        t = bench.max_over_ranks(1.0 + 2.5 * rank, world)            # per-rank times 1.0 and 3.5
        args = argparse.Namespace(requests=11, rate=4.0, nmin=32, nmax=64, remin=100.0, remax=400.0, systems=3)
        served = bench.deal(bench.serve_trace(args), rank, world)
        systems = bench.batch_params(args, rank)
        out.put((rank, t, [q["arrival"] for q in served], [(q["n"], q["mesh_seed"]) for q in systems],
                 bench.aggregate_rate(10, world, t)))
    finally:
        torch.distributed.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r, t, arrivals, systems, rate = out.get(timeout=120)
        res[r] = (t, arrivals, systems, rate)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the slowest rank's time, and the job rate counts both ranks' work
    assert res[0][0] == res[1][0] == 3.5
    assert res[0][3] == res[1][3] == pytest.approx(20 / 3.5)
    # requests dealt round-robin: disjoint, and together the whole trace
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    args = argparse.Namespace(requests=11, rate=4.0, nmin=32, nmax=64, remin=100.0, remax=400.0, systems=3)
    full = [q["arrival"] for q in bench.serve_trace(args)]
    assert sorted(res[0][1] + res[1][1]) == sorted(full)
    assert not set(res[0][1]) & set(res[1][1])
    assert len(res[0][1]) == 6 and len(res[1][1]) == 5
    # each replica solves its own seeded batch
    assert res[0][2] != res[1][2]


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(2.0, 1) == 2.0
    assert bench.deal([1, 2, 3], 0, 1) == [1, 2, 3]
    assert bench.aggregate_rate(4, 1, 2.0) == 2.0
