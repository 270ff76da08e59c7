"""bench.py's multi-rank plumbing on CPU: two gloo ranks (one process each,
rendezvous on 127.0.0.1) run the same helpers the GPU job uses with nccl.
Times are reported as the slowest rank's (max over ranks), the whole-job
value counts every rank's work, and the reference arm runs on rank 0 only:
the other ranks exit 0 without printing."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, REPO)
    import bench

    w, r, local, dist = bench.init_dist("gloo")
    try:
        t = bench.max_over_ranks(1.5 + r, dist, "cpu")  # ranks 0, 1 report 1.5 and 2.5 ms
        same = bench.max_over_ranks(3.0, dist, "cpu")
        dist.barrier()
        q.put((r, w, local, t, same))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[:3] for g in got] == [(0, 2, 0), (1, 2, 1)]
    assert all(g[3] == 2.5 and g[4] == 3.0 for g in got)


def test_single_process_needs_no_process_group(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "1")
    sys.path.insert(0, REPO)
    import bench

    w, r, local, dist = bench.init_dist("gloo")
    assert (w, dist) == (1, None)
    assert bench.max_over_ranks(4.25, None, "cpu") == 4.25


def test_reference_arm_prints_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, REPO)
    import bench

    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"steps": 1, "warmup": 0, "gpus": 2})()
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.run_reference(args) == 0
    assert buf.getvalue() == ""
