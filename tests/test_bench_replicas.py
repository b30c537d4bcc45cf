"""bench.py's multi-process plumbing on the CPU: two gloo ranks rendezvous on
127.0.0.1, agree on the slowest rank's time (max over ranks), and the whole-job
rate of independent replicas is the summed tokens over that time; the
reference arm runs on rank 0 only."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, str(ROOT))
    import bench

    w, r, local, pg = bench.dist_setup()
    try:
        seconds = 1.0 + rank  # rank 1 is the slowest
        mx = bench.allreduce_max(pg, seconds)
        bench.barrier(pg)
        ref = bench.run_reference(None, w, r) if r != 0 else "skipped"
        out.put((r, w, mx, bench.whole_job_rate(w, 1000, 10, mx), ref))
    finally:
        pg.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time_and_rate():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in procs)
    for r, w, mx, rate, ref in res:
        assert w == 2 and mx == pytest.approx(2.0)
        assert rate == pytest.approx(2 * 1000 * 10 / 2.0)
    assert res[1][4] is None  # the reference arm prints nothing on rank 1
