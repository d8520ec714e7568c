"""bench.py's multi-GPU host logic (replicas only) on CPU ranks over gloo:
the timing is the slowest rank's, the value the whole job's, and the
reference arm runs on rank 0 alone."""

import contextlib
import io
import os
import pathlib
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        sec = bench.reduce_max(ws, 1.0 + rank, device="cpu")  # rank r took 1 + r seconds
        bench.barrier(ws, device="cpu")
        value = bench.job_throughput(ws, 1000, 10, sec)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            if rank != 0:  # the reference arm: every rank but 0 returns without work or output
                bench.run_reference(type("A", (), {"steps": 1, "warmup": 1, "gpus": ws})(), ws, rank)
        out[rank] = (sec, value, buf.getvalue())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ws, port = 2, 29517
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    for rank in range(ws):
        sec, value, printed = res[rank]
        assert sec == 2.0                      # the slowest rank
        assert value == pytest.approx(2 * 1000 * 10 / 2.0)
    assert res[1][2] == ""
