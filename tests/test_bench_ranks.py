"""bench.py's multi-rank plumbing on CPU: two gloo ranks, the whole-job throughput takes the
bodies of every rank over the slowest rank's time, and the reference arm runs on rank 0 only."""
import contextlib
import io
import os
import socket

import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        reduce = bench.make_reducer(2, "cpu")
        # rank 0: 1000 bodies in 100 ms; rank 1: 3000 bodies in 150 ms
        value, total_ms = bench.job_throughput([1000, 3000][rank], 4, 10, [100.0, 150.0][rank], reduce)
        out[rank] = (value, total_ms, reduce(float(rank + 1), "sum"))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate():
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(_free_port(), out), nprocs=2, join=True)
    for rank in (0, 1):
        value, total_ms, s = out[rank]
        assert total_ms == 150.0 and s == 3.0
        assert abs(value - (4000 * 4 * 10) / 0.150) < 1e-6 * value


def test_single_rank_is_identity():
    value, total_ms = bench.job_throughput(1000, 4, 10, 100.0, bench.make_reducer(1, "cpu"))
    assert total_ms == 100.0 and abs(value - 400000.0) < 1e-6


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.main(["--impl", "reference", "--steps", "1", "--warmup", "1"])
    assert buf.getvalue() == ""
