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


def _partition_rank(rank, port, out):
    """Each gloo rank computes its share of the 4 096-world batch on its own (no communication),
    then the shares are gathered to check them."""
    import torch
    import torch.distributed as dist
    from natsel_b200 import scenes
    from natsel_b200.partition import partition_worlds, share_loads
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        sizes = [scenes.batch_world_size(k, 4) for k in range(4096)]
        mine = bench.batch_share({"count": 4096, "seed": 4}, rank, 2)
        gathered = [None, None]
        dist.all_gather_object(gathered, mine)
        reduce = bench.make_reducer(2, "cpu")
        bodies = sum(sizes[k] for k in mine)
        value, total_ms = bench.job_throughput(bodies, 4, 10, [100.0, 120.0][rank], reduce)
        out[rank] = (gathered, value, total_ms, share_loads(sizes, partition_worlds(sizes, 2)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_the_batch_by_body_count():
    """bench.py's multi-GPU batched path: the two ranks' shares cover every world exactly once,
    their body counts differ by less than the largest world, and the whole-job throughput counts
    every world's bodies over the slower rank's time."""
    from natsel_b200 import scenes
    out = mp.Manager().dict()
    mp.spawn(_partition_rank, args=(_free_port(), out), nprocs=2, join=True)
    sizes = [scenes.batch_world_size(k, 4) for k in range(4096)]
    for rank in (0, 1):
        gathered, value, total_ms, loads = out[rank]
        assert gathered == out[0][0]
        a, b = gathered
        assert sorted(a + b) == list(range(4096)) and not set(a) & set(b)
        assert abs(loads[0] - loads[1]) <= max(sizes)
        assert total_ms == 120.0
        assert abs(value - sum(sizes) * 4 * 10 / 0.120) < 1e-6 * value


def test_partition_is_balanced_and_deterministic():
    from natsel_b200.partition import partition_worlds, share_loads
    import random
    rng = random.Random(3)
    sizes = [rng.randint(32, 512) for _ in range(1000)]
    for ranks in (1, 2, 3, 8):
        shares = partition_worlds(sizes, ranks)
        assert shares == partition_worlds(sizes, ranks)
        assert sorted(i for s in shares for i in s) == list(range(1000))
        loads = share_loads(sizes, shares)
        # greedy longest-first packing: within the largest item of the best possible split
        assert max(loads) - min(loads) <= max(sizes)


def test_timed_schedule_spreads_over_the_run_and_stays_inside_it():
    """K timed steps every (length - W) // K steps from W + 1; K is capped at the steps the run
    has after the warm-up, so no timed step lies beyond the workload's length."""
    assert bench.timed_schedule(600, 20, 5) == [6 + 29 * k for k in range(20)]
    full = bench.timed_schedule(600, 600, 3)
    assert full == list(range(4, 601))
    assert bench.timed_schedule(1000, 10, 3)[-1] <= 1000
