"""The multi-GPU bench path's host logic on CPU ranks (gloo, world size 2):
shard assignment, sum of the partial counts, max of the times -- the
reference's MPI_Reduce (tc_multigpu/tc_challenge_multigpu.cu:198-206)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, partials, times, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shard, num = bench.shard_of(rank, world)
        total, tmax = bench.combine_ranks(partials[shard], times[rank], "cpu")
        out.put((rank, shard, num, total, tmax))
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_counts_and_take_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    partials = [1_000_000_007, 2_999_999_993]
    times = [12.5, 17.25]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, partials, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [0, 1] and all(r[2] == 2 for r in res)
    assert all(r[3] == sum(partials) for r in res)
    assert all(r[4] == max(times) for r in res)


def test_two_ranks_sum_wrapping_pattern_partials():
    """Pattern partials are c1 - c2 of per-shard sums: a shard's value can
    wrap below zero (mod 2^64); the combined count is their sum mod 2^64."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    full = 123_456_789
    partials = [(full + 5 - (1 << 40)) % (1 << 64), ((1 << 40) - 5) % (1 << 64)]
    partials[1] = (full - partials[0]) % (1 << 64)
    assert partials[0] >= (1 << 63) or partials[1] >= (1 << 63)
    times = [3.0, 2.0]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, partials, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(r[3] == full for r in res)


def test_shard_of_rejects_bad_rank():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    with pytest.raises(ValueError):
        bench.shard_of(2, 2)
