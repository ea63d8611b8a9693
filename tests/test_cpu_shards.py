"""The multi-GPU bench path on CPU: two gloo ranks, each with its own seeded
shard (no data-path collective), timings combined as the maximum over ranks."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        a = bench.make_inputs(rank)[0]
        t = bench.max_over_ranks([1.0 + rank, 5.0 - rank], dist, torch.device("cpu"))
        q.put((rank, float(a[0, 0]), t))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_inputs_and_take_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, a0, t0), (r1, a1, t1) = out
    assert a0 != a1  # independent shards (seed = rank)
    assert t0 == t1 == [2.0, 5.0]  # max over ranks, the same on every rank


def test_single_process_timing_is_unchanged():
    assert bench.max_over_ranks([0.25, 3.0], None, torch.device("cpu")) == [0.25, 3.0]


@pytest.mark.parametrize("rank", [0, 1, 7])
def test_shards_are_deterministic(rank):
    a1, a2 = bench.make_inputs(rank)[0], bench.make_inputs(rank)[0]
    assert torch.equal(a1, a2)
