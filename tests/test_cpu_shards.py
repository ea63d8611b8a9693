"""The multi-GPU partition on CPU: two gloo ranks split the rows of one
broadcast grid (torchscience_b200.shard), each evaluates its block with the
oracle as the per-rank compute, grad_x partials are summed over ranks in
rank order, and the reassembled result equals the single-process one.  The
bench's timing is the maximum over ranks."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from oracle import oracle as O
from torchscience_b200.shard import row_range, shard_rows, sum_over_ranks

ROWS, COLS, STRESS = 97, 80, 301


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _grid(seed=0):
    g = torch.Generator().manual_seed(seed)
    lu = lambda shape, lo, hi: torch.exp(  # noqa: E731
        torch.rand(shape, generator=g, dtype=torch.float64) * (np.log(hi) - np.log(lo)) + np.log(lo))
    a, x = lu((ROWS, 1), 1e-2, 1e3), lu((1, COLS), 1e-3, 2e3)
    gr = torch.randn(ROWS, COLS, generator=g, dtype=torch.float64)
    a_s = lu((STRESS,), 1e-2, 1e3)
    x_s = a_s * (1 + (torch.rand(STRESS, generator=g, dtype=torch.float64) * 2 - 1) * 1e-2)
    g_s = torch.randn(STRESS, generator=g, dtype=torch.float64)
    return a, x, gr, a_s, x_s, g_s


def _step(a, x, g, a_s, x_s, g_s):
    """P and the gradients of one block through the oracle (the reference's
    algorithm restated in C): values, row sums of g dP/da, column sums of
    g dP/dx, and the stress points' elementwise gradients."""
    (p,) = O.restated("regularized_gamma_p", 0, a.numpy(), x.numpy())
    fa, fx = O.restated("regularized_gamma_p", 1, g.numpy(), a.numpy(), x.numpy())
    (ps,) = O.restated("regularized_gamma_p", 0, a_s.numpy(), x_s.numpy())
    fas, fxs = O.restated("regularized_gamma_p", 1, g_s.numpy(), a_s.numpy(), x_s.numpy())
    t = torch.from_numpy
    return t(p), t(fa.sum(1, keepdims=True)), t(fx.sum(0, keepdims=True)), t(ps), t(fas), t(fxs), t(np.abs(fx).sum(0))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        a, x, g, a_s, x_s, g_s = _grid()
        mine = [shard_rows(t, rank, world) for t in (a, x, g, a_s, x_s, g_s)]
        p, ga, gx_part, ps, gas, gxs, _ = _step(*mine)
        gx = sum_over_ranks(gx_part)
        t = bench.max_over_ranks([1.0 + rank, 5.0 - rank], dist, torch.device("cpu"))
        q.put((rank, p, ga, gx, ps, gas, gxs, t))
    finally:
        dist.destroy_process_group()


def test_row_range_covers_every_row_once():
    for n in (0, 1, 5, 97, 4096):
        for world in (1, 2, 3, 8):
            ranges = [row_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        row_range(10, 2, 2)


def test_two_ranks_reassemble_the_single_process_result():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=120) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    p1, ga1, gx1, ps1, gas1, gxs1, gx_terms = _step(*_grid())
    # values and the row input's gradient: the ranks' blocks, concatenated, are the single-process result
    assert torch.equal(torch.cat([r[1] for r in out]), p1)
    assert torch.equal(torch.cat([r[2] for r in out]), ga1)
    assert torch.equal(torch.cat([r[4] for r in out]), ps1)
    assert torch.equal(torch.cat([r[5] for r in out]), gas1)
    assert torch.equal(torch.cat([r[6] for r in out]), gxs1)
    # the column input's gradient: the same on both ranks, the single-process sum up to summation order
    assert torch.equal(out[0][3], out[1][3])
    assert bool(((out[0][3] - gx1).abs().squeeze(0) <= 1e-14 * gx_terms + 1e-300).all())
    assert out[0][7] == out[1][7] == [2.0, 5.0]  # timings: max over ranks, the same on every rank


def test_single_process_timing_is_unchanged():
    assert bench.max_over_ranks([0.25, 3.0], None, torch.device("cpu")) == [0.25, 3.0]


def test_bench_shards_cover_the_workload():
    full = bench.make_inputs(0)
    world = 3
    shards = [bench.make_shard(r, world) for r in range(world)]
    for k in (0, 2, 3, 4, 5):  # a, g and the stress points are split; x is shared
        assert torch.equal(torch.cat([s[k] for s in shards]), full[k])
    assert all(torch.equal(s[1], full[1]) for s in shards)
