"""Row partition of a broadcast grid across ranks (one process per GPU).

Every output element of these operators is independent, so a grid of an
(R, 1) input against a (1, C) input splits into contiguous row blocks, one
per rank, with no exchange for the values or for the gradient of the row
input (each rank's rows of grad_a are final).  The gradient of the column
input is a sum over all rows: each rank reduces its own rows and
:func:`sum_over_ranks` adds the partials, in rank order, so that the result
does not depend on the collective's algorithm and equals the sum of the
ranks' partials taken one after another.

The reference has no distributed code; this is the partition of its
broadcast iteration space that a multi-GPU job uses.
"""

from __future__ import annotations

import torch


def row_range(n_rows: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block [start, stop) of rank `rank` out of `world`: the
    first n_rows % world ranks take one row more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    base, extra = divmod(n_rows, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_rows(t: torch.Tensor, rank: int, world: int, dim: int = 0) -> torch.Tensor:
    """The rank's block of `t` along `dim` (a view); a size-1 (broadcast)
    dimension is returned whole."""
    if t.shape[dim] == 1:
        return t
    start, stop = row_range(t.shape[dim], rank, world)
    return t.narrow(dim, start, stop - start)


def sum_over_ranks(partial: torch.Tensor, group=None) -> torch.Tensor:
    """Sum of every rank's `partial` (same shape on all ranks), added in
    rank order 0, 1, ..., world-1: deterministic, and the same on every rank.
    Gathers world x partial.numel() elements, which for a reduced gradient
    (one value per column) is small."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if world == 1:
        return partial
    parts = [torch.empty_like(partial) for _ in range(world)]
    dist.all_gather(parts, partial.contiguous(), group=group)
    out = parts[0].clone()
    for p in parts[1:]:
        out += p
    return out
