"""Multi-GPU plumbing of the path: one process per GPU, torch.distributed.

* ``exchange_slab_halos``: a field split into slabs along X (the slowest axis),
  one slab per rank, gets its ``ghost`` X planes from the neighbouring ranks'
  interior planes (periodic wrap between the last rank and rank 0, or left
  untouched at the ends).  Point-to-point send/recv into the receiver's own
  buffers (NCCL over NVLink on GPUs, gloo on CPU); the two messages a rank
  exchanges with one peer are posted in the same order on both sides, so they
  also match when the left and right neighbours are the same rank.
* ``partition_grids``: the batched rollouts' grids are independent, so ranks
  take disjoint subsets with no communication; largest grid first to the least
  loaded rank (ties: lowest index) balances the cell counts.
"""
from __future__ import annotations

import torch


def partition_grids(cells, world: int) -> list[list[int]]:
    """Indices of the grids each of ``world`` ranks advances, by greedy cell-count bin-packing.

    Deterministic: every rank computes the same partition from the same sizes."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    loads = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += int(cells[i])
    return [sorted(p) for p in parts]


def exchange_slab_halos(field: torch.Tensor, ghost: int, periodic: bool = True, group=None) -> None:
    """Fill the ``ghost`` low and high X planes of this rank's slab from its neighbours.

    ``field`` is the rank's slab (X_local + 2*ghost, ...) with the interior planes
    ``ghost .. X_local + ghost - 1`` owned by this rank; ranks are ordered along X.
    Collective over ``group``: every rank calls it with slabs of the same plane shape."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    g = int(ghost)
    n = field.shape[0]
    if g == 0 or world == 1 and not periodic:
        return
    if n < 3 * g:
        raise ValueError("a slab needs at least `ghost` interior planes")
    if world == 1:  # periodic on one rank: wrap locally
        field[0:g].copy_(field[n - 2 * g:n - g])
        field[n - g:n].copy_(field[g:2 * g])
        return
    left, right = (rank - 1) % world, (rank + 1) % world
    has_left = periodic or rank > 0
    has_right = periodic or rank < world - 1
    send_lo = field[g:2 * g].contiguous()
    send_hi = field[n - 2 * g:n - g].contiguous()
    recv_lo = torch.empty_like(send_lo)
    recv_hi = torch.empty_like(send_hi)
    glob = (lambda r: dist.get_global_rank(group, r)) if group is not None else (lambda r: r)
    ops = []
    # post order per peer: (low planes to the left, high planes to the right), and receive in the
    # order the peer sends: from the right its low planes first, from the left its high planes second
    if has_left:
        ops.append(dist.P2POp(dist.isend, send_lo, glob(left), group))
    if has_right:
        ops.append(dist.P2POp(dist.isend, send_hi, glob(right), group))
    if has_right:
        ops.append(dist.P2POp(dist.irecv, recv_hi, glob(right), group))
    if has_left:
        ops.append(dist.P2POp(dist.irecv, recv_lo, glob(left), group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    if has_left:
        field[0:g].copy_(recv_lo)
    if has_right:
        field[n - g:n].copy_(recv_hi)


def exchange_local_slabs(fields, halo: int) -> None:
    """``exchange_slab_halos`` (not periodic) for several slabs held by one process:
    fields[r] is slab r's array (rows ordered along X, ``halo`` rows beyond the owned
    block on each cut side); each slab's halo rows take its neighbours' owned rows."""
    h = int(halo)
    for left, right in zip(fields[:-1], fields[1:]):
        lo_send = right[h:2 * h].clone()
        hi_send = left[left.shape[0] - 2 * h:left.shape[0] - h].clone()
        left[left.shape[0] - h:].copy_(lo_send)
        right[:h].copy_(hi_send)
