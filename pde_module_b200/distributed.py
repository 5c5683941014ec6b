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
* ``SlabHeatRollout``: the fused heat rollout of a grid split into slabs along
  X.  Each block of k steps is one halo exchange (``exchange_cut_planes``) and
  one k-step pass of the fused kernel over the slab; the owned planes equal the
  single-array rollout bit for bit.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable

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
    # X is the slowest axis: a run of planes is one contiguous block, sent from
    # and received into the field itself
    send_lo = field[g:2 * g]
    send_hi = field[n - 2 * g:n - g]
    recv_lo = field[0:g]
    recv_hi = field[n - g:n]
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


def slab_partition(X: int, ghost: int, world: int) -> list[tuple[int, int]]:
    """Planes [a, b) of an X-plane array (ghost planes included) that each of
    ``world`` ranks owns: the X - 2*ghost interior planes split evenly (the first
    (X - 2g) % world ranks take one more), rank 0 also owning the low ghost planes
    and the last rank the high ones."""
    nint = int(X) - 2 * int(ghost)
    if world < 1 or nint < world:
        raise ValueError(f"{nint} interior planes cannot be split over {world} ranks")
    base, extra = divmod(nint, world)
    out, start = [], int(ghost)
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((0 if r == 0 else start, start + n if r < world - 1 else int(X)))
        start += n
    return out


def slab_halo(ghost: int, order: int, steps_per_block: int) -> int:
    """Halo planes beside a cut for ``steps_per_block`` steps between exchanges.

    A slab is stepped as a whole array, so its cut faces take the boundary fill
    as well: the fill rewrites the g + 1 planes next to the cut (the ghost planes
    and the node plane) and each step carries that error R = order/2 planes
    further in.  After k steps the planes up to g + k*R from the cut differ from
    the single-array run; the first owned plane sits one plane beyond."""
    return int(ghost) + int(steps_per_block) * (int(order) // 2) + 1


def exchange_cut_planes(field: torch.Tensor, h_lo: int, n_own: int, h_hi: int, group=None) -> None:
    """Fill a slab's halo planes at its cuts from the neighbouring ranks' owned planes.

    ``field`` is (h_lo + n_own + h_hi, ...) with the owned planes h_lo .. h_lo +
    n_own - 1; h_lo > 0 where rank - 1 holds the planes below, h_hi > 0 where
    rank + 1 holds those above, every cut with the same halo h on both sides.
    The lower neighbour's last h owned planes land in planes 0 .. h-1, the upper
    neighbour's first h in the top h; send and receive buffers are the field's
    own contiguous plane runs.  Collective over ``group`` (ranks ordered along X)."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    glob = (lambda r: dist.get_global_rank(group, r)) if group is not None else (lambda r: r)
    top = h_lo + n_own
    ops = []
    if h_lo:
        if n_own < h_lo:
            raise ValueError("a slab needs at least `halo` owned planes")
        ops.append(dist.P2POp(dist.isend, field[h_lo:2 * h_lo], glob(rank - 1), group))
        ops.append(dist.P2POp(dist.irecv, field[0:h_lo], glob(rank - 1), group))
    if h_hi:
        if n_own < h_hi:
            raise ValueError("a slab needs at least `halo` owned planes")
        ops.append(dist.P2POp(dist.isend, field[top - h_hi:top], glob(rank + 1), group))
        ops.append(dist.P2POp(dist.irecv, field[top:top + h_hi], glob(rank + 1), group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


# stepper(src, dst, nsteps, n0): nsteps fused steps of the whole slab array from
# src into dst, the first being step n0 of the run
Stepper = Callable[[torch.Tensor, torch.Tensor, int, int], None]


class SlabHeatRollout:
    """Fused heat rollout (boundary fill + Laplacian + forward Euler, the loop of
    examples/2D_Heat_Equation.py:57-65) of a grid split into slabs along X, one
    slab per rank of ``group``.

    The rank holds its owned planes (``slab_partition``) plus ``halo`` planes on
    each cut side (``slab_halo`` for the pass depth k).  A call runs blocks of k
    steps: an exchange of the halo planes with the neighbour ranks, then one
    k-step pass of the fused rollout over the slab as a whole array, ping-ponging
    between two buffers.  The owned planes equal the single-array rollout bit for
    bit.  ``boundary`` is a GridBoundary with standard face groups on any field of
    the grid's (Y, Z, N) (its rules do not depend on X); X-face groups act at the
    global ends only.  Ramp groups take the global step index (t0 + n*dt).

    ``stepper`` replaces the CUDA pass (host-side tests of the decomposition); by
    default the library's ``pde_heat_rollout_from`` runs on the slab's device."""

    def __init__(self, boundary, dx: float, alpha: float, dt: float, global_x: int, order: int = 2,
                 steps_per_pass: int = 0, group=None, device=None, stepper: Stepper | None = None,
                 rank: int | None = None, world: int | None = None) -> None:
        import torch.distributed as dist
        from ._lib import make_grid
        self.group = group
        # rank / world given: slabs held by one process (exchange_local_slabs between blocks)
        self.local_slabs = world is not None
        self.world = int(world) if world is not None else (dist.get_world_size(group) if dist.is_initialized() else 1)
        self.rank = int(rank) if rank is not None else (dist.get_rank(group) if dist.is_initialized() else 0)
        self.boundary = boundary
        self.dx, self.alpha, self.dt = float(dx), float(alpha), float(dt)
        self.order = int(order)
        self.ghost = int(boundary.ghost_cells)
        self.ncomp = int(boundary.inputs[0])
        Y, Z = int(boundary.grid_shape[1]), int(boundary.grid_shape[2])
        self.global_x = int(global_x)
        a, b = slab_partition(self.global_x, self.ghost, self.world)[self.rank]
        self.own = (a, b)
        self._stepper = stepper
        if stepper is None:
            from ._lib import lib
            probe = make_grid((self.global_x, Y, Z), self.ghost, self.order, self.dx)
            k = lib().pde_heat_pass_depth(C.byref(probe), self.ncomp, int(steps_per_pass))
            if k < 1:
                raise ValueError(f"pde_heat_pass_depth: status {k}")
        else:
            k = int(steps_per_pass) if steps_per_pass > 0 else 1
        self.k = int(k)
        self.halo = slab_halo(self.ghost, self.order, self.k)
        self.h_lo = self.halo if self.rank > 0 else 0
        self.h_hi = self.halo if self.rank < self.world - 1 else 0
        self.n_own = b - a
        if self.world > 1 and self.n_own < self.halo:
            raise ValueError(f"slab of {self.n_own} planes is thinner than its halo ({self.halo})")
        shape = (self.h_lo + self.n_own + self.h_hi, Y, Z, self.ncomp)
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.buffers = [torch.zeros(shape, dtype=torch.float32, device=dev) for _ in range(2)]
        self.cur = 0
        self.grid = make_grid(shape[:3], self.ghost, self.order, self.dx)
        self.rules = boundary.rules() if stepper is None else None
        self.work = torch.zeros(shape, dtype=torch.float32, device=dev) if stepper is None else None
        self.steps_done = 0

    @property
    def field(self) -> torch.Tensor:
        """The current slab array (halo planes included)."""
        return self.buffers[self.cur]

    @property
    def owned(self) -> torch.Tensor:
        """View of the current owned planes: global planes own[0] .. own[1]-1."""
        return self.buffers[self.cur][self.h_lo:self.h_lo + self.n_own]

    def load(self, planes: torch.Tensor) -> None:
        """Set the owned planes (a tensor of this slab's n_own planes, or the whole
        global array, whose owned range is taken); resets the step count."""
        if planes.shape[0] == self.global_x and self.global_x != self.n_own:
            planes = planes[self.own[0]:self.own[1]]
        self.owned.copy_(planes)
        self.steps_done = 0

    def _cuda_pass(self, src: torch.Tensor, dst: torch.Tensor, nsteps: int, n0: int) -> None:
        from ._lib import lib, check, stream_ptr
        check(lib().pde_heat_rollout_from(C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()),
                                          C.c_void_p(self.work.data_ptr()), C.byref(self.grid), self.ncomp,
                                          C.byref(self.rules), self.alpha, self.dt, int(nsteps), self.k,
                                          float(self.t0), self.dt, int(n0), C.c_void_p(stream_ptr(src))),
              "pde_heat_rollout_from")

    def block(self, nsteps: int, t0: float = 0.0) -> None:
        """One pass of nsteps <= k steps over the slab, no exchange (the halo planes
        must hold the neighbours' planes)."""
        if not 0 < nsteps <= self.k:
            raise ValueError(f"a block is 1..{self.k} steps")
        self.t0 = float(t0)
        (self._stepper or self._cuda_pass)(self.buffers[self.cur], self.buffers[1 - self.cur], int(nsteps),
                                           self.steps_done)
        self.cur = 1 - self.cur
        self.steps_done += int(nsteps)

    def __call__(self, nsteps: int, t0: float = 0.0) -> torch.Tensor:
        """Advance ``nsteps``; step n of the run (counted from the last ``load``)
        fills the boundary at t0 + n*dt.  Returns the owned planes.  Collective
        over the group: every rank calls it with the same nsteps."""
        if self.local_slabs and self.world > 1:
            raise RuntimeError("slabs held by one process advance through advance_local_slabs")
        left = int(nsteps)
        while left > 0:
            kb = min(self.k, left)
            if self.world > 1:
                exchange_cut_planes(self.field, self.h_lo, self.n_own, self.h_hi, self.group)
            self.block(kb, t0)
            left -= kb
        return self.owned


def advance_local_slabs(slabs: list[SlabHeatRollout], nsteps: int, t0: float = 0.0) -> None:
    """``SlabHeatRollout.__call__`` for all slabs of a grid held by one process
    (slabs[r] built with rank=r, world=len(slabs)): the same blocks, the halo
    exchange done by copies between the slabs' arrays."""
    left = int(nsteps)
    k = slabs[0].k
    while left > 0:
        kb = min(k, left)
        if len(slabs) > 1:
            exchange_local_slabs([s.field for s in slabs], slabs[0].halo)
        for s in slabs:
            s.block(kb, t0)
        left -= kb
