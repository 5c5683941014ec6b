"""Batched rollouts: many independent 2D grids of uneven sizes in one launch.

The reference advances every grid with its own module chain: for the heat
equation, examples/2D_Heat_Equation.py:57-65 runs GridBoundary -> Laplacian ->
ForwardEuler per step, three launches per step per grid.  Here all grids of a
batch advance ``nsteps`` in ONE persistent kernel that takes (time block, grid,
tile) items from a work queue; a tile starts a time block once its 3x3
neighbouring tiles have finished the previous one.  The call is one memset and
one launch, so a whole rollout can be captured in a CUDA graph (``graph``).

``BatchedHeatRollout``: per grid alpha, dt and dx; the boundary groups (standard
faces, constant values) are shared by all grids.  Each grid's result is
bit-identical to ``HeatRollout`` on that grid alone, hence to the module chain.
``BatchedWaveRollout``: leapfrog u^{n+1} = 2u^n - u^{n-1} + K Lap(u^n) with a
per-grid constant K = dt^2 c^2 and zero Dirichlet nodes, bit-identical to
``pde_wave_forward`` with a constant K field and no source.

Fields are (X, Y, 1, 1) CUDA float32 tensors, advanced in place.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import torch

from .._lib import lib, check, stream_ptr, require_cuda_f32
from .. import _lib


def _per_grid(v, n: int, name: str) -> list[float]:
    if isinstance(v, (int, float)):
        return [float(v)] * n
    v = [float(x) for x in v]
    if len(v) != n:
        raise ValueError(f"{name}: {len(v)} values for {n} grids")
    return v


class _BatchedRollout:
    kind = -1

    def _setup(self, fields, prev, dx, coef, dt, rules, ghost_cells, order, tile, steps_per_pass):
        n = len(fields)
        if n < 1:
            raise ValueError("a batch needs at least one grid")
        self.fields = list(fields)
        self.prev = list(prev) if prev is not None else None
        self.ghost_cells = int(ghost_cells)
        self.order = int(order)
        dev = self.fields[0].device
        for i, f in enumerate(self.fields):
            require_cuda_f32(f, f"fields[{i}]")
            if f.dim() != 4 or f.shape[2] != 1 or f.shape[3] != 1:
                raise ValueError(f"fields[{i}] must be (X, Y, 1, 1), got {tuple(f.shape)}")
            if f.device != dev:
                raise ValueError("all fields of a batch must be on one device")
            if self.prev is not None:
                require_cuda_f32(self.prev[i], f"prev[{i}]")
                if self.prev[i].shape != f.shape:
                    raise ValueError(f"prev[{i}] shape differs from fields[{i}]")
        self.dx = _per_grid(dx, n, "dx")
        self.coef = _per_grid(coef, n, "coef")
        self.dt = _per_grid(dt, n, "dt")
        nbuf = 1 if self.kind == _lib.PDE_BATCH_HEAT else 2
        # one scratch allocation for the whole batch
        sizes = [f.numel() * nbuf for f in self.fields]
        self._scratch = torch.empty(sum(sizes) + 64 * n, device=dev, dtype=torch.float32)
        self._desc = (_lib.PdeBatchGrid * n)()
        off = 0
        for i, f in enumerate(self.fields):
            d = self._desc[i]
            d.field = f.data_ptr()
            d.field_prev = self.prev[i].data_ptr() if self.prev is not None else None
            d.scratch = self._scratch.data_ptr() + 4 * off
            d.shape[0], d.shape[1] = int(f.shape[0]), int(f.shape[1])
            d.dx = self.dx[i]
            d.coef = self.coef[i]
            d.dt = self.dt[i]
            off += sizes[i] + (-sizes[i]) % 64  # keep every scratch 256-byte aligned
        self._rules = rules
        self.tile = tuple(tile) if tile is not None else (0, 0)
        self.steps_per_pass = int(steps_per_pass)
        self._work = None
        self._plan = None
        self._make_plan()

    def _make_plan(self) -> None:
        """(Re)build the launch plan for the current tile and steps_per_pass."""
        n = len(self.fields)
        nbytes = C.c_uint64(0)
        check(lib().pde_batch_work_bytes(self._desc, n, int(self.tile[0]), int(self.tile[1]), C.byref(nbytes)),
              "pde_batch_work_bytes")
        if self._work is None or self._work.numel() < nbytes.value:
            self._work = torch.empty(int(nbytes.value), device=self.fields[0].device, dtype=torch.uint8)
        plan = _lib.PdeBatchPlan()
        rules = C.byref(self._rules) if self._rules is not None else None
        check(lib().pde_batch_plan(self.kind, self._desc, n, self.ghost_cells, self.order, rules,
                                   int(self.tile[0]), int(self.tile[1]), self.steps_per_pass,
                                   C.c_void_p(self._work.data_ptr()), self._work.numel(), C.byref(plan),
                                   C.c_void_p(stream_ptr(self.fields[0]))), "pde_batch_plan")
        self._plan = plan

    def configure(self, tile=None, steps_per_pass=None) -> None:
        """Change the tile (tile_x, tile_y) and/or the time-block depth."""
        if tile is not None:
            self.tile = tuple(tile)
        if steps_per_pass is not None:
            self.steps_per_pass = int(steps_per_pass)
        self._make_plan()

    @property
    def plan(self) -> "_lib.PdeBatchPlan":
        return self._plan

    @property
    def cells(self) -> int:
        """Array cells (ghosts included) of all grids."""
        return sum(int(f.shape[0]) * int(f.shape[1]) for f in self.fields)

    def __call__(self, nsteps: int, t0: float = 0.0) -> list[torch.Tensor]:
        """Advance every grid nsteps.  Heat with time-ramped groups: step n of grid i
        fills its boundary at t0 + n*dt_i (dt_i as a float32)."""
        s = C.c_void_p(stream_ptr(self.fields[0]))
        if self._rules is not None and self._rules.has_ramp:
            check(lib().pde_batch_rollout_at(C.byref(self._plan), int(nsteps), float(t0), s), "pde_batch_rollout_at")
        else:
            check(lib().pde_batch_rollout(C.byref(self._plan), int(nsteps), s), "pde_batch_rollout")
        return self.fields

    def graph(self, nsteps: int) -> torch.cuda.CUDAGraph:
        """Capture one nsteps rollout in a CUDA graph; each replay advances every grid nsteps."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.fields[0].device)
        s.wait_stream(torch.cuda.current_stream(self.fields[0].device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                check(lib().pde_batch_rollout(C.byref(self._plan), int(nsteps), C.c_void_p(s.cuda_stream)),
                      "pde_batch_rollout")
        torch.cuda.current_stream(self.fields[0].device).wait_stream(s)
        return g


class BatchedHeatRollout(_BatchedRollout):
    """Heat rollouts of many 2D grids (per-grid dx, alpha, dt) in one persistent launch.

    ``boundary`` is a GridBoundary built on any one grid of the batch (standard
    face groups, constant values, one component); every grid gets its groups, with
    its own dx for Neumann ghosts.  Default: Dirichlet 0 on ALL, as
    examples/2D_Heat_Equation.py:50."""
    kind = _lib.PDE_BATCH_HEAT

    def __init__(self, fields: Sequence[torch.Tensor], dx, alpha, dt, boundary=None, ghost_cells: int = 1,
                 order: int = 2, tile=None, steps_per_pass: int = 0) -> None:
        if boundary is None:
            from ..FDM.boundary import GridBoundary
            boundary = GridBoundary(fields[0], _per_grid(dx, len(fields), "dx")[0], ghost_cells)
            boundary.dirichlet_BC("ALL", 0.0)
        if boundary.inputs[0] != 1:
            raise ValueError("batched heat rollouts take scalar fields")
        self.boundary = boundary
        self._setup(fields, None, dx, alpha, dt, boundary.rules(), ghost_cells, order, tile, steps_per_pass)


class BatchedWaveRollout(_BatchedRollout):
    """Leapfrog wave rollouts of many 2D grids (per-grid constant K = dt^2 c^2) in one launch.

    ``fields`` hold u^n and ``prev`` u^{n-1}; after a call of nsteps they hold
    u^{n+nsteps} and u^{n+nsteps-1}.  Cells outside the Dirichlet node ring are
    zero (the state of ``WaveSolver``)."""
    kind = _lib.PDE_BATCH_WAVE

    def __init__(self, fields: Sequence[torch.Tensor], prev: Sequence[torch.Tensor], dx, K, ghost_cells: int = 1,
                 tile=None, steps_per_pass: int = 0) -> None:
        if len(prev) != len(fields):
            raise ValueError("prev needs one field per grid")
        self._setup(fields, prev, dx, K, 0.0, None, ghost_cells, 2, tile, steps_per_pass)
