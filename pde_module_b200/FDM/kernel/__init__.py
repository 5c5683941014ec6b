"""Operator plans: the B200 counterpart of the reference's kernel factories.

Reference: FDM/kernel/laplacian.py:7-60, grad.py:8-53, divergence.py:7-45.
The reference specialises a Warp kernel per dtype/shape/stencil; here a plan
records the grid descriptor and component counts that the C ABI needs, and
the kernels themselves are compiled ahead of time for sm_100a.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from .. import _types
from ..._lib import make_grid, PdeGrid


@dataclass
class StencilPlan:
    op: str                 # "laplacian" | "grad" | "divergence"
    grid_shape: tuple       # (X, Y, Z) including ghosts
    ghost_cells: int
    order: int
    dx: float
    ncomp: int              # N of the input vector (rows of a matrix input)
    dimension: int          # number of eligible axes
    fast: bool = False      # PDE_MODE_FAST arithmetic (see include/pde_b200.h)
    grid: PdeGrid = field(repr=False, default=None)

    def __post_init__(self):
        if self.order not in (2, 4):
            raise ValueError("order must be 2 or 4")
        if self.ghost_cells < self.order // 2:
            raise AssertionError("Max shift must be <= ghost cell to avoid out of bounds array access!")
        self.grid = make_grid(self.grid_shape, self.ghost_cells, self.order, self.dx)


def _plan(op, ncomp, grid_shape, dx, ghost_cells, order, fast):
    gs = _types.grid_shape_of(grid_shape)
    return StencilPlan(op, gs, int(ghost_cells), int(order), float(dx), int(ncomp),
                       _types.dimension_of(gs), bool(fast))


def create_Laplacian_kernel(ncomp: int, grid_shape, dx: float, ghost_cells: int, order: int = 2,
                            fast: bool = False) -> StencilPlan:
    return _plan("laplacian", ncomp, grid_shape, dx, ghost_cells, order, fast)


def create_Grad_kernel(ncomp: int, grid_shape, dx: float, ghost_cells: int, order: int = 2,
                       fast: bool = False) -> StencilPlan:
    return _plan("grad", ncomp, grid_shape, dx, ghost_cells, order, fast)


def create_Divergence_kernel(nrows: int, grid_shape, dx: float, ghost_cells: int, order: int = 2,
                             fast: bool = False) -> StencilPlan:
    return _plan("divergence", nrows, grid_shape, dx, ghost_cells, order, fast)
