"""Laplacian module (reference: FDM/module/laplacian.py:10-72)."""
from __future__ import annotations

import torch

from .ExplicitUniformGridStencil import ExplicitUniformGridStencil
from ...stencil.hooks import setup
from ..kernel import create_Laplacian_kernel
from ..functional import laplacian


class Laplacian(ExplicitUniformGridStencil):
    """alpha * (sum over eligible axes of the central second difference), per component.

    Args mirror the reference: inputs (vector length N), dx, ghost_cells,
    stencil (custom stencils raise ValueError, as in the reference),
    float_dtype (float32 only).  ``order=4`` selects the 5-point
    (-1, 16, -30, 16, -1)/(12 dx^2) stencil (needs ghost_cells >= 2).
    """

    def __init__(self, inputs: int, dx: float, ghost_cells: int, stencil=None, float_dtype=torch.float32,
                 order: int = 2, fast: bool = False) -> None:
        if stencil is not None:
            raise ValueError("Custom stencil not implemented yet")
        self.fast = bool(fast)
        super().__init__(inputs, inputs, dx, ghost_cells, float_dtype=float_dtype, order=order)

    @setup
    def initialize_kernel(self, input_array: torch.Tensor, *args, **kwargs) -> None:
        assert len(self.inputs) == 1, "Laplacian Only For Vectors"
        self.kernel = create_Laplacian_kernel(self.inputs[0], input_array.shape, self.dx_value,
                                              self.ghost_cells, self.order,
                                              fast=self.fast)
        self.kernel_dim = self.grid_shape_with_no_ghost_cells(input_array.shape, self.ghost_cells)

    def forward(self, input_array: torch.Tensor, alpha: float = 1.0, *args, **kwargs) -> torch.Tensor:
        return laplacian(self.kernel, input_array, alpha, self.output_array, self.ghost_cells, device=self.device)
