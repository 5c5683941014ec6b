"""Grad module (reference: FDM/module/grad.py:10-87)."""
from __future__ import annotations

import torch

from .ExplicitUniformGridStencil import ExplicitUniformGridStencil
from ...stencil.hooks import setup
from ..kernel import create_Grad_kernel
from ..functional import grad


class Grad(ExplicitUniformGridStencil):
    """Central first differences along every eligible axis, scaled by alpha.

    inputs == 1 (and not force_matrix): output vec(D) per cell, shape (X,Y,Z,D);
    otherwise mat(N, D), shape (X,Y,Z,N,D), column = axis.
    """

    def __init__(self, inputs: int, grid_shape, dx: float, ghost_cells: int, stencil=None,
                 force_matrix: bool = False, float_dtype=torch.float32, order: int = 2, fast: bool = False) -> None:
        if stencil is not None:
            raise ValueError("Custom stencil not implemented yet")
        self.fast = bool(fast)
        self.force_matrix = force_matrix
        dimension = self.calculate_dimension_from_grid_shape(grid_shape)
        assert type(inputs) is int and inputs > 0
        output_shape = dimension if (inputs == 1 and not force_matrix) else (inputs, dimension)
        assert dimension <= 3
        super().__init__(inputs, output_shape, dx, ghost_cells, float_dtype, order=order)

    @setup
    def initialize_kernel(self, input_array: torch.Tensor, *args, **kwargs) -> None:
        assert len(self.inputs) == 1, "Grad Only For Vectors"
        self.kernel = create_Grad_kernel(self.inputs[0], input_array.shape, self.dx_value, self.ghost_cells,
                                         self.order, fast=self.fast)
        assert self.kernel.dimension == (self.outputs[-1]), "grid dimension differs from the constructor's"
        self.kernel_dim = self.grid_shape_with_no_ghost_cells(input_array.shape, self.ghost_cells)

    def forward(self, input_array: torch.Tensor, alpha: float = 1.0) -> torch.Tensor:
        return grad(self.kernel, input_array, alpha, self.output_array, self.ghost_cells, device=self.device)
