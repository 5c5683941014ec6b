"""Divergence module (reference: FDM/module/divergence.py:11-110)."""
from __future__ import annotations

from collections.abc import Iterable

import torch

from .ExplicitUniformGridStencil import ExplicitUniformGridStencil
from ...stencil.hooks import setup
from ..kernel import create_Divergence_kernel
from ..functional import divergence


class Divergence(ExplicitUniformGridStencil):
    """Sum over eligible axes of the central first difference of column ``axis``.

    inputs int (== D): vector input (X,Y,Z,D) -> (X,Y,Z,1);
    inputs (N, D): matrix input (X,Y,Z,N,D) -> (X,Y,Z,N).
    The reference launches its kernel twice per call with the same result;
    this module launches once.
    """

    def __init__(self, inputs, grid_shape, dx: float, ghost_cells: int, stencil=None,
                 float_dtype=torch.float32, order: int = 2, fast: bool = False) -> None:
        if stencil is not None:
            raise ValueError("Custom stencil not implemented yet")
        self.fast = bool(fast)
        dimension = self.calculate_dimension_from_grid_shape(grid_shape)
        is_vector = False
        if isinstance(inputs, Iterable):
            assert all(type(i) is int for i in inputs)
            if len(inputs) == 1:
                inputs = inputs[0]
                is_vector = True
            else:
                assert len(inputs) == 2
        elif type(inputs) is int:
            is_vector = True
        else:
            raise ValueError("Inputs must be int or tuple|list of int")
        if is_vector:
            assert inputs == dimension
            outputs = 1
        else:
            assert inputs[1] == dimension
            outputs = inputs[0]
        self.is_vector = is_vector
        super().__init__(inputs, outputs, dx, ghost_cells, float_dtype=float_dtype, order=order)

    @setup
    def initialize_kernel(self, input_array: torch.Tensor, *args, **kwargs) -> None:
        self.kernel = create_Divergence_kernel(self.outputs[0], input_array.shape, self.dx_value,
                                               self.ghost_cells, self.order,
                                              fast=self.fast)
        self.kernel_dim = self.grid_shape_with_no_ghost_cells(input_array.shape, self.ghost_cells)

    def forward(self, input_array: torch.Tensor, alpha: float = 1.0, *args, **kwargs) -> torch.Tensor:
        return divergence(self.kernel, input_array, alpha, self.ghost_cells, self.output_array,
                          device=self.device)
