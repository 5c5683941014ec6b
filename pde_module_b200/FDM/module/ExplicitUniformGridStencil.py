"""Base of the explicit uniform-grid operators (reference:
FDM/module/ExplicitUniformGridStencil.py:9-179).

Fields are torch CUDA float32 tensors laid out like the reference's Warp
``array3d(dtype=vec(N))`` / ``mat(N, D)``: shape (X, Y, Z, N) or
(X, Y, Z, N, D), C-contiguous, ghosts included, Z == 1 for 2D grids.
"""
from __future__ import annotations

import numpy as np
import torch

from ...stencil.stencil import Stencil, tuplify
from ...stencil.hooks import setup
from ..._lib import require_cuda_f32
from .._types import check_float_dtype, dimension_of, grid_shape_of


class ExplicitUniformGridStencil(Stencil):
    output_array: torch.Tensor | None = None

    def __init__(self, inputs, outputs, dx: float, ghost_cells: int = 0, float_dtype=torch.float32,
                 order: int = 2) -> None:
        super().__init__()
        check_float_dtype(float_dtype)
        if order not in (2, 4):
            raise ValueError("order must be 2 or 4")
        self.dx_value = float(dx)            # Python float: stencil weights are formed from it
        self.dx = np.float32(dx)             # the fp32 dx the reference stores (:27)
        self._inputs = tuplify(inputs)
        self._outputs = tuplify(outputs)
        self.ghost_cells = int(ghost_cells)
        self.order = int(order)
        self.float_dtype = torch.float32

    @property
    def inputs(self) -> tuple:
        assert 1 <= len(self._outputs) <= 2, "AoS stencils input/output can be either vec or matrix"
        return self._inputs

    @property
    def outputs(self) -> tuple:
        assert 1 <= len(self._outputs) <= 2, "AoS stencils input/output can be either vec or matrix"
        return self._outputs

    @property
    def input_dtype_shape(self) -> tuple:
        return self.inputs

    @property
    def output_dtype_shape(self) -> tuple:
        return self.outputs

    @staticmethod
    def calculate_dimension_from_grid_shape(shape) -> int:
        return dimension_of(shape)

    @staticmethod
    def grid_shape_with_no_ghost_cells(grid_shape, ghost_cells: int) -> tuple:
        return tuple(a - 2 * ghost_cells if a > 1 else a for a in grid_shape_of(grid_shape))

    @staticmethod
    def get_ghost_shape(grid_shape, ghost_cells: int) -> tuple:
        return tuple(a + 2 * ghost_cells if a > 1 else a for a in grid_shape_of(grid_shape))

    def check_input(self, input_array: torch.Tensor) -> None:
        require_cuda_f32(input_array, "input_array")
        assert tuple(input_array.shape[3:]) == tuple(self.inputs), (
            f"input components {tuple(input_array.shape[3:])} != {tuple(self.inputs)}")

    @setup(order=-1)
    def initialize_array(self, input_array: torch.Tensor, *args, **kwargs) -> None:
        self.check_input(input_array)
        self.device = input_array.device
        self.output_array = self.create_output_array(input_array, self.outputs)

    def forward(self, input_array, *args, **kwargs):
        raise NotImplementedError()
