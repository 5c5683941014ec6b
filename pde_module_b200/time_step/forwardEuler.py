"""Forward Euler step (reference: time_step/forwardEuler.py:9-81).

new = current + dt * stencil, element by element over the whole array (ghost
cells included), into the module's preallocated output.
"""
from __future__ import annotations

import ctypes as C

import torch

from ..stencil.stencil import Stencil
from ..stencil.hooks import setup
from .._lib import lib, check, stream_ptr, require_cuda_f32


class ForwardEuler(Stencil):
    def __init__(self, *args, **kwargs) -> None:
        # The reference examples construct it as ForwardEuler(u.dtype); arguments are ignored.
        super().__init__()

    @setup
    def initialize_kernel(self, input_array: torch.Tensor, stencil_values: torch.Tensor, dt: float) -> None:
        require_cuda_f32(input_array, "input_array")
        require_cuda_f32(stencil_values, "stencil_values")
        self.device = input_array.device
        self.output_array = torch.zeros_like(input_array)
        self.size = input_array.numel()
        assert input_array.shape == stencil_values.shape == self.output_array.shape

    def forward(self, input_array: torch.Tensor, stencil_values: torch.Tensor, dt: float) -> torch.Tensor:
        if input_array.shape != self.output_array.shape or stencil_values.shape != self.output_array.shape:
            raise AssertionError("ForwardEuler: shapes differ from the first call's")
        require_cuda_f32(input_array, "input_array")
        require_cuda_f32(stencil_values, "stencil_values")
        check(lib().pde_euler(C.c_void_p(input_array.data_ptr()), C.c_void_p(stencil_values.data_ptr()), float(dt),
                              C.c_void_p(self.output_array.data_ptr()), self.size,
                              C.c_void_p(stream_ptr(input_array))), "pde_euler")
        return self.output_array
