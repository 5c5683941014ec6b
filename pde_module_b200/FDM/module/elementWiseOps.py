"""Cell-by-cell products of two fields (reference: FDM/module/elementWiseOps.py:10-88
on stencil/elementWise.py:6-49).

``OuterProduct(na, nb)(A, B)``: vec(na), vec(nb) fields -> mat(na, nb) field with
M[i, j] = A[i] * B[j]; ``scalarVectorMult(outputs)(a, B)``: a vec(1) field times a
vector or matrix field.  One rounding per product, as the reference's kernels;
outputs are the modules' own preallocated tensors.
"""
from __future__ import annotations

import ctypes as C

import torch

from ...stencil.stencil import Stencil
from ...stencil.hooks import setup
from ..._lib import lib, check, stream_ptr, require_cuda_f32


class _ElementWise(Stencil):
    def _check_pair(self, A: torch.Tensor, B: torch.Tensor) -> None:
        require_cuda_f32(A, "array_A")
        require_cuda_f32(B, "array_B")
        assert tuple(A.shape[:3]) == tuple(B.shape[:3]), "input arrays must be the same Shape!"


class OuterProduct(_ElementWise):
    def __init__(self, vec_A: int, vec_B: int, float_dtype=torch.float32) -> None:
        super().__init__()
        self.vec_A, self.vec_B = int(vec_A), int(vec_B)

    @setup
    def initialize_kernel(self, array_A: torch.Tensor, array_B: torch.Tensor, *args, **kwargs) -> None:
        self._check_pair(array_A, array_B)
        # the reference checks both inputs against vec_A (elementWiseOps.py:25-30)
        assert tuple(array_A.shape[3:]) == (self.vec_A,) and tuple(array_B.shape[3:]) == (self.vec_A,)
        self.device = array_A.device
        self.output_array = self.create_output_array(array_A, (self.vec_A, self.vec_B))

    def forward(self, array_A: torch.Tensor, array_B: torch.Tensor, *args, **kwargs) -> torch.Tensor:
        self._check_pair(array_A, array_B)
        cells = array_A.shape[0] * array_A.shape[1] * array_A.shape[2]
        check(lib().pde_outer(C.c_void_p(array_A.data_ptr()), C.c_void_p(array_B.data_ptr()),
                              C.c_void_p(self.output_array.data_ptr()), cells, self.vec_A, self.vec_B,
                              C.c_void_p(stream_ptr(array_A))), "pde_outer")
        return self.output_array


class scalarVectorMult(_ElementWise):
    def __init__(self, outputs, float_dtype=torch.float32) -> None:
        super().__init__()
        self.outputs = (int(outputs),) if isinstance(outputs, int) else tuple(int(o) for o in outputs)
        assert 1 <= len(self.outputs) <= 2

    @setup
    def initialize_kernel(self, array_A: torch.Tensor, array_B: torch.Tensor, *args, **kwargs) -> None:
        self._check_pair(array_A, array_B)
        assert tuple(array_A.shape[3:]) == (1,) and tuple(array_B.shape[3:]) == self.outputs
        self.device = array_A.device
        self.output_array = self.create_output_array(array_B)

    def forward(self, array_A: torch.Tensor, array_B: torch.Tensor, *args, **kwargs) -> torch.Tensor:
        self._check_pair(array_A, array_B)
        cells = array_A.shape[0] * array_A.shape[1] * array_A.shape[2]
        nb = array_B.numel() // max(cells, 1)
        check(lib().pde_scalar_mult(C.c_void_p(array_A.data_ptr()), C.c_void_p(array_B.data_ptr()),
                                    C.c_void_p(self.output_array.data_ptr()), cells, nb,
                                    C.c_void_p(stream_ptr(array_A))), "pde_scalar_mult")
        return self.output_array
