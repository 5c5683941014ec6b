"""Stateless launchers with the reference's signatures.

Reference: FDM/functional/_laplacian.py:5-36, _grad.py:5-36,
_divergence.py:4-24 (note its different argument order).  ``kernel`` is a
StencilPlan from ``pde_module_b200.FDM.kernel``.  The launch runs on the
current torch CUDA stream of the input's device; ``device`` is accepted for
signature compatibility.
"""
from __future__ import annotations

import ctypes as C

import torch

from ..._lib import lib, check, stream_ptr, require_cuda_f32, PDE_MODE_EXACT, PDE_MODE_FAST


def _mode(kernel) -> int:
    return PDE_MODE_FAST if getattr(kernel, "fast", False) else PDE_MODE_EXACT


def _check_io(kernel, input_array, output_array, in_trailing, out_trailing):
    require_cuda_f32(input_array, "input_array")
    require_cuda_f32(output_array, "output_array")
    if tuple(input_array.shape[:3]) != tuple(kernel.grid_shape):
        raise AssertionError(f"input grid {tuple(input_array.shape[:3])} does not match the kernel's "
                             f"{tuple(kernel.grid_shape)}")
    if tuple(input_array.shape[3:]) != tuple(in_trailing):
        raise AssertionError(f"input components {tuple(input_array.shape[3:])} != {tuple(in_trailing)}")
    if tuple(output_array.shape) != tuple(kernel.grid_shape) + tuple(out_trailing):
        raise AssertionError(f"output shape {tuple(output_array.shape)} != "
                             f"{tuple(kernel.grid_shape) + tuple(out_trailing)}")
    if input_array.device != output_array.device:
        raise AssertionError("input and output on different devices")


def laplacian(kernel, input_array: torch.Tensor, alpha: float, output_array: torch.Tensor,
              ghost_cells: int, device=None) -> torch.Tensor:
    if ghost_cells != kernel.ghost_cells:
        raise AssertionError("ghost_cells differs from the kernel's")
    _check_io(kernel, input_array, output_array, (kernel.ncomp,), (kernel.ncomp,))
    check(lib().pde_laplacian_ex(C.c_void_p(input_array.data_ptr()), C.c_void_p(output_array.data_ptr()),
                              C.byref(kernel.grid), kernel.ncomp, float(alpha), _mode(kernel),
                              C.c_void_p(stream_ptr(input_array))), "pde_laplacian")
    return output_array


def grad(kernel, input_array: torch.Tensor, alpha: float, output_array: torch.Tensor,
         ghost_cells: int, device=None) -> torch.Tensor:
    if ghost_cells != kernel.ghost_cells:
        raise AssertionError("ghost_cells differs from the kernel's")
    D = kernel.dimension
    out_tr = tuple(output_array.shape[3:])
    if out_tr not in ((kernel.ncomp, D),) and not (kernel.ncomp == 1 and out_tr == (D,)):
        raise AssertionError(f"grad output components {out_tr} do not match ({kernel.ncomp}, {D})")
    _check_io(kernel, input_array, output_array, (kernel.ncomp,), out_tr)
    check(lib().pde_grad_ex(C.c_void_p(input_array.data_ptr()), C.c_void_p(output_array.data_ptr()),
                         C.byref(kernel.grid), kernel.ncomp, float(alpha), _mode(kernel),
                         C.c_void_p(stream_ptr(input_array))), "pde_grad")
    return output_array


def divergence(kernel, input_array: torch.Tensor, alpha: float, ghost_cells: int,
               output_array: torch.Tensor, device=None) -> torch.Tensor:
    if ghost_cells != kernel.ghost_cells:
        raise AssertionError("ghost_cells differs from the kernel's")
    D = kernel.dimension
    in_tr = tuple(input_array.shape[3:])
    if in_tr not in ((kernel.ncomp, D),) and not (kernel.ncomp == 1 and in_tr == (D,)):
        raise AssertionError(f"divergence input components {in_tr} do not match ({kernel.ncomp}, {D})")
    _check_io(kernel, input_array, output_array, in_tr, (kernel.ncomp,))
    check(lib().pde_divergence_ex(C.c_void_p(input_array.data_ptr()), C.c_void_p(output_array.data_ptr()),
                               C.byref(kernel.grid), kernel.ncomp, float(alpha), _mode(kernel),
                               C.c_void_p(stream_ptr(input_array))), "pde_divergence")
    return output_array
