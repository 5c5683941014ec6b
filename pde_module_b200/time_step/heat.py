"""Fused heat-equation rollout: boundary fill + Laplacian + forward Euler.

Runs ``nsteps`` of the reference's explicit step (examples/2D_Heat_Equation.py:57-65)

    u2 = BC(u);  lap = Laplacian(u2, alpha);  u = ForwardEuler(u2, lap, dt)

in fused sm_100a kernels: 2D grids advance k steps per pass out of shared-memory
tiles (temporal blocking), 3D grids one fused step per pass.  The result is
bit-identical to running the three modules of this package step by step (the
Laplacian module's ghost cells are zero, so Euler copies the boundary-filled
ghosts through).
"""
from __future__ import annotations

import ctypes as C

import torch

from .._lib import lib, check, stream_ptr, require_cuda_f32, make_grid
from ..FDM.boundary import GridBoundary


class HeatRollout:
    def __init__(self, boundary: GridBoundary, dx: float, alpha: float, dt: float, order: int = 2,
                 steps_per_pass: int = 0) -> None:
        self.boundary = boundary
        self.dx = float(dx)
        self.alpha = float(alpha)
        self.dt = float(dt)
        self.order = int(order)
        self.steps_per_pass = int(steps_per_pass)
        self.rules = boundary.rules()
        self.grid = make_grid(boundary.grid_shape, boundary.ghost_cells, self.order, self.dx)
        self.ncomp = boundary.inputs[0]
        self.output_array = None
        self.work = None

    def __call__(self, u: torch.Tensor, nsteps: int) -> torch.Tensor:
        require_cuda_f32(u, "u")
        if tuple(u.shape) != tuple(self.boundary.grid_shape) + (self.ncomp,):
            raise AssertionError(f"field shape {tuple(u.shape)} does not match the boundary's grid")
        if self.output_array is None:
            self.output_array = torch.zeros_like(u)
            self.work = torch.zeros_like(u)
        check(lib().pde_heat_rollout(C.c_void_p(u.data_ptr()), C.c_void_p(self.output_array.data_ptr()),
                                     C.c_void_p(self.work.data_ptr()), C.byref(self.grid), self.ncomp,
                                     C.byref(self.rules), self.alpha, self.dt, int(nsteps), self.steps_per_pass,
                                     C.c_void_p(stream_ptr(u))), "pde_heat_rollout")
        return self.output_array
