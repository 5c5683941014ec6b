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


class HeatSolver:
    """Differentiable 2D heat rollout with a per-cell diffusivity field.

    New: the reference steps the heat equation forward only
    (examples/2D_Heat_Equation.py:57-65, scalar alpha).  Step, on a scalar
    (X, Y, 1, 1) field with the boundary groups of ``boundary``:

        v = BC(u);  S = Lap(v);  u' = v + dt * (alpha o S)    (stencil cells; v elsewhere)

    which is the module chain's step with alpha taken per cell (bit-identical to
    ``HeatRollout`` for a constant field).  ``forward`` keeps ceil(sqrt(N))
    checkpoints of u; ``backward`` recomputes each segment's S from its checkpoint
    (the last segment keeps them from the forward pass) and runs the discrete
    adjoint, returning (dJ/dalpha, dJ/du0)."""

    def __init__(self, boundary: GridBoundary, dx: float, dt: float, nsteps: int, order: int = 2,
                 steps_per_pass: int = 0, checkpoint_every: int | None = None) -> None:
        import math
        if boundary.inputs[0] != 1:
            raise ValueError("HeatSolver takes scalar fields")
        self.boundary = boundary
        self.shape = tuple(boundary.grid_shape)
        assert self.shape[2] == 1 and self.shape[0] > 1 and self.shape[1] > 1, "2D grids (X, Y, 1)"
        self.dx, self.dt, self.N, self.order = float(dx), float(dt), int(nsteps), int(order)
        self.rules = boundary.rules()
        self.grid = make_grid(self.shape, boundary.ghost_cells, self.order, self.dx)
        self.steps_per_pass = int(steps_per_pass)
        self.every = int(checkpoint_every) if checkpoint_every else max(1, int(math.ceil(math.sqrt(self.N))))
        self.checkpoints = []
        self._work = None
        self._last_seg_ready = False

    def _buffers(self, like: torch.Tensor) -> None:
        if self._work is None or self._work.device != like.device:
            cells = self.shape[0] * self.shape[1]
            self._work = torch.zeros(cells, dtype=torch.float32, device=like.device)
            self._seg = torch.zeros((self.every, cells), dtype=torch.float32, device=like.device)

    def _fwd(self, alpha, u, out, nsteps, lstates=None):
        check(lib().pde_heat_forward(C.c_void_p(alpha.data_ptr()), C.c_void_p(u.data_ptr()),
                                     C.c_void_p(out.data_ptr()), C.c_void_p(self._work.data_ptr()),
                                     C.byref(self.grid), C.byref(self.rules), self.dt, int(nsteps),
                                     self.steps_per_pass,
                                     C.c_void_p(lstates.data_ptr()) if lstates is not None else None,
                                     C.c_void_p(stream_ptr(u))), "pde_heat_forward")

    def _check(self, alpha, u):
        require_cuda_f32(alpha, "alpha")
        require_cuda_f32(u, "u")
        if tuple(alpha.shape) != self.shape + (1,) or tuple(u.shape) != self.shape + (1,):
            raise AssertionError(f"alpha and u must be {self.shape + (1,)}")

    def forward(self, alpha: torch.Tensor, u0: torch.Tensor) -> torch.Tensor:
        """u^N; keeps u at n = 0, every, 2*every, ... and the last segment's S."""
        self._check(alpha, u0)
        self._buffers(u0)
        self.checkpoints = []
        self._last_seg_ready = False
        cur, n = u0, 0
        while n < self.N:
            self.checkpoints.append((n, cur.clone()))
            m = min(self.every, self.N - n)
            out = torch.empty_like(cur)
            last = n + m == self.N
            self._fwd(alpha, cur, out, m, self._seg[:m] if last else None)
            self._last_seg_ready = last
            cur, n = out, n + m
        if self.N == 0:
            cur = u0.clone()
        return cur

    def backward(self, alpha: torch.Tensor, dJ_duN: torch.Tensor):
        """(dJ/dalpha, dJ/du0) for the last forward()."""
        lam = dJ_duN.contiguous()
        self._check(alpha, lam)
        self._buffers(alpha)
        galpha = torch.zeros_like(alpha)
        kept, self._last_seg_ready = self._last_seg_ready, False
        scratch = torch.empty_like(lam)
        for n0, u in reversed(self.checkpoints):
            m = min(self.every, self.N - n0)
            seg = self._seg[:m]
            if not (kept and n0 + m == self.N):
                self._fwd(alpha, u, scratch, m, seg)  # recompute S^{n0} .. S^{n0+m-1}
            out = torch.empty_like(lam)
            check(lib().pde_heat_adjoint(C.c_void_p(alpha.data_ptr()), C.c_void_p(lam.data_ptr()),
                                         C.c_void_p(out.data_ptr()), C.c_void_p(seg.data_ptr()),
                                         C.c_void_p(galpha.data_ptr()), C.byref(self.grid), C.byref(self.rules),
                                         self.dt, m, self.steps_per_pass, C.c_void_p(self._work.data_ptr()),
                                         C.c_void_p(stream_ptr(lam))), "pde_heat_adjoint")
            lam = out
        return galpha, lam.clone() if lam is dJ_duN else lam


class _HeatFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, alpha, u0, solver):
        ctx.solver = solver
        ctx.save_for_backward(alpha)
        return solver.forward(alpha.detach().contiguous(), u0.detach().contiguous())

    @staticmethod
    def backward(ctx, g):
        (alpha,) = ctx.saved_tensors
        ga, gu = ctx.solver.backward(alpha.detach().contiguous(), g.contiguous())
        return ga, gu, None


def heat_rollout(alpha: torch.Tensor, u0: torch.Tensor, solver: HeatSolver) -> torch.Tensor:
    """u^N as a differentiable function of the diffusivity field alpha and u0
    (a scalar alpha can be broadcast: ``alpha_s.expand(shape)`` sums its gradient)."""
    return _HeatFn.apply(alpha, u0, solver)
