"""Fractional-step (projection) solver for the 2D lid-driven cavity.

Composed of the reference's operators as its LDC examples use them
(examples/LDC/LDC_Graph_Capture.py:53-68: velocity boundary ALL Dirichlet 0 then
the lid '+Y' component 0 = U; pressure ALL Von Neumann 0) with a Jacobi
pressure-Poisson solve and a projection, which the reference does not have (its
cavity uses artificial compressibility).  One step, in float32:

    u2 = BC_u(u);  u* = u2 + dt*(nu*Laplacian(u2) - Grad(u2) u2)
    rhs = (1/dt) * Divergence(BC_u(u*))
    jacobi_iters sweeps: p <- (pW + pE + pS + pN - dx^2 rhs) / 4   on BC_p(p)
    u = BC_u(u*) + dt * Grad(BC_p(p), -1)

run by fused sm_100a kernels (predictor, divergence, temporally blocked Jacobi
sweeps with a warp-shuffle residual, projection), bit-identical to that
composition of the operators.
"""
from __future__ import annotations

import ctypes as C

import torch

from .._lib import lib, check, stream_ptr, make_grid, PdeLDCParams
from ..FDM.boundary import GridBoundary


class FractionalStepLDC:
    def __init__(self, n: int = 1024, Re: float = 100.0, lid: float = 1.0, cfl: float = 0.2,
                 jacobi_iters: int = 50, jacobi_per_pass: int = 0, ghost_cells: int = 1, device="cuda",
                 dt: float | None = None) -> None:
        g = int(ghost_cells)
        self.n, self.g = int(n), g
        self.dx = 1.0 / (n - 1)            # node-centred, n nodes from 0 to 1
        self.lid = float(lid)
        self.nu = lid * 1.0 / Re           # L = U = 1
        self.dt = float(dt) if dt is not None else cfl * min(self.dx / max(abs(lid), 1e-30),
                                                               self.dx * self.dx / (4.0 * self.nu))
        shape = (n + 2 * g, n + 2 * g, 1)
        self.u = torch.zeros(shape + (2,), dtype=torch.float32, device=device)
        self.p = torch.zeros(shape + (1,), dtype=torch.float32, device=device)
        self.u_bc = GridBoundary(self.u, self.dx, g)
        self.u_bc.dirichlet_BC("ALL", 0.0)
        self.u_bc.dirichlet_BC("+Y", self.lid, 0)
        self.p_bc = GridBoundary(self.p, self.dx, g)
        self.p_bc.vonNeumann_BC("ALL", 0.0)
        self.params = PdeLDCParams(self.nu, self.dt, int(jacobi_iters), int(jacobi_per_pass))
        self.grid = make_grid(shape, g, 2, self.dx)
        self._u_star = torch.zeros_like(self.u)
        self._p_tmp = torch.zeros_like(self.p)
        self._rhs = torch.zeros_like(self.p)
        self.residuals = None

    @property
    def jacobi_per_pass(self) -> int:
        return self.params.jacobi_per_pass

    @jacobi_per_pass.setter
    def jacobi_per_pass(self, k: int) -> None:
        self.params.jacobi_per_pass = int(k)

    def step(self, nsteps: int = 1, residuals: bool = False):
        """Advance nsteps; returns (u, p).  With residuals=True, self.residuals holds
        each step's sum of squared pressure updates over its last Jacobi sweep."""
        rp = None
        if residuals:
            if self.residuals is None or self.residuals.numel() < nsteps:
                self.residuals = torch.zeros(max(nsteps, 1), dtype=torch.float32, device=self.u.device)
            rp = C.c_void_p(self.residuals.data_ptr())
        check(lib().pde_ldc_rollout(C.c_void_p(self.u.data_ptr()), C.c_void_p(self.p.data_ptr()),
                                    C.c_void_p(self._u_star.data_ptr()), C.c_void_p(self._p_tmp.data_ptr()),
                                    C.c_void_p(self._rhs.data_ptr()), rp, C.byref(self.grid),
                                    C.byref(self.u_bc.rules()), C.byref(self.p_bc.rules()), C.byref(self.params),
                                    int(nsteps), C.c_void_p(stream_ptr(self.u))), "pde_ldc_rollout")
        return self.u, self.p
