"""Weakly compressible flow with RK2 time stepping, one fused launch per step.

New: the reference builds this solver in its example examples/LDC/LDC_RK2.py from
its modules (GridBoundary, Laplacian, Grad, Divergence, OuterProduct,
scalarVectorMult, MapWise, RungeKatta2), about forty launches per step.  Here
``pde_wc_rk2`` runs a whole step in one kernel per tile, bit-identical to that
composition of this package's modules (tests/test_wc_gpu.py):

    bc(m, rho) = (rho' u', rho'),  u = m / rho,  u' = BC_u(u),  rho' = BC_rho(rho)
    f(m, rho)  = (((Grad(c2 (rho - rho0), -1) - Div(outer(m, u))) + Lap(u, nu)) + Lap(Lap(u, nu), eps),
                  Div(m, -1))
    y0 = bc(y);  y1 = bc(y0 + dt/2 f(y0));  y' = y0 + dt f(y1)

Fields: momentum m (X, Y, 1, 2) and density rho (X, Y, 1, 1).
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from .._lib import lib, check, stream_ptr, require_cuda_f32, make_grid
from .. import _lib
from ..FDM.boundary import GridBoundary


class WeaklyCompressibleRK2:
    def __init__(self, u_bc: GridBoundary, rho_bc: GridBoundary, dx: float, nu: float, c2: float, rho0: float,
                 damping_eps: float, dt: float) -> None:
        if u_bc.inputs[0] != 2 or rho_bc.inputs[0] != 1:
            raise ValueError("velocity boundary with 2 components, density boundary with 1")
        if u_bc.grid_shape != rho_bc.grid_shape or u_bc.grid_shape[2] != 1:
            raise ValueError("one 2D grid (X, Y, 1) for both boundaries")
        if u_bc.time_dependent or rho_bc.time_dependent:
            raise NotImplementedError("constant-valued boundary groups")
        self.shape = tuple(u_bc.grid_shape)
        self.u_rules, self.rho_rules = u_bc.rules(), rho_bc.rules()
        self.grid = make_grid(self.shape, u_bc.ghost_cells, 2, float(dx))
        self.params = _lib.PdeWCParams(float(nu), float(damping_eps), float(c2), float(rho0), float(dt))
        self.dt = float(dt)
        self.m_out = self.rho_out = self._work = None

    def __call__(self, m: torch.Tensor, rho: torch.Tensor, nsteps: int = 1):
        """Advance (m, rho) by nsteps; returns the module's own output tensors."""
        require_cuda_f32(m, "m")
        require_cuda_f32(rho, "rho")
        if tuple(m.shape) != self.shape + (2,) or tuple(rho.shape) != self.shape + (1,):
            raise AssertionError("fields must be (X, Y, 1, 2) and (X, Y, 1, 1) on the boundaries' grid")
        if self.m_out is None:
            self.m_out, self.rho_out = torch.zeros_like(m), torch.zeros_like(rho)
            self._work = torch.zeros(3 * self.shape[0] * self.shape[1], dtype=torch.float32, device=m.device)
        check(lib().pde_wc_rk2(C.c_void_p(m.data_ptr()), C.c_void_p(rho.data_ptr()),
                               C.c_void_p(self.m_out.data_ptr()), C.c_void_p(self.rho_out.data_ptr()),
                               C.byref(self.grid), C.byref(self.u_rules), C.byref(self.rho_rules),
                               C.byref(self.params), int(nsteps), C.c_void_p(self._work.data_ptr()),
                               C.c_void_p(stream_ptr(m))), "pde_wc_rk2")
        return self.m_out, self.rho_out


def lid_driven_cavity_wc(n: int = 201, Re: float = 100.0, M: float = 0.1, cfl: float = 0.8, U: float = 1.0,
                         rho0: float = 1.0, device="cuda"):
    """The weakly compressible cavity of examples/LDC/LDC_RK2.py: n x n nodes on the
    unit square (one ghost layer), lid speed U on +Y, no-slip elsewhere, zero-gradient
    density, sound speed U / M, dt from the viscous, convective and acoustic limits
    at the given CFL number, biharmonic damping -0.01 dx^4 / (dt nu).
    Returns (solver, m, rho) with the fluid at rest (rho = rho0, m = 0)."""
    dx = 1.0 / (n - 1)
    nu = U * 1.0 / Re
    cs = U / M
    dt = min(cfl * dx * dx / nu, cfl * dx / cs, cfl * dx / (cs + U))
    eps = -0.01 * (math.exp(4 * math.log(dx) - math.log(dt)) / nu)
    shape = (n + 2, n + 2, 1)
    m = torch.zeros(shape + (2,), dtype=torch.float32, device=device)
    rho = torch.full(shape + (1,), float(rho0), dtype=torch.float32, device=device)
    u_bc = GridBoundary(m, dx, 1)
    u_bc.dirichlet_BC("ALL", 0.0)
    u_bc.dirichlet_BC("+Y", U, 0)
    rho_bc = GridBoundary(rho, dx, 1)
    rho_bc.vonNeumann_BC("ALL", 0.0)
    return WeaklyCompressibleRK2(u_bc, rho_bc, dx, nu, cs * cs, rho0, eps, dt), m, rho
