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
                 dt: float | None = None, lid_ramp_time: float | None = None) -> None:
        """lid_ramp_time: the lid speed ramps from 0 to ``lid`` over this time
        (boundary_functions.py:77-92), as the reference's function-BC cavity
        does (Benchmark/Functional_BC/LDC_Graph Function.py:44-113); step n fills
        its boundaries at t = n*dt from the first step of this solver."""
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
        if lid_ramp_time:
            from ..FDM.boundary import get_ramp_func
            self.u_bc.dirichlet_BC("+Y", get_ramp_func(self.lid, float(lid_ramp_time), output_ids=(0,)), 0)
        else:
            self.u_bc.dirichlet_BC("+Y", self.lid, 0)
        self.p_bc = GridBoundary(self.p, self.dx, g)
        self.p_bc.vonNeumann_BC("ALL", 0.0)
        self.params = PdeLDCParams(self.nu, self.dt, int(jacobi_iters), int(jacobi_per_pass))
        self.steps_done = 0
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
        args = [C.c_void_p(self.u.data_ptr()), C.c_void_p(self.p.data_ptr()), C.c_void_p(self._u_star.data_ptr()),
                C.c_void_p(self._p_tmp.data_ptr()), C.c_void_p(self._rhs.data_ptr()), rp, C.byref(self.grid),
                C.byref(self.u_bc.rules()), C.byref(self.p_bc.rules()), C.byref(self.params), int(nsteps)]
        if self.u_bc.time_dependent:
            check(lib().pde_ldc_rollout_at(*args, self.steps_done * self.dt, self.dt, C.c_void_p(stream_ptr(self.u))),
                  "pde_ldc_rollout_at")
        else:
            check(lib().pde_ldc_rollout(*args, C.c_void_p(stream_ptr(self.u))), "pde_ldc_rollout")
        self.steps_done += int(nsteps)
        return self.u, self.p


# ---- the cavity split into slabs along X (one per GPU) ----------------------------
def slab_rows(x_global: int, world: int, halo: int, ghost: int = 1) -> list[tuple[int, int, int, int]]:
    """(own_lo, own_hi, held_lo, held_hi) of each of `world` slabs: contiguous blocks of
    the domain's rows (ghosts included) and `halo` more rows on each cut side."""
    out = []
    for r in range(world):
        lo, hi = r * x_global // world, (r + 1) * x_global // world
        out.append((lo, hi, max(lo - halo, 0), min(hi + halo, x_global)))
    for r, (lo, hi, _, _) in enumerate(out):
        if world > 1 and hi - lo < max(halo, ghost + 2):
            raise ValueError(f"slab {r} owns {hi - lo} rows: at least {max(halo, ghost + 2)} needed")
    return out


class LDCSlab:
    """One slab of the cavity of FractionalStepLDC (same parameters): owned rows
    [own_lo, own_hi) of the (n+2g)^2 domain plus halo rows on its cut sides.  Each
    method runs one phase of a fractional step on this slab (pde_ldc_slab_step); a
    host fills the halo rows between phases (``ldc_slab_steps``)."""

    def __init__(self, rows, n: int = 1024, Re: float = 100.0, lid: float = 1.0, cfl: float = 0.2,
                 jacobi_iters: int = 50, jacobi_per_pass: int = 0, ghost_cells: int = 1, device="cuda",
                 dt: float | None = None) -> None:
        from .. import _lib
        g = int(ghost_cells)
        self.n, self.g = int(n), g
        self.dx = 1.0 / (n - 1)
        self.lid = float(lid)
        self.nu = lid * 1.0 / Re
        self.dt = float(dt) if dt is not None else cfl * min(self.dx / max(abs(lid), 1e-30),
                                                               self.dx * self.dx / (4.0 * self.nu))
        self.own_lo, self.own_hi, self.held_lo, self.held_hi = (int(v) for v in rows)
        X = n + 2 * g
        nloc = self.held_hi - self.held_lo
        shape = (nloc, X, 1)
        z = lambda c: torch.zeros(shape + (c,), dtype=torch.float32, device=device)
        self.u, self.u_star, self.p, self.p_tmp, self.rhs = z(2), z(2), z(1), z(1), z(1)
        # boundary rules of the whole domain (face groups: the same for every slab)
        whole_u = torch.zeros((X, X, 1, 2))
        self.u_bc = GridBoundary(whole_u, self.dx, g)
        self.u_bc.dirichlet_BC("ALL", 0.0)
        self.u_bc.dirichlet_BC("+Y", self.lid, 0)
        self.p_bc = GridBoundary(whole_u[..., :1], self.dx, g)
        self.p_bc.vonNeumann_BC("ALL", 0.0)
        self._u_rules, self._p_rules = self.u_bc.rules(), self.p_bc.rules()
        self.params = PdeLDCParams(self.nu, self.dt, int(jacobi_iters), int(jacobi_per_pass))
        self.grid = make_grid(shape, g, 2, self.dx)
        self.slab = _lib.PdeSlab(X, self.held_lo, self.own_lo, self.own_hi)
        self.resid = torch.zeros(1, dtype=torch.float32, device=device)

    @property
    def owned(self) -> slice:
        """Local rows of the owned block."""
        return slice(self.own_lo - self.held_lo, self.own_hi - self.held_lo)

    def _phase(self, phase, p_in=None, p_out=None, nsweeps=0, last=False, resid=False):
        P = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        check(lib().pde_ldc_slab_step(phase, P(self.u), P(self.u_star), P(p_in), P(p_out), P(self.rhs),
                                      P(self.resid) if resid else None, C.byref(self.grid), C.byref(self.slab),
                                      C.byref(self._u_rules), C.byref(self._p_rules), C.byref(self.params),
                                      int(nsweeps), int(bool(last)), C.c_void_p(stream_ptr(self.u))),
              "pde_ldc_slab_step")

    def predict(self):
        from .. import _lib
        self._phase(_lib.PDE_LDC_PREDICT)

    def divergence(self):
        from .. import _lib
        self._phase(_lib.PDE_LDC_DIVERGENCE)

    def jacobi(self, nsweeps: int, last: bool, residual: bool = False):
        """nsweeps sweeps from p into p_tmp, then the two are swapped."""
        from .. import _lib
        self._phase(_lib.PDE_LDC_JACOBI, self.p, self.p_tmp, nsweeps, last, residual)
        self.p, self.p_tmp = self.p_tmp, self.p

    def project(self):
        from .. import _lib
        self._phase(_lib.PDE_LDC_PROJECT, self.p)


def ldc_slab_steps(slabs, nsteps: int, exchange, residuals: bool = False) -> None:
    """Advance the slabs of one cavity nsteps fractional steps.  ``exchange(fields)``
    fills the halo rows of the listed fields (one per slab, in slab order) from the
    neighbouring slabs: ``exchange_slab_halos`` across ranks, ``exchange_local_slabs``
    for several slabs in one process.  With residuals, each slab's ``resid`` holds the
    sum of squared pressure updates of its owned cells over the last step's last sweep."""
    s0 = slabs[0]
    iters = s0.params.jacobi_iters
    k = s0.params.jacobi_per_pass or 10
    for _ in range(nsteps):
        if residuals:
            for s in slabs:
                s.resid.zero_()
        exchange([s.u for s in slabs])
        for s in slabs:
            s.predict()
        exchange([s.u_star for s in slabs])
        for s in slabs:
            s.divergence()
        exchange([s.rhs for s in slabs])
        done = 0
        while done < iters:
            kk = min(k, iters - done)
            done += kk
            exchange([s.p for s in slabs])
            for s in slabs:
                s.jacobi(kk, done == iters, residuals)
        exchange([s.p for s in slabs])
        for s in slabs:
            s.project()


class SlabFractionalStepLDC:
    """FractionalStepLDC split across the ranks of a process group (one slab of rows
    per rank, one GPU per rank): halo rows are exchanged between phases with
    point-to-point send/recv (NCCL over NVLink), the residual summed with all_reduce."""

    def __init__(self, n: int = 1024, Re: float = 100.0, jacobi_iters: int = 50, jacobi_per_pass: int = 0,
                 group=None, device="cuda", **kw) -> None:
        import torch.distributed as dist
        from ..distributed import exchange_slab_halos
        self.group = group
        world, rank = dist.get_world_size(group), dist.get_rank(group)
        k = jacobi_per_pass or 10
        self.halo = k + 1
        rows = slab_rows(n + 2, world, self.halo)[rank]
        self.slab = LDCSlab(rows, n=n, Re=Re, jacobi_iters=jacobi_iters, jacobi_per_pass=jacobi_per_pass,
                            device=device, **kw)
        self._exchange = lambda fields: exchange_slab_halos(fields[0], self.halo, periodic=False, group=group)

    def step(self, nsteps: int = 1, residuals: bool = False):
        import torch.distributed as dist
        ldc_slab_steps([self.slab], nsteps, self._exchange, residuals)
        if residuals:
            dist.all_reduce(self.slab.resid, group=self.group)
        return self.slab.u, self.slab.p
