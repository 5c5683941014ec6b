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
from ._replay import GraphedSequence


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

    def __call__(self, u: torch.Tensor, nsteps: int, t0: float = 0.0) -> torch.Tensor:
        """Advance ``nsteps``; step n fills the boundary at time t0 + n*dt (only
        ramp groups depend on it), as the loop ``u2 = bc(u, t0 + n*dt)`` does."""
        require_cuda_f32(u, "u")
        if tuple(u.shape) != tuple(self.boundary.grid_shape) + (self.ncomp,):
            raise AssertionError(f"field shape {tuple(u.shape)} does not match the boundary's grid")
        if self.output_array is None:
            self.output_array = torch.zeros_like(u)
            self.work = torch.zeros_like(u)
        args = [C.c_void_p(u.data_ptr()), C.c_void_p(self.output_array.data_ptr()), C.c_void_p(self.work.data_ptr()),
                C.byref(self.grid), self.ncomp, C.byref(self.rules), self.alpha, self.dt, int(nsteps),
                self.steps_per_pass]
        if self.rules.has_ramp:
            check(lib().pde_heat_rollout_at(*args, float(t0), self.dt, C.c_void_p(stream_ptr(u))),
                  "pde_heat_rollout_at")
        else:
            check(lib().pde_heat_rollout(*args, C.c_void_p(stream_ptr(u))), "pde_heat_rollout")
        return self.output_array


class HeatSolver:
    """Differentiable 2D heat rollout with a per-cell diffusivity field.

    New: the reference steps the heat equation forward only
    (examples/2D_Heat_Equation.py:57-65, scalar alpha).  Step, on a scalar
    (X, Y, 1, 1) field with the boundary groups of ``boundary``:

        v = BC(u);  S = Lap(v);  u' = v + dt * (alpha o S)    (stencil cells; v elsewhere)

    which is the module chain's step with alpha taken per cell (bit-identical to
    ``HeatRollout`` for a constant field).  ``forward`` keeps ceil(sqrt(N))
    checkpoints of u and the last segment's S; ``backward`` recomputes every
    other segment's S from its checkpoint and runs the discrete adjoint,
    returning (dJ/dalpha, dJ/du0).  Buffers are allocated once per device; with
    ``graphs`` (default) each sequence is captured as a CUDA graph after its first
    run and replayed afterwards.  One backward() belongs to the latest forward()."""

    def __init__(self, boundary: GridBoundary, dx: float, dt: float, nsteps: int, order: int = 2,
                 steps_per_pass: int = 0, checkpoint_every: int | None = None, graphs: bool = True) -> None:
        if boundary.inputs[0] != 1:
            raise ValueError("HeatSolver takes scalar fields")
        self.boundary = boundary
        self.shape = tuple(boundary.grid_shape)
        assert self.shape[2] == 1 and self.shape[0] > 1 and self.shape[1] > 1, "2D grids (X, Y, 1)"
        self.dx, self.dt, self.N, self.order = float(dx), float(dt), int(nsteps), int(order)
        self.rules = boundary.rules()
        self._t0 = 0.0  # ramp groups: step n fills the boundary at t0 + n*dt
        self.grid = make_grid(self.shape, boundary.ghost_cells, self.order, self.dx)
        self._steps_per_pass = int(steps_per_pass)
        self.graphs = bool(graphs)
        self.set_checkpoint_every(checkpoint_every)

    def set_checkpoint_every(self, every: int | None) -> None:
        """Checkpoint spacing (None: ceil(sqrt(N)) rounded up to a multiple of the pass
        depth, so no segment ends with a short pass); frees the buffers and graphs."""
        import math
        self._every_auto = not every
        if every:
            self.every = int(every)
        else:  # about sqrt(N), rounded up to whole passes of k steps (k = 8 when left to the library)
            k = self._steps_per_pass if self._steps_per_pass > 0 else 8
            e = max(1, int(math.ceil(math.sqrt(self.N))))
            self.every = max(1, min(self.N, -(-e // k) * k))
        self.segments = [(n0, min(self.every, self.N - n0)) for n0 in range(0, self.N, self.every)]
        self._dev = None
        self._seq_f = GraphedSequence(self._run_forward, self.graphs)
        self._seq_b = GraphedSequence(self._run_backward, self.graphs)

    @property
    def steps_per_pass(self) -> int:
        return self._steps_per_pass

    @steps_per_pass.setter
    def steps_per_pass(self, k: int) -> None:
        self._steps_per_pass = int(k)
        if self._every_auto:
            self.set_checkpoint_every(None)  # the spacing follows the pass depth
        else:
            self._seq_f.reset()
            self._seq_b.reset()

    def _buffers(self, like: torch.Tensor) -> None:
        if self._dev == like.device:
            return
        dev, f = like.device, self.shape + (1,)
        cells = self.shape[0] * self.shape[1]
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device=dev)
        self._work = z(cells)
        self._work_r = z(cells)  # the recomputation's own scratch
        self._seg = z(max(self.every, 1), cells)
        self._seg2 = z(max(self.every, 1), cells) if len(self.segments) > 1 else self._seg
        self._side = torch.cuda.Stream(device=dev)
        self._alpha, self._g = z(*f), z(*f)
        self._ck = z(max(len(self.segments), 1), *f)  # u^{n0} per segment
        self._out = z(*f)
        self._lam = z(2, *f)
        self._tmp = z(*f)
        self._ga = z(*f)
        self._dev = dev
        self._seq_f.reset()
        self._seq_b.reset()

    def _fwd(self, alpha, u, out, nsteps, lstates=None, work=None, n0=0):
        work = self._work if work is None else work
        args = [C.c_void_p(alpha.data_ptr()), C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()),
                C.c_void_p(work.data_ptr()), C.byref(self.grid), C.byref(self.rules), self.dt, int(nsteps),
                self.steps_per_pass, C.c_void_p(lstates.data_ptr()) if lstates is not None else None]
        if self.rules.has_ramp:
            check(lib().pde_heat_forward_at(*args, self._t0, self.dt, int(n0), C.c_void_p(stream_ptr(u))),
                  "pde_heat_forward_at")
        else:
            check(lib().pde_heat_forward(*args, C.c_void_p(stream_ptr(u))), "pde_heat_forward")

    def _check(self, alpha, u):
        require_cuda_f32(alpha, "alpha")
        require_cuda_f32(u, "u")
        if tuple(alpha.shape) != self.shape + (1,) or tuple(u.shape) != self.shape + (1,):
            raise AssertionError(f"alpha and u must be {self.shape + (1,)}")

    def _run_forward(self) -> None:
        for j, (n0, m) in enumerate(self.segments):
            last = j == len(self.segments) - 1
            self._fwd(self._alpha, self._ck[j], self._out if last else self._ck[j + 1], m,
                      self._seg[:m] if last else None, n0=n0)
        if not self.segments:
            self._out.copy_(self._ck[0])

    def _run_backward(self) -> None:
        """Segments from the last to the first.  The adjoint of segment j (this
        stream) runs while a second stream recomputes S of segment j-1 into the
        other of two buffers; events order each buffer's reuse."""
        main, side = torch.cuda.current_stream(), self._side
        J = len(self.segments) - 1
        bufs = (self._seg, self._seg2)  # segment j uses bufs[(J - j) % 2]; the forward filled bufs[0]
        self._ga.zero_()
        a, b = self._lam[0], self._lam[1]
        a.copy_(self._g)
        side.wait_stream(main)
        rec_done, adj_done = {}, {}
        for j in range(J, -1, -1):
            if j >= 1:  # recompute S^{n0} .. S^{n0+m-1} of segment j-1 from its checkpoint
                n0, m = self.segments[j - 1]
                with torch.cuda.stream(side):
                    if j + 1 in adj_done:
                        side.wait_event(adj_done[j + 1])  # its buffer was segment j+1's
                    self._fwd(self._alpha, self._ck[j - 1], self._tmp, m, bufs[(J - j + 1) % 2][:m],
                              work=self._work_r, n0=n0)
                    rec_done[j - 1] = torch.cuda.Event()
                    rec_done[j - 1].record(side)
            n0, m = self.segments[j]
            if j in rec_done:
                main.wait_event(rec_done[j])
            seg = bufs[(J - j) % 2][:m]
            check(lib().pde_heat_adjoint(C.c_void_p(self._alpha.data_ptr()), C.c_void_p(a.data_ptr()),
                                         C.c_void_p(b.data_ptr()), C.c_void_p(seg.data_ptr()),
                                         C.c_void_p(self._ga.data_ptr()), C.byref(self.grid), C.byref(self.rules),
                                         self.dt, m, self.steps_per_pass, C.c_void_p(self._work.data_ptr()),
                                         C.c_void_p(main.cuda_stream)), "pde_heat_adjoint")
            adj_done[j] = torch.cuda.Event()
            adj_done[j].record(main)
            a, b = b, a
        main.wait_stream(side)

    def forward(self, alpha: torch.Tensor, u0: torch.Tensor, t0: float = 0.0) -> torch.Tensor:
        """u^N for diffusivity field alpha and initial field u0; with time-ramped
        groups step n fills the boundary at t0 + n*dt (a new t0 re-captures the
        sequences' graphs, which hold the times)."""
        self._check(alpha, u0)
        self._buffers(u0)
        if self.rules.has_ramp and float(t0) != self._t0:
            self._t0 = float(t0)
            self._seq_f.reset()
            self._seq_b.reset()
        self._alpha.copy_(alpha)
        self._ck[0].copy_(u0)
        self._seq_f.run()
        self._fwd_done = True
        return self._out.clone()

    def backward(self, alpha: torch.Tensor, dJ_duN: torch.Tensor):
        """(dJ/dalpha, dJ/du0) for the last forward()."""
        if not getattr(self, "_fwd_done", False):
            raise RuntimeError("backward() needs a forward() first")
        self._check(alpha, dJ_duN.contiguous())
        self._alpha.copy_(alpha)
        self._g.copy_(dJ_duN)
        self._seq_b.run()
        gu = self._lam[len(self.segments) % 2]  # the buffer the last adjoint pass wrote
        return self._ga.clone(), gu.clone()


class _HeatFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, alpha, u0, solver, t0):
        ctx.solver = solver
        ctx.save_for_backward(alpha)
        return solver.forward(alpha.detach().contiguous(), u0.detach().contiguous(), t0)

    @staticmethod
    def backward(ctx, g):
        (alpha,) = ctx.saved_tensors
        ga, gu = ctx.solver.backward(alpha.detach().contiguous(), g.contiguous())
        return ga, gu, None, None


def heat_rollout(alpha: torch.Tensor, u0: torch.Tensor, solver: HeatSolver, t0: float = 0.0) -> torch.Tensor:
    """u^N as a differentiable function of the diffusivity field alpha and u0
    (a scalar alpha can be broadcast: ``alpha_s.expand(shape)`` sums its gradient);
    time-ramped groups are filled at t0 + n*dt."""
    return _HeatFn.apply(alpha, u0, solver, float(t0))
