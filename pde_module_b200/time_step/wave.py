"""Differentiable 2D wave equation: leapfrog rollout and its discrete adjoint.

New (no reference counterpart: the reference's wave examples step a first-order
(u, v) pair with forward Euler, tests/FDM/test_WaveStanding.py:71-76).  On the
cells strictly inside the Dirichlet node ring of an (X, Y, 1, 1) grid, with
K = dt^2 c^2 and L the reference's 5-point Laplacian:

    u^{n+1} = 2 u^n - u^{n-1} + K o L(u^n) + s^n e_src,    u^{-1} = u^0 = u0

``WaveSolver.forward`` runs N steps keeping ceil(sqrt(N)) checkpoints;
``WaveSolver.backward`` recomputes each segment from its checkpoint and runs the
discrete adjoint (mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1})), accumulating
dJ/dK; dJ/du0 = mu^0 - mu^1.  ``wave_rollout`` wraps both in a
torch.autograd.Function of (K, u0), so gradients reach c through K = dt^2 c^2.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .._lib import lib, check, stream_ptr, make_grid, require_cuda_f32
from ._replay import GraphedSequence


class WaveSolver:
    """Leapfrog rollout of N steps and its adjoint with sqrt(N) checkpoints.

    All buffers are allocated once per device: checkpoints (u^{n-1}, u^n) at the
    start of every segment, L(u^n) of one segment, the adjoint's mu pairs.  With
    ``graphs`` (default) the forward and the backward sequences are each captured
    as a CUDA graph after their first (eager) run and replayed afterwards.  One
    backward() belongs to the latest forward()."""

    def __init__(self, shape, dx: float, nsteps: int, src: torch.Tensor | None = None, src_cell=None,
                 ghost_cells: int = 1, steps_per_pass: int = 0, checkpoint_every: int | None = None,
                 graphs: bool = True) -> None:
        self.shape = tuple(int(s) for s in shape[:3])
        assert self.shape[2] == 1, "2D grids (X, Y, 1)"
        self.dx, self.N, self.g = float(dx), int(nsteps), int(ghost_cells)
        self.grid = make_grid(self.shape, self.g, 2, self.dx)
        self.src = src
        if src_cell is None:
            self.src_cell = -1
        elif isinstance(src_cell, (tuple, list)):
            self.src_cell = int(src_cell[0]) * self.shape[1] + int(src_cell[1])
        else:
            self.src_cell = int(src_cell)
        if self.src_cell >= 0:
            require_cuda_f32(src, "src")
            assert src.numel() >= self.N
        self._steps_per_pass = int(steps_per_pass)
        self.graphs = bool(graphs)
        self.set_checkpoint_every(checkpoint_every)

    # -- configuration ---------------------------------------------------------
    def set_checkpoint_every(self, every: int | None) -> None:
        """Checkpoint spacing (None: ceil(sqrt(N)) rounded up to a multiple of the pass
        depth, so no segment ends with a short pass); frees the buffers and graphs."""
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
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device=dev)
        self._work = z(6, self.shape[0] * self.shape[1])
        self._seg = z(max(self.every, 1), self.shape[0] * self.shape[1])
        # a second buffer of L(u^n): the recomputation of segment j-1 fills it while
        # the adjoint of segment j reads the first
        self._seg2 = z(max(self.every, 1), self.shape[0] * self.shape[1]) if len(self.segments) > 1 else self._seg
        self._K, self._u0, self._g = z(*f), z(*f), z(*f)
        self._ck = z(max(len(self.segments), 1), 2, *f)       # (u^{n0-1}, u^{n0}) per segment
        self._out = z(2, *f)                                   # (u^{N-1}, u^N)
        self._mu = z(2, 2, *f)                                 # ping-pong (mu^{n+1}, mu^{n+2}) pairs
        self._tmp = z(2, *f)
        self._gK, self._gu = z(*f), z(*f)
        self._mask = interior_mask(self.shape, self.g, dev)
        self._dev = dev
        self._seq_f.reset()
        self._seq_b.reset()

    def _fwd(self, K, a, b, oa, ob, n0, nsteps, lstates=None, work=None):
        work = self._work if work is None else work
        check(lib().pde_wave_forward(C.c_void_p(K.data_ptr()), C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                     C.c_void_p(oa.data_ptr()), C.c_void_p(ob.data_ptr()),
                                     C.c_void_p(self.src.data_ptr()) if self.src_cell >= 0 else None,
                                     self.src_cell, n0, nsteps, self.steps_per_pass,
                                     C.c_void_p(lstates.data_ptr()) if lstates is not None else None,
                                     C.c_void_p(work.data_ptr()), C.byref(self.grid),
                                     C.c_void_p(stream_ptr(K))), "pde_wave_forward")

    # -- the two launch sequences (static buffers only) ------------------------
    def _run_forward(self) -> None:
        self._ck[0, 0].copy_(self._u0)
        self._ck[0, 1].copy_(self._u0)
        for j, (n0, m) in enumerate(self.segments):
            last = j == len(self.segments) - 1
            o = self._out if last else self._ck[j + 1]
            # the last segment keeps L(u^n): the adjoint starts there without recomputing
            self._fwd(self._K, self._ck[j, 0], self._ck[j, 1], o[0], o[1], n0, m,
                      lstates=self._seg[:m] if last else None)
        if not self.segments:
            self._out[0].copy_(self._u0)
            self._out[1].copy_(self._u0)

    def _run_backward(self) -> None:
        """Segments from the last to the first, each one paired launch sequence
        (pde_wave_pair): the adjoint of segment j beside the recomputation of
        L(u^n) of segment j-1 into the other of two buffers."""
        J = len(self.segments) - 1
        bufs = (self._seg, self._seg2)  # segment j uses bufs[(J - j) % 2]; the forward filled bufs[0]
        self._gK.zero_()
        a, b = self._mu[0], self._mu[1]
        a[0].copy_(self._g)
        a[1].zero_()
        P = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        for j in range(J, -1, -1):
            n0, m = self.segments[j]
            if j >= 1:
                f0, fm = self.segments[j - 1]
                ck, lf = self._ck[j - 1], bufs[(J - j + 1) % 2][:fm]
            else:
                f0, fm, ck, lf = 0, 0, None, None
            check(lib().pde_wave_pair(P(self._K), P(ck[0]) if ck is not None else None,
                                      P(ck[1]) if ck is not None else None, f0, fm, P(lf),
                                      P(a[0]), P(a[1]), P(b[0]), P(b[1]), P(bufs[(J - j) % 2][:m]), P(self._gK), m,
                                      C.c_void_p(self.src.data_ptr()) if self.src_cell >= 0 else None,
                                      self.src_cell, self.steps_per_pass, P(self._work), C.byref(self.grid),
                                      C.c_void_p(stream_ptr(self._K))), "pde_wave_pair")
            a, b = b, a
        torch.sub(a[0], a[1], out=self._gu)  # dJ/du0 = mu^0 + mu^{-1} = mu^0 - mu^1

    # -- public ------------------------------------------------------------------
    def forward(self, K: torch.Tensor, u0: torch.Tensor) -> torch.Tensor:
        """u^N from u^{-1} = u^0 = u0 (restricted to the cells inside the node ring)."""
        require_cuda_f32(K, "K")
        require_cuda_f32(u0, "u0")
        self._buffers(K)
        self._K.copy_(K)
        torch.mul(u0, self._mask, out=self._u0)  # the state lives inside the node ring
        self._seq_f.run()
        self._fwd_done = True
        return self._out[1].clone()

    def backward(self, K: torch.Tensor, dJ_duN: torch.Tensor):
        """(dJ/dK, dJ/du0) for the last forward()."""
        if not getattr(self, "_fwd_done", False):
            raise RuntimeError("backward() needs a forward() first")
        self._K.copy_(K)
        self._g.copy_(dJ_duN)
        self._seq_b.run()
        return self._gK.clone(), self._gu.clone()


class _WaveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, K, u0, solver):
        ctx.solver = solver
        ctx.save_for_backward(K)
        return solver.forward(K.detach().contiguous(), u0.detach().contiguous())

    @staticmethod
    def backward(ctx, g):
        (K,) = ctx.saved_tensors
        gK, gu0 = ctx.solver.backward(K.detach().contiguous(), g)
        return gK, gu0, None


def wave_rollout(K: torch.Tensor, u0: torch.Tensor, solver: WaveSolver) -> torch.Tensor:
    """u^N as a differentiable function of K = dt^2 c^2 and u0."""
    return _WaveFn.apply(K, u0, solver)


def interior_mask(shape, ghost_cells: int = 1, device="cuda") -> torch.Tensor:
    """1 on the cells the wave state lives on (strictly inside the node ring)."""
    X, Y = int(shape[0]), int(shape[1])
    m = torch.zeros((X, Y, 1, 1), dtype=torch.float32, device=device)
    g = ghost_cells
    m[g + 1:X - 1 - g, g + 1:Y - 1 - g] = 1.0
    return m


def ricker(nsteps: int, dt: float, f0: float) -> np.ndarray:
    """Ricker wavelet samples r(n dt), delayed by 1.2/f0."""
    t = np.arange(nsteps) * dt - 1.2 / f0
    a = (np.pi * f0 * t) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def speed_field(shape, seed: int, amplitude: float = 0.1, sigma: float = 8.0) -> np.ndarray:
    """1 + amplitude * (Gaussian-filtered standard normal noise, scaled to max |.| = 1)."""
    from scipy.ndimage import gaussian_filter
    f = gaussian_filter(np.random.default_rng(seed).standard_normal(tuple(shape[:2])), sigma=sigma, mode="wrap")
    return 1.0 + amplitude * f / np.abs(f).max()


def make_problem(n: int = 512, nsteps: int = 2000, seed: int = 6, target_seed: int = 7, cfl: float = 0.5,
                 device="cuda", steps_per_pass: int = 0):
    """The differentiable-wave benchmark problem: n^2 nodes (+1 ghost), speed field
    1 + 0.1 smooth noise, Ricker source at the centre with 10 cells per wavelength at
    c = 1, leapfrog at CFL 0.5, target from another seeded speed field.
    Returns (solver, c, u0, target, dt, mask)."""
    g = 1
    shape = (n + 2 * g, n + 2 * g, 1)
    dx = 1.0 / (n - 1)
    c = speed_field(shape, seed)
    ct = speed_field(shape, target_seed)
    dt = cfl * dx / (np.sqrt(2.0) * max(c.max(), ct.max()))
    f0 = 1.0 / (10.0 * dx)
    # point source of unit strength per cell area: u reaches O(0.1) at the wavefront
    src = torch.from_numpy(((dt * dt / (dx * dx)) * ricker(nsteps, dt, f0)).astype(np.float32)).to(device)
    solver = WaveSolver(shape, dx, nsteps, src=src, src_cell=(shape[0] // 2, shape[1] // 2), ghost_cells=g,
                        steps_per_pass=steps_per_pass)
    c_t = torch.from_numpy(c.astype(np.float32)[:, :, None, None]).to(device)
    ct_t = torch.from_numpy(ct.astype(np.float32)[:, :, None, None]).to(device)
    u0 = torch.zeros(shape + (1,), dtype=torch.float32, device=device)
    with torch.no_grad():
        target = solver.forward((dt * dt) * ct_t * ct_t, u0).clone()
    return solver, c_t, u0, target, float(dt), interior_mask(shape, g, device)
