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


class WaveSolver:
    def __init__(self, shape, dx: float, nsteps: int, src: torch.Tensor | None = None, src_cell=None,
                 ghost_cells: int = 1, steps_per_pass: int = 0, checkpoint_every: int | None = None) -> None:
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
        self.steps_per_pass = int(steps_per_pass)
        self.every = int(checkpoint_every) if checkpoint_every else max(1, int(math.ceil(math.sqrt(self.N))))
        self.checkpoints = []
        self._work = None

    def _buffers(self, like: torch.Tensor):
        if self._work is None or self._work.device != like.device:
            cells = self.shape[0] * self.shape[1]
            self._work = torch.zeros((2, cells), dtype=torch.float32, device=like.device)
            self._seg = torch.zeros((self.every + 1, cells), dtype=torch.float32, device=like.device)
        self._last_seg_ready = getattr(self, "_last_seg_ready", False)

    def _fwd(self, K, a, b, oa, ob, n0, nsteps, states=None):
        check(lib().pde_wave_forward(C.c_void_p(K.data_ptr()), C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                     C.c_void_p(oa.data_ptr()), C.c_void_p(ob.data_ptr()),
                                     C.c_void_p(self.src.data_ptr()) if self.src_cell >= 0 else None,
                                     self.src_cell, n0, nsteps, self.steps_per_pass,
                                     C.c_void_p(states.data_ptr()) if states is not None else None,
                                     C.c_void_p(self._work.data_ptr()), C.byref(self.grid),
                                     C.c_void_p(stream_ptr(K))), "pde_wave_forward")

    def forward(self, K: torch.Tensor, u0: torch.Tensor) -> torch.Tensor:
        """u^N from u^{-1} = u^0 = u0; keeps (u^{n-1}, u^n) at n = 0, every, 2*every, ..."""
        require_cuda_f32(K, "K")
        require_cuda_f32(u0, "u0")
        self._buffers(K)
        self.checkpoints = []
        u0 = u0 * interior_mask(self.shape, self.g, u0.device)  # the state lives inside the node ring
        prev, cur = u0.clone(), u0.clone()
        n = 0
        self._last_seg_ready = False
        while n < self.N:
            self.checkpoints.append((n, prev.clone(), cur.clone()))
            m = min(self.every, self.N - n)
            op, oc = torch.empty_like(cur), torch.empty_like(cur)
            if n + m == self.N:
                # the last segment keeps its states: the adjoint starts there without recomputing
                self._seg[0].copy_(cur.reshape(-1))
                self._fwd(K, prev, cur, op, oc, n, m, states=self._seg[1:m + 1])
                self._last_seg_ready = True
            else:
                self._fwd(K, prev, cur, op, oc, n, m)
            prev, cur, n = op, oc, n + m
        return cur

    def backward(self, K: torch.Tensor, dJ_duN: torch.Tensor):
        """(dJ/dK, dJ/du0) for the last forward()."""
        self._buffers(K)
        gK = torch.zeros_like(K)
        mu1, mu2 = dJ_duN.contiguous().clone(), torch.zeros_like(dJ_duN)
        kept = self._last_seg_ready
        self._last_seg_ready = False
        for n0, prev, cur in reversed(self.checkpoints):
            m = min(self.every, self.N - n0)
            seg = self._seg[: m]
            if kept and n0 + m == self.N:
                pass  # u^{n0} .. u^{N-1} were stored by forward()
            else:
                seg[0].copy_(cur.reshape(-1))
                if m > 1:  # recompute u^{n0+1} .. u^{n0+m-1}
                    op, oc = torch.empty_like(cur), torch.empty_like(cur)
                    self._fwd(K, prev, cur, op, oc, n0, m - 1, states=seg[1:])
            o1, o2 = torch.empty_like(mu1), torch.empty_like(mu2)
            check(lib().pde_wave_adjoint(C.c_void_p(K.data_ptr()), C.c_void_p(mu1.data_ptr()),
                                         C.c_void_p(mu2.data_ptr()), C.c_void_p(o1.data_ptr()),
                                         C.c_void_p(o2.data_ptr()), C.c_void_p(seg.data_ptr()),
                                         C.c_void_p(gK.data_ptr()), m, self.steps_per_pass,
                                         C.c_void_p(self._work.data_ptr()), C.byref(self.grid),
                                         C.c_void_p(stream_ptr(K))), "pde_wave_adjoint")
            mu1, mu2 = o1, o2
        return gK, mu1 - mu2  # dJ/du0 = mu^0 + mu^{-1} = mu^0 - mu^1


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
