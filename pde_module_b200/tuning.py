"""Autotuning of launch configurations.

``tune_stream3d`` times every tile configuration (candidate) of the 3D
streaming kernels for each operator and order on fields of the given interior
shape, with CUDA events over a few repetitions, and selects the fastest through
``pde_stream3d_select`` (process-wide).  ``tune_heat_depth`` picks the
temporal-blocking depth of a HeatRollout.  Both run real kernels on the
current device and synchronise it, so call them at setup, outside any CUDA
graph capture.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib

N_CANDIDATES = 4
_OPS = (("laplacian", _lib.PDE_OP_LAPLACIAN, 1), ("laplacian", _lib.PDE_OP_LAPLACIAN, 3),
        ("grad", _lib.PDE_OP_GRAD, 1), ("divergence", _lib.PDE_OP_DIVERGENCE, 3))


def _time(fn, reps: int) -> float:
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_stream3d(interior=(512, 512, 512), orders=(2, 4), reps: int = 5, kinds=None) -> dict:
    """Select the fastest streaming-kernel candidate per (operator, input components, order).

    Returns {(op, ncomp_in, order): {"best": c, "ms": [t_0, ..., t_3]}}."""
    from .FDM import Laplacian, Grad, Divergence
    lib = _lib.lib()
    out = {}
    for order in orders:
        g = order // 2
        full = tuple(int(s) + 2 * g for s in interior)
        dx = 1.0 / max(interior)
        u = torch.randn(full + (1,), device="cuda")
        v = torch.randn(full + (3,), device="cuda")
        for name, opc, cin in _OPS:
            if kinds is not None and (name, cin) not in kinds:
                continue
            if name == "laplacian":
                mod, x = Laplacian(cin, dx, g, order=order), (u if cin == 1 else v)
            elif name == "grad":
                mod, x = Grad(1, full, dx, g, order=order), u
            else:
                mod, x = Divergence(3, full, dx, g, order=order), v
            times = []
            for c in range(N_CANDIDATES):
                rc = lib.pde_stream3d_select(opc, order, cin, c)
                if rc < 0:
                    _lib.check(rc, "pde_stream3d_select")
                times.append(_time(lambda: mod(x, 1.0), reps))
            best = min(range(N_CANDIDATES), key=lambda c: times[c])
            lib.pde_stream3d_select(opc, order, cin, best)
            out[(name, cin, order)] = {"best": best, "ms": [round(t, 4) for t in times]}
        del u, v
    torch.cuda.synchronize()
    return out


def tune_heat_depth(rollout, u: torch.Tensor, nsteps: int = 256, depths=(1, 2, 4, 8, 16), reps: int = 3) -> int:
    """Set rollout.steps_per_pass to the fastest temporal-blocking depth for field u."""
    best, best_ms = None, None
    for k in depths:
        rollout.steps_per_pass = k
        ms = _time(lambda: rollout(u, nsteps), reps)
        if best_ms is None or ms < best_ms:
            best, best_ms = k, ms
    rollout.steps_per_pass = best
    return best
