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


def set_launch_3d(tile_y: int = 0, tile_z: int = 0, chunks: int = 0) -> None:
    """Launch shape of the 3D streaming heat rollout: tile sides along Y and Z
    (capped at the compiled maxima) and the number of X chunks; 0 = automatic.
    Results do not depend on it."""
    _lib.check(_lib.lib().pde_set_launch_3d(int(tile_y), int(tile_z), int(chunks)), "pde_set_launch_3d")


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


BATCH_TILES = ((32, 64), (64, 64), (32, 128), (64, 32), (16, 128), (48, 96))
BATCH_DEPTHS = (2, 4, 6, 8, 12, 16)


def tune_batched(rollout, nsteps: int = 100, tiles=BATCH_TILES, depths=BATCH_DEPTHS, reps: int = 2) -> dict:
    """Pick the fastest (tile, time-block depth) of a batched rollout.

    Times ``rollout(nsteps)`` for every admissible pair (the halo may not exceed
    a tile side, the shared-memory region must fit) and leaves the rollout
    configured with the best.  The rollout advances its fields in place, so
    they are saved first and restored afterwards.  Returns
    {"best": (tile_x, tile_y, k), "ms": {"TXxTY_k": ms}}."""
    saved = [f.clone() for f in rollout.fields]
    saved_prev = [f.clone() for f in rollout.prev] if rollout.prev is not None else None
    times = {}
    best = None
    for t in tiles:
        for k in depths:
            try:
                rollout.configure(tile=t, steps_per_pass=k)
            except _lib.PdeError:
                continue  # halo wider than the tile, or region too large
            ms = _time(lambda: rollout(nsteps), reps)
            times[f"{t[0]}x{t[1]}_k{k}"] = round(ms, 4)
            if best is None or ms < best[0]:
                best = (ms, t, k)
    rollout.configure(tile=best[1], steps_per_pass=best[2])
    for f, s in zip(rollout.fields, saved):
        f.copy_(s)
    if saved_prev is not None:
        for f, s in zip(rollout.prev, saved_prev):
            f.copy_(s)
    torch.cuda.synchronize()
    return {"best": (best[1][0], best[1][1], best[2]), "ms": times}
