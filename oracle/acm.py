"""ORACLE — TEST INFRASTRUCTURE ONLY.

CPU (NumPy) restatement of PDE_Module's element-wise, absorbing-layer and
Runge-Kutta modules, used by tests/ as the checker.  Nothing in pde_module_b200
imports it.

* OuterProduct — FDM/module/elementWiseOps.py:10-48 (wp.outer per cell: M[i, j] =
  A[i] * B[j], one rounding per product).
* scalarVectorMult — elementWiseOps.py:51-88, FDM/kernel/elementWiseOps.py:6-23
  (a[0] * b per cell).
* FarField — FDM/module/farfield.py:13-151, FDM/kernel/farfield.py:8-77: points of
  the outer layers (per eligible axis, index < L or >= n - L, excluded groups left
  out, :62-90); per point the axis of the nearest array face (first minimum,
  :38-48), the depth dx into the layer (:66-70) and
  out = -(sigma * (dx / L) ** beta) * (u - u_far); zero elsewhere.
* ViscousDampingLayer — FDM/module/viscousDampingLayer.py:13-150,
  FDM/kernel/viscousDampingLayer.py:8-76: the same points and depth,
  out = -(C_max * (dx / L) ** p) * du_dt.
* RungeKatta1 / RungeKatta2 — time_step/rungeKatta.py:21-174, composed from the
  fdm oracle's GridBoundary, Laplacian and ForwardEuler (RungeKatta1 steps with
  dt / 2, as the reference does, :79-83).
* The weakly compressible RK2 step of examples/LDC/LDC_RK2.py (bc and f at
  :116-140: u = m/rho, boundary fills, momentum, divergence, Laplacian, outer
  product, biharmonic damping, pressure gradient), composed of the operators
  above, for the fused kernel's parity (its own operators pinned as above).

The layer profile (dx / L) ** beta is a float32 power (the C library's powf, as
the reference's CPU kernels and NumPy's float32 scalar power both call).

Parity pin: tests/golden/make_acm_golden.py runs the reference modules through
tests/golden/warp_emu.py (tests/golden/acm_golden.npz); tests/test_acm_cpu.py
checks this restatement against them bit for bit.
"""
from __future__ import annotations

import numpy as np

from . import fdm

INT32_MAX = 2 ** 31 - 1


def outer(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    return (A[..., :, None] * B[..., None, :]).astype(np.float32)


def scalar_mult(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    s = A[..., 0].astype(np.float32)
    return (s.reshape(s.shape + (1,) * (B.ndim - 3)) * B).astype(np.float32)


def layer_points(grid_shape, num_layers: int, exclude=()) -> np.ndarray:
    """(n, 3) int32 points of the absorbing layers, in C order (farfield.py:62-90)."""
    idx = np.moveaxis(np.indices(grid_shape, dtype=np.int32), 0, -1).reshape(-1, 3)
    masks = []
    for i, (s, ax) in enumerate(zip(grid_shape, "XYZ")):
        if s > 1:
            if f"-{ax}" not in exclude:
                masks.append(idx[:, i] < num_layers)
            if f"+{ax}" not in exclude:
                masks.append(idx[:, i] >= s - num_layers)
    mask = masks[0]
    for m in masks[1:]:
        mask = np.logical_or(mask, m)
    return idx[mask]


def layer_depth(points: np.ndarray, grid_shape, num_layers: int) -> np.ndarray:
    """Depth dx of each point into its layer (farfield.py:38-48, :62-70)."""
    n = np.array(grid_shape, dtype=np.int64)
    p = points.astype(np.int64)
    dist = np.where(n > 1, np.minimum(p, n - p - 1), INT32_MAX)
    axis = np.argmin(dist, axis=1)  # first minimum
    x = p[np.arange(len(p)), axis]
    na = n[axis]
    hi_lim = (na - 1) - num_layers
    return np.where((na - 1 - x) < x, x - hi_lim, num_layers - x)


def layer_profile(points, grid_shape, num_layers: int, exponent: float) -> np.ndarray:
    """(dx / L) ** exponent per point, in float32, one powf each."""
    d = layer_depth(points, grid_shape, num_layers)
    q = d.astype(np.float32) / np.float32(num_layers)
    e = np.float32(exponent)
    return np.array([np.float32(v) ** e for v in q], dtype=np.float32)


def farfield(u: np.ndarray, grid_shape, num_layers: int, beta: float, cond, sigma: float, exclude=()):
    pts = layer_points(grid_shape, num_layers, exclude)
    prof = layer_profile(pts, grid_shape, num_layers, beta)
    out = np.zeros_like(u, dtype=np.float32)
    damp = (np.float32(sigma) * prof).astype(np.float32)
    c = np.asarray(cond, dtype=np.float32).reshape(u.shape[3:])
    sel = (pts[:, 0], pts[:, 1], pts[:, 2])
    diff = (u[sel] - c).astype(np.float32)
    out[sel] = ((-damp).reshape((-1,) + (1,) * (u.ndim - 3)) * diff).astype(np.float32)
    return out


def damping(du: np.ndarray, grid_shape, num_layers: int, p: float, cmax: float, exclude=()):
    pts = layer_points(grid_shape, num_layers, exclude)
    prof = layer_profile(pts, grid_shape, num_layers, p)
    out = np.zeros_like(du, dtype=np.float32)
    damp = (np.float32(cmax) * prof).astype(np.float32)
    sel = (pts[:, 0], pts[:, 1], pts[:, 2])
    out[sel] = ((-damp).reshape((-1,) + (1,) * (du.ndim - 3)) * du[sel]).astype(np.float32)
    return out


def runge_kutta(order: int, fields, groups, alphas, dx, ghost, dt, steps):
    """RungeKatta1/2 with bc = GridBoundary per field and f = Laplacian(alpha) per field.
    Ghost cells of the Laplacian output are taken as zero (the reference's output
    there is never written)."""
    ys = [np.asarray(u, dtype=np.float32) for u in fields]
    t = 0.0
    for _ in range(steps):
        ys = [fdm.bc_apply(y, g, dx, ghost, t) for y, g in zip(ys, groups)]
        k1 = [fdm.laplacian(y, dx, ghost, a) for y, a in zip(ys, alphas)]
        if order == 1:
            ys = [fdm.forward_euler(y, k, dt / 2) for y, k in zip(ys, k1)]
        else:
            y0 = [y.copy() for y in ys]
            y1 = [fdm.forward_euler(y, k, dt / 2) for y, k in zip(ys, k1)]
            y1 = [fdm.bc_apply(y, g, dx, ghost, t) for y, g in zip(y1, groups)]
            k2 = [fdm.laplacian(y, dx, ghost, a) for y, a in zip(y1, alphas)]
            ys = [fdm.forward_euler(y, k, dt) for y, k in zip(y0, k2)]
        t += dt
    return ys


# ---- weakly compressible RK2 step (examples/LDC/LDC_RK2.py composed of the above) ----
def wc_bc(m, rho, u_groups, rho_groups, dx, ghost):
    """bc(t, m, rho) of LDC_RK2.py: u = m / rho; BC_u(u); BC_rho(rho); m = rho * u."""
    u = (m / rho).astype(np.float32)
    u = fdm.bc_apply(u, u_groups, dx, ghost)
    r = fdm.bc_apply(rho, rho_groups, dx, ghost)
    return scalar_mult(r, u), r


def wc_f(m, rho, dx, ghost, nu, eps, c2, rho0):
    """f(t, m, rho) of LDC_RK2.py (momentum and density rates)."""
    u = (m / rho).astype(np.float32)
    m_div = fdm.divergence(m, dx, ghost, -1.0)
    u_diff = fdm.laplacian(u, dx, ghost, nu)
    u_conv = fdm.divergence(outer(m, u), dx, ghost, 1.0)
    u_damp = fdm.laplacian(u_diff, dx, ghost, eps)
    p = (np.float32(c2) * (rho - np.float32(rho0))).astype(np.float32)
    dp = fdm.grad(p, dx, ghost, -1.0)
    k_m = (((dp - u_conv) + u_diff) + u_damp).astype(np.float32)
    return k_m, m_div


def wc_rk2(m, rho, u_groups, rho_groups, dx, ghost, nu, eps, c2, rho0, dt, nsteps):
    """nsteps of RungeKatta2 (rungeKatta.py:123-174) with the bc and f above."""
    m = np.asarray(m, dtype=np.float32)
    rho = np.asarray(rho, dtype=np.float32)
    for _ in range(nsteps):
        m0, r0 = wc_bc(m, rho, u_groups, rho_groups, dx, ghost)
        km, kr = wc_f(m0, r0, dx, ghost, nu, eps, c2, rho0)
        m1 = fdm.forward_euler(m0, km, dt / 2)
        r1 = fdm.forward_euler(r0, kr, dt / 2)
        m1, r1 = wc_bc(m1, r1, u_groups, rho_groups, dx, ghost)
        km, kr = wc_f(m1, r1, dx, ghost, nu, eps, c2, rho0)
        m = fdm.forward_euler(m0, km, dt)
        rho = fdm.forward_euler(r0, kr, dt)
    return m, rho
