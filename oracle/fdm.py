"""ORACLE — TEST INFRASTRUCTURE ONLY.

CPU (NumPy) restatement of PDE_Module's finite-difference hot path, used by
tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the
checker.  Nothing in pde_module_b200 imports it.

It follows the reference kernels operation by operation so that, in float32,
every product and sum is rounded exactly where the reference's Warp kernel
rounds it (no fused multiply-add):

* Laplacian  — FDM/kernel/laplacian.py:34-59: ``acc = 0; for axis in
  eligible axes: for tap: acc += w[tap] * u[c + shift*e_axis]; out = alpha*acc``
  over the interior launch domain (functional/_laplacian.py:26-35);
  weights FDM/module/laplacian.py:33-35, formed in float64, rounded to float32.
* Grad       — FDM/kernel/grad.py:78-100 (weights module/grad.py:37-39).
* Divergence — FDM/kernel/divergence.py:85-106 (weights module/divergence.py:37-39).
* ForwardEuler — time_step/forwardEuler.py:70-79 (``cur + dt*k``, flat).
* GridBoundary — groups functional_boundary.py:111-137; copy :260-263; per
  group kernel :357-400 with the constant value function
  boundary_functions.py:32-45 and the ramp :77-92.

Order-4 weights and the periodic fill have no reference counterpart; they
are restated from their definitions.  Pass ``dtype=np.float64`` for the
float64 oracle (same operation order, double rounding).

Parity pin: the reference package imports ``warp`` (warp-lang 1.12.1, not
installed here), so tests/golden/make_golden.py runs the reference's own FDM
modules through the Warp-DSL executor tests/golden/warp_emu.py and stores their
outputs in tests/golden/fdm_golden.npz; tests/test_golden_cpu.py checks this
restatement against them bit for bit.
"""
from __future__ import annotations

import numpy as np

DIRICHLET = 1
VON_NEUMANN = 2


# ---------------------------------------------------------------- weights ---
def lap_weights(order: int, dx: float, dtype=np.float32) -> np.ndarray:
    if order == 2:
        w = [1.0 / dx ** 2, -2.0 / dx ** 2, 1.0 / dx ** 2]
    elif order == 4:
        d = 12.0 * dx * dx
        w = [-1.0 / d, 16.0 / d, -30.0 / d, 16.0 / d, -1.0 / d]
    else:
        raise ValueError(order)
    return np.array(w, dtype=np.float64).astype(dtype)


def d1_weights(order: int, dx: float, dtype=np.float32) -> np.ndarray:
    if order == 2:
        w = [-1.0 / (2 * dx), 0.0, 1.0 / (2 * dx)]
    elif order == 4:
        d = 12.0 * dx
        w = [1.0 / d, -8.0 / d, 0.0, 8.0 / d, -1.0 / d]
    else:
        raise ValueError(order)
    return np.array(w, dtype=np.float64).astype(dtype)


# ----------------------------------------------------------------- shapes ---
def eligible_dims(grid_shape) -> tuple:
    return tuple(i for i, s in enumerate(grid_shape[:3]) if s > 1)


def _interior_slices(grid_shape, g, shift=(0, 0, 0)):
    """Slices of the interior launch domain moved by ``shift`` cells."""
    sl = []
    for a in range(3):
        n = grid_shape[a]
        if n > 1:
            sl.append(slice(g + shift[a], n - g + shift[a]))
        else:
            sl.append(slice(0, n))
    return tuple(sl)


# -------------------------------------------------------------- operators ---
def laplacian(u: np.ndarray, dx: float, ghost: int, alpha: float, order: int = 2, dtype=np.float32,
              out: np.ndarray | None = None) -> np.ndarray:
    """u: (X, Y, Z, N).  Returns out with the interior written (ghosts 0)."""
    u = np.asarray(u, dtype=dtype)
    w = lap_weights(order, dx, dtype)
    R = (len(w) - 1) // 2
    gs = u.shape[:3]
    if out is None:
        out = np.zeros_like(u)
    core = _interior_slices(gs, ghost)
    acc = np.zeros(u[core].shape, dtype=dtype)
    for a in eligible_dims(gs):
        for t in range(len(w)):
            sh = [0, 0, 0]
            sh[a] = t - R
            acc = acc + w[t] * u[_interior_slices(gs, ghost, sh)]
    out[core] = dtype(alpha) * acc
    return out


def grad(u: np.ndarray, dx: float, ghost: int, alpha: float, order: int = 2, dtype=np.float32,
         force_matrix: bool = False) -> np.ndarray:
    """u: (X, Y, Z, N) -> (X, Y, Z, N, D), or (X, Y, Z, D) when N == 1 and not force_matrix."""
    u = np.asarray(u, dtype=dtype)
    w = d1_weights(order, dx, dtype)
    R = (len(w) - 1) // 2
    gs = u.shape[:3]
    dims = eligible_dims(gs)
    N = u.shape[3]
    out = np.zeros(gs + (N, len(dims)), dtype=dtype)
    core = _interior_slices(gs, ghost)
    for col, a in enumerate(dims):
        acc = np.zeros(u[core].shape, dtype=dtype)
        for t in range(len(w)):
            sh = [0, 0, 0]
            sh[a] = t - R
            acc = acc + w[t] * u[_interior_slices(gs, ghost, sh)]
        out[core + (slice(None), col)] = dtype(alpha) * acc
    if N == 1 and not force_matrix:
        out = out[:, :, :, 0, :].copy()
    return out


def divergence(u: np.ndarray, dx: float, ghost: int, alpha: float, order: int = 2,
               dtype=np.float32) -> np.ndarray:
    """u: (X, Y, Z, D) vector -> (X, Y, Z, 1); (X, Y, Z, N, D) matrix -> (X, Y, Z, N)."""
    u = np.asarray(u, dtype=dtype)
    if u.ndim == 4:
        u = u[:, :, :, None, :]
    w = d1_weights(order, dx, dtype)
    R = (len(w) - 1) // 2
    gs = u.shape[:3]
    dims = eligible_dims(gs)
    N = u.shape[3]
    assert u.shape[4] == len(dims)
    out = np.zeros(gs + (N,), dtype=dtype)
    core = _interior_slices(gs, ghost)
    acc = np.zeros(u[core][..., 0].shape, dtype=dtype)
    for col, a in enumerate(dims):
        for t in range(len(w)):
            sh = [0, 0, 0]
            sh[a] = t - R
            acc = acc + w[t] * u[_interior_slices(gs, ghost, sh)][..., col]
    out[core] = dtype(alpha) * acc
    return out


def forward_euler(y: np.ndarray, k: np.ndarray, dt: float, dtype=np.float32) -> np.ndarray:
    y = np.asarray(y, dtype=dtype)
    k = np.asarray(k, dtype=dtype)
    return y + dtype(dt) * k


# --------------------------------------------------------------- boundary ---
def exterior_groups(grid_shape, ghost: int) -> dict:
    """Node-id groups of functional_boundary.py:111-137 (C-order flat ids)."""
    gs = tuple(grid_shape[:3])
    ids = np.arange(int(np.prod(gs)), dtype=np.int32).reshape(gs)
    groups, faces = {}, []
    for i, ax in enumerate("XYZ"):
        if gs[i] <= 1:
            continue
        for prefix in "-+":
            sl = [slice(None)] * 3
            sl[i] = ghost if prefix == "-" else -(ghost + 1)
            for x in range(3):
                if gs[x] > 1 and x != i:
                    sl[x] = slice(ghost, -ghost) if ghost > 0 else slice(None)
            groups[prefix + ax] = ids[tuple(sl)].ravel()
            faces.append(groups[prefix + ax])
    groups["ALL"] = np.unique(np.concatenate(faces)).astype(np.int32)
    return groups


def bc_value(func: str, value: float, t: float = 0.0, t_max: float = 1.0, dtype=np.float32):
    v = dtype(value)
    if func == "ramp":
        ramp = np.minimum(dtype(t) / dtype(t_max), dtype(1.0))
        return dtype(ramp * v)
    return v


def bc_apply(u: np.ndarray, groups: list, dx: float, ghost: int, t: float = 0.0,
             dtype=np.float32) -> np.ndarray:
    """Copy, then each group in order.

    groups: list of dicts {ids, type (1/2), comps (tuple), func ('constant'|'ramp'), value, t_max}.
    Reads only the pre-boundary field ``u``.
    """
    u = np.asarray(u, dtype=dtype)
    out = u.copy()
    gs = u.shape[:3]
    dims = eligible_dims(gs)
    N = u.shape[3]
    dx32 = dtype(dx)
    flat_u = u.reshape(-1, N)
    flat_o = out.reshape(-1, N)
    strides = (gs[1] * gs[2], gs[2], 1)
    for G in groups:
        ids = np.asarray(G["ids"], dtype=np.int64)
        if ids.size == 0:
            continue
        ijk = np.stack([ids // (gs[1] * gs[2]), (ids // gs[2]) % gs[1], ids % gs[2]], axis=1)
        v = bc_value(G.get("func", "constant"), G["value"], t, G.get("t_max", 1.0), dtype)
        comps = tuple(G["comps"])
        if G["type"] == DIRICHLET:
            node_vals = flat_u[ids].copy()
            for c in comps:
                node_vals[:, c] = v
            flat_o[ids] = node_vals
        for a in dims:
            inc = np.zeros(len(ids), dtype=np.int64)
            inc[ijk[:, a] == ghost] = 1
            inc[(ijk[:, a] == gs[a] - 1 - ghost) & (inc == 0)] = -1
            sel = inc != 0
            if not sel.any():
                continue
            ghost_ids = ids[sel] - inc[sel] * strides[a]
            adj_ids = ids[sel] + inc[sel] * strides[a]
            for c in comps:
                cur = flat_u[adj_ids, c]
                if G["type"] == DIRICHLET:
                    nv = dtype(2.0) * v - cur
                else:
                    s = (-np.sign(inc[sel]).astype(dtype)) * dtype(2.0)
                    nv = s * dx32 * v + cur
                flat_o[ghost_ids, c] = nv
    return out


def periodic_fill(u: np.ndarray, ghost: int, axes) -> np.ndarray:
    """New (no reference counterpart): wrap every ghost layer along ``axes``,
    axes processed in ascending order over the full extent of the others."""
    out = np.array(u, copy=True)
    gs = out.shape[:3]
    for a in sorted(axes):
        n = gs[a]
        M = n - 2 * ghost
        src = [ghost + ((i - ghost) % M) for i in range(n)]
        idx = [slice(None)] * 3
        for i in list(range(ghost)) + list(range(n - ghost, n)):
            idx_d = list(idx)
            idx_s = list(idx)
            idx_d[a] = i
            idx_s[a] = src[i]
            out[tuple(idx_d)] = out[tuple(idx_s)]
    return out


# ------------------------------------------------------------- rollouts ---
def heat_step(u: np.ndarray, groups: list, dx: float, ghost: int, alpha: float, dt: float, order: int = 2,
              dtype=np.float32, t: float = 0.0) -> np.ndarray:
    """One step of examples/2D_Heat_Equation.py:59-62 with a zero-ghost Laplacian
    output; the boundary is filled at time t (ramp groups)."""
    u2 = bc_apply(u, groups, dx, ghost, t, dtype=dtype)
    lap = laplacian(u2, dx, ghost, alpha, order, dtype)
    return forward_euler(u2, lap, dt, dtype)


def heat_rollout(u: np.ndarray, groups: list, dx: float, ghost: int, alpha: float, dt: float, nsteps: int,
                 order: int = 2, dtype=np.float32, t0: float = 0.0) -> np.ndarray:
    """nsteps of heat_step; step n fills the boundary at t0 + n*dt (Python floats),
    as a loop passing that time to GridBoundary does (functional_boundary.py:237,254-255)."""
    u = np.asarray(u, dtype=dtype)
    for n in range(nsteps):
        u = heat_step(u, groups, dx, ghost, alpha, dt, order, dtype, t0 + n * dt)
    return u


def heat_forward_field(alpha, u0, groups, dx, ghost, dt, nsteps, order=2, dtype=np.float32, t0=0.0):
    """New (the reference's loop, examples/2D_Heat_Equation.py:57-65, has a scalar
    alpha): the heat step with a per-cell diffusivity field, one component,
        v = B(u);  S = L(v) (alpha 1);  u' = v + dt*(alpha o S).
    alpha, u0: (X, Y, Z, 1).  Step n fills the boundary at t0 + n*dt (ramp groups).
    Returns (u^N, [S^0, ..., S^{N-1}]), S as (X, Y, Z) arrays."""
    u = np.asarray(u0, dtype=dtype)
    a = np.asarray(alpha, dtype=dtype)
    S = []
    for n in range(nsteps):
        v = bc_apply(u, groups, dx, ghost, t0 + n * dt, dtype=dtype)
        acc = laplacian(v, dx, ghost, 1.0, order, dtype)
        S.append(acc[..., 0].copy())
        u = forward_euler(v, a * acc, dt, dtype)
    return u, S


def bc_linear_map(grid_shape, groups, dx, ghost):
    """The linear part of the boundary fill B(u) = A u + b (one component):
    (direct, pairs) with direct[i] true where B(u)_i = u_i, and pairs a list of
    (ghost cell, partner cell, coefficient +-1) for B(u)_ghost = c +- u_partner.
    Found by applying bc_apply to cell ids with every value set to 0."""
    n = int(np.prod(grid_shape[:3]))
    ids = (np.arange(n, dtype=np.float64) + 1.0).reshape(tuple(grid_shape[:3]) + (1,))
    zero = [dict(G, value=0.0) for G in groups]
    out = bc_apply(ids, zero, dx, ghost, dtype=np.float64).reshape(-1)
    flat = ids.reshape(-1)
    direct = out == flat
    pairs = []
    for i in np.nonzero((out != flat) & (out != 0.0))[0]:
        p = int(abs(out[i])) - 1
        pairs.append((int(i), p, 1.0 if out[i] > 0 else -1.0))
    return direct.reshape(grid_shape[:3]), pairs


def heat_adjoint(alpha, S, lamN, groups, dx, ghost, dt, order=2, dtype=np.float32):
    """Discrete adjoint of heat_forward_field, one rounding per operation:
        dJ/dalpha += lam o (dt * S^n)          stencil cells, n = N-1 .. 0
        z  = dt * (alpha o lam)                stencil cells, 0 elsewhere
        mu = lam + L^T(z)                      L^T = L, zero outside the array
        lam = B^T(mu): (direct ? mu : 0), then -/+ mu_ghost per pair, ghosts in
              the order x-low, x-high, y-low, y-high of their partner.
    Returns (dJ/dalpha, dJ/du^0) as (X, Y, Z, 1) arrays."""
    a = np.asarray(alpha, dtype=dtype)[..., 0]
    lam = np.array(np.asarray(lamN, dtype=dtype)[..., 0])
    gs = lam.shape
    direct, pairs = bc_linear_map(gs, groups, dx, ghost)
    strides = (gs[1] * gs[2], gs[2], 1)

    def pair_key(pr):
        gcell, pcell, _ = pr
        d = pcell - gcell
        axis = next(ax for ax in range(3) if strides[ax] == abs(d) // 2 and abs(d) % strides[ax] == 0)
        return (pcell, axis, 0 if d > 0 else 1)  # per partner: axis, then the low-side ghost first

    pairs = sorted(pairs, key=pair_key)
    w = lap_weights(order, dx, dtype)
    R = (len(w) - 1) // 2
    core = _interior_slices(gs, ghost)
    st = np.zeros(gs, dtype=bool)
    st[core] = True
    galpha = np.zeros(gs, dtype=dtype)
    dt32 = dtype(dt)
    for n in range(len(S) - 1, -1, -1):
        galpha[st] = galpha[st] + lam[st] * (dt32 * np.asarray(S[n], dtype=dtype)[st])
        z = np.zeros(gs, dtype=dtype)
        z[st] = dt32 * (a[st] * lam[st])
        zp = np.pad(z, [(R, R) if gs[ax] > 1 else (0, 0) for ax in range(3)])
        acc = np.zeros(gs, dtype=dtype)
        for ax in eligible_dims(gs):
            for t in range(len(w)):
                sl = [slice(R, R + gs[b]) if gs[b] > 1 else slice(None) for b in range(3)]
                sl[ax] = slice(t, t + gs[ax])
                acc = acc + w[t] * zp[tuple(sl)]
        mu = lam + acc
        new = np.where(direct, mu, dtype(0)).reshape(-1)
        muf = mu.reshape(-1)
        for gcell, pcell, c in pairs:
            new[pcell] = new[pcell] + muf[gcell] if c > 0 else new[pcell] - muf[gcell]
        lam = new.reshape(gs)
    return galpha[..., None], lam[..., None]


def standard_groups(grid_shape, ghost, spec) -> list:
    """spec: list of (group_name, type, value, comps) -> group dicts with ids."""
    G = exterior_groups(grid_shape, ghost)
    return [dict(ids=G[name], type=typ, value=val, comps=tuple(comps), func="constant")
            for name, typ, val, comps in spec]


# ------------------------------------------------------ per-cell samples ---
def stencil_at(u: np.ndarray, cells: np.ndarray, w: np.ndarray, axes_comps, alpha: float,
               dtype=np.float32) -> np.ndarray:
    """Reference-order stencil sum at selected cells.

    u: (X, Y, Z, C) array (C = flattened trailing components); cells: (M, 3)
    int array; axes_comps: list of (axis, component) pairs visited in order,
    each contributing its taps low to high into one accumulator per cell.
    Used to check full-size (e.g. 512^3) outputs at sampled cells.
    """
    R = (len(w) - 1) // 2
    acc = np.zeros(len(cells), dtype=dtype)
    for a, comp in axes_comps:
        for t in range(len(w)):
            idx = cells.copy()
            idx[:, a] += t - R
            acc = acc + w[t] * u[idx[:, 0], idx[:, 1], idx[:, 2], comp]
    return dtype(alpha) * acc


# ------------------------------------------------- fractional-step cavity ---
def ldc_step(u, p, u_groups, p_groups, dx, ghost, nu, dt, jacobi_iters, dtype=np.float32, t=0.0):
    """One projection step composed of the reference operators (no reference
    counterpart: its cavity uses artificial compressibility,
    examples/LDC/LDC_Graph_Capture.py:71-90).  u (X,Y,1,2), p (X,Y,1,1).

        u2 = BC_u(u); u* = u2 + dt*(nu*Lap(u2) - Grad(u2) u2)
        rhs = (1/dt)*Div(BC_u(u*))
        jacobi_iters x: p <- 0.25*(pW + pE + pS + pN - dx^2*rhs) on BC_p(p)
        u = BC_u(u*) + dt*Grad(BC_p(p), -1)

    Every boundary of the step is filled at time t (ramp groups).
    """
    u2 = bc_apply(u, u_groups, dx, ghost, t, dtype=dtype)
    lap = laplacian(u2, dx, ghost, nu, dtype=dtype)
    G = grad(u2, dx, ghost, 1.0, dtype=dtype)  # (X,Y,1,2,2): row = component, column = axis
    conv = G[..., 0] * u2[..., 0:1] + G[..., 1] * u2[..., 1:2]
    us = forward_euler(u2, lap - conv, dt, dtype)
    us_bc = bc_apply(us, u_groups, dx, ghost, t, dtype=dtype)
    dt32 = float(np.float32(dt))
    inv_dt = float(np.float32(1.0 / dt32)) if dtype == np.float32 else 1.0 / dt
    rhs = divergence(us_bc, dx, ghost, inv_dt, dtype=dtype)
    h2 = dtype(dx * dx)
    X, Y = u.shape[0], u.shape[1]
    c = (slice(ghost, X - ghost), slice(ghost, Y - ghost), 0, 0)
    for _ in range(jacobi_iters):
        pb = bc_apply(p, p_groups, dx, ghost, t, dtype=dtype)
        new = pb.copy()
        s = ((pb[ghost - 1:X - ghost - 1, ghost:Y - ghost, 0, 0] + pb[ghost + 1:X - ghost + 1, ghost:Y - ghost, 0, 0])
             + pb[ghost:X - ghost, ghost - 1:Y - ghost - 1, 0, 0]) + pb[ghost:X - ghost, ghost + 1:Y - ghost + 1, 0, 0]
        new[c] = dtype(0.25) * (s - h2 * rhs[c])
        p = new
    pb = bc_apply(p, p_groups, dx, ghost, t, dtype=dtype)
    gp = grad(pb, dx, ghost, -1.0, dtype=dtype)
    u_new = forward_euler(us_bc, gp, dt, dtype)
    return u_new, p


# ------------------------------------------------------ differentiable wave ---
def _wave_interior(X, Y, ghost):
    m = np.zeros((X, Y), dtype=bool)
    m[ghost + 1:X - 1 - ghost, ghost + 1:Y - 1 - ghost] = True
    return m


def _lap5(u, w, dtype):
    """5-point Laplacian (reference order, alpha 1) at every cell not on the array edge."""
    out = np.zeros_like(u)
    c = u[1:-1, 1:-1]
    acc = dtype(0) + w[0] * u[:-2, 1:-1]
    acc = acc + w[1] * c
    acc = acc + w[2] * u[2:, 1:-1]
    acc = acc + w[0] * u[1:-1, :-2]
    acc = acc + w[1] * c
    acc = acc + w[2] * u[1:-1, 2:]
    out[1:-1, 1:-1] = acc
    return out


def wave_forward(K, u0, src, src_cell, nsteps, dx, ghost=1, dtype=np.float32):
    """New (no reference counterpart).  Leapfrog on the cells strictly inside the
    node ring: u^{n+1} = 2u^n - u^{n-1} + K o L(u^n) + src[n] at src_cell,
    u^{-1} = u^0 = u0.  K, u0: (X, Y, 1, 1).  Returns [u^0, ..., u^N] as (X, Y) arrays."""
    K2 = np.asarray(K, dtype=dtype)[:, :, 0, 0]
    X, Y = K2.shape
    I = _wave_interior(X, Y, ghost)
    w = lap_weights(2, dx, dtype)
    u = np.where(I, np.asarray(u0, dtype=dtype)[:, :, 0, 0], dtype(0))
    um = u.copy()
    sx, sy = (src_cell // Y, src_cell % Y) if src_cell is not None and src_cell >= 0 else (-1, -1)
    states = [u]
    for n in range(nsteps):
        v = dtype(2.0) * u - um
        v = v + K2 * _lap5(u, w, dtype)
        if sx >= 0:
            v[sx, sy] = v[sx, sy] + dtype(src[n])
        v = np.where(I, v, dtype(0))
        um, u = u, v
        states.append(u)
    return states


def wave_adjoint(K, states, muN, dx, ghost=1, dtype=np.float32):
    """Discrete adjoint of wave_forward: mu^n = 2mu^{n+1} - mu^{n+2} + L(K o mu^{n+1}),
    dJ/dK += mu^{n+1} o L(u^n) for n = N-1 .. 0.  Returns (dJ/dK, mu^0, mu^1) as (X, Y)."""
    K2 = np.asarray(K, dtype=dtype)[:, :, 0, 0]
    X, Y = K2.shape
    I = _wave_interior(X, Y, ghost)
    w = lap_weights(2, dx, dtype)
    mu1 = np.where(I, np.asarray(muN, dtype=dtype)[:, :, 0, 0], dtype(0))
    mu2 = np.zeros_like(mu1)
    gK = np.zeros_like(mu1)
    for n in range(len(states) - 2, -1, -1):
        gK = np.where(I, gK + mu1 * _lap5(states[n], w, dtype), gK)
        mu0 = dtype(2.0) * mu1 - mu2
        mu0 = mu0 + _lap5(K2 * mu1, w, dtype)
        mu0 = np.where(I, mu0, dtype(0))
        mu2, mu1 = mu1, mu0
    return gK, mu1, mu2
