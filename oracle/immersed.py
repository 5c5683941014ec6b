"""ORACLE — TEST INFRASTRUCTURE ONLY.

CPU (NumPy) restatement of PDE_Module's ImmersedBoundary
(src/pde_module/FDM/boundary/immersedBoundary.py), the staircase boundary for
solid regions inside the grid, used by tests/ as the checker.  Nothing in
pde_module_b200 imports it.

Geometry (finalize(), immersedBoundary.py:57-66):
* solid cells: nonzero bitmask, listed in C order (np.nonzero, :87-89);
* solid boundary: a solid cell with a fluid (bitmask 0) neighbour along an
  eligible axis (locate_boundary, :406-438); the others are interior solids,
  also flattened to x*Y*Z + y*Z + z (:101-107);
* fluid boundary: the fluid neighbours of boundary cells, unique rows
  (identify_fluid_boundary, :110-131 and :344-378);
* fluid neighbours: per boundary cell and eligible axis, the bitmask at -1 and
  +1 (identify_fluid_neighbors, :133-151 and :381-403).

forward(u, fill) (:176-205, kernels :216-341): copy; per boundary cell and
component, Dirichlet (type 1) sets the value, von Neumann (type 2) sets the
running mean ``avg += (c - avg) / n`` over fluid neighbours in axis order, low
side first, of ``c = u_f - (s * value) * dx`` (s = -1, +1), every operation
rounded to float32; then interior solids take ``fill`` in every component.

Solid cells on the array's outer layer along an eligible axis are refused: the
reference reads outside the array there.

Parity pin: tests/golden/make_ib_golden.py runs the reference module through
tests/golden/warp_emu.py and stores its maps and outputs (tests/golden/ib_golden.npz);
tests/test_immersed_cpu.py checks this restatement against them bit for bit.
"""
from __future__ import annotations

import numpy as np

from .fdm import eligible_dims

DIRICHLET, VON_NEUMANN = 1, 2


def _check_edges(bitmask, dims):
    for a in dims:
        lo = np.take(bitmask, 0, axis=a)
        hi = np.take(bitmask, bitmask.shape[a] - 1, axis=a)
        if np.any(lo != 0) or np.any(hi != 0):
            raise ValueError("solid cells on the array's outer layer (the reference reads outside the array)")


def ib_maps(bitmask: np.ndarray) -> dict:
    """The index maps finalize() builds, from an int8 (X, Y, Z) bitmask."""
    bm = np.asarray(bitmask, dtype=np.int8)
    X, Y, Z = bm.shape
    dims = eligible_dims(bm.shape)
    _check_edges(bm, dims)
    solid = np.stack(np.nonzero(bm), axis=-1).astype(np.int32)  # :87
    is_b = np.zeros(len(solid), dtype=bool)
    nbr = np.zeros((len(solid), len(dims), 2), dtype=np.int8)
    for d, a in enumerate(dims):  # :424-436, :396-401
        e = np.zeros(3, dtype=np.int32)
        e[a] = 1
        lo = solid - e
        hi = solid + e
        nbr[:, d, 0] = bm[lo[:, 0], lo[:, 1], lo[:, 2]]
        nbr[:, d, 1] = bm[hi[:, 0], hi[:, 1], hi[:, 2]]
        is_b |= (nbr[:, d, 0] == 0) | (nbr[:, d, 1] == 0)
    sb = solid[is_b]
    interior = solid[~is_b]
    flat = interior[:, 0].astype(np.int64) * Y * Z + interior[:, 1].astype(np.int64) * Z + interior[:, 2]
    fluid = []
    for d, a in enumerate(dims):  # :367-376
        for i, s in enumerate((-1, 1)):
            adj = sb.copy()
            adj[:, a] += s
            fluid.append(adj[nbr[is_b][:, d, i] == 0])
    fb = np.unique(np.concatenate(fluid, axis=0), axis=0) if fluid else np.zeros((0, 3), np.int32)
    return dict(solid_boundary=sb, interior_solids=interior, fluid_neighbors=nbr[is_b], fluid_boundary=fb,
                flat_array=flat)


def ib_apply(u: np.ndarray, maps: dict, bc_type: np.ndarray, bc_value: np.ndarray, dx: float,
             fill: float = 0.0) -> np.ndarray:
    """forward(u, fill): u (X, Y, Z, N) float32; bc_type (n_sb, N) int8; bc_value (n_sb, N)."""
    u = np.asarray(u, dtype=np.float32)
    out = u.copy()
    dims = eligible_dims(u.shape)
    sb = maps["solid_boundary"]
    nbr = maps["fluid_neighbors"]
    dx32 = np.float32(dx)
    N = u.shape[3]
    for var in range(N):
        bv = np.asarray(bc_value[:, var], dtype=np.float32)
        bt = np.asarray(bc_type[:, var])
        avg = np.zeros(len(sb), dtype=np.float32)
        n = np.ones(len(sb), dtype=np.float32)
        for d, a in enumerate(dims):  # :283-296
            for i, s in enumerate((-1, 1)):
                m = nbr[:, d, i] == 0
                adj = sb.copy()
                adj[:, a] += s
                uf = u[adj[:, 0], adj[:, 1], adj[:, 2], var]
                c = uf - (np.float32(s) * bv) * dx32
                upd = avg + (c - avg) / n
                avg = np.where(m, upd, avg).astype(np.float32)
                n = np.where(m, n + np.float32(1.0), n).astype(np.float32)
        dir_ = bt == DIRICHLET
        neu = bt == VON_NEUMANN
        out[sb[dir_, 0], sb[dir_, 1], sb[dir_, 2], var] = bv[dir_]
        out[sb[neu, 0], sb[neu, 1], sb[neu, 2], var] = avg[neu]
    it = maps["interior_solids"]
    out[it[:, 0], it[:, 1], it[:, 2], :] = np.float32(fill)  # :207-231
    return out
