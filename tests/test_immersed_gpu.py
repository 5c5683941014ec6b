"""Immersed boundary on the GPU: the module (geometry from a boolean function,
finalize on the device, settings, forward) on the cases the reference ran for the
golden vectors (tests/golden/make_ib_golden.py), maps and outputs bit for bit;
the C ABI against the oracle on larger grids (2D cylinder, 3D sphere, random
blobs with overlaps), out of place and in place; solids on the outer layer refused."""
import ctypes as C
import json
import os

import numpy as np
import pytest
import torch

from oracle import immersed as I
import pde_module_b200 as P
from pde_module_b200 import _lib

pytestmark = pytest.mark.gpu

Z = np.load(os.path.join(os.path.dirname(__file__), "golden", "ib_golden.npz"))
META = json.loads(bytes(Z["meta"]).decode())

disc = lambda cx, cy, r: (lambda x, y, z: (x - cx) ** 2 + (y - cy) ** 2 < r * r)
ball = lambda cx, cy, cz, r: (lambda x, y, z: (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 < r * r)
# the geometry and settings make_ib_golden.py gave the reference
CASES = {
    "cyl_noslip": ([disc(0.45, 0.5, 0.22)], [("noslip", "ALL", None, None)]),
    "cyl_mixed": ([disc(0.45, 0.5, 0.22)],
                  [("dirichlet", "ALL", 1.5, 0), ("neumann", "ALL", 0.25, 1), ("neumann", (0, 3), -2.0, 0)]),
    "two_discs": ([disc(0.35, 0.45, 0.18), disc(0.55, 0.5, 0.2)],
                  [("neumann", "ALL", 0.5, None), ("dirichlet", (1, 4), 0.75, 1)]),
    "sphere": ([ball(0.45, 0.5, 0.45, 0.3)], [("neumann", "ALL", -0.3, None), ("dirichlet", "ALL", 2.0, 2)]),
    "box_g2": ([lambda x, y, z: (np.abs(x - 0.5) < 0.2) & (np.abs(y - 0.45) < 0.25)],
               [("neumann", "ALL", 1.0, 0), ("dirichlet", "ALL", -0.5, 1)]),
}


def mesh(shape, g, dx):
    ax = [(np.arange(n) - (g if n > 1 else 0)) * dx for n in shape]
    return np.meshgrid(*ax, indexing="ij")


@pytest.mark.parametrize("name", sorted(CASES))
def test_module_matches_reference_golden(name):
    m = META[name]
    shape, g, dx, fill = tuple(m["shape"]), m["g"], m["dx"], m["fill"]
    u = torch.from_numpy(Z[f"{name}/input"]).cuda()
    ib = P.ImmersedBoundary(u, dx, g)
    for f in CASES[name][0]:
        ib.from_bool_func(f, mesh(shape, g, dx))
    assert np.array_equal(ib.bitmask, Z[f"{name}/bitmask"])
    ib.finalize()
    for k in ("solid_boundary", "interior_solids", "fluid_neighbors", "fluid_boundary", "flat_array"):
        got, ref = getattr(ib, k), Z[f"{name}/{k}"]
        assert got.shape == ref.shape and np.array_equal(got, ref), k
    for method, group, value, comps in CASES[name][1]:
        grp = group if isinstance(group, str) else np.arange(len(ib.solid_boundary))[group[0]::group[1]]
        if method == "dirichlet":
            ib.dirichlet_BC(grp, value, comps)
        elif method == "neumann":
            ib.vonNeumann_BC(grp, value, comps)
        else:
            ib.no_slip(grp)
    assert np.array_equal(ib.boundary_type, Z[f"{name}/boundary_type"])
    assert np.array_equal(ib.boundary_value, Z[f"{name}/boundary_value"])
    out = ib(u, fill)
    assert out.data_ptr() != u.data_ptr()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), Z[f"{name}/output"].view(np.uint32))
    again = ib(u, fill)  # the module reuses its output
    assert again.data_ptr() == out.data_ptr()


def _abi_maps(bm_np, shape, g, dx):
    L = _lib.lib()
    grid = _lib.make_grid(shape, g, 2, dx)
    bm = torch.from_numpy(bm_np).cuda()
    nb = L.pde_ib_work_bytes(C.byref(grid))
    work = torch.empty(nb, dtype=torch.uint8, device="cuda")
    counts = (C.c_int64 * 3)()
    rc = L.pde_ib_maps(C.c_void_p(bm.data_ptr()), C.byref(grid), None, None, None, None, counts,
                       C.c_void_p(work.data_ptr()), nb, None)
    if rc:
        return rc, None
    n_sb, n_is, n_fb = (int(c) for c in counts)
    D = sum(1 for s in shape if s > 1)
    sb = torch.full((max(n_sb, 1), 3), -7, dtype=torch.int32, device="cuda")
    fnb = torch.full((max(n_sb, 1), D, 2), -7, dtype=torch.int8, device="cuda")
    isd = torch.full((max(n_is, 1), 3), -7, dtype=torch.int32, device="cuda")
    fb = torch.full((max(n_fb, 1), 3), -7, dtype=torch.int32, device="cuda")
    rc = L.pde_ib_maps(C.c_void_p(bm.data_ptr()), C.byref(grid), C.c_void_p(sb.data_ptr()), C.c_void_p(fnb.data_ptr()),
                       C.c_void_p(isd.data_ptr()), C.c_void_p(fb.data_ptr()), counts, C.c_void_p(work.data_ptr()), nb,
                       None)
    assert rc == 0
    return 0, dict(grid=grid, sb=sb[:n_sb], fnb=fnb[:n_sb], isd=isd[:n_is], fb=fb[:n_fb])


def _geometry(kind, rng):
    if kind == "cylinder":
        shape, g = (258, 202, 1), 1
        dx = 1.0 / 256
        x, y, z = mesh(shape, g, dx)
        return (((x - 0.3) ** 2 + (y - 0.4) ** 2) < 0.1 ** 2).astype(np.int8), shape, g, dx
    if kind == "sphere":
        shape, g = (66, 60, 70), 2
        dx = 1.0 / 61
        x, y, z = mesh(shape, g, dx)
        return (((x - 0.5) ** 2 + (y - 0.45) ** 2 + (z - 0.55) ** 2) < 0.3 ** 2).astype(np.int8), shape, g, dx
    shape, g = (90, 77, 1), 1
    bm = np.zeros(shape, np.int8)
    for _ in range(12):  # overlapping random rectangles: values up to several
        x0, y0 = rng.integers(1, 70), rng.integers(1, 60)
        bm[x0:x0 + rng.integers(1, 19), y0:y0 + rng.integers(1, 16), 0] += 1
    bm[0, :, :] = 0
    bm[-1, :, :] = 0
    bm[:, 0, :] = 0
    bm[:, -1, :] = 0
    return bm, shape, g, 1.0 / 88


@pytest.mark.parametrize("kind", ["cylinder", "sphere", "blobs"])
@pytest.mark.parametrize("in_place", [False, True])
def test_abi_maps_and_apply_match_oracle(kind, in_place):
    rng = np.random.default_rng(5)
    bm, shape, g, dx = _geometry(kind, rng)
    rc, M = _abi_maps(bm, shape, g, dx)
    assert rc == 0
    ref = I.ib_maps(bm)
    assert np.array_equal(M["sb"].cpu().numpy(), ref["solid_boundary"])
    assert np.array_equal(M["fnb"].cpu().numpy(), ref["fluid_neighbors"])
    assert np.array_equal(M["isd"].cpu().numpy(), ref["interior_solids"])
    assert np.array_equal(M["fb"].cpu().numpy(), ref["fluid_boundary"])
    N = 3 if shape[2] > 1 else 2
    n_sb = len(ref["solid_boundary"])
    u0 = rng.standard_normal(shape + (N,)).astype(np.float32)
    btype = rng.integers(0, 3, size=(n_sb, N)).astype(np.int8)  # 0 = leave the cell as it is
    bval = rng.standard_normal((n_sb, N)).astype(np.float32)
    u = torch.from_numpy(u0).cuda()
    out = u if in_place else torch.full_like(u, float("nan"))
    bt, bv = torch.from_numpy(btype).cuda(), torch.from_numpy(bval).cuda()
    rc = _lib.lib().pde_ib_apply(C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()), C.byref(M["grid"]), N,
                                 C.c_void_p(M["sb"].data_ptr()), C.c_void_p(M["fnb"].data_ptr()),
                                 C.c_void_p(bt.data_ptr()), C.c_void_p(bv.data_ptr()), n_sb,
                                 C.c_void_p(M["isd"].data_ptr()), len(ref["interior_solids"]), 1.25, None)
    assert rc == 0
    expect = I.ib_apply(u0, ref, btype, bval, dx, 1.25)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), expect.view(np.uint32))


def test_solids_on_the_outer_layer_are_refused():
    shape = (20, 18, 1)
    bm = np.zeros(shape, np.int8)
    bm[5:9, 0:4, 0] = 1  # touches y = 0
    rc, _ = _abi_maps(bm, shape, 1, 0.05)
    assert rc == _lib.PDE_ERR_ARG
    u = torch.zeros(shape + (2,), device="cuda")
    ib = P.ImmersedBoundary(u, 0.05, 1)
    ib.bitmask[:] = bm
    with pytest.raises(ValueError):
        ib.finalize()


def test_all_fluid_grid_has_empty_maps_and_copies():
    shape = (16, 12, 1)
    u = torch.randn(shape + (2,), device="cuda")
    ib = P.ImmersedBoundary(u, 0.1, 1)
    ib.finalize()
    assert ib.n_boundary == 0 and ib.n_interior == 0 and len(ib.fluid_boundary) == 0
    assert torch.equal(ib(u), u)
