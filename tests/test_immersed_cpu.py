"""Immersed boundary oracle (oracle/immersed.py) against the golden vectors made
by running the reference's ImmersedBoundary (tests/golden/make_ib_golden.py):
index maps and forward outputs bit for bit; plus the C ABI's argument checks,
which need no GPU."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import immersed as I
from pde_module_b200 import _lib

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ib_golden.npz")
Z = np.load(GOLDEN)
META = json.loads(bytes(Z["meta"]).decode())


@pytest.mark.parametrize("name", sorted(META))
def test_oracle_matches_reference_golden(name):
    m = META[name]
    maps = I.ib_maps(Z[f"{name}/bitmask"])
    for k in ("solid_boundary", "interior_solids", "fluid_neighbors", "fluid_boundary", "flat_array"):
        ref = Z[f"{name}/{k}"]
        assert maps[k].shape == ref.shape and np.array_equal(maps[k], ref), k
    out = I.ib_apply(Z[f"{name}/input"], maps, Z[f"{name}/boundary_type"], Z[f"{name}/boundary_value"], m["dx"],
                     m["fill"])
    assert np.array_equal(out.view(np.uint32), Z[f"{name}/output"].view(np.uint32))


def test_golden_cases_cover_both_types_and_overlaps():
    kinds = set()
    for name in META:
        kinds |= set(np.unique(Z[f"{name}/boundary_type"]).tolist())
    assert kinds == {1, 2}
    assert max(int(Z[f"{n}/bitmask"].max()) for n in META) == 2  # overlapping solids sum to 2
    assert any(META[n]["shape"][2] > 1 for n in META)            # a 3D case


def test_oracle_refuses_solids_on_the_outer_layer():
    bm = np.zeros((8, 9, 1), np.int8)
    bm[0, 4, 0] = 1
    with pytest.raises(ValueError):
        I.ib_maps(bm)


def test_c_abi_argument_checks_need_no_gpu():
    L = _lib.lib()
    g = _lib.make_grid((34, 30, 1), 1, 2, 0.03)
    nb = L.pde_ib_work_bytes(C.byref(g))
    assert nb >= 3 * 12 * ((34 * 30 + 2047) // 2048)
    bad = _lib.make_grid((34, 30, 1), 1, 3, 0.03)
    assert L.pde_ib_work_bytes(C.byref(bad)) == -1
    counts = (C.c_int64 * 3)()
    assert L.pde_ib_maps(None, C.byref(g), None, None, None, None, counts, None, nb, None) == _lib.PDE_ERR_ARG
    assert L.pde_ib_maps(C.c_void_p(16), C.byref(g), None, None, None, None, counts, C.c_void_p(64), 8,
                         None) == _lib.PDE_ERR_ARG  # work too small
    assert L.pde_ib_apply(None, None, C.byref(g), 2, None, None, None, None, 0, None, 0, 0.0,
                          None) == _lib.PDE_ERR_ARG
    assert L.pde_ib_apply(C.c_void_p(16), C.c_void_p(32), C.byref(g), 2, None, None, None, None, 5, None, 0, 0.0,
                          None) == _lib.PDE_ERR_ARG  # boundary cells without their tables
