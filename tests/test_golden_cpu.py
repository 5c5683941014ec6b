"""The oracle against golden fixtures made by PDE_Module's own code.

tests/golden/fdm_golden.npz was written by tests/golden/make_golden.py, which
runs the reference's Laplacian, Grad, Divergence, GridBoundary, ForwardEuler
modules and its heat-equation loop through the Warp-DSL executor
tests/golden/warp_emu.py.  Bitwise equality on every cell the reference
writes (its never-written cells are NaN in the fixtures)."""
import json
import os

import numpy as np
import pytest

from oracle import fdm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fdm_golden.npz")
Z = np.load(GOLDEN)
META = json.loads(str(Z["__meta__"]))


def oracle_case(name, m, dtype=np.float32):
    u = Z[f"{name}__in"]
    op = m["op"]
    if op == "laplacian":
        return fdm.laplacian(u, m["dx"], m["g"], m["alpha"], dtype=dtype)
    if op == "grad":
        return fdm.grad(u, m["dx"], m["g"], m["alpha"], force_matrix=m["force_matrix"], dtype=dtype)
    if op == "divergence":
        return fdm.divergence(u, m["dx"], m["g"], m["alpha"], dtype=dtype)
    if op == "euler":
        return fdm.forward_euler(u, Z["euler__k"], m["dt"], dtype=dtype)
    if op == "bc":
        return fdm.bc_apply(u, bc_groups(m), m["dx"], m["g"], t=m["t"] or 0.0, dtype=dtype)
    if op == "heat":
        groups = fdm.standard_groups(u.shape, m["g"], [("ALL", fdm.DIRICHLET, 0.0, (0,))])
        return fdm.heat_rollout(u, groups, m["dx"], m["g"], m["alpha"], m["dt"], m["nsteps"], dtype=dtype)
    raise KeyError(op)


def bc_groups(m):
    return [dict(ids=np.array(G["ids"], dtype=np.int32), type=G["type"], comps=tuple(G["comps"]),
                 value=G["value"], func=G["func"], t_max=G["t_max"]) for G in m["groups"]]


def test_fixture_covers_the_path():
    ops = {m["op"] for m in META.values()}
    assert ops == {"laplacian", "grad", "divergence", "euler", "bc", "heat"}
    assert len(META) >= 20


@pytest.mark.parametrize("name", sorted(META))
def test_oracle_matches_reference_bitwise(name):
    m = META[name]
    ref = Z[f"{name}__out"]
    got = oracle_case(name, m)
    assert got.shape == ref.shape
    written = ~np.isnan(ref)
    assert written.any()
    assert np.array_equal(got[written], ref[written])


@pytest.mark.parametrize("name", [n for n in sorted(META) if META[n]["op"] == "bc"])
def test_boundary_group_ids_match_reference(name):
    m = META[name]
    shape = Z[f"{name}__in"].shape
    ours = fdm.exterior_groups(shape, m["g"])
    np.testing.assert_array_equal(ours["ALL"], np.array(m["all_ids"], dtype=np.int32))
    for G in m["groups"]:
        for key in ("-X", "+X", "-Y", "+Y", "-Z", "+Z", "ALL"):
            if key in ours and len(ours[key]) == len(G["ids"]) and np.array_equal(ours[key], G["ids"]):
                break
        else:
            assert G["name"].startswith("BC_Group"), "a standard group's ids differ from the reference's"
