"""CUDA path against golden fixtures made by PDE_Module's own code (see
tests/test_golden_cpu.py): bitwise on every cell the reference writes."""
import json
import os

import numpy as np
import pytest
import torch

import pde_module_b200 as P
from pde_module_b200.FDM.boundary import get_ramp_func

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fdm_golden.npz")
Z = np.load(GOLDEN)
META = json.loads(str(Z["__meta__"]))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_ours(name, m):
    u = Z[f"{name}__in"]
    ud = dev(u)
    op = m["op"]
    if op == "laplacian":
        return P.Laplacian(u.shape[3], m["dx"], m["g"])(ud, m["alpha"])
    if op == "grad":
        return P.Grad(u.shape[3], u.shape, m["dx"], m["g"], force_matrix=m["force_matrix"])(ud, m["alpha"])
    if op == "divergence":
        inputs = u.shape[3] if u.ndim == 4 else tuple(u.shape[3:5])
        return P.Divergence(inputs, u.shape, m["dx"], m["g"])(ud, m["alpha"])
    if op == "euler":
        return P.ForwardEuler()(ud, dev(Z["euler__k"]), m["dt"])
    if op == "bc":
        bc = P.GridBoundary(ud, m["dx"], m["g"])
        for kind, where, value, comps in m["spec"]:
            if kind == "dirichlet":
                bc.dirichlet_BC(where, value, comps)
            elif kind == "neumann":
                bc.vonNeumann_BC(where, value, comps)
            elif kind == "impermeable":
                bc.impermeable(where)
            elif kind == "ramp":
                bc.dirichlet_BC(where, get_ramp_func(value[0], value[1], None, comps), comps)
        return bc(ud, t=m["t"])
    if op == "heat":
        bc = P.GridBoundary(ud, m["dx"], m["g"])
        bc.dirichlet_BC("ALL", 0.0)
        fused = P.HeatRollout(bc, m["dx"], m["alpha"], m["dt"], steps_per_pass=4)(ud, m["nsteps"]).clone()
        lap, euler = P.Laplacian(1, m["dx"], m["g"]), P.ForwardEuler()
        x = ud
        for _ in range(m["nsteps"]):
            x2 = bc(x)
            x = euler(x2, lap(x2, m["alpha"]), m["dt"])
        assert torch.equal(fused, x)
        return fused
    raise KeyError(op)


@pytest.mark.parametrize("name", sorted(META))
def test_cuda_matches_reference_bitwise(name):
    ref = Z[f"{name}__out"]
    got = run_ours(name, META[name]).cpu().numpy()
    assert got.shape == ref.shape
    written = ~np.isnan(ref)
    assert np.array_equal(got[written], ref[written])
