"""Element-wise, absorbing-layer and Runge-Kutta modules on the GPU: on the cases
the reference ran for the golden vectors (tests/golden/make_acm_golden.py) bit for
bit, and against the oracle on larger grids; modules reuse their outputs."""
import json
import os

import numpy as np
import pytest
import torch

from oracle import acm, fdm
import pde_module_b200 as P

pytestmark = pytest.mark.gpu

Z = np.load(os.path.join(os.path.dirname(__file__), "golden", "acm_golden.npz"))
META = json.loads(bytes(Z["meta"]).decode())


def same(a, ref):
    m = ~np.isnan(ref)
    return a.shape == ref.shape and np.array_equal(a[m].view(np.uint32), ref[m].view(np.uint32))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("name", [n for n in sorted(META) if META[n]["kind"] in ("outer", "scalar_mult")])
def test_elementwise_matches_golden(name):
    A, B = dev(Z[f"{name}/A"]), dev(Z[f"{name}/B"])
    if META[name]["kind"] == "outer":
        n = A.shape[3]
        op = P.OuterProduct(n, n)
    else:
        op = P.scalarVectorMult(tuple(B.shape[3:]) if B.dim() == 5 else B.shape[3])
    out = op(A, B)
    assert same(out.cpu().numpy(), Z[f"{name}/out"])
    assert op(A, B).data_ptr() == out.data_ptr()


@pytest.mark.parametrize("name", [n for n in sorted(META) if META[n]["kind"] in ("farfield", "damping")])
def test_layers_match_golden(name):
    m = META[name]
    shape, comps = tuple(m["shape"]), tuple(m["comps"])
    u = dev(Z[f"{name}/input"])
    inputs = comps[0] if len(comps) == 1 else comps
    dx = 1.0 / (shape[0] - 3)
    if m["kind"] == "farfield":
        mod = P.FarField(inputs, m["num_layers"], m["beta"], shape, dx, 1)
        if m["exclude"]:
            mod.exclude(*m["exclude"])
        out = mod(u, np.asarray(m["cond"], np.float32).reshape(comps), m["sigma"])
    else:
        mod = P.ViscousDampingLayer(inputs, m["num_layers"], shape, dx, 1, m["p"])
        if m["exclude"]:
            mod.exclude(*m["exclude"])
        out = mod(u, m["cmax"])
    assert np.array_equal(mod.outer_layers, Z[f"{name}/points"])
    assert same(out.cpu().numpy(), Z[f"{name}/out"])


@pytest.mark.parametrize("name", [n for n in sorted(META) if META[n]["kind"].startswith("RungeKatta")])
def test_runge_kutta_matches_golden(name):
    m = META[name]
    shape, dx, dt = tuple(m["shape"]), m["dx"], m["dt"]
    fields, bcs, laps = [], [], []
    for i, (n, groups) in enumerate(m["specs"]):
        u = dev(Z[f"{name}/u0_{i}"])
        bc = P.GridBoundary(u, dx, 1)
        for grp, typ, val, comps in groups:
            (bc.dirichlet_BC if typ == 1 else bc.vonNeumann_BC)(grp, val, comps)
        fields.append(u)
        bcs.append(bc)
        laps.append(P.Laplacian(n, dx, 1))
    alphas = m["alphas"]

    def bc_fn(t, *arrs):
        return tuple(b(a) for b, a in zip(bcs, arrs))

    def f_fn(t, *arrs):
        return tuple(l(a, al) for l, a, al in zip(laps, arrs, alphas))

    cls = P.RungeKatta2 if m["kind"] == "RungeKatta2" else P.RungeKatta1
    rk = cls([f.shape[3] for f in fields], f=f_fn, bc=bc_fn)
    arrs, t = tuple(fields), 0.0
    for _ in range(m["steps"]):
        arrs = rk(t, dt, *arrs)
        t += dt
    for i, a in enumerate(arrs):
        assert same(a.cpu().numpy(), Z[f"{name}/out_{i}"])


def test_large_layers_and_products_match_oracle():
    rng = np.random.default_rng(8)
    shape = (130, 97, 1)
    u = rng.standard_normal(shape + (2,)).astype(np.float32)
    ff = P.FarField(2, 15, 2.0, shape, 0.01, 1)
    ff.exclude("-X")
    out = ff(dev(u), np.array([1.0, 0.0], np.float32), 25.0).cpu().numpy()
    assert np.array_equal(out, acm.farfield(u, shape, 15, 2.0, [1.0, 0.0], 25.0, ("-X",)))
    shape3 = (40, 36, 44)
    du = rng.standard_normal(shape3 + (3,)).astype(np.float32)
    vd = P.ViscousDampingLayer(3, 6, shape3, 0.02, 1, p=3)
    got = vd(dev(du), 4.5).cpu().numpy()
    assert np.array_equal(got, acm.damping(du, shape3, 6, 3.0, 4.5))
    A = rng.standard_normal(shape3 + (3,)).astype(np.float32)
    B = rng.standard_normal(shape3 + (3,)).astype(np.float32)
    assert np.array_equal(P.OuterProduct(3, 3)(dev(A), dev(B)).cpu().numpy(), acm.outer(A, B))
    s = rng.standard_normal(shape3 + (1,)).astype(np.float32)
    assert np.array_equal(P.scalarVectorMult(3)(dev(s), dev(B)).cpu().numpy(), acm.scalar_mult(s, B))

