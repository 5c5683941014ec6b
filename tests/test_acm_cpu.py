"""Element-wise, absorbing-layer and Runge-Kutta oracle (oracle/acm.py) against the
golden vectors made by running the reference's OuterProduct, scalarVectorMult,
FarField, ViscousDampingLayer and RungeKatta1/2 (tests/golden/make_acm_golden.py),
bit for bit on every value the reference writes; plus the C ABI's argument checks."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import acm, fdm
from pde_module_b200 import _lib

Z = np.load(os.path.join(os.path.dirname(__file__), "golden", "acm_golden.npz"))
META = json.loads(bytes(Z["meta"]).decode())


def same(a, ref):
    """Bitwise on the values the reference wrote (NaN marks cells it never writes)."""
    m = ~np.isnan(ref)
    return a.shape == ref.shape and np.array_equal(a[m].view(np.uint32), ref[m].view(np.uint32))


def rk_groups(m):
    sh = tuple(m["shape"])
    G = fdm.exterior_groups(sh, 1)
    out = []
    for n, groups in m["specs"]:
        gl = []
        for grp, typ, val, comps in groups:
            c = tuple(range(n)) if comps is None else ((comps,) if isinstance(comps, int) else tuple(comps))
            gl.append(dict(ids=G[grp], type=typ, value=val, comps=c, func="constant"))
        out.append(gl)
    return out


@pytest.mark.parametrize("name", sorted(META))
def test_oracle_matches_reference_golden(name):
    m = META[name]
    k = m["kind"]
    if k == "outer":
        assert same(acm.outer(Z[f"{name}/A"], Z[f"{name}/B"]), Z[f"{name}/out"])
    elif k == "scalar_mult":
        assert same(acm.scalar_mult(Z[f"{name}/A"], Z[f"{name}/B"]), Z[f"{name}/out"])
    elif k in ("farfield", "damping"):
        sh = tuple(m["shape"])
        assert np.array_equal(acm.layer_points(sh, m["num_layers"], m["exclude"]), Z[f"{name}/points"])
        if k == "farfield":
            o = acm.farfield(Z[f"{name}/input"], sh, m["num_layers"], m["beta"], m["cond"], m["sigma"], m["exclude"])
        else:
            o = acm.damping(Z[f"{name}/input"], sh, m["num_layers"], m["p"], m["cmax"], m["exclude"])
        assert same(o, Z[f"{name}/out"])
    else:
        fields = [Z[f"{name}/u0_{i}"] for i in range(m["nfields"])]
        ys = acm.runge_kutta(2 if k == "RungeKatta2" else 1, fields, rk_groups(m), m["alphas"], m["dx"], 1, m["dt"],
                             m["steps"])
        for i, y in enumerate(ys):
            assert same(y, Z[f"{name}/out_{i}"])


def test_layer_depth_is_one_to_num_layers():
    for shape, L, excl in (((24, 20, 1), 4, ()), ((14, 12, 10), 3, ("+Z",)), ((30, 9, 1), 5, ("-X", "+Y"))):
        d = acm.layer_depth(acm.layer_points(shape, L, excl), shape, L)
        assert d.min() >= 1 and d.max() <= L


def test_c_abi_argument_checks_need_no_gpu():
    L = _lib.lib()
    assert L.pde_outer(None, None, None, 4, 2, 2, None) == _lib.PDE_ERR_ARG
    assert L.pde_scalar_mult(C.c_void_p(16), C.c_void_p(32), C.c_void_p(48), 4, 0, None) == _lib.PDE_ERR_ARG
    cond = (C.c_float * 17)()
    assert L.pde_layer_apply(C.c_void_p(16), C.c_void_p(32), 17, C.c_void_p(48), C.c_void_p(64), 3, 1.0, cond,
                             None) == _lib.PDE_ERR_ARG  # far-field value longer than 16 floats
    assert L.pde_layer_apply(C.c_void_p(16), C.c_void_p(32), 2, None, None, 3, 1.0, None,
                             None) == _lib.PDE_ERR_ARG  # points without their profile


def test_runge_kutta_refuses_mismatched_signatures():
    from pde_module_b200.time_step import RungeKatta2, SignatureMismatchError
    with pytest.raises(SignatureMismatchError):
        RungeKatta2([1], f=lambda t, u: (u,), bc=lambda t, u, p: (u, p))
