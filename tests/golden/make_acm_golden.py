"""Write tests/golden/acm_golden.npz from PDE_Module's element-wise, absorbing-layer
and Runge-Kutta modules.

    python tests/golden/make_acm_golden.py [--reference PATH_TO_PDE_MODULE]

Runs the reference's OuterProduct and scalarVectorMult (FDM/module/elementWiseOps.py),
FarField (FDM/module/farfield.py), ViscousDampingLayer
(FDM/module/viscousDampingLayer.py) and RungeKatta1 / RungeKatta2
(time_step/rungeKatta.py, driving the reference's GridBoundary and Laplacian) on
small seeded float32 fields, executing their Warp-DSL kernels through
tests/golden/warp_emu.py.  Each case stores its inputs, parameters and outputs.
Harness-side only: inert stand-ins for absent plotting libraries, node
coordinates passed to GridBoundary (only user value functions read them), and the
ForwardEuler.input_dtype attribute that RungeKatta's argument check reads but
whose assignment is commented out in time_step/forwardEuler.py:24 (without it the
reference's Runge-Kutta classes fail at their first call).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "acm_golden.npz")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PDE_MODULE_REFERENCE"),
                    help="root of the PDE_Module source tree (or set PDE_MODULE_REFERENCE)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set PDE_MODULE_REFERENCE to the PDE_Module source tree")

    sys.path.insert(0, HERE)
    import warp_emu
    wp = warp_emu.install()
    import importlib.util
    import types as pytypes
    for name in ("matplotlib", "matplotlib.pyplot", "pyvista", "numba"):
        top = name.split(".")[0]
        if top in sys.modules or importlib.util.find_spec(top) is None:
            mod = pytypes.ModuleType(name)
            mod.__getattr__ = lambda n, _nm=name: warp_emu._Anything(f"{_nm}.{n}")
            sys.modules[name] = mod
    sys.path.insert(0, os.path.join(args.reference, "src"))
    import pde_module.FDM.kernel.grad as kgrad
    kgrad.create_n_point_stencil_function = lambda *a, **k: None
    from pde_module.FDM import OuterProduct, scalarVectorMult, FarField, ViscousDampingLayer, Laplacian, GridBoundary
    from pde_module.time_step.rungeKatta import RungeKatta1, RungeKatta2

    rng = np.random.default_rng(20261205)
    store: dict[str, np.ndarray] = {}
    meta: dict[str, dict] = {}
    f32 = wp.float32

    def field(a):
        if a.ndim == 5:
            return wp.array(a, dtype=wp.types.matrix(a.shape[3:5], f32))
        return wp.array(a, dtype=wp.types.vector(a.shape[3], f32))

    def rnd(shape):
        return rng.standard_normal(shape).astype(np.float32)

    def out(arr):
        return np.array(arr.numpy(), dtype=np.float32)

    # ---- element-wise ------------------------------------------------------
    for name, shape, n in (("outer2", (12, 10, 1), 2), ("outer3", (8, 7, 6), 3)):
        A, B = rnd(shape + (n,)), rnd(shape + (n,))
        op = OuterProduct(n, n)
        res = op(field(A), field(B))
        store[f"{name}/A"], store[f"{name}/B"], store[f"{name}/out"] = A, B, out(res)
        meta[name] = dict(kind="outer")
    for name, shape, comps in (("svm_vec", (11, 9, 1), (2,)), ("svm_mat", (6, 5, 4), (2, 2))):
        A, B = rnd(shape + (1,)), rnd(shape + comps)
        op = scalarVectorMult(comps[0] if len(comps) == 1 else comps)
        res = op(field(A), field(B))
        store[f"{name}/A"], store[f"{name}/B"], store[f"{name}/out"] = A, B, out(res)
        meta[name] = dict(kind="scalar_mult")

    # ---- absorbing layers --------------------------------------------------
    def coords(shape):
        return np.zeros(tuple(shape[:3]) + (3,), dtype=np.float32)

    ff_cases = [
        ("ff_vec2", (24, 20, 1), 2, 4, 2.0, (), [1.0, -0.5], 3.7),
        ("ff_vec2_excl", (24, 20, 1), 2, 5, 1.5, ("-X",), [0.25, 0.75], 1.3),
        ("ff_scalar3d", (14, 12, 10), 1, 3, 2.0, ("+Z",), [2.0], 0.9),
        ("ff_mat", (16, 15, 1), (2, 2), 3, 3.0, (), [[1.0, 0.0], [0.5, -1.0]], 2.2),
    ]
    for name, shape, inputs, L, beta, excl, cond, sigma in ff_cases:
        comps = (inputs,) if isinstance(inputs, int) else inputs
        u = rnd(shape + comps)
        dx = 1.0 / (shape[0] - 3)
        ff = FarField(inputs, L, beta, shape, dx, 1)
        if excl:
            ff.exclude(*excl)
        cval = wp.types.vector(comps[0], f32)(cond) if len(comps) == 1 else wp.types.matrix(comps, f32)(cond)
        res = ff(field(u), cval, sigma)
        store[f"{name}/input"], store[f"{name}/out"] = u, out(res)
        store[f"{name}/points"] = np.asarray(ff.outer_layers, dtype=np.int32)
        meta[name] = dict(kind="farfield", shape=list(shape), comps=list(comps), num_layers=L, beta=beta,
                          exclude=list(excl), cond=np.asarray(cond, np.float32).ravel().tolist(), sigma=sigma)
    vd_cases = [
        ("vd_vec2", (22, 18, 1), 2, 5, 2, (), 0.8),
        ("vd_vec3_excl", (12, 11, 10), 3, 3, 3, ("+Z", "-Y"), 1.7),
    ]
    for name, shape, inputs, L, p, excl, cmax in vd_cases:
        u = rnd(shape + (inputs,))
        dx = 1.0 / (shape[0] - 3)
        vd = ViscousDampingLayer(inputs, L, shape, dx, 1, p)
        if excl:
            vd.exclude(*excl)
        res = vd(field(u), cmax)
        store[f"{name}/input"], store[f"{name}/out"] = u, out(res)
        store[f"{name}/points"] = np.asarray(vd.outer_layers, dtype=np.int32)
        meta[name] = dict(kind="damping", shape=list(shape), comps=[inputs], num_layers=L, p=p,
                          exclude=list(excl), cmax=cmax)

    # ---- Runge-Kutta: heat-like fields with boundary groups, three steps ----
    def rk_case(name, cls, shape, specs, alphas, steps):
        g = 1
        dx = 1.0 / (shape[0] - 2 * g - 1)
        dt = 0.1 * dx * dx
        fields, bcs, laps, dtypes = [], [], [], []
        for (n, groups), alpha in zip(specs, alphas):
            u0 = rng.random(shape + (n,)).astype(np.float32)
            fa = field(u0)
            bc = GridBoundary(fa, dx, g, coords(shape))
            for grp, typ, val, comps in groups:
                if typ == 1:
                    bc.dirichlet_BC(grp, val, comps)
                else:
                    bc.vonNeumann_BC(grp, val, comps)
            fields.append(fa)
            bcs.append(bc)
            laps.append(Laplacian(n, dx, g))
            dtypes.append(fa.dtype)
            store[f"{name}/u0_{len(fields) - 1}"] = u0

        def bc_fn(t, *arrs):
            return tuple(b(a) for b, a in zip(bcs, arrs))

        def f_fn(t, *arrs):
            return tuple(l(a, al) for l, a, al in zip(laps, arrs, alphas))

        rk = cls(dtypes if len(dtypes) > 1 else dtypes[0], f=f_fn, bc=bc_fn)
        # Shim: check_args (rungeKatta.py:54-60, :124-131) reads ForwardEuler.input_dtype,
        # whose assignment is commented out in time_step/forwardEuler.py:24; restore it.
        for group in ("forwardEulers", "forwardEulers_1", "forwardEulers_2"):
            for fe, dt_ in zip(getattr(rk, group, ()), dtypes):
                fe.input_dtype = dt_
        arrs = tuple(fields)
        t = 0.0
        for _ in range(steps):
            arrs = rk(t, dt, *arrs)
            t += dt
        for i, a in enumerate(arrs):
            store[f"{name}/out_{i}"] = out(a)
        meta[name] = dict(kind=cls.__name__, shape=list(shape), dx=dx, dt=dt, steps=steps, alphas=list(alphas),
                          specs=[[n, [list(gr[:3]) + [list(gr[3]) if isinstance(gr[3], tuple) else gr[3]]
                                      for gr in groups]] for n, groups in specs], nfields=len(specs))

    rk_case("rk2_two", RungeKatta2, (14, 12, 1),
            [(2, [("ALL", 1, 0.0, None), ("+Y", 1, 1.0, 0)]), (1, [("ALL", 2, 0.0, None)])], [0.7, 1.3], 3)
    rk_case("rk1_one", RungeKatta1, (13, 15, 1), [(1, [("ALL", 1, 0.5, None)])], [1.0], 2)

    store["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **store)
    print(f"wrote {OUT}: {len(meta)} cases")


if __name__ == "__main__":
    main()
