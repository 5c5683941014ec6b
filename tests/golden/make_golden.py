"""Write tests/golden/fdm_golden.npz from PDE_Module's own finite-difference code.

    python tests/golden/make_golden.py [--reference PATH_TO_PDE_MODULE]

Runs the reference's modules (FDM Laplacian / Grad / Divergence / GridBoundary,
ForwardEuler, and the heat-equation loop of examples/2D_Heat_Equation.py) on
small seeded float32 fields, executing their Warp-DSL kernels through
tests/golden/warp_emu.py (warp-lang itself is not installable here).  Each case
stores its input, the reference's output and its parameters.  Cells the
reference never writes (its outputs come from wp.empty) are NaN in the stored
outputs.  Two harness-side shims, both outside the reference's arithmetic:
  * FDM/kernel/grad.py:33 calls create_n_point_stencil_function, which exists
    only as commented-out code (FDM/utils.py:58); Grad cannot be built as
    shipped, so a no-op of that name is injected (its result is unused);
  * plotting/JIT libraries that sibling modules import at module level and that
    are absent here (matplotlib, pyvista, numba) are replaced by inert modules;
  * GridBoundary requires grid_coordinates (functional_boundary.py:81-87) though
    only user value functions read them; the node coordinates are passed.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "fdm_golden.npz")


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
    # Sibling modules of the FDM package import plotting/JIT libraries at module
    # level (e.g. FDM/boundary/immersedBoundary.py:12 imports matplotlib); they
    # are not on this path, so absent ones are replaced by inert modules.
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
    from pde_module.FDM import Laplacian, Grad, Divergence, GridBoundary
    from pde_module.FDM.boundary.boundary_functions import get_ramp_func
    from pde_module.time_step.forwardEuler import ForwardEuler

    rng = np.random.default_rng(20261203)
    store: dict[str, np.ndarray] = {}
    meta: dict[str, dict] = {}

    def vec_field(a):
        return wp.array(a, dtype=wp.types.vector(a.shape[3], wp.float32))

    def mat_field(a):
        return wp.array(a, dtype=wp.types.matrix(a.shape[3:5], wp.float32))

    def out_np(arr):
        o = np.array(arr.numpy(), dtype=np.float32)
        return o

    def coords(shape):
        return np.zeros(tuple(shape[:3]) + (3,), dtype=np.float32)

    def rnd(shape):
        return rng.standard_normal(shape).astype(np.float32)

    def put(name, inp, out, **m):
        store[f"{name}__in"] = inp
        store[f"{name}__out"] = out
        meta[name] = m

    # ---- Laplacian (FDM/module/laplacian.py) ----
    for name, shape, g, dx, alpha in [("lap2d_n1", (12, 10, 1, 1), 1, 0.1, 0.7),
                                      ("lap3d_n2", (7, 6, 5, 2), 1, 0.25, 1.3),
                                      ("lap2d_g2", (9, 11, 1, 1), 2, 1.0 / 7.0, 1.0)]:
        u = rnd(shape)
        out = Laplacian(shape[3], dx, g)(vec_field(u), alpha)
        put(name, u, out_np(out), op="laplacian", dx=dx, g=g, alpha=alpha)

    # ---- Grad (FDM/module/grad.py) ----
    for name, shape, g, dx, alpha, force in [("grad2d_n1", (12, 10, 1, 1), 1, 0.1, -1.0, False),
                                             ("grad2d_n2", (12, 10, 1, 2), 1, 0.1, 1.0, False),
                                             ("grad3d_n1", (7, 6, 5, 1), 1, 0.2, 0.5, False),
                                             ("grad2d_force", (12, 10, 1, 1), 1, 0.3, 1.0, True)]:
        u = rnd(shape)
        out = Grad(shape[3], shape[:3], dx, g, force_matrix=force)(vec_field(u), alpha)
        put(name, u, out_np(out), op="grad", dx=dx, g=g, alpha=alpha, force_matrix=force)

    # ---- Divergence (FDM/module/divergence.py) ----
    for name, shape, g, dx, alpha in [("div2d_vec", (12, 10, 1, 2), 1, 0.1, -0.3),
                                      ("div2d_mat", (12, 10, 1, 2, 2), 1, 0.1, 1.0),
                                      ("div3d_vec", (7, 6, 5, 3), 1, 0.2, 2.0)]:
        u = rnd(shape)
        if len(shape) == 5:
            out = Divergence(tuple(shape[3:5]), shape[:3], dx, g)(mat_field(u), alpha)
        else:
            out = Divergence(shape[3], shape[:3], dx, g)(vec_field(u), alpha)
        put(name, u, out_np(out), op="divergence", dx=dx, g=g, alpha=alpha)

    # ---- ForwardEuler (time_step/forwardEuler.py) ----
    y, k = rnd((12, 10, 1, 2)), rnd((12, 10, 1, 2))
    out = ForwardEuler()(vec_field(y), vec_field(k), 0.013)
    store["euler__k"] = k
    put("euler", y, out_np(out), op="euler", dt=0.013)

    # ---- GridBoundary (FDM/boundary/functional_boundary.py) ----
    def run_bc(name, shape, g, dx, spec, t=None):
        u = rnd(shape)
        f = vec_field(u)
        bc = GridBoundary(f, dx, g, coords(shape))
        groups = []
        for kind, where, value, comps in spec:
            if kind == "dirichlet":
                bc.dirichlet_BC(where, value, comps)
            elif kind == "neumann":
                bc.vonNeumann_BC(where, value, comps)
            elif kind == "impermeable":
                bc.impermeable(where)
            elif kind == "ramp":
                bc.dirichlet_BC(where, get_ramp_func(value[0], value[1], bc.input_dtype, comps), comps)
        values = []  # (value, func, t_max) per group, in the order set_BC created them
        for kind, where, value, comps in spec:
            if kind == "impermeable":
                values += [(0.0, "constant", 1.0), (0.0, "constant", 1.0)]
            elif kind == "ramp":
                values.append((value[0], "ramp", value[1]))
            else:
                values.append((value, "constant", 1.0))
        for (key, fg), (val, fn, tmax) in zip(bc.func_groups.items(), values):
            ids = np.asarray(fg.face_ids, dtype=np.int32)
            comps = fg.output_ids if isinstance(fg.output_ids, (list, tuple)) else (fg.output_ids,)
            groups.append(dict(name=key, ids=ids.tolist(), type=int(fg.boundary_type), comps=list(comps),
                               value=float(val), func=fn, t_max=float(tmax)))
        tt = None if t is None else wp.array(np.array([t], dtype=np.float32), dtype=wp.float32)
        out = bc(f, tt)
        m = dict(op="bc", dx=dx, g=g, spec=[list(s) if not isinstance(s[2], tuple) else
                                            [s[0], s[1], list(s[2]), s[3]] for s in spec],
                 groups=groups, all_ids=np.asarray(bc.groups["ALL"]).tolist(), t=t)
        put(name, u, out_np(out), **m)

    run_bc("bc_dir_all", (12, 10, 1, 1), 1, 0.1, [("dirichlet", "ALL", 0.0, None)])
    run_bc("bc_ldc_u", (12, 10, 1, 2), 1, 0.1, [("dirichlet", "ALL", 0.0, None), ("dirichlet", "+Y", 1.0, 0)])
    run_bc("bc_neu_all", (12, 10, 1, 1), 1, 0.1, [("neumann", "ALL", 0.25, None)])
    run_bc("bc_impermeable", (12, 10, 1, 2), 1, 0.2,
           [("impermeable", "-X", None, None), ("dirichlet", "+X", 0.5, None)])
    run_bc("bc_custom_ids", (12, 10, 1, 2), 1, 0.1,
           [("neumann", "ALL", 0.0, None), ("dirichlet", [13, 14, 25, 40, 61], 0.75, 1)])
    run_bc("bc_ramp", (12, 10, 1, 1), 1, 0.1, [("ramp", "+X", (2.0, 4.0), 0)], t=1.0)
    run_bc("bc3d", (7, 6, 5, 3), 1, 0.2, [("dirichlet", "ALL", 0.0, None), ("neumann", "+Z", 1.0, 2),
                                          ("dirichlet", "-Y", 2.0, 0)])
    run_bc("bc_g2", (9, 11, 1, 1), 2, 0.1, [("dirichlet", "ALL", 0.5, None)])

    # ---- heat loop (examples/2D_Heat_Equation.py:57-65) ----
    shape, g = (18, 16, 1, 1), 1
    dx = 1.0 / 15
    alpha, dt, nsteps = 0.9, 0.2 * (1.0 / 15) ** 2 / 0.9, 10
    x = (np.arange(shape[0]) - g) * dx
    yy = (np.arange(shape[1]) - g) * dx
    X, Y = np.meshgrid(x, yy, indexing="ij")
    u0 = (rng.random(shape[:3]) * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2)[:, :, None] / (2 * 0.1 ** 2)))
    u0 = u0.astype(np.float32)[..., None]
    u = vec_field(u0)
    bc = GridBoundary(u, dx, g, coords(shape))
    bc.dirichlet_BC("ALL", 0.0)
    euler = ForwardEuler(u.dtype)
    lapl = Laplacian(1, dx, g)
    for _ in range(nsteps):
        u2 = bc(u)
        stencil = lapl(u2, alpha)
        u = euler(u2, stencil, dt)
    put("heat", u0, out_np(u), op="heat", dx=dx, g=g, alpha=alpha, dt=dt, nsteps=nsteps)

    store["__meta__"] = np.array(json.dumps(meta))
    np.savez_compressed(OUT, **store)
    print(f"wrote {OUT}: {len(meta)} cases")


if __name__ == "__main__":
    main()
