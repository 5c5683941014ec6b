"""Write tests/golden/ib_golden.npz from PDE_Module's ImmersedBoundary.

    python tests/golden/make_ib_golden.py [--reference PATH_TO_PDE_MODULE]

Runs the reference's FDM/boundary/immersedBoundary.py (geometry from a boolean
function, finalize(), Dirichlet / von Neumann settings, forward with a fill value)
on small seeded float32 vector fields, executing its Warp-DSL kernels through
tests/golden/warp_emu.py (warp-lang is not installable here).  Each case stores the
bitmask, the index maps finalize() builds (solid_boundary, interior_solids,
fluid_neighbors, fluid_boundary, flat_array), the boundary type and value tables,
the input field and the forward result.  Harness-side only: absent plotting
libraries that the module imports at load time are replaced by inert modules.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "ib_golden.npz")


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
    from pde_module.FDM.boundary.immersedBoundary import ImmersedBoundary

    rng = np.random.default_rng(20261204)
    store: dict[str, np.ndarray] = {}
    meta: dict[str, dict] = {}

    def mesh(shape, g, dx):
        ax = [(np.arange(n) - (g if n > 1 else 0)) * dx for n in shape]
        return np.meshgrid(*ax, indexing="ij")

    def case(name, shape, g, solids, settings, fill):
        """solids: boolean functions f(x, y, z); settings: (method, group, value, comps)."""
        N = 3 if shape[2] > 1 else 2
        dx = 1.0 / (shape[0] - 2 * g - 1)
        u = rng.standard_normal(shape + (N,)).astype(np.float32)
        field = wp.array(u, dtype=wp.types.vector(N, wp.float32))
        ib = ImmersedBoundary(field, dx, g)
        M = mesh(shape, g, dx)
        for f in solids:
            ib.from_bool_func(f, M)
        ib.finalize()
        for method, group, value, comps in settings:
            if isinstance(group, str):
                grp = group
            else:
                grp = np.arange(len(ib.solid_boundary))[group[0]::group[1]]
            if method == "dirichlet":
                ib.dirichlet_BC(grp, value, comps)
            elif method == "neumann":
                ib.vonNeumann_BC(grp, value, comps)
            else:
                ib.no_slip(grp)
        out = ib(field, fill)
        store[f"{name}/bitmask"] = np.asarray(ib.bitmask, dtype=np.int8)
        store[f"{name}/solid_boundary"] = np.asarray(ib.solid_boundary, dtype=np.int32)
        store[f"{name}/interior_solids"] = np.asarray(ib.interior_solids, dtype=np.int32)
        store[f"{name}/fluid_neighbors"] = np.asarray(ib.fluid_neighbors, dtype=np.int8)
        store[f"{name}/fluid_boundary"] = np.asarray(ib.fluid_boundary, dtype=np.int32)
        store[f"{name}/flat_array"] = np.asarray(ib.flat_array, dtype=np.int64)
        store[f"{name}/boundary_type"] = np.asarray(ib.boundary_type, dtype=np.int8)
        store[f"{name}/boundary_value"] = np.asarray(ib.boundary_value, dtype=np.float32)
        store[f"{name}/input"] = u
        store[f"{name}/output"] = np.array(out.numpy(), dtype=np.float32)
        meta[name] = dict(shape=list(shape), g=g, dx=dx, fill=fill, ncomp=N)

    disc = lambda cx, cy, r: (lambda x, y, z: (x - cx) ** 2 + (y - cy) ** 2 < r * r)
    ball = lambda cx, cy, cz, r: (lambda x, y, z: (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 < r * r)
    case("cyl_noslip", (34, 30, 1), 1, [disc(0.45, 0.5, 0.22)], [("noslip", "ALL", None, None)], 0.0)
    case("cyl_mixed", (34, 30, 1), 1, [disc(0.45, 0.5, 0.22)],
         [("dirichlet", "ALL", 1.5, 0), ("neumann", "ALL", 0.25, 1), ("neumann", (0, 3), -2.0, 0)], 3.0)
    case("two_discs", (40, 36, 1), 1, [disc(0.35, 0.45, 0.18), disc(0.55, 0.5, 0.2)],
         [("neumann", "ALL", 0.5, None), ("dirichlet", (1, 4), 0.75, 1)], -1.0)
    case("sphere", (20, 18, 16), 1, [ball(0.45, 0.5, 0.45, 0.3)],
         [("neumann", "ALL", -0.3, None), ("dirichlet", "ALL", 2.0, 2)], 0.5)
    case("box_g2", (24, 22, 1), 2, [lambda x, y, z: (np.abs(x - 0.5) < 0.2) & (np.abs(y - 0.45) < 0.25)],
         [("neumann", "ALL", 1.0, 0), ("dirichlet", "ALL", -0.5, 1)], 0.0)

    store["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **store)
    print(f"wrote {OUT}: {len(meta)} cases")


if __name__ == "__main__":
    main()
