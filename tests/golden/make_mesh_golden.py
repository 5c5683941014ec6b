"""Write tests/golden/mesh_golden.npz from PDE_Module's own mesh code.

    python tests/golden/make_mesh_golden.py [--reference PATH_TO_PDE_MODULE]

Builds the reference's UniformGridMesh (mesh/uniformGridMesh/grid.py:10-111 on
functions.py:25-90) for 2D and 3D node counts, several ghost widths, spacings
and origins, and stores per case the coordinate vectors (ghost nodes
included), the nodal grid, nodes per axis, cell count and dimension; and the
shapes and values of create_structured_warp_field (mesh/mesh_functions.py:
108-159) on nodes and cells, with and without a value function.  Warp arrays go
through tests/golden/warp_emu.py (warp-lang is not installable here); absent
plotting/JIT libraries imported by sibling modules are replaced by inert ones.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "mesh_golden.npz")

CASES = [
    # name, dx, nodes_per_axis, origin, ghost_cells
    ("2d_g1", 1.0 / 31, (32, 24, 1), None, 1),
    ("2d_g0_origin", 0.05, (21, 17, 1), (0.5, -0.25, 0.0), None),
    ("3d_g2", 0.1, (11, 9, 7), (0.1, 0.2, 0.3), 2),
    ("3d_g1_fine", 1.0 / 63, (64, 17, 33), None, 1),
]


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
    from pde_module.mesh.uniformGridMesh.grid import UniformGridMesh
    from pde_module.mesh.mesh_functions import create_structured_warp_field

    store: dict[str, np.ndarray] = {}
    meta: dict[str, dict] = {}
    for name, dx, npa, origin, g in CASES:
        m = UniformGridMesh(dx, npa, origin=origin, ghost_cells=g)
        for a, v in enumerate(m.coordinate_vectors):
            store[f"{name}/coord{a}"] = np.asarray(v)
        store[f"{name}/nodal_grid"] = np.asarray(m.nodal_grid)
        meta[name] = dict(dx=dx, nodes_per_axis=list(npa), origin=origin, ghost_cells=g,
                          out_nodes_per_axis=[int(n) for n in m.nodes_per_axis], num_cells=int(m.num_cells),
                          dimension=int(m.dimension))
        for kind in ("node", "cell"):
            f = create_structured_warp_field(m, kind, 2)
            meta[name][f"{kind}_shape"] = [int(s) for s in np.asarray(f.numpy()).shape]
        fn = lambda X, Y, Z: np.stack([X + 2.0 * Y, X * Y - Z], axis=-1).astype(np.float32)
        f = create_structured_warp_field(m, "node", 2, func=fn)
        store[f"{name}/node_func"] = np.asarray(f.numpy(), dtype=np.float32)
    np.savez_compressed(OUT, meta=np.array(json.dumps(meta)), **store)
    print(f"wrote {OUT}: {len(CASES)} cases")


if __name__ == "__main__":
    main()
