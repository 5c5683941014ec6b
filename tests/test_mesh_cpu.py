"""UniformGridMesh and create_structured_field against the reference's own mesh
code (tests/golden/mesh_golden.npz, written by tests/golden/make_mesh_golden.py
from mesh/uniformGridMesh/grid.py:10-111, functions.py:25-90 and
mesh/mesh_functions.py:108-159): coordinate vectors with ghost nodes, the nodal
grid, node counts, cell count, dimension, and field shapes and values, bit for bit."""
import json
import os

import numpy as np
import pytest

from pde_module_b200.mesh import UniformGridMesh, create_structured_field

G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mesh_golden.npz"))
META = json.loads(str(G["meta"]))


@pytest.mark.parametrize("name", sorted(META))
def test_mesh_matches_reference(name):
    c = META[name]
    m = UniformGridMesh(c["dx"], tuple(c["nodes_per_axis"]), origin=c["origin"], ghost_cells=c["ghost_cells"])
    assert list(m.nodes_per_axis) == c["out_nodes_per_axis"]
    assert m.dimension == c["dimension"]
    for a in range(3):
        ref = G[f"{name}/coord{a}"]
        assert m.coordinate_vectors[a].dtype == ref.dtype
        assert np.array_equal(m.coordinate_vectors[a], ref)
    assert np.array_equal(m.nodal_grid, G[f"{name}/nodal_grid"])
    cells = int(np.prod([n - 1 for n in m.nodes_per_axis if n > 1]))
    assert cells == c["num_cells"]
    for kind in ("node", "cell"):
        f = create_structured_field(m, kind, 2, device="cpu")
        assert list(f.shape) == c[f"{kind}_shape"]
    fn = lambda X, Y, Z: np.stack([X + 2.0 * Y, X * Y - Z], axis=-1).astype(np.float32)
    f = create_structured_field(m, "node", 2, func=fn, device="cpu")
    assert np.array_equal(f.numpy(), G[f"{name}/node_func"])
