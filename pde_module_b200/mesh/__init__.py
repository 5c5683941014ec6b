"""Uniform node-centred grids and field construction.

Reference: mesh/uniformGridMesh/grid.py:10-111 (UniformGridMesh),
mesh/uniformGridMesh/functions.py:25-90 (coordinates with ghost nodes),
mesh/mesh_functions.py:108-159 (create_structured_warp_field).  Only the parts
the finite-difference path consumes: coordinates, meshgrid and AoS fields as
torch CUDA tensors.
"""
from __future__ import annotations

from math import prod
from typing import Callable, Optional

import numpy as np
import torch


class UniformGridMesh:
    def __init__(self, dx: float, nodes_per_axis, origin=None, ghost_cells: int | None = None,
                 float_dtype=np.float32) -> None:
        dx = float_dtype(dx)
        self.dx = dx
        self.float_dtype = float_dtype
        self.ghost_cells = 0 if ghost_cells is None else int(ghost_cells)
        assert self.ghost_cells >= 0
        self.origin = np.zeros(3, dtype=float_dtype) if origin is None else np.array(origin, dtype=float_dtype)
        assert len(self.origin) == 3, "Origin must be a tuple of length 3"
        vecs = [np.arange(0, n, dtype=self.origin.dtype) * dx - o for n, o in zip(nodes_per_axis, self.origin)]
        g = self.ghost_cells
        if g:
            out = []
            for v in vecs:
                if len(v) == 1:
                    out.append(v)
                    continue
                left = np.array([v[0] - k * dx for k in range(1, g + 1)])
                right = np.array([v[-1] + k * dx for k in range(1, g + 1)])
                out.append(np.concatenate((left, v, right), dtype=v.dtype))
            vecs = out
        self.coordinate_vectors = tuple(vecs)
        mg = np.meshgrid(*vecs, indexing="ij")
        self.nodal_grid = np.stack(mg, axis=-1)
        self.meshgrid = [self.nodal_grid[..., i] for i in range(3)]
        self.nodes_per_axis = tuple(len(v) for v in vecs)
        self.grid_shape = self.nodes_per_axis
        self.dimension = sum(1 for n in self.nodes_per_axis if n > 1)
        assert 1 <= self.dimension <= 3
        self.num_nodes = prod(self.nodes_per_axis)


def create_structured_field(mesh: UniformGridMesh, type: str, num_outputs, AoS: bool = True,
                            func: Optional[Callable] = None, device="cuda", **kwargs) -> torch.Tensor:
    """AoS float32 field on the mesh nodes ('node') or cells ('cell'), on ``device``."""
    if type == "node":
        shape = tuple(mesh.nodal_grid.shape[:-1])
    elif type == "cell":
        shape = tuple(n - 1 for n in mesh.nodal_grid.shape[:-1])
    else:
        raise ValueError("Valid types are: node and cell")
    trailing = (num_outputs,) if isinstance(num_outputs, int) else tuple(num_outputs)
    if not AoS:
        raise NotImplementedError("fields are array-of-structures (X, Y, Z, N...)")
    if func is not None:
        arr = np.asarray(func(*mesh.meshgrid, **kwargs), dtype=np.float32)
        return torch.from_numpy(np.ascontiguousarray(arr.reshape(shape + trailing))).to(device)
    return torch.zeros(shape + trailing, dtype=torch.float32, device=device)


create_structured_warp_field = create_structured_field
