"""Solid regions inside the grid with a staircase boundary.

Reference: FDM/boundary/immersedBoundary.py:16-205 (module), :207-438 (kernels),
on the Boundary base FDM/boundary/boundary.py:11-222.  The geometry comes from a
boolean function on the node coordinates (``from_bool_func``, summed into an int8
bitmask as the reference does); ``finalize`` builds the index maps on the GPU
(``pde_ib_maps``: solid boundary cells, their fluid neighbours, interior solids,
fluid boundary, all in the reference's C order) and sets every boundary cell to
Dirichlet 0 ('ALL' = every boundary cell).  A call ``ib(u, fill_value)`` copies u
to the module's own output, sets each boundary cell per component (Dirichlet:
the value; von Neumann: the staircase mean over its fluid neighbours) and fills
the interior solids (``pde_ib_apply``), bit-identical to the reference.
The boundary tables go to the device at the first call and again only after a
setting changed (the reference reads them once, at its first call), so repeated
calls copy nothing from the host and can be captured in a CUDA graph.  Solid cells on the array's outer layer are refused (the reference
reads outside the array there).
"""
from __future__ import annotations

import ctypes as C
from typing import Callable

import numpy as np
import torch

from .flags import DIRICHLET, VON_NEUMANN
from ..module.ExplicitUniformGridStencil import ExplicitUniformGridStencil
from ...stencil.hooks import setup
from ... import _lib
from ..._lib import lib, check, stream_ptr


class ImmersedBoundary(ExplicitUniformGridStencil):
    def __init__(self, field: torch.Tensor, dx: float, ghost_cells: int) -> None:
        inputs = tuple(int(s) for s in field.shape[3:])
        if len(inputs) != 1:
            raise AssertionError("input must be vector type")
        assert type(ghost_cells) is int and ghost_cells > 0
        super().__init__(inputs, inputs, dx, ghost_cells)
        self.grid_shape = tuple(int(s) for s in field.shape[:3])
        self.grid_shape_without_ghost = self.grid_shape_with_no_ghost_cells(self.grid_shape, ghost_cells)
        self.dimension = self.calculate_dimension_from_grid_shape(self.grid_shape)
        self.bitmask = np.zeros(self.grid_shape, dtype=np.int8)
        self.groups: dict[str, np.ndarray] = {}
        self._device = field.device
        self._maps = None

    # ---- geometry ----------------------------------------------------------
    def from_bool_func(self, fn: Callable, meshgrid: list) -> None:
        """Add the solid region where fn(*meshgrid) is true (immersedBoundary.py:40-53)."""
        assert meshgrid[0].shape == self.grid_shape
        bitmask = fn(*meshgrid)
        self.bitmask += np.asarray(bitmask).astype(np.int8)

    def finalize(self) -> None:
        """Build the index maps from the bitmask (immersedBoundary.py:57-66)."""
        dev = self._device
        bm = torch.as_tensor(np.ascontiguousarray(self.bitmask), dtype=torch.int8).to(dev)
        grid = _lib.make_grid(self.grid_shape, self.ghost_cells, 2, self.dx_value)
        nbytes = int(lib().pde_ib_work_bytes(C.byref(grid)))
        if nbytes < 0:
            raise AssertionError("invalid grid for an immersed boundary")
        work = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        counts = (C.c_int64 * 3)()
        s = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        rc = lib().pde_ib_maps(C.c_void_p(bm.data_ptr()), C.byref(grid), None, None, None, None, counts,
                               C.c_void_p(work.data_ptr()), nbytes, s)
        if rc == _lib.PDE_ERR_ARG:
            raise ValueError("solid cells on the array's outer layer: the reference reads outside the array there")
        check(rc, "pde_ib_maps")
        n_sb, n_is, n_fb = (int(c) for c in counts)
        D = self.dimension
        i32 = dict(dtype=torch.int32, device=dev)
        sb = torch.zeros((max(n_sb, 1), 3), **i32)
        fnb = torch.zeros((max(n_sb, 1), D, 2), dtype=torch.int8, device=dev)
        isd = torch.zeros((max(n_is, 1), 3), **i32)
        fb = torch.zeros((max(n_fb, 1), 3), **i32)
        check(lib().pde_ib_maps(C.c_void_p(bm.data_ptr()), C.byref(grid), C.c_void_p(sb.data_ptr()),
                                C.c_void_p(fnb.data_ptr()), C.c_void_p(isd.data_ptr()), C.c_void_p(fb.data_ptr()),
                                counts, C.c_void_p(work.data_ptr()), nbytes, s), "pde_ib_maps")
        self._grid = grid
        self._d_sb, self._d_fnb, self._d_is = sb, fnb, isd
        self.n_boundary, self.n_interior = n_sb, n_is
        self.solid_boundary = sb[:n_sb].cpu().numpy()
        self.fluid_neighbors = fnb[:n_sb].cpu().numpy()
        self.interior_solids = isd[:n_is].cpu().numpy()
        self.fluid_boundary = fb[:n_fb].cpu().numpy()
        X, Y, Z = self.grid_shape
        it = self.interior_solids.astype(np.int64)
        self.flat_array = it[:, 0] * Y * Z + it[:, 1] * Z + it[:, 2]
        self.define_boundary_value_and_type_arrays(self.solid_boundary)
        self._maps = True

    def define_boundary_value_and_type_arrays(self, indices: np.ndarray) -> None:
        """Every boundary cell Dirichlet 0; 'ALL' = all of them (boundary.py:51-63)."""
        shape = (len(indices),) + tuple(self.inputs)
        self.boundary_ids = np.arange(len(indices))
        self.boundary_value = np.zeros(shape, dtype=np.float32)
        self.boundary_type = np.ones(shape, dtype=np.int8)
        self.groups["ALL"] = self.boundary_ids
        self._tables_dirty = True

    # ---- boundary settings (boundary.py:65-222) ----------------------------
    def _check_output_ids(self, output_ids):
        if output_ids is None:
            return slice(None)
        if isinstance(output_ids, (int, np.integer)):
            assert 0 <= output_ids < self.inputs[0]
            return int(output_ids)
        if isinstance(output_ids, (list, tuple, np.ndarray)):
            output_ids = np.array(output_ids, dtype=np.int32)
            assert np.all((0 <= output_ids) & (output_ids < self.inputs[0]))
            return output_ids
        raise TypeError(f"Valid Types are: int|np.ndarray|list|tuple|None got {type(output_ids)} instead")

    def set_BC(self, face_ids, value: float, boundary_type: int, outputs_ids=None) -> None:
        assert self._maps, "call finalize() before setting boundary conditions"
        if isinstance(face_ids, str):
            assert face_ids in self.groups
            face_ids = self.groups[face_ids]
        else:
            assert isinstance(face_ids, (np.ndarray, list, tuple, int))
            face_ids = np.array(face_ids, dtype=np.int32)
        outputs_ids = self._check_output_ids(outputs_ids)
        assert isinstance(value, float)
        self.boundary_type[face_ids, outputs_ids] = boundary_type
        self.boundary_value[face_ids, outputs_ids] = value
        self._tables_dirty = True

    def dirichlet_BC(self, group, value: float, outputs_ids=None) -> None:
        if not isinstance(value, (float, int)):
            raise NotImplementedError("immersed boundaries take constant values")
        self.set_BC(group, float(value), DIRICHLET, outputs_ids)

    def vonNeumann_BC(self, group, value: float, outputs_ids=None) -> None:
        self.set_BC(group, value, VON_NEUMANN, outputs_ids)

    def no_slip(self, group) -> None:
        assert self.inputs[0] == self.dimension, (
            "Valid only when input_dtype is vector with same length equal to dimension of field")
        self.dirichlet_BC(group, 0.0)

    # ---- call --------------------------------------------------------------
    @setup(order=1)
    def initialize_kernel(self, input_array: torch.Tensor, *args, **kwargs) -> None:
        if tuple(input_array.shape[:3]) != self.grid_shape:
            raise AssertionError("input grid differs from the field the boundary was built for")
        assert self._maps, "call finalize() first"
        n = max(self.n_boundary, 1)
        self._d_type = torch.zeros((n,) + tuple(self.inputs), dtype=torch.int8, device=input_array.device)
        self._d_value = torch.zeros((n,) + tuple(self.inputs), dtype=torch.float32, device=input_array.device)

    def forward(self, input_array: torch.Tensor, fill_value: float = 0.0, *args, **kwargs) -> torch.Tensor:
        self.check_input(input_array)
        nb = self.n_boundary
        if nb and self._tables_dirty:
            self._d_type[:nb].copy_(torch.from_numpy(self.boundary_type))
            self._d_value[:nb].copy_(torch.from_numpy(self.boundary_value))
        self._tables_dirty = False
        check(lib().pde_ib_apply(C.c_void_p(input_array.data_ptr()), C.c_void_p(self.output_array.data_ptr()),
                                 C.byref(self._grid), self.inputs[0], C.c_void_p(self._d_sb.data_ptr()),
                                 C.c_void_p(self._d_fnb.data_ptr()), C.c_void_p(self._d_type.data_ptr()),
                                 C.c_void_p(self._d_value.data_ptr()), nb, C.c_void_p(self._d_is.data_ptr()),
                                 self.n_interior, float(fill_value), C.c_void_p(stream_ptr(input_array))),
              "pde_ib_apply")
        return self.output_array
