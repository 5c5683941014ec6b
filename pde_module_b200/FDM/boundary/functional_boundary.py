"""Ghost-cell boundary conditions on the outer box of a uniform grid.

Reference: FDM/boundary/functional_boundary.py:57-402.  The module copies its
input to its own output, then applies each boundary group in the order the
groups were set: Dirichlet groups write the node (the node's input vector with
the chosen components replaced) and the adjacent ghost (2*val - adj), Von
Neumann groups write the ghost (adj -/+ 2*dx*val).  Group node ids are built
exactly as the reference builds them (C-order flat ids of the face slices,
``ALL`` their sorted union).  ``periodic`` is new: it fills every ghost layer
along the chosen axes from the opposite side of the interior.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from math import prod
from typing import Any, Callable, Optional

import numpy as np
import torch

from .flags import DIRICHLET, VON_NEUMANN, BC_SRING
from .boundary_functions import BCFunction, get_constant_func
from ..module.ExplicitUniformGridStencil import ExplicitUniformGridStencil
from ...stencil.hooks import setup, before_forward
from ... import _lib
from ..._lib import lib, check, stream_ptr, FACE_BITS


def get_unique_key(dictionary: dict, base_name: str) -> str:
    """reference: utils/utils.py:5-12."""
    candidate, counter = base_name, 1
    while candidate in dictionary:
        candidate = f"{base_name}_{counter}"
        counter += 1
    return candidate


@dataclass
class FunctionBC:
    face_ids: np.ndarray
    boundary_type: int
    output_ids: tuple
    func: BCFunction
    face_mask: int = 0
    device_ids: Optional[torch.Tensor] = field(default=None, repr=False)

    @property
    def comp_mask(self) -> int:
        m = 0
        for i in self.output_ids:
            m |= 1 << int(i)
        return m


class GridBoundary(ExplicitUniformGridStencil):
    """Boundary groups '-X','+X','-Y','+Y','-Z','+Z' (eligible axes) and 'ALL'.

    ``grid_coordinates`` is optional (the reference requires it but only
    user-written value functions read it).
    """

    def __init__(self, field: torch.Tensor, dx: float, ghost_cells: int, grid_coordinates=None) -> None:
        inputs = tuple(int(s) for s in field.shape[3:])
        if len(inputs) != 1:
            raise AssertionError("GridBoundary is implemented for vector fields (X, Y, Z, N)")
        self.dimension = sum(1 for s in field.shape[:3] if s > 1)
        super().__init__(inputs, inputs, dx, ghost_cells)
        self.grid_coordinates = grid_coordinates
        self.grid_shape = tuple(int(s) for s in field.shape[:3])
        self.nodeIDs = np.arange(0, prod(self.grid_shape), 1, dtype=np.int32)
        self.groups: dict[str, np.ndarray] = {}
        self.face_masks: dict[str, int] = {}
        self.func_groups: dict[str, FunctionBC] = {}
        self.periodic_axes = 0
        self._rules = None
        self.define_exterior_groups()

    def define_exterior_groups(self) -> None:
        g = self.ghost_cells
        ids = self.nodeIDs.reshape(self.grid_shape)
        faces = []
        all_mask = 0
        for i, axis in enumerate("XYZ"):
            if self.grid_shape[i] <= 1:
                continue
            for prefix in ("-", "+"):
                key = prefix + axis
                sl = [slice(None)] * 3
                sl[i] = g if prefix == "-" else -(g + 1)
                for x, n in enumerate(self.grid_shape):
                    if n > 1 and x != i:
                        sl[x] = slice(g, -g, 1) if g > 0 else slice(None)
                self.groups[key] = ids[tuple(sl)].ravel()
                self.face_masks[key] = FACE_BITS[key]
                all_mask |= FACE_BITS[key]
                faces.append(self.groups[key])
        self.groups["ALL"] = np.unique(np.concatenate(faces, axis=0)).astype(np.int32)
        self.face_masks["ALL"] = all_mask

    # ---- configuration -------------------------------------------------
    def set_BC(self, face_ids, value, boundary_type: int, output_ids=None) -> None:
        if boundary_type not in (DIRICHLET, VON_NEUMANN):
            raise ValueError("boundary_type must be DIRICHLET or VON_NEUMANN")
        if output_ids is None:
            output_ids = tuple(range(self.inputs[0]))
        assert isinstance(output_ids, (int, list, tuple)), "output id must be an integer"
        ids = (output_ids,) if isinstance(output_ids, int) else tuple(int(i) for i in output_ids)
        if any(i < 0 or i >= self.inputs[0] for i in ids):
            raise AssertionError("output id out of range")
        if not callable(value):
            assert isinstance(value, (float, int)) and not isinstance(value, bool)
            value = get_constant_func(value, None, ids)
        if not isinstance(value, BCFunction):
            raise NotImplementedError("value functions are constant or ramp (get_constant_func/get_ramp_func)")
        if value.output_ids is not None and tuple(value.output_ids) != ids:
            raise NotImplementedError("the value function must set the same components as output_ids")
        if isinstance(face_ids, str):
            assert face_ids in self.groups, f"unknown group {face_ids!r}"
            name = get_unique_key(self.func_groups, f"{None}_{BC_SRING[boundary_type]}")
            fmask = self.face_masks[face_ids]
            arr = self.groups[face_ids]
        else:
            assert isinstance(face_ids, (np.ndarray, list, tuple, int))
            name = get_unique_key(self.func_groups, "BC_Group")
            arr = np.array(face_ids, dtype=np.int32).reshape(-1) if isinstance(face_ids, int) else \
                np.array(face_ids, dtype=np.int32)
            assert arr.ndim == 1, "face_ids should be 1D"
            fmask = 0
        self.func_groups[name] = FunctionBC(arr, boundary_type, ids, value, fmask)
        self._reset()

    def dirichlet_BC(self, face_ids, value, output_ids=None) -> None:
        self.set_BC(face_ids, value, DIRICHLET, output_ids)

    def vonNeumann_BC(self, face_ids, value, output_ids=None) -> None:
        self.set_BC(face_ids, value, VON_NEUMANN, output_ids)

    def no_slip(self, face_ids, output_ids=None) -> None:
        self.set_BC(face_ids, 0.0, DIRICHLET, output_ids)

    def impermeable(self, group: str) -> None:
        assert self.inputs[0] == self.dimension, (
            "Valid only when input_dtype is vector with same length equal to dimension of field")
        assert group in {"-X", "+X", "-Y", "+Y", "-Z", "+Z"}, "{'-X','+X','-Y','+Y','-Z','+Z'} are valid groups"
        axis = "XYZ".index(group[-1])
        self.vonNeumann_BC(group, 0.0)
        self.dirichlet_BC(group, 0.0, axis)

    def periodic(self, axes="ALL") -> None:
        """New: periodic ghosts along the given axes ('X', 'Y', 'Z', iterable of them, or 'ALL')."""
        if axes == "ALL":
            axes = [a for i, a in enumerate("XYZ") if self.grid_shape[i] > 1]
        for a in axes:
            i = "XYZ".index(a.upper()[-1])
            assert self.grid_shape[i] > 1, f"axis {a} is not a grid dimension"
            self.periodic_axes |= 1 << i
        self._reset()

    def _reset(self) -> None:
        self._rules = None
        if not self.initial:
            self._upload()

    # ---- lifecycle ---------------------------------------------------------
    def __call__(self, input_array: torch.Tensor, t=None, params: dict[str, Any] | None = None) -> torch.Tensor:
        if params is None:
            params = {}
        return super().__call__(input_array, t, params)

    @setup(order=1)
    def initialize_kernel(self, input_array: torch.Tensor, *args, **kwargs) -> None:
        if tuple(input_array.shape[:3]) != self.grid_shape:
            raise AssertionError("input grid differs from the field the boundary was built for")
        self.t = torch.zeros(1, dtype=torch.float32, device=input_array.device)
        self.grid = _lib.make_grid(self.grid_shape, self.ghost_cells, 2, self.dx_value)
        self._upload()

    def _upload(self) -> None:
        dev = self.device
        n = len(self.func_groups)
        arr = (_lib.PdeBCGroup * max(n, 1))()
        for i, fg in enumerate(self.func_groups.values()):
            fg.device_ids = torch.as_tensor(fg.face_ids, dtype=torch.int32).to(dev)
            b = arr[i]
            b.node_ids = fg.device_ids.data_ptr() if fg.device_ids.numel() else None
            b.count = int(fg.device_ids.numel())
            b.type = int(fg.boundary_type)
            b.comp_mask = fg.comp_mask
            b.func = _lib.PDE_BC_FUNC_RAMP if fg.func.kind == "ramp" else _lib.PDE_BC_FUNC_CONSTANT
            b.value = float(fg.func.value)
            b.t_max = float(fg.func.t_max)
            b.face_mask = int(fg.face_mask)
        self._c_groups = arr
        self._n_groups = n
        self._has_ramp = any(fg.func.kind == "ramp" for fg in self.func_groups.values())

    @before_forward
    def set_default_params(self, input_array, t, params, **kwargs) -> None:
        for key in self.func_groups:
            params.setdefault(key, 0)
        if t is not None:
            if isinstance(t, torch.Tensor):
                self.t = t
            else:
                self.t.fill_(float(t))

    def forward(self, input_array: torch.Tensor, t=None, params=None, **kwargs) -> torch.Tensor:
        self.check_input(input_array)
        s = C.c_void_p(stream_ptr(input_array))
        tptr = C.c_void_p(self.t.data_ptr()) if self._has_ramp else None
        check(lib().pde_bc_apply(C.c_void_p(input_array.data_ptr()), C.c_void_p(self.output_array.data_ptr()),
                                 C.byref(self.grid), self.inputs[0], self._c_groups, self._n_groups, tptr, s),
              "pde_bc_apply")
        if self.periodic_axes:
            check(lib().pde_periodic_fill(C.c_void_p(self.output_array.data_ptr()), C.byref(self.grid),
                                          self.inputs[0], self.periodic_axes, s), "pde_periodic_fill")
        return self.output_array

    # ---- fused kernels ----------------------------------------------------
    @property
    def fusable(self) -> bool:
        return (self.periodic_axes == 0 and all(fg.face_mask for fg in self.func_groups.values())
                and self.inputs[0] <= _lib.PDE_FUSED_MAX_COMP and len(self.func_groups) <= _lib.PDE_MAX_GROUPS)

    @property
    def time_dependent(self) -> bool:
        """Some group's value depends on t (a ramp)."""
        return any(fg.func.kind == "ramp" for fg in self.func_groups.values())

    def rules(self) -> "_lib.PdeBCRules":
        """The groups compiled for the fused kernels (standard face groups only).
        Ramp groups compile with has_ramp set: the fused heat rollout evaluates them
        per step (HeatRollout's t0); the other fused solvers reject them."""
        if self._rules is None:
            if not self.fusable:
                raise NotImplementedError("fused kernels take standard face groups")
            n = len(self.func_groups)
            arr = (_lib.PdeBCGroup * max(n, 1))()
            for i, fg in enumerate(self.func_groups.values()):
                ramp = fg.func.kind == "ramp"
                arr[i].type = int(fg.boundary_type)
                arr[i].comp_mask = fg.comp_mask
                arr[i].func = _lib.PDE_BC_FUNC_RAMP if ramp else _lib.PDE_BC_FUNC_CONSTANT
                arr[i].value = float(fg.func.value)
                arr[i].t_max = float(fg.func.t_max) if ramp else 1.0
                arr[i].face_mask = int(fg.face_mask)
            grid = _lib.make_grid(self.grid_shape, self.ghost_cells, 2, self.dx_value)
            r = _lib.PdeBCRules()
            check(lib().pde_bc_compile(arr, n, C.byref(grid), self.inputs[0], C.byref(r)), "pde_bc_compile")
            self._rules = r
        return self._rules
