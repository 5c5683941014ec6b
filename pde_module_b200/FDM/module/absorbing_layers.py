"""Absorbing layers along the outer faces of the grid.

References: FDM/module/farfield.py:13-151 (kernel FDM/kernel/farfield.py:8-77) and
FDM/module/viscousDampingLayer.py:13-150 (kernel FDM/kernel/viscousDampingLayer.py:8-76).
A layer is every cell within ``num_layers`` of an eligible face (groups '-X' ..
'+Z', some of which can be excluded, e.g. an inlet).  Each of its cells takes the
axis of its nearest face (first minimum) and its depth dx into the layer; with
profile = (dx / num_layers) ** exponent:

    FarField(u, u_far, sigma_max)     out = -(sigma_max * profile) * (u - u_far)
    ViscousDampingLayer(du_dt, C_max) out = -(C_max * profile) * du_dt

and 0 elsewhere.  The points and the profile are prepared at the first call (the
depth takes num_layers distinct values; each power is one float32 powf, as the
reference's CPU kernels evaluate it), then every call is one GPU pass over the
layer (``pde_layer_apply``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .ExplicitUniformGridStencil import ExplicitUniformGridStencil
from ...stencil.hooks import setup
from ..._lib import lib, check, stream_ptr

_INT32_MAX = 2 ** 31 - 1


class _Layer(ExplicitUniformGridStencil):
    def __init__(self, inputs, num_layers: int, grid_shape, dx: float, ghost_cells: int, exponent: float) -> None:
        super().__init__(inputs, inputs, dx, ghost_cells)
        self.grid_shape = tuple(int(s) for s in grid_shape)
        self.num_layers = int(num_layers)
        self._exponent = np.float32(exponent)
        self.groups: dict[str, np.ndarray] = {}
        self.exclude_group: set = set()
        self.indices = np.moveaxis(np.indices(self.grid_shape, dtype=np.int32), 0, -1).reshape(-1, 3)
        for i, (s, ax) in enumerate(zip(self.grid_shape, "XYZ")):
            if s > 1:
                self.groups[f"-{ax}"] = self.indices[:, i] < self.num_layers
                self.groups[f"+{ax}"] = self.indices[:, i] >= (s - self.num_layers)

    def exclude(self, *groups: str) -> None:
        for group in groups:
            assert group in self.groups.keys()
            self.exclude_group.add(group)

    def _layer_array(self) -> np.ndarray:
        masks = [v for k, v in self.groups.items() if k not in self.exclude_group]
        mask = masks[0]
        for m in masks[1:]:
            mask = np.logical_or(mask, m)
        return self.indices[mask]

    def _profile(self, pts: np.ndarray) -> np.ndarray:
        n = np.array(self.grid_shape, dtype=np.int64)
        p = pts.astype(np.int64)
        dist = np.where(n > 1, np.minimum(p, n - p - 1), _INT32_MAX)
        axis = np.argmin(dist, axis=1)
        x = p[np.arange(len(p)), axis]
        na = n[axis]
        depth = np.where((na - 1 - x) < x, x - ((na - 1) - self.num_layers), self.num_layers - x)
        lut = np.zeros(self.num_layers + 1, dtype=np.float32)
        for d in range(1, self.num_layers + 1):  # depth is 1 .. num_layers: one float32 powf each
            q = np.float32(np.float32(d) / np.float32(self.num_layers))
            lut[d] = np.float32(q ** self._exponent)
        return lut[depth]

    @setup
    def initialize_kernel(self, input_array: torch.Tensor, *args, **kwargs) -> None:
        if tuple(input_array.shape[:3]) != self.grid_shape:
            raise AssertionError("input grid differs from the layer's grid_shape")
        self.outer_layers = self._layer_array()
        Y, Z = self.grid_shape[1], self.grid_shape[2]
        pts = self.outer_layers.astype(np.int64)
        flat = pts[:, 0] * Y * Z + pts[:, 1] * Z + pts[:, 2]
        dev = input_array.device
        self._cells = torch.from_numpy(flat).to(dev)
        self._prof = torch.from_numpy(self._profile(self.outer_layers)).to(dev)
        self._ncomp = int(np.prod(input_array.shape[3:]))

    def _apply(self, x: torch.Tensor, scale: float, cond) -> torch.Tensor:
        self.check_input(x)
        n = int(self._cells.numel())
        check(lib().pde_layer_apply(C.c_void_p(x.data_ptr()), C.c_void_p(self.output_array.data_ptr()), self._ncomp,
                                    C.c_void_p(self._cells.data_ptr()), C.c_void_p(self._prof.data_ptr()), n,
                                    float(scale), cond, C.c_void_p(stream_ptr(x))), "pde_layer_apply")
        return self.output_array


class FarField(_Layer):
    """Sponge layer forcing the field toward a far-field value."""

    def __init__(self, inputs, num_layers: int, beta: float, grid_shape, dx: float, ghost_cells: int,
                 float_dtype=torch.float32) -> None:
        super().__init__(inputs, num_layers, grid_shape, dx, ghost_cells, beta)
        self.beta = beta

    def get_sponge_array(self) -> np.ndarray:
        return self._layer_array()

    def __call__(self, input_array: torch.Tensor, farfield_condition, sigma_max: float) -> torch.Tensor:
        return super().__call__(input_array, farfield_condition, sigma_max)

    def forward(self, input_array: torch.Tensor, farfield_condition, sigma_max: float) -> torch.Tensor:
        cond = np.ascontiguousarray(np.asarray(farfield_condition, dtype=np.float32).reshape(-1))
        if cond.size != self._ncomp:
            raise AssertionError(f"far-field value of {cond.size} floats for a field of {self._ncomp} components")
        return self._apply(input_array, sigma_max, cond.ctypes.data_as(C.c_void_p))


class ViscousDampingLayer(_Layer):
    """Damping proportional to the time derivative inside the layer."""

    def __init__(self, inputs, num_layers: int, grid_shape, dx: float, ghost_cells: int, p: int = 2,
                 float_dtype=torch.float32) -> None:
        super().__init__(inputs, num_layers, grid_shape, dx, ghost_cells, p)
        self.p = np.float32(p)

    def get_damping_array(self) -> np.ndarray:
        return self._layer_array()

    @staticmethod
    def calculate_C_max(c: float, L: float, p: float = 2, R: float = 1e-2) -> float:
        """Largest stable damping coefficient (viscousDampingLayer.py:91-104)."""
        return float((p + 1.0) * c / (2.0 * L) * np.log(1.0 / R))

    def __call__(self, du_dt: torch.Tensor, C_max: float) -> torch.Tensor:
        return super().__call__(du_dt, C_max)

    def forward(self, du_dt: torch.Tensor, C_max: float) -> torch.Tensor:
        return self._apply(du_dt, C_max, None)
