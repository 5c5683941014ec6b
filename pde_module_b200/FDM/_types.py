"""Shape helpers shared by the FDM modules (reference: utils/utils.py:35-52,
FDM/utils.py:7-28, ExplicitUniformGridStencil.py:84-166)."""
from __future__ import annotations

import numpy as np
import torch


def grid_shape_of(shape) -> tuple:
    """(X, Y, Z) of a field shape given with or without trailing component dims."""
    s = tuple(int(v) for v in shape)
    if len(s) < 3:
        raise AssertionError("fields are 3D arrays (X, Y, Z, ...); a 2D grid has Z == 1")
    return s[:3]


def dimension_of(grid_shape) -> int:
    return sum(1 for s in grid_shape_of(grid_shape) if s > 1)


def eligible_dims(grid_shape) -> tuple:
    return tuple(i for i, s in enumerate(grid_shape_of(grid_shape)) if s > 1)


def check_float_dtype(float_dtype) -> None:
    ok = (None, torch.float32, np.float32, "float32")
    if float_dtype not in ok and getattr(float_dtype, "__name__", None) != "float32":
        raise NotImplementedError("the sm_100a kernels compute in float32 only")
