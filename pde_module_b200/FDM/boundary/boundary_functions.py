"""Boundary value functions (reference: FDM/boundary/boundary_functions.py:9-92).

The reference builds Warp functions that return the node's input vector with
the selected components replaced by a constant (or a linear ramp in time up
to ``T_max``).  Here they are descriptors the CUDA boundary kernels evaluate.
"""
from __future__ import annotations

from dataclasses import dataclass


def _ids(output_ids) -> tuple:
    if output_ids is None:
        return None
    if isinstance(output_ids, int):
        return (output_ids,)
    return tuple(int(i) for i in output_ids)


@dataclass(frozen=True)
class BCFunction:
    kind: str                 # "constant" | "ramp"
    value: float
    output_ids: tuple | None  # components set (None: decided by set_BC)
    t_max: float = 1.0

    def __call__(self, t: float = 0.0) -> float:
        """Value at time t, in float32 as the kernels compute it."""
        import numpy as np
        v = np.float32(self.value)
        if self.kind == "ramp":
            ramp = np.minimum(np.float32(t) / np.float32(self.t_max), np.float32(1.0))
            return float(np.float32(ramp * v))
        return float(v)


def get_constant_func(constant: float, input_dtype=None, output_ids=None) -> BCFunction:
    return BCFunction("constant", float(constant), _ids(output_ids))


def get_ramp_func(constant: float, T_max: float, input_dtype=None, output_ids=None) -> BCFunction:
    return BCFunction("ramp", float(constant), _ids(output_ids), float(T_max))
