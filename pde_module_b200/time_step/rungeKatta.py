"""Runge-Kutta time integration of several fields (reference: time_step/rungeKatta.py:21-174).

``f(t, *fields, **kw)`` returns the time derivatives and ``bc(t, *fields, **kw)`` the
boundary-filled fields (their signatures must match).  RungeKatta2 (midpoint):

    y = bc(t, y);  k1 = f(t, y);  y1 = bc(t, y + dt/2 k1);  k2 = f(t + dt/2, y1);  y' = y + dt k2

RungeKatta1 advances y = bc(t, y) by dt/2 * f(t, y), the step the reference
takes.  The Euler updates are this package's ForwardEuler modules (one launch
per field); the midpoint method keeps a copy of the boundary-filled fields in its
own buffers (allocated at the first call), so every later call allocates nothing.
"""
from __future__ import annotations

import inspect
from typing import Callable

import torch

from ..stencil.stencil import Stencil, tuplify
from ..stencil.hooks import setup
from .forwardEuler import ForwardEuler


class SignatureMismatchError(Exception):
    """f and bc of a Runge-Kutta integrator take different arguments."""


class _RungeKutta(Stencil):
    n_euler = 1

    def __init__(self, field_dtypes, f: Callable, bc: Callable) -> None:
        super().__init__()
        self.input_dtypes = tuplify(field_dtypes)
        self.f, self.bc = f, bc
        self.num_fields = len(self.input_dtypes)
        if inspect.signature(f) != inspect.signature(bc):
            raise SignatureMismatchError(
                f"Signature For f {inspect.signature(f)} does not match the signature of bc {inspect.signature(bc)}!")

    @setup
    def check_args(self, t: float, dt: float, *arrays: torch.Tensor, **kwargs) -> None:
        assert len(arrays) == self.num_fields, f"{len(arrays)} fields for an integrator of {self.num_fields}"
        # a field's dtype is torch.float32, or its component shape: an int (vector) or a tuple (matrix)
        for arr, spec in zip(arrays, self.input_dtypes):
            assert isinstance(arr, torch.Tensor) and arr.dtype == torch.float32 and arr.is_cuda
            if isinstance(spec, int):
                spec = (spec,)
            if isinstance(spec, (tuple, list)):
                assert tuple(arr.shape[3:]) == tuple(spec), "arrays and input dtype for euler must match"


class RungeKatta1(_RungeKutta):
    def __init__(self, field_dtypes, f: Callable, bc: Callable) -> None:
        super().__init__(field_dtypes, f, bc)
        self.forwardEulers = tuple(ForwardEuler() for _ in self.input_dtypes)

    def forward(self, t: float, dt: float, *arrays: torch.Tensor, **kwargs) -> tuple:
        arrays = self.bc(t, *arrays, **kwargs)
        k1s = self.f(t, *arrays, **kwargs)
        return tuple(fe(arr, k1, dt / 2) for fe, arr, k1 in zip(self.forwardEulers, arrays, k1s))


class RungeKatta2(_RungeKutta):
    def __init__(self, field_dtypes, f: Callable, bc: Callable) -> None:
        super().__init__(field_dtypes, f, bc)
        self.forwardEulers_1 = tuple(ForwardEuler() for _ in self.input_dtypes)
        self.forwardEulers_2 = tuple(ForwardEuler() for _ in self.input_dtypes)

    @setup
    def set_buffers(self, t: float, dt: float, *arrays: torch.Tensor, **kwargs) -> None:
        self.t0_fields = tuple(torch.empty_like(arr) for arr in arrays)

    def forward(self, t: float, dt: float, *arrays: torch.Tensor, **kwargs) -> tuple:
        arrays = self.bc(t, *arrays, **kwargs)
        for buf, arr in zip(self.t0_fields, arrays):
            buf.copy_(arr)
        k1s = self.f(t, *arrays, **kwargs)
        y1s = [fe(arr, k1, dt / 2) for fe, arr, k1 in zip(self.forwardEulers_1, arrays, k1s)]
        y1s = self.bc(t, *y1s, **kwargs)
        k2s = self.f(t + dt / 2, *y1s, **kwargs)
        return tuple(fe(arr, k2, dt) for fe, arr, k2 in zip(self.forwardEulers_2, self.t0_fields, k2s))
