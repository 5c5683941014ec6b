"""``torch.nn``-like module base of the finite-difference operators.

Reference: stencil/stencil.py:23-132.  A module sets itself up on its first
call (hooks marked ``@setup``: output allocation, plan creation), runs
``@before_forward`` hooks, ``forward``, then ``@after_forward`` hooks, and
returns the same preallocated output tensor on every call, so later calls
allocate nothing and can be captured in a CUDA graph.
"""
from __future__ import annotations

from collections.abc import Iterable
from typing import Any, Optional

import torch


def tuplify(x: Any) -> tuple:
    """Single item -> 1-tuple; strings/bytes count as single items."""
    if isinstance(x, (str, bytes, bytearray)):
        return (x,)
    if isinstance(x, Iterable):
        return tuple(x)
    return (x,)


class Stencil:
    initial: bool = True
    device: Optional[torch.device] = None

    def __init__(self, *args, **kwargs) -> None:
        pass

    @staticmethod
    def create_output_array(input_array: torch.Tensor, trailing: Optional[tuple] = None,
                            zero: bool = True) -> torch.Tensor:
        """Output of the input's grid shape with trailing component dims ``trailing``.

        Zero-initialised by default so cells an operator never writes (ghost
        layers) hold 0 instead of undefined values.
        """
        grid = tuple(input_array.shape[:3])
        shape = grid + (tuple(trailing) if trailing is not None else tuple(input_array.shape[3:]))
        alloc = torch.zeros if zero else torch.empty
        return alloc(shape, dtype=input_array.dtype, device=input_array.device)

    def forward(self, *args, **kwargs) -> Any:
        raise NotImplementedError("forward method in Stencil Object must be implemented by the user")

    def _registry(self, phase: str) -> list:
        name = f"_{phase}_list"
        reg = self.__dict__.get(name)
        if reg is None:
            found = []
            for attr in dir(self):
                if attr.startswith("__"):
                    continue
                try:
                    meth = getattr(self, attr)
                except AttributeError:
                    continue
                if callable(meth) and hasattr(meth, f"_{phase}_order"):
                    found.append(meth)
            reg = sorted(found, key=lambda m: getattr(m, f"_{phase}_order"))
            setattr(self, name, reg)
        return reg

    def setup(self, *args, **kwargs) -> None:
        """Run the setup hooks (also callable explicitly, as in the reference)."""
        self._registry("before_forward")
        self._registry("after_forward")
        for meth in self._registry("setup"):
            meth(*args, **kwargs)
        self.initial = False

    def before_forward(self, *args, **kwargs) -> None:
        for meth in self._registry("before_forward"):
            meth(*args, **kwargs)

    def after_forward(self, *args, **kwargs) -> None:
        for meth in self._registry("after_forward"):
            meth(*args, **kwargs)

    def __call__(self, *args, **kwargs) -> Any:
        if self.initial:
            self.setup(*args, **kwargs)
        self.before_forward(*args, **kwargs)
        out = self.forward(*args, **kwargs)
        self.after_forward(*args, **kwargs)
        return out
