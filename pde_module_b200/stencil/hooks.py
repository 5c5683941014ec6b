"""Method hooks of the module lifecycle (reference: stencil/hooks.py:6-102).

A hooked method carries an ``_<phase>_order`` attribute; ``Stencil`` collects
them once per instance and runs them sorted by order (lower first).
"""
from __future__ import annotations

from typing import Callable, Optional

_PHASES = ("setup", "before_forward", "after_forward")


def _hook(phase: str, fn: Optional[Callable], order: int, debug: bool) -> Callable:
    if not isinstance(order, int):
        raise AssertionError("order must be integer")

    def mark(func: Callable) -> Callable:
        if any(hasattr(func, f"_{p}_order") for p in _PHASES):
            raise AssertionError("Method already registered!")
        setattr(func, f"_{phase}_order", order)
        func._debug = debug
        return func

    return mark if fn is None else mark(fn)


def setup(fn: Optional[Callable] = None, *, order: int = 0, debug: bool = False) -> Callable:
    """Run the method once, on the first call, before forward."""
    return _hook("setup", fn, order, debug)


def before_forward(fn: Optional[Callable] = None, *, order: int = 0, debug: bool = False) -> Callable:
    """Run the method on every call, before forward."""
    return _hook("before_forward", fn, order, debug)


def after_forward(fn: Optional[Callable] = None, *, order: int = 0, debug: bool = False) -> Callable:
    """Run the method on every call, after forward."""
    return _hook("after_forward", fn, order, debug)
