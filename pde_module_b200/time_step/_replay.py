"""Replaying a fixed sequence of library calls as a CUDA graph.

The differentiable solvers run the same launches on the same static buffers
every time (checkpoint segments, recomputation, adjoint passes), so after one
eager run the sequence is captured once and later calls replay it: one graph
launch instead of a Python-driven launch per pass."""
from __future__ import annotations

import gc
import weakref

import torch


class GraphedSequence:
    """``run()`` executes ``fn``: eagerly the first time (then captures it), by
    graph replay afterwards.  ``fn`` must launch on the current stream and only
    touch buffers that live as long as its owner.

    ``fn`` is held through a weak reference when it is a bound method, so an
    owner and its sequences form no reference cycle: owners are freed (and their
    graphs destroyed) when the last reference goes, never by a garbage-collector
    pass that could fall inside another capture, where destroying a graph is not
    permitted.  The collector is also kept off while a capture runs."""

    def __init__(self, fn, enabled: bool = True) -> None:
        self._fn = weakref.WeakMethod(fn) if hasattr(fn, "__self__") else (lambda f=fn: f)
        self.enabled = enabled
        self.graph = None

    def _call(self) -> None:
        fn = self._fn()
        if fn is None:
            raise RuntimeError("the owner of this sequence no longer exists")
        fn()

    def run(self) -> None:
        if self.graph is not None:
            self.graph.replay()
            return
        self._call()
        if not self.enabled:
            return
        cur = torch.cuda.current_stream()
        s = torch.cuda.Stream(device=cur.device)
        s.wait_stream(cur)
        g = torch.cuda.CUDAGraph()
        gc.collect()
        was_enabled = gc.isenabled()
        gc.disable()
        try:
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
                    self._call()
        finally:
            if was_enabled:
                gc.enable()
        cur.wait_stream(s)
        self.graph = g

    def reset(self) -> None:
        self.graph = None
