"""Replaying a fixed sequence of library calls as a CUDA graph.

The differentiable solvers run the same launches on the same static buffers
every time (checkpoint segments, recomputation, adjoint passes), so after one
eager run the sequence is captured once and later calls replay it: one graph
launch instead of a Python-driven launch per pass."""
from __future__ import annotations

import torch


class GraphedSequence:
    """``run()`` executes ``fn``: eagerly the first time (then captures it), by
    graph replay afterwards.  ``fn`` must launch on the current stream and only
    touch buffers that live as long as this object."""

    def __init__(self, fn, enabled: bool = True) -> None:
        self.fn = fn
        self.enabled = enabled
        self.graph = None

    def run(self) -> None:
        if self.graph is not None:
            self.graph.replay()
            return
        self.fn()
        if not self.enabled:
            return
        cur = torch.cuda.current_stream()
        s = torch.cuda.Stream(device=cur.device)
        s.wait_stream(cur)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
                self.fn()
        cur.wait_stream(s)
        self.graph = g

    def reset(self) -> None:
        self.graph = None
