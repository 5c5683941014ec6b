"""Bounded device-side waits (the batched rollout's tile-progress waits; the same
limit bounds the 3D streaming kernels' mbarrier waits): a wait that runs out
returns, records PDE_ERR_TIMEOUT in the library's error word, and lets its
kernel end; once the word is set, every other wait gives up at once.  No GPU
fault is involved: the probe waits on a device word that nothing sets."""
import ctypes as C
import time

import numpy as np
import pytest
import torch

import pde_module_b200 as P
from pde_module_b200 import _lib

pytestmark = pytest.mark.gpu

PDE_ERR_TIMEOUT = -7


@pytest.fixture
def lib():
    L = _lib.lib()
    L.pde_device_error(None)
    yield L
    L.pde_set_wait_limit_ns(0)
    L.pde_device_error(None)


def test_wait_runs_out_and_reports_timeout(lib):
    word = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib.pde_set_wait_limit_ns(1_000_000)  # 1 ms
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    assert lib.pde_wait_probe(C.c_void_p(word.data_ptr()), 1, None) == 0
    err = lib.pde_device_error(None)
    dt = time.perf_counter() - t0
    assert err == PDE_ERR_TIMEOUT
    assert dt < 0.5
    assert lib.pde_device_error(None) == 0  # read and cleared


def test_satisfied_wait_reports_nothing(lib):
    word = torch.full((1,), 3, dtype=torch.int32, device="cuda")
    lib.pde_set_wait_limit_ns(1_000_000)
    assert lib.pde_wait_probe(C.c_void_p(word.data_ptr()), 2, None) == 0
    assert lib.pde_device_error(None) == 0


def test_waits_give_up_at_once_after_a_timeout(lib):
    word = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib.pde_set_wait_limit_ns(1_000_000)
    lib.pde_wait_probe(C.c_void_p(word.data_ptr()), 1, None)  # runs out, sets the error word
    torch.cuda.synchronize()
    assert lib.pde_set_wait_limit_ns(0) == 1_000_000  # back to the 2 s default
    t0 = time.perf_counter()
    for _ in range(3):
        lib.pde_wait_probe(C.c_void_p(word.data_ptr()), 1, None)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert dt < 0.5, f"waits took {dt:.2f} s with the error word set"
    assert lib.pde_device_error(None) == PDE_ERR_TIMEOUT


def test_batched_rollout_under_a_short_limit(lib):
    """A normal batched rollout completes under a 50 ms bound with no timeout and
    the same result as under the default bound."""
    rng = np.random.default_rng(9)
    sides = [(70, 66), (130, 97), (64, 200), (96, 96)]
    u0 = [rng.random(s).astype(np.float32) for s in sides]
    dx = [1.0 / (s[0] - 3) for s in sides]
    alpha = [0.5, 1.0, 0.1, 0.8]
    dt = [0.2 * h * h / a for h, a in zip(dx, alpha)]

    def run():
        fields = [torch.from_numpy(u[:, :, None, None].copy()).cuda() for u in u0]
        roll = P.BatchedHeatRollout(fields, dx, alpha, dt)
        roll(37)
        torch.cuda.synchronize()
        return fields

    ref = run()
    assert lib.pde_device_error(None) == 0
    lib.pde_set_wait_limit_ns(50_000_000)
    got = run()
    assert lib.pde_device_error(None) == 0
    assert all(torch.equal(a, b) for a, b in zip(got, ref))
