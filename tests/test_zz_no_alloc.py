"""pde_heat_rollout_noalloc: the allocation-free fused heat rollout.

Callers that cannot allocate device memory (a memory manager owns every
allocation, cudaMalloc is not allowed in their loop, or a foreign-language
host can only pass the fields it holds) get the rollout's scratch field from a
fixed array inside the library.  This file checks, through the C ABI, that
two calls in a row give exactly what pde_heat_rollout gives with a caller-owned
scratch buffer, and that grids above the array's size are refused.  It is
collected last and also passes alone in a fresh process (the first call looks
the array up)."""
import ctypes as C

import numpy as np
import pytest
import torch

import pde_module_b200 as P
from pde_module_b200 import _lib

pytestmark = pytest.mark.gpu


def _setup(shape, g, seed):
    rng = np.random.default_rng(seed)
    u = torch.from_numpy(rng.random(shape + (1,)).astype(np.float32)).cuda()
    dx = 1.0 / (shape[0] - 2 * g - 1)
    bc = P.GridBoundary(u, dx, g)
    bc.dirichlet_BC("ALL", 0.0)
    bc.vonNeumann_BC("+X", 0.5)
    return u, dx, bc.rules(), _lib.make_grid(shape, g, 2, dx)


def _rollout_with_work(u, grid, rules, dt, nsteps, k):
    out, work = torch.empty_like(u), torch.empty_like(u)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib().pde_heat_rollout(C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()),
                                     C.c_void_p(work.data_ptr()), C.byref(grid), 1, C.byref(rules), 1.0, dt,
                                     nsteps, k, s)
    assert rc == 0
    return out


def _rollout_noalloc(u, grid, rules, dt, nsteps, k):
    out = torch.empty_like(u)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib().pde_heat_rollout_noalloc(C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()),
                                             C.byref(grid), 1, C.byref(rules), 1.0, dt, nsteps, k, s)
    assert rc == 0, _lib.strerror(rc)
    return out


@pytest.mark.parametrize("shape,nsteps,k", [((66, 70, 1), 21, 4), ((20, 18, 22), 5, 0)])
def test_noalloc_matches_caller_scratch_twice(shape, nsteps, k):
    for call, seed in enumerate((11, 12)):  # two calls in a row, different fields
        u, dx, rules, grid = _setup(shape, 1, seed)
        dt = 0.2 * dx * dx
        ref = _rollout_with_work(u, grid, rules, dt, nsteps, k)
        got = _rollout_noalloc(u, grid, rules, dt, nsteps, k)
        torch.cuda.synchronize()
        assert torch.equal(got, ref), f"call {call}"


def test_noalloc_in_place_with_an_odd_number_of_passes():
    """u_in == u_out: the passes alternate between the field and the library's
    array, and an odd count ends with a copy out of the array."""
    shape, k, nsteps = (70, 66, 1), 4, 12  # 3 passes
    for seed in (21, 22):
        u, dx, rules, grid = _setup(shape, 1, seed)
        dt = 0.2 * dx * dx
        ref = u.clone()
        work = torch.empty_like(u)
        s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert _lib.lib().pde_heat_rollout(C.c_void_p(ref.data_ptr()), C.c_void_p(ref.data_ptr()),
                                           C.c_void_p(work.data_ptr()), C.byref(grid), 1, C.byref(rules), 1.0, dt,
                                           nsteps, k, s) == 0
        got = u.clone()
        rc = _lib.lib().pde_heat_rollout_noalloc(C.c_void_p(got.data_ptr()), C.c_void_p(got.data_ptr()),
                                                 C.byref(grid), 1, C.byref(rules), 1.0, dt, nsteps, k, s)
        assert rc == 0, _lib.strerror(rc)
        torch.cuda.synchronize()
        assert torch.equal(got, ref)


def test_noalloc_two_components_exactly_at_the_limit():
    """2 components x 2048 x 1024 cells = PDE_NOALLOC_MAX_FLOATS floats: accepted,
    and equal to the rollout with a caller-owned scratch buffer."""
    shape = (2048, 1024, 1)
    assert shape[0] * shape[1] * 2 == _lib.PDE_NOALLOC_MAX_FLOATS
    rng = np.random.default_rng(31)
    u = torch.from_numpy(rng.random(shape + (2,)).astype(np.float32)).cuda()
    dx = 1.0 / (shape[0] - 3)
    bc = P.GridBoundary(u, dx, 1)
    bc.dirichlet_BC("ALL", 0.0)
    bc.vonNeumann_BC("+Y", 0.5, 1)
    rules, grid = bc.rules(), _lib.make_grid(shape, 1, 2, dx)
    dt = 0.2 * dx * dx
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref, work, got = torch.empty_like(u), torch.empty_like(u), torch.empty_like(u)
    assert _lib.lib().pde_heat_rollout(C.c_void_p(u.data_ptr()), C.c_void_p(ref.data_ptr()),
                                       C.c_void_p(work.data_ptr()), C.byref(grid), 2, C.byref(rules), 1.0, dt, 9, 4,
                                       s) == 0
    rc = _lib.lib().pde_heat_rollout_noalloc(C.c_void_p(u.data_ptr()), C.c_void_p(got.data_ptr()), C.byref(grid), 2,
                                             C.byref(rules), 1.0, dt, 9, 4, s)
    assert rc == 0, _lib.strerror(rc)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)


def test_noalloc_refuses_one_float_above_the_limit():
    shape = (5, (_lib.PDE_NOALLOC_MAX_FLOATS + 1) // 5, 1)
    assert shape[0] * shape[1] == _lib.PDE_NOALLOC_MAX_FLOATS + 1
    grid = _lib.make_grid(shape, 1, 2, 0.01)
    u = torch.zeros(1, device="cuda")  # never read: the size check comes first
    r = _lib.PdeBCRules()
    r.ncomp = 1
    rc = _lib.lib().pde_heat_rollout_noalloc(C.c_void_p(u.data_ptr()), C.c_void_p(u.data_ptr()), C.byref(grid), 1,
                                             C.byref(r), 1.0, 1e-5, 1, 1,
                                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.PDE_ERR_TOO_LARGE


def test_noalloc_refuses_grids_above_its_scratch():
    n = int(np.sqrt(_lib.PDE_NOALLOC_MAX_FLOATS)) + 3
    shape = (n, n, 1)
    grid = _lib.make_grid(shape, 1, 2, 0.01)
    u = torch.zeros(1, device="cuda")  # never read: the size check comes first
    r = _lib.PdeBCRules()
    r.ncomp = 1
    rc = _lib.lib().pde_heat_rollout_noalloc(C.c_void_p(u.data_ptr()), C.c_void_p(u.data_ptr()), C.byref(grid), 1,
                                             C.byref(r), 1.0, 1e-5, 1, 1,
                                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.PDE_ERR_TOO_LARGE
