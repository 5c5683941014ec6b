"""The fused heat and Jacobi passes are launched as programmatic dependents of
the previous pass (the next pass is scheduled while the current one runs, and
waits on griddepcontrol.wait before any global access).  At sizes with many
waves of tiles and many passes, every pass must still see all of the previous
pass's writes: results bit for bit against the oracle, in place and out of place."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import fdm
import pde_module_b200 as P
from pde_module_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("in_place", [False, True])
def test_heat_512_many_passes(in_place):
    n, g, k, steps = 512, 1, 4, 44
    shape = (n + 2 * g, n + 2 * g, 1)
    dx = 1.0 / n
    dt = 0.2 * dx * dx
    u0 = np.random.default_rng(41).random(shape + (1,)).astype(np.float32)
    ud = torch.from_numpy(u0).cuda()
    bc = P.GridBoundary(ud, dx, g)
    bc.dirichlet_BC("ALL", 0.0)
    bc.vonNeumann_BC("+X", 0.5)
    roll = P.HeatRollout(bc, dx, 1.0, dt, steps_per_pass=k)
    if in_place:
        roll(ud, 0)  # allocate the work buffer
        x = ud.clone()
        rc = _lib.lib().pde_heat_rollout(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                                         C.c_void_p(roll.work.data_ptr()), C.byref(roll.grid), 1,
                                         C.byref(roll.rules), 1.0, dt, steps, k,
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0
        got = x.cpu().numpy()
    else:
        got = roll(ud, steps).cpu().numpy()
    G = fdm.exterior_groups(shape, g)
    groups = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0,)), dict(ids=G["+X"], type=2, value=0.5, comps=(0,))]
    ref = fdm.heat_rollout(u0, groups, dx, g, 1.0, dt, steps)
    assert np.array_equal(got, ref)


def test_cavity_512_many_jacobi_passes():
    s = P.FractionalStepLDC(n=512, Re=100.0, jacobi_iters=50, jacobi_per_pass=5)
    rng = np.random.default_rng(42)
    s.u.copy_(torch.from_numpy((0.1 * rng.standard_normal(tuple(s.u.shape))).astype(np.float32)))
    s.p.copy_(torch.from_numpy((0.1 * rng.standard_normal(tuple(s.p.shape))).astype(np.float32)))
    u, p = s.u.cpu().numpy(), s.p.cpu().numpy()
    s.step(3)
    G = fdm.exterior_groups(u.shape, 1)
    ug = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0, 1)), dict(ids=G["+Y"], type=1, value=1.0, comps=(0,))]
    pg = [dict(ids=G["ALL"], type=2, value=0.0, comps=(0,))]
    for _ in range(3):
        u, p = fdm.ldc_step(u, p, ug, pg, s.dx, 1, s.nu, s.dt, 50)
    assert np.array_equal(s.u.cpu().numpy(), u)
    assert np.array_equal(s.p.cpu().numpy(), p)
