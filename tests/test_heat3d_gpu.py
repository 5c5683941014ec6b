"""3D fused heat rollout (2.5D streaming along X, k steps per pass) against the
float32 oracle and the one-step-per-launch kernel, bit for bit.

The reference's loop is examples/2D_Heat_Equation.py:57-65 (BC -> Laplacian ->
Euler) run on a 3D grid; every case also checks the float64 oracle to 1e-5.
Launch shapes are forced small (many tiles and X chunks) so that the cut edges
of tiles and chunks fall inside the grid, next to its ghost layers and nodes."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import fdm
import pde_module_b200 as P
from pde_module_b200 import _lib, tuning
from pde_module_b200.FDM.boundary import get_ramp_func

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _reset_launch():
    yield
    tuning.set_launch_3d(0, 0, 0)
    _lib.lib().pde_set_dispatch(0)


def _groups(shape, g, spec, nsteps, dt):
    G = fdm.exterior_groups(shape, g)
    out = []
    for item in spec:
        name, typ, val, comps = item[:4]
        d = dict(ids=G[name], type=typ, value=val, comps=tuple(comps), func="constant")
        if len(item) > 4:
            d.update(func="ramp", t_max=item[4] * nsteps * dt)
        out.append(d)
    return out


def _boundary(ud, dx, g, spec, nsteps, dt):
    bc = P.GridBoundary(ud, dx, g)
    for item in spec:
        name, typ, val, comps = item[:4]
        if len(item) > 4:
            bc.set_BC(name, get_ramp_func(val, item[4] * nsteps * dt, output_ids=comps), typ, comps)
        else:
            bc.set_BC(name, val, typ, comps)
    return bc


DIR = [("ALL", 1, 0.5, (0,))]
NEU = [("ALL", 2, 0.25, (0,))]
MIX = [("ALL", 1, 0.0, (0,)), ("+Y", 2, 1.0, (0,)), ("-Z", 1, -0.5, (0,)), ("+X", 2, 0.5, (0,))]
MIX2 = [("ALL", 1, 0.0, (0, 1)), ("+Z", 2, 1.0, (1,)), ("-X", 1, 2.0, (0,))]
MIX3 = [("-X", 2, 0.5, (0, 1, 2)), ("+X", 1, -1.0, (2,)), ("ALL", 1, 0.0, (0,)), ("+Y", 1, 0.3, (1,))]
RAMP = [("ALL", 1, 0.0, (0,)), ("+Y", 1, 1.0, (0,), 0.4), ("-X", 2, -0.5, (0,), 0.6)]

CASES = [
    # shape, g, order, N, spec, nsteps, k, launch (tile_y, tile_z, chunks)
    ((40, 37, 45), 1, 2, 1, DIR, 7, 1, (0, 0, 0)),
    ((40, 37, 45), 1, 2, 1, DIR, 7, 2, (0, 0, 0)),
    ((40, 37, 45), 1, 2, 1, DIR, 9, 3, (0, 0, 0)),
    ((40, 37, 45), 1, 2, 1, DIR, 9, 4, (0, 0, 0)),
    ((61, 37, 45), 1, 2, 1, MIX, 9, 2, (8, 8, 2)),
    ((61, 37, 45), 1, 2, 1, MIX, 10, 3, (7, 9, 2)),
    ((61, 37, 45), 1, 2, 1, NEU, 8, 4, (11, 6, 2)),
    ((80, 29, 33), 1, 2, 1, MIX, 5, 1, (5, 7, 4)),
    ((44, 41, 38), 2, 4, 1, DIR, 6, 1, (0, 0, 0)),
    ((44, 41, 38), 2, 4, 1, MIX, 6, 2, (9, 10, 0)),
    ((70, 41, 38), 2, 4, 1, NEU, 7, 3, (12, 9, 2)),
    ((70, 41, 38), 2, 4, 1, MIX, 9, 4, (13, 11, 2)),
    ((46, 35, 39), 3, 2, 1, MIX, 6, 2, (10, 9, 0)),
    ((50, 33, 29), 1, 2, 2, MIX2, 6, 2, (9, 5, 2)),
    ((50, 33, 29), 2, 4, 2, MIX2, 5, 1, (0, 0, 0)),
    ((48, 23, 21), 1, 2, 3, MIX3, 6, 2, (6, 4, 2)),
    ((48, 23, 21), 2, 4, 4, [("ALL", 1, 0.0, (0, 1, 2, 3)), ("+Y", 2, 1.0, (3,))], 4, 2, (7, 3, 0)),
    ((45, 40, 36), 1, 2, 1, RAMP, 11, 3, (9, 8, 2)),
    ((45, 40, 36), 2, 4, 1, RAMP, 7, 2, (0, 0, 0)),
]


@pytest.mark.parametrize("shape,g,order,N,spec,nsteps,k,launch", CASES)
def test_heat3d_matches_oracle(shape, g, order, N, spec, nsteps, k, launch):
    rng = np.random.default_rng(hash((shape, g, order, N, nsteps, k)) % (2 ** 32))
    dx = 1.0 / (shape[0] - 2 * g - 1)
    alpha = 0.9
    dt = 0.15 * dx * dx / alpha
    u0 = rng.random(shape + (N,)).astype(np.float32)
    ud = torch.from_numpy(u0).cuda()
    bc = _boundary(ud, dx, g, spec, nsteps, dt)
    tuning.set_launch_3d(*launch)
    roll = P.HeatRollout(bc, dx, alpha, dt, order=order, steps_per_pass=k)
    t0 = 2 * dt if roll.rules.has_ramp else 0.0
    got = roll(ud, nsteps, t0).cpu().numpy()
    groups = _groups(shape, g, spec, nsteps, dt)
    ref = fdm.heat_rollout(u0, groups, dx, g, alpha, dt, nsteps, order, t0=t0)
    bad = np.argwhere(got != ref)
    assert bad.size == 0, f"{len(bad)} cells differ, first {bad[:5].tolist()}"
    ref64 = fdm.heat_rollout(u0.astype(np.float64), groups, dx, g, alpha, dt, nsteps, order, dtype=np.float64,
                             t0=t0)
    assert np.linalg.norm(got - ref64) / np.linalg.norm(ref64) < 1e-5


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_heat3d_in_place_and_short_last_pass(k):
    shape, g, dx = (52, 47, 43), 1, 1.0 / 50
    rng = np.random.default_rng(5 + k)
    u0 = rng.random(shape + (1,)).astype(np.float32)
    ud = torch.from_numpy(u0).cuda()
    bc = _boundary(ud, dx, g, MIX, 1, 1.0)
    dt = 0.15 * dx * dx
    roll = P.HeatRollout(bc, dx, 1.0, dt, steps_per_pass=k)
    ref = fdm.heat_rollout(u0, _groups(shape, g, MIX, 1, 1.0), dx, g, 1.0, dt, 2 * k + 1)
    out = roll(ud, 2 * k + 1).clone()
    assert np.array_equal(out.cpu().numpy(), ref)
    x = ud.clone()
    rc = _lib.lib().pde_heat_rollout(x.data_ptr(), x.data_ptr(), roll.work.data_ptr(), C.byref(roll.grid), 1,
                                     C.byref(roll.rules), 1.0, dt, 2 * k + 1, k, None)
    assert rc == 0
    torch.cuda.synchronize()
    assert torch.equal(x, out)


@pytest.mark.parametrize("order,g,N", [(2, 1, 1), (4, 2, 1), (2, 1, 3)])
def test_heat3d_matches_single_step_kernel(order, g, N):
    """A multi-wave grid (many tiles and chunks) against the one-step-per-launch
    kernel selected with PDE_DISPATCH_GENERIC, bit for bit."""
    shape = (150, 131, 140) if N == 1 else (96, 70, 66)
    dx = 1.0 / (shape[0] - 2 * g - 1)
    rng = np.random.default_rng(order + 10 * N)
    ud = torch.from_numpy(rng.random(shape + (N,)).astype(np.float32)).cuda()
    spec = [("ALL", 1, 0.0, tuple(range(N))), ("+Y", 2, 1.0, (0,)), ("-Z", 1, 0.25, (N - 1,))]
    bc = _boundary(ud, dx, g, spec, 1, 1.0)
    dt = 0.15 * dx * dx
    outs = []
    for mode, k in ((1, 0), (0, 2), (0, 1), (0, 4 if N == 1 else 2)):
        _lib.lib().pde_set_dispatch(mode)
        roll = P.HeatRollout(bc, dx, 1.0, dt, order=order, steps_per_pass=k)
        outs.append(roll(ud, 9).clone())
    _lib.lib().pde_set_dispatch(0)
    for o in outs[1:]:
        assert torch.equal(o, outs[0])


# Grids that take the double-row map (even Y and Z, plane pitch a multiple of 4
# floats, even g - R): one step per pass runs the surface fill (ghosts, then
# nodes) and the TMA streaming heat step.
SPLIT = [
    # shape, g, order, spec, nsteps, steps_per_pass (0: the library's choice, 1 here)
    ((40, 38, 44), 1, 2, DIR, 7, 1),
    ((41, 36, 40), 1, 2, MIX, 6, 0),
    ((44, 40, 44), 2, 4, MIX, 5, 1),
    ((39, 34, 42), 2, 4, NEU, 6, 0),
    ((45, 40, 36), 1, 2, RAMP, 8, 1),
    ((45, 40, 36), 2, 4, RAMP, 7, 0),
    ((70, 150, 264), 1, 2, MIX, 5, 0),
    ((66, 132, 260), 2, 4, MIX, 4, 0),
]


@pytest.mark.parametrize("shape,g,order,spec,nsteps,k", SPLIT)
def test_heat3d_one_step_streaming(shape, g, order, spec, nsteps, k):
    rng = np.random.default_rng(hash((shape, g, order, nsteps, k)) % (2 ** 32))
    dx = 1.0 / (shape[0] - 2 * g - 1)
    alpha = 0.8
    dt = 0.15 * dx * dx / alpha
    u0 = rng.random(shape + (1,)).astype(np.float32)
    ud = torch.from_numpy(u0).cuda()
    bc = _boundary(ud, dx, g, spec, nsteps, dt)
    roll = P.HeatRollout(bc, dx, alpha, dt, order=order, steps_per_pass=k)
    assert _lib.lib().pde_heat_pass_depth(C.byref(roll.grid), 1, k) == 1
    t0 = 3 * dt if roll.rules.has_ramp else 0.0
    got = roll(ud, nsteps, t0).cpu().numpy()
    assert np.array_equal(ud.cpu().numpy(), u0)  # the input is not written
    groups = _groups(shape, g, spec, nsteps, dt)
    ref = fdm.heat_rollout(u0, groups, dx, g, alpha, dt, nsteps, order, t0=t0)
    bad = np.argwhere(got != ref)
    assert bad.size == 0, f"{len(bad)} cells differ, first {bad[:5].tolist()}"


@pytest.mark.parametrize("nsteps", [1, 4, 5])
def test_heat3d_one_step_streaming_in_place_and_against_blocked(nsteps):
    """In place and out of place, odd and even step counts; equal to the
    temporally blocked kernel at k = 2 and to the one-step generic kernel."""
    shape, g = (52, 46, 44), 1
    dx = 1.0 / 50
    dt = 0.15 * dx * dx
    rng = np.random.default_rng(17 + nsteps)
    ud = torch.from_numpy(rng.random(shape + (1,)).astype(np.float32)).cuda()
    bc = _boundary(ud, dx, g, MIX, 1, 1.0)
    one = P.HeatRollout(bc, dx, 1.0, dt, steps_per_pass=1)
    out = one(ud, nsteps).clone()
    x = ud.clone()
    rc = _lib.lib().pde_heat_rollout(x.data_ptr(), x.data_ptr(), one.work.data_ptr(), C.byref(one.grid), 1,
                                     C.byref(one.rules), 1.0, dt, nsteps, 1, None)
    assert rc == 0
    torch.cuda.synchronize()
    assert torch.equal(x, out)
    blocked = P.HeatRollout(bc, dx, 1.0, dt, steps_per_pass=2)(ud, nsteps).clone()
    assert torch.equal(blocked, out)
    _lib.lib().pde_set_dispatch(1)
    generic = P.HeatRollout(bc, dx, 1.0, dt)(ud, nsteps).clone()
    assert torch.equal(generic, out)
