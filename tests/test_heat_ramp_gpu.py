"""Time-ramped boundary groups in the fused heat rollout (boundary_functions.py:77-92
ramps; the reference's loop passes t to every GridBoundary call,
functional_boundary.py:237,254-255): step n of HeatRollout(u, N, t0) fills the
boundary at t0 + n*dt and is bit-identical to the loop of the three modules given
that time, and to the float32 oracle, on 2D (temporally blocked, several depths)
and 3D grids; ramps that end inside the rollout are covered."""
import numpy as np
import pytest
import torch

from oracle import fdm
import pde_module_b200 as P
from pde_module_b200.FDM.boundary import get_ramp_func

pytestmark = pytest.mark.gpu


def _case(shape, g, N, ramps, consts, seed):
    """ramps / consts: (group, type, value, comps[, t_max]) specs."""
    dx = 1.0 / (shape[0] - 2 * g - 1)
    u0 = np.random.default_rng(seed).random(shape + (N,)).astype(np.float32)
    ud = torch.from_numpy(u0).cuda()
    bc = P.GridBoundary(ud, dx, g)
    groups = []
    G = fdm.exterior_groups(shape, g)
    for name, typ, val, comps in consts:
        bc.set_BC(name, val, typ, comps)
        groups.append(dict(ids=G[name], type=typ, value=val, comps=tuple(comps), func="constant"))
    for name, typ, val, comps, t_max in ramps:
        bc.set_BC(name, get_ramp_func(val, t_max, output_ids=comps), typ, comps)
        groups.append(dict(ids=G[name], type=typ, value=val, comps=tuple(comps), func="ramp", t_max=t_max))
    return dx, u0, ud, bc, groups


CASES = [
    # shape, g, order, N, consts, ramps, nsteps, k, t0 (in units of dt)
    ((34, 40, 1), 1, 2, 1, [("ALL", 1, 0.0, (0,))], [("+Y", 1, 1.0, (0,), 0.4)], 23, 5, 0.0),
    ((34, 40, 1), 1, 2, 1, [("ALL", 1, 0.0, (0,))], [("+Y", 1, 1.0, (0,), 0.4)], 23, 8, 7.0),
    ((30, 33, 1), 1, 2, 2, [("ALL", 1, 0.0, (0, 1))],
     [("+Y", 1, 1.0, (0,), 0.5), ("-X", 2, -0.5, (1,), 0.25)], 17, 3, 2.5),
    ((26, 29, 1), 2, 4, 1, [("ALL", 2, 0.0, (0,))], [("+X", 1, 2.0, (0,), 0.3)], 11, 4, 0.0),
    ((28, 28, 1), 1, 2, 1, [], [("ALL", 1, 1.0, (0,), 0.2)], 19, 1, 0.0),
    ((12, 11, 10), 1, 2, 1, [("ALL", 1, 0.0, (0,))], [("+Z", 1, 1.0, (0,), 0.4)], 6, 0, 1.0),
    ((14, 12, 13), 2, 4, 2, [("ALL", 1, 0.0, (0, 1))], [("-Y", 2, 1.0, (1,), 0.3)], 4, 0, 0.0),
]


@pytest.mark.parametrize("shape,g,order,N,consts,ramps,nsteps,k,t0", CASES)
def test_ramped_rollout_matches_chain_and_oracle(shape, g, order, N, consts, ramps, nsteps, k, t0):
    alpha = 0.9
    dt = 0.2 * (1.0 / (shape[0] - 2 * g - 1)) ** 2 / alpha
    # t_max in units of the rollout's length, so the ramps end inside it
    ramps = [(n, ty, v, c, tm * nsteps * dt) for n, ty, v, c, tm in ramps]
    dx, u0, ud, bc, groups = _case(shape, g, N, ramps, consts, 1 + nsteps)
    t0 = t0 * dt
    lap = P.Laplacian(N, dx, g, order=order)
    euler = P.ForwardEuler()
    u = ud
    for n in range(nsteps):
        u2 = bc(u, t0 + n * dt)
        u = euler(u2, lap(u2, alpha), dt)
    chain = u.cpu().numpy()
    roll = P.HeatRollout(bc, dx, alpha, dt, order=order, steps_per_pass=k)
    assert roll.rules.has_ramp == 1
    fused = roll(ud, nsteps, t0).cpu().numpy()
    assert np.array_equal(fused, chain)
    ref = fdm.heat_rollout(u0, groups, dx, g, alpha, dt, nsteps, order, t0=t0)
    assert np.array_equal(fused, ref)
    # the ramp matters: the same rollout at another start time differs
    other = roll(ud, nsteps, t0 + 3 * dt).cpu().numpy()
    assert not np.array_equal(other, fused)


def test_solvers_without_ramps_reject_them():
    shape, g = (20, 22, 1), 1
    dx, u0, ud, bc, _ = _case(shape, g, 1, [("+Y", 1, 1.0, (0,), 0.1)], [("ALL", 1, 0.0, (0,))], 3)
    with pytest.raises(NotImplementedError):
        P.HeatSolver(bc, dx, 1e-4, 10)
    with pytest.raises(NotImplementedError):
        P.BatchedHeatRollout([ud.clone()], [dx], [1.0], [1e-4], boundary=bc)
