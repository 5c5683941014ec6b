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


def test_cavity_with_a_ramped_lid():
    """FractionalStepLDC(lid_ramp_time=T): step n fills every boundary at n*dt, the
    lid at min(n*dt/T, 1)*U (the reference's function-BC cavity,
    Benchmark/Functional_BC/LDC_Graph Function.py:44-113); bitwise against the
    oracle's composition given those times, over two calls (the ramp ends inside)."""
    n, steps, iters = 40, 6, 12
    dt = 2e-3
    T = 7.5 * dt
    s = P.FractionalStepLDC(n=n, Re=100.0, jacobi_iters=iters, jacobi_per_pass=5, dt=dt, lid_ramp_time=T)
    assert s.u_bc.rules().has_ramp == 1
    rng = np.random.default_rng(51)
    u0 = (0.05 * rng.standard_normal(tuple(s.u.shape))).astype(np.float32)
    s.u.copy_(torch.from_numpy(u0))
    s.step(4)
    s.step(steps - 4)
    G = fdm.exterior_groups(u0.shape, 1)
    ug = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0, 1)),
          dict(ids=G["+Y"], type=1, value=1.0, comps=(0,), func="ramp", t_max=T)]
    pg = [dict(ids=G["ALL"], type=2, value=0.0, comps=(0,))]
    u, p = u0, np.zeros(tuple(s.p.shape), dtype=np.float32)
    for k in range(steps):
        u, p = fdm.ldc_step(u, p, ug, pg, s.dx, 1, s.nu, s.dt, iters, t=k * dt)
    assert np.array_equal(s.u.cpu().numpy(), u)
    assert np.array_equal(s.p.cpu().numpy(), p)


def test_batched_heat_with_a_ramp():
    """Batched heat rollouts with a ramped face group: every grid bit for bit equal
    to its own HeatRollout(u, N, t0) and to the oracle (step n at t0 + n*dt_i)."""
    rng = np.random.default_rng(52)
    sides = [(70, 66), (97, 130), (64, 90)]
    nsteps, t0 = 23, 0.3
    fields, refs = [], []
    for i, (X, Y) in enumerate(sides):
        dx = 1.0 / (X - 3)
        dt = float(np.float32(0.2 * dx * dx / (0.5 + i)))
        u0 = rng.random((X, Y, 1, 1)).astype(np.float32)
        ud = torch.from_numpy(u0).cuda()
        bc = P.GridBoundary(ud, dx, 1)
        bc.set_BC("ALL", 0.0, 1, (0,))
        bc.set_BC("+Y", get_ramp_func(2.0, 10 * dt, output_ids=(0,)), 1, (0,))
        bc.set_BC("-X", get_ramp_func(-1.0, 40 * dt, output_ids=(0,)), 2, (0,))
        one = P.HeatRollout(bc, dx, 0.5 + i, dt, steps_per_pass=4)(ud, nsteps, t0).clone()
        G = fdm.exterior_groups(u0.shape[:3], 1)
        groups = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0,)),
                  dict(ids=G["+Y"], type=1, value=2.0, comps=(0,), func="ramp", t_max=10 * dt),
                  dict(ids=G["-X"], type=2, value=-1.0, comps=(0,), func="ramp", t_max=40 * dt)]
        ref = fdm.heat_rollout(u0, groups, dx, 1, 0.5 + i, dt, nsteps, t0=t0)
        assert np.array_equal(one.cpu().numpy(), ref)
        fields.append(ud.clone())
        refs.append((ref, dx, 0.5 + i, dt, bc))
    roll = P.BatchedHeatRollout(fields, [r[1] for r in refs], [r[2] for r in refs], [r[3] for r in refs],
                                boundary=refs[0][4], steps_per_pass=4)
    roll(nsteps, t0)
    torch.cuda.synchronize()
    from pde_module_b200 import _lib
    assert _lib.lib().pde_device_error(None) == 0
    for f, r in zip(fields, refs):
        assert np.array_equal(f.cpu().numpy(), r[0])


@pytest.mark.parametrize("every", [5, 0])
def test_differentiable_heat_with_a_ramp(every):
    """HeatSolver with a ramped group: the forward (each checkpoint segment at its
    own step times, also when recomputed for the adjoint) and the gradients bit for
    bit against the oracle; the adjoint is the same as without the ramp values."""
    shape, g = (40, 46, 1), 1
    dx = 1.0 / (shape[0] - 3)
    rng = np.random.default_rng(53)
    alpha = (0.5 + rng.random(shape + (1,))).astype(np.float32)
    u0 = rng.random(shape + (1,)).astype(np.float32)
    lamN = rng.standard_normal(shape + (1,)).astype(np.float32)
    N, dt, t0 = 17, 0.2 * dx * dx / 1.5, 0.01
    ud = torch.from_numpy(u0).cuda()
    bc = P.GridBoundary(ud, dx, g)
    bc.set_BC("ALL", 0.0, 1, (0,))
    bc.set_BC("+Y", get_ramp_func(1.0, 9 * dt, output_ids=(0,)), 1, (0,))
    solver = P.HeatSolver(bc, dx, dt, N, steps_per_pass=4, checkpoint_every=every or None)
    ad = torch.from_numpy(alpha).cuda()
    uN = solver.forward(ad, ud, t0)
    ga, gu = solver.backward(ad, torch.from_numpy(lamN).cuda())
    G = fdm.exterior_groups(shape, g)
    groups = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0,)),
              dict(ids=G["+Y"], type=1, value=1.0, comps=(0,), func="ramp", t_max=9 * dt)]
    ref_u, S = fdm.heat_forward_field(alpha, u0, groups, dx, g, dt, N, t0=t0)
    ref_ga, ref_gu = fdm.heat_adjoint(alpha, S, lamN, groups, dx, g, dt)
    assert np.array_equal(uN.cpu().numpy(), ref_u)
    assert np.array_equal(ga.cpu().numpy(), ref_ga)
    assert np.array_equal(gu.cpu().numpy(), ref_gu)
    # another start time: the graphs are captured anew and the forward moves
    uN2 = solver.forward(ad, ud, t0 + 3 * dt)
    ref_u2, _ = fdm.heat_forward_field(alpha, u0, groups, dx, g, dt, N, t0=t0 + 3 * dt)
    assert np.array_equal(uN2.cpu().numpy(), ref_u2)
