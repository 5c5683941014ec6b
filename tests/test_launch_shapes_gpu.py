"""Launch shapes of the temporally blocked 2D kernels leave results unchanged: odd
tile sides set with pde_set_launch_2d, and the automatic tiles that are balanced
against the SM count on grids with a little more than one tile per SM, give the
oracle's values bit for bit (fused heat rollout, differentiable heat, wave,
cavity)."""
import numpy as np
import pytest
import torch

from oracle import fdm
import pde_module_b200 as P
import pde_module_b200._lib as L
from pde_module_b200.time_step.heat import HeatSolver
from pde_module_b200.time_step.wave import WaveSolver

pytestmark = pytest.mark.gpu

ODD = [(9, 13, 256), (17, 29, 512), (33, 58, 1024)]


@pytest.fixture
def launch():
    def set_launch(tx, ty, threads):
        L.check(L.lib().pde_set_launch_2d(tx, ty, threads), "pde_set_launch_2d")
    yield set_launch
    set_launch(0, 0, 0)


def _heat_case(X, Y, N, seed=0):
    g = 1
    spec = [("ALL", 2, 0.3, (0,)), ("+Y", 1, 1.0, (0,)), ("-X", 1, -0.5, (0,))]
    rng = np.random.default_rng(seed)
    shape = (X, Y, 1)
    dx = 1.0 / (X - 2 * g - 1)
    alpha = (0.5 + rng.random(shape)).astype(np.float32)[..., None]
    dt = float(0.2 * dx * dx / alpha.max())
    u0 = rng.random(shape).astype(np.float32)[..., None]
    lamN = rng.standard_normal(shape).astype(np.float32)[..., None]
    bc = P.GridBoundary(torch.from_numpy(u0).cuda(), dx, g)
    for nm, typ, val, comps in spec:
        bc.set_BC(nm, val, typ, comps)
    return fdm.standard_groups(shape, g, spec), g, dx, dt, alpha, u0, lamN, bc


def _heat_run(case, N, k, every=None):
    groups, g, dx, dt, alpha, u0, lamN, bc = case
    solver = HeatSolver(bc, dx, dt, N, steps_per_pass=k, checkpoint_every=every)
    a, u = torch.from_numpy(alpha).cuda(), torch.from_numpy(u0).cuda()
    uN = solver.forward(a, u)
    ga, gu = solver.backward(a, torch.from_numpy(lamN).cuda())
    torch.cuda.synchronize()
    return uN.cpu().numpy(), ga.cpu().numpy(), gu.cpu().numpy()


@pytest.mark.parametrize("tile", ODD)
def test_heat_adjoint_odd_tiles(tile, launch):
    case = _heat_case(66, 71, 10)
    launch(*tile)
    uN, ga, gu = _heat_run(case, 10, 3, 4)
    groups, g, dx, dt, alpha, u0, lamN, _ = case
    ref_uN, S = fdm.heat_forward_field(alpha, u0, groups, dx, g, dt, 10)
    ref_ga, ref_gu = fdm.heat_adjoint(alpha, S, lamN, groups, dx, g, dt)
    assert np.array_equal(uN, ref_uN)
    assert np.array_equal(ga, ref_ga)
    assert np.array_equal(gu, ref_gu)


def test_heat_adjoint_balanced_tiles_at_258():
    """258^2 has 153 tiles of 16x32: the automatic shape enlarges them to 17x29
    (144 tiles, one per SM on a 148-SM part); the oracle agrees bit for bit."""
    case = _heat_case(258, 258, 12, seed=5)
    uN, ga, gu = _heat_run(case, 12, 4, 5)
    groups, g, dx, dt, alpha, u0, lamN, _ = case
    ref_uN, S = fdm.heat_forward_field(alpha, u0, groups, dx, g, dt, 12)
    ref_ga, ref_gu = fdm.heat_adjoint(alpha, S, lamN, groups, dx, g, dt)
    assert np.array_equal(uN, ref_uN)
    assert np.array_equal(ga, ref_ga)
    assert np.array_equal(gu, ref_gu)


def _wave_case(X, Y, N, seed=0):
    rng = np.random.default_rng(seed)
    dx = 1.0 / (X - 3)
    c = (1.0 + 0.1 * rng.random((X, Y))).astype(np.float32)
    dt = 0.5 * dx / (np.sqrt(2.0) * c.max())
    K = ((dt * dt) * c * c).astype(np.float32)[:, :, None, None]
    u0 = np.zeros((X, Y, 1, 1), dtype=np.float32)
    u0[4:-4, 4:-4, 0, 0] = 0.01 * rng.standard_normal((X - 8, Y - 8))
    src = (dt * dt * np.sin(np.arange(N) * 0.3)).astype(np.float32)
    cell = (X // 2) * Y + Y // 3
    g = rng.standard_normal((X, Y, 1, 1)).astype(np.float32)
    return K, u0, src, cell, dx, g


def _wave_check(X, Y, N, k, every):
    K, u0, src, cell, dx, g = _wave_case(X, Y, N)
    solver = WaveSolver((X, Y, 1), dx, N, src=torch.from_numpy(src).cuda(), src_cell=cell, steps_per_pass=k,
                        checkpoint_every=every)
    Kd = torch.from_numpy(K).cuda()
    uN = solver.forward(Kd, torch.from_numpy(u0).cuda())
    gK, gu0 = solver.backward(Kd, torch.from_numpy(g).cuda())
    st = fdm.wave_forward(K, u0, src, cell, N, dx)
    rgK, mu0, mu1 = fdm.wave_adjoint(K, st, g, dx)
    assert np.array_equal(uN.cpu().numpy()[:, :, 0, 0], st[-1])
    assert np.array_equal(gK.cpu().numpy()[:, :, 0, 0], rgK)
    assert np.array_equal(gu0.cpu().numpy()[:, :, 0, 0], mu0 - mu1)


@pytest.mark.parametrize("tile", ODD)
def test_wave_odd_tiles(tile, launch):
    launch(*tile)
    _wave_check(61, 75, 23, 5, 6)


def test_wave_balanced_tiles_at_514():
    """514^2 has 153 tiles of 32x64: the automatic shape enlarges them to 33x58
    (144 tiles) with 1024 threads; forward and adjoint agree with the oracle."""
    _wave_check(514, 514, 20, 6, 7)


# (64, 64, 256): more than 12 region cells per thread, the flat-walk Jacobi kernel;
# the other shapes run the register cell-list kernel
@pytest.mark.parametrize("tile", ODD + [(64, 64, 256)])
def test_cavity_odd_tiles(tile, launch):
    n, steps, iters, k = 70, 3, 12, 4
    launch(*tile)
    s = P.FractionalStepLDC(n=n, Re=100.0, jacobi_iters=iters, jacobi_per_pass=k, dt=2e-3)
    rng = np.random.default_rng(n)
    u0 = (0.1 * rng.standard_normal(tuple(s.u.shape))).astype(np.float32)
    p0 = (0.1 * rng.standard_normal(tuple(s.p.shape))).astype(np.float32)
    s.u.copy_(torch.from_numpy(u0))
    s.p.copy_(torch.from_numpy(p0))
    s.step(steps)
    G = fdm.exterior_groups(u0.shape, 1)
    ug = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0, 1)), dict(ids=G["+Y"], type=1, value=1.0, comps=(0,))]
    pg = [dict(ids=G["ALL"], type=2, value=0.0, comps=(0,))]
    u, p = u0, p0
    for _ in range(steps):
        u, p = fdm.ldc_step(u, p, ug, pg, s.dx, 1, s.nu, s.dt, iters)
    assert np.array_equal(s.u.cpu().numpy(), u)
    assert np.array_equal(s.p.cpu().numpy(), p)


@pytest.mark.parametrize("tile", ODD + [(16, 32, 256)])
def test_fused_heat_rollout_odd_tiles(tile, launch):
    """The fused rollout under pde_set_launch_2d shapes, several components and a
    mixed boundary, 13 steps in passes of 5, against the oracle."""
    shape, g, N = (47, 53, 1), 1, 2
    dx = 1.0 / 44
    dt = 0.2 * dx * dx
    spec = [("ALL", 1, 0.0, (0, 1)), ("+Y", 2, 0.5, (1,)), ("-X", 1, 1.0, (0,))]
    u0 = np.random.default_rng(17).random(shape + (N,)).astype(np.float32)
    ud = torch.from_numpy(u0).cuda()
    bc = P.GridBoundary(ud, dx, g)
    for nm, typ, val, comps in spec:
        bc.set_BC(nm, val, typ, comps)
    launch(*tile)
    out = P.HeatRollout(bc, dx, 0.8, dt, steps_per_pass=5)(ud, 13)
    ref = fdm.heat_rollout(u0, fdm.standard_groups(shape, g, spec), dx, g, 0.8, dt, 13)
    assert np.array_equal(out.cpu().numpy(), ref)


def test_fused_heat_rollout_at_258():
    """The automatic shape on a 258^2 array (22x22 tiles, one per SM, 512 threads);
    20 steps agree with the oracle bit for bit."""
    shape, g = (258, 258, 1), 1
    dx = 1.0 / 256
    dt = 0.2 * dx * dx
    u0 = np.random.default_rng(9).random(shape + (1,)).astype(np.float32)
    ud = torch.from_numpy(u0).cuda()
    bc = P.GridBoundary(ud, dx, g)
    bc.dirichlet_BC("ALL", 0.0)
    out = P.HeatRollout(bc, dx, 1.0, dt, steps_per_pass=8)(ud, 20)
    ref = fdm.heat_rollout(u0, fdm.standard_groups(shape, g, [("ALL", 1, 0.0, (0,))]), dx, g, 1.0, dt, 20)
    assert np.array_equal(out.cpu().numpy(), ref)
