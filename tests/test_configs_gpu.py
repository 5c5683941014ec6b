"""Parity at the benchmark workloads' own sizes and step counts.

* 2D heat 256^2, 1000 steps (examples/2D_Heat_Equation.py:57-65): the fused
  rollout bit for bit against the float32 oracle, and within 1e-5 of float64.
* 3D operators at 512^3, orders 2 and 4, periodic ghosts: Laplacian, Grad and
  Divergence against the float32 oracle on slabs of planes (first, middle, last).
* Lid-driven cavity 1024^2 (50 Jacobi sweeps per step): two fused steps from
  rest and from a random state, bit for bit against the oracle's composition.
* Differentiable wave 512^2, 2000 steps: the adjoint's gradients against float64
  torch autograd of an independently written leapfrog model.
* 3D heat at 512^3 (the 3D sweep's grid), orders 2 and 4, a few steps on the
  library's default path, the whole array bit for bit against the float32 oracle."""
import numpy as np
import pytest
import torch

from oracle import fdm
import pde_module_b200 as P

pytestmark = pytest.mark.gpu


def heat256_initial(n=256, g=1):
    """U[0,1) from seed 0 on the interior times a Gaussian bump (sigma 0.1) at
    node-centred coordinates x_i = i/n (mesh/uniformGridMesh/functions.py:81-84)."""
    rng = np.random.default_rng(0)
    x = np.arange(n) / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    u = np.zeros((n + 2 * g, n + 2 * g, 1, 1), dtype=np.float32)
    u[g:n + g, g:n + g, 0, 0] = (rng.random((n, n)) *
                                 np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / (2 * 0.1 ** 2))).astype(np.float32)
    return u


def test_heat_256_1000_steps():
    n, g, steps = 256, 1, 1000
    dx = 1.0 / n
    dt = 0.2 * dx * dx
    u0 = heat256_initial(n, g)
    ud = torch.from_numpy(u0).cuda()
    bc = P.GridBoundary(ud, dx, g)
    bc.dirichlet_BC("ALL", 0.0)
    got = P.HeatRollout(bc, dx, 1.0, dt)(ud, steps).cpu().numpy()
    groups = fdm.standard_groups(u0.shape[:3], g, [("ALL", 1, 0.0, (0,))])
    ref = fdm.heat_rollout(u0, groups, dx, g, 1.0, dt, steps)
    assert np.array_equal(got, ref)
    ref64 = fdm.heat_rollout(u0.astype(np.float64), groups, dx, g, 1.0, dt, steps, dtype=np.float64)
    err = float(np.linalg.norm(got - ref64) / np.linalg.norm(ref64))
    print(f"heat 256^2 x 1000: relative L2 error vs float64 = {err:.3e}")
    assert err < 1e-5


@pytest.mark.parametrize("order", [2, 4])
def test_operators_512_slabs(order):
    n, g = 512, order // 2
    s = n + 2 * g
    dx = 1.0 / n
    gen = torch.Generator(device="cuda")
    gen.manual_seed(order)
    u = torch.randn((s, s, s, 1), device="cuda", generator=gen)
    v = torch.randn((s, s, s, 3), device="cuda", generator=gen)
    for f in (u, v):
        bc = P.GridBoundary(f, dx, g)
        bc.periodic("ALL")
        f.copy_(bc(f))
    lap = P.Laplacian(1, dx, g, order=order)(u, 0.7)
    grd = P.Grad(1, u.shape, dx, g, order=order)(u, 1.3)
    div = P.Divergence(3, v.shape, dx, g, order=order)(v, 0.9)
    for x0 in (g, s // 2 - 2, s - g - 4):
        x1 = x0 + 4
        us = u[x0 - g:x1 + g].cpu().numpy()
        vs = v[x0 - g:x1 + g].cpu().numpy()
        sl = slice(g, g + 4)
        assert np.array_equal(lap[x0:x1].cpu().numpy(), fdm.laplacian(us, dx, g, 0.7, order)[sl]), ("lap", x0)
        assert np.array_equal(grd[x0:x1].cpu().numpy(), fdm.grad(us, dx, g, 1.3, order)[sl]), ("grad", x0)
        assert np.array_equal(div[x0:x1].cpu().numpy(), fdm.divergence(vs, dx, g, 0.9, order)[sl]), ("div", x0)
    del u, v, lap, grd, div
    torch.cuda.empty_cache()


@pytest.mark.parametrize("start", ["rest", "random"])
def test_cavity_1024_two_steps(start):
    s = P.FractionalStepLDC(n=1024, Re=100.0, jacobi_iters=50)
    if start == "random":
        rng = np.random.default_rng(3)
        s.u.copy_(torch.from_numpy((0.1 * rng.standard_normal(tuple(s.u.shape))).astype(np.float32)))
        s.p.copy_(torch.from_numpy((0.1 * rng.standard_normal(tuple(s.p.shape))).astype(np.float32)))
    u0, p0 = s.u.cpu().numpy(), s.p.cpu().numpy()
    s.step(2)
    G = fdm.exterior_groups(u0.shape, 1)
    ug = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0, 1)), dict(ids=G["+Y"], type=1, value=1.0, comps=(0,))]
    pg = [dict(ids=G["ALL"], type=2, value=0.0, comps=(0,))]
    u, p = u0, p0
    for _ in range(2):
        u, p = fdm.ldc_step(u, p, ug, pg, s.dx, 1, s.nu, s.dt, 50)
    assert np.array_equal(s.u.cpu().numpy(), u)
    assert np.array_equal(s.p.cpu().numpy(), p)


def test_wave_512_gradients_vs_float64():
    from pde_module_b200.time_step import wave as W
    solver, c, u0, target, dt, mask = W.make_problem(n=512, nsteps=2000)
    cd = c.clone().requires_grad_(True)
    ud = u0.clone().requires_grad_(True)
    uN = W.wave_rollout((dt * dt) * cd * cd, ud, solver)
    loss = (((uN - target) * mask) ** 2).sum() / mask.sum()
    loss.backward()
    # float64 autograd of the same leapfrog model, written here independently
    Y = solver.shape[1]
    dx = solver.dx
    w0, w1 = 1.0 / (dx * dx), -2.0 / (dx * dx)
    inside = mask[:, :, 0, 0].double()
    src = solver.src.double()
    sx, sy = divmod(solver.src_cell, Y)
    tgt = target[:, :, 0, 0].double()
    c64 = c[:, :, 0, 0].double().clone().requires_grad_(True)
    u64 = u0[:, :, 0, 0].double().clone().requires_grad_(True)
    K = (dt * dt) * c64 * c64
    u = u64 * inside
    um = u
    for k in range(solver.N):
        lapu = torch.zeros_like(u)
        cc = u[1:-1, 1:-1]
        lapu[1:-1, 1:-1] = (w0 * u[:-2, 1:-1] + w1 * cc + w0 * u[2:, 1:-1]) + (
            w0 * u[1:-1, :-2] + w1 * cc + w0 * u[1:-1, 2:])
        vv = 2.0 * u - um + K * lapu
        e = torch.zeros_like(vv)
        e[sx, sy] = src[k]
        um, u = u, (vv + e) * inside
    l64 = (((u - tgt) * inside) ** 2).sum() / inside.sum()
    l64.backward()
    rel_c = float((cd.grad[:, :, 0, 0].double() - c64.grad).norm() / c64.grad.norm())
    rel_u = float((ud.grad[:, :, 0, 0].double() - u64.grad).norm() / u64.grad.norm())
    print(f"wave 512^2 x 2000: loss {loss.item():.6e} vs {l64.item():.6e}; "
          f"relative error of dJ/dc {rel_c:.3e}, of dJ/du0 {rel_u:.3e}")
    assert abs(loss.item() - l64.item()) <= 1e-4 * abs(l64.item())
    assert rel_c < 1e-4 and rel_u < 1e-3


@pytest.mark.parametrize("order,nsteps", [(2, 3), (4, 2)])
def test_heat3d_512_steps(order, nsteps):
    n, g = 512, order // 2
    shape = (n + 2 * g,) * 3
    dx = 1.0 / (n - 1)
    dt = 0.15 * dx * dx
    u0 = np.random.default_rng(5 + order).random(shape + (1,), dtype=np.float32)
    ud = torch.from_numpy(u0).cuda()
    bc = P.GridBoundary(ud, dx, g)
    bc.dirichlet_BC("ALL", 0.0)
    bc.vonNeumann_BC("+Y", 0.5)
    got = P.HeatRollout(bc, dx, 1.0, dt, order=order)(ud, nsteps).cpu().numpy()
    del ud
    torch.cuda.empty_cache()
    groups = fdm.standard_groups(shape, g, [("ALL", 1, 0.0, (0,)), ("+Y", 2, 0.5, (0,))])
    ref = fdm.heat_rollout(u0, groups, dx, g, 1.0, dt, nsteps, order)
    bad = np.argwhere(got != ref)
    assert bad.size == 0, f"{len(bad)} cells differ, first {bad[:5].tolist()}"
