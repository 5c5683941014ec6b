"""Fused weakly compressible RK2 step (pde_wc_rk2) on the GPU: bit for bit against
the oracle's composition of the reference operators (oracle/acm.py wc_rk2) for
several tile shapes (cut edges inside the grid, tiles smaller than the halo), and
against the same step run as this package's module chain (GridBoundary,
Laplacian, Grad, Divergence, OuterProduct, scalarVectorMult, RungeKatta2 and torch
element-wise arithmetic for the two map-wise lines of examples/LDC/LDC_RK2.py);
the cavity's lid drives the flow."""
import numpy as np
import pytest
import torch

from oracle import acm, fdm
import pde_module_b200 as P
import pde_module_b200._lib as L

pytestmark = pytest.mark.gpu


def _case(shape, seed, lid=1.0):
    rng = np.random.default_rng(seed)
    dx = 1.0 / (shape[0] - 3)
    rho = (1.0 + 0.05 * rng.standard_normal(shape + (1,))).astype(np.float32)
    m = (0.1 * rng.standard_normal(shape + (2,))).astype(np.float32)
    G = fdm.exterior_groups(shape, 1)
    ug = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0, 1)), dict(ids=G["+Y"], type=1, value=lid, comps=(0,))]
    rg = [dict(ids=G["ALL"], type=2, value=0.0, comps=(0,))]
    md, rd = torch.from_numpy(m).cuda(), torch.from_numpy(rho).cuda()
    u_bc = P.GridBoundary(md, dx, 1)
    u_bc.dirichlet_BC("ALL", 0.0)
    u_bc.dirichlet_BC("+Y", lid, 0)
    r_bc = P.GridBoundary(rd, dx, 1)
    r_bc.vonNeumann_BC("ALL", 0.0)
    nu, c2, rho0 = 0.01, 100.0, 1.0
    dt = 0.2 * dx / 10.0
    eps = -0.01 * dx ** 4 / (dt * nu)
    return m, rho, md, rd, u_bc, r_bc, ug, rg, dx, nu, c2, rho0, eps, dt


@pytest.fixture
def launch():
    def set_launch(tx, ty, threads=0):
        L.check(L.lib().pde_set_launch_2d(tx, ty, threads), "pde_set_launch_2d")
    yield set_launch
    set_launch(0, 0, 0)


@pytest.mark.parametrize("shape,tile,steps", [((43, 37, 1), (0, 0), 3), ((43, 37, 1), (8, 8), 2),
                                              ((30, 41, 1), (12, 16), 3), ((67, 70, 1), (32, 32), 2)])
def test_fused_step_matches_oracle(shape, tile, steps, launch):
    m, rho, md, rd, u_bc, r_bc, ug, rg, dx, nu, c2, rho0, eps, dt = _case(shape, 3)
    launch(*tile)
    solver = P.WeaklyCompressibleRK2(u_bc, r_bc, dx, nu, c2, rho0, eps, dt)
    mo, ro = solver(md, rd, steps)
    ref_m, ref_r = acm.wc_rk2(m, rho, ug, rg, dx, 1, nu, eps, c2, rho0, dt, steps)
    assert np.array_equal(mo.cpu().numpy(), ref_m)
    assert np.array_equal(ro.cpu().numpy(), ref_r)


def test_fused_step_matches_module_chain():
    shape = (34, 30, 1)
    m, rho, md, rd, u_bc, r_bc, ug, rg, dx, nu, c2, rho0, eps, dt = _case(shape, 7)
    lap_u, lap_d = P.Laplacian(2, dx, 1), P.Laplacian(2, dx, 1)
    div_m = P.Divergence(2, md.shape, dx, 1)
    div_t = P.Divergence((2, 2), md.shape, dx, 1)
    grad_p = P.Grad(1, rd.shape, dx, 1)
    outer = P.OuterProduct(2, 2)
    momentum = P.scalarVectorMult(2)

    def bc(t, m_, r_):
        u = u_bc(m_ / r_)
        r2 = r_bc(r_)
        return momentum(r2, u), r2

    def f(t, m_, r_):
        u = m_ / r_
        m_div = div_m(m_, -1.0)
        u_diff = lap_u(u, nu)
        u_conv = div_t(outer(m_, u))
        u_damp = lap_d(u_diff, eps)
        p = c2 * (r_ - rho0)
        dp = grad_p(p, -1.0)
        return dp - u_conv + u_diff + u_damp, m_div

    rk = P.RungeKatta2([2, 1], f=f, bc=bc)
    cm, cr = md.clone(), rd.clone()
    for _ in range(2):
        cm, cr = rk(0.0, dt, cm, cr)
        cm, cr = cm.clone(), cr.clone()
    solver = P.WeaklyCompressibleRK2(u_bc, r_bc, dx, nu, c2, rho0, eps, dt)
    mo, ro = solver(md, rd, 2)
    assert torch.equal(mo, cm) and torch.equal(ro, cr)


def test_cavity_lid_drives_the_flow():
    solver, m, rho = P.lid_driven_cavity_wc(n=65)
    mo, ro = solver(m, rho, 400)
    u = (mo / ro).cpu().numpy()[:, :, 0, :]
    assert np.all(np.isfinite(u))
    mid = u.shape[0] // 2
    col = u[mid, 1:-1, 0]
    assert col[-3] > 0.05          # dragged along by the lid near the top
    assert col[len(col) // 4] < 0  # return flow below
    r = ro.cpu().numpy()
    assert abs(float(r.mean()) - 1.0) < 1e-2
