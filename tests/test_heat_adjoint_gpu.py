"""Differentiable heat rollout on the GPU: the forward with a diffusivity field
and the adjoint bitwise against the float32 oracle (several temporal-blocking
depths, checkpoint spacings, orders, boundary kinds, multi-tile grids); the
autograd gradient against float64 torch autograd of the same model."""
import numpy as np
import pytest
import torch

from oracle import fdm
import pde_module_b200 as P
from pde_module_b200.time_step.heat import HeatSolver, heat_rollout

pytestmark = pytest.mark.gpu

SPECS = {
    "dirichlet0": (1, 2, [("ALL", 1, 0.0, (0,))]),
    "mixed": (1, 2, [("ALL", 2, 0.3, (0,)), ("+Y", 1, 1.0, (0,)), ("-X", 1, -0.5, (0,))]),
    "order4_neumann": (2, 4, [("ALL", 1, 0.25, (0,)), ("+X", 2, -1.0, (0,))]),
}


def _setup(name, X, Y, N, seed=0):
    g, order, spec = SPECS[name]
    rng = np.random.default_rng(seed)
    shape = (X, Y, 1)
    dx = 1.0 / (X - 2 * g - 1)
    alpha = (0.5 + rng.random(shape)).astype(np.float32)[..., None]
    dt = float(0.2 * dx * dx / alpha.max() * (0.5 if order == 4 else 1.0))
    u0 = rng.random(shape).astype(np.float32)[..., None]
    lamN = rng.standard_normal(shape).astype(np.float32)[..., None]
    groups = fdm.standard_groups(shape, g, spec)
    u = torch.from_numpy(u0).cuda()
    bc = P.GridBoundary(u, dx, g)
    for nm, typ, val, comps in spec:
        bc.set_BC(nm, val, typ, comps)
    return groups, g, order, dx, dt, alpha, u0, lamN, bc


@pytest.mark.parametrize("name,X,Y,N,k,every", [
    ("dirichlet0", 40, 70, 23, 5, 7),
    ("dirichlet0", 75, 140, 17, 8, None),
    ("mixed", 37, 131, 19, 3, 19),
    ("mixed", 66, 66, 10, 1, 4),
    ("order4_neumann", 45, 100, 13, 4, 5),
])
def test_forward_and_adjoint_bitwise(name, X, Y, N, k, every):
    groups, g, order, dx, dt, alpha, u0, lamN, bc = _setup(name, X, Y, N)
    solver = HeatSolver(bc, dx, dt, N, order=order, steps_per_pass=k, checkpoint_every=every)
    a, u = torch.from_numpy(alpha).cuda(), torch.from_numpy(u0).cuda()
    uN = solver.forward(a, u)
    ref_uN, S = fdm.heat_forward_field(alpha, u0, groups, dx, g, dt, N, order)
    assert np.array_equal(uN.cpu().numpy(), ref_uN)
    ga, gu = solver.backward(a, torch.from_numpy(lamN).cuda())
    torch.cuda.synchronize()
    ref_ga, ref_gu = fdm.heat_adjoint(alpha, S, lamN, groups, dx, g, dt, order)
    assert np.array_equal(ga.cpu().numpy(), ref_ga)
    assert np.array_equal(gu.cpu().numpy(), ref_gu)


def test_constant_field_matches_heat_rollout():
    groups, g, order, dx, dt, alpha, u0, lamN, bc = _setup("mixed", 50, 90, 31)
    a = torch.full((50, 90, 1, 1), 0.8, device="cuda")
    u = torch.from_numpy(u0).cuda()
    solver = HeatSolver(bc, dx, dt, 31, steps_per_pass=6)
    roll = P.HeatRollout(bc, dx, 0.8, dt, steps_per_pass=6)
    assert torch.equal(solver.forward(a, u), roll(u, 31))


def test_autograd_against_float64_torch():
    from tests.test_heat_adjoint_cpu import _torch_grads
    name, X, Y, N = "mixed", 30, 41, 15
    groups, g, order, dx, dt, alpha, u0, lamN, bc = _setup(name, X, Y, N, seed=4)
    tgt = np.random.default_rng(2).standard_normal((X, Y, 1, 1))
    solver = HeatSolver(bc, dx, dt, N, steps_per_pass=4)
    a = torch.from_numpy(alpha).cuda().requires_grad_(True)
    u = torch.from_numpy(u0).cuda().requires_grad_(True)
    uN = heat_rollout(a, u, solver)
    loss = 0.5 * ((uN - torch.from_numpy(tgt).float().cuda()) ** 2).sum()
    loss.backward()
    _, ga64, gu64, _ = _torch_grads(groups, g, order, dx, dt, alpha.astype(np.float64), u0.astype(np.float64),
                                    tgt, N)
    ga = a.grad.cpu().numpy()[:, :, 0, 0]
    gu = u.grad.cpu().numpy()[:, :, 0, 0]
    assert np.linalg.norm(ga - ga64) / np.linalg.norm(ga64) < 1e-4
    assert np.linalg.norm(gu - gu64) / np.linalg.norm(gu64) < 1e-4


def test_scalar_alpha_gradient_by_broadcast():
    groups, g, order, dx, dt, alpha, u0, lamN, bc = _setup("dirichlet0", 34, 34, 12)
    solver = HeatSolver(bc, dx, dt, 12)
    s = torch.tensor(0.9, device="cuda", requires_grad=True)
    u = torch.from_numpy(u0).cuda()
    uN = heat_rollout(s.expand(34, 34, 1, 1).contiguous(), u, solver)
    uN.sum().backward()
    eps = 1e-2
    with torch.no_grad():
        up = solver.forward(torch.full((34, 34, 1, 1), 0.9 + eps, device="cuda"), u).double().sum()
        um = solver.forward(torch.full((34, 34, 1, 1), 0.9 - eps, device="cuda"), u).double().sum()
    fd = float((up - um) / (2 * eps))
    assert abs(float(s.grad) - fd) <= 5e-3 * abs(fd)


def test_graph_replay_with_solvers_replaced_in_a_loop():
    """Solvers rebuilt in a loop (as a tuning sweep does) each capture and replay
    their graphs; dropped solvers are freed outside any capture."""
    groups, g, order, dx, dt, alpha, u0, lamN, bc = _setup("mixed", 48, 80, 40)
    a0, u = torch.from_numpy(alpha).cuda(), torch.from_numpy(u0).cuda()
    ref = None
    for k in (2, 4, 8, 2, 4, 8):
        solver = HeatSolver(bc, dx, dt, 40, steps_per_pass=k)
        for _ in range(2):
            a = a0.clone().requires_grad_(True)
            loss = (heat_rollout(a, u, solver) ** 2).mean()
            loss.backward()
            if ref is None:
                ref = a.grad.clone()
            assert torch.equal(a.grad, ref)
