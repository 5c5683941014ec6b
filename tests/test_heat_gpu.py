"""Fused heat rollout (boundary fill + Laplacian + Euler, temporal blocking in
2D) against the unfused module chain and the float32 oracle, bitwise."""
import numpy as np
import pytest
import torch

from oracle import fdm
import pde_module_b200 as P

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def make_bc(u, dx, g, spec):
    bc = P.GridBoundary(u, dx, g)
    for name, typ, val, comps in spec:
        bc.set_BC(name, val, typ, comps)
    return bc


CASES = [
    # shape, g, order, N, spec, nsteps, k
    ((20, 17, 1), 1, 2, 1, [("ALL", 1, 0.0, (0,))], 23, 5),
    ((33, 65, 1), 1, 2, 1, [("ALL", 1, 0.0, (0,))], 40, 8),
    ((40, 37, 1), 1, 2, 2, [("ALL", 1, 0.0, (0, 1)), ("+Y", 1, 1.0, (0,))], 17, 3),
    ((30, 31, 1), 1, 2, 1, [("ALL", 2, 0.0, (0,))], 12, 12),
    ((26, 29, 1), 2, 4, 1, [("ALL", 1, 0.5, (0,))], 9, 4),
    ((18, 21, 1), 1, 2, 3, [("-X", 2, 0.5, (0, 1, 2)), ("+X", 1, -1.0, (2,)), ("ALL", 1, 0.0, (0,))], 10, 1),
    ((12, 11, 10), 1, 2, 1, [("ALL", 1, 0.0, (0,))], 6, 0),
    ((14, 12, 13), 2, 4, 2, [("ALL", 1, 0.0, (0, 1)), ("+Z", 2, 1.0, (1,))], 4, 0),
]


@pytest.mark.parametrize("shape,g,order,N,spec,nsteps,k", CASES)
def test_fused_rollout_matches_chain_and_oracle(shape, g, order, N, spec, nsteps, k, rng):
    dx = 1.0 / (shape[0] - 2 * g - 1)
    alpha = 0.9
    dt = 0.2 * dx * dx / alpha
    u0 = rng.random(shape + (N,)).astype(np.float32)
    ud = dev(u0)
    bc = make_bc(ud, dx, g, spec)
    lap = P.Laplacian(N, dx, g, order=order)
    euler = P.ForwardEuler()
    u = ud
    for _ in range(nsteps):
        u2 = bc(u)
        u = euler(u2, lap(u2, alpha), dt)
    chain = u.cpu().numpy()
    roll = P.HeatRollout(bc, dx, alpha, dt, order=order, steps_per_pass=k)
    fused = roll(ud, nsteps).cpu().numpy()
    assert np.array_equal(fused, chain)
    ref = fdm.heat_rollout(u0, fdm.standard_groups(shape, g, spec), dx, g, alpha, dt, nsteps, order)
    assert np.array_equal(fused, ref)
    ref64 = fdm.heat_rollout(u0.astype(np.float64), fdm.standard_groups(shape, g, spec), dx, g, alpha, dt,
                             nsteps, order, dtype=np.float64)
    err = np.linalg.norm(fused - ref64) / np.linalg.norm(ref64)
    assert err < 1e-5


def test_rollout_in_place_and_graph_capture(rng):
    shape, g, dx = (34, 30, 1), 1, 1.0 / 31
    u0 = rng.random(shape + (1,)).astype(np.float32)
    ud = dev(u0)
    bc = make_bc(ud, dx, g, [("ALL", 1, 0.0, (0,))])
    roll = P.HeatRollout(bc, dx, 1.0, 0.2 * dx * dx, steps_per_pass=4)
    ref = roll(ud.clone(), 13).clone()
    x = ud.clone()
    roll(x, 0)  # allocate buffers outside the capture
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        gph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gph, stream=s):
            out = roll(x, 13)
    gph.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
