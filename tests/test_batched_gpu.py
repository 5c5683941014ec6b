"""Batched rollouts (one persistent launch over a tile work queue) against the
per-grid fused rollout and the float32 oracle, bitwise, on uneven grids."""
import numpy as np
import pytest
import torch

from oracle import fdm
import pde_module_b200 as P

pytestmark = pytest.mark.gpu


def _grids(n, lo, hi, seed, g=1):
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=(n, 2))
    alpha = np.exp(rng.uniform(np.log(1e-3), 0.0, size=n))
    fields, dx, dts = [], [], []
    for i, (sx, sy) in enumerate(sides):
        shape = (int(sx) + 2 * g, int(sy) + 2 * g, 1, 1)
        fields.append(np.random.default_rng(100 + i).random(shape).astype(np.float32))
        h = 1.0 / (max(sx, sy) - 1)
        dx.append(h)
        dts.append(0.2 * h * h / alpha[i])
    return fields, dx, alpha.tolist(), dts


def _bc(u, dx, g, spec):
    bc = P.GridBoundary(u, dx, g)
    for name, typ, val, comps in spec:
        bc.set_BC(name, val, typ, comps)
    return bc


@pytest.mark.parametrize("tile,k,nsteps", [((32, 64), 8, 37), ((16, 32), 4, 9), ((64, 32), 6, 1),
                                           ((32, 32), 3, 2), ((24, 40), 5, 50)])
def test_batched_heat_matches_per_grid(tile, k, nsteps):
    g = 1
    fields, dx, alpha, dts = _grids(14, 5, 150, seed=7)
    spec = [("ALL", 1, 0.0, (0,))]
    dev = [torch.from_numpy(f).cuda() for f in fields]
    ref = []
    for i, u in enumerate(dev):
        bc = _bc(u, dx[i], g, spec)
        ref.append(P.HeatRollout(bc, dx[i], alpha[i], dts[i], steps_per_pass=k)(u, nsteps).cpu().numpy())
    batch = [u.clone() for u in dev]
    roll = P.BatchedHeatRollout(batch, dx, alpha, dts, tile=tile, steps_per_pass=k)
    roll(nsteps)
    torch.cuda.synchronize()
    assert P._lib.device_error() == 0
    for i in range(len(batch)):
        assert np.array_equal(batch[i].cpu().numpy(), ref[i]), f"grid {i} {fields[i].shape}"
    for i in (0, 3):
        o = fdm.heat_rollout(fields[i], fdm.standard_groups(fields[i].shape[:3], g, spec), dx[i], g, alpha[i],
                             dts[i], nsteps)
        assert np.array_equal(batch[i].cpu().numpy(), o)


def test_batched_heat_neumann_order4():
    g, order = 2, 4
    fields, dx, alpha, dts = _grids(9, 12, 90, seed=11, g=g)
    spec = [("ALL", 1, 0.0, (0,)), ("+X", 2, 0.75, (0,)), ("-Y", 2, -0.5, (0,))]
    dev = [torch.from_numpy(f).cuda() for f in fields]
    batch = [u.clone() for u in dev]
    bc0 = _bc(batch[0], dx[0], g, spec)
    roll = P.BatchedHeatRollout(batch, dx, alpha, dts, boundary=bc0, ghost_cells=g, order=order, tile=(32, 32),
                                steps_per_pass=4)
    roll(21)
    torch.cuda.synchronize()
    for i, u in enumerate(dev):
        bc = _bc(u, dx[i], g, spec)
        ref = P.HeatRollout(bc, dx[i], alpha[i], dts[i], order=order, steps_per_pass=4)(u, 21).cpu().numpy()
        assert np.array_equal(batch[i].cpu().numpy(), ref), f"grid {i}"
    o = fdm.heat_rollout(fields[2], fdm.standard_groups(fields[2].shape[:3], g, spec), dx[2], g, alpha[2], dts[2],
                         21, order)
    assert np.array_equal(batch[2].cpu().numpy(), o)


def test_batched_heat_graph_replay():
    fields, dx, alpha, dts = _grids(8, 30, 200, seed=5)
    a = [torch.from_numpy(f).cuda() for f in fields]
    b = [u.clone() for u in a]
    ra = P.BatchedHeatRollout(a, dx, alpha, dts, steps_per_pass=8)
    rb = P.BatchedHeatRollout(b, dx, alpha, dts, steps_per_pass=8)
    gr = ra.graph(20)
    gr.replay()
    gr.replay()
    rb(20)
    rb(20)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)


@pytest.mark.parametrize("tile,k,nsteps", [((32, 64), 8, 33), ((16, 16), 5, 12)])
def test_batched_wave_matches_oracle(tile, k, nsteps):
    rng = np.random.default_rng(21)
    n = 10
    sides = rng.integers(8, 120, size=(n, 2))
    fields, prev, dx, Ks, u0s = [], [], [], [], []
    for i, (sx, sy) in enumerate(sides):
        X, Y = int(sx) + 2, int(sy) + 2
        h = 1.0 / (max(X, Y) - 3)
        c = 1.0 + 0.5 * rng.random()
        dt = 0.5 * h / (np.sqrt(2.0) * c)
        K = np.float32(dt * dt * c * c)
        u0 = np.zeros((X, Y, 1, 1), dtype=np.float32)
        u0[2:-2, 2:-2, 0, 0] = rng.standard_normal((X - 4, Y - 4))
        u0s.append(u0)
        fields.append(torch.from_numpy(u0).cuda())
        prev.append(torch.from_numpy(u0).cuda())
        dx.append(h)
        Ks.append(float(K))
    roll = P.BatchedWaveRollout(fields, prev, dx, Ks, tile=tile, steps_per_pass=k)
    roll(nsteps)
    torch.cuda.synchronize()
    assert P._lib.device_error() == 0
    for i in range(n):
        Kf = np.full(u0s[i].shape, Ks[i], dtype=np.float32)
        st = fdm.wave_forward(Kf, u0s[i], None, None, nsteps, dx[i])
        assert np.array_equal(fields[i].cpu().numpy()[:, :, 0, 0], st[-1]), f"grid {i}"
        assert np.array_equal(prev[i].cpu().numpy()[:, :, 0, 0], st[-2]), f"grid {i}"


def test_batched_zero_steps_is_identity():
    fields, dx, alpha, dts = _grids(3, 10, 40, seed=1)
    a = [torch.from_numpy(f).cuda() for f in fields]
    P.BatchedHeatRollout(a, dx, alpha, dts)(0)
    for x, f in zip(a, fields):
        assert np.array_equal(x.cpu().numpy(), f)
