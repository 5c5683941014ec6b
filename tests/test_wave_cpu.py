"""The discrete adjoint of the wave rollout (oracle) against float64 torch
autograd of the same model and against central finite differences."""
import numpy as np
import torch

from oracle import fdm


def _problem(X=20, Y=22, N=30, seed=0):
    rng = np.random.default_rng(seed)
    dx = 1.0 / (X - 3)
    c = 1.0 + 0.1 * rng.random((X, Y))
    dt = 0.5 * dx / (np.sqrt(2.0) * c.max())
    K = (dt * dt * c * c)[:, :, None, None]
    u0 = np.zeros((X, Y, 1, 1))
    u0[3:-3, 3:-3, 0, 0] = 0.01 * rng.standard_normal((X - 6, Y - 6))
    src = dt * dt * fdm.np.sin(np.arange(N) * 0.3)
    target = 0.01 * rng.standard_normal((X, Y))
    return K, u0, src, (X // 2) * Y + Y // 2, N, dx, target


def _loss64(K, u0, src, cell, N, dx, target):
    st = fdm.wave_forward(K, u0, src, cell, N, dx, dtype=np.float64)
    I = fdm._wave_interior(*st[-1].shape, 1)
    return np.mean((st[-1] - target)[I] ** 2), st


def _torch_model(K, u0, src, cell, N, dx, target):
    X, Y = K.shape[:2]
    I = torch.from_numpy(fdm._wave_interior(X, Y, 1))
    w = torch.tensor(fdm.lap_weights(2, dx, np.float64))

    def lap(u):
        out = torch.zeros_like(u)
        c = u[1:-1, 1:-1]
        acc = w[0] * u[:-2, 1:-1] + w[1] * c + w[2] * u[2:, 1:-1] + w[0] * u[1:-1, :-2] + w[1] * c + w[2] * u[1:-1, 2:]
        out[1:-1, 1:-1] = acc
        return out

    Kt = torch.tensor(K[:, :, 0, 0], requires_grad=True)
    u0t = torch.tensor(u0[:, :, 0, 0], requires_grad=True)
    u = torch.where(I, u0t, torch.zeros_like(u0t))
    um = u
    sx, sy = cell // Y, cell % Y
    for n in range(N):
        v = 2 * u - um + Kt * lap(u)
        e = torch.zeros_like(v)
        e[sx, sy] = src[n]
        v = torch.where(I, v + e, torch.zeros_like(v))
        um, u = u, v
    loss = torch.mean((u - torch.from_numpy(target))[I] ** 2)
    loss.backward()
    return loss.item(), Kt.grad.numpy(), u0t.grad.numpy()


def test_adjoint_matches_float64_autograd():
    K, u0, src, cell, N, dx, target = _problem()
    J, st = _loss64(K, u0, src, cell, N, dx, target)
    I = fdm._wave_interior(*st[-1].shape, 1)
    muN = np.where(I, 2 * (st[-1] - target) / I.sum(), 0.0)[:, :, None, None]
    gK, mu0, mu1 = fdm.wave_adjoint(K, st, muN, dx, dtype=np.float64)
    Jt, gK_t, gu0_t = _torch_model(K, u0, src, cell, N, dx, target)
    assert abs(J - Jt) <= 1e-12 * max(1.0, abs(Jt))
    np.testing.assert_allclose(gK, gK_t, rtol=1e-9, atol=1e-12 * np.abs(gK_t).max())
    np.testing.assert_allclose(np.where(I, mu0 - mu1, 0), gu0_t, rtol=1e-9, atol=1e-12 * np.abs(gu0_t).max())
    # float32 adjoint (the GPU's arithmetic) stays close to the float64 gradient
    st32 = fdm.wave_forward(K, u0, src, cell, N, dx)
    g32, _, _ = fdm.wave_adjoint(K, st32, muN.astype(np.float32), dx)
    assert np.linalg.norm(g32 - gK_t) / np.linalg.norm(gK_t) < 1e-3


def test_adjoint_matches_central_differences():
    K, u0, src, cell, N, dx, target = _problem(seed=1)
    J, st = _loss64(K, u0, src, cell, N, dx, target)
    I = fdm._wave_interior(*st[-1].shape, 1)
    muN = np.where(I, 2 * (st[-1] - target) / I.sum(), 0.0)[:, :, None, None]
    gK, mu0, mu1 = fdm.wave_adjoint(K, st, muN, dx, dtype=np.float64)
    rng = np.random.default_rng(5)
    d = np.where(I, rng.standard_normal(I.shape), 0.0)[:, :, None, None]
    eps = 1e-4 * np.abs(K).max()
    Jp, _ = _loss64(K + eps * d, u0, src, cell, N, dx, target)
    Jm, _ = _loss64(K - eps * d, u0, src, cell, N, dx, target)
    fd = (Jp - Jm) / (2 * eps)
    ad = np.sum(gK * d[:, :, 0, 0])
    assert abs(fd - ad) <= 1e-5 * abs(ad)
