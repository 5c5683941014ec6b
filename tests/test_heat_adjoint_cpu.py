"""The discrete adjoint of the heat rollout with a diffusivity field (oracle)
against float64 torch autograd of the same model (boundary fill restated in
torch, independent of the oracle's linear-map derivation) and against central
finite differences."""
import numpy as np
import pytest
import torch

from oracle import fdm

SPECS = {
    "dirichlet0": (1, 2, [("ALL", 1, 0.0, (0,))]),
    "mixed": (1, 2, [("ALL", 2, 0.3, (0,)), ("+Y", 1, 1.0, (0,)), ("-X", 1, -0.5, (0,))]),
    "order4_neumann": (2, 4, [("ALL", 1, 0.25, (0,)), ("+X", 2, -1.0, (0,))]),
}


def _problem(name, X=17, Y=21, N=12, seed=0):
    g, order, spec = SPECS[name]
    rng = np.random.default_rng(seed)
    shape = (X, Y, 1)
    dx = 1.0 / (X - 2 * g - 1)
    alpha = (0.5 + rng.random(shape))[..., None]
    dt = 0.2 * dx * dx / alpha.max() * (0.5 if order == 4 else 1.0)
    u0 = rng.random(shape)[..., None]
    tgt = rng.standard_normal(shape)[..., None]
    groups = fdm.standard_groups(shape, g, spec)
    return groups, g, order, dx, dt, alpha, u0, tgt, N


def _torch_bc(u, groups, dx, g):
    """GridBoundary on a (X, Y) float64 tensor: copy, then each group in order,
    ghosts and nodes from the pre-boundary field (functional_boundary.py)."""
    X, Y = u.shape
    out = u.clone()
    for G in groups:
        ids = np.asarray(G["ids"])
        ix, iy = ids // Y, ids % Y
        val = float(G["value"])
        if G["type"] == 1:
            out[ix, iy] = val
        for a, (ii, n) in enumerate(((ix, X), (iy, Y))):
            inc = np.where(ii == g, 1, np.where(ii == n - 1 - g, -1, 0))
            sel = inc != 0
            if not sel.any():
                continue
            gx, gy = ix[sel].copy(), iy[sel].copy()
            ax_, ay_ = ix[sel].copy(), iy[sel].copy()
            if a == 0:
                gx -= inc[sel]
                ax_ += inc[sel]
            else:
                gy -= inc[sel]
                ay_ += inc[sel]
            cur = u[ax_, ay_]
            if G["type"] == 1:
                out[gx, gy] = 2.0 * val - cur
            else:
                s = torch.from_numpy(-np.sign(inc[sel]) * 2.0)
                out[gx, gy] = s * float(dx) * val + cur  # dx unrounded, as the float64 oracle
    return out


def _torch_grads(groups, g, order, dx, dt, alpha, u0, tgt, N):
    X, Y = u0.shape[:2]
    w = torch.tensor(fdm.lap_weights(order, dx, np.float64))
    R = (len(w) - 1) // 2
    a = torch.tensor(alpha[:, :, 0, 0], requires_grad=True)
    u0t = torch.tensor(u0[:, :, 0, 0], requires_grad=True)
    u = u0t
    for _ in range(N):
        v = _torch_bc(u, groups, dx, g)
        acc = torch.zeros((X - 2 * g, Y - 2 * g), dtype=torch.float64)
        for t in range(2 * R + 1):
            acc = acc + w[t] * v[g + t - R:X - g + t - R, g:Y - g]
        for t in range(2 * R + 1):
            acc = acc + w[t] * v[g:X - g, g + t - R:Y - g + t - R]
        S = torch.zeros_like(v)
        S[g:X - g, g:Y - g] = acc
        u = v + dt * (a * S)
    loss = 0.5 * torch.sum((u - torch.from_numpy(tgt[:, :, 0, 0])) ** 2)
    loss.backward()
    return loss.item(), a.grad.numpy(), u0t.grad.numpy(), u.detach().numpy()


def _oracle(groups, g, order, dx, dt, alpha, u0, tgt, N, dtype=np.float64):
    uN, S = fdm.heat_forward_field(alpha, u0, groups, dx, g, dt, N, order, dtype=dtype)
    lam = (uN - np.asarray(tgt, dtype=dtype)).astype(dtype)
    ga, gu = fdm.heat_adjoint(alpha, S, lam, groups, dx, g, dt, order, dtype=dtype)
    J = 0.5 * float(np.sum((uN.astype(np.float64) - tgt) ** 2))
    return J, ga[:, :, 0, 0], gu[:, :, 0, 0], uN


@pytest.mark.parametrize("name", list(SPECS))
def test_heat_adjoint_matches_float64_autograd(name):
    P = _problem(name)
    J, ga, gu, uN = _oracle(*P)
    Jt, ga_t, gu_t, uN_t = _torch_grads(*P)
    np.testing.assert_allclose(uN[:, :, 0, 0], uN_t, rtol=1e-12, atol=1e-12)
    assert abs(J - Jt) <= 1e-12 * max(1.0, abs(Jt))
    np.testing.assert_allclose(ga, ga_t, rtol=1e-9, atol=1e-12 * np.abs(ga_t).max())
    np.testing.assert_allclose(gu, gu_t, rtol=1e-9, atol=1e-12 * np.abs(gu_t).max())
    # the float32 adjoint (the GPU's arithmetic) stays close to the float64 gradient
    _, ga32, gu32, _ = _oracle(*P, dtype=np.float32)
    assert np.linalg.norm(ga32 - ga_t) / np.linalg.norm(ga_t) < 1e-4
    assert np.linalg.norm(gu32 - gu_t) / np.linalg.norm(gu_t) < 1e-4


@pytest.mark.parametrize("name", ["dirichlet0", "mixed"])
def test_heat_adjoint_matches_central_differences(name):
    groups, g, order, dx, dt, alpha, u0, tgt, N = _problem(name, seed=3)
    J, ga, gu, _ = _oracle(groups, g, order, dx, dt, alpha, u0, tgt, N)
    rng = np.random.default_rng(9)
    for field, grad in (("alpha", ga), ("u0", gu)):
        d = rng.standard_normal(alpha.shape)
        eps = 1e-5
        if field == "alpha":
            Jp = _oracle(groups, g, order, dx, dt, alpha + eps * d, u0, tgt, N)[0]
            Jm = _oracle(groups, g, order, dx, dt, alpha - eps * d, u0, tgt, N)[0]
        else:
            Jp = _oracle(groups, g, order, dx, dt, alpha, u0 + eps * d, tgt, N)[0]
            Jm = _oracle(groups, g, order, dx, dt, alpha, u0 - eps * d, tgt, N)[0]
        fd = (Jp - Jm) / (2 * eps)
        an = float(np.sum(grad * d[:, :, 0, 0]))
        assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (field, fd, an)


def test_bc_linear_map_pairs():
    groups, g, order, dx, *_ = _problem("mixed")
    direct, pairs = fdm.bc_linear_map((17, 21, 1), groups, dx, g)
    # every filled ghost pairs with the cell two steps inward, Dirichlet -1, Neumann +1
    for gc, pc, c in pairs:
        gx, gy = divmod(gc, 21)
        px, py = divmod(pc, 21)
        assert (abs(gx - px), abs(gy - py)) in ((2, 0), (0, 2))
        assert c in (-1.0, 1.0)
    assert not direct[g, 5, 0]  # -X face is Dirichlet (last group on that face)
    assert direct[5, 5, 0]
