"""Differentiable wave rollout on the GPU: forward and adjoint bitwise against
the oracle for several temporal-blocking depths and checkpoint spacings; the
autograd gradient of an MSE loss with respect to the speed field against float64
torch autograd of the same model."""
import numpy as np
import pytest
import torch

from oracle import fdm
from pde_module_b200.time_step.wave import WaveSolver, wave_rollout, interior_mask

pytestmark = pytest.mark.gpu


def _setup(X=40, Y=46, N=37, seed=0):
    rng = np.random.default_rng(seed)
    dx = 1.0 / (X - 3)
    c = (1.0 + 0.1 * rng.random((X, Y))).astype(np.float32)
    dt = 0.5 * dx / (np.sqrt(2.0) * c.max())
    K = ((dt * dt) * c * c).astype(np.float32)[:, :, None, None]
    u0 = np.zeros((X, Y, 1, 1), dtype=np.float32)
    u0[4:-4, 4:-4, 0, 0] = 0.01 * rng.standard_normal((X - 8, Y - 8))
    src = (dt * dt * np.sin(np.arange(N) * 0.3)).astype(np.float32)
    cell = (X // 2) * Y + Y // 3
    return K, u0, src, cell, N, dx, c, dt


@pytest.mark.parametrize("k,every", [(1, None), (5, 6), (8, 37), (3, 1)])
def test_forward_and_adjoint_bitwise(k, every):
    K, u0, src, cell, N, dx, _, _ = _setup()
    X, Y = K.shape[:2]
    solver = WaveSolver((X, Y, 1), dx, N, src=torch.from_numpy(src).cuda(), src_cell=cell, steps_per_pass=k,
                        checkpoint_every=every)
    Kd, u0d = torch.from_numpy(K).cuda(), torch.from_numpy(u0).cuda()
    uN = solver.forward(Kd, u0d)
    st = fdm.wave_forward(K, u0, src, cell, N, dx)
    assert np.array_equal(uN.cpu().numpy()[:, :, 0, 0], st[-1])
    rng = np.random.default_rng(3)
    g = rng.standard_normal((X, Y, 1, 1)).astype(np.float32)
    gK, gu0 = solver.backward(Kd, torch.from_numpy(g).cuda())
    rgK, mu0, mu1 = fdm.wave_adjoint(K, st, g, dx)
    assert np.array_equal(gK.cpu().numpy()[:, :, 0, 0], rgK)
    assert np.array_equal(gu0.cpu().numpy()[:, :, 0, 0], mu0 - mu1)


def test_autograd_speed_gradient_matches_float64():
    K, u0, src, cell, N, dx, c, dt = _setup(N=60, seed=2)
    X, Y = K.shape[:2]
    target = (0.001 * np.random.default_rng(4).standard_normal((X, Y, 1, 1))).astype(np.float32)
    solver = WaveSolver((X, Y, 1), dx, N, src=torch.from_numpy(src).cuda(), src_cell=cell, steps_per_pass=4)
    cd = torch.from_numpy(c[:, :, None, None]).cuda().requires_grad_(True)
    u0d = torch.from_numpy(u0).cuda().requires_grad_(True)
    mask = interior_mask((X, Y), 1)
    uN = wave_rollout((dt * dt) * cd * cd, u0d, solver)
    loss = (((uN - torch.from_numpy(target).cuda()) * mask) ** 2).sum() / mask.sum()
    loss.backward()
    # float64 reference with torch autograd on the CPU
    I = torch.from_numpy(fdm._wave_interior(X, Y, 1))
    w = torch.tensor(fdm.lap_weights(2, dx, np.float64))
    c64 = torch.tensor(c.astype(np.float64), requires_grad=True)
    u064 = torch.tensor(u0[:, :, 0, 0].astype(np.float64), requires_grad=True)

    def lap(u):
        out = torch.zeros_like(u)
        cc = u[1:-1, 1:-1]
        out[1:-1, 1:-1] = (w[0] * u[:-2, 1:-1] + w[1] * cc + w[2] * u[2:, 1:-1] + w[0] * u[1:-1, :-2] + w[1] * cc
                           + w[2] * u[1:-1, 2:])
        return out

    K64 = float(np.float32(dt) ** 2) * c64 * c64
    u = torch.where(I, u064, torch.zeros_like(u064))
    um = u
    for n in range(N):
        v = 2 * u - um + K64 * lap(u)
        e = torch.zeros_like(v)
        e[cell // Y, cell % Y] = float(src[n])
        um, u = u, torch.where(I, v + e, torch.zeros_like(v))
    l64 = torch.mean((u - torch.from_numpy(target[:, :, 0, 0].astype(np.float64)))[I] ** 2)
    l64.backward()
    gc = cd.grad.cpu().numpy()[:, :, 0, 0]
    assert abs(loss.item() - l64.item()) <= 1e-3 * l64.item()
    rel = np.linalg.norm(gc - c64.grad.numpy()) / np.linalg.norm(c64.grad.numpy())
    assert rel < 1e-3
    gu = u0d.grad.cpu().numpy()[:, :, 0, 0]
    relu = np.linalg.norm(gu - u064.grad.numpy()) / np.linalg.norm(u064.grad.numpy())
    assert relu < 1e-3


@pytest.mark.parametrize("nf,na,k,launch", [(7, 5, 3, None), (9, 9, 4, None), (0, 6, 4, None), (5, 0, 2, None),
                                             (12, 3, 16, None), (7, 5, 3, (48, 48, 256)), (9, 9, 4, (48, 48, 256))])
def test_pair_equals_separate_calls(nf, na, k, launch):
    """pde_wave_pair (forward recomputation of one segment beside the adjoint of
    another) is bit-identical to pde_wave_forward + pde_wave_adjoint: the packed
    register-list kernel, and with 48x48 tiles of 256 threads (more than 8
    rectangle cells per thread) the general loop."""
    import ctypes as C
    from pde_module_b200 import _lib
    if launch is not None:
        _lib.check(_lib.lib().pde_set_launch_2d(*launch), "pde_set_launch_2d")
    try:
        _pair_vs_separate(nf, na, k)
    finally:
        _lib.lib().pde_set_launch_2d(0, 0, 0)


def _pair_vs_separate(nf, na, k):
    import ctypes as C
    from pde_module_b200 import _lib
    K, u0, src, cell, N, dx, _, _ = _setup(X=70, Y=90, N=20)
    X, Y = K.shape[:2]
    rng = np.random.default_rng(8)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()
    inside = interior_mask((X, Y, 1), 1, "cuda")
    Kd, srcd = dev(K), dev(src)
    up, uc = dev(u0) * inside, dev(rng.standard_normal((X, Y, 1, 1)) * 1e-3) * inside
    m1, m2 = dev(rng.standard_normal((X, Y, 1, 1))) * inside, dev(rng.standard_normal((X, Y, 1, 1))) * inside
    la = dev(rng.standard_normal((max(na, 1), X, Y)))
    gK0 = dev(rng.standard_normal((X, Y, 1, 1)))
    grid = _lib.make_grid((X, Y, 1), 1, 2, dx)
    L = _lib.lib()
    P = lambda t: C.c_void_p(t.data_ptr())
    # separate calls
    lf_ref = torch.zeros((max(nf, 1), X, Y), device="cuda")
    work = torch.zeros((6, X * Y), device="cuda")
    o1, o2 = torch.empty_like(uc), torch.empty_like(uc)
    if nf:
        _lib.check(L.pde_wave_forward(P(Kd), P(up), P(uc), P(o1), P(o2), P(srcd), cell, 3, nf, k, P(lf_ref),
                                      P(work), C.byref(grid), None), "fwd")
    g_ref = gK0.clone()
    r1, r2 = m1.clone(), m2.clone()
    if na:
        r1, r2 = torch.empty_like(m1), torch.empty_like(m2)
        _lib.check(L.pde_wave_adjoint(P(Kd), P(m1), P(m2), P(r1), P(r2), P(la), P(g_ref), na, k, P(work),
                                      C.byref(grid), None), "adj")
    # paired
    lf = torch.zeros_like(lf_ref)
    g = gK0.clone()
    q1, q2 = m1.clone(), m2.clone()
    if na:
        q1, q2 = torch.empty_like(m1), torch.empty_like(m2)
    _lib.check(L.pde_wave_pair(P(Kd), P(up), P(uc), 3, nf, P(lf), P(m1), P(m2), P(q1), P(q2), P(la), P(g), na,
                               P(srcd), cell, k, P(work), C.byref(grid), None), "pair")
    torch.cuda.synchronize()
    ins = inside[:, :, 0, 0].bool()
    for s in range(nf):  # stored Laplacians are defined on the cells inside the node ring
        assert torch.equal(lf[s][ins], lf_ref[s][ins]), s
    assert torch.equal(g, g_ref)
    assert torch.equal(q1, r1) and torch.equal(q2, r2)
