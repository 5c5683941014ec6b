"""Oracle self-checks on CPU: exactness on polynomials, float32 vs float64,
group construction, boundary formulas and the periodic fill."""
import numpy as np
import pytest

from oracle import fdm


def _field(shape, rng, n=1):
    return rng.standard_normal(tuple(shape) + (n,)).astype(np.float32)


@pytest.mark.parametrize("order", [2, 4])
def test_laplacian_exact_on_quadratic(order):
    g = order // 2
    n = 9 + 2 * g
    dx = 0.25
    x = (np.arange(n) - g) * dx
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u = (X ** 2 + 2 * Y ** 2 - Z ** 2)[..., None]
    lap = fdm.laplacian(u, dx, g, 1.0, order, dtype=np.float64)
    core = (slice(g, n - g),) * 3
    np.testing.assert_allclose(lap[core], 4.0, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("order", [2, 4])
def test_grad_div_exact_on_linear(order):
    g = order // 2
    n = 8 + 2 * g
    dx = 0.5
    x = (np.arange(n) - g) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    u = (3 * X - 2 * Y)[:, :, None, None]
    gr = fdm.grad(u, dx, g, 1.0, order, dtype=np.float64)
    core = (slice(g, n - g), slice(g, n - g), 0)
    np.testing.assert_allclose(gr[core][..., 0], 3.0, atol=1e-12)
    np.testing.assert_allclose(gr[core][..., 1], -2.0, atol=1e-12)
    v = np.stack([X * 2.0, Y * 5.0], axis=-1)[:, :, None, :]
    dv = fdm.divergence(v, dx, g, 1.0, order, dtype=np.float64)
    np.testing.assert_allclose(dv[core][..., 0], 7.0, atol=1e-12)


def test_float32_tracks_float64(rng):
    u = _field((12, 10, 9), rng, 3)
    a = fdm.laplacian(u, 0.1, 1, 0.7, 2, np.float32)
    b = fdm.laplacian(u.astype(np.float64), 0.1, 1, 0.7, 2, np.float64)
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel < 1e-6


def test_groups_match_reference_construction():
    gs, g = (7, 6, 1), 1
    G = fdm.exterior_groups(gs, g)
    assert set(G) == {"-X", "+X", "-Y", "+Y", "ALL"}
    ids = np.arange(np.prod(gs)).reshape(gs)
    np.testing.assert_array_equal(G["-X"], ids[1, 1:-1, :].ravel())
    np.testing.assert_array_equal(G["+Y"], ids[1:-1, -2, :].ravel())
    assert G["ALL"].dtype == np.int32
    assert np.all(np.diff(G["ALL"]) > 0)
    # the perimeter of a 5x4 node box
    assert len(G["ALL"]) == 2 * 5 + 2 * 4 - 4


def test_dirichlet_and_neumann_formulas():
    gs, g, dx = (6, 5, 1), 1, 0.5
    u = np.arange(np.prod(gs), dtype=np.float32).reshape(gs + (1,))
    G = fdm.exterior_groups(gs, g)
    out = fdm.bc_apply(u, [dict(ids=G["-X"], type=fdm.DIRICHLET, value=3.0, comps=(0,))], dx, g)
    # node (1, j) := 3, ghost (0, j) := 2*3 - u(2, j)
    for j in range(1, 4):
        assert out[1, j, 0, 0] == 3.0
        assert out[0, j, 0, 0] == np.float32(6.0) - u[2, j, 0, 0]
    out = fdm.bc_apply(u, [dict(ids=G["+Y"], type=fdm.VON_NEUMANN, value=2.0, comps=(0,))], dx, g)
    # high side: inc = -1 -> ghost (i, 4) := +2*dx*val + u(i, 2); node untouched
    for i in range(1, 5):
        assert out[i, 4, 0, 0] == np.float32(2.0 * 0.5 * 2.0) + u[i, 2, 0, 0]
        assert out[i, 3, 0, 0] == u[i, 3, 0, 0]


def test_later_group_overrides_and_keeps_input_components():
    gs, g = (6, 6, 1), 1
    u = np.random.default_rng(0).standard_normal(gs + (2,)).astype(np.float32)
    G = fdm.exterior_groups(gs, g)
    spec = [dict(ids=G["ALL"], type=1, value=0.0, comps=(0, 1)), dict(ids=G["+Y"], type=1, value=1.0, comps=(0,))]
    out = fdm.bc_apply(u, spec, 0.1, g)
    # lid node: component 0 = 1, component 1 = the pre-boundary input (not 0)
    assert out[3, 4, 0, 0] == 1.0 and out[3, 4, 0, 1] == u[3, 4, 0, 1]
    assert out[1, 2, 0, 0] == 0.0 and out[1, 2, 0, 1] == 0.0


def test_periodic_fill_wraps():
    rng = np.random.default_rng(3)
    u = rng.standard_normal((9, 8, 7, 1)).astype(np.float32)
    out = fdm.periodic_fill(u, 2, (0, 1, 2))
    M = [5, 4, 3]
    for i in range(9):
        for j in range(8):
            for k in range(7):
                s = [2 + ((c - 2) % m) for c, m in zip((i, j, k), M)]
                assert out[i, j, k, 0] == u[s[0], s[1], s[2], 0]


def test_heat_rollout_decays():
    n, g = 18, 1
    dx = 1.0 / (n - 2 * g - 1)
    x = (np.arange(n) - g) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    u = (np.sin(np.pi * X) * np.sin(np.pi * Y))[:, :, None, None].astype(np.float32)
    groups = fdm.standard_groups(u.shape, g, [("ALL", fdm.DIRICHLET, 0.0, (0,))])
    dt = 0.2 * dx * dx
    out = fdm.heat_rollout(u, groups, dx, g, 1.0, dt, 50)
    ratio = out[g:-g, g:-g].max() / u[g:-g, g:-g].max()
    expect = np.exp(-2 * np.pi ** 2 * 50 * dt)
    assert abs(ratio - expect) < 0.02
