"""Multi-rank host logic on CPU (gloo): slab halo exchange along X against the
single-array periodic fill, and the batched grids' partition across ranks
(every grid once, balanced, and a distributed batch of oracle rollouts equal to
the single-process one)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pde_module_b200.distributed import partition_grids, exchange_slab_halos


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _init(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))


def _halo_worker(rank, world, port, g, periodic, q):
    try:
        _init(rank, world, port)
        nx, Y, Z, N = 5, 4, 3, 2
        glob = torch.arange(world * nx * Y * Z * N, dtype=torch.float32).reshape(world * nx, Y, Z, N)
        slab = torch.full((nx + 2 * g, Y, Z, N), -1.0)
        slab[g:g + nx] = glob[rank * nx:(rank + 1) * nx]
        exchange_slab_halos(slab, g, periodic=periodic)
        # expected: the global array's periodic (or absent) neighbours
        lo = [(rank * nx - g + j) for j in range(g)]
        hi = [((rank + 1) * nx + j) for j in range(g)]
        ok = torch.equal(slab[g:g + nx], glob[rank * nx:(rank + 1) * nx])
        for j, x in enumerate(lo):
            if periodic or x >= 0:
                ok &= torch.equal(slab[j], glob[x % (world * nx)])
            else:
                ok &= bool((slab[j] == -1.0).all())
        for j, x in enumerate(hi):
            if periodic or x < world * nx:
                ok &= torch.equal(slab[nx + g + j], glob[x % (world * nx)])
            else:
                ok &= bool((slab[nx + g + j] == -1.0).all())
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, bool(ok)))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e)))


@pytest.mark.parametrize("world,g,periodic", [(2, 1, True), (2, 2, True), (2, 1, False), (3, 2, True),
                                              (3, 1, False)])
def test_slab_halo_exchange(world, g, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_halo_worker, args=(r, world, port, g, periodic, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
    assert res == {r: True for r in range(world)}, res


def test_partition_grids_balanced_and_complete():
    rng = np.random.default_rng(3)
    sides = rng.integers(64, 1025, size=(64, 2))
    cells = [int(a) * int(b) for a, b in sides]
    for world in (1, 2, 3, 4, 8):
        parts = partition_grids(cells, world)
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = [sum(cells[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells)
        assert parts == partition_grids(cells, world)  # deterministic
    assert partition_grids([5, 5, 5], 2) == [[0, 2], [1]]
    with pytest.raises(ValueError):
        partition_grids(cells, 0)


def _batched_worker(rank, world, port, q):
    try:
        from oracle import fdm
        _init(rank, world, port)
        rng = np.random.default_rng(3)
        sides = rng.integers(6, 20, size=(7, 2))
        cells = [int(a + 2) * int(b + 2) for a, b in sides]
        mine = partition_grids(cells, world)[rank]
        out = {}
        for i in mine:
            sx, sy = (int(s) for s in sides[i])
            u0 = np.random.default_rng(5 + i).random((sx + 2, sy + 2, 1, 1)).astype(np.float32)
            dx = 1.0 / max(sx, sy)
            groups = fdm.standard_groups((sx + 2, sy + 2, 1), 1, [("ALL", 1, 0.0, (0,))])
            out[i] = fdm.heat_rollout(u0, groups, dx, 1, 0.5, 0.2 * dx * dx / 0.5, 9)
        gathered = [None] * world
        dist.all_gather_object(gathered, out)
        dist.destroy_process_group()
        merged = {}
        for d in gathered:
            assert not set(d) & set(merged)
            merged.update(d)
        q.put((rank, merged))
    except Exception as e:
        q.put((rank, repr(e)))


def test_distributed_batch_equals_single_process():
    from oracle import fdm
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_batched_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
    for r in range(world):
        assert isinstance(res[r], dict), res[r]
    merged = res[0]
    assert sorted(merged) == list(range(7))
    rng = np.random.default_rng(3)
    sides = rng.integers(6, 20, size=(7, 2))
    for i, (sx, sy) in enumerate(sides):
        sx, sy = int(sx), int(sy)
        u0 = np.random.default_rng(5 + i).random((sx + 2, sy + 2, 1, 1)).astype(np.float32)
        dx = 1.0 / max(sx, sy)
        groups = fdm.standard_groups((sx + 2, sy + 2, 1), 1, [("ALL", 1, 0.0, (0,))])
        assert np.array_equal(merged[i], fdm.heat_rollout(u0, groups, dx, 1, 0.5, 0.2 * dx * dx / 0.5, 9))


def test_slab_rows_and_local_exchange():
    from pde_module_b200.time_step.fractional_step import slab_rows
    from pde_module_b200.distributed import exchange_local_slabs
    rows = slab_rows(50, 3, 4)
    assert [r[0] for r in rows] == [0, 16, 33] and rows[-1][1] == 50
    assert all(hl == max(lo - 4, 0) and hh == min(hi + 4, 50) for lo, hi, hl, hh in rows)
    with pytest.raises(ValueError):
        slab_rows(20, 4, 6)  # 5 rows per slab < halo
    glob = torch.arange(50 * 3, dtype=torch.float32).reshape(50, 3)
    fields = [torch.full((hh - hl, 3), -1.0) for lo, hi, hl, hh in rows]
    for f, (lo, hi, hl, hh) in zip(fields, rows):
        f[lo - hl:hi - hl] = glob[lo:hi]
    exchange_local_slabs(fields, 4)
    for f, (lo, hi, hl, hh) in zip(fields, rows):
        assert torch.equal(f, glob[hl:hh])


# ---------------------------------------------------------------- slab heat ---
# Global 3D heat problem of the slab tests: Dirichlet 0.25 on every face, then
# Neumann 0.5 on -Y and a Dirichlet ramp to 0.8 on +Z (t_max inside the run).
def _slab_groups(shape, g, dt, nsteps):
    from oracle import fdm
    G = fdm.exterior_groups(shape, g)
    return [dict(ids=G["ALL"], type=1, value=0.25, comps=(0,), func="constant"),
            dict(ids=G["-Y"], type=2, value=0.5, comps=(0,), func="constant"),
            dict(ids=G["+Z"], type=1, value=0.8, comps=(0,), func="ramp", t_max=0.5 * nsteps * dt)]


def _slab_problem(order, X):
    g = order // 2
    shape = (X, 7 + 2 * g, 6 + 2 * g)
    rng = np.random.default_rng(11)
    u0 = rng.random(shape + (1,)).astype(np.float32)
    dx = 1.0 / (shape[1] - 2 * g - 1)
    return g, shape, u0, dx, 0.15 * dx * dx


def _oracle_stepper(slab, g, order, dx, dt, nsteps_total, t0):
    """The oracle's heat steps over the slab array, with the slab's own face groups."""
    from oracle import fdm

    def step(src, dst, nsteps, n0):
        u = src.numpy()
        groups = _slab_groups(u.shape[:3], g, dt, nsteps_total)
        for n in range(nsteps):
            u = fdm.heat_step(u, groups, dx, g, 1.0, dt, order, np.float32, t0 + (n0 + n) * dt)
        dst.copy_(torch.from_numpy(u))
    return step


def _slab_reference(u0, g, order, dx, dt, nsteps, t0):
    from oracle import fdm
    groups = _slab_groups(u0.shape[:3], g, dt, nsteps)
    u = u0
    for n in range(nsteps):
        u = fdm.heat_step(u, groups, dx, g, 1.0, dt, order, np.float32, t0 + n * dt)
    return u


def _make_slab(rank, world, order, k, X, nsteps, t0, local=False):
    from pde_module_b200.FDM.boundary import GridBoundary
    from pde_module_b200.distributed import SlabHeatRollout
    g, shape, u0, dx, dt = _slab_problem(order, X)
    bc = GridBoundary(torch.zeros(shape + (1,)), dx, g)
    holder = {}
    kw = dict(rank=rank, world=world) if local else {}
    s = SlabHeatRollout(bc, dx, 1.0, dt, X, order=order, steps_per_pass=k, device="cpu",
                        stepper=lambda *a: holder["f"](*a), **kw)
    holder["f"] = _oracle_stepper(s, g, order, dx, dt, nsteps, t0)
    s.load(torch.from_numpy(u0))
    ref = _slab_reference(u0, g, order, dx, dt, nsteps, t0)
    return s, ref


def _slab_worker(rank, world, port, order, k, X, nsteps, t0, q):
    try:
        _init(rank, world, port)
        s, ref = _make_slab(rank, world, order, k, X, nsteps, t0)
        s(nsteps - 2, t0)   # two calls: the step count carries over
        got = s(2, t0).numpy()
        a, b = s.own
        ok = bool(np.array_equal(got, ref[a:b]))
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e)))


def test_slab_partition_and_halo():
    from pde_module_b200.distributed import slab_partition, slab_halo
    for X, g, world in [(516, 2, 4), (514, 1, 8), (25, 2, 3), (10, 1, 1)]:
        parts = slab_partition(X, g, world)
        assert parts[0][0] == 0 and parts[-1][1] == X
        assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
        sizes = [b - a for a, b in parts]
        inner = [sizes[0] - g] + sizes[1:-1] + [sizes[-1] - g] if world > 1 else [sizes[0] - 2 * g]
        assert max(inner) - min(inner) <= 1 and sum(inner) == X - 2 * g
    assert slab_halo(1, 2, 2) == 4 and slab_halo(2, 4, 1) == 5
    with pytest.raises(ValueError):
        slab_partition(6, 2, 3)


@pytest.mark.parametrize("world,order,k,nsteps", [(2, 2, 3, 7), (2, 4, 1, 5), (3, 4, 2, 7), (3, 2, 2, 6)])
def test_slab_heat_rollout_equals_single_array(world, order, k, nsteps):
    """gloo ranks, each stepping its slab (halo planes beside the cuts, exchanged
    every k steps) with the oracle: the owned planes equal the whole-array run,
    with Dirichlet, Neumann and ramp groups and a block that ends short."""
    X = world * (order // 2 + k * (order // 2) + 1) + order + 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_slab_worker, args=(r, world, port, order, k, X, nsteps, 0.25, q))
          for r in range(world)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
    assert res == {r: True for r in range(world)}, res


@pytest.mark.parametrize("world,order,k", [(1, 2, 2), (2, 2, 2), (4, 2, 1), (3, 4, 2)])
def test_local_slabs_equal_single_array(world, order, k):
    """The same decomposition with all slabs in one process (advance_local_slabs)."""
    from pde_module_b200.distributed import advance_local_slabs
    X = world * (order // 2 + k * (order // 2) + 1) + order + 2
    nsteps = 2 * k + 1
    slabs, ref = zip(*[_make_slab(r, world, order, k, X, nsteps, 0.0, local=True) for r in range(world)])
    advance_local_slabs(list(slabs), nsteps)
    for s in slabs:
        a, b = s.own
        assert np.array_equal(s.owned.numpy(), ref[0][a:b]), s.rank
    with pytest.raises(RuntimeError):
        if world > 1:
            slabs[0](1)
        else:
            raise RuntimeError


def _lost_rank_worker(rank, world, port, q):
    """Rank 1 leaves before the exchange; rank 0's exchange must end with an error
    (the peer's connection closes, or the 10 s process-group timeout runs out)."""
    import time
    from datetime import timedelta
    from pde_module_b200.distributed import exchange_cut_planes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))
    if rank == 1:
        q.put((1, "left"))
        q.close()
        q.join_thread()  # the message is out before the process goes
        os._exit(0)  # gone without a goodbye: no destroy_process_group
    field = torch.zeros((4 + 3, 5, 6, 1))
    t0 = time.time()
    try:
        exchange_cut_planes(field, 0, 4, 3)
        q.put((0, "no error"))
    except Exception as e:  # the lost peer is reported, not waited on forever
        q.put((0, f"error after {time.time() - t0:.1f} s: {type(e).__name__}"))


def test_slab_exchange_reports_a_lost_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_lost_rank_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    assert res[1] == "left"
    assert res[0].startswith("error after"), res[0]
