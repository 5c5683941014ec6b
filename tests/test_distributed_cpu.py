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
