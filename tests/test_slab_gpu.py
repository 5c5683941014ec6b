"""Slab decomposition of the fused 3D heat rollout on one GPU: slabs along X,
each with halo planes beside its cuts, advanced in blocks of k steps (one
fused pass per block, halos exchanged between blocks), against the fused
rollout of the whole array, bit for bit.  The ranks are emulated as several
slabs in one process (advance_local_slabs); the exchange across processes is
covered on CPU (test_distributed_cpu.py)."""
import numpy as np
import pytest
import torch

import pde_module_b200 as P
from pde_module_b200.FDM.boundary import get_ramp_func
from pde_module_b200.distributed import SlabHeatRollout, advance_local_slabs

pytestmark = pytest.mark.gpu


def _problem(shape, g, N, ramp, seed):
    """Field U[0,1), dx, and a builder of the boundary: Dirichlet 0.25 on all
    faces, Neumann 0.5 on -Y, and with ramp > 0 a Dirichlet ramp to 0.8 over
    t_max = ramp on +Z (component 0)."""
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    u = torch.rand(shape + (N,), device="cuda", generator=gen)
    dx = 1.0 / (shape[1] - 2 * g - 1)

    def boundary(field):
        bc = P.GridBoundary(field, dx, g)
        bc.dirichlet_BC("ALL", 0.25)
        bc.vonNeumann_BC("-Y", 0.5)
        if ramp:
            bc.set_BC("+Z", get_ramp_func(0.8, ramp, output_ids=(0,)), 1, (0,))
        return bc
    return u, dx, boundary


CASES = [
    # global array shape, order, components, slabs, steps per pass, steps, ramp
    ((61, 37, 33), 2, 1, 2, 2, 9, False),
    ((61, 37, 33), 2, 1, 3, 4, 9, True),
    ((64, 30, 41), 4, 1, 3, 1, 5, False),
    ((70, 30, 41), 4, 1, 2, 2, 7, True),
    ((50, 21, 18), 2, 2, 4, 2, 6, False),
    ((52, 22, 19), 4, 3, 2, 2, 5, True),
    ((45, 20, 26), 2, 1, 1, 3, 7, False),
    # even Y and Z: one step per pass on the streaming kernel after the surface fill
    ((60, 38, 44), 2, 1, 3, 0, 7, True),
    ((64, 36, 40), 4, 1, 2, 0, 5, False),
]


@pytest.mark.parametrize("shape,order,N,world,k,nsteps,ramp", CASES)
def test_slabs_equal_whole_array(shape, order, N, world, k, nsteps, ramp):
    g = order // 2
    dx = 1.0 / (shape[1] - 2 * g - 1)
    dt = 0.15 * dx * dx
    u, dx, boundary = _problem(shape, g, N, 0.5 * nsteps * dt if ramp else 0.0, 3 + world)  # ramp ends mid-run
    whole = P.HeatRollout(boundary(u), dx, 1.0, dt, order=order, steps_per_pass=k)(u.clone(), nsteps, t0=0.1)
    slabs = [SlabHeatRollout(boundary(u), dx, 1.0, dt, shape[0], order=order, steps_per_pass=k, rank=r, world=world)
             for r in range(world)]
    for s in slabs:
        s.load(u)
    advance_local_slabs(slabs, nsteps - 1, t0=0.1)
    advance_local_slabs(slabs, 1, t0=0.1)
    torch.cuda.synchronize()
    for s in slabs:
        a, b = s.own
        assert torch.equal(s.owned, whole[a:b]), (s.rank, a, b)
    if world == 1:
        one = SlabHeatRollout(boundary(u), dx, 1.0, dt, shape[0], order=order, steps_per_pass=k)
        one.load(u)
        assert torch.equal(one(nsteps, t0=0.1), whole)


def test_slab_halo_follows_the_pass_depth():
    """The halo is g + k*R + 1 for the depth the library runs (deeper requests
    are capped: two components run at most 2 steps per pass; a scalar field
    with even Y and Z runs one step per pass by default)."""
    u, dx, boundary = _problem((40, 20, 20), 1, 2, 0.0, 1)
    s = SlabHeatRollout(boundary(u), dx, 1.0, 0.1 * dx * dx, 40, steps_per_pass=4, rank=0, world=2)
    assert s.k == 2 and s.halo == 1 + 2 + 1
    s = SlabHeatRollout(boundary(u[..., :1]), dx, 1.0, 0.1 * dx * dx, 40, steps_per_pass=0, rank=1, world=2)
    assert s.k == 1 and s.h_lo == 3 and s.h_hi == 0
    s = SlabHeatRollout(boundary(u[:, :19, :19, :1]), dx, 1.0, 0.1 * dx * dx, 40, steps_per_pass=0, rank=0, world=2)
    assert s.k == 2 and s.h_lo == 0 and s.h_hi == 4
