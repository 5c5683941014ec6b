"""The C-ABI library on CPU: it loads, exports every symbol the header
declares, validates arguments without touching a GPU, and its host-side
boundary-rule compiler reproduces the group-by-group semantics of the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import fdm
from pde_module_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pde_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|uint64_t|const char\*)\s+(pde_\w+)\s*\(", txt, flags=re.M)))


def test_library_loads_and_exports_header_symbols():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 11
    for s in syms:
        assert hasattr(L, s), s
    assert set(_lib.exported_symbols()) >= set(syms)
    assert L.pde_version() >= 100
    assert L.pde_strerror(_lib.PDE_ERR_GHOST).decode().startswith("ghost")


def test_argument_validation_needs_no_gpu():
    L = _lib.lib()
    g = _lib.make_grid((8, 8, 1), 1, 2, 0.1)
    assert L.pde_laplacian(None, None, C.byref(g), 1, 1.0, None) == _lib.PDE_ERR_ARG
    bad = _lib.make_grid((8, 8, 1), 0, 2, 0.1)
    assert L.pde_laplacian(C.c_void_p(16), C.c_void_p(32), C.byref(bad), 1, 1.0, None) == _lib.PDE_ERR_GHOST
    o3 = _lib.make_grid((8, 8, 1), 1, 3, 0.1)
    assert L.pde_grad(C.c_void_p(16), C.c_void_p(32), C.byref(o3), 1, 1.0, None) == _lib.PDE_ERR_SHAPE
    assert L.pde_euler(None, None, 0.1, None, 4, None) == _lib.PDE_ERR_ARG
    r = _lib.PdeBCRules()
    grp = (_lib.PdeBCGroup * 1)()
    grp[0].type, grp[0].comp_mask, grp[0].face_mask = 1, 1, 0  # custom node list: not fusable
    assert L.pde_bc_compile(grp, 1, C.byref(g), 1, C.byref(r)) == _lib.PDE_ERR_UNSUPPORTED


def test_heat_pass_depth_needs_no_gpu():
    """The depth pde_heat_rollout runs (the slab rollout sizes its halos by it)."""
    L = _lib.lib()
    d = lambda shape, g, order, N, k: L.pde_heat_pass_depth(C.byref(_lib.make_grid(shape, g, order, 0.1)), N, k)
    assert d((66, 66, 1), 1, 2, 1, 0) == 8 and d((66, 66, 1), 1, 2, 1, 5) == 5    # 2D: 8 unless asked
    # 3D: 1 where the one-step streaming path applies (even Y and Z), else 2 (order 2) / 1 (order 4)
    assert d((514, 514, 514), 1, 2, 1, 0) == 1 and d((516, 516, 516), 2, 4, 1, 0) == 1
    assert d((514, 513, 514), 1, 2, 1, 0) == 2 and d((516, 515, 516), 2, 4, 1, 0) == 1
    assert d((40, 40, 40), 1, 2, 1, 9) == 4 and d((40, 40, 40), 1, 2, 3, 4) == 2  # capped per component count
    assert d((40, 4, 40), 1, 2, 1, 3) == 1                                          # 2 interior rows: one step per pass
    assert d((40, 40, 40), 1, 2, 0, 0) == _lib.PDE_ERR_ARG
    assert L.pde_heat_pass_depth(None, 1, 0) == _lib.PDE_ERR_ARG


def test_ramp_rules_compile_and_only_the_timed_rollout_takes_them():
    """A ramp group compiles with has_ramp set; pde_heat_rollout (constant groups)
    refuses such rules before touching any memory, pde_heat_rollout_at validates
    its arguments the same way."""
    L = _lib.lib()
    g = _lib.make_grid((8, 8, 1), 1, 2, 0.1)
    grp = (_lib.PdeBCGroup * 2)()
    grp[0].type, grp[0].comp_mask, grp[0].face_mask, grp[0].func, grp[0].value = 1, 1, 0xF, 0, 0.0
    grp[1].type, grp[1].comp_mask, grp[1].face_mask = 1, 1, 1 << 3  # +Y
    grp[1].func, grp[1].value, grp[1].t_max = _lib.PDE_BC_FUNC_RAMP, 1.0, 0.5
    r = _lib.PdeBCRules()
    assert L.pde_bc_compile(grp, 2, C.byref(g), 1, C.byref(r)) == _lib.PDE_OK
    assert r.has_ramp == 1 and r.group[1].func == _lib.PDE_BC_FUNC_RAMP and r.group[1].t_max == 0.5
    p = [C.c_void_p(16), C.c_void_p(32), C.c_void_p(48)]
    assert L.pde_heat_rollout(*p, C.byref(g), 1, C.byref(r), 1.0, 1e-3, 4, 0, None) == _lib.PDE_ERR_UNSUPPORTED
    assert L.pde_heat_rollout_at(None, None, None, C.byref(g), 1, C.byref(r), 1.0, 1e-3, 4, 0, 0.0, 1e-3,
                                 None) == _lib.PDE_ERR_ARG
    assert L.pde_heat_rollout_at(*p, C.byref(g), 2, C.byref(r), 1.0, 1e-3, 4, 0, 0.0, 1e-3,
                                 None) == _lib.PDE_ERR_ARG  # ncomp differs from the rules'


# ---- rule compiler ----------------------------------------------------------
def compile_rules(shape, g, ncomp, spec, dx=0.1):
    """spec: (name, type, value, comps)"""
    L = _lib.lib()
    arr = (_lib.PdeBCGroup * len(spec))()
    for i, (name, typ, val, comps) in enumerate(spec):
        mask = 0
        for c in comps:
            mask |= 1 << c
        fm = 0
        if name == "ALL":
            for a in range(3):
                if shape[a] > 1:
                    fm |= 3 << (2 * a)
        else:
            fm = _lib.FACE_BITS[name]
        arr[i].type, arr[i].comp_mask, arr[i].func, arr[i].value, arr[i].face_mask = typ, mask, 0, val, fm
    grid = _lib.make_grid(shape, g, 2, dx)
    r = _lib.PdeBCRules()
    assert L.pde_bc_compile(arr, len(spec), C.byref(grid), ncomp, C.byref(r)) == 0
    return r


def apply_rules(u, r, g, dx):
    """NumPy model of the fused kernels' per-cell boundary evaluation (fused.cuh: bc_eval)."""
    gs = u.shape[:3]
    out = u.copy()
    N = u.shape[3]

    def cls(i, n, elig):
        if not elig:
            return 1
        return 0 if i == g else (2 if i == n - 1 - g else 1)

    for c in np.ndindex(*gs):
        ghost_axes, deep = [], False
        for a in range(3):
            if gs[a] == 1:
                continue
            if c[a] < g or c[a] > gs[a] - 1 - g:
                if c[a] in (g - 1, gs[a] - g):
                    ghost_axes.append(a)
                else:
                    deep = True
        for v in range(N):
            if deep or len(ghost_axes) > 1:
                continue
            if ghost_axes:
                a = ghost_axes[0]
                inc = 1 if c[a] == g - 1 else -1
                p = list(c)
                p[a] += inc
                K = cls(p[0], gs[0], gs[0] > 1) * 9 + cls(p[1], gs[1], gs[1] > 1) * 3 + cls(p[2], gs[2], gs[2] > 1)
                gi = r.ghost_group[K][a][v]
                if gi < 0:
                    continue
                p[a] += inc
                G = r.group[gi]
                a_val = u[tuple(p) + (v,)]
                val = np.float32(G.value)
                if G.type == 1:
                    out[c + (v,)] = np.float32(2.0) * val - a_val
                else:
                    out[c + (v,)] = (np.float32(-2 * inc) * np.float32(r.dx32)) * val + a_val
            else:
                K = cls(c[0], gs[0], gs[0] > 1) * 9 + cls(c[1], gs[1], gs[1] > 1) * 3 + cls(c[2], gs[2], gs[2] > 1)
                if K == 13:
                    continue
                gi = r.node_group[K]
                if gi >= 0 and (r.group[gi].comp_mask >> v) & 1:
                    out[c + (v,)] = np.float32(r.group[gi].value)
    return out


SPECS = [
    ((9, 8, 1), 1, 1, [("ALL", 1, 0.0, (0,))]),
    ((9, 8, 1), 1, 2, [("ALL", 1, 0.0, (0, 1)), ("+Y", 1, 1.0, (0,))]),
    ((9, 8, 1), 1, 1, [("ALL", 2, 0.0, (0,))]),
    ((9, 8, 1), 2, 2, [("-X", 2, 0.5, (0, 1)), ("-X", 1, 0.0, (0,)), ("+Y", 2, -1.5, (1,))]),
    ((7, 6, 5), 1, 3, [("ALL", 1, 0.0, (0, 1, 2)), ("+Z", 1, 2.0, (2,)), ("-Y", 2, 0.25, (0,))]),
    ((6, 7, 8), 1, 1, [("-X", 1, 1.0, (0,)), ("+X", 1, -1.0, (0,)), ("ALL", 2, 0.0, (0,))]),
]


@pytest.mark.parametrize("shape,g,N,spec", SPECS)
def test_compiled_rules_match_group_semantics(shape, g, N, spec):
    rng = np.random.default_rng(7)
    dx = 0.1
    u = rng.standard_normal(shape + (N,)).astype(np.float32)
    groups = fdm.standard_groups(shape, g, spec)
    ref = fdm.bc_apply(u, groups, dx, g)
    r = compile_rules(shape, g, N, spec, dx)
    got = apply_rules(u, r, g, dx)
    np.testing.assert_array_equal(got, ref)


def _batch_desc(shapes, ptr0=1 << 20):
    arr = (_lib.PdeBatchGrid * len(shapes))()
    for i, (X, Y) in enumerate(shapes):
        arr[i].field = ptr0 + i * (1 << 16)
        arr[i].field_prev = ptr0 + (1 << 30) + i * (1 << 16)
        arr[i].scratch = ptr0 + (1 << 31) + i * (1 << 16)
        arr[i].shape[0], arr[i].shape[1] = X, Y
        arr[i].dx, arr[i].coef, arr[i].dt = 0.1, 1.0, 0.001
    return arr


def test_batch_plan_validation_needs_no_gpu():
    L = _lib.lib()
    shapes = [(66, 130), (10, 7), (1026, 514)]
    desc = _batch_desc(shapes)
    nb = C.c_uint64(0)
    assert L.pde_batch_work_bytes(desc, 3, 32, 64, C.byref(nb)) == _lib.PDE_OK
    tiles = sum(-(-X // 32) * -(-Y // 64) for X, Y in shapes)
    # descriptor table (device layout, 256-byte aligned) + queue head + one progress word per tile
    assert 4 * tiles + 512 <= nb.value <= 4 * tiles + 256 + 256 * 3
    assert L.pde_batch_work_bytes(desc, 0, 32, 64, C.byref(nb)) == _lib.PDE_ERR_ARG
    bad = _batch_desc([(0, 10)])
    assert L.pde_batch_work_bytes(bad, 1, 32, 64, C.byref(nb)) == _lib.PDE_ERR_SHAPE
    # rules for the heat kind: Dirichlet 0 on every face of a 2D grid
    grp = (_lib.PdeBCGroup * 1)()
    grp[0].type, grp[0].comp_mask, grp[0].face_mask = _lib.PDE_BC_DIRICHLET, 1, 0xF
    rules = _lib.PdeBCRules()
    g2 = _lib.make_grid((66, 130, 1), 1, 2, 0.1)
    assert L.pde_bc_compile(grp, 1, C.byref(g2), 1, C.byref(rules)) == _lib.PDE_OK
    plan = _lib.PdeBatchPlan()
    work = C.c_void_p(1 << 24)
    big = 1 << 30

    def plan_rc(kind=_lib.PDE_BATCH_HEAT, d=desc, n=3, g=1, order=2, r=rules, tx=32, ty=64, k=8, w=work, wb=big):
        return L.pde_batch_plan(kind, d, n, g, order, C.byref(r) if r is not None else None, tx, ty, k, w, wb,
                                C.byref(plan), None)

    assert plan_rc(kind=7) == _lib.PDE_ERR_ARG
    assert plan_rc(order=3) == _lib.PDE_ERR_ARG
    assert plan_rc(kind=_lib.PDE_BATCH_WAVE, order=4, g=2) == _lib.PDE_ERR_UNSUPPORTED
    assert plan_rc(g=0) == _lib.PDE_ERR_GHOST
    assert plan_rc(r=None) == _lib.PDE_ERR_ARG
    assert plan_rc(k=40) == _lib.PDE_ERR_ARG        # halo 41 wider than the 32-cell tile side
    assert plan_rc(tx=16, k=16) == _lib.PDE_ERR_ARG
    assert plan_rc(wb=16) == _lib.PDE_ERR_TOO_LARGE
    assert plan_rc(w=C.c_void_p((1 << 24) + 4)) == _lib.PDE_ERR_ALIGN
    assert plan_rc(tx=256, ty=256, k=16) == _lib.PDE_ERR_TOO_LARGE  # shared-memory region too large
    tiny = _batch_desc([(3, 40)])
    assert plan_rc(d=tiny, n=1) == _lib.PDE_ERR_SHAPE
    # a heat plan with ramp groups runs only through pde_batch_rollout_at
    ramp_plan = _lib.PdeBatchPlan()
    ramp_plan.table = 1 << 24
    ramp_plan.kind, ramp_plan.steps_per_pass, ramp_plan.total_tiles = _lib.PDE_BATCH_HEAT, 4, 1
    ramp_plan.rules.has_ramp = 1
    assert L.pde_batch_rollout(C.byref(ramp_plan), 5, None) == _lib.PDE_ERR_UNSUPPORTED
    assert L.pde_batch_rollout_at(None, 5, 0.0, None) == _lib.PDE_ERR_ARG
    assert L.pde_batch_rollout(None, 5, None) == _lib.PDE_ERR_ARG
    assert L.pde_batch_rollout(C.byref(_lib.PdeBatchPlan()), 5, None) == _lib.PDE_ERR_ARG


def test_wave_pair_validation_needs_no_gpu():
    L = _lib.lib()
    g = _lib.make_grid((20, 20, 1), 1, 2, 0.1)
    p = C.c_void_p(1 << 20)
    args = lambda **kw: dict(dict(K=p, up=p, uc=p, n0=0, nf=3, lf=p, m1=p, m2=p, o1=p, o2=p, la=p, gk=p, na=3,
                                  src=None, cell=-1, k=2, work=p), **kw)

    def call(**kw):
        a = args(**kw)
        return L.pde_wave_pair(a["K"], a["up"], a["uc"], a["n0"], a["nf"], a["lf"], a["m1"], a["m2"], a["o1"],
                               a["o2"], a["la"], a["gk"], a["na"], a["src"], a["cell"], a["k"], a["work"],
                               C.byref(g), None)
    assert call(K=None) == _lib.PDE_ERR_ARG
    assert call(nf=-1) == _lib.PDE_ERR_ARG
    assert call(lf=None) == _lib.PDE_ERR_ARG
    assert call(la=None) == _lib.PDE_ERR_ARG
    assert call(cell=5) == _lib.PDE_ERR_ARG          # a source cell needs source samples
    assert call(nf=0, na=0) == _lib.PDE_OK           # nothing to do
    assert call(nf=0, lf=None, up=None, uc=None, na=0) == _lib.PDE_OK
