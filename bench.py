"""Benchmark of the finite-difference hot path on B200.

Workload (one GPU): the 3D operator sweep on a 512^3 float32 grid — a scalar
field and a 3-component vector field, standard normal values (seeded), ghost
width 1 for order 2 and 2 for order 4, periodic ghosts filled once before
timing.  One step applies, for each order (2 and 4): Laplacian(scalar),
Grad(scalar -> vec3) and Divergence(vec3 -> scalar), i.e. 6 operator
applications over the 512^3 interior.  Metric: cell-updates/s (interior cells
x operator applications / s).  Every input is larger than L2 (126 MB), so no
L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--gpus N > 1 (under torchrun): weak scaling, each rank owns one 512^3 slab of
an (N*512) x 512 x 512 periodic domain; its X ghost planes come from the
neighbouring ranks once before timing (NCCL send/recv), so the timed steps
have no collective.  --impl reference times the CPU restatement of the
reference's operators (oracle/fdm.py, float32, reference operation order) on
the host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_INT = 512
# interior side of the CPU sample of the sweep (both arms time the same sample)
CPU_SAMPLE_N = 128
METRIC = "cell-updates/s (3D operator sweep: Laplacian, Grad, Divergence; order 2 and 4)"
UNIT = "cell-updates/s"
# algorithmic bytes per interior cell: compulsory read once + write once
ALG_BYTES = {"laplacian": 8, "grad": 16, "divergence": 16}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


# ------------------------------------------------------------ clocks ---
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------- CPU baseline ---
def cpu_sweep_sample(n: int, threads: int, reps: int = 1, min_seconds: float = 0.0):
    """Time the float32 oracle over the 6-operator step on an n^3 interior,
    split into X slabs over `threads` threads (NumPy releases the GIL); at least
    `reps` repetitions and at least `min_seconds` of work."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import fdm
    rng = np.random.default_rng(1)
    dx = 1.0 / N_INT
    fields = {}
    for order in (2, 4):
        g = order // 2
        s = n + 2 * g
        fields[order] = (rng.standard_normal((s, s, s, 1), dtype=np.float32),
                         rng.standard_normal((s, s, s, 3), dtype=np.float32))

    def slab_job(order, x0, x1):
        g = order // 2
        u, v = fields[order]
        us, vs = u[x0 - g:x1 + g], v[x0 - g:x1 + g]
        fdm.laplacian(us, dx, g, 1.0, order)
        fdm.grad(us, dx, g, 1.0, order)
        fdm.divergence(vs, dx, g, 1.0, order)

    bounds = np.linspace(0, n, threads + 1).astype(int)
    t0 = time.perf_counter()
    done = 0
    with ThreadPoolExecutor(threads) as ex:
        while done < reps or time.perf_counter() - t0 < min_seconds:
            done += 1
            futs = []
            for order in (2, 4):
                g = order // 2
                for i in range(threads):
                    if bounds[i + 1] > bounds[i]:
                        futs.append(ex.submit(slab_job, order, g + bounds[i], g + bounds[i + 1]))
            for f in futs:
                f.result()
    dt = time.perf_counter() - t0
    return 6 * n ** 3 * done / dt, dt


def _timed_cpu(fn, min_seconds: float):
    t0 = time.perf_counter()
    n = 0
    while n == 0 or time.perf_counter() - t0 < min_seconds:
        fn()
        n += 1
    return n, time.perf_counter() - t0


def cpu_heat_sample(steps: int = 20, min_seconds: float = 2.0) -> dict:
    """The 256^2 heat loop on the host (NumPy float32 restatement, one core), per cell-update."""
    from oracle import fdm
    n, g = 256, 1
    dx = 1.0 / n
    u0 = np.random.default_rng(0).random((n + 2, n + 2, 1, 1)).astype(np.float32)
    groups = fdm.standard_groups(u0.shape[:3], g, [("ALL", 1, 0.0, (0,))])
    reps, dt = _timed_cpu(lambda: fdm.heat_rollout(u0, groups, dx, g, 1.0, 0.2 * dx * dx, steps), min_seconds)
    return {"value": n * n * steps * reps / dt, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"{steps} steps of the 256^2 loop x {reps}, NumPy float32 restatement (oracle/fdm.py)"}


def cpu_ldc_sample(n: int = 256, min_seconds: float = 2.0) -> dict:
    """One fractional step (50 Jacobi sweeps) on the host (NumPy float32 composition), per cell-update."""
    from oracle import fdm
    g = 1
    shape = (n + 2 * g, n + 2 * g, 1)
    dx = 1.0 / (n - 1)
    u = np.zeros(shape + (2,), dtype=np.float32)
    p = np.zeros(shape + (1,), dtype=np.float32)
    ug = fdm.standard_groups(shape, g, [("ALL", 1, 0.0, (0, 1)), ("+Y", 1, 1.0, (0,))])
    pg = fdm.standard_groups(shape, g, [("ALL", 2, 0.0, (0,))])
    nu = 0.01
    dt = 0.2 * min(dx, dx * dx / (4 * nu))
    reps, t = _timed_cpu(lambda: fdm.ldc_step(u, p, ug, pg, dx, g, nu, dt, 50), min_seconds)
    return {"value": n * n * reps / t, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"{reps} fractional steps (50 Jacobi sweeps each) on a {n}^2 grid, NumPy float32 "
                      "composition of the operators (oracle/fdm.py ldc_step); per cell and step"}


def cpu_batched_sample(steps: int = 10, min_seconds: float = 2.0) -> dict:
    """The batched heat workload's first 4 grids on the host, one after the other (NumPy float32)."""
    from oracle import fdm
    sides, alpha, u0, dx, dt = batched_problem()
    grids = range(4)
    cells = sum(int(sides[i][0]) * int(sides[i][1]) for i in grids)

    def run():
        for i in grids:
            u = u0[i][:, :, None, None]
            groups = fdm.standard_groups(u.shape[:3], 1, [("ALL", 1, 0.0, (0,))])
            fdm.heat_rollout(u, groups, dx[i], 1, alpha[i], dt[i], steps)

    reps, t = _timed_cpu(run, min_seconds)
    return {"value": cells * steps * reps / t, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"grids 0-3 of the batch (per-grid loops), {steps} steps x {reps}, NumPy float32 "
                      "restatement (oracle/fdm.py); per cell-update"}


def sweep_config(world: int) -> dict:
    return {"workload": "3D operator sweep 512^3 (Laplacian, Grad, Divergence; order 2 and 4; periodic ghosts)",
            "interior": [N_INT, N_INT, N_INT], "ops_per_step": 6,
            "fields": "scalar (512+2g)^3 and vec3 (512+2g)^3 per order",
            "l2": "inputs larger than L2 (>=543 MB each), no flush",
            "parallelism": f"x-slabs{world}" if world > 1 else "single",
            **({"halo_exchange": "every step, before the operators: the g halo planes of each input field "
                                 "from both X neighbours (periodic), NCCL send/recv into the field's own planes",
                "global_interior": [N_INT * world, N_INT, N_INT]} if world > 1 else {})}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n = CPU_SAMPLE_N
    for _ in range(args.warmup):
        cpu_sweep_sample(n, threads)
    vals = []
    t_all = 0.0
    for _ in range(args.steps):
        v, dt = cpu_sweep_sample(n, threads)
        vals.append(v)
        t_all += dt
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_all / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(sweep_config(args.gpus), cpu_sample_interior=[n, n, n]),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"each step: the 6-operator step on a {n}^3 interior (order 2 and 4), NumPy "
                                   f"float32 restatement of the reference kernels (the reference's own code needs "
                                   f"warp-lang, absent here), X slabs over {threads} threads; value per cell"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU ---
def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    import pde_module_b200 as P
    from pde_module_b200 import _lib

    from pde_module_b200.distributed import exchange_slab_halos
    dx = 1.0 / N_INT
    fast_mods = {}
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1 + rank)
    fields = {}
    for order in (2, 4):
        g = order // 2
        s = N_INT + 2 * g
        u = torch.randn((s, s, s, 1), device="cuda", generator=gen)
        v = torch.randn((s, s, s, 3), device="cuda", generator=gen)
        for f in (u, v):
            bc = P.GridBoundary(f, dx, g)
            bc.periodic("ALL" if world == 1 else ("Y", "Z"))
            f.copy_(bc(f))
        if world > 1:
            exchange_slab_halos(u, g)
            exchange_slab_halos(v, g)
        mods = (P.Laplacian(1, dx, g, order=order), P.Grad(1, u.shape, dx, g, order=order),
                P.Divergence(3, v.shape, dx, g, order=order))
        fast = (P.Laplacian(1, dx, g, order=order, fast=True), P.Grad(1, u.shape, dx, g, order=order, fast=True),
                P.Divergence(3, v.shape, dx, g, order=order, fast=True))
        fields[order] = (u, v, mods)
        fast_mods[order] = fast

    # autotune the streaming kernels' tile configuration for this shape (setup, untimed)
    from pde_module_b200 import tuning
    tuned = {} if args.no_tune else tuning.tune_stream3d(
        (N_INT, N_INT, N_INT), reps=3, kinds=[("laplacian", 1), ("grad", 1), ("divergence", 3)])

    ops = []
    for order in (2, 4):
        u, v, (lap, grd, div) = fields[order]
        ops.append((f"laplacian_o{order}", lambda u=u, lap=lap: lap(u, 1.0), ALG_BYTES["laplacian"]))
        ops.append((f"grad_o{order}", lambda u=u, grd=grd: grd(u, 1.0), ALG_BYTES["grad"]))
        ops.append((f"divergence_o{order}", lambda v=v, div=div: div(v, 1.0), ALG_BYTES["divergence"]))

    fast_ops = []
    for order in (2, 4):
        u, v, _ = fields[order]
        lap, grd, div = fast_mods[order]
        fast_ops.append((f"laplacian_o{order}", lambda u=u, lap=lap: lap(u, 1.0), ALG_BYTES["laplacian"]))
        fast_ops.append((f"grad_o{order}", lambda u=u, grd=grd: grd(u, 1.0), ALG_BYTES["grad"]))
        fast_ops.append((f"divergence_o{order}", lambda v=v, div=div: div(v, 1.0), ALG_BYTES["divergence"]))

    # N > 1: the slabs are cut along X; every step first refreshes each input
    # field's g halo planes from the neighbouring ranks (periodic), in the timed region
    exch = []
    if world > 1:
        for order in (2, 4):
            u, v, _ = fields[order]
            exch.append(lambda u=u, v=v, g=order // 2: (exchange_slab_halos(u, g), exchange_slab_halos(v, g)))

    def step():
        for fn in exch:
            fn()
        for _, fn, _ in ops:
            fn()

    for _ in range(max(args.warmup, 3)):
        step()
        for _, fn, _ in fast_ops:
            fn()
    torch.cuda.synchronize()
    if _lib.device_error() != 0:
        raise RuntimeError("device error during warm-up")

    stream = torch.cuda.current_stream()
    K = args.steps
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in ops]
          for _ in range(K)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    t0.record(stream)
    for k in range(K):
        for fn in exch:
            fn()
        for j, (_, fn, _) in enumerate(ops):
            ev[k][j][0].record(stream)
            fn()
            ev[k][j][1].record(stream)
    t1.record(stream)
    # the same steps with the fast arithmetic mode (reported beside the exact path)
    evf = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in fast_ops]
           for _ in range(K)]
    for k in range(K):
        for j, (_, fn, _) in enumerate(fast_ops):
            evf[k][j][0].record(stream)
            fn()
            evf[k][j][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if world > 1:
        dist.barrier()
    ms = t0.elapsed_time(t1)
    if world > 1:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    per_op = {name: statistics.mean(ev[k][j][0].elapsed_time(ev[k][j][1]) for k in range(K))
              for j, (name, _, _) in enumerate(ops)}
    per_op_fast = {name: statistics.mean(evf[k][j][0].elapsed_time(evf[k][j][1]) for k in range(K))
                   for j, (name, _, _) in enumerate(fast_ops)}
    cells = N_INT ** 3
    ms_step = ms / K
    value = world * cells * len(ops) / (ms_step / 1000.0)
    # each operator alone: R back-to-back launches between two events (inputs larger than L2)
    iso = {}
    R_ISO = 5
    for name, fn, b in ops:
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(R_ISO):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        t_iso = e0.elapsed_time(e1) / R_ISO
        gbs = cells * b / (t_iso / 1000.0) / 1e9
        iso[name] = {"ms": round(t_iso, 4), "achieved_gbs": round(gbs, 1)}

    peak, peak_kind = peaks()
    traffic = traffic_table()
    kern = {}
    for name, _, b in ops:
        gbs = cells * b / (per_op[name] / 1000.0) / 1e9
        kern[name] = {"ms": round(per_op[name], 4), "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    kern_fast = {}
    for name, _, b in fast_ops:
        gbs = cells * b / (per_op_fast[name] / 1000.0) / 1e9
        kern_fast[name] = {"ms": round(per_op_fast[name], 4), "achieved_gbs": round(gbs, 1),
                           "frac": round(gbs / peak, 4)}
    fast_ms_step = sum(per_op_fast.values())
    dom = max(per_op, key=per_op.get)
    dom_b = dict((n, b) for n, _, b in ops)[dom]
    ach = cells * dom_b / (per_op[dom] / 1000.0) / 1e9
    tr = traffic.get(dom)
    roofline = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": tr, "kernel": dom, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": cells * dom_b}

    # end to end through the public API: pinned host fields in, all outputs back
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(fields, ops, world, args, exch)

    heat3d = None
    if world == 1 and not args.no_heat3d:
        heat3d = run_heat3d()
    elif not args.no_heat3d:  # collective: every rank runs its slab
        heat3d = run_heat3d_slabs(world, rank)
    heat = None
    if world == 1 and not args.no_heat:  # a single-GPU workload (replicas only): not run beside other ranks
        heat = run_heat()
        if not args.no_cpu:
            heat["cpu_baseline"] = cpu_heat_sample()
    ldc = None
    if world == 1 and not args.no_ldc:  # a single-GPU workload (replicas only): not run beside other ranks
        ldc = run_ldc()
        if not args.no_cpu:
            ldc["cpu_baseline"] = cpu_ldc_sample()
    wave = None
    if world == 1 and not args.no_wave:  # a single-GPU workload (replicas only): not run beside other ranks
        wave = run_wave()
    wc = None
    if world == 1 and not args.no_wc:  # a single-GPU workload (replicas only): not run beside other ranks
        wc = run_wc()
    batched = None
    if world == 1 and not args.no_batched:  # a single-GPU workload (replicas only): not run beside other ranks
        batched = run_batched(tune=not args.no_tune)
        if not args.no_cpu:
            batched["cpu_baseline"] = cpu_batched_sample()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v, dt = cpu_sweep_sample(CPU_SAMPLE_N, threads, min_seconds=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"the 6-operator step on a {CPU_SAMPLE_N}^3 interior repeated for {dt:.1f} s, NumPy float32 "
                         f"restatement of the reference kernels (oracle/fdm.py), X slabs over {threads} threads"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (standard normal, seeded)",
            "config": sweep_config(world),
            "roofline": roofline, "kernels": kern,
            "kernels_isolated": {n: dict(v, frac=round(v["achieved_gbs"] / peak, 4)) for n, v in iso.items()},
            "fast_mode": {"value": world * cells * len(ops) / (fast_ms_step / 1000.0), "unit": UNIT,
                          "kernels": kern_fast,
                          "note": "PDE_MODE_FAST arithmetic (weights folded, FMA); the headline value is the "
                                  "exact mode, bit-identical to the reference algorithm"},
            "heat_256": heat,
            "ldc_1024": ldc,
            "wave_512": wave,
            "batched_64": batched,
            "wc_cavity": wc,
            "autotune": {f"{k[0]}_n{k[1]}_o{k[2]}": v for k, v in tuned.items()},
            "heat3d_512": heat3d,
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": K * len(ops), "clocks": clocks,
            "summary": leg_summary(kern, heat3d, heat, ldc, wave, batched, wc),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# launch shapes (tile_x, tile_y, threads) tried for the temporally blocked 2D kernels (0: automatic)
TILES_2D = ((0, 0, 0), (32, 64, 1024), (32, 64, 512), (32, 32, 512), (32, 32, 256), (16, 32, 256), (16, 64, 256))


def heat256_initial(n: int = 256, g: int = 1) -> np.ndarray:
    """The 2D heat workload's initial field: U[0,1) from seed 0 on the n x n
    interior times a Gaussian bump of sigma 0.1 centred at (0.5, 0.5), with
    node-centred coordinates x_i = i/n (mesh/uniformGridMesh/functions.py:81-84);
    ghost cells 0.  Shape (n+2g, n+2g, 1, 1), float32."""
    rng = np.random.default_rng(0)
    x = np.arange(n) / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    u = np.zeros((n + 2 * g, n + 2 * g, 1, 1), dtype=np.float32)
    u[g:n + g, g:n + g, 0, 0] = (rng.random((n, n)) *
                                 np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / (2 * 0.1 ** 2))).astype(np.float32)
    return u


def run_heat3d(n: int = 512, steps: int = 12, depths=(1, 2, 3, 4)):
    """3D heat, n^3 interior + 1 ghost (order 2) or 2 (order 4), Dirichlet 0 on
    every face, alpha 1, dt = 0.15 dx^2, u0 = U[0,1) (seeded): the 3D rollout at
    each depth k (k = 1: surface fill and the TMA streaming heat step; k >= 2:
    boundary fill + Laplacian + Euler temporally blocked, k steps per HBM pass),
    CUDA events around `steps` steps of one call (best of 3; each call copies the
    input once), and a bitwise check of the fastest depth against the generic
    one-step kernel.  Fields (0.54 GB each) are larger than L2."""
    import torch
    import pde_module_b200 as P
    from pde_module_b200 import _lib
    peak, peak_kind = peaks()
    out = {"workload": f"3D heat {n}^3, Dirichlet 0 on all faces, alpha 1, dt 0.15 dx^2 (the heat loop of "
                       "examples/2D_Heat_Equation.py on a 3D grid), exact arithmetic"}
    for order in (2, 4):
        g = order // 2
        s = n + 2 * g
        dx = 1.0 / (n - 1)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(11)
        u = torch.rand((s, s, s, 1), device="cuda", generator=gen)
        bc = P.GridBoundary(u, dx, g)
        bc.dirichlet_BC("ALL", 0.0)
        dt = 0.15 * dx * dx
        res = {}
        for k in depths:
            roll = P.HeatRollout(bc, dx, 1.0, dt, order=order, steps_per_pass=k)
            roll(u, steps)
            torch.cuda.synchronize()
            best = None
            for _ in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                roll(u, steps)
                e1.record()
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1) / steps
                best = t if best is None else min(best, t)
            cps = n ** 3 / (best / 1000.0)
            gbs = cps * 8.0 / k / 1e9
            res[k] = {"ms_per_step": round(best, 4), "cell_updates_per_s": cps,
                      "alg_bytes_per_cell_step": round(8.0 / k, 3), "alg_gbs": round(gbs, 1),
                      "frac_of_hbm": round(gbs / peak, 4)}
        kb = min(res, key=lambda q: res[q]["ms_per_step"])
        roll = P.HeatRollout(bc, dx, 1.0, dt, order=order, steps_per_pass=kb)
        fused = roll(u, 4).clone()
        prev = _lib.lib().pde_set_dispatch(1)
        single = P.HeatRollout(bc, dx, 1.0, dt, order=order)(u, 4).clone()
        _lib.lib().pde_set_dispatch(prev)
        torch.cuda.synchronize()
        out[f"order{order}"] = {"best_k": kb, "ms_per_step": res[kb]["ms_per_step"],
                                "cell_updates_per_s": res[kb]["cell_updates_per_s"],
                                "bitwise_equal_to_single_step_kernel": bool(torch.equal(fused, single)),
                                "by_k": {f"k{k}": v for k, v in res.items()}}
        del u, fused, single
    out["note"] = (f"alg_gbs = 8 B per cell and pass / (ms per step x k), of the {peak_kind} HBM peak {peak} GB/s; "
                   "k = 1 on these grids is the one-step path (surface fill, then the TMA streaming heat step, "
                   "HBM-bound); k >= 2 the temporally blocked kernel (bound by one barrier per plane, not HBM)")
    return out


def run_heat3d_slabs(world: int, rank: int, n: int = 512, steps: int = 12) -> dict:
    """3D heat on a (n*world) x n x n interior cut into X slabs of n planes, one
    per rank (weak scaling), order 2 at the library's depth k, Dirichlet 0 on all
    faces: each block of k steps is one halo exchange (g + k + 1 planes to each
    neighbour, NCCL send/recv) and one fused pass.  CUDA events around `steps`
    steps after one untimed call, the max over ranks."""
    import torch
    import torch.distributed as dist
    import pde_module_b200 as P
    from pde_module_b200.distributed import SlabHeatRollout
    g, X = 1, n * world + 2
    dx = 1.0 / (n - 1)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11 + rank)
    bc = P.GridBoundary(torch.empty((4, n + 2, n + 2, 1), device="cuda"), dx, g)
    bc.dirichlet_BC("ALL", 0.0)
    roll = SlabHeatRollout(bc, dx, 1.0, 0.15 * dx * dx, X)
    roll.owned.copy_(torch.rand(roll.owned.shape, device="cuda", generator=gen))
    roll(steps)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    roll(steps)
    e1.record()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1) / steps], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    return {"workload": f"3D heat {n * world}x{n}x{n} in {world} X slabs, Dirichlet 0, order 2, exact",
            "k": roll.k, "halo_planes": roll.halo, "ms_per_step": round(ms, 4),
            "cell_updates_per_s": world * n ** 3 / (ms / 1000.0), "scaling": "weak",
            "exchange": "per block of k steps, inside the timed region"}


def leg_summary(kern, heat3d, heat, ldc, wave, batched, wc) -> dict:
    """The key figure of every leg, short (the line's last key)."""
    def g(d, *path):
        for p in path:
            if not isinstance(d, dict) or p not in d:
                return None
            d = d[p]
        return round(d, 4) if isinstance(d, float) else d
    out = {"sweep_frac": {k: v["frac"] for k, v in kern.items()}}
    if heat3d and "order2" not in heat3d:  # N > 1: the slab rollout
        out["heat3d_slabs"] = {"k": heat3d["k"], "ms_per_step": heat3d["ms_per_step"],
                               "gcups": round(heat3d["cell_updates_per_s"] / 1e9, 1)}
    elif heat3d:
        out["heat3d_512"] = {f"o{o}": {"k": g(heat3d, f"order{o}", "best_k"),
                                       "ms_per_step": g(heat3d, f"order{o}", "ms_per_step"),
                                       "gcups": round(heat3d[f"order{o}"]["cell_updates_per_s"] / 1e9, 1),
                                       "bitwise": g(heat3d, f"order{o}", "bitwise_equal_to_single_step_kernel")}
                             for o in (2, 4)}
    if heat:
        out["heat_256"] = {"gcups": round(heat["fused_cell_updates_per_s"] / 1e9, 1),
                           "x_chain": g(heat, "speedup_vs_chain"),
                           "fwd_adj_ratio": g(heat, "adjoint", "ratio_fwd_adj_over_fwd")}
    if wave:
        out["wave_512"] = {"fwd_ms": g(wave, "forward_ms"), "fwd_adj_ratio": g(wave, "ratio_fwd_adj_over_fwd")}
    if ldc:
        out["ldc_1024"] = {"gcups": round(ldc["cell_updates_per_s"] / 1e9, 2),
                           "jacobi_sweeps_per_s": round(ldc["jacobi_sweeps_per_s"])}
    if batched:
        out["batched_64"] = {"heat_x_per_grid_plain": g(batched, "heat", "speedup_vs_plain_chain"),
                             "heat_x_per_grid_fused": g(batched, "heat", "speedup_vs_per_grid_fused"),
                             "wave_x_per_grid_fused": g(batched, "wave", "speedup_vs_per_grid_fused")}
    if wc:
        out["wc_cavity"] = {"n201_ms": g(wc, "n201", "fused_ms_per_step")}
    return out


def run_heat(steps: int = 1000):
    """2D heat, 256^2 interior + 1 ghost, Dirichlet 0, alpha 1, dt = 0.2 dx^2, u0 =
    U[0,1) (seed 0) x Gaussian bump (sigma 0.1): the fused rollout (boundary fill +
    Laplacian + Euler, k steps per launch) against the module chain of
    examples/2D_Heat_Equation.py (4 launches per step), both replayed as CUDA graphs,
    and checked bitwise against each other."""
    import torch
    import pde_module_b200 as P
    n, g = 256, 1
    dx = 1.0 / n
    dt = 0.2 * dx * dx
    u0 = torch.from_numpy(heat256_initial(n, g)).cuda()
    bc = P.GridBoundary(u0, dx, g)
    bc.dirichlet_BC("ALL", 0.0)
    lap, euler = P.Laplacian(1, dx, g), P.ForwardEuler()

    def chain(u, k):
        for _ in range(k):
            u2 = bc(u)
            u = euler(u2, lap(u2, 1.0), dt)
        return u

    def graph_of(fn):
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            fn()  # warm-up / setup outside capture
            gph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(gph, stream=s):
                out = fn()
        torch.cuda.current_stream().wait_stream(s)
        return gph, out

    def timed(gph, reps=5):
        gph.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            gph.replay()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    res = {}
    g_chain, out_chain = graph_of(lambda: chain(u0, steps))
    res["chain_ms"] = timed(g_chain)
    best = None
    for k in (4, 8, 16, 32):
        roll = P.HeatRollout(bc, dx, 1.0, dt, steps_per_pass=k)
        g_roll, out_roll = graph_of(lambda: roll(u0, steps))
        ms = timed(g_roll)
        res[f"fused_k{k}_ms"] = ms
        if best is None or ms < best[0]:
            best = (ms, k, out_roll, g_roll)
    best[3].replay()
    g_chain.replay()
    torch.cuda.synchronize()
    cells = n * n * steps
    # differentiable form: alpha as a field, gradients w.r.t. alpha and u0 by the adjoint
    # with sqrt(N) checkpoints; loss = mean squared final field
    import pde_module_b200._lib as L
    adj = {}
    for tile, k in [(t, q) for t in TILES_2D for q in (4, 8, 16)]:
        L.check(L.lib().pde_set_launch_2d(*tile), "pde_set_launch_2d")
        solver = P.HeatSolver(bc, dx, dt, steps, steps_per_pass=k)
        a_f = torch.ones_like(u0)

        def fwd():
            with torch.no_grad():
                return solver.forward(a_f, u0)

        def fwd_adj():
            a = a_f.clone().requires_grad_(True)
            u = u0.clone().requires_grad_(True)
            loss = (P.heat_rollout(a, u, solver) ** 2).mean()
            loss.backward()
            return a.grad, u.grad

        def ev(fn, reps=3):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps

        f_ms, fa_ms = ev(fwd), ev(fwd_adj)
        adj[(tile, k)] = (f_ms, fa_ms)
    kb = min(adj, key=lambda q: adj[q][1])
    L.check(L.lib().pde_set_launch_2d(*kb[0]), "pde_set_launch_2d")
    same_fwd = bool(torch.equal(P.HeatSolver(bc, dx, dt, steps, steps_per_pass=kb[1]).forward(torch.ones_like(u0),
                                                                                             u0), out_chain))
    L.check(L.lib().pde_set_launch_2d(0, 0, 0), "pde_set_launch_2d")
    return {"workload": "2D heat 256^2, Dirichlet 0, 1000 steps (examples/2D_Heat_Equation.py loop)",
            "fused_cell_updates_per_s": cells / (best[0] / 1000.0), "fused_k": best[1],
            "chain_cell_updates_per_s": cells / (res["chain_ms"] / 1000.0),
            "speedup_vs_chain": res["chain_ms"] / best[0],
            "bitwise_equal_to_chain": bool(torch.equal(best[2], out_chain)),
            "times_ms": {k: round(v, 4) for k, v in res.items()},
            "adjoint": {"steps_per_pass": kb[1], "launch": list(kb[0]) if kb[0] != (0, 0, 0) else "auto",
                        "forward_ms": adj[kb][0], "forward_adjoint_ms": adj[kb][1],
                        "ratio_fwd_adj_over_fwd": adj[kb][1] / adj[kb][0],
                        "forward_bitwise_equal_to_chain": same_fwd,
                        "by_launch_k": {f"{q[0][0]}x{q[0][1]}t{q[0][2]}_k{q[1]}": [round(v[0], 4), round(v[1], 4)]
                                      for q, v in adj.items()},
                        "note": "alpha as a field, grads w.r.t. alpha and u0, sqrt(N) checkpoints (every 32 "
                                "steps), forward and backward each replayed as one CUDA graph"},
            "note": "both as CUDA graph replays; the working set (0.27 MB) is L2-resident, launch-bound"}


def run_ldc(steps: int = 2000, n: int = 1024):
    """Lid-driven cavity, Re 100, n x n nodes, fractional step with 50 Jacobi sweeps
    per step, dt at CFL 0.2, from rest: the whole rollout captured as one CUDA graph."""
    import torch
    import pde_module_b200 as P
    s = P.FractionalStepLDC(n=n, Re=100.0, jacobi_iters=50)
    u0, p0 = s.u.clone(), s.p.clone()

    def timed_rollout(k, nsteps):
        s.jacobi_per_pass = k
        s.u.copy_(u0)
        s.p.copy_(p0)
        st = torch.cuda.Stream()
        st.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(st):
            s.step(1)
            gph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(gph, stream=st):
                s.step(nsteps)
        torch.cuda.current_stream().wait_stream(st)
        s.u.copy_(u0)
        s.p.copy_(p0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        gph.replay()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    import pde_module_b200._lib as L
    tune = {}
    for tile in ((0, 0, 0), (32, 64, 0), (64, 64, 0), (64, 64, 512), (64, 64, 1024), (48, 96, 0), (48, 96, 512),
                 (32, 128, 0), (32, 128, 512), (44, 88, 512), (64, 128, 1024), (88, 88, 1024)):
        L.check(L.lib().pde_set_launch_2d(*tile), "pde_set_launch_2d")
        for kk in (5, 8, 10, 16):
            tune[(tile, kk)] = timed_rollout(kk, 40)
    tile, k = min(tune, key=tune.get)
    L.check(L.lib().pde_set_launch_2d(*tile), "pde_set_launch_2d")
    ms = timed_rollout(k, steps)
    L.check(L.lib().pde_set_launch_2d(0, 0, 0), "pde_set_launch_2d")
    u = s.u.cpu().numpy()
    cells = n * n * steps
    return {"workload": f"lid-driven cavity Re 100, {n}^2 nodes, fractional step, 50 Jacobi sweeps/step, "
                        f"{steps} steps from rest, dt {s.dt:.3e}",
            "ms": ms, "cell_updates_per_s": cells / (ms / 1000.0),
            "jacobi_sweeps_per_s": 50 * steps / (ms / 1000.0), "jacobi_per_pass": k,
            "jacobi_launch": list(tile) if tile != (0, 0, 0) else "auto",
            "tune_ms_40_steps": {f"{t[0]}x{t[1]}t{t[2]}_k{kk}": round(v, 3) for (t, kk), v in tune.items()},
            "launches_per_step": 3 + -(-50 // k) + (1 if (-(-50 // k)) % 2 else 0),
            "max_abs_u": float(np.abs(u).max()),
            "note": "L2-resident (about 28 MB of fields); CUDA graph replay of the whole rollout"}


def run_wave(n: int = 512, steps: int = 2000):
    """Differentiable wave, n^2 nodes, leapfrog at CFL 0.5, Ricker source, MSE loss
    against a target from another speed field; gradients w.r.t. the speed field and the
    initial field through the adjoint with sqrt(N) checkpoints.  Times the forward
    rollout and forward + adjoint."""
    import torch
    from pde_module_b200.time_step import wave as W
    solver, c, u0, target, dt, mask = W.make_problem(n=n, nsteps=steps)

    def fwd_only():
        with torch.no_grad():
            return W.wave_rollout((dt * dt) * c * c, u0, solver)

    def fwd_adj():
        cc = c.clone().requires_grad_(True)
        uu = u0.clone().requires_grad_(True)
        uN = W.wave_rollout((dt * dt) * cc * cc, uu, solver)
        loss = (((uN - target) * mask) ** 2).sum() / mask.sum()
        loss.backward()
        return loss, cc.grad, uu.grad

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, out

    import pde_module_b200._lib as L
    best = None
    for tile in TILES_2D:
        L.check(L.lib().pde_set_launch_2d(*tile), "pde_set_launch_2d")
        for k in (4, 8, 12, 16):
            solver.steps_per_pass = k  # also drops the captured graphs
            ms, _ = timed(fwd_adj, 1)
            if best is None or ms < best[0]:
                best = (ms, k, tile)
    L.check(L.lib().pde_set_launch_2d(*best[2]), "pde_set_launch_2d")
    solver.steps_per_pass = best[1]
    f_ms, _ = timed(fwd_only)
    fa_ms, (loss, gc, gu) = timed(fwd_adj)
    # the same with every state kept (one segment: no recomputation; 2000 x 1 MB)
    every = solver.every
    solver.set_checkpoint_every(steps)
    fa_all_ms, (loss2, gc2, _) = timed(fwd_adj)
    solver.set_checkpoint_every(every)
    same = bool(torch.equal(gc, gc2))
    L.check(L.lib().pde_set_launch_2d(0, 0, 0), "pde_set_launch_2d")
    cells = n * n * steps
    check = wave_gradient_check(solver, c, u0, target, dt, mask, gc, gu)
    return {"workload": f"differentiable wave {n}^2, {steps} leapfrog steps, CFL 0.5, Ricker source, "
                        f"MSE vs target, grads w.r.t. speed and initial field, sqrt(N) checkpoints "
                        f"(every {solver.every} steps)",
            "forward_ms": f_ms, "forward_adjoint_ms": fa_ms, "ratio_fwd_adj_over_fwd": fa_ms / f_ms,
            "store_all_states": {"forward_adjoint_ms": fa_all_ms, "ratio_fwd_adj_over_fwd": fa_all_ms / f_ms,
                                 "grad_bitwise_equal_to_checkpointed": same},
            "forward_cell_updates_per_s": cells / (f_ms / 1000.0), "steps_per_pass": best[1],
            "launch": list(best[2]) if best[2] != (0, 0, 0) else "auto",
            "loss": float(loss.item()), "grad_c_norm": float(gc.norm().item()),
            "grad_u0_norm": float(gu.norm().item()), "gradient_check": check}


def wave_gradient_check(solver, c, u0, target, dt, mask, gc, gu, eps=1e-3):
    """The full-size gradients against float64 torch autograd of the same leapfrog
    model (weights unrounded, written here independently of the kernels) and a
    float64 central difference J(c + eps d) - J(c - eps d) along a seeded direction d."""
    import torch
    X, Y = solver.shape[0], solver.shape[1]
    dx = solver.dx
    w0, w1 = 1.0 / (dx * dx), -2.0 / (dx * dx)
    inside = mask[:, :, 0, 0].double()
    src = solver.src.double()
    sx, sy = divmod(solver.src_cell, Y)
    tgt = target[:, :, 0, 0].double()

    def J(c64, u064):
        K = (dt * dt) * c64 * c64
        u = u064 * inside
        um = u
        for k in range(solver.N):
            lap = torch.zeros_like(u)
            cc = u[1:-1, 1:-1]
            lap[1:-1, 1:-1] = (w0 * u[:-2, 1:-1] + w1 * cc + w0 * u[2:, 1:-1]) + (
                w0 * u[1:-1, :-2] + w1 * cc + w0 * u[1:-1, 2:])
            v = 2.0 * u - um + K * lap
            e = torch.zeros_like(v)
            e[sx, sy] = src[k]
            um, u = u, (v + e) * inside
        return (((u - tgt) * inside) ** 2).sum() / inside.sum()

    c64 = c[:, :, 0, 0].double().clone().requires_grad_(True)
    u64 = u0[:, :, 0, 0].double().clone().requires_grad_(True)
    loss64 = J(c64, u64)
    loss64.backward()
    g64, gu64 = c64.grad, u64.grad
    g32, gu32 = gc[:, :, 0, 0].double(), gu[:, :, 0, 0].double()
    d = torch.randn(X, Y, generator=torch.Generator(device=c.device).manual_seed(11), device=c.device,
                    dtype=torch.float64) * inside
    with torch.no_grad():
        fd = float((J(c64 + eps * d, u64) - J(c64 - eps * d, u64)) / (2 * eps))
    an64, an32 = float((g64 * d).sum()), float((g32 * d).sum())
    rel = lambda a, b: float((a - b).norm() / b.norm()) if float(b.norm()) > 0 else None
    return {"reference": "float64 torch autograd of the same model (GPU), and a float64 central difference",
            "loss_float64": float(loss64.detach()), "rel_err_grad_c": rel(g32, g64), "rel_err_grad_u0": rel(gu32, gu64),
            "fd_directional": fd, "adjoint_directional_float32": an32, "autograd_directional_float64": an64,
            "rel_err_fd_vs_float64_autograd": abs(fd - an64) / abs(fd), "rel_err_fd_vs_adjoint": abs(fd - an32) / abs(fd),
            "eps": eps}


def batched_problem(n_grids: int = 64, lo: int = 64, hi: int = 1024):
    """64 independent 2D grids: interior sides from rng(3).integers(64, 1025, (64, 2)),
    diffusivity exp(U[ln 1e-3, 0]) from rng(4), u0 = U[0,1) from rng(5 + i), one ghost
    layer, dx = 1 / max(side), dt = 0.2 dx^2 / alpha."""
    sides = np.random.default_rng(3).integers(lo, hi + 1, size=(n_grids, 2))
    alpha = np.exp(np.random.default_rng(4).uniform(np.log(1e-3), 0.0, size=n_grids))
    u0, dx, dt = [], [], []
    for i, (sx, sy) in enumerate(sides):
        u0.append(np.random.default_rng(5 + i).random((int(sx) + 2, int(sy) + 2)).astype(np.float32))
        h = 1.0 / int(max(sx, sy))
        dx.append(h)
        dt.append(0.2 * h * h / float(alpha[i]))
    return sides, alpha.tolist(), u0, dx, dt


def run_wc(sizes=(201, 1025), steps: int = 100, chain_steps: int = 10):
    """Weakly compressible cavity (examples/LDC/LDC_RK2.py): n x n nodes, RK2 steps
    as one fused launch each (pde_wc_rk2) against the same step composed of this
    package's modules (GridBoundary, Laplacian, Grad, Divergence, OuterProduct,
    scalarVectorMult, RungeKatta2, torch arithmetic for the map-wise lines), both
    replayed as CUDA graphs; checks the two agree bit for bit."""
    import torch
    import pde_module_b200 as P

    def graph_ms(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                fn()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {"workload": "weakly compressible lid-driven cavity (LDC_RK2.py: Re 100, M 0.1, CFL 0.8), RK2 steps"}
    for n in sizes:
        solver, m, rho = P.lid_driven_cavity_wc(n=n)
        dx, nu, c2 = 1.0 / (n - 1), 0.01, 100.0
        eps, dt = solver.params.eps, solver.dt
        u_bc = P.GridBoundary(m, dx, 1)
        u_bc.dirichlet_BC("ALL", 0.0)
        u_bc.dirichlet_BC("+Y", 1.0, 0)
        r_bc = P.GridBoundary(rho, dx, 1)
        r_bc.vonNeumann_BC("ALL", 0.0)
        lap_u, lap_d = P.Laplacian(2, dx, 1), P.Laplacian(2, dx, 1)
        div_m, div_t = P.Divergence(2, m.shape, dx, 1), P.Divergence((2, 2), m.shape, dx, 1)
        grad_p, outer, momentum = P.Grad(1, rho.shape, dx, 1), P.OuterProduct(2, 2), P.scalarVectorMult(2)

        def bc(t, m_, r_):
            r2 = r_bc(r_)
            return momentum(r2, u_bc(m_ / r_)), r2

        def f(t, m_, r_):
            u = m_ / r_
            u_diff = lap_u(u, nu)
            return (grad_p(c2 * (r_ - 1.0), -1.0) - div_t(outer(m_, u)) + u_diff + lap_d(u_diff, eps),
                    div_m(m_, -1.0))

        rk = P.RungeKatta2([2, 1], f=f, bc=bc)
        m0 = m + 0.01 * torch.rand_like(m)
        state = [m0.clone(), rho.clone()]

        def chain():
            a, b = state
            for _ in range(chain_steps):
                a, b = rk(0.0, dt, a, b)
            state[0], state[1] = a, b

        fused_ms = graph_ms(lambda: solver(m0, rho, steps)) / steps
        chain_ms = graph_ms(chain) / chain_steps
        a, b = rk(0.0, dt, m0, rho)
        fm, fr = solver(m0, rho, 1)
        cells = n * n  # the nodes (the operators' launch domain)
        out[f"n{n}"] = {"fused_ms_per_step": round(fused_ms, 5), "chain_ms_per_step": round(chain_ms, 5),
                        "speedup": round(chain_ms / fused_ms, 2),
                        "fused_cell_updates_per_s": cells / (fused_ms / 1000.0),
                        "bitwise_equal_to_chain": bool(torch.equal(a, fm) and torch.equal(b, fr))}
    return out


def run_batched(steps: int = 500, chain_steps: int = 50, tune: bool = True):
    """Batched heat and wave rollouts of 64 uneven grids in one persistent launch
    (replayed as a CUDA graph), against per-grid plain launches: the module chain
    GridBoundary -> Laplacian -> ForwardEuler of examples/2D_Heat_Equation.py per grid
    and step (captured as a CUDA graph over chain_steps steps; the time is linear in
    steps and is scaled to the rollout's), and per-grid fused rollouts."""
    import torch
    import pde_module_b200 as P
    from pde_module_b200 import tuning
    sides, alpha, u0, dx, dt = batched_problem()
    n = len(u0)
    interior = int(sum(int(a) * int(b) for a, b in sides))
    cells_arr = int(sum(u.size for u in u0))
    dev0 = [torch.from_numpy(u[:, :, None, None]).cuda() for u in u0]

    def graph_of(fn):
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            fn()
            gph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(gph, stream=s):
                fn()
        torch.cuda.current_stream().wait_stream(s)
        return gph

    def timed(gph, reps=3):
        gph.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            gph.replay()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {"workload": f"batched heat: {n} 2D grids, interior sides U{{64..1024}} (rng 3), alpha log-uniform "
                       f"[1e-3, 1] (rng 4), u0 U[0,1) (rng 5+i), Dirichlet 0, dt = 0.2 dx^2/alpha, {steps} steps",
           "grids": n, "interior_cells": interior, "array_cells": cells_arr}
    # --- batched heat -----------------------------------------------------------
    fields = [u.clone() for u in dev0]
    roll = P.BatchedHeatRollout(fields, dx, alpha, dt)
    if tune:
        t = tuning.tune_batched(roll, nsteps=100)
        out["autotune"] = {"best": list(t["best"]), "ms_100_steps": t["ms"]}
    for f, u in zip(fields, dev0):
        f.copy_(u)
    g_b = graph_of(lambda: roll(steps))
    b_ms = timed(g_b)
    # parity: a fresh rollout against per-grid fused rollouts (bitwise)
    for f, u in zip(fields, dev0):
        f.copy_(u)
    g_b.replay()
    torch.cuda.synchronize()
    err = P._lib.device_error()
    bcs = []
    for i in range(n):
        bc = P.GridBoundary(dev0[i], dx[i], 1)
        bc.dirichlet_BC("ALL", 0.0)
        bcs.append(bc)
    rolls = [P.HeatRollout(bcs[i], dx[i], alpha[i], dt[i], steps_per_pass=8) for i in range(n)]
    same = all(torch.equal(rolls[i](dev0[i], steps), fields[i]) for i in range(n))
    g_pg = graph_of(lambda: [rolls[i](dev0[i], steps) for i in range(n)])
    pg_ms = timed(g_pg)
    # per-grid module chain, chain_steps steps per replay
    laps = [P.Laplacian(1, dx[i], 1) for i in range(n)]
    eulers = [P.ForwardEuler() for _ in range(n)]

    def chain():
        for i in range(n):
            u = dev0[i]
            for _ in range(chain_steps):
                u2 = bcs[i](u)
                u = eulers[i](u2, laps[i](u2, alpha[i]), dt[i])

    g_c = graph_of(chain)
    c_ms = timed(g_c, reps=2) * (steps / chain_steps)
    del g_c
    upd = interior * steps
    out["heat"] = {"batched_ms": b_ms, "batched_cell_updates_per_s": upd / (b_ms / 1000.0),
                   "plain_chain_ms": c_ms, "plain_chain_cell_updates_per_s": upd / (c_ms / 1000.0),
                   "per_grid_fused_ms": pg_ms, "per_grid_fused_cell_updates_per_s": upd / (pg_ms / 1000.0),
                   "speedup_vs_plain_chain": c_ms / b_ms, "speedup_vs_per_grid_fused": pg_ms / b_ms,
                   "tile": [roll.plan.tile_x, roll.plan.tile_y], "steps_per_pass": roll.plan.steps_per_pass,
                   "persistent_blocks": roll.plan.blocks, "total_tiles": roll.plan.total_tiles,
                   "hbm_bytes_algorithmic": 8 * cells_arr * (-(-steps // roll.plan.steps_per_pass) +
                                                             (-(-steps // roll.plan.steps_per_pass)) % 2),
                   "bitwise_equal_to_per_grid": bool(same), "device_error": err,
                   "note": "plain chain = per-grid GridBoundary, Laplacian, ForwardEuler launches, as a CUDA "
                           f"graph of {chain_steps} steps x {n} grids scaled to {steps} steps"}
    del g_b, g_pg
    # --- batched wave: K = dt^2 c^2 = 0.125 dx^2 (CFL 0.5 in 2D), zero Dirichlet ring
    wf = []
    for u in u0:
        w = u.copy()
        w[:2, :] = 0.0; w[-2:, :] = 0.0; w[:, :2] = 0.0; w[:, -2:] = 0.0
        wf.append(torch.from_numpy(w[:, :, None, None]).cuda())
    Ks = [0.125 * h * h for h in dx]
    cur = [w.clone() for w in wf]
    prev = [w.clone() for w in wf]
    wroll = P.BatchedWaveRollout(cur, prev, dx, Ks)
    if tune:
        t = tuning.tune_batched(wroll, nsteps=100)
        out["wave_autotune"] = {"best": list(t["best"])}
    for a, b, w in zip(cur, prev, wf):
        a.copy_(w)
        b.copy_(w)
    g_w = graph_of(lambda: wroll(steps))
    w_ms = timed(g_w)
    for a, b, w in zip(cur, prev, wf):
        a.copy_(w)
        b.copy_(w)
    g_w.replay()
    from pde_module_b200.time_step.wave import WaveSolver
    # per-grid fused forward rollouts (pde_wave_forward, no states kept), one call per grid
    solvers = [WaveSolver(tuple(wf[i].shape[:3]), dx[i], steps, steps_per_pass=8, checkpoint_every=1)
               for i in range(n)]
    Kf = [torch.full_like(wf[i], Ks[i]) for i in range(n)]
    wout = [(torch.empty_like(w), torch.empty_like(w)) for w in wf]
    for i in range(n):
        solvers[i]._buffers(Kf[i])
    g_wp = graph_of(lambda: [solvers[i]._fwd(Kf[i], wf[i], wf[i], wout[i][0], wout[i][1], 0, steps)
                             for i in range(n)])
    wp_ms = timed(g_wp)
    wsame = all(torch.equal(wout[i][1], cur[i]) for i in range(n))
    out["wave"] = {"batched_ms": w_ms, "batched_cell_updates_per_s": upd / (w_ms / 1000.0),
                   "per_grid_fused_ms": wp_ms, "speedup_vs_per_grid_fused": wp_ms / w_ms,
                   "bitwise_equal_to_per_grid": bool(wsame),
                   "tile": [wroll.plan.tile_x, wroll.plan.tile_y], "steps_per_pass": wroll.plan.steps_per_pass}
    del g_w, g_wp
    return out


def run_e2e(fields, ops, world, args, exch=()):
    """The sweep end to end through the module API: every step copies both input
    fields of each order from pinned host memory, runs the six module calls and
    copies every output back.  Copies run on their own streams (host->device and
    device->host engines work at the same time), pipelined by order: order 4's
    inputs travel while order 2 computes and its outputs travel back; events keep
    each device buffer's reuse after its last reader.  Timed on the compute stream
    after it has waited for the last device->host copy."""
    import torch
    import torch.distributed as dist
    groups = []  # per order: (host inputs, device inputs, ops, (host output, module) pairs)
    for gi, order in enumerate((2, 4)):
        u, v, mods = fields[order]
        hin, din = [], []
        for t in (u, v):
            h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            h.copy_(t)
            hin.append(h)
            din.append(t)
        hout = [(torch.empty(m.output_array.shape, dtype=torch.float32, pin_memory=True), m)
                for m in mods if m.output_array is not None]
        groups.append((hin, din, ops[3 * gi:3 * gi + 3], hout))
    h2d = sum(h.numel() * 4 for g in groups for h in g[0])
    d2h = sum(h.numel() * 4 for g in groups for h, _ in g[3])
    K = max(1, min(args.steps, args.e2e_steps))
    comp = torch.cuda.current_stream()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in groups]
    ev_done = [torch.cuda.Event() for _ in groups]  # the group's ops have run: inputs free, outputs ready
    ev_out = [torch.cuda.Event() for _ in groups]   # the group's outputs are on the host: outputs free

    def e2e_step():
        for gi, (hin, din, gops, hout) in enumerate(groups):
            s_in.wait_event(ev_done[gi])  # the previous step's ops no longer read these inputs
            with torch.cuda.stream(s_in):
                for h, d in zip(hin, din):
                    d.copy_(h, non_blocking=True)
            ev_in[gi].record(s_in)
            comp.wait_event(ev_in[gi])
            comp.wait_event(ev_out[gi])  # the previous step's outputs have left
            if exch:  # N > 1: this order's halo planes from the neighbouring ranks
                exch[gi]()
            for _, fn, _ in gops:
                fn()
            ev_done[gi].record(comp)
            s_out.wait_event(ev_done[gi])
            with torch.cuda.stream(s_out):
                for h, m in hout:
                    h.copy_(m.output_array, non_blocking=True)
            ev_out[gi].record(s_out)

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(comp)
    for _ in range(K):
        e2e_step()
    comp.wait_stream(s_out)
    comp.wait_stream(s_in)
    t1.record(comp)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    if world > 1:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    val = world * N_INT ** 3 * len(ops) / (ms / K / 1000.0)
    return {"value": val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": K,
            "path": "pinned host fields -> H2D -> module calls (C ABI) -> D2H of every output; copies on their "
                    "own streams, pipelined by order"}


def run_profile_op(args):
    """One operator on the 512^3 sweep fields, for profilers: 2 untimed calls, then
    --iters timed calls.  --profile-op is lap2|lap4|grad2|grad4|div2|div4."""
    import torch
    import pde_module_b200 as P
    if args.profile_op in ("wave", "heatadj", "batched", "ldc", "heat"):
        return run_profile_2d(args)
    if args.profile_op in ("heat3d_o2", "heat3d_o4"):
        return run_profile_heat3d(args)
    op, order = args.profile_op[:-1], int(args.profile_op[-1])
    n = args.profile_n
    g = order // 2
    s = n + 2 * g
    dx = 1.0 / n
    fast = args.profile_fast
    if op == "div":
        u = torch.randn((s, s, s, 3), device="cuda")
        m = P.Divergence(3, u.shape, dx, g, order=order, fast=fast)
    elif op == "grad":
        u = torch.randn((s, s, s, 1), device="cuda")
        m = P.Grad(1, u.shape, dx, g, order=order, fast=fast)
    else:
        u = torch.randn((s, s, s, 1), device="cuda")
        m = P.Laplacian(1, dx, g, order=order, fast=fast)
    for _ in range(2):
        m(u, 1.0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.iters):
        m(u, 1.0)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.iters
    b = {"lap": 8, "grad": 16, "div": 16}[op]
    print(json.dumps({"profile_op": args.profile_op, "n": n, "ms": ms, "gbs": n ** 3 * b / ms / 1e6}))
    return 0


def run_profile_heat3d(args):
    """The fused 3D heat rollout for profilers: --profile-n^3 interior, order 2 or 4,
    Dirichlet 0 on all faces, --profile-k steps per pass (0: 4 for order 2, 2 for
    order 4), each of --iters calls one pass (k steps)."""
    import torch
    import pde_module_b200 as P
    order = int(args.profile_op[-1])
    n, g = args.profile_n, order // 2
    k = args.profile_k or (4 if order == 2 else 2)
    dx = 1.0 / (n - 1)
    u = torch.rand((n + 2 * g,) * 3 + (1,), device="cuda")
    bc = P.GridBoundary(u, dx, g)
    bc.dirichlet_BC("ALL", 0.0)
    roll = P.HeatRollout(bc, dx, 1.0, 0.15 * dx * dx, order=order, steps_per_pass=k)
    for _ in range(2):
        roll(u, k)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.iters):
        roll(u, k)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / (args.iters * k)
    print(json.dumps({"profile_op": args.profile_op, "n": n, "k": k, "ms_per_step": ms,
                      "cell_updates_per_s": n ** 3 / (ms / 1e3)}))
    return 0


def run_profile_2d(args):
    """The 2D time-stepping kernels for profilers, eager (no graphs), short runs:
    wave    - 512^2 wave problem, 96 steps, forward + adjoint (k = 8, automatic tile)
    heat    - 256^2 fused heat rollout (Dirichlet 0), 96 steps (k = 8, automatic launch shape)
    heatadj - 256^2 heat, alpha field, 96 steps, forward + adjoint (k = 4)
    batched - the 64-grid batched heat rollout, 16 steps (k = 4, 64 x 64 tiles)
    ldc     - the 1024^2 lid-driven cavity, 4 steps (50 Jacobi sweeps each)"""
    import torch
    import pde_module_b200 as P
    from pde_module_b200.time_step import wave as W
    t0 = time.time()
    for _ in range(args.iters):
        if args.profile_op == "wave":
            solver, c, u0, target, dt, mask = W.make_problem(n=512, nsteps=96, steps_per_pass=8)
            solver.graphs = False
            solver.set_checkpoint_every(None)
            K = (dt * dt) * c * c
            uN = solver.forward(K, u0)
            solver.backward(K, (uN - target) * mask)
        elif args.profile_op == "heat":
            n, g = 256, 1
            dx = 1.0 / n
            u0 = torch.rand((n + 2, n + 2, 1, 1), device="cuda")
            bc = P.GridBoundary(u0, dx, g)
            bc.dirichlet_BC("ALL", 0.0)
            P.HeatRollout(bc, dx, 1.0, 0.2 * dx * dx, steps_per_pass=8)(u0, 96)
        elif args.profile_op == "heatadj":
            n, g = 256, 1
            dx = 1.0 / n
            u0 = torch.rand((n + 2, n + 2, 1, 1), device="cuda")
            bc = P.GridBoundary(u0, dx, g)
            bc.dirichlet_BC("ALL", 0.0)
            solver = P.HeatSolver(bc, dx, 0.2 * dx * dx, 96, steps_per_pass=4, graphs=False)
            a = torch.ones_like(u0)
            uN = solver.forward(a, u0)
            solver.backward(a, uN)
        elif args.profile_op == "ldc":
            s = P.FractionalStepLDC(n=1024, Re=100.0, jacobi_iters=50)
            s.step(4)
        else:
            sides, alpha, u0, dx, dt = batched_problem()
            fields = [torch.from_numpy(u[:, :, None, None]).cuda() for u in u0]
            roll = P.BatchedHeatRollout(fields, dx, alpha, dt, tile=(64, 64), steps_per_pass=4)
            roll(16)
    torch.cuda.synchronize()
    print(json.dumps({"profile_op": args.profile_op, "iters": args.iters, "s": round(time.time() - t0, 3)}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-heat", action="store_true")
    ap.add_argument("--no-heat3d", action="store_true")
    ap.add_argument("--no-ldc", action="store_true")
    ap.add_argument("--no-wave", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-wc", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the library's default tile candidates")
    ap.add_argument("--profile-op", default=None, help="run one operator only (lap2, grad4, div2, ...)")
    ap.add_argument("--profile-n", type=int, default=N_INT)
    ap.add_argument("--profile-fast", action="store_true")
    ap.add_argument("--profile-k", type=int, default=0, help="heat3d_o2/o4: steps per pass")
    ap.add_argument("--iters", type=int, default=3)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_op:
        return run_profile_op(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
