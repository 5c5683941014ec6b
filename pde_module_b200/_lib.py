"""ctypes binding of ``libpde_b200.so`` (the C ABI of include/pde_b200.h).

There is no CPU fallback: every operator needs CUDA float32 tensors and the
compiled library.  A missing library raises at first use, naming the build
command.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_native", "libpde_b200.so")

PDE_OK = 0
PDE_ERR_ARG = -1
PDE_ERR_SHAPE = -2
PDE_ERR_GHOST = -3
PDE_ERR_ALIGN = -4
PDE_ERR_CUDA = -5
PDE_ERR_UNSUPPORTED = -6
PDE_ERR_TIMEOUT = -7
PDE_ERR_TOO_LARGE = -8

PDE_MODE_EXACT = 0
PDE_MODE_FAST = 1
PDE_DISPATCH_AUTO = 0
PDE_DISPATCH_GENERIC = 1
PDE_OP_LAPLACIAN = 0
PDE_OP_GRAD = 1
PDE_OP_DIVERGENCE = 2
PDE_BC_DIRICHLET = 1
PDE_BC_VON_NEUMANN = 2
PDE_BC_FUNC_CONSTANT = 0
PDE_BC_FUNC_RAMP = 1
PDE_FUSED_MAX_COMP = 4
PDE_MAX_GROUPS = 16
PDE_NOALLOC_MAX_FLOATS = 1 << 22
PDE_LDC_PREDICT = 0
PDE_LDC_DIVERGENCE = 1
PDE_LDC_JACOBI = 2
PDE_LDC_PROJECT = 3
PDE_BATCH_HEAT = 0
PDE_BATCH_WAVE = 1
FACE_BITS = {"-X": 1 << 0, "+X": 1 << 1, "-Y": 1 << 2, "+Y": 1 << 3, "-Z": 1 << 4, "+Z": 1 << 5}


class PdeGrid(C.Structure):
    _fields_ = [("shape", C.c_int64 * 3), ("ghost_cells", C.c_int32), ("order", C.c_int32), ("dx", C.c_double)]


class PdeBCGroup(C.Structure):
    _fields_ = [
        ("node_ids", C.c_void_p), ("count", C.c_int32), ("type", C.c_int32), ("comp_mask", C.c_uint32),
        ("func", C.c_int32), ("value", C.c_float), ("t_max", C.c_float), ("face_mask", C.c_int32),
    ]


class PdeBCGroupParam(C.Structure):
    _fields_ = [("type", C.c_int32), ("comp_mask", C.c_uint32), ("func", C.c_int32), ("value", C.c_float),
                ("t_max", C.c_float)]


class PdeBCRules(C.Structure):
    _fields_ = [
        ("ncomp", C.c_int32), ("ngroups", C.c_int32), ("dx32", C.c_float), ("has_ramp", C.c_int32),
        ("group", PdeBCGroupParam * PDE_MAX_GROUPS),
        ("node_group", C.c_int8 * 27),
        ("ghost_group", ((C.c_int8 * PDE_FUSED_MAX_COMP) * 3) * 27),
        ("pad", C.c_int8 * 1),
    ]


class PdeLDCParams(C.Structure):
    _fields_ = [("nu", C.c_float), ("dt", C.c_float), ("jacobi_iters", C.c_int32), ("jacobi_per_pass", C.c_int32)]


class PdeWCParams(C.Structure):
    _fields_ = [("nu", C.c_double), ("eps", C.c_double), ("c2", C.c_double), ("rho0", C.c_double),
                ("dt", C.c_double)]


class PdeBatchGrid(C.Structure):
    _fields_ = [("field", C.c_void_p), ("field_prev", C.c_void_p), ("scratch", C.c_void_p),
                ("shape", C.c_int64 * 2), ("dx", C.c_double), ("coef", C.c_float), ("dt", C.c_float)]


class PdeBatchPlan(C.Structure):
    _fields_ = [("table", C.c_void_p), ("kind", C.c_int32), ("ngrids", C.c_int32), ("total_tiles", C.c_int32),
                ("ghost_cells", C.c_int32), ("order", C.c_int32), ("tile_x", C.c_int32), ("tile_y", C.c_int32),
                ("steps_per_pass", C.c_int32), ("blocks", C.c_int32), ("smem_bytes", C.c_int32),
                ("rules", PdeBCRules)]


class PdeSlab(C.Structure):
    _fields_ = [("x_global", C.c_int64), ("x_offset", C.c_int64), ("own_lo", C.c_int64), ("own_hi", C.c_int64)]


class PdeError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {strerror(status)} (status {status})")


# name -> (restype, argtypes)
_SIGS = {
    "pde_version": (C.c_int, []),
    "pde_strerror": (C.c_char_p, [C.c_int]),
    "pde_device_error": (C.c_int, [C.c_void_p]),
    "pde_set_dispatch": (C.c_int, [C.c_int]),
    "pde_stream3d_select": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "pde_laplacian": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.c_float, C.c_void_p]),
    "pde_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.c_float, C.c_void_p]),
    "pde_divergence": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.c_float, C.c_void_p]),
    "pde_laplacian_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.c_float, C.c_int32,
                                   C.c_void_p]),
    "pde_grad_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.c_float, C.c_int32,
                              C.c_void_p]),
    "pde_divergence_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.c_float, C.c_int32,
                                    C.c_void_p]),
    "pde_euler": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_int64, C.c_void_p]),
    "pde_bc_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.POINTER(PdeBCGroup),
                               C.c_int32, C.c_void_p, C.c_void_p]),
    "pde_periodic_fill": (C.c_int, [C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.c_int32, C.c_void_p]),
    "pde_bc_compile": (C.c_int, [C.POINTER(PdeBCGroup), C.c_int32, C.POINTER(PdeGrid), C.c_int32,
                                 C.POINTER(PdeBCRules)]),
    "pde_heat_rollout": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32,
                                   C.POINTER(PdeBCRules), C.c_float, C.c_float, C.c_int32, C.c_int32,
                                   C.c_void_p]),
    "pde_ib_work_bytes": (C.c_int64, [C.POINTER(PdeGrid)]),
    "pde_ib_maps": (C.c_int, [C.c_void_p, C.POINTER(PdeGrid), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.POINTER(C.c_int64), C.c_void_p, C.c_int64, C.c_void_p]),
    "pde_ib_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_float, C.c_void_p]),
    "pde_outer": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_void_p]),
    "pde_scalar_mult": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p]),
    "pde_layer_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64, C.c_float,
                                  C.c_void_p, C.c_void_p]),
    "pde_wc_rk2": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(PdeGrid),
                             C.POINTER(PdeBCRules), C.POINTER(PdeBCRules), C.POINTER(PdeWCParams), C.c_int32,
                             C.c_void_p, C.c_void_p]),
    "pde_heat_rollout_at": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32,
                                      C.POINTER(PdeBCRules), C.c_float, C.c_float, C.c_int32, C.c_int32,
                                      C.c_double, C.c_double, C.c_void_p]),
    "pde_heat_rollout_from": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32,
                                        C.POINTER(PdeBCRules), C.c_float, C.c_float, C.c_int32, C.c_int32,
                                        C.c_double, C.c_double, C.c_int32, C.c_void_p]),
    "pde_heat_pass_depth": (C.c_int, [C.POINTER(PdeGrid), C.c_int32, C.c_int32]),
    "pde_ldc_rollout": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(PdeGrid), C.POINTER(PdeBCRules), C.POINTER(PdeBCRules),
                                  C.POINTER(PdeLDCParams), C.c_int32, C.c_void_p]),
    "pde_ldc_rollout_at": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.POINTER(PdeGrid), C.POINTER(PdeBCRules), C.POINTER(PdeBCRules),
                                     C.POINTER(PdeLDCParams), C.c_int32, C.c_double, C.c_double, C.c_void_p]),
    "pde_ldc_slab_step": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.POINTER(PdeGrid), C.POINTER(PdeSlab), C.POINTER(PdeBCRules),
                                    C.POINTER(PdeBCRules), C.POINTER(PdeLDCParams), C.c_int32, C.c_int32,
                                    C.c_void_p]),
    "pde_wave_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                   C.POINTER(PdeGrid), C.c_void_p]),
    "pde_wave_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.POINTER(PdeGrid), C.c_void_p]),
    "pde_wave_pair": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.POINTER(PdeGrid), C.c_void_p]),
    "pde_set_launch_2d": (C.c_int, [C.c_int32, C.c_int32, C.c_int32]),
    "pde_set_launch_3d": (C.c_int, [C.c_int32, C.c_int32, C.c_int32]),
    "pde_set_wait_limit_ns": (C.c_uint64, [C.c_uint64]),
    "pde_wait_probe": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "pde_heat_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(PdeGrid),
                                   C.POINTER(PdeBCRules), C.c_float, C.c_int32, C.c_int32, C.c_void_p,
                                   C.c_void_p]),
    "pde_heat_forward_at": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(PdeGrid),
                                      C.POINTER(PdeBCRules), C.c_float, C.c_int32, C.c_int32, C.c_void_p,
                                      C.c_double, C.c_double, C.c_int32, C.c_void_p]),
    "pde_heat_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.POINTER(PdeGrid), C.POINTER(PdeBCRules), C.c_float, C.c_int32, C.c_int32,
                                   C.c_void_p, C.c_void_p]),
    "pde_batch_work_bytes": (C.c_int, [C.POINTER(PdeBatchGrid), C.c_int32, C.c_int32, C.c_int32,
                                       C.POINTER(C.c_uint64)]),
    "pde_batch_plan": (C.c_int, [C.c_int32, C.POINTER(PdeBatchGrid), C.c_int32, C.c_int32, C.c_int32,
                                 C.POINTER(PdeBCRules), C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_uint64,
                                 C.POINTER(PdeBatchPlan), C.c_void_p]),
    "pde_batch_rollout": (C.c_int, [C.POINTER(PdeBatchPlan), C.c_int32, C.c_void_p]),
    "pde_batch_rollout_at": (C.c_int, [C.POINTER(PdeBatchPlan), C.c_int32, C.c_double, C.c_void_p]),
    "pde_heat_rollout_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PdeGrid), C.c_int32,
                                           C.POINTER(PdeBCRules), C.c_float, C.c_float, C.c_int32, C.c_int32,
                                           C.c_void_p]),
}

_lib = None
_lock = threading.Lock()


def lib() -> C.CDLL:
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(
                        f"{LIB_PATH} is missing: build it with `python -m pde_module_b200.build_native` "
                        "(pde_module_b200 has no CPU fallback)")
                h = C.CDLL(LIB_PATH)
                for name, (res, args) in _SIGS.items():
                    fn = getattr(h, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = h
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def strerror(status: int) -> str:
    try:
        return lib().pde_strerror(status).decode()
    except Exception:  # library not loadable: still report the code
        return f"status {status}"


def check(status: int, what: str) -> None:
    if status != PDE_OK:
        raise PdeError(status, what)


def make_grid(shape3, ghost_cells: int, order: int, dx: float) -> PdeGrid:
    g = PdeGrid()
    for i in range(3):
        g.shape[i] = int(shape3[i])
    g.ghost_cells = int(ghost_cells)
    g.order = int(order)
    g.dx = float(dx)
    return g


def stream_ptr(t: torch.Tensor | None = None) -> int:
    dev = t.device if t is not None else None
    return torch.cuda.current_stream(dev).cuda_stream


def dptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def require_cuda_f32(t: torch.Tensor, name: str) -> None:
    """The product path runs on CUDA float32 contiguous tensors only."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor (got {type(t).__name__})")
    if t.device.type != "cuda":
        raise RuntimeError(f"{name} must be a CUDA tensor: pde_module_b200 has no CPU path")
    if t.dtype != torch.float32:
        raise TypeError(f"{name} must be float32 (got {t.dtype})")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be C-contiguous")


def device_error(t: torch.Tensor | None = None) -> int:
    return lib().pde_device_error(C.c_void_p(stream_ptr(t)))
