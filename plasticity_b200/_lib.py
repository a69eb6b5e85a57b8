"""ctypes binding of ``libpfem_b200.so`` (the C ABI declared in include/pfem_b200.h).

The library is built in-tree by ``plasticity_b200/build.py``.  There is no CPU
fallback: if the shared library cannot be loaded this module raises, and every
computing entry point returns an error when no CUDA device is usable.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpfem_b200.so")

PFEM_OK = 0
PFEM_ERR_BAD_ARG = -1
PFEM_ERR_CUDA = -2
PFEM_ERR_INVERTED_ELEMENT = -3
PFEM_ERR_LINSOLVE = -4
PFEM_ERR_NOT_CONVERGED = -5
PFEM_ERR_STATE = -6

PFEM_HEX8_SMALL = 0
PFEM_HEX8_FINITE = 1
PFEM_HEX8_FINITE_FBAR = 2
PFEM_FP64 = 0
PFEM_MIXED = 1
PFEM_PRED_PREVIOUS = 0
PFEM_PRED_EXTRAPOLATE = 1
PFEM_PRED_LEARNED = 2
PFEM_KRYLOV_CG = 0
PFEM_KRYLOV_BICGSTAB = 1


class Material(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("sigy0", C.c_double),
                ("Hiso", C.c_double), ("Hkin", C.c_double), ("sigsat", C.c_double),
                ("delta", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("nsteps", C.c_int32), ("maxiter", C.c_int32), ("tol", C.c_double),
                ("precision", C.c_int32), ("krylov", C.c_int32), ("lin_rtol", C.c_double),
                ("eta_min", C.c_double), ("eta_max", C.c_double), ("ew_gamma", C.c_double),
                ("ew_alpha", C.c_double), ("krylov_itmax", C.c_int32), ("predictor", C.c_int32),
                ("amg_rebuild", C.c_int32), ("cheb_degree", C.c_int32), ("verbose", C.c_int32),
                ("line_search", C.c_int32), ("predictor_smooth", C.c_int32), ("max_cuts", C.c_int32),
                ("eta_first", C.c_double), ("amg_stale_ratio", C.c_double), ("ew_need", C.c_int32)]


class SolveResultC(C.Structure):
    _fields_ = [("converged", C.c_int32), ("steps_done", C.c_int32),
                ("newton_iters_total", C.c_int32), ("krylov_iters_total", C.c_int32),
                ("predictor_learned_used", C.c_int32), ("time_total_ms", C.c_double),
                ("time_assembly_ms", C.c_double), ("time_amg_setup_ms", C.c_double),
                ("time_krylov_ms", C.c_double), ("time_predictor_ms", C.c_double),
                ("load_step_cuts", C.c_int32)]


_d = C.POINTER(C.c_double)
_f = C.POINTER(C.c_float)
_i64 = C.POINTER(C.c_int64)
_i32 = C.POINTER(C.c_int32)
_u8 = C.POINTER(C.c_uint8)
_ctx = C.c_void_p

# name -> (restype, argtypes); every symbol include/pfem_b200.h declares
SIGNATURES = {
    "pfem_default_opts": (None, [C.POINTER(SolveOpts)]),
    "pfem_create": (C.c_int, [C.POINTER(_ctx), _d, C.c_int64, _i64, C.c_int64, C.c_int32,
                              C.POINTER(Material), _d, C.c_int32]),
    "pfem_destroy": (None, [_ctx]),
    "pfem_last_error": (C.c_char_p, [_ctx]),
    "pfem_inversion_info": (C.c_int, [_ctx, _i64, _i32, _d]),
    "pfem_pattern": (C.c_int, [_ctx, _i64, _i64, _i64]),
    "pfem_colors": (C.c_int, [_ctx, _i32, _i64]),
    "pfem_set_bcs": (C.c_int, [_ctx, _i64, _d, _u8, C.c_int64, _i64, _d, C.c_int64]),
    "pfem_reset": (C.c_int, [_ctx]),
    "pfem_assemble": (C.c_int, [_ctx, _d, C.c_int32, C.c_int32, _d, _d, _d, _u8]),
    "pfem_newton": (C.c_int, [_ctx, C.c_double, C.POINTER(SolveOpts), _i32, _d, _i32]),
    "pfem_solve": (C.c_int, [_ctx, C.POINTER(SolveOpts), C.POINTER(SolveResultC), _i32, _d, _i32]),
    "pfem_residual": (C.c_int, [_ctx, C.c_double, C.c_int32, _d, _d]),
    "pfem_predict": (C.c_int, [_ctx, C.c_double, C.POINTER(SolveOpts), _d, _d, _d, _i32]),
    "pfem_linear_solve": (C.c_int, [_ctx, _d, _d, C.c_double, C.c_int32, C.POINTER(SolveOpts), _i32]),
    "pfem_amg_apply": (C.c_int, [_ctx, _d, _d]),
    "pfem_amg_dense": (C.c_int, [_ctx, C.c_int32, C.c_int32, _d, _i64]),
    "pfem_get_state": (C.c_int, [_ctx, _d, _d, _d, _d, _d, _u8]),
    "pfem_set_state": (C.c_int, [_ctx, _d, _d, _d]),
    "pfem_get_back_stress": (C.c_int, [_ctx, _d]),
    "pfem_set_back_stress": (C.c_int, [_ctx, _d]),
    "pfem_set_displacement": (C.c_int, [_ctx, _d]),
    "pfem_gauss_stress": (C.c_int, [_ctx, _d]),
    "pfem_profile": (C.c_int, [_ctx, C.c_int32, C.c_int32, _d]),
    "pfem_timer": (C.c_int, [_ctx, C.c_int32, _d]),
    "pfem_kernel_launches": (C.c_int64, []),
    "pfem_tangent_index_bytes": (C.c_int, [_ctx, _i32]),
    "pfem_mlp_init": (C.c_int, [_ctx, C.c_uint64]),
    "pfem_mlp_params": (C.c_int, [_ctx, C.c_int32, _f, C.c_int64]),
    "pfem_mlp_forward": (C.c_int, [_ctx, _f, C.c_int64, _f]),
    "pfem_mlp_loss_grad": (C.c_int, [_ctx, _f, _f, C.c_int64, _f, _f]),
    "pfem_mlp_record": (C.c_int, [_ctx, C.c_int32, C.c_int64, _i64]),
    "pfem_mlp_train": (C.c_int, [_ctx, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _f]),
    "pfem_norm2_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python plasticity_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a, t=_d):
    return None if a is None else a.ctypes.data_as(t)


class PfemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(rc: int, ctx=None):
    if rc != PFEM_OK:
        msg = lib().pfem_last_error(ctx)
        raise PfemError(rc, msg.decode() if msg else "")
