"""ctypes binding of libnmxla.so, the sm_100a library behind numax_b200.

Every compute call goes through the C ABI declared in include/nmx_la.h.
There is no CPU fallback: if the shared library is missing or no sm_100
device is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnmxla.so")

NMX_F32 = 0
NMX_F64 = 1
NMX_ERR_CUDA = -1000
NMX_ERR_ALLOC = -1001
NMX_ERR_UNSUPPORTED = -1002
NMX_ERR_INTERNAL = -1003
NMX_ERR_IO = -1004
NMX_ERR_FORMAT = -1005

_lock = threading.Lock()
_lib = None

vp = C.c_void_p
i32 = C.c_int32
i64 = C.c_int64
ci = C.c_int

# name -> (restype, argtypes); mirrors include/nmx_la.h
SIGNATURES = {
    "nmx_create": (ci, [ci, C.POINTER(vp)]),
    "nmx_destroy": (ci, [vp]),
    "nmx_last_error_string": (C.c_char_p, []),
    "nmx_version": (ci, []),
    "nmx_synchronize": (ci, [vp, vp]),
    "nmx_memcpy_to_host": (ci, [vp, vp, vp, i64, vp]),
    "nmx_tune_set": (ci, [vp, C.c_char_p, i64]),
    "nmx_tune_get": (ci, [vp, C.c_char_p, C.POINTER(i64)]),
    "nmx_potrf_potrs_batched_plan": (ci, [vp, ci, i64, vp, ci, C.POINTER(vp)]),
    "nmx_batched_plan_destroy": (ci, [vp]),
    "nmx_batched_plan_sizes": (ci, [vp, C.POINTER(i64), C.POINTER(i64)]),
    "nmx_potrf_potrs_batched_f64": (ci, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "nmx_potrf_potrs_batched_f32": (ci, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "nmx_batched_plan_autotune": (ci, [vp, vp, vp, vp, vp, vp, vp, ci, vp]),
    "nmx_batched_plan_schedule": (ci, [vp, vp, vp, vp, ci, vp]),
    "nmx_batched_plan_set_shape": (ci, [vp, vp, ci, ci]),
    "nmx_batched_partition": (ci, [i64, vp, ci, ci, vp, vp]),
    "nmx_potrf_potrs_batched_graph_f64": (ci, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "nmx_potrf_potrs_batched_graph_f32": (ci, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "nmx_syevj_batched_plan": (ci, [vp, i64, vp, C.POINTER(vp)]),
    "nmx_syevj_plan_destroy": (ci, [vp]),
    "nmx_syevj_plan_sizes": (ci, [vp, C.POINTER(i64), C.POINTER(i64)]),
    "nmx_syevj_batched_f32": (ci, [vp, vp, vp, vp, vp, vp, C.c_double, ci, ci, vp]),
    "nmx_syevj_plan_autotune": (ci, [vp, vp, vp, vp, vp, vp, C.c_double, ci, ci, ci, vp]),
    "nmx_syevj_plan_schedule": (ci, [vp, vp, vp, vp, vp, ci, vp]),
    "nmx_syevj_batched_graph_f32": (ci, [vp, vp, vp, vp, vp, vp, C.c_double, ci, ci, vp]),
    "nmx_potrf_potrs_batched_noalloc_f64": (ci, [vp, i64, vp, ci, vp, vp, vp, vp, vp, vp]),
    "nmx_syevd_f64": (ci, [vp, i64, vp, i64, vp, vp, i64, vp, vp]),
    "nmx_syevd_f32": (ci, [vp, i64, vp, i64, vp, vp, i64, vp, vp]),
    "nmx_npy_header": (ci, [C.c_char_p, C.POINTER(ci), C.POINTER(ci), vp, ci, C.POINTER(i64)]),
    "nmx_npy_load": (ci, [vp, C.c_char_p, ci, ci, vp, vp, i64, vp]),
    "nmx_npy_save": (ci, [vp, C.c_char_p, ci, ci, vp, vp, vp]),
    "nmx_getrf_f64": (ci, [vp, i64, vp, i64, vp, vp, vp]),
    "nmx_getrf_f32": (ci, [vp, i64, vp, i64, vp, vp, vp]),
    "nmx_getrs_f64": (ci, [vp, i64, i64, vp, i64, vp, vp, i64, vp]),
    "nmx_getrs_f32": (ci, [vp, i64, i64, vp, i64, vp, vp, i64, vp]),
    "nmx_potrf_f64": (ci, [vp, i64, vp, i64, vp, vp]),
    "nmx_potrf_f32": (ci, [vp, i64, vp, i64, vp, vp]),
    "nmx_potrs_f64": (ci, [vp, i64, i64, vp, i64, vp, i64, vp]),
    "nmx_potrs_f32": (ci, [vp, i64, i64, vp, i64, vp, i64, vp]),
    "nmx_geqrf_f32": (ci, [vp, i64, i64, vp, i64, vp, vp]),
    "nmx_geqrf_f64": (ci, [vp, i64, i64, vp, i64, vp, vp]),
    "nmx_orgqr_f32": (ci, [vp, i64, i64, vp, i64, vp, vp, i64, vp]),
    "nmx_orgqr_f64": (ci, [vp, i64, i64, vp, i64, vp, vp, i64, vp]),
    "nmx_ormqr_f32": (ci, [vp, i64, i64, vp, i64, vp, vp, i64, i64, vp]),
    "nmx_ormqr_f64": (ci, [vp, i64, i64, vp, i64, vp, vp, i64, i64, vp]),
    "nmx_qr_solve_f32": (ci, [vp, i64, i64, vp, i64, vp, vp, vp, vp, vp]),
    "nmx_qr_solve_f64": (ci, [vp, i64, i64, vp, i64, vp, vp, vp, vp, vp]),
    "nmx_gesv_ir_f64": (ci, [vp, i64, vp, i64, vp, vp, ci, C.c_double, ci, vp, vp]),
    "nmx_gemm_sub_f32": (ci, [vp, i64, i64, i64, vp, i64, vp, i64, vp, i64, ci, vp]),
    "nmx_gesv_ir_reserve": (ci, [vp, i64, ci]),
    "nmx_lu_slogdet_f64": (ci, [vp, i64, vp, i64, vp, vp, vp]),
    "nmx_lu_slogdet_f32": (ci, [vp, i64, vp, i64, vp, vp, vp]),
    "nmx_lu_unpack_f64": (ci, [vp, i64, vp, i64, vp, vp, i64, vp, i64, vp, i64, vp]),
    "nmx_lu_unpack_f32": (ci, [vp, i64, vp, i64, vp, vp, i64, vp, i64, vp, i64, vp]),
    "nmx_inverse_f64": (ci, [vp, i64, vp, i64, vp, i64, vp, vp, vp]),
    "nmx_inverse_f32": (ci, [vp, i64, vp, i64, vp, i64, vp, vp, vp]),
    "nmx_posv_ir_f64": (ci, [vp, i64, vp, i64, vp, vp, ci, C.c_double, ci, vp, vp]),
    "nmx_posv_ir_reserve": (ci, [vp, i64, ci]),
    "nmx_gemm_f64": (ci, [vp, ci, ci, i64, i64, i64, C.c_double, vp, i64, vp, i64, C.c_double,
                          vp, i64, ci, vp]),
    "nmx_gemm_f32": (ci, [vp, ci, ci, i64, i64, i64, C.c_float, vp, i64, vp, i64, C.c_float,
                          vp, i64, ci, vp]),
}

NMX_IR_BF16 = 1
NMX_IR_FP16 = 2
NMX_IR_FP32 = 3
NMX_IR_BF16X3 = 4
NMX_IR_BF16X6 = 5
NMX_IR_FP64 = 6
NMX_IR_GMRES = 0x10
NMX_IR_AUTO = 0x20
NMX_IR_ESCALATE = 0x40
IR_PRECISION_NAMES = {NMX_IR_BF16: "bf16", NMX_IR_FP16: "fp16", NMX_IR_FP32: "fp32",
                      NMX_IR_BF16X3: "bf16x3", NMX_IR_BF16X6: "bf16x6", NMX_IR_FP64: "fp64"}


class IrStats(C.Structure):
    """nmx_ir_stats (include/nmx_la.h)."""
    _fields_ = [("iterations", C.c_int32), ("gmres_iterations", C.c_int32),
                ("converged", C.c_int32), ("info", C.c_int32), ("used_gmres", C.c_int32),
                ("final_precision", C.c_int32), ("backward_error", C.c_double),
                ("factor_ms", C.c_double), ("refine_ms", C.c_double)]


class NmxError(RuntimeError):
    """A failure reported by libnmxla (argument error or CUDA failure)."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed ({code}): {msg}")
        self.code = code


def load() -> C.CDLL:
    """Load libnmxla.so (building nothing: it must have been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m numax_b200.build` "
                    "(numax_b200 has no CPU fallback)")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def last_error() -> str:
    s = load().nmx_last_error_string()
    return s.decode() if s else ""


def check(fn: str, code: int) -> int:
    """Raise NmxError on a negative status; return info (>= 0) otherwise."""
    if code < 0:
        raise NmxError(fn, code, last_error())
    return code


def call(name: str, *args) -> int:
    return check(name, getattr(load(), name)(*args))


_contexts: dict[int, int] = {}


def context(device: int) -> int:
    """The process-wide nmx context of CUDA device `device` (created lazily)."""
    with _lock:
        h = _contexts.get(device)
    if h is None:
        out = vp()
        call("nmx_create", device, C.byref(out))
        with _lock:
            _contexts.setdefault(device, out.value)
            h = _contexts[device]
    return h
