"""ctypes binding of libqsv.so (declarations in include/qsv.h).

The library is built in-tree (``openqarp_b200/libqsv.so``).  There is no fallback: if it is
missing or fails to load, importing the engine raises ImportError naming the build step.
Status codes map onto the reference's exception classes (src/qarpx/python/bindings.cpp:272-290).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_size_t, c_uint8, c_uint32, c_uint64, c_void_p

import numpy as np

from .errors import CapabilityError, CudaError

_HERE = os.path.dirname(os.path.abspath(__file__))
# QSV_LIBRARY loads another build of the same C-ABI (e.g. one compiled with different tile
# parameters); by default the in-tree build next to this file
LIB_PATH = os.environ.get("QSV_LIBRARY") or os.path.join(_HERE, "libqsv.so")

QSV_OK, QSV_EINVAL, QSV_ERUNTIME, QSV_ECAPABILITY, QSV_ECUDA, QSV_ENOMEM = range(6)
QSV_C128, QSV_C64 = 0, 1


class PassTime(ctypes.Structure):
    _fields_ = [("label", ctypes.c_char * 24), ("launches", c_uint64), ("bytes", c_uint64), ("flops", c_double),
                ("ms", c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("launches", c_uint64), ("passes", c_uint64), ("hbm_bytes", c_uint64),
                ("fused_blocks", c_uint64), ("last_apply_ms", c_double)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libqsv.so not found at {LIB_PATH}: build it with "
            "`make -C openqarp_b200/csrc` (or __graft_entry__.build()).")
    lib = ctypes.CDLL(LIB_PATH)
    P8 = POINTER(c_uint8)
    PD = POINTER(c_double)
    PU64 = POINTER(c_uint64)
    PI32 = POINTER(c_int32)
    sig = {
        "qsv_last_error": (c_char_p, []),
        "qsv_abi_version": (c_int, []),
        "qsv_create": (c_int, [c_int, c_int, c_int, POINTER(c_void_p)]),
        "qsv_destroy": (c_int, [c_void_p]),
        "qsv_set_fusion": (c_int, [c_void_p, c_int, c_int]),
        "qsv_set_executor": (c_int, [c_void_p, c_int]),
        "qsv_set_tile_qubits": (c_int, [c_void_p, c_int]),
        "qsv_set_checkpoint_interval": (c_int, [c_void_p, c_int]),
        "qsv_reset": (c_int, [c_void_p]),
        "qsv_set_state": (c_int, [c_void_p, PD, c_uint64, c_int]),
        "qsv_get_state": (c_int, [c_void_p, PD, c_uint64]),
        "qsv_device_state": (c_int, [c_void_p, POINTER(c_void_p), POINTER(c_void_p)]),
        "qsv_copy_state": (c_int, [c_void_p, c_void_p]),
        "qsv_fuse_count": (c_int, [P8, c_size_t, c_int, c_int, c_int, PI32, PI32]),
        "qsv_fuse_plan": (c_int, [P8, c_size_t, c_int, c_int, c_int, c_void_p, c_size_t, POINTER(c_size_t)]),
        "qsv_tile_plan_count": (c_int, [P8, c_size_t, c_int, c_int, c_int, c_int, PI32, PI32]),
        "qsv_debug_bounds_selftest": (c_int, [c_int, PI32, PI32]),
        "qsv_jit_check": (c_int, [P8, c_size_t, c_int, c_int, c_int, c_int, c_int, c_int, PI32, PI32, PU64]),
        "qsv_apply": (c_int, [c_void_p, P8, c_size_t]),
        "qsv_apply_unfused": (c_int, [c_void_p, P8, c_size_t]),
        "qsv_transition": (c_int, [c_void_p, c_void_p, PU64, PU64, PD, c_size_t, PD]),
        "qsv_sample": (c_int, [c_void_p, PD, c_size_t, PU64]),
        "qsv_sample_seeded": (c_int, [c_void_p, c_uint32, c_size_t, PU64]),
        "qsv_uniforms": (c_int, [c_uint32, c_size_t, PD]),
        "qsv_sample_parities": (c_int, [c_void_p, c_uint32, c_size_t, PU64, c_size_t, PU64]),
        "qsv_exact_probs": (c_int, [c_void_p, c_double, PU64, PD, c_uint64, PU64]),
        "qsv_set_noise": (c_int, [c_void_p, c_int, PI32, PI32, PD]),
        "qsv_set_trajectory_batch": (c_int, [c_void_p, c_uint64]),
        "qsv_run_trajectories": (c_int, [c_void_p, P8, c_size_t, c_uint32, c_size_t, PU64, PU64, PI32]),
        "qsv_adjoint": (c_int, [c_void_p, P8, c_size_t, PI32, PI32, PD, c_int, PU64, PU64, PD,
                                c_size_t, PD, PD]),
        "qsv_adjoint_phi": (c_int, [c_void_p, P8, c_size_t, PI32, PI32, PD, c_int, PD, PD]),
        "qsv_norm2": (c_int, [c_void_p, PD]),
        "qsv_scale": (c_int, [c_void_p, c_double]),
        "qsv_inner": (c_int, [c_void_p, c_void_p, PD]),
        "qsv_synchronize": (c_int, [c_void_p]),
        "qsv_stats": (c_int, [c_void_p, POINTER(Stats)]),
        "qsv_device_info": (c_int, [c_int, c_char_p, c_size_t, POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
        "qsv_set_timing": (c_int, [c_void_p, c_int]),
        "qsv_pass_times": (c_int, [c_void_p, POINTER(PassTime), c_int, POINTER(c_int)]),
        "qsv_qaoa_create": (c_int, [c_int, c_int, PI32, PI32, PI32, PI32, POINTER(c_void_p)]),
        "qsv_qaoa_run": (c_int, [c_void_p, PD, c_int, PD, PD, PD]),
        "qsv_qaoa_destroy": (c_int, [c_void_p]),
        "qsv_cbatch_create": (c_int, [c_int, c_int, POINTER(c_void_p)]),
        "qsv_cbatch_add": (c_int, [c_void_p, c_int, P8, c_size_t, PI32, PI32, PD, c_int, PU64, PU64, PD, c_size_t,
                                   PI32]),
        "qsv_cbatch_set": (c_int, [c_void_p, c_int, P8, c_size_t]),
        "qsv_cbatch_run": (c_int, [c_void_p, PD, PD, PD]),
        "qsv_cbatch_destroy": (c_int, [c_void_p]),
        "qsv_transition_static": (c_int, [c_void_p, c_void_p, c_int, c_int, PU64, PU64, PD, c_size_t,
                                          c_void_p, PD]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()

DECLARED = (
    "qsv_last_error", "qsv_abi_version", "qsv_create", "qsv_destroy", "qsv_set_fusion",
    "qsv_set_executor", "qsv_set_tile_qubits", "qsv_set_checkpoint_interval", "qsv_reset", "qsv_set_state", "qsv_get_state", "qsv_device_state",
    "qsv_copy_state", "qsv_fuse_count", "qsv_fuse_plan", "qsv_tile_plan_count", "qsv_jit_check", "qsv_debug_bounds_selftest", "qsv_apply", "qsv_apply_unfused", "qsv_transition", "qsv_sample",
    "qsv_sample_seeded", "qsv_uniforms", "qsv_sample_parities", "qsv_exact_probs", "qsv_set_noise", "qsv_set_trajectory_batch", "qsv_run_trajectories", "qsv_adjoint", "qsv_adjoint_phi", "qsv_norm2",
    "qsv_scale", "qsv_inner", "qsv_synchronize", "qsv_stats", "qsv_device_info", "qsv_set_timing",
    "qsv_pass_times", "qsv_transition_static",
    "qsv_qaoa_create", "qsv_qaoa_run", "qsv_qaoa_destroy",
    "qsv_cbatch_create", "qsv_cbatch_add", "qsv_cbatch_set", "qsv_cbatch_run", "qsv_cbatch_destroy",
)
STATIC_MAX_TERMS = 4096


def check(rc: int) -> None:
    if rc == QSV_OK:
        return
    msg = (lib.qsv_last_error() or b"").decode("utf-8", "replace")
    if rc == QSV_EINVAL:
        raise ValueError(msg)
    if rc == QSV_ECAPABILITY:
        raise CapabilityError(msg)
    if rc == QSV_ECUDA:
        raise CudaError(msg)
    if rc == QSV_ENOMEM:
        raise MemoryError(msg)
    raise RuntimeError(msg)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


def u64ptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_uint64))


def i32ptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_int32))


def u8ptr(b: bytes):
    return ctypes.cast(ctypes.c_char_p(b), POINTER(c_uint8))
