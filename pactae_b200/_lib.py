"""ctypes binding of include/smp_b200.h.

The library is built in-tree (``pactae_b200/libsmp_b200.so``).  There is no
fallback: if the library is missing or does not load, importing this module
raises, so nothing silently runs a CPU path.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsmp_b200.so"

SMP_OK = 0
SMP_ERR_INVALID_ARG = 1
SMP_ERR_INVALID_INPUT = 2
SMP_ERR_OOM = 3
SMP_ERR_CUDA = 4
SMP_ERR_TIMEOUT = 5
SMP_ERR_BUSY = 6
SMP_ERR_NOT_READY = 7
SMP_ERR_UNSUPPORTED = 8
SMP_ERR_IO = 9

SMP_B200_MAX_N = 1048575
SMP_B200_STATIC_MAX_N = 1024
SMP_B200_BATCH_MAX_N = 16384

SMP_F_DEVICE_PTRS = 0x1
SMP_F_CHECK = 0x2
SMP_F_VALIDATE = 0x4
SMP_F_NO_PRECHECK = 0x8

SMP_GEN_UNIFORM = 0
SMP_GEN_CONGESTED = 1
SMP_GEN_CORRELATED = 2
SMP_GEN_PERFECT = 3
SMP_GEN_REF_CONGESTED = 4
SMP_GEN_GROUPED = 5
SMP_GEN_SOLO = 6

# Every symbol include/smp_b200.h declares.
ABI_SYMBOLS = (
    "smp_b200_create",
    "smp_b200_destroy",
    "smp_b200_strerror",
    "smp_b200_last_error",
    "smp_b200_version",
    "smp_b200_stage",
    "smp_b200_precheck",
    "smp_b200_init",
    "smp_b200_core",
    "smp_b200_post",
    "smp_b200_stats",
    "smp_b200_solve",
    "smp_b200_invert",
    "smp_b200_check",
    "smp_b200_generate",
    "smp_b200_solve_static",
    "smp_b200_batch_create",
    "smp_b200_batch_run",
    "smp_b200_batch_run_plain",
    "smp_b200_batch_destroy", "smp_b200_batch_config",
    "smp_b200_workload_read_n", "smp_b200_workload_read", "smp_b200_workload_write", "smp_b200_workload_filename",
    "smp_b200_solve_batch",
    "smp_b200_batch_instance",
    "smp_b200_server_create",
    "smp_b200_submit",
    "smp_b200_poll",
    "smp_b200_server_stats",
    "smp_b200_server_destroy",
)


class smp_cfg(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("prefix_k", ctypes.c_int32),
        ("tail_threshold", ctypes.c_int32),
        ("bulk_window", ctypes.c_int32),
        ("hbm_budget", ctypes.c_uint64),
        ("tail_window", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("rank_bytes", ctypes.c_int32),
        ("reserved32", ctypes.c_int32),
        ("reserved", ctypes.c_uint64 * 2),
    ]


class smp_stats(ctypes.Structure):
    _fields_ = [
        ("proposals", ctypes.c_int64),
        ("blocking_pairs", ctypes.c_int64),
        ("tail_proposals", ctypes.c_int64),
        ("n", ctypes.c_int32),
        ("perfect", ctypes.c_int32),
        ("tail_men", ctypes.c_int32),
        ("rank_bytes", ctypes.c_int32),
        ("kernel_launches", ctypes.c_int32),
        ("bulk_hops", ctypes.c_int32),
        ("tail_hops", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("stage_ms", ctypes.c_float),
        ("precheck_ms", ctypes.c_float),
        ("init_ms", ctypes.c_float),
        ("core_ms", ctypes.c_float),
        ("post_ms", ctypes.c_float),
        ("check_ms", ctypes.c_float),
        ("total_ms", ctypes.c_float),
        ("invert_ms", ctypes.c_float),
        ("bulk_ms", ctypes.c_float),
        ("tail_ms", ctypes.c_float),
        ("reserved", ctypes.c_float * 2),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if not name.startswith("reserved")}


class smp_instance(ctypes.Structure):
    _fields_ = [
        ("pref_m", ctypes.c_void_p),
        ("pref_w", ctypes.c_void_p),
        ("match", ctypes.c_void_p),
        ("n", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("proposals", ctypes.c_int64),
    ]


class smp_batch_cfg(ctypes.Structure):
    _fields_ = [
        ("block_threads", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32),
        ("window", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("rank_smem_kb", ctypes.c_int32),
        ("tune", ctypes.c_int32),
        ("threshold_n", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class smp_batch_stats(ctypes.Structure):
    _fields_ = [
        ("instances", ctypes.c_int32),
        ("failed", ctypes.c_int32),
        ("proposals", ctypes.c_int64),
        ("ms", ctypes.c_float),
        ("launches", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class smp_server_cfg(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("max_wave", ctypes.c_int32),
        ("route_n", ctypes.c_int32),
        ("waves", ctypes.c_int32),
        ("hbm_budget", ctypes.c_uint64),
        ("block_threads", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32),
        ("large_slots", ctypes.c_uint64),
        ("reserved", ctypes.c_uint64 * 2),
    ]


class smp_result(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("n", ctypes.c_int32),
        ("proposals", ctypes.c_int64),
        ("queue_ms", ctypes.c_double),
        ("latency_ms", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class smp_server_stats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64),
        ("completed", ctypes.c_int64),
        ("waves", ctypes.c_int64),
        ("large", ctypes.c_int64),
        ("admitted_bytes", ctypes.c_int64),
        ("peak_bytes", ctypes.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64

_SIGNATURES = {
    "smp_b200_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.POINTER(smp_cfg)]),
    "smp_b200_destroy": (None, [_P]),
    "smp_b200_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "smp_b200_last_error": (ctypes.c_char_p, [_P]),
    "smp_b200_version": (ctypes.c_char_p, []),
    "smp_b200_stage": (ctypes.c_int, [_P, _P, _P, _I32, _U32]),
    "smp_b200_precheck": (ctypes.c_int, [_P, ctypes.POINTER(_I32)]),
    "smp_b200_init": (ctypes.c_int, [_P]),
    "smp_b200_core": (ctypes.c_int, [_P]),
    "smp_b200_post": (ctypes.c_int, [_P, _P, _U32]),
    "smp_b200_stats": (ctypes.c_int, [_P, ctypes.POINTER(smp_stats)]),
    "smp_b200_solve": (ctypes.c_int, [_P, _P, _P, _I32, _P, _U32, ctypes.POINTER(smp_stats)]),
    "smp_b200_invert": (ctypes.c_int, [_P, _P, _I32, _P, _U32]),
    "smp_b200_check": (ctypes.c_int, [_P, _P, _P, _I32, _P, _U32, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int64)]),
    "smp_b200_generate": (ctypes.c_int, [_P, _I32, _I32, _U64, _U32, _I32, _P, _P, _U32]),
    "smp_b200_solve_static": (ctypes.c_int, [_P, _P, _I32, _P, ctypes.POINTER(ctypes.c_int64), _P]),
    "smp_b200_batch_create": (ctypes.c_int, [_P, ctypes.POINTER(smp_instance), _I32, ctypes.POINTER(smp_batch_cfg),
                                             ctypes.POINTER(_P)]),
    "smp_b200_batch_run": (ctypes.c_int, [_P, ctypes.POINTER(smp_instance), ctypes.POINTER(smp_batch_stats)]),
    "smp_b200_batch_run_plain": (ctypes.c_int, [_P, ctypes.POINTER(smp_instance), ctypes.POINTER(smp_batch_stats)]),
    "smp_b200_batch_destroy": (None, [_P]),
    "smp_b200_batch_config": (ctypes.c_int, [_P, ctypes.POINTER(smp_batch_cfg)]),
    "smp_b200_workload_read_n": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32)]),
    "smp_b200_workload_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, _P, _P]),
    "smp_b200_workload_write": (ctypes.c_int, [ctypes.c_char_p, _P, _P, ctypes.c_int32]),
    "smp_b200_workload_filename": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_char_p,
                                                  ctypes.c_size_t]),
    "smp_b200_solve_batch": (ctypes.c_int, [_P, ctypes.POINTER(smp_instance), _I32, ctypes.POINTER(smp_batch_cfg),
                                            ctypes.POINTER(smp_batch_stats)]),
    "smp_b200_batch_instance": (None, [_U64, _U32, _I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    "smp_b200_server_create": (ctypes.c_int, [ctypes.POINTER(smp_server_cfg), ctypes.POINTER(_P)]),
    "smp_b200_submit": (ctypes.c_int, [_P, _P, _P, _I32, _P, _U32, ctypes.POINTER(ctypes.c_int64)]),
    "smp_b200_poll": (ctypes.c_int, [_P, ctypes.c_int64, _I32, ctypes.POINTER(smp_result)]),
    "smp_b200_server_stats": (ctypes.c_int, [_P, ctypes.POINTER(smp_server_stats)]),
    "smp_b200_server_destroy": (None, [_P]),
}


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python -m pactae_b200.build` "
            "(there is no CPU fallback for the solver)")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()
