"""Python access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and
its --impl reference arm) may import this package.  It is the checker the
CUDA path is compared against, never the thing measured or shipped.

Two libraries:
  _build/liboracle.so  the C restatement in smp_oracle.c (generators,
                       Gs-Seq, Mw-Seq, checker); always built by `make`.
  _ref/libsmpref.so    the reference's own CPU engines compiled from their
                       sources by `make ref` (needs the reference tree at
                       build time; the built library is used afterwards).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libsmpref.so"

GEN_UNIFORM, GEN_CONGESTED, GEN_CORRELATED, GEN_PERFECT, GEN_REF_CONGESTED, GEN_GROUPED, GEN_SOLO = range(7)
REF_ENGINES = {0: "Gs-Seq-CPU", 1: "Mw-Seq-CPU", 2: "Gs-Par-Cpu", 3: "Mw-Par-Cpu"}

_P = ctypes.c_void_p
_lib = None
_ref = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)


def reference_dir() -> Path:
    """The reference tree the recipes compile from: SMP_REFERENCE_DIR if set,
    else the default of oracle/Makefile (its REF variable).  It exists only
    where the reference is mounted; nothing on the GPU path reads it."""
    env = os.environ.get("SMP_REFERENCE_DIR")
    if env:
        return Path(env)
    out = subprocess.run(["make", "-s", "-C", str(HERE), "print-ref"], check=True, capture_output=True, text=True)
    return Path(out.stdout.strip())


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            build()
        L = ctypes.CDLL(str(ORACLE_LIB))
        L.oracle_generate.argtypes = [ctypes.c_int, ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int32,
                                      _P, _P]
        L.oracle_generate_side.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int32, ctypes.c_uint64,
                                           ctypes.c_uint32, ctypes.c_int32, _P]
        L.oracle_gs_seq.argtypes = [_P, _P, ctypes.c_int32, _P, ctypes.POINTER(ctypes.c_int64)]
        L.oracle_mw_seq.argtypes = [_P, _P, ctypes.c_int32, _P, ctypes.POINTER(ctypes.c_int64)]
        L.oracle_check.argtypes = [_P, _P, ctypes.c_int32, _P, ctypes.POINTER(ctypes.c_int64)]
        L.oracle_check.restype = ctypes.c_int64
        L.oracle_invert.argtypes = [_P, ctypes.c_int32, _P]
        L.oracle_is_perfect.argtypes = [_P, ctypes.c_int32]
        L.oracle_batch_instance.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
        L.oracle_philox4x32_10.argtypes = [_P, _P, _P]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def generate(kind: int, n: int, seed: int, salt: int = 0, param: int = 0) -> tuple[np.ndarray, np.ndarray]:
    pm = np.empty((n, n), dtype=np.int32)
    pw = np.empty((n, n), dtype=np.int32)
    if lib().oracle_generate(kind, n, seed, salt, param, _p(pm), _p(pw)) != 0:
        raise ValueError("oracle_generate rejected its arguments")
    return pm, pw


def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.empty(4, dtype=np.uint32)
    lib().oracle_philox4x32_10(_p(c), _p(k), _p(out))
    return out


def gs_seq(pm, pw) -> tuple[np.ndarray, int]:
    pm, pw = _i32(pm), _i32(pw)
    n = pm.shape[0]
    match = np.empty(n, dtype=np.int32)
    props = ctypes.c_int64()
    if lib().oracle_gs_seq(_p(pm), _p(pw), n, _p(match), ctypes.byref(props)) != 0:
        raise ValueError("oracle_gs_seq: invalid input")
    return match, props.value


def mw_seq(pm, pw) -> tuple[np.ndarray, int]:
    pm, pw = _i32(pm), _i32(pw)
    n = pm.shape[0]
    match = np.empty(n, dtype=np.int32)
    props = ctypes.c_int64()
    if lib().oracle_mw_seq(_p(pm), _p(pw), n, _p(match), ctypes.byref(props)) != 0:
        raise ValueError("oracle_mw_seq: invalid input")
    return match, props.value


def check(pm, pw, match) -> tuple[int, int]:
    """(blocking pairs, proposals); blocking = -1 if match is not a perfect
    matching."""
    pm, pw, match = _i32(pm), _i32(pw), _i32(match)
    props = ctypes.c_int64()
    bp = lib().oracle_check(_p(pm), _p(pw), pm.shape[0], _p(match), ctypes.byref(props))
    return int(bp), props.value


def invert(pw) -> np.ndarray:
    pw = _i32(pw)
    n = pw.shape[0]
    rank = np.empty((n, n), dtype=np.int32)
    if lib().oracle_invert(_p(pw), n, _p(rank)) != 0:
        raise ValueError("oracle_invert: a row is not a permutation")
    return rank


def is_perfect(pm) -> bool:
    pm = _i32(pm)
    return bool(lib().oracle_is_perfect(_p(pm), pm.shape[0]))


def batch_instance(seed: int, b: int, n_lo: int, n_hi: int) -> tuple[int, int]:
    n = ctypes.c_int32()
    kind = ctypes.c_int32()
    lib().oracle_batch_instance(seed, b, n_lo, n_hi, ctypes.byref(n), ctypes.byref(kind))
    return n.value, kind.value


# --------------------------------------------------------------------------
# The reference's own CPU engines (oracle/_ref/libsmpref.so).
# --------------------------------------------------------------------------
def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} is not built (make -C oracle ref)")
        R = ctypes.CDLL(str(REF_LIB))
        R.ref_solve.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int32, _P, _P]
        R.ref_threads.argtypes = []
        R.ref_engine_safe.argtypes = [ctypes.c_int, ctypes.c_int32]
        R.ref_obj_create.argtypes = [_P, _P, ctypes.c_int32]
        R.ref_obj_create.restype = ctypes.c_void_p
        R.ref_obj_destroy.argtypes = [ctypes.c_void_p]
        R.ref_obj_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int32, _P, _P]
        _ref = R
    return _ref


def ref_workload_save(filename: str, pm: np.ndarray, pw: np.ndarray) -> None:
    """The reference's SaveSmpWorkload: writes data/workloads/<filename>
    under the current directory."""
    pm = np.ascontiguousarray(pm, np.int32)
    pw = np.ascontiguousarray(pw, np.int32)
    R = ref()
    R.ref_workload_save.argtypes = [ctypes.c_char_p, _P, _P, ctypes.c_int32]
    assert R.ref_workload_save(filename.encode(), pm.ctypes.data, pw.ctypes.data, pm.shape[0]) == 0


def ref_workload_load(filename: str, n: int) -> tuple[np.ndarray, np.ndarray]:
    """The reference's LoadSmpWorkload on data/workloads/<filename>."""
    pm = np.empty((n, n), np.int32)
    pw = np.empty((n, n), np.int32)
    R = ref()
    R.ref_workload_load.argtypes = [ctypes.c_char_p, ctypes.c_int32, _P, _P]
    assert R.ref_workload_load(filename.encode(), n, pm.ctypes.data, pw.ctypes.data) == 0
    return pm, pw


def ref_workload_filename(workload_type: int, n: int, group_size: int) -> str:
    """The reference's GetWorkloadFilename (WorkloadType: PERFECT 0, RANDOM 1,
    CONGESTED 2, SOLO 3)."""
    buf = ctypes.create_string_buffer(256)
    R = ref()
    R.ref_workload_filename.argtypes = [ctypes.c_int, ctypes.c_int32, ctypes.c_int32, ctypes.c_char_p, ctypes.c_int32]
    assert R.ref_workload_filename(workload_type, n, group_size, buf, len(buf)) == 0
    return buf.value.decode()


def ref_threads() -> int:
    return int(ref().ref_threads())


def ref_engine_safe(engine: int, n: int) -> bool:
    return bool(ref().ref_engine_safe(engine, n))


def ref_solve(engine: int, pm, pw) -> tuple[np.ndarray, tuple[float, float, float]]:
    """Run a reference engine; returns (match, (precheck, init, core) ms)."""
    pm, pw = _i32(pm), _i32(pw)
    n = pm.shape[0]
    match = np.empty(n, dtype=np.int32)
    ms = (ctypes.c_double * 3)()
    rc = ref().ref_solve(engine, _p(pm), _p(pw), n, _p(match), ms)
    if rc == -2:
        raise ValueError(f"{REF_ENGINES[engine]} writes out of range at n={n} with {ref_threads()} threads")
    if rc != 0:
        raise RuntimeError(f"ref_solve failed ({rc})")
    return match, (ms[0], ms[1], ms[2])


class RefProblem:
    """The reference's SmpObj built once, solved repeatedly by reference
    engines (each solve constructs the engine, as SmpEngineExecutor does)."""

    def __init__(self, pm, pw):
        pm, pw = _i32(pm), _i32(pw)
        self.n = pm.shape[0]
        self._obj = ref().ref_obj_create(_p(pm), _p(pw), self.n)
        if not self._obj:
            raise RuntimeError("ref_obj_create failed")

    def solve(self, engine: int) -> tuple[np.ndarray, tuple[float, float, float]]:
        match = np.empty(self.n, dtype=np.int32)
        ms = (ctypes.c_double * 3)()
        rc = ref().ref_obj_solve(self._obj, engine, self.n, _p(match), ms)
        if rc == -2:
            raise ValueError(f"{REF_ENGINES[engine]} writes out of range at n={self.n}")
        if rc != 0:
            raise RuntimeError(f"ref_obj_solve failed ({rc})")
        return match, (ms[0], ms[1], ms[2])

    def close(self) -> None:
        if self._obj:
            ref().ref_obj_destroy(self._obj)
            self._obj = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
