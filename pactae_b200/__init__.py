"""pactae_b200 -- a B200 (sm_100a) Gale-Shapley stable-marriage solver.

Python mirror of the reference's engine API (victorliu-sq/PACTAE:
``bamboosmp::SmpObj``, include/smp/smp.h:8-52, and ``AbsSmpEngine``,
include/smp/smp_engine_abs.h:6-74) over the C ABI in include/smp_b200.h.
Every solve runs in libsmp_b200.so on the GPU; there is no CPU path.

    >>> import numpy as np, pactae_b200 as pb
    >>> with pb.Context() as ctx:
    ...     pm, pw = ctx.generate(pb.SMP_GEN_UNIFORM, 2000, seed=1, device=False)
    ...     match, stats = ctx.solve(pm, pw)
"""
from __future__ import annotations

import ctypes
import os
import time
from typing import Any

import numpy as np

from ._lib import (  # noqa: F401  (re-exported constants)
    ABI_SYMBOLS,
    LIB_PATH,
    SMP_B200_MAX_N,
    SMP_ERR_BUSY,
    SMP_ERR_CUDA,
    SMP_ERR_INVALID_ARG,
    SMP_ERR_INVALID_INPUT,
    SMP_ERR_IO,
    SMP_ERR_NOT_READY,
    SMP_ERR_OOM,
    SMP_ERR_TIMEOUT,
    SMP_ERR_UNSUPPORTED,
    SMP_F_CHECK,
    SMP_F_DEVICE_PTRS,
    SMP_F_NO_PRECHECK,
    SMP_F_VALIDATE,
    SMP_GEN_CONGESTED,
    SMP_GEN_CORRELATED,
    SMP_GEN_GROUPED,
    SMP_GEN_PERFECT,
    SMP_GEN_REF_CONGESTED,
    SMP_GEN_SOLO,
    SMP_GEN_UNIFORM,
    SMP_OK,
    lib,
    smp_batch_cfg,
    smp_batch_stats,
    smp_cfg,
    smp_instance,
    smp_result,
    smp_server_cfg,
    smp_server_stats,
    smp_stats,
)

__all__ = ["Batch", "Server", "Context", "SmpError", "SmpObj", "SmpEngineB200", "batch_instance", "version"]


class SmpError(RuntimeError):
    """A non-OK smp_status from the library."""

    def __init__(self, status: int, where: str = "", detail: str = ""):
        self.status = status
        msg = lib.smp_b200_strerror(status).decode()
        if detail:
            msg = f"{msg}: {detail}"
        super().__init__(f"{where}: {msg} (status {status})" if where else f"{msg} (status {status})")


def _check(status: int, where: str, handle: Any = None) -> None:
    if status != SMP_OK:
        detail = lib.smp_b200_last_error(handle).decode() if handle is not None else ""
        raise SmpError(status, where, detail)


def version() -> str:
    return lib.smp_b200_version().decode()


def _is_device_tensor(x: Any) -> bool:
    return hasattr(x, "is_cuda") and bool(getattr(x, "is_cuda"))


def _host_array(x: Any, n: int | None = None, name: str = "array") -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.int32)
    if n is not None and a.size != n * n:
        raise ValueError(f"{name} must hold n*n = {n * n} int32 values, got {a.size}")
    return a


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class Context:
    """One solver context (smp_ctx): a CUDA stream plus grow-only device
    buffers on one device.  Not thread-safe; use one per thread."""

    def __init__(self, device: int = 0, prefix_k: int = 0, tail_threshold: int = 0, hbm_budget: int = 0,
                 bulk_window: int = 0, tail_window: int = 0, mode: int = 0, rank_bytes: int = 0):
        cfg = smp_cfg()
        cfg.device = device
        cfg.prefix_k = prefix_k
        cfg.tail_threshold = tail_threshold
        cfg.hbm_budget = hbm_budget
        cfg.bulk_window = bulk_window
        cfg.tail_window = tail_window
        cfg.mode = mode
        cfg.rank_bytes = rank_bytes
        handle = ctypes.c_void_p()
        _check(lib.smp_b200_create(ctypes.byref(handle), ctypes.byref(cfg)), "smp_b200_create")
        self._h = handle
        self.device = device

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.smp_b200_destroy(self._h)
        self._h = None

    def __enter__(self) -> "Context":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._h is None:
            raise RuntimeError("context is closed")
        return self._h

    # -- whole solve ----------------------------------------------------------
    def solve(self, pref_m: Any, pref_w: Any, n: int | None = None, *, check: bool = False,
              precheck: bool = True, out: Any = None) -> tuple[Any, dict]:
        """Man-optimal stable matching of one instance.

        Host inputs (anything numpy can view as int32 n x n) give a numpy
        result; CUDA tensors (torch, on this context's device) give a CUDA
        tensor and no host copies.  Returns (match, stats)."""
        flags = (SMP_F_CHECK if check else 0) | (0 if precheck else SMP_F_NO_PRECHECK)
        st = smp_stats()
        if _is_device_tensor(pref_m):
            import torch

            n = n or int(pref_m.shape[0])
            for t, name in ((pref_m, "pref_m"), (pref_w, "pref_w")):
                if t.dtype != torch.int32 or not t.is_contiguous() or t.numel() != n * n:
                    raise ValueError(f"{name} must be a contiguous int32 CUDA tensor of n*n values")
            match = out if out is not None else torch.empty(n, dtype=torch.int32, device=pref_m.device)
            torch.cuda.synchronize(pref_m.device)
            rc = lib.smp_b200_solve(self.handle, ctypes.c_void_p(pref_m.data_ptr()),
                                    ctypes.c_void_p(pref_w.data_ptr()), n, ctypes.c_void_p(match.data_ptr()),
                                    flags | SMP_F_DEVICE_PTRS, ctypes.byref(st))
            _check(rc, "smp_b200_solve", self.handle)
            return match, st.as_dict()
        pm = _host_array(pref_m)
        n = n or int(round(np.sqrt(pm.size)))
        pm = _host_array(pm, n, "pref_m")
        pw = _host_array(pref_w, n, "pref_w")
        match = out if out is not None else np.empty(n, dtype=np.int32)
        rc = lib.smp_b200_solve(self.handle, _ptr(pm), _ptr(pw), n, _ptr(match), flags, ctypes.byref(st))
        _check(rc, "smp_b200_solve", self.handle)
        return match, st.as_dict()

    # -- phases (AbsSmpEngine::FindStableMatching, smp_engine_abs.h:10-36) ---
    def stage(self, pref_m: np.ndarray, pref_w: np.ndarray, n: int) -> None:
        self._staged = (_host_array(pref_m, n, "pref_m"), _host_array(pref_w, n, "pref_w"))
        _check(lib.smp_b200_stage(self.handle, _ptr(self._staged[0]), _ptr(self._staged[1]), n, 0),
               "smp_b200_stage")
        self._n = n

    def precheck(self) -> bool:
        v = ctypes.c_int32(0)
        _check(lib.smp_b200_precheck(self.handle, ctypes.byref(v)), "smp_b200_precheck")
        return bool(v.value)

    def init(self) -> None:
        _check(lib.smp_b200_init(self.handle), "smp_b200_init")

    def core(self) -> None:
        _check(lib.smp_b200_core(self.handle), "smp_b200_core")

    def post(self) -> np.ndarray:
        match = np.empty(self._n, dtype=np.int32)
        _check(lib.smp_b200_post(self.handle, _ptr(match), 0), "smp_b200_post")
        return match

    def stats(self) -> dict:
        st = smp_stats()
        _check(lib.smp_b200_stats(self.handle, ctypes.byref(st)), "smp_b200_stats")
        return st.as_dict()

    # -- other entry points ---------------------------------------------------
    def invert(self, pref_w: Any, n: int | None = None) -> Any:
        if _is_device_tensor(pref_w):
            import torch

            n = n or int(pref_w.shape[0])
            rank = torch.empty((n, n), dtype=torch.int32, device=pref_w.device)
            torch.cuda.synchronize(pref_w.device)
            _check(lib.smp_b200_invert(self.handle, ctypes.c_void_p(pref_w.data_ptr()), n,
                                       ctypes.c_void_p(rank.data_ptr()), SMP_F_DEVICE_PTRS), "smp_b200_invert")
            return rank
        pw = _host_array(pref_w)
        n = n or int(round(np.sqrt(pw.size)))
        pw = _host_array(pw, n, "pref_w")
        rank = np.empty((n, n), dtype=np.int32)
        _check(lib.smp_b200_invert(self.handle, _ptr(pw), n, _ptr(rank), 0), "smp_b200_invert")
        return rank

    def check(self, pref_m: Any, pref_w: Any, match: Any, n: int | None = None) -> tuple[int, int]:
        """(blocking pairs, proposals) of a matching, computed on the GPU."""
        bp = ctypes.c_int64(-1)
        props = ctypes.c_int64(0)
        if _is_device_tensor(pref_m):
            import torch

            n = n or int(pref_m.shape[0])
            torch.cuda.synchronize(pref_m.device)
            rc = lib.smp_b200_check(self.handle, ctypes.c_void_p(pref_m.data_ptr()),
                                    ctypes.c_void_p(pref_w.data_ptr()), n, ctypes.c_void_p(match.data_ptr()),
                                    SMP_F_DEVICE_PTRS, ctypes.byref(bp), ctypes.byref(props))
        else:
            pm = _host_array(pref_m)
            n = n or int(round(np.sqrt(pm.size)))
            pm = _host_array(pm, n, "pref_m")
            pw = _host_array(pref_w, n, "pref_w")
            mt = np.ascontiguousarray(match, dtype=np.int32)
            if mt.size != n:
                raise ValueError("match must hold n values")
            rc = lib.smp_b200_check(self.handle, _ptr(pm), _ptr(pw), n, _ptr(mt), 0, ctypes.byref(bp),
                                    ctypes.byref(props))
        _check(rc, "smp_b200_check")
        return int(bp.value), int(props.value)

    def generate_into(self, kind: int, n: int, seed: int, pref_m_ptr: int, pref_w_ptr: int, salt: int = 0,
                      param: int = 0) -> None:
        """Seeded instance written to caller-owned device memory (n*n int32 each)."""
        _check(lib.smp_b200_generate(self.handle, kind, n, seed, salt, param, ctypes.c_void_p(pref_m_ptr),
                                     ctypes.c_void_p(pref_w_ptr), SMP_F_DEVICE_PTRS), "smp_b200_generate")

    def generate(self, kind: int, n: int, seed: int, salt: int = 0, param: int = 0,
                 device: bool = True) -> tuple[Any, Any]:
        """Seeded instance (pref_m, pref_w): CUDA tensors if device, else numpy."""
        if device:
            import torch

            dev = torch.device("cuda", self.device)
            pm = torch.empty((n, n), dtype=torch.int32, device=dev)
            pw = torch.empty((n, n), dtype=torch.int32, device=dev)
            torch.cuda.synchronize(dev)
            _check(lib.smp_b200_generate(self.handle, kind, n, seed, salt, param, ctypes.c_void_p(pm.data_ptr()),
                                         ctypes.c_void_p(pw.data_ptr()), SMP_F_DEVICE_PTRS), "smp_b200_generate")
            return pm, pw
        pm = np.empty((n, n), dtype=np.int32)
        pw = np.empty((n, n), dtype=np.int32)
        _check(lib.smp_b200_generate(self.handle, kind, n, seed, salt, param, _ptr(pm), _ptr(pw), 0),
               "smp_b200_generate")
        return pm, pw


# -- the reference's workload text cache (generate_workloads_flat.h:283-376) ----
def read_workload(path) -> tuple[np.ndarray, np.ndarray]:
    """(pref_m, pref_w) of a workload file in the reference's format
    (LoadSmpWorkload): "n", then n rows of each list."""
    n = ctypes.c_int32()
    _check(lib.smp_b200_workload_read_n(os.fsencode(path), ctypes.byref(n)), "smp_b200_workload_read_n")
    pm = np.empty((n.value, n.value), dtype=np.int32)
    pw = np.empty((n.value, n.value), dtype=np.int32)
    _check(lib.smp_b200_workload_read(os.fsencode(path), n.value, _ptr(pm), _ptr(pw)), "smp_b200_workload_read")
    return pm, pw


def write_workload(path, pref_m: Any, pref_w: Any) -> None:
    """Writes both lists in the reference's format (SaveSmpWorkload)."""
    pm = _host_array(pref_m)
    pw = _host_array(pref_w)
    n = pm.shape[0] if pm.ndim == 2 else int(round(pm.size ** 0.5))
    _check(lib.smp_b200_workload_write(os.fsencode(path), _ptr(pm), _ptr(pw), n), "smp_b200_workload_write")


def workload_filename(kind: int, n: int, group_size: int = 5) -> str:
    """The file name the reference gives a generated workload (GetWorkloadFilename)."""
    buf = ctypes.create_string_buffer(128)
    _check(lib.smp_b200_workload_filename(kind, n, group_size, buf, len(buf)), "smp_b200_workload_filename")
    return buf.value.decode()


def batch_instance(seed: int, b: int, n_lo: int, n_hi: int) -> tuple[int, int]:
    """(n, kind) of instance b of a seeded mix (log-uniform n in [n_lo, n_hi],
    kind uniform / congested / correlated)."""
    n = ctypes.c_int32()
    kind = ctypes.c_int32()
    lib.smp_b200_batch_instance(seed, b, n_lo, n_hi, ctypes.byref(n), ctypes.byref(kind))
    return n.value, kind.value


class Batch:
    """A batch of independent instances solved by one persistent launch
    (smp_b200_batch_*).  instances: sequence of (pref_m, pref_w, match) CUDA
    tensors (int32, n*n / n*n / n) on the context's device; they must stay
    alive while the batch is used."""

    def __init__(self, ctx: Context, instances, block_threads: int = 0, ctas_per_sm: int = 0, window: int = 0,
                 use_graph: bool = True, rank_smem_kb: int = 0, tune: bool = True, threshold_n: int = 0):
        self.ctx = ctx
        self._keep = list(instances)
        count = len(self._keep)
        table = (smp_instance * count)()
        for i, (pm, pw, mt) in enumerate(self._keep):
            n = int(mt.numel())
            if pm.numel() != n * n or pw.numel() != n * n:
                raise ValueError(f"instance {i}: lists must hold n*n values")
            table[i].pref_m = pm.data_ptr()
            table[i].pref_w = pw.data_ptr()
            table[i].match = mt.data_ptr()
            table[i].n = n
        self._table = table
        cfg = smp_batch_cfg()
        cfg.block_threads = block_threads
        cfg.ctas_per_sm = ctas_per_sm
        cfg.window = window
        cfg.use_graph = 1 if use_graph else -1
        cfg.rank_smem_kb = rank_smem_kb
        cfg.tune = 0 if tune else -1
        cfg.threshold_n = threshold_n
        handle = ctypes.c_void_p()
        import torch

        torch.cuda.synchronize()
        _check(lib.smp_b200_batch_create(ctx.handle, table, count, ctypes.byref(cfg), ctypes.byref(handle)),
               "smp_b200_batch_create")
        self._h = handle
        self.count = count

    def _run(self, fn) -> tuple[list[int], list[int], dict]:
        results = (smp_instance * self.count)()
        st = smp_batch_stats()
        _check(fn(self._h, results, ctypes.byref(st)), "smp_b200_batch_run")
        return [r.status for r in results], [r.proposals for r in results], st.as_dict()

    def config(self) -> dict:
        """The shape the batch runs with (after tuning), with threshold_n:
        instances above it run the all-SM pipeline (-1: none)."""
        cfg = smp_batch_cfg()
        _check(lib.smp_b200_batch_config(self._h, ctypes.byref(cfg)), "smp_b200_batch_config")
        return cfg.as_dict()

    def run(self) -> tuple[list[int], list[int], dict]:
        """Batched persistent launch: (statuses, proposals, stats)."""
        return self._run(lib.smp_b200_batch_run)

    def run_plain(self) -> tuple[list[int], list[int], dict]:
        """The same kernel launched once per instance."""
        return self._run(lib.smp_b200_batch_run_plain)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.smp_b200_batch_destroy(self._h)
        self._h = None

    def __enter__(self) -> "Batch":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving loop (smp_b200_server_*): submit() returns a ticket at
    once; poll() waits for the outcome.  Requests with CUDA tensors run on
    them in place (they must stay alive until polled); numpy requests are
    copied in when admitted and the matching copied back."""

    def __init__(self, device: int = 0, max_wave: int = 0, route_n: int = 0, waves: int = 0, hbm_budget: int = 0,
                 block_threads: int = 0, ctas_per_sm: int = 0, large_slots: int = 0):
        cfg = smp_server_cfg()
        cfg.device = device
        cfg.max_wave = max_wave
        cfg.route_n = route_n
        cfg.waves = waves
        cfg.hbm_budget = hbm_budget
        cfg.block_threads = block_threads
        cfg.ctas_per_sm = ctas_per_sm
        cfg.large_slots = large_slots
        handle = ctypes.c_void_p()
        _check(lib.smp_b200_server_create(ctypes.byref(cfg), ctypes.byref(handle)), "smp_b200_server_create")
        self._h = handle
        self._live: dict[int, tuple] = {}

    def submit(self, pref_m: Any, pref_w: Any, match: Any) -> int:
        ticket = ctypes.c_int64()
        if _is_device_tensor(pref_m):
            n = int(match.numel())
            rc = lib.smp_b200_submit(self._h, ctypes.c_void_p(pref_m.data_ptr()), ctypes.c_void_p(pref_w.data_ptr()),
                                     n, ctypes.c_void_p(match.data_ptr()), SMP_F_DEVICE_PTRS, ctypes.byref(ticket))
            keep = (pref_m, pref_w, match)
        else:
            pm = _host_array(pref_m)
            pw = _host_array(pref_w)
            n = int(match.size)
            rc = lib.smp_b200_submit(self._h, _ptr(pm), _ptr(pw), n, _ptr(match), 0, ctypes.byref(ticket))
            keep = (pm, pw, match)
        _check(rc, "smp_b200_submit")
        self._live[ticket.value] = keep
        return ticket.value

    def poll(self, ticket: int, wait_ms: int = -1) -> dict | None:
        res = smp_result()
        rc = lib.smp_b200_poll(self._h, ticket, wait_ms, ctypes.byref(res))
        if rc == SMP_ERR_NOT_READY:
            return None
        _check(rc, "smp_b200_poll")
        self._live.pop(ticket, None)
        return res.as_dict()

    def stats(self) -> dict:
        st = smp_server_stats()
        _check(lib.smp_b200_server_stats(self._h, ctypes.byref(st)), "smp_b200_server_stats")
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.smp_b200_server_destroy(self._h)
        self._h = None
        self._live.clear()

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


class SmpObj:
    """Mirror of bamboosmp::SmpObj (include/smp/smp.h:8-52): the two flat
    row-major preference lists of one instance."""

    def __init__(self, flat_m: Any, flat_w: Any):
        self.flatten_pref_lists_m = np.ascontiguousarray(flat_m, dtype=np.int32).reshape(-1)
        self.flatten_pref_lists_w = np.ascontiguousarray(flat_w, dtype=np.int32).reshape(-1)

    @staticmethod
    def CreateFromFlatLists(flat_m: Any, flat_w: Any, n: int) -> "SmpObj":  # noqa: N802 (reference name)
        obj = SmpObj(flat_m, flat_w)
        if obj.flatten_pref_lists_m.size != n * n or obj.flatten_pref_lists_w.size != n * n:
            raise ValueError("flat lists must hold n*n entries")
        return obj


class SmpEngineB200:
    """Mirror of an AbsSmpEngine subclass (include/smp/smp_engine_abs.h:6-74)
    backed by the GPU: FindStableMatching() runs the precheck, init and core
    phases (each timed with a wall clock, as the reference does) and PostProc,
    and returns the matching as a list with match[m] = w."""

    def __init__(self, smp: SmpObj, n: int, ctx: Context | None = None):
        self.smp = smp
        self.n = int(n)
        self._own = ctx is None
        self.ctx = ctx or Context()
        self.precheck_time_ = 0.0
        self.init_time_ = 0.0
        self.core_time_ = 0.0
        # The reference engines copy the lists to the device in the
        # constructor, outside the timed phases (smp_engine_bamboo.cu:28-29).
        self.ctx.stage(smp.flatten_pref_lists_m, smp.flatten_pref_lists_w, self.n)

    def GetEngineName(self) -> str:  # noqa: N802
        return "B200-GS"

    def FindStableMatching(self) -> list[int]:  # noqa: N802
        t0 = time.perf_counter()
        perfect = self.ctx.precheck()
        t1 = time.perf_counter()
        self.precheck_time_ = (t1 - t0) * 1e3
        if not perfect:
            t0 = time.perf_counter()
            self.ctx.init()
            t1 = time.perf_counter()
            self.init_time_ = (t1 - t0) * 1e3
            t0 = time.perf_counter()
            self.ctx.core()
            t1 = time.perf_counter()
            self.core_time_ = (t1 - t0) * 1e3
        return self.ctx.post().tolist()

    def PrintProfilingInfo(self) -> None:  # noqa: N802
        name = self.GetEngineName()
        total = self.precheck_time_ + self.init_time_ + self.core_time_
        print(f"{name} Profiling Info:")
        print(f"{name} Precheck Time: {self.precheck_time_} ms")
        print(f"{name} Init Time: {self.init_time_} ms")
        print(f"{name} Core Time: {self.core_time_} ms")
        print(f"{name} Total Time: {total} ms")
        print("=" * 66)

    def close(self) -> None:
        if self._own:
            self.ctx.close()
