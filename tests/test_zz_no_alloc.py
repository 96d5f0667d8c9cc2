"""smp_b200_solve_static: the solve that allocates nothing.

Applications whose device memory is already held by their own caching
allocator, processes under a per-process device-memory limit, and loops that
must not stall on cudaMalloc/cudaFree cannot let a library allocate; this
entry point keeps its scratch in a fixed device array compiled into the
library instead.  The test calls it through the C ABI and checks that it
returns the same matching and proposal count as smp_b200_solve on the same
inputs, over calls in a row -- each later call starts from the scratch the
previous one left behind (a different n, a different instance) -- and that a
size beyond the array's limit is refused.  Integer work: the bar is equality.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _p(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def test_static_solve_matches_regular_solve():
    import torch

    import pactae_b200 as pb
    from pactae_b200 import _lib

    lib = _lib.lib
    cases = [
        (pb.SMP_GEN_UNIFORM, 1000, 11, 0),
        (pb.SMP_GEN_CONGESTED, 700, 12, 0),
        (pb.SMP_GEN_UNIFORM, 1000, 11, 0),  # the first case again, after the second one's leftovers
        (pb.SMP_GEN_CORRELATED, 1024, 13, 500),
    ]
    with pb.Context(device=0) as ctx:
        for kind, n, seed, param in cases:
            pm, pw = ctx.generate(kind, n, seed=seed, param=param)
            want, st = ctx.solve(pm, pw)
            out = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
            props = ctypes.c_int64(-1)
            torch.cuda.synchronize()
            rc = lib.smp_b200_solve_static(_p(pm), _p(pw), n, _p(out), ctypes.byref(props), None)
            assert rc == pb.SMP_OK, rc
            assert torch.equal(out, want), (kind, n)
            assert props.value == st["proposals"]

        # one case pinned to the oracle itself, independently of smp_b200_solve
        import oracle

        pm, pw = ctx.generate(pb.SMP_GEN_CORRELATED, 999, seed=14, param=300)
        want, props_want = oracle.gs_seq(pm.cpu().numpy(), pw.cpu().numpy())
        out = torch.full((999,), -1, dtype=torch.int32, device="cuda:0")
        props = ctypes.c_int64(-1)
        torch.cuda.synchronize()
        rc = lib.smp_b200_solve_static(_p(pm), _p(pw), 999, _p(out), ctypes.byref(props), None)
        assert rc == pb.SMP_OK and np.array_equal(out.cpu().numpy(), want) and props.value == props_want

        # beyond the fixed array: refused before anything runs
        big = _lib.SMP_B200_STATIC_MAX_N + 1
        pm, pw = ctx.generate(pb.SMP_GEN_UNIFORM, big, seed=1)
        out = torch.empty(big, dtype=torch.int32, device="cuda:0")
        rc = lib.smp_b200_solve_static(_p(pm), _p(pw), big, _p(out), None, None)
        assert rc == pb.SMP_ERR_UNSUPPORTED


def test_static_solve_rejects_invalid_lists():
    import torch

    import pactae_b200 as pb
    from pactae_b200 import _lib

    with pb.Context(device=0) as ctx:
        pm, pw = ctx.generate(pb.SMP_GEN_UNIFORM, 300, seed=4)
        bad = pw.clone()
        bad[5, 7] = bad[5, 8]  # a woman's row that is not a permutation
        out = torch.empty(300, dtype=torch.int32, device="cuda:0")
        torch.cuda.synchronize()
        rc = _lib.lib.smp_b200_solve_static(_p(pm), _p(bad), 300, _p(out), None, None)
        assert rc == pb.SMP_ERR_INVALID_INPUT
        # and the next call is unaffected
        want, _ = ctx.solve(pm, pw)
        rc = _lib.lib.smp_b200_solve_static(_p(pm), _p(pw), 300, _p(out), None, None)
        assert rc == pb.SMP_OK and torch.equal(out, want)
