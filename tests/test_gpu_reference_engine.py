"""Parity with the reference's own GPU engine, SmpEngineBamboo
(src/smp/smp_engine_bamboo.cu: GPU rank and PR matrices, La3F9CoreKernel,
a host monitor that finishes a lone last chain on the CPU), compiled from the
reference's sources into oracle/_ref/libsmpref_bamboo.so with its release
flags.  On the same instances its matching must equal ours bit for bit: the
man-optimal stable matching is unique.  Skipped where that library was not
built (it needs the reference's sources at build time)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
import pactae_b200 as pb
from conftest import ROOT

pytestmark = pytest.mark.gpu

BAMBOO = ROOT / "oracle" / "_ref" / "libsmpref_bamboo.so"


@pytest.fixture(scope="module")
def bamboo():
    if not BAMBOO.exists():
        pytest.skip("oracle/_ref/libsmpref_bamboo.so not built")
    lib = ctypes.CDLL(str(BAMBOO))
    lib.ref_bamboo_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_double)]
    return lib


def bamboo_solve(lib, pm, pw):
    n = pm.shape[0]
    pm = np.ascontiguousarray(pm, np.int32)
    pw = np.ascontiguousarray(pw, np.int32)
    out = np.full(n, -1, np.int32)
    ms = (ctypes.c_double * 6)()
    rc = lib.ref_bamboo_solve(pm.ctypes.data, pw.ctypes.data, n, out.ctypes.data, ms)
    assert rc == 0
    return out


@pytest.mark.parametrize("kind,n,param", [
    (pb.SMP_GEN_UNIFORM, 2000, 0),
    (pb.SMP_GEN_UNIFORM, 4099, 0),        # a host-input solve of ours: streamed, packed pref_w
    (pb.SMP_GEN_CONGESTED, 600, 0),
    (pb.SMP_GEN_REF_CONGESTED, 500, 0),
    (pb.SMP_GEN_CORRELATED, 1500, 500),
    (pb.SMP_GEN_GROUPED, 1200, 5),
    (pb.SMP_GEN_SOLO, 800, 0),
    (pb.SMP_GEN_PERFECT, 1000, 0),
])
def test_matches_smp_engine_bamboo(ctx, bamboo, kind, n, param):
    pm, pw = oracle.generate(kind, n, 11, 0, param)
    ref = bamboo_solve(bamboo, pm, pw)
    ours, _ = ctx.solve(pm, pw)
    assert np.array_equal(ours, ref)
    assert np.array_equal(ref, oracle.gs_seq(pm, pw)[0])


INIT_GPU = ROOT / "oracle" / "_ref" / "libsmpref_gpu.so"


@pytest.mark.skipif(not INIT_GPU.exists(), reason="oracle/_ref/libsmpref_gpu.so not built")
@pytest.mark.parametrize("kind,n", [(pb.SMP_GEN_REF_CONGESTED, 1000), (pb.SMP_GEN_UNIFORM, 2999),
                                    (pb.SMP_GEN_REF_CONGESTED, 5000)])
def test_invert_matches_smp_init_gpu(ctx, kind, n):
    # The reference's GPU init engine SmpInitEngine3 ("Smp-Init-Gpu",
    # include/smp/smp_init_3.h:68-95, the engine its init study times) and
    # smp_b200_invert must produce the same int32 rank matrix.
    lib = ctypes.CDLL(str(INIT_GPU))
    lib.ref_gpu_rank.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
    pm, pw = oracle.generate(kind, n, 2)
    pm = np.ascontiguousarray(pm, np.int32)
    pw = np.ascontiguousarray(pw, np.int32)
    want = np.empty((n, n), np.int32)
    assert lib.ref_gpu_rank(pm.ctypes.data, pw.ctypes.data, n, want.ctypes.data) == 0
    assert np.array_equal(ctx.invert(pw), want)
