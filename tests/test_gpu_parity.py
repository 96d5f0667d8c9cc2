"""Parity of the CUDA path with the reference, through the C ABI.

Integer work, so the bar is bit-exact: the matching must equal the one the
reference's own engines returned (tests/golden), the proposal count must
equal the reference's, and the GPU stability checker must find no blocking
pair.  Full-size cases (n = 30000) are generated on the device by the
library's generator; the SHA-256 of the generated lists must equal the
digest recorded with the fixture, so the device inputs are the very inputs
the reference solved.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import oracle
import pactae_b200 as pb
from conftest import golden_match, load_cases

pytestmark = pytest.mark.gpu

CASES = load_cases()
SMALL = [c for c in CASES if c["n"] <= 2000]
FULL = [c for c in CASES if c["n"] > 2000]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()


def to_host(t) -> np.ndarray:
    return t if isinstance(t, np.ndarray) else t.cpu().numpy()


# -- generator --------------------------------------------------------------
GEN_CASES = [
    (pb.SMP_GEN_UNIFORM, n, 0) for n in (1, 2, 7, 64, 1000)
] + [
    (pb.SMP_GEN_CONGESTED, 300, 0), (pb.SMP_GEN_CORRELATED, 301, 500), (pb.SMP_GEN_CORRELATED, 100, 0),
    (pb.SMP_GEN_PERFECT, 200, 0), (pb.SMP_GEN_REF_CONGESTED, 150, 0), (pb.SMP_GEN_GROUPED, 250, 5),
    (pb.SMP_GEN_GROUPED, 256, 64), (pb.SMP_GEN_SOLO, 3, 0), (pb.SMP_GEN_SOLO, 129, 0),
]


@pytest.mark.parametrize("kind,n,param", GEN_CASES)
@pytest.mark.parametrize("salt", [0, 5])
def test_device_generator_matches_oracle(ctx, kind, n, param, salt):
    pm_d, pw_d = ctx.generate(kind, n, seed=77, salt=salt, param=param)
    pm, pw = oracle.generate(kind, n, 77, salt, param)
    assert np.array_equal(to_host(pm_d), pm)
    assert np.array_equal(to_host(pw_d), pw)


def test_generator_host_output(ctx):
    pm, pw = ctx.generate(pb.SMP_GEN_UNIFORM, 300, seed=9, device=False)
    opm, opw = oracle.generate(pb.SMP_GEN_UNIFORM, 300, 9)
    assert np.array_equal(pm, opm) and np.array_equal(pw, opw)


# -- solve vs the reference's matchings ------------------------------------
@pytest.mark.parametrize("case", SMALL, ids=[c["name"] for c in SMALL])
def test_solve_host_inputs_match_reference(ctx, case):
    pm, pw = oracle.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
    match, st = ctx.solve(pm, pw, check=True)
    assert np.array_equal(match, golden_match(case["name"]))
    assert st["proposals"] == case["proposals"]
    assert st["blocking_pairs"] == 0


@pytest.mark.parametrize("case", SMALL, ids=[c["name"] for c in SMALL])
def test_solve_device_inputs_match_reference(ctx, case):
    pm, pw = ctx.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
    match, st = ctx.solve(pm, pw)
    assert np.array_equal(to_host(match), golden_match(case["name"]))
    assert st["proposals"] == case["proposals"]


@pytest.mark.slow
@pytest.mark.parametrize("case", FULL, ids=[c["name"] for c in FULL])
def test_full_size_matches_reference(ctx, case):
    import torch

    pm, pw = ctx.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
    assert sha(to_host(pm)) == case["sha256_pref_m"]
    assert sha(to_host(pw)) == case["sha256_pref_w"]
    match, st = ctx.solve(pm, pw, check=True)
    assert sha(to_host(match)) == case["sha256_match"]
    assert np.array_equal(to_host(match), golden_match(case["name"]))
    assert st["proposals"] == case["proposals"]
    assert st["blocking_pairs"] == 0
    del pm, pw
    torch.cuda.empty_cache()


# -- configurations of the pipeline give the same answer ----------------------
@pytest.mark.parametrize("prefix_k,tail", [(-1, -1), (-1, 0), (0, -1), (1, 0), (33, 1), (0, 200)])
def test_pipeline_variants_agree(prefix_k, tail):
    with pb.Context(prefix_k=prefix_k, tail_threshold=tail) as c:
        for case in [x for x in SMALL if x["name"] in (
                "uniform_n2000", "congested_n500", "correlated_n500", "uniform_n33", "solo_n100", "uniform_n1")]:
            pm, pw = oracle.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
            match, st = c.solve(pm, pw)
            assert np.array_equal(match, golden_match(case["name"])), case["name"]
            assert st["proposals"] == case["proposals"]


# -- host-pointer solves of n >= 4096 copy only what they read -----------------
@pytest.mark.parametrize("kind,param,prefix_k,mode", [
    (pb.SMP_GEN_UNIFORM, 0, 0, 1),        # query mode: pref_w arrives in row chunks
    (pb.SMP_GEN_UNIFORM, 0, 8, 2),        # men go beyond an 8-choice prefix: the rest of pref_m follows
    (pb.SMP_GEN_CONGESTED, 0, 0, 3),      # everything is copied first; the men share one list: women propose
    (pb.SMP_GEN_CORRELATED, 500, 0, None),
    (pb.SMP_GEN_PERFECT, 0, 0, None),     # perfect: only the first choices are read
])
def test_streamed_host_solve_matches_oracle(kind, param, prefix_k, mode):
    n = 4099  # rows start off 16-byte boundaries; chunks of uneven size
    pm, pw = oracle.generate(kind, n, 17, 0, param)
    want, props = oracle.gs_seq(pm, pw)
    with pb.Context(prefix_k=prefix_k) as c:
        match, st = c.solve(pm, pw)
        again, st2 = c.solve(pm, pw)
    assert np.array_equal(match, want) and st["proposals"] == props
    assert np.array_equal(again, want) and st2["proposals"] == props
    if mode is not None:
        assert st["mode"] == mode
    if kind == pb.SMP_GEN_PERFECT:
        assert st["perfect"] == 1


def test_phase_api_and_engine_mirror(ctx):
    case = next(c for c in SMALL if c["name"] == "uniform_n2000")
    pm, pw = oracle.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
    smp = pb.SmpObj.CreateFromFlatLists(pm.reshape(-1), pw.reshape(-1), case["n"])
    eng = pb.SmpEngineB200(smp, case["n"], ctx=ctx)
    match = eng.FindStableMatching()
    assert match == golden_match(case["name"]).tolist()
    st = ctx.stats()
    assert st["proposals"] == case["proposals"] and st["perfect"] == 0
    assert eng.init_time_ > 0 and eng.core_time_ > 0


def test_perfect_instance_short_circuits(ctx):
    case = next(c for c in SMALL if c["name"] == "perfect_n1000")
    pm, pw = oracle.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
    match, st = ctx.solve(pm, pw, check=True)
    assert st["perfect"] == 1 and st["proposals"] == case["n"] and st["blocking_pairs"] == 0
    assert np.array_equal(match, pm[:, 0])
    # the phase API skips init and core, like AbsSmpEngine
    smp = pb.SmpObj.CreateFromFlatLists(pm, pw, case["n"])
    eng = pb.SmpEngineB200(smp, case["n"], ctx=ctx)
    assert eng.FindStableMatching() == pm[:, 0].tolist()
    assert eng.init_time_ == 0.0
    # with the precheck off the full pipeline runs and agrees
    match2, st2 = ctx.solve(pm, pw, precheck=False)
    assert np.array_equal(match2, match) and st2["perfect"] == 0


# -- inversion and checker ------------------------------------------------------
@pytest.mark.parametrize("n", [1, 3, 5, 127, 1000])
def test_invert_matches_oracle(ctx, n):
    _, pw = oracle.generate(pb.SMP_GEN_UNIFORM, n, 31)
    assert np.array_equal(ctx.invert(pw), oracle.invert(pw))


def test_checker_counts_blocking_pairs(ctx):
    pm, pw = oracle.generate(pb.SMP_GEN_UNIFORM, 500, 8)
    m, props = oracle.gs_seq(pm, pw)
    assert ctx.check(pm, pw, m) == (0, props)
    for seed in range(3):
        rng = np.random.default_rng(seed)
        bad = m.copy()
        i, j = rng.choice(500, 2, replace=False)
        bad[[i, j]] = bad[[j, i]]
        assert ctx.check(pm, pw, bad) == oracle.check(pm, pw, bad)
    with pytest.raises(pb.SmpError) as e:
        ctx.check(pm, pw, np.zeros(500, np.int32))
    assert e.value.status == pb.SMP_ERR_INVALID_INPUT


# -- invalid inputs are rejected, never run off the end ------------------------
def test_invalid_inputs_rejected(ctx):
    pm, pw = oracle.generate(pb.SMP_GEN_UNIFORM, 200, 3)
    cases = []
    bad = pw.copy()
    bad[7, 3] = bad[7, 4]
    cases.append((pm, bad, 0))                      # duplicate in a woman's row
    bad = pw.copy()
    bad[9, 0] = 5000
    cases.append((pm, bad, 0))                      # out of range in a woman's row
    bad = pm.copy()
    bad[4, 0] = -1
    cases.append((bad, pw, 0))                      # out of range first choice
    bad = pm.copy()
    bad[4, 5] = 200
    cases.append((bad, pw, 0))                      # out of range inside the prefix
    bad = pm.copy()
    bad[4, 150] = bad[4, 151]
    cases.append((bad, pw, pb.SMP_F_VALIDATE))      # duplicate caught by full validation
    import ctypes
    from pactae_b200 import _lib

    for a, b, flags in cases:
        a = np.ascontiguousarray(a, np.int32)
        b = np.ascontiguousarray(b, np.int32)
        out = np.empty(200, np.int32)
        rc = _lib.lib.smp_b200_solve(ctx.handle, ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(b.ctypes.data),
                                     200, ctypes.c_void_p(out.ctypes.data), flags, None)
        assert rc == pb.SMP_ERR_INVALID_INPUT
    # the context is still usable afterwards
    match, _ = ctx.solve(pm, pw)
    assert np.array_equal(match, oracle.gs_seq(pm, pw)[0])


@pytest.mark.parametrize("n,row", [(4999, 10), (4999, 4990), (6000, 3001)])
@pytest.mark.parametrize("defect", ["duplicate", "out_of_range", "negative", "wraps_to_valid"])
@pytest.mark.parametrize("host", [False, True])
def test_bad_row_deep_in_the_inversion(ctx, n, row, defect, host):
    # At these sizes each CTA of the query-mode inversion works through many
    # rows, so a bad row is found after rows that were permutations (row 10
    # is the first row of its CTA).  Host inputs take the streamed path,
    # which packs pref_w to 16 bits on the host: a -1 where the 0 was, or
    # v + 65536 where v was, must not pack into a permutation.
    pm, pw = ctx.generate(pb.SMP_GEN_UNIFORM, n, seed=77)
    pw = pw.clone()
    if defect == "duplicate":
        pw[row, 5] = pw[row, 6]
    elif defect == "out_of_range":
        pw[row, n - 1] = n + 5
    elif defect == "negative":
        pw[row, int((pw[row] == 0).nonzero()[0, 0])] = -1
    else:
        pw[row, 7] += 65536
    if host:
        pm, pw = to_host(pm), to_host(pw)
    with pytest.raises(pb.SmpError) as e:
        ctx.solve(pm, pw)
    assert e.value.status == pb.SMP_ERR_INVALID_INPUT
    # the same context solves the intact instance afterwards
    pm2, pw2 = ctx.generate(pb.SMP_GEN_UNIFORM, n, seed=77)
    match, st = ctx.solve(pm2, pw2)
    if n == 4999 and row == 10 and defect == "duplicate" and not host:
        want, props = oracle.gs_seq(to_host(pm2), to_host(pw2))
        assert np.array_equal(to_host(match), want) and st["proposals"] == props


@pytest.mark.parametrize("kind,n,param", [
    (pb.SMP_GEN_CONGESTED, 4097, 0),      # men alike, women not: the bulk runs with its shared filter
    (pb.SMP_GEN_REF_CONGESTED, 3001, 0),  # both sides alike: plain bulk, displacement-heavy tail
    (pb.SMP_GEN_GROUPED, 3000, 3),
    (pb.SMP_GEN_CORRELATED, 4096, 50),
    (pb.SMP_GEN_SOLO, 1500, 0),           # one chain scanning deep: all of it in the CTA-wide tail
])
def test_deep_chain_families_match_oracle(ctx, kind, n, param):
    # Rank-mode solves whose last chains k_tail hands to the CTA-wide tail
    # kernel, one after another; the matching and the proposal count must not
    # depend on that order.
    pm, pw = ctx.generate(kind, n, seed=11, param=param)
    match, st = ctx.solve(pm, pw, check=True)
    want, props = oracle.gs_seq(to_host(pm), to_host(pw))
    assert np.array_equal(to_host(match), want)
    assert st["proposals"] == props
    assert st["blocking_pairs"] == 0


def twist(pm):
    """One man swaps his last two choices: the men no longer share one list."""
    pm = pm.copy()
    n = pm.shape[0]
    pm[n // 2, [n - 2, n - 1]] = pm[n // 2, [n - 1, n - 2]]
    return pm


@pytest.mark.parametrize("shared", [True, False])
@pytest.mark.parametrize("where", ["man_deep", "man_first_choices", "woman_row", "woman_out_of_range",
                                   "woman_last_row"])
def test_rank_mode_rejects_bad_entries(ctx, where, shared):
    # Congested lists: men alike in every first choice.  With one shared list
    # the women propose after a screen of both lists; with one man's list
    # twisted the screen hands over to the men's rank mode (inversion,
    # transpose, ranks by position).  A bad entry anywhere must end the solve
    # with the status -- a bad man's row also differs from row 0, so those
    # cases reach the rank mode -- and the context must solve the intact
    # instance afterwards.
    n = 1001
    pm, pw = oracle.generate(pb.SMP_GEN_CONGESTED, n, 5)
    pm = pm.copy() if shared else twist(pm)
    pw = pw.copy()
    if where == "man_deep":
        pm[7, 900] = n + 3
    elif where == "man_first_choices":
        pm[11, 3] = -2
    elif where == "woman_row":
        pw[20, 10] = pw[20, 11]
    elif where == "woman_out_of_range":
        pw[30, 5] = n + 7
    else:  # the last row, its last entries: the partial 16-byte word of the check
        pw[n - 1, n - 1] = pw[n - 1, n - 2]
    with pytest.raises(pb.SmpError) as e:
        ctx.solve(pm, pw)
    assert e.value.status == pb.SMP_ERR_INVALID_INPUT
    pm2, pw2 = oracle.generate(pb.SMP_GEN_CONGESTED, n, 5)
    if not shared:
        pm2 = twist(pm2)
    match, st = ctx.solve(pm2, pw2)
    want, props = oracle.gs_seq(pm2, pw2)
    assert np.array_equal(match, want) and st["proposals"] == props
    assert st["mode"] == (3 if shared else 0)


@pytest.mark.parametrize("kind,n,device", [
    (pb.SMP_GEN_CONGESTED, 2, False),
    (pb.SMP_GEN_CONGESTED, 3, False),
    (pb.SMP_GEN_CONGESTED, 17, False),
    (pb.SMP_GEN_CONGESTED, 1001, False),
    (pb.SMP_GEN_REF_CONGESTED, 999, False),   # both sides share one list
    (pb.SMP_GEN_CONGESTED, 4095, True),
    (pb.SMP_GEN_CONGESTED, 6001, True),        # rows start off 16-byte boundaries
    (pb.SMP_GEN_REF_CONGESTED, 5000, True),
])
def test_men_sharing_one_list_women_propose(ctx, kind, n, device):
    # All men share one list: the stable matching is unique and the women
    # propose; the matching and the men's proposal count n(n+1)/2 must equal
    # the oracle's men-proposing run.
    if device:
        pm, pw = ctx.generate(kind, n, seed=13)
    else:
        pm, pw = oracle.generate(kind, n, 13)
    match, st = ctx.solve(pm, pw)
    want, props = oracle.gs_seq(to_host(pm), to_host(pw))
    assert np.array_equal(to_host(match), want)
    assert st["proposals"] == props == n * (n + 1) // 2
    # up to n = 4 one distinct first choice in four already picks the query mode
    assert st["mode"] == (3 if n > 4 else 1)
    if kind == pb.SMP_GEN_REF_CONGESTED:
        # the women share one list too (paired rank for rank); with one
        # woman's list twisted they propose instead
        pw3 = twist(to_host(pw))
        match3, st3 = ctx.solve(to_host(pm), pw3)
        want3, props3 = oracle.gs_seq(to_host(pm), pw3)
        assert np.array_equal(match3, want3) and st3["proposals"] == props3 and st3["mode"] == 3
    # a twisted list goes to the men's rank mode with the same answer as the oracle
    pm2 = twist(to_host(pm))
    match2, st2 = ctx.solve(pm2, to_host(pw))
    want2, props2 = oracle.gs_seq(pm2, to_host(pw))
    assert np.array_equal(match2, want2) and st2["proposals"] == props2 and st2["mode"] != 3


def test_first_solve_of_a_fresh_context_takes_the_shared_list_path():
    # The dispatch reads the plan of the n being solved, so a fresh
    # context's first solve (no earlier plan) takes the women-proposing pass
    # for men sharing a list, as every later solve does.
    for kind in (pb.SMP_GEN_REF_CONGESTED, pb.SMP_GEN_CONGESTED):
        with pb.Context() as c:
            pm, pw = c.generate(kind, 3001, seed=19)
            match, st = c.solve(pm, pw)
            assert st["mode"] == 3 and st["proposals"] == 3001 * 3002 // 2
            want, _ = oracle.gs_seq(to_host(pm), to_host(pw))
            assert np.array_equal(to_host(match), want)


def test_bad_arguments(ctx):
    with pytest.raises(pb.SmpError) as e:
        ctx.generate(pb.SMP_GEN_SOLO, 2, seed=1)
    assert e.value.status == pb.SMP_ERR_INVALID_ARG
    import ctypes
    from pactae_b200 import _lib

    assert _lib.lib.smp_b200_solve(ctx.handle, None, None, 10, None, 0, None) == pb.SMP_ERR_INVALID_ARG
    x = np.zeros(4, np.int32)
    p = ctypes.c_void_p(x.ctypes.data)
    assert _lib.lib.smp_b200_solve(ctx.handle, p, p, 0, p, 0, None) == pb.SMP_ERR_INVALID_ARG
    assert _lib.lib.smp_b200_solve(ctx.handle, p, p, pb.SMP_B200_MAX_N + 1, p, 0, None) == pb.SMP_ERR_INVALID_ARG
    assert _lib.lib.smp_b200_init(ctx.handle) in (pb.SMP_OK, pb.SMP_ERR_INVALID_ARG)


@pytest.mark.parametrize("seed", range(8))
def test_random_instances_against_oracle(ctx, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 3000))
    kind = int(rng.choice([pb.SMP_GEN_UNIFORM, pb.SMP_GEN_CONGESTED, pb.SMP_GEN_CORRELATED, pb.SMP_GEN_GROUPED]))
    param = {pb.SMP_GEN_CORRELATED: int(rng.integers(0, 2000)), pb.SMP_GEN_GROUPED: int(rng.integers(1, 64))}.get(
        kind, 0)
    pm, pw = ctx.generate(kind, n, seed=seed + 500, param=param)
    match, st = ctx.solve(pm, pw)
    want, props = oracle.gs_seq(to_host(pm), to_host(pw))
    assert np.array_equal(to_host(match), want)
    assert st["proposals"] == props


def test_query_bucket_overflow_falls_back_to_rank_mode():
    # Half the men share a first choice with another man (n/2 distinct first
    # choices: query mode), and every man's next 191 choices are the same
    # women, so their buckets receive n queries each, far above capacity.
    n = 2000
    rng = np.random.default_rng(41)
    common = np.arange(n - 191, n)
    pm = np.empty((n, n), np.int32)
    for m in range(n):
        first = m % (n // 2)
        rest = rng.permutation(np.setdiff1d(np.arange(n), np.concatenate([[first], common])))
        pm[m] = np.concatenate([[first], common, rest])
    pw = np.stack([rng.permutation(n) for _ in range(n)]).astype(np.int32)
    want, props = oracle.gs_seq(pm, pw)
    with pb.Context() as c:
        match, st = c.solve(pm, pw)
    assert np.array_equal(match, want) and st["proposals"] == props
    assert st["mode"] == 2  # query round abandoned, rank-mode round solved it


# -- int32 ranks (the layout every n above 65535 uses), forced at small n ------
@pytest.mark.parametrize("tail", [0, -1])
def test_int32_ranks_match_reference(tail):
    # rank_bytes = 4 runs the int32 template family -- the int32 inversion,
    # transpose, bulk, tail (and its CTA-wide hand-over) and checker -- that
    # sizes above 65535 take; with the tail off the matching comes from the
    # bid words (k_match), as it does above 65535.
    names = {"uniform_n2000", "congested_n2000", "correlated_n2000", "grouped5_n300", "solo_n1000",
             "refcongested_n200", "uniform_n33", "uniform_n1", "perfect_n1000"}
    with pb.Context(rank_bytes=4, tail_threshold=tail) as c:
        for case in [x for x in SMALL if x["name"] in names]:
            pm, pw = oracle.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
            match, st = c.solve(pm, pw, check=True)
            assert np.array_equal(match, golden_match(case["name"])), case["name"]
            assert st["proposals"] == case["proposals"] and st["blocking_pairs"] == 0
            if not st["perfect"] and st["mode"] != 3:
                assert st["rank_bytes"] == 4
        # device inputs and the inversion entry point too
        case = next(x for x in SMALL if x["name"] == "correlated_n500")
        pm, pw = c.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
        match, st = c.solve(pm, pw)
        assert np.array_equal(to_host(match), golden_match(case["name"])) and st["rank_bytes"] == 4
        assert np.array_equal(c.invert(to_host(pw)), oracle.invert(to_host(pw)))


def test_rank_bytes_knob_rejects_other_widths():
    with pytest.raises(pb.SmpError) as e:
        pb.Context(rank_bytes=2 + 1)
    assert e.value.status == pb.SMP_ERR_INVALID_ARG


def test_error_text_names_the_failure(ctx):
    pm, pw = oracle.generate(pb.SMP_GEN_UNIFORM, 50, 3)
    bad = pw.copy()
    bad[4, 2] = bad[4, 3]
    with pytest.raises(pb.SmpError) as e:
        ctx.solve(pm, bad)
    assert e.value.status == pb.SMP_ERR_INVALID_INPUT and "invalid input detected on the device" in str(e.value)


@pytest.mark.slow
def test_n_above_65535_uses_int32_ranks():
    # n = 65600: rows of more than 65535 ranks, inverted straight in global
    # memory and verified (k_invert_global / k_invert_verify), int32 ranks
    # throughout, no tail kernel.  Device inputs ~17 GB per matrix; the
    # oracle runs on the host copy when the host has room for it.
    import psutil
    import torch

    n = 65600
    nn = n * n
    if psutil.virtual_memory().available < 6 * nn * 4:
        pytest.skip("host memory too small for the oracle at n = 65600")
    with pb.Context() as c:
        pm, pw = c.generate(pb.SMP_GEN_UNIFORM, n, seed=21)
        match, st = c.solve(pm, pw, check=True)
        assert st["rank_bytes"] == 4 and st["blocking_pairs"] == 0
        got = to_host(match)
        hpm, hpw = to_host(pm), to_host(pw)
        del pm, pw
    torch.cuda.empty_cache()
    want, props = oracle.gs_seq(hpm, hpw)
    assert np.array_equal(got, want) and st["proposals"] == props


@pytest.mark.parametrize("case", ["shared", "twisted", "both_shared", "bad_woman_row", "bad_shared_entry"])
def test_host_input_men_sharing_one_list(case):
    # Host-input solves of n >= 4096 whose men all make the same first choice
    # compare the men's rows on the host while pref_w crosses the link; when
    # they are all equal only row 0 of pref_m is sent and the women propose.
    n = 4099
    kind = pb.SMP_GEN_REF_CONGESTED if case == "both_shared" else pb.SMP_GEN_CONGESTED
    pm, pw = oracle.generate(kind, n, 23)
    pm, pw = pm.copy(), pw.copy()
    if case == "twisted":
        pm = twist(pm)
    elif case == "bad_woman_row":
        pw[n - 7, 11] = pw[n - 7, 12]
    elif case == "bad_shared_entry":
        pm[:, 40] = pm[:, 41]  # the shared list itself is not a permutation
    with pb.Context() as c:
        if case.startswith("bad"):
            with pytest.raises(pb.SmpError) as e:
                c.solve(pm, pw)
            assert e.value.status == pb.SMP_ERR_INVALID_INPUT
            return
        match, st = c.solve(pm, pw)
    want, props = oracle.gs_seq(pm, pw)
    assert np.array_equal(match, want) and st["proposals"] == props
    assert st["mode"] == (0 if case == "twisted" else 3)


@pytest.mark.parametrize("prefix_k", [1, 8, 0])
@pytest.mark.parametrize("kind", [pb.SMP_GEN_CONGESTED, pb.SMP_GEN_REF_CONGESTED])
def test_host_input_shared_list_sends_what_the_women_read(kind, prefix_k):
    # Men sharing one list, host inputs: only row 0 of pref_m, every woman's
    # first K entries and the 1024 women the shared list ranks lowest cross
    # whole; a woman who reaches the end of what the device holds of her row
    # stops, her row is sent and she resumes.  With K = 1 or 8 most women
    # stop at least once (several rounds); with the default K none should.
    n = 4099
    pm, pw = oracle.generate(kind, n, 27)
    want, props = oracle.gs_seq(pm, pw)
    with pb.Context(prefix_k=prefix_k) as c:
        for _ in range(2):  # the context's buffers are reused
            match, st = c.solve(pm, pw)
            assert np.array_equal(match, want) and st["proposals"] == props and st["mode"] == 3


@pytest.mark.parametrize("where", ["deep_row", "prefix", "resumed_row", "both_shared_row0"])
def test_host_input_shared_list_checks_what_it_sends(where):
    # Every entry sent is checked on the device.  A duplicate in the whole
    # row of the woman the shared list ranks last, in the first K entries of
    # a woman's row, or deep in the row of a woman who stops at the end of
    # her first 8 entries and is sent whole: each is reported.
    n = 4099
    kind = pb.SMP_GEN_REF_CONGESTED if where == "both_shared_row0" else pb.SMP_GEN_CONGESTED
    pm, pw = oracle.generate(kind, n, 31)
    pm, pw = pm.copy(), pw.copy()
    shared = pm[0]
    prefix_k = 0
    if where == "both_shared_row0":
        pw[:, n - 9] = pw[:, n - 8]  # every woman's row alike, none a permutation: only row 0 is sent
    elif where == "deep_row":
        w = int(shared[n - 1])
        pw[w, n - 5] = pw[w, n - 4]
    elif where == "prefix":
        w = int(shared[5])
        pw[w, 2] = pw[w, 3]
    else:
        # a woman outside the lowest 1024 of the shared list whose final man
        # lies past her first 8 entries: she stops there and is sent whole
        prefix_k = 8
        want, _ = oracle.gs_seq(pm, pw)
        husband = np.empty(n, np.int64)
        husband[want] = np.arange(n)
        rank_in_l = np.empty(n, np.int64)
        rank_in_l[shared] = np.arange(n)
        depth = np.array([int(np.nonzero(pw[v] == husband[v])[0][0]) for v in range(n)])
        w = int(np.nonzero((depth > 8) & (depth < n - 3) & (rank_in_l < n - 1024))[0][0])
        pw[w, n - 3] = pw[w, n - 2]
    with pb.Context(prefix_k=prefix_k) as c:
        with pytest.raises(pb.SmpError) as e:
            c.solve(pm, pw)
        assert e.value.status == pb.SMP_ERR_INVALID_INPUT
        good_pm, good_pw = oracle.generate(kind, n, 31)
        match, st = c.solve(good_pm, good_pw)
    want, props = oracle.gs_seq(good_pm, good_pw)
    assert np.array_equal(match, want) and st["proposals"] == props


@pytest.mark.parametrize("defect", ["none", "duplicate", "negative", "wraps_to_valid", "men_wrap"])
def test_host_input_rank_mode_sends_packed_lists(defect):
    # Rank-mode host-input solves send both lists packed to 16 bits, in row
    # groups, and widen each group back to int32 on the device.  A defect must
    # survive packing: a duplicate stays one, and -1 or v + 65536 pack to
    # 0xFFFF, which widens to 65535 >= n.  The defect sits in the last row
    # group of pref_w; "men_wrap" puts v + 65536 in every man's second choice,
    # which correlated lists make many men reach.
    n = 4099
    pm, pw = oracle.generate(pb.SMP_GEN_CORRELATED, n, 29, 0, 500)
    pm, pw = pm.copy(), pw.copy()
    row = n - 3
    if defect == "duplicate":
        pw[row, 5] = pw[row, 6]
    elif defect == "negative":
        pw[row, int(np.nonzero(pw[row] == 0)[0][0])] = -1
    elif defect == "wraps_to_valid":
        pw[row, 7] += 65536
    elif defect == "men_wrap":
        pm[:, 1] += 65536
    with pb.Context() as c:
        if defect != "none":
            with pytest.raises(pb.SmpError) as e:
                c.solve(pm, pw)
            assert e.value.status == pb.SMP_ERR_INVALID_INPUT
            pm, pw = oracle.generate(pb.SMP_GEN_CORRELATED, n, 29, 0, 500)
        match, st = c.solve(pm, pw)  # the context is still usable
    want, props = oracle.gs_seq(pm, pw)
    assert np.array_equal(match, want) and st["proposals"] == props and st["mode"] == 0


@pytest.mark.slow
def test_host_input_rank_mode_above_the_query_limit():
    # n = 33000, above the query path's 32767: a rank-mode host-input solve
    # still sends both lists packed (16 bits hold any n <= 65535).  Checked
    # against the device-input solve of the same lists.
    import torch

    n = 33000
    with pb.Context() as c:
        pm, pw = c.generate(pb.SMP_GEN_CORRELATED, n, seed=5, param=500)
        want, st0 = c.solve(pm, pw)
        want = to_host(want)
        hpm, hpw = to_host(pm), to_host(pw)
        del pm, pw
        torch.cuda.empty_cache()
        got, st = c.solve(hpm, hpw)
    assert st0["mode"] == 0 and st["mode"] == 0
    assert np.array_equal(got, want) and st["proposals"] == st0["proposals"]
