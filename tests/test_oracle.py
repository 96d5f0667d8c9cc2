"""The CPU oracle, pinned to the reference.

The reference (victorliu-sq/PACTAE) ships no tests or golden vectors; the
fixtures in tests/golden/ were produced by running the reference's own CPU
engines (compiled from src/smp/smp_engine_{gs_1,mw_1,gs_2,mw_2}.cu) on seeded
inputs, see tests/golden/make_golden.py.  These tests check the oracle's
generator, Gale-Shapley and checker against them, plus the known answers the
reference's code implies (PERFECT returns the top choices,
src/smp/smp_engine_bamboo.cu:291-297; CONGESTED has a closed form).
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import oracle
from conftest import golden_match, load_cases

CASES = load_cases()
SMALL = [c for c in CASES if c["n"] <= 2000]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()


# Published known-answer vectors of Philox4x32-10 (Random123 distribution,
# kat_vectors): counter, key, output.
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,out", PHILOX_KAT)
def test_philox_known_answers(ctr, key, out):
    assert tuple(int(v) for v in oracle.philox(ctr, key)) == out


@pytest.mark.parametrize("case", SMALL, ids=[c["name"] for c in SMALL])
def test_generator_matches_golden_digest(case):
    pm, pw = oracle.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
    assert sha(pm) == case["sha256_pref_m"]
    assert sha(pw) == case["sha256_pref_w"]
    n = case["n"]
    for row in np.concatenate([pm, pw])[: min(2 * n, 64)]:
        assert np.array_equal(np.sort(row), np.arange(n))
    if "pref_m" in case:
        assert pm.tolist() == case["pref_m"] and pw.tolist() == case["pref_w"]


@pytest.mark.parametrize("case", SMALL, ids=[c["name"] for c in SMALL])
def test_gs_and_mw_match_reference(case):
    pm, pw = oracle.generate(case["kind"], case["n"], case["seed"], case["salt"], case["param"])
    ref = golden_match(case["name"])
    gs, gs_props = oracle.gs_seq(pm, pw)
    mw, mw_props = oracle.mw_seq(pm, pw)
    assert np.array_equal(gs, ref)
    assert np.array_equal(mw, ref)
    # every Gale-Shapley execution makes the same set of proposals
    assert gs_props == mw_props == case["proposals"]
    blocking, props = oracle.check(pm, pw, ref)
    assert blocking == 0 and props == case["proposals"]


def test_known_answer_tiny():
    # n = 1: the only matching.
    assert oracle.gs_seq([[0]], [[0]])[0].tolist() == [0]
    # n = 2, both men prefer woman 0, she prefers man 1: man 1 gets her.
    pm = [[0, 1], [0, 1]]
    pw = [[1, 0], [0, 1]]
    m, props = oracle.gs_seq(pm, pw)
    assert m.tolist() == [1, 0] and props == 3
    # 3 x 3 instance worked by hand: men-optimal differs from women-optimal.
    pm = [[0, 1, 2], [1, 2, 0], [2, 0, 1]]
    pw = [[1, 2, 0], [2, 0, 1], [0, 1, 2]]
    m, props = oracle.gs_seq(pm, pw)
    assert m.tolist() == [0, 1, 2] and props == 3
    assert oracle.check(pm, pw, [0, 1, 2])[0] == 0
    assert oracle.check(pm, pw, [2, 0, 1])[0] == 0  # the women-optimal matching is stable too
    assert oracle.check(pm, pw, [1, 0, 2])[0] > 0


@pytest.mark.parametrize("n", [3, 64, 777])
def test_perfect_returns_top_choices(n):
    pm, pw = oracle.generate(oracle.GEN_PERFECT, n, 99)
    assert oracle.is_perfect(pm)
    m, props = oracle.gs_seq(pm, pw)
    assert np.array_equal(m, pm[:, 0]) and props == n


@pytest.mark.parametrize("n", [2, 50, 301])
def test_ref_congested_closed_form(n):
    # Every man has row R, every woman row Q: woman R[i] ends with man Q[i].
    pm, pw = oracle.generate(oracle.GEN_REF_CONGESTED, n, 5)
    m, props = oracle.gs_seq(pm, pw)
    expect = np.empty(n, dtype=np.int32)
    expect[pw[0]] = pm[0]
    assert np.array_equal(m, expect)
    assert props == n * (n + 1) // 2


def test_congested_men_proposal_count():
    n = 300
    pm, pw = oracle.generate(oracle.GEN_CONGESTED, n, 3)
    assert (pm == pm[0]).all()
    _, props = oracle.gs_seq(pm, pw)
    assert props == n * (n + 1) // 2


@pytest.mark.parametrize("n,seed,women", [(40, 1, "uniform"), (301, 2, "uniform"), (257, 3, "correlated")])
def test_shared_men_list_has_one_stable_matching(n, seed, women):
    # The women-proposing solve of instances whose men share one list L
    # rests on this: the men-proposing and the women-proposing runs agree,
    # and both equal the serial dictatorship in which each woman, taken in
    # L's order, takes her best man still untaken.
    pm, _ = oracle.generate(oracle.GEN_CONGESTED, n, seed)
    if women == "uniform":
        _, pw = oracle.generate(oracle.GEN_UNIFORM, n, seed + 10)
    else:
        _, pw = oracle.generate(oracle.GEN_CORRELATED, n, seed + 10, 0, 500)
    assert (pm == pm[0]).all()
    men, _ = oracle.gs_seq(pm, pw)
    wives, _ = oracle.gs_seq(pw, pm)  # the women propose: wives[w] = her man
    from_women = np.empty(n, dtype=np.int32)
    from_women[wives] = np.arange(n, dtype=np.int32)
    assert np.array_equal(men, from_women)
    taken = np.zeros(n, dtype=bool)
    dictator = np.empty(n, dtype=np.int32)
    for w in pm[0]:
        m = next(int(x) for x in pw[w] if not taken[x])
        taken[m] = True
        dictator[m] = w
    assert np.array_equal(men, dictator)


def test_correlated_is_skewed_toward_high_scores():
    n = 400
    pm, _ = oracle.generate(oracle.GEN_CORRELATED, n, 4, 0, 500)
    # with sigma = 0.05 the first choices concentrate on a few top women
    assert len(set(pm[:, 0].tolist())) < n // 4
    pm0, _ = oracle.generate(oracle.GEN_CORRELATED, n, 4, 0, 0)
    assert (pm0 == pm0[0]).all()  # sigma = 0: everyone ranks by the common score


def test_generator_rejects_bad_arguments():
    with pytest.raises(ValueError):
        oracle.generate(oracle.GEN_SOLO, 2, 1)
    with pytest.raises(ValueError):
        oracle.generate(oracle.GEN_GROUPED, 10, 1, 0, 0)
    with pytest.raises(ValueError):
        oracle.generate(99, 10, 1)


def test_invalid_inputs_rejected():
    pm, pw = oracle.generate(oracle.GEN_UNIFORM, 20, 1)
    bad = pw.copy()
    bad[3, 4] = bad[3, 5]  # duplicate in a woman's row
    with pytest.raises(ValueError):
        oracle.invert(bad)
    with pytest.raises(ValueError):
        oracle.gs_seq(pm, bad)
    bad_m = pm.copy()
    bad_m[0, 0] = 20  # out of range
    with pytest.raises(ValueError):
        oracle.gs_seq(bad_m, pw)
    assert oracle.check(pm, pw, np.zeros(20, np.int32))[0] == -1  # not a matching


def test_checker_counts_blocking_pairs():
    pm, pw = oracle.generate(oracle.GEN_UNIFORM, 200, 8)
    m, _ = oracle.gs_seq(pm, pw)
    assert oracle.check(pm, pw, m)[0] == 0
    bad = m.copy()
    bad[[0, 1]] = bad[[1, 0]]
    # brute-force count of blocking pairs of the swapped matching
    rank = oracle.invert(pw)
    husband = np.empty(200, np.int64)
    husband[bad] = np.arange(200)
    brute = 0
    for man in range(200):
        for w in pm[man]:
            if w == bad[man]:
                break
            if rank[w, man] < rank[w, husband[w]]:
                brute += 1
    assert oracle.check(pm, pw, bad)[0] == brute


def test_batch_recipe_is_log_uniform():
    ns, kinds = zip(*(oracle.batch_instance(5, b, 16, 4096) for b in range(4000)))
    ns = np.array(ns)
    assert ns.min() >= 16 and ns.max() <= 4096
    # log-uniform: about half the mass below the geometric midpoint 256
    assert 0.45 < (ns < 256).mean() < 0.55
    assert set(kinds) == {0, 1, 2}


@pytest.mark.skipif(not oracle.ref_available(), reason="reference engines not built")
@pytest.mark.parametrize("seed", range(6))
def test_reference_engines_agree_with_oracle(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(40, 400))
    kind = int(rng.integers(0, 3))
    pm, pw = oracle.generate(kind, n, 1000 + seed, 0, 500 if kind == 2 else 0)
    want, _ = oracle.gs_seq(pm, pw)
    for eng in oracle.REF_ENGINES:
        if oracle.ref_engine_safe(eng, n):
            got, _ = oracle.ref_solve(eng, pm, pw)
            assert np.array_equal(got, want)
