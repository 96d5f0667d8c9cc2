"""The batched path (smp_b200_batch_*): many instances of uneven size in one
persistent launch, against the single-instance solve, the oracle and the
plain one-launch-per-instance run of the same kernel.  Bit-exact."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import pactae_b200 as pb

pytestmark = pytest.mark.gpu

KIND_PARAM = {pb.SMP_GEN_UNIFORM: 0, pb.SMP_GEN_CONGESTED: 0, pb.SMP_GEN_CORRELATED: 500}


def make_batch(ctx, count, seed, n_lo, n_hi):
    import torch

    insts, meta = [], []
    for b in range(count):
        n, kind = pb.batch_instance(seed, b, n_lo, n_hi)
        pm, pw = ctx.generate(kind, n, seed=seed, salt=b, param=KIND_PARAM[kind])
        insts.append((pm, pw, torch.full((n,), -1, dtype=torch.int32, device=pm.device)))
        meta.append((n, kind))
    return insts, meta


@pytest.mark.parametrize("window,use_graph,block", [(0, True, 0), (32, False, 256), (128, True, 128)])
def test_batch_matches_single_solves(ctx, window, use_graph, block):
    insts, meta = make_batch(ctx, 48, seed=5, n_lo=16, n_hi=700)
    with pb.Batch(ctx, insts, window=window, use_graph=use_graph, block_threads=block) as batch:
        for _ in range(2):  # a replay gives the same answers
            status, props, st = batch.run()
            assert st["failed"] == 0 and all(s == 0 for s in status)
            for (pm, pw, mt), p in zip(insts, props):
                want, wst = ctx.solve(pm, pw)
                assert np.array_equal(mt.cpu().numpy(), want.cpu().numpy())
                assert p == wst["proposals"]
            assert st["proposals"] == sum(props)


def test_batch_plain_launches_agree(ctx):
    insts, meta = make_batch(ctx, 24, seed=9, n_lo=16, n_hi=400)
    with pb.Batch(ctx, insts) as batch:
        _, props_b, st_b = batch.run()
        got_b = [mt.cpu().numpy().copy() for _, _, mt in insts]
        for _, _, mt in insts:
            mt.fill_(-1)
        status, props_p, st_p = batch.run_plain()
        assert all(s == 0 for s in status) and props_p == props_b
        assert st_p["launches"] == 24 and st_b["launches"] == 1
        for (_, _, mt), g in zip(insts, got_b):
            assert np.array_equal(mt.cpu().numpy(), g)


def test_batch_against_oracle(ctx):
    insts, meta = make_batch(ctx, 16, seed=21, n_lo=16, n_hi=300)
    with pb.Batch(ctx, insts) as batch:
        _, props, _ = batch.run()
    for (pm, pw, mt), p in zip(insts, props):
        want, wp = oracle.gs_seq(pm.cpu().numpy(), pw.cpu().numpy())
        assert np.array_equal(mt.cpu().numpy(), want) and p == wp


def test_batch_flags_a_bad_instance_only(ctx):
    insts, meta = make_batch(ctx, 12, seed=3, n_lo=32, n_hi=200)
    bad_pw = insts[4][1]
    bad_pw[1, 0] = bad_pw[1, 1]  # not a permutation
    with pb.Batch(ctx, insts) as batch:
        status, props, st = batch.run()
    assert status[4] == pb.SMP_ERR_INVALID_INPUT
    assert st["failed"] == 1
    assert all(s == 0 for i, s in enumerate(status) if i != 4)


def test_batch_men_sharing_one_list(ctx):
    # All men share one list (the congested family): the batch solves these
    # with the women proposing, as the stable matching is unique; matchings
    # and the men's proposal counts must equal the oracle's.  Odd sizes, and
    # near-congested instances (one man's list differs) that must not take
    # that path.
    import torch

    insts, wants = [], []
    for b, n in enumerate([16, 17, 333, 1001, 2048]):
        pm, pw = oracle.generate(pb.SMP_GEN_CONGESTED, n, 40 + b)
        for twist in (False, True):
            pm2 = pm.copy()
            if twist:  # one man swaps two choices: lists no longer shared
                pm2[n // 2, [n - 2, n - 1]] = pm2[n // 2, [n - 1, n - 2]]
            wants.append(oracle.gs_seq(pm2, pw))
            insts.append((torch.from_numpy(pm2).cuda(), torch.from_numpy(pw).cuda(),
                          torch.full((n,), -1, dtype=torch.int32, device="cuda")))
    with pb.Batch(ctx, insts) as batch:
        status, props, st = batch.run()
    assert all(s == 0 for s in status)
    for (_, _, mt), (want, wp), p in zip(insts, wants, props):
        assert np.array_equal(mt.cpu().numpy(), want) and p == wp


@pytest.mark.parametrize("where", ["woman_row", "shared_list"])
def test_batch_men_sharing_one_list_bad_input(ctx, where):
    import torch

    n = 300
    pm, pw = oracle.generate(pb.SMP_GEN_CONGESTED, n, 7)
    pm, pw = pm.copy(), pw.copy()
    if where == "woman_row":
        pw[5, 3] = pw[5, 4]  # a woman's list is not a permutation
    else:
        pm[:, 10] = pm[:, 11]  # the shared list is not a permutation
    good_pm, good_pw = oracle.generate(pb.SMP_GEN_CONGESTED, n, 8)
    insts = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
              torch.full((n,), -1, dtype=torch.int32, device="cuda")) for a, b in ((pm, pw), (good_pm, good_pw))]
    with pb.Batch(ctx, insts) as batch:
        status, props, st = batch.run()
    assert status[0] == pb.SMP_ERR_INVALID_INPUT and status[1] == 0
    want, wp = oracle.gs_seq(good_pm, good_pw)
    assert np.array_equal(insts[1][2].cpu().numpy(), want) and props[1] == wp


# -- shapes: the rank matrix on chip or in the slab, tuned or fixed ------------
@pytest.mark.parametrize("rank_smem_kb", [-1, 32, 96])
def test_shared_and_global_rank_agree(ctx, rank_smem_kb):
    # with 32 KB instances up to n = 128 invert into shared memory, with 96 KB
    # up to n = 221; the rest (and all with -1) use the global slab
    insts, meta = make_batch(ctx, 40, seed=13, n_lo=16, n_hi=300)
    with pb.Batch(ctx, insts, rank_smem_kb=rank_smem_kb, tune=False) as batch:
        cfg = batch.config()
        assert cfg["rank_smem_kb"] == rank_smem_kb and cfg["tune"] == -1
        status, props, st = batch.run()
    assert st["failed"] == 0
    for (pm, pw, mt), p in zip(insts, props):
        want, wp = oracle.gs_seq(pm.cpu().numpy(), pw.cpu().numpy())
        assert np.array_equal(mt.cpu().numpy(), want) and p == wp


def test_autotuned_shape(ctx):
    insts, meta = make_batch(ctx, 64, seed=17, n_lo=16, n_hi=1024)
    with pb.Batch(ctx, insts) as batch:
        cfg = batch.config()
        assert cfg["tune"] == 1
        assert cfg["block_threads"] in (256, 512) and cfg["ctas_per_sm"] in (1, 2, 4)
        assert cfg["window"] in (32, 64, 128, 256) and cfg["rank_smem_kb"] in (-1, 32, 64, 96)
        status, props, st = batch.run()
    assert st["failed"] == 0
    for (pm, pw, mt), p in zip(insts, props):
        want, wst = ctx.solve(pm, pw)
        assert np.array_equal(mt.cpu().numpy(), want.cpu().numpy()) and p == wst["proposals"]


def test_fixed_shape_is_kept(ctx):
    insts, meta = make_batch(ctx, 20, seed=23, n_lo=16, n_hi=500)
    with pb.Batch(ctx, insts, block_threads=256, ctas_per_sm=4, window=64, rank_smem_kb=-1) as batch:
        cfg = batch.config()
        thr = cfg.pop("threshold_n")
        assert cfg == {"block_threads": 256, "ctas_per_sm": 4, "window": 64, "use_graph": 1,
                       "rank_smem_kb": -1, "tune": -1}
        assert thr == -1  # nothing above 1024 to route
        status, props, st = batch.run()
    assert st["failed"] == 0


def test_batch_top_of_the_mix_against_oracle(ctx):
    # The largest instances the mix draws (n in (2048, 4096]) of all three
    # kinds: the grouped slab inversion and, for the congested ones, the
    # women-proposing role swap, checked against the oracle's men-proposing
    # Gale-Shapley; small instances ride along so both rank placements run.
    import torch

    sizes = [(pb.SMP_GEN_UNIFORM, 4096), (pb.SMP_GEN_CONGESTED, 4096), (pb.SMP_GEN_CORRELATED, 4096),
             (pb.SMP_GEN_UNIFORM, 2049), (pb.SMP_GEN_CONGESTED, 3001), (pb.SMP_GEN_CORRELATED, 2600),
             (pb.SMP_GEN_UNIFORM, 100), (pb.SMP_GEN_CORRELATED, 64)]
    insts = []
    for b, (kind, n) in enumerate(sizes):
        pm, pw = ctx.generate(kind, n, seed=31, salt=b, param=KIND_PARAM[kind])
        insts.append((pm, pw, torch.full((n,), -1, dtype=torch.int32, device=pm.device)))
    with pb.Batch(ctx, insts) as batch:
        status, props, st = batch.run()
    assert st["failed"] == 0 and all(s == 0 for s in status)
    for (pm, pw, mt), p in zip(insts, props):
        want, wp = oracle.gs_seq(pm.cpu().numpy(), pw.cpu().numpy())
        assert np.array_equal(mt.cpu().numpy(), want) and p == wp


# -- the largest instances routed to the all-SM pipeline -----------------------
@pytest.mark.parametrize("use_graph", [True, False])
def test_routed_instances_match_the_oracle(ctx, use_graph):
    # Instances above threshold_n run the single-instance pipeline on side
    # streams beside the persistent kernel (forked and joined inside the
    # captured graph); the rest run in the batch.  Every kind on both sides,
    # and a defective instance among the routed ones, which alone fails.
    import torch

    sizes = [(pb.SMP_GEN_UNIFORM, 3000), (pb.SMP_GEN_CONGESTED, 2500), (pb.SMP_GEN_CORRELATED, 2100),
             (pb.SMP_GEN_UNIFORM, 1800), (pb.SMP_GEN_CORRELATED, 1600), (pb.SMP_GEN_UNIFORM, 1400),
             (pb.SMP_GEN_CONGESTED, 1200), (pb.SMP_GEN_UNIFORM, 900), (pb.SMP_GEN_CORRELATED, 300),
             (pb.SMP_GEN_CONGESTED, 200), (pb.SMP_GEN_UNIFORM, 64)]
    insts = []
    for b, (kind, n) in enumerate(sizes):
        pm, pw = ctx.generate(kind, n, seed=41, salt=b, param=KIND_PARAM[kind])
        insts.append((pm, pw, torch.full((n,), -1, dtype=torch.int32, device=pm.device)))
    bad = 5  # n = 1400: routed
    insts[bad][1][7, 2] = insts[bad][1][7, 3]
    with pb.Batch(ctx, insts, use_graph=use_graph, threshold_n=1300) as batch:
        assert batch.config()["threshold_n"] == 1300
        for _ in range(2):  # a replay gives the same answers
            for _, _, mt in insts:
                mt.fill_(-1)
            status, props, st = batch.run()
            assert status[bad] == pb.SMP_ERR_INVALID_INPUT and st["failed"] == 1
            for i, ((pm, pw, mt), p) in enumerate(zip(insts, props)):
                if i == bad:
                    continue
                assert status[i] == 0
                want, wp = oracle.gs_seq(pm.cpu().numpy(), pw.cpu().numpy())
                assert np.array_equal(mt.cpu().numpy(), want) and p == wp, i


def test_autotuned_threshold_is_reported(ctx):
    # A mix reaching n = 4096: the autotuner times routing none and the
    # largest 8, 32 and 128 instances, and keeps the fastest; whichever it
    # keeps, the answers equal the single solves'.
    insts, meta = make_batch(ctx, 160, seed=43, n_lo=16, n_hi=4096)
    with pb.Batch(ctx, insts) as batch:
        thr = batch.config()["threshold_n"]
        assert thr == -1 or thr >= 1024
        status, props, st = batch.run()
    assert st["failed"] == 0
    for k in sorted(range(len(meta)), key=lambda k: -meta[k][0])[:12] + list(range(0, 160, 16)):
        pm, pw, mt = insts[k]
        want, wst = ctx.solve(pm, pw)
        assert np.array_equal(mt.cpu().numpy(), want.cpu().numpy()) and props[k] == wst["proposals"]
