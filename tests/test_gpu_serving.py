"""The serving loop (smp_b200_server_*): requests of uneven size submitted
in a burst are admitted against the HBM budget, batched into overlapping
waves (and the large ones run on the all-SM pipeline concurrently), and each
result is the same as solving that request alone.  Bit-exact."""
from __future__ import annotations

import numpy as np
import pytest

import pactae_b200 as pb

pytestmark = pytest.mark.gpu

KIND_PARAM = {pb.SMP_GEN_UNIFORM: 0, pb.SMP_GEN_CONGESTED: 0, pb.SMP_GEN_CORRELATED: 500}


def make_requests(ctx, count, seed, n_lo, n_hi):
    import torch

    reqs = []
    for b in range(count):
        n, kind = pb.batch_instance(seed, b, n_lo, n_hi)
        pm, pw = ctx.generate(kind, n, seed=seed, salt=b, param=KIND_PARAM[kind])
        reqs.append((pm, pw, torch.full((n,), -1, dtype=torch.int32, device=pm.device)))
    return reqs


@pytest.mark.parametrize("large_slots", [1, 3])
def test_results_alone_equal_results_in_the_mix(ctx, large_slots):
    reqs = make_requests(ctx, 40, seed=6, n_lo=64, n_hi=3000)
    alone = [ctx.solve(pm, pw) for pm, pw, _ in reqs]
    # route_n = 1024: the larger requests take the single-instance pipeline
    # (large_slots of them at once) alongside the waves
    with pb.Server(route_n=1024, max_wave=8, waves=3, large_slots=large_slots) as srv:
        tickets = [srv.submit(pm, pw, mt) for pm, pw, mt in reqs]
        results = [srv.poll(t) for t in tickets]
        st = srv.stats()
    assert st["submitted"] == st["completed"] == 40
    assert st["large"] > 0 and st["waves"] > 1
    for (pm, pw, mt), (want, wst), res in zip(reqs, alone, results):
        assert res["status"] == 0
        assert np.array_equal(mt.cpu().numpy(), want.cpu().numpy())
        assert res["proposals"] == wst["proposals"]
        assert res["latency_ms"] >= res["queue_ms"] >= 0


def test_host_pointer_requests(ctx):
    reqs = make_requests(ctx, 6, seed=8, n_lo=64, n_hi=1500)
    with pb.Server(route_n=512) as srv:
        host = [(pm.cpu().numpy(), pw.cpu().numpy(), np.full(pm.shape[0], -1, np.int32)) for pm, pw, _ in reqs]
        tickets = [srv.submit(*h) for h in host]
        for t, (hpm, hpw, out) in zip(tickets, host):
            assert srv.poll(t)["status"] == 0
            want, _ = ctx.solve(hpm, hpw)
            assert np.array_equal(out, want)


def test_admission_budget_is_respected(ctx):
    reqs = make_requests(ctx, 16, seed=12, n_lo=200, n_hi=800)
    biggest = max(int(mt.numel()) for _, _, mt in reqs)
    budget = 10 * biggest * biggest * 2  # room for about two requests at a time
    with pb.Server(hbm_budget=budget, max_wave=4) as srv:
        tickets = [srv.submit(pm, pw, mt) for pm, pw, mt in reqs]
        assert all(srv.poll(t)["status"] == 0 for t in tickets)
        st = srv.stats()
    assert 0 < st["peak_bytes"] <= budget and st["admitted_bytes"] == 0
    for pm, pw, mt in reqs:
        want, _ = ctx.solve(pm, pw)
        assert np.array_equal(mt.cpu().numpy(), want.cpu().numpy())


def test_oversize_request_is_refused(ctx):
    import torch

    with pb.Server(hbm_budget=10 * 100 * 100) as srv:
        pm, pw = ctx.generate(pb.SMP_GEN_UNIFORM, 101, seed=1)
        with pytest.raises(pb.SmpError) as e:
            srv.submit(pm, pw, torch.empty(101, dtype=torch.int32, device="cuda:0"))
        assert e.value.status == pb.SMP_ERR_BUSY


def test_solves_beside_the_server(ctx):
    # Kernels with dynamic shared memory are launched from the caller's thread
    # (solves) and the server's thread at once, each with its own size.  A
    # launch must not fail because the other thread set the kernel's shared
    # memory limit for a smaller launch just before.
    import numpy as np

    big = make_requests(ctx, 8, seed=21, n_lo=700, n_hi=1600)
    small = make_requests(ctx, 12, seed=22, n_lo=40, n_hi=300)
    alone = [ctx.solve(pm, pw) for pm, pw, _ in big]
    with pb.Server(route_n=256) as srv:
        tickets = [srv.submit(pm, pw, mt) for pm, pw, mt in big]
        with pb.Context() as other:
            for _ in range(3):
                for pm, pw, _ in small:
                    m1, _ = other.solve(pm, pw)
                    m2, _ = other.solve(pm.cpu().numpy(), pw.cpu().numpy())
                    assert np.array_equal(m1.cpu().numpy(), m2)
        for t, (want, wst), (_, _, mt) in zip(tickets, alone, big):
            res = srv.poll(t)
            assert res["status"] == 0
            assert np.array_equal(mt.cpu().numpy(), want.cpu().numpy())
            assert res["proposals"] == wst["proposals"]


def test_large_requests_up_to_16384(ctx):
    # The top of the serving mix (n up to 16384, all three kinds) goes
    # through the large-request route -- each on its own context and stream,
    # several at once, beside a wave of small requests -- and every result
    # must equal the same request solved alone.
    import torch

    sizes = [(pb.SMP_GEN_UNIFORM, 16384), (pb.SMP_GEN_CONGESTED, 12000), (pb.SMP_GEN_CORRELATED, 9000),
             (pb.SMP_GEN_UNIFORM, 5003), (pb.SMP_GEN_CORRELATED, 16384), (pb.SMP_GEN_CONGESTED, 4097)]
    reqs = []
    for b, (kind, n) in enumerate(sizes):
        pm, pw = ctx.generate(kind, n, seed=61, salt=b, param=KIND_PARAM[kind])
        reqs.append((pm, pw, torch.full((n,), -1, dtype=torch.int32, device=pm.device)))
    reqs += make_requests(ctx, 12, seed=62, n_lo=64, n_hi=900)
    alone = [ctx.solve(pm, pw) for pm, pw, _ in reqs]
    with pb.Server(large_slots=3) as srv:
        tickets = [srv.submit(pm, pw, mt) for pm, pw, mt in reqs]
        results = [srv.poll(t) for t in tickets]
        st = srv.stats()
    assert st["large"] >= len(sizes)
    for (pm, pw, mt), (want, wst), res in zip(reqs, alone, results):
        assert res["status"] == 0
        assert np.array_equal(mt.cpu().numpy(), want.cpu().numpy())
        assert res["proposals"] == wst["proposals"]
