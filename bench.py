#!/usr/bin/env python
"""Benchmark of the B200 Gale-Shapley solver (one JSON line on rank 0).

Workload: one stable-marriage instance, n = 30000, both preference sides
independent uniform random permutations (seed 2), int32 -- two 3.6 GB lists
plus the rank matrix, resident in HBM.  A step is one full solve of that
instance (precheck, rank inversion, proposals, tail, matching) through the C
ABI with device pointers.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--gpus N under torchrun runs N replicas (one per GPU, no collective on the
data path: a single instance does not shard).  --impl reference times the
reference's own multithreaded CPU engine (Mw-Par-Cpu) on the host cores on
the same instance, on rank 0 only.

Timing: W untimed warm-up solves, then K solves, each timed on the device
with the library's CUDA events on its own stream; the 7.2 GB inputs exceed
the 126 MB L2 and a 256 MB buffer is written before every timed solve
anyway.  The e2e number times smp_b200_solve with pinned host buffers (both
lists copied in, the matching copied out) by the host clock around the
synchronous call.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "instances/s batched vs plain per-instance launches; n=30k solve ms; p99 latency"
N_DEFAULT = 30000
SEED = 2
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
TRAFFIC_FILE = ROOT / "profiles" / "roofline_traffic.txt"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", "--size", dest="n", type=int, default=N_DEFAULT)
    ap.add_argument("--kind", type=int, default=0, help="workload kind (0 uniform, 1 congested, 2 correlated)")
    ap.add_argument("--param", type=int, default=0)
    ap.add_argument("--init-study", action="store_true",
                    help="the reference's init study (benchmark/figure_5.cu): its GPU init engine beside ours")
    ap.add_argument("--init-sizes", default="1000,5000,10000,15000,30000")
    ap.add_argument("--bamboo-study", action="store_true",
                    help="the reference's GPU engine SmpEngineBamboo beside ours on the same B200 and instances")
    ap.add_argument("--bamboo-cases", default="0:2000:1,0:30000:2",
                    help="kind:n:seed[:param] cases for --bamboo-study (param: the generator's, e.g. the "
                         "group size of kind 5); the reference's Figure 9 matrix at n = 30000 is "
                         "4:30000:9,3:30000:9,5:30000:9:5,6:30000:9")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 8192-instance batched leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg")
    ap.add_argument("--batch-count", type=int, default=8192)
    ap.add_argument("--no-plain", action="store_true", help="skip the one-launch-per-instance baseline")
    ap.add_argument("--no-routing", action="store_true",
                    help="skip timing the batch with its largest instances routed to the all-SM pipeline")
    ap.add_argument("--serving-loads", default="0.1,0.2,0.3,0.4,0.5,0.6,0.7,0.8,0.9,1.0",
                    help="offered loads as fractions of the measured saturation")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (n=2000 on the reference CPU path, congested and "
                         "correlated n=30000, Gs-Seq at n=30000)")
    ap.add_argument("--no-bamboo", action="store_true", help="skip the reference GPU engine beside ours")
    ap.add_argument("--no-solve-loop", action="store_true",
                    help="skip the batch's one-smp_b200_solve-per-instance comparison")
    ap.add_argument("--serving-requests", type=int, default=150)
    return ap.parse_args()


def workload_config(args) -> dict:
    kinds = {0: "uniform random permutations", 1: "congested (men share one row, women uniform)",
             2: f"correlated (sigma={args.param / 1e4})"}
    return {
        "workload": f"single SMP instance n={args.n}, {kinds.get(args.kind, args.kind)}, seed {SEED}, int32 "
                    f"(two {args.n * args.n * 4 / 1e9:.1f} GB preference lists + rank matrix resident in HBM)",
        "n": args.n,
        "kind": args.kind,
        "seed": SEED,
        "l2": "inputs (2 x n^2 x 4 B) exceed the 126 MB L2; a 256 MB buffer is written before each timed solve",
        "parallelism": "replicas" if args.gpus > 1 else "single GPU",
    }


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
class Dist:
    """One rank of the job (RANK / WORLD_SIZE / LOCAL_RANK from torchrun).
    The collectives are a barrier and max / sum of a scalar over ranks, on
    NCCL with a GPU per rank, else on gloo (the CPU tests)."""

    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            timeout = datetime.timedelta(seconds=120)
            if torch.cuda.is_available():
                torch.cuda.set_device(self.local_rank)
                self.device = f"cuda:{self.local_rank}"
                dist.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", self.local_rank))
            else:
                dist.init_process_group("gloo", timeout=timeout)
            self.pg = dist

    def _host_only(self, rank: int) -> "Dist":
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = rank
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        return self

    def barrier(self):
        if self.pg:
            import torch

            t = torch.ones(1, device=self.device)
            self.pg.all_reduce(t)
            if self.device != "cpu":
                torch.cuda.synchronize()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={CLOCK_FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak_hbm() -> tuple[float, str]:
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch(kernel: str, n: int) -> float | None:
    """DRAM bytes per launch of `kernel` at size n from the committed ncu
    summary (lines `kernel=<name> n=<n> dram_bytes=<bytes>`), else None."""
    try:
        for line in TRAFFIC_FILE.read_text().splitlines():
            f = dict(kv.split("=", 1) for kv in line.split() if "=" in kv)
            if f.get("kernel") == kernel and int(f.get("n", -1)) == n:
                return float(f["dram_bytes"])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def run_b200(args, dist: Dist) -> dict | None:
    import numpy as np
    import torch

    import pactae_b200 as pb

    dev = dist.local_rank
    torch.cuda.set_device(dev)
    n = args.n
    ctx = pb.Context(device=dev)
    pm, pw = ctx.generate(args.kind, n, seed=SEED, param=args.param)
    match = torch.empty(n, dtype=torch.int32, device=f"cuda:{dev}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")

    def one():
        flush.random_(0, 255)  # evicts L2 (untimed: the library's events bracket the solve only)
        torch.cuda.synchronize()
        _, st = ctx.solve(pm, pw, out=match)
        return st

    for _ in range(args.warmup):
        one()
    dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    t_wall0 = time.perf_counter()
    steps = [one() for _ in range(args.steps)]
    t_wall = time.perf_counter() - t_wall0
    dist.barrier()
    local_ms = sum(s["total_ms"] for s in steps)
    total_ms = dist.max(local_ms)  # max over ranks of the device time of K solves

    # parity of the timed result (cheap: against the proposals the fixture records)
    st0 = steps[-1]
    launches = int(sum(s["kernel_launches"] for s in steps))

    # e2e through the C ABI with pinned host buffers
    e2e = None
    h_pm = h_pw = None
    if not args.no_e2e:
        h_pm_t = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
        h_pw_t = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
        h_pm_t.copy_(pm)
        h_pw_t.copy_(pw)
        h_match = torch.empty(n, dtype=torch.int32, pin_memory=True)
        h_pm, h_pw, hm = h_pm_t.numpy(), h_pw_t.numpy(), h_match.numpy()
        del pm, pw
        torch.cuda.empty_cache()
        for _ in range(max(1, args.warmup)):
            ctx.solve(h_pm, h_pw, out=hm)
        dist.barrier()
        e2e_times = []
        for _ in range(args.steps):
            flush.random_(0, 255)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, e2e_st = ctx.solve(h_pm, h_pw, out=hm)
            e2e_times.append((time.perf_counter() - t0) * 1e3)
        e2e_total = dist.max(sum(e2e_times))
        assert np.array_equal(hm, match.cpu().numpy()), "e2e matching differs from the device-input solve"
        # A host-input query-mode solve copies each man's first K = 192
        # choices and all of pref_w, streamed in 16 row chunks under the
        # inversion -- when n <= 32767 packed to 16 bits on the host except
        # chunks 4 and 12, which cross as int32; rank mode and the retry copy
        # both lists whole as int32.
        if e2e_st["mode"] == 1:
            rows = [n * (k + 1) // 16 - n * k // 16 for k in range(16)]
            h2d = 4 * n * 192 + sum(r * n * (4 if n > 32767 or k % 8 == 4 else 2) for k, r in enumerate(rows))
        else:
            h2d = 8 * n * n
        e2e = {"value": e2e_total / (args.steps * dist.world), "unit": "ms",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": n * 4,
               "per_rank_ms_per_solve": e2e_total / args.steps,
               "path": "C ABI smp_b200_solve with pinned host buffers"}
    clk = clocks.stop()

    result = None
    if dist.rank == 0:
        ms_per_step = total_ms / args.steps
        peak, peak_kind = measured_peak_hbm()
        P = st0["proposals"]
        swapped = st0["mode"] == 3
        # The roofline unit is one solve: B_alg = 8 n^2 (inversion: read
        # pref_w, write an int32 rank matrix) + 36 B per proposal (4 B of the
        # man's list + one 32 B sector of the rank matrix), over the device
        # time of the whole solve.  When the men share one list the women
        # propose instead: the men's n(n+1)/2 proposals are counted, not made,
        # and the bytes the solve must move are both lists read once (the
        # screen that proves the list is shared and pref_w valid).
        b_solve = 8 * n * n if swapped else 8 * n * n + 36 * P
        solve_ach = b_solve / (ms_per_step * 1e-3) / 1e9
        query = st0["mode"] == 1
        K = 192
        # init phase: the bytes it must move at least (query mode: pref_w once,
        # the first K choices read twice, the bucket lists written and read,
        # the prefix written; rank mode: pref_w read, uint16 rank written,
        # prefix gathered)
        if swapped:
            init_bytes = 8 * n * n
        elif query:
            init_bytes = 4 * n * n + 20 * n * K
        else:
            init_bytes = 4 * n * n + 2 * n * n + 36 * n * K
        init_ms = statistics.mean(s["invert_ms"] for s in steps)
        init_ach = init_bytes / (init_ms * 1e-3) / 1e9
        init_kernels = ("k_swap_pos, k_swap_screen" if swapped else
                        "k_qcount, k_qscan, k_qscatter, k_qinvert" if query else "k_invert, k_prefix")
        phases = {
            "init": {"ms": round(init_ms, 4), "kernels": init_kernels, "min_bytes": init_bytes,
                     "achieved_gbs": round(init_ach, 1), "frac": round(init_ach / peak, 4), "bound": "hbm"},
            "bulk": {"ms": round(st0["bulk_ms"], 4), "kernels": "k_swap_gs (the women propose)" if swapped
                     else "k_bulk", "hops": st0["bulk_hops"], "bound": "latency (dependent L2 loads and atomics)"},
            "tail": {"ms": round(st0["tail_ms"], 4), "kernels": "k_tail_q" if query else "k_tail",
                     "hops": st0["tail_hops"], "bound": "latency (one SM, serial displacement chains)"},
        }
        traffic = traffic_per_launch("solve", n)
        roofline = {
            "kernel": "solve (precheck, init, k_bulk, tail; one solve = one launch unit)",
            "bound": "hbm",
            "achieved": round(solve_ach, 1),
            "peak": peak,
            "unit": "GB/s",
            "frac": round(solve_ach / peak, 4),
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
            "traffic": traffic,
            "traffic_note": "DRAM bytes per solve from ncu (profiles/), scaled from n=12000" if traffic else None,
            "algorithmic_bytes_per_launch": b_solve,
            "formula": ("B_alg = 8 n^2 (both lists read once; the women propose) over the solve's device time"
                        if swapped else "B_alg = 8 n^2 + 36 P over the solve's device time (CUDA events)"),
            "launch_ms": round(ms_per_step, 4),
            "phases": phases,
        }
        result = {
            "metric": METRIC,
            "value": round(total_ms / (args.steps * dist.world), 4),
            "unit": "ms",
            "n_gpus": dist.world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int32",
            "data": "synthetic (seeded Philox generator, same instance the reference fixtures were solved on)",
            "config": workload_config(args),
            "solves_per_s": round(args.steps * dist.world / (total_ms * 1e-3), 2),
            "proposals": P,
            "tail_men": st0["tail_men"],
            "tail_proposals": st0["tail_proposals"],
            "bulk_hops": st0["bulk_hops"],
            "tail_hops": st0["tail_hops"],
            "tail_us_per_hop": round(st0["tail_ms"] * 1e3 / st0["tail_hops"], 4) if st0["tail_hops"] else None,
            "phase_ms": {k: round(st0[k], 4) for k in ("precheck_ms", "init_ms", "core_ms", "post_ms",
                                                         "invert_ms", "bulk_ms", "tail_ms")},
            "wall_s_timed_loop": round(t_wall, 3),
            "roofline": roofline,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
    # CPU baseline: the reference's Mw-Par-Cpu on the same instance, rank 0, N = 1
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline and result is not None:
        result["cpu_baseline"] = cpu_baseline(args, h_pm, h_pw, match.cpu().numpy(), ctx)
    try:
        del pm, pw
    except NameError:
        pass
    torch.cuda.empty_cache()
    # the other configurations and the reference's sequential engine, rank 0 at N = 1
    if dist.rank == 0 and dist.world == 1 and not args.no_configs and result is not None and args.kind == 0:
        result["configs"] = run_configs(ctx, args, h_pm, h_pw, match.cpu().numpy())
        torch.cuda.empty_cache()
    if dist.rank == 0 and dist.world == 1 and not args.no_bamboo and result is not None and args.kind == 0:
        result["reference_gpu_engine"] = bamboo_cases(ctx, [(0, 2000, 1), (0, args.n, SEED)])
        torch.cuda.empty_cache()
    del h_pm, h_pw
    torch.cuda.empty_cache()
    if not args.no_batch:
        bres = run_batched(ctx, args, dist)
        if result is not None:
            result["batched"] = bres
    torch.cuda.empty_cache()
    if not args.no_serving:
        sres = run_serving(ctx, args, dist)
        if result is not None:
            result["serving"] = sres
    ctx.close()
    return result


KIND_PARAM = {0: 0, 1: 0, 2: 500}  # correlated: sigma = 0.05


def run_batched(ctx, args, dist: Dist) -> dict:
    """The batched mix: args.batch_count instances, n log-uniform in
    [16, 4096] (seed 5), kind uniform / congested / correlated per instance,
    inputs resident in HBM.  Batched persistent launch (CUDA graph replay)
    against the same kernel launched once per instance."""
    import torch

    import pactae_b200 as pb

    count = args.batch_count
    metas = [pb.batch_instance(5, b, 16, 4096) for b in range(count)]
    total = sum(n * n for n, _ in metas)
    t0 = time.perf_counter()
    pool_m = torch.empty(total, dtype=torch.int32, device=f"cuda:{dist.local_rank}")
    pool_w = torch.empty(total, dtype=torch.int32, device=f"cuda:{dist.local_rank}")
    match = torch.full((sum(n for n, _ in metas),), -1, dtype=torch.int32, device=f"cuda:{dist.local_rank}")
    insts, off, moff = [], 0, 0
    for b, (n, kind) in enumerate(metas):
        pm, pw = pool_m[off:off + n * n], pool_w[off:off + n * n]
        ctx.generate_into(kind, n, 5, pm.data_ptr(), pw.data_ptr(), salt=b, param=KIND_PARAM[kind])
        insts.append((pm, pw, match[moff:moff + n]))
        off += n * n
        moff += n
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    out = {"workload": f"{count} instances, n log-uniform in [16, 4096] (seed 5), kind uniform/congested/"
                       "correlated(sigma=0.05) per instance, inputs resident in HBM",
           "instances": count, "entries_per_list": total, "generate_s": round(gen_s, 2)}
    t_create = time.perf_counter()
    with pb.Batch(ctx, insts) as batch:
        out["create_s"] = round(time.perf_counter() - t_create, 2)  # includes the autotuner's runs
        out["shape"] = batch.config()
        batch.run()  # warm-up (also the L2 is far smaller than the 97 GB of lists)
        dist.barrier()
        runs = []
        for _ in range(3):
            status, props, st = batch.run()
            runs.append(st)
        assert all(x == 0 for x in status), "a batched instance failed"
        best = dist.max(min(r["ms"] for r in runs))  # best of 3 per rank, max over ranks
        # The same roofline as a single solve, summed over the instances,
        # counting only proposals that are made: an instance whose men share
        # one list (the congested third) is solved with the women proposing,
        # so its men's n(n+1)/2 proposals are counted, not made, and its bytes
        # are both lists read once (8 n^2), as for a single solve.
        made = sum(p for p, (_, kind) in zip(props, metas) if kind != 1)
        b_alg = 8 * total + 36 * made
        peak, _ = measured_peak_hbm()
        ach = b_alg / (best * 1e-3) / 1e9
        inv = 8 * total / (best * 1e-3) / 1e9
        out["roofline"] = {"bound": "hbm", "algorithmic_bytes": b_alg, "achieved": round(ach, 1), "peak": peak,
                           "unit": "GB/s", "frac": round(ach / peak, 4),
                           "formula": "sum over instances of 8 n^2, plus 36 P for instances whose proposals are "
                                      "made (not the women-proposing ones), over the batched launch time",
                           "inversion_only_gbs": round(inv, 1), "inversion_only_frac": round(inv / peak, 4)}
        out.update({"batched_ms": round(best, 3), "batched_ms_runs": [round(r["ms"], 3) for r in runs],
                    "instances_per_s": round(count * dist.world / (best * 1e-3), 1),
                    "proposals": runs[-1]["proposals"], "failed": runs[-1]["failed"],
                    "launches_per_run": runs[-1]["launches"]})
        # spot parity: a sample of instances (the largest first) against the
        # oracle's Gale-Shapley on the host
        import numpy as np

        import oracle

        order = sorted(range(count), key=lambda b: -metas[b][0])
        sample = order[:4] + [order[i] for i in range(4, count, max(1, count // 12))]
        for b in sample:
            pm, pw, mt = insts[b]
            n = mt.numel()
            want, wp = oracle.gs_seq(pm.view(n, n).cpu().numpy(), pw.view(n, n).cpu().numpy())
            assert np.array_equal(mt.cpu().numpy(), want) and props[b] == wp, f"batched instance {b} differs"
        out["oracle_checked"] = len(sample)
        out["threshold_n"] = out["shape"]["threshold_n"]
        if not args.no_routing:
            # The autotuner's routing choice, measured: the tuned shape with
            # none, or the largest 8, 32 and 128 instances, sent to the
            # all-SM single-instance pipeline on side streams beside the
            # persistent kernel (best of 3 graph replays each).
            shape = out["shape"]
            cands = []
            for r in (0, 8, 32, 128):
                thr = -1 if r == 0 else max(metas[order[r]][0], 1024)
                routed = sum(1 for n, _ in metas if thr > 0 and n > thr)
                if r and (routed == 0 or any(c["threshold_n"] == thr for c in cands)):
                    continue
                with pb.Batch(ctx, insts, block_threads=shape["block_threads"], ctas_per_sm=shape["ctas_per_sm"],
                              window=shape["window"], rank_smem_kb=shape["rank_smem_kb"], threshold_n=thr) as b2:
                    b2.run()
                    rr = [b2.run() for _ in range(3)]
                assert all(x == 0 for run in rr for x in run[0]), "a routed batch instance failed"
                cands.append({"routed": routed, "threshold_n": thr, "ms": round(min(run[2]["ms"] for run in rr), 3)})
            out["routing"] = {"chosen_threshold_n": out["threshold_n"], "candidates": cands,
                              "note": "instances above threshold_n run the all-SM single-instance pipeline on "
                                      "four side streams, forked and joined inside the batch's CUDA graph"}
        if not args.no_plain:
            _, pprops, pst = batch.run_plain()
            assert pst["proposals"] == runs[-1]["proposals"] and pst["failed"] == 0
            out.update({"plain_ms": round(pst["ms"], 1),
                        "plain_instances_per_s": round(count / (pst["ms"] * 1e-3), 1),
                        "plain_launches": pst["launches"],
                        "plain_note": "the same kernel launched once per instance with a grid of one CTA",
                        "batched_vs_plain": round(pst["ms"] / best, 1)})
    if not args.no_solve_loop:
        # The realistic per-instance alternative: every instance through the
        # all-SM single-instance solve (smp_b200_solve, device pointers), one
        # call after another; wall clock around the loop and the solves' own
        # device time.
        for pm, pw, mt in insts[:8]:  # warm the buffers for every size class
            ctx.solve(pm.view(mt.numel(), -1), pw.view(mt.numel(), -1), out=mt)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev_ms = 0.0
        for pm, pw, mt in insts:
            n = mt.numel()
            _, st = ctx.solve(pm.view(n, n), pw.view(n, n), out=mt)
            dev_ms += st["total_ms"]
        loop_s = time.perf_counter() - t0
        out.update({"solve_loop_s": round(loop_s, 3), "solve_loop_device_ms": round(dev_ms, 1),
                    "solve_loop_instances_per_s": round(count / loop_s, 1),
                    "batched_vs_solve_loop": round(loop_s * 1e3 / out["batched_ms"], 1),
                    "solve_loop_note": "one smp_b200_solve call per instance (all SMs each), host wall clock"})
    del pool_m, pool_w, match, insts
    return out


def run_serving(ctx, args, dist: Dist) -> dict:
    """Serving: single-instance requests, n log-uniform in [64, 16384] (seed 6),
    the three distributions, drawn from a pool of instances resident in HBM.
    Saturation = throughput of a burst; then Poisson arrivals at fractions of
    it.  Latency is submission to completion (the server's clock)."""
    import threading

    import numpy as np
    import torch

    import pactae_b200 as pb

    dev = f"cuda:{dist.local_rank}"
    pool_size = 48
    pool = []
    for b in range(pool_size):
        n, kind = pb.batch_instance(6, b, 64, 16384)
        pm, pw = ctx.generate(kind, n, seed=6, salt=b, param=KIND_PARAM[kind])
        pool.append((pm, pw, n))
    # each pool instance solved alone: every served matching must equal it
    solo = [ctx.solve(pm, pw)[0].clone() for pm, pw, _ in pool]
    checked = [0]
    rng = np.random.default_rng(6)

    def one_load(srv, rate, count, pool, host=False):
        # pool entries: (pref_m, pref_w, n, the matching solved alone)
        picks = rng.integers(0, len(pool), count)
        if host:
            outs = [np.empty(pool[i][2], dtype=np.int32) for i in picks]
        else:
            outs = [torch.empty(pool[i][2], dtype=torch.int32, device=dev) for i in picks]
        gaps = rng.exponential(1.0 / rate, count) if rate else np.zeros(count)
        tickets = [None] * count
        results = [None] * count

        def submitter():
            t = time.perf_counter()
            for k, i in enumerate(picks):
                t += gaps[k]
                delay = t - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tickets[k] = srv.submit(pool[i][0], pool[i][1], outs[k])

        th = threading.Thread(target=submitter)
        t0 = time.perf_counter()
        th.start()
        for k in range(count):
            while tickets[k] is None:
                time.sleep(0.0002)
            results[k] = srv.poll(tickets[k])
        th.join()
        wall = time.perf_counter() - t0
        lat = np.array([r["latency_ms"] for r in results])
        assert all(r["status"] == 0 for r in results)
        for k, i in enumerate(picks):
            same = np.array_equal(outs[k], pool[i][3]) if host else torch.equal(outs[k], pool[i][3])
            assert same, f"served request {k} differs from its instance solved alone"
        checked[0] += count
        return {"offered_per_s": round(rate, 1) if rate else None, "requests": count,
                "solves_per_s": round(count / wall, 1), "p50_ms": round(float(np.percentile(lat, 50)), 3),
                "p99_ms": round(float(np.percentile(lat, 99)), 3), "mean_n": int(np.mean([pool[i][2] for i in picks]))}

    pool = [(pm, pw, n, m) for (pm, pw, n), m in zip(pool, solo)]
    with pb.Server() as srv:
        one_load(srv, 0, 32, pool)  # warm-up
        sat = one_load(srv, 0, args.serving_requests, pool)
        saturation = sat["solves_per_s"]
        loads = []
        for f in [float(x) for x in args.serving_loads.split(",") if x]:
            r = one_load(srv, f * saturation, args.serving_requests, pool)
            r["load"] = f
            loads.append(r)
        st = srv.stats()
    out = {"workload": "Poisson stream of single instances, n log-uniform in [64, 16384] (seed 6), "
                       "uniform/congested/correlated, pool of 48 instances resident in HBM, "
                       "64 GiB admission budget", "saturation_solves_per_s": saturation,
           "burst": sat, "loads": loads, "waves": st["waves"], "large_path": st["large"],
           "peak_admitted_gb": round(st["peak_bytes"] / 1e9, 2)}
    del pool, solo
    # Host inputs: each request's lists are copied in when it is admitted
    # (10 n^2 bytes held while it runs) and its matching copied back; a
    # 4 GiB budget makes admission wait for room.
    hpool = []
    for b in range(16):
        n, kind = pb.batch_instance(7, b, 64, 16384)
        pm, pw = ctx.generate(kind, n, seed=7, salt=b, param=KIND_PARAM[kind])
        hpm = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
        hpw = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
        hpm.copy_(pm)
        hpw.copy_(pw)
        hpool.append((hpm.numpy(), hpw.numpy(), n, ctx.solve(pm, pw)[0].cpu().numpy()))
        del pm, pw
    budget = 4 << 30
    with pb.Server(hbm_budget=budget) as srv:
        one_load(srv, 0, 8, hpool, host=True)  # warm-up
        hsat = one_load(srv, 0, 64, hpool, host=True)
        hhalf = one_load(srv, 0.5 * hsat["solves_per_s"], 64, hpool, host=True)
        hhalf["load"] = 0.5
        hst = srv.stats()
    out["host_inputs"] = {"workload": "16 pinned host instances, n log-uniform in [64, 16384] (seed 7), "
                                      "lists copied in on admission, matching copied back",
                          "hbm_budget_gib": budget >> 30, "burst": hsat, "half_load": hhalf,
                          "peak_admitted_gb": round(hst["peak_bytes"] / 1e9, 2),
                          "mean_h2d_bytes_per_request": int(np.mean([8 * h[2] ** 2 for h in hpool]))}
    out["matchings_checked"] = checked[0]
    return out


def config_roofline(n: int, st: dict, ms: float) -> dict:
    """The single-solve roofline (8 n^2 + 36 P, or 8 n^2 when the women
    propose) for a solve of `ms` device milliseconds."""
    peak, kind = measured_peak_hbm()
    b = 8 * n * n if st["mode"] == 3 else 8 * n * n + 36 * st["proposals"]
    ach = b / (ms * 1e-3) / 1e9
    return {"algorithmic_bytes": b, "achieved_gbs": round(ach, 1), "peak": peak, "frac": round(ach / peak, 4),
            "peak_source": kind}


def run_configs(ctx, args, c2_pm, c2_pw, c2_match) -> dict:
    """The configurations besides the headline one, each with the reference's
    own CPU engines on the host cores: n = 2000 uniform (seed 1), the CPU
    config, with Gs-Seq-CPU and Mw-Par-Cpu; congested (men share one list,
    seed 3) and correlated (sigma = 0.05, seed 4) at n = 30000, device time
    with the L2 flushed, phases, the host-input solve through the C ABI, and
    Mw-Par-Cpu; and Gs-Seq-CPU on the headline instance.  Every matching is
    checked against the reference engine's."""
    import numpy as np
    import torch

    import oracle
    import pactae_b200 as pb

    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    have_ref = oracle.ref_available()
    cases = [("n2000_uniform", pb.SMP_GEN_UNIFORM, 2000, 1, 0, 20),
             ("n30000_congested", pb.SMP_GEN_CONGESTED, args.n, 3, 0, 5),
             ("n30000_correlated", pb.SMP_GEN_CORRELATED, args.n, 4, 500, 5)]
    for name, kind, n, seed, param, reps in cases:
        pm, pw = ctx.generate(kind, n, seed=seed, param=param)
        m = torch.empty(n, dtype=torch.int32, device=pm.device)
        for _ in range(2):
            ctx.solve(pm, pw, out=m)
        dev = []
        for _ in range(reps):
            flush.random_(0, 255)
            torch.cuda.synchronize()
            _, st = ctx.solve(pm, pw, out=m)
            dev.append(st)
        best = min(dev, key=lambda x: x["total_ms"])
        got = m.cpu().numpy()
        hpm_t = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
        hpw_t = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
        hpm_t.copy_(pm)
        hpw_t.copy_(pw)
        del pm, pw, m
        torch.cuda.empty_cache()
        hpm, hpw = hpm_t.numpy(), hpw_t.numpy()
        hm = torch.empty(n, dtype=torch.int32, pin_memory=True).numpy()
        ctx.solve(hpm, hpw, out=hm)
        e2e = []
        for _ in range(3 if n > 5000 else reps):
            t0 = time.perf_counter()
            _, est = ctx.solve(hpm, hpw, out=hm)
            e2e.append((time.perf_counter() - t0) * 1e3)
        assert np.array_equal(hm, got), f"{name}: host-input matching differs from the device-input one"
        rec = {"n": n, "kind": kind, "seed": seed, "param": param, "mode": best["mode"],
               "proposals": best["proposals"], "device_ms": round(best["total_ms"], 4),
               "device_ms_runs": [round(x["total_ms"], 4) for x in dev],
               "phases_ms": {k: round(best[k], 4) for k in ("precheck_ms", "invert_ms", "init_ms", "bulk_ms", "tail_ms",
                                                           "core_ms", "post_ms")},
               "roofline": config_roofline(n, best, best["total_ms"]),
               "e2e_ms": round(min(e2e), 3), "e2e_path": "C ABI smp_b200_solve with pinned host buffers"}
        if have_ref:
            prob = oracle.RefProblem(hpm, hpw)
            engines = (0, 3) if n <= 5000 else (3,)
            for eng in engines:
                ref_match, ms = prob.solve(eng)
                assert np.array_equal(ref_match, got), f"{name}: {oracle.REF_ENGINES[eng]} matching differs"
                rec[oracle.REF_ENGINES[eng]] = {"ms": round(sum(ms), 3), "phases_ms": [round(x, 3) for x in ms],
                                                "threads": 1 if eng == 0 else oracle.ref_threads()}
            prob.close()
        out[name] = rec
        del hpm_t, hpw_t
    if have_ref and c2_pm is not None:
        # the reference's sequential engine on the headline instance: one run
        prob = oracle.RefProblem(c2_pm, c2_pw)
        ref_match, ms = prob.solve(0)
        prob.close()
        assert np.array_equal(ref_match, c2_match), "Gs-Seq-CPU matching differs from the GPU's"
        out["n30000_uniform_gs_seq_cpu"] = {"ms": round(sum(ms), 3), "phases_ms": [round(x, 3) for x in ms],
                                            "threads": 1, "engine": "Gs-Seq-CPU (src/smp/smp_engine_gs_1.cu)"}
    out["cpu_engines_note"] = ("reference engines compiled from their sources into oracle/_ref; times are their own "
                               "precheck + init + core stopwatch")
    return out


def cpu_baseline(args, h_pm, h_pw, gpu_match, ctx) -> dict:
    import numpy as np

    import oracle

    n = args.n
    if h_pm is None:
        h_pm, h_pw = oracle.generate(args.kind, n, SEED, 0, args.param)
    if oracle.ref_available():
        eng = 3  # Mw-Par-Cpu, min(nproc, 96) threads
        prob = oracle.RefProblem(h_pm, h_pw)
        match, ms = prob.solve(eng)
        prob.close()
        assert np.array_equal(match, gpu_match), "reference CPU matching differs from the GPU's"
        return {"value": round(sum(ms), 3), "unit": "ms", "cores": oracle.ref_threads(), "kind": "reference",
                "sample": f"1 solve of the same n={n} instance by the reference's Mw-Par-Cpu "
                          f"(smp_engine_mw_2.cu), engine-reported precheck+init+core",
                "phases_ms": [round(x, 3) for x in ms]}
    t0 = time.perf_counter()
    match, _ = oracle.gs_seq(h_pm, h_pw)
    dt = (time.perf_counter() - t0) * 1e3
    assert np.array_equal(match, gpu_match)
    return {"value": round(dt, 3), "unit": "ms", "cores": 1, "kind": "port",
            "sample": f"1 solve of the same n={n} instance by the oracle's sequential Gale-Shapley"}


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU engine on the host cores
# ---------------------------------------------------------------------------
def run_reference(args, dist: Dist) -> dict | None:
    if dist.rank != 0:
        return None
    import oracle

    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libsmpref.so (the reference's CPU engines) not built"}
    n = args.n
    pm, pw = oracle.generate(args.kind, n, SEED, 0, args.param)
    prob = oracle.RefProblem(pm, pw)
    del pm, pw
    eng = 3  # Mw-Par-Cpu
    for _ in range(args.warmup):
        prob.solve(eng)
    times = []
    for _ in range(args.steps):
        _, ms = prob.solve(eng)
        times.append(sum(ms))
    prob.close()
    total = sum(times)
    ms_per_step = total / args.steps
    threads = oracle.ref_threads()
    return {
        "metric": METRIC,
        "value": round(ms_per_step, 3),
        "unit": "ms",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic (seeded Philox generator)",
        "config": workload_config(args),
        "impl": "reference",
        "cpu_baseline": {"value": round(ms_per_step, 3), "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": f"each step one solve of the n={n} instance by the reference's Mw-Par-Cpu "
                                   f"(smp_engine_mw_2.cu) with {threads} threads, engine-reported "
                                   "precheck+init+core"},
        "e2e": {"value": round(ms_per_step, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }


def run_init_study(args) -> None:
    """The reference's init study (benchmark/figure_5.cu) on this GPU: its GPU
    init engine Smp-Init-Gpu (SmpInitEngine3, built from its headers into
    oracle/_ref/libsmpref_gpu.so with its release flags) beside this
    library's inversion (smp_b200_invert, the same int32 rank matrix), on the
    reference's CONGESTED workload at n = 1000 .. 30000.  The reference's
    figures are its own report (kernel time = its stopwatch minus its
    transfers); ours are CUDA events around the inversion kernel.  One JSON
    line per n."""
    import ctypes

    import numpy as np
    import torch

    import oracle
    import pactae_b200 as pb

    lib_path = ROOT / "oracle" / "_ref" / "libsmpref_gpu.so"
    if not lib_path.exists():
        print(json.dumps({"init_study": "unavailable", "why": "oracle/_ref/libsmpref_gpu.so not built"}))
        return
    R = ctypes.CDLL(str(lib_path))
    dbl = ctypes.POINTER(ctypes.c_double)
    R.ref_gpu_init.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int, dbl, dbl, dbl]
    ctx = pb.Context(0)
    for n in [int(x) for x in args.init_sizes.split(",")]:
        pm, pw = oracle.generate(pb.SMP_GEN_REF_CONGESTED, n, SEED)
        ref = {}
        for pr in (0, 1):
            runs = []
            for _ in range(4):  # the first run warms the engine up; the best of the other three is kept
                k, t, tot = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
                rc = R.ref_gpu_init(pm.ctypes.data, pw.ctypes.data, n, pr, ctypes.byref(k), ctypes.byref(t),
                                    ctypes.byref(tot))
                runs.append((k.value, t.value, tot.value, rc))
            k, t, tot, rc = min(runs[1:])
            ref["rank_and_pr" if pr else "rank"] = {"kernel_ms": round(k, 3), "transfer_ms": round(t, 3),
                                                     "total_ms": round(tot, 3), "status": rc}
        dpw = torch.from_numpy(pw).cuda()
        ctx.invert(dpw)  # warm-up
        times = []
        for _ in range(3):
            rank = ctx.invert(dpw)
            times.append(ctx.stats()["init_ms"])
        ours = min(times)
        if n <= 5000:
            assert np.array_equal(rank.cpu().numpy(), oracle.invert(pw)), "rank matrix differs from the oracle"
        print(json.dumps({"init_study": "CONGESTED (reference generate_workloads_flat.h:14-47)", "n": n,
                          "reference_smp_init_gpu": ref,
                          "ours_k_invert_ms": round(ours, 4),
                          "rank_kernel_speedup": round(ref["rank"]["kernel_ms"] / ours, 1) if ours > 0 else None,
                          "ours_bytes_per_s": round(8 * n * n / (ours * 1e-3) / 1e9, 1)}), flush=True)
        del dpw, rank
        torch.cuda.empty_cache()
    ctx.close()


class stdout_to_stderr:
    """Sends file descriptor 1 to stderr for the duration (native code that
    prints to stdout included)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def bamboo_cases(ctx, cases) -> list[dict]:
    """The reference's own GPU engine, SmpEngineBamboo (the BambooSMP solve:
    GPU rank and PR matrices, La3F9CoreKernel, a host monitor that finishes a
    last lone chain on the CPU; src/smp/smp_engine_bamboo.cu), built from its
    sources into oracle/_ref/libsmpref_bamboo{,_o3}.so, beside this library's
    solve on the same B200 and the same instances (kind, n, seed).  The
    reference's figures are its engine's own precheck/init/core stopwatch
    (AbsSmpEngine, smp_engine_abs.h:10-36), with its untimed list upload and
    PR-matrix download listed apart; ours are the device-input solve (CUDA
    events) and the host-input solve through the C ABI (wall clock).
    Matchings must be identical.  One record per case."""
    import ctypes

    import numpy as np
    import torch

    libs = {}
    for tag, name in (("ptxas_O0_release", "libsmpref_bamboo.so"), ("ptxas_O3", "libsmpref_bamboo_o3.so")):
        path = ROOT / "oracle" / "_ref" / name
        if path.exists():
            lib = ctypes.CDLL(str(path))
            lib.ref_bamboo_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                             ctypes.POINTER(ctypes.c_double)]
            libs[tag] = lib
    if not libs:
        return [{"bamboo_study": "unavailable", "why": "oracle/_ref/libsmpref_bamboo*.so not built"}]

    def mem_available() -> int:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
        return 0

    records = []
    for case in cases:
        kind, n, seed = case[:3]
        param = case[3] if len(case) > 3 else 0
        # host bytes at peak: our pinned lists (8 n^2), the engine's SmpObj and
        # its construction copies (16 n^2) and its host PR matrix (8 n^2)
        need = 32 * n * n
        if mem_available() < 2 * need:
            records.append({"bamboo_study": f"kind {kind} n={n} seed {seed} param {param}", "unavailable":
                            f"host memory: {mem_available() >> 30} GiB available, {2 * need >> 30} GiB wanted"})
            continue
        dpm, dpw = ctx.generate(kind, n, seed, param=param)
        ours_match, _ = ctx.solve(dpm, dpw)  # warm-up
        dev_ms = []
        for _ in range(3):
            _, st = ctx.solve(dpm, dpw)
            dev_ms.append(st["total_ms"])
        want = ours_match.cpu().numpy()
        hpm_t = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
        hpw_t = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
        hpm_t.copy_(dpm)
        hpw_t.copy_(dpw)
        del dpm, dpw
        torch.cuda.empty_cache()
        hpm, hpw = hpm_t.numpy(), hpw_t.numpy()
        hm = torch.empty(n, dtype=torch.int32, pin_memory=True).numpy()
        ctx.solve(hpm, hpw, out=hm)
        e2e_ms = []
        for _ in range(3):
            t0 = time.perf_counter()
            ctx.solve(hpm, hpw, out=hm)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
        assert np.array_equal(hm, want), "host-input matching differs from the device-input one"
        ref = {}
        for tag, lib in libs.items():
            runs = []
            for _ in range(2):  # the first run warms the engine up
                ms = (ctypes.c_double * 6)()
                got = np.empty(n, np.int32)
                with stdout_to_stderr():  # the engine prints its progress; the bench's stdout is its JSON line
                    rc = lib.ref_bamboo_solve(hpm.ctypes.data, hpw.ctypes.data, n, got.ctypes.data, ms)
                runs.append((rc, list(ms), got))
            rc, ms, got = runs[-1]
            # engine-reported total: precheck + init + core with the lists
            # already on the device (the engine's constructor uploads them,
            # untimed); end to end: that upload plus FindStableMatching,
            # which adds the untimed PR-matrix download and PostProc
            ref[tag] = {"status": rc, "precheck_ms": round(ms[0], 3), "init_ms": round(ms[1], 3),
                        "core_ms": round(ms[2], 3), "engine_total_ms": round(ms[0] + ms[1] + ms[2], 3),
                        "untimed_upload_ms": round(ms[3], 1),
                        "find_stable_matching_wall_ms": round(ms[4], 1),
                        "end_to_end_ms": round(ms[3] + ms[4], 1),
                        "matching_equal": bool(rc == 0 and np.array_equal(got, want)),
                        "engine_total_ms_first_run": round(sum(runs[0][1][:3]), 3)}
        best_dev = min(r["engine_total_ms"] for r in ref.values())
        best_e2e = min(r["end_to_end_ms"] for r in ref.values())
        records.append({"bamboo_study": f"kind {kind} n={n} seed {seed} param {param}", "n": n, "kind": kind,
                        "seed": seed, "param": param,
                        "reference_smp_engine_bamboo": ref,
                        "ours": {"device_input_ms": round(min(dev_ms), 3), "host_input_e2e_ms": round(min(e2e_ms), 2)},
                        "speedup_vs_best_reference": {
                            "device_input_vs_engine_total": round(best_dev / min(dev_ms), 1),
                            "host_input_e2e_vs_end_to_end": round(best_e2e / min(e2e_ms), 1)}})
        del hpm_t, hpw_t
    return records


def run_bamboo_study(args) -> None:
    """--bamboo-study: bamboo_cases over --bamboo-cases, one JSON line each."""
    import pactae_b200 as pb

    ctx = pb.Context(0)
    cases = [tuple(int(x) for x in c.split(":")) for c in args.bamboo_cases.split(",")]
    for rec in bamboo_cases(ctx, cases):
        print(json.dumps(rec), flush=True)
    ctx.close()


def main():
    args = parse_args()
    if args.init_study:
        run_init_study(args)
        return
    if args.bamboo_study:
        run_bamboo_study(args)
        return
    if args.impl == "reference":
        # Host-only arm: rank 0 times the reference's CPU engine; other ranks
        # exit without work and no process group is needed.
        rank = int(os.environ.get("RANK", "0"))
        if rank == 0:
            res = run_reference(args, Dist.__new__(Dist)._host_only(rank))
            print(json.dumps(res), flush=True)
        return
    dist = Dist(args.gpus)
    try:
        res = run_b200(args, dist)
        if res is not None and dist.rank == 0:
            print(json.dumps(res), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
