"""Regenerate the golden fixtures in tests/golden/.

The reference (victorliu-sq/PACTAE) ships no tests, fixtures or golden
vectors, and its workload generators are unseeded.  The fixtures are made by
running the reference's OWN CPU engines -- src/smp/smp_engine_{gs_1,mw_1,
gs_2,mw_2}.cu compiled from their sources into oracle/_ref/libsmpref.so by
`make -C oracle ref` -- on seeded inputs from the oracle generator, and
requiring every engine that can run at that n to return the same matching.

For each case the fixture records the generator parameters, SHA-256 digests
of both generated preference matrices (which pin the generator), the
matching every reference engine returned, and the proposal count.

Run from the repository root (needs the reference tree to build
oracle/_ref; the fixtures it writes do not):

    python tests/golden/make_golden.py [--quick]
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent

U, C, R, P, RC, G, S = (oracle.GEN_UNIFORM, oracle.GEN_CONGESTED, oracle.GEN_CORRELATED, oracle.GEN_PERFECT,
                        oracle.GEN_REF_CONGESTED, oracle.GEN_GROUPED, oracle.GEN_SOLO)

# (name, kind, n, seed, salt, param)
CASES = [
    ("uniform_n1", U, 1, 11, 0, 0),
    ("uniform_n2", U, 2, 12, 0, 0),
    ("uniform_n3", U, 3, 13, 0, 0),
    ("uniform_n5", U, 5, 14, 0, 0),
    ("uniform_n16", U, 16, 15, 0, 0),
    ("uniform_n31", U, 31, 16, 0, 0),
    ("uniform_n32", U, 32, 17, 0, 0),
    ("uniform_n33", U, 33, 18, 0, 0),
    ("uniform_n100", U, 100, 19, 0, 0),
    ("uniform_n257", U, 257, 20, 0, 0),
    ("uniform_n1000_salt7", U, 1000, 21, 7, 0),
    ("uniform_n2000", U, 2000, 1, 0, 0),              # the n=2000 CPU configuration
    ("congested_n64", C, 64, 3, 0, 0),
    ("congested_n500", C, 500, 3, 0, 0),
    ("congested_n2000", C, 2000, 3, 0, 0),
    ("correlated_n64", R, 64, 4, 0, 500),
    ("correlated_n500", R, 500, 4, 0, 500),
    ("correlated_n2000", R, 2000, 4, 0, 500),
    ("perfect_n64", P, 64, 5, 0, 0),
    ("perfect_n1000", P, 1000, 5, 0, 0),
    ("refcongested_n200", RC, 200, 6, 0, 0),
    ("grouped5_n300", G, 300, 7, 0, 5),
    ("grouped50_n1000", G, 1000, 7, 0, 50),
    ("solo_n3", S, 3, 8, 0, 0),
    ("solo_n100", S, 100, 8, 0, 0),
    ("solo_n1000", S, 1000, 8, 0, 0),
]
FULL_CASES = [
    ("uniform_n30000", U, 30000, 2, 0, 0),            # single-instance GPU configuration
    ("congested_n30000", C, 30000, 3, 0, 0),          # contention stress (a)
    ("correlated_n30000", R, 30000, 4, 0, 500),       # contention stress (b), sigma = 0.05
]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()


def make_case(name, kind, n, seed, salt, param) -> dict:
    t0 = time.time()
    pm, pw = oracle.generate(kind, n, seed, salt, param)
    t_gen = time.time() - t0
    results = {}
    for eng, ename in oracle.REF_ENGINES.items():
        if not oracle.ref_engine_safe(eng, n):
            continue
        match, ms = oracle.ref_solve(eng, pm, pw)
        results[ename] = (match, ms)
    names = list(results)
    base = results[names[0]][0]
    for ename in names[1:]:
        if not np.array_equal(results[ename][0], base):
            raise SystemExit(f"{name}: reference engines disagree ({names[0]} vs {ename})")
    blocking, props = oracle.check(pm, pw, base)
    if blocking != 0:
        raise SystemExit(f"{name}: reference matching has {blocking} blocking pairs")
    np.save(OUT / f"match_{name}.npy", base.astype(np.int32))
    rec = {
        "name": name, "kind": kind, "n": n, "seed": seed, "salt": salt, "param": param,
        "sha256_pref_m": digest(pm), "sha256_pref_w": digest(pw),
        "sha256_match": digest(base), "proposals": props,
        "reference_engines": names,
        "reference_ms": {e: [round(x, 3) for x in results[e][1]] for e in names},
    }
    if n <= 16:  # tiny cases keep their inputs, readable in the json
        rec["pref_m"] = pm.tolist()
        rec["pref_w"] = pw.tolist()
    print(f"{name}: n={n} gen {t_gen:.1f}s, engines {names}, proposals {props}", flush=True)
    return rec


def main() -> None:
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libsmpref.so is missing: run `make -C oracle ref` first")
    cases = CASES if "--quick" in sys.argv else CASES + FULL_CASES
    recs = [make_case(*c) for c in cases]
    meta = {
        "generated_by": "tests/golden/make_golden.py",
        "reference_threads": oracle.ref_threads(),
        "cases": recs,
    }
    (OUT / "cases.json").write_text(json.dumps(meta, indent=1) + "\n")


if __name__ == "__main__":
    main()
