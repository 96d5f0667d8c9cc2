"""The reference's workload text cache (generate_workloads_flat.h:283-376),
read and written by the library on the host: byte-identical to the
reference's own SaveSmpWorkload, readable by its LoadSmpWorkload and back,
the same file names, and errors for short, malformed or missing files."""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

import oracle
import pactae_b200 as pb
from pactae_b200 import _lib

# WorkloadType of the reference (include/utils/types.h:85-90) for our kinds
REF_TYPE = {pb.SMP_GEN_PERFECT: 0, pb.SMP_GEN_GROUPED: 1, pb.SMP_GEN_REF_CONGESTED: 2, pb.SMP_GEN_SOLO: 3}


def lists(n: int, seed: int):
    return oracle.generate(pb.SMP_GEN_UNIFORM, n, seed)


def test_round_trip(tmp_path):
    pm, pw = lists(57, 1)
    path = tmp_path / "w.txt"
    pb.write_workload(path, pm, pw)
    got_m, got_w = pb.read_workload(path)
    assert np.array_equal(got_m, pm) and np.array_equal(got_w, pw)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference engines not built")
@pytest.mark.parametrize("n", [1, 33, 700])
def test_same_bytes_as_the_reference_and_readable_both_ways(tmp_path, monkeypatch, n):
    monkeypatch.chdir(tmp_path)
    (tmp_path / "data" / "workloads").mkdir(parents=True)
    pm, pw = lists(n, 2)
    oracle.ref_workload_save("ref.txt", pm, pw)
    ours = tmp_path / "data" / "workloads" / "ours.txt"
    pb.write_workload(ours, pm, pw)
    assert ours.read_bytes() == (tmp_path / "data" / "workloads" / "ref.txt").read_bytes()
    m2, w2 = pb.read_workload(tmp_path / "data" / "workloads" / "ref.txt")
    assert np.array_equal(m2, pm) and np.array_equal(w2, pw)
    m3, w3 = oracle.ref_workload_load("ours.txt", n)
    assert np.array_equal(m3, pm) and np.array_equal(w3, pw)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference engines not built")
@pytest.mark.parametrize("kind", sorted(REF_TYPE))
def test_file_names_match_the_reference(kind):
    for n, g in [(2000, 5), (30000, 7)]:
        assert pb.workload_filename(kind, n, g) == oracle.ref_workload_filename(REF_TYPE[kind], n, g)


def test_many_threads_on_a_larger_file(tmp_path):
    pm, pw = lists(1500, 3)  # ~20 MB of text: one line range per host thread
    path = tmp_path / "big.txt"
    pb.write_workload(path, pm, pw)
    got_m, got_w = pb.read_workload(path)
    assert np.array_equal(got_m, pm) and np.array_equal(got_w, pw)


def test_any_whitespace_layout_is_read(tmp_path):
    # the reference's reader only needs whitespace between values
    pm, pw = lists(20, 4)
    path = tmp_path / "one_line.txt"
    path.write_text(f"{20}\n" + "\t".join(map(str, np.concatenate([pm.ravel(), pw.ravel()]))) + "\n")
    got_m, got_w = pb.read_workload(path)
    assert np.array_equal(got_m, pm) and np.array_equal(got_w, pw)


def _read_status(path, n):
    buf = np.empty(2 * n * n, np.int32)
    return _lib.lib.smp_b200_workload_read(os.fsencode(path), n, ctypes.c_void_p(buf.ctypes.data),
                                           ctypes.c_void_p(buf.ctypes.data + 4 * n * n))


def test_short_malformed_and_missing_files(tmp_path):
    pm, pw = lists(10, 5)
    good = tmp_path / "good.txt"
    pb.write_workload(good, pm, pw)
    text = good.read_text()
    short = tmp_path / "short.txt"
    short.write_text(text[: len(text) // 2])
    assert _read_status(short, 10) == pb.SMP_ERR_INVALID_INPUT
    bad = tmp_path / "bad.txt"
    bad.write_text(text.replace(" ", " x ", 1))
    assert _read_status(bad, 10) == pb.SMP_ERR_INVALID_INPUT
    assert _read_status(good, 11) == pb.SMP_ERR_INVALID_INPUT  # the header says 10
    assert _read_status(tmp_path / "missing.txt", 10) == pb.SMP_ERR_IO
    with pytest.raises(pb.SmpError):
        pb.read_workload(tmp_path / "missing.txt")
