"""The C ABI library on the CPU: it loads, exports exactly what
include/smp_b200.h declares, its header compiles as C and C++, and calls
that need no GPU behave (no compute runs here)."""
from __future__ import annotations

import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import pytest

import pactae_b200 as pb
from pactae_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "smp_b200.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    return set(re.findall(r"SMP_B200_API\s+[\w\s\*]*?\b(smp_b200_\w+)\s*\(", text))


def exported_symbols() -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_symbol():
    declared = declared_symbols()
    assert declared, "no declarations parsed from the header"
    assert declared == set(_lib.ABI_SYMBOLS)
    exported = exported_symbols()
    assert declared <= exported
    # nothing but the ABI leaks out of the shared object
    assert {s for s in exported if not s.startswith("smp_b200_")} == set()
    for name in declared:
        assert hasattr(_lib.lib, name)


def test_library_is_built_for_sm100a():
    # The build recipe compiles for sm_100a only.
    from conftest import load_build_recipe

    pbuild = load_build_recipe()
    assert pbuild.ARCH_FLAGS == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert _lib.LIB_PATH.exists()


@pytest.mark.parametrize("lang,compiler", [("c", "gcc"), ("c++", "g++")])
def test_header_compiles(tmp_path, lang, compiler):
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} missing")
    src = tmp_path / ("t.c" if lang == "c" else "t.cpp")
    src.write_text('#include "smp_b200.h"\nint main(void){ smp_ctx *c = 0; (void)c; return SMP_OK; }\n')
    subprocess.run(["/usr/bin/" + compiler, "-std=c11" if lang == "c" else "-std=c++17", "-Wall", "-Werror",
                    f"-I{ROOT / 'include'}", "-fsyntax-only", str(src)], check=True)


def test_struct_layouts_match_header(tmp_path):
    # sizeof / offsetof of the ABI structs, compiled from the header, equal
    # the ctypes mirrors the Python binding uses.
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "smp_b200.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu\\n\", sizeof(smp_cfg), sizeof(smp_stats),"
        " offsetof(smp_stats, stage_ms), offsetof(smp_stats, total_ms), offsetof(smp_cfg, hbm_budget));"
        " return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["/usr/bin/gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.smp_cfg), ctypes.sizeof(_lib.smp_stats), _lib.smp_stats.stage_ms.offset,
            _lib.smp_stats.total_ms.offset, _lib.smp_cfg.hbm_budget.offset]
    assert got == want


def test_strerror_and_version():
    assert pb.version().startswith("smp_b200")
    for status in range(9):
        assert _lib.lib.smp_b200_strerror(status)
    assert b"unknown" in _lib.lib.smp_b200_strerror(1234)


def test_null_arguments_are_rejected_without_a_gpu():
    assert _lib.lib.smp_b200_create(None, None) == pb.SMP_ERR_INVALID_ARG
    assert _lib.lib.smp_b200_solve(None, None, None, 10, None, 0, None) == pb.SMP_ERR_INVALID_ARG
    assert _lib.lib.smp_b200_stage(None, None, None, 10, 0) == pb.SMP_ERR_INVALID_ARG
    _lib.lib.smp_b200_destroy(None)  # no-op


def test_create_fails_cleanly_without_a_device(cuda_available):
    if cuda_available:
        pytest.skip("a CUDA device is present")
    with pytest.raises(pb.SmpError) as e:
        pb.Context(device=0)
    assert e.value.status == pb.SMP_ERR_CUDA


def test_constants_match_header():
    text = HEADER.read_text()
    for name in ("SMP_F_DEVICE_PTRS", "SMP_F_CHECK", "SMP_F_VALIDATE", "SMP_F_NO_PRECHECK", "SMP_GEN_UNIFORM",
                 "SMP_GEN_CONGESTED", "SMP_GEN_CORRELATED", "SMP_GEN_PERFECT", "SMP_GEN_REF_CONGESTED",
                 "SMP_GEN_GROUPED", "SMP_GEN_SOLO", "SMP_B200_MAX_N"):
        m = re.search(rf"#define {name} (0x[0-9a-fA-F]+|\d+)", text)
        assert m, name
        assert int(m.group(1).rstrip("u"), 0) == getattr(_lib, name)
    for name in ("SMP_OK", "SMP_ERR_INVALID_ARG", "SMP_ERR_INVALID_INPUT", "SMP_ERR_OOM", "SMP_ERR_CUDA",
                 "SMP_ERR_TIMEOUT", "SMP_ERR_BUSY", "SMP_ERR_NOT_READY", "SMP_ERR_UNSUPPORTED"):
        m = re.search(rf"{name} = (\d+)", text)
        assert m and int(m.group(1)) == getattr(_lib, name)


def test_oracle_generator_and_product_constants_agree():
    import oracle

    assert (oracle.GEN_UNIFORM, oracle.GEN_CONGESTED, oracle.GEN_CORRELATED, oracle.GEN_PERFECT,
            oracle.GEN_REF_CONGESTED, oracle.GEN_GROUPED, oracle.GEN_SOLO) == (
        pb.SMP_GEN_UNIFORM, pb.SMP_GEN_CONGESTED, pb.SMP_GEN_CORRELATED, pb.SMP_GEN_PERFECT,
        pb.SMP_GEN_REF_CONGESTED, pb.SMP_GEN_GROUPED, pb.SMP_GEN_SOLO)


def test_batch_recipe_matches_oracle():
    # host-only entry point: the size/kind recipe of a seeded batch mix
    import oracle

    for b in range(3000):
        assert pb.batch_instance(5, b, 16, 4096) == oracle.batch_instance(5, b, 16, 4096)
        assert pb.batch_instance(6, b, 64, 16384) == oracle.batch_instance(6, b, 64, 16384)
