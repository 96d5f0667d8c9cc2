"""The C++ drop-in engine (include/smp_engine_b200.h).

CPU: the standalone driver compiles and links against libsmp_b200.so, and --
when the reference tree is present -- the reference's own executor template
instantiates with SmpEngineB200 derived from the reference's AbsSmpEngine.
GPU: the driver's FindStableMatching result equals smp_b200_solve's and the
checker finds no blocking pair."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("SMP_REFERENCE_DIR", "/root/reference"))
LIBDIR = ROOT / "pactae_b200"


def build_driver(tmp: Path) -> Path:
    exe = tmp / "engine_driver"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "cpp" / "engine_driver.cpp"), "-o", str(exe), f"-L{LIBDIR}", "-lsmp_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_driver_compiles_and_links(tmp_path):
    assert build_driver(tmp_path).exists()


@pytest.mark.skipif(not (REF / "benchmark" / "smp_engine_exec.h").exists(), reason="reference tree not present")
def test_reference_executor_instantiates_engine(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    subprocess.run([nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-c",
                    str(ROOT / "tests" / "cpp" / "reference_executor.cu"), "-o", str(tmp_path / "x.o"),
                    f"-I{ROOT / 'include'}", f"-I{REF / 'include'}", f"-I{REF / 'benchmark'}",
                    f"-I{ROOT / 'oracle' / 'glog_stub'}"], check=True)


@pytest.mark.gpu
@pytest.mark.parametrize("n,kind", [(500, 0), (1200, 1), (3, 6), (800, 3)])
def test_engine_matches_solve_on_gpu(tmp_path, n, kind):
    exe = build_driver(tmp_path)
    out = subprocess.run([str(exe), str(n), str(kind)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ENGINE_OK" in out.stdout
    assert "B200-GS Core Time:" in out.stdout or kind == 3  # PERFECT skips init/core like the reference
