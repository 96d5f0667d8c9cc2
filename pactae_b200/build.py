"""Build recipe for libsmp_b200.so (sm_100a) and the CPU oracle.

``python pactae_b200/build.py`` compiles the CUDA sources in
``pactae_b200/csrc`` with nvcc straight into ``pactae_b200/libsmp_b200.so``
(in-tree, so the built library travels with the working tree).  Every source
is compiled for ``sm_100a`` only.  A rebuild happens only when a source or
header is newer than the library.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libsmp_b200.so"
BUILD_DIR = PKG / "_build"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
]

SOURCES = ["smp_b200.cu", "generate.cu", "batch.cu", "serve.cu", "static_solve.cu", "workload_io.cpp", "host_pack.cpp"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libsmp_b200.so")
    return cand


def _inputs() -> list[Path]:
    files = [p for p in CSRC.iterdir() if p.suffix in (".cu", ".cuh", ".h", ".cpp")]
    files += [p for p in INCLUDE.iterdir() if p.suffix == ".h"]
    files.append(Path(__file__))
    return files


def needs_build() -> bool:
    if not LIB.exists():
        return True
    mtime = LIB.stat().st_mtime
    return any(p.stat().st_mtime > mtime for p in _inputs())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile libsmp_b200.so if needed and return its path."""
    if not force and not needs_build() and not ptxas_info:
        return LIB
    nvcc = _nvcc()
    BUILD_DIR.mkdir(exist_ok=True)
    objs, cmds = [], []
    for src in SOURCES:
        obj = BUILD_DIR / (Path(src).stem + ".o")
        cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(CSRC / src), "-o", str(obj)]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        cmds.append(cmd)
        objs.append(str(obj))
    # the translation units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for r in pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *objs, "-Xcompiler", "-fPIC"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


def build_oracle(verbose: bool = False) -> None:
    """Compile the CPU oracle (test infrastructure) and, when the reference
    sources are present, the reference's own CPU engines and the GPU engines
    the studies time beside this library."""
    oracle = ROOT / "oracle"
    targets = ["all"]
    ref = os.environ.get("SMP_REFERENCE_DIR")
    if not ref:  # the recipe's own default location of the reference tree
        ref = subprocess.run(["make", "-s", "-C", str(oracle), "print-ref"], check=True, capture_output=True,
                             text=True).stdout.strip()
    ref = Path(ref)
    if (ref / "src" / "smp" / "smp_engine_gs_1.cu").exists():
        targets.append("ref")
    if (ref / "include" / "smp" / "smp_init_3.h").exists():
        targets.append("ref-gpu")
    if (ref / "src" / "smp" / "smp_engine_bamboo.cu").exists():
        targets.append("ref-bamboo")
    if (ref / "benchmark" / "smp_engine_exec.h").exists() and LIB.exists():
        targets.append("ref-exec")
    cmd = ["make", "-s", "-C", str(oracle), *targets, f"REF={ref}"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


if __name__ == "__main__":
    force = "--force" in sys.argv
    info = "--ptxas-info" in sys.argv
    print(build(force=force, verbose=True, ptxas_info=info))
    if "--oracle" in sys.argv:
        build_oracle(verbose=True)
