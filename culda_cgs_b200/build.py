"""Build recipe for the sm_100a library, the `culda` command and the checkers.

Everything is built in-tree with nvcc/g++ (no JIT cache), so the shared
objects and binaries travel with the source tree:

    culda_cgs_b200/libculda_b200.so   CUDA kernels + C ABI (include/culda_b200.h)
    culda_cgs_b200/bin/culda          C++ host with the reference's CLI
    culda_cgs_b200/bin/format         C++ host with the reference's preprocessing tool
    culda_cgs_b200/bin/gencorpus      C++ host writing a seeded synthetic corpus in the src_format files
    oracle/liboracle.so               host FP64 oracle + OpenMP CPU baseline (tests/bench only)
    oracle/_ref/...                   the reference's own build (only where its sources exist)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "culda_cgs_b200"
CSRC = PKG / "csrc"
LIB = PKG / "libculda_b200.so"
CLI = PKG / "bin" / "culda"
FORMAT_CLI = PKG / "bin" / "format"
GEN_CLI = PKG / "bin" / "gencorpus"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# portable host ISA: the library is built here and run on the GPU hosts
HOST_ARCH = "-march=x86-64-v2"


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def library_sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def build_library(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    srcs = library_sources()
    deps = srcs + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "culda_b200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-shared",
           "-Xcompiler", f"-fPIC,-fopenmp,{HOST_ARCH},-fvisibility=hidden",
           "-I", str(ROOT / "include"),
           "-o", str(tmp), *map(str, srcs), "-lgomp"]
    if ptxas_info:
        cmd.insert(1, "-Xptxas=-v")
    _run(cmd, verbose)
    os.replace(tmp, LIB)
    return LIB


def _build_host_tool(src: Path, exe: Path, verbose: bool, force: bool) -> Path:
    if not src.exists():
        return exe
    if not force and not _stale(exe, [src, LIB, ROOT / "include" / "culda_b200.h"]):
        return exe
    exe.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", HOST_ARCH, "-I", str(ROOT / "include"), "-o", str(exe), str(src),
           "-L", str(PKG), "-lculda_b200", "-Wl,-rpath,$ORIGIN/.."]
    _run(cmd, verbose)
    return exe


def build_cli(verbose: bool = False, force: bool = False) -> Path:
    return _build_host_tool(CSRC / "cli" / "culda_main.cpp", CLI, verbose, force)


def build_format_cli(verbose: bool = False, force: bool = False) -> Path:
    return _build_host_tool(CSRC / "cli" / "format_main.cpp", FORMAT_CLI, verbose, force)


def build_gencorpus_cli(verbose: bool = False, force: bool = False) -> Path:
    return _build_host_tool(CSRC / "cli" / "gencorpus_main.cpp", GEN_CLI, verbose, force)


def build_all(verbose: bool = False, force: bool = False) -> None:
    build_library(verbose, force)
    build_cli(verbose, force)
    build_format_cli(verbose, force)
    build_gencorpus_cli(verbose, force)
    sys.path.insert(0, str(ROOT))
    from oracle import build_oracle  # the checker is built beside the product, never linked into it

    build_oracle.build(verbose=verbose, force=force)


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv, force="-f" in sys.argv)
