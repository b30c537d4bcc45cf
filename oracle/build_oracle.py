"""Build the checker: oracle/liboracle.so, and the reference's own build in oracle/_ref/.

TEST INFRASTRUCTURE ONLY: nothing in the product links, loads or calls what
this script builds.  The reference build compiles the reference's sources
where they lie (read-only) with nvcc and a compatibility header
(oracle/ref_compat.h); outputs go only to oracle/_ref/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB = HERE / "liboracle.so"
REF_OUT = HERE / "_ref"
# the reference's source tree: CULDA_REFERENCE_SRC, else a `reference` directory
# beside this repository
REFERENCE = Path(os.environ.get("CULDA_REFERENCE_SRC", str(ROOT.parent / "reference")))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(map(str, cmd)), flush=True)
    r = subprocess.run(list(map(str, cmd)), cwd=ROOT, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"oracle build step failed: {' '.join(map(str, cmd[:4]))} ...")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_oracle_lib(verbose=False, force=False) -> Path:
    srcs = [HERE / "cgs_oracle.cpp", HERE / "cgs_cpu.cpp"]
    srcs = [s for s in srcs if s.exists()]
    if force or _stale(LIB, srcs):
        tmp = LIB.with_suffix(".so.tmp")
        # -ffp-contract=off keeps the FP64 restatement free of fused multiply-adds
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-march=x86-64-v2",
              "-I", ROOT / "include", "-o", tmp, *srcs], verbose)
        os.replace(tmp, LIB)
    return LIB


def _nvcc():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def build_reference(verbose=False, force=False) -> bool:
    """Compile the reference's culda, format tool and the golden-vector harness.

    Returns False (and builds nothing) when the reference sources are absent,
    as on the GPU hosts, where the prebuilt files are used."""
    src = REFERENCE / "src_culda"
    if not (src / "main.cpp").exists():
        return False
    REF_OUT.mkdir(exist_ok=True)
    compat = HERE / "ref_compat.h"
    model = sorted((src / "model").glob("*.cpp"))
    kernels = [src / "kernel" / f for f in ("lda_train_kernel.cu", "lda_phi_kernel.cu", "lda_theta_kernel.cu")]
    common = ["-O3", "-std=c++14", *ARCH, "-include", compat, "-w"]
    deps = model + kernels + [compat, src / "main.cpp", src / "train" / "lda_train.cu"]
    culda = REF_OUT / "culda"
    if force or _stale(culda, deps):
        _run([_nvcc(), *common, "-o", culda, src / "main.cpp", src / "train" / "lda_train.cu", *model, *kernels],
             verbose)
    harness = REF_OUT / "ref_harness"
    hsrc = HERE / "ref_harness.cu"
    if hsrc.exists() and (force or _stale(harness, deps + [hsrc])):
        _run([_nvcc(), *common, "-I", src, "-o", harness, hsrc, *model, *kernels], verbose)
    fmt = REF_OUT / "format"
    fsrc = [REFERENCE / "src_format" / "format.cpp", src / "model" / "vocab.cpp"]
    if force or _stale(fmt, fsrc):
        _run(["g++", "-O2", "-w", "-I", "/usr/local/cuda/include", "-o", fmt, *fsrc], verbose)
    return True


def build(verbose=False, force=False) -> None:
    build_oracle_lib(verbose, force)
    build_reference(verbose, force)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
