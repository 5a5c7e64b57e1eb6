"""Build recipe of the engine library (sm_100a) and the command-line program.

    python -m dsmc_erlend_b200.build          # lib/libdsmc_b200.so, lib/dsmc and
                                              # lib/libdsmc_surrogate.so

The CUDA sources are compiled for sm_100a only, with --fmad=false (no
contraction of a*b+c, so FP64 arithmetic is the reference's operation
sequence) and the host sources with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libdsmc_b200.so"
CLI = LIB_DIR / "dsmc"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler",
              "-fPIC,-ffp-contract=off,-O2", "-I", str(ROOT / "include")]

LIB_SOURCES = ["dsmc_capi.cu", "host_api.cpp", "surface.cpp"]
DEPENDS = ["dsmc_device.cuh", "dsmc_scan.cuh", "dsmc_kernels.cuh", "dsmc_bulk.cuh",
           "dsmc_units.cuh", "dsmc_persist.cuh"]

# The surrogate's kernels: ordinary FP32 contraction is fine there (a neural
# network, not the reference's arithmetic).
SG_LIB = LIB_DIR / "libdsmc_surrogate.so"
SG_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-I",
            str(ROOT / "include")]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build(force: bool = False, verbose: bool = False) -> Path:
    LIB_DIR.mkdir(exist_ok=True)
    srcs = [CSRC / s for s in LIB_SOURCES if (CSRC / s).exists()]
    deps = srcs + [CSRC / d for d in DEPENDS] + [ROOT / "include" / "dsmc.h",
                                                 ROOT / "include" / "dsmc_philox.h"]
    if force or _stale(LIB, deps):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-shared", "-o", str(LIB), *map(str, srcs)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    sg = CSRC / "surrogate.cu"
    if sg.exists() and (force or _stale(SG_LIB, [sg, ROOT / "include" / "dsmc_surrogate.h"])):
        cmd = [nvcc(), *ARCH, *SG_FLAGS, "-shared", "-o", str(SG_LIB), str(sg)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    main = CSRC / "main.cpp"
    if main.exists() and (force or _stale(CLI, [main, LIB])):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-o", str(CLI), str(main), "-L", str(LIB_DIR),
               "-ldsmc_b200", "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
