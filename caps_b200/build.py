"""Builds the device engine: every CUDA source under caps_b200/csrc into caps_b200/libcaps_b200.so for sm_100a.

The library is a plain C ABI (include/caps_gpu.h); it links only the CUDA runtime. nvcc cross-compiles here without a
GPU. The build is skipped when the library is newer than every source.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
LIB = HERE / "libcaps_b200.so"
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    return all(p.stat().st_mtime <= t for p in deps)


def build(force: bool = False, verbose: bool = True) -> Path:
    if not force and up_to_date():
        return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", str(ROOT / "include"), *map(str, sources()), "-o", str(LIB) + ".tmp", "-lcudart"]
    if verbose:
        print("[caps_b200] " + " ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
