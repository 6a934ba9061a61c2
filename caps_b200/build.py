"""Builds the device engine: every CUDA source under caps_b200/csrc into caps_b200/libcaps_b200.so for sm_100a.

The library is a plain C ABI (include/caps_gpu.h); it links only the CUDA runtime. nvcc cross-compiles here without a
GPU. The build is skipped when the library is newer than every source.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
LIB = HERE / "libcaps_b200.so"
OBJ = HERE / "_build"
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
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
    """Compiles each translation unit in parallel into caps_b200/_build/, then links the shared library."""
    if not force and up_to_date():
        return LIB
    OBJ.mkdir(exist_ok=True)
    objs = [OBJ / (src.stem + ".o") for src in sources()]
    cmds = [[_nvcc(), *NVCC_FLAGS, "-c", "-I", str(ROOT / "include"), str(src), "-o", str(obj)] for src, obj in zip(sources(), objs)]
    if verbose:
        print("[caps_b200] " + " ".join(cmds[0][:-4]) + " -c <each csrc/*.cu>", file=sys.stderr)
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        results = list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for c, r in zip(cmds, results):
        if r.stderr and verbose:
            print(r.stderr, file=sys.stderr, end="")
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, c, r.stdout, r.stderr)
    subprocess.run([_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *map(str, objs), "-o", str(LIB) + ".tmp", "-lcudart"], check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
