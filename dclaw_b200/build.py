"""Build the CUDA library in-tree for sm_100a.

nvcc -gencode arch=compute_100a,code=sm_100a, FP64, --fmad=false so that
every product and sum rounds exactly as in the reference's x86-64 build
(no fused multiply-add contraction).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "lib" / "libdclaw_b200.so"
SOURCES = [CSRC / "kernels.cu"]
HEADERS = list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "dclaw_b200.h"]

NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "--fmad=false", "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = str(OUT) + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, *[str(s) for s in SOURCES], "-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
