"""Build the CUDA library in-tree for sm_100a.

nvcc -gencode arch=compute_100a,code=sm_100a, FP64, --fmad=false so that
every product and sum rounds exactly as in the reference's x86-64 build
(no fused multiply-add contraction). Each .cu file compiles to an object in
parallel; the objects link into dclaw_b200/lib/libdclaw_b200.so.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "lib" / "libdclaw_b200.so"
OBJ = HERE / "lib" / "obj"
SOURCES = [CSRC / "kernels.cu", CSRC / "adjoint.cu"]
HEADERS = list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "dclaw_b200.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in SOURCES + HEADERS + [Path(__file__)])


def _compile(src: Path, verbose: bool) -> Path:
    obj = OBJ / (src.stem + ".o")
    cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return OUT
    OBJ.mkdir(parents=True, exist_ok=True)
    with ThreadPoolExecutor(len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    tmp = str(OUT) + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", *[str(o) for o in objs], "-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
