"""Build the CUDA library in-tree: yuzen_b200/libyuzen_b200.so (sm_100a only).

    python -m yuzen_b200.build          # or build_library() from Python

Every .cu file under csrc/ is compiled by nvcc for sm_100a with -fmad=false
(no fused multiply-add: the FP64 parity path rounds every product and sum as
the reference's host code does under -ffp-contract=off) and linked into one
shared library.  Objects go to yuzen_b200/_build/ (git-ignored).
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libyuzen_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build yuzen_b200")


def _flags(src: Path) -> list[str]:
    flags = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                    "-I", str(HERE.parent / "include"), "-I", str(CSRC)]
    # every kernel of the library keeps products and sums separately rounded
    flags += ["-fmad=false"]
    if os.environ.get("YZ_PTXAS_VERBOSE"):
        flags += ["-Xptxas", "-v"]
    return flags


def _compile(src: Path) -> Path:
    obj = BUILD / (src.stem + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(
            [src.stat().st_mtime] + [p.stat().st_mtime for p in CSRC.glob("*.cuh")]
            + [p.stat().st_mtime for p in CSRC.glob("*.h")]
            + [(HERE.parent / "include" / "yuzen_b200.h").stat().st_mtime]):
        return obj
    cmd = [nvcc_path()] + _flags(src) + ["-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    if res.stderr.strip() and os.environ.get("YZ_PTXAS_VERBOSE"):
        print(res.stderr, file=sys.stderr)
    return obj


def build_library(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(sources))) as ex:
        objs = list(ex.map(_compile, sources))
    newest = max(o.stat().st_mtime for o in objs)
    if LIB.exists() and LIB.stat().st_mtime >= newest:
        return LIB
    cmd = [nvcc_path()] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIB)] + [str(o) for o in objs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build_library(verbose=True)
