"""Builds lib/libdrmppi.so (the control-step kernels and their C ABI) for sm_100a with nvcc.

Each translation unit is compiled to an object under _build/ (in parallel, skipped when
up to date) and the objects are linked into one shared library, in-tree, so that it
ships with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libdrmppi.so"
INCLUDE = PKG.parent / "include"

SOURCES = ["mppi_kernels.cu", "gate_kernels.cu", "gate_pr_kernels.cu", "grad_kernels.cu", "finish_kernels.cu", "track_kernels.cu", "prmppi_kernels.cu", "api.cu", "api_pr.cu", "noalloc.cu", "predict_kernels.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "--expt-relaxed-constexpr", "-diag-suppress", "177,550"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _deps() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.hpp")) + [INCLUDE / "drmppi.h"]


def _compile(src: str, verbose: bool, ptxas_info: bool) -> Path:
    s = CSRC / src
    o = BUILD / (Path(src).stem + ".o")
    newest = max([s.stat().st_mtime] + [d.stat().st_mtime for d in _deps()])
    if o.exists() and o.stat().st_mtime >= newest and not ptxas_info:
        return o
    cmd = [nvcc(), *FLAGS, "-c", str(s), "-o", str(o)]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if ptxas_info:
        (BUILD / (Path(src).stem + ".ptxas.txt")).write_text(r.stderr)
    return o


def build(verbose: bool = False, ptxas_info: bool = False, jobs: int = 4) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, ptxas_info), SOURCES))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
