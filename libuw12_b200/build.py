"""Builds the CUDA extension in-tree: libuw12_b200/_lib/libuw12_b200.so (sm_100a).

Usage: ``python -m libuw12_b200.build [--force]``.  Sources are compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked
against cuSOLVER (metric / overlap eigensolves) and the CUDA runtime.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT_DIR = HERE / "_lib"
LIB = OUT_DIR / "libuw12_b200.so"
SOURCES = ["gemm_f64.cu", "ozaki.cu", "kernels.cu", "engine.cu", "synth.cu", "capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _flags() -> list:
    return ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-Wall", "--expt-relaxed-constexpr"]


def _deps(src: Path) -> list:
    return [src] + sorted(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "uw12_c.h"]


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    objs = []
    jobs = []
    for name in SOURCES:
        src = CSRC / name
        obj = OUT_DIR / (name + ".o")
        objs.append(obj)
        newest = max(p.stat().st_mtime for p in _deps(src) if p.exists())
        if force or not obj.exists() or obj.stat().st_mtime < newest:
            jobs.append([_nvcc(), *_flags(), "-c", str(src), "-o", str(obj)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    newest_obj = max(o.stat().st_mtime for o in objs)
    if force or jobs or not LIB.exists() or LIB.stat().st_mtime < newest_obj:
        run([_nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
             "-lcusolver", "-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
