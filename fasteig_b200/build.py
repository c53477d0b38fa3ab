"""Build the in-tree CUDA library ``fasteig_b200/libfasteig_b200.so`` for sm_100a.

Usage: ``python -m fasteig_b200.build`` (or ``__graft_entry__.build()``).
Each translation unit is compiled separately (objects under ``_build/``) and
re-compiled only when it or a header changed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = ROOT / "_build"
LIB = HERE / "libfasteig_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
SOURCES = ["spmm.cu", "blocks.cu", "dmma.cu", "dense.cu", "tc_gemm.cu", "batch_ks.cu",
           "lanczos.cu", "ingest.cu", "syevd.cu", "group_kernels.cu", "solver.cpp", "grouped.cpp",
           "server.cpp"]
LIBS: list = []


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + [ROOT / "include" / "fasteig_b200.h"]


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdr_mtime = max(p.stat().st_mtime for p in _headers())
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if not force and o.exists() and o.stat().st_mtime >= max(s.stat().st_mtime, hdr_mtime):
            continue
        lang = ["-x", "cu"] if s.suffix == ".cu" else []
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"), *lang, "-c", str(s),
               "-o", str(o)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose and (r.stdout or r.stderr):
            sys.stderr.write(r.stdout + r.stderr)
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), *LIBS]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link failed")
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
