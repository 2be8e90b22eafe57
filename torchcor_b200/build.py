"""Build ``libtcb200.so`` in-tree: nvcc for sm_100a (CUDA sources) and g++
(host pattern builder), linked into one shared library next to this file.

    python -m torchcor_b200.build [--force]

Object files go to ``torchcor_b200/_build/``; the library is rebuilt when any
source or header is newer than it.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libtcb200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# translation units that must keep float32 expressions as separate roundings (the
# lookup-table builders: their grids pass through removable singularities)
NO_FMA = {"tables.cu"}


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libtcb200.so")
    return cand


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def _compile(src: Path, verbose: bool):
    obj = BUILD / (src.name + ".o")
    if src.suffix == ".cu":
        cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
               "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if src.name in NO_FMA:
            cmd.insert(1, "-fmad=false")
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", "-O3", "-fPIC", "-fopenmp", "-std=c++17", "-I", str(INCLUDE), "-I", str(CSRC),
               "-I", "/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every source for sm_100a and link ``libtcb200.so``; returns its path."""
    if not force and not _stale():
        return LIB
    BUILD.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), sources()))
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    objs = [str(o) for o, _ in results]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-Xcompiler", "-fopenmp", "-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill reports")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
