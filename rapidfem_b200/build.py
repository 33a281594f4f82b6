"""Build the native library ``rapidfem_b200/_lib/librapidfem_b200.so``.

nvcc compiles the CUDA sources for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``); the host C++ sources are compiled by the
same nvcc driver.  The library exports the C ABI of ``include/dgtd.h`` and
``include/dgtd_host.h`` and links only the CUDA runtime (static).

Usage: ``python -m rapidfem_b200.build [--force] [--verbose]``
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "librapidfem_b200.so")
OBJDIR = os.path.join(PKG, "_build")

CU_SOURCES = ["dgtd_capi.cu"]
CPP_SOURCES = ["host/host_op.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _deps():
    files = []
    for d, _, fs in os.walk(CSRC):
        files += [os.path.join(d, f) for f in fs if f.endswith((".cu", ".cuh", ".cpp", ".h"))]
    files += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return files


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
    objs = []
    for src in CU_SOURCES:
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        cmd = [nvcc, *ARCH, "-lineinfo", *common, "-Xptxas", "-v" if verbose else "-O3",
               "-c", os.path.join(CSRC, src), "-o", obj]
        _run(cmd, verbose)
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        cmd = [nvcc, *common, "-Xcompiler", "-fopenmp", "-x", "c++", "-c", os.path.join(CSRC, src), "-o", obj]
        _run(cmd, verbose)
        objs.append(obj)
    tmp = LIB + ".tmp"
    _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lgomp"], verbose)
    os.replace(tmp, LIB)
    return LIB


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
