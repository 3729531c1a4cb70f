"""Builds libipcb200.so (sm_100a) in-tree with nvcc; no torch extension machinery.

Each .cu is compiled to an object in parallel, then linked into one shared
library with the CUDA runtime linked statically, so the library does not
depend on the runtime version torch ships.  ccd.cu is compiled with
-fmad=false: its root finder must round each operation on its own.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libipcb200.so")
OBJ_DIR = os.path.join(HERE, "csrc", "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["lbvh.cu", "dcd.cu", "narrow.cu", "ccd.cu", "bsr.cu", "contact_bsr.cu", "fem.cu", "noalloc.cu"]
NOFMAD = {"ccd.cu"}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh"))]
    files.append(os.path.join(INCLUDE, "ipcb.h"))
    return files


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    newest = max(os.path.getmtime(f) for f in _deps())
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= newest:
        return LIB_PATH
    nvcc = _nvcc()
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
               "--expt-relaxed-constexpr", "-c", os.path.join(CSRC, src), "-o", obj]
        if src in NOFMAD:
            cmd.insert(1, "-fmad=false")
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out)
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    link = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", LIB_PATH, *objs]
    subprocess.run(link, check=True)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
