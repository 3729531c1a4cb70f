"""Builds libipcb200.so and libipcb200_direct.so (sm_100a) in-tree with nvcc;
no torch extension machinery.

Each .cu is compiled to an object in parallel, then linked into its shared
library with the CUDA runtime linked statically, so the libraries do not
depend on the runtime version torch ships.  ccd.cu is compiled with
-fmad=false: its root finder must round each operation on its own.  The
direct solver links cuSOLVER/cuSPARSE and lives in its own library so that
the contact pipeline does not depend on them.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libipcb200.so")
DIRECT_LIB_PATH = os.path.join(LIB_DIR, "libipcb200_direct.so")
OBJ_DIR = os.path.join(HERE, "csrc", "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["lbvh.cu", "dcd.cu", "narrow.cu", "ccd.cu", "bsr.cu", "contact_bsr.cu", "fem.cu", "umma_gemm.cu", "mpnn.cu", "pcg.cu",
           "noalloc.cu", "abd.cu", "terms.cu", "linesearch.cu", "alset.cu", "intersect.cu", "mixed.cu"]
NOFMAD = {"ccd.cu"}
DIRECT_SOURCES = ["direct.cu"]
CUDA_LIB = "/usr/local/cuda/lib64"


def _solver_lib_dirs():
    """cuSOLVER/cuSPARSE directories: the copies torch loads (so one process
    never mixes two cuBLAS builds under the same soname), else the toolkit's."""
    dirs = []
    try:
        import nvidia.cusolver
        import nvidia.cusparse

        for m in (nvidia.cusolver, nvidia.cusparse):
            d = os.path.join(list(m.__path__)[0], "lib")
            if os.path.isdir(d):
                dirs.append(d)
    except ImportError:
        pass
    return dirs if len(dirs) == 2 else [CUDA_LIB]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh"))]
    files += [os.path.join(INCLUDE, h) for h in os.listdir(INCLUDE) if h.endswith(".h")]
    return files


def header_hash(header: str = "ipcb.h") -> str:
    """Hash of the C-ABI header the library is compiled against; the loader
    refuses a library whose hash differs from the header next to it."""
    import hashlib

    with open(os.path.join(INCLUDE, header), "rb") as f:
        return hashlib.sha1(f.read()).hexdigest()[:16]


def _compile(nvcc, sources, verbose):
    procs, objs = [], []
    abi = header_hash()
    for src in sources:
        obj = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
               "--expt-relaxed-constexpr", f'-DIPCB_ABI_HASH="{abi}"', "-c", os.path.join(CSRC, src), "-o", obj]
        if src in NOFMAD:
            cmd.insert(1, "-fmad=false")
        if src in DIRECT_SOURCES:
            cmd += ["-Wno-deprecated-declarations", "-Xcompiler", "-Wno-deprecated-declarations"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    return procs, objs


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    newest = max(os.path.getmtime(f) for f in _deps())
    fresh = all(os.path.exists(p) and os.path.getmtime(p) >= newest for p in (LIB_PATH, DIRECT_LIB_PATH))
    if not force and fresh:
        return LIB_PATH
    nvcc = _nvcc()
    procs, objs = _compile(nvcc, SOURCES, verbose)
    dprocs, dobjs = _compile(nvcc, DIRECT_SOURCES, verbose)
    failed = []
    for src, p in procs + dprocs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out)
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    subprocess.run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", LIB_PATH, *objs], check=True)
    libdirs = _solver_lib_dirs()
    link = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", DIRECT_LIB_PATH, *dobjs]
    for d in libdirs:
        link += ["-L", d, "-Xlinker", "-rpath=" + d]
    link += ["-l:libcusolver.so.11", "-l:libcusparse.so.12"]
    subprocess.run(link, check=True)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
