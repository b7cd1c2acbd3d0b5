"""Builds libawcpml.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python acousticwavecpml.jl_b200/build.py [--force] [-v]

Each translation unit compiles to an object in parallel (objects under
lib/obj/), then nvcc links the shared library. Output:
acousticwavecpml.jl_b200/lib/libawcpml.so (CUDA runtime linked statically, so
the library loads without a toolkit on the library path).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["csrc/awc_api.cu", "csrc/awc_adjoint.cu", "csrc/awc_batch.cu", "csrc/awc_learned.cu",
           "csrc/awc_static.cu", "csrc/awc_tb.cu"]
HEADERS = ["csrc/awc_kernels.cuh", "csrc/awc_tb.cuh", "csrc/awc_ctx.h", "../include/awcpml.h"]
OUT = os.path.join(HERE, "lib", "libawcpml.so")
OBJ = os.path.join(HERE, "lib", "obj")
FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in deps)


def _compile(src, force, verbose):
    obj = os.path.join(OBJ, os.path.basename(src).replace(".cu", ".o"))
    if not force and not _stale(obj, [src] + HEADERS + ["build.py"]):
        return obj, ""
    cmd = [NVCC, *FLAGS, "-c", "-o", obj, os.path.join(HERE, src)]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src} ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force=False, verbose=False):
    if not force and not _stale(OUT, SOURCES + HEADERS + ["build.py"]):
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        done = list(ex.map(lambda s: _compile(s, force, verbose), SOURCES))
    if verbose:
        for _, log in done:
            print(log)
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", OUT] + [o for o, _ in done]
    r = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
