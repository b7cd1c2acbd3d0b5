"""Builds libawcpml.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python acousticwavecpml.jl_b200/build.py

Output: acousticwavecpml.jl_b200/lib/libawcpml.so (CUDA runtime linked
statically, so the library loads without a toolkit on the library path).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["csrc/awc_api.cu", "csrc/awc_adjoint.cu", "csrc/awc_batch.cu", "csrc/awc_learned.cu", "csrc/awc_static.cu"]
HEADERS = ["csrc/awc_kernels.cuh", "csrc/awc_ctx.h", "../include/awcpml.h"]
OUT = os.path.join(HERE, "lib", "libawcpml.so")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale(OUT, SOURCES + HEADERS + ["build.py"]):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-Wall", "-shared", "-cudart", "static", "-o", OUT]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(HERE, s) for s in SOURCES]
    r = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
