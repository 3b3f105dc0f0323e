"""Build libmbc.so in-tree: host C++ with g++, CUDA for sm_100a with nvcc.

    python -m fastmbcui_b200.build          # incremental
    python -m fastmbcui_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
OBJ = os.path.join(ROOT, "_build", "mbc")
LIB = os.path.join(PKG, "libmbc.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX_FLAGS = ["-O3", "-fPIC", "-fopenmp", "-ffp-contract=off", "-std=c++17", "-Wall",
             "-Wno-unknown-pragmas", f"-I{INC}", f"-I{CSRC}"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off", f"-I{INC}", f"-I{CSRC}",
                     "-Xptxas", "-warn-spills"]

HOST_SRC = ["plan.cpp", "capi.cpp", "spatial.cpp"]
CUDA_SRC = ["solver.cu", "context.cu", "noalloc.cu", "mlp.cu", "warmstart.cu", "mesh.cu", "int8_ops.cu", "grad.cu"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _headers():
    out = [os.path.join(INC, "mbc.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".h", ".cuh")):
            out.append(os.path.join(CSRC, f))
    return out


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_nvcc=()) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    jobs = []
    objs = []
    for src in HOST_SRC + CUDA_SRC:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs):
            if src.endswith(".cu"):
                cmd = [nvcc, *NVCC_FLAGS, *extra_nvcc, "-c", path, "-o", obj]
            else:
                cmd = ["g++", *CXX_FLAGS, "-c", path, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=max(1, min(8, len(jobs)))) as ex:
        for err in ex.map(run, jobs):
            if verbose and err:
                print(err)
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
