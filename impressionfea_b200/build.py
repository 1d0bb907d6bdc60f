"""Build of the in-tree CUDA library ``impressionfea_b200/libifea_gpu.so`` for sm_100a.

nvcc compiles every translation unit under ``csrc/`` with ``-gencode arch=compute_100a,code=sm_100a`` and
``--fmad=false`` (the reference's .NET arithmetic does not contract a*b+c). No GPU is needed to build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libifea_gpu.so")
SOURCES = ["solver3d.cu", "solver2d.cu", "spd_capi.cu", "mesh3d.cpp", "mesh2d.cpp", "multifrontal.cpp", "band_noalloc.cu", "mlp.cu", "remesh.cu", "batch.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _deps():
    out = []
    for d in (CSRC, os.path.join(os.path.dirname(HERE), "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".cpp", ".h")):
                out.append(os.path.join(d, f))
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in _deps()):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    jobs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s + ".o")
        cmd = [NVCC] + ARCH + ["-lineinfo", "-O3", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
                               "-Xcompiler", "-Wall", "-Xcompiler", "-Wno-deprecated-declarations", "-diag-suppress", "128", "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        jobs.append((cmd, obj))
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as pool:
        for f in [pool.submit(subprocess.check_call, c) for c, _ in jobs]:
            f.result()
    objs = [o for _, o in jobs]
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcusolver", "-lcusparse", "-lcublas"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
