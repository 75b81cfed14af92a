"""Builds the CUDA gridder library in-tree: yandasoft_b200/libyg_b200.so.

nvcc cross-compiles for sm_100a only (no GPU needed).  Objects go to
yandasoft_b200/_build/, the shared library next to this file so that it
travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libyg_b200.so")
BUILD = os.path.join(HERE, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["yg_gridding.cu", "yg_cf.cu", "yg_image.cu", "yg_gridder.cu", "yg_capi.cu", "yg_spheroidal.cpp",
           "yg_noalloc.cu", "yg_learned.cu", "yg_cycle.cu",
           "yg_autotune.cu", "yg_sort.cu"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(HERE, "..", "include")]


def _newer(src, obj):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "yg.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src):
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if not _newer(path, obj):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + FLAGS + ["-x", "c++", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr + r.stdout
    return obj, None


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        results = list(ex.map(_compile, SOURCES))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + [
            "-L" + os.path.join(CUDA, "lib64"), "-lcufft", "-lcudart",
            "-Xlinker", "-rpath," + os.path.join(CUDA, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr + r.stdout)
    if verbose:
        print(OUT)
    return OUT


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
