"""Build the in-tree shared libraries.

- `librcsr_b200.so`: the CUDA C-ABI library (csrc/*.cu), compiled for sm_100a
  only, one object per translation unit in parallel, then linked.
- `librcsr_host.so`: the host-side compiler (host/rcsr_host.cpp) and the
  exact f64 finalist refit (host/refit.cpp).

Run `python the-rule-and-compass_b200/build.py` or call `build()`.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
CUDA_LIB = os.path.join(HERE, "librcsr_b200.so")
HOST_LIB = os.path.join(HERE, "librcsr_host.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE,
              "-I" + CSRC]
SOURCES = ["ctx.cu", "score.cu", "fit.cu", "rank.cu", "vary.cu", "multi.cu"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "rcsr_b200.h"))
    return hs


def _compile(src, verbose_ptxas=False):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    srcp = os.path.join(CSRC, src)
    if not _stale(obj, [srcp] + _headers()) and not verbose_ptxas:
        return obj, ""
    cmd = [NVCC, *ARCH, *NVCC_FLAGS, "-c", srcp, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build_cuda(verbose_ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    objs = [o for o, _ in results]
    if verbose_ptxas:
        for (o, log), s in zip(results, SOURCES):
            sys.stderr.write(f"== {s}\n{log}")
    if _stale(CUDA_LIB, objs) or verbose_ptxas:
        cmd = [NVCC, *ARCH, "-shared", "-o", CUDA_LIB, *objs, "-lcudart"]
        subprocess.run(cmd, check=True)
    return CUDA_LIB


def build_host():
    """The host library: the compiler (rcsr_host.cpp) and the exact f64
    finalist refit (refit.cpp). -ffp-contract=off keeps every f64 operation
    a separately rounded IEEE operation, which the refit's bit-identity with
    the reference's CPU path relies on."""
    srcs = [os.path.join(HERE, "host", f) for f in ("rcsr_host.cpp", "refit.cpp")]
    deps = srcs + [os.path.join(INCLUDE, "rcsr_refit.h"), os.path.join(INCLUDE, "rcsr_host.h")]
    if _stale(HOST_LIB, deps):
        cmd = ["g++", "-O3", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-pthread",
               "-fopenmp", "-Wall", "-I" + INCLUDE, "-o", HOST_LIB, *srcs]
        subprocess.run(cmd, check=True)
    return HOST_LIB


def build(verbose_ptxas=False):
    build_host()
    build_cuda(verbose_ptxas)


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
    print(CUDA_LIB)
    print(HOST_LIB)
