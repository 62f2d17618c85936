"""Build libmaxlq_b200.so in-tree with nvcc for sm_100a.

    python -m maxlq_b200.build [--force] [--verbose]

The shared library is the product: the C ABI of include/maxlq.h.  It links
the CUDA runtime statically so it loads on any box of this image without a
library path.  Only sm_100a code is generated (B200).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmaxlq_b200.so")
SOURCES = ["engine.cu", "engine_f32.cu", "engine_f64.cu", "solver.cu", "capi.cu", "noalloc.cu", "diag.cu", "lsdev.cu",
           "ncdf.cpp", "kappa.cpp"]
HEADERS = ["common.cuh", "fft.cuh", "kernels.cuh", "functors.cuh", "regfft.cuh", "cfft.cuh", "engine.cuh",
           "engine_common.cuh", "engine_impl.cuh", "solver.cuh", "linesearch.cuh"]
# the device line search rounds every step as the host search does
EXTRA_FLAGS = {"lsdev.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # the system g++ (the environment's CXX wrapper may lack runtime specs)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "maxlq.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc(), "-ccbin", host_cxx(), "-std=c++17", "-O3", "-lineinfo", *ARCH,
              "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
    if ptxas_v:
        common += ["-Xptxas", "-v"]
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmds.append(common + EXTRA_FLAGS.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    # translation units compile in parallel; output of each kept together
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for cmd, r in zip(cmds, results):
        if verbose:
            print(" ".join(cmd), flush=True)
        if r.stdout or r.stderr:
            print(r.stdout + r.stderr, end="", flush=True)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, cmd)
    link = [nvcc(), "-ccbin", host_cxx(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, ptxas_v="--ptxas-v" in sys.argv)
    print(LIB)
