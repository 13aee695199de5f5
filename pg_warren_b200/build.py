"""Builds libwarren_cuda.so in the package directory from csrc/.

Every .cu / .cpp file is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``), in parallel, then linked into
one shared library with the CUDA runtime linked statically.  The library is
built in tree so it travels with the repository to the GPU machine.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBRARY = os.path.join(HERE, "libwarren_cuda.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: a product and a sum stay two roundings, as on the host, so
# floating-point results follow the reference's operation order bit for bit.
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", f"-I{INCLUDE}",
         "--expt-relaxed-constexpr", "--extended-lambda", "-fmad=false"]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [
        os.path.join(INCLUDE, "warren_cuda.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src):
    obj = os.path.join(BUILD, src + ".o")
    deps = [os.path.join(CSRC, src)] + headers() + [__file__]
    if not _stale(obj, deps):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(_compile, srcs))
    if _stale(LIBRARY, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIBRARY + ".tmp", *objs,
               "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(LIBRARY + ".tmp", LIBRARY)
    if verbose:
        print(LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
