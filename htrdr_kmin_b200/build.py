"""Build the CUDA library (sm_100a) in-tree: htrdr_kmin_b200/lib/libhtrdr_gpu.so.

    python -m htrdr_kmin_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libhtrdr_gpu.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    deps.append(os.path.join(ROOT, "include", "htrdr_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, verbose: bool) -> str:
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-c",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
           "-I", os.path.join(ROOT, "include"), "-o", obj, src]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}{r.stderr}")
    return r.stderr if verbose else ""


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object (in parallel: the kernel variants
    make each translation unit slow) and link the shared library."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]
    # the largest translation units first
    order = sorted(range(len(srcs)), key=lambda i: -os.path.getsize(srcs[i]))
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        futs = [ex.submit(_compile, srcs[i], objs[i], verbose) for i in order]
        logs = [f.result() for f in futs]
    if verbose:
        sys.stderr.write("".join(logs))
    tmp = LIB + ".tmp"
    r = subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lpthread"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libhtrdr_gpu.so")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
