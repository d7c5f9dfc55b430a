"""Builds brook_b200/_lib/libbrook_b200.so from brook_b200/csrc with nvcc for sm_100a.

Every source compiles with --fmad=false (each floating-point operation rounds on its own; the
kernels that mirror a fused multiply-add spell it out) and with host contraction off.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libbrook_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "--fmad=false",
         "-Xcompiler", "-fPIC,-ffp-contract=off", "-DBROOK_B200_VERSION=\"0.1.0\"",
         "-I" + os.path.join(HERE, "..", "include")]


def _sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp")))


def _newest_header():
    headers = glob.glob(os.path.join(SRC, "*.h*")) + glob.glob(os.path.join(SRC, "*.cuh")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return max(os.path.getmtime(h) for h in headers)


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return obj
    cmd = [NVCC, *FLAGS, *extra, "-x", "cu", "-c", src, "-o", obj]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{result.stderr}")
    if result.stderr.strip():
        sys.stderr.write(result.stderr)
    return obj


def build(verbose_ptxas=False, jobs=None):
    """Compile (incrementally) and link the shared library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as pool:
        objects = list(pool.map(lambda s: _compile(s, extra), _sources()))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objects):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objects, "-o", LIB]
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"link failed:\n{result.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
