"""Build libswd.so (the CUDA kernels + C ABI) in-tree for sm_100a.

Usage: python -m swd_b200.build [--force]

Each .cu file compiles to its own object so that the FD/pick files get
-fmad=false (no multiply-add contraction: their FP32 arithmetic reproduces the
reference's operation order bit for bit) while the Radon/SoftMax files keep
the default contraction.
"""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
OUT = os.path.join(OUT_DIR, "libswd.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
          "--expt-relaxed-constexpr"]
# file -> extra flags
SOURCES = {
    "fd_host.cu": ["-fmad=false"],
    "fd_warpx.cu": ["-fmad=false"],
    "fd_col2.cu": ["-fmad=false"],
    "model_prep.cu": ["-fmad=false"],
    "radon.cu": [],
    "engine.cu": ["-fmad=false"],
    "pick_noalloc.cu": [],
    "server.cu": [],
    "radon_tc.cu": [],
    "wd.cu": [],
    "fk.cu": [],
}


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "swd.h"), __file__]
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _newest(deps):
        return OUT
    jobs = []
    for src, extra in SOURCES.items():
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        jobs.append((cmd, obj))
    # the translation units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(subprocess.run, cmd, check=True) for cmd, _ in jobs]:
            f.result()
    objs = [obj for _, obj in jobs]
    cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
