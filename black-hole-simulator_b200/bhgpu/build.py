"""Compile libbhgpu.so in-tree for sm_100a.

    python black-hole-simulator_b200/bhgpu/build.py

(run as a script: importing the package loads the library it builds)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
          "-I" + os.path.join(REPO, "include"), "-I" + CSRC]
# --fmad=false keeps the reference's separate multiply/add roundings; the FMA
# and mixed variants contract, and the mixed variant's FP32 arithmetic uses
# flush-to-zero and the fast division/square root
FMAD = {"bh_fp64fma.cu": ["--fmad=true"],
        "bh_mixed.cu": ["--fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
        "bh_mlp.cu": ["--fmad=true"]}


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]


def build(verbose: bool = False) -> str:
    out = os.path.join(HERE, "libbhgpu.so")
    srcs = sources()
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps.append(os.path.join(REPO, "include", "bhgpu.h"))
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    bdir = os.path.join(PKG, "_build")
    os.makedirs(bdir, exist_ok=True)
    jobs = []
    for src in srcs:
        obj = os.path.join(bdir, os.path.basename(src).replace(".cu", ".o"))
        cmd = [NVCC] + ARCH + COMMON + FMAD.get(os.path.basename(src), ["--fmad=false"]) + ["-c", src, "-o", obj]
        jobs.append((cmd, obj))
        if verbose:
            print(" ".join(cmd))
    # the translation units compile independently: in parallel
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda j: subprocess.run(j[0], capture_output=True, text=True), jobs))
    for (cmd, obj), r in zip(jobs, results):
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    objs = [obj for _, obj in jobs]
    cmd = [NVCC] + ARCH + ["-shared", "-o", out] + objs
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
