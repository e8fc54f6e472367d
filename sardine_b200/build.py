"""Builds libsardine_b200.so in-tree with nvcc for sm_100a.

    python -m sardine_b200.build [--verbose]

--fmad=false: the reference never contracts a*b+c into an FMA, and integer
outcomes of the terrain correction (microsecond azimuth times, masks) depend
on the last bit of the double-precision arithmetic.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsardine_b200.so")
SOURCES = ["runtime.cu", "tc.cu", "speckle.cu", "calib.cu", "diag.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC,-O2", "-shared", "-lcudart",
]


def build(verbose: bool = False, force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "sardine_b200.h"))
    if not force and os.path.exists(OUT):
        t_out = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t_out for d in deps):
            return OUT
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", OUT + ".tmp"] + srcs
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libsardine_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(OUT)
