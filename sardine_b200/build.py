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
SOURCES = ["runtime.cu", "tc.cu", "tc_tiles.cu", "speckle.cu", "calib.cu", "diag.cu", "export.cu", "slc.cu", "multilook.cu", "grd.cu", "deramp.cu", "insar.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC,-O2", "-shared", "-lcudart",
]


def build(verbose: bool = False, force: bool = False, extra_flags=(), out: str = None) -> str:
    """Compiles the library (incrementally); `extra_flags` and `out` build a
    variant (e.g. -D switches) into another file with its own objects."""
    global OUT
    if out is not None:
        saved = OUT
        OUT = out
        try:
            return _build(verbose, force, list(extra_flags), os.path.join(os.path.dirname(out), "_build"))
        finally:
            OUT = saved
    return _build(verbose, force, list(extra_flags), os.path.join(HERE, "_build"))


def _build(verbose: bool, force: bool, extra_flags, objdir: str) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "sardine_b200.h"))
    if not force and os.path.exists(OUT):
        t_out = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t_out for d in deps):
            return OUT
    # every translation unit compiles in its own nvcc process, then one link
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.basename(s)[:-3] + ".o") for s in srcs]
    cflags = [f for f in FLAGS if f not in ("-shared", "-lcudart")] + extra_flags
    headers = [d for d in deps if not d.endswith(".cu")]
    t_hdr = max(os.path.getmtime(h) for h in headers)
    procs = []
    for src, obj in zip(srcs, objs):
        # a translation unit recompiles when it or any header is newer than its object
        if (not force and os.path.exists(obj)
                and os.path.getmtime(obj) >= max(os.path.getmtime(src), t_hdr)):
            continue
        cmd = [NVCC] + cflags + (["-Xptxas", "-v"] if verbose else []) + ["-c", "-o", obj, src]
        procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    failed = False
    for pr in procs:
        out, err = pr.communicate()
        if pr.returncode != 0:
            failed = True
            sys.stderr.write(out + err)
        elif verbose:
            sys.stderr.write(err)
    if failed:
        raise RuntimeError("nvcc failed building libsardine_b200.so")
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT + ".tmp"] + objs + ["-lcudart"]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed linking libsardine_b200.so")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(OUT)
