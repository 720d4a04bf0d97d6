"""Builds libfastcone_b200.so (sm_100a) in-tree with nvcc.

    python -m fastcone_b200.build            # or fastcone_b200.build.build()

The library is a plain C-ABI shared object (include/fastcone_b200.h); Python reaches it
through ctypes, C/C++ callers link it directly.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfastcone_b200.so")
OBJDIR = os.path.join(HERE, "_build")

SOURCES = [
    "fcb_common.cpp",
    "fcb_refgeom.cpp",
    "fcb_backproject.cu",
    "fcb_project.cu",
    "fcb_filter.cu",
    "fcb_katsevich.cu",
    "fcb_conv.cu",
    "fcb_probe.cu",
    "fcb_capi.cpp",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "fastcone_b200.h"))
    newest_header = max(os.path.getmtime(h) for h in headers)
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJDIR, src + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
                and os.path.getmtime(obj) >= newest_header):
            continue
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-c", path, "-o", obj]
        if src.endswith(".cpp"):
            cmd[1:1] = ["-x", "cu"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", OUT, *objs, "-lcufft"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
