"""Builds libgpudock.so (CUDA kernels + C-ABI) for sm_100a, in-tree.

    python -m gpudock_b200.build [--verbose]

Output: gpudock_b200/_lib/libgpudock.so, linked against the static CUDA
runtime so that it does not depend on which libcudart the host process
(e.g. torch) has loaded.  Each source is compiled to its own object (in
parallel, only when it or a header changed); the objects are then linked.
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
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libgpudock.so")
SOURCES = ["gd_kernels.cu", "gd_api.cu", "gd_ensemble.cu", "gd_server.cu", "gd_noalloc.cu",
           "gd_similarity.cu", "gd_load.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags():
    return [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
            "-ccbin", shutil.which("g++") or "g++", "-I" + os.path.join(ROOT, "include")]


def _compile(src: str, obj: str, verbose: bool):
    cmd = [nvcc(), *_flags(), "-c", "-o", obj + ".tmp", src]
    if verbose:
        cmd[1:1] = ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd))
    os.replace(obj + ".tmp", obj)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "gpudock.h"))
    t_hdr = max(os.path.getmtime(h) for h in headers)
    objs, todo = [], []
    for s in srcs:
        o = os.path.join(OBJDIR, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(t_hdr,
                                                                        os.path.getmtime(s)):
            todo.append((s, o))
    if not todo and os.path.exists(LIB) and all(
            os.path.getmtime(o) <= os.path.getmtime(LIB) for o in objs):
        return LIB
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_compile, s, o, verbose) for s, o in todo]:
            f.result()
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-ccbin",
           shutil.which("g++") or "g++", "-o", LIB + ".tmp", *objs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc link failed:\n" + " ".join(cmd))
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv
                or "--verbose" in sys.argv))
