"""Builds libtlibttm_cuda.so (the CUDA kernels + C ABI) in-tree with nvcc for sm_100a.

    python -m ttm_b200.build          # rebuild if any source is newer than the library
    python -m ttm_b200.build --force  # rebuild unconditionally

Each .cu under ttm_b200/csrc is compiled separately (in parallel) with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and the objects are
linked into ttm_b200/libtlibttm_cuda.so with the CUDA runtime linked
statically; driver entry points (tensor-map encoding) are resolved at run
time, so the library loads even where no driver is installed.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libtlibttm_cuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libtlibttm_cuda.so")
    return cand


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return (sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(glob.glob(os.path.join(CSRC, "*.h")))
            + sorted(glob.glob(os.path.join(INCLUDE, "**", "*.h"), recursive=True)))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    """Compile and link the library; returns its path."""
    srcs = sources()
    if not force and not _stale(LIB, srcs + headers()):
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()
    flags = NVCC_FLAGS + list(extra_flags or [])
    hdrs = headers()
    procs = []
    objs = []
    for src in srcs:
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            cmd = [cc] + ARCH + flags + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    tmp = LIB + ".tmp"
    cmd = [cc] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout.decode(errors="replace"))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
