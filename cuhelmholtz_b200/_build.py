"""Builds the in-tree shared library cuhelmholtz_b200/lib/libcuhelmholtz_b200.so
with nvcc for sm_100a (no JIT cache: the built file travels with the tree).

usage: python -m cuhelmholtz_b200._build [--force]
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
LIBNAME = "libcuhelmholtz_b200.so"
LIBPATH = os.path.join(LIBDIR, LIBNAME)

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
              "--expt-relaxed-constexpr", "-Xptxas", "-v"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIBPATH):
        return True
    t = os.path.getmtime(LIBPATH)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) \
        + glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def source_digest() -> str:
    """SHA-256 (first 16 hex digits) over the library's CUDA sources and
    headers, by file name: identifies the build a profile was captured on."""
    import hashlib
    h = hashlib.sha256()
    deps = sorted(sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")))
    for d in deps:
        h.update(os.path.basename(d).encode())
        with open(d, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def _compile(src: str, obj: str) -> str:
    cmd = [nvcc_path(), *ARCH_FLAGS, *NVCC_FLAGS, "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
           "-c", "-o", obj, src]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n" + res.stdout + res.stderr)
    return res.stderr


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compiles every translation unit (in parallel) and links the shared
    library; a no-op when the library is newer than all sources."""
    if not force and not _stale():
        return LIBPATH
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]
    jobs = max(1, min(len(srcs), os.cpu_count() or 1))
    logs = []
    with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
        for src, log in zip(srcs, ex.map(_compile, srcs, objs)):
            logs.append(f"== {os.path.basename(src)}\n{log}")
    tmp = LIBPATH + ".tmp"
    cmd = [nvcc_path(), *ARCH_FLAGS, "-shared", "-o", tmp, *objs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write("".join(logs))
    os.replace(tmp, LIBPATH)
    with open(os.path.join(LIBDIR, "ptxas.log"), "w") as fh:
        fh.write("".join(logs))
    return LIBPATH


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
