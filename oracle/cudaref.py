"""Runs the reference's own GPU path -- test infrastructure and a reported
timing only, never the product.

``oracle/_ref/cudaref_run`` is the reference's cudasymmfft ``do_transform``
(cudasymmfft/funcinterface.cu:25-334, cuFFT underneath) and its solver
``cuda_helmholtz_solver`` (cudahelmholtz/cuda_helmholtz_solver.cu:33-380),
compiled unchanged from the reference sources by ``oracle/Makefile``, with a
project-written ``cut_transpose3d`` (oracle/cut_transpose.cu) in place of the
absent libcuTranspose.  ``oracle/_ref/chz_dropin_run`` is the same driver
source compiled against this project's drop-in headers and linked against
``libcuhelmholtz_b200.so`` (C++ linkage).  Both speak one file protocol
(oracle/cudaref_main.cu), so a test can feed one input to both.

The programs need a GPU; they run in child processes, so the reference's
global cuFFT plans and ``__constant__`` state never share a process with the
product library.
"""
from __future__ import annotations

import os
import re
import struct
import subprocess
import tempfile

import numpy as np

from . import fishpack

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BINARY = os.path.join(HERE, "_ref", "cudaref_run")
DROPIN_BINARY = os.path.join(HERE, "_ref", "chz_dropin_run")
TRANSFORM_MAGIC = 0x43485A54


def available(binary: str = REF_BINARY) -> bool:
    return os.path.isfile(binary) and os.access(binary, os.X_OK)


def _parse_times(stdout: str):
    out = []
    for line in stdout.splitlines():
        if line.startswith("cudaref_seconds"):
            parts = line.split()
            out.append((float(parts[1]), float(parts[2])))
    return out


def transform_many(cases, binary: str = REF_BINARY, repeats: int = 1, timeout: float = 1800):
    """Runs do_transform once per case in one child process.

    cases: iterable of (data, nx, ny, nz, x_kind, y_kind, z_kind, inplace),
    data of (nz+2)(ny+2)(nx+2) doubles.  Returns a list of
    (result array of shape (nz+2, ny+2, nx+2), best_s, median_s)."""
    if not available(binary):
        raise RuntimeError(f"reference GPU driver not built: {binary} (run make -C oracle)")
    cases = list(cases)
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        with open(fin, "wb") as fh:
            for data, nx, ny, nz, kx, ky, kz, inplace in cases:
                fh.write(struct.pack("<8i", TRANSFORM_MAGIC, nx, ny, nz, kx, ky, kz, int(bool(inplace))))
                fh.write(np.ascontiguousarray(data, dtype="<f8").tobytes())
        res = subprocess.run([binary, "transform", fin, fout, str(repeats)],
                             capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"{os.path.basename(binary)} transform failed: {res.stdout[-400:]} {res.stderr[-400:]}")
        times = _parse_times(res.stdout)
        raw = np.fromfile(fout, dtype="<f8")
    out, off = [], 0
    for (_, nx, ny, nz, *_rest), (best, med) in zip(cases, times):
        n = (nx + 2) * (ny + 2) * (nz + 2)
        out.append((raw[off:off + n].reshape(nz + 2, ny + 2, nx + 2), best, med))
        off += n
    if len(out) != len(cases):
        raise RuntimeError("reference GPU driver returned fewer cases than given")
    return out


def solve(p, binary: str = REF_BINARY, repeats: int = 1, timeout: float = 1800):
    """Runs cuda_helmholtz_solver on problem p (oracle.gen's dict).  Returns
    (u, best_s, median_s); the times are wall times of the synchronous call,
    f re-uploaded before every repeat."""
    if not available(binary):
        raise RuntimeError(f"reference GPU driver not built: {binary} (run make -C oracle)")
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        fishpack.write_input(fin, p)
        res = subprocess.run([binary, "solve", fin, fout, str(repeats)],
                             capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"{os.path.basename(binary)} solve failed: {res.stdout[-400:]} {res.stderr[-400:]}")
        (best, med), = _parse_times(res.stdout)
        u = np.fromfile(fout, dtype="<f8").reshape(p["nz"] + 1, p["ny"] + 1, p["nx"] + 1)
    return u, best, med


_MAXDIFF = re.compile(r"max diff : ([0-9.eE+-]+)")


def run_test_driver(name: str, *args: int, timeout: float = 600) -> float:
    """Runs one of the reference's own test drivers built by oracle/Makefile
    (testgpu_chz, testgpu_ref, testcpu, and the *rectangle forms) with its
    command-line arguments and returns the "max diff" it prints: the max-norm
    error of the computed u against the analytic case (ufunc.h:12-32)."""
    path = os.path.join(HERE, "_ref", name)
    if not available(path):
        raise RuntimeError(f"{name} not built (run make -C oracle)")
    res = subprocess.run([path, *map(str, args)], capture_output=True, text=True, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"{name} failed ({res.returncode}): {res.stdout[-400:]} {res.stderr[-400:]}")
    m = _MAXDIFF.search(res.stdout)
    if not m:
        raise RuntimeError(f"{name}: no max diff in output: {res.stdout[-400:]}")
    return float(m.group(1))
