"""Runs the reference's CPU solver (FISHPACK hw3crt via the reference wrapper
solver_3d, cudahelmholtz/hw3crt_wrapper.cpp:5-33) -- test infrastructure and
the timed CPU baseline only.

The binary is built by ``oracle/Makefile`` into ``oracle/_ref/hw3crt_run``.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

from .stencil import FACE_KEYS

HERE = os.path.dirname(os.path.abspath(__file__))
BINARY = os.path.join(HERE, "_ref", "hw3crt_run")
MAGIC = 0x43485A31


def available() -> bool:
    return os.path.isfile(BINARY) and os.access(BINARY, os.X_OK)


def write_input(path, p):
    present = 0
    for b, key in enumerate(FACE_KEYS):
        if p.get(key) is not None:
            present |= 1 << b
    with open(path, "wb") as fh:
        fh.write(struct.pack("<8i", MAGIC, p["nx"], p["ny"], p["nz"],
                             p["xbc"], p["ybc"], p["zbc"], present))
        fh.write(struct.pack("<7d", *p["dom"], p["lam"]))
        fh.write(np.ascontiguousarray(p["f"], dtype="<f8").tobytes())
        for key in FACE_KEYS:
            if p.get(key) is not None:
                fh.write(np.ascontiguousarray(p[key], dtype="<f8").tobytes())


def solve(p, repeats=1, timeout=3600):
    """Returns (u, best_seconds, median_seconds).  Raises when hw3crt reports a
    nonzero error code (it needs at least 5 cells per axis)."""
    if not available():
        raise RuntimeError(f"fishpack runner not built: {BINARY} (run make -C oracle)")
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        write_input(fin, p)
        res = subprocess.run([BINARY, fin, fout, str(repeats)],
                             capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"hw3crt_run failed: {res.stderr}")
        best = med = None
        ierror = None
        for line in res.stdout.splitlines():
            if line.startswith("hw3crt_seconds"):
                parts = line.split()
                best, med = float(parts[1]), float(parts[2])
            if line.startswith("State code"):
                ierror = int(line.split(":")[1])
        if ierror != 0:
            raise RuntimeError(f"hw3crt rejected the problem (ierror={ierror})")
        u = np.fromfile(fout, dtype="<f8").reshape(p["nz"] + 1, p["ny"] + 1,
                                                   p["nx"] + 1)
    return u, best, med


def solve_with_pertrb(p, timeout=600):
    """Calls hw3crt directly (not through the wrapper, which drops PERTRB)
    and returns (u, pertrb, ierror)."""
    if not available():
        raise RuntimeError(f"fishpack runner not built: {BINARY} (run make -C oracle)")
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        write_input(fin, p)
        res = subprocess.run([BINARY, fin, fout, "pertrb"], capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"hw3crt_run failed: {res.stderr}")
        pertrb = ierror = None
        for line in res.stdout.splitlines():
            if line.startswith("pertrb"):
                parts = line.split()
                pertrb, ierror = float(parts[1]), int(parts[3])
        u = np.fromfile(fout, dtype="<f8").reshape(p["nz"] + 1, p["ny"] + 1, p["nx"] + 1)
    return u, pertrb, ierror


def solve_many_parallel(p, procs, timeout=3600):
    """Runs ``procs`` independent copies of the same solve concurrently (one
    process each; hw3crt is serial).  Returns the per-process wall times."""
    if not available():
        raise RuntimeError(f"fishpack runner not built: {BINARY}")
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        write_input(fin, p)
        running = []
        for i in range(procs):
            fout = os.path.join(td, f"out{i}.bin")
            running.append(subprocess.Popen([BINARY, fin, fout, "1"],
                                            stdout=subprocess.PIPE,
                                            stderr=subprocess.PIPE, text=True))
        times = []
        for pr in running:
            out, err = pr.communicate(timeout=timeout)
            if pr.returncode != 0:
                raise RuntimeError(f"hw3crt_run failed: {err}")
            for line in out.splitlines():
                if line.startswith("hw3crt_seconds"):
                    times.append(float(line.split()[1]))
    return times
