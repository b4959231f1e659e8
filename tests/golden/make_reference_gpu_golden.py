"""Regenerates the reference-GPU golden fixtures from the reference's own GPU
path: cudasymmfft ``do_transform`` over cuFFT (cudasymmfft/funcinterface.cu:25-334)
and ``cuda_helmholtz_solver`` (cudahelmholtz/cuda_helmholtz_solver.cu:33-380),
compiled unchanged from the reference sources into ``oracle/_ref/cudaref_run``
by ``oracle/Makefile`` (with the project-written cut_transpose3d of
oracle/cut_transpose.cu for the absent libcuTranspose).  Needs a GPU.

* cudaref_transform.npz -- do_transform outputs, in place on 8^3 (64 kind
  triples: every (x, y) kind pair once, every kind 8 times on every axis) and
  12^3 (8 triples), out of place on 8x6x10 (the same 64 triples) and 12x16x20
  (8 triples).  Input of case i: numpy default_rng(seed_i).standard_normal of
  the padded (NZ+2, NY+2, NX+2) array; a SHA-256 of the input bytes guards
  against generator drift.  Entries outside each kind's output window are
  whatever the reference left there (its pre/post kernels and cuFFT do not
  define them); checks compare the windows only.
* cudaref_solve.npz -- solver outputs for all 125 boundary-code triples on
  10x6x8, lambda = -3.7, with the inputs of the FISHPACK sweep fixture (same
  seeds, oracle.gen.random_problem), and the 12 mixed cases on 16x12x20 of the
  FISHPACK mid-size fixture.

usage: python tests/golden/make_reference_gpu_golden.py [out_dir]
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import cudaref  # noqa: E402
from make_golden import (MID_CASES, MID_DIMS, SWEEP_DIMS, SWEEP_LAMBDA,  # noqa: E402
                         SWEEP_TRIPLES, input_digest, sweep_case)

LATIN_64 = [(i % 8, i // 8, (i + 3 * (i // 8)) % 8) for i in range(64)]
SPARSE_8 = [(3, 4, 6), (5, 0, 2), (1, 7, 3), (6, 2, 5), (0, 3, 1), (2, 6, 7), (4, 5, 0), (7, 1, 4)]
TRANSFORM_GROUPS = [  # (name, dims, inplace, triples, first seed)
    ("cube8", (8, 8, 8), True, LATIN_64, 5000),
    ("cube12", (12, 12, 12), True, SPARSE_8, 5100),
    ("box8x6x10", (8, 6, 10), False, LATIN_64, 5200),
    ("box12x16x20", (12, 16, 20), False, SPARSE_8, 5300),
]


def transform_input(dims, seed):
    nx, ny, nz = dims
    return np.random.default_rng(seed).standard_normal((nz + 2, ny + 2, nx + 2))


def array_digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out_dir, exist_ok=True)
    if not cudaref.available():
        raise SystemExit("build the reference GPU driver first: make -C oracle")
    rec = {}
    for name, dims, inplace, triples, seed0 in TRANSFORM_GROUPS:
        cases, seeds, digests = [], [], []
        for i, (kx, ky, kz) in enumerate(triples):
            h = transform_input(dims, seed0 + i)
            cases.append((h, *dims, kx, ky, kz, inplace))
            seeds.append(seed0 + i)
            digests.append(array_digest(h))
        outs = cudaref.transform_many(cases)
        rec[f"{name}_dims"] = np.array(dims)
        rec[f"{name}_inplace"] = np.array(inplace)
        rec[f"{name}_kinds"] = np.array(triples)
        rec[f"{name}_seeds"] = np.array(seeds)
        rec[f"{name}_digests"] = np.array(digests)
        rec[f"{name}_out"] = np.stack([o[0] for o in outs])
    rec["groups"] = np.array([g[0] for g in TRANSFORM_GROUPS])
    np.savez_compressed(os.path.join(out_dir, "cudaref_transform.npz"), **rec)

    us, digests, seeds = [], [], []
    for t, (xbc, ybc, zbc) in enumerate(SWEEP_TRIPLES):
        p = sweep_case(*SWEEP_DIMS, xbc, ybc, zbc, SWEEP_LAMBDA, 1000 + t)
        u, _, _ = cudaref.solve(p)
        us.append(u)
        digests.append(input_digest(p))
        seeds.append(1000 + t)
    mid_us, mid_digests, mid_seeds = [], [], []
    for t, (xbc, ybc, zbc, lam) in enumerate(MID_CASES):
        p = sweep_case(*MID_DIMS, xbc, ybc, zbc, lam, 2000 + t)
        u, _, _ = cudaref.solve(p)
        mid_us.append(u)
        mid_digests.append(input_digest(p))
        mid_seeds.append(2000 + t)
    np.savez_compressed(os.path.join(out_dir, "cudaref_solve.npz"),
                        sweep_dims=np.array(SWEEP_DIMS), sweep_lam=SWEEP_LAMBDA,
                        sweep_triples=np.array(SWEEP_TRIPLES), sweep_seeds=np.array(seeds),
                        sweep_digests=np.array(digests), sweep_u=np.stack(us),
                        mid_dims=np.array(MID_DIMS), mid_cases=np.array(MID_CASES),
                        mid_seeds=np.array(mid_seeds), mid_digests=np.array(mid_digests),
                        mid_u=np.stack(mid_us))
    print("wrote reference-GPU fixtures to", out_dir)


if __name__ == "__main__":
    main()
