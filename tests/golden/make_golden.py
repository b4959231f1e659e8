"""Regenerates the golden fixtures in this directory from the reference's own CPU
solver (FISHPACK hw3crt through the reference wrapper solver_3d,
cudahelmholtz/hw3crt_wrapper.cpp:5-33), built by ``make -C oracle``.

The reference ships no golden vectors or known-answer tests for this path; its
drivers only print the max-norm error against an analytic function
(testcpurectangle.cpp:134-159).  These fixtures pin the oracle to outputs of the
reference's CPU path run in this repository's build container:

* fishpack_sweep_10x6x8.npz  -- all 125 boundary-code triples on a 10x6x8 grid,
  lambda = -3.7, f and Neumann data ~ U[-1, 1] (periodic-compatible);
* fishpack_16x12x20.npz      -- 12 triples on 16x12x20 with varied lambda;
* fishpack_singular.npz      -- lambda = 0 with every code 0 or 3 on 16x12x20
  and 10x14x8: the solution and PERTRB of a direct hw3crt call (the runner's
  "pertrb" mode; the wrapper drops PERTRB);
* fishpack_ufunc_case1.npz   -- the reference's analytic case 1 (ufunc.h:12-32,
  u = sin(2 pi x) sin(2 pi y) sin(2 pi z) / 3, lambda = -1) on 32^3 and
  24x20x28 for a few triples, with fishpack's max-norm error.

Inputs are regenerated from the stored seeds by ``oracle.gen``; a SHA-256 of
the input bytes is stored to detect generator drift.

usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import fishpack, gen  # noqa: E402
from oracle.stencil import FACE_KEYS  # noqa: E402


def input_digest(p) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(p["f"], dtype="<f8").tobytes())
    for key in FACE_KEYS:
        if p.get(key) is not None:
            h.update(key.encode())
            h.update(np.ascontiguousarray(p[key], dtype="<f8").tobytes())
    return h.hexdigest()


def sweep_case(nx, ny, nz, xbc, ybc, zbc, lam, seed):
    return gen.random_problem(nx, ny, nz, xbc, ybc, zbc, lam, seed)


SWEEP_DIMS = (10, 6, 8)
SWEEP_LAMBDA = -3.7
SWEEP_TRIPLES = list(itertools.product(range(5), repeat=3))

MID_DIMS = (16, 12, 20)
MID_CASES = [  # (xbc, ybc, zbc, lambda)
    (1, 2, 0, -2.0), (3, 4, 0, -1.0), (1, 3, 0, -4.0), (0, 0, 0, -0.25),
    (3, 3, 3, -10.0), (2, 4, 1, -0.01), (4, 2, 3, -50.0), (0, 1, 2, -3.0),
    (2, 2, 2, -7.5), (4, 4, 4, -1.5), (0, 3, 4, -0.5), (1, 1, 1, -100.0),
]


def ufunc_problem(nx, ny, nz, xbc, ybc, zbc):
    """The reference's analytic case 1, assembled as testcpurectangle.cpp:58-123
    does: f = lap u + lambda u in the interior, Dirichlet faces = u, Neumann
    faces = du/dn (outward sign convention of ufunc.h's u{x,y,z}func)."""
    lam = -1.0
    pi = 3.14159265358979323846

    def u(x, y, z):
        return 1.0 / 3.0 * np.sin(2 * pi * x) * np.sin(2 * pi * y) * np.sin(2 * pi * z)

    def ux(x, y, z):
        return 2.0 * pi / 3.0 * np.cos(2 * pi * x) * np.sin(2 * pi * y) * np.sin(2 * pi * z)

    def uy(x, y, z):
        return 2.0 * pi / 3.0 * np.sin(2 * pi * x) * np.cos(2 * pi * y) * np.sin(2 * pi * z)

    def uz(x, y, z):
        return 2.0 * pi / 3.0 * np.sin(2 * pi * x) * np.sin(2 * pi * y) * np.cos(2 * pi * z)

    def lap(x, y, z):
        return -4.0 * pi * pi * np.sin(2 * pi * x) * np.sin(2 * pi * y) * np.sin(2 * pi * z)

    dx, dy, dz = 1.0 / nx, 1.0 / ny, 1.0 / nz
    Z, Y, X = np.meshgrid(np.arange(nz + 1) * dz, np.arange(ny + 1) * dy,
                          np.arange(nx + 1) * dx, indexing="ij")
    f = lap(X, Y, Z) + lam * u(X, Y, Z)
    if xbc in (1, 2):
        f[:, :, 0] = u(X[:, :, 0], Y[:, :, 0], Z[:, :, 0])
    if xbc in (1, 4):
        f[:, :, nx] = u(X[:, :, nx], Y[:, :, nx], Z[:, :, nx])
    if ybc in (1, 2):
        f[:, 0, :] = u(X[:, 0, :], Y[:, 0, :], Z[:, 0, :])
    if ybc in (1, 4):
        f[:, ny, :] = u(X[:, ny, :], Y[:, ny, :], Z[:, ny, :])
    if zbc in (1, 2):
        f[0] = u(X[0], Y[0], Z[0])
    if zbc in (1, 4):
        f[nz] = u(X[nz], Y[nz], Z[nz])
    p = dict(nx=nx, ny=ny, nz=nz, xbc=xbc, ybc=ybc, zbc=zbc,
             dom=gen.UNIT_DOMAIN, lam=lam, f=f)
    p["bcl"] = ux(X[:, :, 0], Y[:, :, 0], Z[:, :, 0]) if xbc in (3, 4) else None
    p["bcr"] = ux(X[:, :, nx], Y[:, :, nx], Z[:, :, nx]) if xbc in (2, 3) else None
    p["bcb"] = uy(X[:, 0, :], Y[:, 0, :], Z[:, 0, :]) if ybc in (3, 4) else None
    p["bct"] = uy(X[:, ny, :], Y[:, ny, :], Z[:, ny, :]) if ybc in (2, 3) else None
    p["bcf"] = uz(X[0], Y[0], Z[0]) if zbc in (3, 4) else None
    p["bce"] = uz(X[nz], Y[nz], Z[nz]) if zbc in (2, 3) else None
    p["u_exact"] = u(X, Y, Z)
    return p


SINGULAR_CASES = [  # (dims, codes, seed), lambda = 0
    ((16, 12, 20), (3, 3, 3), 3000), ((16, 12, 20), (0, 3, 0), 3001), ((16, 12, 20), (0, 0, 0), 3002),
    ((16, 12, 20), (3, 0, 3), 3003), ((10, 14, 8), (0, 0, 3), 3004), ((10, 14, 8), (3, 3, 0), 3005),
]

UFUNC_CASES = [((32, 32, 32), (1, 2, 0)), ((32, 32, 32), (3, 4, 0)),
               ((24, 20, 28), (1, 2, 3)), ((24, 20, 28), (4, 3, 1))]


def main():
    if not fishpack.available():
        raise SystemExit("build the fishpack runner first: make -C oracle")
    # sweep
    us, digests, seeds = [], [], []
    for t, (xbc, ybc, zbc) in enumerate(SWEEP_TRIPLES):
        seed = 1000 + t
        p = sweep_case(*SWEEP_DIMS, xbc, ybc, zbc, SWEEP_LAMBDA, seed)
        u, _, _ = fishpack.solve(p)
        us.append(u)
        digests.append(input_digest(p))
        seeds.append(seed)
    np.savez_compressed(os.path.join(HERE, "fishpack_sweep_10x6x8.npz"),
                        dims=np.array(SWEEP_DIMS), lam=SWEEP_LAMBDA,
                        triples=np.array(SWEEP_TRIPLES), seeds=np.array(seeds),
                        digests=np.array(digests), u=np.stack(us))
    # mid-size
    us, digests, seeds = [], [], []
    for t, (xbc, ybc, zbc, lam) in enumerate(MID_CASES):
        seed = 2000 + t
        p = sweep_case(*MID_DIMS, xbc, ybc, zbc, lam, seed)
        u, _, _ = fishpack.solve(p)
        us.append(u)
        digests.append(input_digest(p))
        seeds.append(seed)
    np.savez_compressed(os.path.join(HERE, "fishpack_16x12x20.npz"),
                        dims=np.array(MID_DIMS), cases=np.array(MID_CASES),
                        seeds=np.array(seeds), digests=np.array(digests),
                        u=np.stack(us))
    # singular problems: solution and PERTRB of a direct hw3crt call
    us, pert, digests = [], [], []
    for dims, bcs, seed in SINGULAR_CASES:
        p = gen.random_problem(*dims, *bcs, 0.0, seed)
        u, pertrb, ierror = fishpack.solve_with_pertrb(p)
        if ierror != 0:
            raise SystemExit(f"hw3crt ierror {ierror} on {dims} {bcs}")
        us.append(u.ravel())
        pert.append(pertrb)
        digests.append(input_digest(p))
    np.savez_compressed(os.path.join(HERE, "fishpack_singular.npz"),
                        dims=np.array([c[0] for c in SINGULAR_CASES]),
                        codes=np.array([c[1] for c in SINGULAR_CASES]),
                        seeds=np.array([c[2] for c in SINGULAR_CASES]), digests=np.array(digests),
                        u=np.concatenate(us), offsets=np.cumsum([0] + [len(v) for v in us]),
                        pertrb=np.array(pert))
    # analytic case 1
    rec = []
    for dims, bcs in UFUNC_CASES:
        p = ufunc_problem(*dims, *bcs)
        u, _, _ = fishpack.solve(p)
        maxdiff = float(np.abs(u - p["u_exact"]).max())
        rec.append(list(dims) + list(bcs) + [maxdiff])
    np.savez_compressed(os.path.join(HERE, "fishpack_ufunc_case1.npz"),
                        cases=np.array(rec))
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
