"""GPU parity against the reference's own GPU path and drop-in checks of the
C++-linkage entry points.

* Golden fixtures (tests/golden/cudaref_*.npz, made by
  make_reference_gpu_golden.py from the reference's cudasymmfft do_transform
  over cuFFT and its cuda_helmholtz_solver, compiled unchanged): this
  library's do_transform and solver through the C ABI must match them to
  1e-12 relative on every entry the reference defines.
* Live: the same reference programs (oracle/_ref/cudaref_run) run beside this
  library on the benchmark configurations' sizes, up to 512^3.
* Drop-in: oracle/_ref/chz_dropin_run is the reference-facing driver source
  compiled against include/ and linked against libcuhelmholtz_b200.so, so it
  calls do_transform and cuda_helmholtz_solver with C++ linkage exactly as the
  reference's callers do (cudahelmholtz/testgpu.cu:163-176,
  cuda_helmholtz_solver.cu:313,344); the reference's own test drivers
  testgpu.cu and testgpurectangle.cu, unchanged, are linked against this
  library too and must print the max-norm errors that the reference's GPU and
  CPU builds of the same drivers print.
"""
import os
import sys

import numpy as np
import pytest
import torch

from oracle import cudaref, gen
from oracle import emulation as E
from oracle.stencil import FACE_KEYS
from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLDEN)
from make_golden import SWEEP_DIMS, MID_DIMS, input_digest, sweep_case  # noqa: E402
from make_reference_gpu_golden import array_digest, transform_input  # noqa: E402

TOL = 1e-12

needs_ref = pytest.mark.skipif(not cudaref.available(), reason="oracle/_ref/cudaref_run not built")
needs_dropin = pytest.mark.skipif(not cudaref.available(cudaref.DROPIN_BINARY),
                                  reason="oracle/_ref/chz_dropin_run not built")


def window_mask(nx, ny, nz, kinds):
    """Entries the reference defines: the product of the kinds' output windows
    (the entries outside are left undefined by its pre/post kernels)."""
    m = np.zeros((nz + 2, ny + 2, nx + 2), dtype=bool)
    (x0, x1), (y0, y1), (z0, z1) = (E.out_window(kinds[0], nx), E.out_window(kinds[1], ny),
                                    E.out_window(kinds[2], nz))
    m[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1] = True
    return m


def ours_transform(h, nx, ny, nz, kinds, inplace):
    dev = torch.from_numpy(np.ascontiguousarray(h).ravel()).cuda()
    out = None if inplace else torch.full_like(dev, float("nan"))
    res = api.do_transform(dev, out, nx, ny, nz, *kinds)
    torch.cuda.synchronize()
    return res.cpu().numpy().reshape(nz + 2, ny + 2, nx + 2)


def ours_solve(p):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    fc = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
          for k in FACE_KEYS}
    d = p["dom"]
    api.cuda_helmholtz_solver(d[0], d[1], p["nx"], p["xbc"], fc["bcl"], fc["bcr"],
                              d[2], d[3], p["ny"], p["ybc"], fc["bcb"], fc["bct"],
                              d[4], d[5], p["nz"], p["zbc"], fc["bcf"], fc["bce"], p["lam"], f)
    torch.cuda.synchronize()
    return f.cpu().numpy().reshape(p["nz"] + 1, p["ny"] + 1, p["nx"] + 1)


def window_err(got, ref, m):
    assert not np.isnan(got[m]).any(), "defined entry not written"
    scale = max(1.0, np.abs(ref[m]).max())
    maxe = np.abs(got[m] - ref[m]).max() / scale
    l2 = np.linalg.norm(got[m] - ref[m]) / np.linalg.norm(ref[m])
    return max(maxe, l2)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# ---------------------------------------------------------------------------
# golden fixtures of the reference GPU path
# ---------------------------------------------------------------------------

def _transform_golden():
    return np.load(os.path.join(GOLDEN, "cudaref_transform.npz"))


@pytest.mark.parametrize("group", ["cube8", "cube12", "box8x6x10", "box12x16x20"])
def test_transform_matches_reference_gpu_golden(group):
    g = _transform_golden()
    nx, ny, nz = (int(v) for v in g[f"{group}_dims"])
    inplace = bool(g[f"{group}_inplace"])
    for kinds, seed, digest, ref in zip(g[f"{group}_kinds"], g[f"{group}_seeds"], g[f"{group}_digests"],
                                        g[f"{group}_out"]):
        h = transform_input((nx, ny, nz), int(seed))
        assert array_digest(h) == str(digest), "input generator drifted"
        kinds = tuple(int(k) for k in kinds)
        got = ours_transform(h, nx, ny, nz, kinds, inplace)
        err = window_err(got, ref, window_mask(nx, ny, nz, kinds))
        assert err < TOL, (group, kinds, err)


def test_solver_matches_reference_gpu_golden():
    g = np.load(os.path.join(GOLDEN, "cudaref_solve.npz"))
    lam = float(g["sweep_lam"])
    for t, (xbc, ybc, zbc) in enumerate(g["sweep_triples"]):
        p = sweep_case(*SWEEP_DIMS, int(xbc), int(ybc), int(zbc), lam, int(g["sweep_seeds"][t]))
        assert input_digest(p) == str(g["sweep_digests"][t])
        err = rel(ours_solve(p), g["sweep_u"][t])
        assert err < TOL, ((xbc, ybc, zbc), err)
    for t, (xbc, ybc, zbc, lam) in enumerate(g["mid_cases"]):
        p = sweep_case(*MID_DIMS, int(xbc), int(ybc), int(zbc), float(lam), int(g["mid_seeds"][t]))
        assert input_digest(p) == str(g["mid_digests"][t])
        err = rel(ours_solve(p), g["mid_u"][t])
        assert err < TOL, ((xbc, ybc, zbc, lam), err)


# ---------------------------------------------------------------------------
# live: the reference GPU programs beside this library at the benchmark sizes
# ---------------------------------------------------------------------------

LIVE_TRANSFORMS = [  # (dims, kinds, inplace)
    ((64, 64, 64), (3, 4, 6), True), ((64, 64, 64), (5, 0, 2), True), ((64, 64, 64), (1, 7, 3), True),
    ((64, 64, 64), (6, 2, 5), True),
    ((128, 128, 128), (3, 4, 6), True),            # the 128^3 configuration's DST-I / DST-II / DFT
    ((256, 192, 320), (5, 2, 0), False),           # codes (2, 4, 3): DST-III / DCT-III / DCT-I
    ((256, 192, 320), (6, 3, 0), False),           # codes (0, 1, 3)
    ((48, 40, 96), (4, 7, 1), False),
    ((512, 512, 512), (0, 2, 6), True),            # the 512^3 configuration's forward kinds
]


@needs_ref
@pytest.mark.parametrize("dims,kinds,inplace", LIVE_TRANSFORMS)
def test_transform_live_vs_reference_gpu(dims, kinds, inplace):
    nx, ny, nz = dims
    h = np.random.default_rng(sum(dims) + 7 * kinds[0]).standard_normal((nz + 2, ny + 2, nx + 2))
    (ref, _, _), = cudaref.transform_many([(h, nx, ny, nz, *kinds, inplace)])
    got = ours_transform(h, nx, ny, nz, kinds, inplace)
    err = window_err(got, ref, window_mask(nx, ny, nz, kinds))
    assert err < TOL, err


LIVE_SOLVES = [
    ("128^3 codes (1,2,0), lambda=-2, manufactured", lambda: gen.config1_problem(seed=1, n=128)),
    ("256x192x320 codes (2,4,3)", lambda: gen.config2_problem(2, 4, seed=2)),
    ("256x192x320 codes (0,1,3)", lambda: gen.config2_problem(0, 1, seed=2)),
    ("256^3 codes (1,3,0), lambda=-4", lambda: gen.config5_problem(seed=5, n=256)),
    ("512^3 codes (3,4,0), lambda=-1, 1e3 mode", lambda: gen.config3_problem(seed=3, n=512)),
]


@needs_ref
@pytest.mark.parametrize("name,make", LIVE_SOLVES, ids=[c[0] for c in LIVE_SOLVES])
def test_solver_live_vs_reference_gpu(name, make):
    p = make()
    uref, _, _ = cudaref.solve(p)
    err = rel(ours_solve(p), uref)
    assert err < TOL, (name, err)


# ---------------------------------------------------------------------------
# drop-in: C++-linkage entry points called by a reference-style driver
# ---------------------------------------------------------------------------

@needs_ref
@needs_dropin
def test_dropin_transform_matches_reference_driver():
    cases = []
    for i, kinds in enumerate([(3, 4, 6), (0, 2, 6), (5, 1, 7), (2, 3, 4)]):
        h = np.random.default_rng(900 + i).standard_normal((18, 18, 18))
        cases.append((h, 16, 16, 16, *kinds, True))
        h2 = np.random.default_rng(950 + i).standard_normal((30, 22, 26))
        cases.append((h2, 24, 20, 28, *kinds, False))
    ref = cudaref.transform_many(cases)
    ours = cudaref.transform_many(cases, binary=cudaref.DROPIN_BINARY)
    for (_, nx, ny, nz, kx, ky, kz, _), (r, _, _), (o, _, _) in zip(cases, ref, ours):
        err = window_err(o, r, window_mask(nx, ny, nz, (kx, ky, kz)))
        assert err < TOL, ((nx, ny, nz), (kx, ky, kz), err)


@needs_ref
@needs_dropin
@pytest.mark.parametrize("dims,codes,lam", [((10, 6, 8), (3, 4, 0), -3.7), ((16, 12, 20), (2, 2, 2), -7.5),
                                            ((64, 64, 64), (0, 3, 1), -1.0), ((96, 64, 128), (4, 1, 3), -0.5)])
def test_dropin_solver_matches_reference_driver(dims, codes, lam):
    p = gen.random_problem(*dims, *codes, lam, seed=77)
    uref, _, _ = cudaref.solve(p)
    u, _, _ = cudaref.solve(p, binary=cudaref.DROPIN_BINARY)
    assert rel(u, uref) < TOL


REF_DRIVER_CASES = [(32, (1, 2, 0)), (32, (3, 4, 0)), (64, (1, 1, 1)), (64, (2, 4, 3)), (48, (0, 0, 0)),
                    (64, (3, 0, 4))]
REF_RECT_CASES = [((32, 24, 40), (1, 2, 3)), ((64, 32, 48), (4, 3, 1)), ((40, 48, 32), (0, 2, 4))]


@pytest.mark.skipif(not all(cudaref.available(os.path.join(cudaref.HERE, "_ref", b))
                            for b in ("testgpu_chz", "testgpu_ref", "testcpu")),
                    reason="reference test drivers not built")
@pytest.mark.parametrize("n,codes", REF_DRIVER_CASES)
def test_reference_testgpu_driver_unchanged(n, codes):
    """cudahelmholtz/testgpu.cu, unchanged, linked against this library: its
    printed max-norm error against the analytic u equals the one printed by
    the same driver linked against the reference's GPU solver and by
    testcpu.cpp on FISHPACK (both solve the same discrete system)."""
    ours = cudaref.run_test_driver("testgpu_chz", n, *codes)
    ref_gpu = cudaref.run_test_driver("testgpu_ref", n, *codes)
    ref_cpu = cudaref.run_test_driver("testcpu", n, *codes)
    assert ours > 0
    for other in (ref_gpu, ref_cpu):
        assert abs(ours - other) <= 1e-9 * other + 1e-13, (ours, ref_gpu, ref_cpu)


@pytest.mark.skipif(not all(cudaref.available(os.path.join(cudaref.HERE, "_ref", b))
                            for b in ("testgpurectangle_chz", "testgpurectangle_ref", "testcpurectangle")),
                    reason="reference test drivers not built")
@pytest.mark.parametrize("dims,codes", REF_RECT_CASES)
def test_reference_testgpurectangle_driver_unchanged(dims, codes):
    ours = cudaref.run_test_driver("testgpurectangle_chz", *dims, *codes)
    ref_gpu = cudaref.run_test_driver("testgpurectangle_ref", *dims, *codes)
    ref_cpu = cudaref.run_test_driver("testcpurectangle", *dims, *codes)
    assert ours > 0
    for other in (ref_gpu, ref_cpu):
        assert abs(ours - other) <= 1e-9 * other + 1e-13, (ours, ref_gpu, ref_cpu)
