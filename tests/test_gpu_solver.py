"""GPU parity of the FP64 Helmholtz solver (through the C ABI) against the
reference's CPU solver (FISHPACK golden fixtures), the oracle's restatement of
the reference GPU solver, and manufactured discrete solutions (exact answers)
up to the benchmark sizes.  Tolerance: 1e-12 relative L2 unless stated."""
import itertools
import os
import sys

import numpy as np
import pytest
import torch

from oracle import emulation as E
from oracle import gen, stencil
from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLDEN)
from make_golden import MID_DIMS, SWEEP_DIMS, sweep_case, ufunc_problem  # noqa: E402

TOL = 1e-12


def gpu_solve(p, workspace=None):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    faces = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
             for k in stencil.FACE_KEYS}
    d = p["dom"]
    api.cuda_helmholtz_solver(d[0], d[1], p["nx"], p["xbc"], faces["bcl"], faces["bcr"],
                              d[2], d[3], p["ny"], p["ybc"], faces["bcb"], faces["bct"],
                              d[4], d[5], p["nz"], p["zbc"], faces["bcf"], faces["bce"],
                              p["lam"], f, workspace=workspace)
    torch.cuda.synchronize()
    return f.cpu().numpy().reshape(p["nz"] + 1, p["ny"] + 1, p["nx"] + 1)


def emulated(p):
    d = p["dom"]
    return E.emulate_solver(d[0], d[1], p["nx"], p["xbc"], p["bcl"], p["bcr"],
                            d[2], d[3], p["ny"], p["ybc"], p["bcb"], p["bct"],
                            d[4], d[5], p["nz"], p["zbc"], p["bcf"], p["bce"], p["lam"], p["f"])


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_matches_fishpack_all_125_triples():
    g = np.load(os.path.join(GOLDEN, "fishpack_sweep_10x6x8.npz"))
    for t, trip in enumerate(g["triples"]):
        xbc, ybc, zbc = (int(v) for v in trip)
        p = sweep_case(*SWEEP_DIMS, xbc, ybc, zbc, float(g["lam"]), int(g["seeds"][t]))
        u = gpu_solve(p)
        assert rel(u, g["u"][t]) < TOL, ((xbc, ybc, zbc), rel(u, g["u"][t]))


def test_matches_fishpack_16x12x20():
    g = np.load(os.path.join(GOLDEN, "fishpack_16x12x20.npz"))
    for t, case in enumerate(g["cases"]):
        xbc, ybc, zbc = (int(v) for v in case[:3])
        p = sweep_case(*MID_DIMS, xbc, ybc, zbc, float(case[3]), int(g["seeds"][t]))
        assert rel(gpu_solve(p), g["u"][t]) < TOL


def test_analytic_case1_error_equals_fishpack():
    g = np.load(os.path.join(GOLDEN, "fishpack_ufunc_case1.npz"))
    for row in g["cases"]:
        p = ufunc_problem(*(int(v) for v in row[:6]))
        u = gpu_solve(p)
        maxdiff = np.abs(u - p["u_exact"]).max()
        assert abs(maxdiff - row[6]) <= 1e-10 * row[6] + 1e-13


@pytest.mark.parametrize("bcs", list(itertools.product(range(5), repeat=3)))
def test_matches_oracle_noncubic_mixed_radix(bcs):
    """All 125 triples on 24x20x28 (N/2 = 12, 10, 14: radices 3, 5, 7)."""
    p = gen.random_problem(24, 20, 28, *bcs, -3.3, seed=sum(b * 5 ** i for i, b in enumerate(bcs)))
    assert rel(gpu_solve(p), emulated(p)) < TOL


@pytest.mark.parametrize("dims,bcs,lam", [
    ((32, 96, 48), (3, 1, 2), -5.0),   # x lines of the 32-point register kernel (128 rows per tile)
    ((32, 32, 32), (4, 2, 1), -0.5),
    ((64, 64, 64), (1, 2, 0), -2.0),
    ((96, 80, 112), (3, 4, 0), -1.0),
    ((176, 48, 32), (0, 3, 2), -0.01),
    ((128, 128, 128), (4, 1, 3), -100.0),
])
def test_manufactured_exact(dims, bcs, lam):
    p = gen.manufactured_problem(*dims, *bcs, lam, seed=21)
    u = gpu_solve(p)
    w = stencil.window_slices(*dims, *bcs)
    assert rel(u[w], p["u_exact"][w]) < TOL


def test_config1_128_manufactured():
    p = gen.config1_problem()
    u = gpu_solve(p)
    assert rel(u, p["u_exact"]) < TOL


@pytest.mark.parametrize("xy", [(0, 0), (1, 2), (2, 4), (3, 1), (4, 3)])
def test_config2_shape_vs_oracle(xy):
    p = gen.config2_problem(*xy)
    u = gpu_solve(p)
    assert rel(u, emulated(p)) < TOL


def test_config3_512_manufactured_exact():
    """512^3, codes (3, 4, 0), lambda = -1: the exact discrete solution is
    recovered (size-independent check at the benchmark size)."""
    p = gen.manufactured_problem(512, 512, 512, 3, 4, 0, -1.0, seed=3, nmodes=4)
    u = gpu_solve(p)
    err = rel(u, p["u_exact"])
    assert err < TOL, err


@pytest.mark.parametrize("family", ["generic", "no_tma"])
@pytest.mark.parametrize("bcs", [(1, 2, 0), (3, 4, 0), (0, 0, 0), (2, 1, 4), (4, 3, 2), (1, 1, 1), (3, 3, 3)])
def test_kernel_families_agree(bcs, family):
    """The TMA-pipelined, register-resident and generic kernels give the same
    solve (1e-13)."""
    p = gen.random_problem(64, 32, 128, *bcs, -2.0, seed=5)
    a = gpu_solve(p)
    prev = api.set_kernel_family(family)
    try:
        b = gpu_solve(p)
    finally:
        api.set_kernel_family(prev)
    assert rel(a, b) < 1e-13
    assert rel(a, emulated(p)) < TOL


def test_explicit_workspace_matches_cached():
    p = gen.random_problem(32, 24, 40, 2, 0, 4, -5.0, seed=8)
    ws = torch.empty(api.workspace_size(32, 24, 40) // 8 + 32, dtype=torch.float64, device="cuda")
    a = gpu_solve(p)
    b = gpu_solve(p, workspace=ws)
    assert np.array_equal(a, b)


def test_singular_mode_zeroed_like_reference():
    """lambda = 0 with periodic/Neumann axes: mode (0,0,0) is zeroed
    (_cuda_helmholtz_.inl:301-305)."""
    p = gen.random_problem(16, 12, 20, 0, 3, 3, 0.0, seed=4)
    assert rel(gpu_solve(p), emulated(p)) < TOL


def test_bad_boundary_code_raises():
    f = torch.zeros(9 * 9 * 9, dtype=torch.float64, device="cuda")
    with pytest.raises(api.CHZError):
        api.cuda_helmholtz_solver(0, 1, 8, 7, None, None, 0, 1, 8, 1, None, None, 0, 1, 8, 1,
                                  None, None, -1.0, f)


@pytest.mark.parametrize("dims,bcs,lam", [
    ((40, 24, 512), (3, 4, 0), -1.0),
    ((18, 10, 512), (1, 2, 0), -2.5),    # x window starts at 1: map column 0 rounded down
    ((24, 40, 512), (0, 0, 0), 0.0),     # singular: zero mode removed in the z pass
    ((36, 20, 512), (3, 3, 0), 0.0),
    ((16, 16, 512), (4, 1, 0), -7.0),
    ((16, 24, 256), (3, 4, 0), -1.0),
    ((18, 10, 256), (1, 2, 0), -2.5),
    ((24, 40, 256), (0, 0, 0), 0.0),     # singular
    ((36, 20, 256), (3, 3, 0), 0.0),
])
def test_periodic_z_512_vs_oracle(dims, bcs, lam):
    """Periodic z with N = 512 and 256: the fused forward / division / inverse
    z pass of the TMA kernel on 16-line tiles with the spectrum held in
    registers between the transforms, the singular cases included."""
    p = gen.random_problem(*dims, *bcs, lam, seed=7 + sum(bcs))
    assert rel(gpu_solve(p), emulated(p)) < TOL


@pytest.mark.parametrize("xy", list(itertools.product(range(5), repeat=2)))
def test_config2_all_25_pairs_manufactured(xy):
    """The rectangular configuration's sweep: 256 x 192 x 320, every (x, y)
    code pair with z = 3 (the out-of-place, non-cubic path; the 192- and
    320-point axes on the generic mixed-radix kernel), lambda from the
    configuration's range.  f = A_h u, so the solve must return u itself."""
    import numpy as _np
    xbc, ybc = xy
    lam = float(_np.random.default_rng(1000 + 5 * xbc + ybc).uniform(-50.0, -0.5))
    p = gen.manufactured_problem(256, 192, 320, xbc, ybc, 3, lam, seed=40 + 5 * xbc + ybc)
    u = gpu_solve(p)
    w = stencil.window_slices(256, 192, 320, xbc, ybc, 3)
    assert rel(u[w], p["u_exact"][w]) < TOL
