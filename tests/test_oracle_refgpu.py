"""The oracle pinned to the reference's own GPU path (CPU tests).

tests/golden/cudaref_*.npz hold outputs of the reference's cudasymmfft
do_transform over cuFFT and of its cuda_helmholtz_solver, compiled unchanged
and run on a B200 by make_reference_gpu_golden.py.  The oracle's restatement
(oracle/emulation.py) must reproduce them on every entry the reference
defines, and the reference GPU solver must agree with the reference CPU solver
(FISHPACK, tests/golden/fishpack_*.npz) on the same inputs -- three
implementations of one discrete system."""
import os
import sys

import numpy as np
import pytest

from oracle import emulation as E

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLDEN)
from make_golden import MID_DIMS, SWEEP_DIMS, input_digest, sweep_case  # noqa: E402
from make_reference_gpu_golden import array_digest, transform_input  # noqa: E402

TOL = 1e-12
TRANSFORM = os.path.join(GOLDEN, "cudaref_transform.npz")
SOLVE = os.path.join(GOLDEN, "cudaref_solve.npz")


@pytest.mark.parametrize("group", ["cube8", "cube12", "box8x6x10", "box12x16x20"])
def test_emulation_matches_reference_gpu_transform(group):
    g = np.load(TRANSFORM)
    nx, ny, nz = (int(v) for v in g[f"{group}_dims"])
    for kinds, seed, digest, ref in zip(g[f"{group}_kinds"], g[f"{group}_seeds"], g[f"{group}_digests"],
                                        g[f"{group}_out"]):
        h = transform_input((nx, ny, nz), int(seed))
        assert array_digest(h) == str(digest)
        emu = E.emulate_do_transform(h, nx, ny, nz, *(int(k) for k in kinds))
        m = ~np.isnan(emu)
        assert m.any()
        scale = max(1.0, np.abs(ref[m]).max())
        err = np.abs(emu[m] - ref[m]).max() / scale
        assert err < TOL, (group, tuple(kinds), err)


def test_emulation_matches_reference_gpu_solver():
    g = np.load(SOLVE)
    lam = float(g["sweep_lam"])
    for t, (xbc, ybc, zbc) in enumerate(g["sweep_triples"]):
        p = sweep_case(*SWEEP_DIMS, int(xbc), int(ybc), int(zbc), lam, int(g["sweep_seeds"][t]))
        assert input_digest(p) == str(g["sweep_digests"][t])
        d = p["dom"]
        emu = E.emulate_solver(d[0], d[1], p["nx"], p["xbc"], p["bcl"], p["bcr"], d[2], d[3], p["ny"], p["ybc"],
                               p["bcb"], p["bct"], d[4], d[5], p["nz"], p["zbc"], p["bcf"], p["bce"], p["lam"],
                               p["f"])
        ref = g["sweep_u"][t]
        assert np.linalg.norm(emu - ref) / np.linalg.norm(ref) < TOL, (xbc, ybc, zbc)


def test_reference_gpu_solver_matches_fishpack():
    """Reference GPU solver vs reference CPU solver on the FISHPACK fixtures'
    own inputs (the sweep: all 125 codes triples; 16x12x20 mixed cases)."""
    g = np.load(SOLVE)
    fp = np.load(os.path.join(GOLDEN, "fishpack_sweep_10x6x8.npz"))
    assert np.array_equal(fp["seeds"], g["sweep_seeds"])
    for t in range(len(g["sweep_triples"])):
        ref = fp["u"][t]
        assert np.linalg.norm(g["sweep_u"][t] - ref) / np.linalg.norm(ref) < TOL
    mid = np.load(os.path.join(GOLDEN, "fishpack_16x12x20.npz"))
    assert np.array_equal(mid["seeds"], g["mid_seeds"])
    for t in range(len(g["mid_cases"])):
        ref = mid["u"][t]
        assert np.linalg.norm(g["mid_u"][t] - ref) / np.linalg.norm(ref) < TOL
    assert tuple(g["mid_dims"]) == tuple(MID_DIMS)
