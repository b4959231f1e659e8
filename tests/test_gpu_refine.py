"""GPU tests of the FP32-transform solve with FP64-residual iterative
refinement (chz_helmholtz_solve_refined, through the C ABI).  The reference is
the FP64 solve on the same input (itself checked against the oracle in
test_gpu_solver.py); the target is 1e-12 relative L2."""
import numpy as np
import pytest
import torch

from oracle import gen, stencil
from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _dev(p):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    faces = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
             for k in stencil.FACE_KEYS}
    return f, faces


def _args(p, faces):
    d = p["dom"]
    return (d[0], d[1], p["nx"], p["xbc"], faces["bcl"], faces["bcr"],
            d[2], d[3], p["ny"], p["ybc"], faces["bcb"], faces["bct"],
            d[4], d[5], p["nz"], p["zbc"], faces["bcf"], faces["bce"], p["lam"])


def fp64(p):
    f, faces = _dev(p)
    api.cuda_helmholtz_solver(*_args(p, faces), f)
    torch.cuda.synchronize()
    return f.cpu().numpy()


def refined(p, k, tol=0.0, report=False):
    f, faces = _dev(p)
    done, rr = api.helmholtz_solve_refined(*_args(p, faces), f, max_corrections=k, tol=tol, report=report)
    torch.cuda.synchronize()
    return f.cpu().numpy(), done, rr


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("dims,bcs,lam", [
    ((64, 48, 80), (3, 4, 0), -1.0),
    ((64, 64, 64), (1, 2, 0), -2.0),
    ((32, 64, 128), (0, 0, 0), -0.5),
    ((48, 40, 56), (2, 1, 4), -7.5),      # mixed-radix kernels
    ((128, 32, 64), (4, 3, 2), -100.0),
    ((64, 64, 32), (1, 3, 0), -4.0),
    ((40, 24, 512), (3, 4, 0), -1.0),     # periodic z at N = 512: fused FP32 z pass, pairs through shared memory
    ((72, 8, 512), (1, 0, 0), -3.0),
    ((24, 40, 256), (1, 3, 0), -4.0),     # the same at N = 256
])
def test_refinement_reaches_fp64(dims, bcs, lam):
    p = gen.random_problem(*dims, *bcs, lam, seed=sum(dims) + 7 * sum(bcs))
    ref = fp64(p)
    errs = []
    for k in (0, 1, 2):
        u, done, _ = refined(p, k)
        assert done == k
        errs.append(rel(u, ref))
    assert 1e-9 < errs[0] < 1e-5, errs     # FP32 alone
    assert errs[1] < errs[0] * 1e-3, errs  # each correction gains ~FP32 precision
    assert errs[2] < TOL, errs


@pytest.mark.parametrize("dims,bcs", [((24, 40, 16), (0, 3, 3)), ((32, 32, 32), (0, 0, 0)),
                                       ((48, 32, 40), (3, 3, 3))])
def test_refinement_singular(dims, bcs):
    """lambda = 0 with every code 0 or 3: the constant mode is removed as in the
    FP64 solve, and the incompatible part of b does not stall the refinement."""
    p = gen.random_problem(*dims, *bcs, 0.0, seed=sum(dims))
    p["f"] = p["f"] + 0.7   # a large incompatible (constant) part
    ref = fp64(p)
    u, done, _ = refined(p, 3)
    assert done == 3
    assert rel(u, ref) < TOL, rel(u, ref)


def test_tolerance_mode_stops_and_reports():
    p = gen.random_problem(64, 64, 64, 3, 4, 0, -1.0, seed=3)
    ref = fp64(p)
    u, done, rr = refined(p, 8, tol=1e-12, report=True)
    assert 1 <= done <= 4
    assert 0.0 <= rr
    assert rel(u, ref) < TOL


def test_config3_512_refined_vs_fp64():
    """Precision configuration: 512^3, codes (3,4,0), lambda = -1, f ~ U[-1,1]
    plus a 1e3 smooth mode.  Two corrections reach the FP64 solve to 1e-12."""
    p = gen.config3_problem(seed=3, n=512)
    ref = fp64(p)
    u, done, _ = refined(p, 2)
    err = rel(u, ref)
    assert err < TOL, err


def test_refined_rejects_bad_arguments():
    f = torch.zeros(9 * 9 * 9, dtype=torch.float64, device="cuda")
    with pytest.raises(api.CHZError):
        api.helmholtz_solve_refined(0, 1, 8, 1, None, None, 0, 1, 8, 1, None, None, 0, 1, 8, 1,
                                    None, None, -1.0, f, max_corrections=-1)
