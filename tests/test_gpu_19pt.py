"""GPU tests of the 19-point variant (chz_helmholtz_solve_19pt) against the
oracle's restatement of the reference's _nonpoisson_devide_19points_, which
itself is checked to solve the compact fourth-order scheme."""
import numpy as np
import pytest
import torch

from oracle import emulation as E
from oracle import gen, stencil
from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu


def _solve(p):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    fc = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
          for k in stencil.FACE_KEYS}
    d = p["dom"]
    api.helmholtz_solve_19pt(d[0], d[1], p["nx"], p["xbc"], fc["bcl"], fc["bcr"],
                             d[2], d[3], p["ny"], p["ybc"], fc["bcb"], fc["bct"],
                             d[4], d[5], p["nz"], p["zbc"], fc["bcf"], fc["bce"], p["lam"], f)
    torch.cuda.synchronize()
    return f.cpu().numpy().reshape(p["nz"] + 1, p["ny"] + 1, p["nx"] + 1)


def _emulated(p):
    d = p["dom"]
    return E.emulate_solver(d[0], d[1], p["nx"], p["xbc"], p["bcl"], p["bcr"],
                            d[2], d[3], p["ny"], p["ybc"], p["bcb"], p["bct"],
                            d[4], d[5], p["nz"], p["zbc"], p["bcf"], p["bce"], p["lam"], p["f"], stencil19=True)


@pytest.mark.parametrize("dims,codes,lam", [
    ((32, 24, 40), (1, 3, 1), -2.0),
    ((64, 64, 64), (3, 3, 1), 0.0),
    ((128, 96, 256), (1, 1, 3), -7.0),   # TMA y/z passes
    ((48, 80, 32), (3, 1, 3), -0.5),     # mixed-radix lengths
])
def test_19pt_matches_oracle(dims, codes, lam):
    n = dims
    # one grid spacing on every axis: domain lengths proportional to the cell counts
    dom = (0.0, n[0] / 64.0, 0.0, n[1] / 64.0, 0.0, n[2] / 64.0)
    p = gen.random_problem(*n, *codes, lam, seed=sum(n), dom=dom)
    u = _solve(p)
    ref = _emulated(p)
    assert np.linalg.norm(u - ref) <= 1e-12 * np.linalg.norm(ref)


def test_19pt_zero_mode_is_finite():
    n = (32, 32, 32)
    p = gen.random_problem(*n, 3, 3, 3, 0.0, seed=2)
    u = _solve(p)
    assert np.isfinite(u).all()


def test_19pt_rejects_what_the_reference_kernel_does_not_cover():
    f = torch.zeros(17 * 17 * 17, dtype=torch.float64, device="cuda")
    with pytest.raises(api.CHZError):   # periodic axis
        api.helmholtz_solve_19pt(0, 1, 16, 0, None, None, 0, 1, 16, 1, None, None, 0, 1, 16, 1, None, None,
                                 -1.0, f)
    with pytest.raises(api.CHZError):   # unequal spacing
        api.helmholtz_solve_19pt(0, 2, 16, 1, None, None, 0, 1, 16, 1, None, None, 0, 1, 16, 1, None, None,
                                 -1.0, f)
