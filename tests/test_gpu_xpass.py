"""GPU parity of the solver's x passes at N = 256 and 512, where the pipelined
contiguous kernel moves the right-hand side f (rows of N + 1 values, 8-byte
aligned) as one bulk span per tile and stores the solution rows back with
bulk copies of their 16-byte-aligned interiors plus plain stores of the ends.

Every x boundary code (its forward and inverse kinds), partial tiles (row
counts that are not multiples of the 16-line tile), and f at both 16-byte
phases (a view one value into a larger array) are compared with the oracle's
restatement of the reference solver, to 1e-12 relative."""
import numpy as np
import pytest
import torch

from cuhelmholtz_b200 import api
from oracle import emulation as E
from oracle import gen
from oracle.stencil import FACE_KEYS

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _solve(p, phase):
    n = p["f"].size
    base = torch.zeros(n + 2, dtype=torch.float64, device="cuda")
    f = base[phase:phase + n]
    assert f.data_ptr() % 16 == 8 * phase
    f.copy_(torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()))
    fc = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
          for k in FACE_KEYS}
    api.solve_problem(p, f, fc)
    api.stream_status()
    # the values around f are untouched
    assert float(base[:phase].abs().sum()) == 0.0
    assert float(base[phase + n:].abs().sum()) == 0.0
    return f.cpu().numpy().reshape(p["nz"] + 1, p["ny"] + 1, p["nx"] + 1)


def _oracle(p):
    d = p["dom"]
    return E.emulate_solver(d[0], d[1], p["nx"], p["xbc"], p["bcl"], p["bcr"], d[2], d[3], p["ny"], p["ybc"],
                            p["bcb"], p["bct"], d[4], d[5], p["nz"], p["zbc"], p["bcf"], p["bce"], p["lam"],
                            p["f"])


@pytest.mark.parametrize("n", [256, 512])
@pytest.mark.parametrize("phase", [0, 1])
@pytest.mark.parametrize("xbc,ybc,zbc", [(0, 1, 3), (1, 3, 0), (2, 4, 2), (3, 4, 0), (4, 0, 1)])
def test_x_pass_every_code(xbc, ybc, zbc, phase, n):
    p = gen.random_problem(n, 12, 20, xbc, ybc, zbc, -3.0, seed=600 + 10 * xbc + phase + n)
    got = _solve(p, phase)
    ref = _oracle(p)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < TOL, err


def test_x_pass_512_many_tiles():
    """Enough tiles for several per CTA (the three-stage pipeline wraps
    around: 4 tiles a plane x 160 planes over 148 CTAs) with a partial last
    tile in every plane (49 rows)."""
    p = gen.random_problem(512, 50, 160, 3, 1, 2, -1.5, seed=650)
    got = _solve(p, 1)
    ref = _oracle(p)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < TOL, err
