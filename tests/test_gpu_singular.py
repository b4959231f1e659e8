"""GPU tests of the FISHPACK-compatible singular solve
(chz_helmholtz_solve_pertrb): for lambda = 0 with every code 0 or 3, PERTRB
equals hw3crt's (golden fixtures from a direct hw3crt call) and the solution
equals hw3crt's up to a constant; PERTRB is 0 when the problem is not
singular."""
import os

import numpy as np
import pytest
import torch

from oracle import gen, stencil
from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _solve(p):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    fc = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
          for k in stencil.FACE_KEYS}
    d = p["dom"]
    pert = api.helmholtz_solve_pertrb(d[0], d[1], p["nx"], p["xbc"], fc["bcl"], fc["bcr"],
                                      d[2], d[3], p["ny"], p["ybc"], fc["bcb"], fc["bct"],
                                      d[4], d[5], p["nz"], p["zbc"], fc["bcf"], fc["bce"], p["lam"], f)
    torch.cuda.synchronize()
    return f.cpu().numpy().reshape(p["nz"] + 1, p["ny"] + 1, p["nx"] + 1), pert


def test_pertrb_and_solution_match_fishpack():
    g = np.load(os.path.join(GOLDEN, "fishpack_singular.npz"))
    for t in range(len(g["pertrb"])):
        dims = tuple(int(v) for v in g["dims"][t])
        codes = tuple(int(v) for v in g["codes"][t])
        p = gen.random_problem(*dims, *codes, 0.0, int(g["seeds"][t]))
        u_ref = g["u"][g["offsets"][t]:g["offsets"][t + 1]].reshape(dims[2] + 1, dims[1] + 1, dims[0] + 1)
        u, pert = _solve(p)
        pert_ref = float(g["pertrb"][t])
        assert abs(pert - pert_ref) <= 1e-12 * max(1.0, abs(pert_ref)), (codes, pert, pert_ref)
        d = u - u_ref
        assert np.ptp(d) <= 1e-12 * np.linalg.norm(u_ref), (codes, np.ptp(d))


@pytest.mark.parametrize("dims,codes", [((128, 96, 64), (3, 0, 3)), ((64, 64, 256), (0, 0, 0))])
def test_pertrb_matches_oracle_larger(dims, codes):
    p = gen.random_problem(*dims, *codes, 0.0, seed=sum(dims))
    p["f"] = p["f"] + 0.3   # an incompatible (constant) part
    u, pert = _solve(p)
    ref = stencil.singular_pertrb(p)
    assert abs(pert - ref) <= 1e-12 * max(1.0, abs(ref))


def test_pertrb_zero_when_not_singular():
    p = gen.random_problem(32, 24, 40, 1, 3, 0, 0.0, seed=4)
    _, pert = _solve(p)
    assert pert == 0.0
    p = gen.random_problem(32, 24, 40, 3, 3, 3, -2.0, seed=4)
    _, pert = _solve(p)
    assert pert == 0.0
