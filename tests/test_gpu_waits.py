"""GPU test of the bounded-wait failure path, with no GPU fault.

The pipelined kernels wait on mbarriers for tile copies and finished tiles;
every wait is bounded, and a wait that runs out raises a flag word that
chz_stream_status turns into CHZ_ERROR_TIMEOUT.  Here the self-test kernel
waits on a barrier that nothing arrives at (no copy is issued), with a short
limit; the status must report the timeout, the flag must be cleared by that
report, and the context must stay usable: a solve afterwards is correct and
reports success."""
import numpy as np
import pytest
import torch

from cuhelmholtz_b200 import api
from oracle import emulation as E
from oracle import gen
from oracle.stencil import FACE_KEYS

pytestmark = pytest.mark.gpu


def _solve(p):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    fc = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
          for k in FACE_KEYS}
    api.solve_problem(p, f, fc)
    return f


def test_wait_that_runs_out_surfaces_as_timeout_status():
    api.stream_status()                       # nothing pending
    api.wait_selftest(cycles=2_000_000)       # about a millisecond
    with pytest.raises(api.CHZError) as ei:
        api.stream_status()
    assert ei.value.status == api.CHZ_ERROR_TIMEOUT
    assert api.debug_flags(reset=False) == 0  # the report cleared the flags
    api.stream_status()                       # and the next check is clean

    # the context is still usable: a solve (TMA y and z passes at N = 128) is correct
    p = gen.random_problem(40, 128, 128, 1, 3, 0, -2.0, seed=71)
    u = _solve(p)
    api.stream_status()
    d = p["dom"]
    ref = E.emulate_solver(d[0], d[1], 40, 1, p["bcl"], p["bcr"], d[2], d[3], 128, 3, p["bcb"], p["bct"],
                           d[4], d[5], 128, 0, p["bcf"], p["bce"], p["lam"], p["f"])
    got = u.cpu().numpy().reshape(ref.shape)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


def test_wait_limit_setting_round_trips():
    prev = api.set_wait_limit(5_000_000)
    try:
        assert api.set_wait_limit(10) == 5_000_000       # below the floor: raised to 1e6
        assert api.set_wait_limit(0) == 1_000_000         # <= 0 restores the default
        p = gen.random_problem(32, 128, 64, 3, 3, 3, -1.0, seed=72)
        _solve(p)
        api.stream_status()
    finally:
        api.set_wait_limit(prev)
