"""GPU tests of HostPipeline: solves of host right-hand sides with the copies
in, the solves and the copies out overlapped give, step by step, the same
arrays as synchronous solves, and they solve the problem (checked against the
oracle's residual)."""
import numpy as np
import pytest
import torch

from oracle import gen, stencil
from cuhelmholtz_b200 import api
from cuhelmholtz_b200.pipeline import HostPipeline

pytestmark = pytest.mark.gpu


def _host(a):
    return torch.from_numpy(np.ascontiguousarray(a).ravel()).pin_memory()


def _sync_solve(p, f_np, faces_h):
    d = p["dom"]
    f = torch.from_numpy(np.ascontiguousarray(f_np).ravel()).cuda()
    fc = {k: (None if v is None else v.cuda()) for k, v in faces_h.items()}
    api.cuda_helmholtz_solver(d[0], d[1], p["nx"], p["xbc"], fc["bcl"], fc["bcr"],
                              d[2], d[3], p["ny"], p["ybc"], fc["bcb"], fc["bct"],
                              d[4], d[5], p["nz"], p["zbc"], fc["bcf"], fc["bce"], p["lam"], f)
    torch.cuda.synchronize()
    return f.cpu().numpy()


@pytest.mark.parametrize("dims,bcs,lam,slots", [
    ((128, 96, 64), (3, 4, 0), -1.0, 2),
    ((64, 64, 64), (1, 3, 2), -3.0, 3),
    ((96, 128, 80), (0, 0, 3), -0.5, 2),
])
def test_pipeline_matches_synchronous(dims, bcs, lam, slots):
    nx, ny, nz = dims
    p = gen.random_problem(nx, ny, nz, *bcs, lam, seed=11)
    faces_h = {k: (None if p.get(k) is None else _host(p[k])) for k in stencil.FACE_KEYS}
    rng = np.random.default_rng(4)
    steps = 7
    fs_np = [p["f"] + rng.normal(size=p["f"].shape) for _ in range(steps)]
    f_hosts = [_host(f) for f in fs_np]
    u_hosts = [torch.empty_like(f_hosts[0]).pin_memory() for _ in range(steps)]
    pipe = HostPipeline(nx, ny, nz, bcs, p["dom"], lam, faces=faces_h, slots=slots)
    for _ in range(2):                       # the second pass reuses slots already used
        for u in u_hosts:
            u.fill_(np.nan)
        pipe.solve(f_hosts, u_hosts)
        pipe.join()
        torch.cuda.synchronize()
        for i in range(steps):
            ref = _sync_solve(p, fs_np[i], faces_h)
            assert np.array_equal(u_hosts[i].numpy(), ref), f"step {i}"
    h2d, d2h = pipe.bytes_per_step()
    assert d2h == (nx + 1) * (ny + 1) * (nz + 1) * 8
    assert h2d == d2h + sum(v.numel() * 8 for v in faces_h.values() if v is not None)
    # the last step's result solves its problem
    q = dict(p)
    q["f"] = fs_np[-1]
    u = u_hosts[-1].numpy().reshape(nz + 1, ny + 1, nx + 1)
    r = stencil.residual(u, q["f"], nx, ny, nz, *bcs, p["dom"], lam, {k: p.get(k) for k in stencil.FACE_KEYS})
    assert np.linalg.norm(r) / np.linalg.norm(q["f"]) < 1e-10


def test_pipeline_one_output_buffer_reused():
    # every step writes the same host buffer: the copies out are ordered on one
    # stream, so the buffer ends with the last step's result
    nx = ny = nz = 64
    p = gen.random_problem(nx, ny, nz, 1, 1, 1, -2.0, seed=2)
    faces_h = {k: None for k in stencil.FACE_KEYS}
    rng = np.random.default_rng(9)
    fs_np = [rng.normal(size=p["f"].shape) for _ in range(5)]
    u = torch.empty((nx + 1) * (ny + 1) * (nz + 1), dtype=torch.float64).pin_memory()
    pipe = HostPipeline(nx, ny, nz, (1, 1, 1), p["dom"], -2.0, faces=faces_h)
    pipe.solve([_host(f) for f in fs_np], [u] * 5)
    pipe.join()
    torch.cuda.synchronize()
    assert np.array_equal(u.numpy(), _sync_solve(p, fs_np[-1], faces_h))
