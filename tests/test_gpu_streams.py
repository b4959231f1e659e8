"""GPU tests of stream ordering: solves and transforms issued on several
streams at once (each stream gets its own library workspace) give the same
results as one at a time."""
import numpy as np
import pytest
import torch

from oracle import gen, stencil
from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu


def _args(p, f, fc):
    d = p["dom"]
    return (d[0], d[1], p["nx"], p["xbc"], fc["bcl"], fc["bcr"], d[2], d[3], p["ny"], p["ybc"], fc["bcb"], fc["bct"],
            d[4], d[5], p["nz"], p["zbc"], fc["bcf"], fc["bce"], p["lam"], f)


def _dev(p):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    fc = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
          for k in stencil.FACE_KEYS}
    return f, fc


def test_concurrent_solves_on_four_streams():
    probs = [gen.random_problem(128, 96, 256, 1, 3, 0, -2.0, seed=1),
             gen.random_problem(256, 128, 128, 3, 4, 0, -1.0, seed=2),
             gen.random_problem(64, 160, 96, 2, 0, 4, -5.0, seed=3),
             gen.random_problem(128, 128, 128, 0, 0, 3, -0.5, seed=4)]
    # one at a time on the default stream
    ref = []
    for p in probs:
        f, fc = _dev(p)
        api.cuda_helmholtz_solver(*_args(p, f, fc))
        torch.cuda.synchronize()
        ref.append(f.cpu().numpy())
    # all at once, each on its own stream, three rounds
    streams = [torch.cuda.Stream() for _ in probs]
    devs = [_dev(p) for p in probs]
    for _ in range(3):
        fs = []
        for p, (f0, fc), s in zip(probs, devs, streams):
            with torch.cuda.stream(s):
                f = f0.clone()
                api.cuda_helmholtz_solver(*_args(p, f, fc), stream=s)
                api.helmholtz_solve_refined(*_args(p, f0.clone(), fc), max_corrections=1, stream=s)
                fs.append(f)
        torch.cuda.synchronize()
        for f, r in zip(fs, ref):
            assert np.array_equal(f.cpu().numpy(), r)


def test_concurrent_transforms_on_two_streams():
    rng = np.random.default_rng(5)
    n = 256
    shape = (n + 2) ** 3
    a = torch.tensor(rng.normal(size=shape), device="cuda")
    b = torch.tensor(rng.normal(size=shape), device="cuda")
    ra, rb = torch.zeros_like(a), torch.zeros_like(b)
    api.do_transform(a, ra, n, n, n, 6, 3, 1)
    api.do_transform(b, rb, n, n, n, 0, 2, 5)
    torch.cuda.synchronize()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    oa, ob = torch.zeros_like(a), torch.zeros_like(b)
    for _ in range(4):
        with torch.cuda.stream(s1):
            api.do_transform(a, oa, n, n, n, 6, 3, 1, stream=s1)
        with torch.cuda.stream(s2):
            api.do_transform(b, ob, n, n, n, 0, 2, 5, stream=s2)
    torch.cuda.synchronize()
    assert torch.equal(oa, ra) and torch.equal(ob, rb)
