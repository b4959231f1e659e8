"""GPU tests of the batched solver (chz_batch_plan_create / chz_batch_solve):
many problems of uneven sizes, boundary codes and lambdas in one graph replay
-- of one persistent launch (a device work queue of pass tiles with per-problem
pass counters) or of one launch per pass, whichever the plan measured faster --
checked against one-at-a-time solves and the oracle."""
import numpy as np
import pytest
import torch

from oracle import emulation as E
from oracle import gen, stencil
from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu


def _dev(p):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    faces = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
             for k in stencil.FACE_KEYS}
    return f, faces


def _single(p):
    f, faces = _dev(p)
    d = p["dom"]
    api.cuda_helmholtz_solver(d[0], d[1], p["nx"], p["xbc"], faces["bcl"], faces["bcr"],
                              d[2], d[3], p["ny"], p["ybc"], faces["bcb"], faces["bct"],
                              d[4], d[5], p["nz"], p["zbc"], faces["bcf"], faces["bce"], p["lam"], f)
    torch.cuda.synchronize()
    return f.cpu().numpy()


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_batch_matches_single_solves_and_oracle():
    probs = gen.config4_problems(count=24, seed=9)
    plan = api.BatchPlan(probs)
    devs = [_dev(p) for p in probs]
    plan.solve([d[0] for d in devs], [d[1] for d in devs])
    torch.cuda.synchronize()
    for i, p in enumerate(probs):
        got = devs[i][0].cpu().numpy()
        assert _rel(got, _single(p)) < 1e-13, i
        if i < 4:
            d = p["dom"]
            ref = E.emulate_solver(d[0], d[1], p["nx"], p["xbc"], p["bcl"], p["bcr"], d[2], d[3], p["ny"],
                                   p["ybc"], p["bcb"], p["bct"], d[4], d[5], p["nz"], p["zbc"], p["bcf"],
                                   p["bce"], p["lam"], p["f"])
            assert _rel(got.reshape(ref.shape), ref) < 1e-12, i
    plan.close()


def test_batch_graph_replay_with_new_arrays():
    probs = [gen.random_problem(32, 48, 64, 1, 3, 0, -2.0, seed=1),
             gen.random_problem(64, 32, 48, 0, 2, 4, -0.3, seed=2),
             gen.random_problem(48, 48, 48, 3, 3, 3, -9.0, seed=3)]
    plan = api.BatchPlan(probs)
    for rep in range(2):
        devs = [_dev(p) for p in probs]
        plan.solve([d[0] for d in devs], [d[1] for d in devs])
        torch.cuda.synchronize()
        for i, p in enumerate(probs):
            assert _rel(devs[i][0].cpu().numpy(), _single(p)) < 1e-13, (rep, i)
    plan.close()


def test_config4_512_problems():
    """The batching configuration: 512 problems, sizes in {32, ..., 192}^3,
    codes uniform in 0..4, lambda log-uniform in [-100, -0.01]."""
    probs = gen.config4_problems(count=512, seed=4)
    plan = api.BatchPlan(probs)
    devs = [_dev(p) for p in probs]
    plan.solve([d[0] for d in devs], [d[1] for d in devs])
    torch.cuda.synchronize()
    for i in range(0, 512, 37):
        assert _rel(devs[i][0].cpu().numpy(), _single(probs[i])) < 1e-13, i
    plan.close()


def test_batch_rejects_bad_plans():
    with pytest.raises(api.CHZError):
        api.BatchPlan([dict(nx=8, ny=8, nz=8, xbc=5, ybc=1, zbc=1, lam=-1.0)])
    with pytest.raises(api.CHZError):
        api.BatchPlan([dict(nx=7, ny=8, nz=8, xbc=1, ybc=1, zbc=1, lam=-1.0)])


def test_autotuned_and_default_tiles_agree():
    """The autotuner picks a tile size per pass among 1024..16384 values per
    tile; the tuned plan and the untuned (4096 everywhere) plan give the same
    solves (1e-13), and both match single solves (1e-12)."""
    probs = gen.config4_problems(count=16, seed=13)
    tuned = api.BatchPlan(probs)
    targets, ms = tuned.tiles()
    assert all(t in (1024, 2048, 4096, 8192, 16384) for t in targets), targets
    assert all(m > 0 for m in ms), ms
    prev = api.BatchPlan.set_autotune(False)
    try:
        plain = api.BatchPlan(probs)
    finally:
        api.BatchPlan.set_autotune(prev)
    t2, ms2 = plain.tiles()
    assert t2 == [4096] * 5 and ms2 == [0.0] * 5
    a = [_dev(p) for p in probs]
    b = [_dev(p) for p in probs]
    tuned.solve([d[0] for d in a], [d[1] for d in a])
    plain.solve([d[0] for d in b], [d[1] for d in b])
    torch.cuda.synchronize()
    for p, da, db in zip(probs, a, b):
        ua, ub = da[0].cpu().numpy(), db[0].cpu().numpy()
        assert _rel(ua, ub) < 1e-13
        assert _rel(ua, _single(p)) < 1e-12


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_every_radix_schedule_matches_single_solves(variant):
    """Each radix schedule the autotuner chooses from (8s first; reversed; 4s
    for 8s) gives the single solves' results, over lengths with radices 2..11."""
    from cuhelmholtz_b200 import _lib
    probs = [gen.random_problem(nx, ny, nz, xbc, ybc, zbc, lam, seed=900 + i)
             for i, (nx, ny, nz, xbc, ybc, zbc, lam) in enumerate(
                 [(48, 80, 96, 0, 1, 2, -1.0), (112, 40, 64, 3, 4, 0, -2.5), (176, 56, 32, 2, 3, 1, -0.3),
                  (96, 144, 48, 4, 0, 3, -7.0), (160, 32, 88, 1, 2, 4, -0.05)])]
    prev = _lib.lib().chz_batch_set_radix_schedule(variant)
    prev_t = api.BatchPlan.set_autotune(False)
    try:
        plan = api.BatchPlan(probs)
    finally:
        api.BatchPlan.set_autotune(prev_t)
        _lib.lib().chz_batch_set_radix_schedule(prev)
    assert plan.radix_schedules() == [variant] * 5
    fs, faces = [], []
    for p in probs:
        f, fc = _dev(p)
        fs.append(f)
        faces.append(fc)
    plan.solve(fs, faces)
    api.stream_status()
    for p, f in zip(probs, fs):
        ref, rfc = _dev(p)
        api.solve_problem(p, ref, rfc)
        torch.cuda.synchronize()
        err = float(torch.linalg.vector_norm(f - ref) / torch.linalg.vector_norm(ref))
        assert err < 1e-12, (variant, p["nx"], p["ny"], p["nz"], err)
    plan.close()


def test_batch_is_one_launch_per_solve():
    from cuhelmholtz_b200 import _lib
    probs = [gen.random_problem(32 + 16 * (i % 4), 48, 40, i % 5, (i + 2) % 5, (i + 4) % 5, -1.5, seed=950 + i)
             for i in range(12)]
    plan = api.BatchPlan(probs)
    fs, faces = zip(*[_dev(p) for p in probs])
    plan.solve(list(fs), list(faces))
    torch.cuda.synchronize()
    n0 = _lib.launch_count()
    plan.solve(list(fs), list(faces))
    api.stream_status()
    assert _lib.launch_count() - n0 == 1
    plan.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_each_launch_form_matches_single_solves(mode):
    """Both launch forms (0: persistent work queue; 1: per pass, register-
    resident launches on groups of problems with the same line length and
    kinds and the generic kernel on the rest -- here N = 176 -- then the
    periodic planes) give the single solves' results, periodic axes
    included."""
    probs = [gen.random_problem(nx, ny, nz, xbc, ybc, zbc, lam, seed=970 + i)
             for i, (nx, ny, nz, xbc, ybc, zbc, lam) in enumerate(
                 [(48, 64, 32, 0, 0, 0, -1.0), (96, 40, 56, 1, 0, 3, -4.0), (32, 32, 144, 3, 4, 0, -0.2),
                  (80, 112, 48, 2, 1, 4, -9.0), (64, 48, 96, 0, 3, 2, -0.6), (176, 40, 48, 4, 2, 1, -2.5),
                  (96, 176, 96, 1, 1, 3, -0.8)])]
    prev = api.BatchPlan.set_launch_mode(mode)
    try:
        plan = api.BatchPlan(probs)
    finally:
        api.BatchPlan.set_launch_mode(prev)
    m, ms = plan.launch_mode()
    assert m == mode and ms == [0.0, 0.0]
    # kernels a solve replays: one persistent launch, or per pass the groups
    # (x forward alone has 5 (length, kind) groups here) plus the leftover
    # launch, then the periodic planes
    assert plan.kernels() == 1 if mode == 0 else plan.kernels() >= 5 + 5 + 1
    for _ in range(2):      # two graph replays, each on fresh copies of the right-hand sides
        fs, faces = zip(*[_dev(p) for p in probs])
        plan.solve(list(fs), list(faces))
        api.stream_status()
    for p, f in zip(probs, fs):
        ref = _single(p)
        assert _rel(f.cpu().numpy(), ref) < 1e-13, (mode, p["nx"], p["ny"], p["nz"])
    plan.close()


def test_plan_times_both_launch_forms():
    probs = gen.config4_problems(count=32, seed=21)
    plan = api.BatchPlan(probs)
    m, ms = plan.launch_mode()
    assert m in (0, 1) and ms[0] > 0 and ms[1] > 0
    assert ms[m] == min(ms)
    fs, faces = zip(*[_dev(p) for p in probs])
    plan.solve(list(fs), list(faces))
    api.stream_status()
    for i in (0, 13, 31):
        assert _rel(fs[i].cpu().numpy(), _single(probs[i])) < 1e-13, i
    plan.close()
