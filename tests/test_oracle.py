"""CPU tests of the oracle: the line-by-line restatement of the reference GPU
path (oracle.emulation) against the textbook transforms (oracle.closed_form),
against the reference's own CPU solver (FISHPACK hw3crt via solver_3d) through
the committed golden fixtures, and against manufactured discrete solutions."""
import itertools
import os

import numpy as np
import pytest

from oracle import closed_form as C
from oracle import emulation as E
from oracle import gen, stencil

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _relmax(a, b):
    m = ~np.isnan(b)
    return np.abs(a[m] - b[m]).max() / max(1.0, np.abs(b[m]).max())


@pytest.mark.parametrize("n", [4, 6, 8, 10, 16, 24, 48, 64, 96])
@pytest.mark.parametrize("kind", range(8))
def test_kind_matches_closed_form(n, kind):
    rng = np.random.default_rng(100 + n * 8 + kind)
    x = rng.normal(size=(7, n + 2))
    a = E.emulate_kind(x, kind, n)
    b = C.closed_kind(x, kind, n)
    assert np.array_equal(np.isnan(a), np.isnan(b)), "defined windows differ"
    assert _relmax(a, b) < 1e-13


@pytest.mark.parametrize("dims", [(8, 6, 10), (8, 8, 8), (12, 4, 6)])
def test_3d_emulation_matches_separable_closed_form(dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(7)
    for kx, ky, kz in itertools.product(range(8), repeat=3):
        d = rng.normal(size=E.padded_shape(nx, ny, nz))
        a = E.emulate_do_transform(d, nx, ny, nz, kx, ky, kz)
        b = C.closed_do_transform(d, nx, ny, nz, kx, ky, kz)
        m = ~np.isnan(a)
        assert m.any()
        # wherever the reference defines a value, it is the separable transform
        # (C2R reads the imaginary parts of bins 0 and N/2 as zero in both)
        err = np.abs(a[m] - b[m]).max() / max(1.0, np.abs(b[m]).max())
        assert err < 1e-12, (kx, ky, kz, err)


def _solve_emulated(p):
    d = p["dom"]
    return E.emulate_solver(d[0], d[1], p["nx"], p["xbc"], p["bcl"], p["bcr"],
                            d[2], d[3], p["ny"], p["ybc"], p["bcb"], p["bct"],
                            d[4], d[5], p["nz"], p["zbc"], p["bcf"], p["bce"],
                            p["lam"], p["f"])


def _load_golden(name):
    path = os.path.join(GOLDEN, name)
    assert os.path.exists(path), f"missing fixture {path}"
    return np.load(path)


def test_fixture_inputs_regenerate():
    """The fixtures store seeds; the generator must reproduce the inputs."""
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import SWEEP_DIMS, input_digest, sweep_case  # noqa: E402
    g = _load_golden("fishpack_sweep_10x6x8.npz")
    for t in (0, 17, 62, 124):
        xbc, ybc, zbc = (int(v) for v in g["triples"][t])
        p = sweep_case(*SWEEP_DIMS, xbc, ybc, zbc, float(g["lam"]), int(g["seeds"][t]))
        assert input_digest(p) == str(g["digests"][t])


def test_emulated_solver_matches_fishpack_all_125_triples():
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import SWEEP_DIMS, sweep_case  # noqa: E402
    g = _load_golden("fishpack_sweep_10x6x8.npz")
    worst = 0.0
    for t, trip in enumerate(g["triples"]):
        xbc, ybc, zbc = (int(v) for v in trip)
        p = sweep_case(*SWEEP_DIMS, xbc, ybc, zbc, float(g["lam"]), int(g["seeds"][t]))
        u = _solve_emulated(p)
        assert not np.isnan(u).any()
        ref = g["u"][t]
        rel = np.linalg.norm(u - ref) / np.linalg.norm(ref)
        worst = max(worst, rel)
        assert rel < 1e-12, ((xbc, ybc, zbc), rel)
    assert worst < 1e-12


def test_emulated_solver_matches_fishpack_16x12x20():
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import MID_DIMS, sweep_case  # noqa: E402
    g = _load_golden("fishpack_16x12x20.npz")
    for t, case in enumerate(g["cases"]):
        xbc, ybc, zbc = (int(v) for v in case[:3])
        p = sweep_case(*MID_DIMS, xbc, ybc, zbc, float(case[3]), int(g["seeds"][t]))
        u = _solve_emulated(p)
        ref = g["u"][t]
        assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-12


def test_analytic_case1_matches_fishpack_truncation_error():
    """The reference's own test (ufunc.h case 1): the max-norm error against the
    continuous solution equals fishpack's to many digits."""
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import ufunc_problem  # noqa: E402
    g = _load_golden("fishpack_ufunc_case1.npz")
    for row in g["cases"]:
        dims = tuple(int(v) for v in row[:3])
        bcs = tuple(int(v) for v in row[3:6])
        p = ufunc_problem(*dims, *bcs)
        u = _solve_emulated(p)
        maxdiff = np.abs(u - p["u_exact"]).max()
        assert abs(maxdiff - row[6]) <= 1e-10 * max(1.0, row[6]) + 1e-13
    # O(h^2): the 32^3 (1,2,0) error is ~1e-3, as the survey measured
    assert 5e-4 < g["cases"][0][6] < 2e-3


@pytest.mark.parametrize("bcs", list(itertools.product(range(5), repeat=3))[::7])
def test_manufactured_discrete_solution_recovered(bcs):
    p = gen.manufactured_problem(16, 12, 20, *bcs, -2.5, seed=3)
    u = _solve_emulated(p)
    w = stencil.window_slices(16, 12, 20, *bcs)
    assert np.linalg.norm(u[w] - p["u_exact"][w]) / np.linalg.norm(p["u_exact"][w]) < 1e-12


def test_residual_of_emulated_solution_is_small():
    p = gen.random_problem(16, 12, 8, 3, 4, 0, -1.0, seed=9)
    u = _solve_emulated(p)
    faces = {k: p[k] for k in stencil.FACE_KEYS}
    r = stencil.residual(u, p["f"], 16, 12, 8, 3, 4, 0, p["dom"], p["lam"], faces)
    assert np.linalg.norm(r) / np.linalg.norm(p["f"]) < 1e-12


def test_oracle_rejects_bad_boundary_code():
    with pytest.raises(ValueError):
        E.solver_windows(5, 8)


def _singular_cases():
    g = _load_golden("fishpack_singular.npz")
    out = []
    for t in range(len(g["pertrb"])):
        dims = tuple(int(v) for v in g["dims"][t])
        codes = tuple(int(v) for v in g["codes"][t])
        p = gen.random_problem(*dims, *codes, 0.0, int(g["seeds"][t]))
        u = g["u"][g["offsets"][t]:g["offsets"][t + 1]].reshape(dims[2] + 1, dims[1] + 1, dims[0] + 1)
        out.append((p, u, float(g["pertrb"][t]), str(g["digests"][t])))
    return out


def test_singular_pertrb_matches_fishpack():
    """lambda = 0, every code 0 or 3: the oracle's PERTRB (weighted mean of the
    right-hand side) equals hw3crt's, and the reference GPU path's zero-mode
    solution differs from hw3crt's unnormalised one by a constant only."""
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import input_digest  # noqa: E402
    for p, u_ref, pert_ref, digest in _singular_cases():
        assert input_digest(p) == digest
        pert = stencil.singular_pertrb(p)
        assert abs(pert - pert_ref) <= 1e-12 * max(1.0, abs(pert_ref)), (pert, pert_ref)
        d = _solve_emulated(p) - u_ref
        assert np.ptp(d) <= 1e-12 * np.linalg.norm(u_ref), np.ptp(d)


def test_pertrb_is_zero_when_not_singular():
    p = gen.random_problem(16, 12, 20, 1, 3, 3, 0.0, seed=1)
    assert stencil.singular_pertrb(p) == 0.0
    p = gen.random_problem(16, 12, 20, 3, 3, 3, -1.0, seed=1)
    assert stencil.singular_pertrb(p) == 0.0


def _rhs_with_terms(p):
    """b = f + boundary terms on the unknown window (the 7-point solve's)."""
    n = (p["nx"], p["ny"], p["nz"])
    codes = (p["xbc"], p["ybc"], p["zbc"])
    d = p["dom"]
    w = stencil.window_slices(*n, *codes)
    f = np.asarray(p["f"], dtype=np.float64)
    neumann = -stencil.apply_operator(np.zeros_like(f), *n, *codes, d, 0.0,
                                      {k: p.get(k) for k in stencil.FACE_KEYS})
    outside = np.zeros_like(f)
    mask = np.ones(f.shape, dtype=bool)
    mask[w] = False
    outside[mask] = f[mask]
    dirichlet = np.nan_to_num(stencil.apply_operator(outside, *n, *codes, d, 0.0,
                                                     {k: None for k in stencil.FACE_KEYS}))
    return (f + neumann - dirichlet)[w], w


@pytest.mark.parametrize("codes,lam", [((1, 1, 1), 0.0), ((3, 1, 3), -2.0), ((3, 3, 3), -1.5),
                                       ((1, 3, 1), 0.0)])
def test_19pt_emulation_solves_the_compact_scheme(codes, lam):
    """The reference's 19-point division (dead code in the reference, no
    outputs to pin against) is the compact fourth-order scheme: the emulated
    solution satisfies (L19 + lambda) u = B b on the window, L19 the 19-point
    Laplacian and B the 7-point right-hand-side filter, with the closures the
    transforms imply."""
    n = (12, 16, 10)
    p = gen.random_problem(*n, *codes, lam, seed=7, dom=(0.0, 1.2, 0.0, 1.6, 0.0, 1.0))
    d = p["dom"]
    u = E.emulate_solver(d[0], d[1], p["nx"], p["xbc"], p["bcl"], p["bcr"],
                         d[2], d[3], p["ny"], p["ybc"], p["bcb"], p["bct"],
                         d[4], d[5], p["nz"], p["zbc"], p["bcf"], p["bce"], p["lam"], p["f"], stencil19=True)
    b, w = _rhs_with_terms(p)
    h2 = (n[0] / 1.2) ** 2
    lhs = stencil.apply_19pt(u[w], codes, h2) + lam * u[w]
    rhs = stencil.filter_19pt(b, codes)
    assert np.linalg.norm(lhs - rhs) <= 1e-13 * np.linalg.norm(rhs)
