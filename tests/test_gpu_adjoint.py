"""GPU tests of the adjoint solve (chz_helmholtz_adjoint) and the
torch.autograd wrapper over it.

(1) Dot-product identity: for fixed lambda the solve map
(f, Neumann faces) -> u is linear, so <g, M(df, dfaces)> must equal
<M^T g, (df, dfaces)> to round-off, for every boundary-code triple.
(2) Central finite differences (h = 1e-6, 16 random directions) of
L = 0.5 ||u - u_target||^2 with respect to f, the Neumann faces and lambda,
including the 256^3, BC (1, 3, 0), lambda = -4, f ~ N(0, 1) case, in FP64 and
with FP32 transforms + FP64 refinement."""
import itertools

import numpy as np
import pytest
import torch

from oracle import gen, stencil
from cuhelmholtz_b200 import api
from cuhelmholtz_b200.autograd import helmholtz_solve

pytestmark = pytest.mark.gpu

DOM = (0.0, 1.3, -0.5, 0.7, 0.0, 2.1)


def _face_tensors(nx, ny, nz, rng, requires_grad=False):
    shapes = stencil.face_shapes(nx, ny, nz)
    return {k: torch.tensor(rng.normal(size=int(np.prod(shapes[k]))), device="cuda",
                            requires_grad=requires_grad) for k in stencil.FACE_KEYS}


def _forward(f, faces, dims, bcs, lam, dom=DOM):
    u = f.detach().clone()
    nx, ny, nz = dims
    api.cuda_helmholtz_solver(dom[0], dom[1], nx, bcs[0], faces["bcl"], faces["bcr"],
                              dom[2], dom[3], ny, bcs[1], faces["bcb"], faces["bct"],
                              dom[4], dom[5], nz, bcs[2], faces["bcf"], faces["bce"], lam, u)
    return u


@pytest.mark.parametrize("bcs", list(itertools.product(range(5), repeat=3)))
def test_dot_product_identity(bcs):
    dims = (16, 12, 20)
    nx, ny, nz = dims
    # lambda = 0 with every code 0 or 3 exercises the zero-mode branch
    lam = 0.0 if sum(bcs) % 2 == 0 else -3.0
    rng = np.random.default_rng(1000 + 25 * bcs[0] + 5 * bcs[1] + bcs[2])
    n = (nx + 1) * (ny + 1) * (nz + 1)
    df_dir = torch.tensor(rng.normal(size=n), device="cuda")
    faces_dir = {k: v.detach() for k, v in _face_tensors(nx, ny, nz, rng).items()}
    g = torch.tensor(rng.normal(size=n), device="cuda")

    mu = _forward(df_dir, faces_dir, dims, bcs, lam)
    lhs = float(torch.dot(g, mu))

    f = torch.zeros(n, device="cuda", dtype=torch.float64, requires_grad=True)
    faces = {k: torch.zeros_like(v, requires_grad=True) for k, v in faces_dir.items()}
    u = helmholtz_solve(f, lam, dims, bcs, faces, DOM)
    grads = torch.autograd.grad(u, [f] + [faces[k] for k in stencil.FACE_KEYS], grad_outputs=g)
    rhs = float(torch.dot(grads[0], df_dir))
    for q, k in enumerate(stencil.FACE_KEYS):
        rhs += float(torch.dot(grads[1 + q], faces_dir[k]))
    scale = float(torch.linalg.norm(g) * torch.linalg.norm(mu))
    assert abs(lhs - rhs) <= 1e-12 * scale, (bcs, lhs, rhs, scale)


@pytest.mark.parametrize("dims,bcs,lam", [
    ((32, 24, 40), (3, 4, 0), -2.0),
    ((32, 32, 32), (1, 2, 4), -6.0),
    ((24, 40, 16), (0, 3, 3), 0.0),       # singular operator, zero mode removed
])
def test_dot_product_refined(dims, bcs, lam):
    """Adjoint through FP32 transforms + 3 FP64 corrections."""
    nx, ny, nz = dims
    rng = np.random.default_rng(77 + sum(dims))
    n = (nx + 1) * (ny + 1) * (nz + 1)
    df_dir = torch.tensor(rng.normal(size=n), device="cuda")
    faces_dir = {k: v.detach() for k, v in _face_tensors(nx, ny, nz, rng).items()}
    g = torch.tensor(rng.normal(size=n), device="cuda")
    mu = _forward(df_dir, faces_dir, dims, bcs, lam)
    lhs = float(torch.dot(g, mu))
    f = torch.zeros(n, device="cuda", dtype=torch.float64, requires_grad=True)
    faces = {k: torch.zeros_like(v, requires_grad=True) for k, v in faces_dir.items()}
    u = helmholtz_solve(f, lam, dims, bcs, faces, DOM, precision=1, corrections=3)
    grads = torch.autograd.grad(u, [f] + [faces[k] for k in stencil.FACE_KEYS], grad_outputs=g)
    rhs = float(torch.dot(grads[0], df_dir))
    for q, k in enumerate(stencil.FACE_KEYS):
        rhs += float(torch.dot(grads[1 + q], faces_dir[k]))
    scale = float(torch.linalg.norm(g) * torch.linalg.norm(mu))
    assert abs(lhs - rhs) <= 1e-11 * scale, (lhs, rhs, scale)


def _loss(u, ut):
    return 0.5 * torch.sum((u - ut) ** 2)


def _fd_check(dims, bcs, lam, f0, faces0, ut, precision, corrections, ndir=16, h=1e-6, dom=DOM,
              tol=1e-6, seed=3):
    """Central differences of L along ndir random directions in (f, faces)
    and along lambda, against the autograd gradients."""
    f = f0.clone().requires_grad_(True)
    faces = {k: v.clone().requires_grad_(True) for k, v in faces0.items()}
    lam_t = torch.tensor(lam, dtype=torch.float64, device="cuda", requires_grad=True)
    u = helmholtz_solve(f, lam_t, dims, bcs, faces, dom, precision=precision, corrections=corrections)
    _loss(u, ut).backward()
    keys = list(faces.keys())

    def L(fv, facev, lv):
        with torch.no_grad():
            return float(_loss(helmholtz_solve(fv, lv, dims, bcs, facev, dom, precision=precision,
                                               corrections=corrections), ut))

    rng = np.random.default_rng(seed)
    worst = 0.0
    for _ in range(ndir):
        v = torch.tensor(rng.normal(size=f.numel()), device="cuda")
        vf = {k: torch.tensor(rng.normal(size=faces[k].numel()), device="cuda") for k in keys}
        with torch.no_grad():
            fp = {k: faces0[k] + h * vf[k] for k in keys}
            fm = {k: faces0[k] - h * vf[k] for k in keys}
            fd = (L(f0 + h * v, fp, lam) - L(f0 - h * v, fm, lam)) / (2 * h)
            an = float(torch.dot(f.grad, v)) + sum(float(torch.dot(faces[k].grad, vf[k])) for k in keys)
        err = abs(fd - an) / max(abs(an), 1e-300)
        worst = max(worst, err)
        assert err <= tol, (fd, an, err)
    fd_l = (L(f0, faces0, lam + h) - L(f0, faces0, lam - h)) / (2 * h)
    an_l = float(lam_t.grad)
    err_l = abs(fd_l - an_l) / abs(an_l)
    assert err_l <= tol, (fd_l, an_l, err_l)
    return worst, err_l


@pytest.mark.parametrize("dims,bcs,lam", [
    ((32, 24, 40), (1, 3, 0), -4.0),
    ((32, 32, 32), (4, 2, 3), -9.0),
    ((24, 20, 16), (2, 0, 1), -1.5),
])
@pytest.mark.parametrize("precision", [0, 1])
def test_finite_differences_small(dims, bcs, lam, precision):
    nx, ny, nz = dims
    rng = np.random.default_rng(11 + sum(bcs))
    n = (nx + 1) * (ny + 1) * (nz + 1)
    f0 = torch.tensor(rng.normal(size=n), device="cuda")
    faces0 = {k: v.detach() for k, v in _face_tensors(nx, ny, nz, rng).items()}
    ut = torch.tensor(rng.normal(size=n), device="cuda")
    _fd_check(dims, bcs, lam, f0, faces0, ut, precision, 3, tol=1e-5)


@pytest.mark.parametrize("precision", [0, 1])
def test_finite_differences_256(precision):
    """256^3, BC (1, 3, 0), lambda = -4, f ~ N(0, 1), L = 0.5 ||u - u_target||^2."""
    p = gen.config5_problem()
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    f0 = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    faces0 = {k: torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda()
              for k in stencil.FACE_KEYS if p.get(k) is not None}
    ut = torch.from_numpy(np.ascontiguousarray(p["u_target"]).ravel()).cuda()
    worst, err_l = _fd_check((nx, ny, nz), (p["xbc"], p["ybc"], p["zbc"]), p["lam"], f0, faces0, ut,
                             precision, 3, dom=p["dom"], tol=1e-5)
    print(f"256^3 precision {precision}: worst directional rel err {worst:.2e}, dlambda rel err {err_l:.2e}")


def test_adjoint_rejects_bad_arguments():
    from cuhelmholtz_b200 import _lib
    L = _lib.lib()
    g = torch.zeros(17 * 13 * 21, dtype=torch.float64, device="cuda")
    ws = torch.empty(8, dtype=torch.float64, device="cuda")
    st = L.chz_helmholtz_adjoint(0.0, 1.0, 16, 1, 0.0, 1.0, 12, 1, 0.0, 1.0, 20, 1, -1.0,
                                 g.data_ptr(), g.data_ptr(), g.data_ptr(), None, None, None, None, None, None,
                                 None, 0, 0, ws.data_ptr(), 64, torch.cuda.current_stream().cuda_stream)
    assert st == api.CHZ_ERROR_WORKSPACE
    st = L.chz_helmholtz_adjoint(0.0, 1.0, 16, 7, 0.0, 1.0, 12, 1, 0.0, 1.0, 20, 1, -1.0,
                                 g.data_ptr(), g.data_ptr(), g.data_ptr(), None, None, None, None, None, None,
                                 None, 0, 0, ws.data_ptr(), 64, torch.cuda.current_stream().cuda_stream)
    assert st == api.CHZ_ERROR_INVALID_VALUE
