"""Differentiable Helmholtz solve: a thin torch.autograd.Function over the C ABI.

Forward: chz_helmholtz_solve (FP64) or chz_helmholtz_solve_refined (FP32
transforms + FP64 refinement) on a copy of ``f``.  Backward:
chz_helmholtz_adjoint, which applies the transpose of the whole solve map
(f with its Dirichlet faces, the Neumann arrays, lambda) -> u; its adjoint
solve is the same diagonal solve between two scalings (A^-T = W A^-1 W^-1,
W = 1/2 at Neumann boundary nodes), in the forward pass's precision.
"""
from __future__ import annotations

from typing import Optional, Sequence

import torch

from . import _lib, api

FACE_KEYS = ("bcl", "bcr", "bcb", "bct", "bcf", "bce")


class _Spec:
    def __init__(self, dims, bcs, dom, precision, corrections):
        self.nx, self.ny, self.nz = (int(v) for v in dims)
        self.xbc, self.ybc, self.zbc = (int(v) for v in bcs)
        self.dom = tuple(float(v) for v in dom)
        self.precision = int(precision)
        self.corrections = int(corrections)


def _solve(spec: _Spec, f: torch.Tensor, faces, lam: float) -> None:
    d = spec.dom
    args = (d[0], d[1], spec.nx, spec.xbc, faces[0], faces[1],
            d[2], d[3], spec.ny, spec.ybc, faces[2], faces[3],
            d[4], d[5], spec.nz, spec.zbc, faces[4], faces[5], lam, f)
    if spec.precision == 0:
        api.cuda_helmholtz_solver(*args)
    else:
        api.helmholtz_solve_refined(*args, max_corrections=spec.corrections)


class HelmholtzSolveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, lam, bcl, bcr, bcb, bct, bcf, bce, spec):
        faces = (bcl, bcr, bcb, bct, bcf, bce)
        u = f.detach().contiguous().clone()
        lam_v = float(lam)
        _solve(spec, u, [None if t is None else t.detach().contiguous() for t in faces], lam_v)
        ctx.spec = spec
        ctx.lam = lam_v
        ctx.face_shapes = [None if t is None else t.shape for t in faces]
        ctx.lam_is_tensor = isinstance(lam, torch.Tensor)
        ctx.save_for_backward(u)
        return u

    @staticmethod
    def backward(ctx, gu):
        (u,) = ctx.saved_tensors
        spec = ctx.spec
        gu = gu.contiguous().to(torch.float64)
        df = torch.empty_like(u)
        dfaces = [None if shp is None else torch.empty(shp, dtype=torch.float64, device=u.device)
                  for shp in ctx.face_shapes]
        dlam = torch.zeros((), dtype=torch.float64, device=u.device)
        L = _lib.lib()
        nbytes = int(L.chz_helmholtz_adjoint_workspace_size(spec.nx, spec.ny, spec.nz, spec.precision))
        ws = torch.empty(nbytes // 8 + 64, dtype=torch.float64, device=u.device)
        base = ws.data_ptr()
        aligned = (base + 255) & ~255
        d = spec.dom
        st = L.chz_helmholtz_adjoint(
            d[0], d[1], spec.nx, spec.xbc, d[2], d[3], spec.ny, spec.ybc, d[4], d[5], spec.nz, spec.zbc,
            ctx.lam, gu.data_ptr(), u.data_ptr(), df.data_ptr(),
            *[0 if t is None else t.data_ptr() for t in dfaces],
            dlam.data_ptr(), spec.precision, spec.corrections, aligned,
            ws.numel() * 8 - (aligned - base), torch.cuda.current_stream().cuda_stream)
        api._check(st)
        grads_faces = [None if (t is None or not ctx.needs_input_grad[2 + q]) else t
                       for q, t in enumerate(dfaces)]
        dl = dlam if ctx.lam_is_tensor and ctx.needs_input_grad[1] else None
        return (df if ctx.needs_input_grad[0] else None, dl, *grads_faces, None)


def helmholtz_solve(f: torch.Tensor, lam, dims: Sequence[int], bcs: Sequence[int],
                    faces: Optional[dict] = None, dom=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0),
                    precision: int = 0, corrections: int = 2) -> torch.Tensor:
    """Differentiable solve of lap_h u + lam u = f (the reference's discrete
    system).  ``f``: CUDA float64 tensor of (NZ+1)(NY+1)(NX+1) values
    ([z][y][x], any shape with that many elements); ``lam``: float or 0-dim
    tensor; ``faces``: dict bcl..bce of Neumann arrays (tensors) as the codes
    need.  Returns u (same layout as f); gradients flow to f, lam and faces.
    precision 0 = FP64, 1 = FP32 transforms + ``corrections`` FP64 refinements."""
    faces = faces or {}
    spec = _Spec(dims, bcs, dom, precision, corrections)
    ft = [faces.get(k) for k in FACE_KEYS]
    return HelmholtzSolveFunction.apply(f, lam, *ft, spec)


# ---------------------------------------------------------------------------
# do_transform as a differentiable function
# ---------------------------------------------------------------------------
#
# Each kind is a matrix from its input window to its output window
# (funcinterface.cu:25-40 and the per-kind files cudasymmfft/dst1..dct3,
# dftfunc.cu; the formulas with the reference's "half FFTW" scaling); its
# transpose is another kind between two diagonal scalings along the line:
#   DST_1^T = DST_1                     DCT_1^T = W DCT_1 W^-1 (W = 1/2 at 0, N)
#   DST_2^T g = DST_3(g; g[0] = 0, g[N] doubled)
#   DST_3^T g = DST_2(g) with entry N halved and copied to entry 0 (DST_3 also
#               reads x[0] through its 1/2 (x[0] + x[N]) term)
#   DCT_2^T g = DCT_3(g with g[0] doubled)      DCT_3^T g = DCT_2(g), entry 0 halved
#   R2C^T g = C2R(g with the interior bins halved)
#   C2R^T g = R2C(g) with the interior bins doubled
# The 3-D transform is the tensor product of the three axes' matrices, so its
# transpose applies the three transposes (each axis' scalings commute with the
# other axes' transforms).

from .api import (DCT_1, DCT_2, DCT_3, DST_1, DST_2, DST_3, DFT_C2R, DFT_R2C,  # noqa: E402
                  do_transform, padded_numel)

_ADJOINT_KIND = {DST_1: DST_1, DST_2: DST_3, DST_3: DST_2, DCT_1: DCT_1, DCT_2: DCT_3, DCT_3: DCT_2,
                 DFT_R2C: DFT_C2R, DFT_C2R: DFT_R2C}


# input and output windows [lo, hi] of each kind on a padded line of N + 2
# entries (the per-kind pre/post kernels' loads and stores, dst1..dct3 and
# dftfunc.cu; an out-of-place transform leaves intermediate values elsewhere)
_IN_WIN = {DST_1: lambda n: (1, n - 1), DST_2: lambda n: (1, n), DST_3: lambda n: (0, n),
           DCT_1: lambda n: (0, n), DCT_2: lambda n: (0, n - 1), DCT_3: lambda n: (0, n - 1),
           DFT_R2C: lambda n: (0, n - 1), DFT_C2R: lambda n: (0, n + 1)}
_OUT_WIN = {DST_1: lambda n: (0, n - 1), DST_2: lambda n: (0, n), DST_3: lambda n: (0, n),
            DCT_1: lambda n: (0, n), DCT_2: lambda n: (0, n - 1), DCT_3: lambda n: (0, n - 1),
            DFT_R2C: lambda n: (0, n + 1), DFT_C2R: lambda n: (0, n - 1)}


def _mask(win, n, device):
    lo, hi = win(n)
    m = torch.zeros(n + 2, dtype=torch.float64, device=device)
    m[lo:hi + 1] = 1.0
    return m


def _pre_weights(kind, n, device):
    """Scaling of the output gradient (length n + 2) before the adjoint kind."""
    w = torch.ones(n + 2, dtype=torch.float64, device=device)
    if kind == DST_2:
        w[0] = 0.0
        w[n] = 2.0
    elif kind == DCT_1:
        w[0] = 2.0
        w[n] = 2.0
    elif kind == DCT_2:
        w[0] = 2.0
    elif kind == DFT_R2C:
        w[2:n] = 0.5
    return w


def _post_weights(kind, n, device):
    """Scaling of the adjoint kind's output (length n + 2)."""
    w = torch.ones(n + 2, dtype=torch.float64, device=device)
    if kind == DST_3:
        w[n] = 0.5
    elif kind == DCT_1:
        w[0] = 0.5
        w[n] = 0.5
    elif kind == DCT_3:
        w[0] = 0.5
    elif kind == DFT_C2R:
        w[2:n] = 2.0
        w[1] = 0.0
        w[n + 1] = 0.0
    return w


def _scale3(t, wx, wy, wz):
    return t * wz.view(-1, 1, 1) * wy.view(1, -1, 1) * wx.view(1, 1, -1)


class TransformFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, nx, ny, nz, kx, ky, kz):
        src = x.detach().contiguous().view(-1)
        out = torch.zeros(padded_numel(nx, ny, nz), dtype=torch.float64, device=x.device)
        do_transform(src, out, nx, ny, nz, kx, ky, kz)
        dev = x.device
        out = _scale3(out.view(nz + 2, ny + 2, nx + 2), _mask(_OUT_WIN[kx], nx, dev),
                      _mask(_OUT_WIN[ky], ny, dev), _mask(_OUT_WIN[kz], nz, dev))
        ctx.dims = (nx, ny, nz)
        ctx.kinds = (kx, ky, kz)
        return out.reshape(x.shape)

    @staticmethod
    def backward(ctx, g):
        nx, ny, nz = ctx.dims
        kx, ky, kz = ctx.kinds
        dev = g.device
        g3 = g.contiguous().view(nz + 2, ny + 2, nx + 2).to(torch.float64)
        gin = _scale3(g3, _pre_weights(kx, nx, dev), _pre_weights(ky, ny, dev), _pre_weights(kz, nz, dev))
        gin = gin.contiguous().view(-1)
        res = torch.zeros_like(gin)
        do_transform(gin, res, nx, ny, nz, _ADJOINT_KIND[kx], _ADJOINT_KIND[ky], _ADJOINT_KIND[kz])
        res = _scale3(res.view(nz + 2, ny + 2, nx + 2), _post_weights(kx, nx, dev) * _mask(_IN_WIN[kx], nx, dev),
                      _post_weights(ky, ny, dev) * _mask(_IN_WIN[ky], ny, dev),
                      _post_weights(kz, nz, dev) * _mask(_IN_WIN[kz], nz, dev))
        # DST_3 reads x[0] with the weight of x[N]
        if kx == DST_3:
            res[:, :, 0] = res[:, :, nx]
        if ky == DST_3:
            res[:, 0, :] = res[:, ny, :]
        if kz == DST_3:
            res[0, :, :] = res[nz, :, :]
        return res.reshape(g.shape), None, None, None, None, None, None


def transform(x: torch.Tensor, nx: int, ny: int, nz: int, kx: int, ky: int, kz: int) -> torch.Tensor:
    """Differentiable 3-D mixed transform (the reference's do_transform kinds)
    of the padded (NZ+2, NY+2, NX+2) float64 CUDA tensor ``x`` (any shape with
    that many elements), out of place: entries outside the kinds' output
    windows are 0 (where do_transform leaves them undefined), entries outside
    their input windows do not contribute (their gradient is 0)."""
    return TransformFunction.apply(x, nx, ny, nz, int(kx), int(ky), int(kz))
