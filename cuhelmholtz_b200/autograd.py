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
