"""Test infrastructure: the local steps of the slab-decomposed solve restated
on the host (numpy), so the partition and the two all-to-all exchanges of
``cuhelmholtz_b200.slab`` can be checked across processes (``gloo``) without a
GPU.  Never part of the product: the GPU executor of ``cuhelmholtz_b200.slab``
runs the same steps through the C ABI.

The steps are the reference solver's (cuda_helmholtz_solver.cu:33-380 and
_cuda_helmholtz_.inl) cut at the z transform, exactly as ``emulation.
emulate_solver`` restates them for the whole grid:

* forward: boundary terms (_3d_bc{1..4}_ini_{x,y,z}_, inl:70-227) on the
  slab's unknown planes, the window copied into a zeroed padded array
  (_ini_ex_, inl:230-239), then the x and y forward kinds;
* z: the z forward kind, the division by the eigenvalues of the 7-point
  operator (_divide_ / _periodic_divide_, inl:276-421; the (0,0,0) mode set
  to 0 when the reference does), the z inverse kind;
* inverse: the y and x inverse kinds, the window scaled by the reference's
  ratio (_store_f_, inl:242-251, solver.cu:211-215), the x and y periodic
  copies (_3d_bc0_store_{x,y}_).
"""
from __future__ import annotations

import numpy as np
import torch

from . import emulation as E
from .stencil import FACE_KEYS

_PI = 3.14159265358979323846


def _axis(bc: int, n: int, lo: float, hi: float):
    s, e = E.solver_windows(bc, n)
    d = n / (hi - lo)
    shift = -0.5 * _PI / n if bc == 2 else (0.5 * _PI / n if bc == 4 else 0.0)
    pidiv = _PI / n * (2 if bc == 0 else 1)
    sp1 = n + 1 if bc == 0 else e
    kf, ki = E.solver_kinds(bc)
    return dict(n=n, bc=bc, s=s, e=e, sp0=s, sp1=sp1, d=d, d2=d * d, shift=shift, pidiv=pidiv, kf=kf, ki=ki)


def _entry_terms(a) -> tuple[np.ndarray, np.ndarray]:
    """Per padded entry of one axis: the eigenvalue term
    (2 cos(mode * pidiv + shift) - 2) / h^2 and whether the entry belongs to
    mode 0 (a periodic axis interleaves Re/Im: entries 2m, 2m + 1 are mode m)."""
    n = a["n"]
    idx = np.arange(n + 2)
    mode = idx // 2 if a["bc"] == 0 else idx
    term = (2 * np.cos(mode * a["pidiv"] + a["shift"]) - 2) * a["d2"]
    return term, mode == 0


def _along(arr: np.ndarray, axis: int, kind: int, n: int) -> np.ndarray:
    return np.moveaxis(E.emulate_kind(np.moveaxis(arr, axis, -1), kind, n), -1, axis)


class OracleExecutor:
    """Host restatement of GpuExecutor (same layout, same methods) over CPU
    torch tensors.  faces: the whole problem's face arrays (numpy or None)."""

    def __init__(self, layout, dom, lam, faces=None):
        self.L = layout
        nx, ny, nz = layout.nx, layout.ny, layout.nz
        xbc, ybc, zbc = layout.bcs
        self.lam = float(lam)
        self.X = _axis(xbc, nx, dom[0], dom[1])
        self.Y = _axis(ybc, ny, dom[2], dom[3])
        self.Z = _axis(zbc, nz, dom[4], dom[5])
        faces = faces or {}
        shp = {"bcl": (nz + 1, ny + 1), "bcr": (nz + 1, ny + 1), "bcb": (nz + 1, nx + 1),
               "bct": (nz + 1, nx + 1), "bcf": (ny + 1, nx + 1), "bce": (ny + 1, nx + 1)}
        self.faces = {k: (None if faces.get(k) is None else np.asarray(faces[k], dtype=np.float64).reshape(shp[k]))
                      for k in FACE_KEYS}

    def work_slab(self, r, device):
        _, nzl = self.L.planes[r]
        return torch.zeros((nzl, self.L.ny + 2, self.L.nx + 2), dtype=torch.float64, device=device)

    def pencil(self, q, device):
        return torch.empty((self.L.zcount, self.L.rows[q][1], self.L.nx + 2), dtype=torch.float64, device=device)

    def forward(self, r, f_slab: torch.Tensor, ws: torch.Tensor) -> None:
        L, X, Y, Z = self.L, self.X, self.Y, self.Z
        nx, ny, nz = L.nx, L.ny, L.nz
        z0, nzl = L.planes[r]
        k0, k1 = L.window_planes(r)
        if k1 < k0:
            return
        f = f_slab.numpy().reshape(nzl, ny + 1, nx + 1).copy()
        fc = self.faces
        K = slice(k0 - z0, k1 - z0 + 1)
        J = slice(Y["s"], Y["e"] + 1)
        I = slice(X["s"], X["e"] + 1)
        gk = np.arange(k0, k1 + 1)
        xs, xe, ys, ye = X["s"], X["e"], Y["s"], Y["e"]
        if X["bc"] in (1, 2):
            f[K, J, xs] -= f[K, J, 0] * X["d2"]
        if X["bc"] in (3, 4):
            f[K, J, xs] += 2 * fc["bcl"][gk][:, J] * X["d"]
        if X["bc"] in (1, 4):
            f[K, J, xe] -= f[K, J, nx] * X["d2"]
        if X["bc"] in (2, 3):
            f[K, J, xe] -= 2 * fc["bcr"][gk][:, J] * X["d"]
        if Y["bc"] in (1, 2):
            f[K, ys, I] -= f[K, 0, I] * Y["d2"]
        if Y["bc"] in (3, 4):
            f[K, ys, I] += 2 * fc["bcb"][gk][:, I] * Y["d"]
        if Y["bc"] in (1, 4):
            f[K, ye, I] -= f[K, ny, I] * Y["d2"]
        if Y["bc"] in (2, 3):
            f[K, ye, I] -= 2 * fc["bct"][gk][:, I] * Y["d"]
        zs, ze = Z["s"], Z["e"]
        if k0 <= zs <= k1:
            if Z["bc"] in (1, 2):
                f[zs - z0, J, I] -= f[0 - z0, J, I] * Z["d2"]
            if Z["bc"] in (3, 4):
                f[zs - z0, J, I] += 2 * fc["bcf"][J, I] * Z["d"]
        if k0 <= ze <= k1:
            if Z["bc"] in (1, 4):
                f[ze - z0, J, I] -= f[nz - z0, J, I] * Z["d2"]
            if Z["bc"] in (2, 3):
                f[ze - z0, J, I] -= 2 * fc["bce"][J, I] * Z["d"]
        ex = np.zeros((k1 - k0 + 1, ny + 2, nx + 2))
        ex[:, J, I] = f[K, J, I]
        ex = _along(ex, 2, X["kf"], nx)
        ex = _along(ex, 1, Y["kf"], ny)
        ws.numpy()[K] = ex

    def zpass(self, q, pencil: torch.Tensor) -> None:
        L, X, Y, Z = self.L, self.X, self.Y, self.Z
        nz = L.nz
        j0, nj = L.rows[q]
        pen = pencil.numpy()
        full = np.zeros((nz + 2, nj, L.nx + 2))
        full[Z["s"]:Z["e"] + 1] = pen
        full = _along(full, 0, Z["kf"], nz)
        tx, zx = _entry_terms(X)
        ty, zy = _entry_terms(Y)
        tz, zz = _entry_terms(Z)
        ty, zy = ty[j0:j0 + nj], zy[j0:j0 + nj]
        den = ((tx[None, None, :] + ty[None, :, None]) + tz[:, None, None]) + self.lam
        with np.errstate(divide="ignore"):
            eig = 1.0 / den
        perturb = self.lam == 0.0 and all(b in (0, 3) for b in L.bcs)
        if perturb:
            eig[np.ix_(zz, zy, zx)] = 0.0
        ks = slice(Z["sp0"], Z["sp1"] + 1)
        xs = slice(X["sp0"], X["sp1"] + 1)
        full[ks, :, xs] *= eig[ks, :, xs]
        full = _along(full, 0, Z["ki"], nz)
        pen[:] = full[Z["s"]:Z["e"] + 1]

    def inverse(self, r, ws: torch.Tensor, f_slab: torch.Tensor) -> None:
        L, X, Y, Z = self.L, self.X, self.Y, self.Z
        nx, ny, nz = L.nx, L.ny, L.nz
        z0, nzl = L.planes[r]
        k0, k1 = L.window_planes(r)
        f = f_slab.numpy().reshape(nzl, ny + 1, nx + 1)
        if k1 >= k0:
            K = slice(k0 - z0, k1 - z0 + 1)
            ex = ws.numpy()[K]
            ex = _along(ex, 1, Y["ki"], ny)
            ex = _along(ex, 2, X["ki"], nx)
            ratio = E._c_int_ratio(nx, ny, nz)
            for bc in L.bcs:
                if bc == 0:
                    ratio *= 2
            J = slice(Y["s"], Y["e"] + 1)
            I = slice(X["s"], X["e"] + 1)
            f[K, J, I] = ex[:, J, I] * (1.0 / float(ratio))
        if X["bc"] == 0:
            f[:, :, nx] = f[:, :, 0]
        if Y["bc"] == 0:
            f[:, ny, :] = f[:, 0, :]
