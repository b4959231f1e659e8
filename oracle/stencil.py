"""7-point discrete Helmholtz operator with the reference's boundary closures
(test infrastructure).

The reference solver (cuda_helmholtz_solver.cu:33-380) solves, on the unknown
window of each axis (solver_windows), the vertex-centred system

    (u[i-1] - 2u[i] + u[i+1]) / h^2  (summed over x, y, z)  + lambda u[i] = f[i]

with: periodic wrap u[-1] = u[N-1], u[N] = u[0] (code 0); Dirichlet face values
taken from f's face planes (codes 1, 2 left; 1, 4 right); Neumann ghost points
u[-1] = u[1] - 2h g_left, u[N+1] = u[N-1] + 2h g_right (codes 3, 4 left; 2, 3
right) -- the closures its boundary-term kernels _3d_bc*_ini_* imply
(_cuda_helmholtz_.inl:70-227).
"""
from __future__ import annotations

import numpy as np

from .emulation import solver_windows

FACE_KEYS = ("bcl", "bcr", "bcb", "bct", "bcf", "bce")


def face_shapes(nx, ny, nz):
    return {"bcl": (nz + 1, ny + 1), "bcr": (nz + 1, ny + 1),
            "bcb": (nz + 1, nx + 1), "bct": (nz + 1, nx + 1),
            "bcf": (ny + 1, nx + 1), "bce": (ny + 1, nx + 1)}


def used_faces(xbc, ybc, zbc):
    """Which Neumann face arrays a boundary-code triple reads
    (testgpurectangle.cu:46-57)."""
    return {"bcl": xbc in (3, 4), "bcr": xbc in (2, 3),
            "bcb": ybc in (3, 4), "bct": ybc in (2, 3),
            "bcf": zbc in (3, 4), "bce": zbc in (2, 3)}


def _second_diff(u, axis, bc, n, d2, d1, g_lo, g_hi):
    """(u[i-1] - 2u[i] + u[i+1]) * d2 along ``axis`` for every index 0..n, with
    the closure of boundary code ``bc``.  g_lo/g_hi are face arrays broadcast
    against u with ``axis`` removed (or None)."""
    um = np.moveaxis(u, axis, -1)
    left = np.empty_like(um)
    right = np.empty_like(um)
    left[..., 1:] = um[..., :-1]
    right[..., :-1] = um[..., 1:]
    if bc == 0:
        left[..., 0] = um[..., n - 1]
        right[..., n - 1] = um[..., 0]
        right[..., n] = um[..., 1]
    if bc in (3, 4):
        left[..., 0] = um[..., 1] - 2.0 * g_lo / d1
    else:
        left[..., 0] = np.nan if bc != 0 else left[..., 0]
    if bc in (2, 3):
        right[..., n] = um[..., n - 1] + 2.0 * g_hi / d1
    elif bc != 0:
        right[..., n] = np.nan
    out = (left - 2.0 * um + right) * d2
    return np.moveaxis(out, -1, axis)


def apply_operator(u, nx, ny, nz, xbc, ybc, zbc, dom, lam, faces):
    """A_h u evaluated at every grid node (values outside the unknown window
    are meaningless).  ``u`` has shape (NZ+1, NY+1, NX+1) and holds the
    Dirichlet face values on Dirichlet faces."""
    left, right, bottom, top, front, back = dom
    dx, dy, dz = nx / (right - left), ny / (top - bottom), nz / (back - front)
    faces = {k: (None if faces.get(k) is None else np.asarray(faces[k]))
             for k in FACE_KEYS}

    def g(key, shape):
        v = faces[key]
        return np.zeros(shape) if v is None else v

    u = np.asarray(u, dtype=np.float64)
    lx = _second_diff(u, 2, xbc, nx, dx * dx, dx,
                      g("bcl", (nz + 1, ny + 1)), g("bcr", (nz + 1, ny + 1)))
    ly = _second_diff(u, 1, ybc, ny, dy * dy, dy,
                      g("bcb", (nz + 1, nx + 1)), g("bct", (nz + 1, nx + 1)))
    lz = _second_diff(u, 0, zbc, nz, dz * dz, dz,
                      g("bcf", (ny + 1, nx + 1)), g("bce", (ny + 1, nx + 1)))
    return lx + ly + lz + lam * u


def window_slices(nx, ny, nz, xbc, ybc, zbc):
    xs, xe = solver_windows(xbc, nx)
    ys, ye = solver_windows(ybc, ny)
    zs, ze = solver_windows(zbc, nz)
    return (slice(zs, ze + 1), slice(ys, ye + 1), slice(xs, xe + 1))


def manufacture_rhs(u, nx, ny, nz, xbc, ybc, zbc, dom, lam, faces):
    """Right-hand side f whose exact discrete solution is ``u``: A_h u on the
    unknown window, u's values elsewhere (Dirichlet faces, periodic planes)."""
    f = np.array(u, dtype=np.float64, copy=True)
    w = window_slices(nx, ny, nz, xbc, ybc, zbc)
    f[w] = apply_operator(u, nx, ny, nz, xbc, ybc, zbc, dom, lam, faces)[w]
    return f


def residual(u, f, nx, ny, nz, xbc, ybc, zbc, dom, lam, faces):
    """f - A_h u on the unknown window (zero elsewhere)."""
    r = np.zeros_like(np.asarray(f, dtype=np.float64))
    w = window_slices(nx, ny, nz, xbc, ybc, zbc)
    uu = np.array(u, dtype=np.float64, copy=True)
    # Dirichlet faces of the operator come from f, as in the solver.
    mask = np.ones(uu.shape, dtype=bool)
    mask[w] = False
    uu[mask] = np.asarray(f)[mask]
    r[w] = np.asarray(f)[w] - apply_operator(uu, nx, ny, nz, xbc, ybc, zbc,
                                             dom, lam, faces)[w]
    return r


def singular_pertrb(p):
    """FISHPACK's PERTRB for the singular case (lambda = 0, every code 0 or 3):
    the constant hw3crt subtracts from the right-hand side so that a solution
    exists (the wrapper passes &pertrb to hw3crt_ and drops it,
    cudahelmholtz/hw3crt_wrapper.cpp:20-28).  On this discrete system it is
    the weighted mean of b = f + boundary terms over the unknown window, with
    weight 1/2 per Neumann boundary index (the weights under which the operator
    is symmetric); 0 when the problem is not singular.  Pinned against the
    runner's direct hw3crt call (tests/golden/fishpack_singular.npz)."""
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    bcs = (p["xbc"], p["ybc"], p["zbc"])
    if p["lam"] != 0.0 or any(b not in (0, 3) for b in bcs):
        return 0.0
    faces = {k: p.get(k) for k in FACE_KEYS}
    zero = np.zeros((nz + 1, ny + 1, nx + 1))
    # A_h of the zero field with the Neumann data is minus the boundary terms
    terms = -apply_operator(zero, nx, ny, nz, *bcs, p["dom"], 0.0, faces)
    w = window_slices(nx, ny, nz, *bcs)
    b = (np.asarray(p["f"], dtype=np.float64) + terms)[w]
    wt = np.ones_like(b)
    for axis, bc in ((0, p["zbc"]), (1, p["ybc"]), (2, p["xbc"])):
        if bc == 3:
            for end in (0, -1):
                sl = [slice(None)] * 3
                sl[axis] = end
                wt[tuple(sl)] *= 0.5
    return float((wt * b).sum() / wt.sum())


def _extend(u, codes):
    """u on the unknown window, extended by one ghost layer per axis with the
    homogeneous closures of codes 1 (Dirichlet neighbour 0) and 3 (mirror)."""
    e = np.asarray(u, dtype=np.float64)
    for axis, bc in ((0, codes[2]), (1, codes[1]), (2, codes[0])):
        e = np.moveaxis(e, axis, -1)
        if bc == 1:
            lo = np.zeros_like(e[..., :1])
            hi = np.zeros_like(e[..., :1])
        elif bc == 3:
            lo = e[..., 1:2]
            hi = e[..., -2:-1]
        else:
            raise ValueError("codes 1 and 3 only")
        e = np.concatenate([lo, e, hi], axis=-1)
        e = np.moveaxis(e, -1, axis)
    return e


def apply_19pt(u, codes, h2):
    """The compact 19-point Laplacian (1 / (6 h^2)) (-24 u + 2 sum of the 6 face
    neighbours + sum of the 12 edge neighbours) on the unknown window, with
    homogeneous closures (codes 1 and 3)."""
    e = _extend(u, codes)
    c = e[1:-1, 1:-1, 1:-1]
    faces = (e[:-2, 1:-1, 1:-1] + e[2:, 1:-1, 1:-1] + e[1:-1, :-2, 1:-1] + e[1:-1, 2:, 1:-1]
             + e[1:-1, 1:-1, :-2] + e[1:-1, 1:-1, 2:])
    edges = 0.0
    sl = {-1: slice(0, -2), 0: slice(1, -1), 1: slice(2, None)}
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if abs(dz) + abs(dy) + abs(dx) == 2:
                    edges = edges + e[sl[dz], sl[dy], sl[dx]]
    return (-24.0 * c + 2.0 * faces + edges) * h2 / 6.0


def filter_19pt(b, codes):
    """Right-hand-side filter of the compact scheme, (6 b + sum of the 6 face
    neighbours) / 12, with the same closures."""
    e = _extend(b, codes)
    c = e[1:-1, 1:-1, 1:-1]
    faces = (e[:-2, 1:-1, 1:-1] + e[2:, 1:-1, 1:-1] + e[1:-1, :-2, 1:-1] + e[1:-1, 2:, 1:-1]
             + e[1:-1, 1:-1, :-2] + e[1:-1, 1:-1, 2:])
    return (6.0 * c + faces) / 12.0
