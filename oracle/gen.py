"""Seeded synthetic problems with the benchmark configurations' shapes and value
distributions (test infrastructure; no public dataset is involved).

A problem is a dict: nx, ny, nz, xbc, ybc, zbc, dom (left, right, bottom, top,
front, back), lam, f (NZ+1, NY+1, NX+1) [z][y][x], and the six Neumann face
arrays bcl, bcr, bcb, bct, bcf, bce (None when the codes do not read them).
Optional key u_exact holds a manufactured discrete solution.
"""
from __future__ import annotations

import numpy as np

from .stencil import FACE_KEYS, face_shapes, manufacture_rhs, used_faces

UNIT_DOMAIN = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)


def make_periodic_compatible(p):
    """Copy plane 0 onto plane N of every periodic axis, in f and in the face
    arrays that span that axis (the reference requires periodic data to agree
    at both ends, README.md 'Caution')."""
    f = p["f"]
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    if p["xbc"] == 0:
        f[:, :, nx] = f[:, :, 0]
    if p["ybc"] == 0:
        f[:, ny, :] = f[:, 0, :]
    if p["zbc"] == 0:
        f[nz, :, :] = f[0, :, :]
    for key in FACE_KEYS:
        v = p.get(key)
        if v is None:
            continue
        # x faces are [z][y], y faces [z][x], z faces [y][x]
        ax_names = {"bcl": ("z", "y"), "bcr": ("z", "y"), "bcb": ("z", "x"),
                    "bct": ("z", "x"), "bcf": ("y", "x"), "bce": ("y", "x")}[key]
        for dim, name in enumerate(ax_names):
            if p[name + "bc"] == 0:
                n = p["n" + name]
                if dim == 0:
                    v[n, :] = v[0, :]
                else:
                    v[:, n] = v[:, 0]
    return p


def random_problem(nx, ny, nz, xbc, ybc, zbc, lam, seed, dom=UNIT_DOMAIN,
                   dist="uniform", amp=1.0):
    """f and used Neumann faces drawn from U[-amp, amp] (or N(0, amp^2))."""
    rng = np.random.default_rng(seed)
    draw = ((lambda shape: rng.uniform(-amp, amp, size=shape)) if dist == "uniform"
            else (lambda shape: rng.normal(0.0, amp, size=shape)))
    p = dict(nx=nx, ny=ny, nz=nz, xbc=xbc, ybc=ybc, zbc=zbc, dom=tuple(dom),
             lam=float(lam))
    p["f"] = draw((nz + 1, ny + 1, nx + 1))
    use = used_faces(xbc, ybc, zbc)
    shapes = face_shapes(nx, ny, nz)
    for key in FACE_KEYS:
        p[key] = draw(shapes[key]) if use[key] else None
    return make_periodic_compatible(p)


def _mode_1d(bc, m, x, phase_cos):
    """Boundary-compatible mode on [0, 1] per code (0: cos/sin(2 pi m x),
    1: sin(m pi x), 2: sin((m-1/2) pi x), 3: cos(m pi x), 4: cos((m-1/2) pi x))."""
    if bc == 0:
        return np.cos(2 * np.pi * m * x) if phase_cos else np.sin(2 * np.pi * m * x)
    if bc == 1:
        return np.sin(m * np.pi * x)
    if bc == 2:
        return np.sin((m - 0.5) * np.pi * x)
    if bc == 3:
        return np.cos(m * np.pi * x)
    if bc == 4:
        return np.cos((m - 0.5) * np.pi * x)
    raise ValueError(bc)


def modal_field(nx, ny, nz, xbc, ybc, zbc, nmodes, seed):
    """Sum of ``nmodes`` separable boundary-compatible modes with N(0,1)
    amplitudes and integer wavenumbers in [1, 8], sampled at the nodes of the
    unit cube."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx + 1) / nx
    y = np.arange(ny + 1) / ny
    z = np.arange(nz + 1) / nz
    u = np.zeros((nz + 1, ny + 1, nx + 1))
    for _ in range(nmodes):
        a = rng.normal()
        mx, my, mz = rng.integers(1, 9, size=3)
        cx, cy, cz = rng.integers(0, 2, size=3)
        u += a * (_mode_1d(zbc, mz, z, cz)[:, None, None]
                  * _mode_1d(ybc, my, y, cy)[None, :, None]
                  * _mode_1d(xbc, mx, x, cx)[None, None, :])
    return u


def manufactured_problem(nx, ny, nz, xbc, ybc, zbc, lam, seed, nmodes=4,
                         dom=UNIT_DOMAIN):
    """f = A_h u for a modal u with homogeneous Neumann data, so u is the exact
    discrete solution (the reference's own analytic test, ufunc.h, pins only
    truncation error)."""
    u = modal_field(nx, ny, nz, xbc, ybc, zbc, nmodes, seed)
    p = dict(nx=nx, ny=ny, nz=nz, xbc=xbc, ybc=ybc, zbc=zbc, dom=tuple(dom),
             lam=float(lam))
    use = used_faces(xbc, ybc, zbc)
    shapes = face_shapes(nx, ny, nz)
    faces = {k: (np.zeros(shapes[k]) if use[k] else None) for k in FACE_KEYS}
    p.update(faces)
    p["f"] = manufacture_rhs(u, nx, ny, nz, xbc, ybc, zbc, dom, lam, faces)
    p["u_exact"] = u
    return p


# ---- benchmark configurations ------------------------------------------------

def config1_problem(seed=1, n=128):
    """128^3 cells, BC (1, 2, 0), lambda = -2, manufactured 4-mode u."""
    return manufactured_problem(n, n, n, 1, 2, 0, -2.0, seed, nmodes=4)


def config2_problem(xbc, ybc, seed=2, shape=(256, 192, 320)):
    """256 x 192 x 320, BC (xbc, ybc, 3), lambda ~ U[-50, -0.5], f and Neumann
    data ~ U[-1, 1]."""
    rng = np.random.default_rng(seed * 1000 + xbc * 5 + ybc)
    lam = float(rng.uniform(-50.0, -0.5))
    nx, ny, nz = shape
    return random_problem(nx, ny, nz, xbc, ybc, 3, lam,
                          seed=seed * 1000 + 100 + xbc * 5 + ybc)


def config3_problem(seed=3, n=512):
    """512^3, BC (3, 4, 0), lambda = -1, f ~ U[-1, 1] plus the smooth mode
    1e3 cos(pi x) cos(pi y / 2) cos(2 pi z)."""
    p = random_problem(n, n, n, 3, 4, 0, -1.0, seed)
    x = np.arange(n + 1) / n
    p["f"] += 1e3 * (np.cos(2 * np.pi * x)[:, None, None]
                     * np.cos(np.pi * x / 2)[None, :, None]
                     * np.cos(np.pi * x)[None, None, :])
    return make_periodic_compatible(p)


def config4_problems(count=512, seed=4):
    """``count`` independent solves: each dimension uniform in {32, 48, ..., 192},
    codes uniform in 0..4 per axis, lambda = -10^U(-2, 2), f ~ U[-1, 1]."""
    rng = np.random.default_rng(seed)
    sizes = np.arange(32, 193, 16)
    out = []
    for i in range(count):
        nx, ny, nz = (int(v) for v in rng.choice(sizes, size=3))
        xbc, ybc, zbc = (int(v) for v in rng.integers(0, 5, size=3))
        lam = -float(10.0 ** rng.uniform(-2.0, 2.0))
        out.append(random_problem(nx, ny, nz, xbc, ybc, zbc, lam,
                                  seed=seed * 100000 + i))
    return out


def config5_problem(seed=5, n=256):
    """256^3, BC (1, 3, 0), lambda = -4, f ~ N(0, 1), with a random 3-mode
    target field for the loss 0.5 ||u - u_target||^2."""
    p = random_problem(n, n, n, 1, 3, 0, -4.0, seed, dist="normal")
    p["u_target"] = modal_field(n, n, n, 1, 3, 0, 3, seed + 17)
    return p
