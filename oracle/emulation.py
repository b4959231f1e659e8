"""Line-by-line numpy restatement of the reference GPU path (test infrastructure).

Every function cites the reference kernel it restates (paths relative to the
reference project).  cuFFT is modelled by numpy's pocketfft with cuFFT's
conventions for the reference's plans:

* Z2D (C2R) of length N, in place on a row of N+2 doubles
  (funcinterface.cu:57-60): input bins k = 0..N/2 at (2k, 2k+1); output reals
  at 0..N-1, unnormalised; the imaginary parts of bins 0 and N/2 are discarded;
  row entries N and N+1 are left undefined (NaN here).
* D2Z (R2C) of length N (funcinterface.cu:74-77): reads 0..N-1, writes bins
  0..N/2 interleaved at 0..N+1, unnormalised.

Each kind's result is then restricted to its output window (entries outside are
NaN), lines the reference's pre/post kernels do not visit (other-axis index
N+1) become NaN for the kinds that have pre/post kernels, and a line whose
input window holds an undefined entry defines nothing.  The defined entries of
a 3-D result are thus the product of the per-axis windows, and a comparison
against this oracle covers exactly the entries the reference defines.
"""
from __future__ import annotations

import numpy as np

# transform_kind, cudasymmfft/global.h:6-15 (values are ABI)
DCT_1, DCT_2, DCT_3, DST_1, DST_2, DST_3, DFT_R2C, DFT_C2R = range(8)
KIND_NAMES = ["DCT_1", "DCT_2", "DCT_3", "DST_1", "DST_2", "DST_3",
              "DFT_R2C", "DFT_C2R"]

# Output window [lo, hi] of each kind on a padded line of N+2 entries.
_OUT_WINDOW = {
    DST_1: lambda n: (0, n - 1),    # out[0] = 0 (dst1funcinplace.cu:107)
    DST_2: lambda n: (0, n),        # out[0] = 0 (dst2funcinplace.cu:102)
    DST_3: lambda n: (0, n),        # out[0] = 0 (dst3funcinplace.cu:90)
    DCT_1: lambda n: (0, n),
    DCT_2: lambda n: (0, n - 1),
    DCT_3: lambda n: (0, n - 1),
    DFT_R2C: lambda n: (0, n + 1),
    DFT_C2R: lambda n: (0, n - 1),
}


def out_window(kind: int, n: int) -> tuple[int, int]:
    return _OUT_WINDOW[kind](n)


# Input window [lo, hi] each kind reads (from the pre kernels' loads and the
# cuFFT plan lengths).
_IN_WINDOW = {
    DST_1: lambda n: (1, n - 1), DST_2: lambda n: (1, n), DST_3: lambda n: (0, n),
    DCT_1: lambda n: (0, n), DCT_2: lambda n: (0, n - 1), DCT_3: lambda n: (0, n - 1),
    DFT_R2C: lambda n: (0, n - 1), DFT_C2R: lambda n: (0, n + 1),
}


def in_window(kind: int, n: int) -> tuple[int, int]:
    return _IN_WINDOW[kind](n)


def _c2r(p: np.ndarray, n: int) -> np.ndarray:
    """cuFFT Z2D of length n in place on rows of n+2 doubles."""
    c = p[..., 0:n + 2:2] + 0j
    c.imag = p[..., 1:n + 2:2]
    c[..., 0] = c[..., 0].real
    c[..., n // 2] = c[..., n // 2].real
    out = np.full(p.shape, np.nan)
    out[..., :n] = np.fft.irfft(c, n=n, axis=-1) * n
    return out


def _r2c(p: np.ndarray, n: int) -> np.ndarray:
    """cuFFT D2Z of length n in place on rows of n+2 doubles."""
    x = np.fft.rfft(p[..., :n], axis=-1)
    out = np.empty(p.shape)
    out[..., 0:n + 2:2] = x.real
    out[..., 1:n + 2:2] = x.imag
    # pocketfft returns exact zeros for the imaginary parts of bins 0 and N/2
    # even when the input holds NaN; an undefined input defines nothing.
    bad = np.isnan(p[..., :n]).any(axis=-1)
    out[bad] = np.nan
    return out


def _dst1(a: np.ndarray, n: int) -> np.ndarray:
    """DST_1: preOp/postOp_dst1_inplace, dst1funcinplace.cu:55-112."""
    sh = a[..., :n].copy()
    p = a.copy()
    p[..., 0] = 2 * sh[..., 1]
    p[..., 1] = 0
    p[..., n] = -2 * sh[..., n - 1]
    p[..., n + 1] = 0
    i = np.arange(1, n // 2)
    p[..., 2 * i] = sh[..., 2 * i + 1] - sh[..., 2 * i - 1]
    p[..., 2 * i + 1] = -sh[..., 2 * i]
    y = _c2r(p, n)
    k = np.arange(1, n // 2 + 1)
    s, sn = y[..., k], y[..., n - k]
    ta = (s + sn) / (4 * np.sin(k * np.pi / n))
    tb = (s - sn) / 2
    q = y.copy()
    q[..., k] = (ta + tb) / 2
    q[..., n - k] = (ta - tb) / 2
    q[..., 0] = 0
    return q


def _dst2(a: np.ndarray, n: int) -> np.ndarray:
    """DST_2: preOp/postOp_dst2_inplace, dst2funcinplace.cu:48-108."""
    sh = a[..., 1:n + 1].copy()
    p = a.copy()
    p[..., 0] = sh[..., 0]
    p[..., 1] = 0
    p[..., n] = -sh[..., n - 1]
    p[..., n + 1] = 0
    i = np.arange(1, n // 2)
    p[..., 2 * i] = (sh[..., 2 * i] - sh[..., 2 * i - 1]) / 2
    p[..., 2 * i + 1] = -((sh[..., 2 * i] + sh[..., 2 * i - 1]) / 2)
    y = _c2r(p, n)
    sh = y[..., :n].copy()
    k = np.arange(1, n // 2 + 1)
    ang = k * np.pi / (2 * n)
    sina, cosa = np.sin(ang), np.cos(ang)
    ta = sh[..., k] + sh[..., n - k]
    tb = sh[..., k] - sh[..., n - k]
    q = y.copy()
    q[..., k] = (ta * sina + tb * cosa) / 2
    q[..., n - k] = (ta * cosa - tb * sina) / 2
    q[..., 0] = 0
    q[..., n] = sh[..., 0]
    return q


def _dst3(a: np.ndarray, n: int) -> np.ndarray:
    """DST_3 (called with DATA_SIZE = n+1, funcinterface.cu:93):
    preOp/postOp_dst3_inplace, dst3funcinplace.cu:49-105."""
    p = a.copy()
    t = np.arange(0, n // 2 + 1)
    ang = t * np.pi / (2 * n)
    sina, cosa = np.sin(ang), np.cos(ang)
    ta = a[..., t] + a[..., n - t]
    tb = a[..., t] - a[..., n - t]
    p[..., t] = ta * cosa + tb * sina
    p[..., n - t] = ta * sina - tb * cosa
    x = _r2c(p, n)
    sh = x.copy()
    t1 = np.arange(1, n // 2 + 1)
    sh[..., 2 * t1 + 1] = -sh[..., 2 * t1 + 1]
    q = x.copy()
    q[..., 0] = 0
    q[..., 1] = sh[..., 0] / 2
    q[..., 2 * t1] = (sh[..., 2 * t1 + 1] - sh[..., 2 * t1]) / 2
    t2 = t1[2 * t1 + 1 < n + 1]
    q[..., 2 * t2 + 1] = (sh[..., 2 * t2] + sh[..., 2 * t2 + 1]) / 2
    return q


def _pow2roundup(x: int) -> int:
    """pow2roundup, dct1funcinplace.cu:37-48."""
    r = 1
    while r < x:
        r <<= 1
    return r


def _tree_sum(v: np.ndarray) -> np.ndarray:
    """Shared-memory tree reduction order of preOp_dct1_inplace
    (dct1funcinplace.cu:83-90): sh[i] += sh[i+s], s = nThread/2 .. 1."""
    m = v.shape[-1]
    while m > 1:
        h = m // 2
        v = v[..., :h] + v[..., h:m]
        m = h
    return v[..., 0]


def _dct1(a: np.ndarray, n: int) -> np.ndarray:
    """DCT_1 (DATA_SIZE = n+1): preOp/postOp_dct1_inplace,
    dct1funcinplace.cu:60-131, with the odd-sample sum x1."""
    nthread = _pow2roundup(n // 2)
    sh = np.zeros(a.shape[:-1] + (nthread,))
    sh[..., :n // 2] = a[..., 1:n:2]
    p = a.copy()
    p[..., n + 1] = 0
    p[..., 1] = 0
    t = np.arange(1, n // 2)
    p[..., 2 * t + 1] = sh[..., t - 1] - sh[..., t]
    x1 = _tree_sum(sh)
    y = _c2r(p, n)
    k = np.arange(1, n // 2 + 1)
    s, sn = y[..., k], y[..., n - k]
    ta = (s + sn) * 0.5
    tb = (s - sn) * 0.25 / np.sin(k * np.pi / n)
    q = y.copy()
    q[..., k] = (ta - tb) * 0.5
    q[..., n - k] = (ta + tb) * 0.5
    sh0 = y[..., 0] * 0.5
    q[..., 0] = sh0 + x1
    q[..., n] = sh0 - x1
    return q


def _dct2(a: np.ndarray, n: int) -> np.ndarray:
    """DCT_2: preOp/postOp_dct2_inplace, dct2funcinplace.cu:49-112."""
    sh = a[..., :n].copy()
    p = a.copy()
    p[..., 0] = sh[..., 0]
    p[..., 1] = 0
    p[..., n] = sh[..., n - 1]
    p[..., n + 1] = 0
    i = np.arange(1, n // 2)
    p[..., 2 * i] = (sh[..., 2 * i] + sh[..., 2 * i - 1]) / 2
    p[..., 2 * i + 1] = -((sh[..., 2 * i - 1] - sh[..., 2 * i]) / 2)
    y = _c2r(p, n)
    sh = y[..., :n].copy()
    k = np.arange(1, n // 2 + 1)
    ang = k * np.pi / (2 * n)
    sina, cosa = np.sin(ang), np.cos(ang)
    ta = sh[..., k] + sh[..., n - k]
    tb = sh[..., k] - sh[..., n - k]
    q = y.copy()
    q[..., k] = (ta * cosa + tb * sina) / 2
    q[..., n - k] = (ta * sina - tb * cosa) / 2
    return q


def _dct3(a: np.ndarray, n: int) -> np.ndarray:
    """DCT_3: preOp/postOp_dct3_inplace, dct3funcinplace.cu:47-95."""
    p = a.copy()
    t = np.arange(0, n // 2)
    ang = (t + 1) * np.pi / (2 * n)
    sina, cosa = np.sin(ang), np.cos(ang)
    ta = a[..., t + 1] + a[..., n - t - 1]
    tb = a[..., t + 1] - a[..., n - t - 1]
    p[..., t + 1] = ta * sina + tb * cosa
    p[..., n - t - 1] = ta * cosa - tb * sina
    x = _r2c(p, n)
    sh = x
    q = x.copy()
    q[..., 0] = sh[..., 0] / 2
    t1 = np.arange(1, n // 2 + 1)
    q[..., 2 * t1 - 1] = (sh[..., 2 * t1] - sh[..., 2 * t1 + 1]) / 2
    t2 = t1[2 * t1 < n]
    q[..., 2 * t2] = (sh[..., 2 * t2] + sh[..., 2 * t2 + 1]) / 2
    return q


def _dft_r2c(a: np.ndarray, n: int) -> np.ndarray:
    """DFT_R2C: plain cuFFT D2Z (dftfunc.cu:91-110)."""
    return _r2c(a, n)


def _dft_c2r(a: np.ndarray, n: int) -> np.ndarray:
    """DFT_C2R: plain cuFFT Z2D (dftfunc.cu:132-150)."""
    return _c2r(a, n)


_KIND_FN = {DST_1: _dst1, DST_2: _dst2, DST_3: _dst3, DCT_1: _dct1,
            DCT_2: _dct2, DCT_3: _dct3, DFT_R2C: _dft_r2c, DFT_C2R: _dft_c2r}


def emulate_kind(lines: np.ndarray, kind: int, n: int) -> np.ndarray:
    """One kind on every row of ``lines`` (shape (..., n+2)); entries outside
    the kind's output window become NaN."""
    if lines.shape[-1] != n + 2:
        raise ValueError("rows must hold n+2 entries")
    if n < 2 or n % 2:
        raise ValueError("n must be even and >= 2")
    lines = np.asarray(lines, dtype=np.float64)
    out = _KIND_FN[kind](lines, n)
    lo, hi = out_window(kind, n)
    out[..., :lo] = np.nan
    out[..., hi + 1:] = np.nan
    # A line whose input is undefined defines nothing, not even the constant
    # zero the DST kinds write at index 0 (such lines lie outside the product
    # of the per-axis windows, where the reference holds meaningless values).
    ilo, ihi = in_window(kind, n)
    used = lines[..., ilo:ihi + 1]
    if kind == DFT_C2R:  # the imaginary parts of bins 0 and N/2 are not read
        keep = np.ones(ihi - ilo + 1, dtype=bool)
        keep[[1, n + 1]] = False
        used = used[..., keep]
    out[np.isnan(used).any(axis=-1)] = np.nan
    return out


def padded_shape(nx: int, ny: int, nz: int) -> tuple[int, int, int]:
    """Padded (z, y, x) shape of do_transform's array: rows of NX+2 doubles."""
    return (nz + 2, ny + 2, nx + 2)


def emulate_do_transform(data: np.ndarray, nx: int, ny: int, nz: int,
                         kx: int, ky: int, kz: int) -> np.ndarray:
    """do_transform (funcinterface.cu:25-40): x pass, then y, then z, each over
    the padded array (NZ+2, NY+2, NX+2) in [z][y][x] order.

    The cubic path (funcinterface.cu:42-198) and the non-cubic path (:200-334)
    apply the same per-axis passes; only their transposes differ, and a
    transpose is an exact permutation.  Pre/post kernels visit the lines whose
    other-axis indices lie in 0..N (grid (batch+1) x (nLayer+1), e.g.
    dst1funcinplace.cu:153-156); cuFFT also transforms the lines at N+1, which
    are meaningful only for the DFT kinds (no pre/post kernels)."""
    a = np.array(data, dtype=np.float64, copy=True)
    if a.shape != padded_shape(nx, ny, nz):
        raise ValueError(f"expected padded shape {padded_shape(nx, ny, nz)}")
    sizes = {2: nx, 1: ny, 0: nz}
    for axis, kind in ((2, kx), (1, ky), (0, kz)):
        n = sizes[axis]
        b = np.moveaxis(a, axis, -1)
        res = emulate_kind(b, kind, n)
        if kind not in (DFT_R2C, DFT_C2R):
            others = [ax for ax in (0, 1, 2) if ax != axis]
            # res has the other axes first (in increasing order), then the line
            for pos, ax in enumerate(others):
                idx = [slice(None)] * 3
                idx[pos] = sizes[ax] + 1
                res[tuple(idx)] = np.nan
        a = np.moveaxis(res, -1, axis)
    return np.ascontiguousarray(a)


# --------------------------------------------------------------------------
# Helmholtz solver, cuda_helmholtz_solver.cu:33-380 + _cuda_helmholtz_.inl
# --------------------------------------------------------------------------

_FWD_KIND = {0: DFT_R2C, 1: DST_1, 2: DST_3, 3: DCT_1, 4: DCT_3}
_INV_KIND = {0: DFT_C2R, 1: DST_1, 2: DST_2, 3: DCT_1, 4: DCT_2}


def solver_windows(bc: int, n: int) -> tuple[int, int]:
    """Unknown window (s, e) per boundary code, cuda_helmholtz_solver.cu:78-103."""
    if bc == 0:
        return 0, n - 1
    if bc == 1:
        return 1, n - 1
    if bc == 2:
        return 1, n
    if bc == 3:
        return 0, n
    if bc == 4:
        return 0, n - 1
    raise ValueError("bad boundary condition")


def solver_kinds(bc: int) -> tuple[int, int]:
    return _FWD_KIND[bc], _INV_KIND[bc]


def _c_int_ratio(nx: int, ny: int, nz: int) -> int:
    """`int ratio = NX/2 * NY/2 * NZ/2;` (cuda_helmholtz_solver.cu:211) with
    C's left-to-right integer division."""
    r = nx // 2
    r = r * ny
    r = r // 2
    r = r * nz
    r = r // 2
    return r


def emulate_solver(left, right, nx, xbc, bcl, bcr,
                   bottom, top, ny, ybc, bcb, bct,
                   front, back, nz, zbc, bcf, bce,
                   lam, f, stencil19=False):
    """Returns the array the reference writes into ``f`` (shape (NZ+1, NY+1,
    NX+1), [z][y][x]).  Face arrays: x faces (NZ+1, NY+1), y faces
    (NZ+1, NX+1), z faces (NY+1, NX+1), as laid out in testgpurectangle.cu:46-57.

    stencil19: the non-periodic branch divides with the reference's
    _nonpoisson_devide_19points_ (_cuda_helmholtz_.inl:255-274; its call is
    commented out at cuda_helmholtz_solver.cu:338) instead of _divide_.
    """
    f = np.array(f, dtype=np.float64, copy=True).reshape(nz + 1, ny + 1, nx + 1)
    dx = nx / (right - left)
    dy = ny / (top - bottom)
    dz = nz / (back - front)
    dx2, dy2, dz2 = dx * dx, dy * dy, dz * dz
    pi = 3.14159265358979323846
    shift = {}
    pidiv = {}
    for ax, bc, n in (("x", xbc, nx), ("y", ybc, ny), ("z", zbc, nz)):
        s = 0.0
        if bc == 2:
            s = -0.5 * pi / n
        if bc == 4:
            s = 0.5 * pi / n
        shift[ax] = s
        pidiv[ax] = pi / n * (2 if bc == 0 else 1)
    xs, xe = solver_windows(xbc, nx)
    ys, ye = solver_windows(ybc, ny)
    zs, ze = solver_windows(zbc, nz)

    def face(arr, shape):
        return None if arr is None else np.asarray(arr, dtype=np.float64).reshape(shape)

    bcl = face(bcl, (nz + 1, ny + 1))
    bcr = face(bcr, (nz + 1, ny + 1))
    bcb = face(bcb, (nz + 1, nx + 1))
    bct = face(bct, (nz + 1, nx + 1))
    bcf = face(bcf, (ny + 1, nx + 1))
    bce = face(bce, (ny + 1, nx + 1))

    # boundary-term kernels _3d_bc{1..4}_ini_{x,y,z}_ (_cuda_helmholtz_.inl:70-227)
    K = slice(zs, ze + 1)
    J = slice(ys, ye + 1)
    I = slice(xs, xe + 1)
    if xbc in (1, 2):
        f[K, J, xs] -= f[K, J, 0] * dx2
    if xbc in (3, 4):
        f[K, J, xs] += 2 * bcl[K, J] * dx
    if xbc in (1, 4):
        f[K, J, xe] -= f[K, J, nx] * dx2
    if xbc in (2, 3):
        f[K, J, xe] -= 2 * bcr[K, J] * dx
    if ybc in (1, 2):
        f[K, ys, I] -= f[K, 0, I] * dy2
    if ybc in (3, 4):
        f[K, ys, I] += 2 * bcb[K, I] * dy
    if ybc in (1, 4):
        f[K, ye, I] -= f[K, ny, I] * dy2
    if ybc in (2, 3):
        f[K, ye, I] -= 2 * bct[K, I] * dy
    if zbc in (1, 2):
        f[zs, J, I] -= f[0, J, I] * dz2
    if zbc in (3, 4):
        f[zs, J, I] += 2 * bcf[J, I] * dz
    if zbc in (1, 4):
        f[ze, J, I] -= f[nz, J, I] * dz2
    if zbc in (2, 3):
        f[ze, J, I] -= 2 * bce[J, I] * dz

    # ex: padded, zeroed, window copied in (_ini_ex_, inl:230-239)
    ex = np.zeros(padded_shape(nx, ny, nz))
    ex[K, J, I] = f[K, J, I]
    kx, kxi = solver_kinds(xbc)
    ky, kyi = solver_kinds(ybc)
    kz, kzi = solver_kinds(zbc)
    ex = emulate_do_transform(ex, nx, ny, nz, kx, ky, kz)

    # divide (_divide_ / _periodic_divide_, inl:276-421)
    needperturb = (lam == 0.0 and xbc in (0, 3) and ybc in (0, 3) and zbc in (0, 3))

    def modes(bc, n, s, e):
        if bc == 0:
            m = np.arange(0, n // 2 + 1)
            return m, [2 * m, 2 * m + 1]
        m = np.arange(s, e + 1)
        return m, [m]

    mi, ent_i = modes(xbc, nx, xs, xe)
    mj, ent_j = modes(ybc, ny, ys, ye)
    mk, ent_k = modes(zbc, nz, zs, ze)
    ex_ = (2 * np.cos(mi * pidiv["x"] + shift["x"]) - 2) * dx2
    ey_ = (2 * np.cos(mj * pidiv["y"] + shift["y"]) - 2) * dy2
    ez_ = (2 * np.cos(mk * pidiv["z"] + shift["z"]) - 2) * dz2
    den = ((ex_[None, None, :] + ey_[None, :, None]) + ez_[:, None, None]) + lam
    with np.errstate(divide="ignore"):
        eig = 1.0 / den
    if stencil19:
        # cos(i * pidivnx) etc. (no shift), dx2 only, no zero-mode handling
        if 0 in (xbc, ybc, zbc):
            raise ValueError("the 19-point division is the non-periodic branch's")
        ci = np.cos(mi * pidiv["x"])[None, None, :]
        cj = np.cos(mj * pidiv["y"])[None, :, None]
        ck = np.cos(mk * pidiv["z"])[:, None, None]
        coef = (2.0 / 3.0 * (ci * cj + ci * ck + cj * ck + ci + cj + ck) - 4) * dx2 + lam
        with np.errstate(divide="ignore", invalid="ignore"):
            eig = (0.5 + 1.0 / 6.0 * (ci + cj + ck)) / coef
        needperturb = False
    if needperturb and mi[0] == 0 and mj[0] == 0 and mk[0] == 0:
        eig[0, 0, 0] = 0.0
    for ek in ent_k:
        for ej in ent_j:
            for ei in ent_i:
                ex[np.ix_(ek, ej, ei)] *= eig
    ex = emulate_do_transform(ex, nx, ny, nz, kxi, kyi, kzi)

    # _store_f_ (inl:242-251) with ratio (solver.cu:211-215)
    ratio = _c_int_ratio(nx, ny, nz)
    for bc in (xbc, ybc, zbc):
        if bc == 0:
            ratio *= 2
    f[K, J, I] = ex[K, J, I] * (1.0 / float(ratio))
    # periodic copies _3d_bc0_store_{x,y,z}_ (inl:58-68, 116-126, 173-183)
    if xbc == 0:
        f[:, :, nx] = f[:, :, 0]
    if ybc == 0:
        f[:, ny, :] = f[:, 0, :]
    if zbc == 0:
        f[nz, :, :] = f[0, :, :]
    return f
