"""The eight transform kinds as textbook sums (test infrastructure).

Each kind is the unnormalised scipy.fft DCT/DST of the listed type times 1/2 on
its input window (the reference's "half of FFTW" scaling), or the unnormalised
real DFT.  These are an independent cross-check of ``oracle.emulation``:

=========  ==========================  =========  ==========
kind       formula (k over out window)  in         out
=========  ==========================  =========  ==========
DST_1      sum_{n=1}^{N-1} x_n sin(pi n k / N)             [1,N-1]  [1,N-1], out0=0
DST_2      sum_{n=1}^{N} x_n sin(pi k (2n-1) / 2N)         [1,N]    [1,N],   out0=0
DST_3      sum_{n=1}^{N-1} x_n sin(pi (2k-1) n / 2N)
           + (-1)^(k+1) (x_N + x_0) / 2                    [0,N]    [1,N],   out0=0
DCT_1      x_0/2 + (-1)^k x_N/2 + sum_{n=1}^{N-1} x_n cos(pi n k / N)  [0,N] [0,N]
DCT_2      sum_{n=0}^{N-1} x_n cos(pi k (2n+1) / 2N)       [0,N-1]  [0,N-1]
DCT_3      x_0/2 + sum_{n=1}^{N-1} x_n cos(pi (2k+1) n / 2N)  [0,N-1] [0,N-1]
DFT_R2C    rfft, bins interleaved (re, im)                 [0,N-1]  [0,N+1]
DFT_C2R    N * irfft, Im of bins 0 and N/2 ignored         [0,N+1]  [0,N-1]
=========  ==========================  =========  ==========
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

from .emulation import (DCT_1, DCT_2, DCT_3, DST_1, DST_2, DST_3, DFT_R2C,
                        DFT_C2R, out_window, padded_shape)


def closed_kind(lines: np.ndarray, kind: int, n: int) -> np.ndarray:
    x = np.asarray(lines, dtype=np.float64)
    out = np.full(x.shape, np.nan)
    if kind == DST_1:
        out[..., 1:n] = 0.5 * sfft.dst(x[..., 1:n], type=1, axis=-1)
        out[..., 0] = 0.0
    elif kind == DST_2:
        out[..., 1:n + 1] = 0.5 * sfft.dst(x[..., 1:n + 1], type=2, axis=-1)
        out[..., 0] = 0.0
    elif kind == DST_3:
        y = x[..., 1:n + 1].copy()
        y[..., -1] = y[..., -1] + x[..., 0]
        out[..., 1:n + 1] = 0.5 * sfft.dst(y, type=3, axis=-1)
        out[..., 0] = 0.0
    elif kind == DCT_1:
        out[..., 0:n + 1] = 0.5 * sfft.dct(x[..., 0:n + 1], type=1, axis=-1)
    elif kind == DCT_2:
        out[..., 0:n] = 0.5 * sfft.dct(x[..., 0:n], type=2, axis=-1)
    elif kind == DCT_3:
        out[..., 0:n] = 0.5 * sfft.dct(x[..., 0:n], type=3, axis=-1)
    elif kind == DFT_R2C:
        z = np.fft.rfft(x[..., :n], axis=-1)
        out[..., 0:n + 2:2] = z.real
        out[..., 1:n + 2:2] = z.imag
    elif kind == DFT_C2R:
        c = x[..., 0:n + 2:2] + 1j * np.nan_to_num(x[..., 1:n + 2:2])
        c[..., 0] = c[..., 0].real
        c[..., n // 2] = c[..., n // 2].real
        out[..., 0:n] = np.fft.irfft(c, n=n, axis=-1) * n
    else:
        raise ValueError("bad kind")
    lo, hi = out_window(kind, n)
    out[..., :lo] = np.nan
    out[..., hi + 1:] = np.nan
    return out


def closed_do_transform(data, nx, ny, nz, kx, ky, kz):
    """Separable 3-D application of ``closed_kind`` (x, then y, then z)."""
    a = np.array(data, dtype=np.float64, copy=True)
    assert a.shape == padded_shape(nx, ny, nz)
    for axis, kind, n in ((2, kx, nx), (1, ky, ny), (0, kz, nz)):
        b = np.moveaxis(a, axis, -1)
        a = np.moveaxis(closed_kind(b, kind, n), -1, axis)
    return np.ascontiguousarray(a)
