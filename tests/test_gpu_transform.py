"""GPU parity of do_transform (through the C ABI) against the oracle's
restatement of the reference path.  Every entry the reference defines (the
oracle's non-NaN entries) must match to 1e-12 relative (max-norm over the
array); nothing else is compared."""
import itertools

import numpy as np
import pytest
import torch

from oracle import emulation as E
from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _run(d, nx, ny, nz, kinds, inplace):
    dev = torch.from_numpy(np.ascontiguousarray(d).ravel()).cuda()
    before = dev.clone()
    if inplace:
        res = api.do_transform(dev, None, nx, ny, nz, *kinds)
    else:
        out = torch.full_like(dev, float("nan"))
        res = api.do_transform(dev, out, nx, ny, nz, *kinds)
    torch.cuda.synchronize()
    if not inplace:
        assert torch.equal(dev, before), "out-of-place call modified d_data"
    return res.cpu().numpy().reshape(nz + 2, ny + 2, nx + 2)


def _check(d, nx, ny, nz, kinds, inplace):
    ref = E.emulate_do_transform(d, nx, ny, nz, *kinds)
    got = _run(d, nx, ny, nz, kinds, inplace)
    m = ~np.isnan(ref)
    assert m.any()
    assert not np.isnan(got[m]).any(), "defined entry not written"
    scale = max(1.0, np.abs(ref[m]).max())
    err = np.abs(got[m] - ref[m]).max() / scale
    assert err < TOL, (kinds, err)
    l2 = np.linalg.norm(got[m] - ref[m]) / np.linalg.norm(ref[m])
    assert l2 < TOL, (kinds, l2)


@pytest.mark.parametrize("inplace,dims", [(True, (8, 8, 8)), (False, (8, 6, 10)), (True, (32, 32, 32)),
                                          (False, (64, 32, 128))])
def test_all_kind_triples_small(inplace, dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(11)
    for kinds in itertools.product(range(8), repeat=3):
        d = rng.normal(size=E.padded_shape(nx, ny, nz))
        _check(d, nx, ny, nz, kinds, inplace)


@pytest.fixture(params=["default", "generic", "no_tma"])
def kernel_family(request):
    prev = api.set_kernel_family(request.param)
    yield request.param
    api.set_kernel_family(prev)


@pytest.mark.parametrize("n", [4, 6, 10, 16, 24, 32, 40, 48, 56, 64, 80, 88, 96, 104, 112, 128, 144, 160, 192,
                               256, 320, 384, 512, 1024])
def test_every_kind_per_length(n, kernel_family):
    """Each kind on each axis at one line length (radices 2..13, odd N/2), with
    the register-resident kernels (N = 32..1024, powers of two, and the mixed
    radix plans N = 24, 40, 48, 56, 80, 96, 112, 144, 160, 192, 320, 384; the
    TMA-pipelined strided pass at 192 and 320) and with the generic kernel for
    every length."""
    rng = np.random.default_rng(n)
    other = 6
    for kind in range(8):
        for axis in range(3):
            dims = [other, other, other]
            dims[axis] = n
            kinds = [E.DCT_2, E.DCT_2, E.DCT_2]
            kinds[axis] = kind
            d = rng.normal(size=E.padded_shape(*dims))
            _check(d, *dims, kinds, inplace=False)


@pytest.mark.parametrize("dims,kinds", [
    ((48, 40, 56), (E.DST_3, E.DCT_1, E.DFT_R2C)),
    ((64, 32, 96), (E.DFT_C2R, E.DST_2, E.DCT_3)),
    ((176, 16, 24), (E.DCT_1, E.DST_1, E.DST_3)),
    ((32, 192, 48), (E.DCT_2, E.DFT_R2C, E.DST_1)),
])
def test_noncubic_out_of_place(dims, kinds):
    d = np.random.default_rng(5).normal(size=E.padded_shape(*dims))
    _check(d, *dims, kinds, inplace=False)


def test_config1_standalone_transform_128():
    """128^3 in place, kinds (DST_1, DST_2, DFT_R2C), N(0,1) data."""
    d = np.random.default_rng(1).normal(size=E.padded_shape(128, 128, 128))
    _check(d, 128, 128, 128, (E.DST_1, E.DST_2, E.DFT_R2C), inplace=True)


def test_forward_inverse_round_trip_256():
    """Size-independent property at a large size: each inverse pair scales by
    N/2 per axis (N for DFT), as the solver's ratio assumes."""
    n = 256
    rng = np.random.default_rng(3)
    for fwd, inv, bcn in [((E.DST_3, E.DCT_1, E.DFT_R2C), (E.DST_2, E.DCT_1, E.DFT_C2R), None)]:
        d = np.zeros(E.padded_shape(n, n, n))
        # data on the solver's unknown windows of codes (2, 3, 0)
        d[0:n, 0:n + 1, 1:n + 1] = rng.uniform(-1, 1, size=(n, n + 1, n))
        dev = torch.from_numpy(d.ravel()).cuda()
        api.do_transform(dev, None, n, n, n, *fwd)
        api.do_transform(dev, None, n, n, n, *inv)
        torch.cuda.synchronize()
        got = dev.cpu().numpy().reshape(d.shape)
        scale = (n / 2) * (n / 2) * n
        w = (slice(0, n), slice(0, n + 1), slice(1, n + 1))
        rel = np.linalg.norm(got[w] / scale - d[w]) / np.linalg.norm(d[w])
        assert rel < 1e-13, rel


def test_not_cubic_inplace_raises():
    d = torch.zeros(api.padded_numel(8, 6, 10), dtype=torch.float64, device="cuda")
    with pytest.raises(api.CHZError) as ei:
        api.do_transform(d, None, 8, 6, 10, 0, 0, 0)
    assert ei.value.status == api.CHZ_ERROR_NOT_CUBIC
    # the extension entry point allows it, with the same results as out of place
    h = np.random.default_rng(2).normal(size=E.padded_shape(8, 6, 10))
    dev = torch.from_numpy(h.ravel()).cuda()
    api.do_transform(dev, None, 8, 6, 10, E.DST_2, E.DCT_3, E.DFT_R2C, allow_noncubic_inplace=True)
    torch.cuda.synchronize()
    ref = E.emulate_do_transform(h, 8, 6, 10, E.DST_2, E.DCT_3, E.DFT_R2C)
    got = dev.cpu().numpy().reshape(h.shape)
    m = ~np.isnan(ref)
    assert np.abs(got[m] - ref[m]).max() < TOL * max(1, np.abs(ref[m]).max())


def test_stream_ordering_on_side_stream():
    h = np.random.default_rng(4).normal(size=E.padded_shape(32, 32, 32))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        dev = torch.from_numpy(h.ravel()).cuda(non_blocking=False)
        api.do_transform(dev, None, 32, 32, 32, E.DCT_1, E.DST_3, E.DCT_2, stream=s)
    s.synchronize()
    ref = E.emulate_do_transform(h, 32, 32, 32, E.DCT_1, E.DST_3, E.DCT_2)
    got = dev.cpu().numpy().reshape(h.shape)
    m = ~np.isnan(ref)
    assert np.abs(got[m] - ref[m]).max() < TOL * max(1, np.abs(ref[m]).max())
