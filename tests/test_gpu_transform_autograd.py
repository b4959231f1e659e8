"""GPU tests of the differentiable do_transform (autograd.transform): the
backward pass is the exact transpose of the forward map, checked by the
dot-product identity <g, T x> = <T^T g, x> for every kind triple."""
import itertools

import numpy as np
import pytest
import torch

from oracle import emulation as E
from cuhelmholtz_b200.autograd import transform

pytestmark = pytest.mark.gpu


def _check(nx, ny, nz, kinds, seed):
    rng = np.random.default_rng(seed)
    n = (nx + 2) * (ny + 2) * (nz + 2)
    x = torch.tensor(rng.normal(size=n), device="cuda", requires_grad=True)
    g = torch.tensor(rng.normal(size=n), device="cuda")
    y = transform(x, nx, ny, nz, *kinds)
    (gx,) = torch.autograd.grad(y, x, grad_outputs=g)
    lhs = float(torch.dot(g, y.detach()))
    rhs = float(torch.dot(gx, x.detach()))
    scale = float(torch.linalg.norm(g) * torch.linalg.norm(y.detach()))
    assert abs(lhs - rhs) <= 1e-12 * scale, (kinds, lhs, rhs)
    # the forward values are do_transform's on the output windows
    ref = E.emulate_do_transform(x.detach().cpu().numpy().reshape(E.padded_shape(nx, ny, nz)), nx, ny, nz, *kinds)
    got = y.detach().cpu().numpy().reshape(ref.shape)
    m = ~np.isnan(ref)
    assert np.linalg.norm(got[m] - ref[m]) <= 1e-12 * np.linalg.norm(ref[m])


@pytest.mark.parametrize("kinds", list(itertools.product(range(8), repeat=3)))
def test_transpose_every_kind_triple(kinds):
    _check(8, 6, 10, kinds, seed=sum(k * 8 ** i for i, k in enumerate(kinds)))


@pytest.mark.parametrize("dims,kinds", [((32, 64, 16), (3, 4, 6)), ((64, 48, 128), (0, 5, 7)),
                                        ((128, 128, 128), (1, 2, 6)), ((512, 16, 16), (5, 0, 2))])
def test_transpose_larger(dims, kinds):
    _check(*dims, kinds, seed=7)
