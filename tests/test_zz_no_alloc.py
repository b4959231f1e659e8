"""GPU test of the allocation-free solve entry point, chz_helmholtz_solve_noalloc.

It exists for callers that cannot call cudaMalloc (memory owned by another
allocator, a fixed budget, code that must not wait on the allocator): its work
array and tables are fixed-size __device__ arrays inside the library.  The test
calls it through the C ABI twice in a row, on problems of different sizes and
boundary codes (so the second call runs over the first call's leftovers in the
shared arrays), and compares each result with chz_helmholtz_solve's.  It also
checks that a problem beyond the array's capacity is rejected before any
device work.  This file is collected last so that a failure here does not stop
a -x run before the other tests.
"""
import numpy as np
import pytest
import torch

from cuhelmholtz_b200 import _lib, api
from oracle import gen
from oracle.stencil import FACE_KEYS

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _device(p):
    f = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    faces = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
             for k in FACE_KEYS}
    return f, faces


def _args(p, f, faces):
    d = p["dom"]
    ptr = lambda t: 0 if t is None else t.data_ptr()  # noqa: E731
    return (d[0], d[1], p["nx"], p["xbc"], ptr(faces["bcl"]), ptr(faces["bcr"]),
            d[2], d[3], p["ny"], p["ybc"], ptr(faces["bcb"]), ptr(faces["bct"]),
            d[4], d[5], p["nz"], p["zbc"], ptr(faces["bcf"]), ptr(faces["bce"]),
            p["lam"], f.data_ptr(), torch.cuda.current_stream().cuda_stream)


def _solve(entry, p):
    f, faces = _device(p)
    st = entry(*_args(p, f, faces))
    assert st == 0, _lib.lib().chz_last_error()
    torch.cuda.synchronize()
    return f.cpu().numpy()


def test_noalloc_matches_allocating_solver_on_two_calls_in_a_row():
    L = _lib.lib()
    problems = [gen.random_problem(96, 64, 128, 3, 4, 0, -1.0, seed=31),   # register kernels
                gen.random_problem(48, 40, 56, 2, 0, 1, -7.5, seed=32)]    # mixed-radix kernel
    for p in problems:
        a = _solve(L.chz_helmholtz_solve_noalloc, p)
        b = _solve(L.chz_helmholtz_solve, p)
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel < TOL, rel


@pytest.mark.parametrize("dims,codes", [((48, 40, 512), (3, 4, 0)),    # TMA z pass, spectrum in registers
                                        ((64, 48, 256), (1, 2, 0))])   # the same at N = 256
def test_noalloc_tma_z_pass_on_the_static_arrays(dims, codes):
    """Lengths 256 and 512 on z take the TMA-pipelined z pass, whose tensor
    maps are then built over the __device__ work array."""
    L = _lib.lib()
    p = gen.random_problem(*dims, *codes, -1.0, seed=33)
    for _ in range(2):
        a = _solve(L.chz_helmholtz_solve_noalloc, p)
        b = _solve(L.chz_helmholtz_solve, p)
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel < TOL, rel


def test_noalloc_allocates_no_device_memory():
    """With every library cache released, a call of a size the library has
    just released leaves the device's free memory unchanged (an allocation by
    the library would take at least one 2 MiB page)."""
    L = _lib.lib()
    p = gen.random_problem(72, 56, 80, 0, 3, 2, -2.5, seed=34)
    _solve(L.chz_helmholtz_solve_noalloc, p)      # loads the kernels this size uses
    torch.cuda.synchronize()
    assert L.chz_release_cached() == 0
    torch.cuda.empty_cache()
    free0, _ = torch.cuda.mem_get_info()
    f, faces = _device(p)                          # input and output only (torch allocates them)
    free1, _ = torch.cuda.mem_get_info()
    st = L.chz_helmholtz_solve_noalloc(*_args(p, f, faces))
    assert st == 0, L.chz_last_error()
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    assert free2 == free1, (free0, free1, free2)


def test_noalloc_rejects_problems_beyond_its_scratch():
    L = _lib.lib()
    p = dict(nx=512, ny=512, nz=512, xbc=1, ybc=1, zbc=1, dom=gen.UNIT_DOMAIN, lam=-1.0)
    f = torch.zeros(8, dtype=torch.float64, device="cuda")  # never touched: rejected first
    faces = {k: None for k in FACE_KEYS}
    st = L.chz_helmholtz_solve_noalloc(*_args(p, f, faces))
    assert st == api.CHZ_ERROR_UNSUPPORTED_SIZE
    assert b"scratch" in L.chz_last_error()
