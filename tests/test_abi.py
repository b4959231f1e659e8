"""CPU tests of the C-ABI library: it builds for sm_100a, loads, exports every
symbol the headers in include/ declare, and rejects bad arguments with status
codes before any device work (no GPU needed for these calls)."""
import ctypes
import os
import re
import subprocess

import pytest

from cuhelmholtz_b200 import _build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


@pytest.fixture(scope="module")
def L():
    _build.build_library()
    from cuhelmholtz_b200 import _lib
    return _lib.lib()


def _c_decls():
    text = open(os.path.join(INCLUDE, "cuhelmholtz_b200.h")).read()
    return sorted(set(re.findall(r"\b(chz_[a-z0-9_]+)\s*\(", text)))


def _defined_symbols(demangle):
    args = ["nm", "-D", "--defined-only"] + (["-C"] if demangle else []) + [_build.LIBPATH]
    return subprocess.run(args, capture_output=True, text=True, check=True).stdout


def test_library_exports_every_c_declaration(L):
    syms = _defined_symbols(False)
    names = set(line.split()[-1] for line in syms.splitlines() if line.strip())
    decls = _c_decls()
    assert len(decls) >= 8
    missing = [d for d in decls if d not in names]
    assert not missing, missing


def test_library_exports_reference_cxx_signatures(L):
    """The C++-linkage drop-ins of funcinterface.h and cuda_helmholtz_solver.h
    (the reference's mangled names, e.g. _Z12do_transformPdS_iii14transform_kindS0_S0_)."""
    syms = _defined_symbols(True)
    expected = [
        "do_transform(double*, double*, int, int, int, transform_kind, transform_kind, transform_kind)",
        "do_transform_nocubic(double*, double*, int, int, int, transform_kind, transform_kind, transform_kind)",
        "do_transform_cubic(double*, int, int, int, transform_kind, transform_kind, transform_kind)",
        "freeMemory_cubic()",
        "cuda_helmholtz_solver(double, double, int, int, double*, double*, double, double, int, int, "
        "double*, double*, double, double, int, int, double*, double*, double, double*)",
    ]
    for e in expected:
        assert e in syms, e
    raw = _defined_symbols(False)
    assert "_Z12do_transformPdS_iii14transform_kindS0_S0_" in raw


def test_ctypes_binding_covers_header(L):
    from cuhelmholtz_b200._lib import SIGNATURES
    assert set(_c_decls()) == set(SIGNATURES)


def test_version_and_status_strings(L):
    assert L.chz_version() >= 100
    assert L.chz_status_string(0) == b"CHZ_SUCCESS"
    assert L.chz_status_string(3) == b"CHZ_ERROR_NOT_CUBIC"
    assert L.chz_status_string(99) == b"CHZ_ERROR_UNKNOWN"


FAKE = 0x10000  # never dereferenced: validation fails first


def test_transform_argument_validation(L):
    assert L.chz_do_transform(None, None, 8, 8, 8, 0, 0, 0, None) == 1
    assert L.chz_do_transform(FAKE, None, 8, 8, 8, 9, 0, 0, None) == 1
    assert L.chz_do_transform(FAKE, None, 8, 8, 8, 0, -1, 0, None) == 1
    assert L.chz_do_transform(FAKE, None, 7, 7, 7, 0, 0, 0, None) == 2   # odd
    assert L.chz_do_transform(FAKE, None, 2, 2, 2, 0, 0, 0, None) == 2   # too small
    assert L.chz_do_transform(FAKE, None, 4096, 8, 8, 0, 0, 0, None) == 2
    assert L.chz_do_transform(FAKE, None, 34, 8, 8, 0, 0, 0, None) == 2  # 17 is not a supported radix
    # in place on a non-cube: the reference exits, the C ABI reports it
    assert L.chz_do_transform(FAKE, None, 8, 6, 10, 0, 0, 0, None) == 3
    assert L.chz_do_transform(FAKE, FAKE, 8, 6, 10, 0, 0, 0, None) == 3
    assert b"cubic" in L.chz_last_error()


def _solve(L, nx=8, ny=8, nz=8, bcs=(1, 1, 1), faces=(None,) * 6, f=FAKE, lam=-1.0):
    return L.chz_helmholtz_solve(0.0, 1.0, nx, bcs[0], faces[0], faces[1],
                                 0.0, 1.0, ny, bcs[1], faces[2], faces[3],
                                 0.0, 1.0, nz, bcs[2], faces[4], faces[5], lam, f, None)


def test_solver_argument_validation(L):
    assert _solve(L, bcs=(5, 1, 1)) == 1
    assert b"bad boundary condition" in L.chz_last_error()
    assert _solve(L, bcs=(1, -1, 1)) == 1
    assert _solve(L, nx=9) == 2
    assert _solve(L, f=None) == 1
    # Neumann codes need their face arrays
    assert _solve(L, bcs=(3, 1, 1)) == 1
    assert _solve(L, bcs=(2, 1, 1), faces=(None, None, None, None, None, None)) == 1
    assert _solve(L, bcs=(1, 4, 1)) == 1
    # degenerate domain
    assert L.chz_helmholtz_solve(1.0, 1.0, 8, 1, None, None, 0.0, 1.0, 8, 1, None, None,
                                 0.0, 1.0, 8, 1, None, None, -1.0, FAKE, None) == 1


def test_workspace_size(L):
    assert L.chz_helmholtz_workspace_size(8, 8, 8, 0) >= 10 * 10 * 10 * 8
    assert L.chz_helmholtz_workspace_size(8, 8, 8, 0) % 256 == 0
    assert L.chz_helmholtz_workspace_size(0, 8, 8, 0) == 0
    assert L.chz_helmholtz_solve_ws(0.0, 1.0, 8, 1, None, None, 0.0, 1.0, 8, 1, None, None,
                                    0.0, 1.0, 8, 1, None, None, -1.0, FAKE, None, 0, None) == 6


def test_python_mirror_rejects_host_tensors(L):
    import torch
    from cuhelmholtz_b200 import api
    x = torch.zeros(10 * 10 * 10, dtype=torch.float64)
    with pytest.raises(ValueError):
        api.do_transform(x, None, 8, 8, 8, api.DST_1, api.DST_1, api.DST_1)
