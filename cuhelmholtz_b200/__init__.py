"""cuhelmholtz_b200: B200-native (sm_100a) 3-D mixed DFT/DST/DCT transform and
FFT-diagonalised Helmholtz solver, a drop-in for the hot path of cuHelmholtz.

The compute path is the in-tree CUDA library ``lib/libcuhelmholtz_b200.so``
(C ABI in ``include/cuhelmholtz_b200.h``); this package is a thin host-side
mirror of the reference's interface over that ABI.  There is no CPU fallback.
"""
from .api import (  # noqa: F401
    BatchPlan, CHZError, DCT_1, DCT_2, DCT_3, DST_1, DST_2, DST_3, DFT_R2C, DFT_C2R, KIND_NAMES,
    cuda_helmholtz_solver, do_transform, helmholtz_solve_19pt, helmholtz_solve_pertrb, helmholtz_solve_refined, padded_numel, set_kernel_family,
    solve_problem, workspace_size,
)
from ._lib import lib, library_path  # noqa: F401
from .pipeline import HostPipeline  # noqa: F401

__version__ = "0.1.0"
