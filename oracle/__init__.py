"""CPU oracle for the cuHelmholtz hot path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product imports this package: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs may
use it, and only as the checker (or the timed CPU baseline), never as the thing
measured or shipped.

Contents
--------
``emulation``   line-by-line numpy restatement of the reference GPU path
                (pre/post kernels of cudasymmfft/*.cu, cuFFT conventions, the
                3-D pass order of funcinterface.cu, and cuda_helmholtz_solver.cu
                with _cuda_helmholtz_.inl).  Entries the reference leaves
                undefined are NaN, so a comparison covers exactly what the
                reference defines.
``closed_form`` the same transforms written as the textbook sums (scipy.fft
                DCT/DST types with the reference's 1/2 scaling), used to
                cross-check ``emulation``.
``stencil``     the 7-point discrete Helmholtz operator with the reference's
                boundary closures (manufactured solutions, residuals).
``fishpack``    runs the reference's own CPU solver (``solver_3d`` over
                FISHPACK ``hw3crt``) built by ``oracle/Makefile`` into
                ``oracle/_ref/``.
``gen``         seeded synthetic problem generators with the benchmark
                configurations' shapes and value distributions.

Parity pin: ``emulation``'s solver is checked against fishpack outputs
committed under ``tests/golden/`` (made by ``tests/golden/make_golden.py``).
"""
from .emulation import (  # noqa: F401
    DCT_1, DCT_2, DCT_3, DST_1, DST_2, DST_3, DFT_R2C, DFT_C2R, KIND_NAMES,
    emulate_kind, emulate_do_transform, emulate_solver, padded_shape,
    solver_windows,
)
