"""Python mirror of the reference's interface for the hot path, over the C-ABI.

Same names, argument order and meaning as the reference:

* ``do_transform(d_data, d_out, NX, NY, NZ, X_TRANS, Y_TRANS, Z_TRANS)``
  (cudasymmfft/funcinterface.h:5-12)
* ``cuda_helmholtz_solver(left, right, NX, xbc, bcl, bcr, bottom, top, NY, ybc,
  bcb, bct, front, back, NZ, zbc, bcf, bce, lambda_, f)``
  (cudahelmholtz/cuda_helmholtz_solver.h:5-11)

Arrays are CUDA float64 torch tensors (device memory; torch is only the
allocator and stream provider here).  Where the reference ends the process
(bad boundary code, in-place call on a non-cube, CUDA error) these raise
:class:`CHZError` with the library's status and message.  Calls are
stream-ordered on torch's current stream; they do not synchronise.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _lib

# transform_kind, cudasymmfft/global.h:6-15
DCT_1, DCT_2, DCT_3, DST_1, DST_2, DST_3, DFT_R2C, DFT_C2R = range(8)
KIND_NAMES = ("DCT_1", "DCT_2", "DCT_3", "DST_1", "DST_2", "DST_3", "DFT_R2C", "DFT_C2R")

CHZ_SUCCESS = 0
CHZ_ERROR_INVALID_VALUE = 1
CHZ_ERROR_UNSUPPORTED_SIZE = 2
CHZ_ERROR_NOT_CUBIC = 3
CHZ_ERROR_CUDA = 4
CHZ_ERROR_ALLOC = 5
CHZ_ERROR_WORKSPACE = 6
CHZ_ERROR_TIMEOUT = 7


class CHZError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_lib.lib().chz_status_string(status).decode()}: {message}")


def _check(status: int) -> None:
    if status != CHZ_SUCCESS:
        raise CHZError(status, _lib.lib().chz_last_error().decode())


def _ptr(t: Optional[torch.Tensor], name: str, numel: Optional[int] = None) -> int:
    if t is None:
        return 0
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (device memory)")
    if t.dtype != torch.float64:
        raise ValueError(f"{name} must be float64")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if numel is not None and t.numel() < numel:
        raise ValueError(f"{name} holds {t.numel()} values, needs {numel}")
    return t.data_ptr()


def _stream(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


def padded_numel(nx: int, ny: int, nz: int) -> int:
    return (nx + 2) * (ny + 2) * (nz + 2)


def do_transform(d_data: torch.Tensor, d_out: Optional[torch.Tensor], NX: int, NY: int, NZ: int,
                 X_TRANS: int, Y_TRANS: int, Z_TRANS: int, stream=None,
                 allow_noncubic_inplace: bool = False) -> torch.Tensor:
    """3-D mixed transform on the padded (NZ+2, NY+2, NX+2) array.  Returns the
    tensor holding the result (``d_data`` in place, else ``d_out``)."""
    n = padded_numel(NX, NY, NZ)
    p_in = _ptr(d_data, "d_data", n)
    p_out = _ptr(d_out, "d_out", n) if d_out is not None else 0
    fn = _lib.lib().chz_do_transform_any if allow_noncubic_inplace else _lib.lib().chz_do_transform
    _check(fn(p_in, p_out, NX, NY, NZ, int(X_TRANS), int(Y_TRANS), int(Z_TRANS), _stream(stream)))
    return d_data if (d_out is None or p_out == p_in) else d_out


def _face_len(axis: str, nx: int, ny: int, nz: int) -> int:
    return {"x": (ny + 1) * (nz + 1), "y": (nx + 1) * (nz + 1), "z": (nx + 1) * (ny + 1)}[axis]


def cuda_helmholtz_solver(left, right, NX, xbc, bcl, bcr,
                          bottom, top, NY, ybc, bcb, bct,
                          front, back, NZ, zbc, bcf, bce,
                          lambda_, f, stream=None, workspace: Optional[torch.Tensor] = None):
    """Solves lap_h u + lambda u = f in place on ``f`` ((NZ+1, NY+1, NX+1)
    float64 CUDA tensor).  Returns 0 like the reference."""
    n = (NX + 1) * (NY + 1) * (NZ + 1)
    pf = _ptr(f, "f", n)
    fx, fy, fz = (_face_len(a, NX, NY, NZ) for a in "xyz")
    faces = [_ptr(bcl, "bcl", fx), _ptr(bcr, "bcr", fx), _ptr(bcb, "bcb", fy),
             _ptr(bct, "bct", fy), _ptr(bcf, "bcf", fz), _ptr(bce, "bce", fz)]
    L = _lib.lib()
    if workspace is None:
        st = L.chz_helmholtz_solve(float(left), float(right), NX, xbc, faces[0], faces[1],
                                   float(bottom), float(top), NY, ybc, faces[2], faces[3],
                                   float(front), float(back), NZ, zbc, faces[4], faces[5],
                                   float(lambda_), pf, _stream(stream))
    else:
        if not workspace.is_cuda:
            raise ValueError("workspace must be device memory")
        st = L.chz_helmholtz_solve_ws(float(left), float(right), NX, xbc, faces[0], faces[1],
                                      float(bottom), float(top), NY, ybc, faces[2], faces[3],
                                      float(front), float(back), NZ, zbc, faces[4], faces[5],
                                      float(lambda_), pf, workspace.data_ptr(),
                                      workspace.numel() * workspace.element_size(), _stream(stream))
    _check(st)
    return 0


def helmholtz_solve_19pt(left, right, NX, xbc, bcl, bcr,
                         bottom, top, NY, ybc, bcb, bct,
                         front, back, NZ, zbc, bcf, bce,
                         lambda_, f, stream=None) -> int:
    """cuda_helmholtz_solver with the reference's 19-point division (compact
    fourth-order Laplacian, filtered right-hand side): codes 1 and 3 and one
    grid spacing on all axes.  In place on ``f``."""
    n = (NX + 1) * (NY + 1) * (NZ + 1)
    pf = _ptr(f, "f", n)
    fx, fy, fz = (_face_len(a, NX, NY, NZ) for a in "xyz")
    faces = [_ptr(bcl, "bcl", fx), _ptr(bcr, "bcr", fx), _ptr(bcb, "bcb", fy),
             _ptr(bct, "bct", fy), _ptr(bcf, "bcf", fz), _ptr(bce, "bce", fz)]
    _check(_lib.lib().chz_helmholtz_solve_19pt(
        float(left), float(right), NX, xbc, faces[0], faces[1],
        float(bottom), float(top), NY, ybc, faces[2], faces[3],
        float(front), float(back), NZ, zbc, faces[4], faces[5],
        float(lambda_), pf, _stream(stream)))
    return 0


def helmholtz_solve_pertrb(left, right, NX, xbc, bcl, bcr,
                           bottom, top, NY, ybc, bcb, bct,
                           front, back, NZ, zbc, bcf, bce,
                           lambda_, f, stream=None) -> float:
    """cuda_helmholtz_solver that also returns FISHPACK's PERTRB: for a
    singular problem (lambda = 0, every code 0 or 3) the constant removed from
    the right-hand side so that a solution exists, else 0.  Solves in place
    on ``f`` (the zero-mode solution)."""
    import ctypes
    n = (NX + 1) * (NY + 1) * (NZ + 1)
    pf = _ptr(f, "f", n)
    fx, fy, fz = (_face_len(a, NX, NY, NZ) for a in "xyz")
    faces = [_ptr(bcl, "bcl", fx), _ptr(bcr, "bcr", fx), _ptr(bcb, "bcb", fy),
             _ptr(bct, "bct", fy), _ptr(bcf, "bcf", fz), _ptr(bce, "bce", fz)]
    out = ctypes.c_double(0.0)
    _check(_lib.lib().chz_helmholtz_solve_pertrb(
        float(left), float(right), NX, xbc, faces[0], faces[1],
        float(bottom), float(top), NY, ybc, faces[2], faces[3],
        float(front), float(back), NZ, zbc, faces[4], faces[5],
        float(lambda_), pf, ctypes.byref(out), _stream(stream)))
    return out.value


def helmholtz_solve_refined(left, right, NX, xbc, bcl, bcr,
                            bottom, top, NY, ybc, bcb, bct,
                            front, back, NZ, zbc, bcf, bce,
                            lambda_, f, max_corrections: int = 2, tol: float = 0.0,
                            stream=None, workspace: Optional[torch.Tensor] = None,
                            report: bool = False):
    """FP32 transforms + FP64-residual iterative refinement, in place on
    ``f``.  Returns (corrections_done, last relative residual or -1)."""
    import ctypes
    n = (NX + 1) * (NY + 1) * (NZ + 1)
    pf = _ptr(f, "f", n)
    fx, fy, fz = (_face_len(a, NX, NY, NZ) for a in "xyz")
    faces = [_ptr(bcl, "bcl", fx), _ptr(bcr, "bcr", fx), _ptr(bcb, "bcb", fy),
             _ptr(bct, "bct", fy), _ptr(bcf, "bcf", fz), _ptr(bce, "bce", fz)]
    done = ctypes.c_int(0)
    relr = ctypes.c_double(-1.0)
    ws = workspace.data_ptr() if workspace is not None else None
    wsb = workspace.numel() * workspace.element_size() if workspace is not None else 0
    st = _lib.lib().chz_helmholtz_solve_refined(
        float(left), float(right), NX, xbc, faces[0], faces[1],
        float(bottom), float(top), NY, ybc, faces[2], faces[3],
        float(front), float(back), NZ, zbc, faces[4], faces[5],
        float(lambda_), pf, int(max_corrections), float(tol),
        ctypes.byref(done), ctypes.byref(relr) if report else None, ws, wsb, _stream(stream))
    _check(st)
    return done.value, relr.value


class BatchPlan:
    """Plan for many independent FP64 solves (sizes, codes, domains, lambdas
    fixed at creation); ``solve`` runs the whole batch as one graph replay:
    one persistent launch over a work queue, or one launch per pass, whichever
    measured faster at creation (``launch_mode``).

    problems: sequence of dicts with keys nx, ny, nz, xbc, ybc, zbc, lam and
    optionally dom (left, right, bottom, top, front, back)."""

    def __init__(self, problems):
        import ctypes
        n = len(problems)
        self.count = n
        self.problems = list(problems)
        dims = (ctypes.c_int * (3 * n))(*[v for p in problems for v in (p["nx"], p["ny"], p["nz"])])
        bcs = (ctypes.c_int * (3 * n))(*[v for p in problems for v in (p["xbc"], p["ybc"], p["zbc"])])
        doms = (ctypes.c_double * (6 * n))(*[float(v) for p in problems
                                             for v in p.get("dom", (0, 1, 0, 1, 0, 1))])
        lams = (ctypes.c_double * n)(*[float(p["lam"]) for p in problems])
        self._handle = ctypes.c_void_p()
        _check(_lib.lib().chz_batch_plan_create(n, dims, bcs, doms, lams, ctypes.byref(self._handle)))

    def solve(self, fs, faces=None, stream=None):
        """fs: list of CUDA float64 tensors (solved in place); faces: list of
        dicts {bcl..bce: tensor or None} or None."""
        import ctypes
        n = self.count
        if len(fs) != n:
            raise ValueError(f"expected {n} right-hand sides")
        fp = (ctypes.c_void_p * n)(*[_ptr(f, "f", (p["nx"] + 1) * (p["ny"] + 1) * (p["nz"] + 1))
                                     for f, p in zip(fs, self.problems)])
        keys = ("bcl", "bcr", "bcb", "bct", "bcf", "bce")
        if faces is None:
            fc = None
        else:
            fc = (ctypes.c_void_p * (6 * n))(*[(_ptr(d.get(k), k) or None) if d else None
                                               for d in faces for k in keys])
        _check(_lib.lib().chz_batch_solve(self._handle, fp, fc, _stream(stream)))

    def workspace_bytes(self) -> int:
        return int(_lib.lib().chz_batch_workspace_bytes(self._handle))

    def tiles(self):
        """Tile size (values per tile) the autotuner chose for each of the
        five passes, and the measured time per launch in ms (0: not tuned)."""
        import ctypes
        t = (ctypes.c_int * 5)()
        ms = (ctypes.c_float * 5)()
        _check(_lib.lib().chz_batch_plan_tiles(self._handle, t, ms))
        return list(t), [float(v) for v in ms]

    def radix_schedules(self):
        """Radix schedule the autotuner chose for each of the five passes (0:
        8s first, then 4 / 2, then odd primes; 1: reversed; 2: 4s in place
        of the 8s)."""
        import ctypes
        v = (ctypes.c_int * 5)()
        _check(_lib.lib().chz_batch_plan_radix(self._handle, v))
        return list(v)

    def kernels(self) -> int:
        """Kernel launches one solve of this plan replays (1 in the persistent
        form; per pass its register-resident groups and leftover launch, plus
        the periodic planes, in the per-pass form)."""
        n = int(_lib.lib().chz_batch_plan_kernels(self._handle))
        if n < 0:
            _check(n)
        return n

    def launch_mode(self):
        """The plan's launch form (0: one persistent launch; 1: launches per
        pass, register-resident groups and the generic kernel for the rest)
        and the measured ms of one batched solve in each ([0, 0]: not
        timed)."""
        import ctypes
        m = ctypes.c_int()
        ms = (ctypes.c_float * 2)()
        _check(_lib.lib().chz_batch_plan_launch(self._handle, ctypes.byref(m), ms))
        return int(m.value), [float(v) for v in ms]

    @staticmethod
    def set_launch_mode(mode) -> int:
        """Fixes the launch form of plans created afterwards (0, 1; None or -1
        times both, the default); returns the previous setting."""
        m = -1 if mode is None else int(mode)
        prev = int(_lib.lib().chz_batch_set_launch_mode(m))
        if prev == -2:
            raise ValueError(f"unknown launch form {mode}")
        return prev

    @staticmethod
    def set_autotune(on: bool) -> bool:
        """Turns the plans' autotuner on (default) or off; returns the
        previous setting."""
        return bool(_lib.lib().chz_batch_set_autotune(1 if on else 0))

    def close(self):
        if self._handle:
            _lib.lib().chz_batch_plan_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


KERNEL_FAMILIES = {"default": 0, "generic": 1, "no_tma": 2}


def set_kernel_family(family) -> int:
    """Selects the kernels: "default" (0: TMA-pipelined strided passes,
    register-resident line kernels, mixed-radix elsewhere), "generic" (1, or
    True: the mixed-radix kernel for every pass) or "no_tma" (2).  Returns the
    previous setting (an int, accepted back)."""
    if isinstance(family, str):
        family = KERNEL_FAMILIES[family]
    elif isinstance(family, bool):
        family = 1 if family else 0
    prev = _lib.lib().chz_set_kernel_family(int(family))
    if prev < 0:
        raise ValueError(f"unknown kernel family {family!r}")
    return prev


def debug_flags(reset: bool = True) -> int:
    """Flags raised by the kernels' bounded waits (0: none ran out)."""
    return int(_lib.lib().chz_debug_flags(1 if reset else 0))


def stream_status(stream=None) -> None:
    """Waits for ``stream`` (default: the current one) and raises CHZError
    (CHZ_ERROR_TIMEOUT) when a kernel of this library gave up one of its
    bounded waits since the last check -- the results queued since then are
    not valid -- or CHZ_ERROR_CUDA on a CUDA error."""
    _check(_lib.lib().chz_stream_status(ctypes.c_void_p(_stream(stream))))


def set_wait_limit(cycles: int) -> int:
    """Limit of the kernels' bounded waits in SM clock cycles (>= 1e6; <= 0
    restores the default of 2e9).  Returns the previous limit."""
    return int(_lib.lib().chz_set_wait_limit(int(cycles)))


def wait_selftest(cycles: int = 1_000_000, stream=None) -> None:
    """Queues the self-test kernel whose wait runs out after ``cycles`` SM
    clock cycles (nothing arrives at its barrier); ``stream_status`` then
    raises CHZ_ERROR_TIMEOUT."""
    _check(_lib.lib().chz_wait_selftest(int(cycles), ctypes.c_void_p(_stream(stream))))


def workspace_size(NX: int, NY: int, NZ: int, precision: int = 0) -> int:
    return int(_lib.lib().chz_helmholtz_workspace_size(NX, NY, NZ, precision))


def solve_problem(p: dict, f: torch.Tensor, faces: Optional[dict] = None, stream=None):
    """Convenience: solve a problem dict (keys nx, ny, nz, xbc, ybc, zbc, dom,
    lam) in place on the device tensor ``f``; ``faces`` maps bcl..bce to device
    tensors (or None)."""
    faces = faces or {}
    d = p["dom"]
    return cuda_helmholtz_solver(d[0], d[1], p["nx"], p["xbc"], faces.get("bcl"), faces.get("bcr"),
                                 d[2], d[3], p["ny"], p["ybc"], faces.get("bcb"), faces.get("bct"),
                                 d[4], d[5], p["nz"], p["zbc"], faces.get("bcf"), faces.get("bce"),
                                 p["lam"], f, stream=stream)
