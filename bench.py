#!/usr/bin/env python
"""Benchmark of the hot path: FP64 Helmholtz solves per second on one or more
B200s (one process per GPU, independent replicas), plus the reference's CPU
solver (FISHPACK hw3crt through the reference wrapper) as the baseline arm.

Default workload: 512^3 cells, boundary codes (3, 4, 0), lambda = -1,
f ~ U[-1, 1] + 1e3 cos(pi x) cos(pi y / 2) cos(2 pi z), Neumann data ~ U[-1, 1]
(seeded synthetic data with the precision configuration's shapes and value
distributions).  A step solves a batch of `--batch` such problems, each held in
its own device array; arrays are larger than L2, so no flush is needed.

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (nx, ny, nz, xbc, ybc, zbc, lam, description)
    "helmholtz_fp64_512": (512, 512, 512, 3, 4, 0, -1.0,
                           "FP64 Helmholtz solve 512^3, BC (3,4,0), lambda=-1, f~U[-1,1]+1e3 smooth mode"),
    "helmholtz_fp64_256": (256, 256, 256, 1, 3, 0, -4.0,
                           "FP64 Helmholtz solve 256^3, BC (1,3,0), lambda=-4, f~N(0,1)"),
    "helmholtz_fp64_128": (128, 128, 128, 1, 2, 0, -2.0,
                           "FP64 Helmholtz solve 128^3, BC (1,2,0), lambda=-2, manufactured 4-mode u"),
    "helmholtz_fp64_256x192x320": (256, 192, 320, 2, 4, 3, -7.3,
                                   "FP64 Helmholtz solve 256x192x320, BC (2,4,3), f~U[-1,1]"),
}
DEFAULT_WORKLOAD = "helmholtz_fp64_512"

# Per-pass DRAM bytes (read + write) per launch come from the committed ncu
# summary TRAFFIC_SUMMARY (one capture of each pass, with the digest of the
# CUDA sources it was captured on); a digest that differs from the current
# sources marks the figure stale in the bench line.
TRAFFIC_SUMMARY = os.path.join(ROOT, "profiles", "solve_pass_traffic.md")
METRIC = "solves/s (FP64 Helmholtz solve)"


def make_problem(name, seed):
    from oracle import gen
    nx, ny, nz, xbc, ybc, zbc, lam, _ = WORKLOADS[name]
    if name == "helmholtz_fp64_512":
        return gen.config3_problem(seed=seed, n=nx)
    if name == "helmholtz_fp64_256":
        return gen.config5_problem(seed=seed, n=nx)
    if name == "helmholtz_fp64_128":
        return gen.config1_problem(seed=seed, n=nx)
    return gen.random_problem(nx, ny, nz, xbc, ybc, zbc, lam, seed=seed)


# ---------------------------------------------------------------------------
# algorithmic bytes of the solver schedule (mirrors the host planner)
# ---------------------------------------------------------------------------

def _windows(bc, n):
    s, e = {0: (0, n - 1), 1: (1, n - 1), 2: (1, n), 3: (0, n), 4: (0, n - 1)}[bc]
    sp1 = n + 1 if bc == 0 else e
    return s, e, s, sp1


def solve_pass_bytes(nx, ny, nz, xbc, ybc, zbc, esize=8):
    """Bytes each line pass of one solve must read and write (algorithmic:
    every loaded and stored entry once), by trace label, in launch order."""
    xs, xe, xp0, xp1 = _windows(xbc, nx)
    ys, ye, yp0, yp1 = _windows(ybc, ny)
    zs, ze, zp0, zp1 = _windows(zbc, nz)
    X, Xs = xe - xs + 1, xp1 - xp0 + 1
    Y, Ys = ye - ys + 1, yp1 - yp0 + 1
    Z, Zs = ze - zs + 1, zp1 - zp0 + 1
    return {
        "solve_x_fwd": (Y * Z) * (X + Xs) * esize,            # f -> work
        "solve_y_fwd": (Xs * Z) * (Y + Ys) * esize,
        "solve_z_fwd_div_inv": (Xs * Ys) * (Z + Z) * esize,   # forward, divide, inverse
        "solve_y_inv": (Xs * Z) * (Ys + Y) * esize,
        "solve_x_inv": (Y * Z) * (Xs + X) * esize,            # work -> f
    }


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_ids):
        self.gpu_ids = gpu_ids
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", ",".join(self.gpu_ids), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def nvml_ids_for_visible(devices):
    """nvidia-smi ids (UUIDs) of the given torch device indices."""
    import torch
    out = []
    for d in devices:
        try:
            u = str(torch.cuda.get_device_properties(d).uuid)
            out.append(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            out.append(str(d))
    return out


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


# ---------------------------------------------------------------------------
# CPU baselines (reference CPU solver)
# ---------------------------------------------------------------------------

def cpu_baseline_single(p):
    """One FISHPACK solve of problem p on one host core: the timed CPU
    baseline, and the reference solution the GPU results are compared with.
    Returns (record, u) -- u is None when the runner is not built."""
    from oracle import fishpack
    if not fishpack.available():
        return ({"value": None, "unit": "solves/s", "cores": 1, "kind": "reference",
                 "sample": "unavailable: fishpack runner not built"}, None)
    u, best, _ = fishpack.solve(p, repeats=1)
    return ({"value": 1.0 / best, "unit": "solves/s", "cores": 1, "kind": "reference",
             "seconds_per_solve": best,
             "sample": f"one {p['nx']}x{p['ny']}x{p['nz']} BC ({p['xbc']},{p['ybc']},{p['zbc']}) solve, "
                       "FISHPACK hw3crt via the reference's solver_3d, 1 thread"}, u)


def reference_gpu_solve(p, repeats):
    """The reference's own GPU solver (cudasymmfft over cuFFT, compiled
    unchanged for sm_100a; a child process) on problem p: (record, u), or
    (None, None) when oracle/_ref/cudaref_run is not built."""
    from oracle import cudaref
    if not cudaref.available():
        return None, None
    u, best, med = cudaref.solve(p, repeats=repeats)
    return ({"value": 1.0 / best, "unit": "solves/s", "seconds_per_solve": best, "median_s": med,
             "repeats": repeats,
             "kind": "reference cuda_helmholtz_solver + cudasymmfft over cuFFT, compiled for sm_100a",
             "timing": "wall time of the synchronous call (its per-call plans, allocations and "
                       "synchronisations included), f re-uploaded between calls"}, u)


def rel_l2(a, b):
    import numpy as np
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def load_traffic():
    """{(workload, pass label): DRAM bytes per launch} from the committed ncu
    summary, and whether it was captured on the current CUDA sources."""
    from cuhelmholtz_b200 import _build
    table, digest = {}, None
    if os.path.exists(TRAFFIC_SUMMARY):
        with open(TRAFFIC_SUMMARY) as fh:
            for line in fh:
                line = line.strip()
                if line.startswith("source digest:"):
                    digest = line.split(":", 1)[1].strip().strip("`")
                if line.startswith("| helmholtz_"):
                    cells = [c.strip().strip("`") for c in line.strip("|").split("|")]
                    try:
                        table[(cells[0], cells[1])] = int(cells[3])
                    except (IndexError, ValueError):
                        pass
    return table, digest, (digest is not None and digest == _build.source_digest())


# forward transform kind of each boundary code (the solver's first passes)
FORWARD_KIND = {0: 6, 1: 3, 2: 5, 3: 0, 4: 2}
# the standalone transform of the 128^3 configuration: DST-I, DST-II, DFT (in place)
TRANSFORM_KINDS = {"helmholtz_fp64_128": (3, 4, 6)}


def time_transform(chz, name, nx, ny, nz, bcs, steps, warmup, world, peak):
    """do_transform timed alone: in place on cubic grids, out of place
    otherwise (the reference's rule), FP64, kinds = the workload's forward
    kinds.  Enough arrays are cycled that the working set exceeds L2."""
    import numpy as np
    import torch
    kinds = TRANSFORM_KINDS.get(name, tuple(FORWARD_KIND[b] for b in bcs))
    n = chz.padded_numel(nx, ny, nz)
    inplace = nx == ny == nz
    per = n * 8 * (1 if inplace else 2)
    count = max(2, -(-(256 << 20) // per))
    rng = np.random.default_rng(17)
    base = torch.from_numpy(rng.standard_normal(n)).cuda()
    bufs = [base.clone() for _ in range(count)]
    outs = [None if inplace else torch.empty_like(base) for _ in range(count)]

    def run(i):
        chz.do_transform(bufs[i], outs[i], nx, ny, nz, *kinds)

    for w in range(max(warmup, 1)):
        for i in range(count):
            run(i)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        run(k % count)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, "cuda") / steps
    model_bytes = 48 * nx * ny * nz
    gbs = model_bytes / (ms / 1000.0) / 1e9
    return {"kinds": [chz.KIND_NAMES[k] for k in kinds], "inplace": inplace, "value": world * 1000.0 / ms,
            "unit": "transforms/s", "ms_per_transform": ms, "model_bytes": model_bytes,
            "model": "48 B per point (3 passes x 8 B read + 8 B written), points = NX*NY*NZ",
            "model_gbs": gbs, "frac_of_peak": gbs / peak, "arrays_cycled": count}


def run_reference_arm(args):
    """The reference's CPU implementation of the path on the host cores:
    concurrent single-threaded hw3crt processes (hw3crt is serial)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import fishpack
    name = args.workload
    nx, ny, nz, xbc, ybc, zbc, lam, desc = WORKLOADS[name]
    if not fishpack.available():
        print(json.dumps({"impl": "reference", "unavailable": "fishpack runner (oracle/_ref) not built"}))
        return 0
    p = make_problem(name, seed=3)
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 64 << 30
    per_proc = 3 * (nx + 1) * (ny + 1) * (nz + 1) * 8 + (256 << 20)
    procs = max(1, min(cores, int(avail * 0.6 // per_proc), args.ref_procs))
    small = make_problem("helmholtz_fp64_128", seed=1)
    for _ in range(args.warmup):
        fishpack.solve_many_parallel(small, procs)  # untimed: warms the binary and page cache
    times = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ts = fishpack.solve_many_parallel(p, procs)
        times.append(max(ts))
    wall = time.perf_counter() - t0
    total = sum(times)
    value = procs * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": name, "description": desc, "grid": [nx, ny, nz],
                   "bc": [xbc, ybc, zbc], "lambda": lam, "processes": procs},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": "reference",
                         "sample": f"each step: {procs} concurrent {nx}x{ny}x{nz} solves, one "
                                   "single-threaded FISHPACK hw3crt process per core; warm-up "
                                   "steps solve 128^3"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# multi-rank bookkeeping (one process per GPU, independent replicas)
# ---------------------------------------------------------------------------

def max_over_ranks(ms, world, device):
    """The largest of the ranks' device times (every rank calls this, in the
    same order; a single process returns its own)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, max_ms):
    """Whole-job units per second: all ranks' units over the slowest rank's
    time."""
    return units_per_rank / (max_ms / 1000.0)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def measure_workload(name, args, world, rank, local, headline):
    """Times one workload on this rank: the FP64 solve (device-timed), the
    per-pass roofline from the library's event tracing, do_transform alone,
    the FP32 + FP64-refinement solve and, on the headline workload, the end to
    end figure through the public host-buffer API.  Every rank calls this with
    the same arguments (the max-over-ranks reductions are collectives).
    Returns the record and the host solutions used for the error checks."""
    import numpy as np
    import torch

    import cuhelmholtz_b200 as chz
    from cuhelmholtz_b200 import _lib
    from cuhelmholtz_b200.pipeline import HostPipeline
    from oracle.stencil import FACE_KEYS
    import torch.distributed as dist

    def barrier():
        if world > 1:
            dist.barrier()

    nx, ny, nz, xbc, ybc, zbc, lam, desc = WORKLOADS[name]
    p = make_problem(name, seed=3 + rank)
    npts = (nx + 1) * (ny + 1) * (nz + 1)
    B = args.batch
    steps = args.steps if headline else args.sub_steps
    stream = torch.cuda.current_stream()

    f_host = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).pin_memory()
    u_host = torch.empty_like(f_host).pin_memory()
    fs = [f_host.to("cuda", non_blocking=False) for _ in range(B)]
    faces_h = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).pin_memory())
               for k in FACE_KEYS}
    faces = {k: (None if v is None else v.to("cuda")) for k, v in faces_h.items()}
    dom = p["dom"]

    def solve(f):
        chz.cuda_helmholtz_solver(dom[0], dom[1], nx, xbc, faces["bcl"], faces["bcr"],
                                  dom[2], dom[3], ny, ybc, faces["bcb"], faces["bct"],
                                  dom[4], dom[5], nz, zbc, faces["bcf"], faces["bce"],
                                  lam, f)

    for _ in range(args.warmup):
        for f in fs:
            solve(f)
    torch.cuda.synchronize()

    # ---- device-timed throughput ----
    sampler = ClockSampler(nvml_ids_for_visible([local])) if (rank == 0 and headline) else None
    barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.15)
    launches0 = _lib.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        for f in fs:
            solve(f)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = _lib.launch_count() - launches0
    elapsed_ms = ev0.elapsed_time(ev1)
    clocks = sampler.stop() if sampler else None
    barrier()
    elapsed_max_ms = max_over_ranks(elapsed_ms, world, "cuda")
    value = job_throughput(world * steps * B, elapsed_max_ms)

    # ---- per-kernel times with CUDA events on the launching stream ----
    _lib.trace_enable(True)
    tsteps = max(1, min(steps, 3))
    for _ in range(tsteps):
        for f in fs:
            solve(f)
    torch.cuda.synchronize()
    _lib.trace_enable(False)
    tr = _lib.trace_collect()
    pass_bytes = solve_pass_bytes(nx, ny, nz, xbc, ybc, zbc)
    line_labels = [k for k in pass_bytes if k in tr]
    lp_ms = sum(tr[k][1] for k in line_labels)
    lp_bytes = sum(pass_bytes[k] * tr[k][0] for k in line_labels)
    peak, peak_src = measured_peaks()
    achieved = (lp_bytes / (lp_ms / 1000.0)) / 1e9 if lp_ms > 0 else None
    per_pass = {k: {"launches": tr[k][0], "avg_ms": tr[k][1] / tr[k][0],
                    "gbs": (pass_bytes[k] / (tr[k][1] / tr[k][0] / 1000.0)) / 1e9,
                    "frac": (pass_bytes[k] / (tr[k][1] / tr[k][0] / 1000.0)) / 1e9 / peak}
                for k in line_labels}
    total_trace_ms = sum(v[1] for v in tr.values())
    solve_bytes = lp_bytes / (tsteps * B)
    dom_k = max(line_labels, key=lambda k: tr[k][1]) if line_labels else None
    dom_gbs = per_pass[dom_k]["gbs"] if dom_k else None
    traffic, traffic_digest, traffic_current = load_traffic()
    roofline = {"bound": "hbm", "achieved": dom_gbs, "peak": peak, "unit": "GB/s",
                "frac": (dom_gbs / peak) if dom_gbs else None,
                "traffic": traffic.get((name, dom_k)),
                "traffic_source": os.path.relpath(TRAFFIC_SUMMARY, ROOT),
                "traffic_captured_on_current_sources": traffic_current,
                "kernel": dom_k, "algorithmic_bytes_per_launch": pass_bytes.get(dom_k),
                "peak_source": peak_src, "per_pass": per_pass,
                "all_passes_gbs": achieved,
                "all_passes_frac": (achieved / peak) if achieved else None,
                "line_pass_share_of_traced_time": lp_ms / total_trace_ms if total_trace_ms else None,
                "launches_traced": sum(tr[k][0] for k in line_labels)}

    # ---- the transform alone: do_transform with the workload's forward kinds ----
    transform = None
    if args.transform_steps > 0:
        transform = time_transform(chz, name, nx, ny, nz, (xbc, ybc, zbc), args.transform_steps,
                                   args.warmup, world, peak)

    # ---- the FP64 solution of this input (error checks) ----
    a64 = f_host.to("cuda")
    solve(a64)
    torch.cuda.synchronize()
    u64 = a64.cpu().numpy().reshape(nz + 1, ny + 1, nx + 1)

    # ---- FP32 transforms + FP64 refinement on the same problems ----
    refine, u32 = None, None
    if args.refine_corrections >= 0:
        K = args.refine_corrections

        def solve_refined(f):
            chz.helmholtz_solve_refined(dom[0], dom[1], nx, xbc, faces["bcl"], faces["bcr"],
                                        dom[2], dom[3], ny, ybc, faces["bcb"], faces["bct"],
                                        dom[4], dom[5], nz, zbc, faces["bcf"], faces["bce"],
                                        lam, f, max_corrections=K)
        for _ in range(args.warmup):
            for f in fs:
                solve_refined(f)
        torch.cuda.synchronize()
        barrier()
        r0 = torch.cuda.Event(enable_timing=True)
        r1 = torch.cuda.Event(enable_timing=True)
        r0.record(stream)
        for _ in range(steps):
            for f in fs:
                solve_refined(f)
        r1.record(stream)
        torch.cuda.synchronize()
        rvalue = job_throughput(world * steps * B, max_over_ranks(r0.elapsed_time(r1), world, "cuda"))
        a32 = f_host.to("cuda")
        solve_refined(a32)
        torch.cuda.synchronize()
        u32 = a32.cpu().numpy().reshape(nz + 1, ny + 1, nx + 1)
        del a32
        _lib.trace_enable(True)
        solve_refined(fs[0])
        torch.cuda.synchronize()
        _lib.trace_enable(False)
        rtr = {k: {"launches": v[0], "avg_ms": v[1] / v[0]} for k, v in _lib.trace_collect().items()}
        rbytes = (48 + 72 * K) * nx * ny * nz
        refine = {"value": rvalue, "unit": "solves/s", "corrections": K,
                  "rel_err_vs_fp64": rel_l2(u32, u64), "speedup_vs_fp64": rvalue / value,
                  "model_bytes_per_solve": rbytes,
                  "model": f"{48 + 72 * K} B per point: FP32 solve 48 + {K} x (FP64 residual 20 + "
                           "FP32 solve 48 + FP64 accumulate 4 more); the FP64 solve moves 80",
                  "byte_bound_speedup_vs_fp64": 80.0 / (48 + 72 * K),
                  "per_kernel": rtr, "hbm_gbs_model": rbytes * rvalue / world / 1e9,
                  "frac_model": rbytes * rvalue / world / 1e9 / peak}
    del a64

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if headline:
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        esteps = max(1, min(steps, args.e2e_steps))
        face_bytes = sum(v.numel() * 8 for v in faces_h.values() if v is not None)
        e0.record(stream)
        for _ in range(esteps):
            fs[0].copy_(f_host, non_blocking=True)
            for k, v in faces_h.items():
                if v is not None:
                    faces[k].copy_(v, non_blocking=True)
            solve(fs[0])
            u_host.copy_(fs[0], non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_serial = job_throughput(world * esteps, max_over_ranks(e0.elapsed_time(e1), world, "cuda"))
        # step i's copy in, step i-1's solve and step i-2's copy out overlap
        # (three streams, two device slots); every step still copies its own f
        # (and faces) in and its own u out
        pipe = HostPipeline(nx, ny, nz, (xbc, ybc, zbc), dom, lam, faces=faces_h)
        u_hosts = [u_host, torch.empty_like(f_host).pin_memory()]
        pipe.solve([f_host] * 2, u_hosts)
        pipe.join(stream)
        torch.cuda.synchronize()
        barrier()
        psteps = max(2, esteps)
        e0.record(stream)
        pipe.wait(e0)
        pipe.solve([f_host] * psteps, [u_hosts[i % 2] for i in range(psteps)])
        pipe.join(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_value = job_throughput(world * psteps, max_over_ranks(e0.elapsed_time(e1), world, "cuda"))
        u_api = u_host.numpy().reshape(nz + 1, ny + 1, nx + 1).copy()
        del pipe, u_hosts[1]
        e2e = {"value": e2e_value, "unit": "solves/s",
               "h2d_bytes_per_step": npts * 8 + face_bytes, "d2h_bytes_per_step": npts * 8,
               "steps": psteps, "api": "cuhelmholtz_b200.pipeline.HostPipeline (pinned host f in, u out)",
               "serial_value": e2e_serial,
               "rel_err_vs_device_solve": rel_l2(u_api, u64)}
    del fs
    torch.cuda.synchronize()
    rec = {"workload": name, "description": desc, "grid": [nx, ny, nz], "bc": [xbc, ybc, zbc],
           "lambda": lam, "value": value, "unit": "solves/s", "steps": steps, "batch_per_step": B,
           "ms_per_step": elapsed_max_ms / steps, "npts": npts,
           "hbm_gbs_solve": (solve_bytes * steps * B / (elapsed_ms / 1000.0)) / 1e9,
           "algorithmic_bytes_per_solve": solve_bytes, "roofline": roofline,
           "transform": transform, "fp32_refine": refine, "e2e": e2e,
           "gpu_launches": int(launches), "clocks": clocks}
    return rec, p, u64, u32


def accuracy(rec, p, u64, u32, args, cpu_leg):
    """Errors of the benchmarked results against the reference: FISHPACK's u
    for the same input (the reference's CPU path, timed as the CPU baseline),
    the reference's own GPU solver's u, and the relative residual of the FP64
    solve in FP64 on the host.  Fills rec["accuracy"] and, when cpu_leg,
    rec["cpu_baseline"] and rec["reference_gpu"]."""
    import numpy as np
    from oracle import stencil
    acc = {"metric": "relative L2 over the (N+1)^3 grid"}
    if not args.no_check:
        nx, ny, nz = p["nx"], p["ny"], p["nz"]
        fc = {k: p.get(k) for k in stencil.FACE_KEYS}
        r = stencil.residual(u64, p["f"], nx, ny, nz, p["xbc"], p["ybc"], p["zbc"], p["dom"], p["lam"], fc)
        acc["fp64_rel_residual"] = float(np.linalg.norm(r) / np.linalg.norm(p["f"]))
        del r
    if cpu_leg:
        cpu, ufp = cpu_baseline_single(p)
        rec["cpu_baseline"] = cpu
        if ufp is not None:
            acc["fp64_vs_fishpack"] = rel_l2(u64, ufp)
            if u32 is not None:
                acc["fp32_refine_vs_fishpack"] = rel_l2(u32, ufp)
            del ufp
        rgpu, uref = (None, None) if args.ref_gpu_repeats <= 0 else reference_gpu_solve(p, args.ref_gpu_repeats)
        if rgpu is not None:
            rgpu["our_speedup"] = rec["value"] / rgpu["value"]
            rec["reference_gpu"] = rgpu
            acc["fp64_vs_reference_gpu"] = rel_l2(u64, uref)
            if u32 is not None:
                acc["fp32_refine_vs_reference_gpu"] = rel_l2(u32, uref)
            del uref
    rec["accuracy"] = acc


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        if world == 1 and args.gpus > 1:
            raise SystemExit("launch N>1 with torch.distributed.run (one process per GPU)")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline

    name = args.workload
    rec, p, u64, u32 = measure_workload(name, args, world, rank, local, headline=True)
    if rank == 0:
        accuracy(rec, p, u64, u32, args, cpu_leg)
    del p, u64, u32

    # sub-records: the other single-solve configurations at their own sizes
    subs = {}
    for sub in args.sub_workloads:
        if sub == name:
            continue
        srec, sp, su64, su32 = measure_workload(sub, args, world, rank, local, headline=False)
        if rank == 0:
            accuracy(srec, sp, su64, su32, args, cpu_leg)
        subs[sub] = srec
        del sp, su64, su32
    batch = None
    if args.sub_batch_count > 0:
        batch = measure_batch(args, args.sub_batch_count, args.sub_steps)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": rec["value"], "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": rec["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": name, "description": rec["description"], "grid": rec["grid"],
                   "bc": rec["bc"], "lambda": rec["lambda"], "batch_per_step": args.batch,
                   "parallelism": f"replicas x{world}", "kernel_family": args.kernel_family,
                   "l2": "inputs larger than L2 (each right-hand side 1 array per problem, "
                         f"{rec['npts'] * 8 / 1e9:.2f} GB each)"},
        "hbm_gbs_solve": rec["hbm_gbs_solve"],
        "algorithmic_bytes_per_solve": rec["algorithmic_bytes_per_solve"],
        "roofline": rec["roofline"],
        "cpu_baseline": rec.get("cpu_baseline"),
        "e2e": rec["e2e"],
        "gpu_launches": rec["gpu_launches"],
        "clocks": rec["clocks"],
        "accuracy": rec.get("accuracy"),
        "rel_err_vs_reference": {k: v for k, v in (rec.get("accuracy") or {}).items() if "_vs_" in k},
        "rel_residual": (rec.get("accuracy") or {}).get("fp64_rel_residual"),
        "reference_gpu": rec.get("reference_gpu"),
        "fp32_refine": rec["fp32_refine"],
        "transform": rec["transform"],
        "sub_records": {k: {kk: vv for kk, vv in v.items() if kk not in ("clocks", "e2e")}
                        for k, v in subs.items()},
        "batch": batch,
    }
    print(json.dumps(line))
    return 0


def measure_batch(args, count, steps):
    """Batching configuration: `count` problems (sizes uniform in
    {32, 48, ..., 192} per axis, codes uniform in 0..4, lambda log-uniform in
    [-100, -0.01], f ~ U[-1, 1]) solved by one graph replay per step, against a
    loop of one-at-a-time solves of the same problems."""
    import numpy as np
    import torch

    import cuhelmholtz_b200 as chz
    from cuhelmholtz_b200 import _lib
    from oracle import gen
    from oracle.stencil import FACE_KEYS

    probs = gen.config4_problems(count=count, seed=4)
    npts = sum(p["nx"] * p["ny"] * p["nz"] for p in probs)
    fs = [torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda() for p in probs]
    faces = [{k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
              for k in FACE_KEYS} for p in probs]
    plan = chz.BatchPlan(probs)
    stream = torch.cuda.current_stream()

    def loop():
        for p, f, fc in zip(probs, fs, faces):
            d = p["dom"]
            chz.cuda_helmholtz_solver(d[0], d[1], p["nx"], p["xbc"], fc["bcl"], fc["bcr"],
                                      d[2], d[3], p["ny"], p["ybc"], fc["bcb"], fc["bct"],
                                      d[4], d[5], p["nz"], p["zbc"], fc["bcf"], fc["bce"], p["lam"], f)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    l0 = _lib.launch_count()
    ms = timed(lambda: plan.solve(fs, faces))
    replays = _lib.launch_count() - l0
    assert replays == args.warmup + steps, replays
    targets, tuned_ms = plan.tiles()
    schedules = plan.radix_schedules()
    mode, mode_ms = plan.launch_mode()
    # kernels in one graph replay: the persistent kernel, or per pass the
    # register-resident group launches and the leftover launch, and the
    # periodic planes
    kernels_per_solve = plan.kernels()
    # the same batch with the untuned tile size (4096 values per tile)
    prev = chz.BatchPlan.set_autotune(False)
    try:
        plain = chz.BatchPlan(probs)
    finally:
        chz.BatchPlan.set_autotune(prev)
    ms_plain = timed(lambda: plain.solve(fs, faces))
    plain.close()
    ms_loop = timed(loop)
    # accuracy: the batch's solution of a few problems against the loop's
    errs = []
    for i in range(0, count, max(1, count // 8)):
        p = probs[i]
        a = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
        b = a.clone()
        d = p["dom"]
        fc = faces[i]
        chz.cuda_helmholtz_solver(d[0], d[1], p["nx"], p["xbc"], fc["bcl"], fc["bcr"],
                                  d[2], d[3], p["ny"], p["ybc"], fc["bcb"], fc["bct"],
                                  d[4], d[5], p["nz"], p["zbc"], fc["bcf"], fc["bce"], p["lam"], a)
        fs_i = list(fs)
        fs_i[i] = b
        plan.solve(fs_i, faces)
        torch.cuda.synchronize()
        errs.append(float((torch.linalg.vector_norm(b - a) / torch.linalg.vector_norm(a)).item()))
    plan.close()
    value = count * steps / (ms / 1000.0)
    loop_value = count * steps / (ms_loop / 1000.0)
    peak, peak_src = measured_peaks()
    gbs = 80.0 * npts * steps / (ms / 1000.0) / 1e9
    return {"workload": f"batch_{count}_mixed",
            "description": "sizes uniform in {32..192 step 16}^3, codes 0..4, lambda -10^U(-2,2)",
            "value": value, "unit": "solves/s", "steps": steps, "ms_per_step": ms / steps,
            "points_per_step": npts, "hbm_gbs_model": gbs, "frac_model": gbs / peak,
            "model": "80 B per point (five passes of 16 B)",
            "loop_of_single_solves": {"value": loop_value, "ms_per_step": ms_loop / steps},
            "launch": ("one persistent kernel over a work queue of (pass, problem, tile) items"
                       if mode == 0 else "per pass, one register-resident launch per group of problems with the "
                       "same line length and kinds and one generic launch over the rest, then the periodic planes")
                      + ", replayed from a CUDA graph",
            "kernels_per_solve": kernels_per_solve,
            "launch_form_ms": {"persistent": mode_ms[0], "per_pass": mode_ms[1],
                               "chosen": "persistent" if mode == 0 else "per_pass"},
            "autotune": {"tile_values_per_pass": targets, "tuned_ms_per_pass": tuned_ms,
                         "radix_schedule_per_pass": schedules,
                         "untuned_value": count * steps / (ms_plain / 1000.0)},
            "speedup_vs_loop": value / loop_value, "gpu_launches": int(steps * kernels_per_solve),
            "max_rel_err_vs_single_solves": max(errs) if errs else None}


def run_batch(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rec = measure_batch(args, args.batch_count, args.steps)
    line = {
        "metric": "solves/s (batched FP64 Helmholtz solves)", "value": rec["value"], "unit": "solves/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": rec["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": rec["workload"], "description": rec["description"],
                   "points_per_step": rec["points_per_step"]},
    }
    line.update({k: v for k, v in rec.items() if k not in line and k not in ("workload", "description")})
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--batch", type=int, default=8, help="solves per step (separate arrays)")
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--transform-steps", type=int, default=20,
                    help="timed do_transform calls (0 skips the transform leg)")
    ap.add_argument("--ref-procs", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the FISHPACK and reference-GPU legs (and the errors against them)")
    ap.add_argument("--no-check", action="store_true", help="skip the host residual of the FP64 solve")
    ap.add_argument("--check", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--ref-gpu-repeats", type=int, default=3,
                    help="calls of the reference's own GPU solver timed per workload (0 skips it)")
    ap.add_argument("--sub-workloads", default="helmholtz_fp64_256,helmholtz_fp64_256x192x320",
                    help="comma-separated workloads reported as sub-records ('' for none)")
    ap.add_argument("--sub-steps", type=int, default=10, help="timed steps of each sub-record")
    ap.add_argument("--sub-batch-count", type=int, default=512,
                    help="problems of the batching sub-record (0 skips it)")
    ap.add_argument("--batch-count", type=int, default=0,
                    help="run the batching configuration with this many problems instead")
    ap.add_argument("--refine-corrections", type=int, default=2,
                    help="also time the FP32 + FP64-refinement solve with this many corrections (-1: skip)")
    ap.add_argument("--kernel-family", default="default",
                    choices=["default", "generic", "no_tma"],
                    help="kernel family of the solver's passes (cuhelmholtz_b200.api.set_kernel_family)")
    args = ap.parse_args()
    args.sub_workloads = [w for w in args.sub_workloads.split(",") if w]
    for w in args.sub_workloads:
        if w not in WORKLOADS:
            ap.error(f"unknown sub-workload {w}")
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.kernel_family != "default":
        import cuhelmholtz_b200 as chz
        chz.set_kernel_family(args.kernel_family)
    if args.batch_count > 0:
        return run_batch(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
