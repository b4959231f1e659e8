"""Solves of right-hand sides held in host memory, overlapped.

A caller whose data lives on the host pays two PCIe copies per solve (f in,
u out), each as long as the solve itself or longer.  ``HostPipeline`` runs
step i's host-to-device copy, step i-1's solve and step i-2's device-to-host
copy at once on three streams (the B200's copy engines move both directions
concurrently), with two device slots ordered by CUDA events; every step still
copies its own input in and its own result out.
"""
from __future__ import annotations

from typing import Optional, Sequence

import torch

from . import api

FACE_KEYS = ("bcl", "bcr", "bcb", "bct", "bcf", "bce")


class HostPipeline:
    """Pipelined solves of one problem geometry (sizes, codes, domain,
    lambda) on host right-hand sides.

    faces: dict of Neumann arrays (host tensors, or None) copied with every
    step (they are inputs of the solve too)."""

    def __init__(self, nx: int, ny: int, nz: int, bcs: Sequence[int], dom, lam: float,
                 faces: Optional[dict] = None, slots: int = 2, device=None):
        self.dims = (int(nx), int(ny), int(nz))
        self.bcs = tuple(int(b) for b in bcs)
        self.dom = tuple(float(v) for v in dom)
        self.lam = float(lam)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        n = (nx + 1) * (ny + 1) * (nz + 1)
        self.slots = [torch.empty(n, dtype=torch.float64, device=self.device) for _ in range(slots)]
        faces = faces or {}
        self.faces_h = {k: faces.get(k) for k in FACE_KEYS}
        self.faces_d = [{k: (None if v is None else torch.empty(v.numel(), dtype=torch.float64, device=self.device))
                         for k, v in self.faces_h.items()} for _ in range(slots)]
        self.s_in = torch.cuda.Stream(device=self.device)
        self.s_run = torch.cuda.Stream(device=self.device)
        self.s_out = torch.cuda.Stream(device=self.device)
        self.ev_in = [torch.cuda.Event() for _ in range(slots)]
        self.ev_run = [torch.cuda.Event() for _ in range(slots)]
        self.ev_out = [torch.cuda.Event() for _ in range(slots)]
        self.used = [False] * slots

    def bytes_per_step(self):
        """(host-to-device, device-to-host) bytes of one step."""
        n = self.slots[0].numel() * 8
        faces = sum(v.numel() * 8 for v in self.faces_h.values() if v is not None)
        return n + faces, n

    def solve(self, f_hosts: Sequence[torch.Tensor], u_hosts: Sequence[torch.Tensor]) -> None:
        """u_hosts[i] <- solution for f_hosts[i] (contiguous host tensors; pinned
        for the copies to overlap, otherwise each copy blocks the host).
        Returns once every copy is queued; call ``join()`` and synchronise that
        stream before reading u_hosts.  Raises ValueError for a non-contiguous
        tensor (a reshaped copy would silently drop the result)."""
        nx, ny, nz = self.dims
        xbc, ybc, zbc = self.bcs
        d = self.dom
        k = len(self.slots)
        for t in list(f_hosts) + list(u_hosts):
            if not t.is_contiguous():
                raise ValueError("HostPipeline.solve needs contiguous host tensors")
        for i, (fh, uh) in enumerate(zip(f_hosts, u_hosts)):
            s = i % k
            f = self.slots[s]
            fc = self.faces_d[s]
            with torch.cuda.stream(self.s_in):
                if self.used[s]:
                    self.s_in.wait_event(self.ev_out[s])   # the slot's previous result is out
                f.copy_(fh.view(-1), non_blocking=True)
                for key, v in self.faces_h.items():
                    if v is not None:
                        fc[key].copy_(v.contiguous().view(-1), non_blocking=True)
                self.ev_in[s].record(self.s_in)
            with torch.cuda.stream(self.s_run):
                self.s_run.wait_event(self.ev_in[s])
                api.cuda_helmholtz_solver(d[0], d[1], nx, xbc, fc["bcl"], fc["bcr"],
                                          d[2], d[3], ny, ybc, fc["bcb"], fc["bct"],
                                          d[4], d[5], nz, zbc, fc["bcf"], fc["bce"],
                                          self.lam, f, stream=self.s_run)
                self.ev_run[s].record(self.s_run)
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(self.ev_run[s])
                uh.view(-1).copy_(f, non_blocking=True)
                self.ev_out[s].record(self.s_out)
            self.used[s] = True

    def wait(self, event: torch.cuda.Event) -> None:
        """Work queued after this call starts after ``event``."""
        for s in (self.s_in, self.s_run, self.s_out):
            s.wait_event(event)

    def join(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        """``stream`` (default: the current one) waits for every queued copy
        back to the host."""
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        for used, ev in zip(self.used, self.ev_out):
            if used:
                stream.wait_event(ev)
