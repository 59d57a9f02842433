"""Ragged batches: thousands of Burgers rows with different n, nu, dt, dx.

Rows are packed back to back in one FP32 buffer.  One persistent launch
advances all of them: each warp takes the next row from a device-side counter
in longest-first order (work ~ n), so large rows start early and small ones
fill the tail."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as nat
from .solvers import _SCHEMES

_VALID_N = (8, 16, 32, 64, 128, 256, 512)


class RaggedBurgers:
    def __init__(self, rows_u0, nu, dt, dx, scheme="ssprk3", convection="WENO", device="cuda",
                 warps_per_block=0, grid_blocks=0):
        ns = [int(np.asarray(r).shape[-1]) for r in rows_u0]
        for n in ns:
            if n not in _VALID_N:
                raise ValueError(f"row length {n} not supported (powers of two in [8, 512])")
        if not (len(nu) == len(dt) == len(dx) == len(ns)):
            raise ValueError("nu, dt, dx need one entry per row")
        self.device = torch.device(device)
        self.rows = len(ns)
        self.ns = ns
        off = np.zeros(self.rows, dtype=np.int64)
        off[1:] = np.cumsum(ns)[:-1]
        self.offsets_host = off
        self.total = int(sum(ns))
        dev = self.device
        self.offsets = torch.tensor(off, dtype=torch.int64, device=dev)
        self.n_rows = torch.tensor(ns, dtype=torch.int32, device=dev)
        self.nu = torch.tensor(np.asarray(nu, dtype=np.float32), device=dev)
        self.dt = torch.tensor(np.asarray(dt, dtype=np.float32), device=dev)
        self.dx = torch.tensor(np.asarray(dx, dtype=np.float32), device=dev)
        order = np.argsort(-np.asarray(ns), kind="stable").astype(np.int32)  # longest first
        self.order = torch.tensor(order, device=dev)
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        self.u0 = torch.tensor(np.concatenate([np.asarray(r, dtype=np.float32).reshape(-1) for r in rows_u0]),
                               device=dev)
        d = nat.BurgersRaggedDesc()
        d.rows, d.scheme = self.rows, _SCHEMES[scheme]
        d.convection = nat.INC_CONV_WENO if convection == "WENO" else nat.INC_CONV_FDM
        d.warps_per_block = int(warps_per_block)
        d.offsets, d.n_rows = self.offsets.data_ptr(), self.n_rows.data_ptr()
        d.nu_rows, d.dt_rows, d.dx_rows = self.nu.data_ptr(), self.dt.data_ptr(), self.dx.data_ptr()
        d.order = self.order.data_ptr()
        self.desc = d
        self.grid_blocks = int(grid_blocks) or self.default_grid()

    def default_grid(self) -> int:
        """Blocks of the persistent launch: as many as are resident at once.  The kernel
        keeps up to 255 registers a thread (a row of 512 cells holds 16 cells, their
        increments, compensation and fluxes per lane), so an SM holds eight of its warps;
        a larger grid only adds blocks that start once the queue is empty."""
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        wpb = self.desc.warps_per_block or 4
        return sms * max(1, 8 // wpb)

    def rollout(self, steps, u0=None, out=None):
        """All rows advanced `steps` steps; returns the packed final state."""
        u0 = self.u0 if u0 is None else u0
        out = torch.empty_like(u0) if out is None else out
        with torch.cuda.device(self.device):
            rc = nat.lib().inc_burgers_ragged_rollout(C.byref(self.desc), u0.data_ptr(), int(steps), out.data_ptr(),
                                                      self.queue.data_ptr(), self.grid_blocks,
                                                      nat.stream_of(self.device))
        nat.check(rc, "inc_burgers_ragged_rollout")
        return out

    def unpack(self, packed):
        return [packed[o:o + n] for o, n in zip(self.offsets_host.tolist(), self.ns)]

    @property
    def cells(self):
        return self.total
