"""Slice decomposition of one time-dependent run over ranks (one process per
GPU, ``torch.distributed`` for the plumbing).

Each rank holds a contiguous range of the run's slices: its particles and the
matching field planes.  Within a step the slices are independent; the path
has two exchanges, both the reference's:

* slippage (the multi-rank branch of ``ControlCUDA::applySlippage``,
  src/Core/ControlCUDA.cpp:148-252): at every slice shift each rank sends its
  plane ``last`` (the head of its range for a forward shift) to the next rank
  and receives the previous rank's into ``last``, which becomes its ``first``;
  the first rank (the last one for a backward shift) zeroes the plane that
  arrives from the far end unless the run is periodic.  One plane per shift
  crosses NVLink (NCCL send/recv of device buffers), no collective;
* global diagnostics (``g4_allreduce_sum_inplace``,
  src/Core/DiagnosticCUDA.cpp:81-97): seven sums all-reduced.

Fields are seen through a small plane interface (``nslice``, ``first``,
``plane_out``, ``plane_in``, ``zero_plane``): ``DevicePlanes`` wraps the
library's device field state, ``HostPlanes`` a complex array on the host.
"""
from __future__ import annotations

import ctypes as C

import numpy as np


def split_slices(nslice: int, world: int):
    """Contiguous, balanced slice ranges [(s0, s1), ...] of the ranks."""
    base, extra = divmod(nslice, world)
    out, s = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((s, s + n))
        s += n
    return out


class HostPlanes:
    """A field of complex planes [nslice, ngrid, ngrid] in host memory."""

    def __init__(self, cells: np.ndarray, first: int = 0):
        self.cells = cells
        self.nslice = cells.shape[0]
        self.first = first

    def plane_out(self, i):
        import torch
        return torch.from_numpy(self.cells[i].view(np.float64).copy())

    def plane_in(self, i, buf) -> None:
        self.cells[i] = buf.numpy().view(np.complex128).reshape(self.cells[i].shape)

    def zero_plane(self, i) -> None:
        self.cells[i] = 0


class DevicePlanes:
    """The library's device field state (``device.FieldState``); planes travel
    in device buffers of the state's precision and row pitch."""

    def __init__(self, field):
        self.f = field
        self.nslice = field.nslice
        n = C.c_size_t()
        field.lib.g4b_field_plane_bytes(field.h, C.byref(n))
        self.plane_bytes = n.value
        self.device = field.ctx.device

    @property
    def first(self) -> int:
        return self.f.first

    @first.setter
    def first(self, v: int) -> None:
        self.f.first = v

    def plane_out(self, i):
        import torch
        from ._lib import check
        buf = torch.empty(self.plane_bytes, dtype=torch.uint8, device=f"cuda:{self.device}")
        check(self.f.lib.g4b_field_plane_out(self.f.h, i, C.c_void_p(buf.data_ptr())))
        self.f.ctx.synchronize()  # the copy ran on the library's stream
        return buf

    def plane_in(self, i, buf) -> None:
        import torch
        from ._lib import check
        torch.cuda.current_stream(buf.device).synchronize()  # the receive ran on torch's
        check(self.f.lib.g4b_field_plane_in(self.f.h, i, C.c_void_p(buf.data_ptr())))
        self.f.ctx.synchronize()

    def zero_plane(self, i) -> None:
        from ._lib import check
        check(self.f.lib.g4b_field_zero_plane(self.f.h, i))


class PlaneRing:
    """The ring of ranks a decomposed run's radiation slips along."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def _peer(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def shift(self, field, direction: int, periodic: bool) -> None:
        """One slice shift (src/Core/ControlCUDA.cpp:177-249)."""
        ns = field.nslice
        last = (field.first + ns - 1) % ns
        if direction < 0:
            last = (last + 1) % ns
        nxt, prv = (self.rank + 1) % self.size, (self.rank - 1) % self.size
        if direction < 0:
            nxt, prv = prv, nxt
        if self.size > 1:
            send = field.plane_out(last)
            recv = send.new_empty(send.shape)
            d = self.dist
            ops = [d.P2POp(d.isend, send, self._peer(nxt), self.group),
                   d.P2POp(d.irecv, recv, self._peer(prv), self.group)]
            for req in d.batch_isend_irecv(ops):
                req.wait()
            field.plane_in(last, recv)
        if not periodic:
            if self.rank == 0 and direction > 0:
                field.zero_plane(last)
            if self.rank == self.size - 1 and direction < 0:
                field.zero_plane(last)
        field.first = last if direction > 0 else (last + 1) % ns

    def apply_slippage(self, field, accuslip: float, slippage: float, sample: float,
                       time_run: bool = True, periodic: bool = False):
        """ControlCUDA::applySlippage: accumulate the slippage and shift by one
        slice while it exceeds 0.8 sample; returns (accuslip, shifts)."""
        if not time_run:
            return accuslip, 0
        accuslip += slippage
        count = 0
        while abs(accuslip) > sample * 0.8:
            direction = -1 if accuslip < 0 else 1
            accuslip -= sample * direction
            self.shift(field, direction, periodic)
            count += 1
        return accuslip, count

    def allreduce_sum(self, values, device=None) -> np.ndarray:
        """Sum of per-rank global-diagnostic sums over the ranks
        (src/Core/DiagnosticCUDA.cpp:81-97)."""
        import torch
        t = torch.tensor(np.asarray(values, np.float64), device=device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy()
