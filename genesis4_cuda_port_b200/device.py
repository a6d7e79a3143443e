"""Python handles over the C ABI (include/g4b.h).

These mirror the reference's device-state objects and solver classes:
``Context`` (genesis4_cuda runtime helpers), ``FieldState``
(Genesis4FieldSoA), ``BeamState`` (Genesis4BeamSoA), ``FieldSolverADICUDA``,
``BeamSolverCUDA``/``TrackBeamCUDA`` entry points, ``ControlCUDA.applySlippage``
and the device part of ``DiagnosticCUDA``.  Every call goes through
libg4b200.so; errors raise ``G4BError``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import G4B_FP64, G4B_MIXED, RunDesc, Step, check, dptr  # noqa: F401


class Context:
    """A device and the CUDA stream all work of this context is issued on."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.g4b_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    @property
    def stream(self) -> int:
        return self.lib.g4b_ctx_get_stream(self.h) or 0

    def set_stream(self, stream_ptr: int | None) -> None:
        check(self.lib.g4b_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def synchronize(self) -> None:
        check(self.lib.g4b_ctx_synchronize(self.h))

    def launch_count(self) -> int:
        v = C.c_uint64()
        check(self.lib.g4b_ctx_launch_count(self.h, C.byref(v)))
        return int(v.value)

    def profile(self, enable: bool) -> None:
        """Per-kernel CUDA-event timing on this context's stream."""
        check(self.lib.g4b_ctx_profile(self.h, int(enable)))

    def profile_read(self) -> dict:
        """{kernel name: (launches, total ms)} since profiling was enabled."""
        n = C.c_int()
        check(self.lib.g4b_ctx_profile_read(self.h, 0, None, None, None, C.byref(n)))
        k = n.value
        names = C.create_string_buffer(64 * max(k, 1))
        counts = (C.c_uint64 * max(k, 1))()
        ms = (C.c_double * max(k, 1))()
        check(self.lib.g4b_ctx_profile_read(self.h, k, names, counts, ms, C.byref(n)))
        out = {}
        for i in range(k):
            nm = names.raw[64 * i:64 * (i + 1)].split(b"\0")[0].decode()
            out[nm] = (int(counts[i]), float(ms[i]))
        return out

    def sm_count(self) -> int:
        v = C.c_int()
        check(self.lib.g4b_ctx_sm_count(self.h, C.byref(v)))
        return int(v.value)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.g4b_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FieldState:
    """Radiation field of ``nslice`` planes, ngrid x ngrid complex cells."""

    def __init__(self, ctx: Context, nslice: int, ngrid: int, gridmax: float,
                 xlambda: float, harm: int = 1, precision: int = G4B_FP64,
                 low_memory: bool = False):
        self.ctx, self.lib = ctx, ctx.lib
        self.nslice, self.ngrid, self.gridmax = nslice, ngrid, gridmax
        self.xlambda, self.harm, self.precision = xlambda, harm, precision
        self.dgrid = 2.0 * gridmax / (ngrid - 1)
        self.xks = 2.0 * np.pi / xlambda
        self.accuslip = 0.0
        h = C.c_void_p()
        check(self.lib.g4b_field_create(ctx.h, nslice, ngrid, gridmax, xlambda,
                                        harm, precision, int(low_memory),
                                        C.byref(h)))
        self.h = h

    def upload(self, cells: np.ndarray) -> None:
        a = np.ascontiguousarray(cells, dtype=np.complex128).reshape(-1)
        assert a.size == self.nslice * self.ngrid ** 2
        check(self.lib.g4b_field_upload(self.h, dptr(a.view(np.float64))))

    def download(self) -> np.ndarray:
        out = np.empty((self.nslice, self.ngrid, self.ngrid), np.complex128)
        check(self.lib.g4b_field_download(self.h, dptr(out.reshape(-1).view(np.float64))))
        return out

    @property
    def first(self) -> int:
        v = C.c_int()
        check(self.lib.g4b_field_get_first(self.h, C.byref(v)))
        return int(v.value)

    @first.setter
    def first(self, value: int) -> None:
        check(self.lib.g4b_field_set_first(self.h, int(value)))

    def device_bytes(self) -> int:
        v = C.c_uint64()
        check(self.lib.g4b_field_device_bytes(self.h, C.byref(v)))
        return int(v.value)

    def apply_slippage(self, shift: float, sample: float, time_run: bool = True,
                       periodic: bool = False) -> int:
        """ControlCUDA::applySlippage; returns the number of slice shifts."""
        acc = C.c_double(self.accuslip)
        ns = C.c_int()
        check(self.lib.g4b_slippage(self.h, shift, sample, int(time_run),
                                    int(periodic), C.byref(acc), C.byref(ns)))
        self.accuslip = acc.value
        return int(ns.value)

    def diagnostics(self):
        """Raw per-slice sums (7) and centre cell, indexed by beam slice."""
        stats = np.empty((self.nslice, 7))
        center = np.empty((self.nslice, 2))
        check(self.lib.g4b_diag_field(self.h, dptr(stats.reshape(-1)),
                                      dptr(center.reshape(-1))))
        return stats, center

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.g4b_field_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BeamState:
    """Slice-contiguous FP64 particles x, y, px, py, gamma, theta."""

    NAMES = ("x", "y", "px", "py", "gamma", "theta")

    def __init__(self, ctx: Context, slice_offsets, gamma_ref: float,
                 precision: int = G4B_FP64):
        self.ctx, self.lib = ctx, ctx.lib
        off = np.ascontiguousarray(slice_offsets, dtype=np.int64)
        self.offsets = off
        self.nslice = len(off) - 1
        self.npart = int(off[-1])
        self.gamma_ref = gamma_ref
        h = C.c_void_p()
        check(self.lib.g4b_beam_create(ctx.h, self.nslice,
                                       off.ctypes.data_as(_lib.c_int64_p),
                                       precision, gamma_ref, C.byref(h)))
        self.h = h

    def upload(self, parts: dict) -> None:
        arrs = [np.ascontiguousarray(parts[k], dtype=np.float64) for k in self.NAMES]
        for a in arrs:
            assert a.size == self.npart
        check(self.lib.g4b_beam_upload(self.h, *[dptr(a) for a in arrs]))

    def download(self) -> dict:
        out = {k: np.empty(self.npart) for k in self.NAMES}
        check(self.lib.g4b_beam_download(self.h, *[dptr(out[k]) for k in self.NAMES]))
        return out

    def set_current(self, current) -> None:
        a = np.ascontiguousarray(current, dtype=np.float64)
        assert a.size == self.nslice
        check(self.lib.g4b_beam_set_current(self.h, dptr(a)))

    def set_eloss(self, eloss=None) -> None:
        a = None if eloss is None else np.ascontiguousarray(eloss, dtype=np.float64)
        check(self.lib.g4b_beam_set_eloss(self.h, dptr(a)))

    def set_particle_ez(self, ez=None) -> None:
        """Per-particle loss the push reads in place of the slice loss (None:
        back to the slice loss)."""
        a = None if ez is None else np.ascontiguousarray(ez, dtype=np.float64)
        if a is not None:
            assert a.size == self.npart
        check(self.lib.g4b_beam_set_particle_ez(self.h, dptr(a)))

    def incoherent(self, step: Step, delz: float, *, helical: bool = False, loss: bool = True,
                   spread: bool = True, seed: int = 0, counter: int = 0) -> None:
        """Incoherent synchrotron radiation of one undulator step (Incoherent::apply)."""
        check(self.lib.g4b_beam_incoherent(self.h, C.byref(step), delz, int(helical),
                                           int(loss), int(spread), seed, counter))

    def particle_ez(self) -> np.ndarray:
        out = np.empty(self.npart)
        check(self.lib.g4b_beam_get_particle_ez(self.h, dptr(out)))
        return out

    # TrackBeamCUDA::track / applyR56 and BeamSolverCUDA::advance
    def track(self, step: Step, delz: float, last: bool) -> None:
        check(self.lib.g4b_beam_track(self.h, C.byref(step), delz, int(last)))

    def apply_r56(self, step: Step, lambda0: float) -> None:
        check(self.lib.g4b_beam_r56(self.h, C.byref(step), lambda0))

    def advance(self, fields, fc, step: Step) -> None:
        n = len(fields)
        hs = (C.c_void_p * n)(*[f.h.value for f in fields])
        fcs = np.ascontiguousarray(fc, dtype=np.float64)
        check(self.lib.g4b_beam_advance(self.h, C.cast(hs, _lib.c_void_pp),
                                        dptr(fcs), n, C.byref(step)))

    def diagnostics(self, nharm: int = 1, need_aux: bool = True):
        stats = np.empty((self.nslice, 23))
        bre = np.empty((self.nslice, nharm))
        bim = np.empty((self.nslice, nharm))
        check(self.lib.g4b_diag_beam(self.h, nharm, int(need_aux),
                                     dptr(stats.reshape(-1)), dptr(bre.reshape(-1)),
                                     dptr(bim.reshape(-1))))
        return stats, bre, bim

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.g4b_beam_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FieldSolverADICUDA:
    """The reference's FieldSolverADICUDA: init (factorise) and advance."""

    def __init__(self, ctx: Context):
        self.ctx, self.lib = ctx, ctx.lib
        h = C.c_void_p()
        check(self.lib.g4b_adi_create(ctx.h, C.byref(h)))
        self.h = h

    def init(self, delz: float, dgrid: float, xks: float, ngrid: int) -> None:
        check(self.lib.g4b_adi_init(self.h, delz, dgrid, xks, ngrid))

    def advance(self, field: FieldState, beam: BeamState, step: Step, fc: float,
                enabled: bool = True) -> None:
        check(self.lib.g4b_adi_advance(self.h, field.h, beam.h, C.byref(step), fc,
                                       int(enabled)))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.g4b_adi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FieldSolverFFTCUDA:
    """The reference's FieldSolverFFTCUDA: spectral propagator with the
    optional sigmoid source filter (initSourceFilter), init, advance."""

    def __init__(self, ctx: Context):
        self.ctx, self.lib = ctx, ctx.lib
        h = C.c_void_p()
        check(self.lib.g4b_fft_create(ctx.h, C.byref(h)))
        self.h = h

    def init_source_filter(self, xc: float, yc: float, sig: float, filt: bool) -> None:
        check(self.lib.g4b_fft_init_filter(self.h, xc, yc, sig, int(filt)))

    def init(self, delz: float, dgrid: float, xks: float, ngrid: int) -> None:
        check(self.lib.g4b_fft_init(self.h, delz, dgrid, xks, ngrid))

    def advance(self, field: FieldState, beam: BeamState, step: Step, fc: float,
                enabled: bool = True) -> None:
        check(self.lib.g4b_fft_advance(self.h, field.h, beam.h, C.byref(step), fc,
                                       int(enabled)))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.g4b_fft_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EFieldSolver:
    """Short-range space charge on the device: BeamSolverCUDA::initEField
    (rmax, ngrid, nz, nphi, lambda) and EFieldSolver::shortRange over every
    slice, writing the beam's per-particle loss."""

    def __init__(self, ctx: Context, rmax: float, ngrid: int, nz: int, nphi: int,
                 lambda0: float):
        self.ctx, self.lib = ctx, ctx.lib
        h = C.c_void_p()
        check(self.lib.g4b_efield_create(ctx.h, rmax, ngrid, nz, nphi, lambda0, C.byref(h)))
        self.h = h

    def has_short_range(self) -> bool:
        return bool(self.lib.g4b_efield_has_short_range(self.h))

    def short_range(self, beam: BeamState, gammaz2: float) -> None:
        check(self.lib.g4b_efield_short_range(self.h, beam.h, gammaz2))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.g4b_efield_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Run:
    """The fused mixed-precision form: a whole FEL run resident on the device
    (beam + up to 8 fields sharing the slicing), advanced per lattice step by
    fused kernels replayed as a CUDA graph (g4b_run_* in include/g4b.h)."""

    def __init__(self, ctx: Context, slice_offsets, *, fields, lambda0: float,
                 gamma_ref: float, sample: float = 1.0, time_run: bool = True,
                 periodic: bool = False, nbunch: int = 1):
        """fields: list of (harm, ngrid, gridmax)."""
        self.ctx, self.lib = ctx, ctx.lib
        off = np.ascontiguousarray(slice_offsets, dtype=np.int64)
        self.offsets = off
        self.nslice = len(off) - 1
        self.npart = int(off[-1])
        self.fields = list(fields)
        self.nbunch = nbunch
        d = RunDesc()
        d.nslice = self.nslice
        d.nfield = len(self.fields)
        for i, (h, n, gm) in enumerate(self.fields):
            d.harm[i], d.ngrid[i], d.gridmax[i] = h, n, gm
        d.lambda0, d.gamma_ref, d.sample = lambda0, gamma_ref, sample
        d.time_run, d.periodic, d.nbunch, d.precision = int(time_run), int(periodic), nbunch, G4B_MIXED
        h = C.c_void_p()
        check(self.lib.g4b_run_create(ctx.h, C.byref(d), off.ctypes.data_as(_lib.c_int64_p),
                                      C.byref(h)))
        self.h = h

    def upload_beam(self, parts: dict) -> None:
        arrs = [np.ascontiguousarray(parts[k], dtype=np.float64) for k in BeamState.NAMES]
        check(self.lib.g4b_run_upload_beam(self.h, *[dptr(a) for a in arrs]))

    def download_beam(self, out: dict | None = None) -> dict:
        """out: optional preallocated (e.g. pinned) float64 arrays by name."""
        if out is None:
            out = {k: np.empty(self.npart) for k in BeamState.NAMES}
        check(self.lib.g4b_run_download_beam(self.h, *[dptr(out[k]) for k in BeamState.NAMES]))
        return out

    def upload_field(self, i: int, cells, first: int = 0) -> None:
        """cells None: a zero field."""
        if cells is None:
            check(self.lib.g4b_run_upload_field(self.h, i, None, first))
            return
        a = np.ascontiguousarray(cells, dtype=np.complex128).reshape(-1)
        check(self.lib.g4b_run_upload_field(self.h, i, dptr(a.view(np.float64)), first))

    def download_field(self, i: int, out=None):
        """out: optional preallocated (e.g. pinned) complex128 [nslice, n, n]."""
        n = self.fields[i][1]
        if out is None:
            out = np.empty((self.nslice, n, n), np.complex128)
        first = C.c_int()
        check(self.lib.g4b_run_download_field(self.h, i, dptr(out.reshape(-1).view(np.float64)),
                                              C.byref(first)))
        return out, int(first.value)

    def set_current(self, current) -> None:
        a = np.ascontiguousarray(np.broadcast_to(current, (self.nslice,)), dtype=np.float64)
        check(self.lib.g4b_run_set_current(self.h, dptr(a)))

    def layouts(self) -> list:
        out = (C.c_int * 8)()
        check(self.lib.g4b_run_get_layouts(self.h, out))
        return list(out[: len(self.fields)])

    def set_layouts(self, layouts) -> None:
        arr = (C.c_int * 8)(*layouts)
        check(self.lib.g4b_run_set_layouts(self.h, arr))

    def set_eloss(self, eloss=None) -> None:
        a = None if eloss is None else np.ascontiguousarray(eloss, dtype=np.float64)
        check(self.lib.g4b_run_set_eloss(self.h, dptr(a)))

    def set_lattice(self, steps, fc, slip, hist_steps: int = 0) -> None:
        n = len(steps)
        arr = (Step * n)(*steps)
        fcs = np.ascontiguousarray(fc, dtype=np.float64).reshape(n, len(self.fields))
        sl = np.ascontiguousarray(slip, dtype=np.float64)
        check(self.lib.g4b_run_set_lattice(self.h, n, arr, dptr(fcs.reshape(-1)), dptr(sl),
                                           hist_steps))

    def advance(self, first_step: int, nsteps: int, graph: bool = True) -> None:
        check(self.lib.g4b_run_advance(self.h, first_step, nsteps, int(graph)))

    def prepare(self, first_step: int, nsteps: int) -> None:
        """Capture the CUDA graph of a step range without launching it."""
        check(self.lib.g4b_run_prepare(self.h, first_step, nsteps))

    def history(self, step: int):
        """(beam stats [nslice, 23+2*nbunch], field stats [nfield, nslice, 9])."""
        beam = np.empty((self.nslice, 23 + 2 * self.nbunch))
        field = np.empty((len(self.fields), self.nslice, 9))
        check(self.lib.g4b_run_history(self.h, step, dptr(beam.reshape(-1)),
                                       dptr(field.reshape(-1))))
        return beam, field

    def history_range(self, first: int, n: int):
        """Diagnostics of steps [first, first+n) in one read: (beam [n, nslice,
        23+2*nbunch], field [n, nfield, nslice, 9])."""
        rb = self.nslice * (23 + 2 * self.nbunch)
        rf = len(self.fields) * self.nslice * 9
        out = np.empty((n, rb + rf))
        check(self.lib.g4b_run_history_range(self.h, first, n, dptr(out.reshape(-1))))
        beam = out[:, :rb].reshape(n, self.nslice, 23 + 2 * self.nbunch)
        field = out[:, rb:].reshape(n, len(self.fields), self.nslice, 9)
        return beam, field

    def device_bytes(self) -> int:
        v = C.c_uint64()
        check(self.lib.g4b_run_device_bytes(self.h, C.byref(v)))
        return int(v.value)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.g4b_run_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent mixed-precision runs advanced together by one
    persistent launch per kernel phase (g4b_batch_* in include/g4b.h).  Runs
    are attached as prepared `Run` objects and leave on reaching their last
    step; their state and diagnostics stay readable through the `Run`."""

    def __init__(self, ctx: Context, max_runs: int):
        self.ctx, self.lib = ctx, ctx.lib
        h = C.c_void_p()
        check(self.lib.g4b_batch_create(ctx.h, max_runs, C.byref(h)))
        self.h = h
        self.runs = {}

    def attach(self, run: Run, first_step: int, nsteps: int) -> int:
        slot = C.c_int()
        check(self.lib.g4b_batch_attach(self.h, run.h, first_step, nsteps, C.byref(slot)))
        self.runs[slot.value] = run
        return slot.value

    def detach(self, slot: int) -> None:
        check(self.lib.g4b_batch_detach(self.h, slot))
        self.runs.pop(slot, None)

    def status(self, slot: int):
        """(next lattice step, steps remaining)."""
        nxt, rem = C.c_int(), C.c_int()
        check(self.lib.g4b_batch_status(self.h, slot, C.byref(nxt), C.byref(rem)))
        return nxt.value, rem.value

    def step(self, nsteps: int = 1, graph: bool = True) -> None:
        check(self.lib.g4b_batch_step(self.h, nsteps, int(graph)))

    def tune(self) -> None:
        check(self.lib.g4b_batch_tune(self.h))

    def tune_layouts(self) -> None:
        """Launch shapes, then the ADI row layouts (g4b_batch_tune_layouts)."""
        check(self.lib.g4b_batch_tune_layouts(self.h))

    def shapes(self):
        g = (C.c_int * 4)()
        check(self.lib.g4b_batch_shapes(self.h, g))
        return dict(zip(("beam", "deposit", "adi", "finalize"), list(g)))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.g4b_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mem_info(ctx: Context):
    """(free, total) device bytes."""
    f, t = C.c_uint64(), C.c_uint64()
    check(ctx.lib.g4b_ctx_mem_info(ctx.h, C.byref(f), C.byref(t)))
    return int(f.value), int(t.value)
