"""ctypes binding of the FP64 CPU oracle (oracle/g4_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by the test suite, the smoke check and the
benchmark's CPU-baseline leg, always as the checker or the timed CPU
baseline, never as the product path.  PARITY UNPINNED against upstream
GENESIS 1.3 v4 (see g4_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBPATH = HERE / "_build" / "libg4oracle.so"

dp = C.POINTER(C.c_double)
i64p = C.POINTER(C.c_int64)
ip = C.POINTER(C.c_int)


def build() -> Path:
    """Compile the oracle with the committed Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIBPATH


def _step_type():
    from genesis4_cuda_port_b200._lib import Step
    return Step


class FieldView(C.Structure):
    _fields_ = [("first", C.c_int), ("ngrid", C.c_int), ("nslice", C.c_int),
                ("harm", C.c_int), ("gridmax", C.c_double),
                ("dgrid", C.c_double), ("xks", C.c_double), ("fc", C.c_double),
                ("cells", dp)]


class FieldState(C.Structure):
    _fields_ = [("ngrid", C.c_int), ("harm", C.c_int), ("first", C.c_int),
                ("enabled", C.c_int), ("gridmax", C.c_double),
                ("xlambda", C.c_double), ("fc", C.c_double),
                ("accuslip", C.c_double), ("cells", dp)]


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIBPATH.exists():
        build()
    lib = C.CDLL(str(LIBPATH))
    Step = _step_type()
    sp = C.POINTER(Step)
    lib.g4o_adi_coeffs.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double,
                                   dp, dp, dp, dp]
    lib.g4o_slice_scl.argtypes = [C.c_int, i64p, dp, C.c_double, C.c_double,
                                  C.c_double, C.c_double, dp]
    lib.g4o_deposit.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                C.c_double, sp, i64p, dp, dp, dp, dp, dp, dp]
    lib.g4o_adi_advance.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_int, sp, i64p, dp, dp, dp,
                                    dp, dp, dp, dp]
    lib.g4o_track.argtypes = [C.c_int64, sp, C.c_double, C.c_int, dp, dp, dp, dp, dp]
    lib.g4o_r56.argtypes = [C.c_int64, sp, C.c_double, dp, dp]
    lib.g4o_push.argtypes = [C.c_int, i64p, sp, C.POINTER(FieldView), C.c_int,
                             dp, dp, dp, dp, dp, dp, dp]
    lib.g4o_slippage.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_int, C.c_int, dp, ip, dp]
    lib.g4o_slippage.restype = C.c_int
    lib.g4o_diag_beam.argtypes = [C.c_int, i64p, C.c_int, C.c_int, dp, dp, dp,
                                  dp, dp, dp, dp, dp, dp]
    lib.g4o_diag_field.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp]
    lib.g4o_step.argtypes = [C.c_int, i64p, dp, dp, sp, C.c_double, C.c_double,
                             C.c_double, C.c_int, C.c_int,
                             C.POINTER(FieldState), C.c_int, dp, dp, dp, dp,
                             dp, dp, dp]
    lib.g4o_num_threads.restype = C.c_int
    lib.g4o_set_num_threads.argtypes = [C.c_int]
    _lib = lib
    return lib


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(dp)


def _off(off):
    off = np.ascontiguousarray(off, dtype=np.int64)
    return off, off.ctypes.data_as(i64p)


def num_threads() -> int:
    return int(load().g4o_num_threads())


def set_num_threads(n: int) -> None:
    load().g4o_set_num_threads(int(n))


def adi_coeffs(n, delz, dgrid, xks):
    c = np.empty(2 * n)
    cbet = np.empty(2 * n)
    cwet = np.empty(2 * n)
    r = C.c_double()
    load().g4o_adi_coeffs(n, delz, dgrid, xks, _d(c), _d(cbet), _d(cwet), C.byref(r))
    cv = lambda a: a.view(np.complex128)  # noqa: E731
    return cv(c), cv(cbet), cv(cwet), r.value


def adi_advance(field, *, harm, gridmax, xks, delz, fc, enabled, step, off,
                current, parts, first=0):
    """FieldSolverADICUDA::advance on a complex128 [S, n, n] array in place."""
    S, n, _ = field.shape
    flat = field.reshape(-1).view(np.float64)
    work = np.empty(4 * S * n * n)
    off, offp = _off(off)
    cur = np.ascontiguousarray(current, dtype=np.float64)
    load().g4o_adi_advance(S, n, first, harm, gridmax, xks, delz, fc, int(enabled),
                           C.byref(step), offp, _d(cur), _d(parts["x"]),
                           _d(parts["y"]), _d(parts["gamma"]), _d(parts["theta"]),
                           _d(flat), _d(work))


def deposit(*, nslice, ngrid, first, harm, gridmax, step, off, parts, scl):
    src = np.zeros((nslice, ngrid, ngrid), np.complex128)
    dgrid = 2 * gridmax / (ngrid - 1)
    off, offp = _off(off)
    load().g4o_deposit(nslice, ngrid, first, harm, gridmax, dgrid, C.byref(step),
                       offp, _d(parts["x"]), _d(parts["y"]), _d(parts["gamma"]),
                       _d(parts["theta"]), _d(np.ascontiguousarray(scl, np.float64)),
                       _d(src.reshape(-1).view(np.float64)))
    return src


def slice_scl(off, current, fc, xks, dgrid, delz):
    off, offp = _off(off)
    out = np.empty(len(off) - 1)
    load().g4o_slice_scl(len(off) - 1, offp, _d(np.ascontiguousarray(current, np.float64)),
                         fc, xks, dgrid, delz, _d(out))
    return out


def track(parts, step, delz, last):
    n = parts["x"].size
    load().g4o_track(n, C.byref(step), delz, int(last), _d(parts["x"]), _d(parts["y"]),
                     _d(parts["px"]), _d(parts["py"]), _d(parts["gamma"]))


def r56(parts, step, lambda0):
    load().g4o_r56(parts["x"].size, C.byref(step), lambda0, _d(parts["gamma"]),
                   _d(parts["theta"]))


def push(off, step, fields, parts, slice_eloss=None):
    """fields: list of dicts(cells complex128 [S,n,n], first, harm, gridmax, xlambda, fc)."""
    off, offp = _off(off)
    nf = len(fields)
    views = (FieldView * nf)()
    keep = []
    for i, f in enumerate(fields):
        cells = np.ascontiguousarray(f["cells"], dtype=np.complex128)
        keep.append(cells)
        S, n, _ = cells.shape
        views[i].first = f.get("first", 0)
        views[i].ngrid = n
        views[i].nslice = S
        views[i].harm = f.get("harm", 1)
        views[i].gridmax = f["gridmax"]
        views[i].dgrid = 2 * f["gridmax"] / (n - 1)
        views[i].xks = 2 * np.pi / f["xlambda"]
        views[i].fc = f["fc"]
        views[i].cells = cells.reshape(-1).view(np.float64).ctypes.data_as(dp)
    el = None if slice_eloss is None else np.ascontiguousarray(slice_eloss, np.float64)
    load().g4o_push(len(off) - 1, offp, C.byref(step), views, nf, _d(el),
                    _d(parts["x"]), _d(parts["y"]), _d(parts["px"]), _d(parts["py"]),
                    _d(parts["gamma"]), _d(parts["theta"]))


def slippage(field, shift, sample, time_run, periodic, accuslip, first):
    S, n, _ = field.shape
    acc = C.c_double(accuslip)
    fst = C.c_int(first)
    ns = load().g4o_slippage(S, n, shift, sample, int(time_run), int(periodic),
                             C.byref(acc), C.byref(fst), _d(field.reshape(-1).view(np.float64)))
    return acc.value, fst.value, ns


def diag_beam(off, parts, nharm=1, need_aux=True):
    off, offp = _off(off)
    S = len(off) - 1
    stats = np.empty((S, 23))
    bre = np.empty((S, nharm))
    bim = np.empty((S, nharm))
    load().g4o_diag_beam(S, offp, nharm, int(need_aux), _d(parts["x"]), _d(parts["y"]),
                         _d(parts["px"]), _d(parts["py"]), _d(parts["gamma"]),
                         _d(parts["theta"]), _d(stats.reshape(-1)), _d(bre.reshape(-1)),
                         _d(bim.reshape(-1)))
    return stats, bre, bim


def diag_field(field, first):
    S, n, _ = field.shape
    stats = np.empty((S, 7))
    center = np.empty((S, 2))
    load().g4o_diag_field(S, n, first, _d(field.reshape(-1).view(np.float64)),
                          _d(stats.reshape(-1)), _d(center.reshape(-1)))
    return stats, center


def step(off, current, step_params, lambda0, slippage_shift, sample, time_run,
         periodic, fields, parts, slice_eloss=None):
    """One Gencore main-loop step; fields: list of dicts updated in place
    (cells complex128 [S,n,n], harm, gridmax, xlambda, fc, first, accuslip,
    enabled)."""
    off, offp = _off(off)
    S = len(off) - 1
    nf = len(fields)
    fs = (FieldState * nf)()
    nmax = 0
    for i, f in enumerate(fields):
        cells = f["cells"]
        assert cells.dtype == np.complex128 and cells.flags["C_CONTIGUOUS"]
        n = cells.shape[1]
        nmax = max(nmax, n)
        fs[i].ngrid = n
        fs[i].harm = f.get("harm", 1)
        fs[i].first = f.get("first", 0)
        fs[i].enabled = int(f.get("enabled", True))
        fs[i].gridmax = f["gridmax"]
        fs[i].xlambda = f["xlambda"]
        fs[i].fc = f["fc"]
        fs[i].accuslip = f.get("accuslip", 0.0)
        fs[i].cells = cells.reshape(-1).view(np.float64).ctypes.data_as(dp)
    work = np.empty(4 * S * nmax * nmax)
    el = None if slice_eloss is None else np.ascontiguousarray(slice_eloss, np.float64)
    load().g4o_step(S, offp, _d(np.ascontiguousarray(current, np.float64)), _d(el),
                    C.byref(step_params), lambda0, slippage_shift, sample, int(time_run),
                    int(periodic), fs, nf, _d(parts["x"]), _d(parts["y"]), _d(parts["px"]),
                    _d(parts["py"]), _d(parts["gamma"]), _d(parts["theta"]), _d(work))
    for i, f in enumerate(fields):
        f["first"] = fs[i].first
        f["accuslip"] = fs[i].accuslip
