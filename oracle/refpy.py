"""ctypes binding of oracle/_ref/libg4ref.so: the reference's own CUDA classes
(src/Core/*.cpp of mulingLHY/Genesis4_CUDA_port, compiled unmodified by
oracle/ref/Makefile) driven on host arrays.

TEST INFRASTRUCTURE ONLY.  Used by tests/golden/make_golden.py to record the
reference's outputs as fixtures and by the GPU tests to compare the oracle
and the CUDA path with the reference live.  It needs a GPU to run (the
reference's kernels are CUDA) and the reference tree to build.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBPATH = HERE / "_ref" / "libg4ref.so"
REF_TREE = Path(os.environ.get("G4_REFERENCE_TREE", "/root/reference"))

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)

STEP_FIELDS = ["delz", "aw", "ax", "ay", "kx", "ky", "gradx", "grady", "ku", "gamma_ref",
               "autophase", "qf", "dqx", "dqy", "cx", "cy", "chic_angle", "chic_lb",
               "chic_ld", "chic_lt", "in_undulator"]


def build() -> Path | None:
    """Build libg4ref.so from the reference tree when it is present."""
    if not (REF_TREE / "src" / "Core" / "FieldSolverADICUDA.cpp").exists():
        return None
    subprocess.run(["make", "-s", "-C", str(HERE / "ref"), f"REF={REF_TREE}"], check=True)
    return LIBPATH


def available() -> bool:
    return LIBPATH.exists()


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    from genesis4_cuda_port_b200._lib import Step
    lib = C.CDLL(str(LIBPATH))
    sp = C.POINTER(Step)
    dpp = C.POINTER(dp)
    lib.g4ref_last_error.restype = C.c_char_p
    lib.g4ref_device_count.restype = C.c_int
    lib.g4ref_field_advance.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                        C.c_double, sp, ip, dp, dp, dp, dp, dp, dp, C.c_int,
                                        C.c_double, C.c_double, C.c_double]
    lib.g4ref_beam_advance.argtypes = [C.c_int, ip, sp, C.c_int, ip, ip, ip, dp, dp, dp, dpp,
                                       dp, dp, dp, dp, dp, dp, dp]
    lib.g4ref_time_steps.argtypes = [C.c_int, ip, dp, dp, dp, dp, dp, dp, dp, C.c_int,
                                     C.c_double, C.c_double, dp, C.c_int, sp, dp, dp,
                                     C.c_double, C.c_int, C.c_int, C.c_int, dp]
    lib.g4ref_set_particle_ez.argtypes = [dp]
    lib.g4ref_set_particle_ez.restype = None
    lib.g4ref_track.argtypes = [C.c_int, sp, C.c_double, C.c_int, dp, dp, dp, dp, dp]
    lib.g4ref_r56.argtypes = [C.c_int, sp, C.c_double, dp, dp]
    lib.g4ref_slippage.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                   C.c_int, dp, ip, dp]
    lib.g4ref_diag.argtypes = [C.c_int, ip, dp, dp, dp, dp, dp, dp, C.c_int, dp, dp, dp,
                               C.c_int, ip, ip, dp, dp, C.c_double, dpp]
    lib.g4ref_diag_record.argtypes = [C.c_int, C.c_char_p, dp, C.c_int]
    lib.g4ref_diag_record.restype = C.c_int
    _lib = lib
    return lib


def _chk(rc):
    if rc != 0:
        raise RuntimeError("reference: " + load().g4ref_last_error().decode())


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(dp)


def _i32(off):
    a = np.ascontiguousarray(off, dtype=np.int32)
    return a, a.ctypes.data_as(ip)


def step_to_array(st) -> np.ndarray:
    return np.array([float(getattr(st, k)) for k in STEP_FIELDS])


def step_from_array(a):
    from genesis4_cuda_port_b200._lib import Step
    kw = {k: float(v) for k, v in zip(STEP_FIELDS, a)}
    kw["in_undulator"] = int(kw["in_undulator"])
    return Step(**kw, reserved=0)


def field_advance(cells, *, solver=0, gridmax, xlambda, harm=1, first=0, enabled=True,
                  atomic_source=False, delz, fc, step, off, current, parts,
                  filt=False, xc=0.0, yc=0.0, sig=0.0):
    """One FieldSolverADICUDA / FieldSolverFFTCUDA advance; returns new cells."""
    out = np.ascontiguousarray(cells, dtype=np.complex128).copy()
    S, n, _ = out.shape
    offa, offp = _i32(off)
    cur = np.ascontiguousarray(current, np.float64)
    _chk(load().g4ref_field_advance(solver, S, n, gridmax, xlambda, harm, first, int(enabled),
                                    int(atomic_source), delz, fc, C.byref(step), offp, _d(cur),
                                    _d(parts["x"]), _d(parts["y"]), _d(parts["gamma"]),
                                    _d(parts["theta"]), _d(out.reshape(-1).view(np.float64)),
                                    int(filt), xc, yc, sig))
    return out


def beam_advance(off, step, fields, parts, long_esc=None, particle_field=None):
    """BeamSolverCUDA::advance; fields: dicts(cells, first, harm, gridmax,
    xlambda, fc).  Updates parts['gamma'], parts['theta'] in place.
    particle_field: per-particle getEField values (short range on)."""
    offa, offp = _i32(off)
    nf = len(fields)
    keep = [np.ascontiguousarray(f["cells"], dtype=np.complex128) for f in fields]
    arr_i = lambda k, d=0: np.array([f.get(k, d) for f in fields], np.int32)  # noqa: E731
    first, harm = arr_i("first"), arr_i("harm", 1)
    ngrid = np.array([c.shape[1] for c in keep], np.int32)
    gm = np.array([f["gridmax"] for f in fields])
    xl = np.array([f["xlambda"] for f in fields])
    fc = np.array([f["fc"] for f in fields])
    ptrs = (dp * nf)(*[c.reshape(-1).view(np.float64).ctypes.data_as(dp) for c in keep])
    le = None if long_esc is None else np.ascontiguousarray(long_esc, np.float64)
    pf = None if particle_field is None else np.ascontiguousarray(particle_field, np.float64)
    load().g4ref_set_particle_ez(_d(pf))
    try:
        _beam_advance_call(offa, offp, step, nf, first, ngrid, harm, gm, xl, fc, ptrs, le,
                           parts)
    finally:
        load().g4ref_set_particle_ez(None)


def _beam_advance_call(offa, offp, step, nf, first, ngrid, harm, gm, xl, fc, ptrs, le, parts):
    _chk(load().g4ref_beam_advance(len(offa) - 1, offp, C.byref(step), nf,
                                   first.ctypes.data_as(ip), ngrid.ctypes.data_as(ip),
                                   harm.ctypes.data_as(ip), _d(gm), _d(xl), _d(fc), ptrs,
                                   _d(le), _d(parts["x"]), _d(parts["y"]), _d(parts["px"]),
                                   _d(parts["py"]), _d(parts["gamma"]), _d(parts["theta"])))


def track(parts, step, delz, last):
    _chk(load().g4ref_track(parts["x"].size, C.byref(step), delz, int(last), _d(parts["x"]),
                            _d(parts["y"]), _d(parts["px"]), _d(parts["py"]),
                            _d(parts["gamma"])))


def r56(parts, step, lambda0):
    _chk(load().g4ref_r56(parts["x"].size, C.byref(step), lambda0, _d(parts["gamma"]),
                          _d(parts["theta"])))


def slippage(cells, shift, sample, time_run, periodic, accuslip, first):
    acc = C.c_double(accuslip)
    fst = C.c_int(first)
    S, n, _ = cells.shape
    _chk(load().g4ref_slippage(S, n, shift, sample, int(time_run), int(periodic),
                               C.byref(acc), C.byref(fst),
                               _d(cells.reshape(-1).view(np.float64))))
    return acc.value, fst.value


BEAM_RECORDS = ["energy", "energyspread", "xposition", "xsize", "yposition", "ysize",
                "pxposition", "pyposition", "current", "emitx", "emity", "betax", "betay",
                "alphax", "alphay", "efield", "wakefield", "LSCfield", "SSCfield", "xmin",
                "xmax", "pxmin", "pxmax", "ymin", "ymax", "pymin", "pymax", "emin", "emax",
                "Global/energy", "Global/energyspread", "Global/xposition", "Global/xsize",
                "Global/yposition", "Global/ysize"]
FIELD_RECORDS = ["power", "xposition", "xsize", "yposition", "ysize", "intensity-nearfield",
                 "phase-nearfield", "intensity-farfield", "phase-farfield", "Global/energy",
                 "Global/xposition", "Global/xsize", "Global/yposition", "Global/ysize",
                 "Global/intensity-nearfield", "Global/intensity-farfield", "dgrid",
                 "gridspacing", "ngrid"]


def diag(off, parts, *, nharm, current, fields, slicelength, eloss=None, long_esc=None):
    """DiagnosticCUDA::calc at output step 0; returns (beam records, [field
    records]) as dicts name -> array."""
    offa, offp = _i32(off)
    S = len(offa) - 1
    nf = len(fields)
    keep = [np.ascontiguousarray(f["cells"], dtype=np.complex128) for f in fields]
    ngrid = np.array([c.shape[1] for c in keep], np.int32)
    first = np.array([f.get("first", 0) for f in fields], np.int32)
    gm = np.array([f["gridmax"] for f in fields])
    xl = np.array([f["xlambda"] for f in fields])
    ptrs = (dp * nf)(*[c.reshape(-1).view(np.float64).ctypes.data_as(dp) for c in keep])
    opt = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)  # noqa: E731
    cur, el, le = opt(current), opt(eloss), opt(long_esc)
    lib = load()
    _chk(lib.g4ref_diag(S, offp, _d(parts["x"]), _d(parts["y"]), _d(parts["px"]),
                        _d(parts["py"]), _d(parts["gamma"]), _d(parts["theta"]), nharm,
                        _d(cur), _d(el), _d(le), nf, ngrid.ctypes.data_as(ip),
                        first.ctypes.data_as(ip), _d(gm), _d(xl), slicelength, ptrs))

    def grab(group, name):
        buf = np.empty(max(S, 1))
        n = lib.g4ref_diag_record(group, name.encode(), _d(buf), buf.size)
        if n < 0:
            raise KeyError(name)
        return buf[:n].copy()

    names = list(BEAM_RECORDS)
    for h in range(1, nharm + 1):
        names += ["bunching" if h == 1 else f"bunching{h}",
                  "bunchingphase" if h == 1 else f"bunchingphase{h}"]
    beam = {k: grab(0, k) for k in names}
    flds = [{k: grab(1 + i, k) for k in FIELD_RECORDS} for i in range(nf)]
    return beam, flds


def time_steps(off, parts, current, cells, *, gridmax, xlambda, steps, fc, slip, sample,
               first_step=0, warmup=3, ntimed=10):
    """Milliseconds per step of the reference's own classes stepping one set of
    device-resident state (g4ref_time_steps); parts/cells are not modified."""
    from genesis4_cuda_port_b200._lib import Step
    offa, offp = _i32(off)
    n = len(steps)
    arr = (Step * n)(*steps)
    c = np.ascontiguousarray(cells, dtype=np.complex128)
    fca = np.ascontiguousarray(fc, np.float64)
    sla = np.ascontiguousarray(slip, np.float64)
    cur = np.ascontiguousarray(current, np.float64)
    ms = C.c_double(0.0)
    _chk(load().g4ref_time_steps(len(offa) - 1, offp, _d(parts["x"]), _d(parts["y"]),
                                 _d(parts["px"]), _d(parts["py"]), _d(parts["gamma"]),
                                 _d(parts["theta"]), _d(cur), c.shape[1], gridmax, xlambda,
                                 c.reshape(-1).view(np.float64).ctypes.data_as(dp), n, arr,
                                 _d(fca), _d(sla), sample, first_step, warmup, ntimed,
                                 C.byref(ms)))
    return ms.value
