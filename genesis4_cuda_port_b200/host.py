"""ctypes binding of the host layer's C ABI (include/g4h.h): beam/field
loading and lattice expansion into per-step undulator tables."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import G4BError, Step, dptr

_HOSTLIB = Path(__file__).resolve().parent / "lib" / "libg4host.so"


class BeamSpec(C.Structure):
    """Mirror of ``g4h_beam_spec``."""

    _fields_ = [("nslice", C.c_int), ("npart", C.c_int), ("nbins", C.c_int),
                ("shotnoise", C.c_int), ("seed", C.c_uint64),
                ("gamma0", C.c_double), ("delgam", C.c_double), ("ex", C.c_double),
                ("ey", C.c_double), ("betax", C.c_double), ("betay", C.c_double),
                ("alphax", C.c_double), ("alphay", C.c_double),
                ("xcenter", C.c_double), ("ycenter", C.c_double),
                ("pxcenter", C.c_double), ("pycenter", C.c_double),
                ("reflength", C.c_double), ("slicelength", C.c_double)]

    def __init__(self, **kw):
        super().__init__()
        for k, v in kw.items():
            setattr(self, k, v)


_h = None


def load():
    global _h
    if _h is not None:
        return _h
    _lib.load()  # resolves libg4b200.so first
    if not _HOSTLIB.exists():
        raise RuntimeError(f"{_HOSTLIB} is missing: build it with "
                           "`python -m genesis4_cuda_port_b200.build`")
    h = C.CDLL(str(_HOSTLIB))
    h.g4h_last_error.restype = C.c_char_p
    h.g4h_load_beam.argtypes = [C.POINTER(BeamSpec), _lib.c_double_p] + \
        [_lib.c_double_p] * 6 + [_lib.c_int64_p]
    h.g4h_gaussian_field.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double,
                                     C.c_double, _lib.c_double_p]
    h.g4h_lattice_parse.argtypes = [C.c_char_p, C.c_char_p, C.c_double, C.c_double,
                                    C.c_double, _lib.c_void_pp]
    h.g4h_lattice_destroy.argtypes = [C.c_void_p]
    h.g4h_lattice_nstep.argtypes = [C.c_void_p, _lib.c_int_p]
    h.g4h_lattice_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(Step),
                                   _lib.c_double_p, _lib.c_double_p, _lib.c_int_p]
    h.g4h_lattice_fc.argtypes = [C.c_void_p, C.c_int, C.c_int, _lib.c_double_p]
    h.g4h_coupling.restype = C.c_double
    h.g4h_coupling.argtypes = [C.c_double, C.c_int, C.c_int]
    _h = h
    return h


def _check(rc):
    if rc != 0:
        raise G4BError(rc, load().g4h_last_error().decode())


def library_path() -> Path:
    return _HOSTLIB


def load_beam(spec: BeamSpec, current):
    """Quiet-start (+ shot noise) beam: returns (slice_offsets, parts dict)."""
    n = spec.nslice * spec.npart
    parts = {k: np.empty(n) for k in ("x", "y", "px", "py", "gamma", "theta")}
    off = np.empty(spec.nslice + 1, np.int64)
    cur = np.ascontiguousarray(np.broadcast_to(current, (spec.nslice,)), np.float64)
    _check(load().g4h_load_beam(C.byref(spec), dptr(cur),
                                *[dptr(parts[k]) for k in ("x", "y", "px", "py", "gamma", "theta")],
                                off.ctypes.data_as(_lib.c_int64_p)))
    return off, parts


def gaussian_field(ngrid, gridmax, xlambda, power, w0):
    out = np.empty((ngrid, ngrid), np.complex128)
    _check(load().g4h_gaussian_field(ngrid, gridmax, xlambda, power, w0,
                                     dptr(out.reshape(-1).view(np.float64))))
    return out


def coupling(aw, harm=1, helical=False):
    return float(load().g4h_coupling(aw, harm, int(helical)))


class Lattice:
    """A .lat beamline expanded into per-step tables (upstream Undulator)."""

    def __init__(self, text: str, beamline: str, delz: float, gamma0: float, lambda0: float):
        h = C.c_void_p()
        _check(load().g4h_lattice_parse(text.encode(), beamline.encode(), delz, gamma0,
                                        lambda0, C.byref(h)))
        self.h = h
        n = C.c_int()
        _check(load().g4h_lattice_nstep(h, C.byref(n)))
        self.nstep = n.value
        self.steps, self.slip, self.z, self.marker = [], [], [], []
        for i in range(self.nstep):
            st, sl, z, m = Step(), C.c_double(), C.c_double(), C.c_int()
            _check(load().g4h_lattice_step(h, i, C.byref(st), C.byref(sl), C.byref(z),
                                           C.byref(m)))
            self.steps.append(st)
            self.slip.append(sl.value)
            self.z.append(z.value)
            self.marker.append(m.value)

    def fc(self, i: int, harm: int = 1) -> float:
        v = C.c_double()
        _check(load().g4h_lattice_fc(self.h, i, harm, C.byref(v)))
        return v.value

    def __del__(self):
        try:
            if getattr(self, "h", None):
                load().g4h_lattice_destroy(self.h)
                self.h = None
        except Exception:
            pass
