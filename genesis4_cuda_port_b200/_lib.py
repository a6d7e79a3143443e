"""ctypes binding of the C ABI declared in include/g4b.h.

The shared library is loaded from the package's ``lib/`` directory (built in
tree by ``genesis4_cuda_port_b200.build``).  There is no fallback: if the
library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIBDIR = Path(__file__).resolve().parent / "lib"

c_double_p = C.POINTER(C.c_double)
c_int64_p = C.POINTER(C.c_int64)
c_int_p = C.POINTER(C.c_int)
c_uint64_p = C.POINTER(C.c_uint64)
c_void_pp = C.POINTER(C.c_void_p)

G4B_OK = 0
G4B_FP64 = 0
G4B_MIXED = 1


class G4BError(RuntimeError):
    """A g4b_* call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"g4b error {code}: {message}")
        self.code = code


class Step(C.Structure):
    """Mirror of ``g4b_step`` (include/g4b.h)."""

    _fields_ = [
        ("delz", C.c_double), ("aw", C.c_double), ("ax", C.c_double),
        ("ay", C.c_double), ("kx", C.c_double), ("ky", C.c_double),
        ("gradx", C.c_double), ("grady", C.c_double), ("ku", C.c_double),
        ("gamma_ref", C.c_double), ("autophase", C.c_double),
        ("qf", C.c_double), ("dqx", C.c_double), ("dqy", C.c_double),
        ("cx", C.c_double), ("cy", C.c_double), ("chic_angle", C.c_double),
        ("chic_lb", C.c_double), ("chic_ld", C.c_double),
        ("chic_lt", C.c_double), ("in_undulator", C.c_int),
        ("reserved", C.c_int),
    ]

    def __init__(self, **kw):
        super().__init__()
        for k, v in kw.items():
            setattr(self, k, v)


class RunDesc(C.Structure):
    """Mirror of ``g4b_run_desc`` (include/g4b.h)."""

    _fields_ = [("nslice", C.c_int), ("nfield", C.c_int), ("harm", C.c_int * 8),
                ("ngrid", C.c_int * 8), ("gridmax", C.c_double * 8),
                ("lambda0", C.c_double), ("gamma_ref", C.c_double),
                ("sample", C.c_double), ("time_run", C.c_int), ("periodic", C.c_int),
                ("nbunch", C.c_int), ("precision", C.c_int)]


# name -> (restype, argtypes)
_SIGS = {
    "g4b_last_error": (C.c_char_p, []),
    "g4b_version": (C.c_int, []),
    "g4b_ctx_create": (C.c_int, [C.c_int, c_void_pp]),
    "g4b_ctx_destroy": (C.c_int, [C.c_void_p]),
    "g4b_ctx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "g4b_ctx_get_stream": (C.c_void_p, [C.c_void_p]),
    "g4b_ctx_synchronize": (C.c_int, [C.c_void_p]),
    "g4b_ctx_launch_count": (C.c_int, [C.c_void_p, c_uint64_p]),
    "g4b_ctx_sm_count": (C.c_int, [C.c_void_p, c_int_p]),
    "g4b_ctx_selftest_wait": (C.c_int, [C.c_void_p, C.c_uint, c_int_p]),
    "g4b_ctx_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "g4b_ctx_profile_read": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, c_uint64_p,
                                       c_double_p, c_int_p]),
    "g4b_field_create": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double,
                                   C.c_double, C.c_int, C.c_int, C.c_int,
                                   c_void_pp]),
    "g4b_field_destroy": (C.c_int, [C.c_void_p]),
    "g4b_field_upload": (C.c_int, [C.c_void_p, c_double_p]),
    "g4b_field_download": (C.c_int, [C.c_void_p, c_double_p]),
    "g4b_field_set_first": (C.c_int, [C.c_void_p, C.c_int]),
    "g4b_field_get_first": (C.c_int, [C.c_void_p, c_int_p]),
    "g4b_field_device_bytes": (C.c_int, [C.c_void_p, c_uint64_p]),
    "g4b_beam_create": (C.c_int, [C.c_void_p, C.c_int, c_int64_p, C.c_int,
                                  C.c_double, c_void_pp]),
    "g4b_beam_destroy": (C.c_int, [C.c_void_p]),
    "g4b_beam_upload": (C.c_int, [C.c_void_p] + [c_double_p] * 6),
    "g4b_beam_download": (C.c_int, [C.c_void_p] + [c_double_p] * 6),
    "g4b_beam_set_current": (C.c_int, [C.c_void_p, c_double_p]),
    "g4b_beam_set_eloss": (C.c_int, [C.c_void_p, c_double_p]),
    "g4b_beam_set_particle_ez": (C.c_int, [C.c_void_p, c_double_p]),
    "g4b_beam_get_particle_ez": (C.c_int, [C.c_void_p, c_double_p]),
    "g4b_beam_device_bytes": (C.c_int, [C.c_void_p, c_uint64_p]),
    "g4b_batch_tune_layouts": (C.c_int, [C.c_void_p]),
    "g4b_run_get_layouts": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "g4b_run_set_layouts": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "g4b_default_layout": (C.c_int, [C.c_int]),
    "g4b_isr_rates": (C.c_int, [C.c_double, C.c_double, C.c_int, c_double_p, c_double_p]),
    "g4b_beam_incoherent": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_int,
                                      C.c_int, C.c_uint64, C.c_uint64]),
    "g4b_efield_create": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int,
                                    C.c_double, c_void_pp]),
    "g4b_efield_destroy": (C.c_int, [C.c_void_p]),
    "g4b_efield_has_short_range": (C.c_int, [C.c_void_p]),
    "g4b_efield_short_range": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "g4b_adi_create": (C.c_int, [C.c_void_p, c_void_pp]),
    "g4b_adi_destroy": (C.c_int, [C.c_void_p]),
    "g4b_adi_init": (C.c_int, [C.c_void_p, C.c_double, C.c_double,
                               C.c_double, C.c_int]),
    "g4b_adi_advance": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(Step), C.c_double, C.c_int]),
    "g4b_field_plane_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "g4b_field_plane_out": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "g4b_field_plane_in": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "g4b_field_zero_plane": (C.c_int, [C.c_void_p, C.c_int]),
    "g4b_fft_create": (C.c_int, [C.c_void_p, c_void_pp]),
    "g4b_fft_destroy": (C.c_int, [C.c_void_p]),
    "g4b_fft_init_filter": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                      C.c_int]),
    "g4b_fft_init": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int]),
    "g4b_fft_advance": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Step),
                                  C.c_double, C.c_int]),
    "g4b_beam_track": (C.c_int, [C.c_void_p, C.POINTER(Step), C.c_double,
                                 C.c_int]),
    "g4b_beam_r56": (C.c_int, [C.c_void_p, C.POINTER(Step), C.c_double]),
    "g4b_beam_advance": (C.c_int, [C.c_void_p, c_void_pp, c_double_p, C.c_int,
                                   C.POINTER(Step)]),
    "g4b_slippage": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int,
                               C.c_int, c_double_p, c_int_p]),
    "g4b_diag_beam": (C.c_int, [C.c_void_p, C.c_int, C.c_int, c_double_p,
                                c_double_p, c_double_p]),
    "g4b_diag_field": (C.c_int, [C.c_void_p, c_double_p, c_double_p]),
    "g4b_diag_field_static": (C.c_int, [C.c_void_p, c_double_p, c_double_p]),
    "g4b_run_create": (C.c_int, [C.c_void_p, C.POINTER(RunDesc), c_int64_p, c_void_pp]),
    "g4b_run_destroy": (C.c_int, [C.c_void_p]),
    "g4b_run_history_range": (C.c_int, [C.c_void_p, C.c_int, C.c_int, c_double_p]),
    "g4b_batch_create": (C.c_int, [C.c_void_p, C.c_int, c_void_pp]),
    "g4b_batch_destroy": (C.c_int, [C.c_void_p]),
    "g4b_batch_attach": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, c_int_p]),
    "g4b_batch_detach": (C.c_int, [C.c_void_p, C.c_int]),
    "g4b_batch_status": (C.c_int, [C.c_void_p, C.c_int, c_int_p, c_int_p]),
    "g4b_batch_step": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "g4b_batch_tune": (C.c_int, [C.c_void_p]),
    "g4b_batch_shapes": (C.c_int, [C.c_void_p, c_int_p]),
    "g4b_ctx_mark": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "g4b_ctx_mark_query": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, c_int_p]),
    "g4b_ctx_mem_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "g4b_run_upload_beam": (C.c_int, [C.c_void_p] + [c_double_p] * 6),
    "g4b_run_download_beam": (C.c_int, [C.c_void_p] + [c_double_p] * 6),
    "g4b_run_upload_field": (C.c_int, [C.c_void_p, C.c_int, c_double_p, C.c_int]),
    "g4b_run_download_field": (C.c_int, [C.c_void_p, C.c_int, c_double_p, c_int_p]),
    "g4b_run_set_current": (C.c_int, [C.c_void_p, c_double_p]),
    "g4b_run_set_eloss": (C.c_int, [C.c_void_p, c_double_p]),
    "g4b_run_set_lattice": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Step), c_double_p,
                                      c_double_p, C.c_int]),
    "g4b_run_advance": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "g4b_run_prepare": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "g4b_run_history": (C.c_int, [C.c_void_p, C.c_int, c_double_p, c_double_p]),
    "g4b_run_device_bytes": (C.c_int, [C.c_void_p, c_uint64_p]),
}

_lib = None


def lib_path() -> Path:
    return _LIBDIR / "libg4b200.so"


def load():
    """Load libg4b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not path.exists():
        raise RuntimeError(
            f"{path} is missing: build it with `python -m genesis4_cuda_port_b200.build`"
            " (there is no CPU fallback)")
    lib = C.CDLL(str(path))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols():
    """Every entry point the binding expects the library to export."""
    return sorted(_SIGS)


def check(rc: int) -> None:
    if rc != G4B_OK:
        msg = load().g4b_last_error()
        raise G4BError(rc, msg.decode() if msg else "")


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"], "need C-contiguous float64"
    return a.ctypes.data_as(c_double_p)
