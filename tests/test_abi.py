"""The C-ABI libraries load and export every entry point include/*.h declares
(no GPU needed: nothing is called)."""
import ctypes
import re
from pathlib import Path

import pytest

from genesis4_cuda_port_b200 import _lib, build

ROOT = Path(__file__).resolve().parent.parent


def _declared(header: Path):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(g4[bh]_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def device_lib():
    if not _lib.lib_path().exists():
        build.build_device()
    return ctypes.CDLL(str(_lib.lib_path()))


def test_device_library_exports_every_declared_symbol(device_lib):
    names = _declared(ROOT / "include" / "g4b.h")
    assert len(names) > 20
    missing = [n for n in names if not hasattr(device_lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    names = _declared(ROOT / "include" / "g4b.h")
    assert set(names) <= set(_lib.declared_symbols()) | {"g4b_version"}


def test_errors_are_reported_without_a_gpu(device_lib):
    lib = _lib.load()
    rc = lib.g4b_beam_track(None, None, 0.0, 0)
    assert rc == 1  # G4B_ERR_ARG, nothing thrown across the ABI
    assert b"null" in lib.g4b_last_error()


def test_run_create_rejects_slices_above_the_particle_bound(device_lib):
    """The mixed form's deposition takes at most 65536 particles per slice;
    g4b_run_create says so before it touches the device (no GPU needed)."""
    import numpy as np
    lib = _lib.load()
    d = _lib.RunDesc()
    d.nslice, d.nfield, d.harm[0], d.ngrid[0], d.gridmax[0] = 2, 1, 1, 33, 1e-4
    d.lambda0, d.gamma_ref, d.sample, d.time_run, d.nbunch = 1e-10, 1e4, 1.0, 1, 1
    d.precision = _lib.G4B_MIXED
    out = ctypes.c_void_p()
    off = np.array([0, 65536, 65536 + 65537], np.int64)
    rc = lib.g4b_run_create(None, ctypes.byref(d), off.ctypes.data_as(_lib.c_int64_p),
                            ctypes.byref(out))
    assert rc == 5  # G4B_ERR_RANGE
    assert b"slice 1 holds 65537 particles" in lib.g4b_last_error()
    off = np.array([0, 65536, 2 * 65536], np.int64)
    rc = lib.g4b_run_create(None, ctypes.byref(d), off.ctypes.data_as(_lib.c_int64_p),
                            ctypes.byref(out))
    assert rc == 1 and b"null ctx" in lib.g4b_last_error()
