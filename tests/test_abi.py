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
