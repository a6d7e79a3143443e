"""The G4DS container of the output and dump files: a file written to the
documented layout (include/g4h.h) is read back identically by the host
library's reader and by the pure-Python reader (no GPU needed)."""
import struct

import numpy as np
import pytest

from genesis4_cuda_port_b200 import host
from genesis4_cuda_port_b200._lib import G4BError


def _write(path, sets):
    with open(path, "wb") as f:
        f.write(b"G4DS\x00\x00\x00\x01")
        f.write(struct.pack("<Q", len(sets)))
        for name, arr in sets.items():
            a = np.ascontiguousarray(arr, dtype="<f8")
            nb = name.encode()
            f.write(struct.pack("<I", len(nb)) + nb)
            f.write(struct.pack("<II", 0, a.ndim))
            f.write(struct.pack(f"<{a.ndim}Q", *a.shape))
            f.write(a.tobytes())


def test_readers_agree(tmp_path):
    rng = np.random.default_rng(1)
    sets = {"Beam/energy": rng.normal(size=(3, 5)), "slice000001/field-real": rng.normal(size=(4, 4)),
            "Meta/steps": np.array([17.0])}
    path = tmp_path / "x.out.g4"
    _write(path, sets)
    got = host.read_g4ds(path)
    assert set(got) == set(sets)
    for k, v in sets.items():
        assert np.array_equal(got[k], v)
        assert np.array_equal(host.file_dataset(path, k), v)


def test_reader_rejects_other_files(tmp_path):
    p = tmp_path / "bad.g4"
    p.write_bytes(b"HDF5 not really")
    with pytest.raises(G4BError, match="not a G4DS"):
        host.file_dataset(p, "x")
    with pytest.raises(ValueError):
        host.read_g4ds(p)
