"""g4b_diag_field_static: the field statistics with their device scratch in
a fixed array of the library instead of an allocated buffer.  Called through
the C ABI and compared with g4b_diag_field on the same field, twice in a row
(the second call reuses the array the first one wrote)."""
import ctypes as C

import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from genesis4_cuda_port_b200._lib import G4BError, check, dptr
from tests import synth

pytestmark = pytest.mark.gpu

MAX_SLICES = 4096  # the fixed scratch bound stated in include/g4b.h


@pytest.fixture(scope="module")
def ctx():
    c = dev.Context(0)
    yield c
    c.synchronize()


def _static_diag(fld):
    stats = np.full((fld.nslice, 7), np.nan)
    center = np.full((fld.nslice, 2), np.nan)
    check(fld.lib.g4b_diag_field_static(fld.h, dptr(stats.reshape(-1)),
                                        dptr(center.reshape(-1))))
    return stats, center


@pytest.mark.parametrize("precision", [dev.G4B_FP64, dev.G4B_MIXED])
def test_static_scratch_matches_allocating_entry(ctx, precision):
    nslice, ngrid, gridmax = 7, 45, 160e-6
    cells = synth.field(nslice, ngrid, gridmax, seed=81, amplitude=2e12)
    fld = dev.FieldState(ctx, nslice, ngrid, gridmax, synth.LAMBDA0, precision=precision)
    fld.upload(cells)
    fld.first = 3
    ref_stats, ref_center = fld.diagnostics()
    tol = 1e-12  # the same kernel on the same cells
    for _ in range(2):
        stats, center = _static_diag(fld)
        np.testing.assert_allclose(stats, ref_stats, rtol=tol, atol=0)
        np.testing.assert_allclose(center, ref_center, rtol=tol, atol=0)
    # a different field through the same array right after
    cells2 = synth.field(nslice, ngrid, gridmax, seed=82, amplitude=5e11)
    fld.upload(cells2)
    ref2, cen2 = fld.diagnostics()
    stats, center = _static_diag(fld)
    np.testing.assert_allclose(stats, ref2, rtol=1e-12, atol=0)
    np.testing.assert_allclose(center, cen2, rtol=1e-12, atol=0)
    fld.close()


def test_static_scratch_rejects_more_slices_than_it_holds(ctx):
    fld = dev.FieldState(ctx, MAX_SLICES + 1, 3, 1e-4, synth.LAMBDA0)
    with pytest.raises(G4BError, match="4096"):
        _static_diag(fld)
    fld.close()
    ok = dev.FieldState(ctx, MAX_SLICES, 3, 1e-4, synth.LAMBDA0)
    ok.upload(np.ones((MAX_SLICES, 3, 3), np.complex128))
    stats, center = _static_diag(ok)
    np.testing.assert_allclose(stats[:, 0], 9.0)
    np.testing.assert_allclose(center[:, 0], 1.0)
    ok.close()
