"""Bounded waits end with an error status, not a hang.

Every mbarrier wait in the kernels gives up after a bounded number of polls,
sets the context's device error word and returns.  g4b_ctx_selftest_wait runs
that wait on a barrier phase nothing completes, with a short limit; the call
must report the timeout and leave the context usable for the next step."""
import ctypes as C

import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from genesis4_cuda_port_b200._lib import G4BError
from oracle import pyoracle as orc
from tests import synth

pytestmark = pytest.mark.gpu


def test_wait_gives_up_and_reports():
    ctx = dev.Context(0)
    lib = ctx.lib
    timed_out = C.c_int(-1)
    rc = lib.g4b_ctx_selftest_wait(ctx.h, 4096, C.byref(timed_out))
    assert rc == 6, rc  # G4B_ERR_DEVICE
    assert timed_out.value == 1
    assert b"wait timeout" in lib.g4b_last_error()
    # the error word was cleared when it was reported
    ctx.synchronize()
    # and the context still runs a field step correctly
    nslice, ngrid, gridmax = 2, 33, 1.5e-4
    off, p = synth.beam(nslice, 256, seed=9)
    cells = synth.field(nslice, ngrid, gridmax, seed=10, amplitude=1e11)
    st = synth.und_step()
    beam = dev.BeamState(ctx, off, synth.GAMMA0)
    beam.upload(p)
    beam.set_current(np.full(nslice, synth.CURRENT))
    fld = dev.FieldState(ctx, nslice, ngrid, gridmax, synth.LAMBDA0)
    fld.upload(cells)
    adi = dev.FieldSolverADICUDA(ctx)
    adi.init(st.delz, fld.dgrid, fld.xks, ngrid)
    adi.advance(fld, beam, st, fc=synth.coupling())
    ref = cells.copy()
    orc.adi_advance(ref, harm=1, gridmax=gridmax, xks=fld.xks, delz=st.delz,
                    fc=synth.coupling(), enabled=True, step=st, off=off,
                    current=np.full(nslice, synth.CURRENT), parts=p)
    assert synth.rel_err(fld.download(), ref) < 1e-12
    with pytest.raises(G4BError):
        from genesis4_cuda_port_b200._lib import check
        check(lib.g4b_ctx_selftest_wait(ctx.h, 0, C.byref(timed_out)))
    for o in (adi, fld, beam):
        o.close()
    ctx.close()
