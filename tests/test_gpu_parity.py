"""FP64 drop-in path on the GPU against the FP64 CPU oracle, phase by phase,
through the C ABI.  Tolerances are relative to the largest magnitude of the
oracle's output (FP64; the GPU sums in a different order and the ADI solve is
a reassociated Thomas recurrence)."""
import math

import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from oracle import pyoracle as orc
from tests import synth

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    c = dev.Context(0)
    yield c
    c.synchronize()


def _beam(ctx, off, parts, current=None):
    b = dev.BeamState(ctx, off, synth.GAMMA0)
    b.upload(parts)
    b.set_current(current if current is not None else np.full(len(off) - 1, synth.CURRENT))
    return b


@pytest.mark.parametrize("ngrid,nslice", [(7, 3), (33, 2), (64, 2), (151, 1), (201, 2), (301, 1)])
def test_adi_without_source(ctx, ngrid, nslice):
    gridmax = 200e-6
    f0 = synth.field(nslice, ngrid, gridmax, seed=ngrid)
    step = synth.drift_step(delz=0.015)
    off = np.zeros(nslice + 1, np.int64)
    parts = {k: np.zeros(0) for k in synth.copy_parts(synth.beam(1, 1)[1])}
    fld = dev.FieldState(ctx, nslice, ngrid, gridmax, synth.LAMBDA0)
    fld.upload(f0)
    beam = _beam(ctx, off, {k: np.zeros(0) for k in parts})
    adi = dev.FieldSolverADICUDA(ctx)
    adi.init(step.delz, fld.dgrid, fld.xks, ngrid)
    ref = f0.copy()
    for _ in range(3):
        adi.advance(fld, beam, step, fc=0.0)
        orc.adi_advance(ref, harm=1, gridmax=gridmax, xks=fld.xks, delz=step.delz, fc=0.0,
                        enabled=True, step=step, off=off, current=np.zeros(nslice), parts=parts)
    got = fld.download()
    assert synth.rel_err(got, ref) < TOL


@pytest.mark.parametrize("ngrid,nslice,first", [(33, 3, 1), (151, 2, 0), (201, 3, 2)])
def test_adi_with_deposited_source(ctx, ngrid, nslice, first):
    gridmax = 200e-6
    off, parts = synth.beam(nslice, 3000, seed=ngrid, ragged=True)
    f0 = synth.field(nslice, ngrid, gridmax, seed=7)
    step = synth.und_step()
    fc = synth.coupling()
    cur = np.linspace(1000, 3000, nslice)
    fld = dev.FieldState(ctx, nslice, ngrid, gridmax, synth.LAMBDA0)
    fld.upload(f0)
    fld.first = first
    beam = _beam(ctx, off, parts, cur)
    adi = dev.FieldSolverADICUDA(ctx)
    adi.init(step.delz, fld.dgrid, fld.xks, ngrid)
    adi.advance(fld, beam, step, fc=fc)
    ref = f0.copy()
    orc.adi_advance(ref, harm=1, gridmax=gridmax, xks=fld.xks, delz=step.delz, fc=fc,
                    enabled=True, step=step, off=off, current=cur, parts=parts, first=first)
    got = fld.download()
    assert synth.rel_err(got, ref) < TOL
    # the source alone (field zero) is also reproduced
    fld.upload(np.zeros_like(f0))
    adi.advance(fld, beam, step, fc=fc)
    ref = np.zeros_like(f0)
    orc.adi_advance(ref, harm=1, gridmax=gridmax, xks=fld.xks, delz=step.delz, fc=fc,
                    enabled=True, step=step, off=off, current=cur, parts=parts, first=first)
    assert synth.rel_err(fld.download(), ref) < 1e-11


def test_deposit_is_deterministic(ctx):
    nslice, ngrid, gridmax = 2, 151, 200e-6
    off, parts = synth.beam(nslice, 20000, seed=11)
    step = synth.und_step()
    outs = []
    for _ in range(2):
        fld = dev.FieldState(ctx, nslice, ngrid, gridmax, synth.LAMBDA0)
        beam = _beam(ctx, off, parts)
        adi = dev.FieldSolverADICUDA(ctx)
        adi.init(step.delz, fld.dgrid, fld.xks, ngrid)
        adi.advance(fld, beam, step, fc=synth.coupling())
        outs.append(fld.download())
    assert np.array_equal(outs[0], outs[1])


def test_source_off_outside_undulator_and_for_even_harmonics(ctx):
    nslice, ngrid, gridmax = 1, 33, 200e-6
    off, parts = synth.beam(nslice, 500, seed=12)
    beam = _beam(ctx, off, parts)
    for step, harm in [(synth.drift_step(delz=0.015), 1), (synth.und_step(), 2)]:
        fld = dev.FieldState(ctx, nslice, ngrid, gridmax, synth.LAMBDA0 / harm, harm=harm)
        adi = dev.FieldSolverADICUDA(ctx)
        adi.init(step.delz, fld.dgrid, fld.xks, ngrid)
        adi.advance(fld, beam, step, fc=synth.coupling())
        assert not np.any(fld.download())


@pytest.mark.parametrize("kind", ["drift", "fquad", "und", "chicane", "corrector"])
def test_transverse_track(ctx, kind):
    off, parts = synth.beam(3, 700, seed=13, ragged=True)
    steps = {
        "drift": (synth.drift_step(delz=0.2), False),
        "fquad": (synth.drift_step(delz=0.1, qf=1.5, dqx=1e-5, dqy=-2e-5), False),
        "und": (synth.und_step(ax=3e-6, ay=-2e-6, kx=0.3 * synth.KU ** 2), False),
        "chicane": (synth.drift_step(delz=0.1, chic_angle=2e-3, chic_lb=0.02,
                                     chic_ld=0.01, chic_lt=0.1), False),
        "corrector": (synth.drift_step(delz=0.1, cx=1e-6, cy=-3e-6), True),
    }
    step, last = steps[kind]
    beam = _beam(ctx, off, parts)
    beam.track(step, step.delz * 0.5, last)
    ref = synth.copy_parts(parts)
    orc.track(ref, step, step.delz * 0.5, last)
    got = beam.download()
    for k in ("x", "y", "px", "py"):
        assert synth.rel_err(got[k], ref[k]) < TOL, k


def test_r56(ctx):
    off, parts = synth.beam(2, 500, seed=14)
    step = synth.drift_step(delz=0.1, chic_angle=2e-3, chic_lb=0.02, chic_ld=0.01, chic_lt=0.1)
    beam = _beam(ctx, off, parts)
    beam.apply_r56(step, synth.LAMBDA0)
    ref = synth.copy_parts(parts)
    orc.r56(ref, step, synth.LAMBDA0)
    assert synth.rel_err(beam.download()["theta"], ref["theta"]) < TOL


@pytest.mark.parametrize("nfield", [1, 2])
def test_push(ctx, nfield):
    nslice, ngrid, gridmax = 3, 65, 150e-6
    off, parts = synth.beam(nslice, 2000, seed=15, ragged=True)
    step = synth.und_step(autophase=0.1)
    eloss = np.array([1e-3, -2e-3, 0.0])
    beam = _beam(ctx, off, parts)
    beam.set_eloss(eloss)
    flds, views, fcs = [], [], []
    for i in range(nfield):
        h = 1 + 2 * i
        cells = synth.field(nslice, ngrid, gridmax, seed=20 + i, amplitude=3e13)
        f = dev.FieldState(ctx, nslice, ngrid, gridmax, synth.LAMBDA0 / h, harm=h)
        f.upload(cells)
        f.first = i % nslice
        flds.append(f)
        fcs.append(synth.coupling(harm=h))
        views.append(dict(cells=cells, first=i % nslice, harm=h, gridmax=gridmax,
                          xlambda=synth.LAMBDA0 / h, fc=fcs[-1]))
    beam.advance(flds, fcs, step)
    ref = synth.copy_parts(parts)
    orc.push(off, step, views, ref, slice_eloss=eloss)
    got = beam.download()
    # gamma changes by a small amount: compare the change
    dg = got["gamma"] - parts["gamma"]
    dg_ref = ref["gamma"] - parts["gamma"]
    assert np.max(np.abs(dg_ref)) > 1e-6
    assert synth.rel_err(dg, dg_ref) < 1e-10
    assert synth.rel_err(got["theta"], ref["theta"]) < TOL


def test_slippage_bit_exact(ctx):
    nslice, ngrid = 6, 17
    f0 = synth.field(nslice, ngrid, 100e-6, seed=30)
    fld = dev.FieldState(ctx, nslice, ngrid, 100e-6, synth.LAMBDA0)
    fld.upload(f0)
    ref = f0.copy()
    acc, first = 0.0, 0
    for shift in [1.0, 2.6, -0.4, -1.7, 0.5, 3.0]:
        n_gpu = fld.apply_slippage(shift, 1.0)
        acc, first, n_ref = orc.slippage(ref, shift, 1.0, True, False, acc, first)
        assert n_gpu == n_ref and fld.first == first
        assert fld.accuslip == acc
    assert np.array_equal(fld.download(), ref)


@pytest.mark.parametrize("need_aux,nharm", [(True, 1), (False, 3), (True, 10)])
def test_beam_diagnostics(ctx, need_aux, nharm):
    off, parts = synth.beam(4, 1500, seed=31, ragged=True)
    beam = _beam(ctx, off, parts)
    stats, bre, bim = beam.diagnostics(nharm, need_aux)
    rs, rbre, rbim = orc.diag_beam(off, parts, nharm, need_aux)
    np.testing.assert_allclose(stats, rs, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(bre, rbre, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(bim, rbim, rtol=1e-9, atol=1e-9)


def test_field_diagnostics(ctx):
    nslice, ngrid = 4, 45
    f0 = synth.field(nslice, ngrid, 100e-6, seed=32)
    fld = dev.FieldState(ctx, nslice, ngrid, 100e-6, synth.LAMBDA0)
    fld.upload(f0)
    fld.first = 3
    stats, center = fld.diagnostics()
    rs, rc = orc.diag_field(f0, 3)
    np.testing.assert_allclose(stats, rs, rtol=1e-11, atol=1e-12 * np.max(np.abs(rs)))
    np.testing.assert_array_equal(center, rc)


def test_full_steps_match_oracle(ctx):
    """Five Gencore steps (beam track/advance/R56/track, field track, slippage)
    in the reference order, through the per-phase entry points."""
    nslice, ngrid, gridmax = 4, 65, 160e-6
    off, parts = synth.beam(nslice, 1500, seed=40)
    cells = synth.field(nslice, ngrid, gridmax, seed=41, amplitude=1e12)
    cur = np.full(nslice, synth.CURRENT)
    fc = synth.coupling()
    beam = _beam(ctx, off, parts, cur)
    fld = dev.FieldState(ctx, nslice, ngrid, gridmax, synth.LAMBDA0)
    fld.upload(cells)
    adi = dev.FieldSolverADICUDA(ctx)
    ref_parts = synth.copy_parts(parts)
    ref_field = dict(cells=cells.copy(), gridmax=gridmax, xlambda=synth.LAMBDA0, fc=fc,
                     first=0, accuslip=0.0)
    steps = [synth.und_step(), synth.und_step(), synth.drift_step(delz=0.05, qf=1.5),
             synth.und_step(), synth.und_step()]
    for st in steps:
        slip = 1.0 if st.in_undulator else 0.3
        fcs = fc if st.in_undulator else 0.0
        beam.track(st, st.delz * 0.5, False)
        beam.advance([fld], [fcs], st)
        beam.apply_r56(st, synth.LAMBDA0)
        beam.track(st, st.delz * 0.5, True)
        adi.init(st.delz, fld.dgrid, fld.xks, ngrid)
        adi.advance(fld, beam, st, fc=fcs)
        fld.apply_slippage(slip, 1.0)
        ref_field["fc"] = fcs
        orc.step(off, cur, st, synth.LAMBDA0, slip, 1.0, True, False, [ref_field], ref_parts)
    got = beam.download()
    for k in parts:
        assert synth.rel_err(got[k], ref_parts[k]) < 1e-11, k
    assert fld.first == ref_field["first"]
    assert synth.rel_err(fld.download(), ref_field["cells"]) < 1e-11
