"""The FFT field solver (FieldSolverFFTCUDA) on the GPU against the
reference's own outputs (tests/golden/ref_fft_*.npz, recorded from the
reference's cuFFT-based class) and against the FP64 oracle at the
configurations' grids, with and without the source filter.  Tolerance 1e-12
of the largest magnitude: the transforms differ only in rounding."""
from pathlib import Path

import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from oracle import pyoracle as orc
from oracle import refpy
from tests import synth

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def ctx():
    c = dev.Context(0)
    yield c
    c.synchronize()


def _gpu_fft_step(ctx, cells, *, harm, gridmax, xlambda, first, delz, fc, step, off, current,
                  parts, filt=None, enabled=True):
    S, n, _ = cells.shape
    beam = dev.BeamState(ctx, off, synth.GAMMA0)
    beam.upload(parts)
    beam.set_current(current)
    fld = dev.FieldState(ctx, S, n, gridmax, xlambda, harm=harm)
    fld.upload(cells)
    fld.first = first
    sol = dev.FieldSolverFFTCUDA(ctx)
    if filt is not None:
        sol.init_source_filter(*filt, True)
    sol.init(delz, fld.dgrid, fld.xks, n)
    sol.advance(fld, beam, step, fc=fc, enabled=enabled)
    out = fld.download()
    for o in (sol, fld, beam):
        o.close()
    return out


@pytest.mark.parametrize("name", ["fft_n31", "fft_n32_filter", "fft_n31_h3_filter"])
def test_fft_step_matches_reference_fixture(ctx, name):
    d = dict(np.load(GOLDEN / f"ref_{name}.npz"))
    st = refpy.step_from_array(d["step"])
    p = {k: d["in_" + k].copy() for k in ("x", "y", "px", "py", "gamma", "theta")}
    xc, yc, sig = d["filt"]
    got = _gpu_fft_step(ctx, d["cells_in"], harm=int(d["harm"]), gridmax=float(d["gridmax"]),
                        xlambda=float(d["xlambda"]), first=int(d["first"]), delz=st.delz,
                        fc=float(d["fc"]), step=st, off=d["off"], current=d["current"],
                        parts=p, filt=(xc, yc, sig) if sig > 0 else None)
    ref = d["cells_out"]
    assert synth.rel_err(got, ref) < 1e-12, synth.rel_err(got, ref)


@pytest.mark.parametrize("ngrid,filt", [(151, None), (201, None), (201, (0.2, 0.25, 0.05)),
                                        (255, None), (64, (0.3, 0.3, 0.1))])
def test_fft_step_matches_oracle(ctx, ngrid, filt):
    nslice, gridmax = 3, 2e-4
    off, p = synth.beam(nslice, 1200, seed=ngrid, ragged=True)
    cur = np.linspace(3000.0, 1000.0, nslice)
    cells = synth.field(nslice, ngrid, gridmax, seed=ngrid + 7, amplitude=1e12)
    st = synth.und_step(ax=1e-6, kx=0.5 * synth.KU ** 2, ky=0.5 * synth.KU ** 2)
    fc = synth.coupling()
    ref = cells.copy()
    xc, yc, sig = filt if filt else (0.0, 0.0, 0.0)
    orc.fft_advance(ref, harm=1, gridmax=gridmax, xks=2 * np.pi / synth.LAMBDA0, delz=st.delz,
                    fc=fc, enabled=True, step=st, off=off, current=cur, parts=p, first=1,
                    xc=xc, yc=yc, sig=sig)
    got = _gpu_fft_step(ctx, cells, harm=1, gridmax=gridmax, xlambda=synth.LAMBDA0, first=1,
                        delz=st.delz, fc=fc, step=st, off=off, current=cur, parts=p,
                        filt=filt)
    assert synth.rel_err(ref, cells) > 1e-3
    assert synth.rel_err(got, ref) < 1e-12, synth.rel_err(got, ref)


def test_fft_pure_diffraction_is_unitary_and_reversible(ctx):
    """No source: the propagator has |exp(i k2 dz)| = 1, so the power is kept,
    and a step of -dz undoes a step of +dz."""
    nslice, ngrid, gridmax = 2, 201, 2e-4
    off, p = synth.beam(nslice, 64, seed=3)
    cells = synth.field(nslice, ngrid, gridmax, seed=5, amplitude=1e12)
    st = synth.und_step(in_undulator=0)
    kw = dict(harm=1, gridmax=gridmax, xlambda=synth.LAMBDA0, first=0, fc=0.0, off=off,
              current=np.zeros(nslice), parts=p)
    fwd = _gpu_fft_step(ctx, cells, delz=0.5, step=st, **kw)
    np.testing.assert_allclose(np.sum(np.abs(fwd) ** 2, axis=(1, 2)),
                               np.sum(np.abs(cells) ** 2, axis=(1, 2)), rtol=1e-12)
    back = _gpu_fft_step(ctx, fwd, delz=-0.5, step=st, **kw)
    assert synth.rel_err(back, cells) < 1e-12


LAT = """
D1: DRIFT = { l = 0.2 };
QF: QUADRUPOLE = { l = 0.1, k1 = 2.0 };
QD: QUADRUPOLE = { l = 0.1, k1 = -2.0 };
UND: UNDULATOR = { lambdau = 0.02, nwig = 30, aw = 1.8, helical = False };
CELL: LINE = { UND, D1, QF, D1, UND, D1, QD, D1 };
"""

DECK = """
&setup
rootname = g
lattice = g.lat
beamline = CELL
lambda0 = 1.0e-10
gamma0 = 20000
delz = 0.1
npart = 512
nbins = 4
seed = 11
&end
&time
slen = 1.6e-9
sample = 4
&end
&field
power = 1e5
dgrid = 1.5e-4
ngrid = 65
waist_size = 30e-6
&end
&beam
current = 2500
delgam = 1.0
ex = 0.5e-6
ey = 0.5e-6
&end
&track
fft_fieldsolver = true
source_filter = true
xcut = 0.35
ycut = 0.3
sigmoid = 0.05
&end
"""


def test_fft_deck_matches_the_oracle():
    """A whole deck with fft_fieldsolver and source_filter through Gencore::run
    and the CUDA classes, against the oracle's track / push / R56 / FFT
    advance / slippage in Gencore's order on the same loaded beam and field."""
    from genesis4_cuda_port_b200 import host
    deck = host.Deck(DECK, LAT)
    res = deck.run()
    s = deck.info()
    lam, ns, n, gm = s["lambda0"], s["nslice"], 65, 1.5e-4
    spec = host.BeamSpec(nslice=ns, npart=s["npart"], nbins=4, shotnoise=1, seed=11,
                         gamma0=s["gamma0"], delgam=1.0, ex=0.5e-6, ey=0.5e-6,
                         betax=s["betax"], betay=s["betay"], alphax=s["alphax"],
                         alphay=s["alphay"], xcenter=0.0, ycenter=0.0, pxcenter=0.0,
                         pycenter=0.0, reflength=lam, slicelength=lam * s["sample"])
    cur = np.full(ns, s["current"])
    off, p = host.load_beam(spec, cur)
    cells = np.broadcast_to(host.gaussian_field(n, gm, lam, 1e5, 30e-6), (ns, n, n)).copy()
    lat = host.Lattice(LAT, "CELL", 0.1, s["gamma0"], lam)
    first, acc = 0, 0.0
    xks = 2 * np.pi / lam
    power = [orc.diag_field(cells, first)[0][:, 0]]
    for i in range(s["nrun"]):
        st, fc = lat.steps[i], lat.fc(i, 1)
        orc.track(p, st, st.delz * 0.5, False)
        orc.push(off, st, [dict(cells=cells, first=first, harm=1, gridmax=gm, xlambda=lam,
                                fc=fc)], p)
        orc.r56(p, st, lam)
        orc.track(p, st, st.delz * 0.5, True)
        orc.fft_advance(cells, harm=1, gridmax=gm, xks=xks, delz=st.delz, fc=fc, enabled=True,
                        step=st, off=off, current=cur, parts=p, first=first, xc=0.35, yc=0.3,
                        sig=0.05)
        acc, first, _ = orc.slippage(cells, lat.slip[i], s["sample"], True, False, acc, first)
        power.append(orc.diag_field(cells, first)[0][:, 0])
    dgrid = 2 * gm / (n - 1)
    scl = dgrid * 510998.95 / xks  # raw sum of |u|^2 -> W (DiagnosticCUDA.cpp:686, :735)
    power = np.array(power) * scl * scl / 376.73031346177
    got = res.field[0]["power"]
    assert got.shape == power.shape
    assert abs(power[-1].sum() - power[0].sum()) > 1e-3 * power[0].sum()
    np.testing.assert_allclose(got, power, rtol=1e-9, atol=1e-12 * np.max(power))
