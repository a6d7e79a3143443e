"""Short-range space charge on the device and the push's per-particle loss.

* g4b_efield_short_range against the oracle's restatement of the same model
  (oracle/pyoracle.py short_range), whose physics the CPU tests pin to closed
  forms (tests/test_space_charge.py); bit-identical on a second call.
* The push reading a per-particle loss (the reference's UseParticleEz kernels,
  src/Core/BeamSolverCUDA.cpp:184-195, 633-680) three ways: the drop-in
  kernel, the oracle and the reference's own BeamSolverCUDA, whose
  short-range branch (:525-547) is fed the same per-particle values through
  the stand-in EFieldSolver of oracle/_ref.
* A deck with &efield through the drop-in classes, against the same deck
  without it and the oracle's per-particle loss of the loaded beam.
"""
import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from genesis4_cuda_port_b200._lib import G4BError
from oracle import pyoracle as orc
from oracle import refpy
from tests import synth

pytestmark = pytest.mark.gpu

GZ2 = synth.GAMMA0 ** 2 / (1 + synth.AW ** 2)


@pytest.fixture(scope="module")
def ctx():
    c = dev.Context(0)
    yield c
    c.synchronize()


def _bunched(nslice, npart, seed):
    off, p = synth.beam(nslice, npart, seed=seed, ragged=True)
    rng = np.random.default_rng(seed + 1)
    # a modulation at the first and second harmonic on top of shot noise
    p["theta"] = p["theta"] + 0.3 * np.sin(p["theta"]) + 0.1 * rng.standard_normal(p["theta"].size)
    return off, p


@pytest.mark.parametrize("nz,nphi,ngrid,rmax", [(1, 0, 50, 1.5), (2, 2, 40, 2.0),
                                                (3, 1, 128, 1.2)])
def test_short_range_matches_the_oracle(ctx, nz, nphi, ngrid, rmax):
    off, p = _bunched(4, 3000, seed=11 + nz)
    cur = np.array([2500.0, 1200.0, 3000.0, 800.0])
    el = np.array([1e-4, -2e-4, 0.0, 3e-5])
    beam = dev.BeamState(ctx, off, synth.GAMMA0)
    beam.upload(p)
    beam.set_current(cur)
    beam.set_eloss(el)
    sc = dev.EFieldSolver(ctx, rmax, ngrid, nz, nphi, synth.LAMBDA0)
    assert sc.has_short_range()
    sc.short_range(beam, GZ2)
    got = beam.particle_ez()
    want = orc.short_range(off, p, cur, GZ2, rmax=rmax, ngrid=ngrid, nz=nz, nphi=nphi,
                           lambda0=synth.LAMBDA0, slice_eloss=el)
    el_p = np.repeat(el, np.diff(off))
    sc_part = np.max(np.abs(want - el_p))
    assert sc_part > 1e-3 * np.max(np.abs(el))  # the space-charge part is not negligible
    # same fixed-point mode sums; FP64 rounding of the phases and sums
    assert np.max(np.abs(got - want)) < 1e-9 * sc_part, np.max(np.abs(got - want)) / sc_part
    sc.short_range(beam, GZ2)
    assert np.array_equal(beam.particle_ez(), got)
    for o in (sc, beam):
        o.close()


def test_short_range_off_and_limits(ctx):
    off, p = _bunched(2, 500, seed=3)
    beam = dev.BeamState(ctx, off, synth.GAMMA0)
    beam.upload(p)
    beam.set_current(np.array([1000.0, 1000.0]))
    off_solver = dev.EFieldSolver(ctx, 0.0, 50, 1, 0, synth.LAMBDA0)  # rmax 0: off
    assert not off_solver.has_short_range()
    off_solver.short_range(beam, GZ2)
    with pytest.raises(G4BError):
        beam.particle_ez()  # nothing was set
    with pytest.raises(G4BError):
        dev.EFieldSolver(ctx, 1.0, 1000, 4, 2, synth.LAMBDA0)  # 20 modes x 1000 cells
    for o in (off_solver, beam):
        o.close()


@pytest.mark.skipif(not refpy.available(), reason="oracle/_ref/libg4ref.so not built")
def test_push_with_a_per_particle_loss_three_ways(ctx):
    nslice = 3
    off, p = synth.beam(nslice, 2000, seed=43)
    ku2 = synth.KU ** 2
    st = synth.und_step(ax=1e-6, kx=0.5 * ku2, ky=0.5 * ku2, gradx=5.0)
    cells = synth.field(nslice, 101, 2e-4, seed=44, amplitude=5e10)
    fields = [dict(cells=cells, first=1, harm=1, gridmax=2e-4, xlambda=synth.LAMBDA0,
                   fc=synth.coupling())]
    rng = np.random.default_rng(45)
    pez = rng.normal(0.0, 2e-3, p["x"].size)
    ref = synth.copy_parts(p)
    refpy.beam_advance(off, st, fields, ref, particle_field=pez)
    ora = synth.copy_parts(p)
    orc.push(off, st, fields, ora, particle_ez=pez)
    beam = dev.BeamState(ctx, off, synth.GAMMA0)
    beam.upload(p)
    beam.set_eloss(np.array([1.0, 1.0, 1.0]))  # must be ignored while pez is set
    beam.set_particle_ez(pez)
    fs = dev.FieldState(ctx, nslice, 101, 2e-4, synth.LAMBDA0)
    fs.upload(cells)
    fs.first = 1
    beam.advance([fs], [synth.coupling()], st)
    got = beam.download()
    dg = ref["gamma"] - p["gamma"]
    # the per-particle loss matters at this size
    plain = synth.copy_parts(p)
    orc.push(off, st, fields, plain)
    assert np.max(np.abs((plain["gamma"] - p["gamma"]) - dg)) > 1e-3 * np.max(np.abs(dg))
    for name, q in (("oracle", ora), ("cuda", got)):
        assert np.max(np.abs((q["gamma"] - p["gamma"]) - dg)) < 1e-12 * np.max(np.abs(dg)), name
        # an ulp of theta (~1e-16 at theta of a few radians): the oracle's
        # compiler contracts some products into fused multiply-adds
        np.testing.assert_allclose(q["theta"], ref["theta"], rtol=1e-13, atol=1e-15,
                                   err_msg=name)
    # back to the slice loss
    beam.set_particle_ez(None)
    beam.set_eloss(None)
    beam.upload(p)
    beam.advance([fs], [synth.coupling()], st)
    back = beam.download()
    assert np.max(np.abs((back["gamma"] - p["gamma"]) - (plain["gamma"] - p["gamma"]))) < \
        1e-12 * np.max(np.abs(dg))
    for o in (fs, beam):
        o.close()


EFIELD_DECK = """
&setup
rootname = sc
lattice = sc.lat
beamline = CELL
lambda0 = 1.0e-10
gamma0 = 4000
delz = 0.1
npart = 2048
nbins = 4
seed = 5
&end
&time
slen = 8e-10
sample = 2
&end
&field
power = 1e3
dgrid = 2e-4
ngrid = 65
waist_size = 40e-6
&end
&beam
current = 4000
delgam = 0.5
ex = 0.3e-6
ey = 0.3e-6
betax = 5.0
betay = 5.0
&end
{efield}
&track
&end
"""

EFIELD_LAT = """
UND: UNDULATOR = { lambdau = 0.02, nwig = 50, aw = 1.2, helical = False };
CELL: LINE = { UND };
"""


def test_deck_with_space_charge_changes_the_energy_spread():
    from genesis4_cuda_port_b200 import host
    plain = host.Deck(EFIELD_DECK.format(efield=""), EFIELD_LAT).run()
    sc = host.Deck(EFIELD_DECK.format(efield="&efield\nrmax = 2.0\nngrid = 60\nnz = 2\n"
                                             "nphi = 1\n&end"), EFIELD_LAT).run()
    a, b = plain.beam["energyspread"], sc.beam["energyspread"]
    assert np.all(np.isfinite(b))
    np.testing.assert_array_equal(a[0], b[0])  # step 0: before any push
    assert np.max(np.abs(b[-1] - a[-1])) > 1e-6 * np.max(np.abs(a[-1]))
