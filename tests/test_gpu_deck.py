"""A whole deck through the host classes on the GPU: Gencore::run with the
FP64 CUDA classes against the oracle stepping the same loaded beam, field and
lattice; the fused mixed-precision run of the same deck against the FP64 one."""
import math

import numpy as np
import pytest

from genesis4_cuda_port_b200 import host
from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu

EEV, VACIMP = 510998.95, 376.73031346177

LAT = """
D1: DRIFT = { l = 0.2 };
QF: QUADRUPOLE = { l = 0.1, k1 = 2.0 };
QD: QUADRUPOLE = { l = 0.1, k1 = -2.0 };
C: CHICANE = { l = 0.1, lb = 0.02, delay = 2e-10 };
UND: UNDULATOR = { lambdau = 0.02, nwig = 50, aw = 1.8, helical = False };
CELL: LINE = { UND, D1, QF, C, D1, UND, D1, QD, D1 };
"""


def _deck(precision):
    return f"""
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
&lattice
zmatch = 3.1
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
precision = {precision}
bunchharm = 2
&end
"""


def _oracle(deck):
    s = deck.info()
    lam = s["lambda0"]
    ns = s["nslice"]
    spec = host.BeamSpec(nslice=ns, npart=s["npart"], nbins=4, shotnoise=1, seed=11,
                         gamma0=s["gamma0"], delgam=1.0, ex=0.5e-6, ey=0.5e-6,
                         betax=s["betax"], betay=s["betay"], alphax=s["alphax"],
                         alphay=s["alphay"], xcenter=0.0, ycenter=0.0, pxcenter=0.0,
                         pycenter=0.0, reflength=lam, slicelength=lam * s["sample"])
    cur = np.full(ns, s["current"])
    off, p = host.load_beam(spec, cur)
    plane = host.gaussian_field(65, 1.5e-4, lam, 1e5, 30e-6)
    f = dict(cells=np.broadcast_to(plane, (ns, 65, 65)).copy(), gridmax=1.5e-4, xlambda=lam,
             harm=1, fc=0.0, first=0, accuslip=0.0)
    lat = host.Lattice(LAT, "CELL", 0.1, s["gamma0"], lam)
    dgrid = 2 * 1.5e-4 / 64
    scl = dgrid * EEV / (2 * math.pi / lam)
    power, energy = [], []

    def rec():
        st, _ = orc.diag_field(f["cells"], f["first"])
        power.append(st[:, 0] * scl * scl / VACIMP)
        bs, _, _ = orc.diag_beam(off, p, 1)
        energy.append(bs[:, 0] / bs[:, 12])

    rec()
    for i in range(s["nrun"]):
        f["fc"] = lat.fc(i, 1)
        orc.step(off, cur, lat.steps[i], lam, lat.slip[i], s["sample"], True, False, [f], p)
        rec()
    return np.array(power), np.array(energy)


def test_fp64_deck_matches_the_oracle():
    deck = host.Deck(_deck("fp64"), LAT)
    res = deck.run()
    s = deck.info()
    assert res.nz == s["nrun"] + 1 and res.nslice == s["nslice"] == 4
    pw, en = _oracle(deck)
    got_p = res.field[0]["power"]
    assert abs(pw[-1].sum() - pw[0].sum()) > 1e-3 * pw[0].sum()
    np.testing.assert_allclose(got_p, pw, rtol=1e-9, atol=1e-12 * np.max(pw))
    np.testing.assert_allclose(res.beam["energy"], en, rtol=1e-12)
    assert res.beam["bunching2"].shape == (res.nz, 4)
    assert np.all(np.isfinite(res.field[0]["Global/energy"]))
    np.testing.assert_allclose(res.z[-1], s["zend"])


def test_mixed_deck_tracks_the_fp64_deck():
    r64 = host.Deck(_deck("fp64"), LAT).run()
    rmx = host.Deck(_deck("mixed"), LAT).run()
    p64 = r64.field[0]["power"].sum(axis=1)
    pmx = rmx.field[0]["power"].sum(axis=1)
    assert np.max(np.abs(pmx - p64) / p64) < 1e-3
    b64, bmx = r64.beam["bunching"], rmx.beam["bunching"]
    assert np.max(np.abs(bmx - b64)) < 1e-3
    c64, first64 = r64.final_field(0)
    cmx, firstmx = rmx.final_field(0)
    assert first64 == firstmx
