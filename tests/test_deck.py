"""Input decks on the host (no GPU): namelist parsing, the &track switches,
slice count from &time, marker updates and the &lattice zmatch matching."""
import math

import numpy as np
import pytest

from genesis4_cuda_port_b200 import host
from genesis4_cuda_port_b200._lib import G4BError

LAT = """
D1: DRIFT = { l = 0.2 };
QF: QUADRUPOLE = { l = 0.1, k1 = 2.0 };
QD: QUADRUPOLE = { l = 0.1, k1 = -2.0 };
UND: UNDULATOR = { lambdau = 0.02, nwig = 50, aw = 1.8, helical = False };
M: MARKER = { dumpfield = 1 };
CELL: LINE = { UND, D1, QF, D1, UND, D1, QD, D1 };
BL: LINE = { 4*CELL, M };
"""


def deck(track="use_cuda = 1", time="slen = 3.0e-7\nsample = 4", extra_field="",
         beam="current = 2500\ndelgam = 1.5\nex = 0.5e-6\ney = 0.5e-6"):
    return f"""
&setup
rootname = t
lattice = t.lat
beamline = BL
lambda0 = 1.0e-10
gamma0 = 20000
delz = 0.1
npart = 512
nbins = 4
seed = 7
&end

&lattice
zmatch = 3.0
&end

&time
{time}
&end

&field
power = 1e4
dgrid = 1.5e-4
ngrid = 65
waist_size = 30e-6
&end
{extra_field}
&beam
{beam}
&end

&track
{track}
&end
"""


def test_deck_sizes_and_switches():
    d = host.Deck(deck(track="use_cuda = 1\nlow_memory_adisolver = true\noutput_step = 3"),
                  LAT)
    s = d.info()
    assert s["nslice"] == round(3.0e-7 / (4 * 1.0e-10))
    assert s["time_run"] == 1 and s["sample"] == 4.0
    assert s["low_memory"] == 1 and s["precision"] == 0
    assert s["ngrid"] == [65] and s["gridmax"] == [1.5e-4] and s["harm"] == [1]
    # per cell: 2 undulators of 1 m at delz 0.1 -> 10 steps each; 4 drifts of
    # 0.2 m -> 2 steps each; 2 quads -> 1 step each
    assert s["nstep"] == 4 * (2 * 10 + 4 * 2 + 2)
    assert math.isclose(s["zend"], 4 * 3.0, rel_tol=1e-12)
    assert s["nout"] == 1 + (s["nstep"] + 2) // 3
    assert s["current"] == 2500


def test_precision_and_harmonic_fields():
    d = host.Deck(deck(track="precision = mixed\nbunchharm = 3",
                       extra_field="&field\nharm = 3\nngrid = 65\ndgrid = 1.5e-4\n&end\n"), LAT)
    s = d.info()
    assert s["precision"] == 1 and s["bunchharm"] == 3
    assert s["nfield"] == 2 and s["harm"] == [1, 3]


def test_steady_state_without_time_group():
    text = deck().replace("&time\nslen = 3.0e-7\nsample = 4\n&end\n", "")
    s = host.Deck(text, LAT).info()
    assert s["nslice"] == 1 and s["time_run"] == 0


@pytest.mark.parametrize("bad, msg", [
    ("use_cuda = 1\nfoo = 2", "unknown"),
    ("use_cuda = 0", "use_cuda"),
    ("precision = fp16", "precision"),
    ("fft_fieldsolver = true\nprecision = mixed", "fft_fieldsolver"),
])
def test_track_errors(bad, msg):
    with pytest.raises(G4BError, match=msg):
        host.Deck(deck(track=bad), LAT)


def test_fft_solver_keys_are_accepted():
    """&track fft_fieldsolver / source_filter / xcut / ycut / sigmoid select the
    FFT field solver with its source filter (Track.cpp:95-105)."""
    d = host.Deck(deck(track="fft_fieldsolver = true\nsource_filter = true\nxcut = 0.3\n"
                             "ycut = 0.3\nsigmoid = 0.05"), LAT)
    assert d.info()["precision"] == 0


def _with_efield(text, efield):
    return text.replace("&track", f"&efield\n{efield}\n&end\n\n&track", 1)


def test_efield_group_is_accepted_for_the_fp64_form():
    """&efield rmax / ngrid / nz / nphi (upstream's short-range space charge)
    selects the device solver behind BeamSolverCUDA::initEField."""
    d = host.Deck(_with_efield(deck(), "rmax = 2.0\nngrid = 50\nnz = 2\nnphi = 1"), LAT)
    assert d.info()["precision"] == 0


@pytest.mark.parametrize("efield,track,msg", [
    ("rmax = 2\nnz = 1\nlongrange = true", "use_cuda = 1", "longrange"),
    ("rmax = 2\nnz = 1", "precision = mixed", "space charge"),
    ("rmax = 2\nnz = -1", "use_cuda = 1", "efield"),
    ("rmax = 2\nnz = 1\nfoo = 1", "use_cuda = 1", "unknown"),
])
def test_efield_errors(efield, track, msg):
    with pytest.raises(G4BError, match=msg):
        host.Deck(_with_efield(deck(track=track), efield), LAT)


def test_structure_errors():
    with pytest.raises(G4BError, match="not closed"):
        host.Deck("&setup\nlattice = a\n&beam\n&end\n", LAT)
    with pytest.raises(G4BError, match="needs"):
        host.Deck(deck().split("&track")[0], LAT)
    with pytest.raises(G4BError, match="unknown element"):
        host.Deck(deck().replace("beamline = BL", "beamline = NOPE"), LAT)


def test_zmatch_gives_the_periodic_twiss():
    """Transport (beta, alpha) through one cell with the thick-lens maps of
    the on-axis particle: the matched values come back."""
    d = host.Deck(deck(), LAT)
    s = d.info()
    lat = host.Lattice(LAT, "BL", 0.1, 20000.0, 1.0e-10)
    g0 = 20000.0
    for plane in (0, 1):
        M = np.eye(2)
        for st, z in zip(lat.steps, lat.z):
            if z > 3.0 + 1e-9:
                break
            aw = st.aw
            bp = math.sqrt(1 - (1 + aw * aw) / g0 ** 2)
            quad = st.qf * g0
            q = quad + st.kx * aw * aw / g0 / bp if plane == 0 else -quad + st.ky * aw * aw / g0 / bp
            k = q / math.sqrt(g0 * g0 - 1 - aw * aw)
            L = st.delz
            if k > 0:
                f = math.sqrt(k)
                A = np.array([[math.cos(f * L), math.sin(f * L) / f], [-f * math.sin(f * L), math.cos(f * L)]])
            elif k < 0:
                f = math.sqrt(-k)
                A = np.array([[math.cosh(f * L), math.sinh(f * L) / f], [f * math.sinh(f * L), math.cosh(f * L)]])
            else:
                A = np.array([[1.0, L], [0.0, 1.0]])
            M = A @ M
        beta = s["betax"] if plane == 0 else s["betay"]
        alpha = s["alphax"] if plane == 0 else s["alphay"]
        T = np.array([[beta, -alpha], [-alpha, (1 + alpha * alpha) / beta]])
        T2 = M @ T @ M.T
        np.testing.assert_allclose(T2, T, rtol=1e-9, atol=1e-9)
        assert beta > 0


def test_explicit_beam_twiss_overrides_zmatch():
    s = host.Deck(deck(beam="current = 2500\nbetax = 9.0\nalphax = 0.5"), LAT).info()
    assert s["betax"] == 9.0 and s["alphax"] == 0.5
    assert s["betay"] != 15.0  # still matched


def test_dump_markers_and_zstop():
    s = host.Deck(deck(track="field_dump_step = 10\nzstop = 1.3"), LAT).info()
    assert s["nstep"] == 4 * 30
    # steps end at 0.1, ..., 1.0 (undulator), 1.1, 1.2 (drift), 1.3 (quad)
    assert s["nrun"] == 13
    # the MARKER element at the end of BL sits after the last step
    lat = host.Lattice(LAT, "BL", 0.1, 20000.0, 1.0e-10)
    assert lat.marker[-1] & 2 and not any(m & 2 for m in lat.marker[:-1])
