"""Output and dump files of a deck run, and a run resumed from its dumps.

A marker after the first undulator cell dumps the beam and the field
(ControlCUDA::applyMarker, src/Core/ControlCUDA.cpp:131-146); a second deck
that imports those dumps (&importbeam / &importfield) and runs the rest of
the beamline must reproduce the first run's records from that point on and
its final field, bit for bit (the FP64 drop-in form).  The run's output file
holds the same records as the result object."""
import numpy as np
import pytest

from genesis4_cuda_port_b200 import host

pytestmark = pytest.mark.gpu

LAT = """
D1: DRIFT = { l = 0.2 };
QF: QUADRUPOLE = { l = 0.1, k1 = 2.0 };
QD: QUADRUPOLE = { l = 0.1, k1 = -2.0 };
UND: UNDULATOR = { lambdau = 0.02, nwig = 30, aw = 1.8, helical = False };
M: MARKER = { dumpbeam = 1, dumpfield = 1 };
CELL: LINE = { UND, D1, QF, D1, UND, D1, QD, D1 };
TWO: LINE = { CELL, M, CELL };
"""


def _deck(beamline, extra="", precision="fp64", outdir="out"):
    return f"""
&setup
rootname = run
lattice = g.lat
beamline = {beamline}
lambda0 = 1.0e-10
gamma0 = 20000
delz = 0.1
npart = 512
nbins = 4
seed = 5
outputdir = {outdir}
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
betax = 10.0
betay = 10.0
&end
{extra}
&track
precision = {precision}
&end
"""


def test_dump_and_resume_reproduce_the_run(tmp_path):
    (tmp_path / "out").mkdir()
    full = host.Deck(_deck("TWO"), LAT, str(tmp_path)).run()
    cell_steps = host.Lattice(LAT, "CELL", 0.1, 20000, 1e-10).nstep
    par = tmp_path / "out" / f"run.{cell_steps}.par.g4"
    fld = tmp_path / "out" / f"run.{cell_steps}.fld.g4"
    assert par.exists() and fld.exists()
    dump = host.read_g4ds(par)
    assert dump["slicecount"][0] == 4 and dump["slice000001/gamma"].shape == (512,)
    (tmp_path / "out2").mkdir()
    imports = (f"&importbeam\nfile = {par}\n&end\n&importfield\nfile = {fld}\n"
               "harmonic = 1\n&end\n")
    rest = host.Deck(_deck("CELL", imports, outdir="out2"), LAT, str(tmp_path)).run()
    k = cell_steps  # record k of the full run is the state after the first cell
    assert rest.nz == full.nz - k
    for key in ("power", "intensity-nearfield", "xsize"):
        assert np.array_equal(rest.field[0][key], full.field[0][key][k:]), key
    for key in ("energy", "bunching", "xposition"):
        assert np.array_equal(rest.beam[key], full.beam[key][k:]), key
    f_full, first_full = full.final_field(0)
    f_rest, first_rest = rest.final_field(0)
    ns = f_full.shape[0]
    # the resumed run starts at first = 0 in beam order: compare in beam order
    roll = lambda c, first: c[[(s + first) % ns for s in range(ns)]]  # noqa: E731
    assert np.array_equal(roll(f_rest, first_rest), roll(f_full, first_full))


def test_output_file_holds_the_records(tmp_path):
    res = host.Deck(_deck("CELL", outdir="."), LAT, str(tmp_path)).run()
    path = res.output_file
    assert path.endswith("run.out.g4")
    d = host.read_g4ds(path)
    assert d["Meta/nslice"][0] == res.nslice
    np.testing.assert_array_equal(d["Lattice/zplot"], res.z)
    for key, v in res.beam.items():
        assert np.array_equal(d["Beam/" + key], v), key
    for key, v in res.field[0].items():
        assert np.array_equal(d["Field/" + key], v), key
    assert d["Lattice/aw"].shape == d["Lattice/z"].shape


def test_mixed_run_writes_dumps_at_markers(tmp_path):
    (tmp_path / "out").mkdir()
    res = host.Deck(_deck("TWO", precision="mixed"), LAT, str(tmp_path)).run()
    cell_steps = host.Lattice(LAT, "CELL", 0.1, 20000, 1e-10).nstep
    d = host.read_g4ds(tmp_path / "out" / f"run.{cell_steps}.par.g4")
    f = host.read_g4ds(tmp_path / "out" / f"run.{cell_steps}.fld.g4")
    assert np.all(np.isfinite(d["slice000004/theta"]))
    power = sum(np.sum(f[f"slice{s + 1:06d}/field-real"] ** 2 +
                       f[f"slice{s + 1:06d}/field-imag"] ** 2) for s in range(4))
    # the dump's field is the field of record cell_steps (summed power)
    dgrid = 2 * 1.5e-4 / 64
    scl = dgrid * 510998.95 / (2 * np.pi / 1e-10)
    np.testing.assert_allclose(power * scl * scl / 376.73031346177,
                               res.field[0]["power"][cell_steps].sum(), rtol=1e-6)
    assert res.output_file.endswith("run.out.g4")
