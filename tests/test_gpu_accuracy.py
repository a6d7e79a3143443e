"""The mixed-precision form where its errors can grow: two workloads in the
exponential-gain regime, each run through the FP64 oracle, the FP64 drop-in
and the fused mixed-precision run on identical seeded inputs.

* steady state: 1 slice x 8192, ngrid 151, 1 kW seed, 0.1 um normalised
  emittance, the lattice cell three times (1032 steps); power gain ~1e5;
* periodic time-dependent SASE: 64 slices x 8192 from shot noise, ngrid 201,
  slippage every step with periodic slices, same beam and lattice; power gain
  ~5e4.

Gates (the mixed form's): P(z) within 1e-3 relative before saturation and
per-slice |b1|(z) within 1e-3 absolute of the FP64 oracle; the on-axis
spectrum at the end (|FFT over slices of the centre-cell field|^2) within
1e-2 of its peak; the final energy spread within 1e-3 relative.  The FP64
drop-in stays within 1e-9 of the oracle throughout.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from genesis4_cuda_port_b200 import workloads
from oracle import pyoracle as orc

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402

pytestmark = pytest.mark.gpu

SPECTRUM_TOL = 1e-2
SPREAD_TOL = 1e-3


def oracle_history(wl, off, parts, cells, lat, nstep):
    p = {k: v.copy() for k, v in parts.items()}
    f = dict(cells=cells.copy(), gridmax=wl.gridmax, xlambda=wl.lambda0, fc=0.0, first=0,
             accuslip=0.0)
    cur = np.full(wl.nslice, wl.current)
    pz, b1 = [], []
    for i in range(nstep):
        f["fc"] = lat.fc(i, 1)
        orc.step(off, cur, lat.steps[i], wl.lambda0, lat.slip[i], wl.sample, wl.nslice > 1,
                 wl.periodic, [f], p)
        fs, cen = orc.diag_field(f["cells"], f["first"])
        bs, bre, bim = orc.diag_beam(off, p, 1, False)
        pz.append(fs[:, 0].sum())
        b1.append(np.hypot(bre[:, 0], bim[:, 0]) / np.maximum(bs[:, 12], 1))
    return {"pz": np.array(pz), "b1": np.array(b1), "center": cen[:, 0] + 1j * cen[:, 1],
            "gsum": bs[:, 0].sum(), "g2sum": bs[:, 1].sum(), "count": bs[:, 12].sum()}


@pytest.fixture(scope="module")
def ctx():
    c = dev.Context(0)
    yield c
    c.synchronize()


@pytest.mark.parametrize("make,min_gain", [(workloads.steady_state_high_gain, 1e2),
                                           (workloads.sase_periodic_high_gain, 1e3)],
                         ids=["steady", "sase_periodic"])
def test_mixed_form_within_its_gates_at_high_gain(ctx, make, min_gain):
    wl = make()
    off, parts = wl.make_beam()
    cells = wl.make_field()
    lat = wl.make_lattice()
    n = lat.nstep
    assert n == 1032
    ref = oracle_history(wl, off, parts, cells, lat, n)
    fp64 = bench.fp64_history(ctx, wl, off, parts, cells, lat, n)
    mix = bench.mixed_history(ctx, wl, off, parts, cells, lat, n)
    m64 = bench.accuracy_metrics(fp64, ref)
    mm = bench.accuracy_metrics(mix, ref)
    print(wl.name, "fp64:", m64, "mixed:", mm)
    assert mm["power_gain"] > min_gain, mm
    assert m64["pz_rel_err_max"] < 1e-9 and m64["b1_abs_err_max"] < 1e-9, m64
    assert mm["pz_rel_err_max"] < bench.ACCURACY_GATES["pz_rel"], mm
    assert mm["b1_abs_err_max"] < bench.ACCURACY_GATES["b1_abs"], mm
    assert mm["energy_spread_rel_err"] < SPREAD_TOL, mm
    if wl.nslice > 1:
        assert mm["spectrum_rel_err"] < SPECTRUM_TOL, mm
