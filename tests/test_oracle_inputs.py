"""The oracle's own input builders (quiet-start loader, lattice expansion,
Gaussian seed) against the host layer's: the CPU baseline arm builds its
inputs from the oracle alone, so they must be the same inputs."""
import numpy as np
import pytest

from genesis4_cuda_port_b200 import host, workloads
from oracle import pyoracle as orc
from oracle import refpy


@pytest.mark.parametrize("wl", [workloads.sase(nslice=5), workloads.steady_state(npart=1024)],
                         ids=["sase", "steady"])
def test_loader_bit_identical(wl):
    sp = wl.beam_spec()
    spec = orc.BeamSpec(**{k: getattr(sp, k) for k, _ in orc.BeamSpec._fields_})
    cur = np.linspace(wl.current, 0.5 * wl.current, wl.nslice)
    off_h, ph = host.load_beam(sp, cur)
    off_o, po = orc.load_beam(spec, cur)
    assert np.array_equal(off_h, off_o)
    for k in ph:
        assert np.array_equal(ph[k], po[k]), k


def test_lattice_identical():
    wl = workloads.sase(nslice=2)
    a = wl.make_lattice()
    b = orc.Lattice(wl.lattice, wl.beamline, wl.delz, wl.gamma0, wl.lambda0)
    assert a.nstep == b.nstep == 344
    for i in range(a.nstep):
        assert np.array_equal(refpy.step_to_array(a.steps[i]), refpy.step_to_array(b.steps[i]))
        assert a.slip[i] == b.slip[i]
        for h in (1, 3):
            assert a.fc(i, h) == pytest.approx(b.fc(i, h), rel=1e-15, abs=0)


def test_gaussian_seed_matches():
    a = host.gaussian_field(151, 2e-4, 1.16e-10, 1e3, 30e-6)
    b = orc.gaussian_field(151, 2e-4, 1.16e-10, 1e3, 30e-6)
    np.testing.assert_allclose(b, a, rtol=1e-14, atol=1e-14 * np.max(np.abs(a)))
