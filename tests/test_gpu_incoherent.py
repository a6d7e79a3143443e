"""Incoherent synchrotron radiation on the device against the oracle.

g4b_beam_incoherent draws the same Philox4x32-10 normals as the oracle
(pinned by the generator's known-answer vectors in tests/test_incoherent.py);
the energy changes agree to rounding of log/cos and the moments follow the
closed-form rates.
"""
import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from oracle import pyoracle as orc
from tests import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = dev.Context(0)
    yield c
    c.synchronize()


@pytest.mark.parametrize("helical", [False, True])
def test_incoherent_matches_the_oracle(ctx, helical):
    off, p = synth.beam(5, 40000, seed=21, ragged=True)
    st = synth.und_step(aw=1.3)
    delz = 50.0  # a long step: the noise is far above rounding
    beam = dev.BeamState(ctx, off, synth.GAMMA0)
    beam.upload(p)
    beam.incoherent(st, delz, helical=helical, seed=12345, counter=77)
    got = beam.download()["gamma"]
    want = p["gamma"].copy()
    orc.incoherent(want, aw=1.3, ku=synth.KU, delz=delz, helical=helical, seed=12345,
                   counter=77)
    dg = want - p["gamma"]
    assert np.max(np.abs(dg)) > 1e-6
    assert np.max(np.abs((got - p["gamma"]) - dg)) < 1e-12 * np.max(np.abs(dg))
    beam.close()


def test_incoherent_moments_and_switches(ctx):
    n = 1 << 20
    off = np.array([0, n // 2, n])
    g0 = synth.GAMMA0
    p = {k: np.zeros(n) for k in ("x", "y", "px", "py", "theta")}
    p["gamma"] = np.full(n, g0)
    beam = dev.BeamState(ctx, off, g0)
    beam.upload(p)
    st = synth.und_step(aw=1.0)
    delz = 1000.0
    beam.incoherent(st, delz, seed=3, counter=1)
    dg = beam.download()["gamma"] - g0
    loss, spread = orc.isr_rates(1.0, synth.KU)
    assert np.mean(dg) == pytest.approx(-loss * delz * g0 ** 2, rel=5e-3)
    assert np.var(dg) == pytest.approx(spread * delz * g0 ** 4, rel=1e-2)
    # a drift step does nothing; loss alone is deterministic
    beam.upload(p)
    beam.incoherent(synth.drift_step(), delz, seed=3, counter=2)
    assert np.all(beam.download()["gamma"] == g0)
    beam.incoherent(st, delz, spread=False, seed=3, counter=3)
    lone = beam.download()["gamma"]
    assert np.all(lone == lone[0]) and lone[0] < g0
    beam.close()
