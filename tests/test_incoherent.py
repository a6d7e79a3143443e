"""The incoherent-synchrotron-radiation model of the oracle.

Upstream GENESIS 1.3 v4's Incoherent class (which the reference calls on the
host, src/Core/Beam.cpp:126) is absent from the reference tree; the oracle
restates the device model of g4b_beam_incoherent and is pinned here by the
published pieces it is made of: the Philox4x32-10 known-answer vectors of its
authors (Salmon et al., SC 2011), the moments of the Box-Muller normals, and
the closed-form rates (mean loss (2/3) r_e k_u^2 aw^2 gamma^2; spread growth
(14/15) lambdabar_c r_e k_u^3 K^2 F(K) gamma^4).
"""
import numpy as np
import pytest

from oracle import pyoracle as orc


@pytest.mark.parametrize("ctr,key,want", [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
])
def test_philox_known_answers(ctr, key, want):
    assert orc.philox4x32_10(ctr, key) == want


def test_rates_closed_form():
    aw, ku = 1.0, 2 * np.pi / 0.015
    loss, spread = orc.isr_rates(aw, ku)
    assert loss == pytest.approx(2 / 3 * 2.8179403262e-15 * ku ** 2)
    K = np.sqrt(2)
    F = 1.42 * K + 1 / (1 + 1.5 * K + 0.95 * K * K)
    assert spread == pytest.approx(14 / 15 * 3.8615926796e-13 * 2.8179403262e-15 * ku ** 3 * 2 * F)
    assert orc.isr_rates(0.0, ku) == (0.0, 0.0)
    lh, sh = orc.isr_rates(aw, ku, helical=True)
    assert lh == loss and sh != spread


def test_step_moments_and_determinism():
    n = 1 << 20
    g0 = 11357.0
    aw, ku, delz = 1.0, 2 * np.pi / 0.015, 1000.0  # a long step: measurable moments
    gamma = np.full(n, g0)
    orc.incoherent(gamma, aw=aw, ku=ku, delz=delz, seed=7, counter=3)
    lr, sr = orc.isr_rates(aw, ku)
    dg = gamma - g0
    assert np.mean(dg) == pytest.approx(-lr * delz * g0 ** 2, rel=5e-3)
    assert np.var(dg) == pytest.approx(sr * delz * g0 ** 4, rel=1e-2)
    # the normals: mean 0, variance 1, fourth moment 3, no gross tail excess
    z = (dg + lr * delz * g0 ** 2) / np.sqrt(sr * delz * g0 ** 4)
    assert abs(np.mean(z)) < 5e-3 and abs(np.var(z) - 1) < 5e-3
    assert abs(np.mean(z ** 4) - 3) < 0.05 and np.max(np.abs(z)) < 7
    again = np.full(n, g0)
    orc.incoherent(again, aw=aw, ku=ku, delz=delz, seed=7, counter=3)
    assert np.array_equal(again, gamma)
    other = np.full(n, g0)
    orc.incoherent(other, aw=aw, ku=ku, delz=delz, seed=7, counter=4)
    assert not np.array_equal(other, gamma)
    only_loss = np.full(4, g0)
    orc.incoherent(only_loss, aw=aw, ku=ku, delz=delz, spread=False)
    assert np.all(only_loss == g0 - lr * delz * g0 * g0)
