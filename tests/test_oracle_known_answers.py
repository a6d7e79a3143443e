"""Known-answer checks that pin the FP64 oracle (no GPU).

The reference ships no golden vectors, so the oracle's restatement of each
phase is checked against closed-form physics instead: Gaussian-beam free
propagation and unitarity for the ADI step, constant-rate phase advance for a
zero-field push, drift and thick-quadrupole transfer maps for the transverse
step, the slippage index model, and vanishing bunching of a quiet-start
phase set.
"""
import math

import numpy as np
import pytest

from oracle import pyoracle as orc
from tests import synth


def _gauss_field(n, gridmax, w0, amp=1.0):
    x = np.linspace(-gridmax, gridmax, n)
    X, Y = np.meshgrid(x, x)
    return (amp * np.exp(-(X * X + Y * Y) / w0 ** 2)).astype(np.complex128)[None]


def _rms_size(stats, dgrid):
    p, x1, x2 = stats[0, 0], stats[0, 1], stats[0, 2]
    return math.sqrt(x2 / p - (x1 / p) ** 2) * dgrid


def test_adi_coefficients_solve_the_tridiagonal():
    n, delz, dgrid, xks = 17, 0.01, 2e-6, 5.4e10
    c, cbet, cwet, r = orc.adi_coeffs(n, delz, dgrid, xks)
    assert r == pytest.approx(0.25 * delz / (xks * dgrid * dgrid))
    A = np.zeros((n, n), complex)
    for i in range(n):
        A[i, i] = 1 + 2j * r
        if i > 0:
            A[i, i - 1] = -1j * r
        if i < n - 1:
            A[i, i + 1] = -1j * r
    rhs = np.random.default_rng(0).normal(size=n) + 0j
    # Thomas with the oracle's factors
    y = np.empty(n, complex)
    y[0] = rhs[0] * cbet[0]
    for k in range(1, n):
        y[k] = (rhs[k] - c[k] * y[k - 1]) * cbet[k]
    for k in range(n - 2, -1, -1):
        y[k] = y[k] - cwet[k + 1] * y[k + 1]
    np.testing.assert_allclose(A @ y, rhs, atol=1e-13)


def test_adi_gaussian_beam_free_propagation():
    lam, w0 = 1e-7, 30e-6
    zr = math.pi * w0 * w0 / lam
    n, gridmax = 161, 200e-6
    dgrid = 2 * gridmax / (n - 1)
    f = _gauss_field(n, gridmax, w0)
    nstep = 40
    delz = zr / nstep
    step = synth.drift_step(delz=delz)
    off = np.array([0, 0], np.int64)
    parts = {k: np.zeros(0) for k in ("x", "y", "gamma", "theta")}
    s0, _ = orc.diag_field(f, 0)
    for _ in range(nstep):
        orc.adi_advance(f, harm=1, gridmax=gridmax, xks=2 * np.pi / lam, delz=delz, fc=0.0,
                        enabled=True, step=step, off=off, current=np.zeros(1), parts=parts)
    s1, _ = orc.diag_field(f, 0)
    # intensity rms size is w/2; w(zR) = sqrt(2) w0
    assert _rms_size(s0, dgrid) == pytest.approx(w0 / 2, rel=2e-3)
    assert _rms_size(s1, dgrid) == pytest.approx(math.sqrt(2) * w0 / 2, rel=5e-3)
    # Crank-Nicolson ADI with a symmetric second difference is unitary
    assert s1[0, 0] == pytest.approx(s0[0, 0], rel=1e-12)


def test_zero_field_push_advances_phase_at_constant_rate():
    off, parts = synth.beam(2, 300, seed=3)
    step = synth.und_step(autophase=0.25)
    n = 33
    zero = np.zeros((2, n, n), np.complex128)
    fields = [dict(cells=zero, gridmax=200e-6, xlambda=synth.LAMBDA0, fc=synth.coupling())]
    before = synth.copy_parts(parts)
    orc.push(off, step, fields, parts)
    g = before["gamma"]
    ks = 2 * np.pi / synth.LAMBDA0
    btpar = 1 + before["px"] ** 2 + before["py"] ** 2 + step.aw ** 2 * (
        1 + 0.5 * step.ky * before["y"] ** 2) ** 2
    b0 = np.sqrt(1 - btpar / g ** 2)
    expect = before["theta"] + step.autophase + step.delz * (ks * (1 - 1 / b0) + step.ku)
    np.testing.assert_allclose(parts["gamma"], g, rtol=0, atol=0)
    np.testing.assert_allclose(parts["theta"], expect, rtol=1e-12, atol=1e-9)


def test_drift_and_quadrupole_transfer_maps():
    off, parts = synth.beam(1, 500, seed=4)
    p0 = synth.copy_parts(parts)
    st = synth.drift_step(delz=0.3)
    orc.track(parts, st, 0.3, last=False)
    gz = np.sqrt(p0["gamma"] ** 2 - 1 - p0["px"] ** 2 - p0["py"] ** 2)
    np.testing.assert_allclose(parts["x"], p0["x"] + p0["px"] * 0.3 / gz, rtol=1e-14)
    np.testing.assert_allclose(parts["px"], p0["px"], rtol=0)
    # thick focusing quad in x, defocusing in y
    parts = synth.copy_parts(p0)
    k1, L = 1.5, 0.1
    st = synth.drift_step(delz=L, qf=k1)
    orc.track(parts, st, L, last=False)
    s = k1 * synth.GAMMA0
    fx = np.sqrt(s / gz)
    xe = np.cos(fx * L) * p0["x"] + np.sin(fx * L) / fx * p0["px"] / gz
    pxe = -np.sin(fx * L) * fx * p0["x"] * gz + np.cos(fx * L) * p0["px"]
    fy = np.sqrt(s / gz)
    ye = np.cosh(fy * L) * p0["y"] + np.sinh(fy * L) / fy * p0["py"] / gz
    np.testing.assert_allclose(parts["x"], xe, rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(parts["px"], pxe, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(parts["y"], ye, rtol=1e-12, atol=1e-18)


def test_r56_phase_shift():
    off, parts = synth.beam(1, 200, seed=5)
    p0 = synth.copy_parts(parts)
    st = synth.drift_step(delz=0.1, chic_angle=1e-3, chic_lb=0.02, chic_ld=0.01, chic_lt=0.1)
    orc.r56(parts, st, synth.LAMBDA0)
    a, lb, ld = 1e-3, 0.02, 0.01
    r56 = (4 * lb / math.sin(a) * (1 - a / math.tan(a)) + 2 * ld * math.tan(a) / math.cos(a)) * a
    r56 *= 2 * math.pi / synth.LAMBDA0 / synth.GAMMA0
    np.testing.assert_allclose(parts["theta"], p0["theta"] + r56 * (p0["gamma"] - synth.GAMMA0),
                               rtol=1e-13)


def test_slippage_index_model():
    S, n = 5, 4
    f = np.arange(S * n * n, dtype=float).reshape(S, n, n).astype(np.complex128) + 1
    acc, first, ns = orc.slippage(f, 1.0, 1.0, True, False, 0.0, 0)
    assert (ns, first) == (1, 4) and acc == pytest.approx(0.0)
    assert np.all(f[4] == 0) and np.all(f[:4] != 0)
    acc, first, ns = orc.slippage(f, 2.5, 1.0, True, False, acc, first)
    assert ns == 2 and first == 2 and acc == pytest.approx(0.5)
    acc, first, ns = orc.slippage(f, -1.0, 1.0, True, False, acc, first)
    assert ns == 0 and first == 2 and acc == pytest.approx(-0.5)  # |acc| < 0.8
    acc, first, ns = orc.slippage(f, -0.5, 1.0, True, False, acc, first)
    assert ns == 1 and first == 3 and acc == pytest.approx(0.0)
    assert np.all(f[2] == 0)  # negative slip zeroes the old first plane
    g = f.copy()
    acc, first, ns = orc.slippage(g, 3.0, 1.0, False, False, 0.0, 0)
    assert ns == 0 and np.array_equal(g, f)  # steady state: no-op


def test_quiet_start_bunching_vanishes():
    nb = 4
    base = np.random.default_rng(6).uniform(0, 2 * np.pi, 256)
    theta = (base[:, None] + 2 * np.pi * np.arange(nb)[None] / nb).reshape(-1)
    off = np.array([0, theta.size], np.int64)
    z = np.zeros(theta.size)
    parts = dict(x=z, y=z.copy(), px=z.copy(), py=z.copy(), gamma=z + 1e4, theta=theta)
    stats, bre, bim = orc.diag_beam(off, parts, nharm=3)
    assert abs(bre[0, 0]) / theta.size < 1e-14 and abs(bim[0, 0]) / theta.size < 1e-14
    assert abs(bre[0, 2]) / theta.size < 1e-13
    assert stats[0, 12] == theta.size


def test_uniform_field_push_is_classic_rk4():
    """In a uniform field the gather returns the same value everywhere, so
    the step is one classic RK4 step of (gamma, theta) with a frozen
    coupling: compare with a numpy RK4 of the ODE of
    src/Core/BeamSolverCUDA.cpp:146-223 (Genesis's accumulator form is the
    same scheme)."""
    off, parts = synth.beam(2, 200, seed=8)
    step = synth.und_step(autophase=0.1)
    n, gridmax = 17, 200e-6
    u0 = 4e13 * np.exp(0.7j)
    cells = np.full((2, n, n), u0, np.complex128)
    fc = synth.coupling()
    ks = 2 * np.pi / synth.LAMBDA0
    fields = [dict(cells=cells, gridmax=gridmax, xlambda=synth.LAMBDA0, fc=fc)]
    before = synth.copy_parts(parts)
    orc.push(off, step, fields, parts)
    x, y, px, py = before["x"], before["y"], before["px"], before["py"]
    awloc = 1 + 0.5 * (step.kx * x * x + step.ky * y * y)
    btpar = 1 + px * px + py * py + step.aw ** 2 * awloc ** 2
    rpart = (fc / ks) * awloc * np.conj(u0)

    def f(g, th):
        c = rpart * np.exp(-1j * th)
        b0 = np.sqrt(1 - (btpar - 2 / ks * c.real) / (g * g))
        return c.imag / b0 / g, ks * (1 - 1 / b0) + step.ku

    g, th = before["gamma"].copy(), before["theta"] + step.autophase
    h = step.delz
    k1 = f(g, th)
    k2 = f(g + h / 2 * k1[0], th + h / 2 * k1[1])
    k3 = f(g + h / 2 * k2[0], th + h / 2 * k2[1])
    k4 = f(g + h * k3[0], th + h * k3[1])
    g1 = g + h / 6 * (k1[0] + 2 * k2[0] + 2 * k3[0] + k4[0])
    th1 = th + h / 6 * (k1[1] + 2 * k2[1] + 2 * k3[1] + k4[1])
    inside = (np.abs(x) < gridmax * (1 - 2 / (n - 1))) & (np.abs(y) < gridmax * (1 - 2 / (n - 1)))
    assert inside.mean() > 0.9
    assert np.max(np.abs(g1 - before["gamma"])[inside]) > 1e-5  # the field does work
    np.testing.assert_allclose(parts["gamma"][inside], g1[inside], rtol=1e-13)
    np.testing.assert_allclose(parts["theta"][inside], th1[inside], rtol=0, atol=1e-9)


def test_diagnostic_sums_match_numpy():
    off, parts = synth.beam(3, 400, seed=9, ragged=True)
    stats, bre, bim = orc.diag_beam(off, parts, nharm=2)
    for s in range(3):
        sl = slice(off[s], off[s + 1])
        x, px, g, th = parts["x"][sl], parts["px"][sl], parts["gamma"][sl], parts["theta"][sl]
        ref = [g.sum(), (g * g).sum(), x.sum(), (x * x).sum()]
        np.testing.assert_allclose(stats[s, :4], ref, rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(stats[s, 10], (x * px).sum(), rtol=1e-12, atol=1e-300)
        assert stats[s, 12] == off[s + 1] - off[s]
        np.testing.assert_allclose(bre[s, 1], np.cos(2 * th).sum(), rtol=1e-10, atol=1e-10)
        np.testing.assert_allclose(bim[s, 0], np.sin(th).sum(), rtol=1e-10, atol=1e-10)
    cells = synth.field(2, 21, 100e-6, seed=10)
    fs, cen = orc.diag_field(cells, 1)
    for s0 in range(2):
        s = (2 + s0 - 1) % 2
        w = np.abs(cells[s0]) ** 2
        d = np.arange(21) - 10.0
        np.testing.assert_allclose(fs[s, 0], w.sum(), rtol=1e-12)
        np.testing.assert_allclose(fs[s, 1], (w * d[None, :]).sum(), rtol=1e-10, atol=1e-6 * w.sum())
        np.testing.assert_allclose(fs[s, 4], (w * d[:, None] ** 2).sum(), rtol=1e-12)
        np.testing.assert_allclose(fs[s, 5] + 1j * fs[s, 6], cells[s0].sum(), rtol=1e-12)
        np.testing.assert_allclose(cen[s], [cells[s0, 10, 10].real, cells[s0, 10, 10].imag])
