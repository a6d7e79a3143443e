"""The short-range space-charge model of the oracle against closed forms.

Upstream GENESIS 1.3 v4's EFieldSolver (which the reference calls on the host,
src/Core/BeamSolverCUDA.cpp:523-547) is absent from the reference tree, so
the oracle's model is pinned here by the continuous problem instead:

* a uniform disk of radius a with a bunching b at the reference wavelength
  has, inside a grounded wall at R, the m = 0 solution
  u = S0/kappa^2 + A I0(kappa r) (r < a), B I0 + C K0 (a < r < R), u(R) = 0,
  S0 = b/(pi a^2);
* far inside a wide beam (kappa a >> 1) the field is the one-dimensional
  E_z = -2 I Z0/(k_s pi a^2) Im[b e^{i theta}];
* the radial solve of a higher azimuthal order converges at second order.
"""
import numpy as np
import pytest
from scipy import special

from oracle import pyoracle as orc


def _disk(nring, nper, a, theta):
    """Particles of uniform area density on a polar lattice inside r < a: ring
    k at r^2 = a^2 (k + 1/2)/nring, nper particles per ring (theta(n) gives
    their phases).  With a radial cell of width a/c and nring a multiple of
    c^2, every cell inside the disk holds exactly its area share."""
    k = np.arange(nring)
    r = a * np.sqrt((k + 0.5) / nring)
    phi = (np.arange(nper) + 0.5) * 2 * np.pi / nper
    rr = np.repeat(r, nper)
    pp = np.tile(phi, nring) + np.repeat(k * 0.618, nper)  # staggered rings
    n = rr.size
    th = np.asarray(theta(n), np.float64)
    z = np.zeros(n)
    return dict(x=rr * np.cos(pp), y=rr * np.sin(pp), px=z.copy(), py=z.copy(),
                gamma=np.full(n, 1e4), theta=th)


def _rmax_for(p, cell, ngrid):
    """rmax that puts the wall at ngrid cells of the given width."""
    return ngrid * cell / np.max(np.hypot(p["x"], p["y"]))


def _closed_form_m0(r, a, R, kappa, s0):
    """u(r) of (1/r (r u')' - kappa^2 u) = -s0 [r < a], u(R) = 0, regular at 0."""
    I0, I1 = special.i0, special.i1
    K0, K1 = special.k0, special.k1
    ka, kR = kappa * a, kappa * R
    # unknowns A, B, C: continuity of u and u' at a, u(R) = 0
    M = np.array([[I0(ka), -I0(ka), -K0(ka)],
                  [I1(ka), -I1(ka), K1(ka)],
                  [0.0, I0(kR), K0(kR)]])
    rhs = np.array([-1.0 / kappa ** 2, 0.0, 0.0])
    A, B, C = np.linalg.solve(M, rhs)
    kr = kappa * r
    inside = 1.0 / kappa ** 2 + A * I0(kr)
    outside = B * I0(kr) + C * special.k0(np.maximum(kr, 1e-300))
    return s0 * np.where(r < a, inside, outside)


@pytest.mark.parametrize("kappa_a,c", [(0.5, 20), (2.0, 20), (20.0, 80)])
def test_m0_mode_matches_the_closed_form_of_a_uniform_disk(kappa_a, c):
    a, lam = 20e-6, 1e-9
    ngrid = 3 * c                                   # cell a/c, wall at 3a
    kappa = kappa_a / a
    gz2 = (2 * np.pi / lam / kappa) ** 2
    # half the particles at theta = 0, half at pi/2 (in every ring): b = (1 - i)/2
    p = _disk(5 * c * c, 12, a, lambda n: np.where(np.arange(n) % 2 == 0, 0.0, np.pi / 2))
    n = p["x"].size
    ez, modes = orc.short_range(np.array([0, n]), p, np.array([1000.0]), gz2,
                                rmax=_rmax_for(p, a / c, ngrid), ngrid=ngrid, nz=1, nphi=0,
                                lambda0=lam, return_modes=True)
    md = modes[0]
    dr = md["dr"]
    assert abs(dr - a / c) < 1e-12 * a
    rc = (np.arange(ngrid) + 0.5) * dr
    b = (1 - 1j) / 2
    want = _closed_form_m0(rc, a, ngrid * dr, kappa, b / (np.pi * a ** 2))
    got = md["u"][(1, 0)]
    scale = np.max(np.abs(want))
    # second order in dr (kappa dr <= 1/4 here): below 5e-3
    assert np.max(np.abs(got - want)) < 5e-3 * scale, np.max(np.abs(got - want)) / scale
    assert np.all(np.isfinite(ez))


def test_wide_beam_field_is_the_one_dimensional_limit():
    a, lam, gz2, c = 20e-6, 1e-9, 1.0, 20
    ks = 2 * np.pi / lam
    assert ks * a > 1e5  # kappa a >> 1: one-dimensional inside the beam
    th0 = np.linspace(0, 2 * np.pi, 7)[:-1] + 0.1
    th0[0] += 0.4
    p = _disk(5 * c * c, 12, a, lambda n: th0[np.arange(n) % 6])
    n = p["x"].size
    cur = 500.0
    ez = orc.short_range(np.array([0, n]), p, np.array([cur]), gz2,
                         rmax=_rmax_for(p, a / c, 40), ngrid=40, nz=1, nphi=0, lambda0=lam)
    b = np.mean(np.exp(-1j * p["theta"]))
    assert abs(b) > 0.05
    ez_1d = -2 * cur * orc.VACIMP / (ks * np.pi * a ** 2) * np.imag(
        b * np.exp(1j * p["theta"])) / orc.EEV
    core = np.hypot(p["x"], p["y"]) < 0.9 * a
    np.testing.assert_allclose(ez[core], ez_1d[core], rtol=0,
                               atol=1e-6 * np.max(np.abs(ez_1d)))


def test_higher_azimuthal_order_converges_at_second_order():
    a, R, kdr_ref = 0.4, 1.0, 3.0  # lengths in units of R; kappa R = 3

    def solve(n, m):
        dr = R / n
        lo, hi = np.arange(n) * dr, np.arange(1, n + 1) * dr
        # exact cell-average of S = 1 on r < a (area fraction of each annulus)
        frac = np.clip((np.minimum(hi, a) ** 2 - np.minimum(lo, a) ** 2) /
                       (hi ** 2 - lo ** 2), 0, 1)
        rc = (np.arange(n) + 0.5) * dr
        # acc/(2 pi N) = S * r dr in cell units (dr = 1): S r_c
        acc = frac * 2 * np.pi * (rc / dr) * dr ** 2
        u = orc.sc_solve(acc.astype(complex), 1, m, (kdr_ref * dr) ** 2)
        return rc, u.real

    probe = np.array([0.2, 0.6, 0.8])
    vals = []
    for n in (50, 100, 200, 400):
        rc, u = solve(n, 2)
        vals.append(np.interp(probe, rc, u))
    d1 = np.abs(vals[1] - vals[0])
    d2 = np.abs(vals[2] - vals[1])
    d3 = np.abs(vals[3] - vals[2])
    assert np.all(vals[-1] > 0)
    assert np.all(d2 < d1 / 2.5) and np.all(d3 < d2 / 2.5), (d1, d2, d3)


def test_no_current_or_a_point_beam_gives_the_slice_loss():
    p = _disk(10, 4, 1e-5, lambda n: np.zeros(n))
    n = p["x"].size
    el = np.array([0.3, -0.2])
    off = np.array([0, n // 2, n])
    ez = orc.short_range(off, p, np.array([0.0, 100.0]), 1e4, rmax=2, ngrid=20, nz=2, nphi=1,
                         lambda0=1e-9, slice_eloss=el)
    assert np.all(ez[: n // 2] == el[0])
    q = {k: v.copy() for k, v in p.items()}
    q["x"][:] = 1e-6
    q["y"][:] = 0.0
    ez = orc.short_range(off, q, np.array([100.0, 100.0]), 1e4, rmax=2, ngrid=20, nz=2,
                         nphi=1, lambda0=1e-9, slice_eloss=el)
    assert np.all(ez[: n // 2] == el[0]) and np.all(ez[n // 2:] == el[1])


@pytest.mark.parametrize("nphi", [0, 2])
def test_fully_bunched_beam_has_no_field_on_its_bunch(nphi):
    """All particles at one phase: the field at that phase is zero (odd in theta)."""
    p = _disk(200, 8, 1e-5, lambda n: np.full(n, 0.7))
    n = p["x"].size
    ez = orc.short_range(np.array([0, n]), p, np.array([800.0]), 1e6, rmax=2, ngrid=50,
                         nz=3, nphi=nphi, lambda0=1e-9)
    assert np.max(np.abs(ez)) < 1e-12
