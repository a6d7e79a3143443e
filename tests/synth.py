"""Seeded synthetic inputs with the shapes and value ranges of the benchmark
configurations (planar undulator aw=1.0, lambda_u=15 mm, gamma=11357, 3 kA,
0.4 um normalised emittance at beta=15 m), scaled down for fast tests."""
from __future__ import annotations

import math

import numpy as np
from scipy.special import jv

from genesis4_cuda_port_b200._lib import Step

LAMBDA_U = 0.015
AW = 1.0
GAMMA0 = 11357.0
KU = 2 * math.pi / LAMBDA_U
LAMBDA0 = LAMBDA_U * (1 + AW ** 2) / (2 * GAMMA0 ** 2)
CURRENT = 3000.0
EPS_N = 0.4e-6
BETA = 15.0


def coupling(aw: float = AW, harm: int = 1) -> float:
    """Planar coupling factor aw * JJ_h (odd h)."""
    xi = harm * aw * aw / (2 * (1 + aw * aw))
    m = (harm - 1) // 2
    return aw * (-1) ** m * (jv(m, xi) - jv(m + 1, xi))


def und_step(delz=LAMBDA_U, aw=AW, **kw) -> Step:
    base = dict(delz=delz, aw=aw, ax=0.0, ay=0.0, kx=0.0, ky=KU * KU, gradx=0.0,
                grady=0.0, ku=KU, gamma_ref=GAMMA0, autophase=0.0, qf=0.0, dqx=0.0,
                dqy=0.0, cx=0.0, cy=0.0, chic_angle=0.0, chic_lb=0.0, chic_ld=0.0,
                chic_lt=0.0, in_undulator=1, reserved=0)
    base.update(kw)
    return Step(**base)


def drift_step(delz=0.1, qf=0.0, **kw) -> Step:
    return und_step(delz=delz, aw=0.0, ky=0.0, ku=0.0, qf=qf, in_undulator=0, **kw)


def beam(nslice: int, npart, seed: int = 1, sigma_x: float | None = None,
         energy_spread: float = 1e-4, ragged: bool = False):
    """Gaussian beam, slice-contiguous; npart per slice (or a list)."""
    rng = np.random.default_rng(seed)
    if np.isscalar(npart):
        counts = [int(npart)] * nslice
        if ragged:
            counts = [int(npart * (0.5 + rng.random())) for _ in range(nslice)]
            counts[0] = max(counts[0], 1)
            if nslice > 2:
                counts[1] = 0  # an empty slice
    else:
        counts = list(npart)
    off = np.zeros(nslice + 1, np.int64)
    off[1:] = np.cumsum(counts)
    n = int(off[-1])
    eps = EPS_N / GAMMA0
    sx = sigma_x if sigma_x is not None else math.sqrt(eps * BETA)
    spx = GAMMA0 * math.sqrt(eps / BETA)
    parts = {
        "x": rng.normal(0, sx, n),
        "y": rng.normal(0, sx, n),
        "px": rng.normal(0, spx, n),
        "py": rng.normal(0, spx, n),
        "gamma": GAMMA0 * (1 + energy_spread * rng.normal(0, 1, n)),
        "theta": rng.uniform(0, 2 * math.pi, n),
    }
    return off, parts


def field(nslice: int, ngrid: int, gridmax: float, seed: int = 2,
          amplitude: float = 1e13, waist: float = 30e-6, noise: float = 0.3):
    """Gaussian mode plus seeded complex noise, complex128 [S, n, n]."""
    rng = np.random.default_rng(seed)
    x = np.linspace(-gridmax, gridmax, ngrid)
    X, Y = np.meshgrid(x, x)
    g = np.exp(-(X * X + Y * Y) / waist ** 2)
    out = np.empty((nslice, ngrid, ngrid), np.complex128)
    for s in range(nslice):
        ph = rng.uniform(0, 2 * math.pi)
        nz = rng.normal(size=(ngrid, ngrid)) + 1j * rng.normal(size=(ngrid, ngrid))
        out[s] = amplitude * (g * np.exp(1j * ph) + noise * g * nz)
    return out


def copy_parts(p):
    return {k: v.copy() for k, v in p.items()}


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.max(np.abs(b))
    if scale == 0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / scale)
