"""Benchmark workloads: the FEL configurations the throughput is quoted on,
as .lat beamlines plus beam/field setups.  All inputs are synthetic and
seeded (quiet start + shot noise from the host loader)."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# planar undulator rms aw = 1.0, lambda_u = 15 mm, 3 x 110-period sections
# separated by 0.1 m FODO quadrupoles (k1 = +-1.5 1/m^2)
SASE_LAT = """
UND: UNDULATOR = { lambdau = 0.015, nwig = 110, aw = 1.0, helical = false };
QF: QUADRUPOLE = { l = 0.1, k1 = 1.5 };
QD: QUADRUPOLE = { l = 0.1, k1 = -1.5 };
FEL: LINE = { UND, QF, UND, QD, UND };
"""


@dataclass
class Workload:
    name: str
    nslice: int
    npart: int
    ngrid: int
    gridmax: float = 2e-4
    gamma0: float = 11357.0
    aw: float = 1.0
    lambdau: float = 0.015
    rel_spread: float = 1e-4
    emit_n: float = 0.4e-6
    beta: float = 15.0
    current: float = 3000.0
    nbins: int = 4
    shotnoise: bool = True
    seed_power: float = 0.0
    waist: float = 30e-6
    seed: int = 1
    sample: float = 1.0
    harmonics: tuple = (1,)
    lattice: str = SASE_LAT
    beamline: str = "FEL"
    extra: dict = field(default_factory=dict)

    @property
    def lambda0(self) -> float:
        """Resonant wavelength of the beam's mean particle: the on-axis
        lambda_u (1 + aw^2) / (2 gamma^2) corrected for the matched beam's mean
        transverse momentum <px^2 + py^2> = 2 gamma eps_n / beta and the planar
        undulator's natural-focusing field rise aw^2 ku^2 <y^2>."""
        ku = 2 * math.pi / self.lambdau
        p2 = 2 * self.gamma0 * self.emit_n / self.beta
        foc = self.aw ** 2 * ku * ku * self.emit_n * self.beta / self.gamma0
        return self.lambdau * (1 + self.aw ** 2 + p2 + foc) / (2 * self.gamma0 ** 2)

    @property
    def delz(self) -> float:
        return self.lambdau

    def beam_spec(self):
        from .host import BeamSpec
        return BeamSpec(nslice=self.nslice, npart=self.npart, nbins=self.nbins,
                        shotnoise=int(self.shotnoise), seed=self.seed, gamma0=self.gamma0,
                        delgam=self.rel_spread * self.gamma0, ex=self.emit_n,
                        ey=self.emit_n, betax=self.beta, betay=self.beta, alphax=0.0,
                        alphay=0.0, xcenter=0.0, ycenter=0.0, pxcenter=0.0,
                        pycenter=0.0, reflength=self.lambda0,
                        slicelength=self.lambda0 * self.sample)

    def make_beam(self):
        from .host import load_beam
        return load_beam(self.beam_spec(), np.full(self.nslice, self.current))

    def make_field(self, harm: int = 1):
        from .host import gaussian_field
        plane = gaussian_field(self.ngrid, self.gridmax, self.lambda0 / harm,
                               self.seed_power if harm == 1 else 0.0, self.waist)
        return np.broadcast_to(plane, (self.nslice, self.ngrid, self.ngrid)).copy()

    def make_lattice(self):
        from .host import Lattice
        return Lattice(self.lattice, self.beamline, self.delz, self.gamma0, self.lambda0)

    def alg_bytes_fp64(self) -> dict:
        """Compulsory bytes per step of each FP64 drop-in kernel."""
        N = self.nslice * self.npart
        C = self.nslice * self.ngrid ** 2
        return {
            "track": 72 * N,          # read x,y,px,py,gamma; write x,y,px,py
            "push": 64 * N,           # read 6 doubles, write gamma, theta
            "deposit": 32 * N + 16 * C,
            "adi_x": 48 * C,          # read u, S; write R'
            "adi_y": 32 * C,          # read R'; write u
            "diag_beam": 48 * N,
            "diag_field": 16 * C,
        }


def steady_state(npart=8192, ngrid=151, seed_power=1e3):
    """Steady-state single-slice FEL (FP64, CPU-runnable)."""
    return Workload("steady-state 1 slice x 8192, ngrid 151, 330+14 steps", 1, npart,
                    ngrid, shotnoise=False, seed_power=seed_power)


def sase(nslice=1024, npart=8192, ngrid=201):
    """Time-dependent SASE: 1024 slices at lambda0 spacing, flat-top 3 kA."""
    return Workload(f"time-dependent SASE {nslice} slices x {npart}, ngrid {ngrid}",
                    nslice, npart, ngrid)


def large_sase_h3(nslice=8192, npart=16384, ngrid=255):
    """Large SASE with fundamental and 3rd-harmonic fields."""
    return Workload(f"SASE {nslice} x {npart}, ngrid {ngrid}, h=1 and h=3", nslice,
                    npart, ngrid, harmonics=(1, 3))


WORKLOADS = {"steady": steady_state, "sase": sase, "sase_h3": large_sase_h3}


def lambda_res(lambdau, aw, gamma):
    return lambdau * (1 + aw * aw) / (2 * gamma * gamma)


def zr(w0, lam):
    return math.pi * w0 * w0 / lam
