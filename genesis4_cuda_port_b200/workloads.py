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

# the same cell three times over (1032 steps): long enough for the configs'
# beam at 0.1 um normalised emittance to reach the exponential regime
HIGH_GAIN_LAT = SASE_LAT + "FEL3: LINE = { 3*FEL };\n"


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
    periodic: bool = False
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


def steady_state_high_gain(npart=8192, ngrid=151, seed_power=1e3):
    """Steady-state FEL in the exponential regime: the steady-state beam at
    0.1 um normalised emittance over the cell three times (1032 steps); the
    1 kW seed grows by about 1e5 with the bunching still rising at the end."""
    return Workload(f"steady-state high gain 1 slice x {npart}, ngrid {ngrid}, eps_n 0.1 um, "
                    "3 x 344 steps", 1, npart, ngrid, shotnoise=False, seed_power=seed_power,
                    emit_n=0.1e-6, lattice=HIGH_GAIN_LAT, beamline="FEL3")


def sase_periodic_high_gain(nslice=64, npart=8192, ngrid=201):
    """Time-dependent SASE from shot noise in the exponential regime: the SASE
    beam at 0.1 um normalised emittance, slippage every step with periodic
    slices (radiation leaving the window re-enters at its tail, as inside a
    long flat-top bunch), 1032 steps; the power grows by about 5e4."""
    return Workload(f"periodic SASE high gain {nslice} slices x {npart}, ngrid {ngrid}, "
                    "eps_n 0.1 um, 3 x 344 steps", nslice, npart, ngrid, emit_n=0.1e-6,
                    periodic=True, lattice=HIGH_GAIN_LAT, beamline="FEL3")


WORKLOADS = {"steady": steady_state, "sase": sase, "sase_h3": large_sase_h3}


def _job(wl: Workload, **kw):
    from .host import Job
    j = Job()
    base = dict(nslice=1, npart=wl.npart, ngrid=wl.ngrid, nsteps=10 ** 6, shotnoise=1,
                time_run=0, seed=wl.seed, gridmax=wl.gridmax, gamma=wl.gamma0,
                delgam=wl.rel_spread * wl.gamma0, emit=wl.emit_n, beta=wl.beta,
                current=wl.current, seed_power=0.0, waist=wl.waist, taper=0.0)
    base.update(kw)
    for k, v in base.items():
        setattr(j, k, v)
    return j


def engine(wl: Workload, **kw):
    """Engine configuration of the shared SASE lattice at the workload's
    reference energy."""
    from .host import engine_config
    return engine_config(wl.lattice, wl.beamline, wl.delz, wl.gamma0, wl.lambda0, **kw)


def batched_scan(nruns=256, seed=1):
    """Steady-state scan: nruns single-slice runs with ngrid ~ U[101,301],
    npart ~ U[2048,32768] (multiple of 4), linear taper d(aw)/aw ~ U[0,2%],
    detuning dgamma/gamma ~ U[-5e-4,5e-4], seed power log-U[100 W, 10 kW];
    every run takes the whole lattice.  Returns (workload, jobs, params)."""
    wl = steady_state()
    rng = np.random.default_rng(seed)
    params = []
    jobs = []
    for i in range(nruns):
        p = dict(ngrid=int(rng.integers(101, 302)),
                 npart=int(rng.integers(2048 // 4, 32768 // 4 + 1)) * 4,
                 taper=float(rng.uniform(0.0, 0.02)),
                 detune=float(rng.uniform(-5e-4, 5e-4)),
                 seed_power=float(10 ** rng.uniform(2.0, 4.0)))
        params.append(p)
        jobs.append(_job(wl, ngrid=p["ngrid"], npart=p["npart"], taper=p["taper"],
                         gamma=wl.gamma0 * (1 + p["detune"]), seed_power=p["seed_power"],
                         shotnoise=0, seed=seed + i))
    return wl, jobs, params


def served_stream(nreq=2000, rate=200.0, seed=1):
    """Served stream: Poisson arrivals (rate per second) of runs with
    nslice ~ U{1..64}, ngrid ~ U[101,255], npart ~ U[2048,16384] (multiple of
    4), nsteps ~ U[110,330]; SASE from shot noise, slippage on for nslice > 1.
    Returns (workload, jobs, arrival times [s], params)."""
    wl = sase()
    rng = np.random.default_rng(seed)
    arrival = np.cumsum(rng.exponential(1.0 / rate, nreq))
    jobs, params = [], []
    for i in range(nreq):
        p = dict(nslice=int(rng.integers(1, 65)), ngrid=int(rng.integers(101, 256)),
                 npart=int(rng.integers(2048 // 4, 16384 // 4 + 1)) * 4,
                 nsteps=int(rng.integers(110, 331)))
        params.append(p)
        jobs.append(_job(wl, nslice=p["nslice"], ngrid=p["ngrid"], npart=p["npart"],
                         nsteps=p["nsteps"], time_run=int(p["nslice"] > 1), seed=seed + i))
    return wl, jobs, arrival, params


def lambda_res(lambdau, aw, gamma):
    return lambdau * (1 + aw * aw) / (2 * gamma * gamma)


def zr(w0, lam):
    return math.pi * w0 * w0 / lam
