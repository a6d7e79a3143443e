"""ctypes binding of the FP64 CPU oracle (oracle/g4_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by the test suite, the smoke check and the
benchmark's CPU-baseline leg, always as the checker or the timed CPU
baseline, never as the product path.  PARITY UNPINNED against upstream
GENESIS 1.3 v4 (see g4_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBPATH = HERE / "_build" / "libg4oracle.so"

dp = C.POINTER(C.c_double)
i64p = C.POINTER(C.c_int64)
ip = C.POINTER(C.c_int)


def build() -> Path:
    """Compile the oracle with the committed Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIBPATH


def _step_type():
    from genesis4_cuda_port_b200._lib import Step
    return Step


class FieldView(C.Structure):
    _fields_ = [("first", C.c_int), ("ngrid", C.c_int), ("nslice", C.c_int),
                ("harm", C.c_int), ("gridmax", C.c_double),
                ("dgrid", C.c_double), ("xks", C.c_double), ("fc", C.c_double),
                ("cells", dp)]


class FieldState(C.Structure):
    _fields_ = [("ngrid", C.c_int), ("harm", C.c_int), ("first", C.c_int),
                ("enabled", C.c_int), ("gridmax", C.c_double),
                ("xlambda", C.c_double), ("fc", C.c_double),
                ("accuslip", C.c_double), ("cells", dp)]


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIBPATH.exists():
        build()
    lib = C.CDLL(str(LIBPATH))
    Step = _step_type()
    sp = C.POINTER(Step)
    lib.g4o_adi_coeffs.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double,
                                   dp, dp, dp, dp]
    lib.g4o_slice_scl.argtypes = [C.c_int, i64p, dp, C.c_double, C.c_double,
                                  C.c_double, C.c_double, dp]
    lib.g4o_deposit.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                C.c_double, sp, i64p, dp, dp, dp, dp, dp, dp]
    lib.g4o_adi_advance.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_int, sp, i64p, dp, dp, dp,
                                    dp, dp, dp, dp]
    lib.g4o_track.argtypes = [C.c_int64, sp, C.c_double, C.c_int, dp, dp, dp, dp, dp]
    lib.g4o_r56.argtypes = [C.c_int64, sp, C.c_double, dp, dp]
    lib.g4o_push.argtypes = [C.c_int, i64p, sp, C.POINTER(FieldView), C.c_int,
                             dp, dp, dp, dp, dp, dp, dp]
    lib.g4o_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    lib.g4o_philox4x32_10.restype = None
    lib.g4o_incoherent.argtypes = [C.c_int64, dp, C.c_double, C.c_double, C.c_uint64,
                                   C.c_uint64]
    lib.g4o_incoherent.restype = None
    lib.g4o_push_ez.argtypes = [C.c_int, i64p, sp, C.POINTER(FieldView), C.c_int,
                                dp, dp, dp, dp, dp, dp, dp, dp]
    lib.g4o_slippage.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_int, C.c_int, dp, ip, dp]
    lib.g4o_slippage.restype = C.c_int
    lib.g4o_diag_beam.argtypes = [C.c_int, i64p, C.c_int, C.c_int, dp, dp, dp,
                                  dp, dp, dp, dp, dp, dp]
    lib.g4o_diag_field.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp]
    lib.g4o_step.argtypes = [C.c_int, i64p, dp, dp, sp, C.c_double, C.c_double,
                             C.c_double, C.c_int, C.c_int,
                             C.POINTER(FieldState), C.c_int, dp, dp, dp, dp,
                             dp, dp, dp]
    lib.g4o_num_threads.restype = C.c_int
    lib.g4o_set_num_threads.argtypes = [C.c_int]
    _lib = lib
    return lib


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(dp)


def _off(off):
    off = np.ascontiguousarray(off, dtype=np.int64)
    return off, off.ctypes.data_as(i64p)


def num_threads() -> int:
    return int(load().g4o_num_threads())


def set_num_threads(n: int) -> None:
    load().g4o_set_num_threads(int(n))


def adi_coeffs(n, delz, dgrid, xks):
    c = np.empty(2 * n)
    cbet = np.empty(2 * n)
    cwet = np.empty(2 * n)
    r = C.c_double()
    load().g4o_adi_coeffs(n, delz, dgrid, xks, _d(c), _d(cbet), _d(cwet), C.byref(r))
    cv = lambda a: a.view(np.complex128)  # noqa: E731
    return cv(c), cv(cbet), cv(cwet), r.value


def adi_advance(field, *, harm, gridmax, xks, delz, fc, enabled, step, off,
                current, parts, first=0):
    """FieldSolverADICUDA::advance on a complex128 [S, n, n] array in place."""
    S, n, _ = field.shape
    flat = field.reshape(-1).view(np.float64)
    work = np.empty(4 * S * n * n)
    off, offp = _off(off)
    cur = np.ascontiguousarray(current, dtype=np.float64)
    load().g4o_adi_advance(S, n, first, harm, gridmax, xks, delz, fc, int(enabled),
                           C.byref(step), offp, _d(cur), _d(parts["x"]),
                           _d(parts["y"]), _d(parts["gamma"]), _d(parts["theta"]),
                           _d(flat), _d(work))


def deposit(*, nslice, ngrid, first, harm, gridmax, step, off, parts, scl):
    src = np.zeros((nslice, ngrid, ngrid), np.complex128)
    dgrid = 2 * gridmax / (ngrid - 1)
    off, offp = _off(off)
    load().g4o_deposit(nslice, ngrid, first, harm, gridmax, dgrid, C.byref(step),
                       offp, _d(parts["x"]), _d(parts["y"]), _d(parts["gamma"]),
                       _d(parts["theta"]), _d(np.ascontiguousarray(scl, np.float64)),
                       _d(src.reshape(-1).view(np.float64)))
    return src


def slice_scl(off, current, fc, xks, dgrid, delz):
    off, offp = _off(off)
    out = np.empty(len(off) - 1)
    load().g4o_slice_scl(len(off) - 1, offp, _d(np.ascontiguousarray(current, np.float64)),
                         fc, xks, dgrid, delz, _d(out))
    return out


def track(parts, step, delz, last):
    n = parts["x"].size
    load().g4o_track(n, C.byref(step), delz, int(last), _d(parts["x"]), _d(parts["y"]),
                     _d(parts["px"]), _d(parts["py"]), _d(parts["gamma"]))


def r56(parts, step, lambda0):
    load().g4o_r56(parts["x"].size, C.byref(step), lambda0, _d(parts["gamma"]),
                   _d(parts["theta"]))


def push(off, step, fields, parts, slice_eloss=None, particle_ez=None):
    """fields: list of dicts(cells complex128 [S,n,n], first, harm, gridmax, xlambda, fc);
    particle_ez: per-particle loss read in place of slice_eloss."""
    off, offp = _off(off)
    nf = len(fields)
    views = (FieldView * nf)()
    keep = []
    for i, f in enumerate(fields):
        cells = np.ascontiguousarray(f["cells"], dtype=np.complex128)
        keep.append(cells)
        S, n, _ = cells.shape
        views[i].first = f.get("first", 0)
        views[i].ngrid = n
        views[i].nslice = S
        views[i].harm = f.get("harm", 1)
        views[i].gridmax = f["gridmax"]
        views[i].dgrid = 2 * f["gridmax"] / (n - 1)
        views[i].xks = 2 * np.pi / f["xlambda"]
        views[i].fc = f["fc"]
        views[i].cells = cells.reshape(-1).view(np.float64).ctypes.data_as(dp)
    el = None if slice_eloss is None else np.ascontiguousarray(slice_eloss, np.float64)
    pe = None if particle_ez is None else np.ascontiguousarray(particle_ez, np.float64)
    load().g4o_push_ez(len(off) - 1, offp, C.byref(step), views, nf, _d(el), _d(pe),
                       _d(parts["x"]), _d(parts["y"]), _d(parts["px"]), _d(parts["py"]),
                       _d(parts["gamma"]), _d(parts["theta"]))


def slippage(field, shift, sample, time_run, periodic, accuslip, first):
    S, n, _ = field.shape
    acc = C.c_double(accuslip)
    fst = C.c_int(first)
    ns = load().g4o_slippage(S, n, shift, sample, int(time_run), int(periodic),
                             C.byref(acc), C.byref(fst), _d(field.reshape(-1).view(np.float64)))
    return acc.value, fst.value, ns


def diag_beam(off, parts, nharm=1, need_aux=True):
    off, offp = _off(off)
    S = len(off) - 1
    stats = np.empty((S, 23))
    bre = np.empty((S, nharm))
    bim = np.empty((S, nharm))
    load().g4o_diag_beam(S, offp, nharm, int(need_aux), _d(parts["x"]), _d(parts["y"]),
                         _d(parts["px"]), _d(parts["py"]), _d(parts["gamma"]),
                         _d(parts["theta"]), _d(stats.reshape(-1)), _d(bre.reshape(-1)),
                         _d(bim.reshape(-1)))
    return stats, bre, bim


def diag_field(field, first):
    S, n, _ = field.shape
    stats = np.empty((S, 7))
    center = np.empty((S, 2))
    load().g4o_diag_field(S, n, first, _d(field.reshape(-1).view(np.float64)),
                          _d(stats.reshape(-1)), _d(center.reshape(-1)))
    return stats, center


def step(off, current, step_params, lambda0, slippage_shift, sample, time_run,
         periodic, fields, parts, slice_eloss=None):
    """One Gencore main-loop step; fields: list of dicts updated in place
    (cells complex128 [S,n,n], harm, gridmax, xlambda, fc, first, accuslip,
    enabled)."""
    off, offp = _off(off)
    S = len(off) - 1
    nf = len(fields)
    fs = (FieldState * nf)()
    nmax = 0
    for i, f in enumerate(fields):
        cells = f["cells"]
        assert cells.dtype == np.complex128 and cells.flags["C_CONTIGUOUS"]
        n = cells.shape[1]
        nmax = max(nmax, n)
        fs[i].ngrid = n
        fs[i].harm = f.get("harm", 1)
        fs[i].first = f.get("first", 0)
        fs[i].enabled = int(f.get("enabled", True))
        fs[i].gridmax = f["gridmax"]
        fs[i].xlambda = f["xlambda"]
        fs[i].fc = f["fc"]
        fs[i].accuslip = f.get("accuslip", 0.0)
        fs[i].cells = cells.reshape(-1).view(np.float64).ctypes.data_as(dp)
    work = np.empty(4 * S * nmax * nmax)
    el = None if slice_eloss is None else np.ascontiguousarray(slice_eloss, np.float64)
    load().g4o_step(S, offp, _d(np.ascontiguousarray(current, np.float64)), _d(el),
                    C.byref(step_params), lambda0, slippage_shift, sample, int(time_run),
                    int(periodic), fs, nf, _d(parts["x"]), _d(parts["y"]), _d(parts["px"]),
                    _d(parts["py"]), _d(parts["gamma"]), _d(parts["theta"]), _d(work))
    for i, f in enumerate(fields):
        f["first"] = fs[i].first
        f["accuslip"] = fs[i].accuslip


# ---- FFT field solver ---------------------------------------------------------

def fft_propagator(n, dgrid, xks, xc=0.0, yc=0.0, sig=0.0):
    """Spectral phase table and source filter of FieldSolverFFTCUDA::init
    (src/Core/FieldSolverFFTCUDA.cpp:246-293), in FFT index order: the
    transverse wavenumber of grid offset d = i - (n-1)/2 sits at index
    (i + (n+1)/2) mod n.  Returns (k2 [n,n], sigmoid [n,n] or None)."""
    dk = 4.0 * np.arcsin(1.0) / (n * dgrid)
    shift = -0.5 * (n - 1)
    d = np.arange(n) + shift
    idx = (np.arange(n) + (n + 1) // 2) % n
    k2 = np.empty((n, n))
    dy, dx = np.meshgrid(d, d, indexing="ij")
    k2[np.ix_(idx, idx)] = -(dx * dx + dy * dy) * dk * dk / 2.0 / xks
    if not (xc > 0 and yc > 0 and sig > 0):
        return k2, None
    sg = np.empty((n, n))
    x = dx / n / xc
    y = dy / n / yc
    r = (np.sqrt(x * x + y * y) - 1) / sig
    sg[np.ix_(idx, idx)] = 1.0 / (1 + np.exp(r))
    return k2, sg


def fft_advance(field, *, harm, gridmax, xks, delz, fc, enabled, step, off, current,
                parts, first=0, xc=0.0, yc=0.0, sig=0.0):
    """FieldSolverFFTCUDA::advance (src/Core/FieldSolverFFTCUDA.cpp:325-483) on
    a complex128 [S, n, n] array in place: the same source as the ADI solver
    (deposited by g4o_deposit), forward 2-D transforms of field and source,
    u' = u*exp(i*k2*delz) + 2*filter*S in Fourier space, inverse transform
    divided by n*n."""
    S, n, _ = field.shape
    dgrid = 2 * gridmax / (n - 1)
    k2, sg = fft_propagator(n, dgrid, xks, xc, yc, sig)
    spec = np.fft.fft2(field, axes=(1, 2))
    spec *= np.exp(1j * k2 * delz)[None]
    do_source = bool(step.in_undulator) and enabled and harm % 2 == 1
    off64 = np.ascontiguousarray(off, np.int64)
    if do_source and off64[-1] > 0:
        scl = slice_scl(off64, current, fc, xks, dgrid, delz)
        src = deposit(nslice=S, ngrid=n, first=first, harm=harm, gridmax=gridmax,
                      step=step, off=off64, parts=parts, scl=scl)
        ssp = np.fft.fft2(src, axes=(1, 2))
        if sg is not None:
            ssp *= sg[None]
        spec += 2.0 * ssp
    field[...] = np.fft.ifft2(spec, axes=(1, 2))


# ---- diagnostic records ---------------------------------------------------------

VACIMP = 376.73031346177
EEV = 510998.95


def beam_records(stats, bre, bim, current, *, eloss=None, long_esc=None, first_output=True):
    """Per-slice and global beam records from the per-slice sums, as
    DiagnosticCUDA::calcBeam derives them (src/Core/DiagnosticCUDA.cpp:517-628)
    with every output switched on; first_output adds the current and Twiss
    records written on output step 0."""
    S = stats.shape[0]
    nharm = bre.shape[1]
    cnt = stats[:, 12]
    norm = np.where(cnt > 0, 1.0 / np.where(cnt > 0, cnt, 1.0), 1.0)
    m = stats[:, :12] * norm[:, None]
    g1, g2, x1, x2, y1, y2, px1, px2, py1, py2, xpx, ypy = m.T
    sq = lambda v: np.sqrt(np.abs(v))  # noqa: E731
    out = dict(energy=g1, energyspread=sq(g2 - g1 * g1), xposition=x1, xsize=sq(x2 - x1 * x1),
               yposition=y1, ysize=sq(y2 - y1 * y1), pxposition=px1, pyposition=py1)
    for h in range(nharm):
        br, bi = bre[:, h] * norm, bim[:, h] * norm
        out["bunching" if h == 0 else f"bunching{h + 1}"] = np.hypot(br, bi)
        out["bunchingphase" if h == 0 else f"bunchingphase{h + 1}"] = np.arctan2(bi, br)
    el = np.zeros(S) if eloss is None else np.asarray(eloss, float)
    le = np.zeros(S) if long_esc is None else np.asarray(long_esc, float)
    out.update(efield=el + le, wakefield=el, LSCfield=le, SSCfield=np.zeros(S))
    for k, j in [("xmin", 13), ("xmax", 14), ("pxmin", 15), ("pxmax", 16), ("ymin", 17),
                 ("ymax", 18), ("pymin", 19), ("pymax", 20), ("emin", 21), ("emax", 22)]:
        out[k] = stats[:, j].copy()
    cur = np.asarray(current, float)
    out["current"] = cur.copy()
    if first_output:
        ex = np.sqrt(np.abs((x2 - x1 * x1) * (px2 - px1 * px1) - (xpx - x1 * px1) ** 2))
        ey = np.sqrt(np.abs((y2 - y1 * y1) * (py2 - py1 * py1) - (ypy - y1 * py1) ** 2))
        safe = lambda v: np.where(v > 0, v, 1.0)  # noqa: E731
        out.update(emitx=ex, emity=ey,
                   betax=np.where(ex > 0, (x2 - x1 * x1) / safe(ex) * g1, 0.0),
                   betay=np.where(ey > 0, (y2 - y1 * y1) / safe(ey) * g1, 0.0),
                   alphax=np.where(ex > 0, -(xpx - x1 * px1) / safe(ex), 0.0),
                   alphay=np.where(ey > 0, -(ypy - y1 * py1) / safe(ey), 0.0))
    gc = cur.sum()
    gn = 1.0 / gc if gc > 0 else 1.0
    gg1, gg2 = (cur * g1).sum() * gn, (cur * g2).sum() * gn
    gx1, gx2 = (cur * x1).sum() * gn, (cur * x2).sum() * gn
    gy1, gy2 = (cur * y1).sum() * gn, (cur * y2).sum() * gn
    out.update({"Global/energy": np.array([gg1]),
                "Global/energyspread": np.array([np.sqrt(abs(gg2 - gg1 * gg1))]),
                "Global/xposition": np.array([gx1]),
                "Global/xsize": np.array([np.sqrt(abs(gx2 - gx1 * gx1))]),
                "Global/yposition": np.array([gy1]),
                "Global/ysize": np.array([np.sqrt(abs(gy2 - gy1 * gy1))])})
    return out


def field_records(stats, center, *, ngrid, gridmax, xlambda, slicelength):
    """Per-slice and global field records from the per-slice sums (indexed by
    beam slice), as DiagnosticCUDA::calcField derives them
    (src/Core/DiagnosticCUDA.cpp:680-799), every output switched on."""
    S = stats.shape[0]
    dgrid = 2 * gridmax / (ngrid - 1)
    ks = 4.0 * np.arcsin(1.0) / xlambda
    scl = dgrid * EEV / ks
    p = stats[:, 0]
    x1, x2, y1, y2 = (stats[:, i].copy() for i in (1, 2, 3, 4))
    g = dict(pow=p.sum(), x1=x1.sum(), x2=x2.sum(), y1=y1.sum(), y2=y2.sum())
    pos = p > 0
    for v in (x1, x2, y1, y2):
        v[pos] /= p[pos]
    x2 = np.sqrt(np.abs(x2 - x1 * x1))
    y2 = np.sqrt(np.abs(y2 - y1 * y1))
    cre, cim = center[:, 0], center[:, 1]
    inten = cre * cre + cim * cim
    ff = (stats[:, 5] ** 2 + stats[:, 6] ** 2) * dgrid * dgrid
    out = {"power": p * scl * scl / VACIMP, "xposition": x1 * dgrid, "xsize": x2 * dgrid,
           "yposition": y1 * dgrid, "ysize": y2 * dgrid,
           "intensity-nearfield": inten * EEV * EEV / ks / ks / VACIMP,
           "phase-nearfield": np.arctan2(cim, cre), "intensity-farfield": ff,
           "phase-farfield": np.arctan2(stats[:, 6], stats[:, 5])}
    norm = 1.0 / g["pow"] if g["pow"] > 0 else 1.0
    gx1, gx2, gy1, gy2 = g["x1"] * norm, g["x2"] * norm, g["y1"] * norm, g["y2"] * norm
    out.update({
        "Global/energy": np.array([g["pow"] * scl * scl / VACIMP * slicelength / 299792458.0]),
        "Global/xposition": np.array([gx1 * dgrid]),
        "Global/xsize": np.array([np.sqrt(abs(gx2 - gx1 * gx1)) * dgrid]),
        "Global/yposition": np.array([gy1 * dgrid]),
        "Global/ysize": np.array([np.sqrt(abs(gy2 - gy1 * gy1)) * dgrid]),
        "Global/intensity-nearfield": np.array([inten.sum() / S * EEV * EEV / ks / ks / VACIMP]),
        "Global/intensity-farfield": np.array([ff.sum() / S]),
        "dgrid": np.array([gridmax]), "gridspacing": np.array([dgrid]),
        "ngrid": np.array([float(ngrid)])})
    return out


# ---- beam loading ---------------------------------------------------------------

class BeamSpec(C.Structure):
    """Mirror of g4o_beam_spec (oracle/g4_oracle.h); same fields as the host
    layer's g4h_beam_spec."""
    _fields_ = [("nslice", C.c_int), ("npart", C.c_int), ("nbins", C.c_int),
                ("shotnoise", C.c_int), ("seed", C.c_uint64), ("gamma0", C.c_double),
                ("delgam", C.c_double), ("ex", C.c_double), ("ey", C.c_double),
                ("betax", C.c_double), ("betay", C.c_double), ("alphax", C.c_double),
                ("alphay", C.c_double), ("xcenter", C.c_double), ("ycenter", C.c_double),
                ("pxcenter", C.c_double), ("pycenter", C.c_double),
                ("reflength", C.c_double), ("slicelength", C.c_double)]


def load_beam(spec: BeamSpec, current):
    """Quiet-start beam (g4o_load_beam): (int64 offsets, dict of arrays)."""
    lib = load()
    lib.g4o_load_beam.argtypes = [C.POINTER(BeamSpec), dp, dp, dp, dp, dp, dp, dp, i64p]
    lib.g4o_load_beam.restype = C.c_int
    n = spec.nslice * spec.npart
    parts = {k: np.empty(n) for k in ("x", "y", "px", "py", "gamma", "theta")}
    off = np.empty(spec.nslice + 1, np.int64)
    cur = np.ascontiguousarray(current, np.float64)
    rc = lib.g4o_load_beam(C.byref(spec), _d(cur), *[_d(parts[k]) for k in
                                                     ("x", "y", "px", "py", "gamma", "theta")],
                           off.ctypes.data_as(i64p))
    if rc:
        raise ValueError("g4o_load_beam: npart must be a multiple of nbins")
    return off, parts


# ---- lattice expansion ---------------------------------------------------------

def coupling(aw, harm=1, helical=False):
    """Coupling factor aw*JJ_h of a planar undulator (aw for helical, h = 1):
    JJ_h = J_m(xi) - J_{m+1}(xi), m = (h-1)/2, xi = h aw^2 / (2 (1 + aw^2)),
    sign (-1)^m."""
    from scipy.special import jv
    if harm < 1:
        return 0.0
    if helical:
        return aw if harm == 1 else 0.0
    if harm % 2 == 0:
        return 0.0
    xi = harm * aw * aw / (2.0 * (1.0 + aw * aw))
    m = (harm - 1) // 2
    jj = jv(m, xi) - jv(m + 1, xi)
    return float(aw * (-jj if m % 2 else jj))


class Lattice:
    """A .lat beamline expanded into per-step tables (steps[i] is a g4b_step,
    slip[i] the slippage in units of lambda0, fc(i, h) the coupling), following
    the same expansion rules as the drop-in host layer: undulators in
    round(L/delz) equal steps with slippage dz(1+aw^2)/(2 gamma0^2 lambda0),
    other elements in ceil(L/delz) steps with slippage dz/(2 gamma0^2 lambda0).
    Supports UNDULATOR, QUADRUPOLE, DRIFT and LINE (n*element repetition)."""

    def __init__(self, text, beamline, delz, gamma0, lambda0):
        import math
        import re
        Step = _step_type()
        el = {}
        body = "\n".join(ln.split("#", 1)[0] for ln in text.splitlines())
        for stmt in body.split(";"):
            stmt = stmt.strip()
            if not stmt:
                continue
            m = re.match(r"([^:]+):\s*([A-Za-z]+)\s*=\s*\{(.*)\}\s*$", stmt, re.S)
            if not m:
                raise ValueError(f"cannot parse '{stmt}'")
            label, typ, items = m.group(1).strip().upper(), m.group(2).upper(), m.group(3)
            if typ == "LINE":
                line = []
                for it in items.split(","):
                    it = it.strip()
                    if not it:
                        continue
                    rep, _, name = it.rpartition("*")
                    line.append((int(rep) if rep else 1, name.strip().upper()))
                el[label] = (typ, line)
            else:
                par = {}
                for it in items.split(","):
                    if it.strip():
                        k, v = it.split("=", 1)
                        v = v.strip()
                        vu = v.upper()
                        par[k.strip().lower()] = (1.0 if vu in ("TRUE", "T") else
                                                  0.0 if vu in ("FALSE", "F") else float(v))
                el[label] = (typ, par)

        def flat(name):
            typ, val = el[name]
            if typ != "LINE":
                return [(typ, val)]
            return [e for rep, sub in val for _ in range(rep) for e in flat(sub)]

        g2 = 2.0 * gamma0 * gamma0
        self.steps, self.slip, self.helical = [], [], []
        for typ, p in flat(beamline.upper()):
            if typ == "UNDULATOR":
                lu, nw, aw = p.get("lambdau", 0), p.get("nwig", 0), p.get("aw", 0)
                hel = p.get("helical", 0) != 0
                ku = 2 * math.pi / lu if lu > 0 else 0.0
                kx, ky = p.get("kx", 0.5 if hel else 0.0), p.get("ky", 0.5 if hel else 1.0)
                taper = p.get("taper", 0.0)
                L = lu * nw
                ns = max(1, int(math.floor(L / delz + 0.5)))
                for i in range(ns):
                    dz = L / ns
                    awi = aw * (1.0 + taper * (i + 0.5) / ns)
                    self.steps.append(Step(
                        delz=dz, aw=awi, ax=p.get("ax", 0.0), ay=p.get("ay", 0.0),
                        kx=kx * ku * ku, ky=ky * ku * ku, gradx=p.get("gradx", 0.0),
                        grady=p.get("grady", 0.0), ku=ku, gamma_ref=gamma0,
                        in_undulator=1 if awi > 0 else 0))
                    self.slip.append(dz * (1 + awi * awi) / g2 / lambda0)
                    self.helical.append(hel)
            elif typ in ("DRIFT", "QUADRUPOLE"):
                L = p.get("l", 0.0)
                if L <= 0:
                    continue
                ns = max(1, int(math.ceil(L / delz - 1e-9)))
                for i in range(ns):
                    dz = L / ns
                    kw = dict(delz=dz, gamma_ref=gamma0)
                    if typ == "QUADRUPOLE":
                        kw.update(qf=p.get("k1", 0.0), dqx=p.get("dx", 0.0),
                                  dqy=p.get("dy", 0.0))
                    self.steps.append(Step(**kw))
                    self.slip.append(dz / g2 / lambda0)
                    self.helical.append(False)
            else:
                raise ValueError(f"unsupported element type {typ}")
        self.nstep = len(self.steps)

    def fc(self, i, harm):
        st = self.steps[i]
        return coupling(st.aw, harm, self.helical[i]) if st.in_undulator else 0.0


def gaussian_field(ngrid, gridmax, xlambda, power, w0):
    """One plane of a Gaussian mode of power `power` [W] and waist w0, in the
    field normalisation P = sum |u|^2 (dgrid eev/ks)^2 / vacimp (the host
    layer's seed to within the rounding of exp)."""
    dgrid = 2 * gridmax / (ngrid - 1)
    ks = 2 * np.pi / xlambda
    v = -gridmax + np.arange(ngrid) * dgrid
    yy, xx = np.meshgrid(v, v, indexing="ij")
    g = np.exp(-(xx * xx + yy * yy) / (w0 * w0))
    s = float(np.cumsum((g * g).reshape(-1))[-1])
    unit = dgrid * EEV / ks
    amp = np.sqrt(power * VACIMP / (unit * unit * s)) if (power > 0 and s > 0) else 0.0
    return (g * amp).astype(np.complex128)


# ---------------------------------------------------------------------------
# Short-range space charge.  The reference hands this to upstream GENESIS
# 1.3 v4's EFieldSolver::shortRange on the host (src/Core/BeamSolverCUDA.cpp:
# 523-547), which is absent from the reference tree: this restates the
# device model of g4b_efield_short_range (radial finite-volume solve of
# (1/r d/dr r d/dr - m^2/r^2 - (l k_s)^2/gamma_z^2) u = -S per density mode),
# and tests pin it to the closed-form solution of the continuous problem.
# PARITY UNPINNED against upstream.

SC_FIX = 2.0 ** 40


def sc_solve(acc, npart, m, kdr2):
    """Radial Thomas solve of one mode in cell units: acc = the mode's
    fixed-point cell sums (complex, already divided by 2^40), npart = slice
    particle count, kdr2 = (l k_s dr)^2 / gamma_z^2.  Returns u per cell."""
    n = acc.size
    rhs = -acc / (2.0 * np.pi * npart)
    cp = np.zeros(n)
    d = np.zeros(n, complex)
    pc, pd = 0.0, 0.0
    for j in range(n):
        rc, lo, up = j + 0.5, float(j), float(j + 1)
        diag = -lo - (2.0 * up if j == n - 1 else up) - (m * m / (rc * rc) + kdr2) * rc
        den = diag - lo * pc
        pc = up / den if j < n - 1 else 0.0
        pd = (rhs[j] - lo * pd) / den
        cp[j], d[j] = pc, pd
    u = d.copy()
    for j in range(n - 2, -1, -1):
        u[j] = d[j] - cp[j] * u[j + 1]
    return u


def short_range(off, parts, current, gammaz2, *, rmax, ngrid, nz, nphi, lambda0,
                slice_eloss=None, return_modes=False):
    """Per-particle loss (space charge + slice loss) of every particle."""
    off = np.asarray(off, np.int64)
    ns = off.size - 1
    el = np.zeros(ns) if slice_eloss is None else np.asarray(slice_eloss, np.float64)
    ks = 2.0 * np.pi / lambda0
    coef = -2.0 * VACIMP * ks / (EEV * gammaz2)
    out = np.zeros(int(off[-1]))
    modes = []
    for s in range(ns):
        b, e = int(off[s]), int(off[s + 1])
        npart = e - b
        if npart == 0:
            modes.append(None)
            continue
        x, y, th = parts["x"][b:e], parts["y"][b:e], parts["theta"][b:e]
        xc, yc = x.sum() / npart, y.sum() / npart
        dx, dy = x - xc, y - yc
        r = np.sqrt(dx * dx + dy * dy)
        R = rmax * np.sqrt(np.max(dx * dx + dy * dy))
        if not R > 0 or current[s] == 0:
            out[b:e] = el[s]
            modes.append(None)
            continue
        dr = R / ngrid
        q = r / dr
        ok = (q >= 0) & (q < ngrid)  # NaN or beyond the wall: the last cell
        j = np.where(ok, np.where(ok, q, 0).astype(np.int64), ngrid - 1)
        safe = np.where(r > 0, r, 1.0)
        cph, sph = np.where(r > 0, dx / safe, 1.0), np.where(r > 0, dy / safe, 0.0)
        total = np.zeros(npart)
        us = {}
        for l in range(1, nz + 1):
            cl, sl = np.cos(l * th), np.sin(l * th)
            ph = {0: cl - 1j * sl}
            pr, pi_, qr, qi = cl, -sl, cl, -sl
            for m in range(1, nphi + 1):
                pr, pi_ = pr * cph + pi_ * sph, pi_ * cph - pr * sph
                qr, qi = qr * cph - qi * sph, qi * cph + qr * sph
                ph[m], ph[-m] = pr + 1j * pi_, qr + 1j * qi
            kdr2 = (l * ks * dr) ** 2 / gammaz2
            acc_l = 0.0
            for m in range(-nphi, nphi + 1):
                qre = np.zeros(ngrid, np.int64)
                qim = np.zeros(ngrid, np.int64)
                np.add.at(qre, j, np.rint(ph[m].real * SC_FIX).astype(np.int64))
                np.add.at(qim, j, np.rint(ph[m].imag * SC_FIX).astype(np.int64))
                u = sc_solve((qre + 1j * qim) / SC_FIX, npart, m, kdr2)
                us[(l, m)] = u
                # Im[u e^{i(l theta + m phi)}] = Im[u conj(phase)]
                acc_l = acc_l + np.imag(u[j] * np.conj(ph[m]))
            total += l * acc_l
        out[b:e] = el[s] + coef * current[s] * total
        modes.append(dict(dr=dr, xc=xc, yc=yc, u=us))
    return (out, modes) if return_modes else out


# ---------------------------------------------------------------------------
# Incoherent synchrotron radiation (the device model of g4b_beam_incoherent;
# upstream's Incoherent class, which the reference calls on the host,
# src/Core/Beam.cpp:126, is absent: PARITY UNPINNED against upstream).

RE = 2.8179403262e-15
LAMBDA_C = 3.8615926796e-13


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*[int(v) & 0xFFFFFFFF for v in ctr])
    k = (C.c_uint32 * 2)(*[int(v) & 0xFFFFFFFF for v in key])
    load().g4o_philox4x32_10(c, k)
    return [int(v) for v in c]


def isr_rates(aw, ku, helical=False):
    """(loss, spread): d gamma/dz = -loss gamma^2, d<dgamma^2>/dz = spread gamma^4."""
    if not (aw > 0 and ku > 0):
        return 0.0, 0.0
    K = aw if helical else np.sqrt(2.0) * aw
    F = (1.70 * K + 1 / (1 + 1.88 * K + 0.80 * K * K)) if helical else \
        (1.42 * K + 1 / (1 + 1.5 * K + 0.95 * K * K))
    return 2.0 / 3.0 * RE * ku * ku * aw * aw, 14.0 / 15.0 * LAMBDA_C * RE * ku ** 3 * K * K * F


def incoherent(gamma, *, aw, ku, delz, helical=False, loss=True, spread=True, seed=0,
               counter=0):
    """One step in place on a float64 array."""
    lr, sr = isr_rates(aw, ku, helical)
    load().g4o_incoherent(gamma.size, _d(gamma), lr * delz if loss else 0.0,
                          float(np.sqrt(sr * delz)) if spread else 0.0, seed, counter)
