"""Records the reference's own outputs as golden fixtures for the oracle.

Runs the reference's CUDA classes (oracle/_ref/libg4ref.so, built from the
reference tree by oracle/ref/Makefile, driven through oracle/refpy.py) on
seeded synthetic inputs and writes one .npz per case (inputs and outputs)
into the output directory (default: this directory).  Needs a GPU: the
reference's kernels are CUDA.

    python tests/golden/make_golden.py [OUTDIR]

Cases cover every phase of the reference's time step at small sizes:
FieldSolverADICUDA::advance (source on / off, low-memory source, 3rd
harmonic, shifted slice pointer, ngrid 31 and 101, PCR path),
FieldSolverFFTCUDA::advance (odd and even grids, with and without the source
filter), BeamSolverCUDA::advance (one and two fields, slice energy loss),
TrackBeamCUDA::track / applyR56 (drift, focusing and defocusing quadrupoles
with offsets, corrector, chicane), ControlCUDA::applySlippage (a sequence of
shifts, periodic and not) and DiagnosticCUDA::calc (every record, three
bunching harmonics, two fields, an empty slice).
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refpy  # noqa: E402
from tests import synth  # noqa: E402

GM = 1.5e-4


def _beam(nslice, npart, seed, ragged=False):
    off, p = synth.beam(nslice, npart, seed=seed, ragged=ragged)
    return off.astype(np.int64), p


def _save(out, name, **arrays):
    np.savez(out / f"ref_{name}.npz", **arrays)
    print("wrote", name)


def _parts_arrays(p, prefix="in_"):
    return {prefix + k: v.copy() for k, v in p.items()}


def field_cases(out):
    ku2 = synth.KU ** 2
    base = dict(ax=1e-6, ay=-2e-6, kx=0.3 * ku2, ky=0.7 * ku2, gradx=20.0, grady=-10.0)
    cases = [
        # name, solver, S, n, harm, first, enabled, atomic, in_und, filter
        ("adi_n31", 0, 3, 31, 1, 1, 1, 0, 1, None),
        ("adi_n31_lowmem", 0, 3, 31, 1, 1, 1, 1, 1, None),
        ("adi_n31_h3", 0, 3, 31, 3, 2, 1, 0, 1, None),
        ("adi_n31_nosource", 0, 3, 31, 1, 0, 1, 0, 0, None),
        ("adi_n31_disabled", 0, 3, 31, 1, 0, 0, 0, 1, None),
        ("adi_n101", 0, 2, 101, 1, 1, 1, 0, 1, None),
        ("fft_n31", 1, 3, 31, 1, 1, 1, 0, 1, None),
        ("fft_n32_filter", 1, 2, 32, 1, 1, 1, 0, 1, (0.25, 0.3, 0.05)),
        ("fft_n31_h3_filter", 1, 2, 31, 3, 0, 1, 0, 1, (0.2, 0.2, 0.1)),
    ]
    for k, (name, solver, S, n, harm, first, en, atomic, inund, filt) in enumerate(cases):
        off, p = _beam(S, 300, seed=100 + k, ragged=True)
        cur = np.linspace(3000.0, 1000.0, S)
        cells = synth.field(S, n, GM, seed=200 + k, amplitude=1e12)
        st = synth.und_step(in_undulator=inund, **base)
        xlam = synth.LAMBDA0 / harm
        fc = synth.coupling(harm=harm)
        xc, yc, sig = filt if filt else (0.0, 0.0, 0.0)
        outc = refpy.field_advance(cells, solver=solver, gridmax=GM, xlambda=xlam, harm=harm,
                                   first=first, enabled=bool(en), atomic_source=bool(atomic),
                                   delz=st.delz, fc=fc, step=st, off=off, current=cur,
                                   parts=p, filt=filt is not None, xc=xc, yc=yc, sig=sig)
        _save(out, name, solver=solver, harm=harm, first=first, enabled=en, atomic=atomic,
              gridmax=GM, xlambda=xlam, fc=fc, step=refpy.step_to_array(st), off=off,
              current=cur, cells_in=cells, cells_out=outc, filt=np.array([xc, yc, sig]),
              **_parts_arrays(p))


def push_cases(out):
    ku2 = synth.KU ** 2
    st = synth.und_step(ax=2e-6, ay=1e-6, kx=0.4 * ku2, ky=0.6 * ku2, gradx=15.0,
                        grady=5.0, autophase=0.3)
    for name, harms, grids, firsts in [("push_1field", [1], [31], [2]),
                                       ("push_2field", [1, 3], [31, 25], [1, 3])]:
        S = 4
        off, p = _beam(S, 250, seed=300 + len(harms), ragged=True)
        fields = []
        for i, (h, n, f0) in enumerate(zip(harms, grids, firsts)):
            fields.append(dict(cells=synth.field(S, n, GM, seed=310 + i, amplitude=3e10 / h),
                               first=f0, harm=h, gridmax=GM, xlambda=synth.LAMBDA0 / h,
                               fc=synth.coupling(harm=h)))
        long_esc = np.linspace(-2e3, 4e3, S)
        q = {k: v.copy() for k, v in p.items()}
        refpy.beam_advance(off, st, fields, q, long_esc=long_esc)
        arrays = dict(step=refpy.step_to_array(st), off=off, long_esc=long_esc,
                      harms=np.array(harms), firsts=np.array(firsts), gridmax=GM,
                      out_gamma=q["gamma"], out_theta=q["theta"], **_parts_arrays(p))
        for i, f in enumerate(fields):
            arrays[f"cells{i}"] = f["cells"]
            arrays[f"xlambda{i}"] = f["xlambda"]
            arrays[f"fc{i}"] = f["fc"]
        _save(out, name, **arrays)


def track_cases(out):
    ku2 = synth.KU ** 2
    und = dict(kx=0.2 * ku2, ky=0.8 * ku2, ax=3e-6, ay=-1e-6)
    cases = [
        ("track_drift", synth.drift_step(delz=0.25), 0),
        ("track_quad_focus", synth.drift_step(delz=0.1, qf=2.5, dqx=1e-5, dqy=-2e-5), 0),
        ("track_quad_defocus", synth.drift_step(delz=0.1, qf=-2.5, dqx=-1e-5, dqy=3e-5), 0),
        ("track_und_quad", synth.und_step(qf=0.8, dqx=2e-6, **und), 0),
        ("track_corrector_last", synth.drift_step(delz=0.1, cx=1e-5, cy=-2e-5), 1),
        ("track_chicane_first", synth.drift_step(delz=0.3, chic_angle=0.02, chic_lb=0.05,
                                                 chic_ld=0.1, chic_lt=0.3), 0),
    ]
    for k, (name, st, last) in enumerate(cases):
        off, p = _beam(1, 2000, seed=400 + k)
        q = {kk: v.copy() for kk, v in p.items()}
        refpy.track(q, st, st.delz, last)
        if st.chic_angle != 0.0:
            refpy.r56(q, st, synth.LAMBDA0)
        _save(out, name, step=refpy.step_to_array(st), last=last, lambda0=synth.LAMBDA0,
              **_parts_arrays(p), **{"out_" + kk: v for kk, v in q.items()})


def slippage_cases(out):
    shifts = np.array([1.0, 1.0, 0.5, 0.5, -1.0, 2.0, 0.3, 0.3, 0.3, -0.5, 1.0])
    for name, periodic in [("slippage", 0), ("slippage_periodic", 1)]:
        S, n = 5, 7
        cells = synth.field(S, n, GM, seed=500 + periodic, amplitude=1.0)
        c = cells.copy()
        acc, first = 0.0, 0
        firsts, accs, snaps = [], [], []
        for sh in shifts:
            acc, first = refpy.slippage(c, sh, 1.0, True, bool(periodic), acc, first)
            firsts.append(first)
            accs.append(acc)
            snaps.append(c.copy())
        _save(out, name, periodic=periodic, shifts=shifts, cells_in=cells,
              firsts=np.array(firsts), accs=np.array(accs), cells_after=np.array(snaps))


def diag_cases(out):
    S = 4
    off, p = _beam(S, 350, seed=600, ragged=True)
    fields = [dict(cells=synth.field(S, 31, GM, seed=610, amplitude=1e9), first=1,
                   gridmax=GM, xlambda=synth.LAMBDA0),
              dict(cells=synth.field(S, 25, 1.2e-4, seed=611, amplitude=4e8), first=3,
                   gridmax=1.2e-4, xlambda=synth.LAMBDA0 / 3)]
    cur = np.array([2500.0, 0.0, 3100.0, 1200.0])
    eloss = np.array([1.0, -2.0, 3.0, 0.5])
    long_esc = np.array([10.0, 20.0, -5.0, 0.0])
    slen = synth.LAMBDA0
    beam, flds = refpy.diag(off, p, nharm=3, current=cur, fields=fields, slicelength=slen,
                            eloss=eloss, long_esc=long_esc)
    arrays = dict(off=off, current=cur, eloss=eloss, long_esc=long_esc, slicelength=slen,
                  nharm=3, **_parts_arrays(p))
    for i, f in enumerate(fields):
        arrays[f"cells{i}"] = f["cells"]
        arrays[f"first{i}"] = f["first"]
        arrays[f"gridmax{i}"] = f["gridmax"]
        arrays[f"xlambda{i}"] = f["xlambda"]
        for k, v in flds[i].items():
            arrays[f"field{i}:{k}"] = v
    for k, v in beam.items():
        arrays[f"beam:{k}"] = v
    _save(out, "diag", **arrays)


def main(argv):
    out = Path(argv[1]) if len(argv) > 1 else Path(__file__).resolve().parent
    out.mkdir(parents=True, exist_ok=True)
    lib = refpy.load()
    if lib.g4ref_device_count() < 1:
        raise SystemExit("the reference's kernels need a GPU")
    field_cases(out)
    push_cases(out)
    track_cases(out)
    slippage_cases(out)
    diag_cases(out)


if __name__ == "__main__":
    main(sys.argv)
