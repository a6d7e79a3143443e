"""The fused mixed-precision run against the FP64 CPU oracle.

Per-step tolerances follow from FP32 state (relative ~1e-6 after a few
steps); the end-to-end gates are the ones the mixed form is held to:
P(z) within 1e-3 relative before saturation and |b1|(z) within 1e-3 absolute
of the FP64 oracle on identical seeded inputs, slippage bit-exact."""
import math

import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from genesis4_cuda_port_b200 import workloads
from oracle import pyoracle as orc
from tests import synth

pytestmark = pytest.mark.gpu

P_TOL = 1e-3
B_TOL = 1e-3


@pytest.fixture(scope="module")
def ctx():
    c = dev.Context(0)
    yield c
    c.synchronize()


def _lattice_arrays(steps, harms=(1,)):
    fc = [[(synth.coupling(st.aw, h) if st.in_undulator else 0.0) for h in harms] for st in steps]
    slip = [st.delz * (1 + st.aw ** 2) / (2 * st.gamma_ref ** 2) / synth.LAMBDA0 for st in steps]
    return fc, slip


def _mk_run(ctx, off, parts, cells_list, harms, ngrid, gridmax, steps, current, time_run=True):
    run = dev.Run(ctx, off, fields=[(h, ngrid, gridmax) for h in harms], lambda0=synth.LAMBDA0,
                  gamma_ref=synth.GAMMA0, sample=1.0, time_run=time_run, nbunch=2)
    run.upload_beam(parts)
    for i, c in enumerate(cells_list):
        run.upload_field(i, c, 0)
    run.set_current(current)
    fc, slip = _lattice_arrays(steps, harms)
    run.set_lattice(steps, fc, slip)
    return run, fc, slip


def _oracle_run(off, parts, cells_list, harms, gridmax, steps, fc, slip, current, time_run=True):
    p = synth.copy_parts(parts)
    flds = [dict(cells=c.copy(), gridmax=gridmax, xlambda=synth.LAMBDA0 / h, harm=h, fc=0.0,
                 first=0, accuslip=0.0) for c, h in zip(cells_list, harms)]
    hist = []
    for i, st in enumerate(steps):
        for k, f in enumerate(flds):
            f["fc"] = fc[i][k]
        orc.step(off, current, st, synth.LAMBDA0, slip[i], 1.0, time_run, False, flds, p)
        hist.append([orc.diag_field(f["cells"], f["first"])[0][:, 0].copy() for f in flds])
    return p, flds, hist


@pytest.mark.parametrize("harms", [(1,), (1, 3)])
def test_mixed_steps_track_the_oracle(ctx, harms):
    nslice, ngrid, gridmax = 6, 65, 160e-6
    off, parts = synth.beam(nslice, 2048, seed=50)
    cells = [synth.field(nslice, ngrid, gridmax, seed=51 + h, amplitude=3e13 / h) for h in harms]
    steps = [synth.und_step()] * 4 + [synth.drift_step(delz=0.05, qf=1.5)] + [synth.und_step()] * 3
    cur = np.full(nslice, synth.CURRENT)
    run, fc, slip = _mk_run(ctx, off, parts, cells, harms, ngrid, gridmax, steps, cur)
    run.advance(0, len(steps), graph=False)
    got = run.download_beam()
    ref, flds, _ = _oracle_run(off, parts, cells, harms, gridmax, steps, fc, slip, cur)
    dg = got["gamma"] - parts["gamma"]
    dg_ref = ref["gamma"] - parts["gamma"]
    # energies are stored as FP32 offsets from gamma_ref (|dg| ~ 1-5, resolution
    # ~5e-7): the tolerance is a few of those plus 1e-3 of the energy change
    tol = 4 * np.spacing(np.float32(np.max(np.abs(parts["gamma"] - synth.GAMMA0)))) + \
        1e-3 * np.max(np.abs(dg_ref))
    assert np.max(np.abs(dg_ref)) > 1e-3
    assert np.max(np.abs(dg - dg_ref)) < tol
    assert np.max(np.abs(got["theta"] - ref["theta"])) < 1e-4
    for k in ("x", "y", "px", "py"):
        assert synth.rel_err(got[k], ref[k]) < 1e-5, k
    for i in range(len(harms)):
        cf, first = run.download_field(i)
        assert first == flds[i]["first"]
        assert synth.rel_err(cf, flds[i]["cells"]) < 1e-4


def _max_contrib(x, y, ngrid, gridmax):
    """The deposition's M from positions (FP32 cell arithmetic): the largest
    number of bilinear contributions any output cell receives, the sum of the
    particle counts of its four base cells."""
    x = x.astype(np.float32)
    y = y.astype(np.float32)
    gm = np.float32(gridmax)
    inv = np.float32(1.0 / (2 * gridmax / (ngrid - 1)))
    ok = (x > -gm) & (x < gm) & (y > -gm) & (y < gm)
    ix = np.floor((x[ok] + gm) * inv).astype(np.int64)
    iy = np.floor((y[ok] + gm) * inv).astype(np.int64)
    ok = (ix >= 0) & (ix < ngrid - 1) & (iy >= 0) & (iy < ngrid - 1)
    h = np.zeros((ngrid + 1, ngrid + 1), np.int64)
    np.add.at(h, (iy[ok] + 1, ix[ok] + 1), 1)
    m = h[1:, 1:] + h[:-1, 1:] + h[1:, :-1] + h[:-1, :-1]
    return int(m.max())


def test_recount_when_the_contribution_bound_is_exceeded(ctx):
    """A quadrupole that images the beam's angles onto the grid (phase advance
    pi/2 over one step) concentrates the particles in x: that step's
    deposition counts more contributions per cell than the bound taken from
    the step before (M + M/4 + 4) and is redone at the exact scale.  The
    result is the one a fresh run gives from the same state, whose first
    deposition counts before it accumulates: bit-identical."""
    nslice, ngrid, gridmax = 2, 65, 160e-6
    off, parts = synth.beam(nslice, 2048, seed=70)
    cells = [synth.field(nslice, ngrid, gridmax, seed=71, amplitude=3e13)]
    k = (math.pi / (2 * synth.LAMBDA_U)) ** 2
    steps = [synth.und_step(), synth.und_step(qf=k)]
    cur = np.full(nslice, synth.CURRENT)

    def m_of(b):
        return [_max_contrib(b["x"][off[s]:off[s + 1]], b["y"][off[s]:off[s + 1]], ngrid,
                             gridmax) for s in range(nslice)]

    run, _, _ = _mk_run(ctx, off, parts, cells, (1,), ngrid, gridmax, steps, cur, time_run=False)
    run.advance(0, 1, graph=False)
    b0 = run.download_beam()
    f0, first0 = run.download_field(0)
    run.advance(1, 1, graph=False)
    b1 = run.download_beam()
    f1, _ = run.download_field(0)
    m0, m1 = m_of(b0), m_of(b1)
    assert all(m1[s] > m0[s] + m0[s] // 4 + 4 for s in range(nslice)), (m0, m1)
    assert first0 == 0
    fresh, _, _ = _mk_run(ctx, off, b0, [f0], (1,), ngrid, gridmax, steps, cur, time_run=False)
    fresh.advance(1, 1, graph=False)
    b2 = fresh.download_beam()
    f2, _ = fresh.download_field(0)
    for key in b1:
        assert np.array_equal(b1[key], b2[key]), key
    assert np.array_equal(f1, f2)
    assert np.abs(f1 - f0).max() > 0  # the step deposited a source


def test_particle_results_do_not_depend_on_their_order(ctx):
    """The beam step holds two particles per thread in packed FP32 pairs and
    the deposition adds exact integers, so reversing the particles of every
    slice (new partners, new chunks) must give every particle the same bits.
    A quadrupole sets the thick-lens phase w2 = k (dz/2)^2 at the switch
    between its Taylor series and the closed forms (|w2| = 1e-2), so with a
    1e-3 energy spread the two lanes of many threads take different paths.
    Ragged slices (one empty) leave threads with one particle."""
    nslice, ngrid, gridmax = 3, 65, 160e-6
    off, parts = synth.beam(nslice, 700, seed=90, energy_spread=1e-3, ragged=True)
    cells = [synth.field(nslice, ngrid, gridmax, seed=91, amplitude=2e12)]
    half = synth.LAMBDA_U / 2
    gz0 = math.sqrt(synth.GAMMA0 ** 2 - 1 - synth.AW ** 2)
    q_switch = 1e-2 / half ** 2 * gz0 / synth.GAMMA0
    steps = [synth.und_step(), synth.und_step(qf=q_switch), synth.und_step(),
             synth.und_step(qf=-q_switch), synth.und_step()]
    cur = np.full(nslice, synth.CURRENT)
    # w2 of every particle at the quadrupole step straddles the switch
    g = parts["gamma"]
    gz = np.sqrt(g * g - 1 - synth.AW ** 2 - parts["px"] ** 2 - parts["py"] ** 2)
    w2 = q_switch * synth.GAMMA0 / gz * half ** 2
    assert (w2 < 1e-2).any() and (w2 > 1e-2).any()
    perm = np.concatenate([np.arange(off[s + 1] - 1, off[s] - 1, -1) for s in range(nslice)])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    outs = []
    for order in (None, perm):
        p = parts if order is None else {k: v[order] for k, v in parts.items()}
        run, _, _ = _mk_run(ctx, off, p, cells, (1,), ngrid, gridmax, steps, cur)
        run.advance(0, len(steps), graph=True)
        b = run.download_beam()
        if order is not None:
            b = {k: v[inv] for k, v in b.items()}
        f, first = run.download_field(0)
        outs.append((b, f, first))
    (b1, f1, first1), (b2, f2, first2) = outs
    for key in b1:
        assert np.array_equal(b1[key], b2[key]), key
    assert first1 == first2 and np.array_equal(f1, f2)
    assert np.abs(b1["x"] - parts["x"]).max() > 0


def test_graph_replay_equals_direct_launches_and_is_deterministic(ctx):
    nslice, ngrid, gridmax = 4, 45, 160e-6
    off, parts = synth.beam(nslice, 1024, seed=60)
    cells = [synth.field(nslice, ngrid, gridmax, seed=61, amplitude=1e12)]
    steps = [synth.und_step()] * 6
    cur = np.full(nslice, synth.CURRENT)
    outs = []
    for graph in (False, True, True):
        run, _, _ = _mk_run(ctx, off, parts, cells, (1,), ngrid, gridmax, steps, cur)
        run.advance(0, len(steps), graph=graph)
        b = run.download_beam()
        f, first = run.download_field(0)
        hb, hf = run.history(len(steps) - 1)
        outs.append((b, f, first, hb, hf))
    for o in outs[1:]:
        for k in o[0]:
            assert np.array_equal(o[0][k], outs[0][0][k]), k
        assert np.array_equal(o[1], outs[0][1]) and o[2] == outs[0][2]
        assert np.array_equal(o[3], outs[0][3]) and np.array_equal(o[4], outs[0][4])


def test_mixed_diagnostics_history_matches_oracle_sums(ctx):
    nslice, ngrid, gridmax = 5, 51, 160e-6
    off, parts = synth.beam(nslice, 1536, seed=70, ragged=True)
    cells = [synth.field(nslice, ngrid, gridmax, seed=71, amplitude=1e12)]
    steps = [synth.und_step()] * 3
    cur = np.full(nslice, synth.CURRENT)
    run, fc, slip = _mk_run(ctx, off, parts, cells, (1,), ngrid, gridmax, steps, cur)
    run.advance(0, len(steps), graph=True)
    hb, hf = run.history(len(steps) - 1)
    ref, flds, _ = _oracle_run(off, parts, cells, (1,), gridmax, steps, fc, slip, cur)
    rs, rbre, rbim = orc.diag_beam(off, ref, nharm=2)
    np.testing.assert_allclose(hb[:, 12], rs[:, 12])  # counts exact
    for k in (0, 2, 4, 6, 8):
        np.testing.assert_allclose(hb[:, k], rs[:, k], rtol=1e-5, atol=1e-5 * np.max(np.abs(rs[:, k])))
    n = np.maximum(rs[:, 12], 1)
    np.testing.assert_allclose(hb[:, 23] / n, rbre[:, 0] / n, atol=1e-4)
    np.testing.assert_allclose(hb[:, 24] / n, rbim[:, 0] / n, atol=1e-4)
    fs, fcen = orc.diag_field(flds[0]["cells"], flds[0]["first"])
    np.testing.assert_allclose(hf[0, :, 0], fs[:, 0], rtol=1e-4)
    np.testing.assert_allclose(hf[0, :, 7:9], fcen, rtol=1e-3, atol=1e-4 * np.max(np.abs(fcen)))


def _pz_bunching_gpu_fp64(ctx, wl, off, parts, cells, lat, nstep):
    beam = dev.BeamState(ctx, off, wl.gamma0)
    beam.upload(parts)
    beam.set_current(np.full(wl.nslice, wl.current))
    fld = dev.FieldState(ctx, wl.nslice, wl.ngrid, wl.gridmax, wl.lambda0)
    fld.upload(cells)
    adi = dev.FieldSolverADICUDA(ctx)
    pz, bz = [], []
    for i in range(nstep):
        st = lat.steps[i]
        fc = lat.fc(i, 1)
        beam.track(st, st.delz * 0.5, False)
        beam.advance([fld], [fc], st)
        beam.apply_r56(st, wl.lambda0)
        beam.track(st, st.delz * 0.5, True)
        adi.init(st.delz, fld.dgrid, fld.xks, wl.ngrid)
        adi.advance(fld, beam, st, fc)
        fld.apply_slippage(lat.slip[i], wl.sample, time_run=wl.nslice > 1)
        s, _ = fld.diagnostics()
        bs, bre, bim = beam.diagnostics(1)
        pz.append(s[:, 0].sum())
        bz.append(np.abs(bre[:, 0] + 1j * bim[:, 0]).sum() / bs[:, 12].sum())
    return np.array(pz), np.array(bz)


def test_steady_state_pz_and_bunching_gates(ctx):
    """Steady-state FEL (1 slice, 8192 particles, ngrid 151, 1 kW seed) over the
    whole 344-step lattice: FP64 drop-in ~exact, mixed within the gates."""
    wl = workloads.steady_state()
    off, parts = wl.make_beam()
    cells = wl.make_field()
    lat = wl.make_lattice()
    nstep = lat.nstep
    # oracle
    p = synth.copy_parts(parts)
    f = dict(cells=cells.copy(), gridmax=wl.gridmax, xlambda=wl.lambda0, fc=0.0, first=0,
             accuslip=0.0)
    cur = np.full(1, wl.current)
    pz_ref, bz_ref = [], []
    for i in range(nstep):
        f["fc"] = lat.fc(i, 1)
        orc.step(off, cur, lat.steps[i], wl.lambda0, lat.slip[i], 1.0, False, False, [f], p)
        pz_ref.append(orc.diag_field(f["cells"], 0)[0][0, 0])
        s, bre, bim = orc.diag_beam(off, p, 1)
        bz_ref.append(abs(bre[0, 0] + 1j * bim[0, 0]) / s[0, 12])
    pz_ref, bz_ref = np.array(pz_ref), np.array(bz_ref)
    assert pz_ref[-1] > 1.2 * pz_ref[0]  # the FEL amplifies the seed
    # FP64 drop-in
    pz64, bz64 = _pz_bunching_gpu_fp64(ctx, wl, off, parts, cells, lat, nstep)
    np.testing.assert_allclose(pz64, pz_ref, rtol=1e-9)
    np.testing.assert_allclose(bz64, bz_ref, atol=1e-9)
    # mixed fused run
    run = dev.Run(ctx, off, fields=[(1, wl.ngrid, wl.gridmax)], lambda0=wl.lambda0,
                  gamma_ref=wl.gamma0, sample=1.0, time_run=False, nbunch=1)
    run.upload_beam(parts)
    run.upload_field(0, cells, 0)
    run.set_current(cur)
    run.set_lattice(lat.steps, [[lat.fc(i, 1)] for i in range(nstep)], lat.slip)
    run.advance(0, nstep, graph=True)
    pzm, bzm = [], []
    for i in range(nstep):
        hb, hf = run.history(i)
        pzm.append(hf[0, 0, 0])
        bzm.append(abs(hb[0, 23] + 1j * hb[0, 24]) / hb[0, 12])
    pzm, bzm = np.array(pzm), np.array(bzm)
    # pre-saturation: the whole lattice (power still growing at the end)
    rel = np.max(np.abs(pzm - pz_ref) / pz_ref)
    assert rel < P_TOL, rel
    assert np.max(np.abs(bzm - bz_ref)) < B_TOL
