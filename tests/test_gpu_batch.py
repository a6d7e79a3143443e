"""Batched runs: runs of different grids, particle counts, slice counts,
tapers and lengths advanced together give exactly the results they give
alone (every work item is computed as in the single-run kernels)."""
import numpy as np
import pytest

from genesis4_cuda_port_b200 import device as dev
from tests import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = dev.Context(0)
    yield c
    c.synchronize()


CONFIGS = [
    # nslice, npart/slice, ngrid, taper, detuning, time_run, nsteps
    dict(nslice=1, npart=1024, ngrid=45, taper=0.02, dgam=0.0, time_run=False, nsteps=8),
    dict(nslice=1, npart=2048, ngrid=71, taper=0.0, dgam=3e-4, time_run=False, nsteps=8),
    dict(nslice=3, npart=512, ngrid=33, taper=0.01, dgam=-2e-4, time_run=True, nsteps=6),
    dict(nslice=2, npart=768, ngrid=101, taper=0.0, dgam=0.0, time_run=True, nsteps=7),
    # 32-lane ADI rows (the grids above use 16-lane rows): a batch of mixed
    # row layouts runs their ADI kernels on concurrent streams
    dict(nslice=2, npart=512, ngrid=151, taper=0.005, dgam=1e-4, time_run=True, nsteps=6),
]


def _inputs(k, cfg):
    off, parts = synth.beam(cfg["nslice"], cfg["npart"], seed=200 + k)
    parts["gamma"] = parts["gamma"] * (1 + cfg["dgam"])
    cells = synth.field(cfg["nslice"], cfg["ngrid"], 160e-6, seed=300 + k, amplitude=2e12)
    n = cfg["nsteps"]
    steps = [synth.und_step(aw=synth.AW * (1 - cfg["taper"] * i / n)) for i in range(n - 1)]
    steps.append(synth.drift_step(delz=0.05, qf=1.0))
    fc = [[synth.coupling(st.aw) if st.in_undulator else 0.0] for st in steps]
    slip = [st.delz * (1 + st.aw ** 2) / (2 * synth.GAMMA0 ** 2) / synth.LAMBDA0 for st in steps]
    return off, parts, cells, steps, fc, slip


def _make(ctx, k, cfg):
    off, parts, cells, steps, fc, slip = _inputs(k, cfg)
    run = dev.Run(ctx, off, fields=[(1, cfg["ngrid"], 160e-6)], lambda0=synth.LAMBDA0,
                  gamma_ref=synth.GAMMA0, sample=1.0, time_run=cfg["time_run"], nbunch=1)
    run.upload_beam(parts)
    run.upload_field(0, cells, 0)
    run.set_current(np.full(cfg["nslice"], synth.CURRENT))
    run.set_lattice(steps, fc, slip)
    return run


def _result(run, nsteps):
    beam = run.download_beam()
    cells, first = run.download_field(0)
    hist = [run.history(i) for i in range(nsteps)]
    return beam, cells, first, hist


def _same(a, b):
    for k in a[0]:
        assert np.array_equal(a[0][k], b[0][k]), k
    assert np.array_equal(a[1], b[1])
    assert a[2] == b[2]
    for (hb1, hf1), (hb2, hf2) in zip(a[3], b[3]):
        assert np.array_equal(hb1, hb2) and np.array_equal(hf1, hf2)


def _alone(ctx):
    out = []
    for k, cfg in enumerate(CONFIGS):
        run = _make(ctx, k, cfg)
        run.advance(0, cfg["nsteps"], graph=False)
        out.append(_result(run, cfg["nsteps"]))
        run.close()
    return out


@pytest.mark.parametrize("graph, tune", [(False, False), (True, False), (True, True)])
def test_batch_equals_runs_alone(ctx, graph, tune):
    alone = _alone(ctx)
    batch = dev.Batch(ctx, 8)
    runs = [_make(ctx, k, cfg) for k, cfg in enumerate(CONFIGS)]
    slots = [batch.attach(r, 0, cfg["nsteps"]) for r, cfg in zip(runs, CONFIGS)]
    if tune:
        batch.tune()
    longest = max(cfg["nsteps"] for cfg in CONFIGS)
    batch.step(longest + 2, graph=graph)  # runs leave at their own end
    ctx.synchronize()
    for s, r, cfg, ref in zip(slots, runs, CONFIGS, alone):
        assert batch.status(s) == (cfg["nsteps"], 0)
        _same(_result(r, cfg["nsteps"]), ref)
    if tune:
        g = batch.shapes()
        assert all(v > 0 for v in g.values())
    batch.close()


def test_run_joins_a_batch_in_progress(ctx):
    """A run attached while others are mid-way (continuous batching) ends
    with the results it has alone."""
    alone = _alone(ctx)
    batch = dev.Batch(ctx, len(CONFIGS))
    runs = [_make(ctx, k, cfg) for k, cfg in enumerate(CONFIGS)]
    batch.attach(runs[0], 0, CONFIGS[0]["nsteps"])
    batch.attach(runs[1], 0, CONFIGS[1]["nsteps"])
    batch.step(3, graph=True)
    batch.attach(runs[2], 0, CONFIGS[2]["nsteps"])
    batch.step(2, graph=True)
    batch.attach(runs[3], 0, CONFIGS[3]["nsteps"])
    batch.attach(runs[4], 0, CONFIGS[4]["nsteps"])
    batch.step(12, graph=True)
    ctx.synchronize()
    for r, cfg, ref in zip(runs, CONFIGS, alone):
        _same(_result(r, cfg["nsteps"]), ref)
    batch.close()


def test_many_slices_alone_graphed_and_batched_agree(ctx):
    """A 150-slice time-dependent run with slippage every step: direct
    launches, graph replay and the batch engine give the same bits, state and
    the diagnostics of every step."""
    cfg = dict(nslice=150, npart=256, ngrid=65, taper=0.0, dgam=0.0, time_run=True, nsteps=5)
    alone = _make(ctx, 9, cfg)
    alone.advance(0, cfg["nsteps"], graph=False)
    ref = _result(alone, cfg["nsteps"])
    alone.close()
    graphed = _make(ctx, 9, cfg)
    graphed.advance(0, cfg["nsteps"], graph=True)
    _same(_result(graphed, cfg["nsteps"]), ref)
    graphed.close()
    batch = dev.Batch(ctx, 2)
    run = _make(ctx, 9, cfg)
    batch.attach(run, 0, cfg["nsteps"])
    batch.step(cfg["nsteps"], graph=False)
    ctx.synchronize()
    _same(_result(run, cfg["nsteps"]), ref)
    batch.close()


def test_row_layout_tuner_keeps_batch_equal_to_alone(ctx):
    """g4b_batch_tune_layouts times both ADI row layouts of every grid on a
    scratch field before the first step; every step then runs in the chosen
    layouts, so each run equals an alone run given the same layouts."""
    lib = ctx.lib
    # a grid with at least 32 slices in the batch (ngrid 101: 40 + 2) is
    # timed in both layouts; the others keep their defaults
    cfgs = CONFIGS + [dict(nslice=40, npart=256, ngrid=101, taper=0.0, dgam=0.0,
                           time_run=True, nsteps=6)]
    batch = dev.Batch(ctx, 8)
    runs = [_make(ctx, k, cfg) for k, cfg in enumerate(cfgs)]
    for r, cfg in zip(runs, cfgs):
        batch.attach(r, 0, cfg["nsteps"])
    batch.tune_layouts()
    longest = max(cfg["nsteps"] for cfg in cfgs)
    batch.step(longest + 2, graph=True)
    ctx.synchronize()
    per_grid = {}
    for cfg in cfgs:
        per_grid[cfg["ngrid"]] = per_grid.get(cfg["ngrid"], 0) + cfg["nslice"]
    for k, (r, cfg) in enumerate(zip(runs, cfgs)):
        if per_grid[cfg["ngrid"]] < 32:  # too few slices of this grid to time
            assert r.layouts()[0] == lib.g4b_default_layout(cfg["ngrid"])
        lay = r.layouts()
        default = lib.g4b_default_layout(cfg["ngrid"])
        assert lay[0] == default or (lay[0] >= 100) != (default >= 100)
        alone = _make(ctx, k, cfg)
        alone.set_layouts(lay)
        alone.advance(0, cfg["nsteps"], graph=False)
        _same(_result(r, cfg["nsteps"]), _result(alone, cfg["nsteps"]))
        alone.close()
    batch.close()


def test_both_row_layouts_solve_the_same_system(ctx):
    """The other row layout of a grid changes only the FP32 rounding of the
    row solve; a layout that is not one of the grid's two is refused."""
    # ngrid 101: 16 lanes x 7 by default, 32 lanes x 5 the other; steady
    # state, so the field stays in the window
    k, cfg = 3, dict(CONFIGS[3], time_run=False)
    a = _make(ctx, k, cfg)
    a.advance(0, cfg["nsteps"], graph=False)
    ra = _result(a, cfg["nsteps"])
    b = _make(ctx, k, cfg)
    lay = b.layouts()
    other = 5 if lay[0] >= 100 else 107
    b.set_layouts([other])
    assert b.layouts() == [other]
    b.advance(0, cfg["nsteps"], graph=False)
    rb = _result(b, cfg["nsteps"])
    scale = np.max(np.abs(ra[1]))
    assert scale > 0
    assert not np.array_equal(ra[1], rb[1])
    assert np.max(np.abs(ra[1] - rb[1])) < 1e-4 * scale
    with pytest.raises(Exception):
        b.set_layouts([9])
    a.close()
    b.close()
