"""Slice decomposition over ranks (genesis4_cuda_port_b200.slices), run as
gloo ranks on the CPU with the FP64 oracle doing each rank's compute.

A time-dependent run of 9 slices split over 2 or 3 ranks, each rank stepping
its own slices (track, push, R56, track, ADI field step) and exchanging the
slipped planes through the ring, must give every slice the same bits as the
undivided run with the reference's single-rank slippage, forward and backward
shifts, periodic and not; the all-reduced global sums match the undivided
ones."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from genesis4_cuda_port_b200 import slices
from oracle import pyoracle as orc
from tests import synth

NS, NGRID, GM = 9, 21, 1.5e-4
SHIFTS = [1.0, 1.0, 0.6, 0.6, -1.0, 1.0, 2.0, 1.0]  # slippage per step (sample 1)


def _inputs():
    off, p = synth.beam(NS, 96, seed=21)
    cells = synth.field(NS, NGRID, GM, seed=22, amplitude=1e12)
    cur = np.linspace(3000, 1000, NS)
    return off, p, cells, cur


def _step_pieces(off, cur, p, cells, first, st, fc):
    """Beam::track + Field::track of one step (Gencore.cpp:172-217), no slippage."""
    orc.track(p, st, st.delz * 0.5, False)
    orc.push(off, st, [dict(cells=cells, first=first, harm=1, gridmax=GM,
                            xlambda=synth.LAMBDA0, fc=fc)], p)
    orc.r56(p, st, synth.LAMBDA0)
    orc.track(p, st, st.delz * 0.5, True)
    orc.adi_advance(cells, harm=1, gridmax=GM, xks=2 * np.pi / synth.LAMBDA0, delz=st.delz,
                    fc=fc, enabled=True, step=st, off=off, current=cur, parts=p, first=first)


def _beam_order(cells, first):
    ns = cells.shape[0]
    return cells[[(s + first) % ns for s in range(ns)]]


def _undivided(periodic):
    off, p, cells, cur = _inputs()
    st, fc = synth.und_step(), synth.coupling()
    acc, first = 0.0, 0
    for sh in SHIFTS:
        _step_pieces(off, cur, p, cells, first, st, fc)
        acc, first, _ = orc.slippage(cells, sh, 1.0, True, periodic, acc, first)
    fs, _ = orc.diag_field(cells, first)
    return _beam_order(cells, first), p, fs[:, :5].sum(axis=0)


def _rank(rank, world, port, periodic, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, p, cells, cur = _inputs()
        s0, s1 = slices.split_slices(NS, world)[rank]
        loff = off[s0:s1 + 1] - off[s0]
        lp = {k: v[off[s0]:off[s1]].copy() for k, v in p.items()}
        field = slices.HostPlanes(cells[s0:s1].copy())
        ring = slices.PlaneRing()
        st, fc = synth.und_step(), synth.coupling()
        acc = 0.0
        for sh in SHIFTS:
            _step_pieces(loff, cur[s0:s1], lp, field.cells, field.first, st, fc)
            acc, _ = ring.apply_slippage(field, acc, sh, 1.0, True, periodic)
        fs, _ = orc.diag_field(field.cells, field.first)
        glob = ring.allreduce_sum(fs[:, :5].sum(axis=0))
        q.put((rank, _beam_order(field.cells, field.first), lp, glob))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, False), (3, False), (2, True)])
def test_decomposed_run_equals_undivided(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() % 500) + 10 * world + periodic
    procs = [ctx.Process(target=_rank, args=(r, world, port, periodic, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    got = dict((r, (c, p, g)) for r, c, p, g in (q.get(timeout=300) for _ in range(world)))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    ref_cells, ref_p, ref_glob = _undivided(periodic)
    cells = np.concatenate([got[r][0] for r in range(world)])
    assert np.array_equal(cells, ref_cells)
    off = _inputs()[0]
    for k in ref_p:
        assert np.array_equal(np.concatenate([got[r][1][k] for r in range(world)]), ref_p[k])
    for r in range(world):
        np.testing.assert_allclose(got[r][2], ref_glob, rtol=1e-13)
    assert np.abs(ref_cells).max() > 0 and len(off) == NS + 1


def test_split_slices_is_contiguous_and_balanced():
    assert slices.split_slices(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert slices.split_slices(2, 2) == [(0, 1), (1, 2)]
