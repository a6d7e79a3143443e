"""The device side of the slice decomposition: plane copies out of and into
the library's field state, and the ring's shift logic on device state (one
rank: the same as the library's own slippage, bit for bit).  The exchange
between ranks is covered by the gloo tests in test_slices.py; ranks that
wait on each other are not run on one GPU."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist

from genesis4_cuda_port_b200 import device as dev
from genesis4_cuda_port_b200 import slices
from tests import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [dev.G4B_FP64, dev.G4B_MIXED])
def test_planes_and_single_rank_ring(precision):
    ctx = dev.Context(0)
    ns, n, gm = 6, 33, 1.5e-4
    cells = synth.field(ns, n, gm, seed=31, amplitude=1e10)
    a = dev.FieldState(ctx, ns, n, gm, synth.LAMBDA0, precision=precision)
    b = dev.FieldState(ctx, ns, n, gm, synth.LAMBDA0, precision=precision)
    a.upload(cells)
    b.upload(cells)
    pa = slices.DevicePlanes(a)
    buf = pa.plane_out(2)
    pa.plane_in(4, buf)
    got = a.download()
    assert np.array_equal(got[4], got[2])
    pa.zero_plane(1)
    assert not np.any(a.download()[1])
    a.upload(cells)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", str(29900 + os.getpid() % 50))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        ring = slices.PlaneRing()
        acc = 0.0
        for sh in [1.0, 0.7, 0.7, -1.0, 2.0]:
            acc, _ = ring.apply_slippage(pa, acc, sh, 1.0, True, False)
            b.apply_slippage(sh, 1.0, True, False)
            assert pa.first == b.first and acc == b.accuslip
            assert np.array_equal(a.download(), b.download())
        g = ring.allreduce_sum([1.0, 2.0], device=None)
        assert list(g) == [1.0, 2.0]
    finally:
        dist.destroy_process_group()
    a.close()
    b.close()
    ctx.close()
