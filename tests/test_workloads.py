"""Seeded workload generators of the batched scan and the served stream
(host only)."""
import numpy as np

from genesis4_cuda_port_b200 import workloads


def test_batched_scan_parameters():
    wl, jobs, params = workloads.batched_scan(256)
    a, b = workloads.batched_scan(256)[2], params
    assert a == b  # fixed seed
    n = np.array([p["ngrid"] for p in params])
    npart = np.array([p["npart"] for p in params])
    assert n.min() >= 101 and n.max() <= 301 and len(set(n)) > 100
    assert npart.min() >= 2048 and npart.max() <= 32768 and np.all(npart % 4 == 0)
    assert all(0 <= p["taper"] <= 0.02 and abs(p["detune"]) <= 5e-4 for p in params)
    assert all(100 <= p["seed_power"] <= 1e4 for p in params)
    assert all(j.nslice == 1 and j.time_run == 0 for j in jobs)


def test_served_stream_arrivals():
    wl, jobs, arrival, params = workloads.served_stream(2000, rate=200.0)
    assert np.all(np.diff(arrival) > 0)
    rate = len(arrival) / arrival[-1]
    assert 180 < rate < 220
    assert all(1 <= p["nslice"] <= 64 and 101 <= p["ngrid"] <= 255 for p in params)
    assert all(110 <= p["nsteps"] <= 330 and 2048 <= p["npart"] <= 16384 for p in params)
    assert all(j.time_run == (j.nslice > 1) for j in jobs)
