"""Batched scan and served stream (C++ drivers on the batch engine): each
run's results are the same alone and in the mix, exactly."""
import numpy as np
import pytest

from genesis4_cuda_port_b200 import host, workloads

pytestmark = pytest.mark.gpu

LAT = """
UND: UNDULATOR = { lambdau = 0.015, nwig = 16, aw = 1.0 };
QF: QUADRUPOLE = { l = 0.03, k1 = 1.5 };
BL: LINE = { UND, QF, UND };
"""


def _cfg(**kw):
    wl = workloads.sase()
    return host.engine_config(LAT, "BL", wl.delz, wl.gamma0, wl.lambda0, threads=4, **kw)


def _jobs(n, seed=5):
    wl = workloads.sase()
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        ns = int(rng.integers(1, 5))
        jobs.append(workloads._job(wl, nslice=ns, ngrid=int(rng.choice([33, 45, 65, 71])),
                                   npart=int(rng.integers(64, 257)) * 4,
                                   nsteps=int(rng.integers(12, 35)), time_run=int(ns > 1),
                                   taper=float(rng.uniform(0, 0.02)),
                                   seed_power=float(rng.uniform(0, 1e4)), seed=100 + i))
    return jobs


def _split(rec, jobs):
    out, o = [], 0
    for j in jobs:
        k = j.nslice * 34
        out.append(rec[o:o + k])
        o += k
    return out


def test_scan_batched_equals_one_at_a_time():
    jobs = _jobs(7)
    r_b, p_b, rec_b = host.scan(_cfg(mode=0, tune=True), jobs, records=True)
    r_s, p_s, rec_s = host.scan(_cfg(mode=1), jobs, records=True)
    assert r_b.njobs == 7 and r_b.value > 0 and r_s.value > 0
    assert np.array_equal(rec_b, rec_s)
    assert np.array_equal(p_b, p_s)
    assert np.all(p_b > 0)
    assert all(g > 0 for g in r_b.grids)


def test_served_results_equal_alone():
    jobs = _jobs(9, seed=6)
    arrival = np.cumsum(np.full(9, 0.002))  # overlapping requests
    st, lat, power, rec = host.serve(_cfg(max_runs=4), jobs, arrival, records=True)
    assert st.peak_concurrency >= 2
    assert np.all(lat > 0) and st.p99 >= st.p50 > 0
    assert st.slice_steps == sum(j.nslice * j.nsteps for j in jobs)
    ref = []
    for j in jobs:
        _, _, _, r1 = host.serve(_cfg(max_runs=1), [j], np.zeros(1), records=True)
        ref.append(r1)
    for got, exp in zip(_split(rec, jobs), ref):
        assert np.array_equal(got, exp)
