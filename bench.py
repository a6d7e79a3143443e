#!/usr/bin/env python
"""Throughput of the GENESIS 1.3 v4 time-stepping hot path on B200.

One "step" is one pass of the hot path over every slice of the workload:
beam track/push/R56/track, field deposit + ADI, slippage and the per-slice
diagnostics (the reference's Gencore main loop, src/Core/Gencore.cpp:172-254).
The metric is slice-steps/s = nslice * steps / device time.

Default workload: time-dependent SASE, 1024 slices x 8192 particles, ngrid 201,
planar undulator lattice (3 x 110 periods + FODO quads), synthetic seeded
quiet-start beam with shot noise, no seed field.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one process per GPU): every rank runs an independent
replica of the workload (the path is slice-local and has no exchange step, so
ranks run replicas), value = total slice-steps/s of all ranks over the max-over-ranks
device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "slice-steps/s, mixed vs FP64 plain on 1 B200 at P(z) rel err≤1e-3; p99 latency"
UNIT = "slice-steps/s"


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--nslice", type=int, default=1024)
    p.add_argument("--npart", type=int, default=8192)
    p.add_argument("--ngrid", type=int, default=201)
    p.add_argument("--cpu-slices", type=int, default=128,
                   help="slices per sampled CPU step (oracle baseline)")
    p.add_argument("--cpu-steps", type=int, default=8)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-accuracy", action="store_true")
    p.add_argument("--workload", choices=["sase", "scan", "serve", "sase_h3", "steady", "fft"],
                   default="sase",
                   help="sase: the headline line; the others measure the batched scan, "
                        "the served stream, the large SASE with h=1 and h=3, steady state, "
                        "the FFT field solver")
    p.add_argument("--runs", type=int, default=256, help="scan: runs in the batch")
    p.add_argument("--requests", type=int, default=400, help="serve: requests in the stream")
    p.add_argument("--rate", type=float, default=200.0, help="serve: arrivals per second")
    return p.parse_args(argv)


# ---------------------------------------------------------------- helpers ---

class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def max_over_ranks(ms, dist=None, device="cuda"):
    """Device time of a step range as the max over ranks (the slowest replica
    bounds the job)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, nslice, steps, ms):
    """Whole-job slice-steps/s of `world` independent replicas of an
    nslice-slice workload that all took `steps` steps in at most `ms`."""
    return world * nslice * steps / (ms / 1e3)


def profile_traffic(kernel, wl):
    """DRAM bytes per launch of a mixed kernel from the committed ncu counters
    (profiles/mixed_step_sase1024x8192_n201.traffic.json, captured on 1024
    slices x 8192 particles, ngrid 201), scaled by the particles or cells of
    this workload; None if not profiled."""
    path = ROOT / "profiles" / "mixed_step_sase1024x8192_n201.traffic.json"
    if not path.exists():
        return None
    d = json.loads(path.read_text())
    b = d["bytes_per_launch"].get(kernel)
    if b is None:
        return None
    w = d["workload"]
    if kernel.startswith("adi"):
        scale = wl.nslice * wl.ngrid ** 2 / (w["nslice"] * w["ngrid"] ** 2)
    else:
        scale = wl.nslice * wl.npart / (w["nslice"] * w["npart"])
    return int(b * scale)


def measured_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        d = json.loads(path.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------- CPU arms ---

def oracle_inputs(wl, nslice):
    """The workload's first `nslice` slices built by the oracle alone (its
    quiet-start loader, lattice expansion and Gaussian seed, bit-identical to
    the host layer's): the CPU arms load no library of the product."""
    from oracle import pyoracle as orc
    sp = wl.beam_spec()
    spec = orc.BeamSpec(**{k: getattr(sp, k) for k, _ in orc.BeamSpec._fields_})
    spec.nslice = nslice
    cur = np.full(nslice, wl.current)
    off, parts = orc.load_beam(spec, cur)
    plane = orc.gaussian_field(wl.ngrid, wl.gridmax, wl.lambda0, wl.seed_power, wl.waist)
    cells = np.broadcast_to(plane, (nslice, wl.ngrid, wl.ngrid)).copy()
    lat = orc.Lattice(wl.lattice, wl.beamline, wl.delz, wl.gamma0, wl.lambda0)
    return off, parts, cur, cells, lat


def cpu_steps(wl, off, parts, cur, cells, lat, steps):
    """Time the FP64 oracle over the given lattice step indices (every slice of
    the inputs, diagnostics included); returns seconds per step."""
    from oracle import pyoracle as orc
    fld = dict(cells=cells, gridmax=wl.gridmax, xlambda=wl.lambda0, fc=0.0, first=0,
               accuslip=0.0)
    per = []
    for i in steps:
        t0 = time.perf_counter()
        st = lat.steps[i % lat.nstep]
        fld["fc"] = lat.fc(i % lat.nstep, 1)
        orc.step(off, cur, st, wl.lambda0, lat.slip[i % lat.nstep], wl.sample, True,
                 False, [fld], parts)
        orc.diag_beam(off, parts, 1, True)
        orc.diag_field(fld["cells"], fld["first"])
        per.append(time.perf_counter() - t0)
    return per


def cpu_sample(wl, nslice_sample, nsteps):
    """The FP64 CPU oracle on a bounded sample of the workload: the first
    nslice_sample slices (full particle count and grid), nsteps lattice steps."""
    from oracle import pyoracle as orc
    off, parts, cur, cells, lat = oracle_inputs(wl, nslice_sample)
    dt = sum(cpu_steps(wl, off, parts, cur, cells, lat, range(nsteps)))
    return {"value": nslice_sample * nsteps / dt, "unit": UNIT,
            "cores": orc.num_threads(), "kind": "port",
            "sample": f"{nslice_sample} slices x {nsteps} steps of the same workload "
                      f"(Np={wl.npart}, ngrid={wl.ngrid}), FP64 oracle, OpenMP",
            "seconds": dt}


def run_reference(args, wl, rank, budget_s=240.0):
    """The reference's CPU implementation of the path is upstream GENESIS 1.3 v4
    (not vendored); its FP64 restatement (the oracle) is timed instead, on
    every slice of the workload, inputs built by the oracle itself.  Steps past
    the time budget are not run (the line says how many were)."""
    if rank != 0:
        return
    from oracle import pyoracle as orc
    off, parts, cur, cells, lat = oracle_inputs(wl, wl.nslice)
    warm = cpu_steps(wl, off, parts, cur, cells, lat, range(args.warmup))
    est = warm[-1] if warm else 0.0
    nrun = args.steps
    if est > 0 and est * args.steps > budget_s:
        nrun = max(1, int(budget_s / est))
    per = cpu_steps(wl, off, parts, cur, cells, lat,
                    range(args.warmup, args.warmup + nrun))
    tot = sum(per)
    value = wl.nslice * len(per) / tot
    sample = (f"all {wl.nslice} slices per step, {len(per)} of {args.steps} timed steps"
              f" (time budget {budget_s:.0f} s)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(per), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "nslice": wl.nslice, "npart": wl.npart,
                   "ngrid": wl.ngrid},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": orc.num_threads(),
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    line["reference_cuda"] = reference_cuda(wl, off, parts, cur, cells, lat, args)
    print(json.dumps(line), flush=True)


def reference_cuda(wl, off, parts, cur, cells, lat, args, slip=None):
    """The reference's own CUDA classes (src/Core/*.cpp, compiled unmodified
    into oracle/_ref) stepping the same workload on this GPU from device-
    resident state, in Gencore::run's order: the reference's GPU speed beside
    its CPU arm (slip: per-step slippage in slices, default the lattice's;
    zeros for a steady-state run).  None where the library or a GPU is
    missing."""
    from oracle import refpy
    if not refpy.available():
        return None
    try:
        if refpy.load().g4ref_device_count() < 1:
            return None
        n = lat.nstep
        ms = refpy.time_steps(off, parts, cur, cells, gridmax=wl.gridmax, xlambda=wl.lambda0,
                              steps=lat.steps, fc=[lat.fc(i, 1) for i in range(n)],
                              slip=lat.slip if slip is None else slip, sample=wl.sample,
                              warmup=args.warmup,
                              ntimed=max(1, min(args.steps, 20)))
    except Exception as e:  # the reference's classes throw on what they reject
        return {"unavailable": str(e)[:200]}
    return {"value": wl.nslice / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "steps": max(1, min(args.steps, 20)), "warmup": args.warmup,
            "what": "the reference's FieldSolverADICUDA, BeamSolverCUDA, ControlCUDA and "
                    "DiagnosticCUDA (compiled unmodified) stepping the workload's state "
                    "on this GPU, CUDA events around the timed steps, FP64"}


# ------------------------------------------------------------- GPU arm ---

class Fp64DropIn:
    """The plain FP64 drop-in: per-phase calls in the reference's order through
    the C ABI (Beam::track -> FieldSolverADICUDA::advance -> slippage ->
    DiagnosticCUDA), one host sync per step for the diagnostics."""

    def __init__(self, ctx, wl, off, parts, cells):
        from genesis4_cuda_port_b200 import device as dev
        self.wl = wl
        self.beam = dev.BeamState(ctx, off, wl.gamma0)
        self.fld = dev.FieldState(ctx, wl.nslice, wl.ngrid, wl.gridmax, wl.lambda0)
        self.adi = dev.FieldSolverADICUDA(ctx)
        self.beam.set_current(np.full(wl.nslice, wl.current))
        self.upload(parts, cells)

    def upload(self, parts, cells):
        self.beam.upload(parts)
        self.fld.upload(cells)
        self.fld.first = 0
        self.fld.accuslip = 0.0

    def step(self, lat, i):
        st = lat.steps[i]
        fc = lat.fc(i, 1)
        b, f = self.beam, self.fld
        b.track(st, st.delz * 0.5, False)
        b.advance([f], [fc], st)
        b.apply_r56(st, self.wl.lambda0)
        b.track(st, st.delz * 0.5, True)
        self.adi.init(st.delz, f.dgrid, f.xks, f.ngrid)
        self.adi.advance(f, b, st, fc)
        f.apply_slippage(lat.slip[i], self.wl.sample)
        b.diagnostics(1, True)
        f.diagnostics()

    def download(self):
        return self.beam.download(), self.fld.download()


def kernel_alg_bytes(wl, mixed: bool):
    """Algorithmic (compulsory) bytes of one launch of each kernel: every
    particle array a kernel touches read (and written) once, the field read and
    written once per ADI pass.  Compact source tiles are not counted."""
    N = wl.nslice * wl.npart
    C = wl.nslice * wl.ngrid ** 2
    if mixed:
        return {"run_beam_step": 56 * N, "run_deposit": 20 * N, "run_beam_diag": 28 * N,
                "adi_pass_x": 16 * C, "adi_pass_y": 16 * C, "run_diag_finalize": 0}
    return {"track": 72 * N, "push": 64 * N, "r56": 24 * N, "deposit": 32 * N,
            "adi_pass_x": 32 * C, "adi_pass_y": 32 * C, "diag_beam": 48 * N,
            "diag_field": 16 * C, "slice_scl": 24 * wl.nslice}


class MixedRun:
    """The fused mixed-precision form (g4b_run): state resident on the device,
    five kernels per step replayed as one CUDA graph, diagnostics kept in a
    device-side history."""

    def __init__(self, ctx, wl, off, lat):
        from genesis4_cuda_port_b200 import device as dev
        self.wl, self.lat = wl, lat
        self.run = dev.Run(ctx, off, fields=[(1, wl.ngrid, wl.gridmax)], lambda0=wl.lambda0,
                           gamma_ref=wl.gamma0, sample=wl.sample, time_run=wl.nslice > 1,
                           nbunch=1)
        self.run.set_current(np.full(wl.nslice, wl.current))
        self.run.set_lattice(lat.steps, [[lat.fc(i, 1)] for i in range(lat.nstep)], lat.slip)

    def upload(self, parts, cells):
        self.run.upload_beam(parts)
        self.run.upload_field(0, cells, 0)


def _stats(prof, alg, steps):
    per = {}
    for name, (cnt, tot) in prof.items():
        avg = tot / max(cnt, 1)
        b = alg.get(name, 0)
        per[name] = {"launches": cnt, "ms_per_step": tot / steps, "avg_ms": avg,
                     "alg_bytes": b, "gbs": b / (avg / 1e3) / 1e9 if avg > 0 else 0.0}
    return per


def fp64_history(ctx, wl, off, parts, cells, lat, nstep):
    """The FP64 drop-in over nstep lattice steps (per-phase calls through the C
    ABI): summed power and per-slice |b1| after every step, the final
    per-slice centre-cell field (beam-slice order) and the final beam sums."""
    from genesis4_cuda_port_b200 import device as dev
    beam = dev.BeamState(ctx, off, wl.gamma0)
    beam.upload(parts)
    beam.set_current(np.full(wl.nslice, wl.current))
    fld = dev.FieldState(ctx, wl.nslice, wl.ngrid, wl.gridmax, wl.lambda0)
    fld.upload(cells)
    adi = dev.FieldSolverADICUDA(ctx)
    pz, b1 = [], []
    for i in range(nstep):
        st = lat.steps[i]
        fc = lat.fc(i, 1)
        beam.track(st, st.delz * 0.5, False)
        beam.advance([fld], [fc], st)
        beam.apply_r56(st, wl.lambda0)
        beam.track(st, st.delz * 0.5, True)
        adi.init(st.delz, fld.dgrid, fld.xks, wl.ngrid)
        adi.advance(fld, beam, st, fc)
        fld.apply_slippage(lat.slip[i], wl.sample, time_run=wl.nslice > 1,
                           periodic=wl.periodic)
        fs, cen = fld.diagnostics()
        bs, bre, bim = beam.diagnostics(1)
        pz.append(fs[:, 0].sum())
        b1.append(np.hypot(bre[:, 0], bim[:, 0]) / np.maximum(bs[:, 12], 1))
    out = {"pz": np.array(pz), "b1": np.array(b1), "center": cen[:, 0] + 1j * cen[:, 1],
           "gsum": bs[:, 0].sum(), "g2sum": bs[:, 1].sum(), "count": bs[:, 12].sum()}
    for o in (adi, fld, beam):
        o.close()
    return out


def mixed_history(ctx, wl, off, parts, cells, lat, nstep):
    """The fused mixed-precision run over nstep steps (graph replay), with the
    same quantities as fp64_history read from its device-side history."""
    from genesis4_cuda_port_b200 import device as dev
    run = dev.Run(ctx, off, fields=[(1, wl.ngrid, wl.gridmax)], lambda0=wl.lambda0,
                  gamma_ref=wl.gamma0, sample=wl.sample, time_run=wl.nslice > 1,
                  periodic=wl.periodic, nbunch=1)
    run.upload_beam(parts)
    run.upload_field(0, cells, 0)
    run.set_current(np.full(wl.nslice, wl.current))
    run.set_lattice(lat.steps[:nstep], [[lat.fc(i, 1)] for i in range(nstep)],
                    lat.slip[:nstep], hist_steps=nstep)
    run.advance(0, nstep, graph=True)
    hb, hf = run.history_range(0, nstep)
    run.close()
    last_b, last_f = hb[-1], hf[-1, 0]
    return {"pz": hf[:, 0, :, 0].sum(axis=1),
            "b1": np.hypot(hb[:, :, 23], hb[:, :, 24]) / np.maximum(hb[:, :, 12], 1),
            "center": last_f[:, 7] + 1j * last_f[:, 8],
            "gsum": last_b[:, 0].sum(), "g2sum": last_b[:, 1].sum(),
            "count": last_b[:, 12].sum()}


def accuracy_metrics(test, ref):
    """Errors of one history against a reference history (dicts as returned by
    fp64_history / mixed_history): P(z) relative before saturation (up to the
    reference's power maximum), per-slice |b1|(z) absolute, the on-axis
    spectrum at the end (|FFT over slices of the centre-cell field|^2,
    relative to its peak) and the final energy spread (relative)."""
    pz_t, pz_r = test["pz"], ref["pz"]
    k = int(np.argmax(pz_r)) + 1
    spec = lambda h: np.abs(np.fft.fft(h["center"])) ** 2  # noqa: E731
    sig = lambda h: np.sqrt(max(h["g2sum"] / h["count"] - (h["gsum"] / h["count"]) ** 2, 0.0))  # noqa: E731
    s_t, s_r = spec(test), spec(ref)
    return {"pz_rel_err_max": float(np.max(np.abs(pz_t[:k] - pz_r[:k]) / pz_r[:k])),
            "b1_abs_err_max": float(np.max(np.abs(test["b1"] - ref["b1"]))),
            "spectrum_rel_err": float(np.max(np.abs(s_t - s_r)) / np.max(s_r)),
            "energy_spread_rel_err": float(abs(sig(test) - sig(ref)) / sig(ref)),
            "power_gain": float(pz_r[-1] / pz_r[0]), "b1_final_max": float(ref["b1"][-1].max()),
            "presaturation_steps": k}


ACCURACY_GATES = {"pz_rel": 1e-3, "b1_abs": 1e-3}


def accuracy():
    """The mixed form against the FP64 drop-in (itself held to the FP64
    oracle within 1e-9 by the GPU tests) on the two exponential-gain
    workloads: steady state (1 slice, 1 kW seed) and periodic time-dependent
    SASE (64 slices x 8192 from shot noise, ngrid 201), both over 1032 steps.
    Reports P(z), |b1|(z), on-axis spectrum and final energy-spread errors
    beside the power gain."""
    from genesis4_cuda_port_b200 import device as dev, workloads
    ctx = dev.Context(int(os.environ.get("LOCAL_RANK", "0")))
    out = []
    for wl in (workloads.steady_state_high_gain(), workloads.sase_periodic_high_gain()):
        off, parts = wl.make_beam()
        cells = wl.make_field()
        lat = wl.make_lattice()
        ref = fp64_history(ctx, wl, off, parts, cells, lat, lat.nstep)
        mix = mixed_history(ctx, wl, off, parts, cells, lat, lat.nstep)
        m = accuracy_metrics(mix, ref)
        m["workload"] = wl.name
        m["reference"] = "FP64 drop-in"
        m["gates"] = ACCURACY_GATES
        m["within_gates"] = (m["pz_rel_err_max"] <= ACCURACY_GATES["pz_rel"] and
                             m["b1_abs_err_max"] <= ACCURACY_GATES["b1_abs"])
        out.append(m)
    ctx.close()
    return out


def _engine_clocks():
    return Clocks(int(os.environ.get("LOCAL_RANK", "0")))


def run_scan(args):
    """Batched steady-state scan: every run resident, one persistent launch
    per phase per step (tuned shapes, graph), against the same runs one after
    another through the single-run graph path."""
    from genesis4_cuda_port_b200 import host, workloads
    wl, jobs, params = workloads.batched_scan(args.runs)
    clk = _engine_clocks()
    clk.start()
    time.sleep(0.5)
    rb, _, _ = host.scan(workloads.engine(wl, max_runs=len(jobs), tune=2, mode=0), jobs)
    c = clk.stop()
    rs, _, _ = host.scan(workloads.engine(wl, max_runs=len(jobs), mode=1), jobs)
    line = {"metric": "slice-steps/s, batched steady-state scan", "value": rb.value,
            "unit": UNIT, "n_gpus": 1, "steps": int(rb.slice_steps / len(jobs)),
            "higher_is_better": True, "dtype": "f32 state, f64 theta", "data": "synthetic",
            "config": {"workload": f"batched steady-state scan, {len(jobs)} runs",
                       "ngrid": "U[101,301]", "npart": "U[2048,32768]", "taper": "U[0,2%]",
                       "detuning": "U[-5e-4,5e-4]", "seed_power": "logU[100 W,10 kW]",
                       "prng_seed": 1, "params": params},
            "seconds": rb.seconds, "slice_steps": rb.slice_steps,
            "device_bytes": rb.device_bytes, "launch_shapes": list(rb.grids),
            "row_layouts": {"runs_on_16_lane_rows": rb.layouts_16,
                            "runs_moved_by_the_tuner": rb.layouts_switched},
            "one_at_a_time": {"value": rs.value, "seconds": rs.seconds},
            "batched_over_one_at_a_time": rb.value / rs.value, "clocks": c}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Served stream with continuous batching; p50/p99 latency beside the
    throughput."""
    from genesis4_cuda_port_b200 import host, workloads
    wl, jobs, arrival, params = workloads.served_stream(args.requests, args.rate)
    clk = _engine_clocks()
    clk.start()
    time.sleep(0.5)
    st, lat, power, _ = host.serve(workloads.engine(wl, max_runs=256), jobs, arrival)
    c = clk.stop()
    line = {"metric": "p99 latency, served stream", "value": st.p99, "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f32 state, f64 theta",
            "data": "synthetic",
            "config": {"workload": f"served stream, {len(jobs)} requests, Poisson "
                                   f"{args.rate}/s", "nslice": "U{1..64}",
                       "ngrid": "U[101,255]", "npart": "U[2048,16384]",
                       "nsteps": "U[110,330]", "admission": "free HBM - 4 GB reserve, "
                                                           "256 batch slots"},
            "p50_s": st.p50, "p99_s": st.p99, "mean_s": st.mean,
            "throughput": {"requests_per_s": st.requests_per_s,
                           "slice_steps_per_s": st.slice_steps_per_s},
            "seconds": st.seconds, "peak_concurrency": st.peak_concurrency,
            "batch_steps": st.batch_steps, "clocks": c}
    print(json.dumps(line), flush=True)


def _load_beam_parallel(wl, threads=12):
    """Quiet-start beam of a large workload, slices loaded by worker threads."""
    from concurrent.futures import ThreadPoolExecutor
    from genesis4_cuda_port_b200 import host
    n = wl.nslice * wl.npart
    parts = {k: np.empty(n) for k in ("x", "y", "px", "py", "gamma", "theta")}
    per = max(1, wl.nslice // threads)

    def load(s0):
        s1 = min(wl.nslice, s0 + per)
        sub = type(wl)(**{**wl.__dict__, "nslice": s1 - s0, "seed": wl.seed * 1000003 + s0})
        o, pp = host.load_beam(sub.beam_spec(), np.full(s1 - s0, wl.current))
        for k in parts:
            parts[k][s0 * wl.npart:s1 * wl.npart] = pp[k]

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(load, range(0, wl.nslice, per)))
    off = np.arange(wl.nslice + 1, dtype=np.int64) * wl.npart
    return off, parts


def run_h3(args):
    """Large time-dependent SASE, fundamental and 3rd harmonic fields."""
    import torch
    from genesis4_cuda_port_b200 import device as dev, workloads
    wl = workloads.large_sase_h3()
    ctx = dev.Context(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.ExternalStream(ctx.stream)
    off, parts = _load_beam_parallel(wl)
    lat = wl.make_lattice()
    run = dev.Run(ctx, off, fields=[(1, wl.ngrid, wl.gridmax), (3, wl.ngrid, wl.gridmax)],
                  lambda0=wl.lambda0, gamma_ref=wl.gamma0, sample=wl.sample, time_run=True,
                  nbunch=3)
    run.upload_beam(parts)
    del parts
    run.upload_field(0, None, 0)  # SASE: no seed field
    run.upload_field(1, None, 0)
    run.set_current(np.full(wl.nslice, wl.current))
    run.set_lattice(lat.steps, [[lat.fc(i, 1), lat.fc(i, 3)] for i in range(lat.nstep)],
                    lat.slip, hist_steps=4)
    K, W = args.steps, args.warmup
    run.advance(0, W, graph=False)
    ctx.synchronize()
    run.prepare(W, K)
    clk = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clk.start()
    time.sleep(0.5)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run.advance(W, K, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    c = clk.stop()
    line = {"metric": "slice-steps/s, large SASE h=1 and h=3", "value": wl.nslice * K / (ms / 1e3),
            "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K,
            "higher_is_better": True, "dtype": "f32 state, f64 theta", "data": "synthetic",
            "config": {"workload": wl.name, "nslice": wl.nslice, "npart": wl.npart,
                       "ngrid": wl.ngrid, "fields": "h=1, h=3", "nbunch": 3},
            "device_bytes": run.device_bytes(), "clocks": c}
    print(json.dumps(line), flush=True)


def run_steady(args):
    """Steady state (1 slice, 8192 particles, ngrid 151): latency per step."""
    import torch
    from genesis4_cuda_port_b200 import device as dev, workloads
    wl = workloads.steady_state()
    ctx = dev.Context(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.ExternalStream(ctx.stream)
    off, parts = wl.make_beam()
    lat = wl.make_lattice()
    run = dev.Run(ctx, off, fields=[(1, wl.ngrid, wl.gridmax)], lambda0=wl.lambda0,
                  gamma_ref=wl.gamma0, sample=1.0, time_run=False, nbunch=1)
    cells = wl.make_field()
    run.upload_beam(parts)
    run.upload_field(0, cells, 0)
    run.set_current(np.full(1, wl.current))
    run.set_lattice(lat.steps, [[lat.fc(i, 1)] for i in range(lat.nstep)], lat.slip)
    run.advance(0, args.warmup, graph=False)
    n = lat.nstep
    run.prepare(0, n)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run.advance(0, n, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    line = {"metric": "us per step, steady state", "value": 1e3 * ms / n, "unit": "us/step",
            "higher_is_better": False, "n_gpus": 1, "steps": n, "dtype": "f32 state, f64 theta",
            "data": "synthetic", "config": {"workload": wl.name}}
    del run
    # the reference's own CUDA classes on the same state (steady state: no
    # slippage)
    ref = reference_cuda(wl, off, parts, np.full(1, wl.current), cells, lat, args,
                         slip=np.zeros(lat.nstep))
    if ref and "ms_per_step" in ref:
        ref["us_per_step"] = 1e3 * ref["ms_per_step"]
    line["reference_cuda"] = ref
    print(json.dumps(line), flush=True)


def run_fft(args):
    """The FFT field solver (FieldSolverFFTCUDA form, FP64) on the headline
    field: 1024 slices, ngrid 201, the SASE beam's source every step; device
    time per field step and per kernel (CUDA events on the library's
    stream), beside the ADI solver on the same state."""
    import torch
    from genesis4_cuda_port_b200 import device as dev, workloads
    wl = workloads.sase(args.nslice, args.npart, args.ngrid)
    ctx = dev.Context(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.ExternalStream(ctx.stream)
    off, parts = wl.make_beam()
    lat = wl.make_lattice()
    beam = dev.BeamState(ctx, off, wl.gamma0)
    beam.upload(parts)
    beam.set_current(np.full(wl.nslice, wl.current))
    fld = dev.FieldState(ctx, wl.nslice, wl.ngrid, wl.gridmax, wl.lambda0)
    rng = np.random.default_rng(3)
    cells = (rng.normal(size=(wl.nslice, wl.ngrid, wl.ngrid)) +
             1j * rng.normal(size=(wl.nslice, wl.ngrid, wl.ngrid))) * 1e9
    fld.upload(cells)
    st, fc = lat.steps[0], lat.fc(0, 1)
    out = {}
    for name, solver in (("fft", dev.FieldSolverFFTCUDA(ctx)), ("adi", dev.FieldSolverADICUDA(ctx))):
        solver.init(st.delz, fld.dgrid, fld.xks, wl.ngrid)
        for _ in range(args.warmup):
            solver.advance(fld, beam, st, fc)
        ctx.synchronize()
        ctx.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            solver.advance(fld, beam, st, fc)
        e1.record(stream)
        torch.cuda.synchronize()
        prof = ctx.profile_read()
        ctx.profile(False)
        out[name] = {"ms_per_step": e0.elapsed_time(e1) / args.steps,
                     "kernels": {k: {"launches": c, "avg_ms": t / max(c, 1)}
                                 for k, (c, t) in prof.items()}}
        solver.close()
    C = wl.nslice * wl.ngrid ** 2
    alg = {"fft_rows_fwd": 32 * C, "fft_cols": 32 * C, "fft_rows_inv": 32 * C}
    peak, kind = measured_peak()
    k = out["fft"]["kernels"]
    dom = max((n for n in k if n in alg), key=lambda n: k[n]["avg_ms"])
    gbs = alg[dom] / (k[dom]["avg_ms"] / 1e3) / 1e9
    line = {"metric": "slice-steps/s of the FFT field step (FP64)",
            "value": wl.nslice / (out["fft"]["ms_per_step"] / 1e3), "unit": "slice-steps/s",
            "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out["fft"]["ms_per_step"], "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"FFT field step {wl.nslice} slices, ngrid {wl.ngrid}, "
                                   f"source of {wl.npart} particles per slice"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": gbs, "peak": peak,
                         "peak_source": kind, "unit": "GB/s", "frac": gbs / peak,
                         "alg_bytes_per_launch": alg[dom], "traffic": None},
            "fft": out["fft"], "adi_same_state": out["adi"]}
    print(json.dumps(line), flush=True)


def run_ours(args, wl, rank, world):
    import torch

    from genesis4_cuda_port_b200 import device as dev

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()


    ctx = dev.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    lat = wl.make_lattice()
    off, parts = wl.make_beam()
    cells = wl.make_field()
    nstep = lat.nstep
    K, W = args.steps, args.warmup

    def timed(fn):
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1), dist)

    # ---------------- mixed fused form: the headline ----------------
    mx = MixedRun(ctx, wl, off, lat)
    mx.upload(parts, cells)
    mx.run.advance(0, W, graph=False)          # warm-up (direct launches)
    ctx.synchronize()
    mx.run.prepare(W, K)                        # capture outside the timed region
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.5)
    launches0 = ctx.launch_count()
    ms = timed(lambda: mx.run.advance(W, K, graph=True))
    launches = ctx.launch_count() - launches0
    clk = clocks.stop()
    value = replica_throughput(world, wl.nslice, K, ms)
    # per-kernel CUDA-event timing of the same kernels (direct launches) over
    # the first lattice steps of the timed region again, so that the figures
    # are those of the same steps (all undulator steps on the headline
    # lattice: a drift step's launches do no deposition)
    ctx.profile(True)
    kp = min(K, 30)
    ms_prof = timed(lambda: mx.run.advance(W, kp, graph=False))
    mixed_k = _stats(ctx.profile_read(), kernel_alg_bytes(wl, True), kp)
    ctx.profile(False)

    # mixed end to end: pinned host state -> steps -> host (state + diagnostics)
    e2e = None
    if not args.no_e2e:
        pin = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in parts.items()}
        pcells = torch.from_numpy(cells.view(np.float64)).pin_memory().numpy().view(np.complex128)
        pout = {k: torch.empty(v.shape, dtype=torch.float64).pin_memory().numpy()
                for k, v in parts.items()}
        pcout = torch.empty(cells.view(np.float64).shape,
                            dtype=torch.float64).pin_memory().numpy().view(np.complex128)
        hist = []

        def e2e_run():
            mx.upload(pin, pcells)
            mx.run.advance(0, K, graph=True)
            hist.append(mx.run.history_range(0, K))
            mx.run.download_beam(pout)
            mx.run.download_field(0, pcout)

        e2e_run()  # untimed: captures the graph of steps [0, K) from the uploaded state
        ems = timed(e2e_run)
        state_bytes = sum(v.nbytes for v in parts.values()) + cells.nbytes
        diag_bytes = wl.nslice * (23 + 2 + 9) * 8
        e2e = {"value": world * wl.nslice * K / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(state_bytes / K),
               "d2h_bytes_per_step": int(state_bytes / K + diag_bytes),
               "note": f"FP64 host state in pinned memory -> g4b_run upload -> {K} steps -> "
                       "per-step diagnostics and final beam/field back to the host"}
    del mx

    # ---------------- FP64 plain drop-in, measured beside it ----------------
    eng = Fp64DropIn(ctx, wl, off, parts, cells)
    for i in range(W):
        eng.step(lat, i % nstep)
    ctx.synchronize()
    ms64 = timed(lambda: [eng.step(lat, (W + k) % nstep) for k in range(K)])
    # per-kernel CUDA-event timing of the same lattice steps again (the events
    # between launches would stretch the timed steps)
    ctx.profile(True)
    kp64 = min(K, 10)
    timed(lambda: [eng.step(lat, (W + k) % nstep) for k in range(kp64)])
    fp64_k = _stats(ctx.profile_read(), kernel_alg_bytes(wl, False), kp64)
    ctx.profile(False)
    value64 = replica_throughput(world, wl.nslice, K, ms64)
    del eng

    dom = max(mixed_k, key=lambda n: mixed_k[n]["ms_per_step"])
    peak, peak_kind = measured_peak()
    d = mixed_k[dom]
    roof = {"bound": "hbm", "kernel": dom, "achieved": d["gbs"], "peak": peak,
            "peak_source": peak_kind, "unit": "GB/s", "frac": d["gbs"] / peak,
            "traffic": profile_traffic(dom, wl), "alg_bytes_per_launch": d["alg_bytes"],
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, "
                              "profiles/mixed_step_sase1024x8192_n201.traffic.json",
            "timing": "CUDA events around each launch on the launching stream, "
                      f"{kp} direct-launch steps: the first lattice steps of the graph-timed "
                      "region again"}

    acc = None
    if rank == 0 and not args.no_accuracy:
        acc = accuracy()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(wl, args.cpu_slices, args.cpu_steps)
        cpu.pop("seconds", None)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 state, f64 theta", "data": "synthetic",
            "config": {"workload": wl.name, "nslice": wl.nslice, "npart": wl.npart,
                       "ngrid": wl.ngrid, "form": "mixed fused run, CUDA graph replay",
                       "lattice_steps": nstep, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (mixed state ~1.4 GB per replica)"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": launches, "kernels": mixed_k,
            "fp64_plain": {"value": value64, "ms_per_step": ms64 / K,
                           "form": "FP64 drop-in, per-phase C-ABI calls, host sync per step",
                           "kernels": fp64_k},
            "mixed_over_fp64_plain": value / value64,
            "accuracy": acc,
        }
        print(json.dumps(line), flush=True)
    ctx.synchronize()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main(argv=None):
    args = parse_args(argv)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    from genesis4_cuda_port_b200 import workloads
    wl = workloads.sase(args.nslice, args.npart, args.ngrid)
    if args.impl == "reference":
        run_reference(args, wl, rank)
        return
    if args.workload != "sase":
        if rank == 0:
            {"scan": run_scan, "serve": run_serve, "sase_h3": run_h3,
             "steady": run_steady, "fft": run_fft}[args.workload](args)
        return
    run_ours(args, wl, rank, world)


if __name__ == "__main__":
    main()
