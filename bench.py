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
replica of the workload (the path is slice-local; SURVEY-level decision:
replicas only), value = total slice-steps/s of all ranks over the max-over-ranks
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


def measured_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        d = json.loads(path.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------- CPU arms ---

def cpu_sample(wl, nslice_sample, nsteps, lat):
    """Time the FP64 CPU oracle on a bounded sample of the workload: the first
    nslice_sample slices (full particle count and grid), nsteps lattice steps."""
    from oracle import pyoracle as orc
    sub = type(wl)(**{**wl.__dict__, "nslice": nslice_sample})
    off, parts = sub.make_beam()
    cells = sub.make_field()
    cur = np.full(nslice_sample, wl.current)
    fld = dict(cells=cells, gridmax=wl.gridmax, xlambda=wl.lambda0, fc=0.0, first=0,
               accuslip=0.0)
    t0 = time.perf_counter()
    for i in range(nsteps):
        st = lat.steps[i % lat.nstep]
        fld["fc"] = lat.fc(i % lat.nstep, 1)
        orc.step(off, cur, st, wl.lambda0, lat.slip[i % lat.nstep], wl.sample, True,
                 False, [fld], parts)
        orc.diag_beam(off, parts, 1, True)
        orc.diag_field(fld["cells"], fld["first"])
    dt = time.perf_counter() - t0
    return {"value": nslice_sample * nsteps / dt, "unit": UNIT,
            "cores": orc.num_threads(), "kind": "port",
            "sample": f"{nslice_sample} slices x {nsteps} steps of the same workload "
                      f"(Np={wl.npart}, ngrid={wl.ngrid}), FP64 oracle, OpenMP",
            "seconds": dt}


def run_reference(args, wl, rank):
    """The reference's CPU implementation of the path is upstream GENESIS 1.3 v4
    (not vendored); its FP64 restatement (the oracle) is timed instead."""
    if rank != 0:
        return
    lat = wl.make_lattice()
    per_step = []
    from oracle import pyoracle as orc
    for k in range(args.warmup + args.steps):
        res = cpu_sample(wl, args.cpu_slices, 1, lat)
        if k >= args.warmup:
            per_step.append(res)
    tot = sum(r["seconds"] for r in per_step)
    value = args.cpu_slices * len(per_step) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(per_step), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "nslice": wl.nslice, "npart": wl.npart,
                   "ngrid": wl.ngrid, "sampled_slices_per_step": args.cpu_slices},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": orc.num_threads(),
                         "kind": "port",
                         "sample": f"{args.cpu_slices} of {wl.nslice} slices per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
        return {"run_beam_step": 56 * N, "run_deposit_diag": 28 * N,
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

    def max_over_ranks(ms):
        if dist is None:
            return ms
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

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
        return max_over_ranks(e0.elapsed_time(e1))

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
    value = world * wl.nslice * K / (ms / 1e3)
    # per-kernel CUDA-event timing of the same kernels (direct launches)
    ctx.profile(True)
    kp = min(K, 30)
    ms_prof = timed(lambda: mx.run.advance(W + K, kp, graph=False))
    mixed_k = _stats(ctx.profile_read(), kernel_alg_bytes(wl, True), kp)
    ctx.profile(False)

    # mixed end to end: pinned host state -> steps -> host (state + diagnostics)
    e2e = None
    if not args.no_e2e:
        pin = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in parts.items()}
        pcells = torch.from_numpy(cells.view(np.float64)).pin_memory().numpy().view(np.complex128)
        hist = []

        def e2e_run():
            mx.upload(pin, pcells)
            mx.run.advance(0, K, graph=False)
            for i in range(K):
                hist.append(mx.run.history(i))
            mx.run.download_beam()
            mx.run.download_field(0)

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
    ctx.profile(True)
    ms64 = timed(lambda: [eng.step(lat, (W + k) % nstep) for k in range(K)])
    fp64_k = _stats(ctx.profile_read(), kernel_alg_bytes(wl, False), K)
    ctx.profile(False)
    value64 = world * wl.nslice * K / (ms64 / 1e3)
    del eng

    dom = max(mixed_k, key=lambda n: mixed_k[n]["ms_per_step"])
    peak, peak_kind = measured_peak()
    d = mixed_k[dom]
    roof = {"bound": "hbm", "kernel": dom, "achieved": d["gbs"], "peak": peak,
            "peak_source": peak_kind, "unit": "GB/s", "frac": d["gbs"] / peak,
            "traffic": None, "alg_bytes_per_launch": d["alg_bytes"],
            "timing": "CUDA events around each launch on the launching stream, "
                      f"{kp} direct-launch steps following the graph-timed region"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(wl, args.cpu_slices, args.cpu_steps, lat)
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
    run_ours(args, wl, rank, world)


if __name__ == "__main__":
    main()
