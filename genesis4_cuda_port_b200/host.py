"""ctypes binding of the host layer's C ABI (include/g4h.h): beam/field
loading and lattice expansion into per-step undulator tables."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import G4BError, Step, dptr

_HOSTLIB = Path(__file__).resolve().parent / "lib" / "libg4host.so"


class BeamSpec(C.Structure):
    """Mirror of ``g4h_beam_spec``."""

    _fields_ = [("nslice", C.c_int), ("npart", C.c_int), ("nbins", C.c_int),
                ("shotnoise", C.c_int), ("seed", C.c_uint64),
                ("gamma0", C.c_double), ("delgam", C.c_double), ("ex", C.c_double),
                ("ey", C.c_double), ("betax", C.c_double), ("betay", C.c_double),
                ("alphax", C.c_double), ("alphay", C.c_double),
                ("xcenter", C.c_double), ("ycenter", C.c_double),
                ("pxcenter", C.c_double), ("pycenter", C.c_double),
                ("reflength", C.c_double), ("slicelength", C.c_double)]

    def __init__(self, **kw):
        super().__init__()
        for k, v in kw.items():
            setattr(self, k, v)


class DeckSummary(C.Structure):
    """Mirror of ``g4h_deck_summary``."""

    _fields_ = [("nslice", C.c_int), ("npart", C.c_int), ("nstep", C.c_int),
                ("nfield", C.c_int), ("harm", C.c_int * 8), ("ngrid", C.c_int * 8),
                ("gridmax", C.c_double * 8), ("lambda0", C.c_double),
                ("gamma0", C.c_double), ("sample", C.c_double), ("time_run", C.c_int),
                ("periodic", C.c_int), ("precision", C.c_int), ("low_memory", C.c_int),
                ("output_step", C.c_int), ("nout", C.c_int), ("bunchharm", C.c_int),
                ("nrun", C.c_int), ("betax", C.c_double), ("alphax", C.c_double),
                ("betay", C.c_double), ("alphay", C.c_double), ("current", C.c_double),
                ("zend", C.c_double)]


_h = None


def load():
    global _h
    if _h is not None:
        return _h
    _lib.load()  # resolves libg4b200.so first
    if not _HOSTLIB.exists():
        raise RuntimeError(f"{_HOSTLIB} is missing: build it with "
                           "`python -m genesis4_cuda_port_b200.build`")
    h = C.CDLL(str(_HOSTLIB))
    h.g4h_last_error.restype = C.c_char_p
    h.g4h_load_beam.argtypes = [C.POINTER(BeamSpec), _lib.c_double_p] + \
        [_lib.c_double_p] * 6 + [_lib.c_int64_p]
    h.g4h_gaussian_field.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double,
                                     C.c_double, _lib.c_double_p]
    h.g4h_lattice_parse.argtypes = [C.c_char_p, C.c_char_p, C.c_double, C.c_double,
                                    C.c_double, _lib.c_void_pp]
    h.g4h_lattice_destroy.argtypes = [C.c_void_p]
    h.g4h_lattice_nstep.argtypes = [C.c_void_p, _lib.c_int_p]
    h.g4h_lattice_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(Step),
                                   _lib.c_double_p, _lib.c_double_p, _lib.c_int_p]
    h.g4h_lattice_fc.argtypes = [C.c_void_p, C.c_int, C.c_int, _lib.c_double_p]
    h.g4h_coupling.restype = C.c_double
    h.g4h_coupling.argtypes = [C.c_double, C.c_int, C.c_int]
    h.g4h_deck_parse.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _lib.c_void_pp]
    h.g4h_deck_destroy.argtypes = [C.c_void_p]
    h.g4h_deck_info.argtypes = [C.c_void_p, C.POINTER(DeckSummary)]
    h.g4h_deck_run.argtypes = [C.c_void_p, _lib.c_void_pp]
    h.g4h_result_destroy.argtypes = [C.c_void_p]
    h.g4h_result_info.argtypes = [C.c_void_p, _lib.c_int_p, _lib.c_int_p, _lib.c_int_p,
                                  _lib.c_int_p, _lib.c_double_p]
    h.g4h_result_keys.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_int, _lib.c_int_p]
    h.g4h_result_get.argtypes = [C.c_void_p, C.c_int, C.c_char_p, _lib.c_double_p,
                                 C.c_int64, _lib.c_int64_p]
    h.g4h_result_field.argtypes = [C.c_void_p, C.c_int, _lib.c_double_p, _lib.c_int_p]
    h.g4h_result_output_file.argtypes = [C.c_void_p, C.c_char_p, C.c_int, _lib.c_int_p]
    h.g4h_file_list.argtypes = [C.c_char_p, C.c_char_p, C.c_int, _lib.c_int_p]
    h.g4h_file_read.argtypes = [C.c_char_p, C.c_char_p, _lib.c_double_p, C.c_int64,
                                _lib.c_int64_p, _lib.c_int_p, _lib.c_int64_p]
    _h = h
    return h


def _check(rc):
    if rc != 0:
        raise G4BError(rc, load().g4h_last_error().decode())


def library_path() -> Path:
    return _HOSTLIB


def load_beam(spec: BeamSpec, current):
    """Quiet-start (+ shot noise) beam: returns (slice_offsets, parts dict)."""
    n = spec.nslice * spec.npart
    parts = {k: np.empty(n) for k in ("x", "y", "px", "py", "gamma", "theta")}
    off = np.empty(spec.nslice + 1, np.int64)
    cur = np.ascontiguousarray(np.broadcast_to(current, (spec.nslice,)), np.float64)
    _check(load().g4h_load_beam(C.byref(spec), dptr(cur),
                                *[dptr(parts[k]) for k in ("x", "y", "px", "py", "gamma", "theta")],
                                off.ctypes.data_as(_lib.c_int64_p)))
    return off, parts


def gaussian_field(ngrid, gridmax, xlambda, power, w0):
    out = np.empty((ngrid, ngrid), np.complex128)
    _check(load().g4h_gaussian_field(ngrid, gridmax, xlambda, power, w0,
                                     dptr(out.reshape(-1).view(np.float64))))
    return out


def coupling(aw, harm=1, helical=False):
    return float(load().g4h_coupling(aw, harm, int(helical)))


class Lattice:
    """A .lat beamline expanded into per-step tables (upstream Undulator)."""

    def __init__(self, text: str, beamline: str, delz: float, gamma0: float, lambda0: float):
        h = C.c_void_p()
        _check(load().g4h_lattice_parse(text.encode(), beamline.encode(), delz, gamma0,
                                        lambda0, C.byref(h)))
        self.h = h
        n = C.c_int()
        _check(load().g4h_lattice_nstep(h, C.byref(n)))
        self.nstep = n.value
        self.steps, self.slip, self.z, self.marker = [], [], [], []
        for i in range(self.nstep):
            st, sl, z, m = Step(), C.c_double(), C.c_double(), C.c_int()
            _check(load().g4h_lattice_step(h, i, C.byref(st), C.byref(sl), C.byref(z),
                                           C.byref(m)))
            self.steps.append(st)
            self.slip.append(sl.value)
            self.z.append(z.value)
            self.marker.append(m.value)

    def fc(self, i: int, harm: int = 1) -> float:
        v = C.c_double()
        _check(load().g4h_lattice_fc(self.h, i, harm, C.byref(v)))
        return v.value

    def __del__(self):
        try:
            if getattr(self, "h", None):
                load().g4h_lattice_destroy(self.h)
                self.h = None
        except Exception:
            pass


class Deck:
    """An input deck (.in namelists + .lat beamline), parsed and expanded on
    the host; ``run()`` executes its &track on the GPU (Gencore::run with the
    CUDA classes, or the fused mixed-precision run for ``precision = mixed``)."""

    def __init__(self, text: str, lattice: str | None = None, base_dir: str | None = None):
        h = C.c_void_p()
        _check(load().g4h_deck_parse(text.encode(), lattice.encode() if lattice is not None
                                     else None, (base_dir or "").encode(), C.byref(h)))
        self.h = h
        s = DeckSummary()
        _check(load().g4h_deck_info(h, C.byref(s)))
        self.summary = s

    @classmethod
    def from_file(cls, path: str):
        p = Path(path)
        return cls(p.read_text(), None, str(p.parent))

    def info(self) -> dict:
        s = self.summary
        d = {k: getattr(s, k) for k, _ in DeckSummary._fields_ }
        for k in ("harm", "ngrid", "gridmax"):
            d[k] = list(d[k])[: s.nfield]
        return d

    def run(self) -> "Result":
        r = C.c_void_p()
        _check(load().g4h_deck_run(self.h, C.byref(r)))
        return Result(r)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                load().g4h_deck_destroy(self.h)
                self.h = None
        except Exception:
            pass


class Result:
    """Diagnostics of one deck run: ``beam[key]`` and ``field[i][key]`` are
    arrays shaped (nz, nslice) for per-slice records and (nz,) for Global/
    records, as DiagnosticCUDA::calcBeam / calcField fill them."""

    def __init__(self, h):
        self.h = h
        nz, ns, nf, nst, sec = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_double()
        _check(load().g4h_result_info(h, C.byref(nz), C.byref(ns), C.byref(nf), C.byref(nst),
                                      C.byref(sec)))
        self.nz, self.nslice, self.nfield = nz.value, ns.value, nf.value
        self.nsteps, self.seconds = nst.value, sec.value
        self.z = self._get(-1, "z")
        self.beam = self._group(0)
        self.field = [self._group(i + 1) for i in range(self.nfield)]

    def _get(self, group, key):
        n = C.c_int64()
        _check(load().g4h_result_get(self.h, group, key.encode(), None, 0, C.byref(n)))
        out = np.empty(n.value)
        _check(load().g4h_result_get(self.h, group, key.encode(), dptr(out), n.value, None))
        if group < 0 or key.startswith("Global/") or key in ("dgrid", "gridspacing", "ngrid"):
            return out
        return out.reshape(self.nz, self.nslice)

    def _group(self, g):
        need = C.c_int()
        _check(load().g4h_result_keys(self.h, g, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value)
        _check(load().g4h_result_keys(self.h, g, buf, need.value, None))
        return {k: self._get(g, k) for k in buf.value.decode().split("\n") if k}

    @property
    def output_file(self) -> str:
        """Path of the run's G4DS output file ("" when none was written)."""
        need = C.c_int()
        _check(load().g4h_result_output_file(self.h, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value)
        _check(load().g4h_result_output_file(self.h, buf, need.value, None))
        return buf.value.decode()

    def final_field(self, i: int = 0):
        ngrid = int(self.field[i]["ngrid"][0])
        out = np.empty((self.nslice, ngrid, ngrid), np.complex128)
        first = C.c_int()
        _check(load().g4h_result_field(self.h, i, dptr(out.reshape(-1).view(np.float64)),
                                       C.byref(first)))
        return out, first.value

    def __del__(self):
        try:
            if getattr(self, "h", None):
                load().g4h_result_destroy(self.h)
                self.h = None
        except Exception:
            pass


# ---- many runs on one GPU: batched scan and served stream -------------------

class Job(C.Structure):
    """Mirror of ``g4h_job``: one mixed-precision FEL run."""

    _fields_ = [("nslice", C.c_int), ("npart", C.c_int), ("ngrid", C.c_int),
                ("nsteps", C.c_int), ("shotnoise", C.c_int), ("time_run", C.c_int),
                ("seed", C.c_uint64), ("gridmax", C.c_double), ("gamma", C.c_double),
                ("delgam", C.c_double), ("emit", C.c_double), ("beta", C.c_double),
                ("current", C.c_double), ("seed_power", C.c_double), ("waist", C.c_double),
                ("taper", C.c_double)]


class EngineConfig(C.Structure):
    """Mirror of ``g4h_engine_config``."""

    _fields_ = [("lattice", C.c_char_p), ("beamline", C.c_char_p), ("delz", C.c_double),
                ("gamma_ref", C.c_double), ("lambda0", C.c_double), ("max_runs", C.c_int),
                ("use_graph", C.c_int), ("tune", C.c_int), ("mode", C.c_int),
                ("threads", C.c_int), ("reserve_bytes", C.c_double)]


class ScanResult(C.Structure):
    _fields_ = [("value", C.c_double), ("seconds", C.c_double), ("slice_steps", C.c_double),
                ("device_bytes", C.c_double), ("njobs", C.c_int), ("grids", C.c_int * 4),
                ("layouts_16", C.c_int), ("layouts_switched", C.c_int)]


class ServeStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("p50", C.c_double), ("p99", C.c_double),
                ("mean", C.c_double), ("requests_per_s", C.c_double),
                ("slice_steps", C.c_double), ("slice_steps_per_s", C.c_double),
                ("batch_steps", C.c_double), ("peak_concurrency", C.c_int),
                ("reserved", C.c_int)]


def _bind_engine(h):
    h.g4h_scan.argtypes = [C.POINTER(EngineConfig), C.POINTER(Job), C.c_int,
                           C.POINTER(ScanResult), _lib.c_double_p, _lib.c_double_p]
    h.g4h_serve.argtypes = [C.POINTER(EngineConfig), C.POINTER(Job), _lib.c_double_p, C.c_int,
                            _lib.c_double_p, _lib.c_double_p, _lib.c_double_p,
                            C.POINTER(ServeStats)]


def engine_config(lattice: str, beamline: str, delz: float, gamma_ref: float, lambda0: float,
                  max_runs: int = 256, graph: bool = True, tune: int = 1, mode: int = 0,
                  threads: int = 0, reserve_bytes: float = 4e9) -> EngineConfig:
    """tune: 0 off, 1 launch shapes, 2 ADI row layouts and launch shapes."""
    c = EngineConfig()
    c._keep = (lattice.encode(), beamline.encode())
    c.lattice, c.beamline = c._keep
    c.delz, c.gamma_ref, c.lambda0 = delz, gamma_ref, lambda0
    c.max_runs, c.use_graph, c.tune, c.mode = max_runs, int(graph), int(tune), mode
    c.threads, c.reserve_bytes = threads, reserve_bytes
    return c


def _jobs_array(jobs):
    arr = (Job * len(jobs))()
    for i, j in enumerate(jobs):
        arr[i] = j
    return arr


def scan(cfg: EngineConfig, jobs, records: bool = False):
    """Run every job to its end (batched for cfg.mode 0); returns
    (ScanResult, final power per job [W], raw last-step records or None)."""
    h = load()
    _bind_engine(h)
    arr = _jobs_array(jobs)
    res = ScanResult()
    power = np.empty(len(jobs))
    rec = np.empty(sum(j.nslice for j in jobs) * 34) if records else None
    _check(h.g4h_scan(C.byref(cfg), arr, len(jobs), C.byref(res), dptr(power),
                      dptr(rec) if rec is not None else None))
    return res, power, rec


def serve(cfg: EngineConfig, jobs, arrival, records: bool = False):
    """Served stream: returns (ServeStats, latency [s], final power [W],
    raw last-step records or None)."""
    h = load()
    _bind_engine(h)
    arr = _jobs_array(jobs)
    arrival = np.ascontiguousarray(arrival, np.float64)
    lat = np.empty(len(jobs))
    power = np.empty(len(jobs))
    rec = np.empty(sum(j.nslice for j in jobs) * 34) if records else None
    st = ServeStats()
    _check(h.g4h_serve(C.byref(cfg), arr, dptr(arrival), len(jobs), dptr(lat), dptr(power),
                       dptr(rec) if rec is not None else None, C.byref(st)))
    return st, lat, power, rec


# ---- G4DS files (output records and dumps) ------------------------------------

def read_g4ds(path) -> dict:
    """Every dataset of a G4DS file (the format written by the host layer for
    its output records and marker dumps; described in include/g4h.h) as
    {name: float64 array shaped by its dimensions}.  Pure Python."""
    import struct
    data = Path(path).read_bytes()
    if data[:8] != b"G4DS\x00\x00\x00\x01":
        raise ValueError(f"{path} is not a G4DS file")
    (count,) = struct.unpack_from("<Q", data, 8)
    pos, out = 16, {}
    for _ in range(count):
        (nl,) = struct.unpack_from("<I", data, pos)
        name = data[pos + 4:pos + 4 + nl].decode()
        pos += 4 + nl
        typ, rank = struct.unpack_from("<II", data, pos)
        pos += 8
        dims = struct.unpack_from(f"<{rank}Q", data, pos)
        pos += 8 * rank
        n = int(np.prod(dims)) if rank else 1
        arr = np.frombuffer(data, dtype="<f8" if typ == 0 else "<i8", count=n, offset=pos)
        out[name] = arr.reshape(dims).copy()
        pos += 8 * n
    return out


def file_dataset(path, name) -> np.ndarray:
    """One dataset through the host library's reader (g4h_file_read)."""
    n = C.c_int64()
    rank = C.c_int()
    dims = (C.c_int64 * 8)()
    _check(load().g4h_file_read(str(path).encode(), name.encode(), None, 0, C.byref(n),
                                C.byref(rank), dims))
    out = np.empty(n.value)
    _check(load().g4h_file_read(str(path).encode(), name.encode(), dptr(out), n.value, None,
                                None, None))
    return out.reshape([dims[i] for i in range(rank.value)])
