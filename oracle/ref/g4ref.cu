// g4ref.cu -- drives the reference's own CUDA classes (compiled unmodified
// from the reference tree, see oracle/ref/Makefile) on host arrays.
//
// TEST INFRASTRUCTURE ONLY: the outputs pin the FP64 oracle to the reference.
// The reference's Field/Beam constructors live in src/Core/Field.cpp and
// src/Core/Beam.cpp, which need the absent upstream GENESIS sources; the
// constructors below set the same members the reference's do
// (src/Core/Field.cpp:29-45 and :50-83 for the grid, src/Core/Beam.cpp) and
// nothing else.  The physical constants are the ones the oracle uses.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Beam.h"
#include "BeamSolverCUDA.h"
#include "ControlCUDA.h"
#include "DiagnosticCUDA.h"
#include "Field.h"
#include "FieldSolverADICUDA.h"
#include "FieldSolverFFTCUDA.h"
#include "Genesis4BeamSoA.h"
#include "Genesis4FieldSoA.h"
#include "TrackBeamCUDA.h"
#include "g4ref.h"
#include "mpi.h"

extern const double vacimp = 376.73031346177;
extern const double eev = 510998.95;
extern const double ce = 1.602176634e-19;
bool MPISingle = true;

// ---- single-process MPI: never reached with one rank and MPISingle --------
static int mpi_unreachable(const char* what) {
  throw std::runtime_error(std::string(what) + " called in the single-rank reference build");
}
int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return 0; }
int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return mpi_unreachable("MPI_Allreduce"); }
int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return mpi_unreachable("MPI_Send"); }
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return mpi_unreachable("MPI_Recv"); }
int MPI_Abort(MPI_Comm, int) { return mpi_unreachable("MPI_Abort"); }

// ---- the members of Field and Beam that the CUDA classes read -------------
Field::Field() {
  harm = 1;
  polarization = false;
  disabled = false;
  out_global = true;
  doFFT = doSpatial = doIntensity = doDumpField = true;
  accuslip = 0;
  in = out = nullptr;
  solver = nullptr;
  fieldSoA = new Genesis4FieldSoA();
}
Field::~Field() { delete fieldSoA; }
void Field::pack_field_to_soa() { throw std::runtime_error("Field::pack_field_to_soa: state is uploaded by the wrapper"); }
void Field::unpack_soa_to_field() { throw std::runtime_error("Field::unpack_soa_to_field is not part of this build"); }

Beam::Beam() {
  one4one = false;
  nbins = 4;
  useCudaSolver_ = true;
  beamSoA = new Genesis4BeamSoA();
}
Beam::~Beam() { delete beamSoA; }
void Beam::unpack_soa_to_beam() { throw std::runtime_error("Beam::unpack_soa_to_beam is not part of this build"); }

namespace {

thread_local std::string g_err;
Diagnostic g_diag;

int fail(const std::exception& e) {
  g_err = e.what();
  return -1;
}

void check(cudaError_t e, const char* where) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

// Undulator stand-in holding one lattice step (istep 0).
void load_step(Undulator& u, const g4b_step* st, int harm, double fc) {
  auto one = [](std::vector<double>& v, double x) { v.assign(1, x); };
  one(u.aw, st->aw); one(u.ax, st->ax); one(u.ay, st->ay); one(u.ku, st->ku);
  one(u.kx, st->kx); one(u.ky, st->ky); one(u.gradx, st->gradx); one(u.grady, st->grady);
  one(u.qf, st->qf); one(u.qx, st->dqx); one(u.qy, st->dqy);
  one(u.cx, st->cx); one(u.cy, st->cy);
  one(u.chic_angle, st->chic_angle); one(u.chic_lb, st->chic_lb);
  one(u.chic_ld, st->chic_ld); one(u.chic_lt, st->chic_lt);
  one(u.phasesh, st->autophase);
  u.marker.assign(1, 0);
  u.in_und.assign(1, st->in_undulator);
  u.gammaref = st->gamma_ref;
  u.istep = 0;
  if (harm > 0 && harm < 16) u.fc_by_harm[harm] = fc;
}

// Field::init's grid (src/Core/Field.cpp:50-83) + an uploaded SoA.
void load_field(Field& f, int nslice, int ngrid, double gridmax, double xlambda,
                int harm, int first, const double* cells) {
  f.harm = harm;
  f.xlambda = xlambda;
  f.ngrid = ngrid;
  f.gridmax = gridmax;
  f.dgrid = 2 * gridmax / static_cast<double>(ngrid - 1);
  f.xks = 4. * asin(1) / xlambda;
  f.first = first;
  f.slicelength = xlambda * harm;
  const size_t cells_n = static_cast<size_t>(nslice) * ngrid * ngrid;
  std::vector<double> re(cells_n), im(cells_n);
  for (size_t i = 0; i < cells_n; ++i) { re[i] = cells[2 * i]; im[i] = cells[2 * i + 1]; }
  Genesis4FieldSoA* s = f.fieldSoA;
  s->field_re.copy_from_host(re.data(), cells_n);
  s->field_im.copy_from_host(im.data(), cells_n);
  s->nslice = nslice;
  s->ngrid = ngrid;
  s->total_cells = static_cast<int>(cells_n);
  s->initialized = true;
}

void store_field(Field& f, double* cells) {
  Genesis4FieldSoA* s = f.fieldSoA;
  const size_t n = static_cast<size_t>(s->total_cells);
  std::vector<double> re(n), im(n);
  s->field_re.copy_to_host(re.data(), n);
  s->field_im.copy_to_host(im.data(), n);
  check(cudaStreamSynchronize(0), "synchronize");
  for (size_t i = 0; i < n; ++i) { cells[2 * i] = re[i]; cells[2 * i + 1] = im[i]; }
}

void load_beam(Beam& b, int nslice, const int* off, const double* x, const double* y,
               const double* px, const double* py, const double* gamma,
               const double* theta, const double* current) {
  const int n = off[nslice];
  Genesis4BeamSoA* s = b.beamSoA;
  std::vector<int> sid(n > 0 ? n : 1);
  for (int is = 0; is < nslice; ++is)
    for (int i = off[is]; i < off[is + 1]; ++i) sid[i] = is;
  std::vector<double> zero(n > 0 ? n : 1, 0.0);
  auto put = [&](CudaDeviceBuffer<double>& d, const double* h) {
    d.copy_from_host(h ? h : zero.data(), static_cast<size_t>(n > 0 ? n : 1));
  };
  put(s->x, x); put(s->y, y); put(s->px, px); put(s->py, py);
  put(s->gamma, gamma); put(s->theta, theta);
  s->slice_id.copy_from_host(sid.data(), sid.size());
  s->slice_offsets.copy_from_host(off, static_cast<size_t>(nslice + 1));
  s->nslice = nslice;
  s->total_particles = n;
  s->initialized = true;
  b.current.assign(current ? current : zero.data(), (current ? current : zero.data()) + nslice);
  b.current.resize(nslice, 0.0);
  b.longESC.assign(nslice, 0.0);
  b.eloss.assign(nslice, 0.0);
  // host slices sized as the device layout (BeamSolverCUDA's short-range
  // branch counts them, src/Core/BeamSolverCUDA.cpp:529-542); contents unused
  b.beam.resize(nslice);
  for (int is = 0; is < nslice; ++is) b.beam[is].resize(off[is + 1] - off[is]);
}

void fetch(CudaDeviceBuffer<double>& d, double* h, size_t n) {
  if (!h || n == 0) return;
  d.copy_to_host(h, n);
  check(cudaStreamSynchronize(0), "synchronize");
}

}  // namespace

extern "C" {

const char* g4ref_last_error(void) { return g_err.c_str(); }

int g4ref_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int g4ref_field_advance(int solver, int nslice, int ngrid, double gridmax, double xlambda,
                        int harm, int first, int enabled, int atomic_source, double delz,
                        double fc, const g4b_step* st, const int* off, const double* current,
                        const double* x, const double* y, const double* gamma,
                        const double* theta, double* cells, int filter, double xc, double yc,
                        double sig) {
  try {
    Undulator und;
    load_step(und, st, harm, fc);
    Field fld;
    load_field(fld, nslice, ngrid, gridmax, xlambda, harm, first, cells);
    if (!enabled) fld.disable(1.0);
    Beam beam;
    load_beam(beam, nslice, off, x, y, nullptr, nullptr, gamma, theta, current);
    std::unique_ptr<FieldSolver> s;
    if (solver == 0) s.reset(new FieldSolverADICUDA(atomic_source != 0));
    else s.reset(new FieldSolverFFTCUDA());
    s->initSourceFilter(xc, yc, sig, filter != 0);
    s->init(delz, fld.dgrid, fld.xks, static_cast<unsigned>(ngrid));
    s->advance(delz, &fld, &beam, &und);
    check(cudaGetLastError(), "field advance");
    store_field(fld, cells);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int g4ref_beam_advance(int nslice, const int* off, const g4b_step* st, int nfield,
                       const int* first, const int* ngrid, const int* harm,
                       const double* gridmax, const double* xlambda, const double* fc,
                       const double* const* cells, const double* longESC, const double* x,
                       const double* y, const double* px, const double* py, double* gamma,
                       double* theta) {
  try {
    Undulator und;
    load_step(und, st, 0, 0.0);
    std::vector<std::unique_ptr<Field>> owned;
    std::vector<Field*> fields;
    for (int i = 0; i < nfield; ++i) {
      owned.emplace_back(new Field());
      load_field(*owned.back(), nslice, ngrid[i], gridmax[i], xlambda[i], harm[i], first[i],
                 cells[i]);
      fields.push_back(owned.back().get());
      if (harm[i] > 0 && harm[i] < 16) und.fc_by_harm[harm[i]] = fc[i];
    }
    Beam beam;
    load_beam(beam, nslice, off, x, y, px, py, gamma, theta, nullptr);
    if (longESC) beam.longESC.assign(longESC, longESC + nslice);
    g4ref_sc::off = off;
    BeamSolverCUDA solver;
    solver.advance(st->delz, &beam, &fields, &und);
    check(cudaGetLastError(), "beam advance");
    const size_t n = static_cast<size_t>(off[nslice]);
    fetch(beam.beamSoA->gamma, gamma, n);
    fetch(beam.beamSoA->theta, theta, n);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

void g4ref_set_particle_ez(const double* ez) { g4ref_sc::field = ez; }

int g4ref_track(int npart, const g4b_step* st, double delz, int last_step, double* x,
                double* y, double* px, double* py, const double* gamma) {
  try {
    Undulator und;
    load_step(und, st, 0, 0.0);
    Beam beam;
    const int off[2] = {0, npart};
    load_beam(beam, 1, off, x, y, px, py, gamma, nullptr, nullptr);
    TrackBeamCUDA tracker;
    tracker.track(delz, &beam, &und, last_step != 0);
    check(cudaGetLastError(), "track");
    const size_t n = static_cast<size_t>(npart);
    fetch(beam.beamSoA->x, x, n);
    fetch(beam.beamSoA->y, y, n);
    fetch(beam.beamSoA->px, px, n);
    fetch(beam.beamSoA->py, py, n);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int g4ref_r56(int npart, const g4b_step* st, double lambda0, const double* gamma,
              double* theta) {
  try {
    Undulator und;
    load_step(und, st, 0, 0.0);
    Beam beam;
    const int off[2] = {0, npart};
    load_beam(beam, 1, off, nullptr, nullptr, nullptr, nullptr, gamma, theta, nullptr);
    TrackBeamCUDA tracker;
    tracker.applyR56(&beam, &und, lambda0);
    check(cudaGetLastError(), "r56");
    fetch(beam.beamSoA->theta, theta, static_cast<size_t>(npart));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int g4ref_slippage(int nslice, int ngrid, double slippage, double sample, int time_run,
                   int periodic, double* accuslip, int* first, double* cells) {
  try {
    Field fld;
    load_field(fld, nslice, ngrid, 1.0, 1.0, 1, *first, cells);
    fld.accuslip = *accuslip;
    ControlCUDA control;
    control.init(0, 1, time_run != 0, periodic != 0, sample);
    if (!control.applySlippage(slippage, &fld)) throw std::runtime_error("applySlippage declined");
    check(cudaGetLastError(), "slippage");
    store_field(fld, cells);
    *accuslip = fld.accuslip;
    *first = fld.first;
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int g4ref_diag(int nslice, const int* off, const double* x, const double* y, const double* px,
               const double* py, const double* gamma, const double* theta, int nharm,
               const double* current, const double* eloss, const double* longESC, int nfield,
               const int* ngrid, const int* first, const double* gridmax,
               const double* xlambda, double slicelength, const double* const* cells) {
  try {
    static const char* kBeamSlice[] = {
        "energy", "energyspread", "xposition", "xsize", "yposition", "ysize",
        "pxposition", "pyposition", "current", "emitx", "emity", "betax", "betay",
        "alphax", "alphay", "efield", "wakefield", "LSCfield", "SSCfield", "xmin", "xmax",
        "pxmin", "pxmax", "ymin", "ymax", "pymin", "pymax", "emin", "emax"};
    static const char* kBeamGlobal[] = {"Global/energy", "Global/energyspread",
                                        "Global/xposition", "Global/xsize",
                                        "Global/yposition", "Global/ysize"};
    static const char* kFieldSlice[] = {"power", "xposition", "xsize", "yposition", "ysize",
                                        "intensity-nearfield", "phase-nearfield",
                                        "intensity-farfield", "phase-farfield"};
    static const char* kFieldGlobal[] = {"Global/energy", "Global/xposition", "Global/xsize",
                                         "Global/yposition", "Global/ysize",
                                         "Global/intensity-nearfield",
                                         "Global/intensity-farfield", "dgrid", "gridspacing",
                                         "ngrid"};
    g_diag = Diagnostic();
    g_diag.zout.assign(1, 0.0);
    g_diag.val.resize(3 + nfield);
    auto& bm = g_diag.val[2];
    for (const char* k : kBeamSlice) bm[k].assign(nslice, 0.0);
    for (const char* k : kBeamGlobal) bm[k].assign(1, 0.0);
    for (int h = 1; h <= nharm; ++h) {
      const std::string b = h == 1 ? "bunching" : "bunching" + std::to_string(h);
      const std::string p = h == 1 ? "bunchingphase" : "bunchingphase" + std::to_string(h);
      bm[b].assign(nslice, 0.0);
      bm[p].assign(nslice, 0.0);
    }
    for (int i = 0; i < nfield; ++i) {
      auto& fm = g_diag.val[3 + i];
      for (const char* k : kFieldSlice) fm[k].assign(nslice, 0.0);
      for (const char* k : kFieldGlobal) fm[k].assign(1, 0.0);
    }
    Beam beam;
    load_beam(beam, nslice, off, x, y, px, py, gamma, theta, current);
    if (eloss) beam.eloss.assign(eloss, eloss + nslice);
    if (longESC) beam.longESC.assign(longESC, longESC + nslice);
    std::vector<std::unique_ptr<Field>> owned;
    std::vector<Field*> fields;
    for (int i = 0; i < nfield; ++i) {
      owned.emplace_back(new Field());
      load_field(*owned.back(), nslice, ngrid[i], gridmax[i], xlambda[i], 1, first[i], cells[i]);
      owned.back()->slicelength = slicelength;
      fields.push_back(owned.back().get());
    }
    FilterDiagnostics filter;
    filter.beam.harm = nharm;
    DiagnosticCUDA diag;
    diag.init(filter);
    if (!diag.calc(&beam, &fields, 0.0, g_diag)) throw std::runtime_error("calc declined");
    check(cudaGetLastError(), "diagnostics");
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int g4ref_time_steps(int nslice, const int* off, const double* x, const double* y,
                     const double* px, const double* py, const double* gamma,
                     const double* theta, const double* current, int ngrid, double gridmax,
                     double xlambda, const double* cells, int nstep, const g4b_step* steps,
                     const double* fc, const double* slip, double sample, int first_step,
                     int warmup, int ntimed, double* ms_per_step) {
  try {
    Beam beam;
    load_beam(beam, nslice, off, x, y, px, py, gamma, theta, current);
    beam.reflength = xlambda;
    Field fld;
    load_field(fld, nslice, ngrid, gridmax, xlambda, 1, 0, cells);
    fld.slicelength = xlambda * sample;
    std::vector<Field*> fields{&fld};
    BeamSolverCUDA solver;
    FieldSolverADICUDA adi(false);
    ControlCUDA control;
    control.init(0, 1, true, false, sample);
    FilterDiagnostics filter;
    DiagnosticCUDA diag;
    diag.init(filter);
    const int nout = warmup + ntimed;
    g_diag = Diagnostic();
    g_diag.zout.assign(nout, 0.0);
    g_diag.val.resize(4);
    static const char* kBeam[] = {
        "energy", "energyspread", "xposition", "xsize", "yposition", "ysize",
        "pxposition", "pyposition", "current", "emitx", "emity", "betax", "betay",
        "alphax", "alphay", "efield", "wakefield", "LSCfield", "SSCfield", "xmin", "xmax",
        "pxmin", "pxmax", "ymin", "ymax", "pymin", "pymax", "emin", "emax", "bunching",
        "bunchingphase"};
    static const char* kField[] = {"power", "xposition", "xsize", "yposition", "ysize",
                                   "intensity-nearfield", "phase-nearfield",
                                   "intensity-farfield", "phase-farfield"};
    for (const char* k : kBeam) g_diag.val[2][k].assign((size_t)nout * nslice, 0.0);
    for (const char* k : {"Global/energy", "Global/energyspread", "Global/xposition",
                          "Global/xsize", "Global/yposition", "Global/ysize"})
      g_diag.val[2][k].assign(nout, 0.0);
    for (const char* k : kField) g_diag.val[3][k].assign((size_t)nout * nslice, 0.0);
    for (const char* k : {"Global/energy", "Global/xposition", "Global/xsize",
                          "Global/yposition", "Global/ysize", "Global/intensity-nearfield",
                          "Global/intensity-farfield", "dgrid", "gridspacing", "ngrid"})
      g_diag.val[3][k].assign(nout, 0.0);
    cudaEvent_t t0, t1;
    check(cudaEventCreate(&t0), "event");
    check(cudaEventCreate(&t1), "event");
    double z = 0.0;
    for (int k = 0; k < nout; ++k) {
      if (k == warmup) {
        check(cudaDeviceSynchronize(), "synchronize");
        check(cudaEventRecord(t0, 0), "event");
      }
      const int i = (first_step + k) % nstep;
      const g4b_step& st = steps[i];
      Undulator und;
      load_step(und, &st, 1, fc[i]);
      const double delz = st.delz;
      // Gencore::run's step (src/Core/Gencore.cpp:172-254) with Beam::track's
      // CUDA branch (src/Core/Beam.cpp:117-134) and Field::track
      solver.track(delz * 0.5, &beam, &und, false);
      solver.advance(delz, &beam, &fields, &und);
      solver.applyR56(&beam, &und, xlambda);
      solver.track(delz * 0.5, &beam, &und, true);
      adi.init(delz, fld.dgrid, fld.xks, static_cast<unsigned>(ngrid));
      adi.advance(delz, &fld, &beam, &und);
      if (!control.applySlippage(slip[i], &fld)) throw std::runtime_error("applySlippage declined");
      z += delz;
      if (!diag.calc(&beam, &fields, z, g_diag)) throw std::runtime_error("calc declined");
    }
    check(cudaEventRecord(t1, 0), "event");
    check(cudaEventSynchronize(t1), "synchronize");
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, t0, t1), "elapsed");
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    *ms_per_step = ntimed > 0 ? (double)ms / ntimed : 0.0;
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int g4ref_diag_record(int group, const char* name, double* out, int cap) {
  const int idx = group == 0 ? 2 : 2 + group;
  if (idx >= static_cast<int>(g_diag.val.size())) return -1;
  auto it = g_diag.val[idx].find(name);
  if (it == g_diag.val[idx].end()) return -1;
  const int n = static_cast<int>(it->second.size());
  for (int i = 0; i < n && i < cap; ++i) out[i] = it->second[i];
  return n;
}

}  // extern "C"
