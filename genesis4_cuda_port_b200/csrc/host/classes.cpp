// classes.cpp -- Field, Beam, solvers and slippage over the g4b C ABI.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "g4file.h"
#include "g4h_internal.h"
#include "genesis4.h"

namespace g4h {

const double vacimp = 376.73031346177;
const double eev = 510998.95;
const double ce = 1.602176634e-19;

void check(int rc, const char* where) {
  if (rc != G4B_OK) throw std::runtime_error(std::string(where) + ": " + g4b_last_error());
}

g4b_ctx* cuda_context() {
  static g4b_ctx* ctx = nullptr;
  static std::mutex m;
  std::lock_guard<std::mutex> lock(m);
  if (!ctx) check(g4b_ctx_create(0, &ctx), "genesis4_cuda::initialize");
  return ctx;
}

// ------------------------------------------------------- FieldSolverADICUDA --
FieldSolverADICUDA::FieldSolverADICUDA(bool atomic_source) : atomic_source_(atomic_source) {
  check(g4b_adi_create(cuda_context(), &adi_), "FieldSolverADICUDA");
}

FieldSolverADICUDA::~FieldSolverADICUDA() { g4b_adi_destroy(adi_); }

// FieldSolverADICUDA::init (src/Core/FieldSolverADICUDA.cpp:821-902): the
// library recomputes only when delz or ngrid change.
void FieldSolverADICUDA::init(double delz, double dgrid, double xks, unsigned int ngrid) {
  check(g4b_adi_init(adi_, delz, dgrid, xks, (int)ngrid), "FieldSolverADICUDA::init");
}

// FieldSolverADICUDA::advance (src/Core/FieldSolverADICUDA.cpp:638-818)
void FieldSolverADICUDA::advance(double, Field* field, Beam* beam, Undulator* und) {
  if (!field || !beam || !und)
    throw std::runtime_error("FieldSolverADICUDA::advance received a null field/beam/undulator pointer");
  if (!field->fieldSoA) field->pack_field_to_soa();
  if (!beam->beamSoA) beam->pack_beam_to_soa();
  check(g4b_field_set_first(field->fieldSoA, field->first), "FieldSolverADICUDA::advance");
  const int harm = field->getHarm();
  check(g4b_adi_advance(adi_, field->fieldSoA, beam->beamSoA, &und->current(), und->fc(harm),
                        field->isEnabled() ? 1 : 0),
        "FieldSolverADICUDA::advance");
}

// ------------------------------------------------------- FieldSolverFFTCUDA --
FieldSolverFFTCUDA::FieldSolverFFTCUDA() {
  check(g4b_fft_create(cuda_context(), &fft_), "FieldSolverFFTCUDA");
}

FieldSolverFFTCUDA::~FieldSolverFFTCUDA() { g4b_fft_destroy(fft_); }

// FieldSolverFFTCUDA::initSourceFilter (src/Core/FieldSolverFFTCUDA.cpp:214-222)
void FieldSolverFFTCUDA::initSourceFilter(double xc, double yc, double sig, bool filter) {
  check(g4b_fft_init_filter(fft_, xc, yc, sig, filter ? 1 : 0),
        "FieldSolverFFTCUDA::initSourceFilter");
}

// FieldSolverFFTCUDA::init (src/Core/FieldSolverFFTCUDA.cpp:246-293)
void FieldSolverFFTCUDA::init(double delz, double dgrid, double xks, unsigned int ngrid) {
  check(g4b_fft_init(fft_, delz, dgrid, xks, (int)ngrid), "FieldSolverFFTCUDA::init");
}

// FieldSolverFFTCUDA::advance (src/Core/FieldSolverFFTCUDA.cpp:295-483)
void FieldSolverFFTCUDA::advance(double, Field* field, Beam* beam, Undulator* und) {
  if (!field || !beam || !und)
    throw std::runtime_error(
        "FieldSolverFFTCUDA::advance_gpu received a null field/beam/undulator pointer");
  if (!field->fieldSoA) field->pack_field_to_soa();
  if (!beam->beamSoA) beam->pack_beam_to_soa();
  check(g4b_field_set_first(field->fieldSoA, field->first), "FieldSolverFFTCUDA::advance");
  const int harm = field->getHarm();
  check(g4b_fft_advance(fft_, field->fieldSoA, beam->beamSoA, &und->current(), und->fc(harm),
                        field->isEnabled() ? 1 : 0),
        "FieldSolverFFTCUDA::advance");
}

// -------------------------------------------------------------------- Field --
Field::Field() = default;

Field::~Field() {
  if (fieldSoA) g4b_field_destroy(fieldSoA);
}

// Field::init (src/Core/Field.cpp:50-83): dgrid_in is the grid half width
void Field::init(int nsize, int ngrid_in, double dgrid_in, double xlambda0, double slicelen,
                 double s0_in, int harm_in) {
  slicelength = slicelen;
  s0 = s0_in;
  harm = harm_in;
  rharm = harm_in;
  xlambda = xlambda0 / (double)harm;
  ngrid = ngrid_in;
  gridmax = dgrid_in;
  dgrid = 2 * gridmax / (double)(ngrid - 1);
  field.assign(nsize, std::vector<std::complex<double>>((size_t)ngrid * ngrid));
  xks = 4. * std::asin(1.) / xlambda;
  first = 0;
  dz_save = 0;
  accuslip = 0;
}

// Field::initSolver (src/Core/Field.cpp:87-110): the CUDA FFT solver (with
// its source filter) or the CUDA ADI solver; the upstream CPU solvers are not
// part of this build.
void Field::initSolver(bool isFFT, bool filter, double xc, double yc, double sig,
                       bool use_cuda, bool low_memory_adisolver) {
  if (!use_cuda)
    throw std::runtime_error(
        "Field::initSolver: use_cuda=false selects the upstream CPU solvers, which this "
        "build does not contain");
  low_memory_ = low_memory_adisolver;
  if (isFFT) {
    solver.reset(new FieldSolverFFTCUDA());
    solver->initSourceFilter(xc, yc, sig, filter);
  } else {
    solver.reset(new FieldSolverADICUDA(low_memory_adisolver));
  }
}

void Field::disable(double conv) {  // include/Field.h:117-125
  if (!disabled) rharm = harm;
  rharm *= conv;
  disabled = true;
}

// Field::track (src/Core/Field.cpp:204-212)
void Field::track(double delz, Beam* beam, Undulator* und) {
  if (!solver) throw std::runtime_error("Field::track: initSolver was not called");
  solver->init(delz, dgrid, xks, ngrid);
  solver->advance(delz, this, beam, und);
}

void Field::init_fieldSoA() {
  if (fieldSoA) return;
  check(g4b_field_create(cuda_context(), (int)field.size(), ngrid, gridmax, xlambda,
                         harm, G4B_FP64, low_memory_ ? 1 : 0, &fieldSoA),
        "Field::init_fieldSoA");
}

void Field::pack_field_to_soa() {  // src/Core/Field.cpp:598-634
  init_fieldSoA();
  std::vector<double> host(2 * field.size() * (size_t)ngrid * ngrid);
  for (size_t s = 0; s < field.size(); ++s)
    std::memcpy(host.data() + 2 * s * ngrid * ngrid, field[s].data(),
                sizeof(double) * 2 * ngrid * ngrid);
  check(g4b_field_upload(fieldSoA, host.data()), "Field::pack_field_to_soa");
  check(g4b_field_set_first(fieldSoA, first), "Field::pack_field_to_soa");
}

void Field::unpack_soa_to_field() {  // src/Core/Field.cpp:636-674
  if (!fieldSoA) return;
  std::vector<double> host(2 * field.size() * (size_t)ngrid * ngrid);
  check(g4b_field_download(fieldSoA, host.data()), "Field::unpack_soa_to_field");
  for (size_t s = 0; s < field.size(); ++s)
    std::memcpy(field[s].data(), host.data() + 2 * s * ngrid * ngrid,
                sizeof(double) * 2 * ngrid * ngrid);
}

// --------------------------------------------------------------------- Beam --
Beam::Beam() = default;

Beam::~Beam() {
  if (beamSoA) g4b_beam_destroy(beamSoA);
}

void Beam::init(int nsize, int nbins_in, double reflen, double slicelen, double s0_in,
                bool one4one_in) {  // src/Core/Beam.cpp:36-53
  nbins = nbins_in;
  reflength = reflen;
  slicelength = slicelen;
  s0 = s0_in;
  one4one = one4one_in;
  current.assign(nsize, 0.0);
  eloss.assign(nsize, 0.0);
  longESC.assign(nsize, 0.0);
  beam.assign(nsize, {});
}

void Beam::init_beamSoA() {  // src/Core/Beam.cpp:342-390
  if (beamSoA) return;
  std::vector<int64_t> off(beam.size() + 1, 0);
  for (size_t s = 0; s < beam.size(); ++s) off[s + 1] = off[s] + (int64_t)beam[s].size();
  check(g4b_beam_create(cuda_context(), (int)beam.size(), off.data(), G4B_FP64, gamma_ref,
                        &beamSoA),
        "Beam::init_beamSoA");
}

void Beam::pack_beam_to_soa() {  // src/Core/Beam.cpp:392-455
  init_beamSoA();
  size_t n = 0;
  for (auto& s : beam) n += s.size();
  std::vector<double> x(n), y(n), px(n), py(n), g(n), th(n);
  size_t k = 0;
  for (auto& s : beam)
    for (auto& p : s) {
      x[k] = p.x;
      y[k] = p.y;
      px[k] = p.px;
      py[k] = p.py;
      g[k] = p.gamma;
      th[k] = p.theta;
      ++k;
    }
  check(g4b_beam_upload(beamSoA, x.data(), y.data(), px.data(), py.data(), g.data(), th.data()),
        "Beam::pack_beam_to_soa");
  check(g4b_beam_set_current(beamSoA, current.data()), "Beam::pack_beam_to_soa");
  // BeamSolverCUDA::advance slice energy loss -longESC/511000
  // (src/Core/BeamSolverCUDA.cpp:549-560)
  std::vector<double> el(beam.size());
  for (size_t s = 0; s < beam.size(); ++s) el[s] = -longESC[s] / 511000.0;
  check(g4b_beam_set_eloss(beamSoA, el.data()), "Beam::pack_beam_to_soa");
}

void Beam::unpack_soa_to_beam() {  // src/Core/Beam.cpp:457-525
  if (!beamSoA) return;
  size_t n = 0;
  for (auto& s : beam) n += s.size();
  std::vector<double> x(n), y(n), px(n), py(n), g(n), th(n);
  check(g4b_beam_download(beamSoA, x.data(), y.data(), px.data(), py.data(), g.data(),
                          th.data()),
        "Beam::unpack_soa_to_beam");
  size_t k = 0;
  for (auto& s : beam)
    for (auto& p : s) {
      p.x = x[k];
      p.y = y[k];
      p.px = px[k];
      p.py = py[k];
      p.gamma = g[k];
      p.theta = th[k];
      ++k;
    }
}

void Incoherent::apply(Beam* beam, Undulator* und, double delz) {
  if (!spread_ && !loss_) return;
  check(g4b_beam_incoherent(beam->beamSoA, &und->current(), delz, und->isHelical() ? 1 : 0,
                            loss_ ? 1 : 0, spread_ ? 1 : 0, seed_, counter_++),
        "Incoherent::apply");
}

// Beam::track, CUDA branch (src/Core/Beam.cpp:111-134): incoherent
// synchrotron radiation on the device state after the push; wakes
// (col.apply) reach the push as the slice loss.
void Beam::track(double delz, std::vector<Field*>* field, Undulator* und) {
  for (auto* f : *field) f->setStepsize(delz);
  if (!useCudaSolver_)
    throw std::runtime_error("Beam::track: the upstream CPU beam solver is not in this build");
  if (!beamSoA) pack_beam_to_soa();
  cuda_solver.track(delz * 0.5, this, und, false);
  cuda_solver.advance(delz, this, field, und);
  incoherent.apply(this, und, delz);
  cuda_solver.applyR56(this, und, reflength);
  cuda_solver.track(delz * 0.5, this, und, true);
}

// ------------------------------------------------------ BeamSolver / Track --
void TrackBeamCUDA::track(double delz, Beam* beam, Undulator* und, bool last) {
  check(g4b_beam_track(beam->beamSoA, &und->current(), delz, last ? 1 : 0),
        "TrackBeamCUDA::track");
}

void TrackBeamCUDA::applyR56(Beam* beam, Undulator* und, double lambda0) {
  check(g4b_beam_r56(beam->beamSoA, &und->current(), lambda0), "TrackBeamCUDA::applyR56");
}

BeamSolverCUDA::~BeamSolverCUDA() { g4b_efield_destroy(efield); }

void BeamSolverCUDA::initEField(double rmax, int ngrid, int nz, int nphi, double lambda,
                                bool longr) {
  if (longr)
    throw std::runtime_error("BeamSolverCUDA::initEField: long-range space charge is not built");
  g4b_efield_destroy(efield);
  efield = nullptr;
  check(g4b_efield_create(cuda_context(), rmax, ngrid, nz, nphi, lambda, &efield),
        "BeamSolverCUDA::initEField");
}

// BeamSolverCUDA::advance (src/Core/BeamSolverCUDA.cpp:449-683)
void BeamSolverCUDA::advance(double, Beam* beam, std::vector<Field*>* field, Undulator* und) {
  if (!beam || !field || !und)
    throw std::runtime_error("BeamSolverCUDA::advance received a null beam/field/undulator pointer");
  std::vector<g4b_field*> fl;
  std::vector<double> fc;
  for (Field* f : *field) {
    if (!f) continue;
    if (f->getHarm() != 1 && onlyFundamental) continue;
    if (!f->fieldSoA) f->pack_field_to_soa();
    check(g4b_field_set_first(f->fieldSoA, f->first), "BeamSolverCUDA::advance");
    fl.push_back(f->fieldSoA);
    fc.push_back(und->fc(f->getHarm()));
  }
  if (fl.size() > 8) throw std::runtime_error("BeamSolverCUDA::advance exceeds kMaxBeamSolverFields");
  // short-range space charge: per-particle loss before the push
  // (src/Core/BeamSolverCUDA.cpp:519-547)
  if (g4b_efield_has_short_range(efield)) {
    const g4b_step& st = und->current();
    const double gammaz2 = st.gamma_ref * st.gamma_ref / (1.0 + st.aw * st.aw);
    check(g4b_efield_short_range(efield, beam->beamSoA, gammaz2), "BeamSolverCUDA::advance");
  }
  check(g4b_beam_advance(beam->beamSoA, fl.data(), fc.data(), (int)fl.size(), &und->current()),
        "BeamSolverCUDA::advance");
}

// --------------------------------------------------------------- ControlCUDA --
void ControlCUDA::init(int rank, int size, bool isTime, bool periodic, double sample) {
  rank_ = rank;
  size_ = size;
  timerun_ = isTime;
  periodic_ = periodic;
  sample_ = sample;
}

// ControlCUDA::applySlippage (src/Core/ControlCUDA.cpp:148-252), one rank
bool ControlCUDA::applySlippage(double slippage, Field* field) {
  if (!timerun_) return true;
  if (!field || !field->fieldSoA) return false;
  check(g4b_field_set_first(field->fieldSoA, field->first), "ControlCUDA::applySlippage");
  check(g4b_slippage(field->fieldSoA, slippage, sample_, 1, periodic_ ? 1 : 0, &field->accuslip,
                     nullptr),
        "ControlCUDA::applySlippage");
  check(g4b_field_get_first(field->fieldSoA, &field->first), "ControlCUDA::applySlippage");
  return true;
}

// ControlCUDA::applyMarker (src/Core/ControlCUDA.cpp:131-146): bring the
// state to the host before a dump, then the host-side marker actions.
bool ControlCUDA::applyMarker(Control* control, Beam* beam, std::vector<Field*>* field,
                              Undulator* und, bool& error_IO) {
  const int marker = und->getMarker();
  if (marker & 1) beam->unpack_soa_to_beam();
  if (marker & 2)
    for (Field* f : *field) f->unpack_soa_to_field();
  return control->applyMarker(beam, field, und, error_IO);
}

// ---------------------------------------------------------------- Control --
void Control::init(int, int, const std::string& fnbase, Beam*, std::vector<Field*>*,
                   Undulator*, bool, bool, bool) {
  fnbase_ = fnbase;
  written_.clear();
}

// Marker actions on the host state: beam (bit 0) and field (bit 1) dumps.
// Sorting (bit 2) is not part of this build; the stop bit is the loop's.
bool Control::applyMarker(Beam* beam, std::vector<Field*>* field, Undulator* und,
                          bool& error_IO) {
  const int marker = und->getMarker();
  if (fnbase_.empty() || !(marker & 3)) return false;
  const int step = std::max(0, std::min(und->getStep(), und->nstep()));
  const std::string tag = fnbase_ + "." + std::to_string(step);
  if (marker & 1) {
    const std::string path = tag + ".par.g4";
    if (!write_beam_dump(path, *beam)) {
      error_IO = true;
      return false;
    }
    written_.push_back(path);
  }
  if (marker & 2)
    for (Field* f : *field) {
      const int h = f->getHarm();
      const std::string path = h == 1 ? tag + ".fld.g4" : tag + ".h" + std::to_string(h) + ".fld.g4";
      if (!write_field_dump(path, *f)) {
        error_IO = true;
        return false;
      }
      written_.push_back(path);
    }
  return false;
}

// ------------------------------------------------------------------ dumps --
// Particle dump (upstream .par.h5 names): per slice "sliceNNNNNN/{gamma,
// theta, x, y, px, py, current}", and "beamletsize", "one4one",
// "refposition", "slicecount", "slicelength" (the reference length),
// "slicespacing" (the slice length).
bool write_beam_dump(const std::string& path, const Beam& beam) {
  DataFile f;
  const int ns = (int)beam.beam.size();
  for (int s = 0; s < ns; ++s) {
    const auto& sl = beam.beam[s];
    const uint64_t n = sl.size();
    std::vector<double> v[6];
    for (auto& a : v) a.resize(n);
    for (uint64_t k = 0; k < n; ++k) {
      const Particle& p = sl[k];
      v[0][k] = p.gamma, v[1][k] = p.theta, v[2][k] = p.x, v[3][k] = p.y, v[4][k] = p.px,
      v[5][k] = p.py;
    }
    const std::string g = slice_group(s) + "/";
    const char* names[6] = {"gamma", "theta", "x", "y", "px", "py"};
    for (int c = 0; c < 6; ++c) f.add(g + names[c], {n}, v[c]);
    f.add_scalar(g + "current", s < (int)beam.current.size() ? beam.current[s] : 0.0);
  }
  f.add_scalar("beamletsize", beam.nbins);
  f.add_scalar("one4one", beam.one4one ? 1.0 : 0.0);
  f.add_scalar("refposition", beam.s0);
  f.add_scalar("slicecount", ns);
  f.add_scalar("slicelength", beam.reflength);
  f.add_scalar("slicespacing", beam.slicelength);
  return f.write(path);
}

// Field dump (upstream .fld.h5 names): per slice "sliceNNNNNN/field-real"
// and "field-imag" (ngrid x ngrid, rows along y), and "gridpoints",
// "gridsize", "refposition", "slicecount", "slicespacing", "wavelength"; plus
// "accuslip", the slippage not yet applied, so that a run resumed from the
// dump shifts its slices on the same steps.
bool write_field_dump(const std::string& path, const Field& fld) {
  DataFile f;
  const int ns = (int)fld.field.size();
  const uint64_t n = (uint64_t)fld.ngrid;
  for (int s = 0; s < ns; ++s) {
    const auto& pl = fld.field[(s + fld.first) % ns];  // beam slice s
    std::vector<double> re(n * n), im(n * n);
    for (uint64_t k = 0; k < n * n; ++k) re[k] = pl[k].real(), im[k] = pl[k].imag();
    f.add(slice_group(s) + "/field-real", {n, n}, re);
    f.add(slice_group(s) + "/field-imag", {n, n}, im);
  }
  f.add_scalar("gridpoints", (double)n);
  f.add_scalar("gridsize", fld.dgrid);
  f.add_scalar("refposition", fld.s0);
  f.add_scalar("slicecount", ns);
  f.add_scalar("slicespacing", fld.slicelength);
  f.add_scalar("wavelength", fld.xlambda);
  f.add_scalar("accuslip", fld.accuslip);
  return f.write(path);
}

bool read_beam_dump(const std::string& path, Beam& beam) {
  DataFile f;
  if (!f.read(path)) return false;
  const Dataset* cnt = f.find("slicecount");
  if (!cnt || cnt->data.empty() || (int)cnt->data[0] != (int)beam.beam.size()) {
    set_error(path + ": the dump's slice count differs from the deck's");
    return false;
  }
  for (int s = 0; s < (int)beam.beam.size(); ++s) {
    const std::string g = slice_group(s) + "/";
    const Dataset* v[6] = {f.find(g + "gamma"), f.find(g + "theta"), f.find(g + "x"),
                           f.find(g + "y"), f.find(g + "px"), f.find(g + "py")};
    for (auto* d : v)
      if (!d || d->data.size() != v[0]->data.size()) {
        set_error(path + ": slice " + std::to_string(s + 1) + " is incomplete");
        return false;
      }
    auto& sl = beam.beam[s];
    sl.resize(v[0]->data.size());
    for (size_t k = 0; k < sl.size(); ++k)
      sl[k] = Particle{v[0]->data[k], v[1]->data[k], v[2]->data[k],
                       v[3]->data[k], v[4]->data[k], v[5]->data[k]};
    if (const Dataset* c = f.find(g + "current"))
      if (s < (int)beam.current.size() && !c->data.empty()) beam.current[s] = c->data[0];
  }
  return true;
}

bool read_field_dump(const std::string& path, Field& fld) {
  DataFile f;
  if (!f.read(path)) return false;
  const Dataset* cnt = f.find("slicecount");
  const Dataset* gp = f.find("gridpoints");
  const int ns = (int)fld.field.size();
  if (!cnt || cnt->data.empty() || (int)cnt->data[0] != ns || !gp || gp->data.empty() ||
      (int)gp->data[0] != fld.ngrid) {
    set_error(path + ": the dump's slice count or grid differs from the deck's");
    return false;
  }
  const size_t nn = (size_t)fld.ngrid * fld.ngrid;
  for (int s = 0; s < ns; ++s) {
    const Dataset* re = f.find(slice_group(s) + "/field-real");
    const Dataset* im = f.find(slice_group(s) + "/field-imag");
    if (!re || !im || re->data.size() != nn || im->data.size() != nn) {
      set_error(path + ": slice " + std::to_string(s + 1) + " is incomplete");
      return false;
    }
    for (size_t k = 0; k < nn; ++k) fld.field[s][k] = {re->data[k], im->data[k]};
  }
  fld.first = 0;
  const Dataset* acc = f.find("accuslip");
  fld.accuslip = acc && !acc->data.empty() ? acc->data[0] : 0.0;
  return true;
}

}  // namespace g4h
