// genesis4.h -- the reference's host-side classes for the time-stepping path,
// re-implemented on top of the C ABI of include/g4b.h.
//
// Class names, member functions and their argument meaning follow the
// mulingLHY/Genesis4_CUDA_port overlay (include/Field.h, include/Beam.h,
// include/FieldSolverADICUDA.h, include/BeamSolverCUDA.h,
// include/TrackBeamCUDA.h, include/ControlCUDA.h, include/DiagnosticCUDA.h,
// include/Gencore.h, include/Track.h), so that code calling that path calls
// this one.  Device state lives in g4b_* handles; errors are
// std::runtime_error (the reference's convention, include/Genesis4CudaRuntime.h:13-23).
#pragma once

#include <complex>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Undulator.h"
#include "g4b.h"

namespace g4h {

extern const double vacimp;  // 376.73 Ohm
extern const double eev;     // 510998.95 eV
extern const double ce;      // 1.602176634e-19 C

// g4b status -> std::runtime_error with the library's message.
void check(int rc, const char* where);

// one context (device + stream) per process, created on first use
g4b_ctx* cuda_context();

struct Particle {  // upstream Particle.h layout
  double gamma, theta, x, y, px, py;
};

class Beam;
class Field;

// upstream FieldSolver interface (FieldSolverADICUDA.h:20-25 overrides it)
class FieldSolver {
 public:
  virtual ~FieldSolver() = default;
  virtual void init(double delz, double dgrid, double xks, unsigned int ngrid) = 0;
  virtual void advance(double delz, Field* field, Beam* beam, Undulator* und) = 0;
  virtual void initSourceFilter(double, double, double, bool) {}
};

// FieldSolverADICUDA (include/FieldSolverADICUDA.h:17-65)
class FieldSolverADICUDA : public FieldSolver {
 public:
  explicit FieldSolverADICUDA(bool atomic_source = false);
  ~FieldSolverADICUDA() override;
  void init(double delz, double dgrid, double xks, unsigned int ngrid) override;
  void advance(double delz, Field* field, Beam* beam, Undulator* und) override;

 private:
  g4b_adi* adi_ = nullptr;
  bool atomic_source_;
};

// FieldSolverFFTCUDA (include/FieldSolverFFTCUDA.h:15-20)
class FieldSolverFFTCUDA : public FieldSolver {
 public:
  FieldSolverFFTCUDA();
  ~FieldSolverFFTCUDA() override;
  void init(double delz, double dgrid, double xks, unsigned int ngrid) override;
  void advance(double delz, Field* field, Beam* beam, Undulator* und) override;
  void initSourceFilter(double xc, double yc, double sig, bool filter) override;

 private:
  g4b_fft* fft_ = nullptr;
};

// Field (include/Field.h:32-99)
class Field {
 public:
  Field();
  virtual ~Field();
  void init(int nsize, int ngrid, double dgrid, double xlambda0, double slicelen, double s0,
            int harm);
  void initSolver(bool isFFT, bool filter, double xc, double yc, double sig,
                  bool use_cuda = false, bool low_memory_adisolver = false);
  void track(double delz, Beam* beam, Undulator* und);
  void setStepsize(double delz) { dz_save = delz; }
  void disable(double conv);
  bool isEnabled() const { return !disabled; }
  int getHarm() const { return harm; }
  double getRHarm() const { return rharm; }
  void resetSlippage() { accuslip = 0; }
  void init_fieldSoA();
  void pack_field_to_soa();
  void unpack_soa_to_field();

  std::vector<std::vector<std::complex<double>>> field;
  double xlambda = 0, dgrid = 0, xks = 0, gridmax = 0, dz_save = 0;
  int ngrid = 0, first = 0, harm = 1;
  double slicelength = 0, s0 = 0, accuslip = 0;
  g4b_field* fieldSoA = nullptr;  // device state (Genesis4FieldSoA)

 private:
  std::unique_ptr<FieldSolver> solver;
  bool disabled = false;
  double rharm = 1;
  bool low_memory_ = false;
};

class TrackBeamCUDA {  // include/TrackBeamCUDA.h:7-15
 public:
  void track(double delz, Beam* beam, Undulator* und, bool last);
  void applyR56(Beam* beam, Undulator* und, double lambda0);
};

class BeamSolverCUDA {  // include/BeamSolverCUDA.h:17-37
 public:
  BeamSolverCUDA() = default;
  BeamSolverCUDA(const BeamSolverCUDA&) = delete;
  BeamSolverCUDA& operator=(const BeamSolverCUDA&) = delete;
  ~BeamSolverCUDA();
  // include/BeamSolverCUDA.h:41-43: short-range space charge on the device
  // (g4b_efield); longrange (upstream's long-range model) is not built
  void initEField(double rmax, int ngrid, int nz, int nphi, double lambda, bool longr);
  void advance(double delz, Beam* beam, std::vector<Field*>* field, Undulator* und);
  void track(double delz, Beam* beam, Undulator* und, bool last) {
    tracker.track(delz, beam, und, last);
  }
  void applyR56(Beam* beam, Undulator* und, double reflen) { tracker.applyR56(beam, und, reflen); }
  void checkAllocation(unsigned long) {}
  double getSCField(int) { return 0.0; }

 private:
  bool onlyFundamental = false;
  TrackBeamCUDA tracker;
  g4b_efield* efield = nullptr;
};

// Upstream Incoherent (absent from the reference tree), on the device state:
// init(base, rank, spread, loss) as Beam::initIncoherent (include/Beam.h:124-126)
// calls it; apply(beam, und, delz) as Beam::track does after the push
// (src/Core/Beam.cpp:126).  The seed is base + rank; each apply draws with a
// new counter.
class Incoherent {
 public:
  void init(int base, int rank, bool spread, bool loss) {
    seed_ = (uint64_t)(int64_t)base + (uint64_t)rank;
    spread_ = spread;
    loss_ = loss;
  }
  void apply(Beam* beam, Undulator* und, double delz);

 private:
  uint64_t seed_ = 0, counter_ = 0;
  bool spread_ = false, loss_ = false;
};

// Beam (include/Beam.h:24-105)
class Beam {
 public:
  Beam();
  virtual ~Beam();
  void init(int nsize, int nbins, double reflen, double slicelen, double s0, bool one4one);
  // include/Beam.h:124-126
  void initIncoherent(int base, int rank, bool spread, bool loss) {
    incoherent.init(base, rank, spread, loss);
  }
  // include/Beam.h:128-133
  void initEField(double rmax, int ngrid, int nz, int nphi, double lambda, bool longr) {
    cuda_solver.initEField(rmax, ngrid, nz, nphi, lambda, longr);
  }
  void track(double delz, std::vector<Field*>* field, Undulator* und);
  void setUseCuda(bool in) { useCudaSolver_ = in; }
  void init_beamSoA();
  void pack_beam_to_soa();
  void unpack_soa_to_beam();
  void setBunchingHarmonicOutput(int h) { bharm = h; }
  int getBunchingHarmonics() const { return bharm; }

  std::vector<std::vector<Particle>> beam;
  std::vector<double> current, eloss, longESC;
  double reflength = 0, slicelength = 0, s0 = 0;
  bool one4one = false;
  int nbins = 4;
  double gamma_ref = 0;
  g4b_beam* beamSoA = nullptr;  // device state (Genesis4BeamSoA)

 private:
  Incoherent incoherent;
  BeamSolverCUDA cuda_solver;
  bool useCudaSolver_ = false;
  int bharm = 1;
};

// upstream Setup subset: the output file base (Setup::getRootName,
// Setup::RootName_to_FileName).  With outputdir empty no file is written.
class Setup {
 public:
  std::string rootname = "genesis", outputdir;
  void getRootName(std::string* rn) const { *rn = rootname; }
  void RootName_to_FileName(std::string* fn, const std::string* rn) const {
    *fn = outputdir.empty() ? std::string() : outputdir + "/" + *rn;
  }
};

// upstream Control subset: the marker actions on the host state, which
// ControlCUDA::applyMarker forwards to (src/Core/ControlCUDA.cpp:131-146):
// beam dumps (marker bit 0) as <fnbase>.<steps taken>.par.g4 and field dumps
// (bit 1) as <fnbase>.<steps taken>.fld.g4 (harmonic h > 1: .h<h>.fld.g4),
// in the G4DS format of g4file.cpp.  Slices are written in beam order.
class Control {
 public:
  void init(int rank, int size, const std::string& fnbase, Beam* beam,
            std::vector<Field*>* field, Undulator* und, bool isTime, bool isScan,
            bool periodic);
  bool applyMarker(Beam* beam, std::vector<Field*>* field, Undulator* und, bool& error_IO);
  const std::vector<std::string>& written() const { return written_; }

 private:
  std::string fnbase_;
  std::vector<std::string> written_;
};

// Dump files of one beam / one field (G4DS, the upstream .par.h5 / .fld.h5
// dataset names) and their readers for &importbeam / &importfield.
bool write_beam_dump(const std::string& path, const Beam& beam);
bool write_field_dump(const std::string& path, const Field& field);
bool read_beam_dump(const std::string& path, Beam& beam);
bool read_field_dump(const std::string& path, Field& field);

// slippage / markers (include/ControlCUDA.h:15-23)
class ControlCUDA {
 public:
  void init(int rank, int size, bool isTime, bool periodic, double sample);
  bool applySlippage(double slippage, Field* field);
  bool applyMarker(Control* control, Beam* beam, std::vector<Field*>* field, Undulator* und,
                   bool& error_IO);

 private:
  bool timerun_ = false, periodic_ = false;
  int rank_ = 0, size_ = 1;
  double sample_ = 1.0;
};

// upstream FilterDiagnostics subset (filter_.beam.* / filter_.field.* in
// src/Core/DiagnosticCUDA.cpp)
struct FilterDiagnostics {
  struct {
    int harm = 1;
    bool exclharm = false, auxiliar = true, energy = true, spatial = true, current = true;
    bool twiss = true, global = true;
  } beam;
  struct {
    bool global = true, spatial = true, intensity = true;
  } field;
};

// Output container: val[2] = beam group, val[3+i] = field i (the layout
// DiagnosticCUDA::calc fills, src/Core/DiagnosticCUDA.cpp:395-408).
struct Diagnostic {
  std::vector<double> zout;
  std::vector<std::map<std::string, std::vector<double>>> val;
  std::string output_file;  // written by writeToOutputFile (empty: none)
  void init(int nz, int nslice, int nfield, const FilterDiagnostics& filter);
  // Diagnostic::writeToOutputFile (called at src/Core/Gencore.cpp:297): the
  // records, output positions and lattice tables as <fnbase>.out.g4 (G4DS).
  bool writeToOutputFile(Beam* beam, std::vector<Field*>* field, Setup* setup, Undulator* und);
};

class DiagnosticCUDA {  // include/DiagnosticCUDA.h:17-31
 public:
  void init(FilterDiagnostics& filter) {
    filter_ = filter;
    iz_ = 0;
  }
  bool calc(Beam* beam, std::vector<Field*>* field, double z, Diagnostic& diag);

 private:
  bool calcBeam(Beam* beam, std::map<std::string, std::vector<double>>& out);
  bool calcField(Field* field, std::map<std::string, std::vector<double>>& out);
  FilterDiagnostics filter_;
  int iz_ = 0;
};

// Per-phase wall-clock accumulators (src/Core/Gencore.cpp:163-270), here
// synchronised device time.
struct GencoreTimers {
  double beam = 0, field = 0, slip = 0, diag = 0, unpack = 0;
  int steps = 0;
};

class Gencore {  // include/Gencore.h:20-23
 public:
  // The reference's arguments, then the records (the reference keeps its
  // Diagnostic inside run and writes it to file; here the caller gets it too)
  // and optional phase timers.
  bool run(Beam* beam, std::vector<Field*>* field, Setup* setup, Undulator* und, bool isTime,
           bool isScan, bool periodic, bool use_cuda, FilterDiagnostics& filter,
           Diagnostic& diag, GencoreTimers* timers = nullptr);
};

// Fused mixed-precision run of the same loop (g4b_run): beam and fields stay
// on the device in FP32 (+FP64 theta); the diagnostics are read back at the
// end; the loop stops at dump markers to bring the state to the host.
bool run_mixed(Beam* beam, std::vector<Field*>* field, Setup* setup, Undulator* und,
               bool isTime, bool periodic, FilterDiagnostics& filter, Diagnostic& diag,
               GencoreTimers* timers = nullptr);

// Derived diagnostics from raw per-slice sums (the host part of
// DiagnosticCUDA::calcBeam/calcField, src/Core/DiagnosticCUDA.cpp:449-799).
void finish_beam_diag(const FilterDiagnostics& f, int iz, int nslice, int nharm,
                      const double* stats, const double* bre, const double* bim,
                      const std::vector<double>& current, const std::vector<double>& eloss,
                      const std::vector<double>& longESC,
                      std::map<std::string, std::vector<double>>& out);
void finish_field_diag(const FilterDiagnostics& f, int iz, int nslice, int ngrid, double dgrid,
                       double gridmax, double xlambda, double slicelength, const double* stats,
                       int stats_stride, const double* center, int center_stride,
                       std::map<std::string, std::vector<double>>& out);

}  // namespace g4h
