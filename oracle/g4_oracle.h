/*
 * g4_oracle.h -- FP64 CPU restatement of the GENESIS 1.3 v4 time-stepping hot
 * path as the mulingLHY/Genesis4_CUDA_port CUDA code computes it.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * and the timed CPU baseline of the benchmark.  Nothing in the product links
 * it, calls it or falls back to it.
 *
 * PARITY UNPINNED: the reference compiles only on top of the upstream
 * GENESIS 1.3 v4 sources (tag v4.6.14, cloned at configure time) plus MPI and
 * HDF5, none of which are present, and the reference ships no golden vectors
 * or known-answer tests.  Each function restates the reference's arithmetic
 * from its source (file:line cited per function) and is checked against
 * analytic known answers in the test suite instead.
 *
 * Layouts: field cells are interleaved complex doubles [slice][iy][ix];
 * particles are six double arrays with int64 slice offsets.
 */
#ifndef G4_ORACLE_H_
#define G4_ORACLE_H_

#include <stdint.h>
#include "../include/g4b.h"

#ifdef __cplusplus
extern "C" {
#endif

/* FieldSolverADICUDA::init (src/Core/FieldSolverADICUDA.cpp:821-866).
 * Writes c, cbet, cwet (interleaved complex, n entries each) and r. */
void g4o_adi_coeffs(int n, double delz, double dgrid, double xks,
                    double* c, double* cbet, double* cwet, double* r_out);

/* adi_compute_slice_scl (src/Core/FieldSolverADICUDA.cpp:75-96). */
void g4o_slice_scl(int nslice, const int64_t* off, const double* current,
                   double fc, double xks, double dgrid, double delz,
                   double* scl);

/* adi_zero_source_grid + adi_deposit_source_atomic
 * (src/Core/FieldSolverADICUDA.cpp:98-174): dense source planes, particles
 * summed in index order. */
void g4o_deposit(int nslice, int ngrid, int first, int harm, double gridmax,
                 double dgrid, const g4b_step* st, const int64_t* off,
                 const double* x, const double* y, const double* gamma,
                 const double* theta, const double* scl, double* src);

/* FieldSolverADICUDA::advance (src/Core/FieldSolverADICUDA.cpp:638-818) with
 * the Thomas solves (:222-277, :325-380) and RHS builds (:176-220, :279-323).
 * Source-grid mode.  `field` is updated in place; `work` needs
 * 4*nslice*ngrid^2 doubles. */
void g4o_adi_advance(int nslice, int ngrid, int first, int harm,
                     double gridmax, double xks, double delz, double fc,
                     int enabled, const g4b_step* st, const int64_t* off,
                     const double* current, const double* x, const double* y,
                     const double* gamma, const double* theta, double* field,
                     double* work);

/* TrackBeamCUDA::track incl. applyChicane / applyCorrector
 * (src/Core/TrackBeamCUDA.cpp:27-69, :93-148, :156-255). */
void g4o_track(int64_t npart, const g4b_step* st, double delz, int last_step,
               double* x, double* y, double* px, double* py,
               const double* gamma);

/* TrackBeamCUDA::applyR56 (src/Core/TrackBeamCUDA.cpp:257-278). */
void g4o_r56(int64_t npart, const g4b_step* st, double lambda0,
             const double* gamma, double* theta);

/* One field as the push sees it (BeamSingleFieldView,
 * src/Core/BeamSolverCUDA.cpp:42-52). */
typedef struct g4o_field_view {
  int first, ngrid, nslice, harm;
  double gridmax, dgrid, xks;
  double fc;                 /* und->fc(harm) */
  const double* cells;       /* interleaved complex [slice][iy][ix] */
} g4o_field_view;

/* BeamSolverCUDA::advance + push kernels (src/Core/BeamSolverCUDA.cpp:77-409,
 * :449-683); slice_eloss may be NULL (zero). */
void g4o_push(int nslice, const int64_t* off, const g4b_step* st,
              const g4o_field_view* fields, int nfield,
              const double* slice_eloss, const double* x, const double* y,
              const double* px, const double* py, double* gamma,
              double* theta);
/* The same with a per-particle loss (NULL: the slice loss), the reference's
 * UseParticleEz kernels (src/Core/BeamSolverCUDA.cpp:184-195, 633-680). */
void g4o_push_ez(int nslice, const int64_t* off, const g4b_step* st,
                 const g4o_field_view* fields, int nfield,
                 const double* slice_eloss, const double* particle_ez,
                 const double* x, const double* y, const double* px,
                 const double* py, double* gamma, double* theta);

/* ControlCUDA::applySlippage, one rank (src/Core/ControlCUDA.cpp:148-252). */
int g4o_slippage(int nslice, int ngrid, double shift, double sample,
                 int time_run, int periodic, double* accuslip, int* first,
                 double* field);

/* g4_beam_slice_reduce_kernel (src/Core/DiagnosticCUDA.cpp:188-303):
 * stats[nslice*23], bre/bim[nslice*nharm]. */
void g4o_diag_beam(int nslice, const int64_t* off, int nharm, int need_aux,
                   const double* x, const double* y, const double* px,
                   const double* py, const double* gamma, const double* theta,
                   double* stats, double* bre, double* bim);

/* g4_field_slice_reduce_kernel (src/Core/DiagnosticCUDA.cpp:305-363):
 * stats[nslice*7] and center[nslice*2], indexed by beam slice. */
void g4o_diag_field(int nslice, int ngrid, int first, const double* field,
                    double* stats, double* center);

/* One Gencore main-loop step (src/Core/Gencore.cpp:172-254 with
 * Beam::track, src/Core/Beam.cpp:111-134): beam track/advance/R56/track,
 * field track for every field, slippage.  Fields share the beam's slicing.
 * work needs 4*nslice*max(ngrid)^2 doubles. */
typedef struct g4o_field_state {
  int ngrid, harm, first, enabled;
  double gridmax, xlambda;
  double fc;
  double accuslip;
  double* cells;
} g4o_field_state;

void g4o_step(int nslice, const int64_t* off, const double* current,
              const double* slice_eloss, const g4b_step* st, double lambda0,
              double slippage, double sample, int time_run, int periodic,
              g4o_field_state* fields, int nfield, double* x, double* y,
              double* px, double* py, double* gamma, double* theta,
              double* work);

/* Beam loading: Hammersley quiet start + shot noise, the same operations as
 * the drop-in host layer's loader (the upstream GENESIS loader is absent from
 * the reference tree).  Fields match g4h_beam_spec. */
typedef struct g4o_beam_spec {
  int nslice, npart, nbins, shotnoise;
  uint64_t seed;
  double gamma0, delgam, ex, ey, betax, betay, alphax, alphay;
  double xcenter, ycenter, pxcenter, pycenter, reflength, slicelength;
} g4o_beam_spec;

int g4o_load_beam(const g4o_beam_spec* spec, const double* current, double* x,
                  double* y, double* px, double* py, double* gamma,
                  double* theta, int64_t* slice_offsets);

/* Threads the OpenMP runtime uses (for reporting). */
int g4o_num_threads(void);
void g4o_set_num_threads(int n);

/* Philox4x32-10 (Salmon et al., SC 2011) on one counter block, in place. */
void g4o_philox4x32_10(uint32_t ctr[4], const uint32_t key[2]);
/* Incoherent synchrotron radiation of one step, restating g4b_beam_incoherent:
 * gamma += -loss gamma^2 + sigma gamma^2 z (loss = rate delz, sigma =
 * sqrt(spread rate delz)); z ~ N(0,1) from Philox4x32-10 keyed by seed with
 * counter (index lo, index hi, counter lo, counter hi) and Box-Muller. */
void g4o_incoherent(int64_t n, double* gamma, double loss, double sigma, uint64_t seed,
                    uint64_t counter);

#ifdef __cplusplus
}
#endif

#endif /* G4_ORACLE_H_ */
