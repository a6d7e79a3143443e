/*
 * g4ref.h -- C entry points into the REFERENCE's own CUDA sources, built in
 * place from the reference tree into oracle/_ref/libg4ref.so.
 *
 * TEST INFRASTRUCTURE ONLY.  This library exists to pin the FP64 oracle
 * (oracle/g4_oracle.c) to the reference: it runs the reference's classes
 * FieldSolverADICUDA, FieldSolverFFTCUDA, BeamSolverCUDA, TrackBeamCUDA,
 * ControlCUDA and DiagnosticCUDA (src/Core/*.cpp of mulingLHY/Genesis4_CUDA_port,
 * compiled unmodified with nvcc) on the GPU, on host arrays that this
 * wrapper uploads into the reference's Genesis4BeamSoA / Genesis4FieldSoA.
 * The upstream GENESIS 1.3 v4 classes those sources call (Undulator,
 * FieldSolver, EFieldSolver, Diagnostic, ...) are absent from the reference
 * tree; oracle/ref/upstream/ holds stand-ins that declare exactly the members
 * the reference calls, each returning the value this wrapper sets for one
 * lattice step.  Nothing in the product links or calls this library.
 *
 * Layouts follow include/g4b.h: fields are interleaved complex doubles
 * [slice][iy][ix]; particles are double arrays; slice offsets are int32 as in
 * the reference's Genesis4BeamSoA (include/Genesis4BeamSoA.h:7-21).
 * Every call returns 0, or -1 with a message in g4ref_last_error().
 */
#ifndef G4REF_H_
#define G4REF_H_

#include "../../include/g4b.h"

#ifdef __cplusplus
extern "C" {
#endif

const char* g4ref_last_error(void);
/* Number of CUDA devices visible (0 on a machine without a GPU). */
int g4ref_device_count(void);

/* FieldSolverADICUDA (solver 0, src/Core/FieldSolverADICUDA.cpp:638-902) or
 * FieldSolverFFTCUDA (solver 1, src/Core/FieldSolverFFTCUDA.cpp:214-483):
 * initSourceFilter(xc, yc, sig, filter), init(delz, dgrid, xks, ngrid) and one
 * advance(delz, field, beam, und).  xlambda is this field's wavelength
 * (Field::init divides the fundamental's by harm, src/Core/Field.cpp:57).
 * atomic_source selects the ADI solver's low-memory form. */
int g4ref_field_advance(int solver, int nslice, int ngrid, double gridmax,
                        double xlambda, int harm, int first, int enabled,
                        int atomic_source, double delz, double fc,
                        const g4b_step* st, const int* slice_offsets,
                        const double* current, const double* x,
                        const double* y, const double* gamma,
                        const double* theta, double* cells, int filter,
                        double xc, double yc, double sig);

/* BeamSolverCUDA::advance (src/Core/BeamSolverCUDA.cpp:449-683) over nfield
 * fields; slice energy loss from longESC (may be NULL = 0). */
int g4ref_beam_advance(int nslice, const int* slice_offsets,
                       const g4b_step* st, int nfield, const int* first,
                       const int* ngrid, const int* harm,
                       const double* gridmax, const double* xlambda,
                       const double* fc, const double* const* cells,
                       const double* longESC, const double* x,
                       const double* y, const double* px, const double* py,
                       double* gamma, double* theta);

/* Per-particle field for the next g4ref_beam_advance calls (slice-contiguous,
 * NULL = space charge off): the stand-in EFieldSolver then reports short
 * range on and returns these values from getEField, so BeamSolverCUDA takes
 * its per-particle branch (src/Core/BeamSolverCUDA.cpp:525-547). */
void g4ref_set_particle_ez(const double* ez);

/* TrackBeamCUDA::track (src/Core/TrackBeamCUDA.cpp:156-204), including its
 * corrector / chicane calls. */
int g4ref_track(int npart, const g4b_step* st, double delz, int last_step,
                double* x, double* y, double* px, double* py,
                const double* gamma);

/* TrackBeamCUDA::applyR56 (src/Core/TrackBeamCUDA.cpp:257-278). */
int g4ref_r56(int npart, const g4b_step* st, double lambda0,
              const double* gamma, double* theta);

/* ControlCUDA::init(0, 1, time_run, periodic, sample) + applySlippage
 * (src/Core/ControlCUDA.cpp:122-252) on one field. */
int g4ref_slippage(int nslice, int ngrid, double slippage, double sample,
                   int time_run, int periodic, double* accuslip, int* first,
                   double* cells);

/* DiagnosticCUDA::calc (src/Core/DiagnosticCUDA.cpp:381-799) at output step
 * 0 with every record switched on; the records are kept for
 * g4ref_diag_record.  nharm = bunching harmonics (filter_.beam.harm). */
int g4ref_diag(int nslice, const int* slice_offsets, const double* x,
               const double* y, const double* px, const double* py,
               const double* gamma, const double* theta, int nharm,
               const double* current, const double* eloss,
               const double* longESC, int nfield, const int* ngrid,
               const int* first, const double* gridmax,
               const double* xlambda, double slicelength,
               const double* const* cells);

/* One record of the last g4ref_diag: group 0 = beam, 1 + i = field i.
 * Copies up to cap values and returns the record's length, or -1 if the
 * record does not exist. */
int g4ref_diag_record(int group, const char* name, double* out, int cap);

/* Times ntimed steps (after warmup untimed ones) of the reference's own
 * classes on one set of device-resident state, in Gencore::run's order
 * (src/Core/Gencore.cpp:172-254): BeamSolverCUDA track / advance / applyR56 /
 * track (Beam::track's CUDA branch, src/Core/Beam.cpp:117-134),
 * FieldSolverADICUDA init + advance, ControlCUDA::applySlippage (time run,
 * not periodic) and DiagnosticCUDA::calc, one field of harmonic 1.  Lattice
 * step i of nstep gives the step parameters, fc[i] and slip[i]; steps run
 * from first_step on (wrapping).  *ms_per_step: CUDA-event time per timed
 * step, host work of the classes included. */
int g4ref_time_steps(int nslice, const int* slice_offsets, const double* x, const double* y,
                     const double* px, const double* py, const double* gamma,
                     const double* theta, const double* current, int ngrid, double gridmax,
                     double xlambda, const double* cells, int nstep, const g4b_step* steps,
                     const double* fc, const double* slip, double sample, int first_step,
                     int warmup, int ntimed, double* ms_per_step);

#ifdef __cplusplus
}
#endif

#endif /* G4REF_H_ */
