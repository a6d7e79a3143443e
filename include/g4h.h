/*
 * g4h.h -- C ABI of the C++ host layer (libg4host.so) that sits above g4b.h:
 * input decks, lattice expansion into per-step undulator tables, beam and
 * field loading, and the Gencore step driver with the reference's
 * Field / Beam / FieldSolver / BeamSolver objects.
 *
 * Upstream GENESIS 1.3 v4 provides these parts to the reference (they are not
 * in the reference tree itself); this layer re-derives the subset the hot
 * path needs from published FEL physics.  Status codes follow g4b.h.
 */
#ifndef G4H_H_
#define G4H_H_

#include <stdint.h>

#include "g4b.h"

#ifdef __cplusplus
extern "C" {
#endif

const char* g4h_last_error(void);

/* ---- beam loading (upstream Loading / QuietStart / ShotNoise) -----------
 * Quiet start: each slice holds npart particles in npart/nbins beamlets of
 * nbins particles spaced 2*pi/nbins in phase; the beamlets' (x, y, px, py,
 * gamma, theta0) come from a Hammersley/Halton set (bases 2, 3, 5, 7, 11, 13)
 * mapped to a Gaussian through the inverse normal CDF.  Shot noise perturbs
 * the beamlet phases so that <|b_h|^2> = 1/N_e per harmonic (Fawley,
 * PRST-AB 5, 070701, 2002). */
typedef struct g4h_beam_spec {
  int nslice;
  int npart;          /* particles per slice                              */
  int nbins;          /* particles per beamlet                            */
  int shotnoise;      /* 0/1                                              */
  uint64_t seed;
  double gamma0;      /* mean gamma                                       */
  double delgam;      /* rms gamma spread (absolute)                      */
  double ex, ey;      /* normalised emittances [m rad]                    */
  double betax, betay, alphax, alphay;
  double xcenter, ycenter, pxcenter, pycenter;
  double reflength;   /* lambda0 [m]                                       */
  double slicelength; /* reflength * sample [m]                           */
} g4h_beam_spec;

/* Writes npart*nslice particles (slice-contiguous) and the nslice+1 offsets;
 * current[nslice] gives each slice's current [A] (shot-noise amplitude). */
int g4h_load_beam(const g4h_beam_spec* spec, const double* current,
                  double* x, double* y, double* px, double* py,
                  double* gamma, double* theta, int64_t* slice_offsets);

/* Gaussian mode of power P [W] and waist w0 [m] on an ngrid^2 grid of half
 * width gridmax, at wavelength xlambda; writes interleaved complex cells of
 * one plane (the reference's field normalisation, P = sum |u|^2
 * (dgrid eev/ks)^2 / vacimp). */
int g4h_gaussian_field(int ngrid, double gridmax, double xlambda, double power,
                       double w0, double* cells);

/* ---- lattice -> per-step undulator tables (upstream Lattice/Undulator) ---- */
typedef struct g4h_lattice g4h_lattice;

/* Parses a .lat file subset (UNDULATOR, DRIFT, QUADRUPOLE, CORRECTOR,
 * CHICANE, PHASESHIFTER, MARKER, LINE with n*element repetition) and expands
 * `beamline` into steps of at most delz (undulators: delz per step). */
int g4h_lattice_parse(const char* text, const char* beamline, double delz,
                      double gamma0, double lambda0, g4h_lattice** out);
int g4h_lattice_destroy(g4h_lattice* lat);
int g4h_lattice_nstep(g4h_lattice* lat, int* nstep);
/* Step i: the kernel parameters, plus the upstream Undulator values the
 * driver needs: slippage (in units of lambda0), fc (coupling aw*JJ_h for
 * harmonic h, filled for h = 1..nharm), z at step end and the marker bits. */
int g4h_lattice_step(g4h_lattice* lat, int i, g4b_step* st, double* slippage,
                     double* z, int* marker);
int g4h_lattice_fc(g4h_lattice* lat, int i, int harm, double* fc);

/* Planar / helical coupling factor aw * JJ_h (upstream Undulator::fc). */
double g4h_coupling(double aw, int harm, int helical);

/* ---- input decks and the Track driver ------------------------------------
 * g4h_deck_parse reads a .in deck (&setup, &lattice, &time, &field..., &beam,
 * &track; the reference's &track keys, src/Main/Track.cpp:8-104, plus
 * `precision = fp64 | mixed`) and expands its lattice (lattice_text, or the
 * file &setup names, relative to base_dir).  Parsing needs no GPU.
 * g4h_deck_run then loads the beam and fields and runs Gencore::run
 * (src/Core/Gencore.cpp:19-315) with the CUDA classes, or the fused
 * mixed-precision run; the diagnostics are kept in a g4h_result. */
typedef struct g4h_deck g4h_deck;
typedef struct g4h_result g4h_result;

typedef struct g4h_deck_summary {
  int nslice, npart, nstep, nfield;
  int harm[8], ngrid[8];
  double gridmax[8];
  double lambda0, gamma0, sample;
  int time_run, periodic, precision, low_memory;
  int output_step, nout, bunchharm;
  int nrun;  /* steps taken: up to the first stop marker (zstop) */
  double betax, alphax, betay, alphay;  /* after &lattice zmatch */
  double current, zend;
} g4h_deck_summary;

int g4h_deck_parse(const char* deck_text, const char* lattice_text, const char* base_dir,
                   g4h_deck** out);
int g4h_deck_destroy(g4h_deck* deck);
int g4h_deck_info(g4h_deck* deck, g4h_deck_summary* summary);
int g4h_deck_run(g4h_deck* deck, g4h_result** out);
int g4h_result_destroy(g4h_result* res);
/* nz output records, slices, fields, steps taken, seconds in the loop */
int g4h_result_info(g4h_result* res, int* nz, int* nslice, int* nfield, int* nsteps,
                    double* seconds);
/* Record names of group 0 (beam) or 1..nfield (field i-1), '\n'-separated
 * (the keys of DiagnosticCUDA::calcBeam / calcField). */
int g4h_result_keys(g4h_result* res, int group, char* buf, int buflen, int* needed);
/* One record (group -1, key "z": the output positions); nz*nslice values
 * for per-slice records, nz for Global/ records. */
int g4h_result_get(g4h_result* res, int group, const char* key, double* out,
                   int64_t capacity, int64_t* length);
/* Path of the run's output file (<outputdir>/<rootname>.out.g4, written when
 * the deck names &setup outputdir or was parsed with a base_dir; "" if none).
 * Diagnostic::writeToOutputFile, called at src/Core/Gencore.cpp:297. */
int g4h_result_output_file(g4h_result* res, char* buf, int buflen, int* needed);
/* Final cells of field i (2*nslice*ngrid^2 doubles) and its `first`. */
int g4h_result_field(g4h_result* res, int ifield, double* cells, int* first);

/* ---- output and dump files ------------------------------------------------
 * The upstream HDF5 files (.out.h5 records, .par.h5 particle dumps, .fld.h5
 * field dumps; written by Diagnostic::writeToOutputFile and by the marker
 * actions ControlCUDA::applyMarker forwards to, src/Core/ControlCUDA.cpp:131-146)
 * are written here with the same dataset path names into G4DS files:
 *   "G4DS" 0 0 0 1 | u64 count | per dataset: u32 name length, name,
 *   u32 type (0 = float64, 1 = int64), u32 rank, rank x u64 dims,
 *   product(dims) x 8 bytes, all little-endian.
 * Dumps are read back by the deck groups &importbeam / &importfield. */
/* '\n'-separated dataset names of a file. */
int g4h_file_list(const char* path, char* buf, int buflen, int* needed);
/* One dataset: up to capacity values, its length, rank and dims (<= 8). */
int g4h_file_read(const char* path, const char* name, double* out, int64_t capacity,
                  int64_t* length, int* rank, int64_t* dims);

/* ---- many runs on one GPU: batched scan and served stream ----------------
 * A job is one mixed-precision FEL run on the shared lattice of the engine
 * configuration: its own slice count, grid, particles per slice, taper
 * (linear d(aw)/aw over the run), beam energy (detuning from gamma_ref),
 * seed power and number of lattice steps.  Inputs are prepared by host
 * worker threads (quiet start + shot noise, Gaussian seed); runs execute on
 * the g4b_batch engine of g4b.h. */
typedef struct g4h_job {
  int nslice, npart, ngrid, nsteps;
  int shotnoise, time_run;
  uint64_t seed;
  double gridmax, gamma, delgam, emit, beta, current, seed_power, waist, taper;
} g4h_job;

typedef struct g4h_engine_config {
  const char* lattice;   /* .lat text and the beamline to expand            */
  const char* beamline;
  double delz, gamma_ref, lambda0;
  int max_runs;          /* batch slots                                      */
  int use_graph, tune;   /* tune: 1 launch shapes, 2 also ADI row layouts  */
  int mode;              /* scan: 0 batched, 1 one run after another         */
  int threads;           /* input-preparation threads (0 = cores - 2)        */
  double reserve_bytes;  /* serve: device memory kept free at admission      */
} g4h_engine_config;

typedef struct g4h_scan_result {
  double value;          /* slice-steps/s of the timed stepping loop         */
  double seconds, slice_steps, device_bytes;
  int njobs;
  int grids[4];          /* launch shapes the batch used                     */
  int layouts_16;        /* runs whose ADI rows ended on 16-lane layouts     */
  int layouts_switched;  /* runs the row-layout tuner moved off the default  */
} g4h_scan_result;

typedef struct g4h_serve_stats {
  double seconds, p50, p99, mean, requests_per_s;
  double slice_steps, slice_steps_per_s, batch_steps;
  int peak_concurrency, reserved;
} g4h_serve_stats;

/* final_power[njobs] (W, last step) and records[sum nslice*34] (the last
 * step's raw beam record [nslice][25] then field record [nslice][9]) may be
 * null. */
int g4h_scan(const g4h_engine_config* cfg, const g4h_job* jobs, int njobs,
             g4h_scan_result* result, double* final_power, double* records);
/* arrival[njobs] in seconds from the start, non-decreasing; latency[njobs]
 * receives completion - arrival. */
int g4h_serve(const g4h_engine_config* cfg, const g4h_job* jobs, const double* arrival,
              int njobs, double* latency, double* final_power, double* records,
              g4h_serve_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* G4H_H_ */
