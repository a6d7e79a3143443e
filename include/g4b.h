/*
 * g4b.h -- C ABI of the B200 (sm_100a) GENESIS 1.3 v4 time-stepping core.
 *
 * Every entry point returns an int status (G4B_OK == 0).  Nothing is thrown
 * across the ABI; g4b_last_error() returns the message of the last failing
 * call made on the calling thread.  All handles are opaque.  All work of a
 * context is issued on one CUDA stream (the context's own, or one the caller
 * sets with g4b_ctx_set_stream); entry points that return data to host memory
 * synchronise that stream, all others are asynchronous.
 *
 * Layouts crossing the ABI are the reference's host layouts:
 *   field  : complex<double> cells, [slice][iy][ix], interleaved (re, im)
 *            (Field::field, include/Field.h:66 of the reference);
 *   beam   : six double arrays x, y, px, py, gamma, theta, slice-contiguous,
 *            with int64 slice offsets (Genesis4BeamSoA,
 *            include/Genesis4BeamSoA.h:7-21 of the reference).
 * Device layouts are private (see the design notes shipped with the library).
 *
 * Each declaration names the reference member function it replaces
 * (paths relative to the mulingLHY/Genesis4_CUDA_port tree).
 */
#ifndef G4B_H_
#define G4B_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  G4B_OK = 0,
  G4B_ERR_ARG = 1,      /* bad argument (null handle, size mismatch, ...)   */
  G4B_ERR_CUDA = 2,     /* a CUDA runtime call failed                       */
  G4B_ERR_STATE = 3,    /* call made in the wrong state (e.g. no ADI init)  */
  G4B_ERR_NOMEM = 4,    /* device allocation failed                         */
  G4B_ERR_RANGE = 5,    /* size outside what the kernels support            */
  G4B_ERR_DEVICE = 6    /* a kernel raised its device-side error flag       */
};

/* ---- precision of the device state -------------------------------------- */
enum {
  G4B_FP64 = 0,   /* plain FP64: the drop-in form                          */
  G4B_MIXED = 1   /* FP32 field/source/particles, FP64 phase theta          */
};

typedef struct g4b_ctx g4b_ctx;
typedef struct g4b_field g4b_field;
typedef struct g4b_beam g4b_beam;
typedef struct g4b_adi g4b_adi;

/* Per-step lattice values the kernels consume.  This is the subset of the
 * upstream Undulator API that the reference's CUDA path reads each step:
 * getUndulatorParameters / getQuadrupoleParameters / getCorrectorParameters /
 * getChicaneParameters (src/Core/TrackBeamCUDA.cpp:163-167), ax..grady[istep]
 * (src/Core/FieldSolverADICUDA.cpp:722-729, src/Core/BeamSolverCUDA.cpp:619-631),
 * getaw/getku/autophase/getGammaRef (src/Core/BeamSolverCUDA.cpp:514-522),
 * inUndulator (src/Core/FieldSolverADICUDA.cpp:697). */
typedef struct g4b_step {
  double delz;         /* step length [m]                                   */
  double aw;           /* rms undulator parameter                           */
  double ax, ay;       /* undulator axis offsets [m]                        */
  double kx, ky;       /* natural focusing, already scaled by ku^2 [1/m^2]  */
  double gradx, grady; /* transverse gradient [1/m]                         */
  double ku;           /* undulator wavenumber, 0 outside undulators        */
  double gamma_ref;    /* reference energy gamma0                           */
  double autophase;    /* phase shift added to theta before the push        */
  double qf;           /* quadrupole k1 [1/m^2]                             */
  double dqx, dqy;     /* quadrupole offsets [m]                            */
  double cx, cy;       /* corrector kicks [rad]                             */
  double chic_angle, chic_lb, chic_ld, chic_lt; /* chicane geometry         */
  int in_undulator;    /* und->inUndulator()                                */
  int reserved;
} g4b_step;

/* ---- errors / version ---------------------------------------------------- */
const char* g4b_last_error(void);
int g4b_version(void);

/* ---- context: device, stream, launch counter -----------------------------
 * Replaces genesis4_cuda::initialize / stream / synchronize
 * (include/Genesis4CudaRuntime.h:25-50): the reference runs everything on the
 * legacy default stream; a context owns (or borrows) one explicit stream. */
int g4b_ctx_create(int device, g4b_ctx** out);
int g4b_ctx_destroy(g4b_ctx* ctx);
int g4b_ctx_set_stream(g4b_ctx* ctx, void* cuda_stream); /* NULL = own stream */
void* g4b_ctx_get_stream(g4b_ctx* ctx);
int g4b_ctx_synchronize(g4b_ctx* ctx);
/* Number of kernels this library launched on ctx so far. */
int g4b_ctx_launch_count(g4b_ctx* ctx, uint64_t* count);
/* SM count of the context's device. */
int g4b_ctx_sm_count(g4b_ctx* ctx, int* count);
/* Self-test of the bounded waits every kernel uses on its mbarriers (no
 * counterpart in the reference, whose kernels have no waits): a one-CTA
 * kernel waits on an mbarrier phase that nothing completes, gives up after
 * spin_limit polls (1 .. 2^20), sets the context's device error word and
 * returns.  *timed_out = 1 when the wait gave up; the call then returns
 * G4B_ERR_DEVICE ("wait timeout") and leaves the context usable. */
int g4b_ctx_selftest_wait(g4b_ctx* ctx, unsigned spin_limit, int* timed_out);
/* Per-kernel CUDA-event timing on the context's stream (the reference only
 * has wall-clock phase timers, src/Core/Gencore.cpp:163-270).  Enabling
 * clears the totals; reading synchronises the stream.  names receives
 * 64-byte NUL-terminated kernel names. */
int g4b_ctx_profile(g4b_ctx* ctx, int enable);
int g4b_ctx_profile_read(g4b_ctx* ctx, int max_kernels, char* names,
                         uint64_t* counts, double* total_ms, int* nkernels);

/* ---- field state -----------------------------------------------------------
 * Replaces Genesis4FieldSoA + Field::init_fieldSoA/pack_field_to_soa/
 * unpack_soa_to_field (include/Genesis4FieldSoA.h:7-17,
 * src/Core/Field.cpp:582-674).  gridmax, xlambda and harm follow Field::init
 * (src/Core/Field.cpp:50-83): dgrid = 2*gridmax/(ngrid-1), xks = 2*pi/xlambda.
 * low_memory selects the reference's `low_memory_adisolver` mode (no separate
 * source grid; README.md:36-44). */
int g4b_field_create(g4b_ctx* ctx, int nslice, int ngrid, double gridmax,
                     double xlambda, int harm, int precision, int low_memory,
                     g4b_field** out);
int g4b_field_destroy(g4b_field* f);
int g4b_field_upload(g4b_field* f, const double* host_cells);   /* 2*nslice*ngrid^2 */
int g4b_field_download(g4b_field* f, double* host_cells);
/* Field::first: index of the storage slice holding beam slice 0
 * (include/Field.h:68). */
int g4b_field_set_first(g4b_field* f, int first);
int g4b_field_get_first(g4b_field* f, int* first);
/* Slice decomposition over ranks (the multi-rank branch of
 * ControlCUDA::applySlippage, src/Core/ControlCUDA.cpp:195-244, with its
 * plane pack/unpack kernels :27-66): one storage plane of the field state
 * (ngrid rows of the padded row pitch, in the state's precision; plane_bytes
 * gives its size) copied to or from device memory such as a communication
 * buffer, and a plane zeroed, asynchronously on the context's stream. */
int g4b_field_plane_bytes(g4b_field* f, size_t* bytes);
int g4b_field_plane_out(g4b_field* f, int slice, void* dst_device);
int g4b_field_plane_in(g4b_field* f, int slice, const void* src_device);
int g4b_field_zero_plane(g4b_field* f, int slice);
/* Bytes of device memory the field holds (state + solver scratch). */
int g4b_field_device_bytes(g4b_field* f, uint64_t* bytes);

/* ---- beam state ------------------------------------------------------------
 * Replaces Genesis4BeamSoA + Beam::init_beamSoA/pack_beam_to_soa/
 * unpack_soa_to_beam (include/Genesis4BeamSoA.h:7-21,
 * src/Core/Beam.cpp:342-525).  slice_offsets has nslice+1 entries. */
int g4b_beam_create(g4b_ctx* ctx, int nslice, const int64_t* slice_offsets,
                    int precision, double gamma_ref, g4b_beam** out);
int g4b_beam_destroy(g4b_beam* b);
int g4b_beam_upload(g4b_beam* b, const double* x, const double* y,
                    const double* px, const double* py, const double* gamma,
                    const double* theta);
int g4b_beam_download(g4b_beam* b, double* x, double* y, double* px, double* py,
                      double* gamma, double* theta);
/* Beam::current per slice [A] (include/Beam.h:69); uploaded once, kept on
 * the device (the reference re-uploads it every field step,
 * src/Core/FieldSolverADICUDA.cpp:700-702). */
int g4b_beam_set_current(g4b_beam* b, const double* current);
/* Per-slice longitudinal field loss -longESC/511000 that the push subtracts
 * (src/Core/BeamSolverCUDA.cpp:549-560).  NULL clears it to zero. */
int g4b_beam_set_eloss(g4b_beam* b, const double* slice_eloss);
/* Per-particle longitudinal loss, npart values in particle order, that the
 * push reads in place of the slice loss: the reference's h_particle_ez
 * (getEField(ip) - longESC/511000, src/Core/BeamSolverCUDA.cpp:525-547) and
 * its UseParticleEz kernels (:184-195).  NULL returns to the slice loss. */
int g4b_beam_set_particle_ez(g4b_beam* b, const double* ez);
/* Copies the per-particle loss out (G4B_ERR_STATE when none is set). */
int g4b_beam_get_particle_ez(g4b_beam* b, double* ez);
int g4b_beam_device_bytes(g4b_beam* b, uint64_t* bytes);

/* ---- incoherent synchrotron radiation ---------------------------------------
 * The step the reference leaves to upstream Incoherent::apply(Beam*,
 * Undulator*, delz) on the host particle copies (src/Core/Beam.cpp:126,
 * Beam::initIncoherent(base, rank, spread, loss), include/Beam.h:124-126),
 * here on the device state of an FP64 beam, inside undulators only:
 * gamma -= loss delz gamma^2 (loss = (2/3) r_e ku^2 aw^2) and
 * gamma += sqrt(spread delz) gamma^2 z (spread = (14/15) lambdabar_c r_e ku^3
 * K^2 F(K); planar K = sqrt(2) aw, F = 1.42 K + 1/(1 + 1.5 K + 0.95 K^2);
 * helical K = aw, F = 1.70 K + 1/(1 + 1.88 K + 0.80 K^2)), z ~ N(0,1) from
 * Philox4x32-10 keyed by seed with counter (particle index, counter) and the
 * Box-Muller transform.  Pass a different counter every step. */
int g4b_isr_rates(double aw, double ku, int helical, double* loss, double* spread);
int g4b_beam_incoherent(g4b_beam* b, const g4b_step* st, double delz, int helical,
                        int do_loss, int do_spread, uint64_t seed, uint64_t counter);

/* ---- short-range space charge ------------------------------------------------
 * The solver behind BeamSolverCUDA::initEField (include/BeamSolverCUDA.h:41-43)
 * and EFieldSolver::shortRange, which the reference runs on the host for
 * every slice (src/Core/BeamSolverCUDA.cpp:523-547); here on the device.
 * Per slice: the density modes e^{-i(l theta + m phi)}, l = 1..nz,
 * m = -nphi..nphi, on ngrid radial cells out to rmax x the largest particle
 * radius about the slice centroid; one radial tridiagonal solve per mode of
 * (1/r d/dr r d/dr - m^2/r^2 - (l k_s)^2/gammaz2) u = -S; the particle's
 * loss = -2 Z0 k_s I/(eev gammaz2) sum_l l Im[u_l e^{i l theta}] + slice loss,
 * written to the beam's per-particle buffer (g4b_beam_set_particle_ez).
 * Limits: nz*(2*nphi+1)*ngrid <= 5120, at most 2^22 particles per slice. */
typedef struct g4b_efield g4b_efield;
int g4b_efield_create(g4b_ctx* ctx, double rmax, int ngrid, int nz, int nphi, double lambda,
                      g4b_efield** out);
int g4b_efield_destroy(g4b_efield* e);
/* EFieldSolver::hasShortRange: nz > 0, ngrid > 0 and rmax > 0. */
int g4b_efield_has_short_range(const g4b_efield* e);
/* EFieldSolver::shortRange over every slice of an FP64 beam, with
 * gammaz2 = gamma_ref^2/(1 + aw^2) (src/Core/BeamSolverCUDA.cpp:521); uses the
 * beam's current and slice loss.  A no-op when short range is off. */
int g4b_efield_short_range(g4b_efield* e, g4b_beam* b, double gammaz2);

/* ---- ADI field solver --------------------------------------------------------
 * FieldSolverADICUDA (include/FieldSolverADICUDA.h:20-25). */
int g4b_adi_create(g4b_ctx* ctx, g4b_adi** out);
int g4b_adi_destroy(g4b_adi* adi);
/* FieldSolverADICUDA::init (src/Core/FieldSolverADICUDA.cpp:821-902):
 * factorises the constant tridiagonal (1+2ir, -ir) with r = delz/(4 xks dgrid^2)
 * in FP64; recomputes only when delz or ngrid change. */
int g4b_adi_init(g4b_adi* adi, double delz, double dgrid, double xks, int ngrid);
/* FieldSolverADICUDA::advance (src/Core/FieldSolverADICUDA.cpp:638-818):
 * source deposition (if in_undulator, the field is enabled and harm is odd)
 * and the two ADI half-steps.  fc is und->fc(harm). */
int g4b_adi_advance(g4b_adi* adi, g4b_field* f, g4b_beam* b,
                    const g4b_step* st, double fc, int enabled);

/* ---- beam solver ------------------------------------------------------------
 * TrackBeamCUDA::track (src/Core/TrackBeamCUDA.cpp:156-204), including the
 * chicane matrix on the first half step and the corrector kick on the last. */
int g4b_beam_track(g4b_beam* b, const g4b_step* st, double delz, int last_step);
/* TrackBeamCUDA::applyR56 (src/Core/TrackBeamCUDA.cpp:257-278). */
int g4b_beam_r56(g4b_beam* b, const g4b_step* st, double lambda0);
/* BeamSolverCUDA::advance (src/Core/BeamSolverCUDA.cpp:449-683): RK4 of
 * (gamma, theta) with the bilinear field sample frozen per step, summed over
 * nfield <= 8 fields.  fc[i] = und->fc(harm_i); xks_fund = field xks / harm.
 * xku is und->getku(), replaced by xks_fund/(2 gamma_ref^2) when zero. */
int g4b_beam_advance(g4b_beam* b, g4b_field* const* fields, const double* fc,
                     int nfield, const g4b_step* st);

/* ---- slippage -----------------------------------------------------------------
 * ControlCUDA::applySlippage, single rank (src/Core/ControlCUDA.cpp:148-252):
 * accuslip += shift; while |accuslip| > 0.8*sample shift `first` by one slice
 * and zero the plane entering the window (unless periodic).  Returns the
 * number of whole-slice shifts in *nshift (may be NULL). */
int g4b_slippage(g4b_field* f, double shift, double sample, int time_run,
                 int periodic, double* accuslip, int* nshift);

/* ---- diagnostics -----------------------------------------------------------------
 * Device part of DiagnosticCUDA::calcBeam (src/Core/DiagnosticCUDA.cpp:188-303,
 * :414-447): per slice the 23 raw sums/extrema in the reference's order
 * (g1,g2,x1,x2,y1,y2,px1,px2,py1,py2,xpx,ypy,count,xmin,xmax,pxmin,pxmax,
 * ymin,ymax,pymin,pymax,gmin,gmax) into stats[nslice*23], and the bunching
 * sums sum(cos h theta), sum(sin h theta), h = 1..nharm, into
 * bre/bim[nslice*nharm].  Host arrays; the call synchronises. */
int g4b_diag_beam(g4b_beam* b, int nharm, int need_aux, double* stats,
                  double* bre, double* bim);
/* Device part of DiagnosticCUDA::calcField (src/Core/DiagnosticCUDA.cpp:305-363,
 * :633-659): per beam slice is = (nslice + storage_slice - first) % nslice the
 * 7 sums (power, x1, x2, y1, y2, ff_re, ff_im) into stats[nslice*7] and the
 * centre cell (ngrid^2-1)/2 into center[nslice*2] (re, im). */
int g4b_diag_field(g4b_field* f, double* stats, double* center);
/* g4b_diag_field with no allocation at call time: no counterpart in the
 * reference (its DiagnosticCUDA grows device buffers on demand,
 * src/Core/DiagnosticCUDA.cpp:633-648).  The device scratch is one fixed
 * array in the library, so nslice is limited to 4096 (G4B_ERR_RANGE
 * beyond).  The first call on a device looks up that array's address (which
 * may load the module): make it before any stream capture on that device.
 * No part of the scratch needs to start at zero.  All calls on one device
 * share the array: calls that overlap in time on the same device (two host
 * threads, or two contexts on one device) race and must be serialised by the
 * caller.  Synchronises the context's stream, like g4b_diag_field. */
int g4b_diag_field_static(g4b_field* f, double* stats, double* center);

/* ---- FFT field solver ------------------------------------------------------
 * Replaces FieldSolverFFTCUDA (include/FieldSolverFFTCUDA.h:15-20,
 * src/Core/FieldSolverFFTCUDA.cpp:157-483): the spectral propagator
 *   u' = IFFT2( FFT2(u) exp(i k2 dz) + 2 filter FFT2(S) ) / n^2,
 *   k2 = -(kx^2 + ky^2) / (2 ks),
 * with the ADI solver's deterministic source S and the sigmoid source filter.
 * The batched 2-D transforms are this library's own kernels (no cuFFT).
 * FP64 fields, ngrid <= 256. */
typedef struct g4b_fft g4b_fft;
int g4b_fft_create(g4b_ctx* ctx, g4b_fft** out);
int g4b_fft_destroy(g4b_fft* solver);
/* FieldSolverFFTCUDA::initSourceFilter (src/Core/FieldSolverFFTCUDA.cpp:214-222):
 * the filter 1 / (1 + exp((sqrt((dx/(n xc))^2 + (dy/(n yc))^2) - 1) / sig))
 * is applied only when filter != 0 and xc, yc, sig > 0; it takes effect at
 * the next g4b_fft_init. */
int g4b_fft_init_filter(g4b_fft* solver, double xc, double yc, double sig, int filter);
/* FieldSolverFFTCUDA::init (src/Core/FieldSolverFFTCUDA.cpp:246-293): the
 * tables are rebuilt when ngrid, dgrid or xks change (the reference keys
 * them on ngrid alone); delz is the step the next advance propagates. */
int g4b_fft_init(g4b_fft* solver, double delz, double dgrid, double xks, int ngrid);
/* FieldSolverFFTCUDA::advance (src/Core/FieldSolverFFTCUDA.cpp:295-483). */
int g4b_fft_advance(g4b_fft* solver, g4b_field* f, g4b_beam* b, const g4b_step* step,
                    double fc, int enabled);

/* ---- fused mixed-precision run -------------------------------------------
 * A whole FEL run resident on the device: FP32 particles and complex64
 * fields with the phase theta in FP64, advanced per lattice step by a fused
 * beam step (TrackBeamCUDA::track + BeamSolverCUDA::advance + applyR56 +
 * TrackBeamCUDA::track), a fused deposition + beam diagnostics, the two ADI
 * passes per field (FieldSolverADICUDA::advance, with the slippage of
 * ControlCUDA::applySlippage and the field part of DiagnosticCUDA folded into
 * the second pass), replayed as one CUDA graph.  Beam and fields share the
 * slicing; fields may differ in harmonic and grid.  No counterpart class in
 * the reference: it composes the reference's per-step calls in
 * src/Core/Gencore.cpp:172-254. */
typedef struct g4b_run g4b_run;

typedef struct g4b_run_desc {
  int nslice;
  int nfield;           /* 1..8                                             */
  int harm[8];          /* field harmonics                                  */
  int ngrid[8];
  double gridmax[8];
  double lambda0;       /* reference (fundamental) wavelength [m]           */
  double gamma_ref;
  double sample;        /* slicelength / reflength                          */
  int time_run;         /* slippage on                                      */
  int periodic;
  int nbunch;           /* bunching harmonics in the diagnostics (1..8)     */
  int precision;        /* G4B_MIXED                                        */
} g4b_run_desc;

/* At most 65536 particles per slice (G4B_ERR_RANGE otherwise): the
 * exact-integer deposition keeps at least 2^14 quanta per contribution. */
int g4b_run_create(g4b_ctx* ctx, const g4b_run_desc* desc,
                   const int64_t* slice_offsets, g4b_run** out);
int g4b_run_destroy(g4b_run* run);
int g4b_run_upload_beam(g4b_run* run, const double* x, const double* y,
                        const double* px, const double* py, const double* gamma,
                        const double* theta);
int g4b_run_download_beam(g4b_run* run, double* x, double* y, double* px,
                          double* py, double* gamma, double* theta);
/* cells = NULL uploads a zero field. */
int g4b_run_upload_field(g4b_run* run, int ifield, const double* cells, int first);
int g4b_run_download_field(g4b_run* run, int ifield, double* cells, int* first);
int g4b_run_set_current(g4b_run* run, const double* current);
int g4b_run_set_eloss(g4b_run* run, const double* slice_eloss);
/* Per-step tables: steps[nstep], fc[nstep*nfield] (und->fc(harm) per field),
 * slip[nstep] (und->slippage(), units of lambda0); keeps the diagnostics of
 * the last hist_steps steps (0 = nstep). */
int g4b_run_set_lattice(g4b_run* run, int nstep, const g4b_step* steps,
                        const double* fc, const double* slip, int hist_steps);
/* Enqueue lattice steps [first_step, first_step+nsteps) (asynchronous); with
 * use_graph the range is captured once as a CUDA graph and replayed. */
int g4b_run_advance(g4b_run* run, int first_step, int nsteps, int use_graph);
/* Capture the graph of that range from the current state without launching
 * it (so a timed g4b_run_advance only replays). */
int g4b_run_prepare(g4b_run* run, int first_step, int nsteps);
/* Diagnostics of one step: beam[nslice*(23+2*nbunch)] (raw sums in the
 * order of g4b_diag_beam, bunching interleaved re,im), field[nfield*nslice*9]
 * (the 7 sums of g4b_diag_field, then the centre cell re, im). */
int g4b_run_history(g4b_run* run, int step, double* beam, double* field);
/* Diagnostics of steps [first, first+n) with one read: out[n][step record],
 * a step record being the beam and field blocks of g4b_run_history
 * back to back (n <= the steps the history keeps). */
int g4b_run_history_range(g4b_run* run, int first, int n, double* out);
int g4b_run_device_bytes(g4b_run* run, uint64_t* bytes);

/* ---- batched runs ---------------------------------------------------------
 * No counterpart in the reference (it advances one simulation per process).
 * Many independent mixed-precision runs (each a g4b_run: own slice count,
 * grid, particle count, lattice and slippage) advance together: per step one
 * persistent launch per kernel phase covers every attached run, driven by
 * work lists of (run, chunk / slice / band) items.  A run's results are the
 * same alone and in any mix (every item is computed as in the single-run
 * kernels).  Runs join (attach) and leave (detach, or on reaching their last
 * step) between steps. */
typedef struct g4b_batch g4b_batch;
int g4b_batch_create(g4b_ctx* ctx, int max_runs, g4b_batch** out);
int g4b_batch_destroy(g4b_batch* batch);
/* The run takes part in lattice steps [first_step, first_step + nsteps). */
int g4b_batch_attach(g4b_batch* batch, g4b_run* run, int first_step, int nsteps,
                     int* slot);
int g4b_batch_detach(g4b_batch* batch, int slot);
int g4b_batch_status(g4b_batch* batch, int slot, int* next_step, int* remaining);
/* Advance every attached, unfinished run by nsteps steps (asynchronous);
 * use_graph replays each step's kernels from a CUDA graph. */
int g4b_batch_step(g4b_batch* batch, int nsteps, int use_graph);
/* Autotuner: the next 4 steps try candidate launch shapes (CTAs per SM) for
 * each kernel, timed with CUDA events; the fastest shape per kernel stays. */
int g4b_batch_tune(g4b_batch* batch);
/* Autotuner with row shapes: the launch shapes as g4b_batch_tune, then, for
 * every group of fields sharing an ADI row layout that has another one (a row
 * of n cells as 32 lanes x M elements or as 16 lanes x M' elements, two rows
 * per warp), one timed step in the current layouts and one with the group
 * switched; the faster stays.  The layout sets the FP32 rounding of the row
 * solve (the same linear system), so results of a layout-tuned batch equal an
 * alone run given the same layouts (g4b_run_set_layouts). */
int g4b_batch_tune_layouts(g4b_batch* batch);
/* CTAs of the beam, deposition, ADI and finalize launches in use. */
int g4b_batch_shapes(g4b_batch* batch, int* grids4);
/* ADI row layouts of a run's fields: M (32-lane rows of M elements) or
 * 100 + M (16-lane rows), and setting them (the default layout of the grid,
 * g4b_default_layout, or its other one). */
int g4b_run_get_layouts(g4b_run* run, int* layouts);
int g4b_run_set_layouts(g4b_run* run, const int* layouts);
int g4b_default_layout(int ngrid);
/* Stream marks: g4b_ctx_mark records a point in the context's stream and
 * returns its ticket; g4b_ctx_mark_query reports (or with wait, waits for)
 * the completion of everything enqueued before it.  The last 256 tickets
 * stay valid. */
int g4b_ctx_mark(g4b_ctx* ctx, uint64_t* ticket);
int g4b_ctx_mark_query(g4b_ctx* ctx, uint64_t ticket, int wait, int* done);
/* Free and total device memory (cudaMemGetInfo) for admission decisions. */
int g4b_ctx_mem_info(g4b_ctx* ctx, uint64_t* free_bytes, uint64_t* total_bytes);

#ifdef __cplusplus
}
#endif

#endif /* G4B_H_ */
