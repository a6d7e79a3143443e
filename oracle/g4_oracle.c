/*
 * g4_oracle.c -- FP64 CPU restatement of the reference's time-stepping hot
 * path.  TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline); the
 * product never links or calls it.  PARITY UNPINNED against upstream
 * GENESIS 1.3 v4: see g4_oracle.h.
 *
 * Complex numbers are written out as (re, im) pairs so that the order of
 * every multiply/add follows the reference's thrust::complex expressions.
 * OpenMP parallelises over slices, lines and particles; no loop carries a
 * reduction across threads, so results do not depend on the thread count.
 */
#include "g4_oracle.h"

#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define RE(p, i) ((p)[2 * (i)])
#define IM(p, i) ((p)[2 * (i) + 1])

int g4o_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void g4o_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

static inline void cmul(double ar, double ai, double br, double bi, double* r,
                        double* i) {
  *r = ar * br - ai * bi;
  *i = ar * bi + ai * br;
}

static inline void cinv(double ar, double ai, double* r, double* i) {
  const double d = ar * ar + ai * ai;
  *r = ar / d;
  *i = -ai / d;
}

/* src/Core/FieldSolverADICUDA.cpp:830-866 */
void g4o_adi_coeffs(int n, double delz, double dgrid, double xks, double* c,
                    double* cbet, double* cwet, double* r_out) {
  const double rtmp = 0.25 * delz / (xks * dgrid * dgrid);
  double* mupp = (double*)malloc(sizeof(double) * n);
  double* mmid = (double*)malloc(sizeof(double) * n);
  double* mlow = (double*)malloc(sizeof(double) * n);
  mupp[0] = rtmp;
  mmid[0] = -2 * rtmp;
  mlow[0] = 0;
  for (int i = 1; i < n - 1; i++) {
    mupp[i] = rtmp;
    mmid[i] = -2 * rtmp;
    mlow[i] = rtmp;
  }
  mupp[n - 1] = 0;
  mmid[n - 1] = -2 * rtmp;
  mlow[n - 1] = rtmp;
  /* cwrk1 = (0,-mupp), cwrk2 = (1,-mmid), c = (0,-mlow) */
  for (int i = 0; i < n; i++) {
    RE(c, i) = 0.0;
    IM(c, i) = -mlow[i];
  }
  cinv(1.0, -mmid[0], &RE(cbet, 0), &IM(cbet, 0));
  RE(cwet, 0) = 0.0;
  IM(cwet, 0) = 0.0;
  for (int i = 1; i < n; i++) {
    cmul(0.0, -mupp[i - 1], RE(cbet, i - 1), IM(cbet, i - 1), &RE(cwet, i),
         &IM(cwet, i));
    double tr, ti;
    cmul(RE(c, i), IM(c, i), RE(cwet, i), IM(cwet, i), &tr, &ti);
    cinv(1.0 - tr, -mmid[i] - ti, &RE(cbet, i), &IM(cbet, i));
  }
  if (r_out) *r_out = rtmp;
  free(mupp);
  free(mmid);
  free(mlow);
}

/* src/Core/FieldSolverADICUDA.cpp:75-96 (vacimp, eev: upstream constants). */
#define G4O_VACIMP 376.73031346177
#define G4O_EEV 510998.95

void g4o_slice_scl(int nslice, const int64_t* off, const double* current,
                   double fc, double xks, double dgrid, double delz,
                   double* scl) {
  for (int is = 0; is < nslice; is++) {
    double s = 0.0;
    const int64_t npar = off[is + 1] - off[is];
    if (npar > 0) {
      s = fc * G4O_VACIMP * current[is] * xks * delz;
      s /= 4.0 * G4O_EEV * (double)npar * dgrid * dgrid;
    }
    scl[is] = s;
  }
}

/* src/Core/FieldSolverADICUDA.cpp:98-174 */
void g4o_deposit(int nslice, int ngrid, int first, int harm, double gridmax,
                 double dgrid, const g4b_step* st, const int64_t* off,
                 const double* x, const double* y, const double* gamma,
                 const double* theta, const double* scl, double* src) {
  const int64_t plane = (int64_t)ngrid * ngrid;
  memset(src, 0, sizeof(double) * 2 * plane * nslice);
#pragma omp parallel for schedule(dynamic, 1)
  for (int bs = 0; bs < nslice; bs++) {
    const double s_scl = scl[bs];
    if (s_scl == 0.0) continue;
    const int target = (bs + first) % nslice;
    double* t = src + 2 * plane * target;
    for (int64_t ip = off[bs]; ip < off[bs + 1]; ip++) {
      const double xp = x[ip], yp = y[ip];
      if (!(xp > -gridmax && xp < gridmax && yp > -gridmax && yp < gridmax))
        continue;
      const double wx_raw = (xp + gridmax) / dgrid;
      const double wy_raw = (yp + gridmax) / dgrid;
      const int ix = (int)floor(wx_raw);
      const int iy = (int)floor(wy_raw);
      if (ix < 0 || ix >= ngrid - 1 || iy < 0 || iy >= ngrid - 1) continue;
      const double wx = 1.0 + (double)ix - wx_raw;
      const double wy = 1.0 + (double)iy - wy_raw;
      const double dx = xp - st->ax, dy = yp - st->ay;
      const double faw2 = 1.0 + st->kx * dx * dx + st->ky * dy * dy +
                          2.0 * (st->gradx * dx + st->grady * dy);
      const double part = sqrt(faw2) * s_scl / gamma[ip];
      const double phase = (double)harm * theta[ip];
      const double cre = sin(phase) * part;
      const double cim = cos(phase) * part;
      const int64_t base = ix + (int64_t)iy * ngrid;
      const double w00 = wx * wy, w10 = (1.0 - wx) * wy;
      const double w01 = wx * (1.0 - wy), w11 = (1.0 - wx) * (1.0 - wy);
      RE(t, base) += cre * w00;
      IM(t, base) += cim * w00;
      RE(t, base + 1) += cre * w10;
      IM(t, base + 1) += cim * w10;
      RE(t, base + ngrid) += cre * w01;
      IM(t, base + ngrid) += cim * w01;
      RE(t, base + ngrid + 1) += cre * w11;
      IM(t, base + ngrid + 1) += cim * w11;
    }
  }
}

/* rhs = u + i*r*lap + S along y (dir 0, :176-220) or x (dir 1, :279-323);
 * the missing neighbour at an edge is zero. */
static void rhs_build(int nslice, int ngrid, double r, int dir,
                      const double* src, const double* u, double* out) {
  const int64_t plane = (int64_t)ngrid * ngrid;
  const int64_t total = plane * nslice;
  const int64_t step = dir == 0 ? ngrid : 1;
#pragma omp parallel for schedule(static)
  for (int64_t g = 0; g < total; g++) {
    const int64_t local = g % plane;
    const int64_t pos = dir == 0 ? local / ngrid : local % ngrid;
    const double cr = RE(u, g), ci = IM(u, g);
    double lr, li;
    if (pos == 0) {
      lr = RE(u, g + step) - cr * 2.0;
      li = IM(u, g + step) - ci * 2.0;
    } else if (pos == ngrid - 1) {
      lr = RE(u, g - step) - cr * 2.0;
      li = IM(u, g - step) - ci * 2.0;
    } else {
      lr = RE(u, g + step) + RE(u, g - step) - cr * 2.0;
      li = IM(u, g + step) + IM(u, g - step) - ci * 2.0;
    }
    double rr = cr + (-r * li);
    double ri = ci + (r * lr);
    if (src) {
      rr += RE(src, g);
      ri += IM(src, g);
    }
    RE(out, g) = rr;
    IM(out, g) = ri;
  }
}

/* Thomas solve of every line (:222-277 for dir 1 = rows along x,
 * :325-380 for dir 0 = columns along y); writes u from rhs. */
static void thomas_lines(int nslice, int ngrid, int dir, const double* c,
                         const double* cbet, const double* cwet,
                         const double* rhs, double* u) {
  const int64_t plane = (int64_t)ngrid * ngrid;
  const int64_t nlines = (int64_t)nslice * ngrid;
  const int64_t step = dir == 1 ? 1 : ngrid;
#pragma omp parallel for schedule(static)
  for (int64_t line = 0; line < nlines; line++) {
    const int64_t s = line / ngrid;
    const int64_t l = line - s * ngrid;
    const int64_t base = s * plane + (dir == 1 ? l * ngrid : l);
    double ur, ui;
    cmul(RE(rhs, base), IM(rhs, base), RE(cbet, 0), IM(cbet, 0), &ur, &ui);
    RE(u, base) = ur;
    IM(u, base) = ui;
    for (int k = 1; k < ngrid; k++) {
      const int64_t idx = base + k * step;
      double tr, ti;
      cmul(RE(c, k), IM(c, k), RE(u, idx - step), IM(u, idx - step), &tr, &ti);
      cmul(RE(rhs, idx) - tr, IM(rhs, idx) - ti, RE(cbet, k), IM(cbet, k), &ur,
           &ui);
      RE(u, idx) = ur;
      IM(u, idx) = ui;
    }
    for (int k = ngrid - 2; k >= 0; k--) {
      const int64_t idx = base + k * step;
      double tr, ti;
      cmul(RE(cwet, k + 1), IM(cwet, k + 1), RE(u, idx + step),
           IM(u, idx + step), &tr, &ti);
      RE(u, idx) = RE(u, idx) - tr;
      IM(u, idx) = IM(u, idx) - ti;
    }
  }
}

/* src/Core/FieldSolverADICUDA.cpp:638-818 (source-grid mode). */
void g4o_adi_advance(int nslice, int ngrid, int first, int harm,
                     double gridmax, double xks, double delz, double fc,
                     int enabled, const g4b_step* st, const int64_t* off,
                     const double* current, const double* x, const double* y,
                     const double* gamma, const double* theta, double* field,
                     double* work) {
  const double dgrid = 2.0 * gridmax / (double)(ngrid - 1);
  const int64_t cells = (int64_t)nslice * ngrid * ngrid;
  double* c = (double*)malloc(sizeof(double) * 6 * ngrid);
  double* cbet = c + 2 * ngrid;
  double* cwet = c + 4 * ngrid;
  double r = 0;
  g4o_adi_coeffs(ngrid, delz, dgrid, xks, c, cbet, cwet, &r);
  double* rbuf = work;
  double* src = work + 2 * cells;
  const int do_source = st->in_undulator && enabled && (harm % 2) == 1;
  const int use_source = do_source && off[nslice] > 0;
  if (use_source) {
    double* scl = (double*)malloc(sizeof(double) * nslice);
    g4o_slice_scl(nslice, off, current, fc, xks, dgrid, delz, scl);
    g4o_deposit(nslice, ngrid, first, harm, gridmax, dgrid, st, off, x, y,
                gamma, theta, scl, src);
    free(scl);
  }
  rhs_build(nslice, ngrid, r, 0, use_source ? src : NULL, field, rbuf);
  thomas_lines(nslice, ngrid, 1, c, cbet, cwet, rbuf, field);
  rhs_build(nslice, ngrid, r, 1, use_source ? src : NULL, field, rbuf);
  thomas_lines(nslice, ngrid, 0, c, cbet, cwet, rbuf, field);
  free(c);
}

/* ---- transverse tracking: src/Core/TrackBeamCUDA.cpp ------------------- */

typedef struct {
  int mode; /* 0 drift, 1 focusing, 2 defocusing */
  double strength, offset;
} plane_map;

static plane_map make_plane_map(double strength, double offset) { /* :61-69 */
  plane_map m = {0, strength, 0.0};
  if (strength == 0.0) return m;
  m.offset = offset / strength;
  m.mode = strength > 0.0 ? 1 : 2;
  return m;
}

static inline void advance_plane(plane_map m, double delz, double* coord,
                                 double* mom, double gammaz) { /* :27-59 */
  if (m.mode == 0) {
    *coord += *mom * delz / gammaz;
    return;
  }
  if (m.mode == 1) {
    const double foc = sqrt(m.strength / gammaz);
    const double omg = foc * delz;
    const double a1 = cos(omg);
    const double a2 = sin(omg) / foc;
    const double a3 = -a2 * foc * foc;
    const double xt = *coord - m.offset;
    *coord = a1 * xt + a2 * *mom / gammaz + m.offset;
    *mom = a3 * xt * gammaz + a1 * *mom;
    return;
  }
  const double foc = sqrt(-m.strength / gammaz);
  const double omg = foc * delz;
  const double a1 = cosh(omg);
  const double a2 = sinh(omg) / foc;
  const double a3 = a2 * foc * foc;
  const double xt = *coord - m.offset;
  *coord = a1 * xt + a2 * *mom / gammaz + m.offset;
  *mom = a3 * xt * gammaz + a1 * *mom;
}

typedef struct {
  double v[4][4];
} mat4;

static mat4 mat_identity(void) {
  mat4 m;
  memset(&m, 0, sizeof m);
  for (int i = 0; i < 4; i++) m.v[i][i] = 1.0;
  return m;
}

static void left_multiply(mat4* m, const mat4* e) { /* :80-91 */
  mat4 t;
  memset(&t, 0, sizeof t);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) t.v[i][j] += e->v[i][k] * m->v[k][j];
  *m = t;
}

static mat4 chicane_matrix(double angle, double lb, double ld, double lt) {
  /* :93-148 */
  mat4 m = mat_identity(), d1 = mat_identity(), d2 = mat_identity(),
       d3 = mat_identity(), bp = mat_identity(), bn = mat_identity(),
       ep = mat_identity(), en = mat_identity();
  d1.v[0][1] = ld / cos(angle);
  d1.v[2][3] = ld / cos(angle);
  d2.v[0][1] = lt - 4 * lb - 2 * ld;
  d2.v[2][3] = lt - 4 * lb - 2 * ld;
  d3.v[0][1] = -lt;
  d3.v[2][3] = -lt;
  const double radius = lb / sin(angle);
  const double path = radius * angle;
  bp.v[2][3] = path;
  bp.v[0][0] = cos(angle);
  bp.v[0][1] = radius * sin(angle);
  bp.v[1][0] = -sin(angle) / radius;
  bp.v[1][1] = cos(angle);
  bn.v[2][3] = path;
  bn.v[0][0] = cos(-angle);
  bn.v[0][1] = radius * sin(-angle) * -1;
  bn.v[1][0] = -sin(-angle) / radius * -1;
  bn.v[1][1] = cos(-angle);
  const double edge = tan(angle) / radius;
  ep.v[1][0] = edge;
  ep.v[3][2] = -edge;
  en.v[1][0] = -edge * -1;
  en.v[3][2] = edge * -1;
  left_multiply(&m, &bp);
  left_multiply(&m, &ep);
  left_multiply(&m, &d1);
  left_multiply(&m, &en);
  left_multiply(&m, &bn);
  left_multiply(&m, &d2);
  left_multiply(&m, &bn);
  left_multiply(&m, &en);
  left_multiply(&m, &d1);
  left_multiply(&m, &ep);
  left_multiply(&m, &bp);
  left_multiply(&m, &d3);
  return m;
}

void g4o_track(int64_t npart, const g4b_step* st, double delz, int last_step,
               double* x, double* y, double* px, double* py,
               const double* gamma) { /* :156-255 */
  const double gamma0 = st->gamma_ref;
  const double aw = st->aw;
  const double betpar0 = sqrt(1 - (1 + aw * aw) / gamma0 / gamma0);
  const double quad = st->qf * gamma0;
  const double qnatx = st->kx * aw * aw / gamma0 / betpar0;
  const double qnaty = st->ky * aw * aw / gamma0 / betpar0;
  const double qx = quad + qnatx;
  const double qy = -quad + qnaty;
  const double xoff = quad * st->dqx + qnatx * st->ax;
  const double yoff = -quad * st->dqy + qnaty * st->ay;
  if (last_step) {
    if (st->cx != 0 || st->cy != 0) {
      const double cx = st->cx * gamma0, cy = st->cy * gamma0;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < npart; i++) {
        px[i] += cx;
        py[i] += cy;
      }
    }
  } else if (st->chic_angle != 0) {
    const mat4 m =
        chicane_matrix(st->chic_angle, st->chic_lb, st->chic_ld, st->chic_lt);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < npart; i++) {
      const double gz =
          sqrt(gamma[i] * gamma[i] - 1.0 - px[i] * px[i] - py[i] * py[i]);
      double tmp = x[i];
      x[i] = m.v[0][0] * tmp + m.v[0][1] * px[i] / gz;
      px[i] = m.v[1][0] * tmp * gz + m.v[1][1] * px[i];
      tmp = y[i];
      y[i] = m.v[2][2] * tmp + m.v[2][3] * py[i] / gz;
      py[i] = m.v[3][2] * tmp * gz + m.v[3][3] * py[i];
    }
  }
  const plane_map xm = make_plane_map(qx, xoff);
  const plane_map ym = make_plane_map(qy, yoff);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npart; i++) {
    const double gz = sqrt(gamma[i] * gamma[i] - 1.0 - aw * aw -
                           px[i] * px[i] - py[i] * py[i]);
    advance_plane(xm, delz, &x[i], &px[i], gz);
    advance_plane(ym, delz, &y[i], &py[i], gz);
  }
}

void g4o_r56(int64_t npart, const g4b_step* st, double lambda0,
             const double* gamma, double* theta) { /* :257-278 */
  const double angle = st->chic_angle, lb = st->chic_lb, ld = st->chic_ld;
  const double gamma0 = st->gamma_ref;
  if (angle == 0) return;
  double r56 = (4 * lb / sin(angle) * (1 - angle / tan(angle)) +
                2 * ld * tan(angle) / cos(angle)) *
               angle;
  r56 = r56 * 4 * asin(1.0) / lambda0 / gamma0;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npart; i++) theta[i] += r56 * (gamma[i] - gamma0);
}

/* ---- longitudinal push: src/Core/BeamSolverCUDA.cpp -------------------- */

#define G4O_MAX_FIELDS 8

static inline void sample_field(const g4o_field_view* f, double rtmp,
                                int slice, double x, double y, double awloc,
                                double* rr, double* ri) { /* :87-143 */
  *rr = 0.0;
  *ri = 0.0;
  const int ng = f->ngrid;
  const double gm = f->gridmax;
  if (x <= -gm || x >= gm || y <= -gm || y >= gm) return;
  double wx = (x + gm) / f->dgrid;
  double wy = (y + gm) / f->dgrid;
  const int ix = (int)floor(wx);
  const int iy = (int)floor(wy);
  if (ix < 0 || ix >= ng - 1 || iy < 0 || iy >= ng - 1) return;
  wx = 1.0 + (double)ix - wx;
  wy = 1.0 + (double)iy - wy;
  const int islice = (slice + f->first) % f->nslice;
  const int64_t plane = (int64_t)ng * ng;
  int64_t idx = ix + (int64_t)iy * ng;
  const double* c = f->cells + 2 * plane * islice;
  const double w00 = wx * wy, w10 = (1.0 - wx) * wy;
  const double w01 = wx * (1.0 - wy), w11 = (1.0 - wx) * (1.0 - wy);
  double cre = RE(c, idx) * w00;
  double cim = IM(c, idx) * w00;
  ++idx;
  cre += RE(c, idx) * w10;
  cim += IM(c, idx) * w10;
  idx += ng - 1;
  cre += RE(c, idx) * w01;
  cim += IM(c, idx) * w01;
  ++idx;
  cre += RE(c, idx) * w11;
  cim += IM(c, idx) * w11;
  const double scale = rtmp * awloc;
  *rr = scale * cre;
  *ri = -scale * cim;
}

static inline void ode(double tgam, double tthet, double btpar, double ez,
                       double xks, double xku, int nfield,
                       const double* rharm, const double* rr, const double* ri,
                       double* k2gg, double* k2pp) { /* :146-180 */
  const double ztemp1 = -2.0 / xks;
  double ctr = 0.0, cti = 0.0;
  for (int i = 0; i < nfield; i++) {
    const double arg = rharm[i] * tthet;
    const double c = cos(arg), s = sin(arg);
    ctr += rr[i] * c + ri[i] * s;
    cti += ri[i] * c - rr[i] * s;
  }
  const double btper0 = btpar + ztemp1 * ctr;
  const double btpar0 = sqrt(1.0 - btper0 / (tgam * tgam));
  *k2pp += xks * (1.0 - 1.0 / btpar0) + xku;
  *k2gg += cti / btpar0 / tgam - ez;
}

void g4o_push(int nslice, const int64_t* off, const g4b_step* st,
              const g4o_field_view* fields, int nfield,
              const double* slice_eloss, const double* x, const double* y,
              const double* px, const double* py, double* gamma,
              double* theta) {
  g4o_push_ez(nslice, off, st, fields, nfield, slice_eloss, NULL, x, y, px, py, gamma, theta);
}

void g4o_push_ez(int nslice, const int64_t* off, const g4b_step* st,
                 const g4o_field_view* fields, int nfield,
                 const double* slice_eloss, const double* particle_ez,
                 const double* x, const double* y, const double* px,
                 const double* py, double* gamma,
                 double* theta) { /* :449-683 and :226-409 */
  if (nfield <= 0 || nfield > G4O_MAX_FIELDS) return;
  double rtmp[G4O_MAX_FIELDS], rharm[G4O_MAX_FIELDS];
  double xks_local = 1.0;
  for (int i = 0; i < nfield; i++) {
    xks_local = fields[i].xks / (double)fields[i].harm;
    rtmp[i] = fields[i].fc / fields[i].xks;
    rharm[i] = (double)fields[i].harm;
  }
  double xku = st->ku;
  if (xku == 0.0) xku = xks_local * 0.5 / st->gamma_ref / st->gamma_ref;
  const double aw = st->aw;
  const double delz = st->delz;
#pragma omp parallel for schedule(dynamic, 1)
  for (int is = 0; is < nslice; is++) {
    const double ez_slice = slice_eloss ? slice_eloss[is] : 0.0;
    for (int64_t ip = off[is]; ip < off[is + 1]; ip++) {
      /* load_longitudinal_ez (src/Core/BeamSolverCUDA.cpp:184-195) */
      const double ez = particle_ez ? particle_ez[ip] : ez_slice;
      double g = gamma[ip];
      double th = theta[ip] + st->autophase;
      const double xp = x[ip], yp = y[ip];
      const double dx = xp - st->ax, dy = yp - st->ay;
      const double awloc = 1.0 + 0.5 * (st->kx * dx * dx + st->ky * dy * dy) +
                           st->gradx * dx + st->grady * dy;
      const double btpar =
          1.0 + px[ip] * px[ip] + py[ip] * py[ip] + aw * aw * awloc * awloc;
      double rr[G4O_MAX_FIELDS], ri[G4O_MAX_FIELDS];
      for (int f = 0; f < nfield; f++)
        sample_field(&fields[f], rtmp[f], is, xp, yp, awloc, &rr[f], &ri[f]);
      double k2gg = 0.0, k2pp = 0.0, k3gg, k3pp;
      ode(g, th, btpar, ez, xks_local, xku, nfield, rharm, rr, ri, &k2gg,
          &k2pp);
      double stpz = 0.5 * delz;
      g += stpz * k2gg;
      th += stpz * k2pp;
      k3gg = k2gg;
      k3pp = k2pp;
      k2gg = 0.0;
      k2pp = 0.0;
      ode(g, th, btpar, ez, xks_local, xku, nfield, rharm, rr, ri, &k2gg,
          &k2pp);
      g += stpz * (k2gg - k3gg);
      th += stpz * (k2pp - k3pp);
      k3gg /= 6.0;
      k3pp /= 6.0;
      k2gg *= -0.5;
      k2pp *= -0.5;
      ode(g, th, btpar, ez, xks_local, xku, nfield, rharm, rr, ri, &k2gg,
          &k2pp);
      stpz = delz;
      g += stpz * k2gg;
      th += stpz * k2pp;
      k3gg -= k2gg;
      k3pp -= k2pp;
      k2gg *= 2.0;
      k2pp *= 2.0;
      ode(g, th, btpar, ez, xks_local, xku, nfield, rharm, rr, ri, &k2gg,
          &k2pp);
      g += stpz * (k3gg + k2gg / 6.0);
      th += stpz * (k3pp + k2pp / 6.0);
      gamma[ip] = g;
      theta[ip] = th;
    }
  }
}

/* ---- slippage: src/Core/ControlCUDA.cpp:148-252 (rank 0 of 1) ----------- */
int g4o_slippage(int nslice, int ngrid, double shift, double sample,
                 int time_run, int periodic, double* accuslip, int* first,
                 double* field) {
  if (!time_run) return 0;
  *accuslip += shift;
  const int64_t plane = (int64_t)ngrid * ngrid;
  int nshift = 0;
  int direction = 1;
  while (fabs(*accuslip) > sample * 0.8) {
    direction = *accuslip < 0 ? -1 : 1;
    *accuslip -= sample * direction;
    int last = (*first + nslice - 1) % nslice;
    if (direction < 0) last = (last + 1) % nslice;
    if (!periodic) memset(field + 2 * plane * last, 0, sizeof(double) * 2 * plane);
    *first = last;
    if (direction < 0) *first = (last + 1) % nslice;
    nshift++;
  }
  return nshift;
}

/* ---- diagnostics: src/Core/DiagnosticCUDA.cpp:188-363 ------------------- */
void g4o_diag_beam(int nslice, const int64_t* off, int nharm, int need_aux,
                   const double* x, const double* y, const double* px,
                   const double* py, const double* gamma, const double* theta,
                   double* stats, double* bre, double* bim) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int is = 0; is < nslice; is++) {
    double s[23] = {0};
    double xmin = 1.0e5, xmax = -1.0e5, pxmin = 1.0e5, pxmax = -1.0e5;
    double ymin = 1.0e5, ymax = -1.0e5, pymin = 1.0e5, pymax = -1.0e5;
    double gmin = 1.0e7, gmax = 1.0;
    for (int64_t ip = off[is]; ip < off[is + 1]; ip++) {
      const double xv = x[ip], yv = y[ip], pxv = px[ip], pyv = py[ip],
                   gv = gamma[ip];
      s[0] += gv;
      s[1] += gv * gv;
      s[2] += xv;
      s[3] += xv * xv;
      s[4] += yv;
      s[5] += yv * yv;
      s[6] += pxv;
      s[7] += pxv * pxv;
      s[8] += pyv;
      s[9] += pyv * pyv;
      s[10] += xv * pxv;
      s[11] += yv * pyv;
      s[12] += 1.0;
      if (need_aux) {
        xmin = fmin(xmin, xv);
        xmax = fmax(xmax, xv);
        pxmin = fmin(pxmin, pxv);
        pxmax = fmax(pxmax, pxv);
        ymin = fmin(ymin, yv);
        ymax = fmax(ymax, yv);
        pymin = fmin(pymin, pyv);
        pymax = fmax(pymax, pyv);
        gmin = fmin(gmin, gv);
        gmax = fmax(gmax, gv);
      }
    }
    double* o = stats + 23 * (int64_t)is;
    for (int k = 0; k < 13; k++) o[k] = s[k];
    if (need_aux) {
      o[13] = xmin;
      o[14] = xmax;
      o[15] = pxmin;
      o[16] = pxmax;
      o[17] = ymin;
      o[18] = ymax;
      o[19] = pymin;
      o[20] = pymax;
      o[21] = gmin;
      o[22] = gmax;
    } else {
      for (int k = 13; k < 23; k++) o[k] = 0.0;
    }
    for (int ih = 0; ih < nharm; ih++) {
      const double h = (double)(ih + 1);
      double br = 0.0, bi = 0.0;
      for (int64_t ip = off[is]; ip < off[is + 1]; ip++) {
        const double ph = h * theta[ip];
        br += cos(ph);
        bi += sin(ph);
      }
      bre[(int64_t)is * nharm + ih] = br;
      bim[(int64_t)is * nharm + ih] = bi;
    }
  }
}

void g4o_diag_field(int nslice, int ngrid, int first, const double* field,
                    double* stats, double* center) {
  const int64_t plane = (int64_t)ngrid * ngrid;
  const double shift = -0.5 * (double)(ngrid - 1);
#pragma omp parallel for schedule(dynamic, 1)
  for (int is0 = 0; is0 < nslice; is0++) {
    const double* c = field + 2 * plane * is0;
    const int is = (nslice + is0 - first) % nslice;
    double p = 0, x1 = 0, x2 = 0, y1 = 0, y2 = 0, fr = 0, fi = 0;
    for (int64_t ixy = 0; ixy < plane; ixy++) {
      const int iy = (int)(ixy / ngrid);
      const int ix = (int)(ixy - (int64_t)iy * ngrid);
      const double re = RE(c, ixy), im = IM(c, ixy);
      const double wei = re * re + im * im;
      const double dx = (double)ix + shift, dy = (double)iy + shift;
      p += wei;
      x1 += dx * wei;
      x2 += dx * dx * wei;
      y1 += dy * wei;
      y2 += dy * dy * wei;
      fr += re;
      fi += im;
    }
    double* o = stats + 7 * (int64_t)is;
    o[0] = p;
    o[1] = x1;
    o[2] = x2;
    o[3] = y1;
    o[4] = y2;
    o[5] = fr;
    o[6] = fi;
    const int64_t ic = (plane - 1) / 2;
    center[2 * is] = RE(c, ic);
    center[2 * is + 1] = IM(c, ic);
  }
}

/* ---- one Gencore step (src/Core/Gencore.cpp:172-234) ------------------- */
void g4o_step(int nslice, const int64_t* off, const double* current,
              const double* slice_eloss, const g4b_step* st, double lambda0,
              double slippage, double sample, int time_run, int periodic,
              g4o_field_state* fields, int nfield, double* x, double* y,
              double* px, double* py, double* gamma, double* theta,
              double* work) {
  const int64_t npart = off[nslice];
  const double delz = st->delz;
  /* Beam::track (src/Core/Beam.cpp:117-133) */
  g4o_track(npart, st, delz * 0.5, 0, x, y, px, py, gamma);
  g4o_field_view views[G4O_MAX_FIELDS];
  for (int i = 0; i < nfield && i < G4O_MAX_FIELDS; i++) {
    const g4o_field_state* f = &fields[i];
    const double xl = f->xlambda;
    views[i].first = f->first;
    views[i].ngrid = f->ngrid;
    views[i].nslice = nslice;
    views[i].harm = f->harm;
    views[i].gridmax = f->gridmax;
    views[i].dgrid = 2.0 * f->gridmax / (double)(f->ngrid - 1);
    views[i].xks = 4.0 * asin(1.0) / xl;
    views[i].fc = f->fc;
    views[i].cells = f->cells;
  }
  g4o_push(nslice, off, st, views, nfield, slice_eloss, x, y, px, py, gamma,
           theta);
  g4o_r56(npart, st, lambda0, gamma, theta);
  g4o_track(npart, st, delz * 0.5, 1, x, y, px, py, gamma);
  /* Field::track for every field (src/Core/Gencore.cpp:215-217) */
  for (int i = 0; i < nfield; i++) {
    g4o_field_state* f = &fields[i];
    const double xks = 4.0 * asin(1.0) / f->xlambda;
    g4o_adi_advance(nslice, f->ngrid, f->first, f->harm, f->gridmax, xks, delz,
                    f->fc, f->enabled, st, off, current, x, y, gamma, theta,
                    f->cells, work);
  }
  /* slippage (src/Core/Gencore.cpp:228-230) */
  for (int i = 0; i < nfield; i++) {
    g4o_field_state* f = &fields[i];
    g4o_slippage(nslice, f->ngrid, slippage, sample, time_run, periodic,
                 &f->accuslip, &f->first, f->cells);
  }
}

/* ---- beam loading: Hammersley quiet start + shot noise ------------------
 * The loader of upstream GENESIS 1.3 v4 is absent from the reference tree.
 * This restates, operation for operation, the loader the drop-in host layer
 * uses (beamlets of nbins particles at Hammersley points with radical
 * inverses in bases 2, 3, 5, 7, 11 mapped through the inverse normal CDF,
 * phase base 13; Fawley shot noise from a SplitMix64 stream per slice), so
 * the CPU baseline starts from the same bits without loading the product. */
static double g4o_radical_inverse(uint64_t i, unsigned base) {
  double inv = 1.0 / base, f = inv, r = 0.0;
  while (i) {
    r += f * (double)(i % base);
    i /= base;
    f *= inv;
  }
  return r;
}

/* Inverse normal CDF: P. J. Acklam's rational approximation (2003) refined by
 * one Halley step against erfc. */
static double g4o_inv_normal(double p) {
  static const double a[] = {-3.969683028665376e+01, 2.209460984245205e+02,
                             -2.759285104469687e+02, 1.383577518672690e+02,
                             -3.066479806614716e+01, 2.506628277459239e+00};
  static const double b[] = {-5.447609879822406e+01, 1.615858368580409e+02,
                             -1.556989798598866e+02, 6.680131188771972e+01,
                             -1.328068155288572e+01};
  static const double c[] = {-7.784894002430293e-03, -3.223964580411365e-01,
                             -2.400758277161838e+00, -2.549732539343734e+00,
                             4.374664141464968e+00, 2.938163982698783e+00};
  static const double d[] = {7.784695709041462e-03, 3.224671290700398e-01,
                             2.445134137142996e+00, 3.754408661907416e+00};
  if (p <= 0.0) return -40.0;
  if (p >= 1.0) return 40.0;
  double x;
  const double plow = 0.02425, phigh = 1 - plow;
  if (p < plow) {
    const double q = sqrt(-2 * log(p));
    x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
  } else if (p <= phigh) {
    const double q = p - 0.5, r = q * q;
    x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
        (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1);
  } else {
    const double q = sqrt(-2 * log(1 - p));
    x = -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
  }
  const double e = 0.5 * erfc(-x / sqrt(2.0)) - p;
  const double u = e * sqrt(2 * M_PI) * exp(x * x / 2);
  return x - u / (1 + x * u / 2);
}

static double g4o_uniform(uint64_t* s) {
  *s += 0x9e3779b97f4a7c15ull;
  uint64_t z = *s;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static double g4o_normal(uint64_t* s) {
  const double u1 = g4o_uniform(s), u2 = g4o_uniform(s);
  return sqrt(-2 * log(u1)) * cos(2 * M_PI * u2);
}

int g4o_load_beam(const g4o_beam_spec* sp, const double* current, double* x,
                  double* y, double* px, double* py, double* gamma,
                  double* theta, int64_t* off) {
  if (sp->nslice <= 0 || sp->npart < 0 || sp->nbins <= 0 || sp->npart % sp->nbins)
    return 1;
  const int nbl = sp->npart / sp->nbins;
  const double gref = sp->gamma0;
  const double epx = sp->ex / gref, epy = sp->ey / gref;
  const double sx = sqrt(epx * sp->betax), sy = sqrt(epy * sp->betay);
  const double spx = sqrt(epx / sp->betax), spy = sqrt(epy / sp->betay);
  const double twopi = 2 * M_PI;
  const double ce = 1.602176634e-19, c0 = 299792458.0;
  off[0] = 0;
  for (int s = 0; s < sp->nslice; ++s) off[s + 1] = (int64_t)(s + 1) * sp->npart;
#pragma omp parallel for schedule(dynamic, 1)
  for (int s = 0; s < sp->nslice; ++s) {
    uint64_t rng = sp->seed * 0x100000001b3ull + (uint64_t)s * 0x9e3779b97f4a7c15ull + 1;
    const int64_t base = (int64_t)s * sp->npart;
    const int nbl1 = nbl > 1 ? nbl : 1;
    const double ne = current[s] * sp->slicelength / (ce * c0) / nbl1;
    for (int j = 0; j < nbl; ++j) {
      const uint64_t idx = (uint64_t)s * nbl + j + 1;
      const double g1 = g4o_inv_normal(g4o_radical_inverse(idx, 2));
      const double g2 = g4o_inv_normal(g4o_radical_inverse(idx, 3));
      const double g3 = g4o_inv_normal(g4o_radical_inverse(idx, 5));
      const double g4 = g4o_inv_normal(g4o_radical_inverse(idx, 7));
      const double g5 = g4o_inv_normal(g4o_radical_inverse(idx, 11));
      const double th0 = twopi / sp->nbins * g4o_radical_inverse(idx, 13);
      const double xv = sx * g1 + sp->xcenter;
      const double yv = sy * g3 + sp->ycenter;
      const double xp = spx * (g2 - sp->alphax * g1);
      const double yp = spy * (g4 - sp->alphay * g3);
      const double gv = gref + sp->delgam * g5;
      const double pxv = gv * xp + sp->pxcenter;
      const double pyv = gv * yp + sp->pycenter;
      double an[64], bn[64];
      const int nh = sp->nbins / 2;
      for (int h = 1; h <= nh && h <= 64; ++h) {
        const double sig = (sp->shotnoise && ne > 0) ? sqrt(2.0 / ne) / h : 0.0;
        an[h - 1] = sig * g4o_normal(&rng);
        bn[h - 1] = sig * g4o_normal(&rng);
      }
      for (int k = 0; k < sp->nbins; ++k) {
        const int64_t p = base + (int64_t)j * sp->nbins + k;
        const double th = th0 + twopi * k / sp->nbins;
        double dth = 0.0;
        for (int h = 1; h <= nh && h <= 64; ++h)
          dth += an[h - 1] * cos(h * th) + bn[h - 1] * sin(h * th);
        x[p] = xv;
        y[p] = yv;
        px[p] = pxv;
        py[p] = pyv;
        gamma[p] = gv;
        theta[p] = th + dth;
      }
    }
  }
  return 0;
}

/* ---- incoherent synchrotron radiation -----------------------------------
 * Restates the device model of g4b_beam_incoherent (the reference leaves it
 * to upstream Incoherent::apply on the host, src/Core/Beam.cpp:126; upstream
 * is absent): gamma += -loss gamma^2 + sigma gamma^2 z, z from Philox4x32-10
 * (Salmon et al., SC 2011) keyed by the seed with counter (index, counter)
 * and the Box-Muller transform.  loss and sigma already hold the step
 * length: loss = rate delz, sigma = sqrt(spread rate delz). */
static void philox_round(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
  const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
  c[0] = n0;
  c[1] = lo1;
  c[2] = n2;
  c[3] = lo0;
}

void g4o_philox4x32_10(uint32_t ctr[4], const uint32_t key[2]) {
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    philox_round(ctr, k0, k1);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

static double unit53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}

void g4o_incoherent(int64_t n, double* gamma, double loss, double sigma, uint64_t seed,
                    uint64_t counter) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    const double g = gamma[i], g2 = g * g;
    double dg = -loss * g2;
    if (sigma > 0.0) {
      uint32_t c[4] = {(uint32_t)i, (uint32_t)((uint64_t)i >> 32), (uint32_t)counter,
                       (uint32_t)(counter >> 32)};
      g4o_philox4x32_10(c, key);
      const double u = unit53(c[0], c[1]), v = unit53(c[2], c[3]);
      dg += sigma * g2 * (sqrt(-2.0 * log(u)) * cos(6.283185307179586 * v));
    }
    gamma[i] = g + dg;
  }
}
