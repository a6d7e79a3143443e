// g4b_beam.cu -- beam solver kernels (TrackBeamCUDA, BeamSolverCUDA) for sm_100a.
//
// The push runs one CTA per chunk of <= 256 particles of one slice (the chunk
// table is built once from the slice offsets), so every CTA gathers from one
// field plane and no per-particle slice index is read.
#include <algorithm>
#include <cmath>

#include "g4b_internal.cuh"

namespace g4b {

// ---------------------------------------------------- transverse tracking ---
struct PlaneMap {
  int mode;  // 0 drift, 1 focusing, 2 defocusing
  double strength, offset;
};

// make_plane_map (src/Core/TrackBeamCUDA.cpp:61-69)
static PlaneMap make_plane_map(double strength, double offset) {
  PlaneMap m{0, strength, 0.0};
  if (strength == 0.0) return m;
  m.offset = offset / strength;
  m.mode = strength > 0.0 ? 1 : 2;
  return m;
}

// advance_focusing_plane (src/Core/TrackBeamCUDA.cpp:27-59)
__device__ __forceinline__ void advance_plane(const PlaneMap m, double delz, double& coord,
                                              double& mom, double gammaz) {
  if (m.mode == 0) {
    coord += mom * delz / gammaz;
    return;
  }
  if (m.mode == 1) {
    const double foc = sqrt(m.strength / gammaz);
    const double omg = foc * delz;
    double sn, cs;
    sincos(omg, &sn, &cs);
    const double a1 = cs;
    const double a2 = sn / foc;
    const double a3 = -a2 * foc * foc;
    const double xt = coord - m.offset;
    coord = a1 * xt + a2 * mom / gammaz + m.offset;
    mom = a3 * xt * gammaz + a1 * mom;
    return;
  }
  const double foc = sqrt(-m.strength / gammaz);
  const double omg = foc * delz;
  const double a1 = cosh(omg);
  const double a2 = sinh(omg) / foc;
  const double a3 = a2 * foc * foc;
  const double xt = coord - m.offset;
  coord = a1 * xt + a2 * mom / gammaz + m.offset;
  mom = a3 * xt * gammaz + a1 * mom;
}

struct TrackArgs {
  double *x, *y, *px, *py;
  const double* gamma;
  int64_t n;
  PlaneMap xm, ym;
  double aw, delz;
  // pre-kick: corrector (mode 1) or chicane (mode 2)
  int pre;
  double cx, cy;
  double m00, m01, m10, m11, m22, m23, m32, m33;
};

__global__ void __launch_bounds__(256) track_kernel(const TrackArgs a) {
  ptx::pdl_wait();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    double x = a.x[i], y = a.y[i], px = a.px[i], py = a.py[i];
    const double g = a.gamma[i];
    if (a.pre == 1) {  // applyCorrector (src/Core/TrackBeamCUDA.cpp:206-218)
      px += a.cx;
      py += a.cy;
    } else if (a.pre == 2) {  // applyChicane (:220-255)
      const double gz = sqrt(g * g - 1.0 - px * px - py * py);
      double tmp = x;
      x = a.m00 * tmp + a.m01 * px / gz;
      px = a.m10 * tmp * gz + a.m11 * px;
      tmp = y;
      y = a.m22 * tmp + a.m23 * py / gz;
      py = a.m32 * tmp * gz + a.m33 * py;
    }
    const double gz = sqrt(g * g - 1.0 - a.aw * a.aw - px * px - py * py);
    advance_plane(a.xm, a.delz, x, px, gz);
    advance_plane(a.ym, a.delz, y, py, gz);
    a.x[i] = x;
    a.y[i] = y;
    a.px[i] = px;
    a.py[i] = py;
  }
}

struct Mat4 {
  double v[4][4];
};

static Mat4 mat_identity() {
  Mat4 m{};
  for (int i = 0; i < 4; ++i) m.v[i][i] = 1.0;
  return m;
}

static void left_multiply(Mat4& m, const Mat4& e) {
  Mat4 t{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) t.v[i][j] += e.v[i][k] * m.v[k][j];
  m = t;
}

// build_chicane_matrix (src/Core/TrackBeamCUDA.cpp:93-148)
static Mat4 chicane_matrix(double angle, double lb, double ld, double lt) {
  Mat4 m = mat_identity(), d1 = mat_identity(), d2 = mat_identity(),
       d3 = mat_identity(), bp = mat_identity(), bn = mat_identity(),
       ep = mat_identity(), en = mat_identity();
  d1.v[0][1] = d1.v[2][3] = ld / std::cos(angle);
  d2.v[0][1] = d2.v[2][3] = lt - 4 * lb - 2 * ld;
  d3.v[0][1] = d3.v[2][3] = -lt;
  const double radius = lb / std::sin(angle);
  const double path = radius * angle;
  bp.v[2][3] = path;
  bp.v[0][0] = std::cos(angle);
  bp.v[0][1] = radius * std::sin(angle);
  bp.v[1][0] = -std::sin(angle) / radius;
  bp.v[1][1] = std::cos(angle);
  bn.v[2][3] = path;
  bn.v[0][0] = std::cos(-angle);
  bn.v[0][1] = radius * std::sin(-angle) * -1;
  bn.v[1][0] = -std::sin(-angle) / radius * -1;
  bn.v[1][1] = std::cos(-angle);
  const double edge = std::tan(angle) / radius;
  ep.v[1][0] = edge;
  ep.v[3][2] = -edge;
  en.v[1][0] = -edge * -1;
  en.v[3][2] = edge * -1;
  const Mat4* seq[] = {&bp, &ep, &d1, &en, &bn, &d2, &bn, &en, &d1, &ep, &bp, &d3};
  for (const Mat4* e : seq) left_multiply(m, *e);
  return m;
}

// --------------------------------------------------------------- R56 kick ---
__global__ void __launch_bounds__(256) r56_kernel(int64_t n, const double* gamma,
                                                  double* theta, double r56,
                                                  double gamma0) {
  ptx::pdl_wait();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    theta[i] += r56 * (gamma[i] - gamma0);
}

// ------------------------------------------------------------------- push ---
constexpr int kMaxFields = 8;

struct PushField {
  const double2* cells;
  int first, n, ld, nslice;
  double gridmax, dgrid, rtmp, rharm;
};

struct PushArgs {
  double *gamma, *theta;
  const double *x, *y, *px, *py;
  const int4* chunks;
  const double* eloss;
  const double* pez;  // per-particle loss, or null: the slice's eloss
  PushField f[kMaxFields];
  int nfield;
  double xks, xku, aw, autophase, delz, ax, ay, kx, ky, gradx, grady;
};

// sample_single_field (src/Core/BeamSolverCUDA.cpp:87-143)
__device__ __forceinline__ void sample_field(const PushField& f, int slice, double x,
                                             double y, double awloc, double& rr,
                                             double& ri) {
  rr = 0.0;
  ri = 0.0;
  const int ng = f.n;
  const double gm = f.gridmax;
  if (x <= -gm || x >= gm || y <= -gm || y >= gm) return;
  double wx = (x + gm) / f.dgrid;
  double wy = (y + gm) / f.dgrid;
  const int ix = (int)floor(wx);
  const int iy = (int)floor(wy);
  if (ix < 0 || ix >= ng - 1 || iy < 0 || iy >= ng - 1) return;
  wx = 1.0 + (double)ix - wx;
  wy = 1.0 + (double)iy - wy;
  const int islice = (slice + f.first) % f.nslice;
  const double2* c = f.cells + (size_t)islice * ng * f.ld + (size_t)iy * f.ld + ix;
  const double2 c00 = __ldg(c), c10 = __ldg(c + 1);
  const double2 c01 = __ldg(c + f.ld), c11 = __ldg(c + f.ld + 1);
  const double w00 = wx * wy, w10 = (1.0 - wx) * wy;
  const double w01 = wx * (1.0 - wy), w11 = (1.0 - wx) * (1.0 - wy);
  double cre = c00.x * w00;
  double cim = c00.y * w00;
  cre += c10.x * w10;
  cim += c10.y * w10;
  cre += c01.x * w01;
  cim += c01.y * w01;
  cre += c11.x * w11;
  cim += c11.y * w11;
  const double scale = f.rtmp * awloc;
  rr = scale * cre;
  ri = -scale * cim;
}

// evaluate_longitudinal_ode_multi_field (src/Core/BeamSolverCUDA.cpp:146-180)
template <int NF>
__device__ __forceinline__ void ode(const PushArgs& a, int nf, double tgam, double tthet,
                                    double btpar, double ez, const double* rr,
                                    const double* ri, double& k2gg, double& k2pp) {
  const double ztemp1 = -2.0 / a.xks;
  double ctr = 0.0, cti = 0.0;
#pragma unroll
  for (int i = 0; i < (NF > 0 ? NF : kMaxFields); ++i) {
    if (NF == 0 && i >= nf) break;
    double s, c;
    sincos(a.f[i].rharm * tthet, &s, &c);
    ctr += rr[i] * c + ri[i] * s;
    cti += ri[i] * c - rr[i] * s;
  }
  const double btper0 = btpar + ztemp1 * ctr;
  const double btpar0 = sqrt(1.0 - btper0 / (tgam * tgam));
  k2pp += a.xks * (1.0 - 1.0 / btpar0) + a.xku;
  k2gg += cti / btpar0 / tgam - ez;
}

// push_longitudinal_particles_{single,multi}_field
// (src/Core/BeamSolverCUDA.cpp:226-409); NF = 1 for one field, 0 = generic.
template <int NF>
__global__ void __launch_bounds__(256) push_kernel(const PushArgs a) {
  ptx::pdl_wait();
  const int4 ch = a.chunks[blockIdx.x];
  if ((int)threadIdx.x >= ch.z) return;
  const int slice = ch.x;
  const int64_t ip = (((int64_t)ch.w) << 31) + (int64_t)(unsigned)ch.y + threadIdx.x;
  const int nf = NF > 0 ? NF : a.nfield;
  double gamma = a.gamma[ip];
  double theta = a.theta[ip] + a.autophase;
  const double xp = a.x[ip], yp = a.y[ip], pxp = a.px[ip], pyp = a.py[ip];
  const double dx = xp - a.ax, dy = yp - a.ay;
  const double awloc = 1.0 + 0.5 * (a.kx * dx * dx + a.ky * dy * dy) + a.gradx * dx + a.grady * dy;
  const double btpar = 1.0 + pxp * pxp + pyp * pyp + a.aw * a.aw * awloc * awloc;
  // load_longitudinal_ez (src/Core/BeamSolverCUDA.cpp:184-195)
  const double ez = a.pez ? a.pez[ip] : a.eloss[slice];
  double rr[NF > 0 ? NF : kMaxFields], ri[NF > 0 ? NF : kMaxFields];
#pragma unroll
  for (int i = 0; i < (NF > 0 ? NF : kMaxFields); ++i) {
    if (NF == 0 && i >= nf) {
      rr[i] = ri[i] = 0.0;
      continue;
    }
    sample_field(a.f[i], slice, xp, yp, awloc, rr[i], ri[i]);
  }
  double k2gg = 0.0, k2pp = 0.0, k3gg, k3pp;
  ode<NF>(a, nf, gamma, theta, btpar, ez, rr, ri, k2gg, k2pp);
  double stpz = 0.5 * a.delz;
  gamma += stpz * k2gg;
  theta += stpz * k2pp;
  k3gg = k2gg;
  k3pp = k2pp;
  k2gg = 0.0;
  k2pp = 0.0;
  ode<NF>(a, nf, gamma, theta, btpar, ez, rr, ri, k2gg, k2pp);
  gamma += stpz * (k2gg - k3gg);
  theta += stpz * (k2pp - k3pp);
  k3gg /= 6.0;
  k3pp /= 6.0;
  k2gg *= -0.5;
  k2pp *= -0.5;
  ode<NF>(a, nf, gamma, theta, btpar, ez, rr, ri, k2gg, k2pp);
  stpz = a.delz;
  gamma += stpz * k2gg;
  theta += stpz * k2pp;
  k3gg -= k2gg;
  k3pp -= k2pp;
  k2gg *= 2.0;
  k2pp *= 2.0;
  ode<NF>(a, nf, gamma, theta, btpar, ez, rr, ri, k2gg, k2pp);
  gamma += stpz * (k3gg + k2gg / 6.0);
  theta += stpz * (k3pp + k2pp / 6.0);
  a.gamma[ip] = gamma;
  a.theta[ip] = theta;
}

static unsigned grid_for(g4b_ctx* c, int64_t n, int block) {
  const int64_t want = (n + block - 1) / block;
  const int64_t cap = (int64_t)c->sm_count * 16;
  return (unsigned)std::max<int64_t>(1, std::min(want, cap));
}

}  // namespace g4b

using namespace g4b;

// Row-major 4x4 chicane matrix (build_chicane_matrix,
// src/Core/TrackBeamCUDA.cpp:93-148), shared with the fused form.
void g4b_chicane_matrix(double angle, double lb, double ld, double lt, double* out) {
  const Mat4 m = chicane_matrix(angle, lb, ld, lt);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) out[4 * i + j] = m.v[i][j];
}

extern "C" {

// TrackBeamCUDA::track (src/Core/TrackBeamCUDA.cpp:156-204)
int g4b_beam_track(g4b_beam* b, const g4b_step* st, double delz, int last_step) {
  if (!b || !st) return fail(G4B_ERR_ARG, "g4b_beam_track: null arg");
  if (b->precision != G4B_FP64) return fail(G4B_ERR_ARG, "g4b_beam_track: FP64 beam expected");
  if (b->npart == 0) return G4B_OK;
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  const double gamma0 = st->gamma_ref, aw = st->aw;
  const double betpar0 = std::sqrt(1 - (1 + aw * aw) / gamma0 / gamma0);
  const double quad = st->qf * gamma0;
  const double qnatx = st->kx * aw * aw / gamma0 / betpar0;
  const double qnaty = st->ky * aw * aw / gamma0 / betpar0;
  TrackArgs a{};
  a.x = b->x;
  a.y = b->y;
  a.px = b->px;
  a.py = b->py;
  a.gamma = b->gamma;
  a.n = b->npart;
  a.xm = make_plane_map(quad + qnatx, quad * st->dqx + qnatx * st->ax);
  a.ym = make_plane_map(-quad + qnaty, -quad * st->dqy + qnaty * st->ay);
  a.aw = aw;
  a.delz = delz;
  if (last_step) {
    if (st->cx != 0 || st->cy != 0) {
      a.pre = 1;
      a.cx = st->cx * gamma0;
      a.cy = st->cy * gamma0;
    }
  } else if (st->chic_angle != 0) {
    const Mat4 m = chicane_matrix(st->chic_angle, st->chic_lb, st->chic_ld, st->chic_lt);
    a.pre = 2;
    a.m00 = m.v[0][0];
    a.m01 = m.v[0][1];
    a.m10 = m.v[1][0];
    a.m11 = m.v[1][1];
    a.m22 = m.v[2][2];
    a.m23 = m.v[2][3];
    a.m32 = m.v[3][2];
    a.m33 = m.v[3][3];
  }
  {
    LaunchScope ls(c, "track");
    G4B_CUDA_TRY(launch_pdl(track_kernel, (unsigned)grid_for(c, b->npart, 256), 256, 0, c->stream, a));
  }
  return check_launch(c, "track_kernel");
}

// TrackBeamCUDA::applyR56 (src/Core/TrackBeamCUDA.cpp:257-278)
int g4b_beam_r56(g4b_beam* b, const g4b_step* st, double lambda0) {
  if (!b || !st) return fail(G4B_ERR_ARG, "g4b_beam_r56: null arg");
  const double angle = st->chic_angle, lb = st->chic_lb, ld = st->chic_ld;
  if (angle == 0 || b->npart == 0) return G4B_OK;
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  double r56 = (4 * lb / std::sin(angle) * (1 - angle / std::tan(angle)) +
                2 * ld * std::tan(angle) / std::cos(angle)) *
               angle;
  r56 = r56 * 4 * std::asin(1.0) / lambda0 / st->gamma_ref;
  {
    LaunchScope ls(c, "r56");
    G4B_CUDA_TRY(launch_pdl(r56_kernel, (unsigned)grid_for(c, b->npart, 256), 256, 0, c->stream,
                            b->npart, b->gamma, b->theta, r56, st->gamma_ref));
  }
  return check_launch(c, "r56_kernel");
}

// BeamSolverCUDA::advance (src/Core/BeamSolverCUDA.cpp:449-683)
int g4b_beam_advance(g4b_beam* b, g4b_field* const* fields, const double* fc, int nfield,
                     const g4b_step* st) {
  if (!b || !st || (nfield > 0 && (!fields || !fc)))
    return fail(G4B_ERR_ARG, "g4b_beam_advance: null arg");
  if (nfield > kMaxFields)
    return fail(G4B_ERR_RANGE, "g4b_beam_advance: more than 8 fields");
  if (b->precision != G4B_FP64) return fail(G4B_ERR_ARG, "g4b_beam_advance: FP64 beam expected");
  if (b->npart == 0 || nfield <= 0) return G4B_OK;
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  PushArgs a{};
  a.gamma = b->gamma;
  a.theta = b->theta;
  a.x = b->x;
  a.y = b->y;
  a.px = b->px;
  a.py = b->py;
  a.chunks = b->d_chunks;
  a.eloss = b->d_eloss;
  a.pez = b->use_pez ? b->d_pez : nullptr;
  a.nfield = nfield;
  double xks_local = 1.0;
  for (int i = 0; i < nfield; ++i) {
    g4b_field* f = fields[i];
    if (!f || f->precision != G4B_FP64 || f->nslice != b->nslice)
      return fail(G4B_ERR_ARG, "g4b_beam_advance: field does not match the beam");
    xks_local = f->xks / (double)f->harm;
    a.f[i].cells = static_cast<const double2*>(f->a);
    a.f[i].first = f->first;
    a.f[i].n = f->ngrid;
    a.f[i].ld = f->ld;
    a.f[i].nslice = f->nslice;
    a.f[i].gridmax = f->gridmax;
    a.f[i].dgrid = f->dgrid;
    a.f[i].rtmp = fc[i] / f->xks;
    a.f[i].rharm = (double)f->harm;
  }
  double xku = st->ku;
  if (xku == 0.0) xku = xks_local * 0.5 / st->gamma_ref / st->gamma_ref;
  a.xks = xks_local;
  a.xku = xku;
  a.aw = st->aw;
  a.autophase = st->autophase;
  a.delz = st->delz;
  a.ax = st->ax;
  a.ay = st->ay;
  a.kx = st->kx;
  a.ky = st->ky;
  a.gradx = st->gradx;
  a.grady = st->grady;
  {
    LaunchScope ls(c, "push");
    G4B_CUDA_TRY(launch_pdl(nfield == 1 ? push_kernel<1> : push_kernel<0>, (unsigned)b->nchunk, 256,
                            0, c->stream, a));
  }
  return check_launch(c, "push_kernel");
}

}  // extern "C"
