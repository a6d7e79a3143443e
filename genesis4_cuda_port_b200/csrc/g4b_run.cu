// g4b_run.cu -- the fused mixed-precision form: a whole FEL run resident on
// the device, advanced by a fixed sequence of kernels per step that a CUDA
// graph replays.
//
// Device state (per particle 28 bytes): x,y and px,py as float2 pairs, the
// energy as an FP32 offset dg = gamma - gamma_ref (keeps the ~0.01 per-step
// energy changes above FP32 resolution), the ponderomotive phase theta in
// FP64.  Fields are complex64.  Per step:
//   K1 beam_step : transverse half step (+chicane), RK4 push with the frozen
//                  bilinear field sample, R56, transverse half step
//                  (+corrector), and each slice's bounding box of touched
//                  cells (integer atomics, order independent);
//   K2 deposit : per slice, the deterministic exact-integer deposition of
//                  every field's source into a compact tile, and the beam
//                  diagnostics (FP64 sums): a branch of the captured graph
//                  beside the deposition in runs that fill the GPU, in the
//                  deposition's CTAs (first) in smaller runs;
//   K3/K4 ADI passes per field (pass Y also zeroes the planes this step's
//                  slippage zeroes and writes field-diagnostic partials);
//   K5 diag_finalize : per-slice beam and field diagnostics into the history
//                  buffer.
// The theta derivative ks(1-1/b) + ku is evaluated cancellation-free in FP64
// as ku - ks*eps/(b(1+b)), eps = btper0/gamma^2 (the two ~ku terms cancel to
// the detuning).  Slippage is the host's integer index model: `first` and the
// zeroed planes of every step are known before the step is enqueued.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <tuple>
#include <vector>

#include "g4b_internal.cuh"

namespace g4b {

constexpr int kRunFields = 8;
constexpr int kStepThreads = 128;  // beam step: two particles per thread
constexpr int kStepBlocks = 8;     // resident beam-step CTAs per SM (<= 64 registers)
constexpr int kStepWarps = kStepThreads / 32;
constexpr int kMaxBunch = 8;
constexpr int kBeamRec = 23;  // reference stats order (DiagnosticCUDA.cpp:102-125)

struct MixField {
  const float2* cells;
  int first, n, ld, nslice, harm, do_source;
  float gridmax, dgrid, inv_dgrid;
  float rtmp;      // fc / xks_h
  int4* bbox;      // [nslice]: ixmin, iymin, ixmax, iymax
};

struct PlaneMapF {
  int mode;
  float strength, offset;
};

struct BeamStepArgs {
  float2 *xy, *pxy;
  float* dg;
  double* th;
  const int4* chunks;
  const double* eloss;
  MixField f[kRunFields];
  int nfield;
  float gref_f, aw, aw2, ax, ay, kx, ky, gradx, grady, half;
  float zt0;          // -2 / xks (FP32)
  double gref, xks, xku, delz, autophase;
  PlaneMapF xm, ym;
  int pre;            // 1 chicane before the first half step
  float m00, m01, m10, m11, m22, m23, m32, m33;
  int post;           // 1 corrector before the second half step
  float cx, cy;
  int has_r56;
  double r56, r56_off;
  int* err;
};

// Reduce an FP64 angle to [-pi, pi) before FP32 trigonometry (the
// hardware sine / cosine, __sincosf, has an absolute error below 2^-21.4 on
// that interval).
__device__ __forceinline__ float reduce_angle(double a) {
  const double twopi = 6.283185307179586476925287;
  return (float)__fma_rn(-twopi, rint(a * (1.0 / twopi)), a);
}

// cell of the deposit / gather in FP32 (the same arithmetic in K1 and K2)
__device__ __forceinline__ bool cell_f(const MixField& f, float x, float y, int& ix, int& iy,
                                       float& wx, float& wy) {
  const float gm = f.gridmax;
  if (!(x > -gm && x < gm && y > -gm && y < gm)) return false;
  // explicit roundings: every kernel computes the same cell and weights
  const float wxr = __fmul_rn(x + gm, f.inv_dgrid), wyr = __fmul_rn(y + gm, f.inv_dgrid);
  const float fx = floorf(wxr), fy = floorf(wyr);  // integers below 2^24: exact
  ix = (int)fx;
  iy = (int)fy;
  if (ix < 0 || ix >= f.n - 1 || iy < 0 || iy >= f.n - 1) return false;
  wx = 1.0f + fx - wxr;
  wy = 1.0f + fy - wyr;
  return true;
}

// ---------------------------------------------------- packed FP32 pairs --
// The beam step advances two particles per thread, one in each lane of a
// packed FP32 pair: sm_100 executes add, subtract, multiply and fused
// multiply-add on f32x2 register pairs as one instruction, so every FP32
// operation of the push serves both particles.  Each lane rounds like the
// scalar IEEE round-to-nearest operation, so a particle's result does not
// depend on its partner.
struct P2 {
  float2 v;
};
__device__ __forceinline__ P2 pr(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ P2 bc(float a) { return {make_float2(a, a)}; }
__device__ __forceinline__ float& ln(P2& p, int l) { return l ? p.v.y : p.v.x; }
__device__ __forceinline__ float ln(const P2& p, int l) { return l ? p.v.y : p.v.x; }
__device__ __forceinline__ P2 operator+(P2 a, P2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ P2 operator*(P2 a, P2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ P2 fma2(P2 a, P2 b, P2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ P2 operator-(P2 a, P2 b) {
  P2 r;
  asm("{\n\t.reg .b64 pa, pb, pc;\n\t"
      "mov.b64 pa, {%2, %3};\n\t"
      "mov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pc, pa, pb;\n\t"
      "mov.b64 {%0, %1}, pc;\n\t}"
      : "=f"(r.v.x), "=f"(r.v.y)
      : "f"(a.v.x), "f"(a.v.y), "f"(b.v.x), "f"(b.v.y));
  return r;
}

// Thick-lens map of one plane over `half` (advance_focusing_plane,
// src/Core/TrackBeamCUDA.cpp:27-59) for strength s with k = s/gz and
// w2 = k half^2: a1 = cos w, a2 = sin(w)/sqrt(k), a3 = -k a2 (cosh/sinh for
// k < 0, drift for k = 0).  For |w2| < 1e-2 (every undulator and quadrupole
// step of practical lattices) the functions are their Taylor series in w2,
// a1 = 1 - w2/2 + w2^2/24 - w2^3/720 and a2/half = 1 - w2/6 + w2^2/120 -
// w2^3/5040 (truncation < w2^4/40320 < 3e-13); larger phases use the closed
// forms.  lens_coef is one lane of plane2, rounding for rounding.
__device__ __forceinline__ void lens_coef(float k, float w2, float half, float& a1, float& a2) {
  if (fabsf(w2) < 1e-2f) {
    a1 = __fmaf_rn(w2, __fmaf_rn(w2, __fmaf_rn(w2, -1.0f / 720.0f, 1.0f / 24.0f), -0.5f), 1.0f);
    a2 = __fmul_rn(half, __fmaf_rn(w2, __fmaf_rn(w2, __fmaf_rn(w2, -1.0f / 5040.0f,
                                                                 1.0f / 120.0f),
                                                 -1.0f / 6.0f),
                                   1.0f));
  } else if (k > 0.f) {
    const float foc = sqrtf(k);
    float sn, cs;
    sincosf(foc * half, &sn, &cs);
    a1 = cs;
    a2 = sn / foc;
  } else {
    const float foc = sqrtf(-k);
    a1 = coshf(foc * half);
    a2 = sinhf(foc * half) / foc;
  }
}

// c' = a1 (c - o) + a2 p / gz + o,  p' = a1 p + a3 gz (c - o) with
// a3 gz = -a2 k gz = -a2 s (o: the element's offset).
__device__ __forceinline__ void plane2(const PlaneMapF m, float half, P2& c, P2& p, P2 inv_gz) {
  if (m.mode == 0) {
    c = fma2(p, bc(half) * inv_gz, c);
    return;
  }
  const P2 k = bc(m.strength) * inv_gz;
  const P2 w2 = k * bc(half * half);
  P2 a1, a2;
  if (fmaxf(fabsf(w2.v.x), fabsf(w2.v.y)) < 1e-2f) {
    a1 = fma2(w2, fma2(w2, fma2(w2, bc(-1.0f / 720.0f), bc(1.0f / 24.0f)), bc(-0.5f)), bc(1.0f));
    a2 = bc(half) *
         fma2(w2, fma2(w2, fma2(w2, bc(-1.0f / 5040.0f), bc(1.0f / 120.0f)), bc(-1.0f / 6.0f)),
              bc(1.0f));
  } else {
    lens_coef(k.v.x, w2.v.x, half, a1.v.x, a2.v.x);
    lens_coef(k.v.y, w2.v.y, half, a1.v.y, a2.v.y);
  }
  const P2 o = bc(m.offset);
  const P2 xt = c - o;
  c = fma2(a1, xt, fma2(a2 * inv_gz, p, o));
  p = fma2(a2 * bc(-m.strength), xt, a1 * p);
}

// sin and cos of a small angle (|a| < 0.1: Taylor series to a^5 and a^4,
// truncation below a^7/5040 < 2e-11 and a^6/720 < 1.4e-9, under the FP32
// rounding of the results); larger angles use sincosf.  sincos_small is one
// lane of sincos_small2, rounding for rounding.
__device__ __forceinline__ void sincos_small(float a, float& s, float& c) {
  if (fabsf(a) < 0.1f) {
    const float a2 = __fmul_rn(a, a);
    s = __fmul_rn(a, __fmaf_rn(a2, __fmaf_rn(a2, 1.0f / 120.0f, -1.0f / 6.0f), 1.0f));
    c = __fmaf_rn(a2, __fmaf_rn(a2, 1.0f / 24.0f, -0.5f), 1.0f);
  } else {
    sincosf(a, &s, &c);
  }
}

__device__ __forceinline__ void sincos_small2(P2 a, P2& s, P2& c) {
  if (fmaxf(fabsf(a.v.x), fabsf(a.v.y)) < 0.1f) {
    const P2 a2 = a * a;
    s = a * fma2(a2, fma2(a2, bc(1.0f / 120.0f), bc(-1.0f / 6.0f)), bc(1.0f));
    c = fma2(a2, fma2(a2, bc(1.0f / 24.0f), bc(-0.5f)), bc(1.0f));
  } else {
    sincos_small(a.v.x, s.v.x, c.v.x);
    sincos_small(a.v.y, s.v.y, c.v.y);
  }
}

// NF: number of fields when known at compile time (1, 2), 0 = up to 8.
// One CTA of kStepThreads threads advances a chunk of up to 2 kStepThreads
// particles of one slice: thread t holds particles t (lane x) and
// t + kStepThreads (lane y) of the chunk; a dead y lane repeats x and is
// not stored.
template <int NF>
__device__ __forceinline__ void beam_chunk(const BeamStepArgs& a, const int4 ch) {
  constexpr int kF = NF > 0 ? NF : kRunFields;
  const int nfield = NF > 0 ? NF : a.nfield;
  __shared__ int sbb[kRunFields][4][kStepWarps];
  const int slice = ch.x;
  const int tid = threadIdx.x;
  const bool live = tid < ch.z, live_y = tid + kStepThreads < ch.z;
  const int64_t ipx = (((int64_t)ch.w) << 31) + (int64_t)(unsigned)ch.y + tid;
  const int64_t ipy = live_y ? ipx + kStepThreads : ipx;
  int bb[kF][4];
#pragma unroll
  for (int f = 0; f < kF; ++f) {
    bb[f][0] = bb[f][1] = 1 << 30;
    bb[f][2] = bb[f][3] = -1;
  }
  if (live) {
    const float2 xy0 = a.xy[ipx], xy1 = a.xy[ipy], pp0 = a.pxy[ipx], pp1 = a.pxy[ipy];
    P2 x = pr(xy0.x, xy1.x), y = pr(xy0.y, xy1.y), px = pr(pp0.x, pp1.x), py = pr(pp0.y, pp1.y);
    P2 d = pr(a.dg[ipx], a.dg[ipy]);
    double t[2] = {a.th[ipx], a.th[ipy]};
    // TrackBeamCUDA::track, first half (src/Core/TrackBeamCUDA.cpp:156-204)
    {
      if (a.pre) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
          float &xl = ln(x, l), &pxl = ln(px, l), &yl = ln(y, l), &pyl = ln(py, l);
          const float g = a.gref_f + ln(d, l);
          const float gz = sqrtf(g * g - 1.0f - pxl * pxl - pyl * pyl);
          float tmp = xl;
          xl = a.m00 * tmp + a.m01 * pxl / gz;
          pxl = a.m10 * tmp * gz + a.m11 * pxl;
          tmp = yl;
          yl = a.m22 * tmp + a.m23 * pyl / gz;
          pyl = a.m32 * tmp * gz + a.m33 * pyl;
        }
      }
      const P2 g = bc(a.gref_f) + d;
      const P2 gz2 = fma2(g, g, bc(-1.0f - a.aw2)) - fma2(px, px, py * py);
      const P2 inv_gz = pr(rsqrtf(gz2.v.x), rsqrtf(gz2.v.y));
      plane2(a.xm, a.half, x, px, inv_gz);
      plane2(a.ym, a.half, y, py, inv_gz);
    }
    // BeamSolverCUDA::advance push (src/Core/BeamSolverCUDA.cpp:226-409)
    t[0] += a.autophase;
    t[1] += a.autophase;
    const P2 dxu = x - bc(a.ax), dyu = y - bc(a.ay);
    const P2 awloc =
        fma2(bc(a.gradx), dxu,
             fma2(bc(a.grady), dyu,
                  fma2(bc(0.5f), fma2(bc(a.kx) * dxu, dxu, bc(a.ky) * dyu * dyu), bc(1.0f))));
    const P2 btpar = fma2(bc(a.aw2), awloc * awloc, fma2(py, py, fma2(px, px, bc(1.0f))));
    const float ez = (float)a.eloss[slice];
    // Field sample of each field rotated to the start phase,
    // w = sc (re - i im) e^{-i h theta0} with sc = rtmp awloc: the field term
    // of a stage at phase offset dth is then w e^{-i h dth}.
    P2 wr[kF], wi[kF];
#pragma unroll
    for (int f = 0; f < kF; ++f) {
      wr[f] = wi[f] = bc(0.f);
      if (f >= nfield) continue;
      const MixField& F = a.f[f];
      int islice = slice + F.first;  // both in [0, nslice)
      if (islice >= F.nslice) islice -= F.nslice;
      const float2* base = F.cells + (size_t)islice * F.n * F.ld;
      P2 cre = bc(0.f), cim = bc(0.f), cs0, sn0;
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        int ix, iy;
        float wx, wy;
        if (cell_f(F, ln(x, l), ln(y, l), ix, iy, wx, wy)) {
          const float2* c = base + (size_t)iy * F.ld + ix;
          const float2 c00 = __ldg(c), c10 = __ldg(c + 1), c01 = __ldg(c + F.ld),
                       c11 = __ldg(c + F.ld + 1);
          const float w00 = wx * wy, w10 = (1.f - wx) * wy, w01 = wx * (1.f - wy),
                      w11 = (1.f - wx) * (1.f - wy);
          ln(cre, l) = c00.x * w00 + c10.x * w10 + c01.x * w01 + c11.x * w11;
          ln(cim, l) = c00.y * w00 + c10.y * w10 + c01.y * w01 + c11.y * w11;
        }
        __sincosf(reduce_angle((double)F.harm * t[l]), &ln(sn0, l), &ln(cs0, l));
      }
      wr[f] = (bc(F.rtmp) * awloc) * (cre * cs0 - cim * sn0);
      wi[f] = (bc(-F.rtmp) * awloc) * fma2(cre, sn0, cim * cs0);
    }
    // theta' = ks (1 - 1/b0) + ku with b0 = sqrt(1 - eps), eps = btper0 /
    // gamma^2 ~ 1e-8: the two ~ku terms cancel to the detuning, so the
    // zero-field, start-of-step value A0 = ku - ks eps0 fe(eps0) (fe =
    // 1/(b(1+b))) is formed once in FP64.  Within the step eps differs from
    // eps0 by the relative amount r = (1 + delta/btpar) (g0/gs)^2 - 1, where
    // delta = -(2/ks) Re(c) is the field term (~1e-10 .. 1e-4 of btpar) and
    // gs the stage energy; then ks eps fe(eps) = B0 (1 + r) (1 + O(eps0 r))
    // with B0 = ks eps0 fe(eps0), so theta' = A0 - B0 r to a relative
    // 1e-8 of the field term, and r is formed in FP32 without cancellation.
    // The energy derivative Im(c) / (b0 gs) - ez drops b0 = 1 + O(1e-8).
    P2 A0, nB0, ig0;
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const double g0 = a.gref + (double)ln(d, l);
      // 1/g0: one Newton step from the FP32 reciprocal (relative error
      // ~2^-44, far below what the FP32 results keep)
      double inv_g0 = (double)__fdividef(1.0f, (float)g0);
      inv_g0 = fma(inv_g0, fma(-g0, inv_g0, 1.0), inv_g0);
      const double eps0 = (double)ln(btpar, l) * inv_g0 * inv_g0;
      const double fe0 = 0.5 + eps0 * (0.375 + eps0 * 0.3125);
      const double B0d = a.xks * eps0 * fe0;
      ln(A0, l) = (float)(a.xku - B0d);
      ln(nB0, l) = -(float)B0d;
      ln(ig0, l) = (float)inv_g0;
    }
    // delta / btpar per unit Re(c)
    const P2 zt = bc(a.zt0) * pr(__fdividef(1.0f, btpar.v.x), __fdividef(1.0f, btpar.v.y));
    const P2 nez = bc(-ez);
    // stage derivatives (energy kg, phase kp) at energy offset ds (from g0)
    // and phase offset dth
    auto ode = [&](P2 ds, P2 dth, P2& kg, P2& kp) {
      P2 ctr = bc(0.f), cti = bc(0.f);
#pragma unroll
      for (int f = 0; f < kF; ++f) {
        if (f >= nfield) break;
        P2 sd, cd;
        sincos_small2(bc((float)a.f[f].harm) * dth, sd, cd);
        if (f == 0) {
          ctr = fma2(wr[0], cd, wi[0] * sd);
          cti = wi[0] * cd - wr[0] * sd;
        } else {
          ctr = fma2(wr[f], cd, fma2(wi[f], sd, ctr));
          cti = fma2(wi[f], cd, cti) - wr[f] * sd;
        }
      }
      const P2 e = ds * ig0;               // (gs - g0) / g0, |e| <~ 1e-3
      const P2 bq = e * (e - bc(1.0f));    // g0 / gs - 1, error O(e^3)
      const P2 ar = zt * ctr;              // delta / btpar
      const P2 r = fma2(bq * (bq + bc(2.0f)), ar + bc(1.0f), ar);
      kp = fma2(nB0, r, A0);
      kg = fma2(cti, fma2(ig0, bq, ig0), nez);
    };
    // Fourth-order Runge-Kutta on the step's energy increment dd and phase
    // increment dt (both small, so FP32 keeps their relative precision; the
    // classical combination that src/Core/BeamSolverCUDA.cpp:258-299 forms
    // in accumulator form); theta and the stored energy offset are updated
    // once at the end
    P2 k1g, k1p;
    {
      // first stage at the start point: no phase rotation, gs = g0
      P2 ctr = wr[0], cti = wi[0];
#pragma unroll
      for (int f = 1; f < kF; ++f) {
        if (f >= nfield) break;
        ctr = ctr + wr[f];
        cti = cti + wi[f];
      }
      k1p = fma2(nB0, zt * ctr, A0);
      k1g = fma2(cti, ig0, nez);
    }
    const P2 hh = bc((float)(0.5 * a.delz)), h = bc((float)a.delz);
    // ug, up: the latest stage's derivatives; sg, sp: k1 + 2 k2 + 2 k3 + k4
    P2 ug, up;
    ode(hh * k1g, hh * k1p, ug, up);
    P2 sg = fma2(bc(2.0f), ug, k1g), sp = fma2(bc(2.0f), up, k1p);
    ode(hh * ug, hh * up, ug, up);
    sg = fma2(bc(2.0f), ug, sg);
    sp = fma2(bc(2.0f), up, sp);
    ode(h * ug, h * up, ug, up);
    const P2 h6 = bc((float)(a.delz / 6.0));
    const P2 dd = h6 * (sg + ug);
    const P2 dt = h6 * (sp + up);
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      t[l] += (double)ln(dt, l);
      ln(d, l) = (float)((double)ln(d, l) + (double)ln(dd, l));
      // applyR56 (src/Core/TrackBeamCUDA.cpp:257-278): theta += R56 (gamma - gamma0)
      if (a.has_r56) t[l] += a.r56 * ((double)ln(d, l) + a.r56_off);
    }
    // second half (+corrector on the last half step)
    {
      if (a.post) {
        px = px + bc(a.cx);
        py = py + bc(a.cy);
      }
      const P2 g = bc(a.gref_f) + d;
      const P2 gz2 = fma2(g, g, bc(-1.0f - a.aw2)) - fma2(px, px, py * py);
      const P2 inv_gz = pr(rsqrtf(gz2.v.x), rsqrtf(gz2.v.y));
      plane2(a.xm, a.half, x, px, inv_gz);
      plane2(a.ym, a.half, y, py, inv_gz);
    }
    a.xy[ipx] = make_float2(x.v.x, y.v.x);
    a.pxy[ipx] = make_float2(px.v.x, py.v.x);
    a.dg[ipx] = d.v.x;
    a.th[ipx] = t[0];
    if (live_y) {
      a.xy[ipy] = make_float2(x.v.y, y.v.y);
      a.pxy[ipy] = make_float2(px.v.y, py.v.y);
      a.dg[ipy] = d.v.y;
      a.th[ipy] = t[1];
    }
#pragma unroll
    for (int f = 0; f < kF; ++f) {
      if (f >= nfield) break;
      if (!a.f[f].do_source) continue;
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        int ix, iy;
        float wx, wy;
        if ((l == 0 || live_y) && cell_f(a.f[f], ln(x, l), ln(y, l), ix, iy, wx, wy)) {
          bb[f][0] = min(bb[f][0], ix);
          bb[f][1] = min(bb[f][1], iy);
          bb[f][2] = max(bb[f][2], ix);
          bb[f][3] = max(bb[f][3], iy);
        }
      }
    }
  }
  // per-CTA bounding boxes -> per-slice (integer min/max: order independent)
  const int w = tid >> 5, l = tid & 31;
#pragma unroll
  for (int f = 0; f < kF; ++f) {
    if (f >= nfield) break;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int v = q < 2 ? __reduce_min_sync(0xffffffffu, bb[f][q])
                          : __reduce_max_sync(0xffffffffu, bb[f][q]);
      if (l == 0) sbb[f][q][w] = v;
    }
  }
  __syncthreads();
  if (tid < 4 * nfield) {
    const int f = tid >> 2, q = tid & 3;
    int v = sbb[f][q][0];
    for (int i = 1; i < kStepWarps; ++i) v = q < 2 ? min(v, sbb[f][q][i]) : max(v, sbb[f][q][i]);
    if (a.f[f].do_source) {
      int* b = reinterpret_cast<int*>(&a.f[f].bbox[slice]) + q;
      if (q < 2) {
        if (v < (1 << 30)) atomicMin(b, v);
      } else if (v >= 0) {
        atomicMax(b, v);
      }
    }
  }
}

template <int NF>
__global__ void __launch_bounds__(kStepThreads, kStepBlocks) beam_step_kernel(const __grid_constant__ BeamStepArgs a) {
  ptx::pdl_wait();
  beam_chunk<NF>(a, a.chunks[blockIdx.x]);
}

// Batched form: items[i] = (run, chunk of that run), per-run arguments.
struct BeamBatchArgs {
  const BeamStepArgs* args;
  const int2* items;
  const int* nitems;
};

template <int NF>
__global__ void __launch_bounds__(kStepThreads, kStepBlocks) beam_batch_kernel(const __grid_constant__ BeamBatchArgs b) {
  const int nitems = *b.nitems;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = b.items[it];
    const BeamStepArgs& a = b.args[w.x];
    beam_chunk<NF>(a, a.chunks[w.y]);
    __syncthreads();
  }
}

// ------------------------------------------------------ deposit + beam diag --
struct DepField {
  float2* src;        // compact tiles, cap cells per slice
  int4* desc;
  int4* bbox;
  int* mpred;         // [nslice][kDepSplit] M of the slice's previous deposition (0: none)
  size_t cap;
  int first, n, ld, nslice, harm, do_source;
  float gridmax, dgrid, inv_dgrid;
  double fc, xks, dgrid_d;
};

struct DepArgs {
  const float2* xy;
  const float* dg;
  const double* th;
  const int64_t* off;
  const double* current;
  float* qpred;       // [nslice][kDepSplit] largest charge weight of the previous deposition (0: none)
  DepField f[kRunFields];
  int nfield;
  float ax, ay, kx, ky, gradx, grady, gref_f;
  double delz;
  int* err;
};

struct BeamDiagArgs {
  const float2 *xy, *pxy;
  const float* dg;
  const double* th;
  const int64_t* off;
  int nbunch, need_aux;
  double gref;
  double* beam_part;  // [nslice * kDepParts][23 + 2*nbunch] records
};

// Beam diagnostics (DiagnosticCUDA.cpp:102-125), kDepParts CTAs per slice,
// each over an equal share of the slice's particles: one pass with FP64
// sums (the minima and maxima in FP32, exact for FP32 state) into a record
// of the final layout; the finalize combines a slice's records in a fixed
// order (sums, minima and maxima of records are the record of the union).
// Independent of the deposition, so it runs beside it and the ADI passes.
constexpr int kDepParts = 1;          // beam-diagnostic records per slice
constexpr int kDiagThreads = 256;
constexpr int kDepDiagU = 8;          // particles in flight per thread

// U: particles in flight per thread (each thread adds its particles in the
// same order for every U, so the sums do not depend on it)
template <int NB, int U = kDepDiagU>
__device__ __forceinline__ void diag_slice(const BeamDiagArgs& a, const int bs, const int part) {
  __shared__ double dpart[kDiagThreads / 32][kBeamRec + 2 * kMaxBunch];
  __shared__ double bcomp[kDiagThreads / 32][2 * kMaxBunch];  // bunching compensations
  const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
  const int nall = (int)(a.off[bs + 1] - a.off[bs]);  // at most kRunMaxNp per slice
  const int per = (nall + kDepParts - 1) / kDepParts;
  const int first = min(part * per, nall);
  const int64_t p0 = a.off[bs] + first;
  const int np = min(per, nall - first);
  const float2* xyp = a.xy + p0;
  const float2* pxyp = a.pxy + p0;
  const float* dgp = a.dg + p0;
  const double* thp = a.th + p0;
  const int rec = kBeamRec + 2 * a.nbunch;
  double sm[12];  // sums of x, x^2, y, y^2, px, px^2, py, py^2, x px, y py, dg, dg^2
#pragma unroll
  for (int k = 0; k < 12; ++k) sm[k] = 0.0;
  // minima / maxima of x, px, y, py (reference start values -+1e5) and dg
  float mn[5] = {1.0e5f, 1.0e5f, 1.0e5f, 1.0e5f, INFINITY};
  float mx[5] = {-1.0e5f, -1.0e5f, -1.0e5f, -1.0e5f, -INFINITY};
  // bunching sums: each thread adds its FP32 terms (at most 256: 65536
  // particles over 256 threads) in FP64, within 2^-45 of their magnitude;
  // the warp and the CTA's warps add with compensation (csum_*)
  double bre[NB], bim[NB];
#pragma unroll
  for (int h = 0; h < NB; ++h) bre[h] = bim[h] = 0.0;
  // in a wider CTA only the first kDiagThreads threads sum (the same layout)
  for (int pb = tid < kDiagThreads ? tid : np; pb < np; pb += U * kDiagThreads) {
    float2 lxy[U], lpp[U];
    float ldg[U];
    double lth[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int p = pb + u * kDiagThreads;
      if (p < np) {
        lxy[u] = xyp[p];
        lpp[u] = pxyp[p];
        ldg[u] = dgp[p];
        lth[u] = thp[p];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (pb + u * kDiagThreads >= np) break;
      const double x = lxy[u].x, y = lxy[u].y, px = lpp[u].x, py = lpp[u].y;
      const double d = ldg[u];
      sm[0] += x; sm[1] = __fma_rn(x, x, sm[1]);
      sm[2] += y; sm[3] = __fma_rn(y, y, sm[3]);
      sm[4] += px; sm[5] = __fma_rn(px, px, sm[5]);
      sm[6] += py; sm[7] = __fma_rn(py, py, sm[7]);
      sm[8] = __fma_rn(x, px, sm[8]); sm[9] = __fma_rn(y, py, sm[9]);
      sm[10] += d; sm[11] = __fma_rn(d, d, sm[11]);
      if (a.need_aux) {
        const float f[5] = {lxy[u].x, lpp[u].x, lxy[u].y, lpp[u].y, ldg[u]};
#pragma unroll
        for (int i = 0; i < 5; ++i) {
          mn[i] = fminf(mn[i], f[i]);
          mx[i] = fmaxf(mx[i], f[i]);
        }
      }
      float s1, c1;
      __sincosf(reduce_angle(lth[u]), &s1, &c1);
      float ch = c1, sh = s1;
#pragma unroll
      for (int h = 0; h < NB; ++h) {
        if (h >= a.nbunch) break;
        bre[h] += ch;
        bim[h] += sh;
        const float nc = __fmaf_rn(ch, c1, -__fmul_rn(sh, s1));
        const float ns = __fmaf_rn(sh, c1, __fmul_rn(ch, s1));
        ch = nc;
        sh = ns;
      }
    }
  }
  // per-warp records in the layout of the final one: [0] sum dg,
  // [1] sum dg^2, [2..11] the sums of x .. y py, [13..22] minima / maxima
  // of x, px, y, py, dg
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    double t = sm[k];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (l == 0 && w < kDiagThreads / 32) dpart[w][k < 10 ? k + 2 : k - 10] = t;
  }
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    float lo = mn[i], hi = mx[i];
    for (int o = 16; o > 0; o >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (l == 0 && w < kDiagThreads / 32) {
      dpart[w][13 + 2 * i] = lo;
      dpart[w][14 + 2 * i] = hi;
    }
  }
#pragma unroll
  for (int h = 0; h < NB; ++h) {
    if (h >= a.nbunch) break;
    double tr = bre[h], trc = 0.0, ti = bim[h], tic = 0.0;
    ptx::csum_warp(tr, trc, 32);
    ptx::csum_warp(ti, tic, 32);
    if (l == 0 && w < kDiagThreads / 32) {
      dpart[w][kBeamRec + 2 * h] = tr;
      dpart[w][kBeamRec + 2 * h + 1] = ti;
      bcomp[w][2 * h] = trc;
      bcomp[w][2 * h + 1] = tic;
    }
  }
  __syncthreads();
  if (tid < rec) {
    // record (DiagnosticCUDA.cpp:102-125): [0] sum gamma, [1] sum gamma^2,
    // [12] count, [21] / [22] min / max gamma from the dg extremes (gamma
    // = gref + dg is monotonic in dg)
    const double N = (double)np;
    const int op = tid < 13 ? 0 : (tid < kBeamRec ? ((tid - 13) % 2 == 0 ? 1 : 2) : 0);
    double t = N;
    if (tid >= kBeamRec) {  // bunching: the warps' compensated partials
      const int q = tid - kBeamRec;
      double tc = bcomp[0][q];
      t = dpart[0][tid];
      for (int i = 1; i < kDiagThreads / 32; ++i) ptx::csum_merge(t, tc, dpart[i][tid], bcomp[i][q]);
      t += tc;
    } else if (tid != 12) {
      t = dpart[0][tid];
      for (int i = 1; i < kDiagThreads / 32; ++i) {
        const double u = dpart[i][tid];
        t = op == 0 ? t + u : (op == 1 ? fmin(t, u) : fmax(t, u));
      }
    }
    if (tid == 0) t = __fma_rn(N, a.gref, t);
    if (tid == 1) {
      double sd = dpart[0][0];
      for (int i = 1; i < kDiagThreads / 32; ++i) sd += dpart[i][0];
      t = __fma_rn(__dmul_rn(N, a.gref), a.gref, __fma_rn(__dmul_rn(2.0, a.gref), sd, t));
    }
    if (tid == 21) t = fmin(1.0e7, a.gref + t);
    if (tid == 22) t = fmax(1.0, a.gref + t);
    if (tid >= 13 && tid < kBeamRec && !a.need_aux) t = 0.0;
    a.beam_part[((size_t)bs * kDepParts + part) * rec + tid] = t;
  }
}

template <int NB>
__global__ void __launch_bounds__(kDiagThreads, 2)
    beam_diag_kernel(const __grid_constant__ BeamDiagArgs a) {
  diag_slice<NB>(a, blockIdx.x / kDepParts, blockIdx.x % kDepParts);
}

// Deposition (adi_deposit_source_atomic, FieldSolverADICUDA.cpp:98-174),
// one CTA per slice: a deterministic per-cell reduction in exact integer
// arithmetic.  With M the largest number of contributions any output cell
// receives (the sum of the particle counts of its four base cells) and
// qmax the largest charge weight sqrt(faw2) / gamma, the scale
// S = 2^30 / (M' q') for any M' >= M, q' >= qmax rounds every contribution
// c = rint(S q w (sin h theta, cos h theta)) to an int32 with
// |c| <= 2^30 / M', so no cell sum of 32-bit shared-memory integer atomics
// can overflow (re and im in separate planes, so the 32 lanes of a warp
// spread over the banks).  M' and q' come from the slice's previous
// deposition (M + M/4 + 4 and qmax (1 + 2^-6)): one pass counts the
// particles per base cell, takes qmax and adds the contributions at that
// scale, and the band is redone at the exact scale S = 2^30 / (M qmax) in
// the rare case that the counted M or qmax exceeds its bound.  The first
// deposition after a beam upload counts first.
// Integer addition is associative, so the source does not depend on the
// order in which threads add, and each contribution keeps FP32 resolution
// (2^-24 relative, times at most 1.25 M qmax / (M' q')).  Phases are reduced
// to [-pi, pi) in FP64 and their sine and cosine taken with the hardware
// approximation (absolute error below 2^-21.4 on that interval).  Every
// rounding that could be fused differently is written out with intrinsics,
// so the single-run and the batched kernels give the same bits.  The tile is
// the slice's bounding box of touched cells (from K1); tiles larger than
// kDepMaxCells are processed in row bands.
constexpr int kDepThreads = 256;
// CTAs per slice: CTA `part` takes the tile's row bands part, part +
// kDepSplit, ... (a tile of one band leaves the second CTA idle; one of two
// bands is done by two CTAs side by side instead of one after the other)
constexpr int kDepSplit = 2;
constexpr int kDepAccU = 4;           // particles in flight per thread
constexpr int kDepWideThreads = 512;  // the deposition CTA of runs of few slices
constexpr int kDepMaxCells = 8192;    // output cells per band (a multiple of 4)
constexpr int kDepMaxWidth = 896;     // tile width bound: mixed ngrid <= 880
// re and im planes, then the counts per base cell ((hb + 1) bw <= cells + width)
constexpr size_t kDepSmem = (size_t)(3 * kDepMaxCells + kDepMaxWidth) * 4;

// Charge weight sqrt(faw2) / gamma of one particle (FP32).
__device__ __forceinline__ float dep_charge(const DepArgs& a, const float2 xy, const float dg) {
  const float dxu = xy.x - a.ax, dyu = xy.y - a.ay;
  // 1 + kx dx^2 + ky dy^2 + 2 (gradx dx + grady dy), every rounding explicit
  const float lin = __fmaf_rn(a.grady, dyu, __fmul_rn(a.gradx, dxu));
  const float faw2 = __fmaf_rn(__fmul_rn(a.kx, dxu), dxu,
                               __fmaf_rn(__fmul_rn(a.ky, dyu), dyu, __fmaf_rn(2.0f, lin, 1.0f)));
  return __fdividef(sqrtf(faw2), a.gref_f + dg);
}

// T threads per CTA, U particles in flight per thread: the integer sums and
// the maxima do not depend on either, so every instance gives the same bits.
template <int T = kDepThreads, int U = kDepAccU>
__device__ __forceinline__ void deposit_slice(const DepArgs& a, const int bs, const int part,
                                              unsigned char* smem) {
  __shared__ int4 sbox[kRunFields];
  __shared__ int wsum[T / 32];
  __shared__ float wmax[T / 32];
  const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
  const int64_t p0 = a.off[bs];
  const int np = (int)(a.off[bs + 1] - p0);  // at most kRunMaxNp per slice
  const float2* xyp = a.xy + p0;
  const float* dgp = a.dg + p0;
  const double* thp = a.th + p0;
  if (tid < a.nfield) sbox[tid] = a.f[tid].bbox[bs];
  const float qprev = a.qpred[bs * kDepSplit + part];
  const float q_use = qprev * 1.015625f;  // 0 without a previous deposition
  float q_seen = 0.f;
  bool deposited = false;
  __syncthreads();  // sbox is read by every thread below

  // ---- deposition of every field with a source this step ----
  int* are = reinterpret_cast<int*>(smem);        // [hb * bw] real parts
  int* aim = are + kDepMaxCells;                  // [hb * bw] imaginary parts
  int* hist = aim + kDepMaxCells;                 // [(hb + 1) * bw] counts per base cell
  const double npd = (double)np;
  for (int fi = 0; fi < a.nfield; ++fi) {
    const DepField& F = a.f[fi];
    if (!F.do_source) continue;
    const int target = (bs + F.first) % F.nslice;
    const int4 bb = sbox[fi];
    // adi_compute_slice_scl (src/Core/FieldSolverADICUDA.cpp:75-96)
    double scl = 0.0;
    if (npd > 0) {
      scl = F.fc * 376.73031346177 * a.current[bs] * F.xks * a.delz;
      scl /= 4.0 * 510998.95 * npd * F.dgrid_d * F.dgrid_d;
    }
    if (bb.z < 0 || scl == 0.0) {
      if (tid == 0 && part == 0) F.desc[target] = make_int4(0, 0, 0, 0);
      continue;
    }
    int bx0 = bb.x, bw = bb.z - bb.x + 2;
    const int by0 = bb.y, bh = bb.w - bb.y + 2;
    if (bw & 1) {  // even tile width keeps the rows 16-byte aligned
      ++bw;
      if (bx0 + bw > F.ld) --bx0;
    }
    if (bw > kDepMaxWidth) {  // excluded by g4b_run_create's ngrid limit
      if (tid == 0 && part == 0) {
        atomicOr(a.err, kErrBadSlice);
        F.desc[target] = make_int4(0, 0, 0, 0);
      }
      continue;
    }
    if (tid == 0 && part == 0) F.desc[target] = make_int4(bx0, by0, bw, bh);
    const int hband = max(1, kDepMaxCells / bw);  // bw <= ngrid + 1 < kDepMaxCells
    const float fh = (float)F.harm;
    // row of output cell o: (o + 1/2) / bw in FP32 is never within
    // nout 2^-23 / bw of an integer boundary, so the truncation is exact
    const float inv_bw = 1.0f / (float)bw;
    MixField mf;
    mf.gridmax = F.gridmax;
    mf.dgrid = F.dgrid;
    mf.inv_dgrid = F.inv_dgrid;
    mf.n = F.n;
    // M of this slice's previous deposition of this field (0: none yet)
    // bounds the contributions of the single-pass form below
    const int mprev = F.mpred[bs * kDepSplit + part];
    const int m_use = mprev > 0 ? mprev + (mprev >> 2) + 4 : 0;
    int m_seen = 0;
    for (int yb = part * hband; yb < bh; yb += kDepSplit * hband) {
      const int hb = min(hband, bh - yb);
      const int ylo = by0 + yb;  // first grid row of this band
      const int nout = hb * bw, nbase = (hb + 1) * bw;
      // with `count` the counts per base cell (ext row iy - ylo + 1) and the
      // largest charge weight (qloc), with `add` the contributions at scale
      // Sf of charge weights capped at qc.  A thread takes groups of four
      // consecutive particles: a quiet-start beamlet (nbins = 4 particles at
      // one transverse position) when the four share a base cell, whose
      // rounded contributions it sums in registers and adds, with its count,
      // by one set of atomics instead of four (the same integer sums).
      float qloc = 0.f;
      auto add8 = [&](int cid, const int* v) {
        if (cid >= bw) {  // lower corners: output row ey = cid / bw - 1
          const int o = cid - bw;
          atomicAdd(&are[o], v[0]);
          atomicAdd(&aim[o], v[1]);
          atomicAdd(&are[o + 1], v[2]);
          atomicAdd(&aim[o + 1], v[3]);
        }
        if (cid < nout) {  // upper corners: row ey + 1 inside the band
          atomicAdd(&are[cid], v[4]);
          atomicAdd(&aim[cid], v[5]);
          atomicAdd(&are[cid + 1], v[6]);
          atomicAdd(&aim[cid + 1], v[7]);
        }
      };
      auto pass = [&](const bool count, const bool add, const float Sf, const float qc) {
        for (int g = tid; 4 * g < np; g += T) {
          const int pg = 4 * g;
          float2 lxy[4];
          float ldg[4];
          double lth[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (pg + u < np) {
              lxy[u] = xyp[pg + u];
              ldg[u] = dgp[pg + u];
              if (add) lth[u] = thp[pg + u];
            }
          }
          int cid[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            cid[u] = -1;
            int ix, iy;
            float wx, wy;
            if (pg + u < np && cell_f(mf, lxy[u].x, lxy[u].y, ix, iy, wx, wy) &&
                iy + 1 >= ylo && iy < ylo + hb) {
              const int ex = ix - bx0;
              if (ex < 0 || ex > bw - 2) {
                if (count) atomicOr(a.err, kErrBadSlice);
              } else {
                cid[u] = (iy - ylo + 1) * bw + ex;
              }
            }
          }
          const bool same = cid[0] >= 0 && cid[1] == cid[0] && cid[2] == cid[0] &&
                            cid[3] == cid[0];
          if (count) {
            if (same) {
              atomicAdd(&hist[cid[0]], 4);
            } else {
#pragma unroll
              for (int u = 0; u < 4; ++u)
                if (cid[u] >= 0) atomicAdd(&hist[cid[u]], 1);
            }
          }
          int sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (cid[u] < 0) continue;
            const float qraw = dep_charge(a, lxy[u], ldg[u]);
            if (count) qloc = fmaxf(qloc, qraw);
            if (!add) continue;
            const float q = fminf(qraw, qc) * Sf;
            float sn, cs;
            __sincosf(reduce_angle((double)fh * lth[u]), &sn, &cs);
            const float vre = sn * q, vim = cs * q;
            int ix, iy;
            float x0, y0;
            cell_f(mf, lxy[u].x, lxy[u].y, ix, iy, x0, y0);  // the weights again
            const float w00 = x0 * y0, w10 = (1.f - x0) * y0, w01 = x0 * (1.f - y0),
                        w11 = (1.f - x0) * (1.f - y0);
            const int c[8] = {__float2int_rn(vre * w00), __float2int_rn(vim * w00),
                              __float2int_rn(vre * w10), __float2int_rn(vim * w10),
                              __float2int_rn(vre * w01), __float2int_rn(vim * w01),
                              __float2int_rn(vre * w11), __float2int_rn(vim * w11)};
            if (same) {
#pragma unroll
              for (int k = 0; k < 8; ++k) sum[k] += c[k];
            } else {
              add8(cid[u], c);
            }
          }
          if (add && same) add8(cid[0], sum);
        }
      };
      auto zero_acc = [&]() {
        int4* r4 = reinterpret_cast<int4*>(are);
        int4* i4 = reinterpret_cast<int4*>(aim);
        for (int i = tid; i < (nout + 3) >> 2; i += T) {
          r4[i] = make_int4(0, 0, 0, 0);
          i4[i] = make_int4(0, 0, 0, 0);
        }
      };
      __syncthreads();
      {
        int4* h4 = reinterpret_cast<int4*>(hist);
        for (int i = tid; i < (nbase + 3) >> 2; i += T) h4[i] = make_int4(0, 0, 0, 0);
      }
      const bool single = m_use > 0 && q_use > 0.f && q_use < 3.0e38f;
      double S = 0.0;
      if (single) {
        // one pass: counts, qmax and contributions at the scale of the
        // predicted bounds; kept if neither counted bound exceeds its
        // prediction (then no cell sum can have overflowed and no charge was
        // capped), else redone below at the exact scale
        S = 1073741824.0 / ((double)m_use * (double)q_use);  // 2^30 / (M' q')
        zero_acc();
        __syncthreads();
        pass(true, true, (float)S, q_use);
      } else {
        __syncthreads();
        pass(true, false, 0.f, 0.f);
      }
      __syncthreads();
      // the largest number M of contributions any output cell receives
      int mloc = 0;
      for (int o = tid; o < nout; o += T) {
        const int r = (int)(((float)o + 0.5f) * inv_bw), x = o - r * bw;
        int m = hist[(r + 1) * bw + x] + hist[r * bw + x];
        if (x > 0) m += hist[(r + 1) * bw + x - 1] + hist[r * bw + x - 1];
        mloc = max(mloc, m);
      }
      for (int o = 16; o > 0; o >>= 1) {
        mloc = max(mloc, __shfl_xor_sync(0xffffffffu, mloc, o));
        qloc = fmaxf(qloc, __shfl_xor_sync(0xffffffffu, qloc, o));
      }
      if (l == 0) {
        wsum[w] = mloc;
        wmax[w] = qloc;
      }
      __syncthreads();
      int M = wsum[0];
      float qm = wmax[0];
      for (int i = 1; i < T / 32; ++i) {
        M = max(M, wsum[i]);
        qm = fmaxf(qm, wmax[i]);
      }
      m_seen = max(m_seen, M);
      float2* out = F.src + (size_t)target * F.cap + (size_t)yb * bw;
      if (M == 0 || !(qm > 0.f) || !(qm < 3.0e38f)) {
        if (M > 0) atomicOr(a.err, kErrFixedRange);  // non-finite charge
        for (int i = tid; i < nout; i += T) out[i] = make_float2(0.f, 0.f);
        continue;
      }
      q_seen = fmaxf(q_seen, qm);
      deposited = true;
      if (!single || M > m_use || qm > q_use) {
        S = 1073741824.0 / ((double)M * (double)qm);  // 2^30 / (M qmax)
        zero_acc();
        __syncthreads();
        pass(false, true, (float)S, qm);
      }
      __syncthreads();
      const double unscale = scl / S;
      for (int i = tid; i < nout; i += T)
        out[i] = make_float2((float)((double)are[i] * unscale), (float)((double)aim[i] * unscale));
    }
    if (tid == 0 && part * hband < bh) F.mpred[bs * kDepSplit + part] = m_seen;
  }
  if (tid == 0 && deposited) a.qpred[bs * kDepSplit + part] = q_seen;
}

__global__ void __launch_bounds__(kDepThreads, 2) deposit_kernel(const __grid_constant__ DepArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  ptx::pdl_wait();
  deposit_slice(a, blockIdx.x / kDepSplit, blockIdx.x % kDepSplit, smem);
}

// The beam diagnostics and the deposition of a slice by one CTA, one after
// the other: the form of runs too small to fill the GPU (a graph branch for
// their diagnostics would cost more to instantiate than it saves).  Runs of
// fewer slices than SMs take T = 512 threads, twice the particles in flight
// of a 256-thread CTA for the deposition; the diagnostics use the first
// kDiagThreads threads, so every form gives the same bits.
struct DepDiagLaunch {
  DepArgs d;
  BeamDiagArgs b;
};

template <int NB, int T>
__global__ void __launch_bounds__(T, 512 / T)
    deposit_diag_kernel(const __grid_constant__ DepDiagLaunch a) {
  extern __shared__ __align__(128) unsigned char smem[];
  ptx::pdl_wait();
  const int bs = blockIdx.x / kDepSplit, part = blockIdx.x % kDepSplit;
  // the last part takes the diagnostics: a tile of one band leaves it no
  // deposition, so the slice's diagnostics and deposition run side by side
  if (part == kDepSplit - 1) {
    diag_slice<NB>(a.b, bs, 0);
    __syncthreads();
  }
  deposit_slice<T, kDepAccU>(a.d, bs, part, smem);
}

// Batched forms: items[i] = (run, slice of that run).
struct DepBatchArgs {
  const DepArgs* args;
  const int2* items;
  const int* nitems;
};

__global__ void __launch_bounds__(kDepThreads, 2)
    deposit_batch_kernel(const __grid_constant__ DepBatchArgs b) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int nitems = *b.nitems * kDepSplit;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = b.items[it / kDepSplit];
    deposit_slice(b.args[w.x], w.y, it % kDepSplit, smem);
    __syncthreads();
  }
}

struct DiagBatchArgs {
  const BeamDiagArgs* args;
  const int2* items;
  const int* nitems;
};

template <int NB>
__global__ void __launch_bounds__(kDiagThreads, 2)
    beam_diag_batch_kernel(const __grid_constant__ DiagBatchArgs b) {
  const int nitems = *b.nitems * kDepParts;  // (run, slice) items, kDepParts parts each
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = b.items[it / kDepParts];
    diag_slice<NB>(b.args[w.x], w.y, it % kDepParts);
    __syncthreads();
  }
}

// ---------------------------------------------------------- diag finalize --
// Field diagnostics per beam slice is = (nslice + storage - first) % nslice
// (src/Core/DiagnosticCUDA.cpp:320) from the pass-Y band partials.
struct FinalizeArgs {
  const double* part[kRunFields];  // [nslice][nband][9]
  int4* bbox[kRunFields];
  int nband[kRunFields];
  int first_after[kRunFields];
  int nfield, nslice, rec;
  const double* beam_part;  // [nslice * kDepParts][rec]
  double* beam_hist;        // [nslice][rec] for this step
  double* field_hist;       // [nfield][nslice][9] for this step
};

// Per-slice reductions in fixed order: field diagnostics per beam slice
// is = (nslice + storage - first) % nslice (src/Core/DiagnosticCUDA.cpp:320)
// from the pass-Y band partials (one thread per slice and quantity, adding
// the bands in order), the beam diagnostics from the deposition CTAs'
// records; also resets the deposition boxes for the next step.
__device__ __forceinline__ void finalize_range(const FinalizeArgs& a, int i0, int stride) {
  const int nf = a.nfield * a.nslice;
  const int nb = a.nslice * a.rec;
  for (int i = i0; i < 9 * nf + nb + nf; i += stride) {
    if (i < 9 * nf) {
      const int j = i / 9, q = i - 9 * j;
      const int f = j / a.nslice, s = j - f * a.nslice;
      const double* p = a.part[f] + (size_t)s * a.nband[f] * 9 + q;
      const int nbf = a.nband[f];
      double v = 0.0, vc = 0.0;  // compensated sum of the bands, in band order
      for (int b0 = 0; b0 < nbf; b0 += 32) {  // up to 32 loads in flight
        const int m = min(32, nbf - b0);
        double t[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) t[k] = k < m ? p[(b0 + k) * 9] : 0.0;
#pragma unroll
        for (int k = 0; k < 32; ++k)
          if (k < m) ptx::csum_add(v, vc, t[k]);
      }
      v += vc;
      const int is = (a.nslice + s - a.first_after[f]) % a.nslice;
      a.field_hist[((size_t)f * a.nslice + is) * 9 + q] = v;
    } else if (i < 9 * nf + nb) {
      const int j = i - 9 * nf;
      const int s = j / a.rec, k = j - s * a.rec;
      const int op = k < 13 ? 0 : (k < kBeamRec ? ((k - 13) % 2 == 0 ? 1 : 2) : 0);
      const double* p = a.beam_part + (size_t)s * kDepParts * a.rec + k;
      double t = p[0];
      for (int b = 1; b < kDepParts; ++b) {
        const double u = p[(size_t)b * a.rec];
        t = op == 0 ? t + u : (op == 1 ? fmin(t, u) : fmax(t, u));
      }
      a.beam_hist[(size_t)s * a.rec + k] = t;
    } else {
      const int j = i - 9 * nf - nb;
      const int f = j / a.nslice, s = j - f * a.nslice;
      a.bbox[f][s] = make_int4(1 << 30, 1 << 30, -1, -1);
    }
  }
}

__global__ void diag_finalize_kernel(const __grid_constant__ FinalizeArgs a) {
  ptx::pdl_wait();
  finalize_range(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// Batched form: one CTA per run at a time.
__global__ void finalize_batch_kernel(const FinalizeArgs* args, const int* nruns) {
  const int n = *nruns;
  for (int r = blockIdx.x; r < n; r += gridDim.x) finalize_range(args[r], threadIdx.x, blockDim.x);
}

// Particle conversions between FP64 host arrays (x, y, px, py, gamma, each
// `stride` apart in the staging buffer) and the mixed form's state.
__global__ void beam_f64_to_mixed(const double* stage, size_t stride, size_t m, float gf,
                                  float2* xy, float2* pxy, float* dg) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m;
       i += (size_t)gridDim.x * blockDim.x) {
    xy[i] = make_float2((float)stage[i], (float)stage[stride + i]);
    pxy[i] = make_float2((float)stage[2 * stride + i], (float)stage[3 * stride + i]);
    dg[i] = (float)(stage[4 * stride + i] - (double)gf);
  }
}

__global__ void beam_mixed_to_f64(const float2* xy, const float2* pxy, const float* dg,
                                  double gf, size_t m, double* stage, size_t stride) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m;
       i += (size_t)gridDim.x * blockDim.x) {
    const float2 a = xy[i], b = pxy[i];
    stage[i] = a.x;
    stage[stride + i] = a.y;
    stage[2 * stride + i] = b.x;
    stage[3 * stride + i] = b.y;
    stage[4 * stride + i] = gf + (double)dg[i];
  }
}

static PlaneMapF plane_map_f(double strength, double offset) {
  PlaneMapF m{0, (float)strength, 0.f};
  if (strength == 0.0) return m;
  m.offset = (float)(offset / strength);
  m.mode = strength > 0.0 ? 1 : 2;
  return m;
}

}  // namespace g4b

using namespace g4b;

struct StepPlan {
  g4b_step st;
  double fc[kRunFields];
  int first_before[kRunFields], first_after[kRunFields];
  int zero_start[kRunFields], zero_count[kRunFields];
  int adi_index[kRunFields];
};

struct RunFieldState {
  g4b_field* f = nullptr;
  std::vector<g4b_adi*> adis;   // one factorisation per distinct delz
  std::vector<double> adi_delz;
  int harm = 1;
  int4* d_bbox = nullptr;
  int* d_mpred = nullptr;       // [nslice] deposition contribution bound per slice
  double* d_part = nullptr;
  int nband = 0;
  double accuslip = 0.0;        // host slippage model
  int first = 0;
};

struct g4b_run {
  g4b_ctx* ctx = nullptr;
  g4b_run_desc desc{};
  int nslice = 0, nfield = 0;
  int64_t npart = 0, max_np = 0;
  int64_t* d_off = nullptr;
  int4* d_chunks = nullptr;
  int nchunk = 0;
  float2 *xy = nullptr, *pxy = nullptr;
  float* dg = nullptr;
  double* th = nullptr;
  double *d_current = nullptr, *d_eloss = nullptr;
  std::vector<double> h_current;
  RunFieldState fs[kRunFields];
  // lattice
  std::vector<g4b_step> steps;
  std::vector<double> fc;   // [nstep][nfield]
  std::vector<double> slip;
  // history of diagnostics: per step beam [nslice][rec] then fields
  double* d_hist = nullptr;
  double* d_beam_part = nullptr;   // beam-diagnostic records per slice
  float* d_qpred = nullptr;        // [nslice] largest charge weight of the last deposition
  // second stream and fork / join events of a captured step (diagnostics branch)
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool capturing = false;
  int hist_steps = 0;
  size_t rec_beam = 0, step_doubles = 0;
  // cached graph
  cudaGraphExec_t gexec = nullptr;
  int g_first = -1, g_n = 0;
  std::vector<int> g_state;
  uint64_t bytes = 0;
};

// Chicane transfer matrix shared with the drop-in tracking (row-major 4x4).
void g4b_chicane_matrix(double angle, double lb, double ld, double lt, double* m);

namespace {

constexpr int kRunChunk = 2 * kStepThreads;  // particles per beam-step CTA
constexpr int kRunMaxNp = 65536;              // particles per slice (deposition scale)

// Every argument of one lattice step of one run.
struct StepArgs {
  bool has_beam;
  BeamStepArgs bs;
  DepArgs dd;
  BeamDiagArgs bd;
  AdiPlan adi[kRunFields];
  FinalizeArgs fa;
  int nfin;
};

int plan_step(g4b_run* r, int i, StepPlan& p) {
  p.st = r->steps[i];
  for (int f = 0; f < r->nfield; ++f) {
    RunFieldState& F = r->fs[f];
    p.fc[f] = r->fc[(size_t)i * r->nfield + f];
    p.first_before[f] = F.first;
    // slippage model of ControlCUDA::applySlippage (src/Core/ControlCUDA.cpp:148-252)
    int zs = 0, zc = 0;
    if (r->desc.time_run) {
      F.accuslip += r->slip[i];
      const int ns = r->nslice;
      int direction = 1;
      while (std::fabs(F.accuslip) > r->desc.sample * 0.8) {
        direction = F.accuslip < 0 ? -1 : 1;
        F.accuslip -= r->desc.sample * direction;
        int last = (F.first + ns - 1) % ns;
        if (direction < 0) last = (last + 1) % ns;
        if (!r->desc.periodic) {
          if (zc == 0) {
            zs = last;
            zc = 1;
          } else if (direction > 0 && (last + 1) % ns == zs) {
            zs = last;
            ++zc;
          } else if (direction < 0 && (zs + zc) % ns == last) {
            ++zc;
          } else {
            return fail(G4B_ERR_RANGE, "g4b_run: slippage changes direction within one step");
          }
        }
        F.first = last;
        if (direction < 0) F.first = (last + 1) % ns;
      }
    }
    p.zero_start[f] = zs;
    p.zero_count[f] = std::min(zc, r->nslice);
    p.first_after[f] = F.first;
    int k = -1;
    for (size_t j = 0; j < F.adi_delz.size(); ++j)
      if (F.adi_delz[j] == p.st.delz) k = (int)j;
    if (k < 0) return fail(G4B_ERR_STATE, "g4b_run: step length without a factorisation");
    p.adi_index[f] = k;
  }
  return G4B_OK;
}

// Resolves every kernel argument of lattice step i (plan p) without
// launching anything; the single-run path and the batch engine launch them.
int build_step(g4b_run* r, int i, const StepPlan& p, StepArgs& L) {
  g4b_ctx* c = r->ctx;
  L = StepArgs{};
  const g4b_step& st = p.st;
  const double gref = r->desc.gamma_ref;
  // particles store dg = gamma - (float)gamma_ref; every kernel rebuilds gamma
  // from that same FP32-rounded reference
  const double gbase = (double)(float)gref;
  // K1
  if (r->npart > 0) {
    BeamStepArgs a{};
    a.xy = r->xy;
    a.pxy = r->pxy;
    a.dg = r->dg;
    a.th = r->th;
    a.chunks = r->d_chunks;
    a.eloss = r->d_eloss;
    a.nfield = r->nfield;
    double xks_local = 1.0;
    for (int f = 0; f < r->nfield; ++f) {
      const RunFieldState& F = r->fs[f];
      MixField& m = a.f[f];
      m.cells = static_cast<const float2*>(F.f->a);
      m.first = p.first_before[f];
      m.n = F.f->ngrid;
      m.ld = F.f->ld;
      m.nslice = r->nslice;
      m.harm = F.harm;
      m.do_source = st.in_undulator && (F.harm % 2) == 1;
      m.gridmax = (float)F.f->gridmax;
      m.dgrid = (float)F.f->dgrid;
      m.inv_dgrid = (float)(1.0 / F.f->dgrid);
      m.rtmp = (float)(p.fc[f] / F.f->xks);
      m.bbox = F.d_bbox;
      xks_local = F.f->xks / (double)F.harm;
    }
    a.gref = gbase;
    a.gref_f = (float)gref;
    a.xks = xks_local;
    a.zt0 = (float)(-2.0 / xks_local);
    a.xku = st.ku != 0.0 ? st.ku : xks_local * 0.5 / gref / gref;
    a.delz = st.delz;
    a.half = (float)(0.5 * st.delz);
    a.autophase = st.autophase;
    a.aw = (float)st.aw;
    a.aw2 = (float)(st.aw * st.aw);
    a.ax = (float)st.ax;
    a.ay = (float)st.ay;
    a.kx = (float)st.kx;
    a.ky = (float)st.ky;
    a.gradx = (float)st.gradx;
    a.grady = (float)st.grady;
    const double betpar0 = std::sqrt(1 - (1 + st.aw * st.aw) / gref / gref);
    const double quad = st.qf * gref;
    const double qnatx = st.kx * st.aw * st.aw / gref / betpar0;
    const double qnaty = st.ky * st.aw * st.aw / gref / betpar0;
    a.xm = plane_map_f(quad + qnatx, quad * st.dqx + qnatx * st.ax);
    a.ym = plane_map_f(-quad + qnaty, -quad * st.dqy + qnaty * st.ay);
    if (st.chic_angle != 0) {
      // chicane matrix from the drop-in path's builder (TrackBeamCUDA.cpp:93-148)
      double m[16];
      g4b_chicane_matrix(st.chic_angle, st.chic_lb, st.chic_ld, st.chic_lt, m);
      a.pre = 1;
      a.m00 = (float)m[0];
      a.m01 = (float)m[1];
      a.m10 = (float)m[4];
      a.m11 = (float)m[5];
      a.m22 = (float)m[10];
      a.m23 = (float)m[11];
      a.m32 = (float)m[14];
      a.m33 = (float)m[15];
      const double ang = st.chic_angle, lb = st.chic_lb, ld = st.chic_ld;
      double r56 = (4 * lb / std::sin(ang) * (1 - ang / std::tan(ang)) +
                    2 * ld * std::tan(ang) / std::cos(ang)) * ang;
      a.r56 = r56 * 4 * std::asin(1.0) / r->desc.lambda0 / gref;
      a.r56_off = gbase - gref;  // gamma - gamma0 = dg + (gbase - gamma0)
      a.has_r56 = 1;
    }
    if (st.cx != 0 || st.cy != 0) {
      a.post = 1;
      a.cx = (float)(st.cx * gref);
      a.cy = (float)(st.cy * gref);
    }
    a.err = c->d_error;
    L.has_beam = true;
    L.bs = a;
  }
  // K2
  double* step_hist = r->d_hist + (size_t)(i % r->hist_steps) * r->step_doubles;
  {
    BeamDiagArgs b{};
    b.xy = r->xy;
    b.pxy = r->pxy;
    b.dg = r->dg;
    b.th = r->th;
    b.off = r->d_off;
    b.nbunch = r->desc.nbunch;
    b.need_aux = 1;
    b.gref = gbase;
    b.beam_part = r->d_beam_part;
    L.bd = b;
    DepArgs a{};
    a.xy = r->xy;
    a.dg = r->dg;
    a.th = r->th;
    a.off = r->d_off;
    a.current = r->d_current;
    a.qpred = r->d_qpred;
    a.nfield = r->nfield;
    a.ax = (float)st.ax;
    a.ay = (float)st.ay;
    a.kx = (float)st.kx;
    a.ky = (float)st.ky;
    a.gradx = (float)st.gradx;
    a.grady = (float)st.grady;
    a.delz = st.delz;
    a.gref_f = (float)gbase;
    a.err = c->d_error;
    for (int f = 0; f < r->nfield; ++f) {
      const RunFieldState& F = r->fs[f];
      DepField& d = a.f[f];
      d.src = static_cast<float2*>(F.f->src);
      d.desc = F.f->desc;
      d.bbox = F.d_bbox;
      d.mpred = F.d_mpred;
      d.cap = (size_t)F.f->ngrid * F.f->ld;
      d.first = p.first_before[f];
      d.n = F.f->ngrid;
      d.ld = F.f->ld;
      d.nslice = r->nslice;
      d.harm = F.harm;
      d.do_source = st.in_undulator && (F.harm % 2) == 1 && p.fc[f] != 0.0;
      d.gridmax = (float)F.f->gridmax;
      d.dgrid = (float)F.f->dgrid;
      d.inv_dgrid = (float)(1.0 / F.f->dgrid);
      d.dgrid_d = F.f->dgrid;
      d.fc = p.fc[f];
      d.xks = F.f->xks;
    }
    L.dd = a;
  }
  // K3/K4 per field
  for (int f = 0; f < r->nfield; ++f) {
    RunFieldState& F = r->fs[f];
    F.f->first = p.first_before[f];
    const bool src = st.in_undulator && (F.harm % 2) == 1 && p.fc[f] != 0.0 && r->npart > 0;
    AdiYExtras ex{p.zero_start[f], p.zero_count[f], F.d_part};
    if (int rc = adi_plan(F.adis[p.adi_index[f]], F.f, src ? F.f->src : nullptr, F.f->desc, &ex,
                          L.adi[f]))
      return rc;
    F.f->first = p.first_after[f];
  }
  // K5
  {
    FinalizeArgs a{};
    a.nfield = r->nfield;
    a.nslice = r->nslice;
    a.field_hist = step_hist + r->rec_beam * r->nslice;
    a.beam_hist = step_hist;
    a.beam_part = r->d_beam_part;
    a.rec = (int)r->rec_beam;
    for (int f = 0; f < r->nfield; ++f) {
      a.part[f] = r->fs[f].d_part;
      a.bbox[f] = r->fs[f].d_bbox;
      a.nband[f] = r->fs[f].nband;
      a.first_after[f] = p.first_after[f];
    }
    L.nfin = 10 * r->nfield * r->nslice + r->nslice * (int)r->rec_beam;
    L.fa = a;
  }
  return G4B_OK;
}

// Launches one step of one run from its resolved arguments.
int launch_single(g4b_run* r, const StepArgs& L) {
  g4b_ctx* c = r->ctx;
  // every kernel of the step on the context's stream is a programmatic
  // dependent launch (launch_pdl): it starts while its predecessor drains
  if (L.has_beam) {
    LaunchScope ls(c, "run_beam_step");
    auto kern = r->nfield == 1 ? beam_step_kernel<1>
                               : (r->nfield == 2 ? beam_step_kernel<2> : beam_step_kernel<0>);
    G4B_CUDA_TRY(launch_pdl(kern, (unsigned)r->nchunk, kStepThreads, 0, c->stream, L.bs));
  }
  if (int rc = check_launch(c, "beam_step_kernel")) return rc;
  // The beam diagnostics depend only on K1.  A run with slices enough to
  // fill the GPU twice launches them as a kernel of their own: in a captured
  // graph a branch beside the deposition and the ADI passes (on SMs those
  // leave idle), joined before the finalize.  A smaller run computes them in
  // the deposition's CTAs: the slice's last deposition part, before its band.
  auto diag = [&](cudaStream_t st) {
    LaunchScope ls(c, "run_beam_diag");
    if (r->desc.nbunch == 1)
      beam_diag_kernel<1><<<r->nslice * kDepParts, kDiagThreads, 0, st>>>(L.bd);
    else
      beam_diag_kernel<kMaxBunch><<<r->nslice * kDepParts, kDiagThreads, 0, st>>>(L.bd);
    return check_launch(c, "beam_diag_kernel");
  };
  const bool own = r->nslice >= 2 * c->sm_count;
  const bool branch = own && r->capturing;
  if (branch) {
    G4B_CUDA_TRY(cudaEventRecord(r->ev_fork, c->stream));
    G4B_CUDA_TRY(cudaStreamWaitEvent(r->aux, r->ev_fork, 0));
    if (int rc = diag(r->aux)) return rc;
    G4B_CUDA_TRY(cudaEventRecord(r->ev_join, r->aux));
  }
  if (own) {
    {
      LaunchScope ls(c, "run_deposit");
      G4B_CUDA_TRY(launch_pdl(deposit_kernel, (unsigned)(r->nslice * kDepSplit), kDepThreads,
                              kDepSmem, c->stream, L.dd));
    }
    if (int rc = check_launch(c, "deposit_kernel")) return rc;
    if (!branch)
      if (int rc = diag(c->stream)) return rc;
  } else {
    LaunchScope ls(c, "run_deposit_diag");
    const DepDiagLaunch dl{L.dd, L.bd};
    const unsigned grid = (unsigned)(r->nslice * kDepSplit);
    const bool wide = r->nslice * kDepSplit < c->sm_count;
    const bool one = r->desc.nbunch == 1;
    if (wide)
      G4B_CUDA_TRY(launch_pdl(one ? deposit_diag_kernel<1, kDepWideThreads>
                                  : deposit_diag_kernel<kMaxBunch, kDepWideThreads>,
                              grid, kDepWideThreads, kDepSmem, c->stream, dl));
    else
      G4B_CUDA_TRY(launch_pdl(one ? deposit_diag_kernel<1, kDepThreads>
                                  : deposit_diag_kernel<kMaxBunch, kDepThreads>,
                              grid, kDepThreads, kDepSmem, c->stream, dl));
    if (int rc = check_launch(c, "deposit_diag_kernel")) return rc;
  }
  for (int f = 0; f < r->nfield; ++f)
    if (int rc = adi_launch(r->fs[f].f, L.adi[f])) return rc;
  if (branch) G4B_CUDA_TRY(cudaStreamWaitEvent(c->stream, r->ev_join, 0));
  {
    LaunchScope ls(c, "run_diag_finalize");
    G4B_CUDA_TRY(launch_pdl(diag_finalize_kernel, (unsigned)((L.nfin + 255) / 256), 256, 0,
                            c->stream, L.fa));
  }
  return check_launch(c, "diag_finalize_kernel");
}

int enqueue_step(g4b_run* r, int i, const StepPlan& p) {
  StepArgs L;
  if (int rc = build_step(r, i, p, L)) return rc;
  return launch_single(r, L);
}

std::vector<int> state_key(g4b_run* r) {
  std::vector<int> k;
  for (int f = 0; f < r->nfield; ++f) {
    k.push_back(r->fs[f].first);
    k.push_back(r->fs[f].f->mode);  // the ADI row layout the graph launches
    double a = r->fs[f].accuslip;
    int v[2];
    std::memcpy(v, &a, 8);
    k.push_back(v[0]);
    k.push_back(v[1]);
  }
  return k;
}

}  // namespace

extern "C" {

int g4b_run_create(g4b_ctx* c, const g4b_run_desc* d, const int64_t* off, g4b_run** out) {
  if (!d || !off || !out) return fail(G4B_ERR_ARG, "g4b_run_create: null arg");
  *out = nullptr;
  // The exact-integer deposition scales a slice's contributions so that the
  // fullest cell of its tile sums to at most 2^30; with at most kRunMaxNp
  // particles per slice every contribution keeps at least 2^30 / kRunMaxNp =
  // 2^14 quanta.  Checked before anything touches the device.
  if (d->nslice > 0)
    for (int s = 0; s < d->nslice; ++s)
      if (off[s + 1] - off[s] > kRunMaxNp)
        return fail(G4B_ERR_RANGE, "g4b_run_create: slice " + std::to_string(s) + " holds " +
                                       std::to_string(off[s + 1] - off[s]) +
                                       " particles; the mixed form takes at most " +
                                       std::to_string(kRunMaxNp) + " per slice");
  if (!c) return fail(G4B_ERR_ARG, "g4b_run_create: null ctx");
  if (d->nslice <= 0 || d->nfield < 1 || d->nfield > kRunFields || d->nbunch < 1 ||
      d->nbunch > kMaxBunch || !(d->gamma_ref > 1) || !(d->lambda0 > 0) || !(d->sample > 0))
    return fail(G4B_ERR_ARG, "g4b_run_create: bad descriptor");
  if (d->precision != G4B_MIXED)
    return fail(G4B_ERR_ARG, "g4b_run_create: the fused run holds mixed-precision state");
  for (int f = 0; f < d->nfield; ++f)
    if (d->ngrid[f] + 2 > kDepMaxWidth)
      return fail(G4B_ERR_ARG, "g4b_run_create: ngrid above the mixed form's limit (880)");
  if (off[0] != 0) return fail(G4B_ERR_ARG, "g4b_run_create: slice_offsets[0] != 0");
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  auto r = new (std::nothrow) g4b_run();
  if (!r) return fail(G4B_ERR_NOMEM, "g4b_run_create: host allocation");
  r->ctx = c;
  ctx_retain(c);
  r->desc = *d;
  r->nslice = d->nslice;
  r->nfield = d->nfield;
  r->npart = off[d->nslice];
  std::vector<int4> chunks;
  for (int s = 0; s < d->nslice; ++s) {
    if (off[s + 1] < off[s]) {
      delete r;
      return fail(G4B_ERR_ARG, "g4b_run_create: slice offsets not monotonic");
    }
    r->max_np = std::max<int64_t>(r->max_np, off[s + 1] - off[s]);
    for (int64_t p = off[s]; p < off[s + 1]; p += kRunChunk) {
      const int64_t e = std::min<int64_t>(p + kRunChunk, off[s + 1]);
      chunks.push_back(make_int4(s, (int)(p & 0x7fffffff), (int)(e - p), (int)(p >> 31)));
    }
  }
  r->nchunk = (int)chunks.size();
  const size_t np = (size_t)std::max<int64_t>(r->npart, 1);
  cudaError_t e = cudaSuccess;
  auto A = [&](void** p, size_t b) {
    if (e == cudaSuccess) e = dev_alloc(c, p, b);
    if (e == cudaSuccess) r->bytes += b;
  };
  A((void**)&r->xy, np * 8);
  A((void**)&r->pxy, np * 8);
  A((void**)&r->dg, np * 4);
  A((void**)&r->th, np * 8);
  A((void**)&r->d_off, (d->nslice + 1) * 8);
  A((void**)&r->d_chunks, std::max(1, r->nchunk) * sizeof(int4));
  A((void**)&r->d_current, d->nslice * 8);
  A((void**)&r->d_eloss, d->nslice * 8);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(r->d_off, off, (d->nslice + 1) * 8, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && r->nchunk)
    e = cudaMemcpyAsync(r->d_chunks, chunks.data(), chunks.size() * sizeof(int4),
                        cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(r->d_current, 0, d->nslice * 8, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(r->d_eloss, 0, d->nslice * 8, c->stream);
  if (e != cudaSuccess) {
    g4b_run_destroy(r);
    return cuda_fail(e, "g4b_run_create: device allocation");
  }
  for (int f = 0; f < d->nfield; ++f) {
    RunFieldState& F = r->fs[f];
    F.harm = d->harm[f];
    int rc = g4b_field_create(c, d->nslice, d->ngrid[f], d->gridmax[f],
                              d->lambda0 / (double)d->harm[f], d->harm[f], G4B_MIXED, 0, &F.f);
    if (rc) {
      g4b_run_destroy(r);
      return rc;
    }
    r->bytes += F.f->bytes;
    F.nband = (F.f->ngrid + F.f->band_rows - 1) / F.f->band_rows;
    A((void**)&F.d_bbox, d->nslice * sizeof(int4));
    A((void**)&F.d_mpred, d->nslice * kDepSplit * sizeof(int));
    A((void**)&F.d_part, (size_t)d->nslice * F.nband * 9 * 8);
    if (e != cudaSuccess) {
      g4b_run_destroy(r);
      return cuda_fail(e, "g4b_run_create: device allocation");
    }
    std::vector<int4> init(d->nslice, make_int4(1 << 30, 1 << 30, -1, -1));
    e = cudaMemcpyAsync(F.d_bbox, init.data(), init.size() * sizeof(int4),
                        cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(F.d_mpred, 0, d->nslice * kDepSplit * sizeof(int), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      g4b_run_destroy(r);
      return cuda_fail(e, "g4b_run_create: bbox init");
    }
  }
  r->rec_beam = kBeamRec + 2 * d->nbunch;
  A((void**)&r->d_beam_part, (size_t)d->nslice * kDepParts * r->rec_beam * 8);
  A((void**)&r->d_qpred, d->nslice * kDepSplit * sizeof(float));
  if (e == cudaSuccess)
    e = cudaMemsetAsync(r->d_qpred, 0, d->nslice * kDepSplit * sizeof(float), c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    g4b_run_destroy(r);
    return cuda_fail(e, "g4b_run_create: device allocation");
  }
  r->step_doubles = (size_t)d->nslice * (r->rec_beam + 9 * d->nfield);
  cudaFuncSetAttribute(deposit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kDepSmem);
  cudaFuncSetAttribute(deposit_diag_kernel<1, kDepThreads>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDepSmem);
  cudaFuncSetAttribute(deposit_diag_kernel<kMaxBunch, kDepThreads>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDepSmem);
  cudaFuncSetAttribute(deposit_diag_kernel<1, kDepWideThreads>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDepSmem);
  cudaFuncSetAttribute(deposit_diag_kernel<kMaxBunch, kDepWideThreads>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDepSmem);
  *out = r;
  return G4B_OK;
}

int g4b_run_destroy(g4b_run* r) {
  if (!r) return G4B_OK;
  ctx_quiesce(r->ctx);
  if (r->gexec) cudaGraphExecDestroy(r->gexec);
  if (r->ev_fork) cudaEventDestroy(r->ev_fork);
  if (r->ev_join) cudaEventDestroy(r->ev_join);
  if (r->aux) cudaStreamDestroy(r->aux);
  void* ptrs[] = {r->xy, r->pxy, r->dg, r->th, r->d_off, r->d_chunks, r->d_current,
                  r->d_eloss, r->d_hist, r->d_beam_part, r->d_qpred};
  for (void* p : ptrs) dev_free(r->ctx, p);
  for (int f = 0; f < kRunFields; ++f) {
    RunFieldState& F = r->fs[f];
    for (g4b_adi* a : F.adis) g4b_adi_destroy(a);
    if (F.f) g4b_field_destroy(F.f);
    dev_free(r->ctx, F.d_bbox);
    dev_free(r->ctx, F.d_mpred);
    dev_free(r->ctx, F.d_part);
  }
  ctx_release(r->ctx);
  delete r;
  return G4B_OK;
}

// FP64 particle arrays cross the bus and are converted on the device, in
// chunks through a staging buffer (theta stays FP64 and is copied directly).
int g4b_run_upload_beam(g4b_run* r, const double* x, const double* y, const double* px,
                        const double* py, const double* gamma, const double* theta) {
  if (!r || !x || !y || !px || !py || !gamma || !theta)
    return fail(G4B_ERR_ARG, "g4b_run_upload_beam: null arg");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  const size_t n = (size_t)r->npart;
  cudaStream_t s = r->ctx->stream;
  if (n == 0) return G4B_OK;
  const size_t chunk = std::min(n, (size_t)(64u << 20) / 40);
  double* stage = nullptr;
  G4B_CUDA_TRY(dev_alloc(r->ctx, (void**)&stage, chunk * 40));
  const double* src[5] = {x, y, px, py, gamma};
  cudaError_t e = cudaMemcpyAsync(r->th, theta, n * 8, cudaMemcpyHostToDevice, s);
  const float gf = (float)r->desc.gamma_ref;
  for (size_t p0 = 0; p0 < n && e == cudaSuccess; p0 += chunk) {
    const size_t m = std::min(chunk, n - p0);
    for (int k = 0; k < 5 && e == cudaSuccess; ++k)
      e = cudaMemcpyAsync(stage + k * chunk, src[k] + p0, m * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
      const unsigned grid = (unsigned)std::min<size_t>((m + 255) / 256, 1u << 20);
      beam_f64_to_mixed<<<grid, 256, 0, s>>>(stage, chunk, m, gf, r->xy + p0, r->pxy + p0,
                                             r->dg + p0);
      e = cudaGetLastError();
    }
  }
  dev_free(r->ctx, stage);
  // a new beam: the next deposition counts before it accumulates
  for (int f = 0; f < r->nfield && e == cudaSuccess; ++f)
    e = cudaMemsetAsync(r->fs[f].d_mpred, 0, r->nslice * kDepSplit * sizeof(int), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(r->d_qpred, 0, r->nslice * kDepSplit * sizeof(float), s);
  const cudaError_t es = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "g4b_run_upload_beam");
  if (es != cudaSuccess) return cuda_fail(es, "g4b_run_upload_beam");
  return G4B_OK;
}

int g4b_run_download_beam(g4b_run* r, double* x, double* y, double* px, double* py,
                          double* gamma, double* theta) {
  if (!r) return fail(G4B_ERR_ARG, "g4b_run_download_beam: null run");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  const size_t n = (size_t)r->npart;
  cudaStream_t s = r->ctx->stream;
  if (n == 0) return read_device_error(r->ctx, "g4b_run_download_beam");
  const size_t chunk = std::min(n, (size_t)(64u << 20) / 40);
  double* stage = nullptr;
  G4B_CUDA_TRY(dev_alloc(r->ctx, (void**)&stage, chunk * 40));
  double* dst[5] = {x, y, px, py, gamma};
  cudaError_t e = theta ? cudaMemcpyAsync(theta, r->th, n * 8, cudaMemcpyDeviceToHost, s)
                        : cudaSuccess;
  const double gf = (double)(float)r->desc.gamma_ref;
  for (size_t p0 = 0; p0 < n && e == cudaSuccess; p0 += chunk) {
    const size_t m = std::min(chunk, n - p0);
    const unsigned grid = (unsigned)std::min<size_t>((m + 255) / 256, 1u << 20);
    beam_mixed_to_f64<<<grid, 256, 0, s>>>(r->xy + p0, r->pxy + p0, r->dg + p0, gf, m, stage,
                                           chunk);
    e = cudaGetLastError();
    for (int k = 0; k < 5 && e == cudaSuccess; ++k)
      if (dst[k]) e = cudaMemcpyAsync(dst[k] + p0, stage + k * chunk, m * 8,
                                      cudaMemcpyDeviceToHost, s);
  }
  dev_free(r->ctx, stage);
  const cudaError_t es = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "g4b_run_download_beam");
  if (es != cudaSuccess) return cuda_fail(es, "g4b_run_download_beam");
  return read_device_error(r->ctx, "g4b_run_download_beam");
}

int g4b_run_upload_field(g4b_run* r, int fi, const double* cells, int first) {
  if (!r || fi < 0 || fi >= r->nfield || first < 0 || first >= r->nslice)
    return fail(G4B_ERR_ARG, "g4b_run_upload_field: bad argument");
  RunFieldState& F = r->fs[fi];
  if (cells) {
    if (int rc = g4b_field_upload(F.f, cells)) return rc;
  } else {  // a zero field (no seed)
    G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
    G4B_CUDA_TRY(cudaMemsetAsync(F.f->a, 0, (size_t)F.f->nslice * F.f->ngrid * F.f->ld *
                                                F.f->cell_bytes, r->ctx->stream));
    G4B_CUDA_TRY(cudaStreamSynchronize(r->ctx->stream));
  }
  if (int rc = g4b_field_set_first(F.f, first)) return rc;
  F.first = first;
  F.accuslip = 0.0;
  return G4B_OK;
}

int g4b_run_download_field(g4b_run* r, int fi, double* cells, int* first) {
  if (!r || fi < 0 || fi >= r->nfield || !cells)
    return fail(G4B_ERR_ARG, "g4b_run_download_field: bad argument");
  RunFieldState& F = r->fs[fi];
  if (int rc = g4b_field_download(F.f, cells)) return rc;
  if (first) *first = F.first;
  return read_device_error(r->ctx, "g4b_run_download_field");
}

int g4b_run_set_current(g4b_run* r, const double* current) {
  if (!r || !current) return fail(G4B_ERR_ARG, "g4b_run_set_current: null arg");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  G4B_CUDA_TRY(cudaMemcpyAsync(r->d_current, current, r->nslice * 8, cudaMemcpyHostToDevice,
                               r->ctx->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(r->ctx->stream));
  return G4B_OK;
}

int g4b_run_set_eloss(g4b_run* r, const double* eloss) {
  if (!r) return fail(G4B_ERR_ARG, "g4b_run_set_eloss: null run");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  if (eloss)
    G4B_CUDA_TRY(cudaMemcpyAsync(r->d_eloss, eloss, r->nslice * 8, cudaMemcpyHostToDevice,
                                 r->ctx->stream));
  else
    G4B_CUDA_TRY(cudaMemsetAsync(r->d_eloss, 0, r->nslice * 8, r->ctx->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(r->ctx->stream));
  return G4B_OK;
}

int g4b_run_set_lattice(g4b_run* r, int nstep, const g4b_step* steps, const double* fc,
                        const double* slip, int hist_steps) {
  if (!r || nstep <= 0 || !steps || !fc || !slip)
    return fail(G4B_ERR_ARG, "g4b_run_set_lattice: bad argument");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  r->steps.assign(steps, steps + nstep);
  r->fc.assign(fc, fc + (size_t)nstep * r->nfield);
  r->slip.assign(slip, slip + nstep);
  // one FP64 factorisation per distinct step length and field grid
  for (int f = 0; f < r->nfield; ++f) {
    RunFieldState& F = r->fs[f];
    for (int i = 0; i < nstep; ++i) {
      const double dz = steps[i].delz;
      if (std::find(F.adi_delz.begin(), F.adi_delz.end(), dz) != F.adi_delz.end()) continue;
      g4b_adi* a = nullptr;
      if (int rc = g4b_adi_create(r->ctx, &a)) return rc;
      if (int rc = g4b_adi_init(a, dz, F.f->dgrid, F.f->xks, F.f->ngrid)) {
        g4b_adi_destroy(a);
        return rc;
      }
      F.adis.push_back(a);
      F.adi_delz.push_back(dz);
    }
    if (int rc = adi_configure(F.f)) return rc;
  }
  const int hs = hist_steps > 0 ? hist_steps : nstep;
  dev_free(r->ctx, r->d_hist);
  r->d_hist = nullptr;
  G4B_CUDA_TRY(dev_alloc(r->ctx, (void**)&r->d_hist, (size_t)hs * r->step_doubles * 8));
  G4B_CUDA_TRY(cudaMemsetAsync(r->d_hist, 0, (size_t)hs * r->step_doubles * 8, r->ctx->stream));
  r->hist_steps = hs;
  if (r->gexec) {
    cudaGraphExecDestroy(r->gexec);
    r->gexec = nullptr;
  }
  return G4B_OK;
}

static int run_capture(g4b_run* r, int first_step, int nsteps, cudaGraphExec_t* out) {
  g4b_ctx* c = r->ctx;
  cudaGraph_t g = nullptr;
  if (!r->aux) {
    G4B_CUDA_TRY(cudaStreamCreateWithFlags(&r->aux, cudaStreamNonBlocking));
    G4B_CUDA_TRY(cudaEventCreateWithFlags(&r->ev_fork, cudaEventDisableTiming));
    G4B_CUDA_TRY(cudaEventCreateWithFlags(&r->ev_join, cudaEventDisableTiming));
  }
  const bool prof = c->prof.on;  // no profiler events inside a graph
  c->prof.on = false;
  G4B_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  r->capturing = true;
  int rc = G4B_OK;
  for (int k = 0; k < nsteps && rc == G4B_OK; ++k) {
    const int i = (first_step + k) % (int)r->steps.size();
    StepPlan p;
    rc = plan_step(r, i, p);
    if (rc == G4B_OK) rc = enqueue_step(r, first_step + k, p);
  }
  r->capturing = false;
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  c->prof.on = prof;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  return G4B_OK;
}

// Enqueue lattice steps [first_step, first_step + nsteps) (indices wrap).
// use_graph: 0 = direct launches; 1 = replay a CUDA graph of the whole
// range (captured on first use and reused while the range and the slippage
// state match).
static int run_capture(g4b_run* r, int first_step, int nsteps, cudaGraphExec_t* out);

static int run_prepare(g4b_run* r, int first_step, int nsteps) {
  std::vector<int> key = state_key(r);
  const bool hit = r->gexec && r->g_first == first_step && r->g_n == nsteps && r->g_state == key;
  if (hit) return G4B_OK;
  if (r->gexec) cudaGraphExecDestroy(r->gexec);
  r->gexec = nullptr;
  // capture advances the host slippage model; restore it afterwards
  int first[kRunFields];
  double acc[kRunFields];
  for (int f = 0; f < r->nfield; ++f) {
    first[f] = r->fs[f].first;
    acc[f] = r->fs[f].accuslip;
  }
  int rc = run_capture(r, first_step, nsteps, &r->gexec);
  for (int f = 0; f < r->nfield; ++f) {
    r->fs[f].first = first[f];
    r->fs[f].accuslip = acc[f];
    r->fs[f].f->first = first[f];
  }
  if (rc) return rc;
  r->g_first = first_step;
  r->g_n = nsteps;
  r->g_state = key;
  return G4B_OK;
}

// Capture (without launching) the CUDA graph of steps [first_step,
// first_step + nsteps) from the current state, for a later g4b_run_advance
// with use_graph on the same range.
int g4b_run_prepare(g4b_run* r, int first_step, int nsteps) {
  if (!r || nsteps <= 0 || first_step < 0) return fail(G4B_ERR_ARG, "g4b_run_prepare: bad arg");
  if (r->steps.empty()) return fail(G4B_ERR_STATE, "g4b_run_prepare: no lattice");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  return run_prepare(r, first_step, nsteps);
}

int g4b_run_advance(g4b_run* r, int first_step, int nsteps, int use_graph) {
  if (!r || nsteps < 0 || first_step < 0) return fail(G4B_ERR_ARG, "g4b_run_advance: bad arg");
  if (r->steps.empty()) return fail(G4B_ERR_STATE, "g4b_run_advance: no lattice");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  if (!use_graph) {
    for (int k = 0; k < nsteps; ++k) {
      const int i = (first_step + k) % (int)r->steps.size();
      StepPlan p;
      if (int rc = plan_step(r, i, p)) return rc;
      if (int rc = enqueue_step(r, first_step + k, p)) return rc;
    }
    return G4B_OK;
  }
  if (int rc = run_prepare(r, first_step, nsteps)) return rc;
  r->ctx->launches += (uint64_t)nsteps * (4 + 2 * r->nfield);
  G4B_CUDA_TRY(cudaGraphLaunch(r->gexec, r->ctx->stream));
  // advance the host model exactly as the captured steps did
  for (int k = 0; k < nsteps; ++k) {
    StepPlan p;
    if (int rc = plan_step(r, (first_step + k) % (int)r->steps.size(), p)) return rc;
    for (int f = 0; f < r->nfield; ++f) r->fs[f].f->first = p.first_after[f];
  }
  return G4B_OK;
}

// Diagnostics of lattice step `step` (the history keeps the last hist_steps
// steps): beam[nslice*(23+2*nbunch)] in the reference's stats order, field
// [nfield*nslice*9] = power, x1, x2, y1, y2, farfield re/im, centre re/im,
// indexed by beam slice.  Synchronises.
int g4b_run_history(g4b_run* r, int step, double* beam, double* field) {
  if (!r || step < 0) return fail(G4B_ERR_ARG, "g4b_run_history: bad arg");
  if (!r->d_hist) return fail(G4B_ERR_STATE, "g4b_run_history: no lattice");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  const double* h = r->d_hist + (size_t)(step % r->hist_steps) * r->step_doubles;
  const size_t nb = (size_t)r->nslice * r->rec_beam;
  if (beam)
    G4B_CUDA_TRY(cudaMemcpyAsync(beam, h, nb * 8, cudaMemcpyDeviceToHost, r->ctx->stream));
  if (field)
    G4B_CUDA_TRY(cudaMemcpyAsync(field, h + nb, (size_t)r->nfield * r->nslice * 9 * 8,
                                 cudaMemcpyDeviceToHost, r->ctx->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(r->ctx->stream));
  return read_device_error(r->ctx, "g4b_run_history");
}

// Diagnostics of steps [first, first + n) in one read: out[n][step record],
// a step record being beam [nslice][23 + 2 nbunch] then field [nfield][nslice][9].
int g4b_run_history_range(g4b_run* r, int first, int n, double* out) {
  if (!r || first < 0 || n < 0 || !out) return fail(G4B_ERR_ARG, "g4b_run_history_range: bad arg");
  if (!r->d_hist) return fail(G4B_ERR_STATE, "g4b_run_history_range: no lattice");
  if (n > r->hist_steps)
    return fail(G4B_ERR_RANGE, "g4b_run_history_range: more steps than the history keeps");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  const size_t sd = r->step_doubles;
  int done = 0;
  while (done < n) {
    const int slot = (first + done) % r->hist_steps;
    const int cnt = std::min(n - done, r->hist_steps - slot);
    G4B_CUDA_TRY(cudaMemcpyAsync(out + (size_t)done * sd, r->d_hist + (size_t)slot * sd,
                                 (size_t)cnt * sd * 8, cudaMemcpyDeviceToHost, r->ctx->stream));
    done += cnt;
  }
  G4B_CUDA_TRY(cudaStreamSynchronize(r->ctx->stream));
  return read_device_error(r->ctx, "g4b_run_history_range");
}

int g4b_run_device_bytes(g4b_run* r, uint64_t* bytes) {
  if (!r || !bytes) return fail(G4B_ERR_ARG, "g4b_run_device_bytes: null arg");
  *bytes = r->bytes + (uint64_t)r->hist_steps * r->step_doubles * 8;
  return G4B_OK;
}

}  // extern "C"

// =========================================================== batched runs ===
// Many independent runs advanced together: per step one persistent launch
// per kernel phase covers every attached run.  Each run keeps its own state
// (a g4b_run); the engine resolves every run's step arguments on the host
// (build_step, the same code the single-run path uses), uploads them with
// one copy, and the batch kernels walk work lists of (run, chunk / slice /
// band) items.  Every item is computed exactly as in the single-run kernels,
// so a run's results do not depend on what else is in the batch.

namespace {

// ADI kernel modes (pick_mode): 32-lane rows, then 16-lane rows
constexpr int kNumM = 22;
const int kMList[kNumM] = {1,   3,   5,   7,   9,   11,  13,  15,  17,  21,  25,
                           33,  105, 107, 109, 111, 113, 115, 117, 121, 125, 133};
int m_index(int M) {
  for (int i = 0; i < kNumM; ++i)
    if (kMList[i] == M) return i;
  return -1;
}

// counts block at the head of the staging area
struct BatchCounts {
  int beam, dep, fin, pad;
  int adi[kNumM];
};

template <typename T>
size_t align_up(size_t x) {
  const size_t a = alignof(T) < 128 ? 128 : alignof(T);
  return (x + a - 1) / a * a;
}

}  // namespace

struct g4b_batch {
  g4b_ctx* ctx = nullptr;
  int max_runs = 0;
  std::vector<g4b_run*> runs;   // per slot (nullptr = free)
  std::vector<int> next, last;  // per slot: next lattice step, end (exclusive)
  bool dirty = true;            // composition changed since the last upload
  // staging (pinned host, double-buffered) and device mirror
  size_t off_bs = 0, off_dd = 0, off_bd = 0, off_fa = 0, off_ax = 0, off_ay = 0, off_mx = 0, off_my = 0,
         args_bytes = 0;
  unsigned char* h_args[2] = {nullptr, nullptr};
  unsigned char* d_args = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr};
  int buf = 0;
  // work lists
  std::vector<int2> beam_items, dep_items;
  std::vector<int4> adi_items[kNumM];
  size_t items_cap = 0, h_items_cap[2] = {0, 0};
  unsigned char* d_items = nullptr;
  unsigned char* h_items[2] = {nullptr, nullptr};  // pinned, alternating
  cudaEvent_t items_copied[2] = {nullptr, nullptr};
  int ibuf = 0;
  int stable = 0;               // steps since the composition last changed
  size_t off_beam = 0, off_dep = 0, off_adi[kNumM] = {};
  BatchCounts counts{};
  size_t smem_x[kNumM] = {}, smem_y[kNumM] = {};
  // push kernel field count (1 or 2 when every run has it, else 0 = any:
  // the single-run kernel of the same count), deposition bunching kind
  int nf_kind = 1, nb_kind = 1;
  // launch shapes (CTAs per kernel), chosen by the tuner
  int grid[4] = {0, 0, 0, 0};    // beam, deposit, adi, finalize
  int tune_left = 0, tune_idx = 0;
  std::vector<float> tune_ms[4];

  cudaEvent_t ev[5] = {};
  // concurrent branches of a step: the beam diagnostics beside the
  // deposition and ADI passes; the ADI kernels of different row layouts
  // beside one another
  static constexpr int kAux = 4;
  cudaStream_t aux[kAux] = {};
  cudaEvent_t ev_fork[2] = {}, ev_diag = nullptr, ev_adi[kNumM] = {};
  // graph of one step for the current composition and shapes
  cudaGraphExec_t gexec = nullptr;
  bool graph_valid = false;
  uint64_t steps_done = 0;
};

namespace {

// The tuner's candidates per kernel, in units of SMs.
const int kTuneBeam[4] = {4, 8, 16, 32};
const int kTuneDep[4] = {2, 4, 6, 8};
const int kTuneAdi[4] = {2, 4, 6, 8};

int batch_layout(g4b_batch* b) {
  size_t o = align_up<BatchCounts>(sizeof(BatchCounts));
  const size_t nr = b->max_runs, nf = (size_t)b->max_runs * kRunFields;
  b->off_bs = o;
  o = align_up<BeamStepArgs>(o + nr * sizeof(BeamStepArgs));
  b->off_dd = o;
  o = align_up<DepArgs>(o + nr * sizeof(DepArgs));
  b->off_bd = o;
  o = align_up<BeamDiagArgs>(o + nr * sizeof(BeamDiagArgs));
  b->off_fa = o;
  o = align_up<FinalizeArgs>(o + nr * sizeof(FinalizeArgs));
  b->off_ax = o;
  o = align_up<AdiPassArgs>(o + nf * sizeof(AdiPassArgs));
  b->off_ay = o;
  o = align_up<AdiPassArgs>(o + nf * sizeof(AdiPassArgs));
  b->off_mx = o;
  o = align_up<CUtensorMap>(o + nf * sizeof(CUtensorMap));
  b->off_my = o;
  o = align_up<CUtensorMap>(o + nf * sizeof(CUtensorMap));
  b->args_bytes = o;
  for (int k = 0; k < 2; ++k) {
    G4B_CUDA_TRY(cudaMallocHost(&b->h_args[k], o));
    std::memset(b->h_args[k], 0, o);
    G4B_CUDA_TRY(cudaEventCreateWithFlags(&b->copied[k], cudaEventDisableTiming));
  }
  G4B_CUDA_TRY(cudaMalloc(&b->d_args, o));
  for (auto& e : b->ev) G4B_CUDA_TRY(cudaEventCreate(&e));
  for (auto& e : b->ev_fork) G4B_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto& e : b->ev_adi) G4B_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  G4B_CUDA_TRY(cudaEventCreateWithFlags(&b->ev_diag, cudaEventDisableTiming));
  for (auto& s : b->aux) G4B_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return G4B_OK;
}

// Rebuild the work lists after the set of attached, unfinished runs changed.
int batch_rebuild(g4b_batch* b) {
  b->beam_items.clear();
  b->dep_items.clear();
  for (auto& v : b->adi_items) v.clear();
  std::memset(b->smem_x, 0, sizeof b->smem_x);
  std::memset(b->smem_y, 0, sizeof b->smem_y);
  b->nf_kind = -1;
  b->nb_kind = 1;
  int nactive = 0;
  for (int s = 0; s < b->max_runs; ++s) {
    g4b_run* r = b->runs[s];
    if (!r || b->next[s] >= b->last[s]) continue;
    ++nactive;
    const int kind = r->nfield <= 2 ? r->nfield : 0;
    if (b->nf_kind < 0) b->nf_kind = kind;
    else if (b->nf_kind != kind) b->nf_kind = 0;
    if (r->desc.nbunch != 1) b->nb_kind = 0;
    for (int k = 0; k < r->nchunk; ++k) b->beam_items.push_back(make_int2(s, k));
    for (int sl = 0; sl < r->nslice; ++sl) b->dep_items.push_back(make_int2(s, sl));
    for (int f = 0; f < r->nfield; ++f) {
      g4b_field* F = r->fs[f].f;
      const int mi = m_index(F->mode);
      if (mi < 0) return fail(G4B_ERR_RANGE, "g4b_batch: unsupported grid");
      const int nband = (F->ngrid + F->band_rows - 1) / F->band_rows;
      for (int sl = 0; sl < r->nslice; ++sl)
        for (int bd = 0; bd < nband; ++bd)
          b->adi_items[mi].push_back(make_int4(s * kRunFields + f, sl, bd, 0));
      // shared memory of the largest band in this group
      const int W = F->band_rows, ld = F->ld;
      const size_t cb = F->cell_bytes;
      const size_t out_bytes = (size_t)F->store_nbox * F->store_box_rows * W * cb;
      const size_t tx = (size_t)((W + 2) * ld + W * ld) * cb, ty = (size_t)(W * ld) * cb;
      // pass X: the output staging tile overlays the input tile
      b->smem_x[mi] = std::max(b->smem_x[mi], std::max(tx, out_bytes));
      b->smem_y[mi] = std::max(b->smem_y[mi], (ty + 127) / 128 * 128 + out_bytes);
    }
  }
  b->counts = BatchCounts{};
  b->counts.beam = (int)b->beam_items.size();
  b->counts.dep = (int)b->dep_items.size();
  b->counts.fin = nactive;
  size_t need = 0;
  b->off_beam = 0;
  need = align_up<int2>(b->beam_items.size() * sizeof(int2));
  b->off_dep = need;
  need = align_up<int2>(need + b->dep_items.size() * sizeof(int2));
  for (int m = 0; m < kNumM; ++m) {
    b->counts.adi[m] = (int)b->adi_items[m].size();
    b->off_adi[m] = need;
    need = align_up<int4>(need + b->adi_items[m].size() * sizeof(int4));
  }
  need = std::max<size_t>(need, 256);
  if (need > b->items_cap) {  // stream-ordered: the old lists' readers finish first
    dev_free(b->ctx, b->d_items);
    b->d_items = nullptr;
    b->items_cap = 0;
    G4B_CUDA_TRY(dev_alloc(b->ctx, (void**)&b->d_items, need * 2));
    b->items_cap = need * 2;
  }
  // pinned staging, alternating buffers: wait only for the copy that used
  // this buffer two rebuilds ago
  const int k = b->ibuf;
  if (!b->items_copied[k])
    G4B_CUDA_TRY(cudaEventCreateWithFlags(&b->items_copied[k], cudaEventDisableTiming));
  G4B_CUDA_TRY(cudaEventSynchronize(b->items_copied[k]));
  if (need > b->h_items_cap[k]) {
    if (b->h_items[k]) cudaFreeHost(b->h_items[k]);
    b->h_items[k] = nullptr;
    b->h_items_cap[k] = 0;
    G4B_CUDA_TRY(cudaMallocHost(&b->h_items[k], need * 2));
    b->h_items_cap[k] = need * 2;
  }
  unsigned char* h = b->h_items[k];
  std::memcpy(h + b->off_beam, b->beam_items.data(), b->beam_items.size() * sizeof(int2));
  std::memcpy(h + b->off_dep, b->dep_items.data(), b->dep_items.size() * sizeof(int2));
  for (int m = 0; m < kNumM; ++m)
    std::memcpy(h + b->off_adi[m], b->adi_items[m].data(),
                b->adi_items[m].size() * sizeof(int4));
  G4B_CUDA_TRY(cudaMemcpyAsync(b->d_items, h, need, cudaMemcpyHostToDevice, b->ctx->stream));
  G4B_CUDA_TRY(cudaEventRecord(b->items_copied[k], b->ctx->stream));
  b->ibuf ^= 1;
  b->stable = 0;
  b->dirty = false;
  b->graph_valid = false;
  return G4B_OK;
}

// Resolve this step's arguments of every active run into the staging buffer.
int batch_stage(g4b_batch* b) {
  const int k = b->buf;
  G4B_CUDA_TRY(cudaEventSynchronize(b->copied[k]));  // the copy of two steps ago
  unsigned char* h = b->h_args[k];
  std::memcpy(h, &b->counts, sizeof(BatchCounts));
  auto* bs = reinterpret_cast<BeamStepArgs*>(h + b->off_bs);
  auto* dd = reinterpret_cast<DepArgs*>(h + b->off_dd);
  auto* bd = reinterpret_cast<BeamDiagArgs*>(h + b->off_bd);
  auto* fa = reinterpret_cast<FinalizeArgs*>(h + b->off_fa);
  auto* ax = reinterpret_cast<AdiPassArgs*>(h + b->off_ax);
  auto* ay = reinterpret_cast<AdiPassArgs*>(h + b->off_ay);
  auto* mx = reinterpret_cast<CUtensorMap*>(h + b->off_mx);
  auto* my = reinterpret_cast<CUtensorMap*>(h + b->off_my);
  int nfin = 0;
  for (int s = 0; s < b->max_runs; ++s) {
    g4b_run* r = b->runs[s];
    if (!r || b->next[s] >= b->last[s]) continue;
    const int i = b->next[s];
    StepPlan p;
    if (int rc = plan_step(r, i % (int)r->steps.size(), p)) return rc;
    StepArgs L;
    if (int rc = build_step(r, i, p, L)) return rc;
    bs[s] = L.bs;
    dd[s] = L.dd;
    bd[s] = L.bd;
    fa[nfin++] = L.fa;
    for (int f = 0; f < r->nfield; ++f) {
      ax[s * kRunFields + f] = L.adi[f].x;
      ay[s * kRunFields + f] = L.adi[f].y;
      mx[s * kRunFields + f] = *L.adi[f].tm_x;
      my[s * kRunFields + f] = *L.adi[f].tm_y;
    }
    b->next[s] = i + 1;
    if (b->next[s] >= b->last[s]) b->dirty = true;  // leaves the lists next step
  }
  G4B_CUDA_TRY(cudaMemcpyAsync(b->d_args, h, b->args_bytes, cudaMemcpyHostToDevice,
                               b->ctx->stream));
  G4B_CUDA_TRY(cudaEventRecord(b->copied[k], b->ctx->stream));
  b->buf ^= 1;
  return G4B_OK;
}

// The kernels of one batch step (capturable: no host synchronisation).
int batch_launch(g4b_batch* b, bool timed) {
  g4b_ctx* c = b->ctx;
  const int* counts = reinterpret_cast<const int*>(b->d_args);
  auto ev = [&](int i) {
    if (timed) cudaEventRecord(b->ev[i], c->stream);
  };
  ev(0);
  if (b->counts.beam > 0) {
    BeamBatchArgs a{reinterpret_cast<const BeamStepArgs*>(b->d_args + b->off_bs),
                    reinterpret_cast<const int2*>(b->d_items + b->off_beam), counts + 0};
    LaunchScope ls(c, "batch_beam_step");
    if (b->nf_kind == 1)
      beam_batch_kernel<1><<<b->grid[0], kStepThreads, 0, c->stream>>>(a);
    else if (b->nf_kind == 2)
      beam_batch_kernel<2><<<b->grid[0], kStepThreads, 0, c->stream>>>(a);
    else
      beam_batch_kernel<0><<<b->grid[0], kStepThreads, 0, c->stream>>>(a);
  }
  if (int rc = check_launch(c, "beam_batch_kernel")) return rc;
  ev(1);
  {
    DepBatchArgs a{reinterpret_cast<const DepArgs*>(b->d_args + b->off_dd),
                   reinterpret_cast<const int2*>(b->d_items + b->off_dep), counts + 1};
    LaunchScope ls(c, "batch_deposit");
    deposit_batch_kernel<<<b->grid[1], kDepThreads, kDepSmem, c->stream>>>(a);
  }
  if (int rc = check_launch(c, "deposit_batch_kernel")) return rc;
  // branches (not while the tuner or the profiler times single kernels)
  const bool fork = !timed && !c->prof.on;
  auto diag = [&](cudaStream_t st) {
    DiagBatchArgs a{reinterpret_cast<const BeamDiagArgs*>(b->d_args + b->off_bd),
                    reinterpret_cast<const int2*>(b->d_items + b->off_dep), counts + 1};
    LaunchScope ls(c, "batch_beam_diag");
    if (b->nb_kind == 1)
      beam_diag_batch_kernel<1><<<2 * c->sm_count, kDiagThreads, 0, st>>>(a);
    else
      beam_diag_batch_kernel<kMaxBunch><<<2 * c->sm_count, kDiagThreads, 0, st>>>(a);
    return check_launch(c, "beam_diag_batch_kernel");
  };
  if (fork) {
    G4B_CUDA_TRY(cudaEventRecord(b->ev_fork[0], c->stream));
    G4B_CUDA_TRY(cudaStreamWaitEvent(b->aux[0], b->ev_fork[0], 0));
    if (int rc = diag(b->aux[0])) return rc;
    G4B_CUDA_TRY(cudaEventRecord(b->ev_diag, b->aux[0]));
  } else if (int rc = diag(c->stream)) {
    return rc;
  }
  ev(2);
  for (int pass = 0; pass < 2; ++pass) {
    int ngroups = 0;
    for (int m = 0; m < kNumM; ++m) ngroups += b->counts.adi[m] > 0;
    const bool par = fork && ngroups > 1;
    if (par) G4B_CUDA_TRY(cudaEventRecord(b->ev_fork[1], c->stream));
    int gi = 0;
    for (int m = 0; m < kNumM; ++m) {
      if (b->counts.adi[m] == 0) continue;
      AdiBatchArgs a;
      a.args = reinterpret_cast<const AdiPassArgs*>(b->d_args + (pass ? b->off_ay : b->off_ax));
      a.maps = reinterpret_cast<const CUtensorMap*>(b->d_args + (pass ? b->off_my : b->off_mx));
      a.items = reinterpret_cast<const int4*>(b->d_items + b->off_adi[m]);
      a.nitems = reinterpret_cast<const int*>(b->d_args) + 4 + m;
      const int g = std::min(b->grid[2], b->counts.adi[m]);
      // groups round-robin over the main stream and the branch streams
      // 1..kAux-1 (stream 0 of the branches carries the diagnostics)
      cudaStream_t st = c->stream;
      if (par && gi % g4b_batch::kAux != 0) {
        st = b->aux[gi % g4b_batch::kAux];
        G4B_CUDA_TRY(cudaStreamWaitEvent(st, b->ev_fork[1], 0));
      }
      if (int rc = adi_batch_launch(c, st, kMList[m], pass == 0, a,
                                    pass ? b->smem_y[m] : b->smem_x[m], g))
        return rc;
      if (st != c->stream) G4B_CUDA_TRY(cudaEventRecord(b->ev_adi[gi], st));
      ++gi;
    }
    if (par)
      for (int k = 0; k < gi; ++k)
        if (k % g4b_batch::kAux != 0) G4B_CUDA_TRY(cudaStreamWaitEvent(c->stream, b->ev_adi[k], 0));
    ev(3 + pass);
  }
  if (fork) G4B_CUDA_TRY(cudaStreamWaitEvent(c->stream, b->ev_diag, 0));
  {
    LaunchScope ls(c, "batch_diag_finalize");
    finalize_batch_kernel<<<b->grid[3], 256, 0, c->stream>>>(
        reinterpret_cast<const FinalizeArgs*>(b->d_args + b->off_fa), counts + 2);
  }
  return check_launch(c, "finalize_batch_kernel");
}

void batch_default_grids(g4b_batch* b) {
  const int sm = b->ctx->sm_count;
  b->grid[0] = 2 * kStepBlocks * sm;
  b->grid[1] = 2 * sm;
  b->grid[2] = 4 * sm;
  b->grid[3] = sm;
}

}  // namespace

extern "C" {

int g4b_batch_create(g4b_ctx* c, int max_runs, g4b_batch** out) {
  if (!c || !out || max_runs < 1) return fail(G4B_ERR_ARG, "g4b_batch_create: bad arg");
  *out = nullptr;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  auto b = new (std::nothrow) g4b_batch();
  if (!b) return fail(G4B_ERR_NOMEM, "g4b_batch_create: host allocation");
  b->ctx = c;
  ctx_retain(c);
  b->max_runs = max_runs;
  b->runs.assign(max_runs, nullptr);
  b->next.assign(max_runs, 0);
  b->last.assign(max_runs, 0);
  batch_default_grids(b);
  cudaFuncSetAttribute(deposit_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kDepSmem);
  if (int rc = batch_layout(b)) {
    g4b_batch_destroy(b);
    return rc;
  }
  *out = b;
  return G4B_OK;
}

int g4b_batch_destroy(g4b_batch* b) {
  if (!b) return G4B_OK;
  ctx_quiesce(b->ctx);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  for (int k = 0; k < 2; ++k) {
    if (b->h_args[k]) cudaFreeHost(b->h_args[k]);
    if (b->copied[k]) cudaEventDestroy(b->copied[k]);
  }
  for (auto e : b->ev)
    if (e) cudaEventDestroy(e);
  for (auto e : b->ev_fork)
    if (e) cudaEventDestroy(e);
  for (auto e : b->ev_adi)
    if (e) cudaEventDestroy(e);
  if (b->ev_diag) cudaEventDestroy(b->ev_diag);
  for (auto s : b->aux)
    if (s) cudaStreamDestroy(s);
  if (b->d_args) cudaFree(b->d_args);
  dev_free(b->ctx, b->d_items);
  for (int k = 0; k < 2; ++k) {
    if (b->h_items[k]) cudaFreeHost(b->h_items[k]);
    if (b->items_copied[k]) cudaEventDestroy(b->items_copied[k]);
  }
  ctx_release(b->ctx);
  delete b;
  return G4B_OK;
}

// Attach a prepared run (created, uploaded, lattice set): it takes part in
// the batch's steps from lattice step `first_step` for `nsteps` steps.
int g4b_batch_attach(g4b_batch* b, g4b_run* r, int first_step, int nsteps, int* slot) {
  if (!b || !r || !slot || nsteps < 0 || first_step < 0)
    return fail(G4B_ERR_ARG, "g4b_batch_attach: bad arg");
  if (r->ctx->device != b->ctx->device)
    return fail(G4B_ERR_ARG, "g4b_batch_attach: run on another device");
  if (r->steps.empty()) return fail(G4B_ERR_STATE, "g4b_batch_attach: run has no lattice");
  for (int f = 0; f < r->nfield; ++f)
    if (r->fs[f].f->precision != G4B_MIXED)
      return fail(G4B_ERR_ARG, "g4b_batch_attach: mixed-precision runs only");
  for (int s = 0; s < b->max_runs; ++s)
    if (b->runs[s] == r) return fail(G4B_ERR_STATE, "g4b_batch_attach: run already attached");
  for (int s = 0; s < b->max_runs; ++s) {
    if (b->runs[s]) continue;
    b->runs[s] = r;
    b->next[s] = first_step;
    b->last[s] = first_step + nsteps;
    b->dirty = true;
    *slot = s;
    return G4B_OK;
  }
  return fail(G4B_ERR_RANGE, "g4b_batch_attach: no free slot");
}

// Detach the run in `slot` (the run itself is not destroyed); later steps
// leave it out.  Steps already enqueued may still use it: destroy it only
// after they completed (a g4b_ctx_mark after its last step).
int g4b_batch_detach(g4b_batch* b, int slot) {
  if (!b || slot < 0 || slot >= b->max_runs || !b->runs[slot])
    return fail(G4B_ERR_ARG, "g4b_batch_detach: bad slot");
  b->runs[slot] = nullptr;
  b->dirty = true;
  return G4B_OK;
}

int g4b_batch_status(g4b_batch* b, int slot, int* next_step, int* remaining) {
  if (!b || slot < 0 || slot >= b->max_runs || !b->runs[slot])
    return fail(G4B_ERR_ARG, "g4b_batch_status: bad slot");
  if (next_step) *next_step = b->next[slot];
  if (remaining) *remaining = std::max(0, b->last[slot] - b->next[slot]);
  return G4B_OK;
}

// Start the tuner: the next 4 batch steps run with candidate launch shapes
// (per kernel: CTAs per SM) and time each kernel; the fastest shape of every
// kernel is kept.  Results do not depend on the shapes.
int g4b_batch_tune(g4b_batch* b) {
  if (!b) return fail(G4B_ERR_ARG, "g4b_batch_tune: null batch");
  b->tune_left = 4;
  b->tune_idx = 0;
  for (auto& v : b->tune_ms) v.assign(4, 0.f);
  return G4B_OK;
}

// The ADI row layouts, then the launch shapes as g4b_batch_tune.  For every
// grid size among the attached runs' fields that has two row layouts (32
// lanes of M elements, 16 lanes of M' elements) and at least
// kTuneRowsMinSlices slices in the batch, both passes are timed in each
// layout on a scratch field of that grid (its slice count up to 128, zeros,
// best of three launches after one untimed), before any step: the runs'
// state never advances in a trial layout, so every step of the batch uses
// the chosen layouts and equals an alone run given the same layouts.
constexpr int kTuneRowsMinSlices = 32;

int g4b_batch_tune_layouts(g4b_batch* b) {
  if (!b) return fail(G4B_ERR_ARG, "g4b_batch_tune_layouts: null batch");
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  struct Group {
    int n = 0, nslice = 0;
    double gridmax = 0, xlambda = 0, delz = 0;
    std::vector<g4b_field*> fields;
  };
  std::vector<Group> groups;
  for (int s = 0; s < b->max_runs; ++s) {
    g4b_run* r = b->runs[s];
    if (!r || b->next[s] >= b->last[s] || r->steps.empty()) continue;
    for (int f = 0; f < r->nfield; ++f) {
      g4b_field* F = r->fs[f].f;
      if (!alt_mode(F->ngrid)) continue;
      Group* g = nullptr;
      for (auto& x : groups)
        if (x.n == F->ngrid) g = &x;
      if (!g) {
        groups.emplace_back();
        g = &groups.back();
        g->n = F->ngrid;
        g->gridmax = F->gridmax;
        g->xlambda = F->xlambda;
        g->delz = r->steps[0].delz > 0 ? r->steps[0].delz : 0.015;
      }
      g->nslice += F->nslice;
      g->fields.push_back(F);
    }
  }
  for (Group& g : groups) {
    // a grid with few slices in the batch keeps its default: its passes are
    // launch-bound, and a switch would add a row-layout group (two more
    // launches per step) to the batch
    if (g.nslice < kTuneRowsMinSlices) continue;
    g4b_field* f = nullptr;
    g4b_adi* adi = nullptr;
    int rc = g4b_field_create(c, std::min(g.nslice, 128), g.n, g.gridmax, g.xlambda, 1,
                              G4B_MIXED, 0, &f);
    if (rc == G4B_OK) rc = g4b_adi_create(c, &adi);
    if (rc == G4B_OK) rc = g4b_adi_init(adi, g.delz, f->dgrid, f->xks, g.n);
    const int modes[2] = {pick_mode(g.n, G4B_MIXED), alt_mode(g.n)};
    float best[2] = {1e30f, 1e30f};
    for (int k = 0; k < 2 && rc == G4B_OK; ++k) {
      rc = field_set_layout(f, modes[k]);
      AdiPlan P;
      if (rc == G4B_OK) rc = adi_plan(adi, f, nullptr, f->desc, nullptr, P);
      for (int it = 0; it < 4 && rc == G4B_OK; ++it) {
        cudaEventRecord(b->ev[0], c->stream);
        rc = adi_launch(f, P);
        cudaEventRecord(b->ev[1], c->stream);
        if (rc == G4B_OK) {
          cudaError_t e = cudaEventSynchronize(b->ev[1]);
          if (e != cudaSuccess) rc = cuda_fail(e, "g4b_batch_tune_layouts");
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
        if (it > 0) best[k] = std::min(best[k], ms);
      }
    }
    if (rc == G4B_OK) rc = read_device_error(c, "g4b_batch_tune_layouts");
    g4b_adi_destroy(adi);
    g4b_field_destroy(f);
    if (rc != G4B_OK) return rc;
    const int pick = best[1] < best[0] ? modes[1] : modes[0];
    for (g4b_field* F : g.fields)
      if (int r2 = field_set_layout(F, pick)) return r2;
  }
  b->dirty = true;
  b->graph_valid = false;
  return g4b_batch_tune(b);
}
int g4b_default_layout(int ngrid) { return pick_mode(ngrid, G4B_MIXED); }

// ADI row layouts of a run's fields: M elements per lane on 32-lane rows, or
// 100 + M on 16-lane rows (two rows per warp).
int g4b_run_get_layouts(g4b_run* r, int* modes) {
  if (!r || !modes) return fail(G4B_ERR_ARG, "g4b_run_get_layouts: null arg");
  for (int f = 0; f < r->nfield; ++f) modes[f] = r->fs[f].f->mode;
  return G4B_OK;
}

// Sets them (each the default or the other layout of the field's grid), e.g.
// to rerun a batch-tuned run alone with the same FP32 rounding.
int g4b_run_set_layouts(g4b_run* r, const int* modes) {
  if (!r || !modes) return fail(G4B_ERR_ARG, "g4b_run_set_layouts: null arg");
  G4B_CUDA_TRY(cudaSetDevice(r->ctx->device));
  for (int f = 0; f < r->nfield; ++f)
    if (int rc = field_set_layout(r->fs[f].f, modes[f])) return rc;
  return G4B_OK;
}

// Launch shapes in use: CTAs of the beam, deposition, ADI and finalize kernels.
int g4b_batch_shapes(g4b_batch* b, int* grids) {
  if (!b || !grids) return fail(G4B_ERR_ARG, "g4b_batch_shapes: null arg");
  for (int k = 0; k < 4; ++k) grids[k] = b->grid[k];
  return G4B_OK;
}

// Advance every attached, unfinished run by `nsteps` lattice steps (runs that
// reach their end drop out).  With use_graph the kernels of a step are
// replayed from a CUDA graph captured for the current composition.
int g4b_batch_step(g4b_batch* b, int nsteps, int use_graph) {
  if (!b || nsteps < 0) return fail(G4B_ERR_ARG, "g4b_batch_step: bad arg");
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  for (int k = 0; k < nsteps; ++k) {
    if (b->dirty)
      if (int rc = batch_rebuild(b)) return rc;
    if (b->counts.fin == 0) return G4B_OK;
    if (int rc = batch_stage(b)) return rc;
    if (b->tune_left > 0) {
      const int sm = c->sm_count, t = b->tune_idx;
      b->grid[0] = kTuneBeam[t] * sm;
      b->grid[1] = kTuneDep[t] * sm;
      b->grid[2] = kTuneAdi[t] * sm;
      if (int rc = batch_launch(b, true)) return rc;
      G4B_CUDA_TRY(cudaEventSynchronize(b->ev[4]));
      for (int q = 0; q < 3; ++q) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev[q], b->ev[q + 1]);
        b->tune_ms[q][t] = ms;
      }
      {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev[3], b->ev[4]);
        b->tune_ms[2][t] += ms;  // both ADI passes
      }
      b->tune_idx++;
      if (--b->tune_left == 0) {
        const int* cand[3] = {kTuneBeam, kTuneDep, kTuneAdi};
        for (int q = 0; q < 3; ++q) {
          int best = 0;
          for (int j = 1; j < 4; ++j)
            if (b->tune_ms[q][j] < b->tune_ms[q][best]) best = j;
          b->grid[q] = cand[q][best] * sm;
        }
        b->graph_valid = false;
      }
    } else if (use_graph && b->stable >= 2) {
      // a graph pays once the composition holds for a few steps
      if (!b->graph_valid) {
        if (b->gexec) cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
        cudaGraph_t g;
        const bool prof = c->prof.on;  // no profiler events inside a graph
        c->prof.on = false;
        G4B_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = batch_launch(b, false);
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        c->prof.on = prof;
        if (rc) return rc;
        if (e != cudaSuccess) return cuda_fail(e, "g4b_batch_step: capture");
        e = cudaGraphInstantiate(&b->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "g4b_batch_step: instantiate");
        b->graph_valid = true;
      }
      G4B_CUDA_TRY(cudaGraphLaunch(b->gexec, c->stream));
    } else {
      if (int rc = batch_launch(b, false)) return rc;
    }
    b->steps_done++;
    b->stable++;
  }
  return G4B_OK;
}

}  // extern "C"
