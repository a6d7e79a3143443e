// g4h_loader.cpp -- beam and field loading for the host layer.
//
// Upstream GENESIS 1.3 v4 loads beams with a Hammersley quiet start plus
// shot noise and seeds fields with a Gaussian mode; the upstream sources are
// not part of the reference tree, so this file writes both from their
// published definitions (see g4h.h).  Deterministic for a given seed.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "g4h.h"
#include "g4h_internal.h"

namespace g4h {

static thread_local std::string t_err;
void set_error(const std::string& m) { t_err = m; }
const char* last_error() { return t_err.c_str(); }

double radical_inverse(uint64_t i, unsigned base) {
  double inv = 1.0 / base, f = inv, r = 0.0;
  while (i) {
    r += f * (double)(i % base);
    i /= base;
    f *= inv;
  }
  return r;
}

// Inverse of the standard normal CDF: rational approximation (P. J. Acklam,
// 2003) followed by one Halley step against erfc, accurate to ~1e-15.
double inv_normal(double p) {
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
    const double q = std::sqrt(-2 * std::log(p));
    x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
  } else if (p <= phigh) {
    const double q = p - 0.5, r = q * q;
    x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
        (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1);
  } else {
    const double q = std::sqrt(-2 * std::log(1 - p));
    x = -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
  }
  const double e = 0.5 * std::erfc(-x / std::sqrt(2.0)) - p;
  const double u = e * std::sqrt(2 * M_PI) * std::exp(x * x / 2);
  return x - u / (1 + x * u / 2);
}

// SplitMix64 seeded stream; uniform in (0, 1).
double Rng::uniform() {
  s += 0x9e3779b97f4a7c15ull;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

double Rng::normal() {
  const double u1 = uniform(), u2 = uniform();
  return std::sqrt(-2 * std::log(u1)) * std::cos(2 * M_PI * u2);
}

}  // namespace g4h

using namespace g4h;

extern "C" {

const char* g4h_last_error(void) { return last_error(); }

int g4h_load_beam(const g4h_beam_spec* sp, const double* current, double* x, double* y,
                  double* px, double* py, double* gamma, double* theta, int64_t* off) {
  if (!sp || !current || !x || !y || !px || !py || !gamma || !theta || !off) {
    set_error("g4h_load_beam: null argument");
    return G4B_ERR_ARG;
  }
  if (sp->nslice <= 0 || sp->npart < 0 || sp->nbins <= 0 || sp->npart % sp->nbins) {
    set_error("g4h_load_beam: npart must be a multiple of nbins");
    return G4B_ERR_ARG;
  }
  const int nbl = sp->npart / sp->nbins;  // beamlets per slice
  const double gref = sp->gamma0;
  const double epx = sp->ex / gref, epy = sp->ey / gref;  // geometric
  const double sx = std::sqrt(epx * sp->betax), sy = std::sqrt(epy * sp->betay);
  const double spx = std::sqrt(epx / sp->betax), spy = std::sqrt(epy / sp->betay);
  const double twopi = 2 * M_PI;
  const double ce = 1.602176634e-19, c0 = 299792458.0;
  off[0] = 0;
  for (int s = 0; s < sp->nslice; ++s) {
    Rng rng{sp->seed * 0x100000001b3ull + (uint64_t)s * 0x9e3779b97f4a7c15ull + 1};
    const int64_t base = (int64_t)s * sp->npart;
    // electrons per beamlet for the shot-noise amplitude
    const double ne = current[s] * sp->slicelength / (ce * c0) / std::max(nbl, 1);
    for (int j = 0; j < nbl; ++j) {
      const uint64_t idx = (uint64_t)s * nbl + j + 1;
      const double g1 = inv_normal(radical_inverse(idx, 2));
      const double g2 = inv_normal(radical_inverse(idx, 3));
      const double g3 = inv_normal(radical_inverse(idx, 5));
      const double g4 = inv_normal(radical_inverse(idx, 7));
      const double g5 = inv_normal(radical_inverse(idx, 11));
      const double th0 = twopi / sp->nbins * radical_inverse(idx, 13);
      const double xv = sx * g1 + sp->xcenter;
      const double yv = sy * g3 + sp->ycenter;
      const double xp = spx * (g2 - sp->alphax * g1);
      const double yp = spy * (g4 - sp->alphay * g3);
      const double gv = gref + sp->delgam * g5;
      // momenta are gamma * angle
      const double pxv = gv * xp + sp->pxcenter;
      const double pyv = gv * yp + sp->pycenter;
      // shot noise: delta theta = sum_h a_h cos(h th) + b_h sin(h th),
      // a_h, b_h ~ N(0, 2/(ne h^2)) gives <|b_h|^2> = 1/ne for h < nbins/2
      double an[64], bn[64];
      const int nh = sp->nbins / 2;
      for (int h = 1; h <= nh && h <= 64; ++h) {
        const double sig = (sp->shotnoise && ne > 0) ? std::sqrt(2.0 / ne) / h : 0.0;
        an[h - 1] = sig * rng.normal();
        bn[h - 1] = sig * rng.normal();
      }
      for (int k = 0; k < sp->nbins; ++k) {
        const int64_t p = base + (int64_t)j * sp->nbins + k;
        double th = th0 + twopi * k / sp->nbins;
        double dth = 0.0;
        for (int h = 1; h <= nh && h <= 64; ++h)
          dth += an[h - 1] * std::cos(h * th) + bn[h - 1] * std::sin(h * th);
        x[p] = xv;
        y[p] = yv;
        px[p] = pxv;
        py[p] = pyv;
        gamma[p] = gv;
        theta[p] = th + dth;
      }
    }
    off[s + 1] = base + sp->npart;
  }
  return G4B_OK;
}

int g4h_gaussian_field(int ngrid, double gridmax, double xlambda, double power, double w0,
                       double* cells) {
  if (ngrid < 2 || !(gridmax > 0) || !(xlambda > 0) || !cells || power < 0) {
    set_error("g4h_gaussian_field: bad argument");
    return G4B_ERR_ARG;
  }
  const double dgrid = 2 * gridmax / (ngrid - 1);
  const double ks = 2 * M_PI / xlambda;
  const double eev = 510998.95, vacimp = 376.73031346177;
  double sum = 0.0;
  for (int iy = 0; iy < ngrid; ++iy)
    for (int ix = 0; ix < ngrid; ++ix) {
      const double xv = -gridmax + ix * dgrid, yv = -gridmax + iy * dgrid;
      const double g = std::exp(-(xv * xv + yv * yv) / (w0 * w0));
      cells[2 * ((size_t)iy * ngrid + ix)] = g;
      cells[2 * ((size_t)iy * ngrid + ix) + 1] = 0.0;
      sum += g * g;
    }
  const double unit = dgrid * eev / ks;
  const double amp = (power > 0 && sum > 0) ? std::sqrt(power * vacimp / (unit * unit * sum)) : 0.0;
  for (size_t i = 0; i < (size_t)ngrid * ngrid; ++i) cells[2 * i] *= amp;
  return G4B_OK;
}

}  // extern "C"
