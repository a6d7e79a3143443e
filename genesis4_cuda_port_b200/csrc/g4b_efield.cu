// g4b_efield.cu -- short-range longitudinal space charge on the device.
//
// The reference keeps the space-charge solver on the host: with short-range
// space charge on, BeamSolverCUDA::advance calls EFieldSolver::shortRange for
// every slice on the host particle copies and uploads a per-particle field
// (getEField(ip) + slice loss) that the push reads in place of the slice loss
// (src/Core/BeamSolverCUDA.cpp:523-547, 184-195, 633-680).  Here the whole
// step stays on the device: one CTA per slice builds the slice's azimuthal
// and longitudinal density modes on a radial grid, solves one tridiagonal
// system per mode and writes every particle's field into the beam's
// per-particle buffer, which the push then reads.
//
// Model (per slice, particles i = 1..N, current I):
//   density modulation at harmonic l of the reference wavelength, azimuthal
//   order m:  S_lm(r) = (1/N) sum_i delta(r - r_i) e^{-i(l theta_i + m phi_i)}
//   (radial cell average),
//   (1/r d/dr r d/dr - m^2/r^2 - kappa_l^2) u_lm = -S_lm,  kappa_l = l k_s / gamma_z,
//   u = 0 on the wall r = R, R = rmax * (largest particle radius about the
//   slice centroid),
//   E_z = sum_{l>=1} 2 Re[ i l k_s I Z0 / gamma_z^2 u_l e^{i l theta} ]
//   (the quasi-static field of a modulation moving with the beam), and the
//   push's loss term ez = E_z / (m_e c^2 / e) + slice loss.
// Discretisation: N radial cells of width dr = R/N, centres (j+1/2) dr,
// finite-volume fluxes through the cell faces, the wall half a cell beyond
// the last centre.  Mode sums are exact 2^-40 fixed-point integers (shared
// 64-bit atomics), so the result does not depend on particle order.

#include <algorithm>
#include <cmath>
#include <new>

#include "g4b_internal.cuh"

namespace g4b {
namespace {

constexpr int kScThreads = 256;
constexpr double kScFix = 1099511627776.0;  // 2^40
constexpr double kScUnfix = 1.0 / 1099511627776.0;
constexpr int64_t kScMaxSliceNp = int64_t(1) << 22;  // |mode sum| < 2^62
constexpr double kVacImp = 376.73031346177;   // Z0 [Ohm]
constexpr double kEev = 510998.95;            // m_e c^2 / e [V]

struct ScArgs {
  const double *x, *y, *theta;
  const int64_t* off;
  const double* current;  // [A] per slice
  const double* eloss;    // per-slice loss the push would otherwise use
  double* pez;            // out: per-particle loss
  int nslice, ngrid, nz, nphi, nmode;
  double rmax, ks, gammaz2, coef;  // coef = -2 Z0 k_s / (eev gamma_z^2)
};

__device__ __forceinline__ double block_sum_max(double v, double* sh, bool is_max) {
  // fixed order: warp xor tree, then one thread over the warp partials
  for (int o = 16; o > 0; o >>= 1) {
    const double t = __shfl_xor_sync(0xffffffffu, v, o);
    v = is_max ? fmax(v, t) : v + t;
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = sh[0];
  for (int i = 1; i < (int)(blockDim.x >> 5); ++i) r = is_max ? fmax(r, sh[i]) : r + sh[i];
  return r;
}

__device__ __forceinline__ void fix_add(unsigned long long* acc, double re, double im) {
  atomicAdd(acc, (unsigned long long)__double2ll_rn(re * kScFix));
  atomicAdd(acc + 1, (unsigned long long)__double2ll_rn(im * kScFix));
}

__global__ void __launch_bounds__(kScThreads) short_range_kernel(const ScArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double shd[kScThreads / 32];
  const int n = a.ngrid, nmode = a.nmode, nm = 2 * a.nphi + 1;
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(smem);  // [mode][cell][2]
  double2* u = reinterpret_cast<double2*>(acc + 2 * (size_t)nmode * n);   // [mode][cell]
  double* cp = reinterpret_cast<double*>(u + (size_t)nmode * n);          // Thomas c'
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int s = blockIdx.x; s < a.nslice; s += gridDim.x) {
    const int64_t p0 = a.off[s], p1 = a.off[s + 1], np = p1 - p0;
    if (np <= 0) continue;  // uniform across the CTA
    const double eloss = a.eloss[s], cur = a.current[s];
    double sx = 0.0, sy = 0.0;
    for (int64_t p = p0 + tid; p < p1; p += nt) {
      sx += a.x[p];
      sy += a.y[p];
    }
    sx = block_sum_max(sx, shd, false);
    sy = block_sum_max(sy, shd, false);
    const double xc = sx / (double)np, yc = sy / (double)np;
    double r2 = 0.0;
    for (int64_t p = p0 + tid; p < p1; p += nt) {
      const double dx = a.x[p] - xc, dy = a.y[p] - yc;
      r2 = fmax(r2, dx * dx + dy * dy);
    }
    r2 = block_sum_max(r2, shd, true);
    const double R = a.rmax * sqrt(r2);
    if (!(R > 0.0) || cur == 0.0) {
      for (int64_t p = p0 + tid; p < p1; p += nt) a.pez[p] = eloss;
      continue;
    }
    const double dr = R / (double)n;
    for (int i = tid; i < 2 * nmode * n; i += nt) acc[i] = 0ull;
    __syncthreads();
    for (int64_t p = p0 + tid; p < p1; p += nt) {
      const double dx = a.x[p] - xc, dy = a.y[p] - yc;
      const double r = sqrt(dx * dx + dy * dy);
      const double q = r / dr;  // NaN or beyond the wall: the last cell
      const int j = q >= 0.0 && q < (double)n ? (int)q : n - 1;
      const double cph = r > 0.0 ? dx / r : 1.0, sph = r > 0.0 ? dy / r : 0.0;
      const double th = a.theta[p];
      for (int l = 1; l <= a.nz; ++l) {
        double sl, cl;
        sincos((double)l * th, &sl, &cl);
        unsigned long long* base = acc + 2 * ((size_t)(l - 1) * nm + a.nphi) * n;
        fix_add(base + 2 * j, cl, -sl);  // m = 0: e^{-i l theta}
        double pr = cl, pi = -sl, qr = cl, qi = -sl;
        for (int m = 1; m <= a.nphi; ++m) {
          // e^{-i(l theta + m phi)} and e^{-i(l theta - m phi)}
          const double tr = pr * cph + pi * sph, ti = pi * cph - pr * sph;
          const double ur = qr * cph - qi * sph, ui = qi * cph + qr * sph;
          pr = tr;
          pi = ti;
          qr = ur;
          qi = ui;
          fix_add(base + 2 * ((size_t)m * n + j), pr, pi);
          fix_add(base - 2 * ((size_t)m * n) + 2 * j, qr, qi);
        }
      }
    }
    __syncthreads();
    // one tridiagonal solve per mode (Thomas, FP64), in cell units of dr
    for (int t = tid; t < nmode; t += nt) {
      const int l = t / nm + 1, m = t % nm - a.nphi;
      const double kdr = (double)l * a.ks * dr;
      const double k2 = kdr * kdr / a.gammaz2;
      const double rs = -kScUnfix / (6.283185307179586 * (double)np);
      double2* ut = u + (size_t)t * n;
      double* ct = cp + (size_t)t * n;
      const unsigned long long* at = acc + 2 * (size_t)t * n;
      double prev_c = 0.0, prev_dr = 0.0, prev_di = 0.0;
      for (int j = 0; j < n; ++j) {
        const double rc = (double)j + 0.5;
        const double lo = (double)j, up = (double)(j + 1);
        const double diag = -lo - (j == n - 1 ? 2.0 * up : up) -
                            ((double)(m * m) / (rc * rc) + k2) * rc;
        const double bre = rs * (double)(long long)at[2 * j];
        const double bim = rs * (double)(long long)at[2 * j + 1];
        const double den = diag - lo * prev_c;
        prev_c = j < n - 1 ? up / den : 0.0;
        prev_dr = (bre - lo * prev_dr) / den;
        prev_di = (bim - lo * prev_di) / den;
        ct[j] = prev_c;
        ut[j] = make_double2(prev_dr, prev_di);
      }
      for (int j = n - 2; j >= 0; --j) {
        const double2 nx = ut[j + 1];
        ut[j].x -= ct[j] * nx.x;
        ut[j].y -= ct[j] * nx.y;
      }
    }
    __syncthreads();
    const double scale = a.coef * cur;
    for (int64_t p = p0 + tid; p < p1; p += nt) {
      const double dx = a.x[p] - xc, dy = a.y[p] - yc;
      const double r = sqrt(dx * dx + dy * dy);
      const double q = r / dr;  // NaN or beyond the wall: the last cell
      const int j = q >= 0.0 && q < (double)n ? (int)q : n - 1;
      const double cph = r > 0.0 ? dx / r : 1.0, sph = r > 0.0 ? dy / r : 0.0;
      const double th = a.theta[p];
      double sum = 0.0;
      for (int l = 1; l <= a.nz; ++l) {
        double sl, cl;
        sincos((double)l * th, &sl, &cl);
        const double2* base = u + ((size_t)(l - 1) * nm + a.nphi) * n;
        // Im[u_lm e^{i(l theta + m phi)}]
        double2 c = base[j];
        double im = c.x * sl + c.y * cl;
        double pr = cl, pi = sl, qr = cl, qi = sl;
        for (int m = 1; m <= a.nphi; ++m) {
          const double tr = pr * cph - pi * sph, ti = pi * cph + pr * sph;
          const double ur = qr * cph + qi * sph, ui = qi * cph - qr * sph;
          pr = tr;
          pi = ti;
          qr = ur;
          qi = ui;
          c = base[(size_t)m * n + j];
          im += c.x * pi + c.y * pr;
          c = base[j - (ptrdiff_t)m * n];
          im += c.x * qi + c.y * qr;
        }
        sum += (double)l * im;
      }
      a.pez[p] = eloss + scale * sum;
    }
    __syncthreads();  // the next slice reuses the shared arrays
  }
}

}  // namespace
}  // namespace g4b

using namespace g4b;

struct g4b_efield {
  g4b_ctx* ctx = nullptr;
  double rmax = 0, lambda = 0, ks = 0;
  int ngrid = 0, nz = 0, nphi = 0;
  size_t smem = 0;
};

namespace {
int ensure_pez(g4b_beam* b) {
  if (b->d_pez) return G4B_OK;
  G4B_CUDA_TRY(dev_alloc(b->ctx, (void**)&b->d_pez,
                         (size_t)std::max<int64_t>(1, b->npart) * sizeof(double)));
  b->bytes += (uint64_t)std::max<int64_t>(1, b->npart) * sizeof(double);
  return G4B_OK;
}
}  // namespace

extern "C" {

int g4b_efield_create(g4b_ctx* c, double rmax, int ngrid, int nz, int nphi, double lambda,
                      g4b_efield** out) {
  if (!c || !out) return fail(G4B_ERR_ARG, "g4b_efield_create: null arg");
  if (ngrid < 0 || nz < 0 || nphi < 0 || !(lambda > 0.0) || !(rmax >= 0.0))
    return fail(G4B_ERR_ARG, "g4b_efield_create: bad parameters");
  const size_t nmode = (size_t)nz * (2 * nphi + 1);
  const size_t smem = nmode * (size_t)ngrid * (16 + 16 + 8);
  if (smem > 200u * 1024u)
    return fail(G4B_ERR_RANGE, "g4b_efield_create: nz*(2*nphi+1)*ngrid above 5120");
  g4b_efield* e = new (std::nothrow) g4b_efield();
  if (!e) return fail(G4B_ERR_NOMEM, "g4b_efield_create: host allocation");
  e->ctx = c;
  ctx_retain(c);
  e->rmax = rmax;
  e->ngrid = ngrid;
  e->nz = nz;
  e->nphi = nphi;
  e->lambda = lambda;
  e->ks = 4.0 * std::asin(1.0) / lambda;
  e->smem = smem;
  *out = e;
  return G4B_OK;
}

int g4b_efield_destroy(g4b_efield* e) {
  if (!e) return G4B_OK;
  ctx_release(e->ctx);
  delete e;
  return G4B_OK;
}

int g4b_efield_has_short_range(const g4b_efield* e) {
  return e && e->nz > 0 && e->ngrid > 0 && e->rmax > 0.0 ? 1 : 0;
}

int g4b_efield_short_range(g4b_efield* e, g4b_beam* b, double gammaz2) {
  if (!e || !b) return fail(G4B_ERR_ARG, "g4b_efield_short_range: null arg");
  if (b->precision != G4B_FP64)
    return fail(G4B_ERR_ARG, "g4b_efield_short_range: FP64 beam expected");
  if (b->ctx != e->ctx) return fail(G4B_ERR_ARG, "g4b_efield_short_range: contexts differ");
  if (!(gammaz2 > 0.0)) return fail(G4B_ERR_ARG, "g4b_efield_short_range: gammaz2 <= 0");
  if (!g4b_efield_has_short_range(e)) return G4B_OK;
  if (b->max_slice_np > kScMaxSliceNp)
    return fail(G4B_ERR_RANGE, "g4b_efield_short_range: more than 2^22 particles in a slice");
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  if (int rc = ensure_pez(b)) return rc;
  b->use_pez = 1;
  if (b->npart == 0) return G4B_OK;
  ScArgs a{};
  a.x = b->x;
  a.y = b->y;
  a.theta = b->theta;
  a.off = b->d_off;
  a.current = b->d_current;
  a.eloss = b->d_eloss;
  a.pez = b->d_pez;
  a.nslice = b->nslice;
  a.ngrid = e->ngrid;
  a.nz = e->nz;
  a.nphi = e->nphi;
  a.nmode = e->nz * (2 * e->nphi + 1);
  a.rmax = e->rmax;
  a.ks = e->ks;
  a.gammaz2 = gammaz2;
  a.coef = -2.0 * kVacImp * e->ks / (kEev * gammaz2);
  G4B_CUDA_TRY(cudaFuncSetAttribute(short_range_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)e->smem));
  const unsigned grid = (unsigned)std::max(1, std::min(b->nslice, c->sm_count * 8));
  {
    LaunchScope ls(c, "short_range");
    short_range_kernel<<<grid, kScThreads, e->smem, c->stream>>>(a);
  }
  return check_launch(c, "short_range_kernel");
}

int g4b_beam_set_particle_ez(g4b_beam* b, const double* ez) {
  if (!b) return fail(G4B_ERR_ARG, "g4b_beam_set_particle_ez: null beam");
  if (b->precision != G4B_FP64)
    return fail(G4B_ERR_ARG, "g4b_beam_set_particle_ez: FP64 beam expected");
  if (!ez) {
    b->use_pez = 0;
    return G4B_OK;
  }
  G4B_CUDA_TRY(cudaSetDevice(b->ctx->device));
  if (int rc = ensure_pez(b)) return rc;
  if (b->npart > 0) {
    G4B_CUDA_TRY(cudaMemcpyAsync(b->d_pez, ez, (size_t)b->npart * sizeof(double),
                                 cudaMemcpyHostToDevice, b->ctx->stream));
    G4B_CUDA_TRY(cudaStreamSynchronize(b->ctx->stream));
  }
  b->use_pez = 1;
  return G4B_OK;
}

int g4b_beam_get_particle_ez(g4b_beam* b, double* ez) {
  if (!b || !ez) return fail(G4B_ERR_ARG, "g4b_beam_get_particle_ez: null arg");
  if (!b->use_pez) return fail(G4B_ERR_STATE, "g4b_beam_get_particle_ez: no per-particle field");
  G4B_CUDA_TRY(cudaSetDevice(b->ctx->device));
  if (b->npart > 0) {
    G4B_CUDA_TRY(cudaMemcpyAsync(ez, b->d_pez, (size_t)b->npart * sizeof(double),
                                 cudaMemcpyDeviceToHost, b->ctx->stream));
  }
  G4B_CUDA_TRY(cudaStreamSynchronize(b->ctx->stream));
  return read_device_error(b->ctx, "g4b_beam_get_particle_ez");
}

}  // extern "C"
