// g4b_incoherent.cu -- incoherent synchrotron radiation of an undulator step.
//
// The reference applies it on the host after the push, through upstream
// GENESIS 1.3 v4's Incoherent::apply on the host particle copies
// (src/Core/Beam.cpp:126), which in its CUDA path are stale: the push has
// already moved the device state.  Here it acts on the device state.
//
// Model (published rates of spontaneous undulator radiation; Saldin,
// Schneidmiller and Yurkov, NIM A 381 (1996) 545), per particle of energy
// gamma in an undulator of wavenumber k_u and rms parameter aw:
//   mean loss     d gamma/dz       = -(2/3) r_e k_u^2 aw^2 gamma^2
//   spread growth d <dgamma^2>/dz  = (14/15) lambdabar_c r_e k_u^3 K^2 F(K) gamma^4
//   planar  K = sqrt(2) aw, F(K) = 1.42 K + 1/(1 + 1.5 K + 0.95 K^2)
//   helical K = aw,         F(K) = 1.70 K + 1/(1 + 1.88 K + 0.80 K^2)
// Over a step delz: gamma -= loss delz gamma^2 and gamma += sqrt(spread delz)
// gamma^2 z with z ~ N(0, 1), both from the particle's energy before the step.
// z comes from a counter-based generator (Philox4x32-10, Salmon et al., SC
// 2011) keyed by the seed, counting (particle index, step counter), and the
// Box-Muller transform: the noise of a particle does not depend on the
// launch shape or on the other particles.

#include <cmath>

#include "g4b_internal.cuh"

namespace g4b {
namespace {

constexpr double kRe = 2.8179403262e-15;        // classical electron radius [m]
constexpr double kLambdaC = 3.8615926796e-13;   // reduced Compton wavelength [m]

struct IsrArgs {
  double* gamma;
  int64_t n;
  double loss, sigma;  // loss rate x delz / gamma^2; sqrt(spread rate x delz) / gamma^2
  uint32_t key0, key1, ctr0, ctr1;
};

__device__ __forceinline__ void philox_round(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
  const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
  const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
  const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
  c[0] = n0;
  c[1] = lo1;
  c[2] = n2;
  c[3] = lo0;
}

__device__ __forceinline__ void philox4x32_10(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    philox_round(c, k0, k1);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// a uniform in (0, 1) from two 32-bit words: 27 + 26 bits, centred
__device__ __forceinline__ double unit53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}

__global__ void __launch_bounds__(256) isr_kernel(const IsrArgs a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    const double g = a.gamma[i];
    const double g2 = g * g;
    double dg = -a.loss * g2;
    if (a.sigma > 0.0) {
      uint32_t c[4] = {(uint32_t)i, (uint32_t)((uint64_t)i >> 32), a.ctr0, a.ctr1};
      philox4x32_10(c, a.key0, a.key1);
      const double u = unit53(c[0], c[1]), v = unit53(c[2], c[3]);
      const double z = sqrt(-2.0 * log(u)) * cos(6.283185307179586 * v);
      dg += a.sigma * g2 * z;
    }
    a.gamma[i] = g + dg;
  }
}

}  // namespace
}  // namespace g4b

using namespace g4b;

extern "C" {

int g4b_isr_rates(double aw, double ku, int helical, double* loss, double* spread) {
  if (!loss || !spread) return fail(G4B_ERR_ARG, "g4b_isr_rates: null arg");
  *loss = 0.0;
  *spread = 0.0;
  if (!(aw > 0.0) || !(ku > 0.0)) return G4B_OK;
  const double K = helical ? aw : std::sqrt(2.0) * aw;
  const double F = helical ? 1.70 * K + 1.0 / (1.0 + 1.88 * K + 0.80 * K * K)
                           : 1.42 * K + 1.0 / (1.0 + 1.5 * K + 0.95 * K * K);
  *loss = 2.0 / 3.0 * kRe * ku * ku * aw * aw;
  *spread = 14.0 / 15.0 * kLambdaC * kRe * ku * ku * ku * K * K * F;
  return G4B_OK;
}

int g4b_beam_incoherent(g4b_beam* b, const g4b_step* st, double delz, int helical,
                        int do_loss, int do_spread, uint64_t seed, uint64_t counter) {
  if (!b || !st) return fail(G4B_ERR_ARG, "g4b_beam_incoherent: null arg");
  if (b->precision != G4B_FP64)
    return fail(G4B_ERR_ARG, "g4b_beam_incoherent: FP64 beam expected");
  if (!st->in_undulator || b->npart == 0 || (!do_loss && !do_spread)) return G4B_OK;
  double loss = 0.0, spread = 0.0;
  g4b_isr_rates(st->aw, st->ku, helical, &loss, &spread);
  if (loss == 0.0 && spread == 0.0) return G4B_OK;
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  IsrArgs a{};
  a.gamma = b->gamma;
  a.n = b->npart;
  a.loss = do_loss ? loss * delz : 0.0;
  a.sigma = do_spread ? std::sqrt(spread * delz) : 0.0;
  a.key0 = (uint32_t)seed;
  a.key1 = (uint32_t)(seed >> 32);
  a.ctr0 = (uint32_t)counter;
  a.ctr1 = (uint32_t)(counter >> 32);
  const int64_t want = (b->npart + 255) / 256;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, c->sm_count * 16));
  {
    LaunchScope ls(c, "incoherent");
    isr_kernel<<<grid, 256, 0, c->stream>>>(a);
  }
  return check_launch(c, "isr_kernel");
}

}  // extern "C"
