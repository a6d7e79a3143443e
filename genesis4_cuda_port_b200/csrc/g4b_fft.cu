// g4b_fft.cu -- the spectral field solver (FieldSolverFFTCUDA,
// src/Core/FieldSolverFFTCUDA.cpp:157-483) for sm_100a, with its 2-D
// transforms written here (no cuFFT).
//
// One field step u' = IFFT2( FFT2(u) exp(i k2 dz) + 2 filter FFT2(S) ) / n^2:
//
//   deposition : the deterministic FP64 source of the ADI solver (compact
//                per-slice tiles; src/Core/FieldSolverFFTCUDA.cpp:77-155 is the
//                same arithmetic as the ADI deposition);
//   pass A     : each warp transforms one row of a slice along x; the CTA's
//                eight rows leave transposed ([slice][kx][ky]) so that pass B
//                reads contiguous lines; with the source filter on, the source
//                rows are transformed beside them;
//   pass B     : each warp takes one kx line of the transposed spectrum,
//                transforms it along y, multiplies by the propagator
//                exp(i k2 dz) (adding 2 filter S^ when filtered), transforms it
//                back along y and stores it in place;
//   pass C     : the CTA gathers eight ky lines back from the transposed layout;
//                each warp transforms its row back along x, scales by 1/n^2,
//                adds 2 S (unfiltered: the inverse transform of 2 S^ is 2 S)
//                and writes the natural layout.
//
// A line of any length n <= 256 is transformed by Bluestein's chirp-z
// algorithm: with w_j = exp(-i pi j^2 / n), DFT_n(x)_k = w_k (a * h)_k, a_j =
// x_j w_j, h_t = conj(w_t), a circular convolution of length 512 >= 2n - 1
// done as FFT_512 -> multiply by the precomputed FFT_512(h) -> inverse FFT.
// The 512-point FFT lives in one warp: lane l holds x[32 r + l] in register
// r (r < 16).  With j = j0 + 8 j1 + 64 j2 and k = k0 + 8 k1 + 64 k2 it is
// three radix-8 stages (decimation in frequency):
//   A: per (j0, j1) an 8-point DFT over j2 -> k0, times W_512^((j0 + 8 j1) k0);
//   B: per (j0, k0) an 8-point DFT over j1 -> k1, times W_64^(j0 k1);
//   C: per (k1, k0) an 8-point DFT over j0 -> k2.
// Each lane holds two groups of eight (registers 2 s + b), so every stage
// runs in registers; between stages the warp regroups its 512 values through
// a private shared-memory buffer (rows of nine entries: no bank conflicts),
// two exchanges in place of the five shuffle rounds of a cross-lane radix-2
// form.  The output is in the permuted order (lane l, register 2 s + b) ->
// k0 + 8 k1 + 64 k2 with q = l + 32 b, k0 = q / 8, k1 = q % 8, k2 = brev3(s),
// which only the pointwise multiply sees; the inverse runs the stages back
// (decimation in time, conjugate twiddles) and returns natural order.
#include <algorithm>
#include <cmath>
#include <complex>
#include <new>
#include <vector>

#include "g4b_internal.cuh"

namespace g4b {
namespace {

constexpr int kFftM = 512;       // Bluestein length
constexpr int kFftMaxN = 256;    // 2 n - 1 <= 512
constexpr int kFftWarps = 8;     // lines per CTA
constexpr int kFftPitch = kFftWarps + 1;  // transposition tile pitch (odd: no bank conflicts)

struct FftArgs {
  const double2* tw;      // W_512^j, j < 512
  const double2* chirp;   // w_j, j < n
  const double2* hf;      // FFT_512(conj w) / 512, permuted order (lane * 16 + r)
  const double2* hi;      // FFT_512(w) / 512, permuted order
  const double2* prop_t;  // exp(i k2 dz), [kx][ky]
  const double* sig_t;    // source filter, [kx][ky] (filtered runs)
  const double2* u;       // field, [slice][iy][ld]
  double2* out;           // pass C: field written back
  double2* T;             // spectrum, [slice][kx][ld]
  double2* ST;            // source spectrum, [slice][kx][ld] (filtered runs)
  const double2* src;     // compact source tiles
  const int4* desc;       // per-slice tile (x0, y0, width, height)
  size_t src_cap;
  int n, ld, nband;
  double scale;           // 1 / n^2
};

__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ double2 zmulc(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__host__ __device__ constexpr int brev3(int k) { return ((k & 1) << 2) | (k & 2) | ((k & 4) >> 2); }

constexpr int kXbRow = 9;              // padded row of eight
constexpr int kXb = 8 * 8 * kXbRow;    // exchange buffer per warp (double2)
constexpr double kS = 0.70710678118654752440;

__device__ __forceinline__ double2 mul_w1(double2 z) {  // x (1 - i)/sqrt2
  return make_double2(kS * (z.x + z.y), kS * (z.y - z.x));
}
__device__ __forceinline__ double2 mul_w2(double2 z) { return make_double2(z.y, -z.x); }  // x (-i)
__device__ __forceinline__ double2 mul_w3(double2 z) {  // x (-1 - i)/sqrt2
  return make_double2(kS * (z.y - z.x), -kS * (z.x + z.y));
}
__device__ __forceinline__ double2 mul_c1(double2 z) {  // x (1 + i)/sqrt2
  return make_double2(kS * (z.x - z.y), kS * (z.x + z.y));
}
__device__ __forceinline__ double2 mul_c2(double2 z) { return make_double2(-z.y, z.x); }  // x i
__device__ __forceinline__ double2 mul_c3(double2 z) {  // x (-1 + i)/sqrt2
  return make_double2(-kS * (z.x + z.y), kS * (z.x - z.y));
}

// 8-point DFT of v[2 s + B], s = 0..7 (radix-2, decimation in frequency):
// X[k] lands in slot brev3(k).
template <int B>
__device__ __forceinline__ void dft8(double2 (&v)[16]) {
#define G4B_A(s) v[2 * (s) + B]
  {
    double2 x = G4B_A(0), y = G4B_A(4);
    G4B_A(0) = zadd(x, y);
    G4B_A(4) = zsub(x, y);
    x = G4B_A(1), y = G4B_A(5);
    G4B_A(1) = zadd(x, y);
    G4B_A(5) = mul_w1(zsub(x, y));
    x = G4B_A(2), y = G4B_A(6);
    G4B_A(2) = zadd(x, y);
    G4B_A(6) = mul_w2(zsub(x, y));
    x = G4B_A(3), y = G4B_A(7);
    G4B_A(3) = zadd(x, y);
    G4B_A(7) = mul_w3(zsub(x, y));
  }
#pragma unroll
  for (int blk = 0; blk < 8; blk += 4) {
    double2 x = G4B_A(blk), y = G4B_A(blk + 2);
    G4B_A(blk) = zadd(x, y);
    G4B_A(blk + 2) = zsub(x, y);
    x = G4B_A(blk + 1), y = G4B_A(blk + 3);
    G4B_A(blk + 1) = zadd(x, y);
    G4B_A(blk + 3) = mul_w2(zsub(x, y));
  }
#pragma unroll
  for (int blk = 0; blk < 8; blk += 2) {
    const double2 x = G4B_A(blk), y = G4B_A(blk + 1);
    G4B_A(blk) = zadd(x, y);
    G4B_A(blk + 1) = zsub(x, y);
  }
}

// Unnormalised inverse of dft8 (decimation in time, conjugate twiddles):
// input in its output order, x[j] in slot j.
template <int B>
__device__ __forceinline__ void idft8(double2 (&v)[16]) {
#pragma unroll
  for (int blk = 0; blk < 8; blk += 2) {
    const double2 x = G4B_A(blk), y = G4B_A(blk + 1);
    G4B_A(blk) = zadd(x, y);
    G4B_A(blk + 1) = zsub(x, y);
  }
#pragma unroll
  for (int blk = 0; blk < 8; blk += 4) {
    double2 x = G4B_A(blk), y = G4B_A(blk + 2);
    G4B_A(blk) = zadd(x, y);
    G4B_A(blk + 2) = zsub(x, y);
    x = G4B_A(blk + 1), y = mul_c2(G4B_A(blk + 3));
    G4B_A(blk + 1) = zadd(x, y);
    G4B_A(blk + 3) = zsub(x, y);
  }
  {
    double2 x = G4B_A(0), y = G4B_A(4);
    G4B_A(0) = zadd(x, y);
    G4B_A(4) = zsub(x, y);
    x = G4B_A(1), y = mul_c1(G4B_A(5));
    G4B_A(1) = zadd(x, y);
    G4B_A(5) = zsub(x, y);
    x = G4B_A(2), y = mul_c2(G4B_A(6));
    G4B_A(2) = zadd(x, y);
    G4B_A(6) = zsub(x, y);
    x = G4B_A(3), y = mul_c3(G4B_A(7));
    G4B_A(3) = zadd(x, y);
    G4B_A(7) = zsub(x, y);
  }
#undef G4B_A
}

// Multiplies slot s of group B by W^(e k), k = brev3(s), e given by the
// table entries w1 = W^e, w2 = W^(2e), w4 = W^(4e) (CONJ: by the conjugates).
template <bool CONJ>
__device__ __forceinline__ double2 tmul(double2 z, double2 w) { return CONJ ? zmulc(z, w) : zmul(z, w); }
// slot s holds k = brev3(s): 1 -> 4, 2 -> 2, 3 -> 6, 4 -> 1, 5 -> 5, 6 -> 3, 7 -> 7
template <int B, bool CONJ>
__device__ __forceinline__ void twiddle8(double2 (&v)[16], double2 w1, double2 w2, double2 w4) {
  v[2 * 4 + B] = tmul<CONJ>(v[2 * 4 + B], w1);
  v[2 * 2 + B] = tmul<CONJ>(v[2 * 2 + B], w2);
  v[2 * 1 + B] = tmul<CONJ>(v[2 * 1 + B], w4);
  double2 w = zmul(w2, w1);  // k = 3
  v[2 * 6 + B] = tmul<CONJ>(v[2 * 6 + B], w);
  w = zmul(w4, w1);  // k = 5
  v[2 * 5 + B] = tmul<CONJ>(v[2 * 5 + B], w);
  w = zmul(w4, w2);  // k = 6
  v[2 * 3 + B] = tmul<CONJ>(v[2 * 3 + B], w);
  w = zmul(w, w1);  // k = 7
  v[2 * 7 + B] = tmul<CONJ>(v[2 * 7 + B], w);
}

// Forward 512-point DFT (exp(-2 pi i jk / 512)) of x[32 r + lane] = v[r];
// tw = W_512^j (j < 512), xb = this warp's kXb-entry exchange buffer.
__device__ __forceinline__ void fft512_fwd(double2 (&v)[16], int lane, const double2* tw,
                                           double2* xb) {
  const int lo = lane & 7, hi = lane >> 3;
  // stage A: group b is (j0, j1) = (lo, 4 b + hi), g = j0 + 8 j1 = lane + 32 b
  dft8<0>(v);
  dft8<1>(v);
  twiddle8<0, false>(v, tw[lane], tw[2 * lane], tw[4 * lane]);
  twiddle8<1, false>(v, tw[lane + 32], tw[2 * lane + 64], tw[4 * lane + 128]);
  // regroup by (j0, k0): entry k0 * 72 + j1 * 9 + j0
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int s = 0; s < 8; ++s) xb[brev3(s) * 8 * kXbRow + (4 * b + hi) * kXbRow + lo] = v[2 * s + b];
  __syncwarp();
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int j1 = 0; j1 < 8; ++j1) v[2 * j1 + b] = xb[(hi + 4 * b) * 8 * kXbRow + j1 * kXbRow + lo];
  __syncwarp();
  // stage B: group b is (j0, k0) = (lo, hi + 4 b); W_64^(j0 k1) = W_512^(8 j0 k1)
  dft8<0>(v);
  dft8<1>(v);
  {
    const double2 w1 = tw[8 * lo], w2 = tw[16 * lo], w4 = tw[32 * lo];
    twiddle8<0, false>(v, w1, w2, w4);
    twiddle8<1, false>(v, w1, w2, w4);
  }
  // regroup by (k1, k0): entry k0 * 72 + k1 * 9 + j0
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int s = 0; s < 8; ++s) xb[(hi + 4 * b) * 8 * kXbRow + brev3(s) * kXbRow + lo] = v[2 * s + b];
  __syncwarp();
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int j0 = 0; j0 < 8; ++j0) v[2 * j0 + b] = xb[(hi + 4 * b) * 8 * kXbRow + lo * kXbRow + j0];
  __syncwarp();
  // stage C: group b is (k1, k0) = (lo, hi + 4 b)
  dft8<0>(v);
  dft8<1>(v);
}

// Unnormalised inverse (exp(+2 pi i jk / 512)) of fft512_fwd: input in its
// output order, output v[r] of lane l = 512 x[32 r + l].
__device__ __forceinline__ void fft512_inv(double2 (&v)[16], int lane, const double2* tw,
                                           double2* xb) {
  const int lo = lane & 7, hi = lane >> 3;
  idft8<0>(v);
  idft8<1>(v);
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int j0 = 0; j0 < 8; ++j0) xb[(hi + 4 * b) * 8 * kXbRow + lo * kXbRow + j0] = v[2 * j0 + b];
  __syncwarp();
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int s = 0; s < 8; ++s) v[2 * s + b] = xb[(hi + 4 * b) * 8 * kXbRow + brev3(s) * kXbRow + lo];
  __syncwarp();
  {
    const double2 w1 = tw[8 * lo], w2 = tw[16 * lo], w4 = tw[32 * lo];
    twiddle8<0, true>(v, w1, w2, w4);
    twiddle8<1, true>(v, w1, w2, w4);
  }
  idft8<0>(v);
  idft8<1>(v);
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int j1 = 0; j1 < 8; ++j1) xb[(hi + 4 * b) * 8 * kXbRow + j1 * kXbRow + lo] = v[2 * j1 + b];
  __syncwarp();
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int s = 0; s < 8; ++s) v[2 * s + b] = xb[brev3(s) * 8 * kXbRow + (4 * b + hi) * kXbRow + lo];
  __syncwarp();
  twiddle8<0, true>(v, tw[lane], tw[2 * lane], tw[4 * lane]);
  twiddle8<1, true>(v, tw[lane + 32], tw[2 * lane + 64], tw[4 * lane + 128]);
  idft8<0>(v);
  idft8<1>(v);
}

// DFT_n of one line (INV: the unnormalised inverse, exp(+2 pi i jk / n)),
// v[j] = x[32 j + lane] with zeros at and beyond n; returns the transform in
// the same layout (entries at and beyond n are not meaningful).
template <bool INV>
__device__ __forceinline__ void line_dft(double2 (&v)[16], int lane, int n, const double2* tw,
                                         const double2* chirp, const double2* H, double2* xb) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int i = 32 * j + lane;
    if (i < n) v[j] = INV ? zmulc(v[j], chirp[i]) : zmul(v[j], chirp[i]);
    else v[j] = make_double2(0.0, 0.0);
  }
  fft512_fwd(v, lane, tw, xb);
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = zmul(v[r], H[lane * 16 + r]);
  fft512_inv(v, lane, tw, xb);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int i = 32 * j + lane;
    if (i < n) v[j] = INV ? zmulc(v[j], chirp[i]) : zmul(v[j], chirp[i]);
  }
}

// The circular convolution of Bluestein's algorithm: FFT, times the
// precomputed FFT of the chirp (1/512 included), inverse FFT.
__device__ __forceinline__ void bluestein_conv(double2 (&v)[16], int lane, const double2* tw,
                                               const double2* H, double2* xb) {
  fft512_fwd(v, lane, tw, xb);
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = zmul(v[r], H[lane * 16 + r]);
  fft512_inv(v, lane, tw, xb);
}

// Shared tables of a CTA: tw[512] | chirp[256] | H (one or two of 512).
__device__ __forceinline__ void load_tables(double2* sm, const FftArgs& a, bool hf, bool hi) {
  double2* tw = sm;
  double2* ch = sm + kFftM;
  double2* h0 = ch + kFftMaxN;
  for (int i = threadIdx.x; i < kFftM; i += blockDim.x) tw[i] = a.tw[i];
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) ch[i] = a.chirp[i];
  if (hf)
    for (int i = threadIdx.x; i < kFftM; i += blockDim.x) h0[i] = a.hf[i];
  if (hi)
    for (int i = threadIdx.x; i < kFftM; i += blockDim.x) h0[(hf ? kFftM : 0) + i] = a.hi[i];
}
constexpr int kTabDoubles2 = kFftM + kFftMaxN;  // tw + chirp

// Source row iy of slice s from its compact tile (zero outside the tile).
__device__ __forceinline__ void load_src_row(double2 (&v)[16], const FftArgs& a, int s, int iy,
                                             int lane) {
  const int4 d = a.desc[s];
  const bool in_rows = d.z > 0 && iy >= d.y && iy < d.y + d.w;
  const double2* row = a.src + (size_t)s * a.src_cap + (size_t)(iy - d.y) * d.z - d.x;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int i = 32 * j + lane;
    v[j] = (in_rows && i >= d.x && i < d.x + d.z && i < a.n) ? row[i] : make_double2(0.0, 0.0);
  }
}

// pass A: rows forward along x, written transposed.  SRC: the source rows too.
// The warps' exchange buffers double as the transposition tile once every
// warp's transform is done.
template <bool SRC>
__global__ void __launch_bounds__(kFftWarps * 32, 2) fft_rows_fwd_kernel(const FftArgs a) {
  extern __shared__ __align__(16) double2 sm[];
  load_tables(sm, a, true, false);
  const double2* tw = sm;
  const double2* ch = sm + kFftM;
  const double2* hf = ch + kFftMaxN;
  double2* xall = sm + kTabDoubles2 + kFftM;  // kFftWarps exchange buffers
  double2* tile = xall;                       // [kx][kFftPitch], after the transforms
  const int n = a.n, s = blockIdx.x / a.nband, band = blockIdx.x % a.nband;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2* xb = xall + warp * kXb;
  const int iy0 = band * kFftWarps, iy = iy0 + warp;
  const int rows = min(kFftWarps, n - iy0);
  __syncthreads();
  for (int part = 0; part < (SRC ? 2 : 1); ++part) {
    double2 v[16];
    if (warp < rows) {
      if (part == 0) {
        const double2* row = a.u + ((size_t)s * n + iy) * a.ld;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int i = 32 * j + lane;
          v[j] = i < n ? row[i] : make_double2(0.0, 0.0);
        }
      } else {
        load_src_row(v, a, s, iy, lane);
      }
      line_dft<false>(v, lane, n, tw, ch, hf, xb);
    }
    __syncthreads();  // every transform done: the buffers become the tile
    if (warp < rows) {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int k = 32 * j + lane;
        if (k < n) tile[k * kFftPitch + warp] = v[j];
      }
    }
    __syncthreads();
    double2* dst = part == 0 ? a.T : a.ST;
    for (int idx = threadIdx.x; idx < n * kFftWarps; idx += blockDim.x) {
      const int k = idx / kFftWarps, r = idx % kFftWarps;
      if (r < rows) dst[((size_t)s * n + k) * a.ld + iy0 + r] = tile[k * kFftPitch + r];
    }
    if (SRC && part == 0) __syncthreads();  // the tile is read before the next transforms
  }
}

// pass B: lines along y, forward, propagator (+ filtered source), inverse.
template <bool FILTER>
__global__ void __launch_bounds__(kFftWarps * 32, FILTER ? 1 : 2) fft_cols_kernel(const FftArgs a) {
  extern __shared__ __align__(16) double2 sm[];
  load_tables(sm, a, true, true);
  const double2* tw = sm;
  const double2* ch = sm + kFftM;
  const double2* hf = ch + kFftMaxN;
  const double2* hi = hf + kFftM;
  double2* xall = sm + kTabDoubles2 + 2 * kFftM;  // kFftWarps exchange buffers
  double2* stage = xall + kFftWarps * kXb;        // [warp][256] filtered source spectrum
  const int n = a.n, s = blockIdx.x / a.nband, band = blockIdx.x % a.nband;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2* xb = xall + warp * kXb;
  const int kx = band * kFftWarps + warp;
  __syncthreads();
  if (kx >= n) return;
  double2* line = a.T + ((size_t)s * n + kx) * a.ld;
  const double2* prop = a.prop_t + (size_t)kx * n;
  // The forward transform's closing chirp w_k and the inverse's opening
  // conj(w_k) meet at the propagator and cancel (|w_k| = 1): between the two
  // convolutions the line is multiplied by exp(i k2 dz) alone (and the
  // filtered source spectrum enters without its closing chirp).
  double2 v[16];
  if (FILTER) {
    const double2* sline = a.ST + ((size_t)s * n + kx) * a.ld;
    const double* sg = a.sig_t + (size_t)kx * n;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int i = 32 * j + lane;
      v[j] = i < n ? zmul(sline[i], ch[i]) : make_double2(0.0, 0.0);
    }
    bluestein_conv(v, lane, tw, hf, xb);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int k = 32 * j + lane;
      if (k < n) {
        const double f = 2.0 * sg[k];
        stage[warp * kFftMaxN + k] = make_double2(v[j].x * f, v[j].y * f);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int i = 32 * j + lane;
    v[j] = i < n ? zmul(line[i], ch[i]) : make_double2(0.0, 0.0);
  }
  bluestein_conv(v, lane, tw, hf, xb);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int k = 32 * j + lane;
    if (k < n) {
      v[j] = zmul(v[j], prop[k]);
      if (FILTER) v[j] = zadd(v[j], stage[warp * kFftMaxN + k]);
    } else {
      v[j] = make_double2(0.0, 0.0);
    }
  }
  bluestein_conv(v, lane, tw, hi, xb);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int i = 32 * j + lane;
    if (i < n) line[i] = zmulc(v[j], ch[i]);
  }
}

// pass C: rows back along x from the transposed layout, scaled, + 2 S.  The
// gather tile becomes the warps' exchange buffers once every warp has read
// its row from it.
template <bool ADD_SRC>
__global__ void __launch_bounds__(kFftWarps * 32, 2) fft_rows_inv_kernel(const FftArgs a) {
  extern __shared__ __align__(16) double2 sm[];
  load_tables(sm, a, false, true);
  const double2* tw = sm;
  const double2* ch = sm + kFftM;
  const double2* hi = ch + kFftMaxN;
  double2* xall = sm + kTabDoubles2 + kFftM;  // [kx][kFftPitch], then exchange buffers
  double2* tile = xall;
  const int n = a.n, s = blockIdx.x / a.nband, band = blockIdx.x % a.nband;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int iy0 = band * kFftWarps, iy = iy0 + warp;
  const int rows = min(kFftWarps, n - iy0);
  for (int idx = threadIdx.x; idx < n * kFftWarps; idx += blockDim.x) {
    const int k = idx / kFftWarps, r = idx % kFftWarps;
    tile[k * kFftPitch + r] =
        r < rows ? a.T[((size_t)s * n + k) * a.ld + iy0 + r] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2 v[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int k = 32 * j + lane;
    v[j] = k < n ? tile[k * kFftPitch + warp] : make_double2(0.0, 0.0);
  }
  __syncthreads();  // every row read: the tile becomes the exchange buffers
  if (warp >= rows) return;
  line_dft<true>(v, lane, n, tw, ch, hi, xall + warp * kXb);
  // the source row of the compact tile (zero outside it), read as it is added
  const int4 d = ADD_SRC ? a.desc[s] : make_int4(0, 0, 0, 0);
  const bool in_rows = ADD_SRC && d.z > 0 && iy >= d.y && iy < d.y + d.w;
  const double2* srow = a.src + (size_t)s * a.src_cap + (size_t)(iy - d.y) * d.z - d.x;
  double2* row = a.out + ((size_t)s * n + iy) * a.ld;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int x = 32 * j + lane;
    if (x < n) {
      double2 o = make_double2(v[j].x * a.scale, v[j].y * a.scale);
      if (in_rows && x >= d.x && x < d.x + d.z) {
        const double2 sv = srow[x];
        o = make_double2(fma(2.0, sv.x, o.x), fma(2.0, sv.y, o.y));
      }
      row[x] = o;
    }
  }
}

// exp(i k2 dz) of the transposed phase table, FP64 cos / sin per element as
// the reference's propagator kernel computes them
// (src/Core/FieldSolverFFTCUDA.cpp:157-188).
__global__ void fft_prop_kernel(const double* k2_t, double delz, int nn, double2* prop_t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) {
    const double ph = k2_t[i] * delz;
    prop_t[i] = make_double2(cos(ph), sin(ph));
  }
}

}  // namespace
}  // namespace g4b

using namespace g4b;

struct g4b_fft {
  g4b_ctx* ctx = nullptr;
  int ngrid = 0;
  double delz = 0, dgrid = 0, xks = 0, prop_delz = 0;
  double xc = 1, yc = 1, sig = 1;   // FieldSolverFFTCUDA's member defaults
  bool want_filter = false;         // initSourceFilter's request
  bool filter = false;              // in effect (shape valid at init)
  bool ready = false;
  double2 *tw = nullptr, *chirp = nullptr, *hf = nullptr, *hi = nullptr, *prop_t = nullptr;
  double* k2_t = nullptr;
  double* sig_t = nullptr;
  double2* st = nullptr;            // transposed source spectrum (filtered runs)
  size_t st_cells = 0;
};

namespace {

using cld = std::complex<long double>;

// FFT_512 of h by the definition, in long double, divided by 512 and stored
// in the warp FFT's output order (lane l, register r <-> k0 + 8 k1 + 64 k2).
std::vector<double2> permuted_spectrum(const std::vector<cld>& h) {
  const long double pi = 3.141592653589793238462643383279502884L;
  std::vector<cld> H(kFftM);
  for (int k = 0; k < kFftM; ++k) {
    cld acc = 0;
    for (int t = 0; t < kFftM; ++t) {
      if (h[t] == cld(0)) continue;
      const long double ang = -2.0L * pi * (long double)((k * t) % kFftM) / kFftM;
      acc += h[t] * cld(cosl(ang), sinl(ang));
    }
    H[k] = acc / (long double)kFftM;
  }
  std::vector<double2> out(kFftM);
  for (int l = 0; l < 32; ++l)
    for (int r = 0; r < 16; ++r) {
      const int q = l + 32 * (r & 1);
      const cld v = H[(q >> 3) + 8 * (q & 7) + 64 * brev3(r >> 1)];
      out[l * 16 + r] = make_double2((double)v.real(), (double)v.imag());
    }
  return out;
}

template <typename T>
int upload(g4b_ctx* c, T** d, const std::vector<T>& h) {
  if (*d) dev_free(c, *d);
  *d = nullptr;
  G4B_CUDA_TRY(dev_alloc(c, (void**)d, h.size() * sizeof(T)));
  G4B_CUDA_TRY(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice,
                               c->stream));
  return G4B_OK;
}

int set_smem(const void* fn, size_t bytes) {
  G4B_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)bytes));
  return G4B_OK;
}

}  // namespace

extern "C" {

int g4b_fft_create(g4b_ctx* c, g4b_fft** out) {
  if (!c || !out) return fail(G4B_ERR_ARG, "g4b_fft_create: null arg");
  g4b_fft* s = new (std::nothrow) g4b_fft();
  if (!s) return fail(G4B_ERR_NOMEM, "g4b_fft_create: host allocation");
  s->ctx = c;
  ctx_retain(c);
  *out = s;
  return G4B_OK;
}

int g4b_fft_destroy(g4b_fft* s) {
  if (!s) return G4B_OK;
  g4b_ctx* c = s->ctx;
  cudaSetDevice(c->device);
  for (void* p : {(void*)s->tw, (void*)s->chirp, (void*)s->hf, (void*)s->hi,
                  (void*)s->prop_t, (void*)s->k2_t, (void*)s->sig_t, (void*)s->st})
    dev_free(c, p);
  delete s;
  ctx_release(c);
  return G4B_OK;
}

// FieldSolverFFTCUDA::initSourceFilter (src/Core/FieldSolverFFTCUDA.cpp:214-222).
int g4b_fft_init_filter(g4b_fft* s, double xc, double yc, double sig, int filter) {
  if (!s) return fail(G4B_ERR_ARG, "g4b_fft_init_filter: null arg");
  s->xc = xc;
  s->yc = yc;
  s->sig = sig;
  s->want_filter = filter != 0 && sig > 0 && xc > 0 && yc > 0;
  s->ready = false;  // the filter table follows the next init
  return G4B_OK;
}

// FieldSolverFFTCUDA::init (src/Core/FieldSolverFFTCUDA.cpp:246-293): the
// spectral phase k2 = -(dx^2 + dy^2) dk^2 / (2 ks), dk = 2 pi / (n dgrid), in
// FFT index order, and the sigmoid source filter; plus the Bluestein tables.
int g4b_fft_init(g4b_fft* s, double delz, double dgrid, double xks, int ngrid) {
  if (!s) return fail(G4B_ERR_ARG, "g4b_fft_init: null arg");
  if (ngrid < 2 || ngrid > kFftMaxN)
    return fail(G4B_ERR_RANGE, "g4b_fft_init: ngrid must be in [2, 256]");
  if (!(dgrid > 0) || !(xks > 0)) return fail(G4B_ERR_ARG, "g4b_fft_init: bad dgrid or xks");
  s->delz = delz;
  g4b_ctx* c = s->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  if (!(s->ready && s->ngrid == ngrid && s->dgrid == dgrid && s->xks == xks)) {
    const int n = ngrid;
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<double2> tw(kFftM), chirp(n);
    for (int j = 0; j < kFftM; ++j) {
      const long double ang = -2.0L * pi * j / kFftM;
      tw[j] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    std::vector<cld> hfw(kFftM, 0), hiw(kFftM, 0);
    for (int j = 0; j < n; ++j) {
      const long long q = ((long long)j * j) % (2LL * n);
      const long double ang = -pi * (long double)q / n;
      const cld w(cosl(ang), sinl(ang));
      chirp[j] = make_double2((double)w.real(), (double)w.imag());
      hfw[j] = std::conj(w);
      hiw[j] = w;
      if (j > 0) {
        hfw[kFftM - j] = std::conj(w);
        hiw[kFftM - j] = w;
      }
    }
    const std::vector<double2> hf = permuted_spectrum(hfw), hi = permuted_spectrum(hiw);
    // the reference's tables, transposed to [kx][ky]
    const bool shape_ok = s->xc > 0 && s->yc > 0 && s->sig > 0;
    const double dk = 4. * asin(1.) / (static_cast<double>(n) * dgrid);
    const double shift = -0.5 * static_cast<double>(n - 1);
    std::vector<double> k2_t((size_t)n * n), sig_t((size_t)n * n);
    for (int iy = 0; iy < n; iy++) {
      const double dy = static_cast<double>(iy) + shift;
      const double y = shape_ok ? dy / static_cast<double>(n) / s->yc : 0.0;
      for (int ix = 0; ix < n; ix++) {
        const double dx = static_cast<double>(ix) + shift;
        const double x = shape_ok ? dx / static_cast<double>(n) / s->xc : 0.0;
        const int iiy = (iy + (n + 1) / 2) % n, iix = (ix + (n + 1) / 2) % n;
        const size_t t = (size_t)iix * n + iiy;  // [kx][ky]
        k2_t[t] = -(dx * dx + dy * dy) * dk * dk / 2. / xks;
        if (shape_ok) {
          const double r = (sqrt(x * x + y * y) - 1) / s->sig;
          sig_t[t] = 1. / (1 + exp(r));
        } else {
          sig_t[t] = 1.0;
        }
      }
    }
    if (int rc = upload(c, &s->tw, tw)) return rc;
    if (int rc = upload(c, &s->chirp, chirp)) return rc;
    if (int rc = upload(c, &s->hf, hf)) return rc;
    if (int rc = upload(c, &s->hi, hi)) return rc;
    if (int rc = upload(c, &s->k2_t, k2_t)) return rc;
    if (int rc = upload(c, &s->sig_t, sig_t)) return rc;
    if (s->prop_t) dev_free(c, s->prop_t);
    s->prop_t = nullptr;
    G4B_CUDA_TRY(dev_alloc(c, (void**)&s->prop_t, (size_t)n * n * sizeof(double2)));
    s->prop_delz = std::nan("");
    s->filter = s->want_filter && shape_ok;
    s->ngrid = n;
    s->dgrid = dgrid;
    s->xks = xks;
    s->ready = true;
  }
  if (!(s->prop_delz == delz)) {
    const int nn = s->ngrid * s->ngrid;
    {
      LaunchScope ls(c, "fft_prop");
      fft_prop_kernel<<<(nn + 255) / 256, 256, 0, c->stream>>>(s->k2_t, delz, nn, s->prop_t);
    }
    if (int rc = check_launch(c, "fft_prop_kernel")) return rc;
    s->prop_delz = delz;
  }
  return G4B_OK;
}

// FieldSolverFFTCUDA::advance (src/Core/FieldSolverFFTCUDA.cpp:295-483).
int g4b_fft_advance(g4b_fft* s, g4b_field* f, g4b_beam* b, const g4b_step* st, double fc,
                    int enabled) {
  if (!s || !f || !b || !st) return fail(G4B_ERR_ARG, "g4b_fft_advance: null arg");
  if (!s->ready || s->ngrid != f->ngrid)
    return fail(G4B_ERR_STATE, "g4b_fft_advance: called before g4b_fft_init for this ngrid");
  if (b->nslice != f->nslice)
    return fail(G4B_ERR_ARG, "g4b_fft_advance: beam and field slice counts differ");
  if (f->precision != G4B_FP64 || b->precision != G4B_FP64)
    return fail(G4B_ERR_ARG, "g4b_fft_advance: the drop-in path holds FP64 state");
  g4b_ctx* c = f->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  const int n = f->ngrid;
  const bool do_source = st->in_undulator && enabled && (f->harm % 2) == 1 && b->npart > 0;
  if (do_source)
    if (int rc = fp64_deposit(f, b, st, fc)) return rc;
  const bool filt = do_source && s->filter;
  if (filt) {
    const size_t need = (size_t)f->nslice * n * f->ld;
    if (s->st_cells < need) {
      dev_free(c, s->st);
      s->st = nullptr;
      s->st_cells = 0;
      G4B_CUDA_TRY(dev_alloc(c, (void**)&s->st, need * sizeof(double2)));
      s->st_cells = need;
    }
  }
  FftArgs a{};
  a.tw = s->tw;
  a.chirp = s->chirp;
  a.hf = s->hf;
  a.hi = s->hi;
  a.prop_t = s->prop_t;
  a.sig_t = s->sig_t;
  a.u = static_cast<const double2*>(f->a);
  a.out = static_cast<double2*>(f->a);
  a.T = static_cast<double2*>(f->b);
  a.ST = s->st;
  a.src = static_cast<const double2*>(f->src);
  a.desc = f->desc;
  a.src_cap = (size_t)f->ngrid * f->ld;
  a.n = n;
  a.ld = f->ld;
  a.nband = (n + kFftWarps - 1) / kFftWarps;
  a.scale = 1.0 / ((double)n * (double)n);
  const unsigned grid = (unsigned)(f->nslice * a.nband);
  const size_t tab = (size_t)kTabDoubles2 * sizeof(double2);
  // exchange buffers of the warps, which in passes A and C also hold the
  // transposition tile (kFftMaxN x kFftPitch entries)
  const size_t xbuf = std::max((size_t)kFftWarps * kXb, (size_t)kFftMaxN * kFftPitch) *
                      sizeof(double2);
  const size_t smem_a = tab + kFftM * sizeof(double2) + xbuf;
  const size_t smem_b = tab + 2 * kFftM * sizeof(double2) +
                        (size_t)kFftWarps * kXb * sizeof(double2) +
                        (filt ? (size_t)kFftWarps * kFftMaxN * sizeof(double2) : 0);
  const size_t smem_c = tab + kFftM * sizeof(double2) + xbuf;
  {
    auto ka = filt ? fft_rows_fwd_kernel<true> : fft_rows_fwd_kernel<false>;
    if (int rc = set_smem((const void*)ka, smem_a)) return rc;
    LaunchScope ls(c, "fft_rows_fwd");
    ka<<<grid, kFftWarps * 32, smem_a, c->stream>>>(a);
  }
  if (int rc = check_launch(c, "fft_rows_fwd_kernel")) return rc;
  {
    auto kb = filt ? fft_cols_kernel<true> : fft_cols_kernel<false>;
    if (int rc = set_smem((const void*)kb, smem_b)) return rc;
    LaunchScope ls(c, "fft_cols");
    kb<<<grid, kFftWarps * 32, smem_b, c->stream>>>(a);
  }
  if (int rc = check_launch(c, "fft_cols_kernel")) return rc;
  {
    const bool add = do_source && !filt;
    auto kc = add ? fft_rows_inv_kernel<true> : fft_rows_inv_kernel<false>;
    if (int rc = set_smem((const void*)kc, smem_c)) return rc;
    LaunchScope ls(c, "fft_rows_inv");
    kc<<<grid, kFftWarps * 32, smem_c, c->stream>>>(a);
  }
  return check_launch(c, "fft_rows_inv_kernel");
}

}  // extern "C"
