// g4b_diag.cu -- per-slice beam and field diagnostics (DiagnosticCUDA) for sm_100a.
//
// One CTA per slice reads its particles (or its field plane) once and keeps
// every moment in registers; reductions run in a fixed order (warp xor tree,
// then warps in index order), so results are reproducible run to run.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "g4b_internal.cuh"

namespace g4b {

constexpr int kDiagThreads = 256;
constexpr int kDiagWarps = kDiagThreads / 32;
constexpr int kMaxHarmPass = 8;  // harmonics accumulated per pass

enum class Red { Sum, Min, Max };

__device__ __forceinline__ double warp_red(double v, Red op) {
  for (int o = 16; o > 0; o >>= 1) {
    const double t = __shfl_xor_sync(0xffffffffu, v, o);
    v = op == Red::Sum ? v + t : (op == Red::Min ? fmin(v, t) : fmax(v, t));
  }
  return v;
}

// g4_beam_slice_reduce_kernel (src/Core/DiagnosticCUDA.cpp:188-303); HP
// harmonics accumulated per pass over the particles.  For the fundamental
// alone (HP = 1) three CTAs per SM at 80 registers: 157 -> 119 us per
// 1024 x 8192 particles against one CTA size for all (the same arithmetic).
template <int HP>
__global__ void __launch_bounds__(kDiagThreads, HP == 1 ? 3 : 1)
    beam_diag_kernel(int nslice, int nharm, int need_aux, const int64_t* off,
                     const double* x, const double* y, const double* px, const double* py,
                     const double* gamma, const double* theta, double* stats, double* bre,
                     double* bim) {
  __shared__ double part[kDiagWarps][23 + 2 * HP];
  ptx::pdl_wait();
  const int is = blockIdx.x;
  if (is >= nslice) return;
  const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
  const int64_t p0 = off[is], p1 = off[is + 1];
  double v[23];
#pragma unroll
  for (int k = 0; k < 13; ++k) v[k] = 0.0;
  v[13] = 1.0e5; v[14] = -1.0e5;  // xmin xmax
  v[15] = 1.0e5; v[16] = -1.0e5;  // pxmin pxmax
  v[17] = 1.0e5; v[18] = -1.0e5;  // ymin ymax
  v[19] = 1.0e5; v[20] = -1.0e5;  // pymin pymax
  v[21] = 1.0e7; v[22] = 1.0;     // gmin gmax
  const int h0n = min(nharm, HP);
  double br[HP], bi[HP];
#pragma unroll
  for (int h = 0; h < HP; ++h) br[h] = bi[h] = 0.0;
  for (int64_t p = p0 + tid; p < p1; p += kDiagThreads) {
    const double xv = x[p], yv = y[p], pxv = px[p], pyv = py[p], gv = gamma[p];
    v[0] += gv;
    v[1] += gv * gv;
    v[2] += xv;
    v[3] += xv * xv;
    v[4] += yv;
    v[5] += yv * yv;
    v[6] += pxv;
    v[7] += pxv * pxv;
    v[8] += pyv;
    v[9] += pyv * pyv;
    v[10] += xv * pxv;
    v[11] += yv * pyv;
    v[12] += 1.0;
    if (need_aux) {
      v[13] = fmin(v[13], xv); v[14] = fmax(v[14], xv);
      v[15] = fmin(v[15], pxv); v[16] = fmax(v[16], pxv);
      v[17] = fmin(v[17], yv); v[18] = fmax(v[18], yv);
      v[19] = fmin(v[19], pyv); v[20] = fmax(v[20], pyv);
      v[21] = fmin(v[21], gv); v[22] = fmax(v[22], gv);
    }
    const double th = theta[p];
#pragma unroll
    for (int h = 0; h < HP; ++h) {
      if (h < h0n) {
        double s, c;
        sincos((double)(h + 1) * th, &s, &c);
        br[h] += c;
        bi[h] += s;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 23; ++k) {
    const Red op = k < 13 ? Red::Sum : ((k - 13) % 2 == 0 ? Red::Min : Red::Max);
    const double r = warp_red(v[k], op);
    if (l == 0) part[w][k] = r;
  }
#pragma unroll
  for (int h = 0; h < HP; ++h) {
    if (h < h0n) {
      const double rr = warp_red(br[h], Red::Sum), ri = warp_red(bi[h], Red::Sum);
      if (l == 0) {
        part[w][23 + 2 * h] = rr;
        part[w][24 + 2 * h] = ri;
      }
    }
  }
  __syncthreads();
  if (tid < 23) {
    const int k = tid;
    const Red op = k < 13 ? Red::Sum : ((k - 13) % 2 == 0 ? Red::Min : Red::Max);
    double r = part[0][k];
    for (int i = 1; i < kDiagWarps; ++i) {
      const double t = part[i][k];
      r = op == Red::Sum ? r + t : (op == Red::Min ? fmin(r, t) : fmax(r, t));
    }
    if (k >= 13 && !need_aux) r = 0.0;
    stats[(size_t)is * 23 + k] = r;
  } else if (tid >= 32 && tid < 32 + 2 * h0n) {
    const int k = tid - 32;
    double r = part[0][23 + k];
    for (int i = 1; i < kDiagWarps; ++i) r += part[i][23 + k];
    const int h = k >> 1;
    if (k & 1)
      bim[(size_t)is * nharm + h] = r;
    else
      bre[(size_t)is * nharm + h] = r;
  }
  // further harmonics, HP at a time
  for (int hb = HP; hb < nharm; hb += HP) {
    const int hn = min(nharm - hb, HP);
#pragma unroll
    for (int h = 0; h < HP; ++h) br[h] = bi[h] = 0.0;
    for (int64_t p = p0 + tid; p < p1; p += kDiagThreads) {
      const double th = theta[p];
#pragma unroll
      for (int h = 0; h < HP; ++h) {
        if (h < hn) {
          double s, c;
          sincos((double)(hb + h + 1) * th, &s, &c);
          br[h] += c;
          bi[h] += s;
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < HP; ++h) {
      if (h < hn) {
        const double rr = warp_red(br[h], Red::Sum), ri = warp_red(bi[h], Red::Sum);
        if (l == 0) {
          part[w][2 * h] = rr;
          part[w][2 * h + 1] = ri;
        }
      }
    }
    __syncthreads();
    if (tid < 2 * hn) {
      double r = part[0][tid];
      for (int i = 1; i < kDiagWarps; ++i) r += part[i][tid];
      const int h = hb + (tid >> 1);
      if (tid & 1)
        bim[(size_t)is * nharm + h] = r;
      else
        bre[(size_t)is * nharm + h] = r;
    }
  }
}

// g4_field_slice_reduce_kernel (src/Core/DiagnosticCUDA.cpp:305-363)
template <typename C>
__global__ void __launch_bounds__(kDiagThreads)
    field_diag_kernel(int nslice, int n, int ld, int first, const C* cells, double* stats,
                      double* center) {
  __shared__ double part[kDiagWarps][7];
  const int is0 = blockIdx.x;
  if (is0 >= nslice) return;
  const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
  const C* c = cells + (size_t)is0 * n * ld;
  const int is = (nslice + is0 - first) % nslice;
  const double shift = -0.5 * (double)(n - 1);
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  const int plane = n * n;
  // a warp per row: coalesced row reads with no index division, the row's
  // sums first, then its y moments from the row's power
  for (int iy = w; iy < n; iy += kDiagWarps) {
    const C* row = c + (size_t)iy * ld;
    double p = 0, px = 0, pxx = 0, sre = 0, sim = 0;
    for (int ix = l; ix < n; ix += 32) {
      const C u = row[ix];
      const double re = u.x, im = u.y;
      const double wei = re * re + im * im;
      const double dx = (double)ix + shift;
      p += wei;
      px += dx * wei;
      pxx += dx * dx * wei;
      sre += re;
      sim += im;
    }
    const double dy = (double)iy + shift;
    v[0] += p;
    v[1] += px;
    v[2] += pxx;
    v[3] += dy * p;
    v[4] += dy * dy * p;
    v[5] += sre;
    v[6] += sim;
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    const double r = warp_red(v[k], Red::Sum);
    if (l == 0) part[w][k] = r;
  }
  __syncthreads();
  if (tid < 7) {
    double r = part[0][tid];
    for (int i = 1; i < kDiagWarps; ++i) r += part[i][tid];
    stats[(size_t)is * 7 + tid] = r;
  } else if (tid == 32) {
    const int ic = (plane - 1) / 2;
    const C u = c[(size_t)(ic / n) * ld + (ic % n)];
    center[2 * is] = u.x;
    center[2 * is + 1] = u.y;
  }
}

}  // namespace g4b

using namespace g4b;

namespace {
struct DiagScratch {
  double* d = nullptr;
  size_t cap = 0;
};
// Grow-on-demand scratch of the diagnostics entry points, one buffer per
// calling host thread and device: a thread may drive contexts on several
// devices, and a buffer is only ever used (and freed) with its own device
// current.  Freed with the process (small).
constexpr int kDiagScratchDevices = 64;
int diag_scratch(int device, DiagScratch** out) {
  static thread_local DiagScratch per_device[kDiagScratchDevices];
  if (device < 0 || device >= kDiagScratchDevices)
    return fail(G4B_ERR_RANGE, "diagnostics: device index above 63");
  *out = &per_device[device];
  return G4B_OK;
}
int ensure(DiagScratch& s, size_t n) {
  if (s.cap >= n) return G4B_OK;
  if (s.d) cudaFree(s.d);
  s.d = nullptr;
  s.cap = 0;
  G4B_CUDA_TRY(cudaMalloc(&s.d, n * sizeof(double)));
  s.cap = n;
  return G4B_OK;
}
}  // namespace

namespace {

// ---- field diagnostics with fixed scratch ----------------------------------
// Some callers must not allocate device memory when they ask for the field
// statistics: a host that hands the device's memory to its own pool and
// forbids growth during a run, or a loop whose latency budget has no room for
// cudaMalloc's implicit device-wide synchronisation.  For them the scratch of
// field_diag_kernel lives in one fixed file-scope device array instead of the
// grow-on-demand buffer above.  Its size bounds the slices per call.
constexpr int kStaticDiagMaxSlices = 4096;               // 4096 x 9 doubles = 288 KiB
static __device__ __align__(256) double g_field_diag_scratch[kStaticDiagMaxSlices * 9];

constexpr int kStaticDiagMaxDevices = 64;
std::atomic<double*> g_field_diag_scratch_ptr[kStaticDiagMaxDevices];
std::mutex g_field_diag_scratch_mutex;

// Address of the array on `device` (which must be current).  The first call
// on a device asks the runtime for the symbol address (which may load the
// module); later calls read the cached pointer.
int static_diag_scratch(int device, double** out) {
  if (device < 0 || device >= kStaticDiagMaxDevices)
    return fail(G4B_ERR_RANGE, "g4b_diag_field_static: device index above 63");
  double* p = g_field_diag_scratch_ptr[device].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_field_diag_scratch_mutex);
    p = g_field_diag_scratch_ptr[device].load(std::memory_order_relaxed);
    if (!p) {
      const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_field_diag_scratch);
      if (e != cudaSuccess) return cuda_fail(e, "g4b_diag_field_static: cudaGetSymbolAddress");
      g_field_diag_scratch_ptr[device].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return G4B_OK;
}

}  // namespace

extern "C" {

int g4b_diag_beam(g4b_beam* b, int nharm, int need_aux, double* stats, double* bre,
                  double* bim) {
  if (!b || !stats || nharm < 1 || !bre || !bim)
    return fail(G4B_ERR_ARG, "g4b_diag_beam: bad argument");
  if (b->precision != G4B_FP64) return fail(G4B_ERR_ARG, "g4b_diag_beam: FP64 beam expected");
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  DiagScratch* scratch = nullptr;
  if (int rc = diag_scratch(c->device, &scratch)) return rc;
  const size_t ns = b->nslice;
  const size_t need = ns * 23 + 2 * ns * nharm;
  if (int rc = ensure(*scratch, need)) return rc;
  double* d_stats = scratch->d;
  double* d_bre = d_stats + ns * 23;
  double* d_bim = d_bre + ns * nharm;
  {
    LaunchScope ls(c, "diag_beam");
    auto kern = nharm == 1 ? beam_diag_kernel<1> : beam_diag_kernel<kMaxHarmPass>;
    G4B_CUDA_TRY(launch_pdl(kern, (unsigned)b->nslice, kDiagThreads, 0, c->stream, b->nslice,
                            nharm, need_aux, b->d_off, b->x, b->y, b->px, b->py, b->gamma,
                            b->theta, d_stats, d_bre, d_bim));
  }
  if (int rc = check_launch(c, "beam_diag_kernel")) return rc;
  G4B_CUDA_TRY(cudaMemcpyAsync(stats, d_stats, ns * 23 * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  G4B_CUDA_TRY(cudaMemcpyAsync(bre, d_bre, ns * nharm * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  G4B_CUDA_TRY(cudaMemcpyAsync(bim, d_bim, ns * nharm * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G4B_OK;
}

int g4b_diag_field(g4b_field* f, double* stats, double* center) {
  if (!f || !stats || !center) return fail(G4B_ERR_ARG, "g4b_diag_field: null arg");
  g4b_ctx* c = f->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  DiagScratch* scratch = nullptr;
  if (int rc = diag_scratch(c->device, &scratch)) return rc;
  const size_t ns = f->nslice;
  if (int rc = ensure(*scratch, ns * 9)) return rc;
  double* d_stats = scratch->d;
  double* d_center = d_stats + ns * 7;
  {
    LaunchScope ls(c, "diag_field");
    if (f->precision == G4B_FP64)
      field_diag_kernel<double2><<<f->nslice, kDiagThreads, 0, c->stream>>>(
          f->nslice, f->ngrid, f->ld, f->first, static_cast<const double2*>(f->a), d_stats,
          d_center);
    else
      field_diag_kernel<float2><<<f->nslice, kDiagThreads, 0, c->stream>>>(
          f->nslice, f->ngrid, f->ld, f->first, static_cast<const float2*>(f->a), d_stats,
          d_center);
  }
  if (int rc = check_launch(c, "field_diag_kernel")) return rc;
  G4B_CUDA_TRY(cudaMemcpyAsync(stats, d_stats, ns * 7 * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  G4B_CUDA_TRY(cudaMemcpyAsync(center, d_center, ns * 2 * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G4B_OK;
}

// Same statistics as g4b_diag_field, with the device scratch in a fixed
// file-scope array: nothing is allocated on the device or through the CUDA
// runtime's allocators.  Every scratch entry the call reads back is written
// by its own kernel first, so no part of the array has to start at zero.
int g4b_diag_field_static(g4b_field* f, double* stats, double* center) {
  if (!f || !stats || !center) return fail(G4B_ERR_ARG, "g4b_diag_field_static: null arg");
  if (f->nslice > kStaticDiagMaxSlices)
    return fail(G4B_ERR_RANGE, "g4b_diag_field_static: " + std::to_string(f->nslice) +
                                   " slices exceed the fixed scratch of " +
                                   std::to_string(kStaticDiagMaxSlices));
  g4b_ctx* c = f->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  double* d_stats = nullptr;
  if (int rc = static_diag_scratch(c->device, &d_stats)) return rc;
  const size_t ns = f->nslice;
  double* d_center = d_stats + ns * 7;
  if (f->precision == G4B_FP64)
    field_diag_kernel<double2><<<f->nslice, kDiagThreads, 0, c->stream>>>(
        f->nslice, f->ngrid, f->ld, f->first, static_cast<const double2*>(f->a), d_stats,
        d_center);
  else
    field_diag_kernel<float2><<<f->nslice, kDiagThreads, 0, c->stream>>>(
        f->nslice, f->ngrid, f->ld, f->first, static_cast<const float2*>(f->a), d_stats,
        d_center);
  count_launch(c);
  if (int rc = check_launch(c, "field_diag_kernel")) return rc;
  G4B_CUDA_TRY(cudaMemcpyAsync(stats, d_stats, ns * 7 * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  G4B_CUDA_TRY(cudaMemcpyAsync(center, d_center, ns * 2 * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G4B_OK;
}

}  // extern "C"
