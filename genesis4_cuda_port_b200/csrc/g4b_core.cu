// g4b_core.cu -- context, field and beam state, slippage, error plumbing.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

#include "g4b_internal.cuh"

namespace g4b {

static thread_local std::string t_last_error;

void set_error(const std::string& msg) { t_last_error = msg; }

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? G4B_ERR_NOMEM : G4B_ERR_CUDA;
}

cudaError_t dev_alloc(g4b_ctx* c, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  return cudaMallocAsync(p, bytes, c->stream);
}

void dev_free(g4b_ctx* c, void* p) {
  if (p) cudaFreeAsync(p, c->stream);
}

int check_launch(g4b_ctx* ctx, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  (void)ctx;
  return G4B_OK;
}

int read_device_error(g4b_ctx* ctx, const char* what) {
  int h = 0;
  G4B_CUDA_TRY(cudaMemcpyAsync(&h, ctx->d_error, sizeof(int),
                               cudaMemcpyDeviceToHost, ctx->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (h != 0) {
    G4B_CUDA_TRY(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    char buf[160];
    snprintf(buf, sizeof buf, "%s: device error flag 0x%x (%s%s%s)", what, h,
             (h & kErrWaitTimeout) ? "wait timeout " : "",
             (h & kErrFixedRange) ? "fixed-point range " : "",
             (h & kErrBadSlice) ? "bad slice" : "");
    return fail(G4B_ERR_DEVICE, buf);
  }
  return G4B_OK;
}

static cudaEvent_t pool_get(Profiler& p) {
  if (!p.pool.empty()) {
    cudaEvent_t e = p.pool.back();
    p.pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

static void prof_resolve(g4b_ctx* c) {
  Profiler& p = c->prof;
  if (p.pending.empty()) return;
  cudaStreamSynchronize(c->stream);
  for (auto& q : p.pending) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, q.a, q.b) == cudaSuccess) {
      p.count[q.name] += 1;
      p.ms[q.name] += t;
    }
    p.pool.push_back(q.a);
    p.pool.push_back(q.b);
  }
  p.pending.clear();
}

void prof_begin(g4b_ctx* c, const char* name) {
  Profiler& p = c->prof;
  if (!p.on) return;
  int id = -1;
  for (size_t i = 0; i < p.names.size(); ++i)
    if (p.names[i] == name) id = (int)i;
  if (id < 0) {
    id = (int)p.names.size();
    p.names.push_back(name);
    p.count.push_back(0);
    p.ms.push_back(0.0);
  }
  p.open_a = pool_get(p);
  p.open_name = id;
  cudaEventRecord(p.open_a, c->stream);
}

void prof_end(g4b_ctx* c) {
  Profiler& p = c->prof;
  if (!p.on || p.open_name < 0) return;
  cudaEvent_t b = pool_get(p);
  cudaEventRecord(b, c->stream);
  p.pending.push_back({p.open_name, p.open_a, b});
  p.open_name = -1;
  if (p.pending.size() > 8192) prof_resolve(c);
}

// The context's device resources (stream, error flag, events) live until the
// last reference goes: objects created on a context keep working after
// g4b_ctx_destroy released the handle.
static void ctx_teardown(g4b_ctx* c) {
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->d_error) cudaFree(c->d_error);
  c->d_error = nullptr;
  for (auto& q : c->prof.pending) {
    cudaEventDestroy(q.a);
    cudaEventDestroy(q.b);
  }
  c->prof.pending.clear();
  for (auto e : c->marks) cudaEventDestroy(e);
  c->marks.clear();
  for (auto e : c->prof.pool) cudaEventDestroy(e);
  c->prof.pool.clear();
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->stream = nullptr;
}

void ctx_release(g4b_ctx* c) {
  if (--c->refs == 0) {
    ctx_teardown(c);
    delete c;
  }
}

void ctx_quiesce(g4b_ctx* c) {
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
}

int pick_M(int n) {
  static const int kM[] = {1, 3, 5, 7, 9, 11, 13, 15, 17, 21, 25, 33};
  for (int m : kM)
    if (32 * m >= n) return m;
  return 0;
}

static int pick_M16(int n) {
  static const int kM16[] = {5, 7, 9, 11, 13, 15, 17, 21, 25, 33};
  for (int m : kM16)
    if (16 * m >= n) return m;
  return 0;
}

int pick_mode(int n, int precision) {
  const int m32 = pick_M(n);
  if (precision == G4B_FP64 || m32 == 0) return m32;
  const int m16 = pick_M16(n);
  return m16 && 16 * m16 < 32 * m32 ? 100 + m16 : m32;
}

int alt_mode(int n) {
  const int m32 = pick_M(n), m16 = pick_M16(n);
  if (!m32 || !m16) return 0;
  return pick_mode(n, G4B_MIXED) == m32 ? 100 + m16 : m32;
}

int field_set_layout(g4b_field* f, int mode) {
  if (!f) return fail(G4B_ERR_ARG, "field layout: null field");
  if (mode == f->mode) return G4B_OK;
  if (f->precision != G4B_MIXED ||
      (mode != pick_mode(f->ngrid, G4B_MIXED) && mode != alt_mode(f->ngrid)))
    return fail(G4B_ERR_RANGE, "field layout: not a row layout of this grid");
  const int old = f->mode;
  f->mode = mode;
  if (int rc = adi_configure(f)) {
    f->mode = old;
    return rc;
  }
  return G4B_OK;
}

static int encode_store_map(g4b_ctx* ctx, CUtensorMap* map, void* base, int n,
                            int ld, int nslice, size_t cell_bytes, int band,
                            int box_rows) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ctx->encode_fn);
  if (!fn) return fail(G4B_ERR_STATE, "cuTensorMapEncodeTiled unavailable");
  const size_t real = cell_bytes / 2;
  cuuint64_t dims[3] = {(cuuint64_t)2 * n, (cuuint64_t)n, (cuuint64_t)nslice};
  cuuint64_t strides[2] = {(cuuint64_t)ld * cell_bytes,
                           (cuuint64_t)n * ld * cell_bytes};
  cuuint32_t box[3] = {(cuuint32_t)(2 * band), (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map,
                  real == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                            : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  3, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[128];
    snprintf(buf, sizeof buf, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return fail(G4B_ERR_CUDA, buf);
  }
  return G4B_OK;
}

}  // namespace g4b

using namespace g4b;

extern "C" {

const char* g4b_last_error(void) { return t_last_error.c_str(); }

int g4b_version(void) { return 100; }

int g4b_ctx_create(int device, g4b_ctx** out) {
  if (!out) return fail(G4B_ERR_ARG, "g4b_ctx_create: null out");
  *out = nullptr;
  int ndev = 0;
  G4B_CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev)
    return fail(G4B_ERR_ARG, "g4b_ctx_create: device index out of range");
  G4B_CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  G4B_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(G4B_ERR_DEVICE, "g4b_ctx_create: this build targets sm_100a (B200)");
  g4b_ctx* c = new (std::nothrow) g4b_ctx();
  if (!c) return fail(G4B_ERR_NOMEM, "g4b_ctx_create: host allocation");
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "cudaStreamCreateWithFlags");
  }
  c->own_stream = true;
  {
    // keep released stream-ordered blocks in the pool (process-local setting)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  e = cudaMalloc(&c->d_error, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_error, 0, sizeof(int));
  if (e != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return cuda_fail(e, "cudaMalloc(error flag)");
  }
  cudaDriverEntryPointQueryResult q;
  e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &c->encode_fn,
                              cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess) c->encode_fn = nullptr;
  *out = c;
  return G4B_OK;
}

int g4b_ctx_destroy(g4b_ctx* c) {
  if (!c || c->destroyed) return G4B_OK;
  c->destroyed = true;
  ctx_release(c);
  return G4B_OK;
}

int g4b_ctx_set_stream(g4b_ctx* c, void* s) {
  if (!c) return fail(G4B_ERR_ARG, "g4b_ctx_set_stream: null ctx");
  if (s == nullptr) {
    if (!c->own_stream) {
      G4B_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      c->own_stream = true;
    }
    return G4B_OK;
  }
  if (c->own_stream && c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  c->stream = static_cast<cudaStream_t>(s);
  c->own_stream = false;
  return G4B_OK;
}

void* g4b_ctx_get_stream(g4b_ctx* c) { return c ? (void*)c->stream : nullptr; }

int g4b_ctx_synchronize(g4b_ctx* c) {
  if (!c) return fail(G4B_ERR_ARG, "g4b_ctx_synchronize: null ctx");
  G4B_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return read_device_error(c, "g4b_ctx_synchronize");
}

static constexpr size_t kMarkRing = 256;

int g4b_ctx_mark(g4b_ctx* c, uint64_t* ticket) {
  if (!c || !ticket) return fail(G4B_ERR_ARG, "g4b_ctx_mark: null arg");
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  if (c->marks.empty()) {
    c->marks.resize(kMarkRing, nullptr);
    for (auto& e : c->marks) G4B_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const uint64_t t = c->mark_next++;
  G4B_CUDA_TRY(cudaEventRecord(c->marks[t % kMarkRing], c->stream));
  *ticket = t;
  return G4B_OK;
}

int g4b_ctx_mark_query(g4b_ctx* c, uint64_t ticket, int wait, int* done) {
  if (!c || !done) return fail(G4B_ERR_ARG, "g4b_ctx_mark_query: null arg");
  if (ticket >= c->mark_next || c->mark_next - ticket > kMarkRing)
    return fail(G4B_ERR_ARG, "g4b_ctx_mark_query: unknown or recycled ticket");
  cudaEvent_t e = c->marks[ticket % kMarkRing];
  if (wait) {
    G4B_CUDA_TRY(cudaEventSynchronize(e));
    *done = 1;
    return G4B_OK;
  }
  const cudaError_t q = cudaEventQuery(e);
  if (q == cudaErrorNotReady) {
    *done = 0;
    return G4B_OK;
  }
  if (q != cudaSuccess) return cuda_fail(q, "g4b_ctx_mark_query");
  *done = 1;
  return G4B_OK;
}

int g4b_ctx_mem_info(g4b_ctx* c, uint64_t* free_bytes, uint64_t* total_bytes) {
  if (!c || !free_bytes || !total_bytes) return fail(G4B_ERR_ARG, "g4b_ctx_mem_info: null arg");
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  size_t f = 0, t = 0;
  G4B_CUDA_TRY(cudaMemGetInfo(&f, &t));
  // blocks released to the default pool are free for this process too
  cudaMemPool_t pool;
  uint64_t reserved = 0, used = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, c->device) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
      reserved > used)
    f += reserved - used;
  *free_bytes = f;
  *total_bytes = t;
  return G4B_OK;
}

int g4b_ctx_launch_count(g4b_ctx* c, uint64_t* count) {
  if (!c || !count) return fail(G4B_ERR_ARG, "g4b_ctx_launch_count: null arg");
  *count = c->launches.load();
  return G4B_OK;
}

int g4b_ctx_profile(g4b_ctx* c, int enable) {
  if (!c) return fail(G4B_ERR_ARG, "g4b_ctx_profile: null ctx");
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  prof_resolve(c);
  Profiler& p = c->prof;
  if (enable) {
    p.names.clear();
    p.count.clear();
    p.ms.clear();
  }
  p.on = enable != 0;
  return G4B_OK;
}

int g4b_ctx_profile_read(g4b_ctx* c, int max_kernels, char* names, uint64_t* counts,
                         double* total_ms, int* nkernels) {
  if (!c || !nkernels) return fail(G4B_ERR_ARG, "g4b_ctx_profile_read: null arg");
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  prof_resolve(c);
  Profiler& p = c->prof;
  const int n = (int)p.names.size();
  *nkernels = n;
  for (int i = 0; i < n && i < max_kernels; ++i) {
    if (names) {
      std::strncpy(names + 64 * i, p.names[i].c_str(), 63);
      names[64 * i + 63] = 0;
    }
    if (counts) counts[i] = p.count[i];
    if (total_ms) total_ms[i] = p.ms[i];
  }
  return G4B_OK;
}

int g4b_ctx_sm_count(g4b_ctx* c, int* count) {
  if (!c || !count) return fail(G4B_ERR_ARG, "g4b_ctx_sm_count: null arg");
  *count = c->sm_count;
  return G4B_OK;
}

}  // extern "C"

namespace {
// One CTA arrives on an mbarrier announcing 16 bytes that no copy will ever
// deliver (no asynchronous operation targets this barrier), so the phase
// cannot complete: the bounded wait gives up after `limit` polls, sets the
// error word and returns.
__global__ void wait_selftest_kernel(int* err, uint32_t limit, int* arrived) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    g4b::ptx::mbar_init(&bar, 1);
    g4b::ptx::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) g4b::ptx::mbar_expect_tx(&bar, 16u);
  const bool ok = g4b::ptx::mbar_wait_bounded(&bar, 0u, err, limit);
  if (threadIdx.x == 0) *arrived = ok ? 1 : 0;
}
}  // namespace

extern "C" {

int g4b_ctx_selftest_wait(g4b_ctx* c, unsigned spin_limit, int* timed_out) {
  if (!c || !timed_out) return fail(G4B_ERR_ARG, "g4b_ctx_selftest_wait: null arg");
  if (spin_limit == 0 || spin_limit > (1u << 20))
    return fail(G4B_ERR_RANGE, "g4b_ctx_selftest_wait: spin_limit must be in [1, 2^20]");
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  int* d = nullptr;  // the kernel's "arrived" answer
  G4B_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d), sizeof(int), c->stream));
  G4B_CUDA_TRY(cudaMemsetAsync(d, 0xff, sizeof(int), c->stream));
  wait_selftest_kernel<<<1, 32, 0, c->stream>>>(c->d_error, spin_limit, d);
  count_launch(c);
  const cudaError_t le = cudaGetLastError();
  int arrived = -1;
  cudaError_t e = le;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&arrived, d, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(d, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "g4b_ctx_selftest_wait");
  *timed_out = arrived == 0 ? 1 : 0;
  // the kernel's timeout is reported (and cleared) like any device error
  return read_device_error(c, "g4b_ctx_selftest_wait");
}

// ------------------------------------------------------------------ field ---

int g4b_field_create(g4b_ctx* c, int nslice, int ngrid, double gridmax,
                     double xlambda, int harm, int precision, int low_memory,
                     g4b_field** out) {
  if (!c || !out) return fail(G4B_ERR_ARG, "g4b_field_create: null arg");
  *out = nullptr;
  if (nslice <= 0 || ngrid < 2 || !(gridmax > 0) || !(xlambda > 0) || harm < 1)
    return fail(G4B_ERR_ARG, "g4b_field_create: bad dimensions");
  if (precision != G4B_FP64 && precision != G4B_MIXED)
    return fail(G4B_ERR_ARG, "g4b_field_create: unknown precision");
  if (pick_M(ngrid) == 0)
    return fail(G4B_ERR_RANGE, "g4b_field_create: ngrid above 1056 is not supported");
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  g4b_field* f = new (std::nothrow) g4b_field();
  if (!f) return fail(G4B_ERR_NOMEM, "g4b_field_create: host allocation");
  f->ctx = c;
  ctx_retain(c);
  f->nslice = nslice;
  f->ngrid = ngrid;
  f->harm = harm;
  f->precision = precision;
  f->low_memory = low_memory ? 1 : 0;
  f->gridmax = gridmax;
  f->dgrid = 2.0 * gridmax / (double)(ngrid - 1);  // Field::init, Field.cpp:61
  f->xlambda = xlambda;
  f->xks = 4.0 * std::asin(1.0) / xlambda;          // Field::init, Field.cpp:78
  f->cell_bytes = precision == G4B_FP64 ? 16 : 8;
  f->ld = precision == G4B_FP64 ? ngrid : ngrid + (ngrid & 1);
  f->mode = pick_mode(ngrid, precision);
  f->band_rows = precision == G4B_FP64 ? 9 : 10;  // rows per ADI band (both row layouts)
  // TMA store boxes of <= 256 rows; a multiple of 8 rows keeps every box's
  // shared-memory source 128-byte aligned (W * cell * 8 is a multiple of 128).
  f->store_nbox = (ngrid + 255) / 256;
  f->store_box_rows = ((ngrid + f->store_nbox - 1) / f->store_nbox + 7) / 8 * 8;
  const size_t bytes = (size_t)nslice * ngrid * f->ld * f->cell_bytes + 256;
  cudaError_t e = dev_alloc(c, &f->a, bytes);
  if (e == cudaSuccess) e = dev_alloc(c, &f->b, bytes);
  if (e == cudaSuccess) e = dev_alloc(c, &f->src, bytes);
  if (e == cudaSuccess) e = dev_alloc(c, (void**)&f->desc, nslice * sizeof(int4));
  if (e == cudaSuccess) e = cudaMemsetAsync(f->desc, 0, nslice * sizeof(int4), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(f->a, 0, bytes, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(f->b, 0, bytes, c->stream);
  if (e != cudaSuccess) {
    g4b_field_destroy(f);
    return cuda_fail(e, "g4b_field_create: device allocation");
  }
  f->bytes = 3 * bytes;
  int rc = encode_store_map(c, &f->tm_store_b, f->b, ngrid, f->ld, nslice,
                            f->cell_bytes, f->band_rows, f->store_box_rows);
  if (rc == G4B_OK)
    rc = encode_store_map(c, &f->tm_store_a, f->a, ngrid, f->ld, nslice,
                          f->cell_bytes, f->band_rows, f->store_box_rows);
  if (rc != G4B_OK) {
    g4b_field_destroy(f);
    return rc;
  }
  *out = f;
  return G4B_OK;
}

int g4b_field_destroy(g4b_field* f) {
  if (!f) return G4B_OK;
  ctx_quiesce(f->ctx);
  dev_free(f->ctx, f->a);
  dev_free(f->ctx, f->b);
  dev_free(f->ctx, f->src);
  dev_free(f->ctx, f->desc);
  ctx_release(f->ctx);
  delete f;
  return G4B_OK;
}

// Host (re,im) doubles [slice][iy][ix] <-> device cells [slice][iy][ld].
// Row-wise conversions between FP64 cells (rows of n, unpadded) and the
// mixed form's complex64 rows (pitch ld).
__global__ void cells_f64_to_f32(const double2* src, float2* dst, int n, int ld, size_t rows) {
  const size_t total = rows * (size_t)n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / n, k = i - r * n;
    const double2 v = src[i];
    dst[r * ld + k] = make_float2((float)v.x, (float)v.y);
  }
}

__global__ void cells_f32_to_f64(const float2* src, double2* dst, int n, int ld, size_t rows) {
  const size_t total = rows * (size_t)n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / n, k = i - r * n;
    const float2 v = src[r * ld + k];
    dst[i] = make_double2((double)v.x, (double)v.y);
  }
}

static int field_copy(g4b_field* f, double* host, bool upload) {
  g4b_ctx* c = f->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  const size_t n = f->ngrid;
  const size_t rows = (size_t)f->nslice * n;
  if (f->precision == G4B_FP64) {
    // pitch == row length: one contiguous copy
    const size_t bytes = rows * n * 16;
    if (upload)
      G4B_CUDA_TRY(cudaMemcpyAsync(f->a, host, bytes, cudaMemcpyHostToDevice, c->stream));
    else
      G4B_CUDA_TRY(cudaMemcpyAsync(host, f->a, bytes, cudaMemcpyDeviceToHost, c->stream));
    G4B_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return G4B_OK;
  }
  // mixed: FP64 rows cross the bus and are converted on the device, in
  // chunks of whole rows through a staging buffer
  const size_t row_bytes = n * 16;
  const size_t chunk_rows = std::max<size_t>(1, std::min(rows, (size_t)(64u << 20) / row_bytes));
  double2* stage = nullptr;
  G4B_CUDA_TRY(dev_alloc(c, (void**)&stage, chunk_rows * row_bytes));
  cudaError_t e = cudaSuccess;
  float2* a = static_cast<float2*>(f->a);
  for (size_t r0 = 0; r0 < rows && e == cudaSuccess; r0 += chunk_rows) {
    const size_t nr = std::min(chunk_rows, rows - r0);
    const unsigned grid = (unsigned)std::min<size_t>((nr * n + 255) / 256, 65535u * 32u);
    if (upload) {
      e = cudaMemcpyAsync(stage, host + r0 * 2 * n, nr * row_bytes, cudaMemcpyHostToDevice,
                          c->stream);
      if (e == cudaSuccess)
        cells_f64_to_f32<<<grid, 256, 0, c->stream>>>(stage, a + r0 * f->ld, (int)n, f->ld, nr);
    } else {
      cells_f32_to_f64<<<grid, 256, 0, c->stream>>>(a + r0 * f->ld, stage, (int)n, f->ld, nr);
      e = cudaMemcpyAsync(host + r0 * 2 * n, stage, nr * row_bytes, cudaMemcpyDeviceToHost,
                          c->stream);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  dev_free(c, stage);
  const cudaError_t es = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "field copy");
  if (es != cudaSuccess) return cuda_fail(es, "field copy");
  return G4B_OK;
}

int g4b_field_upload(g4b_field* f, const double* host) {
  if (!f || !host) return fail(G4B_ERR_ARG, "g4b_field_upload: null arg");
  return field_copy(f, const_cast<double*>(host), true);
}

int g4b_field_download(g4b_field* f, double* host) {
  if (!f || !host) return fail(G4B_ERR_ARG, "g4b_field_download: null arg");
  return field_copy(f, host, false);
}

int g4b_field_set_first(g4b_field* f, int first) {
  if (!f || first < 0 || first >= f->nslice)
    return fail(G4B_ERR_ARG, "g4b_field_set_first: bad argument");
  f->first = first;
  return G4B_OK;
}

int g4b_field_get_first(g4b_field* f, int* first) {
  if (!f || !first) return fail(G4B_ERR_ARG, "g4b_field_get_first: null arg");
  *first = f->first;
  return G4B_OK;
}

int g4b_field_device_bytes(g4b_field* f, uint64_t* bytes) {
  if (!f || !bytes) return fail(G4B_ERR_ARG, "g4b_field_device_bytes: null arg");
  *bytes = f->bytes;
  return G4B_OK;
}

// ------------------------------------------------------------------- beam ---

static constexpr int kChunk = 256;  // particles per push CTA

int g4b_beam_create(g4b_ctx* c, int nslice, const int64_t* off, int precision,
                    double gamma_ref, g4b_beam** out) {
  if (!c || !out || !off) return fail(G4B_ERR_ARG, "g4b_beam_create: null arg");
  *out = nullptr;
  if (nslice <= 0) return fail(G4B_ERR_ARG, "g4b_beam_create: nslice <= 0");
  if (precision != G4B_FP64)
    return fail(G4B_ERR_ARG, "g4b_beam_create: this entry point holds FP64 state");
  if (off[0] != 0) return fail(G4B_ERR_ARG, "g4b_beam_create: slice_offsets[0] != 0");
  for (int s = 0; s < nslice; ++s)
    if (off[s + 1] < off[s])
      return fail(G4B_ERR_ARG, "g4b_beam_create: slice_offsets not monotonic");
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  g4b_beam* b = new (std::nothrow) g4b_beam();
  if (!b) return fail(G4B_ERR_NOMEM, "g4b_beam_create: host allocation");
  b->ctx = c;
  ctx_retain(c);
  b->nslice = nslice;
  b->precision = precision;
  b->gamma_ref = gamma_ref;
  b->npart = off[nslice];
  b->h_off.assign(off, off + nslice + 1);
  std::vector<int4> chunks;
  for (int s = 0; s < nslice; ++s) {
    b->max_slice_np = std::max<int64_t>(b->max_slice_np, off[s + 1] - off[s]);
    for (int64_t p = off[s]; p < off[s + 1]; p += kChunk) {
      const int64_t e = std::min<int64_t>(p + kChunk, off[s + 1]);
      chunks.push_back(make_int4(s, (int)(p & 0x7fffffff), (int)(e - p),
                                 (int)(p >> 31)));
    }
  }
  b->nchunk = (int)chunks.size();
  const size_t np = (size_t)std::max<int64_t>(b->npart, 1);
  cudaError_t e = cudaSuccess;
  double** arrs[6] = {&b->x, &b->y, &b->px, &b->py, &b->gamma, &b->theta};
  for (double** a : arrs)
    if (e == cudaSuccess) e = dev_alloc(c, (void**)a, np * sizeof(double));
  if (e == cudaSuccess) e = dev_alloc(c, (void**)&b->d_off, (nslice + 1) * sizeof(int64_t));
  if (e == cudaSuccess) e = dev_alloc(c, (void**)&b->d_current, nslice * sizeof(double));
  if (e == cudaSuccess) e = dev_alloc(c, (void**)&b->d_eloss, nslice * sizeof(double));
  if (e == cudaSuccess) e = dev_alloc(c, (void**)&b->d_scl, nslice * sizeof(double));
  if (e == cudaSuccess)
    e = dev_alloc(c, (void**)&b->d_chunks, std::max(1, b->nchunk) * sizeof(int4));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_off, off, (nslice + 1) * sizeof(int64_t),
                        cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && b->nchunk)
    e = cudaMemcpyAsync(b->d_chunks, chunks.data(), chunks.size() * sizeof(int4),
                        cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_current, 0, nslice * sizeof(double), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_eloss, 0, nslice * sizeof(double), c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    g4b_beam_destroy(b);
    return cuda_fail(e, "g4b_beam_create: device allocation");
  }
  b->bytes = np * 6 * sizeof(double) + (nslice + 1) * 8 + 3 * nslice * 8 +
             chunks.size() * sizeof(int4);
  *out = b;
  return G4B_OK;
}

int g4b_beam_destroy(g4b_beam* b) {
  if (!b) return G4B_OK;
  ctx_quiesce(b->ctx);
  void* ptrs[] = {b->x, b->y, b->px, b->py, b->gamma, b->theta, b->d_off,
                  b->d_current, b->d_eloss, b->d_scl, b->d_chunks, b->d_pez};
  for (void* p : ptrs) dev_free(b->ctx, p);
  ctx_release(b->ctx);
  delete b;
  return G4B_OK;
}

int g4b_beam_upload(g4b_beam* b, const double* x, const double* y,
                    const double* px, const double* py, const double* gamma,
                    const double* theta) {
  if (!b || !x || !y || !px || !py || !gamma || !theta)
    return fail(G4B_ERR_ARG, "g4b_beam_upload: null arg");
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  const size_t bytes = (size_t)b->npart * sizeof(double);
  const double* src[6] = {x, y, px, py, gamma, theta};
  double* dst[6] = {b->x, b->y, b->px, b->py, b->gamma, b->theta};
  for (int i = 0; i < 6 && bytes; ++i)
    G4B_CUDA_TRY(cudaMemcpyAsync(dst[i], src[i], bytes, cudaMemcpyHostToDevice, c->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G4B_OK;
}

int g4b_beam_download(g4b_beam* b, double* x, double* y, double* px, double* py,
                      double* gamma, double* theta) {
  if (!b) return fail(G4B_ERR_ARG, "g4b_beam_download: null beam");
  g4b_ctx* c = b->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  const size_t bytes = (size_t)b->npart * sizeof(double);
  double* dst[6] = {x, y, px, py, gamma, theta};
  const double* src[6] = {b->x, b->y, b->px, b->py, b->gamma, b->theta};
  for (int i = 0; i < 6 && bytes; ++i)
    if (dst[i])
      G4B_CUDA_TRY(cudaMemcpyAsync(dst[i], src[i], bytes, cudaMemcpyDeviceToHost, c->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return G4B_OK;
}

int g4b_beam_set_current(g4b_beam* b, const double* current) {
  if (!b || !current) return fail(G4B_ERR_ARG, "g4b_beam_set_current: null arg");
  G4B_CUDA_TRY(cudaSetDevice(b->ctx->device));
  G4B_CUDA_TRY(cudaMemcpyAsync(b->d_current, current, b->nslice * sizeof(double),
                               cudaMemcpyHostToDevice, b->ctx->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(b->ctx->stream));
  return G4B_OK;
}

int g4b_beam_set_eloss(g4b_beam* b, const double* eloss) {
  if (!b) return fail(G4B_ERR_ARG, "g4b_beam_set_eloss: null beam");
  G4B_CUDA_TRY(cudaSetDevice(b->ctx->device));
  if (!eloss) {
    G4B_CUDA_TRY(cudaMemsetAsync(b->d_eloss, 0, b->nslice * sizeof(double), b->ctx->stream));
  } else {
    G4B_CUDA_TRY(cudaMemcpyAsync(b->d_eloss, eloss, b->nslice * sizeof(double),
                                 cudaMemcpyHostToDevice, b->ctx->stream));
  }
  G4B_CUDA_TRY(cudaStreamSynchronize(b->ctx->stream));
  return G4B_OK;
}

int g4b_beam_device_bytes(g4b_beam* b, uint64_t* bytes) {
  if (!b || !bytes) return fail(G4B_ERR_ARG, "g4b_beam_device_bytes: null arg");
  *bytes = b->bytes;
  return G4B_OK;
}

// --------------------------------------------------------------- slippage ---
// ControlCUDA::applySlippage, single rank (src/Core/ControlCUDA.cpp:148-252):
// the field never moves; `first` rotates and the plane entering the window is
// zeroed, so the result is bit-exact by construction.
int g4b_slippage(g4b_field* f, double shift, double sample, int time_run,
                 int periodic, double* accuslip, int* nshift) {
  if (!f || !accuslip) return fail(G4B_ERR_ARG, "g4b_slippage: null arg");
  if (nshift) *nshift = 0;
  if (!time_run) return G4B_OK;
  g4b_ctx* c = f->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  *accuslip += shift;
  const int ns = f->nslice;
  const size_t plane_bytes = (size_t)f->ngrid * f->ld * f->cell_bytes;
  int count = 0;
  int direction = 1;
  while (std::fabs(*accuslip) > sample * 0.8) {
    direction = *accuslip < 0 ? -1 : 1;
    *accuslip -= sample * direction;
    int last = (f->first + ns - 1) % ns;
    if (direction < 0) last = (last + 1) % ns;
    if (!periodic) {
      G4B_CUDA_TRY(cudaMemsetAsync(static_cast<char*>(f->a) + plane_bytes * last, 0,
                                   plane_bytes, c->stream));
    }
    f->first = last;
    if (direction < 0) f->first = (last + 1) % ns;
    ++count;
  }
  if (nshift) *nshift = count;
  return G4B_OK;
}

// One storage plane (ngrid rows of ld cells, the state's precision) to / from
// device memory, on the context's stream: the pack / unpack of the slippage
// plane exchange between ranks (src/Core/ControlCUDA.cpp:27-66, :195-235).
int g4b_field_plane_bytes(g4b_field* f, size_t* bytes) {
  if (!f || !bytes) return fail(G4B_ERR_ARG, "g4b_field_plane_bytes: null arg");
  *bytes = (size_t)f->ngrid * f->ld * f->cell_bytes;
  return G4B_OK;
}

int g4b_field_plane_out(g4b_field* f, int slice, void* dst_device) {
  if (!f || !dst_device) return fail(G4B_ERR_ARG, "g4b_field_plane_out: null arg");
  if (slice < 0 || slice >= f->nslice) return fail(G4B_ERR_RANGE, "g4b_field_plane_out: slice");
  G4B_CUDA_TRY(cudaSetDevice(f->ctx->device));
  const size_t pb = (size_t)f->ngrid * f->ld * f->cell_bytes;
  G4B_CUDA_TRY(cudaMemcpyAsync(dst_device, static_cast<const char*>(f->a) + pb * slice, pb,
                               cudaMemcpyDeviceToDevice, f->ctx->stream));
  return G4B_OK;
}

int g4b_field_plane_in(g4b_field* f, int slice, const void* src_device) {
  if (!f || !src_device) return fail(G4B_ERR_ARG, "g4b_field_plane_in: null arg");
  if (slice < 0 || slice >= f->nslice) return fail(G4B_ERR_RANGE, "g4b_field_plane_in: slice");
  G4B_CUDA_TRY(cudaSetDevice(f->ctx->device));
  const size_t pb = (size_t)f->ngrid * f->ld * f->cell_bytes;
  G4B_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(f->a) + pb * slice, src_device, pb,
                               cudaMemcpyDeviceToDevice, f->ctx->stream));
  return G4B_OK;
}

int g4b_field_zero_plane(g4b_field* f, int slice) {
  if (!f) return fail(G4B_ERR_ARG, "g4b_field_zero_plane: null arg");
  if (slice < 0 || slice >= f->nslice) return fail(G4B_ERR_RANGE, "g4b_field_zero_plane: slice");
  G4B_CUDA_TRY(cudaSetDevice(f->ctx->device));
  const size_t pb = (size_t)f->ngrid * f->ld * f->cell_bytes;
  G4B_CUDA_TRY(cudaMemsetAsync(static_cast<char*>(f->a) + pb * slice, 0, pb, f->ctx->stream));
  return G4B_OK;
}

}  // extern "C"
