// g4b_internal.cuh -- private state and device helpers of the sm_100a core.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/g4b.h"

namespace g4b {

// ---------------------------------------------------------------- errors ----
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);

#define G4B_CUDA_TRY(expr)                                  \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return ::g4b::cuda_fail(_e, #expr); \
  } while (0)

// Device-side error flag bits (written by kernels, read by the host).
enum : int {
  kErrWaitTimeout = 1,     // an mbarrier wait exceeded its iteration bound
  kErrFixedRange = 2,      // a deposit value fell outside its fixed-point range
  kErrBadSlice = 4,        // a particle index/slice outside the state
};

// Spin bound of every mbarrier wait: far above any legitimate wait.
constexpr uint32_t kWaitSpinLimit = 1u << 26;

// ----------------------------------------------------------------- state ----
struct TensorMapEncoder;

}  // namespace g4b

namespace g4b {
// Per-kernel CUDA-event timing on the context's stream (off by default).
struct Profiler {
  bool on = false;
  struct Pending {
    int name;
    cudaEvent_t a, b;
  };
  std::vector<std::string> names;
  std::vector<uint64_t> count;
  std::vector<double> ms;
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t open_a = nullptr;
  int open_name = -1;
};
}  // namespace g4b

struct g4b_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 0;
  std::atomic<uint64_t> launches{0};
  int* d_error = nullptr;  // device error flag (bit set, see kErr*)
  void* encode_fn = nullptr;  // cuTensorMapEncodeTiled
  g4b::Profiler prof;
  // lifetime: the handle plus every object created on it hold a reference;
  // g4b_ctx_destroy releases the handle's, so objects may be destroyed after
  // their context (the struct lives until the last reference goes)
  std::atomic<int> refs{1};
  bool destroyed = false;
  // stream marks (g4b_ctx_mark): a ring of events, ticket % size
  std::vector<cudaEvent_t> marks;
  uint64_t mark_next = 0;
};

struct g4b_field {
  g4b_ctx* ctx = nullptr;
  int nslice = 0, ngrid = 0, ld = 0;  // ld: row pitch in cells
  int harm = 1, precision = G4B_FP64, low_memory = 0, first = 0;
  double gridmax = 0, dgrid = 0, xlambda = 0, xks = 0;
  size_t cell_bytes = 16;   // sizeof(complex) on the device
  void* a = nullptr;        // state, natural layout [slice][iy][ld]
  void* b = nullptr;        // pass-Y right-hand side, transposed [slice][ix][ld]
  void* src = nullptr;      // source: compact per-slice tiles (n*ld cells reserved each)
  int4* desc = nullptr;     // per-slice source tile (x0, y0, width, height)
  // TMA tensor maps for the transposed stores of the two ADI passes.
  CUtensorMap tm_store_b;   // pass X writes b
  CUtensorMap tm_store_a;   // pass Y writes a
  int store_box_rows = 0;   // rows per TMA store box
  int store_nbox = 0;       // boxes per band
  int band_rows = 0;        // W: rows per CTA (one or two per warp)
  int mode = 0;             // ADI row layout (pick_mode)
  uint64_t bytes = 0;
};

struct g4b_beam {
  g4b_ctx* ctx = nullptr;
  int nslice = 0, precision = G4B_FP64;
  int64_t npart = 0;
  double gamma_ref = 0;
  std::vector<int64_t> h_off;
  int64_t* d_off = nullptr;
  // FP64 state
  double *x = nullptr, *y = nullptr, *px = nullptr, *py = nullptr;
  double *gamma = nullptr, *theta = nullptr;
  double* d_current = nullptr;
  double* d_eloss = nullptr;
  double* d_scl = nullptr;           // per-slice source scale
  // per-particle loss (space charge + slice loss); the push reads it in
  // place of d_eloss while use_pez is set
  double* d_pez = nullptr;
  int use_pez = 0;
  // CTA work chunks: (slice, begin, end) over the particle index space.
  int nchunk = 0;
  int4* d_chunks = nullptr;          // x = slice, y = begin lo, z = end lo, w = hi bits
  int64_t max_slice_np = 0;
  uint64_t bytes = 0;
};

struct g4b_adi {
  g4b_ctx* ctx = nullptr;
  int ngrid = 0;
  double delz = 0, dgrid = 0, xks = 0, r = 0;
  int M = 0;                 // elements per lane (odd), 32-lane rows (FP64 fields)
  int mode32 = 0;            // row layout of FP32 fields (pick_mode)
  int mode32_alt = 0;        // the other FP32 row layout (alt_mode), 0 if none
  // Tables in lane-minor order, complex (double2) and their FP32 copies.
  double2* d_tab64 = nullptr;   // [3][M][32]: cbet, G, H ; then [2][5][32] scans
  float2* d_tab32 = nullptr;
  float2* d_tab32_alt = nullptr;  // tables of mode32_alt
  bool ready = false;
};

namespace g4b {

// Context lifetime helpers (see g4b_ctx::refs).
inline void ctx_retain(g4b_ctx* c) { c->refs++; }
void ctx_release(g4b_ctx* c);
// Make the context's device current and drain its stream, if it is still open.
void ctx_quiesce(g4b_ctx* c);

// Launch bookkeeping: every kernel launch goes through this.
inline void count_launch(g4b_ctx* ctx, int n = 1) { ctx->launches += n; }

// Brackets one kernel launch with profiler events when profiling is on:
//   { LaunchScope ls(ctx, "name"); kernel<<<...>>>(...); }
void prof_begin(g4b_ctx* ctx, const char* name);
void prof_end(g4b_ctx* ctx);
struct LaunchScope {
  g4b_ctx* c;
  LaunchScope(g4b_ctx* ctx, const char* name) : c(ctx) { prof_begin(ctx, name); }
  ~LaunchScope() {
    prof_end(c);
    count_launch(c);
  }
};

// Stream-ordered device memory from the device's default pool: allocation and
// release are ordered on the context's stream, so neither waits for other
// streams' work (cudaFree would synchronise the whole device); released
// blocks stay in the pool for reuse.
cudaError_t dev_alloc(g4b_ctx* ctx, void** p, size_t bytes);
// slice scale + deterministic FP64 deposition into f's compact source tiles
int fp64_deposit(g4b_field* f, g4b_beam* b, const g4b_step* st, double fc);
void dev_free(g4b_ctx* ctx, void* p);

int check_launch(g4b_ctx* ctx, const char* what);
int read_device_error(g4b_ctx* ctx, const char* what);

// Launches kern with programmatic stream serialization: it may start while
// the preceding kernel of its stream drains (in a captured graph, a
// programmatic edge), and waits for that kernel's completion and writes in
// ptx::pdl_wait before its first access to global memory (a load whose
// address needs no earlier load, read through the read-only path, could be
// issued before the wait: such data is read with plain loads).
#if defined(__CUDACC__)
template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*kern)(P...), unsigned grid, unsigned block, size_t smem,
                              cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<A&&>(args)...);
}
#endif

struct AdiPassArgs {
  const void* in;      // pass X: field (natural); pass Y: R' (transposed)
  const void* src;     // pass X only: compact per-slice source tiles; nullptr = none
  const int4* desc;    // per-slice source tile (x0, y0, width, height); width 0 = none
  size_t src_cap;      // cells reserved per slice in `src`
  const void* tab;     // lane-minor tables of this precision
  int n, ld, nband;
  int out_off;         // byte offset of the output staging tile (pass X: 0, over the input)
  int box_rows, nbox;  // TMA store boxes per band
  double r;
  int* err;
  // pass Y extras (fused form): planes [zero_start, zero_start+zero_count)
  // (mod nslice) are written as zeros (the slippage of this step), and, when
  // diag is non-null, each CTA writes 9 partial sums of the plane it solved
  // (power, x1, x2, y1, y2, sum re, sum im, centre re, centre im) to
  // diag[(slice * nband + band) * 9].
  int nslice, zero_start, zero_count;
  double* diag;
};

// Shared ADI entry used by the drop-in and the fused path.  The extras of the
// fused form (may be null): zero the planes the step's slippage zeroes, and
// write per-band field-diagnostic partial sums (9 per band).
struct AdiYExtras {
  int zero_start, zero_count;
  double* diag;
};
int adi_run(g4b_adi* adi, g4b_field* f, const void* src, const int4* desc,
            const AdiYExtras* ex);
// The two passes of one field step, resolved but not launched.
struct AdiPlan {
  AdiPassArgs x, y;
  const CUtensorMap* tm_x;  // host copies of the field's store maps
  const CUtensorMap* tm_y;
  size_t smem_x, smem_y;
  size_t smem_x_max;        // pass X with a source tile (the largest)
  int M, precision;
  unsigned grid;            // CTAs per pass: nslice * nband
};
int adi_plan(g4b_adi* adi, g4b_field* f, const void* src, const int4* desc,
             const AdiYExtras* ex, AdiPlan& plan);
int adi_launch(g4b_field* f, const AdiPlan& plan);
// Batched passes (mixed precision): items[i] = (run, slice, band, 0) of the
// runs whose ADI uses M elements per lane; args / maps indexed by run.
struct AdiBatchArgs {
  const AdiPassArgs* args;
  const CUtensorMap* maps;
  const int4* items;
  const int* nitems;
};
int adi_batch_launch(g4b_ctx* c, cudaStream_t st, int M, bool px, const AdiBatchArgs& b, size_t smem,
                     int grid);
// Sets the launch attributes of the ADI kernels for this field's grid (done
// before any stream capture).
int adi_configure(g4b_field* f);

// Lane-minor table offsets (in complex elements) for rows of L lanes with M
// elements each.
inline size_t tab_cbet(int M, int L) { (void)M; (void)L; return 0; }
inline size_t tab_G(int M, int L) { return (size_t)M * L; }
inline size_t tab_H(int M, int L) { return (size_t)2 * M * L; }
inline size_t tab_scanF(int M, int L) { return (size_t)3 * M * L; }
inline size_t tab_scanB(int M, int L) { return (size_t)3 * M * L + 5 * L; }
inline size_t tab_S(int M, int L) { return (size_t)3 * M * L + 10 * L; }
inline size_t tab_total(int M, int L) { return (size_t)4 * M * L + 10 * L; }

// Elements per lane for 32-lane rows (0 if n > 1056).
int pick_M(int n);
// Row layout ("mode") of the ADI kernels for a grid of n: M for 32-lane rows,
// 100 + M for 16-lane rows (FP32 fields whose rows fit 16 M slots more
// closely than 32 M).
int pick_mode(int n, int precision);
// The other FP32 row layout of an n-point row (32 lanes <-> 16 lanes), 0 if none.
int alt_mode(int n);
// Switches an FP32 field between its two row layouts (pick_mode / alt_mode).
// The solve is the same linear system; its FP32 rounding depends on the layout.
int field_set_layout(g4b_field* f, int mode);
inline int mode_M(int mode) { return mode % 100; }
inline int mode_L(int mode) { return mode >= 100 ? 16 : 32; }

}  // namespace g4b

// ------------------------------------------------------------ PTX helpers ---
#if defined(__CUDACC__)
namespace g4b {
namespace ptx {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Compensated FP64 accumulation (Neumaier's variant of Kahan summation): s
// holds the running sum, c the rounding errors of its additions (TwoSum), so
// that s + c carries the sum to about twice FP64 precision independently of
// the number of terms.
__device__ __forceinline__ void csum_add(double& s, double& c, double x) {
  const double t = s + x;
  c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
  s = t;
}
// Combine another compensated partial (s2, c2) into (s, c).
__device__ __forceinline__ void csum_merge(double& s, double& c, double s2, double c2) {
  csum_add(s, c, s2);
  c += c2;
}
// Butterfly reduction of compensated partials over the lanes of width-w groups.
__device__ __forceinline__ void csum_warp(double& s, double& c, int width) {
  for (int o = width / 2; o > 0; o >>= 1) {
    const double s2 = __shfl_xor_sync(0xffffffffu, s, o);
    const double c2 = __shfl_xor_sync(0xffffffffu, c, o);
    csum_merge(s, c, s2, c2);
  }
}

// Bounded wait: returns false (and sets the device error flag) if the phase
// did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  int* err_flag,
                                                  uint32_t limit = kWaitSpinLimit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
  }
  atomicOr(err_flag, kErrWaitTimeout);
  return false;
}

// 1-D bulk copy global -> shared, completing on an mbarrier.  Both addresses
// 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem,
                                         uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Tensor store shared -> global (3-D box), bulk-group completion.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map,
                                             const void* src_smem, int x, int y,
                                             int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group "
      "[%0, {%2, %3, %4}], [%1];" ::"l"(map),
      "r"(smem_u32(src_smem)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// Make a tensor map written through the generic proxy (host copy into
// global memory) visible to the tensor-map proxy before its first use.
__device__ __forceinline__ void fence_tensormap_acquire(const void* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

// Programmatic dependent launch (launch_pdl): block until the preceding
// kernel of the stream has completed and its writes are visible (returns at
// once in a kernel launched without the attribute).  No kernel triggers its
// dependents early: they launch as its last CTAs exit, which hides the
// launch latency and the ramp-up, not the tail.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_read0() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait0() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

}  // namespace ptx
}  // namespace g4b
#endif
