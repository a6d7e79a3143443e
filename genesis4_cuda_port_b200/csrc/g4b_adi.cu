// g4b_adi.cu -- ADI field solver (FieldSolverADICUDA) for sm_100a.
//
// One field step = deposition + two fused half-step kernels:
//
//   pass X : for a band of W rows of one slice, 1-D bulk copies stage rows
//            r0-1 .. r0+W of the field and rows r0 .. r0+W-1 of the source in
//            shared memory; each warp forms R = u + i r d2y(u) + S for its row,
//            solves (1 - i r d2x) u' = R, and immediately forms the second
//            half-step's right-hand side R' = u' + i r d2x(u') + S (its
//            Laplacian runs along the row just solved).  R' is written
//            transposed ([slice][ix][iy]) through a TMA tensor store.
//   pass Y : each warp loads one contiguous row of R' (a column of the plane),
//            solves (1 - i r d2y) u'' = R' and writes u'' transposed back into
//            the natural layout.
//
// The tridiagonal solve is the reference's Thomas algorithm
// (src/Core/FieldSolverADICUDA.cpp:222-277) written as two first-order linear
// recurrences, y_k = cbet_k R_k + q_k y_{k-1} and u_k = y_k + s_k u_{k+1}
// with q_k = s_k = i r cbet_k, evaluated by a warp: every lane runs the
// recurrence over its own M consecutive elements, the lane carries are
// combined by a 5-step Kogge-Stone scan of affine maps, and each lane adds
// its carry times a precomputed product of coefficients.  All coefficients
// (cbet, prefix/suffix products, scan multipliers) depend only on ngrid and r
// and are computed once on the host in FP64 (FieldSolverADICUDA::init,
// :821-902).
#include <algorithm>
#include <cmath>
#include <complex>
#include <new>

#include <atomic>

#include "g4b_internal.cuh"

namespace g4b {

template <typename T> struct CT;
template <> struct CT<double> { using type = double2; };
template <> struct CT<float> { using type = float2; };

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }

// a + b*c
template <typename C>
__device__ __forceinline__ C cfma(C b, C c, C a) {
  C r;
  r.x = fma(b.x, c.x, fma(-b.y, c.y, a.x));
  r.y = fma(b.x, c.y, fma(b.y, c.x, a.y));
  return r;
}

// b*c with the fused roundings written out (the same bits in every kernel)
template <typename C>
__device__ __forceinline__ C cmul(C b, C c) {
  C r;
  r.x = fma(b.x, c.x, -(b.y * c.y));
  r.y = fma(b.x, c.y, b.y * c.x);
  return r;
}

// shuffles within groups of L lanes (L = 32: the warp; L = 16: its halves)
template <int L, typename C>
__device__ __forceinline__ C shfl_up_c(C v, int d) {
  v.x = __shfl_up_sync(0xffffffffu, v.x, d, L);
  v.y = __shfl_up_sync(0xffffffffu, v.y, d, L);
  return v;
}

template <int L, typename C>
__device__ __forceinline__ C shfl_down_c(C v, int d) {
  v.x = __shfl_down_sync(0xffffffffu, v.x, d, L);
  v.y = __shfl_down_sync(0xffffffffu, v.y, d, L);
  return v;
}


// ------------------------------------------------------ row arithmetic ---
// Forced inline into the single-run and the batched pass kernels: the same
// operations in the same order, hence the same bits, in every kernel.
// Tables of a row layout (L lanes of M elements), lane-minor:
//   cbet [M][L], G prefix products [M][L], H suffix products [M][L],
//   forward scan multipliers [5][L], backward scan multipliers [5][L],
//   S: s_k = i r cbet_k (0 at the last row) [M][L].
template <int M, int L, typename C> struct RowTabs {
  const C *cb, *G, *H, *F, *B, *S;
  __device__ __forceinline__ explicit RowTabs(const C* tab)
      : cb(tab), G(tab + M * L), H(tab + 2 * M * L), F(tab + 3 * M * L),
        B(tab + 3 * M * L + 5 * L), S(tab + 3 * M * L + 10 * L) {}
};

// Pass X right-hand side of the band row at tile slot row + 1 (neighbours at
// slots row and row + 2): R = u + i r d2y(u) + S
// (src/Core/FieldSolverADICUDA.cpp:197-220); elements j >= jn are zero.
template <typename T, int M, typename C>
__device__ __forceinline__ void px_rhs(C (&v)[M], const C* tile, int ld, int row, int gl, int jn,
                                       T r, unsigned long long smask, const C* srow) {
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int k = gl * M + j;
    C R = C{0, 0};
    if (j < jn) {
      const C u = tile[(row + 1) * ld + k];
      const C up = tile[(row + 2) * ld + k];
      const C dn = tile[row * ld + k];
      const T lr = fma((T)-2, u.x, up.x + dn.x);
      const T li = fma((T)-2, u.y, up.y + dn.y);
      R.x = fma(-r, li, u.x);
      R.y = fma(r, lr, u.y);
      if ((smask >> j) & 1ull) R = cadd(R, srow[k]);
    }
    v[j] = R;
  }
}

// Local part of the forward recurrence y_k = cbet_k (R_k + i r y_{k-1}) over
// lane gl's elements, with a zero carry in.
template <typename T, int M, int L, typename C>
__device__ __forceinline__ void fwd_local(C (&v)[M], const RowTabs<M, L, C>& tb, int gl, T r) {
  v[0] = cmul(__ldg(&tb.cb[gl]), v[0]);
#pragma unroll
  for (int j = 1; j < M; ++j) {
    const C cb = __ldg(&tb.cb[j * L + gl]);
    C t;
    t.x = fma(-r, v[j - 1].y, v[j].x);
    t.y = fma(r, v[j - 1].x, v[j].y);
    v[j] = cmul(cb, t);
  }
}

// Local part of the backward recurrence u_k = y_k + s_k u_{k+1}.
template <int M, int L, typename C>
__device__ __forceinline__ void bwd_local(C (&v)[M], const RowTabs<M, L, C>& tb, int gl) {
#pragma unroll
  for (int j = M - 2; j >= 0; --j) v[j] = cfma(__ldg(&tb.S[j * L + gl]), v[j + 1], v[j]);
}

// v_j += P_j carry (P: the prefix or suffix products of lane gl).
template <int M, int L, typename C>
__device__ __forceinline__ void add_carry(C (&v)[M], const C* P, int gl, C carry) {
#pragma unroll
  for (int j = 0; j < M; ++j) v[j] = cfma(__ldg(&P[j * L + gl]), carry, v[j]);
}

// The tridiagonal solve (1 - i r d2) u = R of one row held by a group of L
// lanes, M consecutive elements each (lane gl: elements gl*M .. gl*M+M-1):
// local recurrences, the lane carries combined by a Kogge-Stone scan of
// affine maps, each lane's carry times the products of its coefficients.
template <typename T, int M, int L, typename C>
__device__ __forceinline__ void row_solve(C (&v)[M], const C* tab, int gl, T r) {
  constexpr int kScan = L == 32 ? 5 : 4;  // log2 L
  const RowTabs<M, L, C> tb(tab);
  fwd_local<T, M, L>(v, tb, gl, r);
  C b = v[M - 1];
#pragma unroll
  for (int t = 0; t < kScan; ++t) {
    const int d = 1 << t;
    const C o = shfl_up_c<L>(b, d);
    if (gl >= d) b = cfma(__ldg(&tb.F[t * L + gl]), o, b);
  }
  C yin = shfl_up_c<L>(b, 1);
  if (gl == 0) yin = C{0, 0};
  add_carry<M, L>(v, tb.G, gl, yin);
  bwd_local<M, L>(v, tb, gl);
  b = v[0];
#pragma unroll
  for (int t = 0; t < kScan; ++t) {
    const int d = 1 << t;
    const C o = shfl_down_c<L>(b, d);
    if (gl + d < L) b = cfma(__ldg(&tb.B[t * L + gl]), o, b);
  }
  C uin = shfl_down_c<L>(b, 1);
  if (gl == L - 1) uin = C{0, 0};
  add_carry<M, L>(v, tb.H, gl, uin);
}

// R' = u' + i r d2x(u') + S (src/Core/FieldSolverADICUDA.cpp:279-323) of a
// solved row, in place with the original left neighbour carried along.
template <typename T, int M, int L, typename C>
__device__ __forceinline__ void px_rprime(C (&v)[M], int gl, T r, unsigned long long smask,
                                          const C* srow) {
  C prev = shfl_up_c<L>(v[M - 1], 1);
  if (gl == 0) prev = C{0, 0};
  C right = shfl_down_c<L>(v[0], 1);
  if (gl == L - 1) right = C{0, 0};
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int k = gl * M + j;
    const C cur = v[j];
    const C upp = j < M - 1 ? v[j + 1] : right;
    const T lr = fma((T)-2, cur.x, upp.x + prev.x);
    const T li = fma((T)-2, cur.y, upp.y + prev.y);
    C R;
    R.x = fma(-r, li, cur.x);
    R.y = fma(r, lr, cur.y);
    if ((smask >> j) & 1ull) R = cadd(R, srow[k]);
    v[j] = R;
    prev = cur;
  }
}

// Warps per CTA and CTAs per SM (launch bounds) of the ADI kernels: FP64 9
// warps of 32-lane rows, three CTAs per SM up to M = 7 (ngrid 224: pass X's
// three tiles still fit the SM's shared memory; 416 -> 338 us per pass X of
// 1024 x 201^2 against two); FP32 10 warps of 32-lane rows or 5 warps of two
// 16-lane rows each (10 rows per band either way; smaller CTAs of 16-lane
// rows keep six on an SM so that one CTA's loads and stores overlap the
// others' solves).
template <typename T, int L> struct BandW {
  static constexpr int value = sizeof(T) == 8 ? 9 : (L == 16 ? 5 : 10);
};
template <typename T, int M, int L> struct AdiBlocks {
  static constexpr int value =
      sizeof(T) == 8 ? (M <= 7 ? 3 : 2)
                     : (L == 16 ? (M <= 9 ? 8 : (M <= 17 ? 6 : 4)) : (M <= 9 ? 4 : 2));
};

// One band of W rows (pass X) or W transposed columns (pass Y) of slice s.
// A row is solved by L lanes holding M elements each: L = 32, one row per
// warp; L = 16, two rows per warp (one per half), for rows that fit 16 M
// slots more closely than 32 M.  bar is an initialised mbarrier; parity the
// phase this band waits on.  Returns false, with nothing solved or stored, if
// the band's rows did not arrive within the bounded wait (the device error
// flag then says so); the result is the same in every thread of the CTA.
template <typename T, int M, bool PX, int L>
__device__ __forceinline__ bool adi_band(const AdiPassArgs& a, const CUtensorMap* tm_out, int s,
                                         int band, unsigned char* smem, uint64_t* bar,
                                         uint32_t parity) {
  using C = typename CT<T>::type;
  constexpr int R = 32 / L;                     // rows per warp
  constexpr int W = BandW<T, L>::value * R;     // rows per band
  const int n = a.n, ld = a.ld;
  const int r0 = band * W;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gl = lane & (L - 1);                // lane within the row's group
  const int row = warp * R + (lane >> 4) * (R - 1);  // row within the band
  constexpr int kTileRows = PX ? W + 2 : W;
  const bool has_src = PX && a.src != nullptr;

  C* tile = reinterpret_cast<C*>(smem);
  C* stile = tile + kTileRows * ld;
  C* out = reinterpret_cast<C*>(smem + a.out_off);
  __shared__ double dpart[PX ? 1 : W][9];  // pass Y: per-row diagnostic partials

  const size_t plane = (size_t)n * ld;
  const int lo = PX ? max(r0 - 1, 0) : r0;
  const int hi = PX ? min(r0 + W, n - 1) : min(r0 + W - 1, n - 1);
  const int slot0 = PX ? lo - (r0 - 1) : 0;
  // the source is non-zero only on the slice's tile: rows [sy0, sy0+sbh),
  // columns [sx0, sx0+sbw); stile holds the tile rows of this band.  The
  // descriptor is written by the deposition, which may still be draining
  // when this kernel starts (launch_pdl): a plain load, which stays after
  // ptx::pdl_wait, not a read-only-path load the compiler may issue earlier
  const int4 sd = has_src ? a.desc[s] : make_int4(0, 0, 0, 0);
  const int sx0 = sd.x, sbw = sd.z;
  const int srow_lo = max(r0, sd.y);
  const int srow_hi = min(min(r0 + W, n), sd.y + sd.w);
  const bool band_src = has_src && sbw > 0 && srow_lo < srow_hi;
  if (tid == 0) {
    const C* in = reinterpret_cast<const C*>(a.in) + (size_t)s * plane;
    const uint32_t bytes_in = (uint32_t)((hi - lo + 1) * ld * sizeof(C));
    const uint32_t bytes_s =
        band_src ? (uint32_t)((srow_hi - srow_lo) * sbw * sizeof(C)) : 0u;
    ptx::mbar_expect_tx(bar, bytes_in + bytes_s);
    ptx::bulk_g2s(tile + slot0 * ld, in + (size_t)lo * ld, bytes_in, bar);
    if (band_src) {
      const C* sp = reinterpret_cast<const C*>(a.src) + (size_t)s * a.src_cap +
                    (size_t)(srow_lo - sd.y) * sbw;
      ptx::bulk_g2s(stile + (srow_lo - r0) * sbw, sp, bytes_s, bar);
    }
  }
  if (PX) {
    // rows outside the plane are the zero Dirichlet halo (missing neighbour
    // is zero, src/Core/FieldSolverADICUDA.cpp:197-207)
    for (int t = 0; t < kTileRows; ++t) {
      const int g = r0 - 1 + t;
      if (g < 0 || g > n - 1)
        for (int k = tid; k < ld; k += blockDim.x) tile[t * ld + k] = C{0, 0};
    }
  }
  const bool arrived = ptx::mbar_wait_bounded(bar, parity, a.err);
  if (!__syncthreads_and(arrived)) return false;
  const T r = (T)a.r;
  const int iy = r0 + row;
  const bool active = iy < n;
  const bool row_src = band_src && iy >= srow_lo && iy < srow_hi;
  const C* srow = stile + row * sbw - sx0;  // srow[k] for k in [sx0, sx0+sbw)
  // bit j set: this lane's element j lies in the source tile's columns
  unsigned long long smask = 0ull;
  if (row_src) {
    const int jlo = min(max(sx0 - gl * M, 0), M), jhi = min(max(sx0 + sbw - gl * M, 0), M);
    smask = ((1ull << jhi) - 1ull) & ~((1ull << jlo) - 1ull);
  }
  // elements j < jn lie in the row (none for a row past the plane)
  const int jn = active ? min(max(n - gl * M, 0), M) : 0;
  C v[M];

  // a warp with any row in the plane solves both (a row past the plane is
  // all zeros), so that every lane takes part in the group shuffles
  if (__any_sync(0xffffffffu, active)) {
    if (PX) {
      px_rhs<T, M>(v, tile, ld, row, gl, jn, r, smask, srow);
    } else {
#pragma unroll
      for (int j = 0; j < M; ++j) v[j] = j < jn ? tile[row * ld + gl * M + j] : C{0, 0};
    }
    row_solve<T, M, L>(v, reinterpret_cast<const C*>(a.tab), gl, r);
    if (PX) px_rprime<T, M, L>(v, gl, r, smask, srow);
  } else {
#pragma unroll
    for (int j = 0; j < M; ++j) v[j] = C{0, 0};
  }

  if (!PX && a.zero_count > 0) {
    const int zs = (s - a.zero_start + a.nslice) % a.nslice;
    if (zs < a.zero_count) {
#pragma unroll
      for (int j = 0; j < M; ++j) v[j] = C{0, 0};
    }
  }
  if (!PX && a.diag != nullptr) {
    // field diagnostics of this band (g4_field_slice_reduce_kernel,
    // src/Core/DiagnosticCUDA.cpp:305-363): this lane group holds column
    // ix = r0 + row, rows iy = gl*M + j of the solved plane
    // each lane sums its M cells in the state precision T (exact cell
    // offsets; partials of <= 33 terms, rounding at the level of the state's
    // own); the lanes of a column add in FP64 (<= 32 terms); the power and
    // the other sums of the band's warps and (in the finalize) of the bands
    // are added with compensation (csum_*), as are the slices on the host
    const T shift = (T)(-0.5 * (double)(n - 1));
    const double dx = (double)iy + (double)shift;  // iy is the column index in pass Y
    T tp = 0, ty1 = 0, ty2 = 0, tre = 0, tim = 0;
    double cre = 0, cim = 0;
    const int ic = (n * n - 1) / 2;
    const int icy = ic / n, icx = ic - icy * n;
    if (active) {
      // cells past the row end hold exact zeros (their coefficients are 0)
      const T dy0 = (T)(gl * M) + shift;  // exact: small integers and halves
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const T re = v[j].x, im = v[j].y;
        const T wei = fma(re, re, im * im);
        const T dy = dy0 + (T)j;
        tp += wei;
        ty1 = fma(dy, wei, ty1);
        ty2 = fma(dy * dy, wei, ty2);
        tre += re;
        tim += im;
      }
      const int jc = iy == icx ? icy - gl * M : -1;
      if (jc >= 0 && jc < M) {
#pragma unroll
        for (int j = 0; j < M; ++j)
          if (j == jc) {
            cre = (double)v[j].x;
            cim = (double)v[j].y;
          }
      }
    }
    // power over the column in FP64; the moments and sums over the column's
    // lanes in the state precision; the x moments follow from the column's
    // power (x is the column); the centre cell comes from the one lane that
    // holds it
    double sp = (double)tp;
    for (int o = L / 2; o > 0; o >>= 1) sp += __shfl_xor_sync(0xffffffffu, sp, o);
    T vals[4] = {ty1, ty2, tre, tim};
#pragma unroll
    for (int q = 0; q < 4; ++q)
      for (int o = L / 2; o > 0; o >>= 1) vals[q] += __shfl_xor_sync(0xffffffffu, vals[q], o);
    if (gl == 0) {
      dpart[row][0] = sp;
      dpart[row][1] = dx * sp;
      dpart[row][2] = dx * dx * sp;
      dpart[row][3] = (double)vals[0];
      dpart[row][4] = (double)vals[1];
      dpart[row][5] = (double)vals[2];
      dpart[row][6] = (double)vals[3];
      dpart[row][7] = 0.0;
      dpart[row][8] = 0.0;
    }
    __syncwarp();
    if (cre != 0.0 || cim != 0.0) {  // the lane holding the centre cell
      dpart[row][7] = cre;
      dpart[row][8] = cim;
    }
  }
  if (PX) __syncthreads();  // out overlays the input tile
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const int k = gl * M + j;
    if (j < jn) out[k * W + row] = v[j];
  }
  ptx::fence_proxy_async();
  __syncthreads();  // the staged rows and the diagnostic partials are complete
  if (tid == 0) {
    for (int i = 0; i < a.nbox; ++i)
      ptx::tma_store_3d(tm_out, out + (size_t)i * a.box_rows * W, 2 * r0,
                        i * a.box_rows, s);
    ptx::bulk_commit();
  }
  // the band's diagnostic sums, over its rows in order, while the stores run
  if (!PX && a.diag != nullptr && tid >= 32 && tid < 32 + 9) {
    const int q = tid - 32;
    double t = dpart[0][q], tc = 0.0;
    for (int w = 1; w < W; ++w) ptx::csum_add(t, tc, dpart[w][q]);
    a.diag[((size_t)s * a.nband + band) * 9 + q] = t + tc;
  }
  if (tid == 0) ptx::bulk_wait_read0();
  return true;
}

template <typename T, int M, bool PX, int L>
__global__ void __launch_bounds__(BandW<T, L>::value * 32, AdiBlocks<T, M, L>::value)
    adi_pass_kernel(const __grid_constant__ AdiPassArgs a,
                    const __grid_constant__ CUtensorMap tm_out) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    ptx::mbar_init(&bar, 1);
    ptx::fence_mbar_init();
  }
  __syncthreads();
  ptx::pdl_wait();
  adi_band<T, M, PX, L>(a, &tm_out, blockIdx.x / a.nband, blockIdx.x % a.nband, smem, &bar, 0u);
}

// Persistent form over a work list of (run, slice, band) items of many runs
// (one mbarrier, one phase per item; tensor maps read from global memory).
template <typename T, int M, bool PX, int L>
__global__ void __launch_bounds__(BandW<T, L>::value * 32, AdiBlocks<T, M, L>::value)
    adi_batch_kernel(const __grid_constant__ AdiBatchArgs b) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    ptx::mbar_init(&bar, 1);
    ptx::fence_mbar_init();
  }
  __syncthreads();
  const int nitems = *b.nitems;
  uint32_t parity = 0;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = b.items[it];
    const CUtensorMap* tm = b.maps + w.x;
    if (threadIdx.x == 0) ptx::fence_tensormap_acquire(tm);
    // a band whose rows never arrived leaves the barrier's phase open: stop
    // (the error flag reports it) rather than wait on it again
    if (!adi_band<T, M, PX, L>(b.args[w.x], tm, w.y, w.z, smem, &bar, parity)) return;
    parity ^= 1u;
    __syncthreads();
  }
}

// ------------------------------------------------------------ deposition ---
// Deterministic replacement of adi_zero_source_grid + adi_deposit_source_atomic
// (src/Core/FieldSolverADICUDA.cpp:98-174).  One CTA per beam slice:
//  1. a pass over the slice's particles finds the largest per-particle weight
//     q = sqrt(faw2)/gamma and the bounding box of the touched cells;
//  2. the box is accumulated in shared memory as int64 fixed point with the
//     exponent 2^E chosen so that count * max q * 2^E < 2^62 (integer adds are
//     associative, so the result does not depend on the order of the atomics);
//  3. the CTA writes only the box, scl * sum * 2^-E, as a compact tile of the
//     target slice, and the tile's (x0, y0, width, height) descriptor; the
//     source is zero outside the box.  Boxes larger than the shared-memory
//     accumulator are done in row bands.
struct DepositArgs {
  const double *x, *y, *gamma, *theta;
  const int64_t* off;
  const double* scl;
  double2* src;        // compact tiles, src_cap cells per slice
  int4* desc;          // per target slice
  size_t src_cap;
  int nslice, n, ld, first, harm, acc_cells;
  double gridmax, dgrid, ax, ay, kx, ky, gradx, grady;
  int* err;
};

__device__ __forceinline__ bool dep_cell(const DepositArgs& a, double xp, double yp,
                                         int& ix, int& iy, double& wx, double& wy) {
  if (!(xp > -a.gridmax && xp < a.gridmax && yp > -a.gridmax && yp < a.gridmax))
    return false;
  const double wx_raw = (xp + a.gridmax) / a.dgrid;
  const double wy_raw = (yp + a.gridmax) / a.dgrid;
  ix = (int)floor(wx_raw);
  iy = (int)floor(wy_raw);
  if (ix < 0 || ix >= a.n - 1 || iy < 0 || iy >= a.n - 1) return false;
  wx = 1.0 + (double)ix - wx_raw;
  wy = 1.0 + (double)iy - wy_raw;
  return true;
}

__device__ __forceinline__ double dep_weight(const DepositArgs& a, double xp,
                                             double yp, double g) {
  const double dx = xp - a.ax, dy = yp - a.ay;
  const double faw2 = 1.0 + a.kx * dx * dx + a.ky * dy * dy +
                      2.0 * (a.gradx * dx + a.grady * dy);
  return sqrt(faw2) / g;
}

template <typename V>
__device__ __forceinline__ V block_reduce(V v, V* sh, bool is_max) {
  // fixed-order reduction: warp xor-tree, then warp 0 over the warp partials
  for (int o = 16; o > 0; o >>= 1) {
    V t = __shfl_xor_sync(0xffffffffu, v, o);
    v = is_max ? (t > v ? t : v) : (t < v ? t : v);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  V r = sh[0];
  for (int i = 1; i < nw; ++i) r = is_max ? (sh[i] > r ? sh[i] : r) : (sh[i] < r ? sh[i] : r);
  return r;
}

constexpr int kDepFp64U = 2;  // particles in flight per thread (FP64 deposition)

__global__ void __launch_bounds__(512, 2) deposit_slice_kernel(const DepositArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double shd[16];
  __shared__ int shi[16];
  ptx::pdl_wait();
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(smem);
  const int bs = blockIdx.x;
  const int tid = threadIdx.x;
  const int target = (bs + a.first) % a.nslice;
  double2* S = a.src + (size_t)target * a.src_cap;
  const int64_t p0 = a.off[bs], p1 = a.off[bs + 1];
  const double scl = a.scl[bs];

  double qmax = 0.0;
  int ixmin = 1 << 30, iymin = 1 << 30, ixmax = -1, iymax = -1, cnt = 0;
  const int nt = blockDim.x;
  if (scl != 0.0) {
    // kDepFp64U particles in flight per thread: their loads are issued
    // before any of them is processed
    for (int64_t pb = p0 + tid; pb < p1; pb += (int64_t)kDepFp64U * nt) {
      double lx[kDepFp64U], ly[kDepFp64U], lg[kDepFp64U];
#pragma unroll
      for (int u = 0; u < kDepFp64U; ++u) {
        const int64_t p = pb + (int64_t)u * nt;
        if (p < p1) {
          lx[u] = a.x[p];
          ly[u] = a.y[p];
          lg[u] = a.gamma[p];
        }
      }
#pragma unroll
      for (int u = 0; u < kDepFp64U; ++u) {
        if (pb + (int64_t)u * nt >= p1) break;
        int ix, iy;
        double wx, wy;
        if (!dep_cell(a, lx[u], ly[u], ix, iy, wx, wy)) continue;
        const double q = fabs(dep_weight(a, lx[u], ly[u], lg[u]));
        qmax = q > qmax ? q : qmax;
        if (!(q <= 1e300)) qmax = INFINITY;  // NaN or inf
        ixmin = min(ixmin, ix);
        ixmax = max(ixmax, ix);
        iymin = min(iymin, iy);
        iymax = max(iymax, iy);
        ++cnt;
      }
    }
  }
  qmax = block_reduce<double>(qmax, shd, true);
  ixmin = block_reduce<int>(ixmin, shi, false);
  ixmax = block_reduce<int>(ixmax, shi, true);
  iymin = block_reduce<int>(iymin, shi, false);
  iymax = block_reduce<int>(iymax, shi, true);
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  __syncthreads();
  if ((tid & 31) == 0) shi[tid >> 5] = cnt;
  __syncthreads();
  int total = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) total += shi[i];
  __syncthreads();

  const bool any = total > 0 && qmax > 0.0;
  if (any && !(qmax < INFINITY) && tid == 0) atomicOr(a.err, kErrFixedRange);
  const bool ok = any && qmax < INFINITY;
  int bx0 = 0, by0 = 0, bw = 0, bh = 0;
  double scale = 0.0, unscale = 0.0;
  if (ok) {
    bx0 = ixmin;
    by0 = iymin;
    bw = ixmax - ixmin + 2;  // corners ix..ix+1
    bh = iymax - iymin + 2;
    int e;
    frexp(qmax * (double)total, &e);  // qmax*total < 2^e
    scale = ldexp(1.0, 62 - e);
    unscale = scl * ldexp(1.0, e - 62);
  }
  if (tid == 0) a.desc[target] = make_int4(bx0, by0, ok ? bw : 0, bh);
  if (!ok) return;
  const int band_h = max(1, min(bh, a.acc_cells / bw));
  const double hphase = (double)a.harm;

  for (int yb = by0; yb < by0 + bh; yb += band_h) {
    const int hb = min(band_h, by0 + bh - yb);
    // four 32-bit planes per band: low and high words of the real and the
    // imaginary 64-bit sums (a 64-bit shared atomic costs about four 32-bit
    // ones; the low word's carry goes to the high word, so every sum is the
    // exact 64-bit integer whatever the order of the adds)
    const int ncell = hb * bw;
    unsigned int* lre = reinterpret_cast<unsigned int*>(acc);
    unsigned int* lim = lre + ncell;
    int* hre = reinterpret_cast<int*>(lim + ncell);
    int* him = hre + ncell;
    for (int i = tid; i < 2 * ncell; i += blockDim.x) acc[i] = 0ull;
    __syncthreads();
    for (int64_t pb = p0 + tid; pb < p1; pb += (int64_t)kDepFp64U * nt) {
      double lx[kDepFp64U], ly[kDepFp64U], lg[kDepFp64U], lt[kDepFp64U];
#pragma unroll
      for (int u = 0; u < kDepFp64U; ++u) {
        const int64_t p = pb + (int64_t)u * nt;
        if (p < p1) {
          lx[u] = a.x[p];
          ly[u] = a.y[p];
          lg[u] = a.gamma[p];
          lt[u] = a.theta[p];
        }
      }
#pragma unroll
      for (int u = 0; u < kDepFp64U; ++u) {
      if (pb + (int64_t)u * nt >= p1) break;
      int ix, iy;
      double wx, wy;
      const double xp = lx[u], yp = ly[u];
      if (!dep_cell(a, xp, yp, ix, iy, wx, wy)) continue;
      if (iy + 1 < yb || iy >= yb + hb) continue;
      const double q = dep_weight(a, xp, yp, lg[u]);
      double sn, cs;
      sincos(hphase * lt[u], &sn, &cs);
      const double vre = sn * q * scale, vim = cs * q * scale;
      const double w[4] = {wx * wy, (1.0 - wx) * wy, wx * (1.0 - wy),
                           (1.0 - wx) * (1.0 - wy)};
      const int cx[4] = {ix, ix + 1, ix, ix + 1};
      const int cy[4] = {iy, iy, iy + 1, iy + 1};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int ry = cy[c] - yb;
        if (ry < 0 || ry >= hb) continue;
        const int cell = ry * bw + (cx[c] - bx0);
        const long long cr = __double2ll_rn(vre * w[c]), ci = __double2ll_rn(vim * w[c]);
        const unsigned int rlo = (unsigned int)cr, ilo = (unsigned int)ci;
        const unsigned int rold = atomicAdd(&lre[cell], rlo);
        const unsigned int iold = atomicAdd(&lim[cell], ilo);
        atomicAdd(&hre[cell], (int)(cr >> 32) + (rold + rlo < rold ? 1 : 0));
        atomicAdd(&him[cell], (int)(ci >> 32) + (iold + ilo < iold ? 1 : 0));
      }
      }
    }
    __syncthreads();
    double2* out = S + (size_t)(yb - by0) * bw;
    for (int i = tid; i < ncell; i += blockDim.x) {
      const long long sr = (long long)(((unsigned long long)(unsigned int)hre[i] << 32) | lre[i]);
      const long long si = (long long)(((unsigned long long)(unsigned int)him[i] << 32) | lim[i]);
      out[i] = make_double2((double)sr * unscale, (double)si * unscale);
    }
    __syncthreads();
  }
}

// adi_compute_slice_scl (src/Core/FieldSolverADICUDA.cpp:75-96)
__global__ void slice_scl_kernel(int nslice, const int64_t* off, const double* current,
                                 double fc, double xks, double dgrid, double delz,
                                 double vacimp, double eev, double* scl) {
  ptx::pdl_wait();
  const int is = blockIdx.x * blockDim.x + threadIdx.x;
  if (is >= nslice) return;
  double s = 0.0;
  const int64_t npar = off[is + 1] - off[is];
  if (npar > 0) {
    s = fc * vacimp * current[is] * xks * delz;
    s /= 4.0 * eev * (double)npar * dgrid * dgrid;
  }
  scl[is] = s;
}

// ------------------------------------------------------------- host side ---

static constexpr double kVacimp = 376.73031346177;  // upstream `vacimp`
static constexpr double kEev = 510998.95;          // upstream `eev`

template <typename T, int M, bool PX, int L>
static int configure_pass_t(int device) {
  static std::atomic<uint64_t> configured{0};  // per instantiation, one bit per device
  if (device < 64 && (configured.load() >> device) & 1) return G4B_OK;
  // static + dynamic shared memory must fit the 227 KB a CTA may use
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, adi_pass_kernel<T, M, PX, L>);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncGetAttributes(adi_pass)");
  e = cudaFuncSetAttribute(adi_pass_kernel<T, M, PX, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           227 * 1024 - (int)fa.sharedSizeBytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(adi_pass)");
  if (device < 64) configured.fetch_or(1ull << device);
  return G4B_OK;
}

template <typename T, int M, bool PX, int L>
static int launch_pass_t(g4b_field* f, const AdiPassArgs& args, const CUtensorMap& tm,
                         size_t smem) {
  constexpr int W = BandW<T, L>::value;  // warps per CTA
  auto kern = adi_pass_kernel<T, M, PX, L>;
  if (int rc = configure_pass_t<T, M, PX, L>(f->ctx->device)) return rc;
  const unsigned grid = (unsigned)(f->nslice * args.nband);
  {
    LaunchScope ls(f->ctx, PX ? "adi_pass_x" : "adi_pass_y");
    G4B_CUDA_TRY(launch_pdl(kern, grid, W * 32, smem, f->ctx->stream, args, tm));
  }
  return check_launch(f->ctx, "adi_pass_kernel");
}

// Kernel modes: M (odd elements per lane) with 32-lane rows, 100 + M with
// 16-lane rows (FP32 only).
#define G4B_MODES32(X) X(1, 32) X(3, 32) X(5, 32) X(7, 32) X(9, 32) X(11, 32) X(13, 32) \
  X(15, 32) X(17, 32) X(21, 32) X(25, 32) X(33, 32)
#define G4B_MODES16(X) X(5, 16) X(7, 16) X(9, 16) X(11, 16) X(13, 16) X(15, 16) X(17, 16) \
  X(21, 16) X(25, 16) X(33, 16)

template <typename T, bool PX>
static int configure_pass_m(int mode, int device) {
#define G4B_CFG(m, l) \
  case (l == 16 ? 100 : 0) + m: return configure_pass_t<T, m, PX, l>(device);
  if constexpr (sizeof(T) == 8) {
    switch (mode) { G4B_MODES32(G4B_CFG) }
  } else {
    switch (mode) { G4B_MODES32(G4B_CFG) G4B_MODES16(G4B_CFG) }
  }
#undef G4B_CFG
  return fail(G4B_ERR_RANGE, "adi: unsupported elements per lane");
}

int adi_configure(g4b_field* f) {
  const int M = f->mode;
  const int d = f->ctx->device;
  if (f->precision == G4B_FP64) {
    if (int rc = configure_pass_m<double, true>(M, d)) return rc;
    return configure_pass_m<double, false>(M, d);
  }
  if (int rc = configure_pass_m<float, true>(M, d)) return rc;
  return configure_pass_m<float, false>(M, d);
}

template <typename T, bool PX>
static int launch_pass_m(int mode, g4b_field* f, const AdiPassArgs& args,
                         const CUtensorMap& tm, size_t smem) {
#define G4B_LAUNCH(m, l) \
  case (l == 16 ? 100 : 0) + m: return launch_pass_t<T, m, PX, l>(f, args, tm, smem);
  if constexpr (sizeof(T) == 8) {
    switch (mode) { G4B_MODES32(G4B_LAUNCH) }
  } else {
    switch (mode) { G4B_MODES32(G4B_LAUNCH) G4B_MODES16(G4B_LAUNCH) }
  }
#undef G4B_LAUNCH
  return fail(G4B_ERR_RANGE, "adi: unsupported elements per lane");
}

int adi_plan(g4b_adi* adi, g4b_field* f, const void* src, const int4* desc,
             const AdiYExtras* ex, AdiPlan& P) {
  const int n = f->ngrid, ld = f->ld, W = f->band_rows;
  AdiPassArgs args{};
  args.n = n;
  args.ld = ld;
  args.nband = (n + W - 1) / W;
  args.r = adi->r;
  args.err = f->ctx->d_error;
  args.box_rows = f->store_box_rows;
  args.nbox = f->store_nbox;
  if (f->precision == G4B_FP64)
    args.tab = adi->d_tab64;
  else if (f->mode == adi->mode32)
    args.tab = adi->d_tab32;
  else if (f->mode == adi->mode32_alt && adi->d_tab32_alt)
    args.tab = adi->d_tab32_alt;
  else
    return fail(G4B_ERR_STATE, "adi: solver and field row layouts differ");
  const size_t cb = f->cell_bytes;
  const size_t out_bytes = (size_t)f->store_nbox * f->store_box_rows * W * cb;
  auto smem_for = [&](bool px, bool with_src) {
    size_t tile = (size_t)((px ? W + 2 : W) * ld) * cb;
    if (px && with_src) tile += (size_t)W * ld * cb;
    // pass X: the output staging tile reuses the input tile's memory
    // (written after a barrier that ends every read of the input), which
    // keeps three CTAs of 16-lane rows on an SM; pass Y: after the input
    if (px) {
      args.out_off = 0;
      return std::max(tile, out_bytes);
    }
    const size_t out_off = (tile + 127) / 128 * 128;
    args.out_off = (int)out_off;
    return out_off + out_bytes;
  };
  P.M = f->precision == G4B_FP64 ? adi->M : f->mode;
  if (P.M != f->mode) return fail(G4B_ERR_STATE, "adi: solver and field row layouts differ");
  P.precision = f->precision;
  P.grid = (unsigned)(f->nslice * args.nband);
  P.tm_x = &f->tm_store_b;
  P.tm_y = &f->tm_store_a;
  // pass X: a -> b (transposed R')
  args.in = f->a;
  args.src = src;
  args.desc = desc;
  args.src_cap = (size_t)f->ngrid * f->ld;
  P.smem_x_max = smem_for(true, true);
  P.smem_x = smem_for(true, src != nullptr);
  if (P.smem_x + 2048 > 227 * 1024)
    return fail(G4B_ERR_RANGE, "adi: pass X tile exceeds shared memory");
  P.x = args;
  // pass Y: b -> a (natural)
  args.in = f->b;
  args.src = nullptr;
  args.nslice = f->nslice;
  if (ex) {
    args.zero_start = ex->zero_start;
    args.zero_count = ex->zero_count;
    args.diag = ex->diag;
  }
  P.smem_y = smem_for(false, false);
  P.y = args;
  return G4B_OK;
}

int adi_launch(g4b_field* f, const AdiPlan& P) {
  int rc = P.precision == G4B_FP64
               ? launch_pass_m<double, true>(P.M, f, P.x, *P.tm_x, P.smem_x)
               : launch_pass_m<float, true>(P.M, f, P.x, *P.tm_x, P.smem_x);
  if (rc) return rc;
  return P.precision == G4B_FP64
             ? launch_pass_m<double, false>(P.M, f, P.y, *P.tm_y, P.smem_y)
             : launch_pass_m<float, false>(P.M, f, P.y, *P.tm_y, P.smem_y);
}

int adi_run(g4b_adi* adi, g4b_field* f, const void* src, const int4* desc,
            const AdiYExtras* ex) {
  AdiPlan P;
  if (int rc = adi_plan(adi, f, src, desc, ex, P)) return rc;
  return adi_launch(f, P);
}

template <int M, bool PX, int L>
static int batch_launch_t(g4b_ctx* c, cudaStream_t st, const AdiBatchArgs& b, size_t smem,
                          int grid) {
  static std::atomic<uint64_t> configured{0};
  auto kern = adi_batch_kernel<float, M, PX, L>;
  if (c->device >= 64 || !((configured.load() >> c->device) & 1)) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kern);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncGetAttributes(adi_batch)");
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             227 * 1024 - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(adi_batch)");
    if (c->device < 64) configured.fetch_or(1ull << c->device);
  }
  {
    LaunchScope ls(c, PX ? "batch_adi_x" : "batch_adi_y");
    kern<<<grid, BandW<float, L>::value * 32, smem, st>>>(b);
  }
  return check_launch(c, "adi_batch_kernel");
}

int adi_batch_launch(g4b_ctx* c, cudaStream_t st, int mode, bool px, const AdiBatchArgs& b,
                     size_t smem, int grid) {
#define G4B_BATCH_CASE(m, l)                                                   \
  case (l == 16 ? 100 : 0) + m:                                                \
    return px ? batch_launch_t<m, true, l>(c, st, b, smem, grid)               \
              : batch_launch_t<m, false, l>(c, st, b, smem, grid);
  switch (mode) { G4B_MODES32(G4B_BATCH_CASE) G4B_MODES16(G4B_BATCH_CASE) }
#undef G4B_BATCH_CASE
  return fail(G4B_ERR_RANGE, "adi: unsupported elements per lane");
}

// adi_compute_slice_scl + the deterministic deposition
// (src/Core/FieldSolverADICUDA.cpp:75-174) of an FP64 beam into the field's
// compact source tiles; shared by the ADI and FFT solvers.
int fp64_deposit(g4b_field* f, g4b_beam* b, const g4b_step* st, double fc) {
  g4b_ctx* c = f->ctx;
  const int harm = f->harm;
  {
    LaunchScope ls(c, "slice_scl");
    G4B_CUDA_TRY(launch_pdl(slice_scl_kernel, (unsigned)((b->nslice + 127) / 128), 128, 0,
                            c->stream, b->nslice, b->d_off, b->d_current, fc, f->xks, f->dgrid,
                            st->delz, kVacimp, kEev, b->d_scl));
  }
  if (int rc = check_launch(c, "slice_scl_kernel")) return rc;
  DepositArgs da{};
  da.x = b->x;
  da.y = b->y;
  da.gamma = b->gamma;
  da.theta = b->theta;
  da.off = b->d_off;
  da.scl = b->d_scl;
  da.src = static_cast<double2*>(f->src);
  da.desc = f->desc;
  da.src_cap = (size_t)f->ngrid * f->ld;
  da.nslice = f->nslice;
  da.n = f->ngrid;
  da.ld = f->ld;
  da.first = f->first;
  da.harm = harm;
  da.gridmax = f->gridmax;
  da.dgrid = f->dgrid;
  da.ax = st->ax;
  da.ay = st->ay;
  da.kx = st->kx;
  da.ky = st->ky;
  da.gradx = st->gradx;
  da.grady = st->grady;
  da.err = c->d_error;
  const size_t acc_bytes = 96 * 1024;
  da.acc_cells = (int)(acc_bytes / 16);
  G4B_CUDA_TRY(cudaFuncSetAttribute(deposit_slice_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)acc_bytes));  // per device, cheap
  {
    LaunchScope ls(c, "deposit");
    G4B_CUDA_TRY(launch_pdl(deposit_slice_kernel, (unsigned)f->nslice, 512, acc_bytes, c->stream, da));
  }
  if (int rc = check_launch(c, "deposit_slice_kernel")) return rc;
  return G4B_OK;
}

}  // namespace g4b

using namespace g4b;

extern "C" {


int g4b_adi_create(g4b_ctx* c, g4b_adi** out) {
  if (!c || !out) return fail(G4B_ERR_ARG, "g4b_adi_create: null arg");
  g4b_adi* a = new (std::nothrow) g4b_adi();
  if (!a) return fail(G4B_ERR_NOMEM, "g4b_adi_create: host allocation");
  a->ctx = c;
  ctx_retain(c);
  *out = a;
  return G4B_OK;
}

int g4b_adi_destroy(g4b_adi* a) {
  if (!a) return G4B_OK;
  ctx_quiesce(a->ctx);
  dev_free(a->ctx, a->d_tab64);
  dev_free(a->ctx, a->d_tab32);
  dev_free(a->ctx, a->d_tab32_alt);
  ctx_release(a->ctx);
  delete a;
  return G4B_OK;
}

// FieldSolverADICUDA::init (src/Core/FieldSolverADICUDA.cpp:821-866): the
// Thomas factors of the constant matrix, then the scan tables derived from
// them, all in FP64.
int g4b_adi_init(g4b_adi* a, double delz, double dgrid, double xks, int ngrid) {
  if (!a) return fail(G4B_ERR_ARG, "g4b_adi_init: null adi");
  if (ngrid < 2 || !(dgrid > 0) || !(xks > 0))
    return fail(G4B_ERR_ARG, "g4b_adi_init: bad arguments");
  if (a->ready && delz == a->delz && ngrid == a->ngrid && dgrid == a->dgrid &&
      xks == a->xks)
    return G4B_OK;
  const int M = pick_M(ngrid);
  if (!M) return fail(G4B_ERR_RANGE, "g4b_adi_init: ngrid above 1056 is not supported");
  using cd = std::complex<double>;
  const int n = ngrid;
  const double r = 0.25 * delz / (xks * dgrid * dgrid);
  std::vector<double> mupp(n), mmid(n), mlow(n);
  mupp[0] = r;
  mmid[0] = -2 * r;
  mlow[0] = 0;
  for (int i = 1; i < n - 1; ++i) {
    mupp[i] = r;
    mmid[i] = -2 * r;
    mlow[i] = r;
  }
  mupp[n - 1] = 0;
  mmid[n - 1] = -2 * r;
  mlow[n - 1] = r;
  std::vector<cd> c(n), cbet(n), cwet(n);
  for (int i = 0; i < n; ++i) c[i] = cd(0.0, -mlow[i]);
  cbet[0] = cd(1.0, 0.0) / cd(1.0, -mmid[0]);
  cwet[0] = cd(0.0, 0.0);
  for (int i = 1; i < n; ++i) {
    cwet[i] = cd(0.0, -mupp[i - 1]) * cbet[i - 1];
    cbet[i] = cd(1.0, 0.0) / (cd(1.0, -mmid[i]) - c[i] * cwet[i]);
  }
  // Tables of one row layout: L lanes of M elements, recurrence
  // coefficients on the padded index range [0, L M).
  auto tables = [&](const int M, const int L) {
    const int P = L * M;
    std::vector<cd> cb(P, 0.0), q(P, 0.0), sv(P, 0.0), G(P), H(P);
    for (int k = 0; k < n; ++k) cb[k] = cbet[k];
    for (int k = 1; k < n; ++k) q[k] = -c[k] * cbet[k];         // y_k += q_k y_{k-1}
    for (int k = 0; k + 1 < n; ++k) sv[k] = -cwet[k + 1];       // u_k += s_k u_{k+1}
    std::vector<cd> A(L), B(L);
    for (int lane = 0; lane < L; ++lane) {
      const int k0 = lane * M, k1 = k0 + M - 1;
      cd g = 1.0;
      for (int k = k0; k <= k1; ++k) {
        g *= q[k];
        G[k] = g;
      }
      cd h = 1.0;
      for (int k = k1; k >= k0; --k) {
        h *= sv[k];
        H[k] = h;
      }
      A[lane] = G[k1];
      B[lane] = H[k0];
    }
    std::vector<cd> t(tab_total(M, L), 0.0);
    for (int j = 0; j < M; ++j)
      for (int lane = 0; lane < L; ++lane) {
        const int k = lane * M + j;
        t[tab_cbet(M, L) + j * L + lane] = cb[k];
        t[tab_G(M, L) + j * L + lane] = G[k];
        t[tab_H(M, L) + j * L + lane] = H[k];
        t[tab_S(M, L) + j * L + lane] = sv[k];
      }
    std::vector<cd> af = A, ab = B;
    for (int st = 0; (1 << st) < L; ++st) {
      const int d = 1 << st;
      for (int lane = 0; lane < L; ++lane) {
        t[tab_scanF(M, L) + st * L + lane] = af[lane];
        t[tab_scanB(M, L) + st * L + lane] = ab[lane];
      }
      std::vector<cd> nf = af, nb = ab;
      for (int lane = 0; lane < L; ++lane) {
        if (lane >= d) nf[lane] = af[lane] * af[lane - d];
        if (lane + d < L) nb[lane] = ab[lane] * ab[lane + d];
      }
      af.swap(nf);
      ab.swap(nb);
    }
    return t;
  };
  // FP64 fields solve rows with 32 lanes; FP32 fields with the layout of
  // their mode (16-lane rows where those fit the row more closely)
  // (and the tables of the other FP32 layout, which the batch tuner may pick)
  const int mode32 = pick_mode(n, G4B_MIXED), mode32_alt = alt_mode(n);
  const std::vector<cd> c64 = tables(M, 32);
  auto to32 = [&](int mode) {
    const std::vector<cd> c = tables(mode_M(mode), mode_L(mode));
    std::vector<float2> t(c.size());
    for (size_t k = 0; k < c.size(); ++k) t[k] = make_float2((float)c[k].real(), (float)c[k].imag());
    return t;
  };
  std::vector<double2> t64(c64.size());
  for (size_t k = 0; k < c64.size(); ++k) t64[k] = make_double2(c64[k].real(), c64[k].imag());
  const std::vector<float2> t32 = to32(mode32);
  const std::vector<float2> t32a = mode32_alt ? to32(mode32_alt) : std::vector<float2>();
  g4b_ctx* ctx = a->ctx;
  G4B_CUDA_TRY(cudaSetDevice(ctx->device));
  if (a->d_tab64) {
    cudaStreamSynchronize(ctx->stream);
    dev_free(a->ctx, a->d_tab64);
    dev_free(a->ctx, a->d_tab32);
    dev_free(a->ctx, a->d_tab32_alt);
    a->d_tab64 = nullptr;
    a->d_tab32 = nullptr;
    a->d_tab32_alt = nullptr;
  }
  G4B_CUDA_TRY(dev_alloc(a->ctx, (void**)&a->d_tab64, t64.size() * sizeof(double2)));
  G4B_CUDA_TRY(dev_alloc(a->ctx, (void**)&a->d_tab32, t32.size() * sizeof(float2)));
  if (!t32a.empty())
    G4B_CUDA_TRY(dev_alloc(a->ctx, (void**)&a->d_tab32_alt, t32a.size() * sizeof(float2)));
  G4B_CUDA_TRY(cudaMemcpyAsync(a->d_tab64, t64.data(), t64.size() * sizeof(double2),
                               cudaMemcpyHostToDevice, ctx->stream));
  G4B_CUDA_TRY(cudaMemcpyAsync(a->d_tab32, t32.data(), t32.size() * sizeof(float2),
                               cudaMemcpyHostToDevice, ctx->stream));
  if (!t32a.empty())
    G4B_CUDA_TRY(cudaMemcpyAsync(a->d_tab32_alt, t32a.data(), t32a.size() * sizeof(float2),
                                 cudaMemcpyHostToDevice, ctx->stream));
  G4B_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  a->ngrid = ngrid;
  a->delz = delz;
  a->dgrid = dgrid;
  a->xks = xks;
  a->r = r;
  a->M = M;
  a->mode32 = mode32;
  a->mode32_alt = mode32_alt;
  a->ready = true;
  return G4B_OK;
}

// FieldSolverADICUDA::advance (src/Core/FieldSolverADICUDA.cpp:638-818).
int g4b_adi_advance(g4b_adi* adi, g4b_field* f, g4b_beam* b, const g4b_step* st,
                    double fc, int enabled) {
  if (!adi || !f || !b || !st) return fail(G4B_ERR_ARG, "g4b_adi_advance: null arg");
  if (!adi->ready || adi->ngrid != f->ngrid)
    return fail(G4B_ERR_STATE,
                "g4b_adi_advance: called before g4b_adi_init for this ngrid");
  if (b->nslice != f->nslice)
    return fail(G4B_ERR_ARG, "g4b_adi_advance: beam and field slice counts differ");
  if (f->precision != G4B_FP64 || b->precision != G4B_FP64)
    return fail(G4B_ERR_ARG, "g4b_adi_advance: the drop-in path holds FP64 state");
  g4b_ctx* c = f->ctx;
  G4B_CUDA_TRY(cudaSetDevice(c->device));
  const int harm = f->harm;
  const bool do_source = st->in_undulator && enabled && (harm % 2) == 1;
  const bool use_source = do_source && b->npart > 0;
  const void* src = nullptr;
  if (use_source) {
    if (int rc = fp64_deposit(f, b, st, fc)) return rc;
    src = f->src;
  }
  return adi_run(adi, f, src, f->desc, nullptr);
}

}  // extern "C"
