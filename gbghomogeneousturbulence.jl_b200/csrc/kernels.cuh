// The __global__ kernels of the library (CUDA build only): each runs one CTA body of passes.cuh
// or tracers.cuh with NT threads per block. Included by the engine and by the allocation-free
// entry point.
#pragma once

#include "adjoint.cuh"
#include "passes.cuh"
#include "tracers.cuh"

namespace gbght {

// ------------------------------------------------------------------------------------------------
// Kernels (CUDA build).
// ------------------------------------------------------------------------------------------------
#ifndef GBGHT_EMU
#define CTA_CTX Cta c{int(threadIdx.x), int(blockIdx.x), int(blockIdx.y), int(blockIdx.z)}
extern __shared__ __align__(1024) unsigned char g_smem[];

__device__ __forceinline__ void init_bars(uint64_t* bar, int n) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < n; ++i) mbar_init(bar + i, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async();
  }
  __syncthreads();
}

// Each kernel's CTA runs a __device__ function of its arguments, so that a member-batched kernel
// (one launch over the members of a group, below) runs the same code with one member's arguments.
template <class T, int N, int TL, int NT>
__device__ __forceinline__ void y_inverse_cta(const Cta& c, const TmaMaps& m, const Geometry& g, int comp,
                                              const Cplx<T>* tw, unsigned int* status) {
  Cplx<T>* sm = reinterpret_cast<Cplx<T>*>(g_smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + N * TL);
  init_bars(bar, 1);
  const int kx0 = c.bx * TL, z = c.by;
  if (c.tid == 0) {
    const int row0 = (comp * N + z) * g.NY2;
    mbar_expect_tx(bar, uint32_t(2 * (g.K + 1) * TL * sizeof(Cplx<T>)));
    tma_load_2d(sm, &m.a_ld, 2 * kx0, row0, bar);                            // q 0..K   → rows 0..K
    tma_load_2d(sm + (N - g.K - 1) * TL, &m.a_ld, 2 * kx0, row0 + g.K, bar);  // q K..2K → rows N−K−1..N−1
  }
  mbar_wait(bar, 0, status);
  y_inverse_compute<T, N, TL, NT>(c, sm, g, tw);
  fence_proxy_async();
  __syncthreads();
  if (c.tid == 0) {
    constexpr int BY = box_rows<N>();
    for (int y0 = 0; y0 < N; y0 += BY) tma_store_2d(&m.b, 2 * kx0, (comp * N + z) * N + y0, sm + y0 * TL);
    bulk_commit();
    bulk_wait_read();
  }
}
template <class T, int N, int TL, int NT>
__global__ void __launch_bounds__(NT, sizeof(T) == 8 ? 2 : 3) k_y_inverse(const __grid_constant__ TmaMaps m, Geometry g, int c0,
                                                     const Cplx<T>* tw, unsigned int* status) {
  CTA_CTX;
  y_inverse_cta<T, N, TL, NT>(c, m, g, c0 + c.bz, tw, status);
}

template <class T, int N, int TL, int NT>
__device__ __forceinline__ void y_forward_cta(const Cta& c, const TmaMaps& m, const Geometry& g, int comp,
                                              const Cplx<T>* tw, unsigned int* status) {
  Cplx<T>* sm = reinterpret_cast<Cplx<T>*>(g_smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + N * TL);
  init_bars(bar, 1);
  const int kx0 = c.bx * TL, z = c.by;
  constexpr int BY = box_rows<N>();
  if (c.tid == 0) {
    mbar_expect_tx(bar, uint32_t(N * TL * sizeof(Cplx<T>)));
    for (int y0 = 0; y0 < N; y0 += BY) tma_load_2d(sm + y0 * TL, &m.b, 2 * kx0, (comp * N + z) * N + y0, bar);
  }
  mbar_wait(bar, 0, status);
  tile_fft<T, N, TL, NT, -1>(c, sm, tw);
  fence_proxy_async();
  __syncthreads();
  if (c.tid == 0) {
    const int row0 = (comp * N + z) * g.NY2;
    tma_store_2d(&m.a_st1, 2 * kx0, row0, sm);                                  // rows 0..K     → q 0..K
    tma_store_2d(&m.a_st2, 2 * kx0, row0 + g.K + 1, sm + (N - g.K) * TL);         // rows N−K..N−1 → q K+1..2K
    bulk_commit();
    bulk_wait_read();
  }
}
template <class T, int N, int TL, int NT>
__global__ void __launch_bounds__(NT, sizeof(T) == 8 ? 2 : 3) k_y_forward(const __grid_constant__ TmaMaps m, Geometry g, const Cplx<T>* tw,
                                                     unsigned int* status) {
  CTA_CTX;
  y_forward_cta<T, N, TL, NT>(c, m, g, c.bz, tw, status);
}

template <class T, int N, int NT>
__device__ __forceinline__ void x_products_cta(const Cta& c, const Geometry& g, Cplx<T>* B, int has_scalar, int KXS,
                                               const Cplx<T>* tw, unsigned int* status) {
  Cplx<T>* sm = reinterpret_cast<Cplx<T>*>(g_smem);
  Cplx<T>* stg = sm + N * XShape<T>::ACT_INV;
  uint64_t* bar = reinterpret_cast<uint64_t*>(stg + (XShape<T>::STAGED ? 7 * XShape<T>::P * KXS : 0));
  init_bars(bar, 1);
  body_x_products<T, N, NT>(c, sm, stg, KXS, bar, int(gridDim.x), g, B, has_scalar, tw, status);
}
template <class T, int N, int NT>
__global__ void __launch_bounds__(NT, XShape<T>::STAGED ? 2 : 3) k_x_products(Geometry g, Cplx<T>* B, int has_scalar,
                                                                             int KXS, const Cplx<T>* tw,
                                                                             unsigned int* status) {
  CTA_CTX;
  x_products_cta<T, N, NT>(c, g, B, has_scalar, KXS, tw, status);
}

// Shared memory: the ACT_V lines, NT doubles, the staging rows (3·PV·KXS), one barrier (32 bytes).
template <class T, int N, int NT>
__device__ __forceinline__ void x_velocity_cta(const Cta& c, const Geometry& g, const Cplx<T>* B, T* u,
                                               unsigned long long* maxbits, int KXS, const Cplx<T>* tw,
                                               unsigned int* status) {
  Cplx<T>* sm = reinterpret_cast<Cplx<T>*>(g_smem);
  double* red = reinterpret_cast<double*>(sm + N * XShape<T>::ACT_V);
  Cplx<T>* stg = reinterpret_cast<Cplx<T>*>(red + NT);
  uint64_t* bar = reinterpret_cast<uint64_t*>(stg + 3 * XShape<T>::PV * KXS);
  init_bars(bar, 1);
  const double mx = body_x_velocity<T, N, NT>(c, sm, red, stg, KXS, bar, int(gridDim.x), g, B, u, tw, status);
  if (c.tid == 0) atomicMax(maxbits, static_cast<unsigned long long>(__double_as_longlong(mx)));
}
template <class T, int N, int NT>
__global__ void __launch_bounds__(NT, 2) k_x_velocity(Geometry g, const Cplx<T>* B, T* u, unsigned long long* maxbits,
                                                      int KXS, const Cplx<T>* tw, unsigned int* status) {
  CTA_CTX;
  x_velocity_cta<T, N, NT>(c, g, B, u, maxbits, KXS, tw, status);
}

// The owned rows of a z tile (ZOwn) live in TMEM where every warp is fully active in every
// stage, else in registers. `run(rows)` runs the body between the allocation and the release.
// `slot` is 4 bytes of shared memory for the allocation's address.
template <class T, int N, int TL, int NT, int KM, class F>
__device__ __forceinline__ double with_z_rows(uint32_t* slot, const F& run) {
  using O = ZOwn<T, N, TL, NT, KM>;
  using Sh = ZTmemShape<T, N, O, NT>;
  if constexpr (Sh::kUse) {
    const int warp = int(threadIdx.x) >> 5;
    if (warp == 0) tmem_alloc(slot, Sh::NCOLS);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t base = *slot + (uint32_t((warp & 3) * 32) << 16) + uint32_t((warp >> 2) * Sh::COLS);
    ZRowsTmem<T, O> rows{base};
    const double e = run(rows);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc(*slot, Sh::NCOLS);
    return e;
  } else {
    ZRowsReg<T, O> rows;
    return run(rows);
  }
}

// Shared memory: ZLayout (the FFT tile, NT doubles, barriers, the TMEM address, the twiddle table,
// the staging region).
template <class T, int N, int TL, int NT, int KIND, int KM, bool WIDE>
__device__ __forceinline__ void z_epilogue_cta(const Cta& c, const TmaMaps& m, const Geometry& g, Cplx<T>* A,
                                               Cplx<T>* S, Cplx<T>* H, const StageArgs& st, const double* amp,
                                               double* partial, const Cplx<T>* tw, unsigned int* status) {
  using L = ZLayout<T, N, TL, NT>;
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(g_smem);
  double* red = reinterpret_cast<double*>(g_smem + L::kRed);
  uint64_t* bar = reinterpret_cast<uint64_t*>(g_smem + L::kBar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(g_smem + L::kSlot);
  Cplx<T>* R = reinterpret_cast<Cplx<T>*>(g_smem + L::kStage);
  Cplx<T>* twS = reinterpret_cast<Cplx<T>*>(g_smem + L::kTw);
  for (int i = c.tid; i < N; i += NT) twS[i] = tw[i];
  init_bars(bar, 3);   // its barrier also publishes the twiddle table
  const double e = with_z_rows<T, N, TL, NT, KM>(slot, [&](auto& rows) {
    return body_z_epilogue<T, N, TL, NT, KIND, WIDE>(c, W, R, bar, red, g, m, rows, A, S, H, st, amp, twS, status);
  });
  if (c.tid == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = e;
}
template <class T, int N, int TL, int NT, int KIND, int KM = N / 3 + 1, bool WIDE = false>
__global__ void __launch_bounds__(NT, NT > 256 ? 1 : (sizeof(T) == 8 ? 2 : 4)) k_z_epilogue(const __grid_constant__ TmaMaps m, Geometry g, Cplx<T>* A,
                                                      Cplx<T>* S, Cplx<T>* H, StageArgs st, const double* amp,
                                                      double* partial, const Cplx<T>* tw, unsigned int* status) {
  CTA_CTX;
  z_epilogue_cta<T, N, TL, NT, KIND, KM, WIDE>(c, m, g, A, S, H, st, amp, partial, tw, status);
}

template <class T, int N, int TL, int NT, int KM>
__device__ __forceinline__ void z_init_cta(const Cta& c, const Geometry& g, Cplx<T>* A, const Cplx<T>* S,
                                           int has_scalar, double* partial, const Cplx<T>* tw, int vorticity,
                                           int pstride, int shift) {
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(g_smem);
  double* red = reinterpret_cast<double*>(W + N * TL);
  uint32_t* slot = reinterpret_cast<uint32_t*>(red + NT);
  const double e = with_z_rows<T, N, TL, NT, KM>(slot, [&](auto& rows) {
    return body_z_init<T, N, TL, NT>(c, W, red, g, rows, A, S, has_scalar, tw, vorticity, shift);
  });
  // pstride: the tiles per row of the partials (the full grid's, when a launch covers fewer columns);
  // no partials for the displaced grid's fields
  if (c.tid == 0 && partial) partial[blockIdx.y * (pstride ? pstride : gridDim.x) + blockIdx.x] = e;
}
template <class T, int N, int TL, int NT, int KM = N / 3 + 1>
__global__ void __launch_bounds__(NT, NT > 256 ? 1 : 2) k_z_init(Geometry g, Cplx<T>* A, const Cplx<T>* S, int has_scalar, double* partial,
                                                  const Cplx<T>* tw, int vorticity = 1, int pstride = 0,
                                                  int shift = 0) {
  CTA_CTX;
  z_init_cta<T, N, TL, NT, KM>(c, g, A, S, has_scalar, partial, tw, vorticity, pstride, shift);
}
// PhaseShift's shift back of the displaced products into A (body_z_shift_back). Grid (KXP/TL, NY2).
template <class T, int N, int TL, int NT, int KM>
__global__ void __launch_bounds__(NT, NT > 256 ? 1 : 2) k_z_shift_back(Geometry g, Cplx<T>* A, const Cplx<T>* A2, int nc,
                                                        const Cplx<T>* tw) {
  CTA_CTX;
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(g_smem);
  body_z_shift_back<T, N, TL, NT, ZOwn<T, N, TL, NT, KM>>(c, W, g, A, A2, nc, tw);
}
template <class T, int NT, int CH>
__global__ void __launch_bounds__(NT) k_below_scale(Geometry g, double L, const Cplx<T>* S, double* out) {
  CTA_CTX;
  double* tab = reinterpret_cast<double*>(g_smem);
  body_below_scale<T, NT, CH>(c, tab, tab + CH * (g.K + 1), g, L, S, out);
}
template <class T, int NT>
__global__ void __launch_bounds__(NT) k_det_sum(const T* s6, size_t n, size_t chunk, double* out) {
  CTA_CTX;
  __shared__ double red[NT];
  body_det_sum<T, NT>(c, red, s6, n, chunk, out);
}
template <class T>
__global__ void k_inject_source(Geometry g, Cplx<T>* A, const Cplx<double>* su, const Cplx<double>* sp, SourceArgs a) {
  inject_source<T>(long(blockIdx.x) * blockDim.x + threadIdx.x, g, A, su, sp, a);
}
template <class T>
__global__ void k_reality(Geometry g, Cplx<T>* S, int ncomp) {
  reality_mode<T>(int(blockIdx.x * blockDim.x + threadIdx.x), g, S, ncomp);
}
// A band forcing's amplitude (or rescale factor, see forcing_amplitude) for field slots
// [c0, c0 + nc) of S. The whole-field sum adds whole[i·stride] (i < nwhole: the epilogue's tile
// partials, or the observables rows), the Dirichlet sum dir[i·stride] likewise when dir is given;
// the band sum runs over the box |m_a| ≤ mb. Each is summed per thread in a strided order and then
// by a fixed tree, so the result is the same on every run. out[0..2] = (A, band, whole).
template <class T>
__device__ __forceinline__ void force_amp_cta(const Geometry& g, const Cplx<T>* S, int c0, int nc, const double* whole,
                                              const double* dir, int nwhole, int stride, double lo2, double hi2,
                                              const AmpArgs& a, double* out, unsigned int* status) {
  __shared__ double red[256], bred[256], dred[256];
  double s = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < nwhole; i += 256) {
    s += whole[size_t(i) * stride];
    if (dir) d += dir[size_t(i) * stride];
  }
  red[threadIdx.x] = s;
  dred[threadIdx.x] = d;
  int mb = int(sqrt(hi2) / g.s) + 1;
  if (mb > g.K) mb = g.K;
  const int side = 2 * mb + 1, nbox = nc * side * side * (mb + 1);
  double b = 0.0;
  for (int i = threadIdx.x; i < nbox; i += 256) {
    const int kx = i % (mb + 1), mz = (i / (mb + 1)) % side - mb, my = (i / ((mb + 1) * side)) % side - mb;
    const int cc = c0 + i / ((mb + 1) * side * side);
    const double kxd = g.s * kx, kyd = g.s * my, kzd = g.s * mz;
    const double k2 = (kxd * kxd + kyd * kyd) + kzd * kzd;
    if (!(k2 >= lo2 && k2 <= hi2)) continue;
    const int qy = my >= 0 ? my : my + g.NY2, qz = mz >= 0 ? mz : mz + g.NY2;
    const Cplx<T> v = S[idxS(g, cc, qy, qz, kx)];
    b += (kx == 0 ? 1.0 : 2.0) * (double(v.x) * v.x + double(v.y) * v.y);
  }
  bred[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {   // fixed-order trees
    if (threadIdx.x < w) {
      red[threadIdx.x] += red[threadIdx.x + w];
      bred[threadIdx.x] += bred[threadIdx.x + w];
      dred[threadIdx.x] += dred[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double n6 = double(g.N) * g.N * g.N * double(g.N) * g.N * g.N;
    double band_obs, whole_obs;
    bool empty;
    const double A = forcing_amplitude(a, red[0], bred[0], dred[0], n6, &band_obs, &whole_obs, &empty);
    if (empty) atomicOr(status, 0x2u);
    out[0] = A;
    out[1] = band_obs;
    out[2] = whole_obs;
  }
}
template <class T>
__global__ void k_force_amp(Geometry g, const Cplx<T>* S, int c0, int nc, const double* whole, const double* dir,
                            int nwhole, int stride, double lo2, double hi2, AmpArgs a, double* out,
                            unsigned int* status) {
  force_amp_cta<T>(g, S, c0, nc, whole, dir, nwhole, stride, lo2, hi2, a, out, status);
}

// VarianceRescaling's post-step rescale of slots [c0, c0 + nc) over the box |m_a| ≤ mb
// (grid-stride), by the factor in factor[0]. A factor of exactly 1 (an empty band) leaves the
// field untouched.
template <class T>
__global__ void k_rescale(Geometry g, Cplx<T>* S, int c0, int nc, double lo2, double hi2, const double* factor) {
  const double s = factor[0];
  if (s == 1.0) return;
  int mb = int(sqrt(hi2) / g.s) + 1;
  if (mb > g.K) mb = g.K;
  const long side = 2 * mb + 1, nbox = long(nc) * side * side * (mb + 1);
  for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nbox; i += long(gridDim.x) * blockDim.x)
    rescale_mode<T>(i, g, S, c0, mb, lo2, hi2, s);
}
template <class T, int NT>
__global__ void __launch_bounds__(NT) k_observables(Geometry g, const Cplx<T>* S, int has_scalar, double* out) {
  CTA_CTX;
  body_observables<T, NT>(c, reinterpret_cast<double*>(g_smem), g, S, has_scalar, out);
}
template <class T, int NT>
__global__ void __launch_bounds__(NT) k_spectrum(Geometry g, const Cplx<T>* S, int c0, int nc, int nshell, double* out) {
  CTA_CTX;
  double* hist = reinterpret_cast<double*>(g_smem);
  body_spectrum<T, NT>(c, hist, hist + nshell, g, S, c0, nc, nshell, out);
}
template <class T>
__global__ void k_tracers(int64_t M, const T* u, int N, double L, double* X, double* F, const __grid_constant__ AdamsStep w,
                          const uint32_t* order) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < M) tracer_one<T>(order ? int64_t(order[i]) : i, M, u, N, L, X, F, w);
}
// The warp-cooperative form for the Catmull–Rom gather: 16 lanes per tracer (two tracers per
// warp, tracers taken in the traversal order), see tracer_group.
template <class T>
__global__ void __launch_bounds__(256) k_tracers_group(int64_t M, const T* u, int N, double L, double* X, double* F,
                                                     const __grid_constant__ AdamsStep w, const uint32_t* order) {
  const int64_t i = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 4;
  const int sub = int(threadIdx.x & 15u);
  const bool live = i < M;
  const int64_t p = live ? (order ? int64_t(order[i]) : i) : 0;
  tracer_group<T>(p, M, u, N, L, X, F, w, sub, live);
}

// The traversal rebuild, a counting sort by tile: keys and tile counts, an exclusive scan of the
// counts (one block), then each tracer takes the next slot of its tile. The order within a tile
// follows the atomics and may differ between rebuilds; the gathers' results do not depend on it.
static __global__ void k_trav_count(int64_t M, const double* X, int N, double dx, uint32_t* key, uint32_t* count) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= M) return;
  const uint32_t k = traversal_key(X, p, M, N, dx);
  key[p] = k;
  atomicAdd(count + k, 1u);
}
constexpr int kScanThreads = 1024;
// Exclusive scan of the tile counts in one block: warp w scans the contiguous segment
// [w·seg, (w+1)·seg) in coalesced chunks of 32 with shuffles, after a first pass that sums the
// segments and scans those sums.
static __global__ void __launch_bounds__(kScanThreads) k_trav_scan(uint32_t* count, int nbins) {
  __shared__ uint32_t wsum[kScanThreads / 32];
  const int lane = int(threadIdx.x) & 31, w = int(threadIdx.x) >> 5;
  constexpr int NWARP = kScanThreads / 32;
  const int seg = ((nbins + NWARP - 1) / NWARP + 31) / 32 * 32;
  const int b0 = w * seg, b1 = min(nbins, b0 + seg);
  uint32_t s = 0;
  for (int b = b0 + lane; b < b1; b += 32) s += count[b];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) wsum[w] = s;
  __syncthreads();
  if (w == 0) {   // exclusive scan of the segment sums
    const uint32_t v = wsum[lane];
    uint32_t inc = v;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, off);
      if (lane >= off) inc += t;
    }
    wsum[lane] = inc - v;
  }
  __syncthreads();
  uint32_t carry = wsum[w];
  for (int base = b0; base < b1; base += 32) {
    const int b = base + lane;
    const uint32_t v = b < b1 ? count[b] : 0u;
    uint32_t inc = v;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, off);
      if (lane >= off) inc += t;
    }
    if (b < b1) count[b] = carry + inc - v;
    carry += __shfl_sync(0xffffffffu, inc, 31);
  }
}
static __global__ void k_trav_scatter(int64_t M, const uint32_t* key, uint32_t* offset, uint32_t* order) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= M) return;
  order[atomicAdd(offset + key[p], 1u)] = uint32_t(p);
}
// The bounded wait's expiry, made on purpose: one thread arms a barrier for a copy of 128 bytes
// that is never issued and waits at most `limit` cycles. The wait gives up, raises
// GBGHT_DEV_TIMEOUT in `status` and returns, as a wait on a lost copy would; no copy is in
// flight when the block exits, and the barrier is retired first.
static __global__ void k_expire_wait(unsigned int* status, long long limit) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  mbar_expect_tx(&bar, 128u);
  mbar_wait_for(&bar, 0u, status, limit);
  mbar_inval(&bar);
}

template <class T>
__global__ void k_import(Geometry g, const Cplx<double>* ref, Cplx<T>* Sc, unsigned int* flag) {
  import_mode<T>(size_t(blockIdx.x) * blockDim.x + threadIdx.x, g, ref, Sc, flag);
}
template <class T>
__global__ void k_export(Geometry g, const Cplx<T>* Sc, Cplx<double>* ref) {
  export_mode<T>(size_t(blockIdx.x) * blockDim.x + threadIdx.x, g, Sc, ref);
}
template <class T>
__global__ void k_to_T(const double* in, T* out, size_t n) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = T(in[i]);
}

// ---- the adjoint of the step (adjoint.cuh) ------------------------------------------------------
// x pass: shared memory = the NIN lines of N elements.
template <class T, int N, int NT>
__global__ void __launch_bounds__(NT, 2) k_x_adjoint(Geometry g, const Cplx<T>* Bf, Cplx<T>* Ba, int has_scalar,
                                                     const Cplx<T>* tw) {
  CTA_CTX;
  body_x_adjoint<T, N, NT>(c, reinterpret_cast<Cplx<T>*>(g_smem), g, Bf, Ba, has_scalar, tw);
}
// z pass: shared memory = the FFT tile (N·TL) and the retained rows (6·NY2·TL).
template <class T, int N, int TL, int NT>
__global__ void __launch_bounds__(NT) k_adj_z(Geometry g, AdjArgs a, Cplx<T>* Aa, Cplx<T>* L, Cplx<T>* LH,
                                              const Cplx<T>* Q, const double* coef, const Cplx<T>* tw) {
  CTA_CTX;
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(g_smem);
  body_adj_z<T, N, TL, NT>(c, W, W + N * TL, g, a, Aa, L, LH, Q, coef, tw);
}
// The band coefficients of one stage: 256 strided partial sums per field, then a fixed tree.
template <class T>
__global__ void k_adj_band(Geometry g, const Cplx<T>* Q, const Cplx<T>* LH, AdjBandArgs a, const double* amp,
                           double* coef, double* grad) {
  __shared__ double su[256], sp[256];
  double u = 0.0, p = 0.0;
  if (a.eps_u != 0.0) {
    const int mb = band_box_side(g, a.hi2), side = 2 * mb + 1, n = 3 * side * side * (mb + 1);
    for (int i = threadIdx.x; i < n; i += 256) u += band_pair_term<T>(g, Q, LH, 0, mb, a.lo2, a.hi2, i);
  }
  if (a.eps_p != 0.0) {
    const int mb = band_box_side(g, a.shi2), side = 2 * mb + 1, n = side * side * (mb + 1);
    for (int i = threadIdx.x; i < n; i += 256) p += band_pair_term<T>(g, Q, LH, 3, mb, a.slo2, a.shi2, i);
  }
  su[threadIdx.x] = u;
  sp[threadIdx.x] = p;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      su[threadIdx.x] += su[threadIdx.x + w];
      sp[threadIdx.x] += sp[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) adj_band_finish(a, amp, su[0], sp[0], coef, grad);
}
template <class T>
__global__ void k_tracer_adjoint(int64_t M, const T* u, double* lu, int N, double L, const double* X, const double* f0,
                                 double* lX, double* lf, int push, double b0, double beta_star, double beta_m) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p < M) tracer_adjoint_one<T>(p, M, u, lu, N, L, X, f0, lX, lf, push, b0, beta_star, beta_m);
}
template <class T, int N, int NW>
__global__ void __launch_bounds__(32 * NW) k_phys_forward(Geometry g, const double* lu, Cplx<T>* Ba, const Cplx<T>* tw) {
  CTA_CTX;
  body_phys_forward<T, N, NW, 32 * NW>(c, reinterpret_cast<Cplx<T>*>(g_smem), g, lu, Ba, tw);
}
template <class T>
__global__ void k_adj_add(size_t nS, int nc, Cplx<T>* L, const Cplx<T>* S, double wu, double wp) {
  adj_add_mode<T>(size_t(blockIdx.x) * blockDim.x + threadIdx.x, nS, nc, L, S, wu, wp);
}

// ------------------------------------------------------------------------------------------------
// Member-batched kernels: one launch runs a pass for every member of a group of runs with the same
// kernels (precision, N, dealiasing instantiation, scheme, scalar and forcing kinds). Each member's
// arguments are a GroupMember in device memory; the member index is the grid dimension the pass
// does not use (z for the 2-D passes, y for the 1-D ones; the y passes fold it into z with the
// component). A member's CTAs run the single-run kernel's CTA function with that member's
// arguments: the same arithmetic, in a separate compilation, so a member stepped in a group agrees
// with its lone step to round-off. The tensor maps are read from the member's record in global
// memory, written by the host before the launch and acquired by the thread that issues the copies.
// ------------------------------------------------------------------------------------------------
constexpr int kGroupStages = 5;
// the maps of a member's record, acquired by the thread that issues the TMA copies
__device__ __forceinline__ void acquire_maps(const TmaMaps& m) {
  if (threadIdx.x == 0) {
    tensormap_acquire(&m.a_ld);
    tensormap_acquire(&m.a_st1);
    tensormap_acquire(&m.a_st2);
    tensormap_acquire(&m.b);
    tensormap_acquire(&m.az);
    tensormap_acquire(&m.s3);
    tensormap_acquire(&m.h3);
  }
}
template <class T>
struct alignas(64) GroupMember {
  TmaMaps maps;
  Geometry g;
  Cplx<T>* A;
  Cplx<T>* B;
  Cplx<T>* S;
  Cplx<T>* H;
  T* U;
  double* partial;
  double* amp;
  unsigned int* status;
  unsigned long long* maxbits;
  int ntile;                      // the epilogue's tile partials (ConstantPower's whole-field sum)
  double band_lo2, band_hi2;      // the velocity forcing's band
  AmpArgs vamp;                   // the velocity forcing's amplitude arguments
  StageArgs st[kGroupStages];     // the step's stages
};

template <class T, int N, int TL, int NT>
__global__ void __launch_bounds__(NT, sizeof(T) == 8 ? 2 : 3) kg_y_inverse(const GroupMember<T>* grp, int c0, int nc,
                                                                         const Cplx<T>* tw) {
  const GroupMember<T>& M = grp[blockIdx.z / nc];
  acquire_maps(M.maps);
  const Cta c{int(threadIdx.x), int(blockIdx.x), int(blockIdx.y), int(blockIdx.z % nc)};
  y_inverse_cta<T, N, TL, NT>(c, M.maps, M.g, c0 + c.bz, tw, M.status);
}
template <class T, int N, int TL, int NT>
__global__ void __launch_bounds__(NT, sizeof(T) == 8 ? 2 : 3) kg_y_forward(const GroupMember<T>* grp, int nc,
                                                                         const Cplx<T>* tw) {
  const GroupMember<T>& M = grp[blockIdx.z / nc];
  acquire_maps(M.maps);
  const Cta c{int(threadIdx.x), int(blockIdx.x), int(blockIdx.y), int(blockIdx.z % nc)};
  y_forward_cta<T, N, TL, NT>(c, M.maps, M.g, c.bz, tw, M.status);
}
template <class T, int N, int NT>
__global__ void __launch_bounds__(NT, XShape<T>::STAGED ? 2 : 3) kg_x_products(const GroupMember<T>* grp, int has_scalar,
                                                                              int KXS, const Cplx<T>* tw) {
  const GroupMember<T>& M = grp[blockIdx.y];
  const Cta c{int(threadIdx.x), int(blockIdx.x), 0, 0};
  x_products_cta<T, N, NT>(c, M.g, M.B, has_scalar, KXS, tw, M.status);
}
template <class T, int N, int NT>
__global__ void __launch_bounds__(NT, 2) kg_x_velocity(const GroupMember<T>* grp, int KXS, const Cplx<T>* tw) {
  const GroupMember<T>& M = grp[blockIdx.y];
  const Cta c{int(threadIdx.x), int(blockIdx.x), 0, 0};
  x_velocity_cta<T, N, NT>(c, M.g, M.B, M.U, M.maxbits, KXS, tw, M.status);
}
template <class T, int N, int TL, int NT, int KIND, int KM, bool WIDE>
__global__ void __launch_bounds__(NT, NT > 256 ? 1 : (sizeof(T) == 8 ? 2 : 4)) kg_z_epilogue(const GroupMember<T>* grp,
                                                                                            int stage, const Cplx<T>* tw) {
  const GroupMember<T>& M = grp[blockIdx.z];
  acquire_maps(M.maps);
  const Cta c{int(threadIdx.x), int(blockIdx.x), int(blockIdx.y), 0};
  z_epilogue_cta<T, N, TL, NT, KIND, KM, WIDE>(c, M.maps, M.g, M.A, M.S, M.H, M.st[stage], M.amp, M.partial, tw,
                                               M.status);
}
// the first tile column of A rebuilt after the reality projection (grid (1, NY2, members))
template <class T, int N, int TL, int NT, int KM>
__global__ void __launch_bounds__(NT, NT > 256 ? 1 : 2) kg_z_init_column(const GroupMember<T>* grp, int has_scalar,
                                                                       int pstride, const Cplx<T>* tw) {
  const GroupMember<T>& M = grp[blockIdx.z];
  const Cta c{int(threadIdx.x), int(blockIdx.x), int(blockIdx.y), 0};
  z_init_cta<T, N, TL, NT, KM>(c, M.g, M.A, M.S, has_scalar, M.partial, tw, 1, pstride, 0);
}
template <class T>
__global__ void kg_reality(const GroupMember<T>* grp, int ncomp) {
  const GroupMember<T>& M = grp[blockIdx.y];
  reality_mode<T>(int(blockIdx.x * blockDim.x + threadIdx.x), M.g, M.S, ncomp);
}
// ConstantPower's velocity amplitude from the epilogue's tile partials (grid (members), 256 threads)
template <class T>
__global__ void __launch_bounds__(256) kg_force_amp(const GroupMember<T>* grp) {
  const GroupMember<T>& M = grp[blockIdx.x];
  force_amp_cta<T>(M.g, M.S, 0, 3, M.partial, nullptr, M.ntile, 1, M.band_lo2, M.band_hi2, M.vamp, M.amp, M.status);
}
template <class T>
__global__ void kg_zero_maxbits(const GroupMember<T>* grp, int n) {
  const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i < n) *grp[i].maxbits = 0ull;
}
#endif

}  // namespace gbght
