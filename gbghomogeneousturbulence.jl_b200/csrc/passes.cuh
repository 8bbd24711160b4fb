// The passes of one IF-RK stage, written as CTA bodies (see gbght_common.cuh for the execution
// model).
//
// Layouts in HBM (complex elements; K is the largest retained |m| per axis, NY2 = 2K+1, KXP is
// K+1 rounded up to a whole number of 128-byte rows). Every retained mode of the 2/3 ball has
// |m_x|, |m_y|, |m_z| ≤ K, so the spectral state is stored compactly. The transforms are pruned
// to that box: an inverse pass never reads a mode outside the box, and a forward pass never writes
// one.
//   compact index q ∈ [0, NY2) ↔ m = q for q ≤ K, m = q − NY2 for q > K
//   FFT row of q: e(q) = q (q ≤ K) or q + N − NY2 (q > K)
//   S-layout  [c][ky'][kz'][kx]  state û, φ̂ and the accumulators h        (NY2·NY2·KXP)
//   A-layout  [c][z][ky'][kx]    z-transformed spectra                     (N·NY2·KXP)
//   B-layout  [c][z][y][kx]      y- and z-transformed spectra              (N·N·KXP)
//   physical  [c][z][y][x]       real values, x contiguous                 (N·N·N)
// Component slots: 0-2 velocity, 3-5 vorticity, 6 scalar (A and B). After the x-pass, B slots
// 0-2 hold FFT(u×ω) and slots 3-5 hold FFT(uφ) (x transformed only). After the forward y-pass,
// A slots 0-5 hold them y-transformed as well.
//
// A stage runs: y-inverse (A→B), x-pass (B→B: c2r, products, r2c), y-forward (B→A), then
// z-forward + epilogue + z-inverse (A, S, H → S, H, A).
#pragma once

#include "fft_tile.cuh"
#include "tma.cuh"
#include "tmem.cuh"
#include "warp_fft.cuh"

namespace gbght {

struct Geometry {
  int N, K, NY2, KXP;
  double s;          // 2π/L, the fundamental wavenumber
  double cut2;       // square of the dealias cutoff T(2/3)·T(N/2)·T(2π/L); ∞ under HouLi (no cutoff)
  double inv_norm;   // 1/N³, the inverse transform's normalisation
  int houli;         // 1: HouLi's smooth filter multiplies the nonlinear terms (no sharp cutoff)
  double filt_strength, filt_half_order, inv_kny2;   // its strength, order/2, 1/κ_Ny²
};

// HouLi's filter exp(−strength·(|κ|/κ_Ny)^order) at |κ|² = k2 (src/SimulationDomain.jl:365-376).
GBGHT_HD double dealias_filter(const Geometry& g, double k2) {
  return exp(-g.filt_strength * pow(k2 * g.inv_kny2, g.filt_half_order));
}

GBGHT_HD int q_to_m(int q, int K, int NY2) { return q <= K ? q : q - NY2; }
GBGHT_HD int q_to_row(int q, int K, int N, int NY2) { return q <= K ? q : q + N - NY2; }

// PhaseShift's translation symbol e^{iπ·m/N} for the integer wavenumber sum m = mx + my + mz: the
// factor that samples a mode on the grid displaced by half a cell along every axis (κ·δ = π·m/N
// for δ = L/(2N) per axis); its conjugate shifts a displaced term back. m is reduced to (−N, N]
// first, so the argument of sincospi stays within [−1, 1].
template <class T>
GBGHT_HD Cplx<T> half_cell_phase(int m, int N) {
  int r = m % (2 * N);
  if (r > N) r -= 2 * N;
  if (r <= -N) r += 2 * N;
  double sn, cs;
#ifdef __CUDA_ARCH__
  sincospi(double(r) / double(N), &sn, &cs);
#else
  const double a = 3.14159265358979323846 * (double(r) / double(N));
  sn = std::sin(a);
  cs = std::cos(a);
#endif
  return cmk<T>(T(cs), T(sn));
}

GBGHT_HD size_t idxA(const Geometry& g, int c, int z, int q, int kx) {
  return ((size_t(c) * g.N + z) * g.NY2 + q) * g.KXP + kx;
}
GBGHT_HD size_t idxB(const Geometry& g, int c, int z, int y, int kx) {
  return ((size_t(c) * g.N + z) * g.N + y) * g.KXP + kx;
}
GBGHT_HD size_t idxS(const Geometry& g, int c, int qy, int qz, int kx) {
  return ((size_t(c) * g.NY2 + qy) * g.NY2 + qz) * g.KXP + kx;
}

// ================================================================================================
// Tensor maps for the TMA tile copies (device build only).
//   a_ld   A as rows of KXP elements (dims {2·KXP reals, 7·N·NY2 rows}), box {2·TLY, K+1}
//   a_st1  the same rows, box {2·TLY, K+1};  a_st2: box {2·TLY, K}
//   b      B as rows (dims {2·KXP, 7·N·N}), box {2·TLY, BY}, BY the largest divisor of N ≤ 256
//   az     A as (x, q, c·N + z) (dims {2·KXP, NY2, 7·N}), box {2·TLZ, 1, BZ}, BZ = BY
//   s3/h3  S and H as (x, q_z, c·NY2 + q_y) (dims {2·KXP, NY2, 4·NY2}), box {2·TLZ, K+1, 1}
// Innermost coordinates are 2·kx0 reals with kx0 a multiple of the tile width, so every copy
// starts on a 64- or 128-byte boundary.
// ================================================================================================
// Rows per box of the tensor maps along a length-N dimension: the largest divisor of N ≤ 256.
template <int N> constexpr int box_rows() { return N > 256 ? (N % 256 == 0 ? 256 : N / 2) : N; }

struct TmaMaps {
#if defined(__CUDACC__) && !defined(GBGHT_EMU)
  CUtensorMap a_ld, a_st1, a_st2, b, az, s3, h3;
#else
  int unused;
#endif
};

// ================================================================================================
// y-inverse: A[c][z][ky'][tile] → B[c][z][y][tile], one tile of TL kx columns per CTA.
// Grid: (KXP/TL, N, ncomp); c = c0 + bz. The tile is N rows of TL elements (rows of 128 bytes).
// Compact rows q ≤ K land in rows 0..K, rows q > K in rows N−NY2+q; the rows between are zero.
// ================================================================================================
template <class T, int N, int TL>
GBGHT_HD void y_inverse_load_host(const Cta& c, Cplx<T>* sm, const Geometry& g, const Cplx<T>* A, int c0) {
  const int kx0 = c.bx * TL, z = c.by, comp = c0 + c.bz;
  for (int e = 0; e < N; ++e)
    for (int l = 0; l < TL; ++l) {
      int q = -1;
      if (e <= g.K) q = e;
      else if (e >= N - g.K) q = e - N + g.NY2;
      sm[e * TL + l] = q >= 0 ? A[idxA(g, comp, z, q, kx0 + l)] : czero<T>();
    }
}

template <class T, int N, int TL>
GBGHT_HD void y_store_host(const Cta& c, const Cplx<T>* sm, const Geometry& g, Cplx<T>* B, int comp) {
  const int kx0 = c.bx * TL, z = c.by;
  for (int y = 0; y < N; ++y)
    for (int l = 0; l < TL; ++l) B[idxB(g, comp, z, y, kx0 + l)] = sm[y * TL + l];
}

template <class T, int N, int TL>
GBGHT_HD void y_forward_load_host(const Cta& c, Cplx<T>* sm, const Geometry& g, const Cplx<T>* B) {
  const int kx0 = c.bx * TL, z = c.by, comp = c.bz;
  for (int y = 0; y < N; ++y)
    for (int l = 0; l < TL; ++l) sm[y * TL + l] = B[idxB(g, comp, z, y, kx0 + l)];
}

template <class T, int N, int TL>
GBGHT_HD void y_forward_store_host(const Cta& c, const Cplx<T>* sm, const Geometry& g, Cplx<T>* A) {
  const int kx0 = c.bx * TL, z = c.by, comp = c.bz;
  for (int q = 0; q < g.NY2; ++q)
    for (int l = 0; l < TL; ++l) A[idxA(g, comp, z, q, kx0 + l)] = sm[q_to_row(q, g.K, N, g.NY2) * TL + l];
}

// zero rows K < e < N−K, then the inverse transform
template <class T, int N, int TL, int NT>
GBGHT_HD void y_inverse_compute(const Cta& c, Cplx<T>* sm, const Geometry& g, const Cplx<T>* GBGHT_RESTRICT tw) {
  for (int i = c.tid; i < (N - 2 * g.K - 1) * TL; i += NT) sm[(g.K + 1) * TL + i] = czero<T>();
  GBGHT_SYNC();
  tile_fft<T, N, TL, NT, +1>(c, sm, tw);
}

// ================================================================================================
// x-pass: for P points (z, y0..y0+P−1), c2r of u, ω, φ, the products u×ω and uφ, and r2c of the
// six products. The spectra stay in B's slots (in place). Two tiles per CTA.
// P = TL/4 points (2 in FP64, 4 in FP32) share a tile of lines, each line N elements in shared
// memory, transformed by one warp (warp_fft.cuh):
//   inverse: line 3p+0 = u_x + i·u_y, 3p+1 = u_z + i·ω_x, 3p+2 = ω_y + i·ω_z (point p), and line
//            3P + p/2 = φ(p) + i·φ(p+1) for even p: 3P + P/2 lines in use
//   forward: line 3p+0 = n_x + i·n_y, 3p+1 = n_z + i·f_x, 3p+2 = f_y + i·f_z, n = u×ω, f = uφ
// Two real lines a, b share one complex transform ("two for one"). Inverse: Z[e] = A[e] + i·B[e]
// for 0 ≤ e ≤ K, and Z[N−e] = conj(A[e]) + i·conj(B[e]); only the real parts of the kx = 0 bins
// enter, as in a c2r. Forward: A[k] = (Z[k] + conj Z[N−k])/2, B[k] = (Z[k] − conj Z[N−k])/(2i).
// The spectra come in through a staging area of rows [c][p][KXS] (KXS ≥ K+1 elements, a
// multiple of 16 bytes), filled by bulk copies from B.
// ================================================================================================
template <class T> struct XShape {
  static constexpr int TL = 128 / int(sizeof(Cplx<T>));
  static constexpr int P = TL / 4;                 // points per tile (x pass)
  static constexpr int ACT_INV = 3 * P + P / 2;
  static constexpr int ACT_FWD = 3 * P;
  static constexpr int NW = sizeof(Cplx<T>) == 16 ? 7 : 8;   // warps of the x pass (≥ 1 turnaround item per thread)
  // A tile's spectra are staged in shared memory by bulk copies, overlapping the next tile's load
  // with the current tile's transforms. (Unstaged, with the first inverse stage reading global
  // memory, the FP32 pass fits three CTAs per SM but took 4.18 ms per 512³ launch against 3.02 ms
  // staged at two, so both forms stage.)
  static constexpr bool STAGED = true;
  static constexpr int PV = TL / 2;                // points per tile (deposit pass)
  static constexpr int ACT_V = PV + PV / 2;
};

GBGHT_HD int x_kxs(int K, int elem_bytes) {
  const int per = 16 / elem_bytes;   // elements per 16 bytes (1 for FP64 complex, 2 for FP32)
  return ((K + 1 + per - 1) / per) * per;
}

// One line of an (e, l)-indexed source, for the warp-per-line transform.
template <class Src>
struct LineOfSource {
  static constexpr bool kExternal = true;
  const Src& s;
  int l;
  GBGHT_HD auto load(int e) const { return s.load(e, l); }
};

// Source of the x-pass inverse's first stage: row e of line l from the staging rows [c][p][KXS]
// in shared memory, packed two-for-one (a c2r input: only the real part of the kx = 0 bin, rows
// K < e < N−K zero), scaled by 1/N³. Lines 3p..3p+2 pair comps (0,1), (2,3), (4,5) of point p;
// line 3P + h pairs φ of points 2h, 2h+1.
template <class T, int N, int P>
struct XStagedSource {
  static constexpr bool kExternal = true;
  const Geometry& g;
  const Cplx<T>* stg;
  int KXS, has_scalar;
  T sc;
  const Cplx<T>* B = nullptr;   // unstaged (XShape<T>::STAGED false): the tile's rows in B
  int z = 0, y0 = 0;
  GBGHT_HD Cplx<T> row(int r, int m) const {
    if constexpr (XShape<T>::STAGED) return stg[r * KXS + m];
    else return B[idxB(g, r / P, z, y0 + r % P, m)];
  }
  GBGHT_HD Cplx<T> load(int e, int l) const {
    const int K = g.K;
    if (e > K && e < N - K) return czero<T>();
    int ra, rb;   // staging rows of the pair
    if (l < 3 * P) {
      const int p = l / 3, pr = l % 3;
      ra = (2 * pr) * P + p;
      rb = (2 * pr + 1) * P + p;
    } else {
      if (!has_scalar) return czero<T>();
      const int h = l - 3 * P;
      ra = 6 * P + 2 * h;
      rb = ra + 1;
    }
    const int m = e <= K ? e : N - e;
    const Cplx<T> a = row(ra, m), b = row(rb, m);
    if (e == 0) return cmk<T>(a.x * sc, b.x * sc);
    if (e <= K) return cmk<T>((a.x - b.y) * sc, (a.y + b.x) * sc);
    return cmk<T>((a.x + b.y) * sc, (b.x - a.y) * sc);
  }
};

// Staging of one x tile: the rows B[c][z][y0+p][0..KXS) of comps c < nin, as untiled bulk copies
// completing on `bar` (device), or plain copies (host-check build).
template <class T, int P, bool ON = true>
struct XStaging {
  const Geometry& g;
  const Cplx<T>* B;
  Cplx<T>* stg;
  int KXS, nin;
  uint64_t* bar;
  unsigned int* status;
  GBGHT_HD void issue(const Cta& c, int z, int y0) const {
    if constexpr (!ON) return;
#ifdef __CUDA_ARCH__
    if (c.tid == 0) {
      const uint32_t row = uint32_t(KXS * sizeof(Cplx<T>));
      mbar_expect_tx(bar, row * uint32_t(nin * P));
      for (int cc = 0; cc < nin; ++cc)
        for (int p = 0; p < P; ++p) bulk_load(stg + (cc * P + p) * KXS, B + idxB(g, cc, z, y0 + p, 0), row, bar);
    }
#else
    (void)c;
    for (int cc = 0; cc < nin; ++cc)
      for (int p = 0; p < P; ++p)
        for (int e = 0; e < KXS; ++e) stg[(cc * P + p) * KXS + e] = B[idxB(g, cc, z, y0 + p, e)];
#endif
  }
  GBGHT_HD void wait(uint32_t phase) const {
    if constexpr (!ON) return;
#ifdef __CUDA_ARCH__
    mbar_wait(bar, phase, status);
#else
    (void)phase;
#endif
  }
};
template <class T> using XProductStaging = XStaging<T, XShape<T>::P, XShape<T>::STAGED>;

// A host-device function kept out of line on the device: one copy of a body that a kernel calls
// several times, to keep the kernel's code within the instruction cache.
#ifdef __CUDACC__
#define GBGHT_HD_OUTLINE __host__ __device__ __noinline__
#else
#define GBGHT_HD_OUTLINE inline
#endif

// The turnaround of an x tile. Every plan starts and ends with the same radix R, so butterfly j of
// the inverse's last stage produces exactly the points x = j + r·N/R (r < R) that butterfly j of
// the forward's first stage consumes. One thread per (j, point p) therefore runs, in registers:
// - the last inverse stage of lines 3p, 3p+1, 3p+2 (u, ω) and of p's φ line;
// - the products n = u×ω and f = uφ at those R points;
// - the first forward stage of the three product lines.
// Only the product lines' first-stage outputs (rows j·R + r) go back to shared memory. All reads
// come before the barrier and all writes after it, since the outputs overwrite rows that other
// threads read.
template <class T, int N, int NT>
GBGHT_HD void x_turnaround(const Cta& c, Cplx<T>* sm, const Cplx<T>* GBGHT_RESTRICT tw) {
  constexpr int P = XShape<T>::P;
  constexpr int S = Radices<N>::n - 1;
  constexpr int R = Radices<N>::r[S];
  static_assert(S > 0 && R == Radices<N>::r[0], "the turnaround needs two stages or more and equal end radices");
  constexpr int NB = N / R;
  constexpr int ITEMS = NB * P;
  constexpr int SLOTS = (ITEMS + NT - 1) / NT;
  Cplx<T> out[SLOTS][3][R];
  const auto inv_last = [&](int line, int j, Cplx<T>* v) {
    const Cplx<T>* L = sm + line * N;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = L[lidx<T>(j + r * NB)];
    Cplx<T> w[R];
    twiddles<T, R, +1>(tw, j, w);
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = v[r] * w[r];
    dft<T, R, +1>(v);
  };
  const auto products = [&](int p, const Cplx<T>* a, const Cplx<T>* b, const Cplx<T>* d, const Cplx<T>* ph,
                            Cplx<T> (&o)[3][R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const T ux = a[r].x, uy = a[r].y, uz = b[r].x, wx = b[r].y, wy = d[r].x, wz = d[r].y;
      const T phi = (p & 1) ? ph[r].y : ph[r].x;
      o[0][r] = cmk<T>(uy * wz - uz * wy, uz * wx - ux * wz);
      o[1][r] = cmk<T>(ux * wy - uy * wx, ux * phi);
      o[2][r] = cmk<T>(uy * phi, uz * phi);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) dft<T, R, -1>(o[k]);
  };
  // When the items leave enough threads idle (FP64), those threads run the φ lines' last stage
  // in place meanwhile, and each item reads φ after a barrier instead of transforming its φ line
  // itself (that transform is shared by two points).
  constexpr int PHI = NB * (P / 2);
  constexpr bool kPhiAside = SLOTS == 1 && ITEMS + PHI <= NT;
  if constexpr (kPhiAside) {
    const int it = c.tid;
    const int j = it % NB, p = it / NB;
    Cplx<T> a[R], b[R], d[R];
    if (it < ITEMS) {
      inv_last(3 * p, j, a);        // u_x + i·u_y
      inv_last(3 * p + 1, j, b);    // u_z + i·ω_x
      inv_last(3 * p + 2, j, d);    // ω_y + i·ω_z
    } else if (it < ITEMS + PHI) {
      const int k = it - ITEMS, jj = k % NB, h = k / NB;
      Cplx<T> v[R];
      inv_last(3 * P + h, jj, v);   // φ(2h) + i·φ(2h+1), back into its line (rows jj + r·NB)
      Cplx<T>* L = sm + (3 * P + h) * N;
#pragma unroll
      for (int r = 0; r < R; ++r) L[lidx<T>(jj + r * NB)] = v[r];
    }
    GBGHT_SYNC();
    if (it < ITEMS) {
      const Cplx<T>* L = sm + (3 * P + p / 2) * N;
      Cplx<T> ph[R];
#pragma unroll
      for (int r = 0; r < R; ++r) ph[r] = L[lidx<T>(j + r * NB)];
      products(p, a, b, d, ph, out[0]);
    }
  } else {
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int it = c.tid + s * NT;
      if (SLOTS * NT == ITEMS || it < ITEMS) {
        const int j = it % NB, p = it / NB;
        Cplx<T> ph[R], a[R], b[R], d[R];
        inv_last(3 * P + p / 2, j, ph);   // φ(2h) + i·φ(2h+1)
        inv_last(3 * p, j, a);            // u_x + i·u_y
        inv_last(3 * p + 1, j, b);        // u_z + i·ω_x
        inv_last(3 * p + 2, j, d);        // ω_y + i·ω_z
        products(p, a, b, d, ph, out[s]);
      }
    }
  }
  GBGHT_SYNC();
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    const int it = c.tid + s * NT;
    if (SLOTS * NT == ITEMS || it < ITEMS) {
      const int j = it % NB, p = it / NB;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        Cplx<T>* L = sm + (3 * p + k) * N;
#pragma unroll
        for (int r = 0; r < R; ++r) L[lidx<T>(j * R + r)] = out[s][k][r];
      }
    }
  }
  GBGHT_SYNC();
}

// One x tile: the inverse of the staged spectra (the first stage reads the staging; after it the
// staging is free and the next tile's copies are issued), the turnaround (last inverse stage,
// products, first forward stage), the rest of the forward transform, and the unpack into B.
template <class T, int N, int NT>
GBGHT_HD void x_tile(const Cta& c, Cplx<T>* sm, const XProductStaging<T>& stage,
                                    const XStagedSource<T, N, XShape<T>::P>& src0, const Geometry& g,
                                    Cplx<T>* GBGHT_RESTRICT B, int nout, int z, int y0, int next_z, int next_y0,
                                    const Cplx<T>* GBGHT_RESTRICT tw) {
  using X = XShape<T>;
  constexpr int P = X::P, NW = X::NW;
  const int KX1 = g.K + 1;
  XStagedSource<T, N, P> src = src0;   // the tile's position, for the unstaged source
  src.z = z;
  src.y0 = y0;
  const auto lines = [&](int l) { return sm + l * N; };
  const auto from_stg = [&](int l) { return LineOfSource<XStagedSource<T, N, P>>{src, l}; };
  const auto in_smem = [&](int l) { return LineBuf<T>{sm + l * N}; };
  warp_fft_lines<T, N, NW, NT, +1, 0, 1>(c, X::ACT_INV, lines, from_stg, in_smem, tw);
  // The staging is free once every warp's first stage has read it. On the device only the issuing
  // warp waits for that (barrier 1: the other warps arrive, with release semantics, and go on to
  // their next stages, which touch only their own lines); the lines themselves are next read across
  // warps at the turnaround, after the block barrier there.
#if defined(__CUDA_ARCH__) && !defined(GBGHT_EMU)
  if (next_z >= 0) {
    if (c.tid < 32) {
      asm volatile("barrier.sync 1, %0;" ::"r"(NT) : "memory");
      stage.issue(c, next_z, next_y0);
    } else {
      asm volatile("barrier.arrive 1, %0;" ::"r"(NT) : "memory");
    }
  }
#else
  GBGHT_SYNC();
  if (next_z >= 0) stage.issue(c, next_z, next_y0);
#endif
  if constexpr (Radices<N>::n >= 2) {
    // inverse stages up to the last, then the turnaround (last inverse stage, products, first
    // forward stage), then the forward's remaining stages
    warp_fft_lines<T, N, NW, NT, +1, 1, Radices<N>::n - 1>(c, X::ACT_INV, lines, from_stg, in_smem, tw);
    GBGHT_SYNC();
    x_turnaround<T, N, NT>(c, sm, tw);
    warp_fft_lines<T, N, NW, NT, -1, 1>(c, X::ACT_FWD, lines, in_smem, in_smem, tw);
  } else {
  warp_fft_lines<T, N, NW, NT, +1, 1>(c, X::ACT_INV, lines, from_stg, in_smem, tw);
  GBGHT_SYNC();
  for (int x = c.tid; x < N; x += NT) {
    const int ix = lidx<T>(x);
#pragma unroll
    for (int h = 0; h < P / 2; ++h) {
      const Cplx<T> lp = sm[(3 * P + h) * N + ix];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int p = 2 * h + q;
        const Cplx<T> L0 = sm[(3 * p) * N + ix], L1 = sm[(3 * p + 1) * N + ix], L2 = sm[(3 * p + 2) * N + ix];
        const T ux = L0.x, uy = L0.y, uz = L1.x, wx = L1.y, wy = L2.x, wz = L2.y;
        const T ph = q == 0 ? lp.x : lp.y;
        const T nx = uy * wz - uz * wy, ny = uz * wx - ux * wz, nz = ux * wy - uy * wx;
        sm[(3 * p) * N + ix] = cmk<T>(nx, ny);
        sm[(3 * p + 1) * N + ix] = cmk<T>(nz, ux * ph);
        sm[(3 * p + 2) * N + ix] = cmk<T>(uy * ph, uz * ph);
      }
    }
  }
  GBGHT_SYNC();
  warp_fft_lines<T, N, NW, NT, -1>(c, X::ACT_FWD, lines, in_smem, in_smem, tw);
  }
  // unpack each line (by its owning warp) into B: line 3p+pr → comps (2pr, 2pr+1) of point p;
  // columns past K get zeros
  for (int t = c.tid; t < 32 * NW; t += NT) {
    const int w = t >> 5, lane = t & 31;
    for (int line = w; line < X::ACT_FWD; line += NW) {
      const int p = line / 3, pr = line % 3;
      const int ca = 2 * pr, cb = 2 * pr + 1;
      const Cplx<T>* L = sm + line * N;
      for (int k = lane; k < g.KXP; k += 32) {
        Cplx<T> a = czero<T>(), b = czero<T>();
        if (k < KX1) {
          const Cplx<T> zk = L[lidx<T>(k)];
          const Cplx<T> zc = conj(L[lidx<T>((N - k) % N)]);
          const Cplx<T> sp = zk + zc, sd = zk - zc;
          a = cmk<T>(sp.x * T(0.5), sp.y * T(0.5));
          b = cmk<T>(sd.y * T(0.5), -sd.x * T(0.5));
        }
        if (ca < nout) B[idxB(g, ca, z, y0 + p, k)] = a;
        if (cb < nout) B[idxB(g, cb, z, y0 + p, k)] = b;
      }
    }
  }
  // The next tile's first inverse stage rewrites each line from the warp that owns it here (line l
  // belongs to warp l mod NW in every warp-per-line stage and in the unpack), and every cross-warp
  // read of the lines (the turnaround) ended at a block barrier, so the warp's own order suffices.
  warp_sync();
}

// Tiles I, I+1, … < XT of this CTA (tile index bx + i·grid); tile I's spectra are already being
// copied into the staging rows.
constexpr int XT = 2;
template <class T, int N, int NT, int I>
GBGHT_HD void x_tile_chain(const Cta& c, Cplx<T>* sm, const XProductStaging<T>& stage,
                           const XStagedSource<T, N, XShape<T>::P>& src, const Geometry& g, Cplx<T>* B, int nout,
                           int grid, int ntiles, const Cplx<T>* tw) {
  if constexpr (I < XT) {
    constexpr int P = XShape<T>::P;
    const int tiles_y = N / P;
    const int t = c.bx + I * grid, tn = t + grid;
    const bool more = I + 1 < XT && tn < ntiles;
    stage.wait(uint32_t(I & 1));
    x_tile<T, N, NT>(c, sm, stage, src, g, B, nout, t / tiles_y, P * (t % tiles_y), more ? tn / tiles_y : -1,
                     more ? P * (tn % tiles_y) : 0, tw);
    if (more) x_tile_chain<T, N, NT, I + 1>(c, sm, stage, src, g, B, nout, grid, ntiles, tw);
  }
}

// The x pass over the tiles bx, bx + grid, …: one warp per line, lines at sm + l·N, the next
// tile's spectra prefetched into the staging rows while the current tile is transformed.
template <class T, int N, int NT>
GBGHT_HD void body_x_products(const Cta& c, Cplx<T>* sm, Cplx<T>* stg, int KXS, uint64_t* bar, int grid,
                              const Geometry& g, Cplx<T>* GBGHT_RESTRICT B, int has_scalar,
                              const Cplx<T>* GBGHT_RESTRICT tw, unsigned int* status) {
  using X = XShape<T>;
  constexpr int P = X::P;
  const int nin = has_scalar ? 7 : 6, nout = has_scalar ? 6 : 3;
  const int tiles_y = N / P, ntiles = tiles_y * N;
  const XProductStaging<T> stage{g, B, stg, KXS, nin, bar, status};
  XStagedSource<T, N, P> src{g, stg, KXS, has_scalar, T(g.inv_norm)};
  src.B = B;
  // XT tiles per CTA, written out by template recursion rather than looped (a loop around the
  // tile makes the compiler keep the tile's index arithmetic live across iterations, and the
  // kernel spills): tile bx + i·grid, with the spectra of tile i + 1 copied in while tile i is
  // transformed.
  if (c.bx >= ntiles) return;
  stage.issue(c, c.bx / tiles_y, P * (c.bx % tiles_y));
  x_tile_chain<T, N, NT, 0>(c, sm, stage, src, g, B, nout, grid, ntiles, tw);
}

// Source of the deposit's inverse from the staging rows [c][p][KXS] (c = 0..2) in shared memory:
// line p (p < PV) = u_x + i·u_y of point p; line PV + h = u_z(2h) + i·u_z(2h+1). Packed two-for-one
// as in XStagedSource (a c2r input: only the real part of the kx = 0 bin, rows K < e < N−K zero),
// scaled by 1/N³.
template <class T, int N, int PV>
struct XVelocityStagedSource {
  static constexpr bool kExternal = true;
  const Geometry& g;
  const Cplx<T>* stg;
  int KXS;
  T sc;
  GBGHT_HD Cplx<T> load(int e, int l) const {
    const int K = g.K;
    if (e > K && e < N - K) return czero<T>();
    int ra, rb;   // staging rows of the pair
    if (l < PV) {
      ra = l;
      rb = PV + l;
    } else {
      ra = 2 * PV + 2 * (l - PV);
      rb = ra + 1;
    }
    const int m = e <= K ? e : N - e;
    const Cplx<T> a = stg[ra * KXS + m], b = stg[rb * KXS + m];
    if (e == 0) return cmk<T>(a.x * sc, b.x * sc);
    if (e <= K) return cmk<T>((a.x - b.y) * sc, (a.y + b.x) * sc);
    return cmk<T>((a.x + b.y) * sc, (b.x - a.y) * sc);
  }
};

GBGHT_HD double max_nan(double a, double b) { return (b > a || b != b) ? b : a; }

// One deposit tile (PV points z, y0..y0+PV−1): the inverse of the staged spectra (after its first
// stage the staging is free and the next tile's copies are issued), then the physical velocity
// written out; returns this thread's max |u|² (NaN wins).
template <class T, int N, int NT, class TW>
GBGHT_HD double x_velocity_tile(const Cta& c, Cplx<T>* sm, const XStaging<T, XShape<T>::PV>& stage,
                                const XVelocityStagedSource<T, N, XShape<T>::PV>& src, T* GBGHT_RESTRICT u_phys,
                                int z, int y0, int next_z, int next_y0, const TW& tw) {
  using X = XShape<T>;
  constexpr int PV = X::PV, NW = 6;
  const auto lines = [&](int l) { return sm + l * N; };
  const auto from_stg = [&](int l) { return LineOfSource<XVelocityStagedSource<T, N, PV>>{src, l}; };
  const auto in_smem = [&](int l) { return LineBuf<T>{sm + l * N}; };
  warp_fft_lines<T, N, NW, NT, +1, 0, 1>(c, X::ACT_V, lines, from_stg, in_smem, tw);
  GBGHT_SYNC();
  if (next_z >= 0) stage.issue(c, next_z, next_y0);
  warp_fft_lines<T, N, NW, NT, +1, 1>(c, X::ACT_V, lines, from_stg, in_smem, tw);
  GBGHT_SYNC();
  double m = 0.0;
  const size_t comp = size_t(N) * N * N;
  for (int i = c.tid; i < PV * N; i += NT) {
    const int x = i % N, p = i / N;
    const int ix = lidx<T>(x);
    const Cplx<T> uxy = sm[p * N + ix];
    const Cplx<T> uzz = sm[(PV + (p >> 1)) * N + ix];
    const T uz = (p & 1) ? uzz.y : uzz.x;
    const size_t base = (size_t(z) * N + (y0 + p)) * N + x;
    u_phys[base] = uxy.x;
    u_phys[comp + base] = uxy.y;
    u_phys[2 * comp + base] = uz;
    const double sp = (double(uxy.x) * double(uxy.x) + double(uxy.y) * double(uxy.y)) + double(uz) * double(uz);
    m = max_nan(m, sp);
  }
  GBGHT_SYNC();   // the lines are rewritten by the next tile's inverse
  return m;
}

// Tiles I, I+1, … < XT of this CTA (tile bx + i·grid), written out by template recursion as in
// the x pass; tile I's spectra are already being copied into the staging rows.
template <class T, int N, int NT, int I, class TW>
GBGHT_HD double x_velocity_chain(const Cta& c, Cplx<T>* sm, const XStaging<T, XShape<T>::PV>& stage,
                                 const XVelocityStagedSource<T, N, XShape<T>::PV>& src, T* u_phys, int grid,
                                 int ntiles, const TW& tw) {
  if constexpr (I < XT) {
    constexpr int PV = XShape<T>::PV;
    const int tiles_y = N / PV;
    const int t = c.bx + I * grid, tn = t + grid;
    const bool more = I + 1 < XT && tn < ntiles;
    stage.wait(uint32_t(I & 1));
    double m = x_velocity_tile<T, N, NT>(c, sm, stage, src, u_phys, t / tiles_y, PV * (t % tiles_y),
                                         more ? tn / tiles_y : -1, more ? PV * (tn % tiles_y) : 0, tw);
    if (more) m = max_nan(m, x_velocity_chain<T, N, NT, I + 1>(c, sm, stage, src, u_phys, grid, ntiles, tw));
    return m;
  } else {
    return 0.0;
  }
}

// The deposit's x pass over the tiles bx, bx + grid, …: physical velocity of PV points per tile
// written out, max |u|² returned to thread 0. One warp per line (ACT_V lines at sm + l·N); the next
// tile's spectra are prefetched into the staging rows (3·PV rows of KXS) while the current tile is
// transformed. `red` holds NT doubles.
template <class T, int N, int NT, class TW>
GBGHT_HD double body_x_velocity(const Cta& c, Cplx<T>* sm, double* red, Cplx<T>* stg, int KXS, uint64_t* bar,
                                int grid, const Geometry& g, const Cplx<T>* GBGHT_RESTRICT B,
                                T* GBGHT_RESTRICT u_phys, const TW& tw, unsigned int* status) {
  using X = XShape<T>;
  constexpr int PV = X::PV;
  const int tiles_y = N / PV, ntiles = tiles_y * N;
  double m = 0.0;
  if (c.bx < ntiles) {
    const XStaging<T, PV> stage{g, B, stg, KXS, 3, bar, status};
    const XVelocityStagedSource<T, N, PV> src{g, stg, KXS, T(g.inv_norm)};
    stage.issue(c, c.bx / tiles_y, PV * (c.bx % tiles_y));
    m = x_velocity_chain<T, N, NT, 0>(c, sm, stage, src, u_phys, grid, ntiles, tw);
  }
  red[c.tid] = m;
  GBGHT_SYNC();
  if (c.tid == 0) {
    double r = 0.0;
    for (int i = 0; i < NT; ++i) r = max_nan(r, red[i]);
    return r;
  }
  return 0.0;
}

// ================================================================================================
// z-forward + epilogue + z-inverse helpers
// ================================================================================================

// I/O of one z tile (the TL kx columns kx0.. of row ky' = qy, all z). The forward transforms'
// first stage reads a staged copy (below), and their last stage keeps only the retained rows, in
// the thread that computes them (ZOwn below).
//
// Staged z tiles: A slot `slot` of the tile (N rows of TL elements, the layout of the tile FFT's
// buffer) copied by the TMA engine (map az) into buffer `bf` (0 or 1) of the staging region, so
// the copy of the next transform's input runs while the current one computes. The copy completes
// a phase of barrier bf; the caller tracks the parities. The host-check build copies at issue.
template <class T, int N, int TL>
struct ZStagedSource {
  static constexpr bool kExternal = true;
  const Cplx<T>* P;
  GBGHT_HD Cplx<T> load(int e, int l) const { return P[e * TL + l]; }
};

template <class T, int N, int TL>
struct ZStaging {
  const Geometry& g;
  const Cplx<T>* A;
  const TmaMaps& maps;
  Cplx<T>* R;           // the staging region: two buffers of N·TL elements
  uint64_t* bar;        // barriers 0 and 1
  unsigned int* status;
  int qy, kx0;
  GBGHT_HD Cplx<T>* buf(int bf) const { return R + bf * (N * TL); }
  GBGHT_HD void issue(const Cta& c, int bf, int slot) const {
#if defined(__CUDA_ARCH__)
    if (c.tid == 0) {
      constexpr int BZ = box_rows<N>();
      mbar_expect_tx(bar + bf, uint32_t(N * TL * sizeof(Cplx<T>)));
      for (int z0 = 0; z0 < N; z0 += BZ) tma_load_3d(buf(bf) + z0 * TL, &maps.az, 2 * kx0, qy, slot * N + z0, bar + bf);
    }
#else
    (void)c;
    Cplx<T>* P = buf(bf);
    for (int e = 0; e < N; ++e)
      for (int l = 0; l < TL; ++l) P[e * TL + l] = A[idxA(g, slot, e, qy, kx0 + l)];
#endif
  }
  GBGHT_HD void wait(int bf, int parity) const {
#if defined(__CUDA_ARCH__)
    mbar_wait(bar + bf, uint32_t(parity), status);
#else
    (void)bf;
    (void)parity;
#endif
  }
};

// Staged state for one half of the epilogue: half h holds the compact rows q in [h·(K+1),
// (h+1)·(K+1)) of up to six components of S and H (the tile's TL columns), copied by the TMA engine
// (maps s3 and h3) into the staging region as component i at rows i·rows(K) (K + 1 rounded up so
// that every copy starts on a 128-byte boundary). Component codes: c for S slot c, 4 + c for H
// slot c. Rows past 2K read as zero.
template <class T, int N, int TL>
struct ZStateStaging {
  static constexpr int kRowBytes = TL * int(sizeof(Cplx<T>));
  GBGHT_HD static int rows(int K) { return ((K + 1) * kRowBytes + 127) / 128 * 128 / kRowBytes; }
  const Geometry& g;
  const Cplx<T>* S;
  const Cplx<T>* H;
  const TmaMaps& maps;
  Cplx<T>* R;
  uint64_t* bar;        // barrier 2
  unsigned int* status;
  int qy, kx0;
  GBGHT_HD void issue(const Cta& c, int h, const int* codes, int n) const {
    const int KR = g.K + 1, KS = rows(g.K);
#if defined(__CUDA_ARCH__)
    if (c.tid == 0) {
      mbar_expect_tx(bar, uint32_t(n * KR * TL * sizeof(Cplx<T>)));
      for (int i = 0; i < n; ++i)
        tma_load_3d(R + i * KS * TL, codes[i] < 4 ? &maps.s3 : &maps.h3, 2 * kx0, h * KR, (codes[i] & 3) * g.NY2 + qy,
                    bar);
    }
#else
    (void)c;
    for (int i = 0; i < n; ++i) {
      const Cplx<T>* src = codes[i] < 4 ? S : H;
      for (int t = 0; t < KR; ++t)
        for (int l = 0; l < TL; ++l) {
          const int q = h * KR + t;
          R[(i * KS + t) * TL + l] = q < g.NY2 ? src[idxS(g, codes[i] & 3, qy, q, kx0 + l)] : czero<T>();
        }
    }
#endif
  }
  GBGHT_HD void wait(int parity) const {
#if defined(__CUDA_ARCH__)
    mbar_wait(bar, uint32_t(parity), status);
#else
    (void)parity;
#endif
  }
  // component i of the staged list at compact row q of half h, column l
  GBGHT_HD Cplx<T> at(int i, int q, int h, int l) const { return R[(i * rows(g.K) + (q - h * (g.K + 1))) * TL + l]; }
};

// Shared memory of the z epilogue: the FFT tile W, NT doubles, four barriers, the TMEM address,
// the twiddle table, then the staging region (two A tiles, or six state components of K + 1 rows).
template <class T, int N, int TL, int NT>
struct ZLayout {
  static constexpr size_t kRed = size_t(N) * TL * sizeof(Cplx<T>);
  static constexpr size_t kBar = kRed + size_t(NT) * sizeof(double);
  static constexpr size_t kSlot = kBar + 4 * sizeof(uint64_t);
  static constexpr size_t kTw = kSlot + 16;
  static constexpr size_t kStage = (kTw + size_t(N) * sizeof(Cplx<T>) + 127) / 128 * 128;
  // ncomp: the most state components staged at once (6 with H staged, 4 without)
  GBGHT_HD static size_t stage_elems(int K, int ncomp = 6) {
    const size_t a = 2 * size_t(N) * TL, b = size_t(ncomp) * ZStateStaging<T, N, TL>::rows(K) * TL;
    return a > b ? a : b;
  }
  GBGHT_HD static size_t bytes(int K, int ncomp = 6) { return kStage + stage_elems(K, ncomp) * sizeof(Cplx<T>); }
};

// Per-thread ownership of a z tile's retained rows. In tile_fft_io, slot b of thread t takes
// butterfly j = (t + b·NT) / TL of line l = (t + b·NT) mod TL in every stage. The plans start and
// end with the same radix R, so the last stage of a forward transform writes rows j + r·N/R, which
// are the rows the first stage of an inverse transform reads: the thread that produces a retained
// value is the thread that consumes it, and the retained rows stay in its registers between the
// transforms (no shared-memory copy, no barrier). Row bands r whose rows j + r·N/R have |m| > K for
// every j get no register.
template <class T, int N, int TL, int NT, int KM = N / 3 + 1>
struct ZOwn {
  static constexpr int R = Radices<N>::r[0];
  static_assert(R == Radices<N>::r[Radices<N>::n - 1], "the z epilogue needs equal first and last radix");
  static constexpr int NB = N / R;
  static constexpr int TOT = NB * TL;
  static constexpr int BPT = (TOT + NT - 1) / NT;
  // bounds K = max |m| of the retained box: N/3 + 1 for the 2/3 ball at every side length, N/2 − 1
  // under HouLi (everything but the Nyquist planes)
  static constexpr int KMAX = KM;
  static constexpr int lead() { int a = 0; while (a < R && a * NB <= KMAX) ++a; return a; }
  static constexpr int tail() { int b = R; while (b > 0 && b * NB - 1 >= N - KMAX) --b; return b; }
  static constexpr int A0 = lead(), B0 = tail() > lead() ? tail() : lead();
  static constexpr int NSLOT = A0 + (R - B0);
  GBGHT_HD static constexpr bool may(int r) { return r < A0 || r >= B0; }
  GBGHT_HD static constexpr int slot(int r) { return r < A0 ? r : r - B0 + A0; }
  // Retained rows of the leading bands have q = m ≤ K (half 0), those of the trailing bands
  // q = m + NY2 > K (half 1).
  GBGHT_HD static constexpr int half(int r) { return r < A0 ? 0 : 1; }
  static_assert(A0 * NB - 1 < N - KMAX && B0 * NB > KMAX, "a row band mixes both halves of the retained rows");
};

// Storage of the owned rows: three components × BPT × NSLOT complex values per thread.
// ZRowsReg keeps them in registers (the host-check build, and small N); ZRowsTmem keeps them in the
// thread's private TMEM lane. Both expose put / put_done / get / get3; put_done makes the puts
// visible to later gets.
template <class T, class O>
struct ZRowsReg {
  using Own = O;
  Cplx<T> v[3][O::BPT][O::NSLOT];
  GBGHT_HD void put(int c, int b, int sl, Cplx<T> x) { v[c][b][sl] = x; }
  GBGHT_HD void put_done() const {}
  GBGHT_HD Cplx<T> get(int c, int b, int sl) const { return v[c][b][sl]; }
  GBGHT_HD void get3(int b, int sl, Cplx<T>& a0, Cplx<T>& a1, Cplx<T>& a2) const {
    a0 = v[0][b][sl];
    a1 = v[1][b][sl];
    a2 = v[2][b][sl];
  }
};

// TMEM columns per thread and per CTA for the owned rows of a z tile.
template <class T, int N, class O, int NT>
struct ZTmemShape {
  static constexpr int WPC = int(sizeof(Cplx<T>)) / 4;            // 32-bit words per value
  static constexpr int COLS = 3 * O::BPT * O::NSLOT * WPC;         // per thread
  static constexpr int WPQ = (NT / 32 + 3) / 4;                    // warps per lane quarter
  static constexpr int NEED = COLS * WPQ;
  static constexpr int NCOLS = NEED <= 32 ? 32 : NEED <= 64 ? 64 : NEED <= 128 ? 128 : NEED <= 256 ? 256 : 512;
  // Warp-collective access needs every thread of every warp active in every stage.
  static constexpr bool kUse = N >= 64 && NT % 32 == 0 && O::BPT * NT == O::TOT && NEED <= 256;
};

#if defined(__CUDACC__) && !defined(GBGHT_EMU)
template <class T, class O>
struct ZRowsTmem {
  using Own = O;
  static constexpr int WPC = int(sizeof(Cplx<T>)) / 4;
  uint32_t base;   // this thread's warp: lane quarter and column block
  __device__ static uint32_t col(int c, int b, int sl) { return uint32_t(((c * O::BPT + b) * O::NSLOT + sl) * WPC); }
  __device__ static Cplx<T> unpack(const uint32_t* w) {
    if constexpr (WPC == 4)
      return cmk<T>(__hiloint2double(int(w[1]), int(w[0])), __hiloint2double(int(w[3]), int(w[2])));
    else
      return cmk<T>(__uint_as_float(w[0]), __uint_as_float(w[1]));
  }
  // put and get3 follow per-row branches: reconverge the warp before the collective access.
  __device__ void put(int c, int b, int sl, Cplx<T> x) const {
    __syncwarp();
    if constexpr (WPC == 4)
      tmem_st4(base + col(c, b, sl), uint32_t(__double2loint(x.x)), uint32_t(__double2hiint(x.x)),
               uint32_t(__double2loint(x.y)), uint32_t(__double2hiint(x.y)));
    else
      tmem_st2(base + col(c, b, sl), __float_as_uint(x.x), __float_as_uint(x.y));
  }
  __device__ void put_done() const { tmem_wait_st(); }
  __device__ Cplx<T> get(int c, int b, int sl) const {
    uint32_t w[WPC];
    if constexpr (WPC == 4) tmem_ld4(base + col(c, b, sl), w);
    else tmem_ld2(base + col(c, b, sl), w);
    return unpack(w);
  }
  __device__ void get3(int b, int sl, Cplx<T>& a0, Cplx<T>& a1, Cplx<T>& a2) const {
    __syncwarp();
    uint32_t w[3 * WPC];
    if constexpr (WPC == 4) tmem_ld4x3(base + col(0, b, sl), base + col(1, b, sl), base + col(2, b, sl), w);
    else tmem_ld2x3(base + col(0, b, sl), base + col(1, b, sl), base + col(2, b, sl), w);
    a0 = unpack(w);
    a1 = unpack(w + WPC);
    a2 = unpack(w + 2 * WPC);
  }
};
#endif

// The last stage of a forward transform into component `comp` of the owned rows.
template <class T, class O, class Rows>
struct ZOwnSink {
  static constexpr bool kIndexed = true;
  Rows& rows;
  int comp;
  GBGHT_HD void store_rb(int, int, Cplx<T> v, int r, int b) const {
    if (O::may(r)) rows.put(comp, b, O::slot(r), v);
  }
};

// The first stage of an inverse transform from x[b][slot] on retained rows, zero elsewhere.
template <class T, int N, class O>
struct ZOwnSource {
  static constexpr bool kExternal = true;
  static constexpr bool kIndexed = true;
  const Geometry& g;
  const Cplx<T> (&x)[O::BPT][O::NSLOT];
  GBGHT_HD Cplx<T> load_rb(int e, int, int r, int b) const {
    if (!O::may(r)) return czero<T>();
    const Cplx<T> v = x[b][O::slot(r)];
    return (e <= g.K || e >= N - g.K) ? v : czero<T>();
  }
};

// Every slot of the thread with a register: slot b, band r (slot index sl), whether the row
// e = j + r·N/R is retained, its compact index q and m_z, and the column l. The loops unroll, so
// (b, sl) are compile-time indices.
template <class T, int N, int TL, int NT, int HALF = -1, class O = ZOwn<T, N, TL, NT>, class F>
GBGHT_HD void for_own_slots(const Cta& c, const Geometry& g, const F& f) {
#pragma unroll
  for (int b = 0; b < O::BPT; ++b) {
    const int idx = c.tid + b * NT;
    const bool active = O::BPT * NT == O::TOT || idx < O::TOT;
    const int l = idx % TL, j = idx / TL;
#pragma unroll
    for (int r = 0; r < O::R; ++r) {
      if (!O::may(r) || (HALF >= 0 && O::half(r) != HALF)) continue;
      const int e = j + r * O::NB;
      const bool ret = active && (e <= g.K || e >= N - g.K);
      const int q = e <= g.K ? e : e - N + g.NY2;
      const int mz = e <= g.K ? e : e - N;
      f(b, O::slot(r), ret, q, mz, l);
    }
  }
}

// Inverse: the first stage reads value(q, l) for retained rows and zero elsewhere; the last stage
// writes A slot `slot` rows z straight to global memory.
template <class T, int N, int TL, class F>
struct ZValueSource {
  static constexpr bool kExternal = true;
  const Geometry& g;
  const F& value;
  GBGHT_HD Cplx<T> load(int e, int l) const {
    if (e <= g.K) return value(e, l);
    if (e >= N - g.K) return value(e - N + g.NY2, l);
    return czero<T>();
  }
};
template <class T, int N, int TL>
struct ZGlobalSink {
  const Geometry& g;
  Cplx<T>* A;
  int slot, qy, kx0;
  GBGHT_HD void store(int e, int l, Cplx<T> v) const { A[idxA(g, slot, e, qy, kx0 + l)] = v; }
};

// Forward z-transform of the tile staged in buffer bf (barrier parity `parity`) into component
// `comp` of the owned rows. `after()` runs once the first stage has read the buffer (after the
// barrier that ends the stage), for the caller to start the next copy into it. Kept inline: out
// of line, the staging objects and the row store go through local memory and the kernel slows.
template <class T, int N, int TL, int NT, class O, class Rows, class After, class TW>
GBGHT_HD void z_forward_staged(const Cta& c, Cplx<T>* W, const ZStaging<T, N, TL>& stg, int bf, int parity, Rows& rows,
                               int comp, const After& after, const TW& tw) {
  stg.wait(bf, parity);
  const ZStagedSource<T, N, TL> src{stg.buf(bf)};
  const ZOwnSink<T, O, Rows> dst{rows, comp};
  if constexpr (Radices<N>::n == 1) {
    tile_fft_io<T, N, TL, NT, -1>(c, W, tw, src, dst);
    after();
  } else {
    const TileBuf<T, TL> tb{W};
    tile_fft_io<T, N, TL, NT, -1, TL, 0, 1>(c, W, tw, src, tb);
    after();
    tile_fft_io<T, N, TL, NT, -1, TL, 1>(c, W, tw, tb, dst);
  }
  rows.put_done();
}

// The owned values of one component, passed by value (in registers) to the out-of-line inverse.
template <class T, class O>
struct OwnVals {
  Cplx<T> v[O::BPT][O::NSLOT];
};

// Inverse z-transform of the owned values x (retained rows) into A slot `slot` of the tile. One
// out-of-line copy serves the epilogue's seven inverse transforms.
template <class T, int N, int TL, int NT, class O, class TW>
GBGHT_HD_OUTLINE void z_inverse_own(const Cta c, Cplx<T>* W, const Geometry g, Cplx<T>* A, int slot, int qy, int kx0,
                                    const OwnVals<T, O> x, const TW tw) {
  const ZOwnSource<T, N, O> src{g, x.v};
  const ZGlobalSink<T, N, TL> dst{g, A, slot, qy, kx0};
  tile_fft_io<T, N, TL, NT, +1>(c, W, tw, src, dst);
}

// z-forward source: A slot `slot` of the tile, straight from global memory (the adjoint's z pass,
// PhaseShift's shift back). For the shift back, the forward's last stage keeps the owned retained
// rows in x, and the inverse's last stage averages into the A slot (a ← ½·a + v).
template <class T, int N, int TL>
struct ZGlobalSource {
  static constexpr bool kExternal = true;
  const Geometry& g;
  const Cplx<T>* A;
  int slot, qy, kx0;
  GBGHT_HD Cplx<T> load(int e, int l) const { return A[idxA(g, slot, e, qy, kx0 + l)]; }
};
template <class T, class O>
struct OwnValsSink {
  static constexpr bool kIndexed = true;
  Cplx<T> (&x)[O::BPT][O::NSLOT];
  GBGHT_HD void store_rb(int, int, Cplx<T> v, int r, int b) const {
    if (O::may(r)) x[b][O::slot(r)] = v;
  }
};
template <class T, int N, int TL>
struct ZAverageSink {
  const Geometry& g;
  Cplx<T>* A;
  int slot, qy, kx0;
  GBGHT_HD void store(int e, int l, Cplx<T> v) const {
    Cplx<T>& a = A[idxA(g, slot, e, qy, kx0 + l)];
    a = scale(a, T(0.5)) + v;
  }
};
template <class T, int N, int TL, int NT, class O, class TW>
GBGHT_HD_OUTLINE void z_average_own(const Cta c, Cplx<T>* W, const Geometry g, Cplx<T>* A, int slot, int qy, int kx0,
                                    const OwnVals<T, O> x, const TW tw) {
  const ZOwnSource<T, N, O> src{g, x.v};
  const ZAverageSink<T, N, TL> dst{g, A, slot, qy, kx0};
  tile_fft_io<T, N, TL, NT, +1>(c, W, tw, src, dst);
}

// The displaced products shifted back and averaged with the primary ones, one tile per CTA (grid
// (KXP/TL, NY2)). For each of the nc product components: the z-forward of the displaced grid's
// y-forward output D (slot c of A2), the retained rows multiplied by e^{−iπ(mx+my+mz)/N}/(2N) (the
// back translation, the 1/N of the round trip, the average's ½), the z-inverse, and A ← ½·A + that.
// The rows outside the retained box are dropped: the z epilogue keeps only retained rows of A's
// z-forward, so what it reads is ½(P + e^{−iκ·δ}·P_δ), P and P_δ the two grids' transformed products
// (`_velocity_nonlinear!(::PhaseShift)` and `_scalar_nonlinear!(::PhaseShift)`,
// src/Generator.jl:502-519,668-704, average before the truncation).
template <class T, int N, int TL, int NT, class O>
GBGHT_HD void body_z_shift_back(const Cta& c, Cplx<T>* W, const Geometry& g, Cplx<T>* GBGHT_RESTRICT A,
                                const Cplx<T>* GBGHT_RESTRICT A2, int nc, const Cplx<T>* GBGHT_RESTRICT tw) {
  const int kx0 = c.bx * TL, qy = c.by;
  const int my = q_to_m(qy, g.K, g.NY2);
  const T inv2n = T(0.5 / double(N));
  for (int cc = 0; cc < nc; ++cc) {
    OwnVals<T, O> x;
    const ZGlobalSource<T, N, TL> src{g, A2, cc, qy, kx0};
    const OwnValsSink<T, O> dst{x.v};
    tile_fft_io<T, N, TL, NT, -1>(c, W, tw, src, dst);
    for_own_slots<T, N, TL, NT, -1, O>(c, g, [&](int b, int sl, bool ret, int, int mz, int l) {
      x.v[b][sl] = ret ? scale(x.v[b][sl] * conj(half_cell_phase<T>(kx0 + l + my + mz, N)), inv2n) : czero<T>();
    });
    z_average_own<T, N, TL, NT, O>(c, W, g, A, cc, qy, kx0, x, tw);
  }
}

// Inverse z-transform of value(q, l) (retained rows q) into A slot `slot` of the tile.
template <class T, int N, int TL, int NT, class F, class TW>
GBGHT_HD void z_inverse1(const Cta& c, Cplx<T>* W, const Geometry& g, Cplx<T>* A, int slot, int qy, int kx0,
                         const F& value, const TW& tw) {
  const ZValueSource<T, N, TL, F> src{g, value};
  const ZGlobalSink<T, N, TL> dst{g, A, slot, qy, kx0};
  tile_fft_io<T, N, TL, NT, +1>(c, W, tw, src, dst);
}

// Component o of iκ × û at wavenumber (kX, kY, kZ).
template <class T>
GBGHT_HD Cplx<T> curl_of(int o, Cplx<T> u0, Cplx<T> u1, Cplx<T> u2, T kX, T kY, T kZ) {
  Cplx<T> cr;
  if (o == 0) cr = scale(u2, kY) - scale(u1, kZ);
  else if (o == 1) cr = scale(u0, kZ) - scale(u2, kX);
  else cr = scale(u1, kX) - scale(u0, kY);
  return mul_i(cr);
}

// Component o of the strain rate Ŝ_ij = ½ i(κ_j û_i + κ_i û_j), in the order S11, S22, S33, S12,
// S13, S23 (src/Observables.jl:470, `symmetric_gradient`).
template <class T>
GBGHT_HD Cplx<T> strain_of(int o, Cplx<T> u0, Cplx<T> u1, Cplx<T> u2, T kX, T kY, T kZ) {
  const T h = T(0.5);
  switch (o) {
    case 0: return mul_i(scale(u0, kX));
    case 1: return mul_i(scale(u1, kY));
    case 2: return mul_i(scale(u2, kZ));
    case 3: return mul_i(scale(scale(u0, kY) + scale(u1, kX), h));
    case 4: return mul_i(scale(scale(u0, kZ) + scale(u2, kX), h));
    default: return mul_i(scale(scale(u1, kZ) + scale(u2, kY), h));
  }
}

// ⟨det S⟩'s partial sums: block b adds the determinants of the points [b·chunk, (b+1)·chunk) of
// the six physical components (S11, S22, S33, S12, S13, S23, n points apart), per thread and then
// in thread order through `red` (NT doubles), into out[b].
template <class T, int NT>
GBGHT_HD void body_det_sum(const Cta& c, double* red, const T* GBGHT_RESTRICT s6, size_t n, size_t chunk,
                           double* GBGHT_RESTRICT out) {
  const size_t p0 = size_t(c.bx) * chunk;
  const size_t p1 = p0 + chunk < n ? p0 + chunk : n;
  double acc = 0.0;
  for (size_t p = p0 + c.tid; p < p1; p += NT) {
    const double a = s6[p], d = s6[n + p], f = s6[2 * n + p];
    const double b = s6[3 * n + p], cc = s6[4 * n + p], e = s6[5 * n + p];
    acc += a * (d * f - e * e) - b * (b * f - e * cc) + cc * (b * e - d * cc);
  }
  red[c.tid] = acc;
  GBGHT_SYNC();
  if (c.tid == 0) {
    double s = 0.0;
    for (int i = 0; i < NT; ++i) s += red[i];
    out[c.bx] = s;
  }
}

// The z-inverse of the owned velocity rows into A slots 0..2, and of iκ × û into slots 3..5
// (3..5 only when `vorticity`); with `vorticity` = 2 the six strain components into slots 0..5.
template <class T, int N, int TL, int NT, class O, class Rows, class TW>
GBGHT_HD void z_inverse_velocity(const Cta& c, Cplx<T>* W, const Geometry& g, Cplx<T>* A, int qy, int kx0, double ky,
                                 const Rows& rows, int vorticity, const TW& tw) {
  for (int o = 0; o < 3 && vorticity != 2; ++o) {
    OwnVals<T, O> x;
#pragma unroll
    for (int b = 0; b < O::BPT; ++b)
#pragma unroll
      for (int sl = 0; sl < O::NSLOT; ++sl) x.v[b][sl] = rows.get(o, b, sl);
    z_inverse_own<T, N, TL, NT, O>(c, W, g, A, o, qy, kx0, x, tw);
  }
  if (!vorticity) return;
  const T kY = T(ky);
  if (vorticity == 2) {   // the strain rate instead: S11, S22, S33 into slots 0..2, S12, S13, S23 into 3..5
    for (int o = 0; o < 6; ++o) {
      OwnVals<T, O> x;
      for_own_slots<T, N, TL, NT, -1, O>(c, g, [&](int b, int sl, bool, int, int mz, int l) {
        Cplx<T> u0, u1, u2;
        rows.get3(b, sl, u0, u1, u2);
        x.v[b][sl] = strain_of<T>(o, u0, u1, u2, T(g.s * double(kx0 + l)), kY, T(g.s * double(mz)));
      });
      z_inverse_own<T, N, TL, NT, O>(c, W, g, A, o, qy, kx0, x, tw);
    }
    return;
  }
  for (int o = 0; o < 3; ++o) {
    OwnVals<T, O> x;
    for_own_slots<T, N, TL, NT, -1, O>(c, g, [&](int b, int sl, bool, int, int mz, int l) {
      Cplx<T> u0, u1, u2;
      rows.get3(b, sl, u0, u1, u2);
      x.v[b][sl] = curl_of<T>(o, u0, u1, u2, T(g.s * double(kx0 + l)), kY, T(g.s * double(mz)));
    });
    z_inverse_own<T, N, TL, NT, O>(c, W, g, A, 3 + o, qy, kx0, x, tw);
  }
}

// ================================================================================================
// z-forward + epilogue + z-inverse, one tile (ky', kx0..kx0+TL) per CTA. Grid: (KXP/TL, NY2).
//
// Epilogue per retained mode, stage i of the 2N loop (src/Propagator.jl:326-419):
//   N̂_φ = −𝔻 iκ·FFT(uφ) − G·û_i                          (src/Generator.jl:708-720; G is an extension)
//   N̂_u = 𝔻 ℙ FFT(u×ω), κ = 0 zeroed, + A 𝟙_band û_i     (src/Generator.jl:484-534, Forcing.jl:1104-1117)
//   h ← dt·N̂ (i = 0) or a_i h + dt·N̂
//   q ← E(q + b_i h), h ← E h (i < S−1), E = exp(c_i |κ|² + r_i), c_i = −D·(d_i·dt),
//   r_i = (d_i·dt)·A on a Linear forcing's band and 0 elsewhere (src/Generator.jl:565-581)
//   last stage: û ← ℙ û                                  (src/Propagator.jl:401)
// and the z-inverse of the new û, iκ×û and φ̂ into A slots 0..6 for the next stage's y-inverse.
// `red` holds NT doubles; the CTA's sum of the Hermitian-weighted |û_new|² is returned to thread 0.
// ================================================================================================
struct StageArgs {
  int kind;             // StageKind: the scheme's update at this stage
  double a, b, dt;      // tableau a_i, b_i (low storage) and the step
  double cu, cphi;      // exponents c = −D·δ of the stage's first factor E₁, velocity and scalar
  double cu2, cphi2;    // the second factor E₂ of a two-factor SSPRK3 stage
  int first, last;      // the step's first stage (state = the step's start), its last
  int read_h, write_h;  // the stage reads / writes the second register H
  int has_scalar;
  int forced, sforced;  // a per-stage source A·𝟙_band·f on the velocity, on the scalar
                        // (ConstantPower, VarianceController); A in force_amp[0], force_amp[4]
  double band_lo2, band_hi2;   // squared edges of the velocity forcing's band
  double lin_u, lin_phi;       // δ·A of a Linear forcing in E₁, velocity and scalar (0: none)
  double lin_u2, lin_phi2;     // the same in E₂
  double sband_lo2, sband_hi2; // squared edges of the scalar forcing's band
  double G[3];          // mean scalar gradient (extension)
};

// The stage kinds. Low storage (src/Propagator.jl:326-419): h ← Δt·N (first) or a h + Δt·N,
// q ← E₁(q + b h), h ← E₁ h. IFHeun (:456-544), predictor: q ← E₁(q + Δt N₁), h ← E₁q + (Δt/2)(E₁N₁);
// corrector: q ← h + (Δt/2) N₂. IFSSPRK3 (:599-691), with q⁽⁰⁾ kept in h: stage 1 h ← q,
// q ← E₁(q + Δt N) (E₁ = E(Δt)); stage 2 q ← ¼·E₁(q + Δt N) + E₂(¾ h) (E₁ = E(−Δt/2), E₂ = E(Δt/2));
// stage 3 q ← E₂(⅓ h) + ⅔·E₁(q + Δt N) (E₁ = E(Δt/2), E₂ = E(Δt)). Each grouping is the reference's.
enum StageKind { kLowStorage = 0, kHeunPredictor = 1, kHeunCorrector = 2, kSsp1 = 3, kSsp2 = 4, kSsp3 = 5 };

// KIND is the stage kind, fixed at compile time: each kind has its own epilogue instantiation, so
// no stage carries another kind's arithmetic (a runtime switch here made the kernel 1.76× slower).
template <class T, int KIND>
GBGHT_HD Cplx<T> scheme_update(const StageArgs& st, Cplx<T> q, Cplx<T> h, Cplx<T> n, T E1, T E2, Cplx<T>* hw) {
  const T dt = T(st.dt);
  if (KIND == kHeunPredictor) {
    *hw = scale(q, E1) + scale(scale(n, E1), dt / T(2));
    return scale(q + scale(n, dt), E1);
  }
  if (KIND == kHeunCorrector) return h + scale(n, dt / T(2));
  if (KIND == kSsp1) {
    *hw = q;
    return scale(q + scale(n, dt), E1);
  }
  if (KIND == kSsp2) return scale(scale(q + scale(n, dt), E1), T(0.25)) + scale(scale(h, T(0.75)), E2);
  if (KIND == kSsp3) return scale(scale(h, T(1.0 / 3.0)), E2) + scale(scale(q + scale(n, dt), E1), T(2.0 / 3.0));
  const Cplx<T> hh = st.first ? scale(n, dt) : scale(h, T(st.a)) + scale(n, dt);   // low storage
  *hw = scale(hh, E1);
  return scale(q + scale(hh, T(st.b)), E1);
}

template <class T, int N, int TL, int NT, int KIND, bool WIDE, class Rows>
GBGHT_HD double body_z_epilogue(const Cta& c, Cplx<T>* W, Cplx<T>* R, uint64_t* bar, double* red, const Geometry& g,
                                const TmaMaps& maps, Rows& rows, Cplx<T>* GBGHT_RESTRICT A, Cplx<T>* GBGHT_RESTRICT S,
                                Cplx<T>* GBGHT_RESTRICT H, const StageArgs& st, const double* GBGHT_RESTRICT force_amp,
                                const Cplx<T>* twS, unsigned int* status) {
  using O = typename Rows::Own;
  // WIDE: the instantiation of the wide box (HouLi, PhaseShift). The filter's branches exist only
  // there: in the TwoThirds one even a branch never taken slowed the FP64 epilogue by a third
  // (2.68 → 3.65 ms at 512³). The wide box's rows (K up to N/2 − 1) would make six staged state
  // components outgrow two CTAs' shared memory per SM, so there the registers H are read from
  // global memory in the update instead of staged (at most four staged components).
  constexpr bool kWide = WIDE;
  constexpr bool kStageH = !WIDE;
  using H0 = std::integral_constant<int, 0>;
  const SharedTwiddles<T> tw{twS};
  using H1 = std::integral_constant<int, 1>;
  const int kx0 = c.bx * TL, qy = c.by;
  const double s = g.s;
  const double ky = s * double(q_to_m(qy, g.K, g.NY2));
  const bool withG = st.G[0] != 0.0 || st.G[1] != 0.0 || st.G[2] != 0.0;

  // Staging: the three forward transforms of a part read A tiles copied into buffers 0, 1, 0 of
  // the staging region; once the last has read its tile, the region takes the state of half 0,
  // then (after a barrier) that of half 1. Buffer 0 and the state barrier complete two phases per
  // part, buffer 1 one.
  const ZStaging<T, N, TL> stg{g, A, maps, R, bar, status, qy, kx0};
  const ZStateStaging<T, N, TL> sst{g, S, H, maps, R, bar + 2, status, qy, kx0};
  int par1 = 0;
  const auto forward3 = [&](int c0, const int* codes, int n) {
    z_forward_staged<T, N, TL, NT, O>(c, W, stg, 0, 0, rows, 0, [&] { stg.issue(c, 0, c0 + 2); }, tw);
    z_forward_staged<T, N, TL, NT, O>(c, W, stg, 1, par1, rows, 1, [] {}, tw);
    par1 ^= 1;
    z_forward_staged<T, N, TL, NT, O>(c, W, stg, 0, 1, rows, 2, [&] { sst.issue(c, 0, codes, n); }, tw);
  };

  // ---------------- scalar -------------------------------------------------------------------------
  if (st.has_scalar) {
    stg.issue(c, 0, 3);
    stg.issue(c, 1, 4);
    int codes[6], n = 0;
    codes[n++] = 3;                      // φ̂
    if (st.read_h && kStageH) codes[n++] = 4 + 3;   // h_φ
    const int iG = n;
    if (withG) {                         // û for −G·û
      codes[n++] = 0;
      codes[n++] = 1;
      codes[n++] = 2;
    }
    forward3(3, codes, n);
    const double A_s = st.sforced ? force_amp[4] : 0.0;
    OwnVals<T, O> x;
    const auto half = [&](auto hc) {
      constexpr int h = decltype(hc)::value;
      sst.wait(h);
      for_own_slots<T, N, TL, NT, h, O>(c, g, [&](int b, int sl, bool ret, int q, int mz, int l) {
        Cplx<T> fx, fy, fz;
        rows.get3(b, sl, fx, fy, fz);
        Cplx<T> phi = czero<T>();
        if (ret) {
          const int kx = kx0 + l;
          const double kxd = s * double(kx), kzd = s * double(mz);
          const double k2 = (kxd * kxd + ky * ky) + kzd * kzd;
          const bool keep = kx <= g.K && k2 <= g.cut2;
          const size_t si = idxS(g, 3, qy, q, kx);
          phi = sst.at(0, q, h, l);
          Cplx<T> nphi = czero<T>();
          if (keep) {
            // −i(κx fx + κy fy + κz fz)
            const Cplx<T> dsum = cmk<T>(T(kxd) * fx.x + T(ky) * fy.x + T(kzd) * fz.x,
                                        T(kxd) * fx.y + T(ky) * fy.y + T(kzd) * fz.y);
            nphi = mul_mi(dsum);
            if constexpr (kWide)
              if (g.houli) nphi = scale(nphi, T(dealias_filter(g, k2)));
          }
          if (withG) {
            const Cplx<T> ux = sst.at(iG, q, h, l), uy = sst.at(iG + 1, q, h, l), uz = sst.at(iG + 2, q, h, l);
            const T G0 = T(st.G[0]), G1 = T(st.G[1]), G2 = T(st.G[2]);
            nphi = nphi - cmk<T>(G0 * ux.x + G1 * uy.x + G2 * uz.x, G0 * ux.y + G1 * uy.y + G2 * uz.y);
          }
          if (A_s != 0.0 && k2 >= st.sband_lo2 && k2 <= st.sband_hi2) nphi = nphi + scale(phi, T(A_s));
          const bool sband = k2 >= st.sband_lo2 && k2 <= st.sband_hi2;
          const T E1 = KIND == kHeunCorrector ? T(1) : T(exp(st.cphi * k2 + (sband ? st.lin_phi : 0.0)));
          const T E2 = KIND >= kSsp2 ? T(exp(st.cphi2 * k2 + (sband ? st.lin_phi2 : 0.0))) : T(0);
          Cplx<T> hw = czero<T>();
          const Cplx<T> hphi = st.read_h ? (kStageH ? sst.at(1, q, h, l) : H[si]) : czero<T>();
          phi = scheme_update<T, KIND>(st, phi, hphi, nphi, E1, E2, &hw);
          S[si] = phi;
          if (st.write_h) H[si] = hw;
        }
        x.v[b][sl] = phi;
      });
    };
    half(H0{});
    GBGHT_SYNC();
    sst.issue(c, 1, codes, n);
    half(H1{});
    GBGHT_SYNC();
    // the velocity part's first two tiles load during the scalar's inverse transform
    stg.issue(c, 0, 0);
    stg.issue(c, 1, 1);
    z_inverse_own<T, N, TL, NT, O>(c, W, g, A, 6, qy, kx0, x, tw);
  } else {
    stg.issue(c, 0, 0);
    stg.issue(c, 1, 1);
  }

  // ---------------- velocity -----------------------------------------------------------------------
  int codes[6], n = 0;
  codes[n++] = 0;
  codes[n++] = 1;
  codes[n++] = 2;
  if (st.read_h && kStageH) {
    codes[n++] = 4;
    codes[n++] = 5;
    codes[n++] = 6;
  }
  forward3(0, codes, n);
  const double A_f = st.forced ? force_amp[0] : 0.0;
  double esum = 0.0;
  const auto half = [&](auto hc) {
    constexpr int h = decltype(hc)::value;
    sst.wait(h);
    for_own_slots<T, N, TL, NT, h, O>(c, g, [&](int b, int sl, bool ret, int q, int mz, int l) {
      Cplx<T> f0, f1, f2;
      rows.get3(b, sl, f0, f1, f2);
      Cplx<T> u0 = czero<T>(), u1 = czero<T>(), u2 = czero<T>();
      if (ret) {
        const int kx = kx0 + l;
        const double kxd = s * double(kx), kzd = s * double(mz);
        const double k2 = (kxd * kxd + ky * ky) + kzd * kzd;
        const bool keep = kx <= g.K && k2 <= g.cut2;
        const size_t s0 = idxS(g, 0, qy, q, kx), s1 = idxS(g, 1, qy, q, kx), s2 = idxS(g, 2, qy, q, kx);
        u0 = sst.at(0, q, h, l);
        u1 = sst.at(1, q, h, l);
        u2 = sst.at(2, q, h, l);
        Cplx<T> n0 = czero<T>(), n1 = czero<T>(), n2 = czero<T>();
        if (keep && k2 > 0.0) {
          const T kX = T(kxd), kY = T(ky), kZ = T(kzd);
          const T ik2 = T(1.0 / k2);
          const Cplx<T> kd = cmk<T>((kX * f0.x + kY * f1.x + kZ * f2.x) * ik2, (kX * f0.y + kY * f1.y + kZ * f2.y) * ik2);
          n0 = f0 - scale(kd, kX);
          n1 = f1 - scale(kd, kY);
          n2 = f2 - scale(kd, kZ);
          if (kWide && g.houli) {
            const T F = T(dealias_filter(g, k2));
            n0 = scale(n0, F);
            n1 = scale(n1, F);
            n2 = scale(n2, F);
          }
        }
        if (A_f != 0.0 && k2 >= st.band_lo2 && k2 <= st.band_hi2) {
          const T Af = T(A_f);
          n0 = n0 + scale(u0, Af);
          n1 = n1 + scale(u1, Af);
          n2 = n2 + scale(u2, Af);
        }
        const bool vband = k2 >= st.band_lo2 && k2 <= st.band_hi2;
        const T E1 = KIND == kHeunCorrector ? T(1) : T(exp(st.cu * k2 + (vband ? st.lin_u : 0.0)));
        const T E2 = KIND >= kSsp2 ? T(exp(st.cu2 * k2 + (vband ? st.lin_u2 : 0.0))) : T(0);
        const bool rh = st.read_h;
        Cplx<T> w0 = czero<T>(), w1 = czero<T>(), w2 = czero<T>();
        const Cplx<T> h0 = rh ? (kStageH ? sst.at(3, q, h, l) : H[s0]) : czero<T>();
        const Cplx<T> h1 = rh ? (kStageH ? sst.at(4, q, h, l) : H[s1]) : czero<T>();
        const Cplx<T> h2 = rh ? (kStageH ? sst.at(5, q, h, l) : H[s2]) : czero<T>();
        u0 = scheme_update<T, KIND>(st, u0, h0, n0, E1, E2, &w0);
        u1 = scheme_update<T, KIND>(st, u1, h1, n1, E1, E2, &w1);
        u2 = scheme_update<T, KIND>(st, u2, h2, n2, E1, E2, &w2);
        if (st.last) {
          if (k2 > 0.0) {
            const T kX = T(kxd), kY = T(ky), kZ = T(kzd);
            const T ik2 = T(1.0 / k2);
            const Cplx<T> kd = cmk<T>((kX * u0.x + kY * u1.x + kZ * u2.x) * ik2, (kX * u0.y + kY * u1.y + kZ * u2.y) * ik2);
            u0 = u0 - scale(kd, kX);
            u1 = u1 - scale(kd, kY);
            u2 = u2 - scale(kd, kZ);
          }
        }
        if (st.write_h) {
          H[s0] = w0;
          H[s1] = w1;
          H[s2] = w2;
        }
        S[s0] = u0;
        S[s1] = u1;
        S[s2] = u2;
        const double w = kx == 0 ? 1.0 : 2.0;
        esum += w * ((double(u0.x) * u0.x + double(u0.y) * u0.y) + (double(u1.x) * u1.x + double(u1.y) * u1.y) +
                     (double(u2.x) * u2.x + double(u2.y) * u2.y));
      }
      rows.put(0, b, sl, u0);
      rows.put(1, b, sl, u1);
      rows.put(2, b, sl, u2);
    });
  };
  half(H0{});
  GBGHT_SYNC();
  sst.issue(c, 1, codes, n);
  half(H1{});
  rows.put_done();
  red[c.tid] = esum;
  GBGHT_SYNC();
  double total = 0.0;
  if (c.tid == 0)
    for (int i = 0; i < NT; ++i) total += red[i];
  // z-inverse of û and of ω̂ = iκ × û
  z_inverse_velocity<T, N, TL, NT, O>(c, W, g, A, qy, kx0, ky, rows, 1, tw);
  return total;
}

// ================================================================================================
// StochasticOU's force (src/Forcing.jl:1362-1415), added to a stage's right-hand side through the
// products the z epilogue transforms last: after the y-forward pass, A holds the products
// transformed in x and y, still physical in z. Adding g(z) = Σ_mz N²·a(m)·e^{2πi m_z z/N} to a
// column (m_x, m_y) adds N³·a(m) to the z-transformed product at every m_z of the companion. The
// velocity's force a_u is transverse, so the epilogue's Leray projection keeps it; the scalar's
// force s enters the flux slots as f = iκ s/|κ|², whose −iκ·f the epilogue forms is s. Thread t
// takes one column of the companion's retained box (|m_y| < Nc/2, 0 ≤ m_x < Nc/2) at one z. The
// companion arrays are complex128 [comp][kz][ky][kx] (kx ≤ Nc/2); only band modes are added.
// ================================================================================================
struct SourceArgs {
  int nc;                        // companion points per axis
  int vel, sca;                  // which fields carry the force
  double lo2, hi2, slo2, shi2;   // the bands, squared edges
};
template <class T>
GBGHT_HD void inject_source(long t, const Geometry& g, Cplx<T>* A, const Cplx<double>* su, const Cplx<double>* sp,
                            const SourceArgs& a) {
  const int nc = a.nc, half = nc / 2, ncol = (nc - 1) * half;
  if (t >= long(ncol) * g.N) return;
  const int col = int(t % ncol), z = int(t / ncol);
  const int mx = col % half, my = col / half - (half - 1);
  const int qy = my >= 0 ? my : my + g.NY2;
  const double n2 = double(g.N) * double(g.N);
  const size_t comp = size_t(nc) * nc * (half + 1);
  double acc[6][2] = {};
  for (int mz = -(half - 1); mz <= half - 1; ++mz) {
    const double kxd = g.s * mx, kyd = g.s * my, kzd = g.s * mz;
    const double k2 = (kxd * kxd + kyd * kyd) + kzd * kzd;
    const double th = 2.0 * double(mz) * double(z) / double(g.N);
    double sn, cs;
#ifdef __CUDA_ARCH__
    sincospi(th, &sn, &cs);
#else
    sn = std::sin(M_PI * th);
    cs = std::cos(M_PI * th);
#endif
    const size_t at = (size_t((mz + nc) % nc) * nc + size_t((my + nc) % nc)) * (half + 1) + mx;
    if (a.vel && k2 >= a.lo2 && k2 <= a.hi2)
      for (int c = 0; c < 3; ++c) {
        const Cplx<double> v = su[c * comp + at];
        acc[c][0] += n2 * (v.x * cs - v.y * sn);
        acc[c][1] += n2 * (v.x * sn + v.y * cs);
      }
    if (a.sca && k2 >= a.slo2 && k2 <= a.shi2 && k2 > 0.0) {
      const Cplx<double> v = sp[at];
      const double kk[3] = {kxd, kyd, kzd};
      for (int c = 0; c < 3; ++c) {   // f_c = i κ_c s/|κ|²
        const double fr = -v.y * kk[c] / k2, fi = v.x * kk[c] / k2;
        acc[3 + c][0] += n2 * (fr * cs - fi * sn);
        acc[3 + c][1] += n2 * (fr * sn + fi * cs);
      }
    }
  }
  for (int c = 0; c < 6; ++c) {
    if ((c < 3 && !a.vel) || (c >= 3 && !a.sca)) continue;
    Cplx<T>& r = A[idxA(g, c, z, qy, mx)];
    r = r + cmk<T>(T(acc[c][0]), T(acc[c][1]));
  }
}

// ================================================================================================
// Reality projection of the kx = 0 plane of S slots [0, ncomp) (src/Propagator.jl:411-412): each
// pair (m_y, m_z) ↔ (−m_y, −m_z) is replaced by its Hermitian part. One thread per compact mode;
// the member with the smaller flat index writes both. Grid covers NY2·NY2 threads.
// ================================================================================================
template <class T>
GBGHT_HD void reality_mode(int idx, const Geometry& g, Cplx<T>* S, int ncomp) {
  const int NY2 = g.NY2;
  if (idx >= NY2 * NY2) return;
  const int qy = idx / NY2, qz = idx % NY2;
  const int py = qy == 0 ? 0 : NY2 - qy;   // compact index of −m
  const int pz = qz == 0 ? 0 : NY2 - qz;
  const int pidx = py * NY2 + pz;
  if (pidx < idx) return;
  for (int cc = 0; cc < ncomp; ++cc) {
    const size_t a = idxS(g, cc, qy, qz, 0), b = idxS(g, cc, py, pz, 0);
    const Cplx<T> va = S[a], vb = S[b];
    const Cplx<T> h = cmk<T>(T(0.5) * (va.x + vb.x), T(0.5) * (va.y - vb.y));
    S[a] = h;
    S[b] = conj(h);
  }
}

// ================================================================================================
// ConstantPower amplitude (src/Forcing.jl:1091-1117) for the stage state: the band sum is taken in
// a fixed order by one thread; the whole-field sum adds the per-tile partials in a fixed order.
// ================================================================================================
template <class T>
GBGHT_HD double band_energy_raw(const Geometry& g, const Cplx<T>* S, double lo2, double hi2, int c0 = 0, int nc = 3) {
  // Hermitian-weighted Σ|f̂|² of slots [c0, c0 + nc) over the band, unnormalised; m_a bounded by
  // the band edge
  int mb = int(std::sqrt(hi2) / g.s) + 1;
  if (mb > g.K) mb = g.K;
  double sum = 0.0;
  for (int cc = c0; cc < c0 + nc; ++cc)
    for (int my = -mb; my <= mb; ++my)
      for (int mz = -mb; mz <= mb; ++mz)
        for (int kx = 0; kx <= mb; ++kx) {
          const double kxd = g.s * kx, kyd = g.s * my, kzd = g.s * mz;
          const double k2 = (kxd * kxd + kyd * kyd) + kzd * kzd;
          if (!(k2 >= lo2 && k2 <= hi2)) continue;
          const int qy = my >= 0 ? my : my + g.NY2, qz = mz >= 0 ? mz : mz + g.NY2;
          const Cplx<T> v = S[idxS(g, cc, qy, qz, kx)];
          const double w = kx == 0 ? 1.0 : 2.0;
          sum += w * (double(v.x) * v.x + double(v.y) * v.y);
        }
  return sum;
}

// ================================================================================================
// The number a band forcing solves for from a field's raw, unnormalised sums (whole Σw|f̂|², band
// Σ_band w|f̂|², Dirichlet Σw|κ|²|f̂|², each divided by N⁶ to give the mean over the box):
//  - ConstantPower: A = ε/(2 k_band) (src/Forcing.jl:1091-1117);
//  - VarianceController: A = (ε_f − G(k − k∞)/tℓ)/(2 k_band), ε_f = 2·c·D·⟨f, |κ|²f⟩
//    (src/Forcing.jl:1041-1067);
//  - VarianceRescaling: the factor √(target_band/k_band) of the post-step rescale, target_band the
//    target (:band) or max(0, target − k + k_band) (:total) (src/Forcing.jl:575-596).
// c is ½ for the velocity and 1 for the scalar (`_target_factor`, :456). An empty band — not above
// 10·eps·whole (`_band_is_empty`, :110-111) — gives A = 0, or the factor 1 (the band left alone),
// and raises *empty.
// ================================================================================================
struct AmpArgs {
  int kind;              // ForcingKind
  double rate;           // ConstantPower ε
  double target, gain, turnover_time;
  int over;              // VarianceRescaling: 0 band, 1 total
  double factor;         // ½ velocity, 1 scalar
  double diffusivity;    // ν or ν/Sc
  double eps_T;          // the field precision's machine epsilon
};

GBGHT_HD double forcing_amplitude(const AmpArgs& a, double whole_raw, double band_raw, double dir_raw,
                                  double n6, double* band_obs, double* whole_obs, bool* empty) {
  const double band = a.factor * (band_raw / n6), whole = a.factor * (whole_raw / n6);
  *band_obs = band;
  *whole_obs = whole;
  if (a.kind == 4) {   // VarianceRescaling: the emptiness test on the raw sums, as the reference
    *empty = !(std::isfinite(band_raw) && band_raw > 10.0 * a.eps_T * whole_raw);
    if (*empty) return 1.0;
    const double target_band = a.over == 1 ? std::fmax(0.0, a.target - whole + band) : a.target;
    return std::sqrt(target_band / band);
  }
  *empty = !(std::isfinite(band) && band > 10.0 * a.eps_T * whole);
  if (*empty) return 0.0;
  if (a.kind == 3) {   // VarianceController
    const double dissipation = 2.0 * a.factor * a.diffusivity * (dir_raw / n6);
    const double restoring = a.gain * (whole - a.target) / a.turnover_time;
    return (dissipation - restoring) / (2.0 * band);
  }
  return a.rate / (2.0 * band);   // ConstantPower
}

// VarianceRescaling's rescale of one mode of the box |m_a| ≤ mb over slots c0..: i enumerates
// (slot, my, mz, kx) with kx fastest; a mode in the band becomes f + (s − 1)·f, the reference's
// convolve!(f, f, band, s − 1, 1) (src/Forcing.jl:595).
template <class T>
GBGHT_HD void rescale_mode(long i, const Geometry& g, Cplx<T>* S, int c0, int mb, double lo2, double hi2,
                           double factor) {
  const int side = 2 * mb + 1;
  const int kx = int(i % (mb + 1)), mz = int((i / (mb + 1)) % side) - mb, my = int((i / ((mb + 1) * side)) % side) - mb;
  const int cc = c0 + int(i / (long(mb + 1) * side * side));
  const double kxd = g.s * kx, kyd = g.s * my, kzd = g.s * mz;
  const double k2 = (kxd * kxd + kyd * kyd) + kzd * kzd;
  if (!(k2 >= lo2 && k2 <= hi2)) return;
  const int qy = my >= 0 ? my : my + g.NY2, qz = mz >= 0 ? mz : mz + g.NY2;
  Cplx<T>& v = S[idxS(g, cc, qy, qz, kx)];
  v = v + scale(v, T(factor - 1.0));
}
// ================================================================================================
// z-inverse of the current state into A slots 0..6 (u, iκ×û, φ), and the tile's Hermitian-weighted
// Σ|û|², with the same tiling as the epilogue. Used after an import to start a step. With `shift`
// each mode is first multiplied by e^{iπ(mx+my+mz)/N}: the fields on PhaseShift's displaced grid
// (the translation `to_shifted`, src/Generator.jl:169-175), into another A-layout array; the
// energy sum is still the state's.
// ================================================================================================
template <class T, int N, int TL, int NT, class Rows>
GBGHT_HD double body_z_init(const Cta& c, Cplx<T>* W, double* red, const Geometry& g, Rows& rows,
                            Cplx<T>* GBGHT_RESTRICT A, const Cplx<T>* GBGHT_RESTRICT S, int has_scalar,
                            const Cplx<T>* GBGHT_RESTRICT tw, int vorticity = 1, int shift = 0) {
  using O = typename Rows::Own;
  const int kx0 = c.bx * TL, qy = c.by;
  const int my = q_to_m(qy, g.K, g.NY2);
  const double ky = g.s * double(my);
  double esum = 0.0;
  // the retained rows of half 0, then of half 1: the epilogue's order, so the tile's energy sum
  // (the next stage's forcing amplitude reads it) is the epilogue's to the last bit
  const auto own = [&](int b, int sl, bool ret, int q, int mz, int l) {
    Cplx<T> u0 = czero<T>(), u1 = czero<T>(), u2 = czero<T>();
    if (ret) {
      const int kx = kx0 + l;
      u0 = S[idxS(g, 0, qy, q, kx)];
      u1 = S[idxS(g, 1, qy, q, kx)];
      u2 = S[idxS(g, 2, qy, q, kx)];
      const double w = kx == 0 ? 1.0 : 2.0;
      esum += w * ((double(u0.x) * u0.x + double(u0.y) * u0.y) + (double(u1.x) * u1.x + double(u1.y) * u1.y) +
                   (double(u2.x) * u2.x + double(u2.y) * u2.y));
      if (shift) {   // the state sampled on the displaced grid (PhaseShift)
        const Cplx<T> p = half_cell_phase<T>(kx + my + mz, N);
        u0 = u0 * p;
        u1 = u1 * p;
        u2 = u2 * p;
      }
    }
    rows.put(0, b, sl, u0);
    rows.put(1, b, sl, u1);
    rows.put(2, b, sl, u2);
  };
  for_own_slots<T, N, TL, NT, 0, O>(c, g, own);
  for_own_slots<T, N, TL, NT, 1, O>(c, g, own);
  rows.put_done();
  red[c.tid] = esum;
  GBGHT_SYNC();
  double total = 0.0;
  if (c.tid == 0)
    for (int i = 0; i < NT; ++i) total += red[i];
  z_inverse_velocity<T, N, TL, NT, O>(c, W, g, A, qy, kx0, ky, rows, vorticity, tw);
  if (has_scalar) {
    const auto phi = [&](int q, int l) {
      const Cplx<T> v = S[idxS(g, 3, qy, q, kx0 + l)];
      return shift ? v * half_cell_phase<T>(kx0 + l + my + q_to_m(q, g.K, g.NY2), N) : v;
    };
    z_inverse1<T, N, TL, NT>(c, W, g, A, 6, qy, kx0, phi, tw);
  }
  return total;
}

// ================================================================================================
// State import and export: one component in the reference layout [kz][ky][kx] (kx ≤ N/2,
// complex128) against one compact S component. One thread per reference mode i.
// Import keeps the retained 2/3 ball and reports content anywhere else (Nyquist planes included)
// in bit 0 of `flag`; export writes the compact box and zero elsewhere.
// ================================================================================================
template <class T>
GBGHT_HD void import_mode(size_t i, const Geometry& g, const Cplx<double>* ref, Cplx<T>* Sc, unsigned int* flag) {
  const int N = g.N, NH = N / 2 + 1;
  if (i >= size_t(N) * N * NH) return;
  const int kx = int(i % NH), ky = int((i / NH) % N), kz = int(i / (size_t(NH) * N));
  const Cplx<double> v = ref[i];
  const int my = ky <= N / 2 ? ky : ky - N, mz = kz <= N / 2 ? kz : kz - N;
  const bool in_box = kx <= g.K && (my < 0 ? -my : my) <= g.K && (mz < 0 ? -mz : mz) <= g.K &&
                      !(N % 2 == 0 && (ky == N / 2 || kz == N / 2));
  bool retained = false;
  if (in_box) {
    const double kxd = g.s * kx, kyd = g.s * my, kzd = g.s * mz;
    retained = (kxd * kxd + kyd * kyd) + kzd * kzd <= g.cut2;
  }
  if (retained) {
    const int qy = my >= 0 ? my : my + g.NY2, qz = mz >= 0 ? mz : mz + g.NY2;
    Sc[idxS(g, 0, qy, qz, kx)] = cmk<T>(T(v.x), T(v.y));
  } else if (v.x != 0.0 || v.y != 0.0) {
#ifdef __CUDA_ARCH__
    atomicOr(flag, 1u);
#else
    *flag |= 1u;
#endif
  }
}

template <class T>
GBGHT_HD void export_mode(size_t i, const Geometry& g, const Cplx<T>* Sc, Cplx<double>* ref) {
  const int N = g.N, NH = N / 2 + 1;
  if (i >= size_t(N) * N * NH) return;
  const int kx = int(i % NH), ky = int((i / NH) % N), kz = int(i / (size_t(NH) * N));
  const int my = ky <= N / 2 ? ky : ky - N, mz = kz <= N / 2 ? kz : kz - N;
  Cplx<double> v = cmk<double>(0.0, 0.0);
  if (kx <= g.K && (my < 0 ? -my : my) <= g.K && (mz < 0 ? -mz : mz) <= g.K) {
    const int qy = my >= 0 ? my : my + g.NY2, qz = mz >= 0 ? mz : mz + g.NY2;
    const Cplx<T> w = Sc[idxS(g, 0, qy, qz, kx)];
    v = cmk<double>(double(w.x), double(w.y));
  }
  ref[i] = v;
}

// ================================================================================================
// Observables: per ky' row, the Hermitian-weighted sums Σ|û|², Σκ²|û|², Σ|φ̂|², Σκ²|φ̂|²
// (unnormalised), summed per thread and then in thread order. Grid: (NY2). `red` holds 4·NT.
// has_scalar = 2 takes the scalar sums only (the velocity sums are left at zero).
// ================================================================================================
template <class T, int NT>
GBGHT_HD void body_observables(const Cta& c, double* red, const Geometry& g, const Cplx<T>* GBGHT_RESTRICT S,
                               int has_scalar, double* GBGHT_RESTRICT out) {
  const int qy = c.bx;
  const int NY2 = g.NY2, KX1 = g.K + 1;
  const double ky = g.s * double(q_to_m(qy, g.K, NY2));
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = c.tid; i < NY2 * KX1; i += NT) {
    const int qz = i / KX1, kx = i % KX1;
    const double kxd = g.s * kx, kzd = g.s * q_to_m(qz, g.K, NY2);
    const double k2 = (kxd * kxd + ky * ky) + kzd * kzd;
    const double w = kx == 0 ? 1.0 : 2.0;
    if (has_scalar != 2) {
      double e = 0.0;
      for (int cc = 0; cc < 3; ++cc) {
        const Cplx<T> v = S[idxS(g, cc, qy, qz, kx)];
        e += double(v.x) * v.x + double(v.y) * v.y;
      }
      acc[0] += w * e;
      acc[1] += w * k2 * e;
    }
    if (has_scalar) {
      const Cplx<T> v = S[idxS(g, 3, qy, qz, kx)];
      const double p = double(v.x) * v.x + double(v.y) * v.y;
      acc[2] += w * p;
      acc[3] += w * k2 * p;
    }
  }
  for (int j = 0; j < 4; ++j) red[j * NT + c.tid] = acc[j];
  GBGHT_SYNC();
  if (c.tid == 0)
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int i = 0; i < NT; ++i) s += red[j * NT + i];
      out[qy * 4 + j] = s;
    }
}

// ================================================================================================
// Energy and dissipation below scale (src/Observables.jl:253-263): per ky' row and chunk of CH box
// sides l = nL/N (n = n0+1 … n0+CH), the Hermitian-weighted Σ W_l²|û|² and Σ κ² W_l²|û|² with
// W_l(κ) = ∏_a sinc(κ_a l/2). The sinc factors of the chunk are tabulated per |m| in `tab`
// (CH·(K+1) doubles); each sum runs per thread and then in thread order through `red` (NT
// doubles). out[(qy·N + n − 1)·2 + {0, 1}]. Grid: (NY2, ⌈N/CH⌉).
// ================================================================================================
template <class T, int NT, int CH>
GBGHT_HD void body_below_scale(const Cta& c, double* tab, double* red, const Geometry& g, double L,
                               const Cplx<T>* GBGHT_RESTRICT S, double* GBGHT_RESTRICT out) {
  const int qy = c.bx, n0 = c.by * CH, N = g.N;
  const int KX1 = g.K + 1, NY2 = g.NY2;
  const int nch = N - n0 < CH ? N - n0 : CH;
  for (int i = c.tid; i < CH * KX1; i += NT) {
    const int j = i / KX1, m = i % KX1;
    const double l = double(n0 + j + 1) * L / double(N);
    const double y = (g.s * double(m)) * l / 2.0;
    tab[i] = m == 0 ? 1.0 : sin(y) / y;
  }
  GBGHT_SYNC();
  const int my = q_to_m(qy, g.K, NY2);
  const double ky = g.s * double(my);
  const double* ty = tab + (my < 0 ? -my : my);
  double ak[CH], ae[CH];
  for (int j = 0; j < CH; ++j) ak[j] = ae[j] = 0.0;
  for (int i = c.tid; i < NY2 * KX1; i += NT) {
    const int qz = i / KX1, kx = i % KX1;
    const int mz = q_to_m(qz, g.K, NY2);
    const double kxd = g.s * kx, kzd = g.s * mz;
    const double k2 = (kxd * kxd + ky * ky) + kzd * kzd;
    double e = 0.0;
    for (int cc = 0; cc < 3; ++cc) {
      const Cplx<T> v = S[idxS(g, cc, qy, qz, kx)];
      e += double(v.x) * v.x + double(v.y) * v.y;
    }
    const double we = (kx == 0 ? 1.0 : 2.0) * e;
    const double* tz = tab + (mz < 0 ? -mz : mz);
    for (int j = 0; j < CH; ++j) {
      const double W = (tab[j * KX1 + kx] * ty[j * KX1]) * tz[j * KX1];
      const double p = (W * W) * we;
      ak[j] += p;
      ae[j] += k2 * p;
    }
  }
  for (int j = 0; j < nch; ++j)
    for (int which = 0; which < 2; ++which) {
      red[c.tid] = which == 0 ? ak[j] : ae[j];
      GBGHT_SYNC();
      if (c.tid == 0) {
        double s = 0.0;
        for (int i = 0; i < NT; ++i) s += red[i];
        out[(size_t(qy) * N + n0 + j) * 2 + which] = s;
      }
      GBGHT_SYNC();
    }
}

// ================================================================================================
// Shell spectrum: per ky' row, the Hermitian-weighted Σ|f̂|² of each shell n = floor(|κ|/Δκ + ½),
// for S slots [c0, c0+nc). Each kz' line is summed by thread 0 in kx order, so the result does
// not depend on the launch. Grid: (NY2). `hist` holds nshell doubles, `vals` KXP·2 doubles.
// ================================================================================================
template <class T, int NT>
GBGHT_HD void body_spectrum(const Cta& c, double* hist, double* vals, const Geometry& g,
                            const Cplx<T>* GBGHT_RESTRICT S, int c0, int nc, int nshell,
                            double* GBGHT_RESTRICT out) {
  const int qy = c.bx;
  const int NY2 = g.NY2, KX1 = g.K + 1;
  const double ky = g.s * double(q_to_m(qy, g.K, NY2));
  for (int i = c.tid; i < nshell; i += NT) hist[i] = 0.0;
  GBGHT_SYNC();
  for (int qz = 0; qz < NY2; ++qz) {
    const double kzd = g.s * q_to_m(qz, g.K, NY2);
    for (int kx = c.tid; kx < KX1; kx += NT) {
      const double kxd = g.s * kx;
      const double k2 = (kxd * kxd + ky * ky) + kzd * kzd;
      double e = 0.0;
      for (int cc = c0; cc < c0 + nc; ++cc) {
        const Cplx<T> v = S[idxS(g, cc, qy, qz, kx)];
        e += double(v.x) * v.x + double(v.y) * v.y;
      }
      vals[2 * kx] = (kx == 0 ? 1.0 : 2.0) * e;
      vals[2 * kx + 1] = floor(sqrt(k2) / g.s + 0.5);
    }
    GBGHT_SYNC();
    if (c.tid == 0)
      for (int kx = 0; kx < KX1; ++kx) {
        const int n = int(vals[2 * kx + 1]);
        if (n < nshell) hist[n] += vals[2 * kx];
      }
    GBGHT_SYNC();
  }
  for (int i = c.tid; i < nshell; i += NT) out[size_t(qy) * nshell + i] = hist[i];
}

}  // namespace gbght
