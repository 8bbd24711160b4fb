// The tile FFT: TL independent complex lines of length N, held in shared memory as N rows of TL
// elements (element e of line l at buf[e*TL + l]). The lines are transformed together.
//
// Algorithm: Stockham autosort, decimation in time, mixed radix (Govindaraju et al., "High
// Performance Discrete Fourier Transforms on Graphics Processors", SC 2008). Stage s has radix R,
// and NS is the product of the radices before it. Butterfly j of a line reads
// x[j + r·N/R] (r < R) and twiddles each input by w^(r·(j mod NS)·N/(NS·R)), with w = e^(∓2πi/N).
// It then takes an R-point DFT and writes y[(j / NS)·NS·R + j mod NS + r·NS]. Each stage works in
// place: every thread loads its butterflies, the block synchronises, then every thread stores.
//
// Consecutive threads take the same butterfly of consecutive lines (idx = j·TL + l; the threads of
// lines at or past ACT stay idle). A quarter warp of 8 threads therefore touches one row of the
// tile, for every stage's reads and writes.
// Rows are 64 or 128 bytes, so the shared-memory accesses are free of bank conflicts whatever the
// stage's stride.
//
// SIGN = -1 is the forward (unnormalised) transform, SIGN = +1 the inverse (unnormalised).
// `tw` holds e^(-2πi k/N) for k in [0, N), computed on the host in extended precision.
#pragma once

#include <type_traits>

#include "gbght_common.cuh"

namespace gbght {

// Radix plans, innermost stage first. Every supported N is 2^a·3^b. Every plan starts and ends
// with the same radix, so the rows a thread writes in a forward transform's last stage are the rows
// it reads in an inverse transform's first stage (the z epilogue keeps them in registers).
template <int N> struct Radices;
template <> struct Radices<8>   { static constexpr int n = 1; static constexpr int r[1] = {8}; };
template <> struct Radices<12>  { static constexpr int n = 3; static constexpr int r[3] = {2, 3, 2}; };
template <> struct Radices<16>  { static constexpr int n = 2; static constexpr int r[2] = {4, 4}; };
template <> struct Radices<24>  { static constexpr int n = 4; static constexpr int r[4] = {2, 3, 2, 2}; };
template <> struct Radices<32>  { static constexpr int n = 3; static constexpr int r[3] = {4, 2, 4}; };
template <> struct Radices<48>  { static constexpr int n = 3; static constexpr int r[3] = {4, 3, 4}; };
template <> struct Radices<64>  { static constexpr int n = 2; static constexpr int r[2] = {8, 8}; };
template <> struct Radices<96>  { static constexpr int n = 4; static constexpr int r[4] = {4, 3, 2, 4}; };
template <> struct Radices<128> { static constexpr int n = 3; static constexpr int r[3] = {8, 2, 8}; };
template <> struct Radices<192> { static constexpr int n = 3; static constexpr int r[3] = {8, 3, 8}; };
template <> struct Radices<256> { static constexpr int n = 3; static constexpr int r[3] = {8, 4, 8}; };
template <> struct Radices<384> { static constexpr int n = 4; static constexpr int r[4] = {8, 2, 3, 8}; };
template <> struct Radices<512> { static constexpr int n = 3; static constexpr int r[3] = {8, 8, 8}; };

template <int N> constexpr int stage_ns(int s) {
  int p = 1;
  for (int i = 0; i < s; ++i) p *= Radices<N>::r[i];
  return p;
}

// ---- small DFTs in registers ------------------------------------------------------------------

template <class T, int SIGN> GBGHT_HD void dft2(Cplx<T>* v) {
  Cplx<T> a = v[0], b = v[1];
  v[0] = a + b;
  v[1] = a - b;
}

template <class T, int SIGN> GBGHT_HD void dft3(Cplx<T>* v) {
  // X_k = Σ a_n e^(SIGN·2πi nk/3)
  const T c1 = T(-0.5);
  const T s1 = T(SIGN) * T(0.86602540378443864676372317075294);
  Cplx<T> a0 = v[0], a1 = v[1], a2 = v[2];
  Cplx<T> t = a1 + a2, d = a1 - a2;
  Cplx<T> m = cmk<T>(a0.x + c1 * t.x, a0.y + c1 * t.y);
  // s1 · i · d
  Cplx<T> r = cmk<T>(-s1 * d.y, s1 * d.x);
  v[0] = a0 + t;
  v[1] = m + r;
  v[2] = m - r;
}

template <class T, int SIGN> GBGHT_HD void dft4(Cplx<T>* v) {
  Cplx<T> a0 = v[0], a1 = v[1], a2 = v[2], a3 = v[3];
  Cplx<T> t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, d = a1 - a3;
  Cplx<T> t3 = (SIGN < 0) ? mul_mi(d) : mul_i(d);
  v[0] = t0 + t2;
  v[2] = t0 - t2;
  v[1] = t1 + t3;
  v[3] = t1 - t3;
}

template <class T, int SIGN> GBGHT_HD void dft8(Cplx<T>* v) {
  // even/odd split into two 4-point DFTs, then combine with w8^k = e^(SIGN·iπk/4)
  Cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
  Cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
  dft4<T, SIGN>(e);
  dft4<T, SIGN>(o);
  const T h = T(0.70710678118654752440084436210485);
  // w8^1 = (h, SIGN·h), w8^2 = SIGN·i, w8^3 = (-h, SIGN·h)
  Cplx<T> o1 = cmk<T>(h * (o[1].x - T(SIGN) * o[1].y), h * (o[1].y + T(SIGN) * o[1].x));
  Cplx<T> o2 = (SIGN < 0) ? mul_mi(o[2]) : mul_i(o[2]);
  Cplx<T> o3 = cmk<T>(-h * (o[3].x + T(SIGN) * o[3].y), h * (T(SIGN) * o[3].x - o[3].y));
  v[0] = e[0] + o[0];
  v[4] = e[0] - o[0];
  v[1] = e[1] + o1;
  v[5] = e[1] - o1;
  v[2] = e[2] + o2;
  v[6] = e[2] - o2;
  v[3] = e[3] + o3;
  v[7] = e[3] - o3;
}

template <class T, int R, int SIGN> GBGHT_HD void dft(Cplx<T>* v) {
  if constexpr (R == 2) dft2<T, SIGN>(v);
  else if constexpr (R == 3) dft3<T, SIGN>(v);
  else if constexpr (R == 4) dft4<T, SIGN>(v);
  else if constexpr (R == 8) dft8<T, SIGN>(v);
  else static_assert(R == 2, "unsupported radix");
}

// ---- the tile transform -------------------------------------------------------------------------

// Index of element e of line l in a tile of TL lines.
template <int TL>
GBGHT_HD int tix(int e, int l) { return e * TL + l; }

// The twiddle table e^(-2πi k/N): a pointer is a table in global memory (read through the
// read-only path); SharedTwiddles is a copy in shared memory, for kernels whose L1 cannot keep the
// table next to their streaming traffic.
template <class T>
struct SharedTwiddles {
  const Cplx<T>* p;
};
template <class T> GBGHT_HD Cplx<T> tw_at(const Cplx<T>* GBGHT_RESTRICT tw, int k) { return ldgc(tw + k); }
template <class T> GBGHT_HD Cplx<T> tw_at(const SharedTwiddles<T>& tw, int k) { return tw.p[k]; }

// Twiddles w^(jm·r·TWS), r = 1..R−1, from one table read: w₂ = w₁², w₃ = w₂w₁, w₄ = w₂², w₅ = w₄w₁,
// w₆ = w₄w₂, w₇ = w₄w₃ (at most three products deep, so a few ulp of error).
template <class T, int R, int SIGN, class TW>
GBGHT_HD void twiddles(const TW& tw, int k, Cplx<T>* w) {
  w[1] = tw_at<T>(tw, k);
  if constexpr (SIGN > 0) w[1] = conj(w[1]);
  if constexpr (R > 2) w[2] = w[1] * w[1];
  if constexpr (R > 3) w[3] = w[2] * w[1];
  if constexpr (R > 4) {
    w[4] = w[2] * w[2];
    w[5] = w[4] * w[1];
    w[6] = w[4] * w[2];
    w[7] = w[4] * w[3];
  }
}

// A source or sink with kIndexed = true is called as load_rb(e, l, r, b) / store_rb(e, l, v, r, b),
// with the radix index r and the thread's butterfly slot b as compile-time constants after
// unrolling, so it can keep values in a per-thread register array.
template <class F, class = void>
struct is_indexed : std::false_type {};
template <class F>
struct is_indexed<F, std::void_t<decltype(F::kIndexed)>> : std::bool_constant<F::kIndexed> {};

// The tile buffer as the default source of the first stage and sink of the last one.
template <class T, int TL>
struct TileBuf {
  static constexpr bool kExternal = false;   // the first stage reads the tile it writes
  Cplx<T>* buf;
  GBGHT_HD Cplx<T> load(int e, int l) const { return buf[tix<TL>(e, l)]; }
  GBGHT_HD void store(int e, int l, Cplx<T> v) const { buf[tix<TL>(e, l)] = v; }
};

// ACT ≤ TL lines are transformed; lines ACT..TL−1 are left untouched. The first stage reads its
// inputs through `src.load(e, l)` (a source with kExternal = true never aliases the tile) and the last stage writes its outputs through
// `dst.store(e, l, v)`; every other access goes through the tile in shared memory. With the
// defaults both are the tile itself, and the transform is in place. With an external source the
// first stage loads straight into registers (from global memory, say), and with an external sink
// the last stage stores straight out, so neither costs a pass through shared memory.
//
// Stages [S, S_END) run; a call that stops early leaves the partial transform in the tile, and a
// later call with S = the stop resumes it (the caller can act between the two, after the barrier
// that ends every stage).
template <class T, int N, int TL, int NT, int SIGN, int ACT = TL, int S = 0,
          int S_END = Radices<N>::n, class Src, class Dst, class TW>
GBGHT_HD void tile_fft_io(const Cta& c, Cplx<T>* buf, const TW& tw, const Src& src, const Dst& dst) {
  if constexpr (S < S_END) {
    constexpr int R = Radices<N>::r[S];
    constexpr int NS = stage_ns<N>(S);
    constexpr int NB = N / R;
    constexpr int TOT = NB * TL;
    constexpr int BPT = (TOT + NT - 1) / NT;
    constexpr int TWS = N / (NS * R);
    constexpr bool FIRST = S == 0, LAST = S + 1 == Radices<N>::n;
    Cplx<T> v[BPT][R];
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
      const int idx = c.tid + b * NT;
      const int l = idx % TL, j = idx / TL;
      if ((BPT * NT == TOT || idx < TOT) && (ACT == TL || l < ACT)) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if constexpr (FIRST) {
            if constexpr (is_indexed<Src>::value) v[b][r] = src.load_rb(j + r * NB, l, r, b);
            else v[b][r] = src.load(j + r * NB, l);
          } else {
            v[b][r] = buf[tix<TL>(j + r * NB, l)];
          }
        }
      }
    }
    if constexpr (!FIRST || !Src::kExternal) GBGHT_SYNC();
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
      const int idx = c.tid + b * NT;
      const int l = idx % TL, j = idx / TL;
      if ((BPT * NT == TOT || idx < TOT) && (ACT == TL || l < ACT)) {
        const int jm = j % NS;
        if constexpr (NS > 1) {
          Cplx<T> w[R];
          twiddles<T, R, SIGN>(tw, jm * TWS, w);
#pragma unroll
          for (int r = 1; r < R; ++r) v[b][r] = v[b][r] * w[r];
        }
        dft<T, R, SIGN>(v[b]);
        const int base = (j / NS) * NS * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if constexpr (LAST) {
            if constexpr (is_indexed<Dst>::value) dst.store_rb(base + r * NS, l, v[b][r], r, b);
            else dst.store(base + r * NS, l, v[b][r]);
          } else {
            buf[tix<TL>(base + r * NS, l)] = v[b][r];
          }
        }
      }
    }
    GBGHT_SYNC();
    tile_fft_io<T, N, TL, NT, SIGN, ACT, S + 1, S_END>(c, buf, tw, src, dst);
  }
}

template <class T, int N, int TL, int NT, int SIGN, int ACT = TL>
GBGHT_HD void tile_fft(const Cta& c, Cplx<T>* buf, const Cplx<T>* GBGHT_RESTRICT tw) {
  const TileBuf<T, TL> tb{buf};
  tile_fft_io<T, N, TL, NT, SIGN, ACT>(c, buf, tw, tb, tb);
}

}  // namespace gbght
