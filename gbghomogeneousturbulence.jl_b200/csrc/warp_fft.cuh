// Warp-per-line FFT: each warp owns whole lines of length N in shared memory and transforms them
// with no block-wide barrier (its radix stages are separated by __syncwarp only).
//
// A line is N contiguous complex elements, XOR-swizzled within each 128-byte row. For FP64, element
// e sits at lidx(e) = e with its 16-byte chunk index (e mod 8) XORed with the row index mod 8. For FP32,
// the element's index within its row (e mod 16) is XORed with (5 × row) mod 16. The access patterns
// of the Stockham stages below are reads x[j + r·N/R], writes y[(j/NS)·NS·R + j mod NS + r·NS], and
// the column walks of the x pass. FP64 serves them free of bank conflicts. FP32 is conflict-free on
// the 512-point plan and within 6% of the ideal wavefront count on the others.
//
// The algorithm is the Stockham autosort of fft_tile.cuh (same radices, same twiddles, same
// results), with butterfly j of a stage taken by lane j mod 32 of the owning warp. As there, the
// first stage can read from an external source and the last stage can write to an external sink.
//
// Execution model: the caller iterates `for (t = c.tid; t < 32·NW; t += NT)`. On the device
// NT = 32·NW, so each thread takes one (warp, lane). In the host-check build NT = 1 and one
// thread plays every lane in turn. A stage's loads for all lanes of a warp complete before any
// store, so the in-place stages are exact in both builds.
#pragma once

#include "fft_tile.cuh"

namespace gbght {

template <class T>
GBGHT_HD int lidx(int e) {
  if constexpr (sizeof(Cplx<T>) == 16) return e ^ ((e >> 3) & 7);
  else return e ^ (((e >> 4) * 5) & 15);
}

GBGHT_HD void warp_sync() {
#ifdef __CUDA_ARCH__
  __syncwarp();
#endif
}

template <class T>
struct LineBuf {
  static constexpr bool kExternal = false;
  Cplx<T>* line;
  GBGHT_HD Cplx<T> load(int e) const { return line[lidx<T>(e)]; }
  GBGHT_HD void store(int e, Cplx<T> v) const { line[lidx<T>(e)] = v; }
};

// Transform line `w` of each of NW warps (lines w + k·NW when nlines > NW), stages [S, S_END).
// `lines(w)` returns the shared-memory base of line w; `src(w)`/`dst(w)` the first-stage source
// and last-stage sink of line w. Only lines w < nlines are transformed.
template <class T, int N, int NW, int NT, int SIGN, int S = 0, int S_END = Radices<N>::n, class LineOf, class SrcOf,
          class DstOf>
GBGHT_HD void warp_fft_lines(const Cta& c, int nlines, const LineOf& lines, const SrcOf& src, const DstOf& dst,
                             const Cplx<T>* GBGHT_RESTRICT tw) {
  if constexpr (S < S_END) {
    constexpr int R = Radices<N>::r[S];
    constexpr int NS = stage_ns<N>(S);
    constexpr int NB = N / R;
    constexpr int BPL = (NB + 31) / 32;          // butterflies per lane
    constexpr int TWS = N / (NS * R);
    constexpr bool FIRST = S == 0, LAST = S + 1 == Radices<N>::n;
    constexpr int NTOT = 32 * NW;
    constexpr int SLOTS = (NTOT + NT - 1) / NT;  // (warp, lane) pairs per thread: 1 on the device
    for (int base_line = 0; base_line < nlines; base_line += NW) {
      Cplx<T> v[SLOTS][BPL][R];
#pragma unroll
      for (int s = 0; s < SLOTS; ++s) {
        const int t = c.tid + s * NT;
        const int w = t >> 5, lane = t & 31, ln = base_line + w;
        if (t < NTOT && ln < nlines) {
          Cplx<T>* L = lines(ln);
          const auto sr = src(ln);
#pragma unroll
          for (int b = 0; b < BPL; ++b) {
            const int j = lane + 32 * b;
            if (NB % 32 == 0 || j < NB) {
#pragma unroll
              for (int r = 0; r < R; ++r) {
                if constexpr (FIRST) v[s][b][r] = sr.load(j + r * NB);
                else v[s][b][r] = L[lidx<T>(j + r * NB)];
              }
            }
          }
        }
      }
      warp_sync();
#pragma unroll
      for (int s = 0; s < SLOTS; ++s) {
        const int t = c.tid + s * NT;
        const int w = t >> 5, lane = t & 31, ln = base_line + w;
        if (t < NTOT && ln < nlines) {
          Cplx<T>* L = lines(ln);
          const auto ds = dst(ln);
#pragma unroll
          for (int b = 0; b < BPL; ++b) {
            const int j = lane + 32 * b;
            if (NB % 32 == 0 || j < NB) {
              const int jm = j % NS;
              if constexpr (NS > 1) {
                Cplx<T> wv[R];
                twiddles<T, R, SIGN>(tw, jm * TWS, wv);
#pragma unroll
                for (int r = 1; r < R; ++r) v[s][b][r] = v[s][b][r] * wv[r];
              }
              dft<T, R, SIGN>(v[s][b]);
              const int base = (j / NS) * NS * R + jm;
#pragma unroll
              for (int r = 0; r < R; ++r) {
                if constexpr (LAST) ds.store(base + r * NS, v[s][b][r]);
                else L[lidx<T>(base + r * NS)] = v[s][b][r];
              }
            }
          }
        }
      }
      warp_sync();
    }
    warp_fft_lines<T, N, NW, NT, SIGN, S + 1, S_END>(c, nlines, lines, src, dst, tw);
  }
}

}  // namespace gbght
