// Lagrangian tracers: periodic wrap, Catmull–Rom gather, and the Heun (= ABM(1)) push.
//
// Positions are FP64 in both precision forms. The wrap and the displacement are evaluated with
// round-to-nearest operations and no fused multiply-add, in the order the reference's update
// reads (src/ParticlePropagator.jl:288-315), so a cell index floor(x/Δx) is reproducible.
#pragma once

#include "gbght_common.cuh"

#include <utility>

namespace gbght {

GBGHT_HD double add_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
GBGHT_HD double sub_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
GBGHT_HD double mul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
GBGHT_HD double div_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}

// x − L·floor(x/L); a tiny negative result is lifted by L; a result equal to L maps to 0.
GBGHT_HD double wrap_periodic(double x, double L) {
  double y = sub_rn(x, mul_rn(L, floor(div_rn(x, L))));
  if (y < 0.0) y = add_rn(y, L);
  if (y >= L) y = 0.0;
  return y;
}

// Catmull–Rom weights for taps i−1, i, i+1, i+2 at fraction t (Catmull & Rom 1974).
GBGHT_HD void catmull_rom(double t, double w[4]) {
  w[0] = mul_rn(mul_rn(t, sub_rn(mul_rn(t, sub_rn(2.0, t)), 1.0)), 0.5);
  w[1] = mul_rn(add_rn(mul_rn(mul_rn(t, t), sub_rn(mul_rn(3.0, t), 5.0)), 2.0), 0.5);
  w[2] = mul_rn(mul_rn(t, add_rn(mul_rn(t, sub_rn(4.0, mul_rn(3.0, t))), 1.0)), 0.5);
  w[3] = mul_rn(mul_rn(mul_rn(t, t), sub_rn(t, 1.0)), 0.5);
}

// Cell i = floor(x/Δx) reduced into [0, N), and the fraction t = x/Δx − floor(x/Δx). A
// non-finite position gives cell 0 and a non-finite fraction, so the gathered value is NaN and
// no index leaves the field.
GBGHT_HD void cell_fraction(double x, double dx, int N, int& i, double& t) {
  const double q = div_rn(x, dx);
  if (!(q - q == 0.0)) {
    i = 0;
    t = q - q;
    return;
  }
  const double f = floor(q);
  const double r = sub_rn(f, mul_rn(double(N), floor(div_rn(f, double(N)))));
  i = int(r);
  if (i < 0 || i >= N) i = 0;
  t = sub_rn(q, f);
}

// The four x taps ix − 1 .. ix + 2 of one row of a physical field (rows 16-byte aligned: N·sizeof(T)
// is a multiple of 16 for every supported N). Away from the row's ends the taps come in 16-byte
// vector loads where their alignment allows (two for FP64 on an even start, one for FP32 on a start
// divisible by 4), else in narrower aligned pieces; at the ends, one by one with the periodic wrap.
// The values, and so every sum of them, are those of four scalar loads. The warp-cooperative gather
// uses it (the lanes of a tracer share ix, so they take one branch); the per-tracer gather loads its
// taps one by one, since its lanes' alignments differ and the branches diverge (its FP32 push took
// 1.87 ms per 10⁶ tracers with these loads, 1.00 ms without).
template <class T>
GBGHT_HD void row_taps(const T* GBGHT_RESTRICT row, int ix, int N, double v[4]) {
  const int x0 = ix - 1;
#ifdef __CUDA_ARCH__
  if (x0 >= 0 && x0 + 3 < N) {
    if constexpr (sizeof(T) == 8) {
      const double* r = reinterpret_cast<const double*>(row);
      if ((x0 & 1) == 0) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(r + x0));
        const double2 b = __ldg(reinterpret_cast<const double2*>(r + x0 + 2));
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
      } else {
        const double2 a = __ldg(reinterpret_cast<const double2*>(r + x0 + 1));
        v[0] = __ldg(r + x0); v[1] = a.x; v[2] = a.y; v[3] = __ldg(r + x0 + 3);
      }
    } else {
      const float* r = reinterpret_cast<const float*>(row);
      if ((x0 & 3) == 0) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(r + x0));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
      } else if ((x0 & 1) == 0) {
        const float2 a = __ldg(reinterpret_cast<const float2*>(r + x0));
        const float2 b = __ldg(reinterpret_cast<const float2*>(r + x0 + 2));
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
      } else {
        const float2 a = __ldg(reinterpret_cast<const float2*>(r + x0 + 1));
        v[0] = __ldg(r + x0); v[1] = a.x; v[2] = a.y; v[3] = __ldg(r + x0 + 3);
      }
    }
    return;
  }
#endif
  for (int a = 0; a < 4; ++a) v[a] = double(ldg(row + (x0 + a + N) % N));
}

// Gather the three components of a physical field [3][N][N][N] at X; sums run x innermost,
// then y, then z.
template <class T>
GBGHT_HD void gather3(const T* GBGHT_RESTRICT u, int N, double dx, double x, double y, double z,
                      double out[3]) {
  int ix, iy, iz;
  double tx, ty, tz;
  cell_fraction(x, dx, N, ix, tx);
  cell_fraction(y, dx, N, iy, ty);
  cell_fraction(z, dx, N, iz, tz);
  double wx[4], wy[4], wz[4];
  catmull_rom(tx, wx);
  catmull_rom(ty, wy);
  catmull_rom(tz, wz);
  int ys[4], zs[4];
  for (int a = 0; a < 4; ++a) {
    ys[a] = (iy + a - 1 + N) % N;
    zs[a] = (iz + a - 1 + N) % N;
  }
  const size_t comp = size_t(N) * N * N;
  for (int c = 0; c < 3; ++c) {
    const T* f = u + c * comp;
    double acc_z = 0.0;
    for (int cz = 0; cz < 4; ++cz) {
      double acc_y = 0.0;
      for (int cy = 0; cy < 4; ++cy) {
        const T* row = f + (size_t(zs[cz]) * N + ys[cy]) * N;
        double tap[4];   // the row's loads first, so that they overlap (the push took 1.65 ms with
                         // each load inside its sum, 1.27 ms so, at 512³ FP64 with 10⁶ tracers)
        for (int a = 0; a < 4; ++a) tap[a] = double(ldg(row + (ix + a - 1 + N) % N));
        double acc_x = 0.0;
        for (int cx = 0; cx < 4; ++cx) acc_x = add_rn(acc_x, mul_rn(wx[cx], tap[cx]));
        acc_y = add_rn(acc_y, mul_rn(wy[cy], acc_x));
      }
      acc_z = add_rn(acc_z, mul_rn(wz[cz], acc_y));
    }
    out[c] = acc_z;
  }
}

// ================================================================================================
// Wider interpolation stencils (src/Particles.jl:61-70; the schemes of GBGPeriodicFields, which is
// not vendored, restated from their published definitions):
//  - LagrangeSpline(n): the degree n − 1 Lagrange polynomial through the n taps around the cell;
//  - LalescuSpline(n; smoothness m) (Lalescu, Teaca & Carati 2010): on each cell, the degree 2m + 1
//    Hermite polynomial matching at both ends the value and the derivatives 1..m, each derivative
//    estimated by the centred difference of the (n − 1)-point Lagrange polynomial about that end.
//    LalescuSpline(4; 1) is Catmull–Rom.
// Either is a set of n weight polynomials w_j(t), j = 0..n−1 for the taps i − n/2 + 1 + j at the
// fraction t of cell i; their coefficients are built once on the host (make_stencil).
// ================================================================================================
constexpr int kStencilMax = 8;
struct Stencil {
  int n;                                     // taps per axis; 0 selects the Catmull–Rom gather above
  int deg;                                   // the weights' polynomial degree
  double c[kStencilMax][kStencilMax];        // w_j(t) = Σ_d c[j][d]·t^d
};

GBGHT_HD void stencil_weights(const Stencil& s, double t, double* w) {
  for (int j = 0; j < s.n; ++j) {
    double v = s.c[j][s.deg];
    for (int d = s.deg - 1; d >= 0; --d) v = fma(v, t, s.c[j][d]);
    w[j] = v;
  }
}

// The gather of gatherN: the sums run x innermost, then y, then z.
template <class T>
GBGHT_HD void gatherN(const T* GBGHT_RESTRICT u, int N, double dx, double x, double y, double z, const Stencil& s,
                      double out[3]) {
  int ix, iy, iz;
  double tx, ty, tz;
  cell_fraction(x, dx, N, ix, tx);
  cell_fraction(y, dx, N, iy, ty);
  cell_fraction(z, dx, N, iz, tz);
  double wx[kStencilMax], wy[kStencilMax], wz[kStencilMax];
  stencil_weights(s, tx, wx);
  stencil_weights(s, ty, wy);
  stencil_weights(s, tz, wz);
  const int off = s.n / 2 - 1;
  const size_t comp = size_t(N) * N * N;
  for (int c = 0; c < 3; ++c) {
    const T* f = u + c * comp;
    double acc_z = 0.0;
    for (int cz = 0; cz < s.n; ++cz) {
      const int zz = ((iz + cz - off) % N + N) % N;
      double acc_y = 0.0;
      for (int cy = 0; cy < s.n; ++cy) {
        const int yy = ((iy + cy - off) % N + N) % N;
        const T* row = f + (size_t(zz) * N + yy) * N;
        double tap[kStencilMax];   // the row's loads first, so that they overlap
        for (int cx = 0; cx < s.n; ++cx) tap[cx] = double(ldg(row + ((ix + cx - off) % N + N) % N));
        double acc_x = 0.0;
        for (int cx = 0; cx < s.n; ++cx) acc_x = add_rn(acc_x, mul_rn(wx[cx], tap[cx]));
        acc_y = add_rn(acc_y, mul_rn(wy[cy], acc_x));
      }
      acc_z = add_rn(acc_z, mul_rn(wz[cz], acc_y));
    }
    out[c] = acc_z;
  }
}

// The configured gather: Catmull–Rom (n = 0), or a wider stencil.
template <class T>
GBGHT_HD void gather_any(const T* GBGHT_RESTRICT u, int N, double dx, double x, double y, double z, const Stencil& s,
                         double out[3]) {
  if (s.n == 0) gather3(u, N, dx, x, y, z, out);
  else gatherN(u, N, dx, x, y, z, s, out);
}

// Host: the coefficients of a stencil. kind 1 LalescuSpline(n; m), 2 LagrangeSpline(n); n even in
// [4, 8]; 1 ≤ m ≤ min(3, n − 2). Returns nullptr, or why the stencil is refused.
inline const char* make_stencil(int kind, int n, int m, Stencil* s) {
  *s = Stencil{};
  if (n < 4 || n > kStencilMax || n % 2) return "the stencil width must be 4, 6 or 8 points per axis";
  const int off = n / 2 - 1;
  // p ← p·(t − a)/b, coefficients in increasing degree
  const auto mul_lin = [](double* p, int deg, double a, double b) {
    for (int d = deg + 1; d >= 0; --d) p[d] = ((d > 0 ? p[d - 1] : 0.0) - a * p[d]) / b;
  };
  if (kind == 2) {   // Lagrange through the taps x_j = j − off
    s->n = n;
    s->deg = n - 1;
    for (int j = 0; j < n; ++j) {
      double p[kStencilMax + 1] = {1.0};
      int deg = 0;
      for (int q = 0; q < n; ++q) {
        if (q == j) continue;
        mul_lin(p, deg, double(q - off), double(j - q));
        ++deg;
      }
      for (int d = 0; d < n; ++d) s->c[j][d] = p[d];
    }
    return nullptr;
  }
  if (kind != 1) return "unknown interpolation scheme";
  if (m < 1 || m > 3 || m > n - 2) return "LalescuSpline's smoothness must lie in [1, min(3, n − 2)]";
  const int D = 2 * m + 1;   // Hermite degree
  // d[e][k][j]: the k-th derivative at end e (t = 0, 1) of the (n − 1)-point Lagrange polynomial
  // centred there, as weights on the taps
  double dk[2][4][kStencilMax] = {};
  for (int e = 0; e < 2; ++e) {
    const int np = n - 1, half = (np - 1) / 2;
    for (int i = 0; i < np; ++i) {
      const int si = i - half;   // point relative to the end
      double p[kStencilMax + 1] = {1.0};
      int deg = 0;
      for (int q = 0; q < np; ++q) {
        if (q == i) continue;
        mul_lin(p, deg, double(q - half), double(si - (q - half)));
        ++deg;
      }
      const int tap = e + si + off;   // stencil tap of point si about end e
      double fact = 1.0;
      for (int k = 0; k <= m; ++k) {
        if (k > 0) fact *= k;
        dk[e][k][tap] += fact * p[k];
      }
    }
  }
  // the Hermite basis: H[e][k](t) of degree D with H^(l)(e') = δ(e, e')·δ(k, l), l ≤ m
  double Amat[8][9];
  double H[2][4][8] = {};
  for (int e = 0; e < 2; ++e)
    for (int k = 0; k <= m; ++k) {
      // rows: the conditions (end e', derivative l); columns: monomials t^d, d ≤ D; last column rhs
      for (int ee = 0; ee < 2; ++ee)
        for (int l = 0; l <= m; ++l) {
          const int row = ee * (m + 1) + l;
          for (int d = 0; d <= D; ++d) {
            double v = 0.0;
            if (d >= l) {
              double f = 1.0;
              for (int r = 0; r < l; ++r) f *= double(d - r);
              v = ee == 0 ? (d == l ? f : 0.0) : f;   // d^l/dt^l t^d at 0 or 1
            }
            Amat[row][d] = v;
          }
          Amat[row][D + 1] = (ee == e && l == k) ? 1.0 : 0.0;
        }
      const int R = D + 1;
      for (int col = 0; col < R; ++col) {   // Gauss–Jordan with partial pivoting
        int piv = col;
        for (int r = col + 1; r < R; ++r)
          if (std::fabs(Amat[r][col]) > std::fabs(Amat[piv][col])) piv = r;
        for (int q = 0; q <= R; ++q) std::swap(Amat[col][q], Amat[piv][q]);
        for (int r = 0; r < R; ++r) {
          if (r == col) continue;
          const double fct = Amat[r][col] / Amat[col][col];
          for (int q = col; q <= R; ++q) Amat[r][q] -= fct * Amat[col][q];
        }
      }
      for (int d = 0; d <= D; ++d) H[e][k][d] = Amat[d][R] / Amat[d][d];
    }
  s->n = n;
  s->deg = D;
  for (int j = 0; j < n; ++j)
    for (int d = 0; d <= D; ++d) {
      double v = 0.0;
      for (int e = 0; e < 2; ++e)
        for (int k = 0; k <= m; ++k) v += dk[e][k][j] * H[e][k][d];
      s->c[j][d] = v;
    }
  return nullptr;
}

// Traversal order (src/Particles.jl:220-271): tracers are visited tile by tile, in tiles of 8³
// cells, so the 64-point gathers of neighbouring threads share cache lines. Only the visiting
// order changes; every tracer's arithmetic is the same. The key is the tile of the cell that
// cell_fraction gives the position.
GBGHT_HD int traversal_tiles(int N) { return (N + 7) / 8; }
GBGHT_HD uint32_t traversal_key(const double* GBGHT_RESTRICT X, int64_t p, int64_t M, int N, double dx) {
  int i[3];
  for (int c = 0; c < 3; ++c) {
    double t;
    cell_fraction(X[c * M + p], dx, N, i[c], t);
  }
  const uint32_t T = uint32_t(traversal_tiles(N));
  return (uint32_t(i[2] >> 3) * T + uint32_t(i[1] >> 3)) * T + uint32_t(i[0] >> 3);
}

// One step of the Adams family for every tracer (src/ParticlePropagator.jl:282-307): the
// predictor X* = X + Σ_j b_j f_{n−j} over J samples of the trail, and, when corrected (ABM),
// X ← X* + β*·f* + Σ_j (β_{j+1} − b_j) f_{n−j} with f* gathered at X*. J = 0 moves nothing.
// The trail is a ring of sample slots [slot][3][M]; out_slot ≥ 0 receives the sample at the new
// positions (the closing particle deposit, or a gather alone when J = 0).
constexpr int kTrailMax = 8;
struct AdamsStep {
  int J;                    // samples the predictor integrates over (0: no push)
  int corrected;            // gather f* at X* and correct
  int out_slot;             // slot of the sample at the new positions; −1: none
  int slot[kTrailMax];      // ring slot of f_{n−j}, j = 0 the newest
  double b[kTrailMax];      // predictor weights
  double beta_star;         // corrector weight on f*
  double beta_m[kTrailMax]; // corrector weights β_{j+1} − b_j
  Stencil stencil;          // the interpolation scheme's weights (n = 0: Catmull–Rom)
};

// One tracer. X is [3][M]; F is the trail's slots, 3·M doubles apart. Each displacement is summed
// term by term in the weights' order, then added, and the position wrapped into [0, L).
// gather(x, y, z, out) interpolates the field; only a caller with `writes` stores (the
// warp-cooperative form runs the tracer's scalar arithmetic on every lane of its group).
template <class G>
GBGHT_HD void tracer_step(int64_t p, int64_t M, double L, double* GBGHT_RESTRICT X, double* GBGHT_RESTRICT F,
                          const AdamsStep& w, const G& gather, bool writes) {
  const size_t S3 = 3 * size_t(M);
  double x[3] = {X[p], X[M + p], X[2 * M + p]};
  if (w.J > 0) {
    double disp[3];
    for (int c = 0; c < 3; ++c) disp[c] = mul_rn(w.b[0], F[size_t(w.slot[0]) * S3 + size_t(c) * M + p]);
    for (int j = 1; j < w.J; ++j)
      for (int c = 0; c < 3; ++c)
        disp[c] = add_rn(disp[c], mul_rn(w.b[j], F[size_t(w.slot[j]) * S3 + size_t(c) * M + p]));
    double xs[3];
    for (int c = 0; c < 3; ++c) xs[c] = wrap_periodic(add_rn(x[c], disp[c]), L);
    if (w.corrected) {
      double fs[3];
      gather(xs[0], xs[1], xs[2], fs);
      for (int c = 0; c < 3; ++c) disp[c] = mul_rn(w.beta_star, fs[c]);
      for (int j = 0; j < w.J; ++j)
        for (int c = 0; c < 3; ++c)
          disp[c] = add_rn(disp[c], mul_rn(w.beta_m[j], F[size_t(w.slot[j]) * S3 + size_t(c) * M + p]));
      for (int c = 0; c < 3; ++c) x[c] = wrap_periodic(add_rn(xs[c], disp[c]), L);
    } else {
      for (int c = 0; c < 3; ++c) x[c] = xs[c];
    }
    if (writes)
      for (int c = 0; c < 3; ++c) X[c * M + p] = x[c];
  }
  if (w.out_slot < 0) return;
  double f[3];
  gather(x[0], x[1], x[2], f);
  if (writes)
    for (int c = 0; c < 3; ++c) F[size_t(w.out_slot) * S3 + size_t(c) * M + p] = f[c];
}
template <class T>
GBGHT_HD void tracer_one(int64_t p, int64_t M, const T* GBGHT_RESTRICT u, int N, double L,
                         double* GBGHT_RESTRICT X, double* GBGHT_RESTRICT F, const AdamsStep& w) {
  const double dx = div_rn(L, double(N));
  tracer_step(p, M, L, X, F, w,
              [&](double x, double y, double z, double* out) { gather_any(u, N, dx, x, y, z, w.stencil, out); }, true);
}

#if defined(__CUDACC__) && !defined(GBGHT_EMU)
// The warp-cooperative tracer step: a group of 16 lanes per tracer. Lane a < 3 carries the
// tracer's coordinate a through the Adams sums and the wrap, and takes axis a's cell and
// Catmull–Rom weights; the group reads them by shuffles. Lane (cz, cy) = (sub / 4, sub mod 4) sums
// the x taps of its (z, y) row for the three components, the lanes cy = 0 take the y sums over their
// four rows and lane 0 the z sums. Every operation is the per-tracer path's (tracer_one, gather3),
// on the same values in the same order with the same roundings, so the results are bit for bit
// those of k_tracers. All 32 lanes of the warp run it (a group past M runs tracer 0 and stores
// nothing).
constexpr unsigned kFullWarp = 0xffffffffu;
template <class T>
__device__ __forceinline__ double gather3_group(const T* GBGHT_RESTRICT u, int N, double dx, double xa, int sub) {
  int i = 0;
  double w[4] = {0.0, 0.0, 0.0, 0.0};
  if (sub < 3) {
    double t;
    cell_fraction(xa, dx, N, i, t);
    catmull_rom(t, w);
  }
  const int ix = __shfl_sync(kFullWarp, i, 0, 16), iy = __shfl_sync(kFullWarp, i, 1, 16),
            iz = __shfl_sync(kFullWarp, i, 2, 16);
  double wx[4], wy[4], wz[4];
  for (int a = 0; a < 4; ++a) {
    wx[a] = __shfl_sync(kFullWarp, w[a], 0, 16);
    wy[a] = __shfl_sync(kFullWarp, w[a], 1, 16);
    wz[a] = __shfl_sync(kFullWarp, w[a], 2, 16);
  }
  const int cz = sub >> 2, cy = sub & 3;
  const int zz = (iz + cz - 1 + N) % N, yy = (iy + cy - 1 + N) % N;
  const size_t comp = size_t(N) * N * N;
  double f[3];
  for (int c = 0; c < 3; ++c) {
    const T* row = u + c * comp + (size_t(zz) * N + yy) * N;
    double tap[4];
    row_taps(row, ix, N, tap);
    double acc_x = 0.0;
    for (int cx = 0; cx < 4; ++cx) acc_x = add_rn(acc_x, mul_rn(wx[cx], tap[cx]));
    const double x1 = __shfl_down_sync(kFullWarp, acc_x, 1, 16);
    const double x2 = __shfl_down_sync(kFullWarp, acc_x, 2, 16);
    const double x3 = __shfl_down_sync(kFullWarp, acc_x, 3, 16);
    double acc_y = 0.0;
    acc_y = add_rn(acc_y, mul_rn(wy[0], acc_x));
    acc_y = add_rn(acc_y, mul_rn(wy[1], x1));
    acc_y = add_rn(acc_y, mul_rn(wy[2], x2));
    acc_y = add_rn(acc_y, mul_rn(wy[3], x3));
    const double y1 = __shfl_down_sync(kFullWarp, acc_y, 4, 16);
    const double y2 = __shfl_down_sync(kFullWarp, acc_y, 8, 16);
    const double y3 = __shfl_down_sync(kFullWarp, acc_y, 12, 16);
    double acc_z = 0.0;
    acc_z = add_rn(acc_z, mul_rn(wz[0], acc_y));
    acc_z = add_rn(acc_z, mul_rn(wz[1], y1));
    acc_z = add_rn(acc_z, mul_rn(wz[2], y2));
    acc_z = add_rn(acc_z, mul_rn(wz[3], y3));
    f[c] = __shfl_sync(kFullWarp, acc_z, 0, 16);
  }
  return sub == 1 ? f[1] : sub == 2 ? f[2] : f[0];   // lane a < 3: component a
}
template <class T>
__device__ __forceinline__ void tracer_group(int64_t p, int64_t M, const T* GBGHT_RESTRICT u, int N, double L,
                                             double* GBGHT_RESTRICT X, double* GBGHT_RESTRICT F, const AdamsStep& w,
                                             int sub, bool live) {
  const double dx = div_rn(L, double(N));
  const size_t S3 = 3 * size_t(M);
  const int c = sub < 3 ? sub : 0;   // lanes 3..15 repeat coordinate 0 and store nothing
  const bool store = live && sub < 3;
  double x = X[c * M + p];
  if (w.J > 0) {
    double disp = mul_rn(w.b[0], F[size_t(w.slot[0]) * S3 + size_t(c) * M + p]);
    for (int j = 1; j < w.J; ++j) disp = add_rn(disp, mul_rn(w.b[j], F[size_t(w.slot[j]) * S3 + size_t(c) * M + p]));
    const double xs = wrap_periodic(add_rn(x, disp), L);
    if (w.corrected) {
      const double fs = gather3_group(u, N, dx, xs, sub);
      disp = mul_rn(w.beta_star, fs);
      for (int j = 0; j < w.J; ++j)
        disp = add_rn(disp, mul_rn(w.beta_m[j], F[size_t(w.slot[j]) * S3 + size_t(c) * M + p]));
      x = wrap_periodic(add_rn(xs, disp), L);
    } else {
      x = xs;
    }
    if (store) X[c * M + p] = x;
  }
  if (w.out_slot < 0) return;
  const double f = gather3_group(u, N, dx, x, sub);
  if (store) F[size_t(w.out_slot) * S3 + size_t(c) * M + p] = f;
}
#endif

// 4-point Gauss–Legendre Adams weights (src/ParticlePropagator.jl:263-280), host side.
inline void adams_weights(const double* nodes, int n, double h, double* out) {
  static const double gn[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563,
                               0.8611363115940526};
  static const double gw[4] = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461,
                               0.3478548451374538};
  for (int j = 0; j < n; ++j) {
    double weight = 0.0;
    for (int k = 0; k < 4; ++k) {
      const double t = h * (gn[k] + 1) / 2;
      double basis = 1.0;
      for (int m = 0; m < n; ++m) {
        if (m == j) continue;
        basis *= (t - nodes[m]) / (nodes[j] - nodes[m]);
      }
      weight += gw[k] * h / 2 * basis;
    }
    out[j] = weight;
  }
}

// The step's weights from the trail's sample times (newest first, at most kTrailMax): the
// predictor through the nodes t_{n−j} − t_n, the corrector through (h, nodes…).
inline void adams_step_weights(const double* times, int J, double h, bool corrected, AdamsStep* w) {
  double nodes[kTrailMax + 1];
  for (int j = 0; j < J; ++j) nodes[j] = times[j] - times[0];
  adams_weights(nodes, J, h, w->b);
  w->J = J;
  w->corrected = corrected ? 1 : 0;
  if (!corrected) return;
  double with_end[kTrailMax + 1], beta[kTrailMax + 1];
  with_end[0] = h;
  for (int j = 0; j < J; ++j) with_end[j + 1] = nodes[j];
  adams_weights(with_end, J + 1, h, beta);
  w->beta_star = beta[0];
  for (int j = 0; j < J; ++j) w->beta_m[j] = beta[j + 1] - w->b[j];
}

}  // namespace gbght
