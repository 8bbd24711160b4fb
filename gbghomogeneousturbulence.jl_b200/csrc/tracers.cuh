// Lagrangian tracers: periodic wrap, Catmull–Rom gather, and the Heun (= ABM(1)) push.
//
// Positions are FP64 in both precision forms. The wrap and the displacement are evaluated with
// round-to-nearest operations and no fused multiply-add, in the order the reference's update
// reads (src/ParticlePropagator.jl:288-315), so a cell index floor(x/Δx) is reproducible.
#pragma once

#include "gbght_common.cuh"

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
  int xs[4], ys[4], zs[4];
  for (int a = 0; a < 4; ++a) {
    xs[a] = (ix + a - 1 + N) % N;
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
        double acc_x = 0.0;
        for (int cx = 0; cx < 4; ++cx) acc_x = add_rn(acc_x, mul_rn(wx[cx], double(ldg(row + xs[cx]))));
        acc_y = add_rn(acc_y, mul_rn(wy[cy], acc_x));
      }
      acc_z = add_rn(acc_z, mul_rn(wz[cz], acc_y));
    }
    out[c] = acc_z;
  }
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
};

// One tracer. X is [3][M]; F is the trail's slots, 3·M doubles apart. Each displacement is summed
// term by term in the weights' order, then added, and the position wrapped into [0, L).
template <class T>
GBGHT_HD void tracer_one(int64_t p, int64_t M, const T* GBGHT_RESTRICT u, int N, double L,
                         double* GBGHT_RESTRICT X, double* GBGHT_RESTRICT F, const AdamsStep& w) {
  const double dx = div_rn(L, double(N));
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
      gather3(u, N, dx, xs[0], xs[1], xs[2], fs);
      for (int c = 0; c < 3; ++c) disp[c] = mul_rn(w.beta_star, fs[c]);
      for (int j = 0; j < w.J; ++j)
        for (int c = 0; c < 3; ++c)
          disp[c] = add_rn(disp[c], mul_rn(w.beta_m[j], F[size_t(w.slot[j]) * S3 + size_t(c) * M + p]));
      for (int c = 0; c < 3; ++c) x[c] = wrap_periodic(add_rn(xs[c], disp[c]), L);
    } else {
      for (int c = 0; c < 3; ++c) x[c] = xs[c];
    }
    for (int c = 0; c < 3; ++c) X[c * M + p] = x[c];
  }
  if (w.out_slot < 0) return;
  double f[3];
  gather3(u, N, dx, x[0], x[1], x[2], f);
  for (int c = 0; c < 3; ++c) F[size_t(w.out_slot) * S3 + size_t(c) * M + p] = f[c];
}

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
