// The discrete adjoint of one low-storage IF-RK step (IFLowStorageRK4 / RK3), as CTA bodies.
//
// The reference has no AD; the step it differentiates is `_low_storage_2n_step!`
// (src/Propagator.jl:326-419) with the generator's verbs `velocity_rhs!` / `scalar_rhs!`
// (src/Generator.jl:484-534,648-730) and the ConstantPower source (src/Forcing.jl:1091-1117). The
// adjoint is taken for the inner products ⟨a, b⟩ = Σ_x a·b (physical) and Σ w·Re(conj(x)·y)
// (spectral, w the Hermitian weights), under which irfft* = rfft/N³, rfft* = N³·irfft, and ℙ, the
// mask, the curl iκ×, the integrating factor and the reality projection are self-adjoint. For
// n = u×ω the adjoint sends n̄ to ū = ω×n̄ and ω̄ = n̄×u; for f = uφ it sends f̄ to ū = φf̄ and
// φ̄ = f̄·u. The state lives on the retained 2/3 ball, so every adjoint field is restricted to it.
//
// Reverse stage i of S, with λ the adjoint of the stage's output state and λ_h of its register:
//   prologue   λ_v = E_i λ,  λ_h = b_i λ_v + E_i (a_{i+1} λ_h'),  λ_N = Δt λ_h
//              sources: m̂ = ℙ𝔻 λ_N (κ = 0 zeroed), f̂_c = i𝔻κ_c λ_Nφ
//   x pass     m = N³·irfft(m̂), f = N³·irfft(f̂); ū = ω×m + φf, ω̄ = m×u, φ̄ = f·u
//   combine    λ ← λ_v + rfft(ū)/N³ + iκ×rfft(ω̄)/N³ + A·𝟙λ_N + c·𝟙q_i − G λ_Nφ
//              λ_φ ← λ_vφ + rfft(φ̄)/N³ + A_φ·𝟙λ_Nφ + c_φ·𝟙p_i
// with u, ω, φ the stage's forward fields (recomputed from the saved stage state q_i, p_i), and
// A, c the ConstantPower amplitude and its state derivative (c = ⟨𝟙q_i, λ_N⟩·(−4·c_f·A²/ε), c_f = ½
// for the velocity and 1 for the scalar). The combine of stage i and the prologue of stage i − 1
// run in one z pass, as the forward epilogue fuses the update with the next stage's inverse.
#pragma once

#include "passes.cuh"
#include "tracers.cuh"

namespace gbght {

// ================================================================================================
// The adjoint x pass: for P points (z, y0..y0+P−1), the c2r of the stage's forward fields (B slots
// 0..6 of `Bf`: u, ω, φ, scaled by 1/N³) and of the adjoint sources (slots 0..5 of `Ba`: m, f,
// unscaled), the products ū = ω×m + φf, ω̄ = m×u, φ̄ = f·u, and the r2c of the seven products into
// slots 0..6 of `Ba` (scaled by 1/N³), in place. One warp per line, as the forward x pass.
//   inverse lines (per point p): 6p+0 = u_x + i·u_y, 6p+1 = u_z + i·ω_x, 6p+2 = ω_y + i·ω_z,
//            6p+3 = m_x + i·m_y, 6p+4 = m_z + i·f_x, 6p+5 = f_y + i·f_z; and 6P + h = φ(2h) + i·φ(2h+1)
//   forward lines: 3p+0 = ū_x + i·ū_y, 3p+1 = ū_z + i·ω̄_x, 3p+2 = ω̄_y + i·ω̄_z, 3P + h = φ̄(2h) + i·φ̄(2h+1)
// The first inverse stage reads the half spectra straight from global memory (two for one, a c2r
// input: only the real part of a kx = 0 bin enters, rows K < e < N−K are zero).
// ================================================================================================
template <class T> struct XAdjShape {
  static constexpr int P = XShape<T>::P;          // points per tile: 2 (FP64), 4 (FP32)
  static constexpr int NIN = 6 * P + P / 2;       // inverse lines
  static constexpr int NOUT = 3 * P + P / 2;      // forward lines
  static constexpr int NW = 8;                    // warps per CTA
};

template <class T, int N>
struct XAdjSource {
  static constexpr bool kExternal = true;
  const Geometry& g;
  const Cplx<T>* Bf;   // forward fields, B layout
  const Cplx<T>* Ba;   // adjoint sources, B layout
  int z, y0, has_scalar;
  T scf;               // 1/N³ for the forward fields
  GBGHT_HD Cplx<T> load(int e, int l) const {
    constexpr int P = XAdjShape<T>::P;
    const int K = g.K;
    if (e > K && e < N - K) return czero<T>();
    const Cplx<T>* base;
    int ca, cb, pa, pb;
    T sc;
    if (l < 6 * P) {
      const int p = l / 6, pr = l % 6;
      pa = pb = p;
      if (pr < 3) {
        base = Bf;
        ca = 2 * pr;
        cb = ca + 1;
        sc = scf;
      } else {
        base = Ba;
        ca = 2 * (pr - 3);
        cb = ca + 1;
        sc = T(1);
        if (!has_scalar && ca >= 2) {   // no scalar: the f lines are zero (m_z stays)
          if (ca == 2) {
            const int m = e <= K ? e : N - e;
            const Cplx<T> a = Ba[idxB(g, 2, z, y0 + p, m)];
            if (e == 0) return cmk<T>(a.x, T(0));
            if (e <= K) return a;
            return conj(a);
          }
          return czero<T>();
        }
      }
    } else {
      if (!has_scalar) return czero<T>();
      const int h = l - 6 * P;
      base = Bf;
      ca = cb = 6;
      pa = 2 * h;
      pb = 2 * h + 1;
      sc = scf;
    }
    const int m = e <= K ? e : N - e;
    const Cplx<T> a = base[idxB(g, ca, z, y0 + pa, m)], b = base[idxB(g, cb, z, y0 + pb, m)];
    if (e == 0) return cmk<T>(a.x * sc, b.x * sc);
    if (e <= K) return cmk<T>((a.x - b.y) * sc, (a.y + b.x) * sc);
    return cmk<T>((a.x + b.y) * sc, (b.x - a.y) * sc);
  }
};

// One adjoint x tile.
template <class T, int N, int NT>
GBGHT_HD void x_adjoint_tile(const Cta& c, Cplx<T>* sm, const Geometry& g, const Cplx<T>* GBGHT_RESTRICT Bf,
                             Cplx<T>* Ba, int has_scalar, int z, int y0, const Cplx<T>* GBGHT_RESTRICT tw) {
  using X = XAdjShape<T>;
  constexpr int P = X::P, NW = X::NW;
  const XAdjSource<T, N> src{g, Bf, Ba, z, y0, has_scalar, T(g.inv_norm)};
  const auto lines = [&](int l) { return sm + l * N; };
  const auto from_src = [&](int l) { return LineOfSource<XAdjSource<T, N>>{src, l}; };
  const auto in_smem = [&](int l) { return LineBuf<T>{sm + l * N}; };
  warp_fft_lines<T, N, NW, NT, +1>(c, X::NIN, lines, from_src, in_smem, tw);
  GBGHT_SYNC();
  // the products at every x; all loads of a point set come before its stores, and each x belongs
  // to one thread
  for (int x = c.tid; x < N; x += NT) {
    const int ix = lidx<T>(x);
    Cplx<T> o[3 * P];
    T ph_out[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const Cplx<T> L0 = sm[(6 * p) * N + ix], L1 = sm[(6 * p + 1) * N + ix], L2 = sm[(6 * p + 2) * N + ix];
      const Cplx<T> L3 = sm[(6 * p + 3) * N + ix], L4 = sm[(6 * p + 4) * N + ix], L5 = sm[(6 * p + 5) * N + ix];
      const Cplx<T> lp = sm[(6 * P + p / 2) * N + ix];
      const T ux = L0.x, uy = L0.y, uz = L1.x, wx = L1.y, wy = L2.x, wz = L2.y;
      const T mx = L3.x, my = L3.y, mz = L4.x, fx = L4.y, fy = L5.x, fz = L5.y;
      const T phi = (p & 1) ? lp.y : lp.x;
      // ū = ω×m + φf, ω̄ = m×u, φ̄ = f·u
      const T bx = (wy * mz - wz * my) + phi * fx, by = (wz * mx - wx * mz) + phi * fy, bz = (wx * my - wy * mx) + phi * fz;
      const T cx = my * uz - mz * uy, cy = mz * ux - mx * uz, cz = mx * uy - my * ux;
      o[3 * p] = cmk<T>(bx, by);
      o[3 * p + 1] = cmk<T>(bz, cx);
      o[3 * p + 2] = cmk<T>(cy, cz);
      ph_out[p] = (fx * ux + fy * uy) + fz * uz;
    }
#pragma unroll
    for (int k = 0; k < 3 * P; ++k) sm[k * N + ix] = o[k];
#pragma unroll
    for (int h = 0; h < P / 2; ++h) sm[(3 * P + h) * N + ix] = cmk<T>(ph_out[2 * h], ph_out[2 * h + 1]);
  }
  GBGHT_SYNC();
  warp_fft_lines<T, N, NW, NT, -1>(c, X::NOUT, lines, in_smem, in_smem, tw);
  GBGHT_SYNC();
  // unpack: line 3p+pr → slots (2pr, 2pr+1) of point p; line 3P+h → slot 6 of points 2h, 2h+1;
  // scaled by 1/N³; columns past K get zeros
  const int KX1 = g.K + 1;
  const T sc = T(g.inv_norm);
  for (int t = c.tid; t < 32 * NW; t += NT) {
    const int w = t >> 5, lane = t & 31;
    for (int line = w; line < X::NOUT; line += NW) {
      int ca, cb, pa, pb;
      if (line < 3 * P) {
        pa = pb = line / 3;
        ca = 2 * (line % 3);
        cb = ca + 1;
      } else {
        ca = cb = 6;
        pa = 2 * (line - 3 * P);
        pb = pa + 1;
      }
      const Cplx<T>* L = sm + line * N;
      for (int k = lane; k < g.KXP; k += 32) {
        Cplx<T> a = czero<T>(), b = czero<T>();
        if (k < KX1) {
          const Cplx<T> zk = L[lidx<T>(k)];
          const Cplx<T> zc = conj(L[lidx<T>((N - k) % N)]);
          const Cplx<T> sp = zk + zc, sd = zk - zc;
          a = cmk<T>(sp.x * T(0.5) * sc, sp.y * T(0.5) * sc);
          b = cmk<T>(sd.y * T(0.5) * sc, -sd.x * T(0.5) * sc);
        }
        if (ca < 6 || has_scalar) {
          Ba[idxB(g, ca, z, y0 + pa, k)] = a;
          Ba[idxB(g, cb, z, y0 + pb, k)] = b;
        }
      }
    }
  }
  GBGHT_SYNC();   // the lines are rewritten by the next tile
}

// The adjoint x pass: tile bx of the (N/P)·N tiles, one per CTA (a loop over tiles inside the
// CTA keeps the tile's index arithmetic live and spills).
template <class T, int N, int NT>
GBGHT_HD void body_x_adjoint(const Cta& c, Cplx<T>* sm, const Geometry& g, const Cplx<T>* GBGHT_RESTRICT Bf,
                             Cplx<T>* Ba, int has_scalar, const Cplx<T>* GBGHT_RESTRICT tw) {
  constexpr int P = XAdjShape<T>::P;
  const int tiles_y = N / P;
  x_adjoint_tile<T, N, NT>(c, sm, g, Bf, Ba, has_scalar, c.bx / tiles_y, P * (c.bx % tiles_y), tw);
}

// ================================================================================================
// The adjoint z pass, one tile (ky' = qy, kx0..kx0+TL) per CTA, grid (KXP/TL, NY2): the combine of
// reverse stage i (z-forward of the x pass's products, the per-mode update of λ), then the prologue
// of reverse stage j (λ_v, λ_h into L and LH, the sources m̂, f̂ z-inverse transformed into A slots
// 0..5). At the start of the reverse pass (`start`), L holds λ of the step's output (after the
// reality projection, its own adjoint) and the combine is replaced by the Leray projection.
// Shared memory: the FFT tile W (N·TL) and the retained rows R ([6][NY2][TL]).
// ================================================================================================
struct AdjArgs {
  int add_only;         // the launch adds the z-forward of A slots 0..2 to λ's velocity (nothing else)
  int combine;          // the launch ends reverse stage i
  int prologue;         // the launch starts reverse stage j
  int has_scalar;
  double dt;
  double G[3];          // mean scalar gradient
  int forced, sforced;  // ConstantPower on the velocity, on the scalar (stage i's A and c in coef)
  double band_lo2, band_hi2, sband_lo2, sband_hi2;   // the fields' forcing bands (squared edges)
  double cu, cphi, lin_u, lin_phi;                   // stage j's factor exp(c·|κ|² + lin·𝟙band)
  double b;             // b_j
  double a_next;        // a_i: the register carried into stage j is a_i·λ_h (0 at the start)
};

// z-forward sink: the retained rows of the transform into R component `comp` (added with `add`).
template <class T, int N, int TL>
struct ZRetainedSink {
  const Geometry& g;
  Cplx<T>* R;
  int comp;
  bool add;
  GBGHT_HD void store(int e, int l, Cplx<T> v) const {
    int q = -1;
    if (e <= g.K) q = e;
    else if (e >= N - g.K) q = e - N + g.NY2;
    if (q < 0) return;
    Cplx<T>& r = R[(size_t(comp) * g.NY2 + q) * TL + l];
    r = add ? r + v : v;
  }
};
// z-inverse source: the retained rows of R component `comp`, zero elsewhere.
template <class T, int N, int TL>
struct ZRetainedSource {
  static constexpr bool kExternal = true;
  const Geometry& g;
  const Cplx<T>* R;
  int comp;
  GBGHT_HD Cplx<T> load(int e, int l) const {
    int q = -1;
    if (e <= g.K) q = e;
    else if (e >= N - g.K) q = e - N + g.NY2;
    return q < 0 ? czero<T>() : R[(size_t(comp) * g.NY2 + q) * TL + l];
  }
};
// Leray projection ℙ(κ)v = v − κ(κ·v)/|κ|², the identity at κ = 0 (the forward epilogue's form).
template <class T>
GBGHT_HD void leray3(Cplx<T>* v, double kxd, double kyd, double kzd, double k2) {
  if (!(k2 > 0.0)) return;
  const T kX = T(kxd), kY = T(kyd), kZ = T(kzd), ik2 = T(1.0 / k2);
  const Cplx<T> kd = cmk<T>((kX * v[0].x + kY * v[1].x + kZ * v[2].x) * ik2, (kX * v[0].y + kY * v[1].y + kZ * v[2].y) * ik2);
  v[0] = v[0] - scale(kd, kX);
  v[1] = v[1] - scale(kd, kY);
  v[2] = v[2] - scale(kd, kZ);
}

// L, LH: λ and λ_h (S layout, 4 components); Q: stage i's saved state (S layout); coef = (A, c,
// A_φ, c_φ) of stage i's ConstantPower sources; Aa: the adjoint A slots (read 0..6 at a combine,
// written 0..5 at a prologue).
template <class T, int N, int TL, int NT>
GBGHT_HD void body_adj_z(const Cta& c, Cplx<T>* W, Cplx<T>* R, const Geometry& g, const AdjArgs& a,
                         Cplx<T>* GBGHT_RESTRICT Aa, Cplx<T>* GBGHT_RESTRICT L, Cplx<T>* GBGHT_RESTRICT LH,
                         const Cplx<T>* GBGHT_RESTRICT Q, const double* GBGHT_RESTRICT coef,
                         const Cplx<T>* GBGHT_RESTRICT tw) {
  const int kx0 = c.bx * TL, qy = c.by, NY2 = g.NY2;
  const double s = g.s;
  const double ky = s * double(q_to_m(qy, g.K, NY2));
  const auto Rat = [&](int comp, int q, int l) -> Cplx<T>& { return R[(size_t(comp) * NY2 + q) * TL + l]; };
  const auto zfwd = [&](int slot, int comp, bool add) {
    const ZGlobalSource<T, N, TL> src{g, Aa, slot, qy, kx0};
    const ZRetainedSink<T, N, TL> dst{g, R, comp, add};
    tile_fft_io<T, N, TL, NT, -1>(c, W, tw, src, dst);
  };
  if (a.add_only) {   // λ_u += the z-forward of A slots 0..2 on the ball (the tracers' part)
    for (int k = 0; k < 3; ++k) zfwd(k, k, false);
    for (int idx = c.tid; idx < NY2 * TL; idx += NT) {
      const int q = idx / TL, l = idx % TL, kx = kx0 + l;
      const double kxd = s * double(kx), kzd = s * double(q_to_m(q, g.K, NY2));
      const double k2 = (kxd * kxd + ky * ky) + kzd * kzd;
      if (!(kx <= g.K && k2 <= g.cut2)) continue;
      for (int cc = 0; cc < 3; ++cc) {
        const size_t at = idxS(g, cc, qy, q, kx);
        L[at] = L[at] + Rat(cc, q, l);
      }
    }
    return;
  }
  if (a.combine) {
    // ω̄ (slots 3..5), its curl in place, then + ū (slots 0..2); φ̄ (slot 6) into component 3
    for (int k = 0; k < 3; ++k) zfwd(3 + k, k, false);
    for (int idx = c.tid; idx < NY2 * TL; idx += NT) {
      const int q = idx / TL, l = idx % TL;
      const T kX = T(s * double(kx0 + l)), kY = T(ky), kZ = T(s * double(q_to_m(q, g.K, NY2)));
      const Cplx<T> f0 = Rat(0, q, l), f1 = Rat(1, q, l), f2 = Rat(2, q, l);
      for (int o = 0; o < 3; ++o) Rat(o, q, l) = curl_of<T>(o, f0, f1, f2, kX, kY, kZ);
    }
    GBGHT_SYNC();
    for (int k = 0; k < 3; ++k) zfwd(k, k, true);
    if (a.has_scalar) zfwd(6, 3, false);
  }
  const double A_u = a.forced ? coef[0] : 0.0, c_u = a.forced ? coef[1] : 0.0;
  const double A_p = a.sforced ? coef[2] : 0.0, c_p = a.sforced ? coef[3] : 0.0;
  const T dt = T(a.dt);
  const int nc = a.has_scalar ? 4 : 3;
  for (int idx = c.tid; idx < NY2 * TL; idx += NT) {
    const int q = idx / TL, l = idx % TL, kx = kx0 + l;
    const double kxd = s * double(kx), kzd = s * double(q_to_m(q, g.K, NY2));
    const double k2 = (kxd * kxd + ky * ky) + kzd * kzd;
    const bool ret = kx <= g.K && k2 <= g.cut2;
    const bool vband = k2 >= a.band_lo2 && k2 <= a.band_hi2;
    const bool sband = k2 >= a.sband_lo2 && k2 <= a.sband_hi2;
    Cplx<T> lq[4], lh[4];
    for (int cc = 0; cc < 4; ++cc) {
      lq[cc] = czero<T>();
      lh[cc] = czero<T>();
    }
    if (ret) {
      for (int cc = 0; cc < nc; ++cc) lq[cc] = L[idxS(g, cc, qy, q, kx)];
      if (a.combine) {
        for (int cc = 0; cc < nc; ++cc) lh[cc] = LH[idxS(g, cc, qy, q, kx)];
        // λ ← λ_v + rfft(ū)/N³ + iκ×rfft(ω̄)/N³ (+ the band source's adjoint) − G λ_Nφ
        for (int cc = 0; cc < 3; ++cc) lq[cc] = lq[cc] + Rat(cc, q, l);
        if (A_u != 0.0 && vband)
          for (int cc = 0; cc < 3; ++cc)
            lq[cc] = lq[cc] + scale(scale(lh[cc], dt), T(A_u)) + scale(Q[idxS(g, cc, qy, q, kx)], T(c_u));
        if (a.has_scalar) {
          const Cplx<T> lnp = scale(lh[3], dt);
          for (int cc = 0; cc < 3; ++cc) lq[cc] = lq[cc] - scale(lnp, T(a.G[cc]));
          lq[3] = lq[3] + Rat(3, q, l);
          if (A_p != 0.0 && sband) lq[3] = lq[3] + scale(lnp, T(A_p)) + scale(Q[idxS(g, 3, qy, q, kx)], T(c_p));
        }
      } else {
        leray3<T>(lq, kxd, ky, kzd, k2);   // the end-of-step Leray projection's adjoint
      }
    }
    if (!a.prologue) {
      for (int cc = 0; cc < nc; ++cc) L[idxS(g, cc, qy, q, kx)] = lq[cc];
      continue;
    }
    // prologue of stage j: λ_v = E λ, λ_h = b λ_v + E (a_next λ_h)
    const T Eu = T(exp(a.cu * k2 + (vband ? a.lin_u : 0.0)));
    const T Ep = T(exp(a.cphi * k2 + (sband ? a.lin_phi : 0.0)));
    Cplx<T> src[6];
    for (int cc = 0; cc < nc; ++cc) {
      const T E = cc < 3 ? Eu : Ep;
      const Cplx<T> lv = scale(lq[cc], E);
      const Cplx<T> nh = scale(lv, T(a.b)) + scale(scale(lh[cc], T(a.a_next)), E);
      L[idxS(g, cc, qy, q, kx)] = ret ? lv : czero<T>();
      LH[idxS(g, cc, qy, q, kx)] = ret ? nh : czero<T>();
      lh[cc] = ret ? nh : czero<T>();
    }
    // sources: m̂ = ℙ λ_N with κ = 0 zeroed, f̂_c = iκ_c λ_Nφ (both on the ball)
    for (int cc = 0; cc < 3; ++cc) src[cc] = scale(lh[cc], dt);
    if (k2 > 0.0) leray3<T>(src, kxd, ky, kzd, k2);
    else src[0] = src[1] = src[2] = czero<T>();
    const Cplx<T> lnp = scale(lh[3], dt);
    src[3] = mul_i(scale(lnp, T(kxd)));
    src[4] = mul_i(scale(lnp, T(ky)));
    src[5] = mul_i(scale(lnp, T(kzd)));
    for (int cc = 0; cc < 6; ++cc) Rat(cc, q, l) = ret ? src[cc] : czero<T>();
  }
  GBGHT_SYNC();
  if (!a.prologue) return;
  const int nsrc = a.has_scalar ? 6 : 3;
  for (int k = 0; k < nsrc; ++k) {
    const ZRetainedSource<T, N, TL> src{g, R, k};
    const ZGlobalSink<T, N, TL> dst{g, Aa, k, qy, kx0};
    tile_fft_io<T, N, TL, NT, +1>(c, W, tw, src, dst);
  }
}

// ================================================================================================
// The ConstantPower source's adjoint coefficients of stage i. For a field f with amplitude
// A = ε/(2·c_f·⟨f, 𝟙f⟩) (saved by the forward pass; 0 for an empty band) and λ_N = Δt·λ_h:
//   c = ⟨𝟙f, λ_N⟩·(−4·c_f·A²/ε)   (the state derivative of A·𝟙f paired with λ_N),
//   ∂L/∂ε += (A/ε)·N⁶⟨𝟙f, λ_N⟩    (the forcing rate's gradient, in the unnormalised product),
// with ⟨a, b⟩ = Σ_band w·Re(conj(a)·b)/N⁶ over the box |m_a| ≤ mb. `band_pair_raw` is that sum
// before the division, over slots [c0, c0 + nc).
// ================================================================================================
GBGHT_HD int band_box_side(const Geometry& g, double hi2) {
  int mb = int(std::sqrt(hi2) / g.s) + 1;
  return mb > g.K ? g.K : mb;
}
template <class T>
GBGHT_HD double band_pair_term(const Geometry& g, const Cplx<T>* Q, const Cplx<T>* LH, int c0, int mb, double lo2,
                               double hi2, int i) {
  const int side = 2 * mb + 1;
  const int kx = i % (mb + 1), mz = (i / (mb + 1)) % side - mb, my = (i / ((mb + 1) * side)) % side - mb;
  const int cc = c0 + i / ((mb + 1) * side * side);
  const double kxd = g.s * kx, kyd = g.s * my, kzd = g.s * mz;
  const double k2 = (kxd * kxd + kyd * kyd) + kzd * kzd;
  if (!(k2 >= lo2 && k2 <= hi2 && k2 <= g.cut2)) return 0.0;
  const int qy = my >= 0 ? my : my + g.NY2, qz = mz >= 0 ? mz : mz + g.NY2;
  const size_t at = idxS(g, cc, qy, qz, kx);
  const Cplx<T> a = Q[at], b = LH[at];
  return (kx == 0 ? 1.0 : 2.0) * (double(a.x) * double(b.x) + double(a.y) * double(b.y));
}
// coef = (A_u, c_u, A_φ, c_φ) from the saved amplitudes amp = (A_u, A_φ); grad[0..1] += the
// forcing amplitudes' gradients. One field is done when its `eps` is nonzero.
struct AdjBandArgs {
  double dt, n6;
  double lo2, hi2, slo2, shi2;
  double eps_u, eps_p;   // ConstantPower ε of each field (0: not a ConstantPower field)
};
GBGHT_HD void adj_band_finish(const AdjBandArgs& a, const double* amp, double su, double sp, double* coef,
                              double* grad) {
  const double A_u = amp[0], A_p = amp[1];
  const double pu = a.dt * (su / a.n6), pp = a.dt * (sp / a.n6);
  coef[0] = a.eps_u != 0.0 ? A_u : 0.0;
  coef[1] = (a.eps_u != 0.0 && A_u != 0.0) ? pu * (-4.0 * 0.5 * A_u * A_u / a.eps_u) : 0.0;
  coef[2] = a.eps_p != 0.0 ? A_p : 0.0;
  coef[3] = (a.eps_p != 0.0 && A_p != 0.0) ? pp * (-4.0 * 1.0 * A_p * A_p / a.eps_p) : 0.0;
  // the rate's gradient pairs λ_N with ∂(A·𝟙f)/∂ε = (A/ε)·𝟙f in the unnormalised spectral product
  if (a.eps_u != 0.0 && A_u != 0.0) grad[0] += (A_u / a.eps_u) * (a.dt * su);
  if (a.eps_p != 0.0 && A_p != 0.0) grad[1] += (A_p / a.eps_p) * (a.dt * sp);
}

// λ += w_u·û (velocity) and λ_φ += w_φ·φ̂ at one compact mode i of the box (the gradient of a
// quadratic observable of the state: k has w_u = 1/N⁶, ⟨φ²⟩ has w_φ = 2/N⁶).
template <class T>
GBGHT_HD void adj_add_mode(size_t i, size_t nS, int nc, Cplx<T>* L, const Cplx<T>* S, double wu, double wp) {
  if (i >= nS) return;
  for (int cc = 0; cc < nc; ++cc) {
    const double w = cc < 3 ? wu : wp;
    if (w != 0.0) L[cc * nS + i] = L[cc * nS + i] + scale(S[cc * nS + i], T(w));
  }
}

// ================================================================================================
// The tracers' adjoint (src/ParticlePropagator.jl:288-315,378-386), Heun with Catmull–Rom. The wrap
// is locally the identity and a cell index locally constant, so the gather f(X) = Σ w(X)·u at the
// taps has the adjoint λ ↦ (scatter of w·λ onto the taps, Σ ∂w/∂X·(u·λ) per position).
//   particle deposit f = u(X):                 λ_u += Wᵀλ_f, λ_X += ∂_X(u·λ_f), λ_f ← 0
//   Heun push and closing deposit at step h:   X* = X + b₀f₀, f* = u(X*), X' = X* + β*f* + (β₀ − b₀)f₀,
//                                              f' = u(X'); given (λ_X', λ_f'), λ_u collects both
//                                              gathers' scatters and (λ_X, λ_f₀) replace (λ_X', λ_f').
// λ_u is a physical field [3][N³] in FP64, added to by atomics; its rfft/N³ on the ball then joins λ.
// ================================================================================================
// d/dt of the Catmull–Rom weights.
GBGHT_HD void catmull_rom_slopes(double t, double s[4]) {
  s[0] = ((-3.0 * t + 4.0) * t - 1.0) * 0.5;
  s[1] = (9.0 * t - 10.0) * t * 0.5;
  s[2] = ((-9.0 * t + 8.0) * t + 1.0) * 0.5;
  s[3] = (3.0 * t - 2.0) * t * 0.5;
}

GBGHT_HD void add_to(double* p, double v) {
#ifdef __CUDA_ARCH__
  atomicAdd(p, v);
#else
  *p += v;
#endif
}

// The gather's adjoint at (x, y, z) for values λ[3]: w·λ scattered into lu ([3][N³]); returns the
// positions' part in lX[3] (per unit length).
template <class T>
GBGHT_HD void gather3_adjoint(const T* GBGHT_RESTRICT u, double* lu, int N, double dx, double x, double y, double z,
                              const double lam[3], double lX[3]) {
  int ix, iy, iz;
  double tx, ty, tz;
  cell_fraction(x, dx, N, ix, tx);
  cell_fraction(y, dx, N, iy, ty);
  cell_fraction(z, dx, N, iz, tz);
  double wx[4], wy[4], wz[4], sx[4], sy[4], sz[4];
  catmull_rom(tx, wx);
  catmull_rom(ty, wy);
  catmull_rom(tz, wz);
  catmull_rom_slopes(tx, sx);
  catmull_rom_slopes(ty, sy);
  catmull_rom_slopes(tz, sz);
  const size_t comp = size_t(N) * N * N;
  lX[0] = lX[1] = lX[2] = 0.0;
  for (int cz = 0; cz < 4; ++cz) {
    const int zz = (iz + cz - 1 + N) % N;
    for (int cy = 0; cy < 4; ++cy) {
      const int yy = (iy + cy - 1 + N) % N;
      for (int cx = 0; cx < 4; ++cx) {
        const int xx = (ix + cx - 1 + N) % N;
        const size_t at = (size_t(zz) * N + yy) * N + xx;
        double fl = 0.0;
        for (int c = 0; c < 3; ++c) fl += double(ldg(u + c * comp + at)) * lam[c];
        lX[0] += sx[cx] * wy[cy] * wz[cz] * fl;
        lX[1] += wx[cx] * sy[cy] * wz[cz] * fl;
        lX[2] += wx[cx] * wy[cy] * sz[cz] * fl;
        const double w = wz[cz] * wy[cy] * wx[cx];
        for (int c = 0; c < 3; ++c) add_to(lu + c * comp + at, w * lam[c]);
      }
    }
  }
  for (int c = 0; c < 3; ++c) lX[c] /= dx;
}

// One tracer p. `push` = 1: the Heun push and closing deposit with the forward's own weights b₀, β*
// and β_m = β₀ − b₀ (adams_step_weights for one sample: h, h/2, −h/2 as the quadrature rounds them),
// so X* and X' are the forward's to the bit; X and f₀ are the positions and the newest sample before
// the push. `push` = 0: the particle deposit alone at X. lX, lf: the cotangents [3][M], replaced.
template <class T>
GBGHT_HD void tracer_adjoint_one(int64_t p, int64_t M, const T* GBGHT_RESTRICT u, double* lu, int N, double L,
                                 const double* GBGHT_RESTRICT X, const double* GBGHT_RESTRICT f0, double* lX,
                                 double* lf, int push, double b0, double beta_star, double beta_m) {
  const double dx = div_rn(L, double(N));
  double x[3], lXn[3], lfn[3], g[3];
  for (int c = 0; c < 3; ++c) {
    x[c] = X[c * M + p];
    lXn[c] = lX[c * M + p];
    lfn[c] = lf[c * M + p];
  }
  if (!push) {
    gather3_adjoint<T>(u, lu, N, dx, x[0], x[1], x[2], lfn, g);
    for (int c = 0; c < 3; ++c) {
      lX[c * M + p] = lXn[c] + g[c];
      lf[c * M + p] = 0.0;
    }
    return;
  }
  double f[3], xs[3], fs[3], xn[3];
  for (int c = 0; c < 3; ++c) {
    f[c] = f0[c * M + p];
    xs[c] = wrap_periodic(add_rn(x[c], mul_rn(b0, f[c])), L);
  }
  gather3(u, N, dx, xs[0], xs[1], xs[2], fs);
  for (int c = 0; c < 3; ++c)
    xn[c] = wrap_periodic(add_rn(xs[c], add_rn(mul_rn(beta_star, fs[c]), mul_rn(beta_m, f[c]))), L);
  gather3_adjoint<T>(u, lu, N, dx, xn[0], xn[1], xn[2], lfn, g);
  double lXt[3], lfs[3], lf0[3];
  for (int c = 0; c < 3; ++c) {
    lXt[c] = lXn[c] + g[c];
    lfs[c] = beta_star * lXt[c];
    lf0[c] = beta_m * lXt[c];
  }
  gather3_adjoint<T>(u, lu, N, dx, xs[0], xs[1], xs[2], lfs, g);
  for (int c = 0; c < 3; ++c) {
    const double lxs = lXt[c] + g[c];
    lX[c * M + p] = lxs;
    lf[c * M + p] = lf0[c] + b0 * lxs;
  }
}

// The r2c of one pair of physical lines of λ_u (component c, rows y and y + 1 of plane z) into B
// slot c: line pair `pair` of the [3][N][N/2] pairs, scaled by 1/N³; columns past K get zeros.
template <class T, int N>
struct PhysPairSource {
  static constexpr bool kExternal = true;
  const double* lu;
  size_t base;   // element (c, z, y, 0)
  GBGHT_HD Cplx<T> load(int e) const { return cmk<T>(T(lu[base + e]), T(lu[base + N + e])); }
};
template <class T, int N, int NW, int NT>
GBGHT_HD void body_phys_forward(const Cta& c, Cplx<T>* sm, const Geometry& g, const double* GBGHT_RESTRICT lu,
                                Cplx<T>* Ba, const Cplx<T>* GBGHT_RESTRICT tw) {
  const int npairs = 3 * N * (N / 2);
  const int pair0 = c.bx * NW;
  const auto lines = [&](int l) { return sm + l * N; };
  const auto src = [&](int l) {
    const int pr = pair0 + l;
    const int cc = pr / (N * (N / 2)), rem = pr % (N * (N / 2)), z = rem / (N / 2), y = 2 * (rem % (N / 2));
    return PhysPairSource<T, N>{lu, ((size_t(cc) * N + z) * N + y) * N};
  };
  const auto in_smem = [&](int l) { return LineBuf<T>{sm + l * N}; };
  const int nl = npairs - pair0 < NW ? npairs - pair0 : NW;
  warp_fft_lines<T, N, NW, NT, -1>(c, nl, lines, src, in_smem, tw);
  GBGHT_SYNC();
  const T sc = T(g.inv_norm);
  for (int t = c.tid; t < 32 * NW; t += NT) {
    const int w = t >> 5, lane = t & 31;
    if (w >= nl) continue;
    const int pr = pair0 + w;
    const int cc = pr / (N * (N / 2)), rem = pr % (N * (N / 2)), z = rem / (N / 2), y = 2 * (rem % (N / 2));
    const Cplx<T>* Lp = sm + w * N;
    for (int k = lane; k < g.KXP; k += 32) {
      Cplx<T> a = czero<T>(), b = czero<T>();
      if (k <= g.K) {
        const Cplx<T> zk = Lp[lidx<T>(k)];
        const Cplx<T> zc = conj(Lp[lidx<T>((N - k) % N)]);
        const Cplx<T> sp = zk + zc, sd = zk - zc;
        a = cmk<T>(sp.x * T(0.5) * sc, sp.y * T(0.5) * sc);
        b = cmk<T>(sd.y * T(0.5) * sc, -sd.x * T(0.5) * sc);
      }
      Ba[idxB(g, cc, z, y, k)] = a;
      Ba[idxB(g, cc, z, y + 1, k)] = b;
    }
  }
}

}  // namespace gbght
