// Engine implementation: device buffers, kernel launches, and the sequence of one IF-RK step.
//
// Built by nvcc for sm_100a (the library), or by a host C++ compiler with -DGBGHT_EMU for the
// CPU check of the kernel bodies (see gbght_engine.cuh).
#include "gbght_engine.cuh"
#include "kernels.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>

namespace gbght {

// ------------------------------------------------------------------------------------------------
// Runtime: device memory and copies.
// ------------------------------------------------------------------------------------------------
#ifdef GBGHT_EMU
using Stream = void*;
static const char* rt_alloc(void** p, size_t n) {
  *p = std::calloc(1, n ? n : 1);
  return *p ? nullptr : "host allocation failed";
}
static void rt_free(void* p) { std::free(p); }
static const char* rt_memset(void* p, int v, size_t n, Stream) { std::memset(p, v, n); return nullptr; }
static const char* rt_h2d(void* d, const void* h, size_t n, Stream) { std::memcpy(d, h, n); return nullptr; }
static const char* rt_d2h(void* h, const void* d, size_t n, Stream) { std::memcpy(h, d, n); return nullptr; }
static const char* rt_d2d(void* d, const void* s, size_t n, Stream) { std::memcpy(d, s, n); return nullptr; }
static const char* rt_sync(Stream) { return nullptr; }
static const char* rt_check() { return nullptr; }
static const char* rt_copy(void* d, const void* s, size_t n, Stream) { std::memcpy(d, s, n); return nullptr; }
#else
using Stream = cudaStream_t;
static thread_local char g_cuda_msg[256];
static const char* cuda_err(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return nullptr;
  std::snprintf(g_cuda_msg, sizeof g_cuda_msg, "%s: %s", what, cudaGetErrorString(e));
  return g_cuda_msg;
}
static const char* rt_alloc(void** p, size_t n) {
  const char* e = cuda_err(cudaMalloc(p, n ? n : 16), "cudaMalloc");
  if (!e) e = cuda_err(cudaMemset(*p, 0, n ? n : 16), "cudaMemset");
  return e;
}
static void rt_free(void* p) { if (p) cudaFree(p); }
static const char* rt_memset(void* p, int v, size_t n, Stream s) { return cuda_err(cudaMemsetAsync(p, v, n, s), "cudaMemsetAsync"); }
static const char* rt_h2d(void* d, const void* h, size_t n, Stream s) {
  return cuda_err(cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync H2D");
}
static const char* rt_d2d(void* d, const void* src, size_t n, Stream s) {
  return cuda_err(cudaMemcpyAsync(d, src, n, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync D2D");
}
static const char* rt_d2h(void* h, const void* d, size_t n, Stream s) {
  const char* e = cuda_err(cudaMemcpyAsync(h, d, n, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync D2H");
  if (!e) e = cuda_err(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return e;
}
static const char* rt_sync(Stream s) { return cuda_err(cudaStreamSynchronize(s), "cudaStreamSynchronize"); }
static const char* rt_check() { return cuda_err(cudaGetLastError(), "kernel launch"); }
// A copy between any two of host memory and device memory (unified addressing tells them apart),
// then a synchronisation.
static const char* rt_copy(void* d, const void* src, size_t n, Stream s) {
  const char* e = cuda_err(cudaMemcpyAsync(d, src, n, cudaMemcpyDefault, s), "cudaMemcpyAsync");
  if (!e) e = cuda_err(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return e;
}
#endif


// ------------------------------------------------------------------------------------------------
// Launch shapes.
// ------------------------------------------------------------------------------------------------
template <class T> struct Shape {
  static constexpr int TLY = 128 / int(sizeof(Cplx<T>));   // y passes: 128-byte rows
  static constexpr int TLZ = 4;                             // z epilogue: 4 columns (64-byte rows in FP64)
};
constexpr int clamp_nt(int v) { return v < 64 ? 64 : (v > 256 ? 256 : v); }

#ifdef GBGHT_EMU
constexpr int kNT(int) { return 1; }
constexpr int kNTZ(int) { return 1; }
#else
constexpr int kNT(int v) { return clamp_nt(v); }
constexpr int kNTZ(int v) { return v < 64 ? 64 : (v > 512 ? 512 : v); }
#endif

template <class F>
static void emu_grid(int gx, int gy, int gz, size_t smem, F&& body) {
  std::vector<double> sm((smem + sizeof(double) - 1) / sizeof(double) + 8);
  for (int bz = 0; bz < gz; ++bz)
    for (int by = 0; by < gy; ++by)
      for (int bx = 0; bx < gx; ++bx) {
        Cta c{0, bx, by, bz};
        body(c, reinterpret_cast<void*>(sm.data()));
      }
}


// ------------------------------------------------------------------------------------------------
// Host helpers.
// ------------------------------------------------------------------------------------------------
static int compute_K(int N, double s, double cut2) {
  int K = 0;
  while (K + 1 < N / 2 + 1) {
    const double k = s * double(K + 1);
    if (k * k <= cut2) ++K;
    else break;
  }
  return K;
}


template <class T, int N, int DEA>
class EngineImpl final : public Engine {
  // the retained box's bound on |m|: the 2/3 ball's (TwoThirds), or all but the Nyquist planes (the
  // wide instantiation: HouLi, and PhaseShift's √2·N/3 ball below it)
  static constexpr int KM = DEA ? N / 2 - 1 : N / 3 + 1;
  static constexpr int TLY = Shape<T>::TLY;
  // The y tiles' TMA copies start at row offsets K+1, N−K−1 and N−K, which must be 128-byte
  // aligned in shared memory: rows of exactly 128 bytes make every row offset aligned.
  static_assert(TLY * sizeof(Cplx<T>) == 128, "y tiles need 128-byte rows");
  static constexpr int TLZ = Shape<T>::TLZ;
  static constexpr int NTY = kNT(N * TLY / 8);
  static constexpr int NTX = kNT(N);            // (unused by the warp-per-line x passes)
#ifdef GBGHT_EMU
  static constexpr int NTXP = 1, NTXV = 1;
#else
  static constexpr int NTXP = 32 * XShape<T>::NW, NTXV = 32 * 6;   // one warp per line
#endif
  // z epilogue: one thread per butterfly of the first and last radix-R stage (N/R·TLZ of them),
  // up to 512
  static constexpr int NTZ = kNTZ(N * TLZ / Radices<N>::r[0]);
  static constexpr int NTR = kNT(256);
#ifdef GBGHT_EMU
  static constexpr int NTXA = 1, NTZA = 1;
#else
  static constexpr int NTXA = 32 * XAdjShape<T>::NW;   // the adjoint x pass: one warp per line
  static constexpr int NTZA = kNT(N * TLZ / 8);       // the adjoint z pass
#endif

 public:
  ~EngineImpl() override {
#ifndef GBGHT_EMU
    if (stream_) cudaStreamSynchronize(stream_);
    for (auto& pr : pending_) {
      cudaEventDestroy(pr.a);
      cudaEventDestroy(pr.b);
    }
    for (cudaEvent_t e : pool_) cudaEventDestroy(e);
    for (cudaEvent_t e : timer_ev_)
      if (e) cudaEventDestroy(e);
#endif
    for (void* p : allocs_) rt_free(p);
#ifndef GBGHT_EMU
    if (grp_) rt_free(grp_);
    if (stream_) cudaStreamDestroy(stream_);
#endif
  }

  const char* init(const RunParams& p) override {
    p_ = p;
    const double s = 2.0 * M_PI / p.L;
    g_.N = N;
    g_.s = s;
    if (DEA && p.dealias == 2) {
      // PhaseShift (src/SimulationDomain.jl:177-184,362): the closed ball at (2√2/3)·κ_Ny = √2·N/3·κ₀,
      // inside the wide box's bound
      const double cutoff = (2.0 * std::sqrt(2.0) / 3.0) * (double(N) / 2.0) * s;
      cutoff_ = cutoff;
      g_.cut2 = cutoff * cutoff;
      g_.K = compute_K(N, s, g_.cut2);
      phase_ = true;
    } else if (DEA) {   // HouLi (src/SimulationDomain.jl:365-376): every mode but the Nyquist planes, filtered
      const double kny = (double(N) / 2.0) * s;
      cutoff_ = kny;
      g_.cut2 = INFINITY;
      g_.K = N / 2 - 1;
      g_.houli = 1;
      g_.filt_strength = p.houli_strength > 0 ? p.houli_strength
                                              : -std::log(sizeof(T) == 8 ? DBL_EPSILON : double(FLT_EPSILON));
      g_.filt_half_order = 0.5 * double(p.houli_order);
      g_.inv_kny2 = 1.0 / (kny * kny);
    } else {
      const double cutoff = (2.0 / 3.0) * (double(N) / 2.0) * s;
      cutoff_ = cutoff;
      g_.cut2 = cutoff * cutoff;
      g_.K = compute_K(N, s, g_.cut2);
    }
    g_.NY2 = 2 * g_.K + 1;
    g_.KXP = ((g_.K + 1 + TLY - 1) / TLY) * TLY;
    g_.inv_norm = 1.0 / (double(N) * double(N) * double(N));
    if (g_.NY2 > N) return "grid too small for the retained band";
    if (g_.K > ZOwn<T, N, TLZ, NTZ, KM>::KMAX) return "retained band wider than the z tile's row slots";
    nS_ = size_t(g_.NY2) * g_.NY2 * g_.KXP;
    nA_ = size_t(N) * g_.NY2 * g_.KXP;
    nB_ = size_t(N) * N * g_.KXP;
    nP_ = size_t(N) * N * N;
    ntile_ = (g_.KXP / TLZ) * g_.NY2;
    nshell_ = int(std::floor(std::sqrt(3.0) * N / 2.0 + 0.5)) + 1;
#ifndef GBGHT_EMU
    const char* e = cuda_err(cudaSetDevice(p.device), "cudaSetDevice");
    if (e) return e;
    e = cuda_err(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    if (e) return e;
    if ((e = set_smem_attributes())) return e;
    if ((e = cuda_err(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, p.device),
                      "cudaDeviceGetAttribute")))
      return e;
#endif
    const char* err = nullptr;
    if ((err = alloc(&S_, 4 * nS_ * sizeof(Cplx<T>)))) return err;
    if ((err = alloc(&H_, 4 * nS_ * sizeof(Cplx<T>)))) return err;
    if ((err = alloc(&A_, 7 * nA_ * sizeof(Cplx<T>)))) return err;
    if ((err = alloc(&B_, 7 * nB_ * sizeof(Cplx<T>)))) return err;
    if (phase_ && (err = alloc(&A2_, 7 * nA_ * sizeof(Cplx<T>)))) return err;   // the displaced grid's A
    if ((err = alloc(&U_, 3 * nP_ * sizeof(T)))) return err;
    if ((err = alloc(&tw_, N * sizeof(Cplx<T>)))) return err;
    if ((err = alloc(&partial_, ntile_ * sizeof(double)))) return err;
    if ((err = alloc(&amp_, 16 * sizeof(double)))) return err;   // 4 per field and role
    if ((err = alloc(&maxbits_, sizeof(unsigned long long)))) return err;
    if ((err = alloc(&status_, sizeof(unsigned int)))) return err;
    if ((err = alloc(&flag_, sizeof(unsigned int)))) return err;
    // B doubles as the staging of one reference-layout component at import and export
    if (7 * nB_ * sizeof(Cplx<T>) < ref_comp_elems() * sizeof(Cplx<double>)) return "B too small to stage a component";
    if ((err = alloc(&obs_, size_t(g_.NY2) * 4 * sizeof(double)))) return err;
    if ((err = alloc(&fobs_, size_t(g_.NY2) * 4 * sizeof(double)))) return err;
    if ((err = alloc(&spec_, size_t(g_.NY2) * nshell_ * sizeof(double)))) return err;
    if (p.tracers > 0) {
      if (p.tracers > int64_t(UINT32_MAX)) return "too many tracers for a 32-bit traversal order";
      if ((err = alloc(&X_, 3 * size_t(p.tracers) * sizeof(double)))) return err;
      if (p.trail_capacity < 1 || p.trail_capacity > kTrailMax) return "bad trail capacity";
      if ((err = alloc(&F_, size_t(p.trail_capacity) * 3 * size_t(p.tracers) * sizeof(double)))) return err;
      const size_t nt = size_t(traversal_tiles(N));
      nbins_ = int(nt * nt * nt);
      if ((err = alloc(&tkey_, size_t(p.tracers) * sizeof(uint32_t)))) return err;
      if ((err = alloc(&torder_, size_t(p.tracers) * sizeof(uint32_t)))) return err;
      if ((err = alloc(&tcount_, size_t(nbins_) * sizeof(uint32_t)))) return err;
    }
    for (int f = 0; f < 2; ++f) {   // StochasticOU: the companion grid's force
      const ForcingParams& fp = f == 0 ? p.vf : p.sf;
      if (fp.kind != kForceStochastic) continue;
      const int nc = 2 * (int(fp.highest_shell) + 1);
      src_nc_[f] = nc;
      if ((err = alloc(&src_[f], size_t(f == 0 ? 3 : 1) * nc * nc * (nc / 2 + 1) * sizeof(Cplx<double>)))) return err;
    }
#ifndef GBGHT_EMU
    if ((err = make_maps())) return err;
    if (phase_ && (err = make_maps_on(&maps_ps_, A2_, B_))) return err;
#endif
    // twiddles e^(-2πi k/N) in extended precision
    std::vector<Cplx<T>> tw(N);
    for (int k = 0; k < N; ++k) {
      const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)N;
      tw[k] = cmk<T>(T(cosl(a)), T(-sinl(a)));
    }
    if ((err = rt_h2d(tw_, tw.data(), N * sizeof(Cplx<T>), stream_))) return err;
    return rt_sync(stream_);
  }

  int K() const override { return g_.K; }
  double cutoff() const override { return cutoff_; }

  // ---- state import / export (the reference layout, host or device memory) --------------------------
  // Each component of a host array crosses through B (scratch between steps), and a kernel converts
  // it on the device; a device array of the run's device is read or written by the kernel in place.
  // Import compacts into H, which is dead between steps, so a refused import (content outside the
  // retained ball) leaves S as it was.
  size_t ref_comp_elems() const { return size_t(N) * N * (N / 2 + 1); }
  // 1: memory of the run's device (device or managed), 0: host memory, −1: another device's memory.
  int where(const void* p) const {
#ifdef GBGHT_EMU
    (void)p;
    return 0;
#else
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();   // an unregistered host pointer on older runtimes
      return 0;
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return a.device == p_.device ? 1 : -1;
    return 0;
#endif
  }
  const char* import_state(const double* uh, const double* ph, bool* outside) override {
    const int nc = p_.scalar ? 4 : 3;
    const size_t nref = ref_comp_elems();
    *outside = false;
    const int wu = where(uh), wp = nc == 4 ? where(ph) : 0;
    if (wu < 0 || wp < 0) return "a state array is device memory of another device";
    bu_fresh_ = false;   // B is overwritten
    Cplx<double>* stage = reinterpret_cast<Cplx<double>*>(B_);
    const char* err = rt_memset(H_, 0, 4 * nS_ * sizeof(Cplx<T>), stream_);
    if (!err) err = rt_memset(flag_, 0, sizeof(unsigned int), stream_);
    for (int cc = 0; cc < nc && !err; ++cc) {
      const double* src = cc < 3 ? uh + size_t(cc) * nref * 2 : ph;
      const Cplx<double>* ref = reinterpret_cast<const Cplx<double>*>(src);
      if (!(cc < 3 ? wu : wp)) {
        err = rt_h2d(stage, src, nref * sizeof(Cplx<double>), stream_);
        if (err) break;
        ref = stage;
      }
#ifdef GBGHT_EMU
      for (size_t i = 0; i < nref; ++i) import_mode<T>(i, g_, ref, H_ + cc * nS_, flag_);
#else
      k_import<T><<<unsigned((nref + 255) / 256), 256, 0, stream_>>>(g_, ref, H_ + cc * nS_, flag_);
      err = rt_check();
#endif
    }
    unsigned int fl = 0;
    if (!err) err = rt_d2h(&fl, flag_, sizeof fl, stream_);
    if (err) return err;
    if (fl & 1u) {
      *outside = true;
      return nullptr;
    }
    if ((err = rt_d2d(S_, H_, 4 * nS_ * sizeof(Cplx<T>), stream_))) return err;
    if ((err = rt_memset(H_, 0, 4 * nS_ * sizeof(Cplx<T>), stream_))) return err;
    if ((err = z_init())) return err;
    return rt_sync(stream_);
  }

  const char* export_state(double* uh, double* ph) override {
    const size_t nref = ref_comp_elems();
    const int nc = (p_.scalar && ph) ? 4 : 3;
    const int wu = where(uh), wp = nc == 4 ? where(ph) : 0;
    if (wu < 0 || wp < 0) return "a state array is device memory of another device";
    bu_fresh_ = false;   // B is overwritten
    Cplx<double>* stage = reinterpret_cast<Cplx<double>*>(B_);
    for (int cc = 0; cc < nc; ++cc) {
      double* dst = cc < 3 ? uh + size_t(cc) * nref * 2 : ph;
      const bool direct = (cc < 3 ? wu : wp) == 1;
      Cplx<double>* ref = direct ? reinterpret_cast<Cplx<double>*>(dst) : stage;
#ifdef GBGHT_EMU
      for (size_t i = 0; i < nref; ++i) export_mode<T>(i, g_, S_ + cc * nS_, ref);
#else
      k_export<T><<<unsigned((nref + 255) / 256), 256, 0, stream_>>>(g_, S_ + cc * nS_, ref);
      if (const char* e = rt_check()) return e;
#endif
      if (!direct)
        if (const char* e = rt_d2h(dst, ref, nref * sizeof(Cplx<double>), stream_)) return e;
    }
    return rt_sync(stream_);
  }

  // ---- the step ---------------------------------------------------------------------------------
  // The common part of a stage's arguments: the forcings, the bands, the mean gradient.
  StageArgs stage_base(double dt) const {
    StageArgs st{};
    st.dt = dt;
    st.has_scalar = p_.scalar;
    st.forced = stage_source(p_.vf.kind);
    st.sforced = p_.scalar && stage_source(p_.sf.kind);
    st.band_lo2 = band_lo2();
    st.band_hi2 = band_hi2();
    st.sband_lo2 = sband_lo2();
    st.sband_hi2 = sband_hi2();
    st.G[0] = p_.G[0];
    st.G[1] = p_.G[1];
    st.G[2] = p_.G[2];
    return st;
  }
  // The integrating factors of a span δ: E = exp(−D·δ·|κ|² + δ·A), A a Linear forcing's rate on
  // its band (src/Generator.jl:565-581). `second` selects the stage's second factor.
  void set_factor(StageArgs& st, double delta, bool second) const {
    const double cu = -(p_.viscosity * delta), cphi = -((p_.viscosity / p_.schmidt) * delta);
    const double lu = p_.vf.kind == kForceLinear ? delta * p_.vf.rate : 0.0;
    const double lphi = p_.sf.kind == kForceLinear ? delta * p_.sf.rate : 0.0;
    if (second) {
      st.cu2 = cu;
      st.cphi2 = cphi;
      st.lin_u2 = lu;
      st.lin_phi2 = lphi;
    } else {
      st.cu = cu;
      st.cphi = cphi;
      st.lin_u = lu;
      st.lin_phi = lphi;
    }
  }
  // The stages of one step of the run's scheme, with their arguments, into out[] (at most
  // kStepStages); returns their count.
  static constexpr int kStepStages = 5;
  int stage_list(double dt, const double* a, const double* b, const double* d, int S, StageArgs* out) const {
    if (p_.scheme == 2) {   // IFHeun: predictor, corrector
      out[0] = stage_base(dt);
      out[0].kind = kHeunPredictor;
      out[0].first = 1;
      out[0].write_h = 1;
      set_factor(out[0], dt, false);
      out[1] = stage_base(dt);
      out[1].kind = kHeunCorrector;
      out[1].last = 1;
      out[1].read_h = 1;
      return 2;
    }
    if (p_.scheme == 3) {   // IFSSPRK3: forward to t_n+1, back to the midpoint, forward again
      const double span1[3] = {dt, -dt / 2, dt / 2}, span2[3] = {0.0, dt / 2, dt};
      for (int i = 0; i < 3; ++i) {
        StageArgs& st = out[i];
        st = stage_base(dt);
        st.kind = kSsp1 + i;
        st.first = i == 0;
        st.last = i == 2;
        st.read_h = i > 0;
        st.write_h = i == 0;
        set_factor(st, span1[i], false);
        if (i > 0) set_factor(st, span2[i], true);
      }
      return 3;
    }
    for (int i = 0; i < S && i < kStepStages; ++i) {   // the low-storage 2N schemes
      StageArgs& st = out[i];
      st = stage_base(dt);
      st.kind = kLowStorage;
      st.a = a[i];
      st.b = b[i];
      st.first = i == 0;
      st.last = i == S - 1;
      st.read_h = !st.first;
      st.write_h = !st.last;
      set_factor(st, d[i] * dt, false);
    }
    return S;
  }
  const char* step(double dt, const double* a, const double* b, const double* d, int S) override {
    if (S > kStepStages) return "a scheme of more stages than the step holds";
    StageArgs st[kStepStages];
    const int n = stage_list(dt, a, b, d, S, st);
    for (int i = 0; i < n; ++i)
      if (const char* err = stage(st[i])) return err;
    return rt_check();
  }

  const char* deposit(double* max_speed2) override {
    if (const char* err = deposit_launch()) return err;
    return deposit_read(max_speed2);
  }
  const char* deposit_launch() override {
    const char* err = rt_memset(maxbits_, 0, sizeof(unsigned long long), stream_);
    if (err) return err;
    y_inverse(0, 3);
    bu_fresh_ = true;
    x_velocity();
    return rt_check();
  }
  void* cuda_stream() const override {
#ifdef GBGHT_EMU
    return nullptr;
#else
    return stream_;
#endif
  }
  bool deposit_fresh() const override { return bu_fresh_; }
  bool profiling() const override { return prof_on_; }

  // ---- member-batched stepping (an ensemble's groups) ----------------------------------------------
  // The key: precision, N, the dealiasing instantiation, the scheme, the scalar, the velocity
  // forcing's kind. Runs that step alone: PhaseShift (its displaced passes), StochasticOU sources,
  // VarianceController and VarianceRescaling (row sums, the post-step rescale).
  uint64_t group_key() const override {
#ifdef GBGHT_EMU
    return 0;
#else
    const int vk = p_.vf.kind, sk = p_.scalar ? p_.sf.kind : int(kForceNone);
    if (phase_ || src_[0] || src_[1]) return 0;
    if (!(vk == kForceNone || vk == kForceConstantPower || vk == kForceLinear)) return 0;
    if (!(sk == kForceNone || sk == kForceLinear)) return 0;
    uint64_t k = uint64_t(sizeof(T));
    k = k * 1024 + uint64_t(N);
    k = k * 4 + uint64_t(DEA);
    k = k * 8 + uint64_t(p_.scheme);
    k = k * 2 + uint64_t(p_.scalar);
    k = k * 8 + uint64_t(vk);
    return k;
#endif
  }
#ifdef GBGHT_EMU
  const char* group_prepare(Engine* const*, int, double, const double*, const double*, const double*, int) override {
    return "member-batched stepping runs on the device only";
  }
  const char* group_launch() override { return "member-batched stepping runs on the device only"; }
#else
  const char* group_prepare(Engine* const* ms, int n, double dt, const double* a, const double* b, const double* d,
                            int S) override {
    if (n < 1 || S > kStepStages || kStepStages > kGroupStages) return "bad group";
    std::vector<GroupMember<T>> h(static_cast<size_t>(n));
    std::vector<EngineImpl*> members(static_cast<size_t>(n));
    const uint64_t key = group_key();
    for (int i = 0; i < n; ++i) {
      EngineImpl* m = dynamic_cast<EngineImpl*>(ms[i]);
      if (!m || key == 0 || m->group_key() != key) return "a group member launches other kernels";
      members[size_t(i)] = m;
      GroupMember<T>& r = h[size_t(i)];
      std::memset(static_cast<void*>(&r), 0, sizeof r);
      r.maps = m->maps_;
      r.g = m->g_;
      r.A = m->A_;
      r.B = m->B_;
      r.S = m->S_;
      r.H = m->H_;
      r.U = m->U_;
      r.partial = m->partial_;
      r.amp = m->amp_;
      r.status = m->status_;
      r.maxbits = m->maxbits_;
      r.ntile = int(m->ntile_);
      r.band_lo2 = m->band_lo2();
      r.band_hi2 = m->band_hi2();
      r.vamp = m->amp_args(m->p_.vf, false);
      grp_nst_ = m->stage_list(dt, a, b, d, S, r.st);
    }
    const size_t bytes = size_t(n) * sizeof(GroupMember<T>);
    if (bytes > grp_bytes_) {
      if (grp_) rt_free(grp_);
      grp_ = nullptr;
      grp_bytes_ = 0;
      if (const char* e = rt_alloc(reinterpret_cast<void**>(&grp_), bytes)) return e;
      grp_bytes_ = bytes;
    }
    if (const char* e = rt_h2d(grp_, h.data(), bytes, stream_)) return e;
    for (int i = 0; i < grp_nst_; ++i) grp_st_[i] = h[0].st[i];
    grp_members_ = members;
    return rt_sync(stream_);
  }
  const char* group_launch() override {
    const int n = int(grp_members_.size());
    if (n < 1 || !grp_) return "the group is not prepared";
    for (EngineImpl* m : grp_members_)
      if (!m->bu_fresh_) return "a group member's deposit is not current";
    const int ninv = p_.scalar ? 7 : 6, nfwd = p_.scalar ? 6 : 3, nc = p_.scalar ? 4 : 3;
    const int KXS = x_kxs(g_.K, int(sizeof(Cplx<T>)));
    const int gx = g_.KXP / TLZ;
    const int xgrid = ((N / XShape<T>::P) * N + XT - 1) / XT, vgrid = ((N / XShape<T>::PV) * N + XT - 1) / XT;
    const GroupMember<T>* G = grp_;
    for (int i = 0; i < grp_nst_; ++i) {
      const StageArgs& st = grp_st_[i];
      // the first stage reuses the deposit's y-inverse of the velocity slots
      const int c0 = i == 0 ? 3 : 0;
      kg_y_inverse<T, N, TLY, NTY><<<dim3(g_.KXP / TLY, N, (ninv - c0) * n), NTY, smem_y(), stream_>>>(G, c0, ninv - c0, tw_);
      kg_x_products<T, N, NTXP><<<dim3(xgrid, n), NTXP, smem_x(), stream_>>>(G, p_.scalar, KXS, tw_);
      kg_y_forward<T, N, TLY, NTY><<<dim3(g_.KXP / TLY, N, nfwd * n), NTY, smem_y(), stream_>>>(G, nfwd, tw_);
      if (st.forced) kg_force_amp<T><<<n, 256, 0, stream_>>>(G);
      const dim3 zg(unsigned(gx), unsigned(g_.NY2), unsigned(n));
      switch (st.kind) {
        case kHeunPredictor: kg_z_epilogue<T, N, TLZ, NTZ, kHeunPredictor, KM, (DEA != 0)><<<zg, NTZ, smem_ze(), stream_>>>(G, i, tw_); break;
        case kHeunCorrector: kg_z_epilogue<T, N, TLZ, NTZ, kHeunCorrector, KM, (DEA != 0)><<<zg, NTZ, smem_ze(), stream_>>>(G, i, tw_); break;
        case kSsp1: kg_z_epilogue<T, N, TLZ, NTZ, kSsp1, KM, (DEA != 0)><<<zg, NTZ, smem_ze(), stream_>>>(G, i, tw_); break;
        case kSsp2: kg_z_epilogue<T, N, TLZ, NTZ, kSsp2, KM, (DEA != 0)><<<zg, NTZ, smem_ze(), stream_>>>(G, i, tw_); break;
        case kSsp3: kg_z_epilogue<T, N, TLZ, NTZ, kSsp3, KM, (DEA != 0)><<<zg, NTZ, smem_ze(), stream_>>>(G, i, tw_); break;
        default: kg_z_epilogue<T, N, TLZ, NTZ, kLowStorage, KM, (DEA != 0)><<<zg, NTZ, smem_ze(), stream_>>>(G, i, tw_);
      }
      if (st.last) {   // the reality projection, then the first tile column of A rebuilt
        kg_reality<T><<<dim3(unsigned((g_.NY2 * g_.NY2 + 255) / 256), unsigned(n)), 256, 0, stream_>>>(G, nc);
        kg_z_init_column<T, N, TLZ, NTZ, KM><<<dim3(1, unsigned(g_.NY2), unsigned(n)), NTZ, smem_z(), stream_>>>(
            G, p_.scalar, gx, tw_);
      }
    }
    // the closing deposit: the velocity's y-inverse into B slots 0..2, its physical values and max|u|²
    kg_zero_maxbits<T><<<unsigned((n + 127) / 128), 128, 0, stream_>>>(G, n);
    kg_y_inverse<T, N, TLY, NTY><<<dim3(g_.KXP / TLY, N, 3 * n), NTY, smem_y(), stream_>>>(G, 0, 3, tw_);
    kg_x_velocity<T, N, NTXV><<<dim3(vgrid, n), NTXV, smem_xv(), stream_>>>(G, KXS, tw_);
    for (EngineImpl* m : grp_members_) m->bu_fresh_ = true;
    return rt_check();
  }
#endif
  const char* deposit_read(double* max_speed2) override {
    const char* err = nullptr;
    unsigned long long bits = 0;
    if ((err = rt_d2h(&bits, maxbits_, sizeof bits, stream_))) return err;
    double m;
    std::memcpy(&m, &bits, sizeof m);
    *max_speed2 = m;
    unsigned int st = 0;
    if ((err = rt_d2h(&st, status_, sizeof st, stream_))) return err;
    if (st & GBGHT_DEV_TIMEOUT) return kDeviceTimeoutMessage;
    return nullptr;
  }

  const char* forcing_source(int field, const double* amplitudes, int nc) override {
    if (field < 0 || field > 1 || !src_[field]) return "the field carries no StochasticOU forcing";
    if (nc != src_nc_[field]) return "the force is given on a companion grid of another size";
    if (where(amplitudes) < 0) return "the force is device memory of another device";
    const size_t n = size_t(field == 0 ? 3 : 1) * nc * nc * (nc / 2 + 1) * sizeof(Cplx<double>);
    return rt_copy(src_[field], amplitudes, n, stream_);
  }
  const char* velocity_export(double* u) override {
    std::vector<T> host(3 * nP_);
    const char* err = rt_d2h(host.data(), U_, 3 * nP_ * sizeof(T), stream_);
    if (err) return err;
    for (size_t i = 0; i < 3 * nP_; ++i) u[i] = double(host[i]);
    return nullptr;
  }

  const char* velocity_import(const double* u) override {
    std::vector<T> host(3 * nP_);
    for (size_t i = 0; i < 3 * nP_; ++i) host[i] = T(u[i]);
    const char* err = rt_h2d(U_, host.data(), 3 * nP_ * sizeof(T), stream_);
    if (err) return err;
    return rt_sync(stream_);
  }

  // the four raw sums of body_observables over all ky' rows (mode 2: the scalar sums only)
  const char* observable_sums(int mode, double s[4]) {
#ifdef GBGHT_EMU
    emu_grid(g_.NY2, 1, 1, 4 * sizeof(double), [&](const Cta& c, void* sm) {
      body_observables<T, 1>(c, static_cast<double*>(sm), g_, S_, mode, obs_);
    });
#else
    pbegin(PROF_OBSERVABLES);
    k_observables<T, NTR><<<g_.NY2, NTR, 4 * NTR * sizeof(double), stream_>>>(g_, S_, mode, obs_);
    pend();
#endif
    const char* err = rt_check();
    if (err) return err;
    std::vector<double> host(size_t(g_.NY2) * 4);
    if ((err = rt_d2h(host.data(), obs_, host.size() * sizeof(double), stream_))) return err;
    for (int j = 0; j < 4; ++j) s[j] = 0.0;
    for (int qy = 0; qy < g_.NY2; ++qy)
      for (int j = 0; j < 4; ++j) s[j] += host[qy * 4 + j];
    return nullptr;
  }
  const char* scalar_variance(double* var) override {
    double s[4];
    if (const char* err = observable_sums(p_.scalar ? 2 : 0, s)) return err;
    *var = s[2] / (double(N) * N * N * double(N) * N * N);
    return nullptr;
  }
  const char* observables(Observables* o) override {
    double s[4];
    if (const char* err = observable_sums(p_.scalar, s)) return err;
    const double n6 = double(N) * N * N * double(N) * N * N;
    const double kappa = p_.viscosity / p_.schmidt;
    o->k = 0.5 * (s[0] / n6);
    o->eps = p_.viscosity * (s[1] / n6);
    o->var = s[2] / n6;
    o->chi = 2.0 * kappa * (s[3] / n6);
    return nullptr;
  }

  // derivative_skewness (src/Observables.jl:466-478): C·3⟨det S⟩/⟨S:S⟩^{3/2}, ⟨S:S⟩ = ½Σκ²|û|².
  // The strain's z-inverse replaces the A slots, its y-inverse takes B slots 0..5, the deposit's x
  // pass turns each triple into physical components in a transient buffer, and the determinants
  // are summed in a fixed order. The A slots are rebuilt from the state afterwards.
  const char* skewness(double* out) override {
    double sums[4];
    if (const char* err = observable_sums(0, sums)) return err;
    const double n6 = double(N) * N * N * double(N) * N * N;
    const double ss = 0.5 * (sums[1] / n6);
    if (!(ss > 0)) {
      *out = 0.0;
      return nullptr;
    }
    const size_t n3 = size_t(N) * N * N;
    constexpr int NTD = 256;
    const size_t chunk = size_t(64) * NTD;
    const size_t nblk = (n3 + chunk - 1) / chunk;
    T* s6 = nullptr;
    double* part = nullptr;
    unsigned long long* mb = nullptr;
    const char* err = rt_alloc(reinterpret_cast<void**>(&s6), 6 * n3 * sizeof(T));
    if (!err) err = rt_alloc(reinterpret_cast<void**>(&part), nblk * sizeof(double));
    if (!err) err = rt_alloc(reinterpret_cast<void**>(&mb), sizeof(unsigned long long));
    if (!err) err = z_init(2);
    if (!err) {
      y_inverse(0, 6);
      x_velocity_into(B_, s6, mb);
      x_velocity_into(B_ + idxB(g_, 3, 0, 0, 0), s6 + 3 * n3, mb);
#ifdef GBGHT_EMU
      emu_grid(int(nblk), 1, 1, sizeof(double), [&](const Cta& c, void* sm) {
        body_det_sum<T, 1>(c, static_cast<double*>(sm), s6, n3, chunk, part);
      });
#else
      pbegin(PROF_OBSERVABLES);
      k_det_sum<T, NTD><<<unsigned(nblk), NTD, 0, stream_>>>(s6, n3, chunk, part);
      pend();
#endif
      err = rt_check();
    }
    std::vector<double> host(nblk);
    if (!err) err = rt_d2h(host.data(), part, nblk * sizeof(double), stream_);
    const char* err2 = z_init(1);   // the A slots hold the state's z-inverse again
    rt_free(s6);
    rt_free(part);
    rt_free(mb);
    if (err) return err;
    if (err2) return err2;
    double sum = 0.0;
    for (size_t b = 0; b < nblk; ++b) sum += host[b];
    const double mean_det = sum / double(n3);
    const double C = (4.0 / 7.0) * std::sqrt(15.0 / 2.0);
    *out = 3.0 * C * mean_det / std::pow(ss, 1.5);
    return nullptr;
  }
  const char* below_scale(double nu, double* k, double* eps) override {
    constexpr int CH = 16;
    double sums[4];
    if (const char* err = observable_sums(0, sums)) return err;
    const size_t nrow = size_t(N) * 2;
    double* rows = nullptr;
    const char* err = rt_alloc(reinterpret_cast<void**>(&rows), size_t(g_.NY2) * nrow * sizeof(double));
    if (err) return err;
    const int nchunk = (N + CH - 1) / CH;
#ifdef GBGHT_EMU
    emu_grid(g_.NY2, nchunk, 1, (size_t(CH) * (g_.K + 1) + 1) * sizeof(double), [&](const Cta& c, void* sm) {
      double* tab = static_cast<double*>(sm);
      body_below_scale<T, 1, CH>(c, tab, tab + CH * (g_.K + 1), g_, p_.L, S_, rows);
    });
#else
    const size_t smem = (size_t(CH) * (g_.K + 1) + NTR) * sizeof(double);
    pbegin(PROF_OBSERVABLES);
    k_below_scale<T, NTR, CH><<<dim3(g_.NY2, nchunk, 1), NTR, smem, stream_>>>(g_, p_.L, S_, rows);
    pend();
#endif
    err = rt_check();
    std::vector<double> host(size_t(g_.NY2) * nrow);
    if (!err) err = rt_d2h(host.data(), rows, host.size() * sizeof(double), stream_);
    rt_free(rows);
    if (err) return err;
    const double n6 = double(N) * N * N * double(N) * N * N;
    const double whole = sums[0] / n6, dirichlet = sums[1] / n6;
    for (int n = 0; n < N; ++n) {
      double rk = 0.0, re = 0.0;
      for (int qy = 0; qy < g_.NY2; ++qy) {
        rk += host[size_t(qy) * nrow + size_t(n) * 2];
        re += host[size_t(qy) * nrow + size_t(n) * 2 + 1];
      }
      k[n] = (whole - rk / n6) / 2;
      eps[n] = nu * (dirichlet - re / n6);
    }
    return nullptr;
  }
  const char* spectrum(int which, double* out, int nshell) override {
    const int c0 = which == 0 ? 0 : 3, nc = which == 0 ? 3 : 1;
    const size_t smem = (size_t(nshell_) + 2 * size_t(g_.KXP)) * sizeof(double);
#ifdef GBGHT_EMU
    emu_grid(g_.NY2, 1, 1, smem, [&](const Cta& c, void* sm) {
      double* hist = static_cast<double*>(sm);
      body_spectrum<T, 1>(c, hist, hist + nshell_, g_, S_, c0, nc, nshell_, spec_);
    });
#else
    k_spectrum<T, 32><<<g_.NY2, 32, smem, stream_>>>(g_, S_, c0, nc, nshell_, spec_);
#endif
    const char* err = rt_check();
    if (err) return err;
    std::vector<double> host(size_t(g_.NY2) * nshell_);
    if ((err = rt_d2h(host.data(), spec_, host.size() * sizeof(double), stream_))) return err;
    const double n6 = double(N) * N * N * double(N) * N * N;
    const double scale = which == 0 ? 1.0 / (2.0 * g_.s) : 1.0 / g_.s;
    for (int n = 0; n < nshell && n < nshell_; ++n) {
      double s = 0.0;
      for (int qy = 0; qy < g_.NY2; ++qy) s += host[size_t(qy) * nshell_ + n];
      out[n] = (s / n6) * scale;
    }
    for (int n = nshell_; n < nshell; ++n) out[n] = 0.0;
    return nullptr;
  }

  // ---- tracers ----------------------------------------------------------------------------------
  const char* tracers_set(const double* X) override {
    if (!X_) return "the run carries no tracers";
    if (where(X) < 0) return "the positions are device memory of another device";
    return rt_copy(X_, X, 3 * size_t(p_.tracers) * sizeof(double), stream_);
  }
  const char* tracers_get(double* X) override {
    if (!X_) return "the run carries no tracers";
    if (where(X) < 0) return "the positions are device memory of another device";
    return rt_copy(X, X_, 3 * size_t(p_.tracers) * sizeof(double), stream_);
  }
  const char* tracer_sample_get(double* F, int slot) override {
    if (!F_) return "the run carries no tracers";
    if (slot < 0 || slot >= p_.trail_capacity) return "no such trail slot";
    const size_t n = 3 * size_t(p_.tracers);
    if (where(F) < 0) return "the sample is device memory of another device";
    return rt_copy(F, F_ + size_t(slot) * n, n * sizeof(double), stream_);
  }
  const char* tracer_sample_set(const double* F, int slot) override {
    if (!F_) return "the run carries no tracers";
    if (slot < 0 || slot >= p_.trail_capacity) return "no such trail slot";
    const size_t n = 3 * size_t(p_.tracers);
    if (where(F) < 0) return "the sample is device memory of another device";
    return rt_copy(F_ + size_t(slot) * n, F, n * sizeof(double), stream_);
  }
  const char* tracers_run(const AdamsStep& w) override {
    if (!X_) return "the run carries no tracers";
    if (w.J < 0 || w.J > p_.trail_capacity || w.out_slot >= p_.trail_capacity) return "bad tracer step";
    for (int j = 0; j < w.J; ++j)
      if (w.slot[j] < 0 || w.slot[j] >= p_.trail_capacity) return "bad tracer step";
    if (const char* e = rebuild_traversal()) return e;
    AdamsStep ws = w;
    ws.stencil = p_.stencil;
    run_tracers(p_.tracers, X_, F_, ws, torder_);
    return rt_check();
  }
  const char* gather(const double* X, int64_t M, double* out) override {
    if (M <= 0) return nullptr;
    double *dX = nullptr, *dF = nullptr;
    const char* err = rt_alloc(reinterpret_cast<void**>(&dX), 3 * size_t(M) * sizeof(double));
    if (!err) err = rt_alloc(reinterpret_cast<void**>(&dF), 3 * size_t(M) * sizeof(double));
    if (!err) err = rt_h2d(dX, X, 3 * size_t(M) * sizeof(double), stream_);
    if (!err) {
      AdamsStep w{};   // a gather alone, into slot 0 of a one-slot trail
      w.stencil = p_.stencil;
      run_tracers(M, dX, dF, w);
      err = rt_check();
    }
    if (!err) err = rt_d2h(out, dF, 3 * size_t(M) * sizeof(double), stream_);
    rt_free(dX);
    rt_free(dF);
    return err;
  }

  const char* sync() override { return rt_sync(stream_); }

  const char* profile(int enable) override {
#ifndef GBGHT_EMU
    const char* e = collect();
    if (e) return e;
#endif
    for (int k = 0; k < PROF_KINDS; ++k) {
      prof_ms_[k] = 0.0;
      prof_n_[k] = 0;
    }
    prof_on_ = enable != 0;
    return nullptr;
  }
  const char* profile_read(int kind, int64_t* launches, double* total_ms) override {
    if (kind < 0 || kind >= PROF_KINDS) return "unknown kernel kind";
#ifndef GBGHT_EMU
    const char* e = collect();
    if (e) return e;
#endif
    *launches = prof_n_[kind];
    *total_ms = prof_ms_[kind];
    return nullptr;
  }
  const char* timer(int op, double* ms) override {
#ifdef GBGHT_EMU
    (void)op;
    if (ms) *ms = 0.0;
    return nullptr;
#else
    if (!timer_ev_[0]) {
      for (auto& e : timer_ev_) {
        const char* err = cuda_err(cudaEventCreate(&e), "cudaEventCreate");
        if (err) return err;
      }
    }
    if (op == 0) return cuda_err(cudaEventRecord(timer_ev_[0], stream_), "cudaEventRecord");
    const char* err = cuda_err(cudaEventRecord(timer_ev_[1], stream_), "cudaEventRecord");
    if (!err) err = cuda_err(cudaEventSynchronize(timer_ev_[1]), "cudaEventSynchronize");
    float f = 0.f;
    if (!err) err = cuda_err(cudaEventElapsedTime(&f, timer_ev_[0], timer_ev_[1]), "cudaEventElapsedTime");
    if (ms) *ms = double(f);
    return err;
#endif
  }

  const char* expire_wait(long long cycles) override {
#ifdef GBGHT_EMU
    (void)cycles;
    *status_ |= GBGHT_DEV_TIMEOUT;   // the host-check build has no barrier to wait on
#else
    k_expire_wait<<<1, 32, 0, stream_>>>(status_, cycles);
    if (const char* e = rt_check()) return e;
#endif
    unsigned int st = 0;
    const char* err = rt_d2h(&st, status_, sizeof st, stream_);
    if (err) return err;
    return (st & GBGHT_DEV_TIMEOUT) ? kDeviceTimeoutMessage : nullptr;
  }

  // ---- the adjoint of the step ----------------------------------------------------------------------
  static constexpr int kMaxStages = 5;
  const char* adjoint_init(int snapshots) override {
    if (adj_ready_) {
      if (snapshots == nsnap_) return nullptr;
      return "the adjoint registers exist already with another snapshot count";
    }
    const size_t s4 = 4 * nS_ * sizeof(Cplx<T>);
    const char* err = nullptr;
    if ((err = alloc(&L_, s4))) return err;
    if ((err = alloc(&LH_, s4))) return err;
    if ((err = alloc(&Qs_, kMaxStages * s4))) return err;
    if ((err = alloc(&Aa_, 7 * nA_ * sizeof(Cplx<T>)))) return err;
    if ((err = alloc(&Ba_, 7 * nB_ * sizeof(Cplx<T>)))) return err;
    if (snapshots > 0 && (err = alloc(&snaps_, size_t(snapshots) * s4))) return err;
    if ((err = alloc(&ampsave_, 2 * kMaxStages * sizeof(double)))) return err;
    if ((err = alloc(&coef_, 4 * sizeof(double)))) return err;
    if ((err = alloc(&grad_, 2 * sizeof(double)))) return err;
    if (p_.tracers > 0) {
      const size_t m3 = 3 * size_t(p_.tracers) * sizeof(double);
      if ((err = alloc(&LX_, m3))) return err;
      if ((err = alloc(&LF_, m3))) return err;
      if ((err = alloc(&LU_, 3 * nP_ * sizeof(double)))) return err;
      if (snapshots > 0 && (err = alloc(&snapX_, size_t(snapshots) * 2 * m3))) return err;
    }
#ifndef GBGHT_EMU
    if ((err = make_maps_on(&maps_adj_, Aa_, Ba_))) return err;
#endif
    nsnap_ = snapshots;
    adj_ready_ = true;
    return rt_sync(stream_);
  }
  const char* adjoint_import(const double* lu, const double* lp, bool* outside) override {
    if (!adj_ready_) return "the adjoint is not set up";
    const int nc = p_.scalar ? 4 : 3;
    const size_t nref = ref_comp_elems();
    *outside = false;
    const int wu = where(lu), wp = nc == 4 ? where(lp) : 0;
    if (wu < 0 || wp < 0) return "an adjoint array is device memory of another device";
    bu_fresh_ = false;   // B is the host staging
    Cplx<double>* stage = reinterpret_cast<Cplx<double>*>(B_);
    const char* err = rt_memset(L_, 0, 4 * nS_ * sizeof(Cplx<T>), stream_);
    if (!err) err = rt_memset(flag_, 0, sizeof(unsigned int), stream_);
    for (int cc = 0; cc < nc && !err; ++cc) {
      const double* src = cc < 3 ? lu + size_t(cc) * nref * 2 : lp;
      const Cplx<double>* ref = reinterpret_cast<const Cplx<double>*>(src);
      if (!(cc < 3 ? wu : wp)) {
        if ((err = rt_h2d(stage, src, nref * sizeof(Cplx<double>), stream_))) break;
        ref = stage;
      }
#ifdef GBGHT_EMU
      for (size_t i = 0; i < nref; ++i) import_mode<T>(i, g_, ref, L_ + cc * nS_, flag_);
#else
      k_import<T><<<unsigned((nref + 255) / 256), 256, 0, stream_>>>(g_, ref, L_ + cc * nS_, flag_);
      err = rt_check();
#endif
    }
    unsigned int fl = 0;
    if (!err) err = rt_d2h(&fl, flag_, sizeof fl, stream_);
    if (err) return err;
    if (fl & 1u) {
      *outside = true;
      return rt_memset(L_, 0, 4 * nS_ * sizeof(Cplx<T>), stream_);
    }
    return rt_sync(stream_);
  }
  const char* adjoint_export(double* lu, double* lp) override {
    if (!adj_ready_) return "the adjoint is not set up";
    const size_t nref = ref_comp_elems();
    const int nc = (p_.scalar && lp) ? 4 : 3;
    const int wu = where(lu), wp = nc == 4 ? where(lp) : 0;
    if (wu < 0 || wp < 0) return "an adjoint array is device memory of another device";
    bu_fresh_ = false;
    Cplx<double>* stage = reinterpret_cast<Cplx<double>*>(B_);
    for (int cc = 0; cc < nc; ++cc) {
      double* dst = cc < 3 ? lu + size_t(cc) * nref * 2 : lp;
      const bool direct = (cc < 3 ? wu : wp) == 1;
      Cplx<double>* ref = direct ? reinterpret_cast<Cplx<double>*>(dst) : stage;
#ifdef GBGHT_EMU
      for (size_t i = 0; i < nref; ++i) export_mode<T>(i, g_, L_ + cc * nS_, ref);
#else
      k_export<T><<<unsigned((nref + 255) / 256), 256, 0, stream_>>>(g_, L_ + cc * nS_, ref);
      if (const char* e = rt_check()) return e;
#endif
      if (!direct)
        if (const char* e = rt_d2h(dst, ref, nref * sizeof(Cplx<double>), stream_)) return e;
    }
    return rt_sync(stream_);
  }
  const char* adjoint_add(double wu, double wp) override {
    if (!adj_ready_) return "the adjoint is not set up";
    const int nc = p_.scalar ? 4 : 3;
#ifdef GBGHT_EMU
    for (size_t i = 0; i < nS_; ++i) adj_add_mode<T>(i, nS_, nc, L_, S_, wu, wp);
#else
    k_adj_add<T><<<unsigned((nS_ + 255) / 256), 256, 0, stream_>>>(nS_, nc, L_, S_, wu, wp);
#endif
    return rt_check();
  }
  const char* adjoint_gradient(double* g2, int reset) override {
    if (!adj_ready_) return "the adjoint is not set up";
    if (const char* e = rt_d2h(g2, grad_, 2 * sizeof(double), stream_)) return e;
    return reset ? rt_memset(grad_, 0, 2 * sizeof(double), stream_) : nullptr;
  }
  const char* adjoint_clear() override {
    if (!adj_ready_) return "the adjoint is not set up";
    const char* e = rt_memset(L_, 0, 4 * nS_ * sizeof(Cplx<T>), stream_);
    if (!e) e = rt_memset(grad_, 0, 2 * sizeof(double), stream_);
    return e ? e : rt_sync(stream_);
  }
  const char* snapshot_save(int slot, int f_slot) override {
    if (slot < 0 || slot >= nsnap_) return "no such snapshot slot";
    const char* e = rt_d2d(snaps_ + size_t(slot) * 4 * nS_, S_, 4 * nS_ * sizeof(Cplx<T>), stream_);
    if (!e && X_ && snapX_) {
      const size_t m3 = 3 * size_t(p_.tracers);
      e = rt_d2d(snapX_ + size_t(slot) * 2 * m3, X_, m3 * sizeof(double), stream_);
      if (!e) e = rt_d2d(snapX_ + size_t(slot) * 2 * m3 + m3, F_ + size_t(f_slot) * m3, m3 * sizeof(double), stream_);
    }
    return e;
  }
  const char* snapshot_load(int slot, int f_slot) override {
    if (slot < 0 || slot >= nsnap_) return "no such snapshot slot";
    const char* e = rt_d2d(S_, snaps_ + size_t(slot) * 4 * nS_, 4 * nS_ * sizeof(Cplx<T>), stream_);
    if (!e && X_ && snapX_) {
      const size_t m3 = 3 * size_t(p_.tracers);
      e = rt_d2d(X_, snapX_ + size_t(slot) * 2 * m3, m3 * sizeof(double), stream_);
      if (!e) e = rt_d2d(F_ + size_t(f_slot) * m3, snapX_ + size_t(slot) * 2 * m3 + m3, m3 * sizeof(double), stream_);
    }
    if (!e) e = z_init();
    return e;
  }
  const char* adjoint_tracers_import(const double* lX, const double* lf) override {
    if (!adj_ready_ || !LX_) return "the adjoint of the tracers is not set up";
    const size_t m3 = 3 * size_t(p_.tracers) * sizeof(double);
    if (where(lX) < 0 || where(lf) < 0) return "a tracer cotangent is device memory of another device";
    const char* e = rt_copy(LX_, lX, m3, stream_);
    return e ? e : rt_copy(LF_, lf, m3, stream_);
  }
  const char* adjoint_tracers_export(double* lX, double* lf) override {
    if (!adj_ready_ || !LX_) return "the adjoint of the tracers is not set up";
    const size_t m3 = 3 * size_t(p_.tracers) * sizeof(double);
    if (where(lX) < 0 || where(lf) < 0) return "a tracer cotangent is device memory of another device";
    const char* e = rt_copy(lX, LX_, m3, stream_);
    return e ? e : rt_copy(lf, LF_, m3, stream_);
  }
  const char* adjoint_deposit_tracers() override {
    if (!adj_ready_ || !LX_) return "the adjoint of the tracers is not set up";
    tracer_adjoint(nullptr, 0);
    return rt_check();
  }

  // The reverse of one low-storage step at the current state q: the forward stages again, keeping
  // each stage's state and amplitudes; then, per stage in reverse, the stage's forward fields
  // (z- and y-inverse of the saved state), the adjoint x pass, its y-forward, the band coefficients
  // and the adjoint z pass; finally the state is put back.
  const char* adjoint_step(double dt, const double* a, const double* b, const double* d, int S, const AdamsStep* push,
                           int f_slot) override {
    if (!adj_ready_) return "the adjoint is not set up";
    if (push && !LX_) return "the adjoint of the tracers is not set up";
    if (S < 1 || S > kMaxStages) return "the adjoint needs a low-storage scheme";
    const size_t s4 = 4 * nS_;
    for (int i = 0; i < S; ++i) {
      if (const char* e = rt_d2d(Qs_ + i * s4, S_, s4 * sizeof(Cplx<T>), stream_)) return e;
      StageArgs st = stage_base(dt);
      st.kind = kLowStorage;
      st.a = a[i];
      st.b = b[i];
      st.first = i == 0;
      st.last = i == S - 1;
      st.read_h = !st.first;
      st.write_h = !st.last;
      set_factor(st, d[i] * dt, false);
      amp_save_to_ = ampsave_ + 2 * i;
      const char* e = stage(st);
      amp_save_to_ = nullptr;
      if (e) return e;
    }
    if (push) {   // the iteration's tracer part, reversed first: it ran last
      if (const char* e = deposit_launch()) return e;
      tracer_adjoint(push, f_slot);
    }
    const int nc = p_.scalar ? 4 : 3;
    const int ninv = p_.scalar ? 7 : 6, nsrc = p_.scalar ? 6 : 3, nprod = p_.scalar ? 7 : 6;
    // the end-of-step projections in reverse: the reality projection (self-adjoint), then the
    // start launch applies the Leray projection and opens the last stage
#ifdef GBGHT_EMU
    for (int i = 0; i < g_.NY2 * g_.NY2; ++i) reality_mode<T>(i, g_, L_, nc);
#else
    k_reality<T><<<(g_.NY2 * g_.NY2 + 255) / 256, 256, 0, stream_>>>(g_, L_, nc);
#endif
    AdjArgs base = adj_base(dt);
    AdjArgs st = base;
    st.combine = 0;
    st.prologue = 1;
    adj_factor(st, d[S - 1] * dt);
    st.b = b[S - 1];
    st.a_next = 0.0;
    adj_z(st, nullptr);
    for (int i = S - 1; i >= 0; --i) {
      if (const char* e = z_init(1, 0, Qs_ + i * s4)) return e;   // the stage's u, ω, φ
      y_inverse_on(0, ninv, maps_, A_, B_);
      y_inverse_on(0, nsrc, maps_adj_, Aa_, Ba_);
      x_adjoint();
      y_forward_on(nprod, maps_adj_, Ba_, Aa_);
      if (base.forced || base.sforced) adj_band(dt, i);
      st = base;
      st.combine = 1;
      st.prologue = i > 0;
      if (i > 0) {
        adj_factor(st, d[i - 1] * dt);
        st.b = b[i - 1];
        st.a_next = a[i];
      }
      adj_z(st, Qs_ + i * s4);
      if (const char* e = rt_check()) return e;
    }
    // the state as it was, its z-inverse in A, and its deposit (the tracers' part overwrote it)
    if (const char* e = rt_d2d(S_, Qs_, s4 * sizeof(Cplx<T>), stream_)) return e;
    if (const char* e = z_init()) return e;
    if (push)
      if (const char* e = deposit_launch()) return e;
    return rt_check();
  }

  const char* status(uint32_t* word) override {
    unsigned int v = 0;
    const char* err = rt_d2h(&v, status_, sizeof v, stream_);
    if (err) return err;
    *word = v;
    return rt_memset(status_, 0, sizeof v, stream_);
  }

 private:
  // ---- per-kernel CUDA-event timing (profile on) ---------------------------------------------------
#ifndef GBGHT_EMU
  struct Pending {
    int kind;
    cudaEvent_t a, b;
  };
  cudaEvent_t take_event() {
    if (!pool_.empty()) {
      cudaEvent_t e = pool_.back();
      pool_.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  void pbegin(int kind) {
    if (!prof_on_) return;
    cur_kind_ = kind;
    cur_a_ = take_event();
    cudaEventRecord(cur_a_, stream_);
  }
  void pend() {
    if (!prof_on_ || !cur_a_) return;
    cudaEvent_t b = take_event();
    cudaEventRecord(b, stream_);
    pending_.push_back(Pending{cur_kind_, cur_a_, b});
    cur_a_ = nullptr;
  }
  const char* collect() {
    if (pending_.empty()) return nullptr;
    const char* e = rt_sync(stream_);
    if (e) return e;
    for (auto& pr : pending_) {
      float f = 0.f;
      cudaEventElapsedTime(&f, pr.a, pr.b);
      prof_ms_[pr.kind] += double(f);
      prof_n_[pr.kind] += 1;
      pool_.push_back(pr.a);
      pool_.push_back(pr.b);
    }
    pending_.clear();
    return nullptr;
  }
  std::vector<Pending> pending_;
  std::vector<cudaEvent_t> pool_;
  cudaEvent_t cur_a_ = nullptr;
  int cur_kind_ = 0;
  cudaEvent_t timer_ev_[2] = {nullptr, nullptr};
#else
  void pbegin(int) {}
  void pend() {}
#endif
  bool prof_on_ = false;
  double prof_ms_[PROF_KINDS] = {};
  int64_t prof_n_[PROF_KINDS] = {};

  template <class P> const char* alloc(P** p, size_t n) {
    void* v = nullptr;
    const char* err = rt_alloc(&v, n);
    if (err) return err;
    allocs_.push_back(v);
    *p = static_cast<P*>(v);
    return nullptr;
  }

  // Squared edges of shells lowest..highest, shell h covering [h − ½, h + ½)·2π/L; an infinite
  // highest shell stands for the grid's corner shell ⌈√3 N/2⌉ (src/Forcing.jl:435-441).
  double shell_lo2(int lowest) const {
    const double lo = (lowest - 0.5) * g_.s;
    return lo * lo;
  }
  double shell_hi2(double highest) const {
    const double top = std::isfinite(highest) ? highest : std::ceil(std::sqrt(3.0) * N / 2.0);
    const double hi = (top + 0.5) * g_.s;
    return hi * hi;
  }
  double band_lo2() const { return shell_lo2(p_.vf.lowest_shell); }
  double band_hi2() const { return shell_hi2(p_.vf.highest_shell); }
  double sband_lo2() const { return shell_lo2(p_.sf.lowest_shell); }
  double sband_hi2() const { return shell_hi2(p_.sf.highest_shell); }
  // ConstantPower and VarianceController act through a per-stage source A·𝟙_band·f
  static bool stage_source(int kind) { return kind == kForceConstantPower || kind == kForceController; }
  AmpArgs amp_args(const ForcingParams& f, bool scalar) const {
    AmpArgs a{};
    a.kind = f.kind;
    a.rate = f.rate;
    a.target = f.target;
    a.gain = f.gain;
    a.turnover_time = f.turnover_time;
    a.over = f.over;
    a.factor = scalar ? 1.0 : 0.5;
    a.diffusivity = scalar ? p_.viscosity / p_.schmidt : p_.viscosity;
    a.eps_T = sizeof(T) == 8 ? DBL_EPSILON : double(FLT_EPSILON);
    return a;
  }

  static constexpr size_t kBarBytes = 32;
  // the adjoint's x pass (its lines) and z pass (the FFT tile and six retained-row components)
  size_t smem_xa() const { return size_t(XAdjShape<T>::NIN) * N * sizeof(Cplx<T>); }
  size_t smem_za() const { return (size_t(N) * TLZ + size_t(6) * g_.NY2 * TLZ) * sizeof(Cplx<T>); }
  size_t smem_y() const { return size_t(N) * TLY * sizeof(Cplx<T>) + kBarBytes; }
  size_t smem_x() const {
    return size_t(N) * XShape<T>::ACT_INV * sizeof(Cplx<T>) +
           (XShape<T>::STAGED ? size_t(7) * XShape<T>::P * x_kxs(g_.K, int(sizeof(Cplx<T>))) * sizeof(Cplx<T>) : 0) +
           kBarBytes;
  }
  size_t smem_xv() const {
    return size_t(N) * XShape<T>::ACT_V * sizeof(Cplx<T>) + size_t((NTXV + 1) & ~1) * sizeof(double) +
           size_t(3) * XShape<T>::PV * x_kxs(g_.K, int(sizeof(Cplx<T>))) * sizeof(Cplx<T>) + kBarBytes;
  }
  // z init: the FFT tile, NT doubles, the TMEM address
  size_t smem_z() const {
    return size_t(N) * TLZ * sizeof(Cplx<T>) + size_t(NTZ) * sizeof(double) + 16;
  }
  // z epilogue: the FFT tile, NT doubles, barriers, the TMEM address, the staging region
  // the wide instantiation stages at most four state components (H is read from global memory)
  size_t smem_ze() const { return ZLayout<T, N, TLZ, NTZ>::bytes(g_.K, DEA ? 4 : 6); }

#ifndef GBGHT_EMU
  const char* set_smem_attributes() {
    const char* e = nullptr;
    // The attribute belongs to the kernel, not to this run: runs of the same precision and N with
    // different retained bands (TwoThirds beside HouLi or PhaseShift) share kernels whose shared
    // memory grows with K, so the attribute is only ever raised, never lowered below what another
    // run's launches need.
    auto set = [&](const void* f, size_t bytes) {
      if (e) return;
      cudaFuncAttributes fa{};
      e = cuda_err(cudaFuncGetAttributes(&fa, f), "cudaFuncGetAttributes");
      if (!e && size_t(fa.maxDynamicSharedSizeBytes) < bytes)
        e = cuda_err(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)),
                     "cudaFuncSetAttribute");
    };
    set(reinterpret_cast<const void*>(k_y_inverse<T, N, TLY, NTY>), smem_y());
    set(reinterpret_cast<const void*>(k_y_forward<T, N, TLY, NTY>), smem_y());
    set(reinterpret_cast<const void*>(kg_y_inverse<T, N, TLY, NTY>), smem_y());
    set(reinterpret_cast<const void*>(kg_y_forward<T, N, TLY, NTY>), smem_y());
    set(reinterpret_cast<const void*>(kg_x_products<T, N, NTXP>), smem_x());
    set(reinterpret_cast<const void*>(kg_x_velocity<T, N, NTXV>), smem_xv());
    set(reinterpret_cast<const void*>(kg_z_epilogue<T, N, TLZ, NTZ, kLowStorage, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(kg_z_epilogue<T, N, TLZ, NTZ, kHeunPredictor, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(kg_z_epilogue<T, N, TLZ, NTZ, kHeunCorrector, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(kg_z_epilogue<T, N, TLZ, NTZ, kSsp1, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(kg_z_epilogue<T, N, TLZ, NTZ, kSsp2, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(kg_z_epilogue<T, N, TLZ, NTZ, kSsp3, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(kg_z_init_column<T, N, TLZ, NTZ, KM>), smem_z());
    set(reinterpret_cast<const void*>(k_x_products<T, N, NTXP>), smem_x());
    set(reinterpret_cast<const void*>(k_x_velocity<T, N, NTXV>), smem_xv());
    set(reinterpret_cast<const void*>(k_z_epilogue<T, N, TLZ, NTZ, kLowStorage, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(k_z_epilogue<T, N, TLZ, NTZ, kHeunPredictor, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(k_z_epilogue<T, N, TLZ, NTZ, kHeunCorrector, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(k_z_epilogue<T, N, TLZ, NTZ, kSsp1, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(k_z_epilogue<T, N, TLZ, NTZ, kSsp2, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(k_z_epilogue<T, N, TLZ, NTZ, kSsp3, KM, (DEA != 0)>), smem_ze());
    set(reinterpret_cast<const void*>(k_z_init<T, N, TLZ, NTZ, KM>), smem_z());
    set(reinterpret_cast<const void*>(k_z_shift_back<T, N, TLZ, NTZ, KM>), smem_z());
    set(reinterpret_cast<const void*>(k_x_adjoint<T, N, NTXA>), smem_xa());
    set(reinterpret_cast<const void*>(k_adj_z<T, N, TLZ, NTZA>), smem_za());
    set(reinterpret_cast<const void*>(k_phys_forward<T, N, 8>), size_t(8) * N * sizeof(Cplx<T>));
    return e;
  }

  // Tensor maps over A and B (see TmaMaps in passes.cuh), encoded through the driver entry point.
  const char* make_maps() { return make_maps_on(&maps_, A_, B_); }
  const char* make_maps_on(TmaMaps* mp, Cplx<T>* A, Cplx<T>* B) {
    TmaMaps& maps = *mp;
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    const char* e = cuda_err(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q),
                             "cudaGetDriverEntryPoint(cuTensorMapEncodeTiled)");
    if (e) return e;
    if (!fn || q != cudaDriverEntryPointSuccess) return "cuTensorMapEncodeTiled is unavailable";
    Encode encode = reinterpret_cast<Encode>(fn);
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const cuuint64_t inner = cuuint64_t(2) * g_.KXP;                // reals per row
    const cuuint64_t pitch = cuuint64_t(g_.KXP) * sizeof(Cplx<T>);  // bytes per row
    const cuuint32_t ones[3] = {1, 1, 1};
    auto map2 = [&](CUtensorMap* m, void* base, cuuint64_t rows, cuuint32_t bx, cuuint32_t by) -> bool {
      const cuuint64_t dims[2] = {inner, rows};
      const cuuint64_t strides[1] = {pitch};
      const cuuint32_t box[2] = {bx, by};
      return encode(m, dt, 2, base, dims, strides, box, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    const cuuint32_t bxy = 2 * TLY, bxz = 2 * TLZ;
    const cuuint32_t K1 = cuuint32_t(g_.K + 1), K0 = cuuint32_t(g_.K);
    const cuuint32_t BY = cuuint32_t(box_rows<N>());
    if (!map2(&maps.a_ld, A, cuuint64_t(7) * N * g_.NY2, bxy, K1)) return "tensor map a_ld";
    if (!map2(&maps.a_st1, A, cuuint64_t(7) * N * g_.NY2, bxy, K1)) return "tensor map a_st1";
    if (!map2(&maps.a_st2, A, cuuint64_t(7) * N * g_.NY2, bxy, K0)) return "tensor map a_st2";
    if (!map2(&maps.b, B, cuuint64_t(7) * N * N, bxy, BY)) return "tensor map b";
    {
      const cuuint64_t dims[3] = {inner, cuuint64_t(g_.NY2), cuuint64_t(7) * N};
      const cuuint64_t strides[2] = {pitch, pitch * g_.NY2};
      const cuuint32_t box[3] = {bxz, 1, BY};
      if (encode(&maps.az, dt, 3, A, dims, strides, box, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return "tensor map az";
    }
    for (int which = 0; which < 2; ++which) {   // s3 over S, h3 over H
      const cuuint64_t dims[3] = {inner, cuuint64_t(g_.NY2), cuuint64_t(4) * g_.NY2};
      const cuuint64_t strides[2] = {pitch, pitch * g_.NY2};
      const cuuint32_t box[3] = {bxz, K1, 1};
      if (encode(which == 0 ? &maps.s3 : &maps.h3, dt, 3, which == 0 ? S_ : H_, dims, strides, box, ones,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return which == 0 ? "tensor map s3" : "tensor map h3";
    }
    return nullptr;
  }
#endif

  // The y passes over an (A, B) pair: the run's own (A_, B_, maps_) or the adjoint's.
  void y_inverse(int c0, int nc) { y_inverse_on(c0, nc, maps_, A_, B_); }
  void y_forward(int nc) { y_forward_on(nc, maps_, B_, A_); }
  void y_inverse_on(int c0, int nc, const TmaMaps& m, Cplx<T>* A, Cplx<T>* B) {
#ifdef GBGHT_EMU
    (void)m;
    emu_grid(g_.KXP / TLY, N, nc, smem_y(), [&](const Cta& c, void* sm) {
      Cplx<T>* t = static_cast<Cplx<T>*>(sm);
      y_inverse_load_host<T, N, TLY>(c, t, g_, A, c0);
      y_inverse_compute<T, N, TLY, 1>(c, t, g_, tw_);
      y_store_host<T, N, TLY>(c, t, g_, B, c0 + c.bz);
    });
#else
    (void)A;
    (void)B;
    pbegin(PROF_Y_INVERSE);
    k_y_inverse<T, N, TLY, NTY><<<dim3(g_.KXP / TLY, N, nc), NTY, smem_y(), stream_>>>(m, g_, c0, tw_, status_);
    pend();
#endif
  }
  void y_forward_on(int nc, const TmaMaps& m, Cplx<T>* B, Cplx<T>* A) {
#ifdef GBGHT_EMU
    (void)m;
    emu_grid(g_.KXP / TLY, N, nc, smem_y(), [&](const Cta& c, void* sm) {
      Cplx<T>* t = static_cast<Cplx<T>*>(sm);
      y_forward_load_host<T, N, TLY>(c, t, g_, B);
      tile_fft<T, N, TLY, 1, -1>(c, t, tw_);
      y_forward_store_host<T, N, TLY>(c, t, g_, A);
    });
#else
    (void)A;
    (void)B;
    pbegin(PROF_Y_FORWARD);
    k_y_forward<T, N, TLY, NTY><<<dim3(g_.KXP / TLY, N, nc), NTY, smem_y(), stream_>>>(m, g_, tw_, status_);
    pend();
#endif
  }
  void x_products() {
    using X = XShape<T>;
    const int KXS = x_kxs(g_.K, int(sizeof(Cplx<T>)));
    const int ntiles = (N / X::P) * N;
    const int grid = (ntiles + XT - 1) / XT;   // XT tiles per CTA
#ifdef GBGHT_EMU
    emu_grid(grid, 1, 1, smem_x(), [&](const Cta& c, void* sm) {
      Cplx<T>* t = static_cast<Cplx<T>*>(sm);
      Cplx<T>* stg = t + N * X::ACT_INV;
      body_x_products<T, N, 1>(c, t, stg, KXS, nullptr, grid, g_, B_, p_.scalar, tw_, status_);
    });
#else
    pbegin(PROF_X_PRODUCTS);
    k_x_products<T, N, NTXP><<<grid, NTXP, smem_x(), stream_>>>(g_, B_, p_.scalar, KXS, tw_, status_);
    pend();
#endif
  }
  void x_velocity() { x_velocity_into(B_, U_, maxbits_); }
  // The deposit's x pass over three B slots starting at `src`: their c2r into `out` ([3][N³]) and
  // the max of the sum of their squares into `mb`.
  void x_velocity_into(const Cplx<T>* src, T* out, unsigned long long* mb_out) {
    using X = XShape<T>;
    const int KXS = x_kxs(g_.K, int(sizeof(Cplx<T>)));
    const int ntiles = (N / X::PV) * N;
    const int grid = (ntiles + XT - 1) / XT;   // XT tiles per CTA
#ifdef GBGHT_EMU
    unsigned long long* mb = mb_out;
    emu_grid(grid, 1, 1, smem_xv(), [&](const Cta& c, void* sm) {
      Cplx<T>* t = static_cast<Cplx<T>*>(sm);
      double* red = reinterpret_cast<double*>(t + N * X::ACT_V);
      Cplx<T>* stg = reinterpret_cast<Cplx<T>*>(red + 2);   // NT = 1 double, padded to 16 bytes
      const double m = body_x_velocity<T, N, 1>(c, t, red, stg, KXS, nullptr, grid, g_, src, out, tw_, status_);
      unsigned long long bits;
      std::memcpy(&bits, &m, sizeof bits);
      if (bits > *mb) *mb = bits;
    });
#else
    pbegin(PROF_X_VELOCITY);
    k_x_velocity<T, N, NTXV><<<grid, NTXV, smem_xv(), stream_>>>(g_, src, out, mb_out, KXS, tw_, status_);
    pend();
#endif
  }
  void z_epilogue(const StageArgs& st) {
    switch (st.kind) {   // one instantiation per stage kind
      case kHeunPredictor: return z_epilogue_kind<kHeunPredictor>(st);
      case kHeunCorrector: return z_epilogue_kind<kHeunCorrector>(st);
      case kSsp1: return z_epilogue_kind<kSsp1>(st);
      case kSsp2: return z_epilogue_kind<kSsp2>(st);
      case kSsp3: return z_epilogue_kind<kSsp3>(st);
      default: return z_epilogue_kind<kLowStorage>(st);
    }
  }
  template <int KIND>
  void z_epilogue_kind(const StageArgs& st) {
#ifdef GBGHT_EMU
    const int gx = g_.KXP / TLZ;
    emu_grid(gx, g_.NY2, 1, ZLayout<T, N, TLZ, 1>::bytes(g_.K, DEA ? 4 : 6), [&](const Cta& c, void* sm) {
      using L = ZLayout<T, N, TLZ, 1>;
      unsigned char* base = static_cast<unsigned char*>(sm);
      Cplx<T>* W = reinterpret_cast<Cplx<T>*>(base);
      double* red = reinterpret_cast<double*>(base + L::kRed);
      Cplx<T>* R = reinterpret_cast<Cplx<T>*>(base + L::kStage);
      ZRowsReg<T, ZOwn<T, N, TLZ, 1, KM>> rows;
      partial_[c.by * gx + c.bx] =
          body_z_epilogue<T, N, TLZ, 1, KIND, (DEA != 0)>(c, W, R, nullptr, red, g_, maps_, rows, A_, S_, H_, st, amp_, tw_, status_);
    });
#else
    pbegin(PROF_Z_EPILOGUE);
    k_z_epilogue<T, N, TLZ, NTZ, KIND, KM, (DEA != 0)><<<dim3(g_.KXP / TLZ, g_.NY2, 1), NTZ, smem_ze(), stream_>>>(
        maps_, g_, A_, S_, H_, st, amp_, partial_, tw_, status_);
    pend();
#endif
  }
  // The z-inverse of the state into the A slots (u, iκ×û, φ), or with `vorticity` = 2 of the six
  // strain components into slots 0..5.
  // `columns` = 1 rebuilds only the first tile column (kx = 0..TLZ−1) and its partial sums.
  // `from` replaces the state by another S-layout array (a saved stage state of the adjoint).
  const char* z_init(int vorticity = 1, int columns = 0, const Cplx<T>* from = nullptr) {
    const Cplx<T>* Ssrc = from ? from : S_;
    bu_fresh_ = false;   // A is rewritten
    const int with_scalar = vorticity == 2 ? 0 : p_.scalar;
    const int gx = g_.KXP / TLZ, gl = columns ? columns : gx;
#ifdef GBGHT_EMU
    emu_grid(gl, g_.NY2, 1, smem_z(), [&](const Cta& c, void* sm) {
      Cplx<T>* W = static_cast<Cplx<T>*>(sm);
      double* red = reinterpret_cast<double*>(W + N * TLZ);
      ZRowsReg<T, ZOwn<T, N, TLZ, 1, KM>> rows;
      partial_[c.by * gx + c.bx] =
          body_z_init<T, N, TLZ, 1>(c, W, red, g_, rows, A_, Ssrc, with_scalar, tw_, vorticity);
    });
#else
    k_z_init<T, N, TLZ, NTZ, KM><<<dim3(gl, g_.NY2, 1), NTZ, smem_z(), stream_>>>(g_, A_, Ssrc, with_scalar, partial_,
                                                                            tw_, vorticity, gx);
#endif
    return rt_check();
  }
  // ---- PhaseShift (src/Generator.jl:502-519,668-704) -------------------------------------------------
  // The stage's second evaluation, on the grid displaced by half a cell along every axis: the state's
  // fields there (z-inverse with the translation), their products through the same y and x passes
  // (B is free again once the primary y-forward has read it), and the shift back averaged into the
  // primary products in A.
  void displaced(int ninv, int nfwd) {
    const int gx = g_.KXP / TLZ;
#ifdef GBGHT_EMU
    emu_grid(gx, g_.NY2, 1, smem_z(), [&](const Cta& c, void* sm) {
      Cplx<T>* W = static_cast<Cplx<T>*>(sm);
      double* red = reinterpret_cast<double*>(W + N * TLZ);
      ZRowsReg<T, ZOwn<T, N, TLZ, 1, KM>> rows;
      body_z_init<T, N, TLZ, 1>(c, W, red, g_, rows, A2_, S_, p_.scalar, tw_, 1, 1);
    });
#else
    pbegin(PROF_Z_SHIFT);
    k_z_init<T, N, TLZ, NTZ, KM><<<dim3(gx, g_.NY2, 1), NTZ, smem_z(), stream_>>>(g_, A2_, S_, p_.scalar, nullptr,
                                                                            tw_, 1, 0, 1);
    pend();
#endif
    y_inverse_on(0, ninv, maps_ps_, A2_, B_);
    x_products();
    y_forward_on(nfwd, maps_ps_, B_, A2_);
#ifdef GBGHT_EMU
    emu_grid(gx, g_.NY2, 1, smem_z(), [&](const Cta& c, void* sm) {
      body_z_shift_back<T, N, TLZ, 1, ZOwn<T, N, TLZ, 1, KM>>(c, static_cast<Cplx<T>*>(sm), g_, A_, A2_, nfwd, tw_);
    });
#else
    pbegin(PROF_Z_SHIFT);
    k_z_shift_back<T, N, TLZ, NTZ, KM><<<dim3(gx, g_.NY2, 1), NTZ, smem_z(), stream_>>>(g_, A_, A2_, nfwd, tw_);
    pend();
#endif
  }
  // ---- adjoint launches -------------------------------------------------------------------------------
  // The tracers' adjoint at the deposited field U: the Heun push and closing deposit (w, the sample
  // before the push in trail slot f_slot) or, with w = nullptr, the particle deposit alone; then
  // λ_u += rfft(λ_u physical)/N³ on the ball.
  void tracer_adjoint(const AdamsStep* w, int f_slot) {
    const int64_t M = p_.tracers;
    const double* f0 = F_ + size_t(f_slot) * 3 * size_t(M);
    rt_memset(LU_, 0, 3 * nP_ * sizeof(double), stream_);
    const int push = w ? 1 : 0;
    const double b0 = w ? w->b[0] : 0.0, bs = w ? w->beta_star : 0.0, bm = w ? w->beta_m[0] : 0.0;
    constexpr int NWP = 8;
#ifdef GBGHT_EMU
    for (int64_t p = 0; p < M; ++p) tracer_adjoint_one<T>(p, M, U_, LU_, N, p_.L, X_, f0, LX_, LF_, push, b0, bs, bm);
    const int npairs = 3 * N * (N / 2);
    emu_grid((npairs + NWP - 1) / NWP, 1, 1, size_t(NWP) * N * sizeof(Cplx<T>), [&](const Cta& c, void* sm) {
      body_phys_forward<T, N, NWP, 1>(c, static_cast<Cplx<T>*>(sm), g_, LU_, Ba_, tw_);
    });
#else
    pbegin(PROF_TRACERS);
    k_tracer_adjoint<T><<<unsigned((M + 127) / 128), 128, 0, stream_>>>(M, U_, LU_, N, p_.L, X_, f0, LX_, LF_, push, b0,
                                                                        bs, bm);
    pend();
    const int npairs = 3 * N * (N / 2);
    pbegin(PROF_X_ADJOINT);
    k_phys_forward<T, N, NWP><<<unsigned((npairs + NWP - 1) / NWP), 32 * NWP, size_t(NWP) * N * sizeof(Cplx<T>),
                                stream_>>>(g_, LU_, Ba_, tw_);
    pend();
#endif
    y_forward_on(3, maps_adj_, Ba_, Aa_);
    AdjArgs a{};
    a.add_only = 1;
    adj_z(a, nullptr);
  }
  AdjArgs adj_base(double dt) const {
    AdjArgs a{};
    a.has_scalar = p_.scalar;
    a.dt = dt;
    for (int k = 0; k < 3; ++k) a.G[k] = p_.G[k];
    a.forced = p_.vf.kind == kForceConstantPower;
    a.sforced = p_.scalar && p_.sf.kind == kForceConstantPower;
    a.band_lo2 = band_lo2();
    a.band_hi2 = band_hi2();
    a.sband_lo2 = sband_lo2();
    a.sband_hi2 = sband_hi2();
    return a;
  }
  // the integrating factor of a span δ, as the forward stage's (set_factor)
  void adj_factor(AdjArgs& a, double delta) const {
    StageArgs st{};
    set_factor(st, delta, false);
    a.cu = st.cu;
    a.cphi = st.cphi;
    a.lin_u = st.lin_u;
    a.lin_phi = st.lin_phi;
  }
  void x_adjoint() {
    using X = XAdjShape<T>;
    const int ntiles = (N / X::P) * N;
#ifdef GBGHT_EMU
    emu_grid(ntiles, 1, 1, smem_xa(), [&](const Cta& c, void* sm) {
      body_x_adjoint<T, N, 1>(c, static_cast<Cplx<T>*>(sm), g_, B_, Ba_, p_.scalar, tw_);
    });
#else
    pbegin(PROF_X_ADJOINT);
    k_x_adjoint<T, N, NTXA><<<ntiles, NTXA, smem_xa(), stream_>>>(g_, B_, Ba_, p_.scalar, tw_);
    pend();
#endif
  }
  void adj_z(const AdjArgs& a, const Cplx<T>* Q) {
#ifdef GBGHT_EMU
    emu_grid(g_.KXP / TLZ, g_.NY2, 1, smem_za(), [&](const Cta& c, void* sm) {
      Cplx<T>* W = static_cast<Cplx<T>*>(sm);
      body_adj_z<T, N, TLZ, 1>(c, W, W + N * TLZ, g_, a, Aa_, L_, LH_, Q, coef_, tw_);
    });
#else
    pbegin(PROF_Z_ADJOINT);
    k_adj_z<T, N, TLZ, NTZA><<<dim3(g_.KXP / TLZ, g_.NY2, 1), NTZA, smem_za(), stream_>>>(g_, a, Aa_, L_, LH_, Q,
                                                                                        coef_, tw_);
    pend();
#endif
  }
  // stage i's ConstantPower coefficients from its saved state and amplitudes and λ_h in LH
  void adj_band(double dt, int i) {
    AdjBandArgs a{};
    a.dt = dt;
    a.n6 = double(N) * N * N * double(N) * N * N;
    a.lo2 = band_lo2();
    a.hi2 = band_hi2();
    a.slo2 = sband_lo2();
    a.shi2 = sband_hi2();
    a.eps_u = p_.vf.kind == kForceConstantPower ? p_.vf.rate : 0.0;
    a.eps_p = p_.scalar && p_.sf.kind == kForceConstantPower ? p_.sf.rate : 0.0;
    const Cplx<T>* Q = Qs_ + size_t(i) * 4 * nS_;
    const double* amp = ampsave_ + 2 * i;
#ifdef GBGHT_EMU
    double su = 0.0, sp = 0.0;
    if (a.eps_u != 0.0) {
      const int mb = band_box_side(g_, a.hi2), side = 2 * mb + 1, n = 3 * side * side * (mb + 1);
      for (int k = 0; k < n; ++k) su += band_pair_term<T>(g_, Q, LH_, 0, mb, a.lo2, a.hi2, k);
    }
    if (a.eps_p != 0.0) {
      const int mb = band_box_side(g_, a.shi2), side = 2 * mb + 1, n = side * side * (mb + 1);
      for (int k = 0; k < n; ++k) sp += band_pair_term<T>(g_, Q, LH_, 3, mb, a.slo2, a.shi2, k);
    }
    adj_band_finish(a, amp, su, sp, coef_, grad_);
#else
    pbegin(PROF_FORCE_AMP);
    k_adj_band<T><<<1, 256, 0, stream_>>>(g_, Q, LH_, a, amp, coef_, grad_);
    pend();
#endif
  }
  // StochasticOU's force into the y-forward products (inject_source)
  void inject() {
    SourceArgs a{};
    a.nc = src_nc_[0] ? src_nc_[0] : src_nc_[1];
    if (src_[0] && src_[1] && src_nc_[0] != src_nc_[1]) {   // two companions of different sizes
      SourceArgs b{};
      b.nc = src_nc_[1];
      b.sca = 1;
      b.slo2 = sband_lo2();
      b.shi2 = sband_hi2();
      inject_launch(b);
      a.nc = src_nc_[0];
      a.vel = 1;
    } else {
      a.vel = src_[0] != nullptr;
      a.sca = src_[1] != nullptr;
      a.slo2 = sband_lo2();
      a.shi2 = sband_hi2();
    }
    a.lo2 = band_lo2();
    a.hi2 = band_hi2();
    inject_launch(a);
  }
  void inject_launch(const SourceArgs& a) {
    const long n = long(a.nc - 1) * (a.nc / 2) * N;
#ifdef GBGHT_EMU
    for (long t = 0; t < n; ++t) inject_source<T>(t, g_, A_, src_[0], src_[1], a);
#else
    pbegin(PROF_FORCE_AMP);
    k_inject_source<T><<<unsigned((n + 255) / 256), 256, 0, stream_>>>(g_, A_, src_[0], src_[1], a);
    pend();
#endif
  }
  void reality() {
    const int n = g_.NY2 * g_.NY2;
    const int nc = p_.scalar ? 4 : 3;
#ifdef GBGHT_EMU
    for (int i = 0; i < n; ++i) reality_mode<T>(i, g_, S_, nc);
#else
    pbegin(PROF_REALITY);
    k_reality<T><<<(n + 255) / 256, 256, 0, stream_>>>(g_, S_, nc);
    pend();
#endif
  }
  // The observables' row sums of the state into fobs_ (mode 0 velocity, 1 both, 2 scalar), for the
  // band forcings that read the whole field's variance and dissipation.
  void row_sums(int mode) {
#ifdef GBGHT_EMU
    emu_grid(g_.NY2, 1, 1, 4 * sizeof(double), [&](const Cta& c, void* sm) {
      body_observables<T, 1>(c, static_cast<double*>(sm), g_, S_, mode, fobs_);
    });
#else
    pbegin(PROF_OBSERVABLES);
    k_observables<T, NTR><<<g_.NY2, NTR, 4 * NTR * sizeof(double), stream_>>>(g_, S_, mode, fobs_);
    pend();
#endif
  }
  // One field's amplitude (or rescale factor) into out[0..2]; see k_force_amp.
  void amp_launch(const AmpArgs& a, int c0, int nc, const double* whole, const double* dir, int nwhole, int stride,
                  double lo2, double hi2, double* out) {
#ifdef GBGHT_EMU
    // the same association as the device tree: 256 strided partial sums, then pairwise halving
    double red[256], dred[256];
    for (int t = 0; t < 256; ++t) {
      double s = 0.0, d = 0.0;
      for (int i = t; i < nwhole; i += 256) {
        s += whole[size_t(i) * stride];
        if (dir) d += dir[size_t(i) * stride];
      }
      red[t] = s;
      dred[t] = d;
    }
    for (int w = 128; w > 0; w >>= 1)
      for (int t = 0; t < w; ++t) {
        red[t] += red[t + w];
        dred[t] += dred[t + w];
      }
    const double band = band_energy_raw<T>(g_, S_, lo2, hi2, c0, nc);
    const double n6 = double(N) * N * N * double(N) * N * N;
    bool empty;
    out[0] = forcing_amplitude(a, red[0], band, dred[0], n6, &out[1], &out[2], &empty);
    if (empty) *status_ |= 0x2u;
#else
    pbegin(PROF_FORCE_AMP);
    k_force_amp<T><<<1, 256, 0, stream_>>>(g_, S_, c0, nc, whole, dir, nwhole, stride, lo2, hi2, a, out, status_);
    pend();
#endif
  }
  // The per-stage amplitudes at the stage state: the velocity's in amp_[0], the scalar's in amp_[4].
  // The velocity's ConstantPower takes its whole-field sum from the previous epilogue's tile
  // partials; every other source reads the observables' row sums.
  void force_amp(const StageArgs& st) {
    const bool vrows = st.forced && p_.vf.kind != kForceConstantPower;
    if (vrows || st.sforced) row_sums(vrows ? (st.sforced ? 1 : 0) : 2);
    if (st.forced) {
      if (vrows)
        amp_launch(amp_args(p_.vf, false), 0, 3, fobs_, fobs_ + 1, g_.NY2, 4, band_lo2(), band_hi2(), amp_);
      else
        amp_launch(amp_args(p_.vf, false), 0, 3, partial_, nullptr, int(ntile_), 1, band_lo2(), band_hi2(), amp_);
    }
    if (st.sforced)
      amp_launch(amp_args(p_.sf, true), 3, 1, fobs_ + 2, fobs_ + 3, g_.NY2, 4, sband_lo2(), sband_hi2(), amp_ + 4);
  }
  // VarianceRescaling after the last stage (`finalize!`, src/Generator.jl:396-400): the factor from
  // the end-of-step state, then the band's rescale; velocity first, then the scalar.
  void rescale(int c0, int nc, double lo2, double hi2, const double* factor) {
    int mb = int(std::sqrt(hi2) / g_.s) + 1;
    if (mb > g_.K) mb = g_.K;
    const long side = 2 * mb + 1, nbox = long(nc) * side * side * (mb + 1);
#ifdef GBGHT_EMU
    if (factor[0] != 1.0)
      for (long i = 0; i < nbox; ++i) rescale_mode<T>(i, g_, S_, c0, mb, lo2, hi2, factor[0]);
#else
    const long blocks = std::min<long>((nbox + 255) / 256, long(sm_count_) * 8);
    pbegin(PROF_FORCE_AMP);
    k_rescale<T><<<unsigned(blocks), 256, 0, stream_>>>(g_, S_, c0, nc, lo2, hi2, factor);
    pend();
#endif
  }
  // Returns whether a field was rescaled (the A slots then no longer hold its z-inverse).
  bool project() {
    const bool v = p_.vf.kind == kForceRescaling, s = p_.sf.kind == kForceRescaling;
    if (!v && !s) return false;
    row_sums(v ? (s ? 1 : 0) : 2);
    if (v) {
      amp_launch(amp_args(p_.vf, false), 0, 3, fobs_, nullptr, g_.NY2, 4, band_lo2(), band_hi2(), amp_ + 8);
      rescale(0, 3, band_lo2(), band_hi2(), amp_ + 8);
    }
    if (s) {
      amp_launch(amp_args(p_.sf, true), 3, 1, fobs_ + 2, nullptr, g_.NY2, 4, sband_lo2(), sband_hi2(), amp_ + 12);
      rescale(3, 1, sband_lo2(), sband_hi2(), amp_ + 12);
    }
    return true;
  }
  const char* stage(const StageArgs& st) {
    const int ninv = p_.scalar ? 7 : 6;
    const int nfwd = p_.scalar ? 6 : 3;
    // B slots 0..2 still hold the deposit's y-inverse of the same A slots at a step's first stage
    if (st.first && bu_fresh_) y_inverse(3, ninv - 3);
    else y_inverse(0, ninv);
    bu_fresh_ = false;
    x_products();
    y_forward(nfwd);
    if (phase_) displaced(ninv, nfwd);
    if (src_[0] || src_[1]) inject();
    if (st.forced || st.sforced) force_amp(st);
    if (amp_save_to_) {   // the adjoint's forward pass keeps the stage's amplitudes
      const char* e = rt_d2d(amp_save_to_, amp_, sizeof(double), stream_);
      if (!e) e = rt_d2d(amp_save_to_ + 1, amp_ + 4, sizeof(double), stream_);
      if (e) return e;
    }
    z_epilogue(st);
    if (st.last) {
      const bool rescaled = project();
      reality();
      // The last epilogue left the z-inverse of the unrescaled state in A; the deposit and the next
      // stage read A, so it is rebuilt from the rescaled state. The reality projection changes only
      // the kx = 0 plane's anti-Hermitian part, which the real inverse does not see in exact
      // arithmetic but does see at round-off; the first tile column of A (and its energy partial)
      // is rebuilt from the projected state, so A is exactly what an import of the end-of-step
      // state builds, and a run restored from a checkpoint continues this one bit for bit.
      if (rescaled) return z_init();
      return z_init(1, 1);
    }
    return rt_check();
  }
  void run_tracers(int64_t M, double* X, double* F, const AdamsStep& w, const uint32_t* order = nullptr) {
#ifdef GBGHT_EMU
    for (int64_t i = 0; i < M; ++i) tracer_one<T>(order ? int64_t(order[i]) : i, M, U_, N, p_.L, X, F, w);
#else
    const int bs = 128;
    pbegin(PROF_TRACERS);
    // Catmull–Rom, warp-cooperative (16 lanes per tracer): chosen, or automatic in FP64 with sparse
    // tracers (under one per 50 grid points), where it is the faster: 1.25 against 1.27 ms per
    // 10⁶-tracer push at 512³ (one per 134 points). With dense tracers the per-tracer form's warps
    // share cache lines and win (10⁶ at 256³, one per 17 points), and in FP32 it wins at 512³ too
    // (0.91 against 1.14 ms).
    const bool sparse = double(M) * 50.0 < double(N) * double(N) * double(N);
    const bool warp = p_.tracer_gather == 2 || (p_.tracer_gather == 0 && sizeof(T) == 8 && sparse);
    if (w.stencil.n == 0 && warp) {
      const int64_t threads = 16 * M;
      k_tracers_group<T><<<unsigned((threads + 255) / 256), 256, 0, stream_>>>(M, U_, N, p_.L, X, F, w, order);
    } else {
      k_tracers<T><<<unsigned((M + bs - 1) / bs), bs, 0, stream_>>>(M, U_, N, p_.L, X, F, w, order);
    }
    pend();
#endif
  }
  // The traversal order of the run's tracers from their current positions (rebuilt before every
  // tracer pass, as the reference's automatic mode does each iteration).
  const char* rebuild_traversal() {
    const int64_t M = p_.tracers;
    const double dx = div_rn(p_.L, double(N));
    const char* err = rt_memset(tcount_, 0, size_t(nbins_) * sizeof(uint32_t), stream_);
    if (err) return err;
#ifdef GBGHT_EMU
    for (int64_t p = 0; p < M; ++p) {
      tkey_[p] = traversal_key(X_, p, M, N, dx);
      ++tcount_[tkey_[p]];
    }
    uint32_t run = 0;
    for (int b = 0; b < nbins_; ++b) {
      const uint32_t c = tcount_[b];
      tcount_[b] = run;
      run += c;
    }
    for (int64_t p = 0; p < M; ++p) torder_[tcount_[tkey_[p]]++] = uint32_t(p);
#else
    const unsigned grid = unsigned((M + 255) / 256);
    pbegin(PROF_TRAVERSAL);
    k_trav_count<<<grid, 256, 0, stream_>>>(M, X_, N, dx, tkey_, tcount_);
    pend();
    pbegin(PROF_TRAVERSAL);
    k_trav_scan<<<1, kScanThreads, 0, stream_>>>(tcount_, nbins_);
    pend();
    pbegin(PROF_TRAVERSAL);
    k_trav_scatter<<<grid, 256, 0, stream_>>>(M, tkey_, tcount_, torder_);
    pend();
#endif
    return rt_check();
  }

  RunParams p_{};
  Geometry g_{};
  TmaMaps maps_{};
  double cutoff_ = 0.0;
  size_t nS_ = 0, nA_ = 0, nB_ = 0, nP_ = 0, ntile_ = 0;
  int nshell_ = 0;
  int sm_count_ = 4;
  bool bu_fresh_ = false;   // B slots 0..2 = y-inverse of the current A slots 0..2 (set by the deposit)
  Stream stream_ = nullptr;
  std::vector<void*> allocs_;
  Cplx<T>*S_ = nullptr, *H_ = nullptr, *A_ = nullptr, *B_ = nullptr, *tw_ = nullptr;
  T* U_ = nullptr;
  double *partial_ = nullptr, *amp_ = nullptr, *obs_ = nullptr, *fobs_ = nullptr, *spec_ = nullptr;
  double *X_ = nullptr, *F_ = nullptr;
  unsigned long long* maxbits_ = nullptr;
  unsigned int* status_ = nullptr;
  unsigned int* flag_ = nullptr;     // import: content outside the retained ball
  uint32_t *tkey_ = nullptr, *torder_ = nullptr, *tcount_ = nullptr;   // the traversal sort
  int nbins_ = 0;
  Cplx<double>* src_[2] = {nullptr, nullptr};   // StochasticOU: each field's companion force
  int src_nc_[2] = {0, 0};
  // the adjoint (allocated by adjoint_init): λ and λ_h, the saved stage states and amplitudes, the
  // adjoint A and B slots with their tensor maps, the band coefficients, the rates' gradients, the
  // snapshot slots
  bool adj_ready_ = false;
  int nsnap_ = 0;
  Cplx<T>*L_ = nullptr, *LH_ = nullptr, *Qs_ = nullptr, *Aa_ = nullptr, *Ba_ = nullptr, *snaps_ = nullptr;
  double *ampsave_ = nullptr, *coef_ = nullptr, *grad_ = nullptr;
  double* amp_save_to_ = nullptr;
  TmaMaps maps_adj_{};
  // PhaseShift: the displaced grid's A-layout array (its z-inverse fields, then its y-forward
  // products) and the y passes' maps over it and B
  bool phase_ = false;
  Cplx<T>* A2_ = nullptr;
  TmaMaps maps_ps_{};
#ifndef GBGHT_EMU
  // a member-batched group led by this run: the members' launch records on the device, the
  // members, the step's stages
  GroupMember<T>* grp_ = nullptr;
  size_t grp_bytes_ = 0;
  std::vector<EngineImpl*> grp_members_;
  StageArgs grp_st_[kStepStages]{};
  int grp_nst_ = 0;
#endif
  double *LX_ = nullptr, *LF_ = nullptr, *LU_ = nullptr, *snapX_ = nullptr;   // the tracers' adjoint
};

#if defined(GBGHT_UNIT_FACTORY)
template <class T, int N, int DEA> Engine* new_engine();   // defined in the per-(T, N, dealiasing) units
#else
template <class T, int N, int DEA>
Engine* new_engine() {
  return new EngineImpl<T, N, DEA>();
}
#endif

#if defined(GBGHT_UNIT_T) && defined(GBGHT_UNIT_N)
// one (precision, N, dealiasing) per translation unit, so the library's kernels compile in parallel
#ifndef GBGHT_UNIT_D
#define GBGHT_UNIT_D 0
#endif
template Engine* new_engine<GBGHT_UNIT_T, GBGHT_UNIT_N, GBGHT_UNIT_D>();
#endif

#if !defined(GBGHT_UNIT_T)
bool supported_N(int N) {
  switch (N) {
    case 8: case 12: case 16: case 24: case 32: case 48: case 64: case 96: case 128: case 192:
    case 256: case 384: case 512:
      return true;
    default:
      return false;
  }
}

template <class T, int D>
static Engine* make_for(int N) {
  switch (N) {
    case 8: return new_engine<T, 8, D>();
    case 12: return new_engine<T, 12, D>();
    case 16: return new_engine<T, 16, D>();
    case 24: return new_engine<T, 24, D>();
    case 32: return new_engine<T, 32, D>();
    case 48: return new_engine<T, 48, D>();
    case 64: return new_engine<T, 64, D>();
    case 96: return new_engine<T, 96, D>();
    case 128: return new_engine<T, 128, D>();
    case 192: return new_engine<T, 192, D>();
    case 256: return new_engine<T, 256, D>();
    case 384: return new_engine<T, 384, D>();
    case 512: return new_engine<T, 512, D>();
    default: return nullptr;
  }
}

Engine* make_engine(int N, int precision, int dealias, std::string* err) {
  if (!supported_N(N)) {
    *err = "grid_points_per_axis must be one of 8 12 16 24 32 48 64 96 128 192 256 384 512";
    return nullptr;
  }
  Engine* e = nullptr;
  // HouLi and PhaseShift share the wide instantiation (the box up to the Nyquist planes)
  if (dealias == 1 || dealias == 2) e = precision == 1 ? make_for<float, 1>(N) : make_for<double, 1>(N);
  else e = precision == 1 ? make_for<float, 0>(N) : make_for<double, 0>(N);
  if (!e) *err = "unsupported configuration";
  return e;
}
#endif

}  // namespace gbght
