// An allocation-free form of the deposit's velocity recovery (include/gbght.h,
// gbght_velocity_physical_noalloc).
//
// Who needs it: a caller whose device memory is owned by another allocator cannot call cudaMalloc.
// One example is a host framework whose memory pool has reserved the device, such as the caching
// allocators of Julia's CUDA.jl or of PyTorch configured to take the whole GPU. Another is a loop
// that keeps the reference's rule of no field-scale allocation inside a step
// (docs/ARCHITECTURE.md:921-930 of the reference). Such a caller owns the input spectrum and the
// output field and hands them in. Every intermediate lives here, in one file-scope
// __device__ array of kScratchBytes, which each GPU that loads the library holds until the
// process exits. This path calls no cudaMalloc, no cudaFree, and no routine that allocates; on the
// host it uses static storage only (the twiddle table and the per-device set-up below).
//
// The array is shared by every call on a device and keeps the contents of the last call. Each call
// clears what must start at zero: the compact spectrum, the maximum and the flag word. Two calls
// whose work overlaps on the GPU (on different streams, or from different host threads) race on
// the array. Serialise them.
//
// Set-up, per device: the first call looks up the array's device address with
// cudaGetSymbolAddress (in host code the array's name stands for a host-side shadow, not a device
// address, so it is never passed to a kernel directly). The tensor maps of the y pass and the
// twiddle table in the array are rebuilt only when a call's grid differs from the previous call's
// on that device. Every call synchronises its stream once, to read back max|u| and the flag word,
// so no call can be made inside a stream capture.
#include "../../include/gbght.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "kernels.cuh"

namespace gbght {
void set_global_error(const std::string& msg);   // gbght_capi.cu
}

namespace {

using gbght::Cplx;
using gbght::Geometry;

// Large enough for the largest supported grid, N = 64 in FP64 (about 10 MB in use).
constexpr size_t kScratchBytes = size_t(12) << 20;
constexpr int kMaxN = 64;
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

int fail(int code, const std::string& m) {
  gbght::set_global_error(m);
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  return fail(GBGHT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// The scratch layout for one N, in bytes from the array's start (each region 256-byte aligned).
struct Layout {
  Geometry g;
  size_t tw, S, A, B, partial, maxbits, flag, end;
};

size_t up256(size_t v) { return (v + 255) & ~size_t(255); }

Layout layout_for(int N, double L) {
  Layout o{};
  Geometry& g = o.g;
  const double s = 2.0 * M_PI / L;
  const double cutoff = (2.0 / 3.0) * (double(N) / 2.0) * s;
  g.N = N;
  g.s = s;
  g.cut2 = cutoff * cutoff;
  int K = 0;
  while (K + 1 < N / 2 + 1 && (s * (K + 1)) * (s * (K + 1)) <= g.cut2) ++K;
  g.K = K;
  g.NY2 = 2 * K + 1;
  constexpr int TLY = 128 / int(sizeof(Cplx<double>));
  g.KXP = ((K + 1 + TLY - 1) / TLY) * TLY;
  g.inv_norm = 1.0 / (double(N) * N * N);
  const size_t c = sizeof(Cplx<double>);
  size_t at = 0;
  o.tw = at;
  at = up256(at + size_t(N) * c);
  o.S = at;
  at = up256(at + size_t(3) * g.NY2 * g.NY2 * g.KXP * c);
  o.A = at;
  at = up256(at + size_t(3) * N * g.NY2 * g.KXP * c);
  o.B = at;
  at = up256(at + size_t(3) * N * N * g.KXP * c);
  constexpr int TLZ = 64 / int(sizeof(Cplx<double>));
  o.partial = at;
  at = up256(at + size_t(g.KXP / TLZ) * g.NY2 * sizeof(double));
  o.maxbits = at;
  at = up256(at + sizeof(unsigned long long));
  o.flag = at;
  at = up256(at + sizeof(unsigned int));
  o.end = at;
  return o;
}

// reference layout [c][kz][ky][kx] (kx ≤ N/2) → compact S [c][ky'][kz'][kx]; a nonzero mode
// outside the retained 2/3 ball sets the flag word
__global__ void k_compact_reference(Geometry g, const Cplx<double>* __restrict__ uh, Cplx<double>* S,
                                    unsigned int* flag) {
  const int N = g.N, NH = N / 2 + 1;
  const size_t n = size_t(3) * N * N * NH;
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int kx = int(i % NH);
  const int ky = int((i / NH) % N);
  const int kz = int((i / (size_t(NH) * N)) % N);
  const int cc = int(i / (size_t(NH) * N * N));
  const Cplx<double> v = uh[i];
  const int my = ky <= N / 2 ? ky : ky - N, mz = kz <= N / 2 ? kz : kz - N;
  bool retained = false;
  if (kx <= g.K && abs(my) <= g.K && abs(mz) <= g.K) {
    const double kxd = g.s * kx, kyd = g.s * my, kzd = g.s * mz;
    retained = (kxd * kxd + kyd * kyd) + kzd * kzd <= g.cut2;
  }
  if (retained) {
    const int qy = my >= 0 ? my : my + g.NY2, qz = mz >= 0 ? mz : mz + g.NY2;
    S[gbght::idxS(g, cc, qy, qz, kx)] = v;
  } else if (v.x != 0.0 || v.y != 0.0) {
    atomicOr(flag, 1u);
  }
}

using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                            const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                            CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// What a device keeps between calls: the array's address, and the grid (N, L) whose tensor maps
// are encoded and whose twiddles sit at the start of the array. A call with another grid
// overwrites both (its layout also reuses the bytes that held the old twiddles).
struct DeviceSetup {
  bool ready = false;
  unsigned char* base = nullptr;   // device address of g_noalloc_scratch on this device
  int N = 0;
  double L = 0.0;
  gbght::TmaMaps maps{};
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;
Encode g_encode = nullptr;
// The host copy of the twiddles e^(−2πi k/N), k < N, of the last grid uploaded (static storage;
// cudaMemcpyAsync from pageable memory has consumed it when it returns).
Cplx<double> g_tw_host[kMaxN];

int encode_maps(const Layout& o, unsigned char* base, gbght::TmaMaps* m) {
  if (!g_encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDriverEntryPoint");
    if (!fn || q != cudaDriverEntryPointSuccess) return fail(GBGHT_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    g_encode = reinterpret_cast<Encode>(fn);
  }
  Encode encode = g_encode;
  const Geometry& g = o.g;
  const int N = g.N;
  constexpr int TLY = 128 / int(sizeof(Cplx<double>));
  const cuuint64_t inner = cuuint64_t(2) * g.KXP, pitch = cuuint64_t(g.KXP) * sizeof(Cplx<double>);
  const cuuint32_t ones[2] = {1, 1};
  auto map2 = [&](CUtensorMap* mp, void* ptr, cuuint64_t rows, cuuint32_t by) {
    const cuuint64_t dims[2] = {inner, rows};
    const cuuint64_t strides[1] = {pitch};
    const cuuint32_t box[2] = {cuuint32_t(2 * TLY), by};
    return encode(mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, ptr, dims, strides, box, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  if (!map2(&m->a_ld, base + o.A, cuuint64_t(3) * N * g.NY2, cuuint32_t(g.K + 1)) ||
      !map2(&m->b, base + o.B, cuuint64_t(3) * N * N, cuuint32_t(N)))
    return fail(GBGHT_ERR_CUDA, "tensor map encoding failed");
  return GBGHT_OK;
}

// The grid-dependent set-up of a device, redone only when the grid changes: the tensor maps, and
// the twiddles copied into the array from the static host table. Called with g_setup_mutex held.
int prepare_grid(DeviceSetup& ds, const Layout& o, double L, cudaStream_t st) {
  const int N = o.g.N;
  if (ds.N == N && ds.L == L) return GBGHT_OK;
  ds.N = 0;
  if (int rc = encode_maps(o, ds.base, &ds.maps)) return rc;
  for (int k = 0; k < N; ++k) {   // extended precision, as the run's own table
    const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)N;
    g_tw_host[k] = gbght::cmk<double>(double(cosl(a)), double(-sinl(a)));
  }
  cudaError_t e = cudaMemcpyAsync(ds.base + o.tw, g_tw_host, N * sizeof(Cplx<double>), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (twiddles)");
  ds.N = N;
  ds.L = L;
  return GBGHT_OK;
}

template <int N>
int run_n(const Layout& o, unsigned char* base, const gbght::TmaMaps& maps, const double* u_hat, double* u,
          cudaStream_t st) {
  constexpr int TLY = 128 / int(sizeof(Cplx<double>));
  constexpr int TLZ = 64 / int(sizeof(Cplx<double>));
  constexpr int NTY = N * TLY / 8 < 64 ? 64 : (N * TLY / 8 > 256 ? 256 : N * TLY / 8);
  constexpr int NTX = 32 * 6;   // the deposit's x pass: one warp per line
  constexpr int NTZ = N * TLZ / 8 < 64 ? 64 : (N * TLZ / 8 > 256 ? 256 : N * TLZ / 8);
  const Geometry& g = o.g;
  auto* tw = reinterpret_cast<Cplx<double>*>(base + o.tw);
  auto* S = reinterpret_cast<Cplx<double>*>(base + o.S);
  auto* A = reinterpret_cast<Cplx<double>*>(base + o.A);
  auto* B = reinterpret_cast<Cplx<double>*>(base + o.B);
  auto* partial = reinterpret_cast<double*>(base + o.partial);
  auto* maxbits = reinterpret_cast<unsigned long long*>(base + o.maxbits);
  auto* flag = reinterpret_cast<unsigned int*>(base + o.flag);
  cudaError_t e;
  // what must start at zero: the compact spectrum (modes of the box outside the ball), the
  // maximum and the flag word
  if ((e = cudaMemsetAsync(S, 0, o.A - o.S, st)) != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  if ((e = cudaMemsetAsync(base + o.maxbits, 0, o.end - o.maxbits, st)) != cudaSuccess)
    return cuda_fail(e, "cudaMemsetAsync");
  const size_t nref = size_t(3) * N * N * (N / 2 + 1);
  k_compact_reference<<<unsigned((nref + 255) / 256), 256, 0, st>>>(g, reinterpret_cast<const Cplx<double>*>(u_hat),
                                                                  S, flag);
  const size_t smem_z = size_t(N) * TLZ * sizeof(Cplx<double>) + size_t(NTZ) * sizeof(double) + 16;
  gbght::k_z_init<double, N, TLZ, NTZ><<<dim3(g.KXP / TLZ, g.NY2, 1), NTZ, smem_z, st>>>(g, A, S, 0, partial, tw, 0);
  const size_t smem_y = size_t(N) * TLY * sizeof(Cplx<double>) + 32;
  gbght::k_y_inverse<double, N, TLY, NTY><<<dim3(g.KXP / TLY, N, 3), NTY, smem_y, st>>>(maps, g, 0, tw, flag);
  const int KXS = gbght::x_kxs(g.K, int(sizeof(Cplx<double>)));
  const size_t smem_xv = size_t(N) * gbght::XShape<double>::ACT_V * sizeof(Cplx<double>) + size_t(NTX) * sizeof(double) +
                         size_t(3) * gbght::XShape<double>::PV * KXS * sizeof(Cplx<double>) + 32;
  const int ntiles_x = (N / gbght::XShape<double>::PV) * N;
  gbght::k_x_velocity<double, N, NTX><<<unsigned((ntiles_x + gbght::XT - 1) / gbght::XT), NTX, smem_xv, st>>>(
      g, B, u, maxbits, KXS, tw, flag);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "kernel launch");
  return GBGHT_OK;
}

}  // namespace

extern "C" int gbght_velocity_physical_noalloc(int grid_points_per_axis, double side_length, const double* u_hat,
                                               double* u, double* max_speed, void* stream) {
  const int N = grid_points_per_axis;
  if (!(N == 8 || N == 12 || N == 16 || N == 24 || N == 32 || N == 48 || N == 64))
    return fail(GBGHT_ERR_ARGUMENT, "grid_points_per_axis must be one of 8 12 16 24 32 48 64 (at most " +
                                        std::to_string(kMaxN) + "): the scratch array holds " +
                                        std::to_string(kScratchBytes >> 20) + " MiB");
  if (!(std::isfinite(side_length) && side_length > 0)) return fail(GBGHT_ERR_ARGUMENT, "side_length must be positive");
  if (!u_hat || !u) return fail(GBGHT_ERR_ARGUMENT, "u_hat and u must be device pointers");
  const Layout o = layout_for(N, side_length);
  if (o.end > kScratchBytes) return fail(GBGHT_ERR_ARGUMENT, "the grid does not fit the scratch array");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(GBGHT_ERR_ARGUMENT, "device ordinal out of range");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  gbght::TmaMaps maps{};
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& ds = g_setup[dev];
    if (!ds.ready) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
      ds.base = static_cast<unsigned char*>(p);
      ds.ready = true;
    }
    if (int rc = prepare_grid(ds, o, side_length, st)) return rc;
    base = ds.base;
    maps = ds.maps;
  }
  int rc = GBGHT_OK;
  switch (N) {
    case 8: rc = run_n<8>(o, base, maps, u_hat, u, st); break;
    case 12: rc = run_n<12>(o, base, maps, u_hat, u, st); break;
    case 16: rc = run_n<16>(o, base, maps, u_hat, u, st); break;
    case 24: rc = run_n<24>(o, base, maps, u_hat, u, st); break;
    case 32: rc = run_n<32>(o, base, maps, u_hat, u, st); break;
    case 48: rc = run_n<48>(o, base, maps, u_hat, u, st); break;
    case 64: rc = run_n<64>(o, base, maps, u_hat, u, st); break;
  }
  if (rc) return rc;
  // read back the maximum of |u|² and the flag word (the call's one synchronisation)
  unsigned long long bits = 0;
  unsigned int words[2] = {0, 0};
  if ((e = cudaMemcpyAsync(&bits, base + o.maxbits, sizeof bits, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(words, base + o.flag, sizeof(unsigned int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_fail(e, "reading back the maximum");
  if (words[0] & 1u)
    return fail(GBGHT_ERR_ARGUMENT, "the spectrum has content outside the retained 2/3 ball");
  if (words[0] & gbght::GBGHT_DEV_TIMEOUT)
    return fail(GBGHT_ERR_DEVICE, "a bulk copy did not complete within its bounded wait");
  double m2;
  std::memcpy(&m2, &bits, sizeof m2);
  if (max_speed) *max_speed = std::sqrt(m2);
  return GBGHT_OK;
}
