// Common definitions for the B200 IF-RK step kernels: complex arithmetic, the CTA context and
// the barrier macro.
//
// Every kernel body in this library is a function of a `Cta` context. Threads are addressed as
// `c.tid` in [0, NT). Each body is split into phases separated by GBGHT_SYNC(). Inside a phase a
// thread keeps its values in arrays sized for NT threads, so the body's result does not depend on
// how the phases' loops interleave. The __global__ wrappers in gbght_kernels.cu run the bodies
// with NT threads per block. The same bodies compile as plain C++ with NT = 1, where the barrier
// is a no-op; the kernels' index arithmetic can then be checked on a CPU.
#pragma once

#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define GBGHT_HD __host__ __device__ __forceinline__
#define GBGHT_RESTRICT __restrict__
#else
#define GBGHT_HD inline
#define GBGHT_RESTRICT
#endif
#ifdef __CUDA_ARCH__
#define GBGHT_SYNC() __syncthreads()
#else
#define GBGHT_SYNC() ((void)0)
#endif

namespace gbght {

template <class T>
struct alignas(2 * sizeof(T)) Cplx {
  T x, y;
};

template <class T> GBGHT_HD Cplx<T> cmk(T x, T y) { Cplx<T> r; r.x = x; r.y = y; return r; }
template <class T> GBGHT_HD Cplx<T> operator+(Cplx<T> a, Cplx<T> b) { return cmk<T>(a.x + b.x, a.y + b.y); }
template <class T> GBGHT_HD Cplx<T> operator-(Cplx<T> a, Cplx<T> b) { return cmk<T>(a.x - b.x, a.y - b.y); }
template <class T> GBGHT_HD Cplx<T> operator*(Cplx<T> a, Cplx<T> b) {
  return cmk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class T> GBGHT_HD Cplx<T> scale(Cplx<T> a, T s) { return cmk<T>(a.x * s, a.y * s); }
template <class T> GBGHT_HD Cplx<T> conj(Cplx<T> a) { return cmk<T>(a.x, -a.y); }
// multiply by +i or -i
template <class T> GBGHT_HD Cplx<T> mul_i(Cplx<T> a) { return cmk<T>(-a.y, a.x); }
template <class T> GBGHT_HD Cplx<T> mul_mi(Cplx<T> a) { return cmk<T>(a.y, -a.x); }
template <class T> GBGHT_HD Cplx<T> czero() { return cmk<T>(T(0), T(0)); }

// The execution context of one CTA (thread block).
struct Cta {
  int tid;      // thread index in [0, NT)
  int bx, by, bz;
};

// Read-only global load (L1/texture path on the device).
template <class T> GBGHT_HD T ldg(const T* p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}
template <class T> GBGHT_HD Cplx<T> ldgc(const Cplx<T>* p) {
#ifdef __CUDA_ARCH__
  Cplx<T> r;
  r.x = __ldg(&p->x);
  r.y = __ldg(&p->y);
  return r;
#else
  return *p;
#endif
}

}  // namespace gbght
