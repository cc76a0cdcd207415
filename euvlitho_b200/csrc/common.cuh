// Shared device helpers for the EUV mask-3D library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "../../include/euvl_b200.h"

namespace euv {

struct cplx {
  double x, y;
};

__host__ __device__ __forceinline__ cplx mk(double a, double b) { cplx r; r.x = a; r.y = b; return r; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx operator-(cplx a) { return mk(-a.x, -a.y); }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return mk(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ cplx operator*(cplx a, double s) { return mk(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ cplx cmul_i(cplx a) { return mk(-a.y, a.x); }  // i*a
__host__ __device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  // Smith's algorithm (scaled division, avoids overflow of |b|^2)
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return mk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.x * r + b.y;
    return mk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
__host__ __device__ __forceinline__ double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }
__host__ __device__ __forceinline__ double cabs(cplx a) { return hypot(a.x, a.y); }

// Principal square root, branch cut on the negative real axis with the sign of
// the imaginary part deciding the side (C99 csqrt semantics), from
// sqrt(z) = sqrt((|z|+x)/2) + i sign(y) sqrt((|z|-x)/2), evaluated without
// cancellation: t = sqrt((|z|+|x|)/2), then the other part is |y|/(2t).
__host__ __device__ __forceinline__ cplx csqrt_p(cplx z) {
  double x = z.x, y = z.y;
  if (x == 0.0 && y == 0.0) return mk(0.0, y);
  double t = sqrt(0.5 * (hypot(x, y) + fabs(x)));
  if (x >= 0.0) return mk(t, y / (2.0 * t));
  return mk(fabs(y) / (2.0 * t), copysign(t, y));
}

// exp(z) for complex z.
__host__ __device__ __forceinline__ cplx cexp_(cplx z) {
  double e = exp(z.x);
  double s, c;
  sincos(z.y, &s, &c);
  return mk(e * c, e * s);
}

__device__ __forceinline__ cplx ld(const euv_c64* p) {
  double2 v = *reinterpret_cast<const double2*>(p);
  return mk(v.x, v.y);
}
__device__ __forceinline__ void st(euv_c64* p, cplx v) {
  *reinterpret_cast<double2*>(p) = make_double2(v.x, v.y);
}
__host__ __device__ __forceinline__ cplx fromc(euv_c64 a) { return mk(a.re, a.im); }

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The one spin loop of every device wait in the library: polls ready() and,
// every 256 polls, abort() and the %globaltimer clock.  Returns 1 when ready,
// 0 when aborted (another role gave up), -1 after limit_ns nanoseconds.
template <class Ready, class Abort>
__device__ __forceinline__ int bounded_spin(Ready ready, Abort abort, unsigned long long limit_ns) {
  const unsigned long long t0 = globaltimer();
  for (uint32_t it = 0;; ++it) {
    if (ready()) return 1;
    if ((it & 255u) == 255u) {
      if (abort()) return 0;
      if (globaltimer() - t0 > limit_ns) return -1;
    }
  }
}

}  // namespace euv

#define EUV_CUDA_TRY(expr)                                     \
  do {                                                         \
    cudaError_t _e = (expr);                                   \
    if (_e != cudaSuccess) {                                   \
      euv_set_error("%s:%d CUDA error %s (%s)", __FILE__,      \
                    __LINE__, cudaGetErrorString(_e), #expr);  \
      return EUV_ERR_CUDA;                                     \
    }                                                          \
  } while (0)

// Every kernel launch of the library is followed by this check, which also
// counts the launch (euv_kernel_launches()).
#define EUV_LAUNCH_CHECK()        \
  do {                            \
    euv_count_launch();           \
    EUV_CUDA_TRY(cudaGetLastError()); \
  } while (0)

extern "C" void euv_set_error(const char* fmt, ...);
extern "C" void euv_count_launch(void);

namespace euv {
// The tuning table's pick for (knob, k0, k1), 0 when there is none (api.cu).
int tune_lookup(int knob, int k0, int k1);

// Raise a kernel's dynamic shared-memory limit once per device (the first call
// happens outside any stream capture; later calls do nothing).
template <typename K>
inline cudaError_t ensure_smem(K kernel, int bytes, int* done_per_device) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (__atomic_load_n(&done_per_device[dev], __ATOMIC_ACQUIRE) >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) __atomic_store_n(&done_per_device[dev], bytes, __ATOMIC_RELEASE);
  return e;
}
}  // namespace euv
