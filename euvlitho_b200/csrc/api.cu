// Error reporting and version of the C ABI.
#include <stdarg.h>
#include <stdio.h>
#include "common.cuh"

static thread_local char g_err[1024] = "";
static unsigned long long g_launches = 0;

extern "C" void euv_count_launch(void) { __atomic_fetch_add(&g_launches, 1ull, __ATOMIC_RELAXED); }

extern "C" unsigned long long euv_kernel_launches(void) {
  return __atomic_load_n(&g_launches, __ATOMIC_RELAXED);
}

extern "C" void euv_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

extern "C" const char* euv_last_error(void) { return g_err; }

extern "C" const char* euv_version(void) { return "euvl_b200 0.1 (sm_100a)"; }

// ---------------------------------------------------------------- wait probe
namespace euv {
// One thread waits for *flag != 0 with the library's bounded spin; on expiry
// it records EUV_STATUS_TIMEOUT and returns, leaving the context usable.
__global__ void wait_probe_kernel(const int* flag, unsigned long long limit_ns, int* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const volatile int* f = flag;
  const int r = bounded_spin([&] { return *f != 0; }, [] { return false; }, limit_ns);
  if (r < 0) atomicOr(status, EUV_STATUS_TIMEOUT);
}
}  // namespace euv

extern "C" int euv_wait_probe(const int* d_flag, long long limit_ns, int* d_status, void* stream) {
  if (!d_flag || !d_status || limit_ns < 0 || limit_ns > 2000000000ll) {
    euv_set_error("euv_wait_probe: bad arguments (limit_ns=%lld, at most 2e9)", limit_ns);
    return EUV_ERR_BAD_ARG;
  }
  euv::wait_probe_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(d_flag, (unsigned long long)limit_ns,
                                                              d_status);
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}
