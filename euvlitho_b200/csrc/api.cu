// Error reporting and version of the C ABI.
#include <stdarg.h>
#include <stdio.h>

#include <mutex>

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

// ---------------------------------------------------------------- tuning table
// Picks written by an autotuner (or by hand) that override a kernel's built-in
// choice for one problem shape; looked up on the host at every launch.
namespace {
struct TuneEntry {
  int knob, k0, k1, value;
};
constexpr int kTuneCap = 1024;
TuneEntry g_tune[kTuneCap];
int g_tune_n = 0;
std::mutex g_tune_mu;

bool knob_value_ok(int knob, int value) {
  switch (knob) {
    case EUV_KNOB_ABBE_SPLIT: return value >= 1 && value <= 64;
    case EUV_KNOB_LU_CLUSTER: return value == 1 || value == 2 || value == 4 || value == 8;
    case EUV_KNOB_ZGEMM_ROWS: return value == 32 || value == 64;
    case EUV_KNOB_LU_SUBST_COLS: return value == 8 || value == 12;
    default: return false;
  }
}
}  // namespace

namespace euv {
int tune_lookup(int knob, int k0, int k1) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  for (int i = 0; i < g_tune_n; ++i)
    if (g_tune[i].knob == knob && g_tune[i].k0 == k0 && g_tune[i].k1 == k1) return g_tune[i].value;
  return 0;
}
}  // namespace euv

extern "C" int euv_tune_set(int knob, int k0, int k1, int value) {
  if (value != 0 && !knob_value_ok(knob, value)) {
    euv_set_error("euv_tune_set: value %d not allowed for knob %d", value, knob);
    return EUV_ERR_BAD_ARG;
  }
  std::lock_guard<std::mutex> g(g_tune_mu);
  for (int i = 0; i < g_tune_n; ++i)
    if (g_tune[i].knob == knob && g_tune[i].k0 == k0 && g_tune[i].k1 == k1) {
      if (value == 0) {
        g_tune[i] = g_tune[--g_tune_n];
      } else {
        g_tune[i].value = value;
      }
      return EUV_OK;
    }
  if (value == 0) return EUV_OK;
  if (g_tune_n >= kTuneCap) {
    euv_set_error("euv_tune_set: table full (%d entries)", kTuneCap);
    return EUV_ERR_BAD_ARG;
  }
  g_tune[g_tune_n++] = TuneEntry{knob, k0, k1, value};
  return EUV_OK;
}

extern "C" int euv_tune_get(int knob, int k0, int k1) { return euv::tune_lookup(knob, k0, k1); }

extern "C" void euv_tune_clear(void) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune_n = 0;
}
