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
