// Error reporting and version of the C ABI.
#include <stdarg.h>
#include <stdio.h>
#include "common.cuh"

static thread_local char g_err[1024] = "";

extern "C" void euv_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

extern "C" const char* euv_last_error(void) { return g_err; }

extern "C" const char* euv_version(void) { return "euvl_b200 0.1 (sm_100a)"; }
