// Error reporting and version of the C ABI.
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace pk {

static thread_local char g_error[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}

}  // namespace pk

extern "C" const char *pk_version(void) { return "jaxpower_b200 0.1.0 (sm_100a)"; }

extern "C" const char *pk_last_error(void) { return pk::g_error; }
