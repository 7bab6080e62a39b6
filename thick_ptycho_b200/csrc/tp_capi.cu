// Library-wide C-ABI entry points: error string and version.
#include <stdarg.h>
#include <stdio.h>

#include <string>

#include "tp_errors.h"

namespace tp {
static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int check_cuda(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return TP_OK;
  return set_error(TP_ERR_CUDA, "%s failed: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}
}  // namespace tp

extern "C" const char *tp_last_error_string(void) { return tp::g_last_error.c_str(); }

extern "C" int tp_version(void) { return 100; /* 0.1.0 */ }
