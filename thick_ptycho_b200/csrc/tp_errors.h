// Host-side error channel shared by the libtpcuda translation units.
#pragma once

#include <cuda_runtime.h>

#include "tpcuda.h"

namespace tp {
// Record `msg` as this thread's last error and return `code`.
int set_error(int code, const char *fmt, ...);
// Map a CUDA runtime error to TP_ERR_CUDA with context; TP_OK on success.
int check_cuda(cudaError_t e, const char *what);
// Device address of the library's device error word on the current device
// (resolved once per device), or NULL.
int *device_error_ptr();
}  // namespace tp

#define TP_CHECK_CUDA(expr)                                    \
  do {                                                         \
    int _rc = ::tp::check_cuda((expr), #expr);                 \
    if (_rc != TP_OK) return _rc;                              \
  } while (0)
