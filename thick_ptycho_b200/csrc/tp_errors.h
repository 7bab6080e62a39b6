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
// (resolved once per device and context), or NULL.
int *device_error_ptr();

// Cache of one __device__ symbol's address per device.  An entry is tied to
// the context it was resolved in (its unique context id), so a context that
// replaces it (after cudaDeviceReset) resolves the address again.
constexpr int kMaxSymbolDevices = 64;
struct SymbolCache {
  unsigned long long ctx_id[kMaxSymbolDevices] = {};
  void *addr[kMaxSymbolDevices] = {};
};
// Device address of `symbol` (the host-side stand-in of a __device__
// variable) on the current device, through `cache`; thread-safe.
int symbol_address(const void *symbol, SymbolCache &cache, void **out);
}  // namespace tp

#define TP_CHECK_CUDA(expr)                                    \
  do {                                                         \
    int _rc = ::tp::check_cuda((expr), #expr);                 \
    if (_rc != TP_OK) return _rc;                              \
  } while (0)
