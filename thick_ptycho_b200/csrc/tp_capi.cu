// Library-wide C-ABI entry points: error string and version.
#include <stdarg.h>
#include <stdio.h>

#include <cuda.h>

#include <mutex>
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

// Unique id of this thread's current context (0 when none is current), from
// the driver's cuCtxGetCurrent / cuCtxGetId reached through the runtime (the
// library does not link libcuda itself).
static unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current == nullptr || get_id == nullptr || get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

static std::mutex g_symbol_mu;

int symbol_address(const void *symbol, SymbolCache &cache, void **out) {
  int dev = 0;
  TP_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxSymbolDevices) return set_error(TP_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_symbol_mu);
  unsigned long long id = current_context_id();
  if (id == 0 || cache.ctx_id[dev] != id || cache.addr[dev] == nullptr) {
    void *p = nullptr;
    // resolving the symbol also makes the device's primary context current
    TP_CHECK_CUDA(cudaGetSymbolAddress(&p, symbol));
    id = current_context_id();
    cache.addr[dev] = p;
    cache.ctx_id[dev] = id;
  }
  *out = cache.addr[dev];
  return TP_OK;
}
}  // namespace tp

extern "C" const char *tp_last_error_string(void) { return tp::g_last_error.c_str(); }

extern "C" int tp_version(void) { return 100; /* 0.1.0 */ }
