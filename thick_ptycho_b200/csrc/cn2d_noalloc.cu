// tp_cn2d_march_noalloc: factorise + march without any device allocation.
//
// Some callers cannot allocate device memory.  A reconstruction service or
// host framework may own the whole device budget as a pre-reserved pool and
// hand this library only the input and output buffers.  Other callers run
// latency-bounded loops where a cudaMalloc (which may synchronise the device
// and has no latency bound) is not allowed after start-up.  For them this
// entry point keeps the per-slice factor set in a file-scope device array of
// fixed size instead of a caller-provided workspace.
//
// The array is kStaticScratchBytes (32 MiB).  Every GPU that loads this
// library reserves it for the life of the process.  Problems whose factor set
// is larger (tp_cn2d_factor_bytes(N, nz) > 32 MiB, e.g. N = 2048 with more
// than 337 slices) are rejected with TP_ERR_WORKSPACE.
//
// All calls share the one array, and each call overwrites the part it uses
// before reading it, so nothing carries over between calls.  Calls that
// overlap on the GPU (on different streams, or from different host threads
// without ordering) race on the array and corrupt each other's results.
//
// Set-up: the first call on each device resolves the array's device address
// with cudaGetSymbolAddress while that device is current, and caches it for
// that device's context; a call in a new context (after cudaDeviceReset)
// resolves it again.  The first call on a device should come before any
// stream capture on that device.
#include "tp_errors.h"
#include "tpcuda.h"

namespace tp {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_cn2d_static_scratch[kStaticScratchBytes];

static SymbolCache g_scratch_addr;

// Device address of g_cn2d_static_scratch on the current device.  The host
// symbol is only a stand-in; kernels must be given this address instead.
static int static_scratch(void **out) { return symbol_address(g_cn2d_static_scratch, g_scratch_addr, out); }

}  // namespace tp

extern "C" int tp_cn2d_march_noalloc(const tp_cn2d_op *op, const void *n_field, int32_t n_dtype,
                                     const tp_cn2d_march_args *args, tp_stream_t stream) {
  using namespace tp;
  if (op == nullptr || args == nullptr) return set_error(TP_ERR_INVALID, "op/args is NULL");
  const size_t need = tp_cn2d_factor_bytes(op->n, op->nz);
  if (need == 0) return set_error(TP_ERR_UNSUPPORTED, "N=%d, nz=%d unsupported", op->n, op->nz);
  if (need > kStaticScratchBytes)
    return set_error(TP_ERR_WORKSPACE,
                     "tp_cn2d_march_noalloc: factor set of N=%d, nz=%d needs %zu bytes, more than the %zu-byte "
                     "static scratch; use tp_cn2d_factor + tp_cn2d_march with a caller workspace",
                     op->n, op->nz, need, kStaticScratchBytes);
  void *scratch = nullptr;
  int rc = static_scratch(&scratch);
  if (rc != TP_OK) return rc;
  rc = tp_cn2d_factor(op, n_field, n_dtype, args->mode, scratch, kStaticScratchBytes, stream);
  if (rc != TP_OK) return rc;
  return tp_cn2d_march(op, scratch, args, stream);
}
