// Shared device helpers for libtpcuda: complex arithmetic, bulk-copy (TMA)
// staging with bounded mbarrier waits, bulk stores, and the error channel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tp {

constexpr int kLanes = 32;

// Device-side error channel: kernels never trap; a bounded wait that gives up
// writes a code here and returns, the host reads it after the stream syncs.
enum DeviceError : int { kDevOk = 0, kDevMbarTimeout = 1 };

// ----------------------------------------------------------------- complex64
__device__ __forceinline__ float2 c2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return c2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return c2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return c2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a*b + c
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  return c2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
// c - a*b
__device__ __forceinline__ float2 cfnma(float2 a, float2 b, float2 c) {
  return c2(fmaf(-a.x, b.x, fmaf(a.y, b.y, c.x)), fmaf(-a.x, b.y, fmaf(-a.y, b.x, c.y)));
}
// s*a + c for real s
__device__ __forceinline__ float2 caxpy(float s, float2 a, float2 c) { return c2(fmaf(s, a.x, c.x), fmaf(s, a.y, c.y)); }
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return c2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 shfl_up2(float2 v, int d) {
  return c2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ float2 shfl_down2(float2 v, int d) {
  return c2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}

// The same operations on complex128 (the check build's march state).
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cfnma(double2 a, double2 b, double2 c) {
  return make_double2(fma(-a.x, b.x, fma(a.y, b.y, c.x)), fma(-a.x, b.y, fma(-a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 caxpy(double s, double2 a, double2 c) {
  return make_double2(fma(s, a.x, c.x), fma(s, a.y, c.y));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double2 shfl_up2(double2 v, int d) {
  return make_double2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ double2 shfl_down2(double2 v, int d) {
  return make_double2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}

// A pair of complex128 values (two rows of a stored field in one 32-byte unit).
struct __align__(32) zpair {
  double x, y, z, w;
};

// ------------------------------------------------- state type of the 2D march
// cx is the complex type of the 2D march's state, factor sets and stored
// fields: complex64, or complex128 in the check build (compiled with
// TP_C128_CHECK), which runs the same algorithms -- partitioned solve,
// truncated spikes, PCR skip, Cayley step, pair-sum store -- with every
// stored value and all arithmetic in fp64, so that they can be compared with
// the complex128 oracle far below complex64 round-off.  rx is its real type
// and cx2 a pair of cx (two rows in one vector access).
#ifdef TP_C128_CHECK
using cx = double2;
using rx = double;
using cx2 = zpair;
#else
using cx = float2;
using rx = float;
using cx2 = float4;
#endif
// A floating-point literal of the real type (TP_R(0.5) is 0.5f, or 0.5 in
// the complex128 check build).
#ifdef TP_C128_CHECK
#define TP_R(x) x
#else
#define TP_R(x) x##f
#endif
__host__ __device__ __forceinline__ cx mkcx(rx x, rx y) {
  cx v;
  v.x = x;
  v.y = y;
  return v;
}
__host__ __device__ __forceinline__ cx czero() { return mkcx(rx(0), rx(0)); }
__host__ __device__ __forceinline__ cx2 mkcx2(cx a, cx b) {
  cx2 v;
  v.x = a.x;
  v.y = a.y;
  v.z = b.x;
  v.w = b.y;
  return v;
}
__host__ __device__ __forceinline__ cx cx2_lo(cx2 v) { return mkcx(v.x, v.y); }
__host__ __device__ __forceinline__ cx cx2_hi(cx2 v) { return mkcx(v.z, v.w); }
// global dst += v without a return value (vector reductions in the normal build)
__device__ __forceinline__ void red_add_cx(cx *dst, cx v) {
#ifdef TP_C128_CHECK
  atomicAdd(&dst->x, v.x);
  atomicAdd(&dst->y, v.y);
#else
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(dst), "f"(v.x), "f"(v.y) : "memory");
#endif
}
__device__ __forceinline__ void red_add_cx2(cx2 *dst, cx2 v) {
#ifdef TP_C128_CHECK
  atomicAdd(&dst->x, v.x);
  atomicAdd(&dst->y, v.y);
  atomicAdd(&dst->z, v.z);
  atomicAdd(&dst->w, v.w);
#else
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(dst), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
#endif
}

// ---------------------------------------------------------------- complex128
__host__ __device__ __forceinline__ double2 z2(double x, double y) { return make_double2(x, y); }
__host__ __device__ __forceinline__ double2 zadd(double2 a, double2 b) { return z2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 zsub(double2 a, double2 b) { return z2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return z2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 zconj(double2 a) { return z2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 zneg(double2 a) { return z2(-a.x, -a.y); }
__host__ __device__ __forceinline__ double2 zscale(double2 a, double s) { return z2(a.x * s, a.y * s); }
// a / b by Smith's scaling (avoids overflow of |b|^2 for extreme values)
__host__ __device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return z2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  double r = b.x / b.y, d = b.x * r + b.y;
  return z2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ float2 to_f2(double2 a) { return make_float2((float)a.x, (float)a.y); }
// fp64 value to the march's complex type (rounded to complex64 in the normal build)
__host__ __device__ __forceinline__ cx to_cx(double2 a) { return mkcx((rx)a.x, (rx)a.y); }
__device__ __forceinline__ double2 shfl_up_z(double2 v, int d) {
  return z2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ double2 shfl_down_z(double2 v, int d) {
  return z2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}

// ------------------------------------------------- bulk copy (TMA) + mbarrier
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// Global -> shared bulk copy completing on `bar`.  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Tiled tensor loads (TMA, no multicast): the box of the tensor map `tmap`
// (the generic address of a __grid_constant__ CUtensorMap) at coordinates
// c0 (innermost) .. c2 / c3 into shared memory, completing on `bar`; box
// positions outside the tensor read as zero.  c0 times the element size must
// be a multiple of 16 bytes (callers pass c0 = 0).
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, int c0, int c1, int c2, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_addr(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const void *tmap, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_addr(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}
// Shared -> global bulk copy, tracked by the issuing thread's bulk groups
// (commit with bulk_commit; the source may be rewritten after
// bulk_wait_read, the global result is complete after bulk_wait).  Addresses
// 16-byte aligned, bytes a multiple of 16.  The generic-proxy writes of the
// source must be followed by fence_proxy_async_smem and a barrier before the
// issuing thread copies.
__device__ __forceinline__ void bulk_s2g(void *gdst, const void *ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_addr(ssrc)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Every committed bulk group of this thread has finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Every committed bulk group of this thread has completed.
__device__ __forceinline__ void bulk_wait() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// 8-byte global -> shared asynchronous copy (no registers; completes at
// cp_async_wait_all).  Both addresses 8-byte aligned.
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
// Asynchronous global -> shared copy of one cx (8 or 16 bytes, aligned to its size).
__device__ __forceinline__ void cp_async_cx(cx *dst, const cx *src) {
#ifdef TP_C128_CHECK
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
#else
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
#endif
}
// 16-byte global -> shared asynchronous copy (L2 only).  Both addresses
// 16-byte aligned.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n cp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and records kDevMbarTimeout) after `max_iter`
// polls.  Each try_wait already suspends the thread for a hardware-chosen
// interval, so 1<<22 polls is far beyond any bulk copy's latency.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err,
                                                  uint32_t max_iter = 1u << 22) {
  for (uint32_t it = 0; it < max_iter; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicOr(err, (int)kDevMbarTimeout);
  return false;
}

}  // namespace tp
