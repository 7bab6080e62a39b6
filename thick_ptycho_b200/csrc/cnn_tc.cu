// Learned correction of the 3D FFT preconditioner: 3x3 bf16 convolutions on
// the 5th-generation tensor cores, and the per-pixel filter they produce.
//
// The network maps the index perturbation of one slice (the diagonal d of the
// object term in the 3D step operator) to a 13-tap complex filter per pixel;
// the preconditioner is then  y = z + sum_t F_t(x) z(x + o_t),  z the plain
// FFT-preconditioned vector.  The correction is linear in z, so BiCGStab
// keeps a fixed linear preconditioner, and the network runs once per slice
// (shared by every probe and every Krylov iteration).  The reference has no
// learned component: this is the project's own addition on the 3D path.
//
// conv3x3_tc_kernel: implicit GEMM, D[128 pixels x 32 out] += A_tap[128 x 16]
// B_tap[16 x 32] over the 9 taps and the input channels, one tcgen05.mma
// (kind::f16, bf16 operands, fp32 accumulator in TMEM) per (block, tap,
// 16-channel step), issued by one thread.  Operands sit in shared memory in
// the canonical K-major no-swizzle layout: a core matrix is 8 rows of 16 bytes
// (8 pixels x 8 channels), 8-row groups 128 bytes apart (SBO), channel chunks
// one chunk plane apart (LBO).  Because activations are channel-chunked
// ("padded-linear", cnn_internal.cuh), a tap's A operand is the staged input
// slab shifted by (dy * Wp + dx) pixel rows: no im2col.  One CTA of 4 warps
// computes 4 x 128 consecutive output pixels; its input slab (with a one-row
// halo above and below) and the layer's weights arrive by bulk copies
// (cp.async.bulk, no multicast) on an mbarrier; the epilogue reads the TMEM
// accumulators with tcgen05.ld (warp w owns lanes 32w..32w+31) and applies
// bias + ReLU, the ReLU mask of the backward pass, or writes the filter.
// Every wait is bounded and records kDevMbarTimeout instead of hanging.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cnn_internal.cuh"
#include "tp_common.cuh"
#include "tp_errors.h"
#include "tpcuda.h"

namespace tp {

using bf16 = __nv_bfloat16;

ConvGeom conv_geom(int H, int W, int batch) {
  ConvGeom g{};
  g.H = H;
  g.W = W;
  g.Wp = W + 2;
  g.batch = batch;
  g.S = (long long)(H + 2) * g.Wp;
  g.G0 = 8;
  const long long G1 = ((kConvTile + g.Wp + 8 + 7) / 8) * 8;
  g.CS = ((g.G0 + (long long)batch * g.S + G1 + 7) / 8) * 8;
  g.l_begin = g.G0 + g.Wp;
  g.l_end = g.G0 + (long long)batch * g.S - g.Wp;
  return g;
}

size_t act_bytes(const ConvGeom &g, int channels) { return (size_t)(channels / 8) * (size_t)g.CS * 16; }

int conv_tiles(const ConvGeom &g) { return (int)((g.l_end - g.l_begin + kConvTile - 1) / kConvTile); }

// ------------------------------------------------------------ tcgen05 helpers
// Shared-memory matrix descriptor: start, leading (K) and stride (M/N) byte
// offsets in 16-byte units, version 1 (sm_100), no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 32 consecutive fp32 columns of this warp's 32 TMEM lanes (one lane per thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ void unpack_bf8(uint4 u, float (&f)[8]) {
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162 *>(&w[i]);
    const float2 t = __bfloat1622float2(h);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}

// Interior test of a linear pixel; (p, yp, xp) = image and padded coordinates.
__device__ __forceinline__ bool px_inside(const ConvGeom &g, long long l, int &p, int &yp, int &xp) {
  if (l < g.l_begin || l >= g.l_end) return false;
  const long long rel = l - g.G0;
  p = (int)(rel / g.S);
  const long long rem = rel - (long long)p * g.S;
  yp = (int)(rem / g.Wp);
  xp = (int)(rem - (long long)yp * g.Wp);
  return p < g.batch && yp >= 1 && yp <= g.H && xp >= 1 && xp <= g.W;
}

struct ConvArgs {
  ConvGeom g;
  const bf16 *in;     // CIN channels, padded-linear
  const bf16 *w;      // [9][CIN/8][32][8]
  const float *bias;  // [32] or NULL
  const bf16 *aux;    // kEpiMask: the layer's forward input (32 channels)
  bf16 *out;          // kEpiRelu / kEpiMask: 32 channels, padded-linear
  float2 *filt;       // kEpiFilter: (13, batch*H*W)
  float out_scale;    // kEpiFilter: F = out_scale * (conv + bias)
  int *err;
};

__host__ __device__ inline uint32_t conv_slab_pixels(int Wp) { return (uint32_t)(kConvTile + 2 * Wp + 2); }
__host__ __device__ inline size_t conv_smem_bytes(int cin, int Wp) {
  return (size_t)9 * cin * kConvCout * 2 + (size_t)(cin / 8) * conv_slab_pixels(Wp) * 16 + 32;
}

template <int CIN, int EPI>
__global__ void __launch_bounds__(128) conv3x3_tc_kernel(const ConvArgs a) {
  constexpr int COUT = kConvCout;
  constexpr int B = kConvBlocks;
  constexpr uint32_t W_BYTES = 9 * CIN * COUT * 2;
  constexpr uint32_t NCOL = B * COUT;  // 128 TMEM columns
  extern __shared__ __align__(128) uint8_t smem[];
  const ConvGeom &g = a.g;
  const uint32_t R = conv_slab_pixels(g.Wp);
  const uint32_t a_bytes = (CIN / 8) * R * 16;
  uint8_t *sw = smem;
  uint8_t *sa = smem + W_BYTES;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sa + a_bytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long l0 = g.l_begin + (long long)blockIdx.x * kConvTile;

  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, NCOL);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = *tslot;

  if (tid == 0) {
    mbar_arrive_expect_tx(&bars[0], W_BYTES + a_bytes);
    bulk_g2s(sw, a.w, W_BYTES, &bars[0]);
    const long long src0 = l0 - g.Wp - 1;
#pragma unroll
    for (int j = 0; j < CIN / 8; ++j) bulk_g2s(sa + (size_t)j * R * 16, a.in + ((size_t)j * g.CS + src0) * 8, R * 16, &bars[0]);
  }
  bool ok = mbar_wait_bounded(&bars[0], 0, a.err);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) mbar_wait_bounded(&bars[0], 0, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
      tc_fence_after();
      tmem_dealloc(taddr, NCOL);
    }
    return;
  }

  if (tid == 0) {
    tc_fence_after();
    const uint32_t sA = smem_addr(sa), sW = smem_addr(sw);
    constexpr uint32_t idesc = umma_idesc_bf16(128, COUT);
#pragma unroll 1
    for (int b = 0; b < B; ++b) {
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const int ty = tap / 3, tx = tap % 3;
#pragma unroll
        for (int kk = 0; kk < CIN / 16; ++kk) {
          const uint32_t apix = (uint32_t)(2 * kk) * R + (uint32_t)(b * 128 + ty * g.Wp + tx);
          const uint32_t aaddr = sA + apix * 16;
          const uint32_t baddr = sW + (uint32_t)((tap * (CIN / 8) + 2 * kk) * COUT * 16);
          umma_bf16(taddr + (uint32_t)(b * COUT), umma_desc(aaddr, R * 16, 128), umma_desc(baddr, COUT * 16, 128), idesc,
                    (tap | kk) != 0);
        }
      }
    }
    umma_commit(&bars[1]);
  }
  ok = mbar_wait_bounded(&bars[1], 0, a.err);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) mbar_wait_bounded(&bars[1], 0, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
      tc_fence_after();
      tmem_dealloc(taddr, NCOL);
    }
    return;
  }
  tc_fence_after();

  float bias[COUT];
#pragma unroll
  for (int c = 0; c < COUT; ++c) bias[c] = (a.bias != nullptr) ? a.bias[c] : 0.f;

#pragma unroll 1
  for (int b = 0; b < B; ++b) {
    float v[32];
    tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * COUT), v);
    __syncwarp();
    const long long l = l0 + b * 128 + warp * 32 + lane;
    int p = 0, yp = 0, xp = 0;
    if (!px_inside(g, l, p, yp, xp)) continue;  // the next tcgen05.ld follows a __syncwarp
    if constexpr (EPI == kEpiFilter) {
      const size_t np = (size_t)g.batch * g.H * g.W;
      const size_t pix = (size_t)p * g.H * g.W + (size_t)(yp - 1) * g.W + (xp - 1);
#pragma unroll
      for (int t = 0; t < kFilterTaps; ++t)
        a.filt[(size_t)t * np + pix] =
            make_float2(a.out_scale * (v[2 * t] + bias[2 * t]), a.out_scale * (v[2 * t + 1] + bias[2 * t + 1]));
    } else {
#pragma unroll
      for (int j = 0; j < COUT / 8; ++j) {
        float t[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) t[c] = v[8 * j + c] + bias[8 * j + c];
        if constexpr (EPI == kEpiRelu) {
#pragma unroll
          for (int c = 0; c < 8; ++c) t[c] = fmaxf(t[c], 0.f);
        } else {
          float m[8];
          unpack_bf8(*reinterpret_cast<const uint4 *>(a.aux + ((size_t)j * g.CS + l) * 8), m);
#pragma unroll
          for (int c = 0; c < 8; ++c) t[c] = (m[c] > 0.f) ? t[c] : 0.f;
        }
        uint4 o;
        o.x = pack_bf2(t[0], t[1]);
        o.y = pack_bf2(t[2], t[3]);
        o.z = pack_bf2(t[4], t[5]);
        o.w = pack_bf2(t[6], t[7]);
        *reinterpret_cast<uint4 *>(a.out + ((size_t)j * g.CS + l) * 8) = o;
      }
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(taddr, NCOL);
  }
}

// ------------------------------------------------------------ weight gradient
// dW[tap][c][o] = sum_q x[q + off_tap][c] dy[q][o] and db[o] = sum_q dy[q][o]
// over the computed pixels (dy is zero off the interior).  Thread (tap, c) of
// 10*CIN threads keeps its 32 sums in registers (tap 9 is the bias, c = 0
// only); a persistent CTA loops over tiles staged by bulk copies and adds its
// sums to dW/db once at the end (fp32 CUDA cores: this runs only in training).
template <int CIN>
__global__ void __launch_bounds__(10 * CIN) conv3x3_wgrad_kernel(const ConvGeom g, const bf16 *x, const bf16 *dy,
                                                                 float *dw, float *db, int ntiles, int *err) {
  constexpr int COUT = kConvCout;
  extern __shared__ __align__(128) uint8_t smem[];
  const uint32_t R = conv_slab_pixels(g.Wp);
  bf16 *sx = reinterpret_cast<bf16 *>(smem);
  bf16 *sdy = reinterpret_cast<bf16 *>(smem + (size_t)(CIN / 8) * R * 16);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + (size_t)(CIN / 8) * R * 16 + (size_t)(COUT / 8) * kConvTile * 16);
  const int tid = threadIdx.x;
  const int tap = tid / CIN, c = tid % CIN;
  const int ty = tap / 3, tx = tap % 3;
  const bool active = tap < 9 || c == 0;
  float acc[COUT];
#pragma unroll
  for (int o = 0; o < COUT; ++o) acc[o] = 0.f;
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long l0 = g.l_begin + (long long)tile * kConvTile;
    if (tid == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(bar, (CIN / 8) * R * 16 + (COUT / 8) * kConvTile * 16);
      for (int j = 0; j < CIN / 8; ++j)
        bulk_g2s(sx + (size_t)j * R * 8, x + ((size_t)j * g.CS + (l0 - g.Wp - 1)) * 8, R * 16, bar);
      for (int j = 0; j < COUT / 8; ++j)
        bulk_g2s(sdy + (size_t)j * kConvTile * 8, dy + ((size_t)j * g.CS + l0) * 8, kConvTile * 16, bar);
    }
    const bool ok = mbar_wait_bounded(bar, phase, err);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      if (tid == 0) mbar_wait_bounded(bar, phase ^ 1u, nullptr);
      __syncthreads();
      return;
    }
    if (active) {
      const bf16 *xs = sx + (size_t)(c / 8) * R * 8 + (c % 8);
      const int off = ty * g.Wp + tx;
#pragma unroll 2
      for (int q = 0; q < kConvTile; ++q) {
        const float xv = (tap < 9) ? __bfloat162float(xs[(size_t)(q + off) * 8]) : 1.f;
#pragma unroll
        for (int j = 0; j < COUT / 8; ++j) {
          float d[8];
          unpack_bf8(*reinterpret_cast<const uint4 *>(sdy + ((size_t)j * kConvTile + q) * 8), d);
#pragma unroll
          for (int k = 0; k < 8; ++k) acc[8 * j + k] = fmaf(xv, d[k], acc[8 * j + k]);
        }
      }
    }
    __syncthreads();
  }
  if (!active) return;
  if (tap < 9) {
#pragma unroll
    for (int o = 0; o < COUT; ++o) atomicAdd(&dw[((size_t)tap * CIN + c) * COUT + o], acc[o]);
  } else if (db != nullptr) {
#pragma unroll
    for (int o = 0; o < COUT; ++o) atomicAdd(&db[o], acc[o]);
  }
}

__host__ __device__ inline size_t wgrad_smem_bytes(int cin, int Wp) {
  return (size_t)(cin / 8) * conv_slab_pixels(Wp) * 16 + (size_t)(kConvCout / 8) * kConvTile * 16 + 16;
}

// ------------------------------------------------------------ elementwise parts
__global__ void cnn_features_kernel(const ConvGeom g, const float2 *__restrict__ diag, long long diag_stride,
                                    const float2 *__restrict__ kc, float kappa, bf16 *feat) {
  const long long hw = (long long)g.H * g.W, np = hw * g.batch;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < np; e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / hw, i = e - p * hw;
    const int y = (int)(i / g.W), xx = (int)(i - (long long)y * g.W);
    float2 d = diag[p * diag_stride + i];
    if (kc != nullptr) {
      const float2 k = kc[i];
      d = make_float2(d.x - k.x, d.y - k.y);
    }
    const long long l = g.G0 + p * g.S + (long long)(y + 1) * g.Wp + (xx + 1);
    uint4 c0, c1;
    c0.x = pack_bf2(kappa * d.x, kappa * d.y);
    c0.y = pack_bf2(1.f, xx == 0 ? 1.f : 0.f);
    c0.z = pack_bf2(xx == g.W - 1 ? 1.f : 0.f, y == 0 ? 1.f : 0.f);
    c0.w = pack_bf2(y == g.H - 1 ? 1.f : 0.f, 0.f);
    c1 = make_uint4(0u, 0u, 0u, 0u);
    *reinterpret_cast<uint4 *>(feat + ((size_t)0 * g.CS + l) * 8) = c0;
    *reinterpret_cast<uint4 *>(feat + ((size_t)1 * g.CS + l) * 8) = c1;
  }
}

// y[v] = z[v] + sum_t F_t z[v](x + o_t), vector v using filter image v / per_image.
__global__ void cnn_filter_apply_kernel(int H, int W, int nvec, int per_image, int nimg, int conj,
                                        const float2 *__restrict__ F, const float2 *__restrict__ z, float2 *y) {
  const size_t hw = (size_t)H * W, np = hw * nimg;
  const int v = blockIdx.y;
  const size_t fimg = (per_image > 0) ? (size_t)(v / per_image) * hw : 0;
  const float2 *zv = z + (size_t)v * hw;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < hw; i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / W), f = (int)(i - (size_t)b * W);
    y[(size_t)v * hw + i] = filter_apply_px(F, fimg, np, zv, H, W, b, f, conj);
  }
}

// Gradient of sum_v |y_v - target_v|^2 * scale_v w.r.t. the filter, given
// e_v = scale_v (y_v - target_v):  dF_t(x) = 2 sum_v conj(z_v(x + o_t)) e_v(x)
// (d/dRe + i d/dIm), times out_scale (F = out_scale * last layer), written as
// the 32-channel bf16 gradient of the last layer (channels 2t, 2t+1;
// channels 26..31 zero).  One thread per pixel of
// each filter image sums over the image's `per_image` vectors.
__global__ void cnn_filter_grad_kernel(const ConvGeom g, int per_image, const float2 *__restrict__ z,
                                       const float2 *__restrict__ e, float out_scale, bf16 *dy) {
  const long long hw = (long long)g.H * g.W, np = hw * g.batch;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < np;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long img = idx / hw, i = idx - img * hw;
    const int b = (int)(i / g.W), f = (int)(i - (long long)b * g.W);
    float2 acc[kFilterTaps];
#pragma unroll
    for (int t = 0; t < kFilterTaps; ++t) acc[t] = make_float2(0.f, 0.f);
    for (int s = 0; s < per_image; ++s) {
      const size_t v = (size_t)img * per_image + s;
      const float2 ev = e[v * hw + i];
#pragma unroll
      for (int t = 0; t < kFilterTaps; ++t) {
        const int bb = b + filter_tap_dy(t), ff = f + filter_tap_dx(t);
        if (bb < 0 || bb >= g.H || ff < 0 || ff >= g.W) continue;
        const float2 zv = z[v * hw + (size_t)bb * g.W + ff];
        // conj(z) * e
        acc[t].x = fmaf(zv.x, ev.x, fmaf(zv.y, ev.y, acc[t].x));
        acc[t].y = fmaf(zv.x, ev.y, fmaf(-zv.y, ev.x, acc[t].y));
      }
    }
    const long long l = g.G0 + img * g.S + (long long)(b + 1) * g.Wp + (f + 1);
    float ch[32];
#pragma unroll
    for (int t = 0; t < kFilterTaps; ++t) {
      ch[2 * t] = 2.f * out_scale * acc[t].x;
      ch[2 * t + 1] = 2.f * out_scale * acc[t].y;
    }
#pragma unroll
    for (int c = 2 * kFilterTaps; c < 32; ++c) ch[c] = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      uint4 o;
      o.x = pack_bf2(ch[8 * j], ch[8 * j + 1]);
      o.y = pack_bf2(ch[8 * j + 2], ch[8 * j + 3]);
      o.z = pack_bf2(ch[8 * j + 4], ch[8 * j + 5]);
      o.w = pack_bf2(ch[8 * j + 6], ch[8 * j + 7]);
      *reinterpret_cast<uint4 *>(dy + ((size_t)j * g.CS + l) * 8) = o;
    }
  }
}

// ------------------------------------------------------------ host
static int max_smem_optin() {
  int dev = 0, v = 232448;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v;
}

static int check_geom(const ConvGeom &g) {
  if (g.H < 1 || g.W < 1 || g.batch < 1) return set_error(TP_ERR_INVALID, "bad CNN image size %dx%d x%d", g.H, g.W, g.batch);
  if (conv_smem_bytes(32, g.Wp) > (size_t)max_smem_optin())
    return set_error(TP_ERR_UNSUPPORTED, "CNN image width %d needs %zu B of shared memory", g.W, conv_smem_bytes(32, g.Wp));
  return TP_OK;
}

int cnn_features(const ConvGeom &g, const float2 *diag, long long diag_stride, const float2 *kc, float kappa, void *feat,
                 cudaStream_t st) {
  int rc = check_geom(g);
  if (rc != TP_OK) return rc;
  cnn_features_kernel<<<592, 256, 0, st>>>(g, diag, diag_stride, kc, kappa, static_cast<bf16 *>(feat));
  return check_cuda(cudaGetLastError(), "cnn_features_kernel launch");
}

template <int CIN, int EPI>
static int launch_conv(const ConvArgs &a, cudaStream_t st) {
  auto kern = conv3x3_tc_kernel<CIN, EPI>;
  // At least 58 KB of shared memory per CTA caps residency at 3 CTAs per SM,
  // so the CTAs of an SM never ask for more than its 512 TMEM columns (128
  // each) and tcgen05.alloc never has to wait for another CTA's columns.
  size_t smem = conv_smem_bytes(CIN, a.g.Wp);
  if (smem < 58 * 1024) smem = 58 * 1024;
  TP_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<conv_tiles(a.g), 128, smem, st>>>(a);
  return check_cuda(cudaGetLastError(), "conv3x3_tc_kernel launch");
}

int conv_layer(const ConvGeom &g, int cin, int epi, const void *in, const void *w, const float *bias, const void *aux,
               void *out, void *filt, float out_scale, cudaStream_t st) {
  int rc = check_geom(g);
  if (rc != TP_OK) return rc;
  if (in == nullptr || w == nullptr) return set_error(TP_ERR_INVALID, "conv3x3: NULL input or weights");
  if ((epi == kEpiRelu || epi == kEpiMask) && out == nullptr) return set_error(TP_ERR_INVALID, "conv3x3: NULL output");
  if (epi == kEpiMask && aux == nullptr) return set_error(TP_ERR_INVALID, "conv3x3: the ReLU mask needs the forward input");
  if (epi == kEpiFilter && filt == nullptr) return set_error(TP_ERR_INVALID, "conv3x3: NULL filter output");
  const uintptr_t al = reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(w) |
                       reinterpret_cast<uintptr_t>(out) | reinterpret_cast<uintptr_t>(aux);
  if (al & 15u) return set_error(TP_ERR_INVALID, "conv3x3: buffers must be 16-byte aligned");
  int *err = device_error_ptr();
  if (err == nullptr) return set_error(TP_ERR_CUDA, "cannot resolve the device error word");
  ConvArgs a{};
  a.g = g;
  a.in = static_cast<const bf16 *>(in);
  a.w = static_cast<const bf16 *>(w);
  a.bias = bias;
  a.aux = static_cast<const bf16 *>(aux);
  a.out = static_cast<bf16 *>(out);
  a.filt = static_cast<float2 *>(filt);
  a.out_scale = out_scale;
  a.err = err;
  if (cin == 16 && epi == kEpiRelu) return launch_conv<16, kEpiRelu>(a, st);
  if (cin == 32 && epi == kEpiRelu) return launch_conv<32, kEpiRelu>(a, st);
  if (cin == 32 && epi == kEpiMask) return launch_conv<32, kEpiMask>(a, st);
  if (cin == 32 && epi == kEpiFilter) return launch_conv<32, kEpiFilter>(a, st);
  return set_error(TP_ERR_UNSUPPORTED, "conv3x3: no kernel for cin=%d epilogue=%d", cin, epi);
}

// features (16) | a1 | a2 | a3 (32 each)
size_t cnn_forward_ws_bytes(const ConvGeom &g) { return act_bytes(g, 16) + 3 * act_bytes(g, 32); }

int cnn_forward(const ConvGeom &g, const tp_cnn_model &m, const float2 *diag, long long diag_stride, const float2 *kc,
                void *ws, float2 *filt, cudaStream_t st) {
  char *base = static_cast<char *>(ws);
  void *feat = base;
  void *a1 = base + act_bytes(g, 16);
  void *a2 = static_cast<char *>(a1) + act_bytes(g, 32);
  void *a3 = static_cast<char *>(a2) + act_bytes(g, 32);
  int rc = cnn_features(g, diag, diag_stride, kc, m.kappa, feat, st);
  if (rc == TP_OK) rc = conv_layer(g, 16, kEpiRelu, feat, m.w[0], m.b[0], nullptr, a1, nullptr, 1.f, st);
  if (rc == TP_OK) rc = conv_layer(g, 32, kEpiRelu, a1, m.w[1], m.b[1], nullptr, a2, nullptr, 1.f, st);
  if (rc == TP_OK) rc = conv_layer(g, 32, kEpiRelu, a2, m.w[2], m.b[2], nullptr, a3, nullptr, 1.f, st);
  if (rc == TP_OK) rc = conv_layer(g, 32, kEpiFilter, a3, m.w[3], m.b[3], nullptr, nullptr, filt, m.out_scale, st);
  return rc;
}

}  // namespace tp

using namespace tp;

extern "C" size_t tp_cnn_act_bytes(int32_t nf, int32_t nb, int32_t batch, int32_t channels) {
  if (nf < 1 || nb < 1 || batch < 1 || channels < 8 || channels % 8 != 0) return 0;
  return act_bytes(conv_geom(nb, nf, batch), channels);
}

extern "C" int tp_cnn_features(int32_t nf, int32_t nb, int32_t batch, const void *diag, float kappa, void *feat,
                               tp_stream_t stream) {
  if (diag == nullptr || feat == nullptr) return set_error(TP_ERR_INVALID, "tp_cnn_features: NULL argument");
  return cnn_features(conv_geom(nb, nf, batch), static_cast<const float2 *>(diag), (long long)nf * nb, nullptr, kappa,
                      feat, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tp_conv3x3_bf16(int32_t nf, int32_t nb, int32_t batch, int32_t cin, int32_t epilogue, const void *in,
                               const void *weights, const float *bias, const void *aux, void *out, float out_scale,
                               tp_stream_t stream) {
  const ConvGeom g = conv_geom(nb, nf, batch);
  return conv_layer(g, cin, epilogue, in, weights, bias, aux, epilogue == kEpiFilter ? nullptr : out,
                    epilogue == kEpiFilter ? out : nullptr, out_scale, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tp_conv3x3_wgrad(int32_t nf, int32_t nb, int32_t batch, int32_t cin, const void *x, const void *dy,
                                float *dw, float *db, tp_stream_t stream) {
  const ConvGeom g = conv_geom(nb, nf, batch);
  int rc = check_geom(g);
  if (rc != TP_OK) return rc;
  if (x == nullptr || dy == nullptr || dw == nullptr) return set_error(TP_ERR_INVALID, "tp_conv3x3_wgrad: NULL argument");
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(dy)) & 15u)
    return set_error(TP_ERR_INVALID, "tp_conv3x3_wgrad: buffers must be 16-byte aligned");
  int *err = device_error_ptr();
  if (err == nullptr) return set_error(TP_ERR_CUDA, "cannot resolve the device error word");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0, sms = 148;
  TP_CHECK_CUDA(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = conv_tiles(g);
  const int grid = ntiles < 2 * sms ? ntiles : 2 * sms;
  const size_t smem = wgrad_smem_bytes(cin, g.Wp);
  if (smem > (size_t)max_smem_optin()) return set_error(TP_ERR_UNSUPPORTED, "wgrad needs %zu B of shared memory", smem);
  if (cin == 16) {
    TP_CHECK_CUDA(cudaFuncSetAttribute(conv3x3_wgrad_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    conv3x3_wgrad_kernel<16><<<grid, 160, smem, st>>>(g, static_cast<const bf16 *>(x), static_cast<const bf16 *>(dy),
                                                       dw, db, ntiles, err);
  } else if (cin == 32) {
    TP_CHECK_CUDA(cudaFuncSetAttribute(conv3x3_wgrad_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    conv3x3_wgrad_kernel<32><<<grid, 320, smem, st>>>(g, static_cast<const bf16 *>(x), static_cast<const bf16 *>(dy),
                                                       dw, db, ntiles, err);
  } else {
    return set_error(TP_ERR_UNSUPPORTED, "tp_conv3x3_wgrad: cin must be 16 or 32");
  }
  return check_cuda(cudaGetLastError(), "conv3x3_wgrad_kernel launch");
}

extern "C" int tp_cnn_filter_apply(int32_t nf, int32_t nb, int32_t nvec, int32_t per_image, int32_t conj,
                                   const void *filt, const void *z, void *y, tp_stream_t stream) {
  if (filt == nullptr || z == nullptr || y == nullptr || nvec < 1 || nf < 1 || nb < 1 || per_image < 0)
    return set_error(TP_ERR_INVALID, "tp_cnn_filter_apply: bad argument");
  const int nimg = per_image > 0 ? (nvec + per_image - 1) / per_image : 1;
  const size_t hw = (size_t)nf * nb;
  const int gx = (int)((hw + 255) / 256 < 4096 ? (hw + 255) / 256 : 4096);
  cnn_filter_apply_kernel<<<dim3(gx, nvec), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      nb, nf, nvec, per_image, nimg, conj, static_cast<const float2 *>(filt), static_cast<const float2 *>(z),
      static_cast<float2 *>(y));
  return check_cuda(cudaGetLastError(), "cnn_filter_apply_kernel launch");
}

extern "C" int tp_cnn_filter_grad(int32_t nf, int32_t nb, int32_t nimg, int32_t per_image, const void *z, const void *e,
                                  float out_scale, void *dy, tp_stream_t stream) {
  if (z == nullptr || e == nullptr || dy == nullptr || per_image < 1 || nimg < 1)
    return set_error(TP_ERR_INVALID, "tp_cnn_filter_grad: bad argument");
  const ConvGeom g = conv_geom(nb, nf, nimg);
  int rc = check_geom(g);
  if (rc != TP_OK) return rc;
  cnn_filter_grad_kernel<<<592, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      g, per_image, static_cast<const float2 *>(z), static_cast<const float2 *>(e), out_scale, static_cast<bf16 *>(dy));
  return check_cuda(cudaGetLastError(), "cnn_filter_grad_kernel launch");
}

extern "C" size_t tp_cnn_forward_ws_bytes(int32_t nf, int32_t nb, int32_t batch) {
  if (nf < 1 || nb < 1 || batch < 1) return 0;
  return cnn_forward_ws_bytes(conv_geom(nb, nf, batch));
}

extern "C" int tp_cnn_forward(int32_t nf, int32_t nb, int32_t batch, const tp_cnn_model *model, const void *diag,
                              void *ws, size_t ws_bytes, void *filt, tp_stream_t stream) {
  if (model == nullptr || diag == nullptr || ws == nullptr || filt == nullptr)
    return set_error(TP_ERR_INVALID, "tp_cnn_forward: NULL argument");
  const ConvGeom g = conv_geom(nb, nf, batch);
  if (ws_bytes < cnn_forward_ws_bytes(g))
    return set_error(TP_ERR_WORKSPACE, "tp_cnn_forward: workspace %zu B < %zu B", ws_bytes, cnn_forward_ws_bytes(g));
  return cnn_forward(g, *model, static_cast<const float2 *>(diag), (long long)nf * nb, nullptr, ws,
                     static_cast<float2 *>(filt), reinterpret_cast<cudaStream_t>(stream));
}
