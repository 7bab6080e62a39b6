// Internal declarations of the learned 3D preconditioner (cnn_tc.cu), shared
// with the 3D march (cn3d.cu).
//
// Activations live in a "padded-linear" bf16 layout: each image of H x W
// pixels is surrounded by a one-pixel zero border (Hp = H + 2 rows of
// Wp = W + 2), the images of a batch follow each other, and the channels are
// stored in chunks of 8: element (chunk j, pixel l, channel 8j + c) sits at
// ((j * CS + l) * 8 + c).  A 3x3 tap is then a constant shift of the linear
// pixel index (dy * Wp + dx), so the implicit-GEMM A operand of a tap is a
// contiguous run of 16-byte pixel rows in shared memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tpcuda.h"

namespace tp {

constexpr int kConvBlocks = 4;                 // 128-pixel M blocks per CTA
constexpr int kConvTile = 128 * kConvBlocks;   // output pixels per CTA
constexpr int kConvCout = 32;                  // output channels of every layer
constexpr int kFilterTaps = 13;                // taps of the learned per-pixel filter

// Offsets (row, column) of the filter taps: the centre, the 8 neighbours and
// the 4 axial pixels at distance 2.
__host__ __device__ inline int filter_tap_dy(int t) {
  const int v[kFilterTaps] = {0, 0, 0, -1, 1, -1, -1, 1, 1, 0, 0, -2, 2};
  return v[t];
}
__host__ __device__ inline int filter_tap_dx(int t) {
  const int v[kFilterTaps] = {0, -1, 1, 0, 0, -1, 1, -1, 1, -2, 2, 0, 0};
  return v[t];
}

struct ConvGeom {
  int H, W, Wp, batch;
  long long S;        // pixels of one padded image, (H + 2) * Wp
  long long G0;       // zero guard before the first image
  long long CS;       // pixels per channel chunk (guards included)
  long long l_begin;  // first computed linear pixel
  long long l_end;    // one past the last computed linear pixel
};

ConvGeom conv_geom(int H, int W, int batch);
size_t act_bytes(const ConvGeom &g, int channels);
int conv_tiles(const ConvGeom &g);

enum ConvEpi { kEpiRelu = 0, kEpiMask = 1, kEpiFilter = 2 };

// Features of the index perturbation of one slice per image:
// [kappa Re d, kappa Im d, 1, x == 0, x == W-1, y == 0, y == H-1, 0 ...]
// (16 channels), d = diag[img] - kc (kc may be NULL).
int cnn_features(const ConvGeom &g, const float2 *diag, long long diag_stride, const float2 *kc, float kappa,
                 void *feat, cudaStream_t st);

// One 3x3 layer with 32 output channels (tcgen05 implicit GEMM).
int conv_layer(const ConvGeom &g, int cin, int epi, const void *in, const void *w, const float *bias, const void *aux,
               void *out, void *filt, float out_scale, cudaStream_t st);

// Four-layer forward from the features to the per-pixel filter (13, batch*H*W)
// float2.  `ws` holds the activations (cnn_forward_ws_bytes).
size_t cnn_forward_ws_bytes(const ConvGeom &g);
int cnn_forward(const ConvGeom &g, const tp_cnn_model &m, const float2 *diag, long long diag_stride, const float2 *kc,
                void *ws, float2 *filt, cudaStream_t st);

// y = z + sum_t F_t(x) z(x + o_t) (F conjugated when conj != 0) for `nvec`
// vectors of H*W; vector v uses filter image v / per_image (per_image = 0: image 0).
__device__ __forceinline__ float2 filter_apply_px(const float2 *__restrict__ F, size_t fimg, size_t np,
                                                   const float2 *__restrict__ z, int H, int W, int b, int f, int conj) {
  const size_t i = (size_t)b * W + f;
  float2 acc = z[i];
#pragma unroll
  for (int t = 0; t < kFilterTaps; ++t) {
    const int bb = b + filter_tap_dy(t), ff = f + filter_tap_dx(t);
    if (bb < 0 || bb >= H || ff < 0 || ff >= W) continue;
    float2 w = F[(size_t)t * np + fimg + i];
    if (conj) w.y = -w.y;
    const float2 v = z[(size_t)bb * W + ff];
    acc.x = fmaf(w.x, v.x, fmaf(-w.y, v.y, acc.x));
    acc.y = fmaf(w.x, v.y, fmaf(w.y, v.x, acc.y));
  }
  return acc;
}

}  // namespace tp
