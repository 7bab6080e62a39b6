// Reconstruction-loop pieces of the reference's NLCG (2D), on stored fields.
//
// Both kernels read full fields in the chunked layout written by
// tp_cn2d_march (tp_cn2d_layout) and use the reference's constant gradient
// operator grad_A = -(diag(G) + subdiag(G)), G = (dz/2)(k/i)
// (forward_model.py:128-153), which pairs block b of the vector form (slice
// b+1) with u_{b+1} + u_b for b >= 1 and with u_1 alone for b = 0 (the
// reference's full-system gradient drops C_0 u_0, forward_model.py:151-153).
//
//   cn2d_refgrad_kernel: the reference's compute_grad_least_squares
//     (pwe_reconstructor.py:100-164): with the reference adjoint lambda
//     (mode ADJOINT, flipped output: column b pairs with block b),
//     S_b = sum_p conj(u_p[b+1] + [b>=1] u_p[b]) lambda_p[b],
//     grad_re = Re(conj(G) S_b), grad_im = Im(conj(G) S_b), z-major (L*N).
//   cn2d_alpha_source_kernel: the source grad_A @ u_p of compute_alphak
//     (pwe_reconstructor.py:166-219) in the march's src_probe layout
//     (P, L, N): src[p][b] = -G (u_p[b+1] + [b>=1] u_p[b]).
#include <cuda_runtime.h>

#include "cn2d_internal.cuh"
#include "tp_errors.h"

namespace tp {

// Matrix row of offset `off` within a chunked slice (-1 for padding rows).
__device__ __forceinline__ int chunk_row(int off, int M, int C, int pair, int N) {
  int i, k;
  if (pair) {
    const int q = off >> 1;
    k = q % C;
    i = (q / C) * 2 + (off & 1);
  } else {
    i = off / C;
    k = off % C;
  }
  const int g = k * M + i;
  return g < N ? g : -1;
}

__global__ void cn2d_refgrad_kernel(int P, int L, int nz, int Npad, int N, int M, int C, int pair, float2 G,
                                    const float2 *__restrict__ u, const float2 *__restrict__ lam, float *gre,
                                    float *gim) {
  const size_t total = (size_t)L * Npad;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(e / Npad), off = (int)(e - (size_t)b * Npad);
    const int g = chunk_row(off, M, C, pair, N);
    if (g < 0) continue;
    float2 S = make_float2(0.f, 0.f);
    for (int p = 0; p < P; ++p) {
      const size_t base = (size_t)p * nz * Npad + off;
      float2 w = u[base + (size_t)(b + 1) * Npad];
      if (b >= 1) w = cadd(w, u[base + (size_t)b * Npad]);
      S = cadd(S, cmulc(lam[base + (size_t)b * Npad], w));  // lambda * conj(w)
    }
    const float2 t = cmulc(S, G);  // conj(G) S
    gre[(size_t)b * N + g] = t.x;
    gim[(size_t)b * N + g] = t.y;
  }
}

__global__ void cn2d_alpha_source_kernel(int P, int L, int nz, int Npad, int N, int M, int C, int pair, float2 G,
                                         const float2 *__restrict__ u, float2 *src) {
  const size_t total = (size_t)P * L * Npad;
  const float2 mG = make_float2(-G.x, -G.y);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int off = (int)(e % Npad);
    const size_t pb = e / Npad;
    const int b = (int)(pb % L);
    const size_t p = pb / L;
    const int g = chunk_row(off, M, C, pair, N);
    if (g < 0) continue;
    const size_t base = p * nz * Npad + off;
    float2 w = u[base + (size_t)(b + 1) * Npad];
    if (b >= 1) w = cadd(w, u[base + (size_t)b * Npad]);
    src[(p * L + b) * N + g] = cmul(mG, w);
  }
}

static int recon_setup(const tp_cn2d_op *op, int P, Partition *pt) {
  if (op == nullptr || P < 1) return set_error(TP_ERR_INVALID, "bad reconstruction-kernel arguments");
  if (op->exact_ref_coeff || op->empty_px != 0)
    return set_error(TP_ERR_UNSUPPORTED, "the reference NLCG pieces need exact_ref_coeff = 0 and no empty-space padding");
  return partition_for(op->n, pt);
}

}  // namespace tp

using namespace tp;

extern "C" int tp_cn2d_ref_gradient(const tp_cn2d_op *op, int32_t num_probes, const void *u_store,
                                    const void *lam_store, float *grad_re, float *grad_im, tp_stream_t stream) {
  Partition pt{};
  int rc = recon_setup(op, num_probes, &pt);
  if (rc != TP_OK) return rc;
  if (u_store == nullptr || lam_store == nullptr || grad_re == nullptr || grad_im == nullptr)
    return set_error(TP_ERR_INVALID, "tp_cn2d_ref_gradient: NULL argument");
  const float2 G = make_float2(0.f, (float)(-0.5 * op->dz * op->k));  // (dz/2)(k/i)
  cn2d_refgrad_kernel<<<1184, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      num_probes, op->nz - 1, op->nz, pt.C * pt.M, op->n, pt.M, pt.C, pt.team, G, static_cast<const float2 *>(u_store),
      static_cast<const float2 *>(lam_store), grad_re, grad_im);
  return check_cuda(cudaGetLastError(), "cn2d_refgrad_kernel launch");
}

extern "C" int tp_cn2d_alpha_source(const tp_cn2d_op *op, int32_t num_probes, const void *u_store, void *src,
                                    tp_stream_t stream) {
  Partition pt{};
  int rc = recon_setup(op, num_probes, &pt);
  if (rc != TP_OK) return rc;
  if (u_store == nullptr || src == nullptr) return set_error(TP_ERR_INVALID, "tp_cn2d_alpha_source: NULL argument");
  const float2 G = make_float2(0.f, (float)(-0.5 * op->dz * op->k));
  cn2d_alpha_source_kernel<<<2368, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      num_probes, op->nz - 1, op->nz, pt.C * pt.M, op->n, pt.M, pt.C, pt.team, G, static_cast<const float2 *>(u_store),
      static_cast<float2 *>(src));
  return check_cuda(cudaGetLastError(), "cn2d_alpha_source_kernel launch");
}
