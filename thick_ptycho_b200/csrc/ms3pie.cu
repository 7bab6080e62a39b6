// Multislice 3PIE reconstruction (reconstruction/ms_reconstructor.py:40-190)
// on the GPU.
//
// 3PIE updates the object probe by probe: every probe's forward march sees
// the estimate left by the previous probe, so the algorithm is sequential
// over probes and slices.  One CTA runs it all: epochs x probes in scan
// order; per probe a forward multislice march (transmit, FFT, angular
// spectrum kernel H, inverse FFT) storing the field in a caller workspace,
// the modulus constraint on the exit wave
// (psi_c = F^-1(sqrt(I) F psi / (|F psi| + 1e-12))), then from the detector
// plane to the entrance, for every slice z (last first): psi <- F^-1(conj(H)
// F psi), psi <- psi conj(T_z), dpsi = psi - u_z and
// n_z += (alpha / (epoch + 1)) conj(u_z) dpsi / (max|u_z|^2 + 1e-12) / (i k dz).
// Every FFT is the shared-memory Stockham FFT of fft.cuh on one CTA; the
// estimate n is kept in fp64, transmissions are applied as psi + psi (T - 1)
// with T - 1 evaluated in fp64 (T is 1 + O(k dn dz)).
#include <cuda_runtime.h>
#include <math.h>

#include "fft.cuh"
#include "tp_errors.h"
#include "tpcuda.h"

namespace tp {

constexpr int kPieThreads = 1024;

struct PieParams {
  int n, nz, P, iters, phase_retrieval;
  double k, dx, dz, alpha, nmr, nmi;
  double2 *n_est;          // (n, nz) row-major, in/out
  const float2 *probes;    // (P, n)
  const float *intensity;  // (P, n) (phase retrieval)
  const float2 *exit_known;  // (P, n) (known exit waves)
  float2 *u;               // workspace (nz, n): the current probe's forward field
  double *loss;            // (iters)
};

// T - 1 = exp(i k (n - n_m) dz) - 1, fp64, with the medium's absorption.
__device__ __forceinline__ double2 trans_m1(const PieParams &q, double2 nv) {
  const double ar = q.k * q.dz * (nv.x - q.nmr), ai = q.k * q.dz * (nv.y - q.nmi);
  // exp(i (ar + i ai)) - 1 = exp(-ai) (cos ar + i sin ar) - 1
  double s, c;
  sincos(ar, &s, &c);
  const double e = exp(-ai);
  const double em1 = expm1(-ai);
  // e cos ar - 1 = (e - 1) cos ar + (cos ar - 1) = em1 cos ar - 2 sin^2(ar/2)
  const double sh = sin(0.5 * ar);
  return z2(em1 * c - 2.0 * sh * sh, e * s);
}

__device__ __forceinline__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  __syncthreads();
  return s;  // valid in thread 0
}

__device__ __forceinline__ double block_max_all(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    red[0] = m;
  }
  __syncthreads();
  const double m = red[0];
  __syncthreads();
  return m;
}

__global__ void __launch_bounds__(kPieThreads) ms_3pie_kernel(const FftPlan pl, const PieParams q) {
  extern __shared__ __align__(16) float2 psm[];
  __shared__ double red[kPieThreads / 32];
  const int n = q.n, tid = threadIdx.x, nth = blockDim.x;
  float2 *tw = psm, *H = tw + n, *A = H + n, *B = A + n;
  fft_twiddles(tw, n, tid, nth);
  for (int j = tid; j < n; j += nth) {  // angular-spectrum kernel, global phase removed (ms_solver.py:49-72)
    const int f = (j <= (n - 1) / 2) ? j : j - n;
    const double kx = 2.0 * M_PI * (double)f / ((double)n * q.dx);
    const double in = q.k * q.k - kx * kx;
    const double kz = in > 0.0 ? sqrt(in) : 0.0;
    double s, c;
    sincos((kz - q.k) * q.dz, &s, &c);
    H[j] = make_float2((float)c, (float)s);
  }
  __syncthreads();
  const float inv_n = 1.f / (float)n;
  float2 *cur = A, *oth = B;  // the working vector lives in cur
  for (int it = 0; it < q.iters; ++it) {
    double err2 = 0.0;
    const double step = q.alpha / (double)(it + 1);
    for (int p = 0; p < q.P; ++p) {
      // ---- forward march: u_0 = probe, u_{z+1} = F^-1(H F(u_z T_z))
      for (int x = tid; x < n; x += nth) {
        const float2 v = q.probes[(size_t)p * n + x];
        cur[x] = v;
        q.u[x] = v;
      }
      __syncthreads();
      for (int z = 0; z < q.nz - 1; ++z) {
        for (int x = tid; x < n; x += nth) {
          const double2 tm = trans_m1(q, q.n_est[(size_t)x * q.nz + z]);
          const float2 v = cur[x];
          cur[x] = cfma(to_f2(tm), v, v);
        }
        __syncthreads();
        float2 *F = fft_block(cur, oth, pl, tw, false, 1, tid, nth);
        for (int x = tid; x < n; x += nth) F[x] = cmul(F[x], H[x]);
        __syncthreads();
        float2 *o = (F == cur) ? oth : cur;
        float2 *R = fft_block(F, o, pl, tw, true, 1, tid, nth);
        float2 *Ro = (R == cur) ? oth : cur;
        for (int x = tid; x < n; x += nth) {
          const float2 v = make_float2(R[x].x * inv_n, R[x].y * inv_n);
          R[x] = v;
          q.u[(size_t)(z + 1) * n + x] = v;
        }
        __syncthreads();
        cur = R;
        oth = Ro;
      }
      // ---- modulus constraint on the exit wave (cur holds u_{nz-1})
      if (q.phase_retrieval) {
        float2 *F = fft_block(cur, oth, pl, tw, false, 1, tid, nth);
        for (int x = tid; x < n; x += nth) {
          const float2 v = F[x];
          const double mag = sqrt((double)v.x * v.x + (double)v.y * v.y);
          const double a = sqrt((double)q.intensity[(size_t)p * n + x]) / (mag + 1e-12);
          F[x] = make_float2((float)(a * v.x), (float)(a * v.y));
        }
        __syncthreads();
        float2 *o = (F == cur) ? oth : cur;
        float2 *R = fft_block(F, o, pl, tw, true, 1, tid, nth);
        float2 *Ro = (R == cur) ? oth : cur;
        for (int x = tid; x < n; x += nth) R[x] = make_float2(R[x].x * inv_n, R[x].y * inv_n);
        __syncthreads();
        cur = R;
        oth = Ro;
      } else {
        for (int x = tid; x < n; x += nth) cur[x] = q.exit_known[(size_t)p * n + x];
        __syncthreads();
      }
      double e2 = 0.0;
      const float2 *ex = q.u + (size_t)(q.nz - 1) * n;
      for (int x = tid; x < n; x += nth) {
        const float2 d = csub(cur[x], ex[x]);
        e2 += (double)d.x * d.x + (double)d.y * d.y;
      }
      const double s2 = block_sum(e2, red);
      if (tid == 0) err2 += s2;
      // ---- back propagation with the slice updates (last slice first)
      for (int z = q.nz - 1; z >= 0; --z) {
        float2 *F = fft_block(cur, oth, pl, tw, false, 1, tid, nth);
        for (int x = tid; x < n; x += nth) F[x] = cmulc(F[x], H[x]);  // conj(H)
        __syncthreads();
        float2 *o = (F == cur) ? oth : cur;
        float2 *R = fft_block(F, o, pl, tw, true, 1, tid, nth);
        float2 *Ro = (R == cur) ? oth : cur;
        const float2 *uz = q.u + (size_t)z * n;
        double m = 0.0;
        for (int x = tid; x < n; x += nth) {
          const float2 v = uz[x];
          m = fmax(m, (double)v.x * v.x + (double)v.y * v.y);
        }
        const double scale = block_max_all(m, red) + 1e-12;
        const double2 cstep = z2(0.0, -step / (q.k * q.dz * scale));  // step / (scale i k dz)
        for (int x = tid; x < n; x += nth) {
          const size_t ni = (size_t)x * q.nz + z;
          const double2 nv = q.n_est[ni];
          const double2 tm = trans_m1(q, nv);
          float2 psi = make_float2(R[x].x * inv_n, R[x].y * inv_n);
          psi = cadd(psi, cmulc(psi, to_f2(tm)));  // psi conj(T) = psi + psi conj(T - 1)
          R[x] = psi;
          const float2 uv = uz[x];
          const double2 d = z2((double)psi.x - uv.x, (double)psi.y - uv.y);
          const double2 g = zmul(z2(uv.x, -uv.y), d);  // conj(u) dpsi
          q.n_est[ni] = zadd(nv, zmul(cstep, g));
        }
        __syncthreads();
        cur = R;
        oth = Ro;
      }
    }
    if (tid == 0) q.loss[it] = sqrt(err2 / ((double)q.P * n));
  }
}

}  // namespace tp

using namespace tp;

extern "C" size_t tp_ms2d_3pie_workspace_bytes(int32_t n, int32_t nz) {
  if (n < 1 || nz < 2) return 0;
  return (size_t)n * nz * sizeof(float2);
}

extern "C" int tp_ms2d_3pie(const tp_ms2d_op *op, const void *probes, int32_t num_probes, const void *data,
                            int32_t phase_retrieval, int32_t iters, double alpha_obj, void *n_est, double *loss,
                            void *workspace, size_t workspace_bytes, tp_stream_t stream) {
  if (op == nullptr || probes == nullptr || data == nullptr || n_est == nullptr || loss == nullptr ||
      workspace == nullptr || num_probes < 1 || iters < 0 || op->nz < 2)
    return set_error(TP_ERR_INVALID, "bad tp_ms2d_3pie arguments");
  const FftPlan pl = make_fft_plan(op->n);
  if (pl.npass == 0) return set_error(TP_ERR_UNSUPPORTED, "FFT length %d unsupported (need 2^a 3^b 5^c <= 4096)", op->n);
  if (workspace_bytes < tp_ms2d_3pie_workspace_bytes(op->n, op->nz))
    return set_error(TP_ERR_WORKSPACE, "3PIE workspace %zu B < %zu B", workspace_bytes,
                     tp_ms2d_3pie_workspace_bytes(op->n, op->nz));
  PieParams q{};
  q.n = op->n;
  q.nz = op->nz;
  q.P = num_probes;
  q.iters = iters;
  q.phase_retrieval = phase_retrieval != 0;
  q.k = op->k;
  q.dx = op->dx;
  q.dz = op->dz;
  q.alpha = alpha_obj;
  q.nmr = op->n_medium[0];
  q.nmi = op->n_medium[1];
  q.n_est = static_cast<double2 *>(n_est);
  q.probes = static_cast<const float2 *>(probes);
  q.intensity = static_cast<const float *>(data);
  q.exit_known = static_cast<const float2 *>(data);
  q.u = static_cast<float2 *>(workspace);
  q.loss = loss;
  const size_t smem = (size_t)4 * op->n * sizeof(float2);
  TP_CHECK_CUDA(cudaFuncSetAttribute(ms_3pie_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ms_3pie_kernel<<<1, kPieThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(pl, q);
  return check_cuda(cudaGetLastError(), "ms_3pie_kernel launch");
}
