// Batched 1D FFTs, far-field / amplitude-loss heads and the 2D multislice
// (angular-spectrum) march with its adjoint, all on the shared-memory FFT of
// fft.cuh.
//
// Replaces: numpy.fft in the far field (forward_model/base/base_solver.py:
// 234-242) and the phase-retrieval projection (reconstruction/
// base_reconstructor.py:171-207); the multislice solver's per-probe loop
// (forward_model/multislice/ms_solver.py:49-159).
#include <cuda_runtime.h>

#include "fft.cuh"
#include "tp_errors.h"
#include "tpcuda.h"

namespace tp {

constexpr int kFftThreads = 256;

static int fft_rows_per_cta(int n) {
  int r = kFftMaxN / n;
  if (r > 8) r = 8;
  return r < 1 ? 1 : r;
}

// ------------------------------------------------------------------ 1D FFT
__global__ void __launch_bounds__(kFftThreads) fft1d_kernel(const FftPlan pl, int batch, const float2 *__restrict__ in,
                                                            float2 *__restrict__ out, int inverse, int rows) {
  extern __shared__ __align__(16) float2 fsm[];
  const int n = pl.n;
  float2 *tw = fsm, *a = fsm + n, *b = a + rows * n;
  const int r0 = blockIdx.x * rows;
  const int nb = min(rows, batch - r0);
  fft_twiddles(tw, n, threadIdx.x, blockDim.x);
  for (int e = threadIdx.x; e < nb * n; e += blockDim.x) a[e] = in[(size_t)r0 * n + e];
  __syncthreads();
  float2 *res = fft_block(a, b, pl, tw, inverse != 0, nb, threadIdx.x, blockDim.x);
  const float s = inverse ? 1.f / (float)n : 1.f;
  for (int e = threadIdx.x; e < nb * n; e += blockDim.x) {
    const float2 v = res[e];
    out[(size_t)r0 * n + e] = make_float2(v.x * s, v.y * s);
  }
}

// |FFT(exit)|^2 (intensity, unnormalised, no shift)
__global__ void __launch_bounds__(kFftThreads) farfield_kernel(const FftPlan pl, int batch, const float2 *__restrict__ in,
                                                               float *__restrict__ out, int rows) {
  extern __shared__ __align__(16) float2 fsm[];
  const int n = pl.n;
  float2 *tw = fsm, *a = fsm + n, *b = a + rows * n;
  const int r0 = blockIdx.x * rows;
  const int nb = min(rows, batch - r0);
  fft_twiddles(tw, n, threadIdx.x, blockDim.x);
  for (int e = threadIdx.x; e < nb * n; e += blockDim.x) a[e] = in[(size_t)r0 * n + e];
  __syncthreads();
  float2 *res = fft_block(a, b, pl, tw, false, nb, threadIdx.x, blockDim.x);
  for (int e = threadIdx.x; e < nb * n; e += blockDim.x) {
    const float2 v = res[e];
    out[(size_t)r0 * n + e] = fmaf(v.x, v.x, v.y * v.y);
  }
}

// loss = sum (|F e| - a)^2 ;  grad = sum_k F^H[2 (|U|-a) U/|U|]  (torch convention)
__global__ void __launch_bounds__(kFftThreads) amp_residual_kernel(const FftPlan pl, int batch,
                                                                   const float2 *__restrict__ ex,
                                                                   const float *__restrict__ amp,
                                                                   float2 *__restrict__ grad, double *loss, int rows) {
  extern __shared__ __align__(16) float2 fsm[];
  __shared__ double red[kFftThreads / 32];
  const int n = pl.n;
  float2 *tw = fsm, *a = fsm + n, *b = a + rows * n;
  const int r0 = blockIdx.x * rows;
  const int nb = min(rows, batch - r0);
  fft_twiddles(tw, n, threadIdx.x, blockDim.x);
  for (int e = threadIdx.x; e < nb * n; e += blockDim.x) a[e] = ex[(size_t)r0 * n + e];
  __syncthreads();
  float2 *U = fft_block(a, b, pl, tw, false, nb, threadIdx.x, blockDim.x);
  double acc = 0.0;
  for (int e = threadIdx.x; e < nb * n; e += blockDim.x) {
    const float2 u = U[e];
    const double mag = sqrt((double)u.x * u.x + (double)u.y * u.y);
    const double d = mag - (double)amp[(size_t)r0 * n + e];
    acc += d * d;
    const float f = mag > 0.0 ? (float)(2.0 * d / mag) : 0.f;
    U[e] = make_float2(f * u.x, f * u.y);
  }
  __syncthreads();
  float2 *other = (U == a) ? b : a;
  float2 *G = fft_block(U, other, pl, tw, true, nb, threadIdx.x, blockDim.x);  // unnormalised inverse = F^H
  for (int e = threadIdx.x; e < nb * n; e += blockDim.x) grad[(size_t)r0 * n + e] = G[e];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += red[w];
    atomicAdd(loss, s);
  }
}

// ---------------------------------------------------------------- multislice
struct MsParams {
  int n, nz, L, P;
  double k, dx, dz;
  double nmr, nmi;  // medium index
  const void *field;
  int dtype;
  const float2 *trans;  // (L, n)
  const float2 *probes;
  float2 *u_store;  // (P, nz, n) or null
  float2 *exit_out;
  const float2 *u_fwd;   // backward: forward field (P, nz, n)
  const float2 *src_exit;
  float2 *grad_t;  // backward: (L, n) accumulator of sum_p conj(T_z u_z) g_z
};

// T_z[x] - 1 with T_z[x] = exp(i k (n[x,z] - n_medium) dz), z = 0..L-1
// (ms_solver.py:86-88).  The table holds the deviation from one, computed in
// fp64 (expm1, -2 sin^2): T is 1 + O(k dn dz) and rounding it to fp32 every
// slice would bias the march.
__global__ void ms_transmission_kernel(const MsParams q, float2 *__restrict__ trans) {
  const size_t total = (size_t)q.L * q.n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(idx % q.n), z = (int)(idx / q.n);
    double nr, ni;
    if (q.dtype == TP_C128) {
      const double2 v = static_cast<const double2 *>(q.field)[(size_t)x * q.nz + z];
      nr = v.x;
      ni = v.y;
    } else {
      const float2 v = static_cast<const float2 *>(q.field)[(size_t)x * q.nz + z];
      nr = v.x;
      ni = v.y;
    }
    const double ph = q.k * (nr - q.nmr) * q.dz, am1 = expm1(-q.k * (ni - q.nmi) * q.dz);
    double s, c, sh, ch;
    sincos(ph, &s, &c);
    sincos(0.5 * ph, &sh, &ch);
    // e^a (c + i s) - 1 = (e^a - 1) c + (c - 1) + i e^a s,  c - 1 = -2 sin^2(ph/2)
    trans[idx] = make_float2((float)(am1 * c - 2.0 * sh * sh), (float)((am1 + 1.0) * s));
  }
}

// H[j] - 1 with H[j] = exp(i (kz - k) dz), kz = sqrt(max(k^2 - kx^2, 0)),
// kx = 2 pi fftfreq(n, dx) (ms_solver.py:49-72); fp64, kept as the deviation
// from one like the transmission.
__device__ __forceinline__ void ms_kernel_H(float2 *H, const MsParams &q, int tid, int nth) {
  for (int j = tid; j < q.n; j += nth) {
    const int f = (j < (q.n + 1) / 2) ? j : j - q.n;
    const double kx = 2.0 * 3.14159265358979323846 * (double)f / ((double)q.n * q.dx);
    const double kz = sqrt(fmax(q.k * q.k - kx * kx, 0.0));
    const double th = (kz - q.k) * q.dz;
    double s, c, sh, ch;
    sincos(th, &s, &c);
    sincos(0.5 * th, &sh, &ch);
    H[j] = make_float2((float)(-2.0 * sh * sh), (float)s);
  }
}

// One CTA marches `rows` probes through all slices (the field stays in
// shared memory).  Each slice is evaluated in delta form,
//   X = psi + (T_z - 1) psi,   psi' = X + IFFT((H - 1) . FFT(X)),
// so the FFT round-off scales with the small update instead of the field
// (the same reason the CN march keeps "1 + eps" coefficients).  X stays in
// registers: a thread owns elements tid + j*nth, j < E (E = 8, 16 or 32:
// rows * n <= E * kFftThreads).
constexpr int kMsElems = 32;  // the largest E

template <int E>
__global__ void __launch_bounds__(kFftThreads) ms_march_kernel(const FftPlan pl, const MsParams q, int rows) {
  extern __shared__ __align__(16) float2 fsm[];
  const int n = q.n, tid = threadIdx.x, nth = blockDim.x;
  float2 *tw = fsm, *H = tw + n, *a = H + n, *b = a + rows * n;
  const int p0 = blockIdx.x * rows;
  const int nb = min(rows, q.P - p0);
  const int tot = nb * n;
  fft_twiddles(tw, n, tid, nth);
  ms_kernel_H(H, q, tid, nth);
  float2 X[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int e = tid + j * nth;
    if (e < tot) {
      X[j] = q.probes[(size_t)p0 * n + e];
      if (q.u_store) q.u_store[((size_t)(p0 + e / n) * q.nz) * n + e % n] = X[j];
    }
  }
  __syncthreads();
  const float s = 1.f / (float)n;
  for (int z = 0; z < q.L; ++z) {
    const float2 *Tz = q.trans + (size_t)z * n;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = tid + j * nth;
      if (e < tot) {
        X[j] = cfma(Tz[e % n], X[j], X[j]);
        a[e] = X[j];
      }
    }
    __syncthreads();
    float2 *F = fft_block(a, b, pl, tw, false, nb, tid, nth);
    float2 *o = (F == a) ? b : a;
    for (int e = tid; e < tot; e += nth) F[e] = cmul(F[e], H[e % n]);
    __syncthreads();
    float2 *R = fft_block(F, o, pl, tw, true, nb, tid, nth);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = tid + j * nth;
      if (e < tot) {
        X[j] = make_float2(fmaf(R[e].x, s, X[j].x), fmaf(R[e].y, s, X[j].y));
        if (q.u_store) q.u_store[((size_t)(p0 + e / n) * q.nz + z + 1) * n + e % n] = X[j];
        if (z == q.L - 1 && q.exit_out) q.exit_out[(size_t)p0 * n + e] = X[j];
      }
    }
    __syncthreads();
  }
}

// Adjoint march (delta form as the forward): g = lambda + IFFT(conj(H - 1) .
// FFT(lambda)); grad_t[z] += sum_p g conj(T_z u_z); lambda <- conj(T_z) g,
// from lambda = src_exit at the exit plane.
template <int E>
__global__ void __launch_bounds__(kFftThreads) ms_backward_kernel(const FftPlan pl, const MsParams q, int rows) {
  extern __shared__ __align__(16) float2 fsm[];
  const int n = q.n, tid = threadIdx.x, nth = blockDim.x;
  float2 *tw = fsm, *H = tw + n, *a = H + n, *b = a + rows * n;
  const int p0 = blockIdx.x * rows;
  const int nb = min(rows, q.P - p0);
  const int tot = nb * n;
  fft_twiddles(tw, n, tid, nth);
  ms_kernel_H(H, q, tid, nth);
  float2 X[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int e = tid + j * nth;
    if (e < tot) {
      X[j] = q.src_exit[(size_t)p0 * n + e];
      a[e] = X[j];
    }
  }
  __syncthreads();
  const float s = 1.f / (float)n;
  for (int z = q.L - 1; z >= 0; --z) {
    float2 *F = fft_block(a, b, pl, tw, false, nb, tid, nth);
    float2 *o = (F == a) ? b : a;
    for (int e = tid; e < tot; e += nth) F[e] = cmulc(F[e], H[e % n]);
    __syncthreads();
    float2 *G = fft_block(F, o, pl, tw, true, nb, tid, nth);
    const float2 *Tz = q.trans + (size_t)z * n;
    // g = X + s*G ; contribution g conj(T u); X <- conj(T) g = g + conj(T-1) g
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = tid + j * nth;
      if (e < tot) {
        const float2 g = make_float2(fmaf(G[e].x, s, X[j].x), fmaf(G[e].y, s, X[j].y));
        const float2 tm1 = Tz[e % n];
        const float2 u = q.u_fwd[((size_t)(p0 + e / n) * q.nz + z) * n + e % n];
        const float2 tu = cfma(tm1, u, u);
        const float2 c = cmulc(g, tu);
        float2 *dst = q.grad_t + (size_t)z * n + e % n;
        asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(dst), "f"(c.x), "f"(c.y) : "memory");
        X[j] = cadd(g, cmulc(g, tm1));
        a[e] = X[j];
      }
    }
    __syncthreads();
  }
}

static size_t fft_smem(int n, int rows, int extra) { return (size_t)(extra * n + 2 * rows * n) * sizeof(float2); }

int ms_transmission_launch(int n_total, int nz, double k, double dz, double nmr, double nmi, const void *field,
                           int dtype, float2 *trans, cudaStream_t st) {
  MsParams q{};
  q.n = n_total;
  q.nz = nz;
  q.L = nz - 1;
  q.k = k;
  q.dz = dz;
  q.nmr = nmr;
  q.nmi = nmi;
  q.field = field;
  q.dtype = dtype;
  ms_transmission_kernel<<<592, 256, 0, st>>>(q, trans);
  return check_cuda(cudaGetLastError(), "ms_transmission_kernel launch");
}

static int fft_launch_setup(const void *kern, size_t smem) {
  return check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                    "cudaFuncSetAttribute(fft)");
}

}  // namespace tp

using namespace tp;

static int fft_plan_or_error(int n, FftPlan *pl) {
  *pl = make_fft_plan(n);
  if (pl->npass == 0)
    return set_error(TP_ERR_UNSUPPORTED, "FFT length %d unsupported (need 2^a 3^b 5^c <= %d)", n, kFftMaxN);
  return TP_OK;
}

extern "C" int tp_fft1d(int32_t n, int32_t batch, const void *in, void *out, int32_t inverse, tp_stream_t stream) {
  FftPlan pl;
  int rc = fft_plan_or_error(n, &pl);
  if (rc) return rc;
  if (in == nullptr || out == nullptr || batch < 1) return set_error(TP_ERR_INVALID, "bad tp_fft1d arguments");
  const int rows = fft_rows_per_cta(n);
  const size_t smem = fft_smem(n, rows, 1);
  rc = fft_launch_setup((const void *)fft1d_kernel, smem);
  if (rc) return rc;
  fft1d_kernel<<<(batch + rows - 1) / rows, kFftThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      pl, batch, static_cast<const float2 *>(in), static_cast<float2 *>(out), inverse, rows);
  return check_cuda(cudaGetLastError(), "fft1d_kernel launch");
}

extern "C" int tp_farfield_intensity(int32_t n, int32_t batch, const void *exit_waves, float *intensity,
                                     tp_stream_t stream) {
  FftPlan pl;
  int rc = fft_plan_or_error(n, &pl);
  if (rc) return rc;
  if (exit_waves == nullptr || intensity == nullptr || batch < 1) return set_error(TP_ERR_INVALID, "bad farfield args");
  const int rows = fft_rows_per_cta(n);
  const size_t smem = fft_smem(n, rows, 1);
  rc = fft_launch_setup((const void *)farfield_kernel, smem);
  if (rc) return rc;
  farfield_kernel<<<(batch + rows - 1) / rows, kFftThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      pl, batch, static_cast<const float2 *>(exit_waves), intensity, rows);
  return check_cuda(cudaGetLastError(), "farfield_kernel launch");
}

extern "C" int tp_amplitude_residual(int32_t n, int32_t batch, const void *exit_waves, const float *amplitude,
                                     void *grad_out, double *loss_out, tp_stream_t stream) {
  FftPlan pl;
  int rc = fft_plan_or_error(n, &pl);
  if (rc) return rc;
  if (!exit_waves || !amplitude || !grad_out || !loss_out || batch < 1)
    return set_error(TP_ERR_INVALID, "bad amplitude-residual args");
  const int rows = fft_rows_per_cta(n);
  const size_t smem = fft_smem(n, rows, 1);
  rc = fft_launch_setup((const void *)amp_residual_kernel, smem);
  if (rc) return rc;
  amp_residual_kernel<<<(batch + rows - 1) / rows, kFftThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      pl, batch, static_cast<const float2 *>(exit_waves), amplitude, static_cast<float2 *>(grad_out), loss_out, rows);
  return check_cuda(cudaGetLastError(), "amp_residual_kernel launch");
}

static int ms_params(const tp_ms2d_op *op, MsParams *q) {
  if (op == nullptr) return set_error(TP_ERR_INVALID, "op is NULL");
  if (op->nz < 2) return set_error(TP_ERR_INVALID, "nz=%d must be >= 2", op->nz);
  *q = MsParams{};
  q->n = op->n;
  q->nz = op->nz;
  q->L = op->nz - 1;
  q->k = op->k;
  q->dx = op->dx;
  q->dz = op->dz;
  q->nmr = op->n_medium[0];
  q->nmi = op->n_medium[1];
  return TP_OK;
}

extern "C" int tp_ms2d_transmission(const tp_ms2d_op *op, const void *n_field, int32_t n_dtype, void *trans,
                                    tp_stream_t stream) {
  MsParams q;
  int rc = ms_params(op, &q);
  if (rc) return rc;
  if (!n_field || !trans) return set_error(TP_ERR_INVALID, "n_field/trans is NULL");
  return ms_transmission_launch(q.n, q.nz, q.k, q.dz, q.nmr, q.nmi, n_field, n_dtype, static_cast<float2 *>(trans),
                                reinterpret_cast<cudaStream_t>(stream));
}

// Probes per CTA: at most what kMsElems field values per thread hold and
// what fits in 200 KB of shared memory (two FFT buffers per probe, H and the
// twiddles), at most 4, and no more than needed to give every SM a CTA.
static int ms_rows(int n, int num_probes) {
  int r = (kMsElems * kFftThreads) / n;
  const int rs = (200 * 1024 / (int)sizeof(float2) - 2 * n) / (2 * n);
  if (rs < r) r = rs;
  if (r > 4) r = 4;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int fill = (num_probes + sms - 1) / sms;
  if (r > fill) r = fill < 1 ? 1 : fill;
  return r;
}

// Field values per thread for `rows` probes of length n (a compiled E).
static int ms_elems(int n, int rows) {
  const int e = (rows * n + kFftThreads - 1) / kFftThreads;
  return e <= 8 ? 8 : (e <= 16 ? 16 : 32);
}

extern "C" int tp_ms2d_march(const tp_ms2d_op *op, const void *trans, const void *probes, int32_t num_probes,
                             void *u_store, void *exit_out, tp_stream_t stream) {
  MsParams q;
  int rc = ms_params(op, &q);
  if (rc) return rc;
  FftPlan pl;
  rc = fft_plan_or_error(op->n, &pl);
  if (rc) return rc;
  if (!trans || !probes || num_probes < 1) return set_error(TP_ERR_INVALID, "bad ms march args");
  q.P = num_probes;
  q.trans = static_cast<const float2 *>(trans);
  q.probes = static_cast<const float2 *>(probes);
  q.u_store = static_cast<float2 *>(u_store);
  q.exit_out = static_cast<float2 *>(exit_out);
  const int rows = ms_rows(op->n, num_probes);
  if (rows < 1) return set_error(TP_ERR_UNSUPPORTED, "N=%d too large for the multislice kernel", op->n);
  const size_t smem = fft_smem(op->n, rows, 2);
  const int E = ms_elems(op->n, rows);
  auto kern = E == 8 ? ms_march_kernel<8> : (E == 16 ? ms_march_kernel<16> : ms_march_kernel<32>);
  rc = fft_launch_setup((const void *)kern, smem);
  if (rc) return rc;
  kern<<<(num_probes + rows - 1) / rows, kFftThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(pl, q, rows);
  return check_cuda(cudaGetLastError(), "ms_march_kernel launch");
}

extern "C" int tp_ms2d_backward(const tp_ms2d_op *op, const void *trans, const void *u_fwd, const void *src_exit,
                                int32_t num_probes, void *grad_t, tp_stream_t stream) {
  MsParams q;
  int rc = ms_params(op, &q);
  if (rc) return rc;
  FftPlan pl;
  rc = fft_plan_or_error(op->n, &pl);
  if (rc) return rc;
  if (!trans || !u_fwd || !src_exit || !grad_t || num_probes < 1) return set_error(TP_ERR_INVALID, "bad ms backward args");
  q.P = num_probes;
  q.trans = static_cast<const float2 *>(trans);
  q.u_fwd = static_cast<const float2 *>(u_fwd);
  q.src_exit = static_cast<const float2 *>(src_exit);
  q.grad_t = static_cast<float2 *>(grad_t);
  const int rows = ms_rows(op->n, num_probes);
  if (rows < 1) return set_error(TP_ERR_UNSUPPORTED, "N=%d too large for the multislice kernel", op->n);
  const size_t smem = fft_smem(op->n, rows, 2);
  const int E = ms_elems(op->n, rows);
  auto kern = E == 8 ? ms_backward_kernel<8> : (E == 16 ? ms_backward_kernel<16> : ms_backward_kernel<32>);
  rc = fft_launch_setup((const void *)kern, smem);
  if (rc) return rc;
  kern<<<(num_probes + rows - 1) / rows, kFftThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(pl, q, rows);
  return check_cuda(cudaGetLastError(), "ms_backward_kernel launch");
}
