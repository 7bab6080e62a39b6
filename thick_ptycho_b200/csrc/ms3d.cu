// 3D angular-spectrum multislice (forward march and its adjoint).
//
// The reference's multislice solver is 2D only (forward_model/multislice/
// ms_solver.py:28-31 rejects a 3D simulation space); this is the same
// propagator on an (n1, n2) transverse grid:
//   psi <- IFFT2(H . FFT2(psi . T_z)),  T_z = exp(i k (n[:, z] - n_medium) dz),
//   H = exp(i (k_z - k) dz),  k_z = sqrt(max(k^2 - k1^2 - k2^2, 0)),
//   k1 = 2 pi fftfreq(n1, d1), k2 = 2 pi fftfreq(n2, d2)
// (the 2D kernel of ms_solver.py:49-72 with the transverse wavenumber made
// two-dimensional).  Element (a, b) of a slice sits at a * n2 + b, the
// C-order flattening of the reference's (nx, ny) arrays.
//
// A 256 x 256 slice (512 KB) does not fit one CTA's shared memory, so each
// slice is two kernels over all probes:
//   rows:    inverse row FFTs of the spectrum W, psi_{z+1} = X_z + result
//            (delta form, X_z = psi_z T_z), store, X_{z+1} = psi_{z+1} T_{z+1},
//            forward row FFTs into W;
//   columns: column FFTs, times (H - 1)/N, inverse column FFTs, in place.
// The field psi and the spectrum W (P x N complex64 each) are updated in place
// by the CTA that owns the rows, so a march needs no ping-pong buffers; at
// 64 probes of 256 x 256 both fit in L2.  T - 1 and H - 1 are kept as
// deviations from one, evaluated in fp64, so the fp32 FFT round-off scales
// with the per-slice update, not the field.
#include <cuda_runtime.h>

#include "fft.cuh"
#include "tp_errors.h"
#include "tpcuda.h"

namespace tp {

constexpr int kMs3Threads = 256;

// host helper of ms2d.cu: the fp64 T - 1 table of an (n_total, nz) index field
int ms_transmission_launch(int n_total, int nz, double k, double dz, double nmr, double nmi, const void *field,
                           int dtype, float2 *trans, cudaStream_t st);

struct Ms3Params {
  int n1, n2, N, nz, L, P;
  const float2 *trans;  // (L, N): T_z - 1
  const float2 *hm1t;   // (n2, n1): (H - 1) / N, transposed
  const float2 *tw1, *tw2;
  float2 *psi;          // (P, N): field (forward) or lambda (adjoint), in place
  float2 *W;            // (P, N): spectrum work buffer, in place
  const float2 *probes, *src_exit, *u_fwd;
  float2 *u_store, *exit_out, *grad_t;
};

enum Ms3Phase : int { kMs3FwdStart = 0, kMs3FwdStep = 1, kMs3BwdStart = 2, kMs3BwdStep = 3 };

// Twiddle table W_n^t = exp(-2 pi i t / n) (fp64, rounded once) for the row
// (n2) and column (n1) lengths.
__global__ void ms3_twiddle_kernel(int n, float2 *tw) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double sv, cv;
    sincospi(-2.0 * (double)t / (double)n, &sv, &cv);
    tw[t] = make_float2((float)cv, (float)sv);
  }
}

// (H - 1) / N at hm1t[b * n1 + a]; H - 1 = exp(i th) - 1 = -2 sin^2(th/2) + i sin th.
__global__ void ms3_kernel_h_kernel(int n1, int n2, double k, double d1, double d2, double dz, float2 *hm1t) {
  const int N = n1 * n2;
  const double inv = 1.0 / (double)N;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N; e += gridDim.x * blockDim.x) {
    const int b = e / n1, a = e - b * n1;
    const int fa = (a < (n1 + 1) / 2) ? a : a - n1;
    const int fb = (b < (n2 + 1) / 2) ? b : b - n2;
    const double k1 = 2.0 * 3.14159265358979323846 * (double)fa / ((double)n1 * d1);
    const double k2 = 2.0 * 3.14159265358979323846 * (double)fb / ((double)n2 * d2);
    const double kz = sqrt(fmax(k * k - k1 * k1 - k2 * k2, 0.0));
    const double th = (kz - k) * dz;
    double s, c, sh, ch;
    sincos(th, &s, &c);
    sincos(0.5 * th, &sh, &ch);
    hm1t[e] = make_float2((float)(-2.0 * sh * sh * inv), (float)(s * inv));
  }
}

// Rows (columns) per CTA of the compile-time plans: at most 16 and 4096 elements.
__host__ __device__ constexpr int ms3_fixed_per_cta(int n) { return 4096 / n > 16 ? 16 : 4096 / n; }

// Row pass of slice z (phase selects start / step, forward / adjoint).
// Grid (n1 / rpc, P): a CTA owns rpc rows of one probe.  The spectrum rows
// (into a) and the step's third operand (T_{z+1} forward, u_z adjoint, into
// the unpadded buffer c) are copied asynchronously at entry; with a
// compile-time plan (N2 > 0, rpc = ms3_fixed_per_cta(N2)) every thread owns
// EPT fixed elements whose field and T_z values are loaded into registers at
// entry too, so all loads overlap the inverse FFT.
template <int N2>
__global__ void __launch_bounds__(kMs3Threads) ms3_rows_kernel(const FftPlan pl, const Ms3Params q, int phase, int z,
                                                               int rpc_rt) {
  extern __shared__ __align__(16) float2 fsm[];
  constexpr bool FIX = N2 > 0;
  constexpr int RPC = FIX ? ms3_fixed_per_cta(N2 > 0 ? N2 : 1) : 1;
  constexpr int EPT = FIX ? RPC * N2 / kMs3Threads : 1;
  const int n = FIX ? N2 : q.n2, pr = blockIdx.y;
  const int rpc = FIX ? RPC : rpc_rt;
  float2 *tw = fsm, *a = tw + n, *b = a + rpc * fstride<N2>(n), *cbuf = b + rpc * fstride<N2>(n);
  const size_t pbase = (size_t)pr * q.N;
  const int g0 = blockIdx.x * rpc * n;  // first element of the CTA's rows within the slice
  const int tot = rpc * n;
  const int tid = threadIdx.x;
  auto slot = [&](int e) { return fslot<N2>(e / n, e % n, n); };
  load_twiddles(tw, q.tw2, n);
  float2 *out = a;  // the buffer transformed forward into W at the end
  bool fwd_fft = true;
  if (phase == kMs3FwdStart) {
    const float2 *T0 = q.trans;
    for (int e = tid; e < tot; e += kMs3Threads) {
      const int g = g0 + e;
      const float2 v = q.probes[pbase + g];
      q.psi[pbase + g] = v;
      if (q.u_store) q.u_store[(size_t)pr * q.nz * q.N + g] = v;
      a[slot(e)] = cfma(T0[g], v, v);
    }
  } else if (phase == kMs3BwdStart) {
    for (int e = tid; e < tot; e += kMs3Threads) {
      const int g = g0 + e;
      const float2 v = q.src_exit[pbase + g];
      q.psi[pbase + g] = v;
      a[slot(e)] = v;
    }
  } else {
    const float2 *Tz = q.trans + (size_t)z * q.N;
    const bool last = (phase == kMs3FwdStep) && (z + 1 == q.L);
    const float2 *third = phase == kMs3FwdStep ? (last ? nullptr : q.trans + (size_t)(z + 1) * q.N + g0)
                                               : q.u_fwd + ((size_t)pr * q.nz + z) * q.N + g0;
    for (int e = tid; e < tot; e += kMs3Threads) {
      cp_async8(&a[slot(e)], &q.W[pbase + g0 + e]);
      if (third) cp_async8(&cbuf[e], &third[e]);
    }
    float2 pz[EPT], tz[EPT];
    if constexpr (FIX) {
#pragma unroll
      for (int j = 0; j < EPT; ++j) {
        const int g = g0 + tid + j * kMs3Threads;
        pz[j] = q.psi[pbase + g];
        tz[j] = Tz[g];
      }
    }
    cp_async_wait_all();
    __syncthreads();
    const float2 *R = fft_rows<N2>(a, b, pl, tw, true, rpc);
    out = (R == a) ? b : a;
    if (phase == kMs3FwdStep) {
      // psi_{z+1} = X_z + IFFT2((H-1) FFT2 X_z), X_z = psi_z + (T_z - 1) psi_z
      float2 *us = q.u_store ? q.u_store + ((size_t)pr * q.nz + z + 1) * q.N : nullptr;
      auto one = [&](int e, float2 pv, float2 tm1) {
        const int g = g0 + e;
        const float2 v = cadd(cfma(tm1, pv, pv), R[slot(e)]);
        q.psi[pbase + g] = v;
        if (us) us[g] = v;
        if (last) {
          if (q.exit_out) q.exit_out[pbase + g] = v;
        } else {
          out[slot(e)] = cfma(cbuf[e], v, v);  // X_{z+1} = psi_{z+1} T_{z+1}
        }
      };
      if constexpr (FIX) {
#pragma unroll
        for (int j = 0; j < EPT; ++j) one(tid + j * kMs3Threads, pz[j], tz[j]);
      } else {
        for (int e = tid; e < tot; e += kMs3Threads) one(e, q.psi[pbase + g0 + e], Tz[g0 + e]);
      }
      fwd_fft = !last;
    } else {
      // g_z = lambda_{z+1} + IFFT2(conj(H-1) FFT2 lambda_{z+1});
      // grad_t[z] += g_z conj(T_z u_z);  lambda_z = conj(T_z) g_z
      float2 *gt = q.grad_t + (size_t)z * q.N;
      auto one = [&](int e, float2 lam1, float2 tm1) {
        const int g = g0 + e;
        const float2 gv = cadd(lam1, R[slot(e)]);
        const float2 u = cbuf[e];  // u_z
        const float2 c = cmulc(gv, cfma(tm1, u, u));
        asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(gt + g), "f"(c.x), "f"(c.y) : "memory");
        const float2 lam = cadd(gv, cmulc(gv, tm1));
        q.psi[pbase + g] = lam;
        if (z > 0) out[slot(e)] = lam;
      };
      if constexpr (FIX) {
#pragma unroll
        for (int j = 0; j < EPT; ++j) one(tid + j * kMs3Threads, pz[j], tz[j]);
      } else {
        for (int e = tid; e < tot; e += kMs3Threads) one(e, q.psi[pbase + g0 + e], Tz[g0 + e]);
      }
      fwd_fft = z > 0;
    }
  }
  if (!fwd_fft) return;
  __syncthreads();
  float2 *scratch = (out == a) ? b : a;
  const float2 *F = fft_rows<N2>(out, scratch, pl, tw, false, rpc);
  for (int e = tid; e < tot; e += kMs3Threads) q.W[pbase + g0 + e] = F[slot(e)];
}

// Column pass: FFT along a, times (H - 1)/N (conjugated for the adjoint),
// inverse FFT along a, in place on W.  Grid (n2 / cpc, P).  The columns are
// copied asynchronously and, with a compile-time plan, the CTA's (H - 1)/N
// block is loaded into registers under the forward FFT.
template <int N1>
__global__ void __launch_bounds__(kMs3Threads) ms3_cols_kernel(const FftPlan pl, const Ms3Params q, int conj_h,
                                                               int cpc_rt) {
  extern __shared__ __align__(16) float2 fsm[];
  constexpr bool FIX = N1 > 0;
  constexpr int CPC = FIX ? ms3_fixed_per_cta(N1 > 0 ? N1 : 1) : 1;
  constexpr int EPT = FIX ? CPC * N1 / kMs3Threads : 1;
  const int n = FIX ? N1 : q.n1, pr = blockIdx.y;
  const int cpc = FIX ? CPC : cpc_rt;
  const int tid = threadIdx.x;
  float2 *tw = fsm, *a = tw + n, *b = a + cpc * fstride<N1>(n);
  const int b0 = blockIdx.x * cpc;
  float2 *base = q.W + (size_t)pr * q.N;
  const float2 *h = q.hm1t + (size_t)b0 * n;
  load_twiddles(tw, q.tw1, n);
  for (int e = tid; e < cpc * n; e += kMs3Threads) {
    const int c = e % cpc, r = e / cpc;  // coalesced over c
    cp_async8(&a[fslot<N1>(c, r, n)], &base[(size_t)r * q.n2 + b0 + c]);
  }
  float2 hv[EPT];
  if constexpr (FIX) {
#pragma unroll
    for (int j = 0; j < EPT; ++j) hv[j] = h[tid + j * kMs3Threads];
  }
  cp_async_wait_all();
  __syncthreads();
  float2 *F = fft_rows<N1>(a, b, pl, tw, false, cpc);
  float2 *o = (F == a) ? b : a;
  auto mul = [&](int e, float2 hh) {
    const int c = e / n, r = e - c * n;
    const int sl = fslot<N1>(c, r, n);
    F[sl] = conj_h ? cmulc(F[sl], hh) : cmul(F[sl], hh);
  };
  if constexpr (FIX) {
#pragma unroll
    for (int j = 0; j < EPT; ++j) mul(tid + j * kMs3Threads, hv[j]);
  } else {
    for (int e = tid; e < cpc * n; e += kMs3Threads) mul(e, h[e]);
  }
  __syncthreads();
  const float2 *R = fft_rows<N1>(F, o, pl, tw, true, cpc);
  for (int e = tid; e < cpc * n; e += kMs3Threads) {
    const int c = e % cpc, r = e / cpc;
    base[(size_t)r * q.n2 + b0 + c] = R[fslot<N1>(c, r, n)];
  }
}

using Ms3Rows = void (*)(const FftPlan, const Ms3Params, int, int, int);
using Ms3Cols = void (*)(const FftPlan, const Ms3Params, int, int);

template <int N>
static Ms3Rows ms3_rows_of() { return ms3_rows_kernel<N>; }
template <int N>
static Ms3Cols ms3_cols_of() { return ms3_cols_kernel<N>; }

// Compile-time plans for the common lengths, per axis.
static Ms3Rows pick_rows(int n) {
  switch (n) {
    case 32: return ms3_rows_of<32>();
    case 64: return ms3_rows_of<64>();
    case 128: return ms3_rows_of<128>();
    case 192: return ms3_rows_of<192>();
    case 256: return ms3_rows_of<256>();
    case 512: return ms3_rows_of<512>();
    default: return ms3_rows_of<0>();
  }
}
static Ms3Cols pick_cols(int n) {
  switch (n) {
    case 32: return ms3_cols_of<32>();
    case 64: return ms3_cols_of<64>();
    case 128: return ms3_cols_of<128>();
    case 192: return ms3_cols_of<192>();
    case 256: return ms3_cols_of<256>();
    case 512: return ms3_cols_of<512>();
    default: return ms3_cols_of<0>();
  }
}

// Transforms per CTA: at most 16 and 4096 elements, and a divisor of the count.
static int ms3_per_cta(int n, int count) {
  int r = 4096 / n;
  if (r > 16) r = 16;
  if (r < 1) r = 1;
  while (count % r != 0) --r;
  return r;
}

struct Ms3Work {
  float2 *psi, *W, *hm1t, *tw1, *tw2;
  size_t bytes;
};

static size_t a256(size_t b) { return (b + 255) & ~(size_t)255; }

static Ms3Work ms3_layout(char *base, int n1, int n2, int P) {
  Ms3Work w{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    float2 *p = base ? reinterpret_cast<float2 *>(base + off) : nullptr;
    off += a256(bytes);
    return p;
  };
  const size_t N = (size_t)n1 * n2;
  w.psi = take((size_t)P * N * sizeof(float2));
  w.W = take((size_t)P * N * sizeof(float2));
  w.hm1t = take(N * sizeof(float2));
  w.tw1 = take((size_t)n1 * sizeof(float2));
  w.tw2 = take((size_t)n2 * sizeof(float2));
  w.bytes = off;
  return w;
}

static int ms3_check_op(const tp_ms3d_op *op) {
  if (op == nullptr) return set_error(TP_ERR_INVALID, "op is NULL");
  if (op->nz < 2) return set_error(TP_ERR_INVALID, "nz=%d must be >= 2", op->nz);
  if (make_fft_plan(op->n1).npass == 0 || make_fft_plan(op->n2).npass == 0)
    return set_error(TP_ERR_UNSUPPORTED, "3D multislice grid %d x %d: each side must be 2^a 3^b 5^c <= %d", op->n1,
                     op->n2, kFftMaxN);
  if (!(op->k > 0.0) || !(op->d1 > 0.0) || !(op->d2 > 0.0))
    return set_error(TP_ERR_INVALID, "k, d1, d2 must be positive");
  return TP_OK;
}

// Runs the forward march (backward = false) or the adjoint march.
static int ms3_run(const tp_ms3d_op *op, Ms3Params q, bool backward, void *workspace, size_t workspace_bytes,
                   cudaStream_t st) {
  const int n1 = op->n1, n2 = op->n2;
  if (workspace == nullptr || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
    return set_error(TP_ERR_INVALID, "3D multislice workspace must be non-NULL and 256-byte aligned");
  Ms3Work w = ms3_layout(static_cast<char *>(workspace), n1, n2, q.P);
  if (workspace_bytes < w.bytes)
    return set_error(TP_ERR_WORKSPACE, "3D multislice workspace %zu B < %zu B", workspace_bytes, w.bytes);
  q.psi = w.psi;
  q.W = w.W;
  q.hm1t = w.hm1t;
  q.tw1 = w.tw1;
  q.tw2 = w.tw2;
  ms3_twiddle_kernel<<<(n1 + 255) / 256, 256, 0, st>>>(n1, w.tw1);
  ms3_twiddle_kernel<<<(n2 + 255) / 256, 256, 0, st>>>(n2, w.tw2);
  ms3_kernel_h_kernel<<<(q.N + 255) / 256 < 1184 ? (q.N + 255) / 256 : 1184, 256, 0, st>>>(n1, n2, op->k, op->d1,
                                                                                           op->d2, op->dz, w.hm1t);
  TP_CHECK_CUDA(cudaGetLastError());
  const FftPlan p1 = make_fft_plan(n1), p2 = make_fft_plan(n2);
  // compile-time plans (padded layout, fixed transforms per CTA) where the
  // other axis splits into whole CTAs, else the runtime plan
  const bool fix_r = fft_fixed_size(n2) && n1 % ms3_fixed_per_cta(n2) == 0;
  const bool fix_c = fft_fixed_size(n1) && n2 % ms3_fixed_per_cta(n1) == 0;
  const Ms3Rows rows = fix_r ? pick_rows(n2) : ms3_rows_of<0>();
  const Ms3Cols cols = fix_c ? pick_cols(n1) : ms3_cols_of<0>();
  const int srow = fix_r ? n2 + n2 / 8 + 1 : n2, scol = fix_c ? n1 + n1 / 8 + 1 : n1;
  const int rpc = fix_r ? ms3_fixed_per_cta(n2) : ms3_per_cta(n2, n1);
  const int cpc = fix_c ? ms3_fixed_per_cta(n1) : ms3_per_cta(n1, n2);
  const size_t smem_r = (size_t)(n2 + 2 * rpc * srow + rpc * n2) * sizeof(float2);
  const size_t smem_c = (size_t)(n1 + 2 * cpc * scol) * sizeof(float2);
  TP_CHECK_CUDA(cudaFuncSetAttribute(rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_r));
  TP_CHECK_CUDA(cudaFuncSetAttribute(cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_c));
  const dim3 gr(n1 / rpc, q.P), gc(n2 / cpc, q.P);
  if (!backward) {
    rows<<<gr, kMs3Threads, smem_r, st>>>(p2, q, kMs3FwdStart, 0, rpc);
    for (int z = 0; z < q.L; ++z) {
      cols<<<gc, kMs3Threads, smem_c, st>>>(p1, q, 0, cpc);
      rows<<<gr, kMs3Threads, smem_r, st>>>(p2, q, kMs3FwdStep, z, rpc);
    }
  } else {
    rows<<<gr, kMs3Threads, smem_r, st>>>(p2, q, kMs3BwdStart, q.L, rpc);
    for (int z = q.L - 1; z >= 0; --z) {
      cols<<<gc, kMs3Threads, smem_c, st>>>(p1, q, 1, cpc);
      rows<<<gr, kMs3Threads, smem_r, st>>>(p2, q, kMs3BwdStep, z, rpc);
    }
  }
  return check_cuda(cudaGetLastError(), "ms3d march launch");
}

static Ms3Params ms3_params(const tp_ms3d_op *op, int P) {
  Ms3Params q{};
  q.n1 = op->n1;
  q.n2 = op->n2;
  q.N = op->n1 * op->n2;
  q.nz = op->nz;
  q.L = op->nz - 1;
  q.P = P;
  return q;
}

}  // namespace tp

using namespace tp;

extern "C" size_t tp_ms3d_workspace_bytes(int32_t n1, int32_t n2, int32_t num_probes) {
  if (n1 < 1 || n2 < 1 || num_probes < 1) return 0;
  return ms3_layout(nullptr, n1, n2, num_probes).bytes;
}

extern "C" int tp_ms3d_transmission(const tp_ms3d_op *op, const void *n_field, int32_t n_dtype, void *trans,
                                    tp_stream_t stream) {
  int rc = ms3_check_op(op);
  if (rc) return rc;
  if (!n_field || !trans) return set_error(TP_ERR_INVALID, "n_field/trans is NULL");
  return ms_transmission_launch(op->n1 * op->n2, op->nz, op->k, op->dz, op->n_medium[0], op->n_medium[1], n_field,
                                n_dtype, static_cast<float2 *>(trans), reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tp_ms3d_march(const tp_ms3d_op *op, const void *trans, const void *probes, int32_t num_probes,
                             void *u_store, void *exit_out, void *workspace, size_t workspace_bytes,
                             tp_stream_t stream) {
  int rc = ms3_check_op(op);
  if (rc) return rc;
  if (!trans || !probes || num_probes < 1) return set_error(TP_ERR_INVALID, "bad 3D multislice march args");
  Ms3Params q = ms3_params(op, num_probes);
  q.trans = static_cast<const float2 *>(trans);
  q.probes = static_cast<const float2 *>(probes);
  q.u_store = static_cast<float2 *>(u_store);
  q.exit_out = static_cast<float2 *>(exit_out);
  return ms3_run(op, q, false, workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tp_ms3d_backward(const tp_ms3d_op *op, const void *trans, const void *u_fwd, const void *src_exit,
                                int32_t num_probes, void *grad_t, void *workspace, size_t workspace_bytes,
                                tp_stream_t stream) {
  int rc = ms3_check_op(op);
  if (rc) return rc;
  if (!trans || !u_fwd || !src_exit || !grad_t || num_probes < 1)
    return set_error(TP_ERR_INVALID, "bad 3D multislice backward args");
  Ms3Params q = ms3_params(op, num_probes);
  q.trans = static_cast<const float2 *>(trans);
  q.u_fwd = static_cast<const float2 *>(u_fwd);
  q.src_exit = static_cast<const float2 *>(src_exit);
  q.grad_t = static_cast<float2 *>(grad_t);
  return ms3_run(op, q, true, workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
}
