// 3D paraxial Crank–Nicolson march (2D transverse, 5-point operator), batched
// over probes, each slice solved by FFT-preconditioned BiCGStab.
//
// Replaces the reference's per-slice sparse LU of the 2D operator
// (iterative_lu.py:103-133 with operator_matrices.py:75-126) and its
// per-probe z-march (iterative_lu.py:138-197).
//
// Step s solves (I - P_s) u_new = (I + P_r) u + b, P = sigma*T(K + diag(c_s)),
// in delta form: (I - P_s) d = (P_r + P_s) u + b, u_new = u + d.  The update d
// is O(|P| |u|) ~ 4e-2 |u|, so the Krylov tolerance and the complex64
// round-off act on the small update, not on u (the same "1 + eps" reason as
// the 2D kernels).  BiCGStab (van der Vorst) runs on every probe of the batch
// at once: all vectors are (P, N) complex64 (complex128 in the check build),
// inner products are accumulated in fp64 per probe, and a probe stops
// updating once ||r|| <= tol ||rhs||; after the iterations each solve is
// judged by its true residual ||rhs - (I - P_s) d||.  Preconditioner: the
// periodic 5-point operator diagonalised by a 2D FFT, applied as
// IFFT2(FFT2(v) / (1 - sigma*T K_per(kf, kb))),
// K_per = mu_x (2 cos kf - 2) + mu_y (2 cos kb - 2), with register four-step
// transforms for square 64..256 grids and the shared-memory Stockham FFT of
// fft.cuh otherwise; optionally followed by the learned per-pixel correction.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>

#include <mutex>

#include "cnn_internal.cuh"
#include "fft.cuh"
#include "tp_common.cuh"
#include "tp_errors.h"
#include "tpcuda.h"

namespace tp {

constexpr int k3Threads = 256;

struct C3Params {
  int nf, nb, N, nz, L, P;
  int exact, is_delta, dtype, conj_t;
  double sigma, k, dz;
  double2 mu_x, mu_y;  // preconditioner symbol coefficients (sigma and T applied)
  const void *field;
  const cx *kc, *kw, *ke, *ks, *kn;  // diagonals of sigma*T(K)
};

// Per-probe BiCGStab scalars (fp64).
struct __align__(16) Krylov {
  double2 rho_prev, rho_cur, alpha, omega;
  double2 acc_r0v, acc_ts, acc_r0r;
  double acc_tt, acc_rr, bnorm2, res2;
  int done, iters, pad0, pad1;
};

// stats[0] total iterations, [1] solves, [2] solves whose true residual
// exceeded the tolerance, [3] largest iteration count of one solve.
enum { kStatIters = 0, kStatSolves = 1, kStatFailed = 2, kStatMaxIters = 3 };

// Step state of a march, kept on the device so that one launch sequence (or
// one CUDA graph with device-side loops) serves every step: t is the current
// step (1..L; 0 before the first), s its slice, it the BiCGStab iterations
// of this step, pending = 1 while a probe of the step is still iterating.
// Learned form: cheap = 1 when every solve of the previous step took one
// iteration (last_max, written by the step's statistics kernel); the first
// iteration of such a step applies the learned correction to the first of
// its two preconditioner applications only.  BiCGStab's recursions stay
// consistent with any pair of preconditioned vectors (x += alpha y + omega z,
// r = s - omega A z), and a solve converged in one iteration saves a filter
// pass; solves that need more iterations keep the correction in both.
struct __align__(16) C3State {
  int t, s, it, pending;
  int cheap, last_max, pad0, pad1;
};

// Start step t = state.t + 1.  In a graph, `outer` is the condition of the
// step loop (set to 0 at the last step, so the loop ends after L bodies) and
// `inner` that of the iteration loop (re-armed for the new step).
__global__ void c3_advance_kernel(C3State *st, int L, int backward, int use_cond, cudaGraphConditionalHandle outer,
                                  cudaGraphConditionalHandle inner) {
  const int t = st->t + 1;
  st->t = t;
  st->s = backward ? (L + 1 - t) : t;
  st->it = 0;
  st->pending = 1;
  st->cheap = (t > 1 && st->last_max <= 1) ? 1 : 0;
  if (use_cond) {
    cudaGraphSetConditional(outer, t < L ? 1u : 0u);
    cudaGraphSetConditional(inner, 1u);
  }
}

__device__ __forceinline__ double2 load_field(const C3Params &q, size_t idx) {
  if (q.dtype == TP_C128) return static_cast<const double2 *>(q.field)[idx];
  const cx v = static_cast<const cx *>(q.field)[idx];
  return z2(v.x, v.y);
}

// coef(n) of base_simulation_space.py:356-360
__device__ __forceinline__ double2 coef3(const C3Params &q, double2 v) {
  const double2 d = q.is_delta ? v : z2(v.x - 1.0, v.y);
  if (!q.exact) return z2(q.k * d.y, -q.k * d.x);
  const double2 w = zadd(zscale(d, 2.0), zmul(d, d));
  return z2(0.5 * q.k * w.y, -0.5 * q.k * w.x);
}

// sigma*T(K) diagonals from K's (T = conjugate transpose for the adjoints).
__global__ void c3_diag_kernel(int N, int nf, double sigma, int conj_t, const cx *kc, const cx *kw,
                               const cx *ke, const cx *ks, const cx *kn, cx *oc, cx *ow,
                               cx *oe, cx *os, cx *on) {
  const rx sg = (rx)sigma;
  auto tf = [&](cx v) { return mkcx(sg * v.x, sg * (conj_t ? -v.y : v.y)); };
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const cx z = mkcx(TP_R(0.0), TP_R(0.0));
    oc[i] = tf(kc[i]);
    if (!conj_t) {
      ow[i] = tf(kw[i]);
      oe[i] = tf(ke[i]);
      os[i] = tf(ks[i]);
      on[i] = tf(kn[i]);
    } else {
      ow[i] = (i >= 1) ? tf(ke[i - 1]) : z;
      oe[i] = (i + 1 < N) ? tf(kw[i + 1]) : z;
      os[i] = (i >= nf) ? tf(kn[i - nf]) : z;
      on[i] = (i + nf < N) ? tf(ks[i + nf]) : z;
    }
  }
}

// cd[i] = sigma*T(K)_c[i] + sigma*T(c_s(i)) for slice s (1-based), fp64 -> fp32,
// s = the current step's slice + next (next = 1: the slice after it, used by
// the exact adjoint from its second step on).
__global__ void c3_center_kernel(const C3Params q, const C3State *st, int next, cx *__restrict__ cd) {
  if (next && st->t == 1) return;
  const int s = st->s + next;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < q.N; i += gridDim.x * blockDim.x) {
    const size_t base = (size_t)i * q.nz;
    const double2 c = zscale(zadd(coef3(q, load_field(q, base + s - 1)), coef3(q, load_field(q, base + s))), 0.25 * q.dz);
    const double2 v = zscale(q.conj_t ? zconj(c) : c, q.sigma);
    const cx k = q.kc[i];
    cd[i] = mkcx((rx)(k.x + v.x), (rx)(k.y + v.y));
  }
}

// Object diagonals of slices s0+1 .. s0+count in the forward orientation,
// out[(s - s0 - 1) * N + i] = c_s(i) (sigma = 1, no transpose): the learned
// filters' inputs.  The adjoint modes apply the conjugate of the forward
// slice's filter (the transposed operator of a complex-symmetric K is its
// elementwise conjugate, so its corrected inverse is the conjugate one).
__global__ void c3_obj_diag_kernel(const C3Params q, int s0, int count, cx *__restrict__ out) {
  const size_t total = (size_t)count * q.N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int s = s0 + 1 + (int)(e / q.N), i = (int)(e % q.N);
    const size_t base = (size_t)i * q.nz;
    const double2 c = zscale(zadd(coef3(q, load_field(q, base + s - 1)), coef3(q, load_field(q, base + s))), 0.25 * q.dz);
    out[e] = to_cx(c);
  }
}

__device__ __forceinline__ cx apply_P(const C3Params &q, const cx *__restrict__ cd, const cx *__restrict__ x,
                                          int i) {
  cx r = cmul(cd[i], x[i]);
  const int f = i % q.nf;
  if (f > 0) r = cfma(q.kw[i], x[i - 1], r);
  if (f < q.nf - 1) r = cfma(q.ke[i], x[i + 1], r);
  if (i >= q.nf) r = cfma(q.ks[i], x[i - q.nf], r);
  if (i + q.nf < q.N) r = cfma(q.kn[i], x[i + q.nf], r);
  return r;
}

__device__ __forceinline__ void block_reduce_add(double v, double *dst, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) s += red[j];
    atomicAdd(dst, s);
  }
  __syncthreads();
}

// Sum M per-thread values over the CTA; thread m < M then calls fin(m, sum).
template <int M, class Fin>
__device__ __forceinline__ void block_reduce_many(double (&v)[M], double *red, Fin fin) {
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double x = v[m];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[m * nw + wp] = x;
  }
  __syncthreads();
  if (threadIdx.x < M) {
    double sum = 0.0;
    for (int j = 0; j < nw; ++j) sum += red[threadIdx.x * nw + j];
    fin(threadIdx.x, sum);
  }
}

// The stencil kernels below give each thread one element of kStencilProbes
// probes per loop trip: the operator's diagonals at the element are read once
// for all of them (they are shared by the probes), and every load of the trip
// precedes its stores, so the probes' loads are in flight together.  Grid
// (gx, ceil(P / kStencilProbes)), gx chosen so that the grid is one wave of
// resident CTAs (stencil_grid).
constexpr int kStencilProbes = 4;

// The off-diagonal couplings of element i (zero across an edge).
struct Stencil {
  cx w, e, s, n;
  int f;
};
__device__ __forceinline__ Stencil stencil_at(const C3Params &q, int i) {
  const cx z = mkcx(TP_R(0.0), TP_R(0.0));
  Stencil k;
  k.f = i % q.nf;
  k.w = k.f > 0 ? q.kw[i] : z;
  k.e = k.f < q.nf - 1 ? q.ke[i] : z;
  k.s = i >= q.nf ? q.ks[i] : z;
  k.n = i + q.nf < q.N ? q.kn[i] : z;
  return k;
}
// K_off x at element i (same operation order as apply_P).
__device__ __forceinline__ cx stencil_off(const C3Params &q, const Stencil &k, const cx *__restrict__ x, int i,
                                              cx acc) {
  if (k.f > 0) acc = cfma(k.w, x[i - 1], acc);
  if (k.f < q.nf - 1) acc = cfma(k.e, x[i + 1], acc);
  if (i >= q.nf) acc = cfma(k.s, x[i - q.nf], acc);
  if (i + q.nf < q.N) acc = cfma(k.n, x[i + q.nf], acc);
  return acc;
}

// Probes p0 .. p0 + kStencilProbes - 1 of this CTA that still iterate.
__device__ __forceinline__ unsigned pending_mask(const Krylov *K, int p0, int P) {
  unsigned m = 0;
#pragma unroll
  for (int j = 0; j < kStencilProbes; ++j)
    if (p0 + j < P && !K[p0 + j].done) m |= 1u << j;
  return m;
}

// r0 = rhs = (P_l + P_r) u + src and its norm; the first iteration reads r0
// as r and takes x = p = v = 0 without reading them.  The step t decides the
// terms: the exact adjoint's right-hand side uses the next slice's operator
// (cdr) and has no u term at t = 1 (lambda_{L+1} = 0); the per-probe source
// enters at t = 1; src_shared is (L, N) by step.
__global__ void __launch_bounds__(k3Threads) c3_init_kernel(const C3Params q, const C3State *st, int adj_exact,
                                                            const cx *__restrict__ cdl, const cx *__restrict__ cdn,
                                                            const cx *__restrict__ u, const cx *__restrict__ src_exit,
                                                            const cx *__restrict__ src_shared, cx *r0,
                                                            Krylov *K) {
  __shared__ double red[kStencilProbes * (k3Threads / 32)];
  const int p0 = blockIdx.y * kStencilProbes;
  const int np = q.P - p0 < kStencilProbes ? q.P - p0 : kStencilProbes;
  const int t = st->t;
  const int use_u = !(adj_exact && t == 1);
  const cx *cdr = (adj_exact && t > 1) ? cdn : cdl;
  const cx *src = (t == 1) ? src_exit : nullptr;
  const cx *shared = src_shared ? src_shared + (size_t)(t - 1) * q.N : nullptr;
  double acc[kStencilProbes] = {};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < q.N; i += gridDim.x * blockDim.x) {
    // (P_l + P_r) u = (cd_l + cd_r) u + 2 K_off u: the two operators differ only on the diagonal
    Stencil k{};
    cx dsum = mkcx(TP_R(0.0), TP_R(0.0));
    if (use_u) {
      k = stencil_at(q, i);
      dsum = cadd(cdl[i], cdr[i]);
    }
    const cx sh = shared != nullptr ? shared[i] : mkcx(TP_R(0.0), TP_R(0.0));
    cx bv[kStencilProbes];
#pragma unroll
    for (int j = 0; j < kStencilProbes; ++j) {
      if (j >= np) break;
      const size_t off = (size_t)(p0 + j) * q.N;
      cx b = mkcx(TP_R(0.0), TP_R(0.0));
      if (use_u) {
        const cx *uu = u + off;
        const cx o = stencil_off(q, k, uu, i, mkcx(TP_R(0.0), TP_R(0.0)));
        b = cfma(dsum, uu[i], cadd(o, o));
      }
      if (src != nullptr) b = cadd(b, src[off + i]);
      if (shared != nullptr) b = cadd(b, sh);
      bv[j] = b;
    }
#pragma unroll
    for (int j = 0; j < kStencilProbes; ++j) {
      if (j >= np) break;
      const cx b = bv[j];
      r0[(size_t)(p0 + j) * q.N + i] = b;
      acc[j] += (double)b.x * b.x + (double)b.y * b.y;
    }
  }
  block_reduce_many(acc, red, [&](int m, double v) {
    if (m < np) atomicAdd(&K[p0 + m].bnorm2, v);
  });
}

// Per probe: start a solve (rho = <r0, r0>, done when the right-hand side is zero).
__global__ void c3_start_kernel(Krylov *K, int P) {
  const int pr = blockIdx.x * blockDim.x + threadIdx.x;
  if (pr >= P) return;
  Krylov &k = K[pr];
  k.rho_prev = z2(1, 0);
  k.rho_cur = z2(k.bnorm2, 0.0);
  k.alpha = z2(1, 0);
  k.omega = z2(1, 0);
  k.iters = 0;
  k.done = (k.bnorm2 == 0.0) ? 1 : 0;
  k.acc_r0v = k.acc_ts = k.acc_r0r = z2(0, 0);
  k.acc_tt = 0.0;
  k.acc_rr = 0.0;
}

// Commit an iteration of every probe (one CTA loops over the probes), count
// it in the step state and record whether a probe is still iterating.  In a
// graph, `inner` (the iteration loop's condition) stays 1 only while a probe
// is pending and fewer than max_iter iterations ran, so the loop is bounded.
__global__ void c3_commit_kernel(Krylov *K, int P, double tol2, C3State *st, int max_iter, int use_cond,
                                 cudaGraphConditionalHandle inner) {
  int pend = 0;
  for (int pr = threadIdx.x; pr < P; pr += blockDim.x) {
    Krylov &k = K[pr];
    if (!k.done) {
      const double den = k.acc_r0v.x * k.acc_r0v.x + k.acc_r0v.y * k.acc_r0v.y;
      k.alpha = den > 0.0 ? zdiv(k.rho_cur, k.acc_r0v) : z2(0, 0);
      k.omega = (k.acc_tt > 0.0) ? zscale(k.acc_ts, 1.0 / k.acc_tt) : z2(0, 0);
      k.rho_prev = k.rho_cur;
      k.rho_cur = k.acc_r0r;
      k.iters += 1;
      const double om2 = k.omega.x * k.omega.x + k.omega.y * k.omega.y;
      const double rp2 = k.rho_prev.x * k.rho_prev.x + k.rho_prev.y * k.rho_prev.y;
      if (k.acc_rr <= tol2 * k.bnorm2 || om2 == 0.0 || rp2 == 0.0) k.done = 1;
    }
    pend |= !k.done;
    k.acc_r0v = k.acc_ts = k.acc_r0r = z2(0, 0);
    k.acc_tt = 0.0;
    k.acc_rr = 0.0;
  }
  pend = __syncthreads_or(pend);
  if (threadIdx.x == 0) {
    const int it = st->it + 1;
    st->it = it;
    st->pending = pend;
    if (use_cond) cudaGraphSetConditional(inner, (pend && it < max_iter) ? 1u : 0u);
  }
}

// Twiddle table W_n^t = exp(-2 pi i t / n) (fp64 sincospi, rounded once).
__global__ void c3_twiddle_kernel(int n, cx *tw) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double sv, cv;
    sincospi(-2.0 * (double)t / (double)n, &sv, &cv);
    tw[t] = mkcx((rx)cv, (rx)sv);
  }
}

// Inverse of the periodic symbol, scaled by 1/(nf nb) (the normalisation of
// the inverse 2D transform), transposed: sym[f * nb + b] =
// 1 / ((1 - mu_x (2 cos(2 pi f/nf) - 2) - mu_y (2 cos(2 pi b/nb) - 2)) nf nb).
__global__ void c3_symbol_kernel(const C3Params q, cx *sym) {
  const double sc = 1.0 / ((double)q.nf * (double)q.nb);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < q.N; e += gridDim.x * blockDim.x) {
    const int f = e / q.nb, bb = e - f * q.nb;
    double sf, cf, sb, cbv;
    sincospi(2.0 * (double)f / (double)q.nf, &sf, &cf);
    sincospi(2.0 * (double)bb / (double)q.nb, &sb, &cbv);
    const double ax = 2.0 * cf - 2.0, ay = 2.0 * cbv - 2.0;
    const double2 lam = z2(1.0 - (q.mu_x.x * ax + q.mu_y.x * ay), -(q.mu_x.y * ax + q.mu_y.y * ay));
    sym[e] = to_cx(zscale(zdiv(z2(1, 0), lam), sc));
  }
}

// Forward row FFTs of the preconditioner input, formed on the fly:
//   mode 0: p := r + beta (p - omega v)  (p updated in place), input p
//   mode 1: s := r - alpha v             (s written),          input s
//   mode 2: input r as is (K may be NULL: every probe is transformed)
// The first iteration of a step (st->it == 0) starts from x = p = v = 0 and
// r = r0, which the step head does not write: mode 0 takes p = r0 (and does
// not store it: the second iteration reads r0 as its p), mode 1 reads r0 as r.
// Grid (nb / rpc, P).
template <int NF>
__global__ void __launch_bounds__(k3Threads) c3_prec_rows_kernel(const FftPlan pl, const C3Params q, int mode,
                                                                 const cx *r, cx *p, const cx *v, cx *s,
                                                                 cx *hat, const Krylov *K, int rpc, int fft_on,
                                                                 const cx *twg, const cx *r0,
                                                                 const C3State *st) {
  extern __shared__ __align__(16) cx fsm[];
  const int n = NF > 0 ? NF : q.nf, pr = blockIdx.y;
  if (K != nullptr && K[pr].done) return;
  cx *tw = fsm, *a = tw + n, *b = a + rpc * fstride<NF>(n);
  const size_t off = (size_t)pr * q.N + (size_t)blockIdx.x * rpc * n;
  const int tot = rpc * n;
  auto slot = [&](int e) { return fslot<NF>(e / n, e % n, n); };
  if (fft_on) load_twiddles(tw, twg, n);
  if (mode == 2) {
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      if (fft_on) a[slot(e)] = r[off + e];
      else hat[off + e] = r[off + e];
    }
  } else if (mode == 0) {
    const int it = st->it;
    if (it == 0) {
      for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        const cx pv = r0[off + e];
        if (fft_on) a[slot(e)] = pv;
        else hat[off + e] = pv;
      }
    } else {
      const Krylov &k = K[pr];
      const double den = k.rho_prev.x * k.rho_prev.x + k.rho_prev.y * k.rho_prev.y;
      const double2 beta = den > 0.0 ? zmul(zdiv(k.rho_cur, k.rho_prev), zdiv(k.alpha, k.omega)) : z2(0, 0);
      const cx bt = to_cx(beta), om = to_cx(k.omega);
      const cx *pin = (it == 1) ? r0 : p;
      for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        const cx pv = cfma(bt, cfnma(om, v[off + e], pin[off + e]), r[off + e]);
        p[off + e] = pv;
        if (fft_on) a[slot(e)] = pv;
        else hat[off + e] = pv;
      }
    }
  } else {
    const Krylov &k = K[pr];
    const double den = k.acc_r0v.x * k.acc_r0v.x + k.acc_r0v.y * k.acc_r0v.y;
    const double2 alpha = den > 0.0 ? zdiv(k.rho_cur, k.acc_r0v) : z2(0, 0);
    const cx al = to_cx(alpha);
    const cx *rin = (st->it == 0) ? r0 : r;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      const cx sv = cfnma(al, v[off + e], rin[off + e]);
      s[off + e] = sv;
      if (fft_on) a[slot(e)] = sv;
      else hat[off + e] = sv;
    }
  }
  if (!fft_on) return;
  __syncthreads();
  const cx *res = fft_rows<NF>(a, b, pl, tw, false, rpc);
  for (int e = threadIdx.x; e < tot; e += blockDim.x) hat[off + e] = res[slot(e)];
}

// Column FFTs, multiplication by the (scaled) inverse symbol, inverse column
// FFTs (in place on hat).  Grid (nf / cpc, P): a CTA transposes cpc columns of
// length nb into smem.
template <int NB>
__global__ void __launch_bounds__(k3Threads) c3_prec_cols_kernel(const FftPlan pl, const C3Params q, cx *hat,
                                                                 const Krylov *K, int cpc, const cx *twg,
                                                                 const cx *__restrict__ sym) {
  extern __shared__ __align__(16) cx fsm[];
  const int nb = NB > 0 ? NB : q.nb, nf = q.nf, pr = blockIdx.y;
  if (K != nullptr && K[pr].done) return;
  cx *tw = fsm, *a = tw + nb, *b = a + cpc * fstride<NB>(nb);
  const int f0 = blockIdx.x * cpc;
  cx *base = hat + (size_t)pr * q.N;
  load_twiddles(tw, twg, nb);
  for (int e = threadIdx.x; e < cpc * nb; e += blockDim.x) {
    const int c = e % cpc, bb = e / cpc;  // coalesced over c; asynchronous copies
    cp_async_cx(&a[fslot<NB>(c, bb, nb)], &base[(size_t)bb * nf + f0 + c]);
  }
  cp_async_wait_all();
  __syncthreads();
  cx *F = fft_rows<NB>(a, b, pl, tw, false, cpc);
  cx *o = (F == a) ? b : a;
  const cx *sy = sym + (size_t)f0 * nb;
  for (int e = threadIdx.x; e < cpc * nb; e += blockDim.x) {
    const int c = e / nb, bb = e - c * nb;
    const int sl = fslot<NB>(c, bb, nb);
    F[sl] = cmul(F[sl], sy[e]);
  }
  __syncthreads();
  cx *R = fft_rows<NB>(F, o, pl, tw, true, cpc);
  for (int e = threadIdx.x; e < cpc * nb; e += blockDim.x) {
    const int c = e % cpc, bb = e / cpc;
    base[(size_t)bb * nf + f0 + c] = R[fslot<NB>(c, bb, nb)];
  }
}

// Inverse row FFTs of hat into out (the 1/(nf nb) scale is in the symbol);
// into out_first instead (when given) in the first iteration of a step whose
// state says cheap (the learned form's plain second application).
template <int NF>
__global__ void __launch_bounds__(k3Threads) c3_prec_rows_inv_kernel(const FftPlan pl, const C3Params q,
                                                                     const cx *hat, cx *out, const Krylov *K,
                                                                     int rpc, const cx *twg, cx *out_first,
                                                                     const C3State *st) {
  extern __shared__ __align__(16) cx fsm[];
  const int n = NF > 0 ? NF : q.nf, pr = blockIdx.y;
  if (K != nullptr && K[pr].done) return;
  cx *tw = fsm, *a = tw + n, *b = a + rpc * fstride<NF>(n);
  const size_t off = (size_t)pr * q.N + (size_t)blockIdx.x * rpc * n;
  const int tot = rpc * n;
  auto slot = [&](int e) { return fslot<NF>(e / n, e % n, n); };
  load_twiddles(tw, twg, n);
  for (int e = threadIdx.x; e < tot; e += blockDim.x) cp_async_cx(&a[slot(e)], &hat[off + e]);
  cp_async_wait_all();
  __syncthreads();
  const cx *res = fft_rows<NF>(a, b, pl, tw, true, rpc);
  cx *dst = (out_first != nullptr && st->it == 0 && st->cheap) ? out_first : out;
  for (int e = threadIdx.x; e < tot; e += blockDim.x) dst[off + e] = res[slot(e)];
}

// ab[f] = 2 cos(2 pi f / nf) - 2 (f < nf), ab[nf + b] = 2 cos(2 pi b / nb) - 2
// (fp64, rounded once): the factors of the periodic symbol.
__global__ void c3_symbol_factors_kernel(int nf, int nb, rx *ab) {
  for (int e = threadIdx.x; e < nf + nb; e += blockDim.x) {
    const int j = e < nf ? e : e - nf, n = e < nf ? nf : nb;
    ab[e] = (rx)(2.0 * cospi(2.0 * (double)j / (double)n) - 2.0);
  }
}

// Padded twiddle table of the four-step transforms of length n = R1 R2:
// tw[k1 * (R2 + 1) + n2] = W_n^{n2 k1} (fp64 sincospi, rounded once).
__global__ void c3_twiddle4_kernel(int n, int r1, int r2, cx *tw) {
  for (int e = threadIdx.x; e < r1 * (r2 + 1); e += blockDim.x) {
    const int k1 = e / (r2 + 1), n2 = e % (r2 + 1);
    double sv, cv;
    sincospi(-2.0 * (double)((n2 * k1) % n) / (double)n, &sv, &cv);
    tw[e] = n2 < r2 ? mkcx((rx)cv, (rx)sv) : mkcx(TP_R(0.0), TP_R(0.0));
  }
}

// The preconditioner input of mode 0 / 1 / 2 at element e of a probe's vector
// (see c3_prec_rows_kernel); loads only: the caller stores p (mode 0 after
// the first iteration) or s (mode 1) after all its loads, so that they are
// issued together rather than one memory latency per element.
struct PrecInput {
  int mode, first;
  cx bt, om, al;
  const cx *r, *pin, *v, *r0;
  cx *p, *s;
  __device__ __forceinline__ cx operator()(size_t e) const {
    if (mode == 2) return r[e];
    if (mode == 0) {
      if (first) return r0[e];
      return cfma(bt, cfnma(om, v[e], pin[e]), r[e]);
    }
    return cfnma(al, v[e], first ? r0[e] : r[e]);
  }
  // where the formed input is stored (nullptr: not stored)
  __device__ __forceinline__ cx *dest() const {
    if (mode == 0 && !first) return p;
    if (mode == 1) return s;
    return nullptr;
  }
};

__device__ __forceinline__ PrecInput prec_input(int mode, const cx *r, cx *p, const cx *v, cx *s,
                                                const cx *r0, const Krylov *K, int pr, const C3State *st) {
  PrecInput in{};
  in.mode = mode;
  in.r = r;
  in.p = p;
  in.v = v;
  in.s = s;
  in.r0 = r0;
  if (mode == 2) return in;
  const int it = st->it;
  in.first = it == 0;
  const Krylov &k = K[pr];
  if (mode == 0) {
    if (it > 0) {
      const double den = k.rho_prev.x * k.rho_prev.x + k.rho_prev.y * k.rho_prev.y;
      const double2 beta = den > 0.0 ? zmul(zdiv(k.rho_cur, k.rho_prev), zdiv(k.alpha, k.omega)) : z2(0, 0);
      in.bt = to_cx(beta);
      in.om = to_cx(k.omega);
      in.pin = (it == 1) ? r0 : p;
    }
  } else {
    const double den = k.acc_r0v.x * k.acc_r0v.x + k.acc_r0v.y * k.acc_r0v.y;
    in.al = to_cx(den > 0.0 ? zdiv(k.rho_cur, k.acc_r0v) : z2(0, 0));
  }
  return in;
}

// Four-step preconditioner kernels for nf = nb = R1 R2 (R1 >= R2): 256
// threads, 256 / R1 rows (or columns) per CTA, one short DFT per thread and
// stage, one shared-memory transpose per transform.
//
// Forward row transforms of the preconditioner input (formed as in
// c3_prec_rows_kernel) into hat, natural frequency order.  Grid (nb / RPC, P).
template <int R1, int R2>
__global__ void __launch_bounds__(256) c3_rows4_kernel(const C3Params q, int mode, const cx *r, cx *p,
                                                       const cx *v, cx *s, cx *hat, const Krylov *K,
                                                       const cx *__restrict__ twg, const cx *r0,
                                                       const C3State *st) {
  constexpr int N = R1 * R2, RPC = 256 / R1, S = R1 * (R2 + 1);
  __shared__ cx buf[RPC * S];
  __shared__ cx tw[R1 * (R2 + 1)];
  const int pr = blockIdx.y;
  if (K != nullptr && K[pr].done) return;
  for (int e = threadIdx.x; e < R1 * (R2 + 1); e += 256) tw[e] = twg[e];
  const PrecInput in = prec_input(mode, r, p, v, s, r0, K, pr, st);
  const size_t off = (size_t)pr * q.N + (size_t)blockIdx.x * RPC * N;
  __syncthreads();
  if (threadIdx.x < RPC * R2) {  // stage A: (row, n2)
    const int row = threadIdx.x / R2, n2 = threadIdx.x % R2;
    cx x[16];
    const size_t e0 = off + (size_t)row * N + n2;
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) x[n1] = in(e0 + R2 * n1);
    if (cx *dst = in.dest()) {
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) dst[e0 + R2 * n1] = x[n1];
    }
    dft_reg<R1>(x, -TP_R(1.0));
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1)
      buf[row * S + k1 * (R2 + 1) + n2] = k1 ? cmul(x[k1], tw[k1 * (R2 + 1) + n2]) : x[0];
  }
  __syncthreads();
  {  // stage C: (row, k1)
    const int row = threadIdx.x / R1, k1 = threadIdx.x % R1;
    cx x[16];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) x[n2] = buf[row * S + k1 * (R2 + 1) + n2];
    dft_reg<R2>(x, -TP_R(1.0));
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) hat[off + row * N + k1 + R1 * k2] = x[k2];
  }
}

// Column transforms of hat in place: forward, times the inverse symbol,
// inverse.  The symbol 1 / ((1 - mu_x a_f - mu_y a_b) nf nb) is formed on the
// fly from the real tables a_f = 2 cos(2 pi f / nf) - 2 (ab[f]) and a_b
// (ab[nf + b]), so no symbol array is read between the two transforms.
// Grid (nf / CPC, P).
template <int R1, int R2>
__global__ void __launch_bounds__(256, R1 * R2 == 256 ? 3 : 4) c3_cols4_kernel(const C3Params q, cx *hat, const Krylov *K,
                                                       const cx *__restrict__ twg,
                                                       const rx *__restrict__ ab) {
  constexpr int N = R1 * R2, CPC = 256 / R1;
  __shared__ cx buf[N * CPC];  // [k1][n2][c]
  __shared__ cx tw[R1 * (R2 + 1)];
  __shared__ rx bcos[N];
  const int pr = blockIdx.y;
  if (K != nullptr && K[pr].done) return;
  for (int e = threadIdx.x; e < R1 * (R2 + 1); e += 256) tw[e] = twg[e];
  const int nf = q.nf, f0 = blockIdx.x * CPC;
  for (int e = threadIdx.x; e < N; e += 256) bcos[e] = ab[nf + e];
  cx *base = hat + (size_t)pr * q.N + f0;
  __syncthreads();
  cx x[16];
  if (threadIdx.x < CPC * R2) {  // stage A: (c, n2), c fastest
    const int c = threadIdx.x % CPC, n2 = threadIdx.x / CPC;
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) x[n1] = base[(size_t)(R2 * n1 + n2) * nf + c];
    dft_reg<R1>(x, -TP_R(1.0));
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1)
      buf[(k1 * R2 + n2) * CPC + c] = k1 ? cmul(x[k1], tw[k1 * (R2 + 1) + n2]) : x[0];
  }
  __syncthreads();
  {  // stage C and its inverse: (c, k1)
    const int c = threadIdx.x % CPC, k1 = threadIdx.x / CPC;
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) x[n2] = buf[(k1 * R2 + n2) * CPC + c];
    dft_reg<R2>(x, -TP_R(1.0));
    {
      const rx sc = (rx)(1.0 / ((double)nf * (double)N));
      const rx af = ab[f0 + c];
      const rx ax = (rx)q.mu_x.x * af, ay = (rx)q.mu_x.y * af;
      const rx mx = (rx)q.mu_y.x, my = (rx)q.mu_y.y;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        const rx bb = bcos[k1 + R1 * k2];
        const rx dr = TP_R(1.0) - ax - mx * bb, di = -(ay + my * bb);
#ifdef TP_C128_CHECK
        const rx m = sc / (dr * dr + di * di);
#else
        const rx m = __fdividef(sc, dr * dr + di * di);  // a preconditioner value: the fast quotient
#endif
        x[k2] = cmul(x[k2], mkcx(dr * m, -di * m));
      }
    }
    dft_reg<R2>(x, TP_R(1.0));
    __syncthreads();  // every stage-C read is done before the buffer is rewritten
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2)
      buf[(k1 * R2 + n2) * CPC + c] = n2 ? cmulc(x[n2], tw[k1 * (R2 + 1) + n2]) : x[0];
  }
  __syncthreads();
  if (threadIdx.x < CPC * R2) {  // inverse stage A: (c, n2)
    const int c = threadIdx.x % CPC, n2 = threadIdx.x / CPC;
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) x[k1] = buf[(k1 * R2 + n2) * CPC + c];
    dft_reg<R1>(x, TP_R(1.0));
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) base[(size_t)(R2 * n1 + n2) * nf + c] = x[n1];
  }
}

// Inverse row transforms of hat into out (the 1/(nf nb) scale is in the
// symbol; out_first as in c3_prec_rows_inv_kernel).  Grid (nb / RPC, P).
template <int R1, int R2>
__global__ void __launch_bounds__(256) c3_rows4_inv_kernel(const C3Params q, const cx *hat, cx *out,
                                                           const Krylov *K, const cx *__restrict__ twg,
                                                           cx *out_first, const C3State *st) {
  constexpr int N = R1 * R2, RPC = 256 / R1, S = R1 * (R2 + 1);
  __shared__ cx buf[RPC * S];
  __shared__ cx tw[R1 * (R2 + 1)];
  const int pr = blockIdx.y;
  if (K != nullptr && K[pr].done) return;
  for (int e = threadIdx.x; e < R1 * (R2 + 1); e += 256) tw[e] = twg[e];
  const size_t off = (size_t)pr * q.N + (size_t)blockIdx.x * RPC * N;
  cx *dst = (out_first != nullptr && st->it == 0 && st->cheap) ? out_first : out;
  __syncthreads();
  {  // inverse stage C: (row, k1)
    const int row = threadIdx.x / R1, k1 = threadIdx.x % R1;
    cx x[16];
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) x[k2] = hat[off + row * N + k1 + R1 * k2];
    dft_reg<R2>(x, TP_R(1.0));
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2)
      buf[row * S + k1 * (R2 + 1) + n2] = n2 ? cmulc(x[n2], tw[k1 * (R2 + 1) + n2]) : x[0];
  }
  __syncthreads();
  if (threadIdx.x < RPC * R2) {  // inverse stage A: (row, n2)
    const int row = threadIdx.x / R2, n2 = threadIdx.x % R2;
    cx x[16];
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) x[k1] = buf[row * S + k1 * (R2 + 1) + n2];
    dft_reg<R1>(x, TP_R(1.0));
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) dst[off + row * N + R2 * n1 + n2] = x[n1];
  }
}

// out = (I - P) y with fused fp64 dots: WHICH 0: acc_r0v += <r0, out>;
// WHICH 1: acc_ts += <out, s>, acc_tt += <out, out>.
template <int WHICH>
__global__ void __launch_bounds__(k3Threads, WHICH == 0 ? 4 : 3) c3_matvec_kernel(const C3Params q, const cx *__restrict__ cd,
                                                              const cx *__restrict__ y, cx *__restrict__ out,
                                                              const cx *__restrict__ r0, const cx *__restrict__ s,
                                                              Krylov *K) {
  constexpr int A = WHICH == 0 ? 2 : 3;  // sums per probe
  __shared__ double red[A * kStencilProbes * (k3Threads / 32)];
  const int p0 = blockIdx.y * kStencilProbes;
  const unsigned pend = pending_mask(K, p0, q.P);
  if (pend == 0) return;
  const cx *c_in = WHICH == 0 ? r0 : s;
  double acc[A * kStencilProbes] = {};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < q.N; i += gridDim.x * blockDim.x) {
    const Stencil k = stencil_at(q, i);
    const cx dc = cd[i];
    cx tv[kStencilProbes], cv[kStencilProbes];
#pragma unroll
    for (int j = 0; j < kStencilProbes; ++j) {
      if (!(pend & (1u << j))) continue;
      const size_t off = (size_t)(p0 + j) * q.N;
      const cx *yy = y + off;
      const cx yi = yy[i];
      tv[j] = csub(yi, stencil_off(q, k, yy, i, cmul(dc, yi)));
      cv[j] = c_in[off + i];
    }
#pragma unroll
    for (int j = 0; j < kStencilProbes; ++j) {
      if (!(pend & (1u << j))) continue;
      const cx t = tv[j], c = cv[j];
      out[(size_t)(p0 + j) * q.N + i] = t;
      if (WHICH == 0) {  // conj(r0) t
        acc[A * j] += (double)c.x * t.x + (double)c.y * t.y;
        acc[A * j + 1] += (double)c.x * t.y - (double)c.y * t.x;
      } else {  // conj(t) s, |t|^2
        acc[A * j] += (double)t.x * c.x + (double)t.y * c.y;
        acc[A * j + 1] += (double)t.x * c.y - (double)t.y * c.x;
        acc[A * j + 2] += (double)t.x * t.x + (double)t.y * t.y;
      }
    }
  }
  block_reduce_many(acc, red, [&](int m, double v) {
    const int j = m / A, c = m % A;
    if (!(pend & (1u << j))) return;
    Krylov &kr = K[p0 + j];
    double *dst = WHICH == 0 ? (c == 0 ? &kr.acc_r0v.x : &kr.acc_r0v.y)
                             : (c == 0 ? &kr.acc_ts.x : (c == 1 ? &kr.acc_ts.y : &kr.acc_tt));
    atomicAdd(dst, v);
  });
}

// omega = <t,s>/<t,t>; x += alpha y + omega z (x = 0 before the first
// iteration of a step: not read then); r = s - omega t; accumulate <r0, r>
// and ||r||^2 for the next iteration.
__global__ void __launch_bounds__(k3Threads) c3_update_kernel(const C3Params q, cx *x, cx *r,
                                                              const cx *__restrict__ r0, const cx *__restrict__ y,
                                                              const cx *__restrict__ z, const cx *__restrict__ s,
                                                              const cx *__restrict__ t, Krylov *K,
                                                              const C3State *st) {
  __shared__ double red[3 * (k3Threads / 32)];
  const int pr = blockIdx.y;
  Krylov &k = K[pr];
  if (k.done) return;
  const size_t off = (size_t)pr * q.N;
  const double den = k.acc_r0v.x * k.acc_r0v.x + k.acc_r0v.y * k.acc_r0v.y;
  const double2 alpha = den > 0.0 ? zdiv(k.rho_cur, k.acc_r0v) : z2(0, 0);
  const double2 omega = (k.acc_tt > 0.0) ? zscale(k.acc_ts, 1.0 / k.acc_tt) : z2(0, 0);
  const cx al = to_cx(alpha), om = to_cx(omega);
  const bool first = st->it == 0;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < q.N; i += gridDim.x * blockDim.x) {
    const cx x0 = first ? mkcx(TP_R(0.0), TP_R(0.0)) : x[off + i];
    x[off + i] = cfma(om, z[off + i], cfma(al, y[off + i], x0));
    const cx rv = cfnma(om, t[off + i], s[off + i]);
    r[off + i] = rv;
    const cx c = r0[off + i];
    a0 += (double)c.x * rv.x + (double)c.y * rv.y;
    a1 += (double)c.x * rv.y - (double)c.y * rv.x;
    a2 += (double)rv.x * rv.x + (double)rv.y * rv.y;
  }
  double acc[3] = {a0, a1, a2};
  block_reduce_many(acc, red, [&](int m, double v) { atomicAdd(m == 0 ? &k.acc_r0r.x : (m == 1 ? &k.acc_r0r.y : &k.acc_rr), v); });
}

// True residual of each solve: res2 = ||rhs - (I - P) d||^2 (rhs = r0, d = x),
// then u += d, stored into node `to` of u_store (to = t, or L - t for the
// flipped reference adjoint) and, at the last step, into exit_out.
__global__ void __launch_bounds__(k3Threads, 4) c3_finish_kernel(const C3Params q, const C3State *st,
                                                              const cx *__restrict__ cd,
                                                              const cx *__restrict__ x, const cx *__restrict__ r0,
                                                              cx *u, Krylov *K, cx *u_store, int flip,
                                                              cx *exit_out) {
  __shared__ double red[kStencilProbes * (k3Threads / 32)];
  const int p0 = blockIdx.y * kStencilProbes;
  const int np = q.P - p0 < kStencilProbes ? q.P - p0 : kStencilProbes;
  const int t = st->t;
  const size_t node = flip ? q.L - t : t;
  // a probe whose right-hand side was zero did not iterate: its update is 0
  // (x then holds an earlier step's values)
  unsigned iterated = 0;
#pragma unroll
  for (int j = 0; j < kStencilProbes; ++j)
    if (j < np && K[p0 + j].iters > 0) iterated |= 1u << j;
  double acc[kStencilProbes] = {};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < q.N; i += gridDim.x * blockDim.x) {
    Stencil k{};
    cx dc = mkcx(TP_R(0.0), TP_R(0.0));
    if (iterated) {
      k = stencil_at(q, i);
      dc = cd[i];
    }
    cx unv[kStencilProbes];
#pragma unroll
    for (int j = 0; j < kStencilProbes; ++j) {
      if (j >= np) break;
      const size_t off = (size_t)(p0 + j) * q.N;
      const bool it = iterated & (1u << j);
      const cx xi = it ? x[off + i] : mkcx(TP_R(0.0), TP_R(0.0));
      const cx mx = it ? csub(xi, stencil_off(q, k, x + off, i, cmul(dc, xi))) : xi;
      const cx d = csub(r0[off + i], mx);
      acc[j] += (double)d.x * d.x + (double)d.y * d.y;
      unv[j] = cadd(u[off + i], xi);
    }
#pragma unroll
    for (int j = 0; j < kStencilProbes; ++j) {
      if (j >= np) break;
      const int pr = p0 + j;
      const size_t off = (size_t)pr * q.N;
      u[off + i] = unv[j];
      if (u_store) u_store[((size_t)pr * q.nz + node) * q.N + i] = unv[j];
      if (exit_out && t == q.L) exit_out[off + i] = unv[j];
    }
  }
  block_reduce_many(acc, red, [&](int m, double v) {
    if (m < np) atomicAdd(&K[p0 + m].res2, v);
  });
}

#ifndef TP_C128_CHECK
// ------------------------------------------------ TMA-tiled stencil kernels
// The right-hand side, both matvecs and the finish with their inputs staged
// by the tensor-memory accelerator: a CTA owns probe group blockIdx.y
// (kStencilProbes probes) and the row blocks blockIdx.x, blockIdx.x +
// gridDim.x, ... of kTmaRows image rows.  For each row block one thread
// issues three tiled tensor loads into a shared-memory stage -- the stencil
// input of the group's probes with a one-row halo (rows outside the image
// read as zero), the slice's diagonal(s) and its four off-diagonals -- and
// the stages are double-buffered, so the next block's copies are in flight
// while this one is computed from shared memory (the kernels that read
// their inputs from global memory wait one memory latency per loop trip).
// The vectors of the workspace block and the slice diagonals are equally
// spaced, so three tensor maps serve every kernel (the vector or diagonal is
// the outer coordinate).  The arithmetic is that of c3_init_kernel,
// c3_matvec_kernel and c3_finish_kernel, element by element; waits on the
// stages are bounded (kDevMbarTimeout) and a CTA that gives up waits for its
// copies in flight before it returns.
constexpr int kTmaRows = 2;
enum { kTmaInit = 0, kTmaMatvec0 = 1, kTmaMatvec1 = 2, kTmaFinish = 3 };
// workspace vector and diagonal indices (c3_layout order)
enum { kVecU = 0, kVecX = 1, kVecR0 = 3, kVecV = 5, kVecS = 6, kVecY = 7, kVecZ = 8, kVecT = 9, kNumVecs = 11 };
enum { kDiagCdl = 0, kDiagCdr = 1, kDiagW = 3, kNumDiags = 8 };

struct TmaArgs {
  int vin;       // the staged stencil input (with its halo rows)
  int vc0, vc1;  // the other staged vectors (tile rows only): matvec r0 or s; finish r0 and u
  cx *out;       // init: r0; matvec: v or t; finish: u
  const cx *src_exit, *src_shared;
  cx *u_store, *exit_out;
  int adj_exact, flip;
};

// vectors staged without halo: 0 (init), 1 (matvec), 2 (finish)
template <int KIND>
__host__ __device__ constexpr int tma_plain_vecs() {
  return KIND == kTmaInit ? 0 : (KIND == kTmaFinish ? 2 : 1);
}
template <int KIND, int NF>
__host__ __device__ constexpr uint32_t tma_stage_bytes() {
  return (uint32_t)((kStencilProbes * (kTmaRows + 2 + tma_plain_vecs<KIND>() * kTmaRows) +
                     (KIND == kTmaInit ? 6 : 5) * kTmaRows) *
                    NF * sizeof(cx));
}

template <int KIND, int NF>
__global__ void __launch_bounds__(k3Threads, 1) c3_tma_kernel(const __grid_constant__ CUtensorMap mh,
                                                              const __grid_constant__ CUtensorMap mv,
                                                              const __grid_constant__ CUtensorMap md,
                                                              const __grid_constant__ CUtensorMap md4, const C3Params q,
                                                              const C3State *st, const TmaArgs a, Krylov *K, int *err) {
  constexpr int TR = kTmaRows, H = TR + 2, SP = kStencilProbes, TE = TR * NF;
  constexpr int NV = tma_plain_vecs<KIND>();
  constexpr int ND = KIND == kTmaInit ? 2 : 1;  // diagonals staged before the off-diagonals
  constexpr uint32_t HB = SP * H * NF * sizeof(cx), VB = SP * TE * sizeof(cx), DB = TE * sizeof(cx);
  constexpr uint32_t STAGE = tma_stage_bytes<KIND, NF>();
  static_assert(STAGE == HB + NV * VB + (ND + 4) * DB, "stage layout");
  constexpr int A = KIND == kTmaMatvec1 ? 3 : (KIND == kTmaMatvec0 ? 2 : 1);  // sums per probe
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double red[A * SP * (k3Threads / 32)];
  __shared__ __align__(8) uint64_t bar[2];
  const int p0 = blockIdx.y * SP;
  const int np = q.P - p0 < SP ? q.P - p0 : SP;
  const int t = st->t;
  unsigned act = 0, iterated = 0;
#pragma unroll
  for (int j = 0; j < SP; ++j) {
    if (j >= np) continue;
    if (KIND == kTmaMatvec0 || KIND == kTmaMatvec1) {
      if (!K[p0 + j].done) act |= 1u << j;
    } else {
      act |= 1u << j;
      if (KIND == kTmaFinish && K[p0 + j].iters > 0) iterated |= 1u << j;
    }
  }
  if (act == 0) return;
  const int nblk = q.nb / TR;
  const int nmine = blockIdx.x < nblk ? (nblk - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // init: the right-hand side's terms (see c3_init_kernel)
  const int use_u = KIND == kTmaInit ? !(a.adj_exact && t == 1) : 1;
  const int dsec = (a.adj_exact && t > 1) ? kDiagCdr : kDiagCdl;
  const cx *src = (KIND == kTmaInit && t == 1) ? a.src_exit : nullptr;
  const cx *shared = (KIND == kTmaInit && a.src_shared) ? a.src_shared + (size_t)(t - 1) * q.N : nullptr;
  const size_t node = a.flip ? q.L - t : t;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int k) {  // thread 0: the stage of my k-th row block
    const int buf = k & 1, rb = blockIdx.x + k * gridDim.x;
    unsigned char *sb = smem + buf * STAGE;
    mbar_arrive_expect_tx(&bar[buf], STAGE);
    tma_load_4d(sb, &mh, 0, rb * TR - 1, p0, a.vin, &bar[buf]);
    if (NV > 0) tma_load_4d(sb + HB, &mv, 0, rb * TR, p0, a.vc0, &bar[buf]);
    if (NV > 1) tma_load_4d(sb + HB + VB, &mv, 0, rb * TR, p0, a.vc1, &bar[buf]);
    tma_load_3d(sb + HB + NV * VB, &md, 0, rb * TR, kDiagCdl, &bar[buf]);
    if (KIND == kTmaInit) tma_load_3d(sb + HB + NV * VB + DB, &md, 0, rb * TR, dsec, &bar[buf]);
    tma_load_3d(sb + HB + NV * VB + ND * DB, &md4, 0, rb * TR, kDiagW, &bar[buf]);
  };
  if (threadIdx.x == 0) {
    if (nmine > 0) issue(0);
    if (nmine > 1) issue(1);
  }
  double acc[A * SP] = {};
  const cx zero = czero();
  for (int k = 0; k < nmine; ++k) {
    const int buf = k & 1;
    const bool got = mbar_wait_bounded(&bar[buf], (uint32_t)((k >> 1) & 1), err);
    if (__syncthreads_or(!got)) {
      // give up: the copies in flight (this stage's, and the next one's if
      // issued) land in shared memory before the CTA exits
      if (threadIdx.x == 0) {
        mbar_wait_bounded(&bar[buf], (uint32_t)((k >> 1) & 1), nullptr);
        if (k + 1 < nmine) mbar_wait_bounded(&bar[buf ^ 1], (uint32_t)(((k + 1) >> 1) & 1), nullptr);
      }
      __syncthreads();
      return;
    }
    const unsigned char *sb = smem + buf * STAGE;
    const cx *tl = reinterpret_cast<const cx *>(sb);                        // [SP][H][NF]
    const cx *v0 = reinterpret_cast<const cx *>(sb + HB);                   // [SP][TR][NF]
    const cx *v1 = reinterpret_cast<const cx *>(sb + HB + VB);              // [SP][TR][NF]
    const cx *d1 = reinterpret_cast<const cx *>(sb + HB + NV * VB);         // [TR][NF]
    const cx *d2 = reinterpret_cast<const cx *>(sb + HB + NV * VB + DB);    // init: second diagonal
    const cx *dof = reinterpret_cast<const cx *>(sb + HB + NV * VB + ND * DB);  // [4][TR][NF]: w, e, s, n
    const int rb = blockIdx.x + k * gridDim.x;
#pragma unroll
    for (int e = threadIdx.x; e < TE; e += k3Threads) {
      const int row = e / NF, f = e - row * NF;
      const int i = (rb * TR + row) * NF + f;
      const cx kw = f > 0 ? dof[e] : zero, ke = f < NF - 1 ? dof[TE + e] : zero;
      const cx ks = i >= NF ? dof[2 * TE + e] : zero, kn = i + NF < q.N ? dof[3 * TE + e] : zero;
      const cx dc = d1[e];
      // K_off x at the element from the staged rows of probe j (the order of stencil_off)
      auto off = [&](const cx *xt, cx acc0) {
        const int c0 = (row + 1) * NF + f;
        if (f > 0) acc0 = cfma(kw, xt[c0 - 1], acc0);
        if (f < NF - 1) acc0 = cfma(ke, xt[c0 + 1], acc0);
        if (i >= NF) acc0 = cfma(ks, xt[c0 - NF], acc0);
        if (i + NF < q.N) acc0 = cfma(kn, xt[c0 + NF], acc0);
        return acc0;
      };
      if (KIND == kTmaInit) {
        const cx dsum = cadd(dc, d2[e]);
        const cx sh = shared != nullptr ? shared[i] : zero;
        cx bv[SP];
#pragma unroll
        for (int j = 0; j < SP; ++j) {
          if (!((act >> j) & 1u)) continue;
          const size_t offp = (size_t)(p0 + j) * q.N;
          cx b = zero;
          if (use_u) {
            const cx *xt = tl + j * H * NF;
            const cx o = off(xt, zero);
            b = cfma(dsum, xt[(row + 1) * NF + f], cadd(o, o));
          }
          if (src != nullptr) b = cadd(b, src[offp + i]);
          if (shared != nullptr) b = cadd(b, sh);
          bv[j] = b;
        }
#pragma unroll
        for (int j = 0; j < SP; ++j) {
          if (!((act >> j) & 1u)) continue;
          const cx b = bv[j];
          a.out[(size_t)(p0 + j) * q.N + i] = b;
          acc[j] += (double)b.x * b.x + (double)b.y * b.y;
        }
      } else if (KIND == kTmaMatvec0 || KIND == kTmaMatvec1) {
        cx tv[SP], cv[SP];
#pragma unroll
        for (int j = 0; j < SP; ++j) {
          if (!((act >> j) & 1u)) continue;
          const cx *xt = tl + j * H * NF;
          const cx yi = xt[(row + 1) * NF + f];
          tv[j] = csub(yi, off(xt, cmul(dc, yi)));
          cv[j] = v0[j * TE + e];
        }
#pragma unroll
        for (int j = 0; j < SP; ++j) {
          if (!((act >> j) & 1u)) continue;
          const cx tt = tv[j], c = cv[j];
          a.out[(size_t)(p0 + j) * q.N + i] = tt;
          if (KIND == kTmaMatvec0) {  // conj(r0) t
            acc[A * j] += (double)c.x * tt.x + (double)c.y * tt.y;
            acc[A * j + 1] += (double)c.x * tt.y - (double)c.y * tt.x;
          } else {  // conj(t) s, |t|^2
            acc[A * j] += (double)tt.x * c.x + (double)tt.y * c.y;
            acc[A * j + 1] += (double)tt.x * c.y - (double)tt.y * c.x;
            acc[A * j + 2] += (double)tt.x * tt.x + (double)tt.y * tt.y;
          }
        }
      } else {  // finish
        cx unv[SP];
#pragma unroll
        for (int j = 0; j < SP; ++j) {
          if (!((act >> j) & 1u)) continue;
          const bool itd = (iterated >> j) & 1u;
          const cx *xt = tl + j * H * NF;
          const cx xi = itd ? xt[(row + 1) * NF + f] : zero;
          const cx mx = itd ? csub(xi, off(xt, cmul(dc, xi))) : xi;
          const cx d = csub(v0[j * TE + e], mx);
          acc[j] += (double)d.x * d.x + (double)d.y * d.y;
          unv[j] = cadd(v1[j * TE + e], xi);
        }
#pragma unroll
        for (int j = 0; j < SP; ++j) {
          if (!((act >> j) & 1u)) continue;
          const int pr = p0 + j;
          const size_t offp = (size_t)pr * q.N;
          a.out[offp + i] = unv[j];
          if (a.u_store) a.u_store[((size_t)pr * q.nz + node) * q.N + i] = unv[j];
          if (a.exit_out && t == q.L) a.exit_out[offp + i] = unv[j];
        }
      }
    }
    __syncthreads();  // every thread is done with this stage
    if (threadIdx.x == 0 && k + 2 < nmine) {
      fence_proxy_async_smem();
      issue(k + 2);
    }
  }
  block_reduce_many(acc, red, [&](int m, double v) {
    const int j = m / A, c = m % A;
    if (!((act >> j) & 1u)) return;
    Krylov &kr = K[p0 + j];
    double *dst;
    if (KIND == kTmaInit) dst = &kr.bnorm2;
    else if (KIND == kTmaFinish) dst = &kr.res2;
    else if (KIND == kTmaMatvec0) dst = c == 0 ? &kr.acc_r0v.x : &kr.acc_r0v.y;
    else dst = c == 0 ? &kr.acc_ts.x : (c == 1 ? &kr.acc_ts.y : &kr.acc_tt);
    atomicAdd(dst, v);
  });
}
#endif  // TP_C128_CHECK

// After a step (one CTA loops over the probes): accumulate the statistics
// (when `stats` is given) and clear the per-probe sums of the next step.
__global__ void c3_stats_kernel(Krylov *K, int P, double tol2, int *stats, C3State *st) {
  __shared__ int mx;
  if (threadIdx.x == 0) mx = 0;
  __syncthreads();
  for (int pr = threadIdx.x; pr < P; pr += blockDim.x) {
    Krylov &k = K[pr];
    atomicMax(&mx, k.iters);
    if (stats != nullptr) {
      atomicAdd(&stats[kStatIters], k.iters);
      atomicAdd(&stats[kStatSolves], 1);
      atomicMax(&stats[kStatMaxIters], k.iters);
      // the true residual may exceed the recursive one by round-off; allow 10x
      if (k.res2 > 100.0 * tol2 * k.bnorm2) atomicAdd(&stats[kStatFailed], 1);
    }
    k.res2 = 0.0;
    k.bnorm2 = 0.0;
  }
  __syncthreads();
  if (threadIdx.x == 0) st->last_max = mx;
}

// Store the state (P, N) into slice `t` of u_store (P, nz, N) and/or exit.
__global__ void c3_store_kernel(int N, int P, int nz, int t, const cx *__restrict__ u, cx *u_store,
                                cx *exit_out) {
  const size_t total = (size_t)P * N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t pr = e / N, i = e % N;
    if (u_store) u_store[(pr * nz + t) * N + i] = u[e];
    if (exit_out) exit_out[e] = u[e];
  }
}

// grad_c[s-1][i] += sum_p lambda_p[i] conj(u_p,s[i] + u_p,s-1[i]) for the
// current step's slice s (no atomics: one thread owns element i and loops
// over the probes).
__global__ void c3_grad_kernel(int N, int P, int nz, const C3State *st, const cx *__restrict__ lam,
                               const cx *__restrict__ u_fwd, cx *grad_c) {
  constexpr int G = 8;  // probes whose loads are issued together
  const int s = st->s;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    cx acc = mkcx(TP_R(0.0), TP_R(0.0));
    for (int p0 = 0; p0 < P; p0 += G) {
      cx a[G], b[G], l[G];
#pragma unroll
      for (int j = 0; j < G; ++j) {
        if (p0 + j < P) {
          const size_t pr = p0 + j;
          a[j] = u_fwd[(pr * nz + s) * N + i];
          b[j] = u_fwd[(pr * nz + s - 1) * N + i];
          l[j] = lam[pr * N + i];
        }
      }
#pragma unroll
      for (int j = 0; j < G; ++j)
        if (p0 + j < P) acc = cadd(acc, cmulc(l[j], cadd(a[j], b[j])));
    }
    cx g = grad_c[(size_t)(s - 1) * N + i];
    grad_c[(size_t)(s - 1) * N + i] = cadd(g, acc);
  }
}

#ifndef TP_C128_CHECK  // the learned preconditioner is not part of the complex128 check build
// Learned correction of the preconditioned vector: out = z + sum_t F_t z(x + o_t)
// with the filter of the current step's slice s (conj(F) in the adjoint
// modes).  The filters of all slices are computed before the march, in
// chunks of `chunk` slices: slice s uses image (s-1) % chunk of chunk
// (s-1) / chunk, tap-major within the chunk (13, chunk * N).
//
// A CTA owns a block of cw <= 256 columns and rb = 2 * (256 / cw) rows for
// kFilterProbes probes; thread (pair, column) filters the two vertically
// adjacent pixels (b0 + 2 pair, f) and (b0 + 2 pair + 1, f) and keeps their
// 2 x 13 taps in registers (read once for all the CTA's probes).  The rows of
// every pending probe, with a 2-pixel border, are copied into shared memory
// in one wave of cp.async copies, positions outside the image set to zero, so
// each tap reads a fixed offset and the taps reaching outside the image add
// zero.  The two pixels' 26 taps read 18 distinct neighbours.
// Grid (ceil(nf / cw), ceil(nb / rb), ceil(P / kFilterProbes)).
constexpr int kFilterProbes = 8;

__host__ __device__ constexpr int filter_cw(int nf) { return nf < 256 ? nf : 256; }
__host__ __device__ constexpr int filter_rb(int nf) { return 2 * (256 / filter_cw(nf)); }

__global__ void __launch_bounds__(k3Threads, 2) c3_filter_kernel(const C3Params q, const C3State *st, int chunk,
                                                                 const cx *__restrict__ Fall,
                                                                 const cx *__restrict__ z, cx *__restrict__ out,
                                                                 const Krylov *K, int second) {
  extern __shared__ __align__(16) cx ztile[];  // [kFilterProbes][rb + 4][cw + 4]
  // the second application of a cheap first iteration stays plain (C3State)
  if (second && st->it == 0 && st->cheap) return;
  const int nf = q.nf, nb = q.nb;
  const int cw = filter_cw(nf), rb = filter_rb(nf), W = cw + 4, H = rb + 4;
  const int c0 = blockIdx.x * cw, b0 = blockIdx.y * rb, p0 = blockIdx.z * kFilterProbes;
  const int np_cta = q.P - p0 < kFilterProbes ? q.P - p0 : kFilterProbes;
  unsigned pend = 0;
  for (int j = 0; j < np_cta; ++j)
    if (K == nullptr || !K[p0 + j].done) pend |= 1u << j;
  // tile row y holds image row b0 - 2 + y, columns c0 - 2 .. c0 + cw + 1 (zero outside the image)
  const cx zero = mkcx(TP_R(0.0), TP_R(0.0));
  const bool pairs16 = ((nf | cw) & 1) == 0;  // 16-byte copies of column pairs
  for (int j = 0; j < np_cta; ++j) {
    if (!((pend >> j) & 1u)) continue;
    const cx *src = z + (size_t)(p0 + j) * q.N;
    for (int y = 0; y < H; ++y) {
      const int b = b0 - 2 + y;
      cx *dst = ztile + (j * H + y) * W;
      if (b < 0 || b >= nb) {
        for (int x = threadIdx.x; x < W; x += blockDim.x) dst[x] = zero;
        continue;
      }
      const cx *srow = src + (size_t)b * nf;
      if (pairs16) {
        for (int m = 2 * threadIdx.x; m < cw; m += 2 * blockDim.x) {
          if (c0 + m < nf) {
            cp_async16(&dst[2 + m], &srow[c0 + m]);
          } else {
            dst[2 + m] = zero;
            dst[3 + m] = zero;
          }
        }
      } else {
        for (int m = threadIdx.x; m < cw; m += blockDim.x) {
          if (c0 + m < nf) cp_async_cx(&dst[2 + m], &srow[c0 + m]);
          else dst[2 + m] = zero;
        }
      }
      if (threadIdx.x < 4) {  // border columns x = 0, 1, cw + 2, cw + 3
        const int x = threadIdx.x < 2 ? threadIdx.x : cw + threadIdx.x;
        const int f = c0 - 2 + x;
        if (f >= 0 && f < nf) cp_async_cx(&dst[x], &srow[f]);
        else dst[x] = zero;
      }
    }
  }
  // the taps of the thread's two pixels while the copies are in flight
  const int pr = threadIdx.x / cw, fx = threadIdx.x - pr * cw;
  const int f = c0 + fx, ba = b0 + 2 * pr;
  const bool act = pr < rb / 2 && f < nf;
  const bool va = act && ba < nb, vb = act && ba + 1 < nb;
  const int sl = st->s - 1;
  const size_t np = (size_t)chunk * q.N;
  const cx *F = Fall + (size_t)(sl / chunk) * kFilterTaps * np + (size_t)(sl % chunk) * q.N;
  const rx cs = q.conj_t ? -TP_R(1.0) : TP_R(1.0);
  cx wa[kFilterTaps], wb[kFilterTaps];
#pragma unroll
  for (int t = 0; t < kFilterTaps; ++t) {
    const cx a = va ? F[(size_t)t * np + (size_t)ba * nf + f] : mkcx(TP_R(0.0), TP_R(0.0));
    const cx b = vb ? F[(size_t)t * np + (size_t)(ba + 1) * nf + f] : mkcx(TP_R(0.0), TP_R(0.0));
    wa[t] = mkcx(a.x, cs * a.y);
    wb[t] = mkcx(b.x, cs * b.y);
  }
  cp_async_wait_all();
  __syncthreads();
  if (!va) return;
  for (int j = 0; j < np_cta; ++j) {
    const int pj = p0 + j;
    if (!((pend >> j) & 1u)) continue;
    // row k of the window is tile row 2 pr + k, k = 0..5; pixel a sits in row 2, b in row 3
    const cx *rw = ztile + j * H * W + 2 * pr * W + fx + 2;
    const cx m2 = rw[0];
    const cx m1l = rw[W - 1], m1c = rw[W], m1r = rw[W + 1];
    const cx a_l2 = rw[2 * W - 2], a_l1 = rw[2 * W - 1], a_c = rw[2 * W], a_r1 = rw[2 * W + 1], a_r2 = rw[2 * W + 2];
    const cx b_l2 = rw[3 * W - 2], b_l1 = rw[3 * W - 1], b_c = rw[3 * W], b_r1 = rw[3 * W + 1], b_r2 = rw[3 * W + 2];
    const cx p2l = rw[4 * W - 1], p2c = rw[4 * W], p2r = rw[4 * W + 1];
    const cx p3 = rw[5 * W];
    // taps (dy, dx): (0,0) (0,-1) (0,1) (-1,0) (1,0) (-1,-1) (-1,1) (1,-1) (1,1) (0,-2) (0,2) (-2,0) (2,0)
    cx A = a_c;
    A = cfma(wa[0], a_c, A);
    A = cfma(wa[1], a_l1, A);
    A = cfma(wa[2], a_r1, A);
    A = cfma(wa[3], m1c, A);
    A = cfma(wa[4], b_c, A);
    A = cfma(wa[5], m1l, A);
    A = cfma(wa[6], m1r, A);
    A = cfma(wa[7], b_l1, A);
    A = cfma(wa[8], b_r1, A);
    A = cfma(wa[9], a_l2, A);
    A = cfma(wa[10], a_r2, A);
    A = cfma(wa[11], m2, A);
    A = cfma(wa[12], p2c, A);
    cx B = b_c;
    B = cfma(wb[0], b_c, B);
    B = cfma(wb[1], b_l1, B);
    B = cfma(wb[2], b_r1, B);
    B = cfma(wb[3], a_c, B);
    B = cfma(wb[4], p2c, B);
    B = cfma(wb[5], a_l1, B);
    B = cfma(wb[6], a_r1, B);
    B = cfma(wb[7], p2l, B);
    B = cfma(wb[8], p2r, B);
    B = cfma(wb[9], b_l2, B);
    B = cfma(wb[10], b_r2, B);
    B = cfma(wb[11], m1c, B);
    B = cfma(wb[12], p3, B);
    cx *dst = out + (size_t)pj * q.N + (size_t)ba * nf + f;
    dst[0] = A;
    if (vb) dst[nf] = B;
  }
}

// The same correction without shared memory, for nf = NF in {64, 128, 192,
// 256}: a CTA of NF threads owns one row pair and kFilterProbes probes; each
// thread keeps its two pixels' taps in registers, loads its own column's six
// rows (b - 2 .. b + 3, zero outside the image) of each probe from global
// memory, and takes the columns f -+ 1 and f -+ 2 from the neighbouring lanes
// by warp shuffles (the two lanes at each end of a warp load the columns
// beyond it).  No staging copies, no barrier: ~30 us per pass at 256 x 256,
// 64 probes, against ~42 us for the shared-memory tile kernel above.
// Grid (ceil(nb / 2), ceil(P / kFilterProbes)).
template <int NF>
__global__ void __launch_bounds__(NF, 2) c3_filter_shfl_kernel(const C3Params q, const C3State *st, int chunk,
                                                               const cx *__restrict__ Fall,
                                                               const cx *__restrict__ z, cx *__restrict__ out,
                                                               const Krylov *K, int second) {
  static_assert(NF % 32 == 0 && NF <= 256, "one thread per column, whole warps");
  if (second && st->it == 0 && st->cheap) return;
  const int nb = q.nb;
  const int lane = threadIdx.x & 31, f = threadIdx.x;
  const int ba = blockIdx.x * 2, p0 = blockIdx.y * kFilterProbes;
  const int np_cta = q.P - p0 < kFilterProbes ? q.P - p0 : kFilterProbes;
  unsigned pend = 0;
  for (int j = 0; j < np_cta; ++j)
    if (K == nullptr || !K[p0 + j].done) pend |= 1u << j;
  const bool vb = ba + 1 < nb;
  const int sl = st->s - 1;
  const size_t npx = (size_t)chunk * q.N;
  const cx *F = Fall + (size_t)(sl / chunk) * kFilterTaps * npx + (size_t)(sl % chunk) * q.N;
  const float cs = q.conj_t ? -1.f : 1.f;
  const cx zero = czero();
  cx wa[kFilterTaps], wb[kFilterTaps];
#pragma unroll
  for (int t = 0; t < kFilterTaps; ++t) {
    const cx a = F[(size_t)t * npx + (size_t)ba * NF + f];
    const cx b = vb ? F[(size_t)t * npx + (size_t)(ba + 1) * NF + f] : zero;
    wa[t] = mkcx(a.x, cs * a.y);
    wb[t] = mkcx(b.x, cs * b.y);
  }
  for (int j = 0; j < np_cta; ++j) {
    if (!((pend >> j) & 1u)) continue;  // the same for every thread: the shuffles below stay converged
    const cx *zp = z + (size_t)(p0 + j) * q.N;
    cx c[6];  // rows ba - 2 .. ba + 3 of column f
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int row = ba - 2 + r;
      c[r] = (row >= 0 && row < nb) ? zp[(size_t)row * NF + f] : zero;
    }
    cx w1[4], e1[4], w2[2], e2[2];  // columns f - 1, f + 1 (rows ba - 1 .. ba + 2), f - 2, f + 2 (rows ba, ba + 1)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      w1[k] = shfl_up2(c[k + 1], 1);
      e1[k] = shfl_down2(c[k + 1], 1);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      w2[k] = shfl_up2(c[k + 2], 2);
      e2[k] = shfl_down2(c[k + 2], 2);
    }
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int row = ba - 1 + k;
        w1[k] = (f >= 1 && row >= 0 && row < nb) ? zp[(size_t)row * NF + f - 1] : zero;
      }
    }
    if (lane < 2) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int row = ba + k;
        w2[k] = (f >= 2 && row < nb) ? zp[(size_t)row * NF + f - 2] : zero;
      }
    }
    if (lane == 31) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int row = ba - 1 + k;
        e1[k] = (f + 1 < NF && row >= 0 && row < nb) ? zp[(size_t)row * NF + f + 1] : zero;
      }
    }
    if (lane >= 30) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int row = ba + k;
        e2[k] = (f + 2 < NF && row < nb) ? zp[(size_t)row * NF + f + 2] : zero;
      }
    }
    // taps (dy, dx): (0,0) (0,-1) (0,1) (-1,0) (1,0) (-1,-1) (-1,1) (1,-1) (1,1) (0,-2) (0,2) (-2,0) (2,0)
    cx A = c[2];
    A = cfma(wa[0], c[2], A);
    A = cfma(wa[1], w1[1], A);
    A = cfma(wa[2], e1[1], A);
    A = cfma(wa[3], c[1], A);
    A = cfma(wa[4], c[3], A);
    A = cfma(wa[5], w1[0], A);
    A = cfma(wa[6], e1[0], A);
    A = cfma(wa[7], w1[2], A);
    A = cfma(wa[8], e1[2], A);
    A = cfma(wa[9], w2[0], A);
    A = cfma(wa[10], e2[0], A);
    A = cfma(wa[11], c[0], A);
    A = cfma(wa[12], c[4], A);
    cx B = c[3];
    B = cfma(wb[0], c[3], B);
    B = cfma(wb[1], w1[2], B);
    B = cfma(wb[2], e1[2], B);
    B = cfma(wb[3], c[2], B);
    B = cfma(wb[4], c[4], B);
    B = cfma(wb[5], w1[1], B);
    B = cfma(wb[6], e1[1], B);
    B = cfma(wb[7], w1[3], B);
    B = cfma(wb[8], e1[3], B);
    B = cfma(wb[9], w2[1], B);
    B = cfma(wb[10], e2[1], B);
    B = cfma(wb[11], c[1], B);
    B = cfma(wb[12], c[5], B);
    cx *dst = out + (size_t)(p0 + j) * q.N + (size_t)ba * NF + f;
    dst[0] = A;
    if (vb) dst[NF] = B;
  }
}

// The same correction with each probe's six rows b - 2 .. b + 3 staged in
// shared memory by one bulk copy per probe: a CTA issues the copies of all
// its pending probes at once (one mbarrier each; rows outside the image are
// not copied but zero-filled) and filters each probe as its copy lands, so
// the loads of the later probes overlap the arithmetic of the earlier ones.
// Every tap reads shared memory at a fixed offset (row, column f + dx;
// columns outside the image read zero), and the multiply-adds run in the
// order of c3_filter_shfl_kernel, so both kernels give the same bits.  Waits
// are bounded (kDevMbarTimeout); a thread that gives up waits for the CTA's
// other copies before it returns.  nf = NF in {64, 128, 192, 256}, z 16-byte
// aligned; a CTA of NF threads, one row pair, kFilterProbes probes.
// Grid (ceil(nb / 2), ceil(P / kFilterProbes)).
constexpr int kFilterRows = 6;

template <int NF>
__global__ void __launch_bounds__(NF, 2) c3_filter_bulk_kernel(const C3Params q, const C3State *st, int chunk,
                                                               const cx *__restrict__ Fall,
                                                               const cx *__restrict__ z, cx *__restrict__ out,
                                                               const Krylov *K, int second, int *err) {
  static_assert(NF % 32 == 0 && NF <= 256, "one thread per column, whole warps");
  constexpr int RW = kFilterRows;
  extern __shared__ __align__(128) cx zs[];  // [kFilterProbes][RW][NF]
  __shared__ __align__(8) uint64_t bar[kFilterProbes];
  if (second && st->it == 0 && st->cheap) return;
  const int nb = q.nb, f = threadIdx.x;
  const int ba = blockIdx.x * 2, p0 = blockIdx.y * kFilterProbes;
  const int np_cta = q.P - p0 < kFilterProbes ? q.P - p0 : kFilterProbes;
  unsigned pend = 0;
  for (int j = 0; j < np_cta; ++j)
    if (K == nullptr || !K[p0 + j].done) pend |= 1u << j;
  if (pend == 0) return;
  // staged rows r_lo .. r_hi - 1 (image rows ba - 2 + r) lie inside the image
  const int r_lo = ba < 2 ? 2 - ba : 0;
  const int r_hi = ba + 4 > nb ? nb - ba + 2 : RW;
  if (threadIdx.x == 0) {
    for (int j = 0; j < kFilterProbes; ++j) mbar_init(&bar[j], 1);
    fence_mbar_init();
  }
  if (r_lo > 0 || r_hi < RW) {
    for (int j = 0; j < np_cta; ++j) {
      if (!((pend >> j) & 1u)) continue;
      for (int r = 0; r < RW; ++r)
        if (r < r_lo || r >= r_hi) zs[(j * RW + r) * NF + f] = czero();
    }
  }
  __syncthreads();
  if (threadIdx.x < np_cta && ((pend >> threadIdx.x) & 1u)) {
    const int j = threadIdx.x;
    const uint32_t bytes = (uint32_t)((r_hi - r_lo) * NF * sizeof(cx));
    mbar_arrive_expect_tx(&bar[j], bytes);
    bulk_g2s(&zs[(j * RW + r_lo) * NF], z + (size_t)(p0 + j) * q.N + (size_t)(ba - 2 + r_lo) * NF, bytes, &bar[j]);
  }
  const bool vb = ba + 1 < nb;
  const int sl = st->s - 1;
  const size_t npx = (size_t)chunk * q.N;
  const cx *F = Fall + (size_t)(sl / chunk) * kFilterTaps * npx + (size_t)(sl % chunk) * q.N;
  const float cs = q.conj_t ? -1.f : 1.f;
  const cx zero = czero();
  cx wa[kFilterTaps], wb[kFilterTaps];
#pragma unroll
  for (int t = 0; t < kFilterTaps; ++t) {
    const cx a = F[(size_t)t * npx + (size_t)ba * NF + f];
    const cx b = vb ? F[(size_t)t * npx + (size_t)(ba + 1) * NF + f] : zero;
    wa[t] = mkcx(a.x, cs * a.y);
    wb[t] = mkcx(b.x, cs * b.y);
  }
  const bool hw1 = f >= 1, he1 = f + 1 < NF, hw2 = f >= 2, he2 = f + 2 < NF;
  for (int j = 0; j < np_cta; ++j) {
    if (!((pend >> j) & 1u)) continue;
    if (!mbar_wait_bounded(&bar[j], 0, err)) {
      for (int k = j + 1; k < np_cta; ++k)
        if ((pend >> k) & 1u) mbar_wait_bounded(&bar[k], 0, nullptr);
      return;
    }
    const cx *zr = zs + j * RW * NF + f;  // column f of the probe's staged rows
    cx c[RW];
#pragma unroll
    for (int r = 0; r < RW; ++r) c[r] = zr[r * NF];
    cx w1[4], e1[4], w2[2], e2[2];  // columns f - 1, f + 1 (rows ba - 1 .. ba + 2), f - 2, f + 2 (rows ba, ba + 1)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      w1[k] = hw1 ? zr[(k + 1) * NF - 1] : zero;
      e1[k] = he1 ? zr[(k + 1) * NF + 1] : zero;
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      w2[k] = hw2 ? zr[(k + 2) * NF - 2] : zero;
      e2[k] = he2 ? zr[(k + 2) * NF + 2] : zero;
    }
    // taps (dy, dx): (0,0) (0,-1) (0,1) (-1,0) (1,0) (-1,-1) (-1,1) (1,-1) (1,1) (0,-2) (0,2) (-2,0) (2,0)
    cx A = c[2];
    A = cfma(wa[0], c[2], A);
    A = cfma(wa[1], w1[1], A);
    A = cfma(wa[2], e1[1], A);
    A = cfma(wa[3], c[1], A);
    A = cfma(wa[4], c[3], A);
    A = cfma(wa[5], w1[0], A);
    A = cfma(wa[6], e1[0], A);
    A = cfma(wa[7], w1[2], A);
    A = cfma(wa[8], e1[2], A);
    A = cfma(wa[9], w2[0], A);
    A = cfma(wa[10], e2[0], A);
    A = cfma(wa[11], c[0], A);
    A = cfma(wa[12], c[4], A);
    cx B = c[3];
    B = cfma(wb[0], c[3], B);
    B = cfma(wb[1], w1[2], B);
    B = cfma(wb[2], e1[2], B);
    B = cfma(wb[3], c[2], B);
    B = cfma(wb[4], c[4], B);
    B = cfma(wb[5], w1[1], B);
    B = cfma(wb[6], e1[1], B);
    B = cfma(wb[7], w1[3], B);
    B = cfma(wb[8], e1[3], B);
    B = cfma(wb[9], w2[1], B);
    B = cfma(wb[10], e2[1], B);
    B = cfma(wb[11], c[1], B);
    B = cfma(wb[12], c[5], B);
    cx *dst = out + (size_t)(p0 + j) * q.N + (size_t)ba * NF + f;
    dst[0] = A;
    if (vb) dst[NF] = B;
  }
}
#endif  // TP_C128_CHECK

// out = (I - P_s) x (no inner products): right-hand sides of the white-noise
// training pairs.  Grid (chunks, P).
__global__ void __launch_bounds__(k3Threads) c3_apply_a_kernel(const C3Params q, const cx *__restrict__ cd,
                                                               const cx *__restrict__ x, cx *out) {
  const size_t off = (size_t)blockIdx.y * q.N;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < q.N; i += gridDim.x * blockDim.x)
    out[off + i] = csub(x[off + i], apply_P(q, cd, x + off, i));
}

// x = uniform complex white noise in [-1, 1]^2 from a counter hash of
// (step, probe, row): reproducible, independent of the launch shape.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__global__ void c3_noise_kernel(int N, int P, int step, cx *x) {
  const size_t total = (size_t)P * N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const uint64_t h = mix64(((uint64_t)step << 40) ^ (uint64_t)e);
    const rx a = (rx)(h >> 40) * (TP_R(1.0) / TP_R(16777216.0)), b = (rx)((h >> 16) & 0xFFFFFFu) * (TP_R(1.0) / TP_R(16777216.0));
    x[e] = mkcx(TP_R(2.0) * a - TP_R(1.0), TP_R(2.0) * b - TP_R(1.0));
  }
}

// stats[4] = how the march ran: 1 as one CUDA graph with device-side loops, 0 step by step.
__global__ void c3_flag_kernel(int *stats, int graph) { stats[4] = graph; }

// out[i] = cd[i] - kc[i]: the object part sigma*T(c_s) of the slice's diagonal.
__global__ void c3_diag_diff_kernel(int N, const cx *__restrict__ cd, const cx *__restrict__ kc, cx *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    out[i] = mkcx(cd[i].x - kc[i].x, cd[i].y - kc[i].y);
}

// ------------------------------------------------------------------ host
struct C3Work {
  cx *u, *x, *r, *r0, *p, *v, *s, *y, *z, *t, *hat;
  cx *cdl, *cdr;
  cx *dc, *dw, *de, *ds, *dn;
  cx *sym, *twf, *twb;  // preconditioner symbol (N) and twiddle tables
  cx *tw4;              // padded twiddle table of the four-step transforms
  rx *ab;                // 2 cos(2 pi f / nf) - 2, then the same for b / nb
  Krylov *K;
  C3State *st;
  size_t bytes;
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

static C3Work c3_layout(char *base, int N, int P) {
  C3Work w{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char *ptr = base ? base + off : nullptr;
    off += align256(bytes);
    return ptr;
  };
  const size_t vec = (size_t)P * N * sizeof(cx);
  cx **vecs[] = {&w.u, &w.x, &w.r, &w.r0, &w.p, &w.v, &w.s, &w.y, &w.z, &w.t, &w.hat};
  for (cx **v : vecs) *v = reinterpret_cast<cx *>(take(vec));
  cx **diag[] = {&w.cdl, &w.cdr, &w.dc, &w.dw, &w.de, &w.ds, &w.dn, &w.sym};
  for (cx **d : diag) *d = reinterpret_cast<cx *>(take((size_t)N * sizeof(cx)));
  w.twf = reinterpret_cast<cx *>(take((size_t)kFftMaxN * sizeof(cx)));
  w.twb = reinterpret_cast<cx *>(take((size_t)kFftMaxN * sizeof(cx)));
  w.tw4 = reinterpret_cast<cx *>(take((size_t)four_tw_len(256) * sizeof(cx)));
  w.ab = reinterpret_cast<rx *>(take((size_t)2 * kFftMaxN * sizeof(rx)));
  w.K = reinterpret_cast<Krylov *>(take((size_t)P * sizeof(Krylov)));
  w.st = reinterpret_cast<C3State *>(take(sizeof(C3State)));
  w.bytes = off;
  return w;
}

using RowsKernel = void (*)(const FftPlan, const C3Params, int, const cx *, cx *, const cx *, cx *,
                           cx *, const Krylov *, int, int, const cx *, const cx *, const C3State *);
using ColsKernel = void (*)(const FftPlan, const C3Params, cx *, const Krylov *, int, const cx *,
                           const cx *);
using InvKernel = void (*)(const FftPlan, const C3Params, const cx *, cx *, const Krylov *, int, const cx *, cx *,
                          const C3State *);
struct PrecKernels {
  RowsKernel rows;
  ColsKernel cols;
  InvKernel inv;
  int fixed;  // compile-time plans in the padded shared-memory layout
};

template <int NF, int NB>
static PrecKernels prec_kernels_t() {
  return {c3_prec_rows_kernel<NF>, c3_prec_cols_kernel<NB>, c3_prec_rows_inv_kernel<NF>, NF > 0 ? 1 : 0};
}

// Square transverse grids of the common sizes get compile-time FFT plans.
static PrecKernels prec_kernels(int nf, int nb) {
  if (nf == nb) {
    switch (nf) {
      case 32: return prec_kernels_t<32, 32>();
      case 64: return prec_kernels_t<64, 64>();
      case 128: return prec_kernels_t<128, 128>();
      case 192: return prec_kernels_t<192, 192>();
      case 256: return prec_kernels_t<256, 256>();
      case 512: return prec_kernels_t<512, 512>();
      default: break;
    }
  }
  return prec_kernels_t<0, 0>();
}

using Rows4Kernel = void (*)(const C3Params, int, const cx *, cx *, const cx *, cx *, cx *,
                            const Krylov *, const cx *, const cx *, const C3State *);
using Cols4Kernel = void (*)(const C3Params, cx *, const Krylov *, const cx *, const rx *);
using Inv4Kernel = void (*)(const C3Params, const cx *, cx *, const Krylov *, const cx *, cx *, const C3State *);
struct Prec4Kernels {
  Rows4Kernel rows = nullptr;
  Cols4Kernel cols = nullptr;
  Inv4Kernel inv = nullptr;
  int r1 = 0, r2 = 0;
};

template <int R1, int R2>
static Prec4Kernels prec4_kernels_t() {
  return {c3_rows4_kernel<R1, R2>, c3_cols4_kernel<R1, R2>, c3_rows4_inv_kernel<R1, R2>, R1, R2};
}

// Register four-step kernels for square grids of 64, 128, 192 and 256 (rows
// kernel nullptr otherwise).
static Prec4Kernels prec4_kernels(int nf, int nb) {
  if (nf != nb || !four_step_size(nf)) return {};
  static_assert(four_r1(64) == 8 && four_r1(128) == 16 && four_r1(192) == 16 && four_r1(256) == 16, "plans");
  switch (nf) {
    case 64: return prec4_kernels_t<8, 8>();
    case 128: return prec4_kernels_t<16, 8>();
#ifndef TP_C128_CHECK  // complex128 tiles of 192 and 256 exceed 48 KB of static shared memory
    case 192: return prec4_kernels_t<16, 12>();
    default: return prec4_kernels_t<16, 16>();
#else
    default: return {};
#endif
  }
}

// Grid of a stencil kernel: ceil(P / kStencilProbes) probe groups times as
// many element blocks as fill one wave of resident CTAs (at least 1, at most
// one element per thread).
template <class Kern>
static dim3 stencil_grid(Kern kernel, int N, int P) {
  int dev = 0, sms = 148, occ = 1;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, k3Threads, 0) != cudaSuccess || occ < 1) occ = 1;
  (void)cudaGetLastError();
  const int gy = (P + kStencilProbes - 1) / kStencilProbes;
  int gx = (sms * occ) / gy;
  const int gmax = (N + k3Threads - 1) / k3Threads;
  if (gx > gmax) gx = gmax;
  if (gx < 1) gx = 1;
  return dim3(gx, gy);
}

// FFT rows per CTA: at most 16 and 4096 elements, and a divisor of the row count.
static int fft_rows_of(int n, int rows) {
  int r = 4096 / n;
  if (r > 16) r = 16;
  if (r < 1) r = 1;
  while (rows % r != 0) --r;
  return r;
}

// Learned-preconditioner workspace: the CNN activations of one chunk of
// slices, the per-pixel filters of every slice (chunked, see c3_filter_kernel),
// the object diagonals of one chunk and the plain-preconditioned vectors (P, N).
constexpr int kCnnChunk = 64;

static int cnn_chunk(int L) { return L < kCnnChunk ? L : kCnnChunk; }

struct C3Learned {
  char *cnn;
  cx *F, *dg, *zt;
  int chunk, nchunks;
  size_t cnn_bytes, bytes;
};

static C3Learned c3_learned_layout(char *base, int nf, int nb, int nz, int P) {
  C3Learned l{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char *ptr = base ? base + off : nullptr;
    off += align256(bytes);
    return ptr;
  };
  const size_t N = (size_t)nf * nb;
  const int L = nz - 1;
  l.chunk = cnn_chunk(L);
  l.nchunks = (L + l.chunk - 1) / l.chunk;
#ifndef TP_C128_CHECK
  l.cnn_bytes = cnn_forward_ws_bytes(conv_geom(nb, nf, l.chunk));
#else
  l.cnn_bytes = 0;
#endif
  l.cnn = take(l.cnn_bytes);
  l.F = reinterpret_cast<cx *>(take((size_t)l.nchunks * kFilterTaps * l.chunk * N * sizeof(cx)));
  l.dg = reinterpret_cast<cx *>(take((size_t)l.chunk * N * sizeof(cx)));
  l.zt = reinterpret_cast<cx *>(take((size_t)P * N * sizeof(cx)));
  l.bytes = off;
  return l;
}

// Streams used only to record graphs (never to run work), one set per host thread.
struct CaptureStreams {
  cudaStream_t s[3] = {nullptr, nullptr, nullptr};
  int dev = -1;
  ~CaptureStreams() {
    for (cudaStream_t &x : s)
      if (x) cudaStreamDestroy(x);
  }
};

static int capture_streams(cudaStream_t **out) {
  static thread_local CaptureStreams cs;
  int dev = 0;
  TP_CHECK_CUDA(cudaGetDevice(&dev));
  if (cs.dev != dev) {
    for (cudaStream_t &x : cs.s) {
      if (x) cudaStreamDestroy(x);
      x = nullptr;
    }
    for (cudaStream_t &x : cs.s) TP_CHECK_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    cs.dev = dev;
  }
  *out = cs.s;
  return TP_OK;
}

// Append a WHILE node (condition `h`, created on the graph being recorded by
// `rec`, default value `dflt` at every launch) after the nodes recorded so
// far on `rec`; returns its body graph.
static int add_while(cudaStream_t rec, unsigned dflt, cudaGraphConditionalHandle *h, cudaGraph_t *body) {
  cudaStreamCaptureStatus status;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  TP_CHECK_CUDA(cudaStreamGetCaptureInfo(rec, &status, nullptr, &g, &deps, &nd));
  if (status != cudaStreamCaptureStatusActive) return set_error(TP_ERR_CUDA, "add_while: stream is not recording");
  TP_CHECK_CUDA(cudaGraphConditionalHandleCreate(h, g, dflt, cudaGraphCondAssignDefault));
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = *h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  TP_CHECK_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
  *body = p.conditional.phGraph_out[0];
  TP_CHECK_CUDA(cudaStreamUpdateCaptureDependencies(rec, &node, 1, cudaStreamSetCaptureDependencies));
  return TP_OK;
}

#ifndef TP_C128_CHECK
// cuTensorMapEncodeTiled, reached through the runtime (the library does not
// link libcuda itself); nullptr when the driver does not provide it.
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiled tensor_map_encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(f);
    (void)cudaGetLastError();
  });
  return fn;
}

struct TmaMaps {
  CUtensorMap mh, mv, md, md4;
};

// The TMA stencil kernels' tensor maps over workspace w: the vector block
// (nf, nb, P, vector) with a (nf, kTmaRows + 2, kStencilProbes, 1) box, and
// the slice diagonals (nf, nb, diagonal) with (nf, kTmaRows, 1) and
// (nf, kTmaRows, 4) boxes.  False if the driver offers no encoder, the
// workspace is not equally spaced or a map is refused.
static bool make_tma_maps(const C3Work &w, int nf, int nb, int P, TmaMaps *m) {
  EncodeTiled enc = tensor_map_encoder();
  if (enc == nullptr) return false;
  const size_t N = (size_t)nf * nb;
  const cuuint64_t vstride = align256((size_t)P * N * sizeof(cx)), dstride = align256(N * sizeof(cx));
  if ((size_t)(reinterpret_cast<char *>(w.x) - reinterpret_cast<char *>(w.u)) != vstride ||
      (size_t)(reinterpret_cast<char *>(w.hat) - reinterpret_cast<char *>(w.u)) != 10 * vstride ||
      (size_t)(reinterpret_cast<char *>(w.sym) - reinterpret_cast<char *>(w.cdl)) != 7 * dstride)
    return false;
  const cuuint64_t row = (cuuint64_t)nf * sizeof(cx);
  const cuuint64_t vdims[4] = {(cuuint64_t)nf, (cuuint64_t)nb, (cuuint64_t)P, (cuuint64_t)kNumVecs};
  const cuuint64_t vstr[3] = {row, (cuuint64_t)N * sizeof(cx), vstride};
  const cuuint32_t vbox[4] = {(cuuint32_t)nf, (cuuint32_t)(kTmaRows + 2), (cuuint32_t)kStencilProbes, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const auto ok = [](CUresult r) { return r == CUDA_SUCCESS; };
  if (!ok(enc(&m->mh, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, w.u, vdims, vstr, vbox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)))
    return false;
  const cuuint32_t pbox[4] = {(cuuint32_t)nf, (cuuint32_t)kTmaRows, (cuuint32_t)kStencilProbes, 1};
  if (!ok(enc(&m->mv, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, w.u, vdims, vstr, pbox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)))
    return false;
  const cuuint64_t ddims[3] = {(cuuint64_t)nf, (cuuint64_t)nb, (cuuint64_t)kNumDiags};
  const cuuint64_t dstr[2] = {row, dstride};
  const cuuint32_t dbox1[3] = {(cuuint32_t)nf, (cuuint32_t)kTmaRows, 1};
  const cuuint32_t dbox4[3] = {(cuuint32_t)nf, (cuuint32_t)kTmaRows, 4};
  if (!ok(enc(&m->md, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, w.cdl, ddims, dstr, dbox1, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)))
    return false;
  if (!ok(enc(&m->md4, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, w.cdl, ddims, dstr, dbox4, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)))
    return false;
  return true;
}

using TmaKernel = void (*)(const CUtensorMap, const CUtensorMap, const CUtensorMap, const CUtensorMap, const C3Params,
                           const C3State *, const TmaArgs, Krylov *, int *);
struct TmaLaunch {
  TmaKernel kern = nullptr;
  size_t smem = 0;
  dim3 grid;
};

template <int KIND, int NF>
static int tma_launch_t(int nb, int P, TmaLaunch *out) {
  auto kern = c3_tma_kernel<KIND, NF>;
  const size_t smem = 2 * (size_t)tma_stage_bytes<KIND, NF>();
  TP_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, sms = 148, occ = 1;
  TP_CHECK_CUDA(cudaGetDevice(&dev));
  TP_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, k3Threads, smem) != cudaSuccess || occ < 1) occ = 1;
  (void)cudaGetLastError();
  const int gy = (P + kStencilProbes - 1) / kStencilProbes, nblk = nb / kTmaRows;
  int gx = (sms * occ) / gy;
  if (gx > nblk) gx = nblk;
  if (gx < 1) gx = 1;
  out->kern = kern;
  out->smem = smem;
  out->grid = dim3(gx, gy);
  return TP_OK;
}

// The launch of stencil kind KIND at transverse width nf (kern nullptr: no
// tensor-memory kernel for that width).
template <int KIND>
static int tma_launch(int nf, int nb, int P, TmaLaunch *out) {
  switch (nf) {
    case 64: return tma_launch_t<KIND, 64>(nb, P, out);
    case 128: return tma_launch_t<KIND, 128>(nb, P, out);
    case 192: return tma_launch_t<KIND, 192>(nb, P, out);
    case 256: return tma_launch_t<KIND, 256>(nb, P, out);
    default: return TP_OK;
  }
}
#endif  // TP_C128_CHECK

}  // namespace tp

using namespace tp;

extern "C" size_t tp_cn3d_learned_ws_bytes(int32_t nf, int32_t nb, int32_t nz, int32_t num_probes) {
  if (nf < 1 || nb < 1 || nz < 2 || num_probes < 1) return 0;
  return c3_learned_layout(nullptr, nf, nb, nz, num_probes).bytes;
}

extern "C" size_t tp_cn3d_workspace_bytes(int32_t n_total, int32_t num_probes) {
  if (n_total < 1 || num_probes < 1) return 0;
  return c3_layout(nullptr, n_total, num_probes).bytes;
}

extern "C" int tp_cn3d_march(const tp_cn3d_op *op, const void *n_field, int32_t n_dtype, const tp_cn3d_march_args *a,
                             void *workspace, size_t workspace_bytes, tp_stream_t stream) {
  if (op == nullptr || a == nullptr || n_field == nullptr || workspace == nullptr)
    return set_error(TP_ERR_INVALID, "tp_cn3d_march: NULL argument");
  const int nf = op->nf, nb = op->nb, N = nf * nb, P = a->num_probes, nz = op->nz, L = nz - 1;
  if (nf < 2 || nb < 2 || nz < 2 || P < 1) return set_error(TP_ERR_INVALID, "bad 3D sizes nf=%d nb=%d nz=%d P=%d", nf, nb, nz, P);
  if (a->mode < TP_MODE_FORWARD || a->mode > TP_MODE_ADJOINT_EXACT) return set_error(TP_ERR_INVALID, "bad mode");
  if ((a->grad_c != nullptr) != (a->u_fwd != nullptr) || (a->grad_c != nullptr && a->mode != TP_MODE_ADJOINT_EXACT))
    return set_error(TP_ERR_INVALID, "the gradient needs TP_MODE_ADJOINT_EXACT with u_fwd and grad_c");
  if (a->mode == TP_MODE_ADJOINT_EXACT && a->probes != nullptr)
    return set_error(TP_ERR_INVALID, "TP_MODE_ADJOINT_EXACT starts from lambda = 0 (probes must be NULL)");
  if ((reinterpret_cast<uintptr_t>(workspace) & 255u) != 0) return set_error(TP_ERR_INVALID, "workspace must be 256-byte aligned");
  C3Work w = c3_layout(static_cast<char *>(workspace), N, P);
  if (workspace_bytes < w.bytes) return set_error(TP_ERR_WORKSPACE, "3D workspace %zu B < %zu B", workspace_bytes, w.bytes);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

  C3Params q{};
  q.nf = nf;
  q.nb = nb;
  q.N = N;
  q.nz = nz;
  q.L = L;
  q.P = P;
  q.exact = op->exact_ref_coeff;
  q.is_delta = op->field_is_delta;
  q.dtype = n_dtype;
  q.conj_t = (a->mode == TP_MODE_ADJOINT || a->mode == TP_MODE_ADJOINT_EXACT) ? 1 : 0;
  q.sigma = (a->mode == TP_MODE_REVERSE) ? -1.0 : 1.0;
  q.k = op->k;
  q.dz = op->dz;
  auto tr = [&](const double v[2]) { return z2(q.sigma * v[0], q.sigma * (q.conj_t ? -v[1] : v[1])); };
  q.mu_x = tr(op->mu_x);
  q.mu_y = tr(op->mu_y);
  q.field = n_field;
  q.kc = w.dc;
  q.kw = w.dw;
  q.ke = w.de;
  q.ks = w.ds;
  q.kn = w.dn;

  const FftPlan pf = make_fft_plan(nf), pb = make_fft_plan(nb);
  const int fft_on = a->precond != 0 && pf.npass > 0 && pb.npass > 0;
  const bool learned = a->precond == 2;
  C3Learned lw{};
  if (learned) {
#ifdef TP_C128_CHECK
    return set_error(TP_ERR_UNSUPPORTED, "the complex128 check build has no learned preconditioner");
#endif
    if (a->model == nullptr || a->learned_ws == nullptr)
      return set_error(TP_ERR_INVALID, "learned preconditioner: NULL model or workspace");
    if (!fft_on) return set_error(TP_ERR_UNSUPPORTED, "learned preconditioner needs FFT-plannable nf, nb (got %d, %d)", nf, nb);
    if (a->mode == TP_MODE_REVERSE) return set_error(TP_ERR_UNSUPPORTED, "learned preconditioner: REVERSE mode is not supported");
    if ((reinterpret_cast<uintptr_t>(a->learned_ws) & 255u) != 0)
      return set_error(TP_ERR_INVALID, "learned workspace must be 256-byte aligned");
    lw = c3_learned_layout(static_cast<char *>(a->learned_ws), nf, nb, nz, P);
    if (a->learned_ws_bytes < lw.bytes)
      return set_error(TP_ERR_WORKSPACE, "learned workspace %zu B < %zu B", a->learned_ws_bytes, lw.bytes);
  }
  const bool train = a->train_every > 0;
  if (train && (a->train_z0 == nullptr || a->train_sol == nullptr || a->train_diag == nullptr))
    return set_error(TP_ERR_INVALID, "train_every needs train_z0, train_sol and train_diag");
  const int rpc = fft_rows_of(nf, nb), cpc = fft_rows_of(nb, nf);
  const int use_fft = fft_on;
  // kernels of the preconditioner: compile-time FFT plans for the common sizes
  PrecKernels pk = prec_kernels(nf, nb);
  const Prec4Kernels p4 = (fft_on && (a->kernels & 1) == 0) ? prec4_kernels(nf, nb) : Prec4Kernels{};
  const bool four = p4.rows != nullptr;
  const int rpc4 = four ? 256 / p4.r1 : 1;
  const int srow_f = pk.fixed ? nf + nf / 8 + 1 : nf, srow_b = pk.fixed ? nb + nb / 8 + 1 : nb;
  const size_t smem_rows = (size_t)(nf + 2 * rpc * srow_f) * sizeof(cx);
  const size_t smem_cols = (size_t)(nb + 2 * cpc * srow_b) * sizeof(cx);
  if (use_fft) {
    TP_CHECK_CUDA(cudaFuncSetAttribute(pk.rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_rows));
    TP_CHECK_CUDA(cudaFuncSetAttribute(pk.inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_rows));
    TP_CHECK_CUDA(cudaFuncSetAttribute(pk.cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cols));
  }

  const int rows_cta = use_fft ? rpc : 1;
  const int max_iter = a->max_iter > 0 ? a->max_iter : 20;
  const double tol2 = (a->tol > 0 ? a->tol : 1e-6) * (a->tol > 0 ? a->tol : 1e-6);
  int *stats = a->stats;
  const bool backward = a->mode != TP_MODE_FORWARD;
  const bool flip = a->mode == TP_MODE_ADJOINT;
  const int adj_exact = a->mode == TP_MODE_ADJOINT_EXACT ? 1 : 0;
  cx *ust = static_cast<cx *>(a->u_store);
  cx *exit_out = static_cast<cx *>(a->exit_out);
#ifndef TP_C128_CHECK
  // learned filter: column blocks of at most 256, two rows per thread
  const int fcw = filter_cw(nf), frb = filter_rb(nf);
  const dim3 fgrid((nf + fcw - 1) / fcw, (nb + frb - 1) / frb, (P + kFilterProbes - 1) / kFilterProbes);
  const size_t smem_filter = (size_t)kFilterProbes * (frb + 4) * (fcw + 4) * sizeof(cx);
  if (learned)
    TP_CHECK_CUDA(cudaFuncSetAttribute(c3_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_filter));
  // widths with one thread per column take the bulk-staged kernel (bit 2 of
  // kernels: the register-shuffle kernel), other widths the tile kernel
  using ShflFilter = void (*)(const C3Params, const C3State *, int, const cx *, const cx *, cx *, const Krylov *, int);
  using BulkFilter = void (*)(const C3Params, const C3State *, int, const cx *, const cx *, cx *, const Krylov *, int,
                              int *);
  const ShflFilter shfl_filter = nf == 64    ? c3_filter_shfl_kernel<64>
                                 : nf == 128 ? c3_filter_shfl_kernel<128>
                                 : nf == 192 ? c3_filter_shfl_kernel<192>
                                 : nf == 256 ? c3_filter_shfl_kernel<256>
                                             : nullptr;
  BulkFilter bulk_filter = nf == 64    ? c3_filter_bulk_kernel<64>
                           : nf == 128 ? c3_filter_bulk_kernel<128>
                           : nf == 192 ? c3_filter_bulk_kernel<192>
                           : nf == 256 ? c3_filter_bulk_kernel<256>
                                       : nullptr;
  int *ferr = nullptr;
  if (!learned || (a->kernels & 4) != 0 || (reinterpret_cast<uintptr_t>(lw.zt) & 15) != 0) bulk_filter = nullptr;
  if (bulk_filter && (ferr = device_error_ptr()) == nullptr) bulk_filter = nullptr;
  const size_t smem_bulk_f = (size_t)kFilterProbes * kFilterRows * nf * sizeof(cx);
  if (bulk_filter)
    TP_CHECK_CUDA(cudaFuncSetAttribute(bulk_filter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bulk_f));
  const dim3 sgrid_f((nb + 1) / 2, (P + kFilterProbes - 1) / kFilterProbes);
  // the correction y = z + F z of application `second` (0 or 1) of an iteration
  auto filter = [&](cudaStream_t s, cx *dst, int second) {
    if (bulk_filter)
      bulk_filter<<<sgrid_f, nf, smem_bulk_f, s>>>(q, w.st, lw.chunk, lw.F, lw.zt, dst, w.K, second, ferr);
    else if (shfl_filter)
      shfl_filter<<<sgrid_f, nf, 0, s>>>(q, w.st, lw.chunk, lw.F, lw.zt, dst, w.K, second);
    else
      c3_filter_kernel<<<fgrid, k3Threads, smem_filter, s>>>(q, w.st, lw.chunk, lw.F, lw.zt, dst, w.K, second);
  };
#endif
  const dim3 vgrid((N + 256 * 8 - 1) / (256 * 8), P);
  const dim3 sg_init = stencil_grid(c3_init_kernel, N, P), sg_fin = stencil_grid(c3_finish_kernel, N, P);
  const dim3 sg_mv0 = stencil_grid(c3_matvec_kernel<0>, N, P), sg_mv1 = stencil_grid(c3_matvec_kernel<1>, N, P);
#ifndef TP_C128_CHECK
  // stencil kernels with tensor-memory staging where the width has an instantiation
  TmaMaps tmaps{};
  TmaLaunch t_init, t_mv0, t_mv1, t_fin;
  bool tma = (a->kernels & 2) == 0 && (nf == 64 || nf == 128 || nf == 192 || nf == 256) && nb % kTmaRows == 0 &&
             make_tma_maps(w, nf, nb, P, &tmaps);
  if (tma) {
    int r = tma_launch<kTmaInit>(nf, nb, P, &t_init);
    if (r == TP_OK) r = tma_launch<kTmaMatvec0>(nf, nb, P, &t_mv0);
    if (r == TP_OK) r = tma_launch<kTmaMatvec1>(nf, nb, P, &t_mv1);
    if (r == TP_OK) r = tma_launch<kTmaFinish>(nf, nb, P, &t_fin);
    if (r != TP_OK) return r;
    tma = t_init.kern && t_mv0.kern && t_mv1.kern && t_fin.kern;
  }
  int *derr = tma ? device_error_ptr() : nullptr;
  if (tma && derr == nullptr) return set_error(TP_ERR_CUDA, "device error word unavailable");
#endif
  const int pgrid = (P + 127) / 128;
  const int one_cta = P >= 1024 ? 1024 : ((P + 31) / 32) * 32;
  const int eb = 296;
#ifndef TP_C128_CHECK
  const ConvGeom gch = learned ? conv_geom(nb, nf, lw.chunk) : ConvGeom{};
#endif

  // ---- launch sequences (recorded into a graph, or issued step by step)
  // M0^{-1} in -> out (mode 0/1/2 input of the row kernel; Kp NULL = all probes)
  auto precondition = [&](cudaStream_t s, int mode, const cx *rin, cx *out, const Krylov *Kp,
                          cx *out_first = nullptr) {
    if (four) {
      p4.rows<<<dim3(nb / rpc4, P), 256, 0, s>>>(q, mode, rin, w.p, w.v, w.s, w.hat, Kp, w.tw4, w.r0, w.st);
      p4.cols<<<dim3(nf / rpc4, P), 256, 0, s>>>(q, w.hat, Kp, w.tw4, w.ab);
      p4.inv<<<dim3(nb / rpc4, P), 256, 0, s>>>(q, w.hat, out, Kp, w.tw4, out_first, w.st);
      return;
    }
    pk.rows<<<dim3(nb / rows_cta, P), k3Threads, use_fft ? smem_rows : 0, s>>>(
        pf, q, mode, rin, w.p, w.v, w.s, use_fft ? w.hat : out, Kp, rows_cta, use_fft, w.twf, w.r0, w.st);
    if (use_fft) {
      pk.cols<<<dim3(nf / cpc, P), k3Threads, smem_cols, s>>>(pb, q, w.hat, Kp, cpc, w.twb, w.sym);
      pk.inv<<<dim3(nb / rpc, P), k3Threads, smem_rows, s>>>(pf, q, w.hat, out, Kp, rpc, w.twf, out_first, w.st);
    }
  };
  auto prologue = [&](cudaStream_t s) -> int {
    if (use_fft) {
      c3_twiddle_kernel<<<(nf + 255) / 256, 256, 0, s>>>(nf, w.twf);
      c3_twiddle_kernel<<<(nb + 255) / 256, 256, 0, s>>>(nb, w.twb);
      if (four) {
        c3_twiddle4_kernel<<<1, 256, 0, s>>>(nf, p4.r1, p4.r2, w.tw4);
        c3_symbol_factors_kernel<<<1, 256, 0, s>>>(nf, nb, w.ab);
      } else {
        c3_symbol_kernel<<<eb, 256, 0, s>>>(q, w.sym);
      }
    }
    c3_diag_kernel<<<eb, 256, 0, s>>>(N, nf, q.sigma, q.conj_t, static_cast<const cx *>(op->kc),
                                      static_cast<const cx *>(op->kw), static_cast<const cx *>(op->ke),
                                      static_cast<const cx *>(op->ks), static_cast<const cx *>(op->kn), w.dc,
                                      w.dw, w.de, w.ds, w.dn);
#ifndef TP_C128_CHECK
    if (learned && !a->learned_reuse) {
      // the filters of every slice, chunk by chunk (the CNN activations' zero
      // borders are never written by the kernels)
      TP_CHECK_CUDA(cudaMemsetAsync(lw.cnn, 0, lw.cnn_bytes, s));
      C3Params qf = q;  // forward orientation
      qf.sigma = 1.0;
      qf.conj_t = 0;
      for (int c = 0; c < lw.nchunks; ++c) {
        const int s0 = c * lw.chunk, cnt = (L - s0) < lw.chunk ? (L - s0) : lw.chunk;
        if (cnt < lw.chunk) TP_CHECK_CUDA(cudaMemsetAsync(lw.dg, 0, (size_t)lw.chunk * N * sizeof(cx), s));
        c3_obj_diag_kernel<<<eb * 2, 256, 0, s>>>(qf, s0, cnt, lw.dg);
        const int rc = cnn_forward(gch, *a->model, lw.dg, N, nullptr, lw.cnn,
                                   lw.F + (size_t)c * kFilterTaps * lw.chunk * N, s);
        if (rc != TP_OK) return rc;
      }
    }
#endif
    TP_CHECK_CUDA(cudaMemsetAsync(w.u, 0, (size_t)P * N * sizeof(cx), s));
    if (a->probes != nullptr)
      TP_CHECK_CUDA(cudaMemcpyAsync(w.u, a->probes, (size_t)P * N * sizeof(cx), cudaMemcpyDeviceToDevice, s));
    TP_CHECK_CUDA(cudaMemsetAsync(w.K, 0, (size_t)P * sizeof(Krylov), s));
    TP_CHECK_CUDA(cudaMemsetAsync(w.st, 0, sizeof(C3State), s));
    if (ust) c3_store_kernel<<<eb, 256, 0, s>>>(N, P, nz, flip ? L : 0, w.u, ust, nullptr);
    return TP_OK;
  };
  // (I - P) y -> v with <r0, v> (which 0), (I - P) z -> t with <t, s>, |t|^2 (which 1)
  auto matvec = [&](cudaStream_t s, int which) {
#ifndef TP_C128_CHECK
    if (tma) {
      TmaArgs ta{};
      ta.vin = which ? kVecZ : kVecY;
      ta.vc0 = which ? kVecS : kVecR0;
      ta.out = which ? w.t : w.v;
      const TmaLaunch &tl = which ? t_mv1 : t_mv0;
      tl.kern<<<tl.grid, k3Threads, tl.smem, s>>>(tmaps.mh, tmaps.mv, tmaps.md, tmaps.md4, q, w.st, ta, w.K, derr);
      return;
    }
#endif
    if (which == 0) c3_matvec_kernel<0><<<sg_mv0, k3Threads, 0, s>>>(q, w.cdl, w.y, w.v, w.r0, w.s, w.K);
    else c3_matvec_kernel<1><<<sg_mv1, k3Threads, 0, s>>>(q, w.cdl, w.z, w.t, w.r0, w.s, w.K);
  };
  // true residual, u += x, store
  auto finish = [&](cudaStream_t s) {
#ifndef TP_C128_CHECK
    if (tma) {
      TmaArgs ta{};
      ta.vin = kVecX;
      ta.vc0 = kVecR0;
      ta.vc1 = kVecU;
      ta.out = w.u;
      ta.u_store = ust;
      ta.exit_out = exit_out;
      ta.flip = flip ? 1 : 0;
      t_fin.kern<<<t_fin.grid, k3Threads, t_fin.smem, s>>>(tmaps.mh, tmaps.mv, tmaps.md, tmaps.md4, q, w.st, ta, w.K, derr);
      return;
    }
#endif
    c3_finish_kernel<<<sg_fin, k3Threads, 0, s>>>(q, w.st, w.cdl, w.x, w.r0, w.u, w.K, ust, flip ? 1 : 0, exit_out);
  };
  // step head: slice state, operators, right-hand side, Krylov start
  auto step_head = [&](cudaStream_t s, int use_cond, cudaGraphConditionalHandle outer, cudaGraphConditionalHandle inner) {
    c3_advance_kernel<<<1, 1, 0, s>>>(w.st, L, backward ? 1 : 0, use_cond, outer, inner);
    c3_center_kernel<<<eb, 256, 0, s>>>(q, w.st, 0, w.cdl);
    if (adj_exact) c3_center_kernel<<<eb, 256, 0, s>>>(q, w.st, 1, w.cdr);
#ifndef TP_C128_CHECK
    if (tma) {
      TmaArgs ta{};
      ta.vin = kVecU;
      ta.out = w.r0;
      ta.src_exit = static_cast<const cx *>(a->src_exit);
      ta.src_shared = static_cast<const cx *>(a->src_shared);
      ta.adj_exact = adj_exact;
      t_init.kern<<<t_init.grid, k3Threads, t_init.smem, s>>>(tmaps.mh, tmaps.mv, tmaps.md, tmaps.md4, q, w.st, ta, w.K, derr);
    } else
#endif
      c3_init_kernel<<<sg_init, k3Threads, 0, s>>>(q, w.st, adj_exact, w.cdl, w.cdr, w.u,
                                                  static_cast<const cx *>(a->src_exit),
                                                  static_cast<const cx *>(a->src_shared), w.r0, w.K);
    c3_start_kernel<<<pgrid, 128, 0, s>>>(w.K, P);
  };
  // one BiCGStab iteration of every pending probe
  auto iteration = [&](cudaStream_t s, int use_cond, cudaGraphConditionalHandle inner) {
    // p = r + beta (p - omega v); y = Prec(p); v = M y
    precondition(s, 0, w.r, learned ? lw.zt : w.y, w.K);
#ifndef TP_C128_CHECK
    if (learned) filter(s, w.y, 0);
#endif
    matvec(s, 0);
    // s = r - alpha v; z = Prec(s); t = M z
    precondition(s, 1, w.r, learned ? lw.zt : w.z, w.K, learned ? w.z : nullptr);
#ifndef TP_C128_CHECK
    if (learned) filter(s, w.z, 1);
#endif
    matvec(s, 1);
    c3_update_kernel<<<vgrid, k3Threads, 0, s>>>(q, w.x, w.r, w.r0, w.y, w.z, w.s, w.t, w.K, w.st);
    c3_commit_kernel<<<1, one_cta, 0, s>>>(w.K, P, tol2, w.st, max_iter, use_cond, inner);
  };
  // step tail: u += x (true residual, store), statistics, gradient
  auto step_tail = [&](cudaStream_t s) {
    finish(s);
    c3_stats_kernel<<<1, one_cta, 0, s>>>(w.K, P, tol2, stats, w.st);
    if (a->grad_c)
      c3_grad_kernel<<<eb, 256, 0, s>>>(N, P, nz, w.st, w.u, static_cast<const cx *>(a->u_fwd),
                                        static_cast<cx *>(a->grad_c));
  };

  // ---- one graph: prologue, then WHILE(step) { head; WHILE(iteration) {..}; tail }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  TP_CHECK_CUDA(cudaStreamIsCapturing(st, &cap));
  const bool use_graph = !train && cap == cudaStreamCaptureStatusNone && a->launch == 0 && a->host_check != 0;
  if (use_graph) {
    cudaStream_t *rs = nullptr;
    int rc = capture_streams(&rs);
    if (rc != TP_OK) return rc;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    TP_CHECK_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h_step = 0, h_iter = 0;
    cudaGraph_t body_step = nullptr, body_iter = nullptr;
    auto record = [&]() -> int {
      TP_CHECK_CUDA(cudaStreamBeginCaptureToGraph(rs[0], g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      int r = prologue(rs[0]);
      if (r == TP_OK) r = add_while(rs[0], 1u, &h_step, &body_step);
      cudaGraph_t g_end = nullptr;
      const cudaError_t e0 = cudaStreamEndCapture(rs[0], &g_end);
      if (r != TP_OK) return r;
      TP_CHECK_CUDA(e0);
      // step body
      TP_CHECK_CUDA(cudaStreamBeginCaptureToGraph(rs[1], body_step, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      // h_iter is created on the step body (it is re-armed by the advance kernel)
      {
        cudaStreamCaptureStatus status;
        cudaGraph_t gb = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        r = check_cuda(cudaStreamGetCaptureInfo(rs[1], &status, nullptr, &gb, &deps, &nd), "cudaStreamGetCaptureInfo");
        if (r == TP_OK) r = check_cuda(cudaGraphConditionalHandleCreate(&h_iter, gb, 1u, 0), "cudaGraphConditionalHandleCreate");
      }
      if (r == TP_OK) {
        step_head(rs[1], 1, h_step, h_iter);
        r = check_cuda(cudaGetLastError(), "step head launches");
      }
      if (r == TP_OK) {
        // the iteration loop, on a node whose handle already exists
        cudaStreamCaptureStatus status;
        cudaGraph_t gb = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        r = check_cuda(cudaStreamGetCaptureInfo(rs[1], &status, nullptr, &gb, &deps, &nd), "cudaStreamGetCaptureInfo");
        if (r == TP_OK) {
          cudaGraphNodeParams p = {};
          p.type = cudaGraphNodeTypeConditional;
          p.conditional.handle = h_iter;
          p.conditional.type = cudaGraphCondTypeWhile;
          p.conditional.size = 1;
          cudaGraphNode_t node;
          r = check_cuda(cudaGraphAddNode(&node, gb, deps, nd, &p), "cudaGraphAddNode (iteration loop)");
          if (r == TP_OK) {
            body_iter = p.conditional.phGraph_out[0];
            r = check_cuda(cudaStreamUpdateCaptureDependencies(rs[1], &node, 1, cudaStreamSetCaptureDependencies),
                           "cudaStreamUpdateCaptureDependencies");
          }
        }
      }
      if (r == TP_OK) {
        step_tail(rs[1]);
        r = check_cuda(cudaGetLastError(), "step tail launches");
      }
      cudaGraph_t b_end = nullptr;
      const cudaError_t e1 = cudaStreamEndCapture(rs[1], &b_end);
      if (r != TP_OK) return r;
      TP_CHECK_CUDA(e1);
      // iteration body
      TP_CHECK_CUDA(cudaStreamBeginCaptureToGraph(rs[2], body_iter, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      iteration(rs[2], 1, h_iter);
      r = check_cuda(cudaGetLastError(), "iteration launches");
      cudaGraph_t i_end = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(rs[2], &i_end);
      if (r != TP_OK) return r;
      TP_CHECK_CUDA(e2);
      TP_CHECK_CUDA(cudaGraphInstantiate(&ge, g, 0));
      return TP_OK;
    };
    rc = record();
    if (rc == TP_OK) {
      rc = check_cuda(cudaGraphLaunch(ge, st), "cudaGraphLaunch (3D march)");
      // an executable graph still running is freed when it completes
      cudaGraphExecDestroy(ge);
      cudaGraphDestroy(g);
      if (rc != TP_OK) return rc;
      if (stats) c3_flag_kernel<<<1, 1, 0, st>>>(stats, 1);
      return check_cuda(cudaGetLastError(), "tp_cn3d_march graph");
    }
    // the graph could not be recorded (nothing of it ran): run step by step
    // below; stats[4] = 0 reports it
    if (ge) cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    (void)cudaGetLastError();
  }

  // ---- step by step on the caller's stream
  int rc = prologue(st);
  if (rc != TP_OK) return rc;
  for (int t = 1; t <= L; ++t) {
    // a training pair copies x, which a probe with a zero right-hand side
    // never writes in its step
    if (train) TP_CHECK_CUDA(cudaMemsetAsync(w.x, 0, (size_t)P * N * sizeof(cx), st));
    step_head(st, 0, 0, 0);
    for (int it = 0; it < max_iter; ++it) {
      iteration(st, 0, 0);
      if (a->host_check && it + 1 < max_iter) {
        // stop launching iterations once every probe has converged
        C3State hs{};
        TP_CHECK_CUDA(cudaMemcpyAsync(&hs, w.st, sizeof(C3State), cudaMemcpyDeviceToHost, st));
        TP_CHECK_CUDA(cudaStreamSynchronize(st));
        if (hs.pending == 0) break;
      }
    }
    finish(st);
    if (train && t % a->train_every == 0) {
      // training pair of this step: z0 = M0^{-1} v and x with (I - P_s) x = v,
      // v the step's right-hand side r0 and x its converged update
      // (train_kind 0), or x white noise and v = (I - P_s) x (train_kind 1);
      // plus the slice's object diagonal
      const size_t k = (size_t)(t / a->train_every - 1);
      cx *tz = static_cast<cx *>(a->train_z0) + k * P * N;
      cx *tx = static_cast<cx *>(a->train_sol) + k * P * N;
      const cx *v = w.r0;
      if (a->train_kind == 1) {
        c3_noise_kernel<<<eb, 256, 0, st>>>(N, P, t, tx);
        c3_apply_a_kernel<<<vgrid, k3Threads, 0, st>>>(q, w.cdl, tx, w.t);
        v = w.t;
      } else {
        TP_CHECK_CUDA(cudaMemcpyAsync(tx, w.x, (size_t)P * N * sizeof(cx), cudaMemcpyDeviceToDevice, st));
      }
      precondition(st, 2, v, tz, nullptr);
      c3_diag_diff_kernel<<<eb, 256, 0, st>>>(N, w.cdl, w.dc, static_cast<cx *>(a->train_diag) + k * N);
    }
    c3_stats_kernel<<<1, one_cta, 0, st>>>(w.K, P, tol2, stats, w.st);
    if (a->grad_c)
      c3_grad_kernel<<<eb, 256, 0, st>>>(N, P, nz, w.st, w.u, static_cast<const cx *>(a->u_fwd),
                                         static_cast<cx *>(a->grad_c));
  }
  if (stats) c3_flag_kernel<<<1, 1, 0, st>>>(stats, 0);
  return check_cuda(cudaGetLastError(), "tp_cn3d_march launches");
}
