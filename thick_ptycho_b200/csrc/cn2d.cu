// 2D paraxial Crank–Nicolson march (1D transverse), batched over probes.
//
// Replaces the reference's per-slice sparse LU (iterative_lu.py:103-133) and
// per-probe z-march (iterative_lu.py:138-197, base/base_solver.py:124-143).
//
// Step t of a march solves  M_s u_t = R_s u_{t-1} + b_t  with
//   M_s = I - P_s,  R_s = I + P_s,  P_s = sigma * T(K + diag(c_s)),
// where sigma = -1 for REVERSE, T = conjugate transpose for the adjoints and
// s = t (forward) or L+1-t (backward).  For ADJOINT_EXACT the right-hand side
// of step t uses P_{s+1} (the exact transpose of the forward recursion).
//
// Numerics: every coefficient is held as a deviation from the identity
// ("1 + eps" form): x*(1+eps) is evaluated as x + x*eps.  Rounding a diagonal
// of size ~1 to fp32 would otherwise perturb the operator by 6e-8 absolute
// every slice, a systematic error that grows linearly with the number of
// slices (4e-5 relative after 1023 slices at N = 2048); in this form the
// complex64 march stays at ~3e-6 of the complex128 result.
//
// Tridiagonal solve (one warp per probe, 32 lanes): the N_pad = 32*M rows are
// cut into 32 chunks of M rows, one per lane.  The last row of each chunk is
// a separator; the M-1 interior rows are eliminated in terms of the two
// neighbouring separators (Schur complement), which leaves a 32-unknown
// tridiagonal system solved by 5 levels of warp-shuffle parallel cyclic
// reduction.  Everything that depends only on the matrix (interior LU
// factors, the two spike vectors, the PCR multipliers) is probe-independent;
// it is computed once per slice in fp64 by cn2d_factor_kernel and streamed
// into shared memory with bulk (TMA) copies, so each probe pays only for
// right-hand-side work.  Data layout of one slice of the factor set (cx
// [rows][32 lanes], row i of lane k is matrix row k*M + i):
//   QD  [M][32]  diagonal of P_s
//   LF  [M][32]  interior forward multipliers (row 0 unused)
//   EP  [M][32]  interior inverse pivots minus one
//   V   [M][32]  spike: response of the interior to the left separator
//   W   [M][32]  spike: response of the interior to the own separator
//   LR  [13][32] per-lane reduced-system data: M sub / super at the
//                separator, 5 PCR alpha, 5 PCR gamma, 1/d_final - 1
// The full field is stored in the same chunked layout (row k*M+i at offset
// i*32+k of a slice), so every warp-wide load/store moves 256 contiguous bytes.

#include <cuda_runtime.h>
#include <stdio.h>

#include "cn2d_internal.cuh"
#include "tp_common.cuh"
#include "tp_errors.h"
#include "tpcuda.h"

namespace tp {

// Warp path: 32 chunks (one per lane), 5 PCR levels, 13 records per chunk.
constexpr int kRecMA = 0, kRecMC = 1, kRecAlpha = 2, kRecGamma = 7, kRecRDE = 12;
constexpr int kMarchWarps = 4;

// Rows-per-lane values of the warp path with compiled kernels.
static const int kRowSet[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64};

static int rows_per_lane_for(int n) {
  int need = (n + kLanes - 1) / kLanes;
  for (int m : kRowSet)
    if (m >= need) return m;
  return -1;
}

int partition_for(int n, Partition *pt) {
  if (n == 512 || n == 1024 || n == 2048) {
    pt->C = kTeamChunks;
    pt->M = n / kTeamChunks;
    pt->team = 1;
    pt->levels = 7;
  } else {
    const int m = rows_per_lane_for(n);
    if (n < 4 || m < 0)
      return set_error(TP_ERR_UNSUPPORTED, "N=%d unsupported (4 <= N <= %d)", n, kWarpChunks * kMaxRowsPerLane);
    pt->C = kWarpChunks;
    pt->M = m;
    pt->team = 0;
    pt->levels = 5;
  }
  pt->nrec = 3 + 2 * pt->levels;
  return TP_OK;
}

int team_spike_rows(const tp_cn2d_op *op, int M) {
  const double b = hypot(op->k_off[0], op->k_off[1]);
  const double d0 = hypot(1.0 - op->k_diag[0], op->k_diag[1]);
  if (b == 0.0) return 1;
  const double disc = d0 * d0 - 4.0 * b * b;
  if (disc <= 0.0) return M - 1;
  const double rho = (d0 - sqrt(disc)) / (2.0 * b);
  if (!(rho > 0.0) || rho >= 0.5) return M - 1;
  int t = (int)ceil(log(kSpikeDrop) / log(rho)) + 1;
  if (t < 1) t = 1;
  if (t > M - 1) t = M - 1;
  return t;
}

// --------------------------------------------------------------------------
// Factorisation (fp64)
// --------------------------------------------------------------------------


__device__ __forceinline__ double2 load_n(const FactorParams &f, int row, int col) {
  size_t idx = (size_t)row * f.nz + col;
  if (f.dtype == TP_C128) return static_cast<const double2 *>(f.n)[idx];
  float2 v = static_cast<const float2 *>(f.n)[idx];
  return z2(v.x, v.y);
}

// coef(n) of base_simulation_space.py:356-360 (v = n, or n - 1 if is_delta)
__device__ __forceinline__ double2 coef_of(const FactorParams &f, double2 v) {
  double2 d = f.is_delta ? v : z2(v.x - 1.0, v.y);
  if (!f.exact) return z2(f.k * d.y, -f.k * d.x);            // (k/i) d
  double2 w = zadd(zscale(d, 2.0), zmul(d, d));               // n^2 - 1
  return z2(0.5 * f.k * w.y, -0.5 * f.k * w.x);               // (k/2i) w
}

// C_s at matrix row g for slice index sl (0-based; nodes sl, sl+1).
__device__ __forceinline__ double2 obj_c(const FactorParams &f, int g, int sl) {
  int r = g - f.empty_px;
  if (r < 0 || r >= f.n_obj) return z2(0.0, 0.0);
  double2 c0 = coef_of(f, load_n(f, r, sl)), c1 = coef_of(f, load_n(f, r, sl + 1));
  return zscale(zadd(c0, c1), 0.25 * f.dz);
}

__device__ __forceinline__ double2 k_sub(const FactorParams &f, int g) {  // K[g, g-1]
  return (g == f.N - 1) ? f.k_nm : f.k_off;
}
__device__ __forceinline__ double2 k_sup(const FactorParams &f, int g) {  // K[g, g+1]
  return (g == 0) ? f.k_01 : f.k_off;
}
__device__ __forceinline__ double2 p_diag(const FactorParams &f, int g, int sl) {
  if (g >= f.N) return z2(0.0, 0.0);
  double2 d = zadd((g == 0) ? f.k_d0 : ((g == f.N - 1) ? f.k_dn : f.k_diag), obj_c(f, g, sl));
  if (f.conj_t) d = zconj(d);
  return zscale(d, f.sigma);
}
__device__ __forceinline__ double2 p_sub(const FactorParams &f, int g) {  // P[g, g-1]
  if (g < 1 || g > f.N - 1) return z2(0.0, 0.0);
  double2 v = f.conj_t ? zconj(k_sup(f, g - 1)) : k_sub(f, g);
  return zscale(v, f.sigma);
}
__device__ __forceinline__ double2 p_sup(const FactorParams &f, int g) {  // P[g, g+1]
  if (g < 0 || g > f.N - 2) return z2(0.0, 0.0);
  double2 v = f.conj_t ? zconj(k_sub(f, g + 1)) : k_sup(f, g);
  return zscale(v, f.sigma);
}

// One block of C threads per slice, one thread per chunk.
__global__ void __launch_bounds__(128) cn2d_factor_kernel(const FactorParams f) {
  extern __shared__ double2 fsm[];  // [5][C]: ra, rd, rc, v_first, w_first
  const int c = threadIdx.x;
  const int sl = f.sl0 + blockIdx.x;
  const int M = f.M, C = f.C;
  cx *base = reinterpret_cast<cx *>(f.factors + (size_t)sl * f.slice_bytes);
  cx *QD = base, *LF = base + M * C, *EP = base + 2 * M * C, *V = base + 3 * M * C, *W = base + 4 * M * C,
         *LR = base + 5 * M * C;

  double2 pl[kMaxRowsPerLane], msl[kMaxRowsPerLane], fv[kMaxRowsPerLane];
  const int g0 = c * M;
  double2 p_prev = z2(1, 0), msup_prev = z2(0, 0), fvv = z2(0, 0);
  double2 me_a = z2(0, 0), me_d = z2(1, 0), me_c = z2(0, 0);
  for (int i = 0; i < M; ++i) {
    const int g = g0 + i;
    const double2 pd = p_diag(f, g, sl);
    QD[i * C + c] = to_cx(pd);
    const double2 md = z2(1.0 - pd.x, -pd.y);
    const double2 msub = zneg(p_sub(f, g));
    const double2 msup = zneg(p_sup(f, g));
    if (i < M - 1) {
      double2 l, p;
      if (i == 0) {
        l = z2(0, 0);
        p = md;
        fvv = zneg(msub);  // spike v forward part: -M[g0, g0-1] e_0
      } else {
        l = zdiv(msub, p_prev);
        p = zsub(md, zmul(l, msup_prev));
        fvv = zneg(zmul(l, fvv));
      }
      LF[i * C + c] = to_cx(l);
      EP[i * C + c] = to_cx(zdiv(z2(1.0 - p.x, -p.y), p));  // 1/p - 1
      pl[i] = p;
      msl[i] = msup;
      fv[i] = fvv;
      p_prev = p;
      msup_prev = msup;
    } else {
      me_d = md;
      me_a = msub;
      me_c = msup;
      LF[i * C + c] = czero();
      EP[i * C + c] = czero();
      V[i * C + c] = czero();
      W[i * C + c] = czero();
    }
  }
  double2 v_last, w_last, v_first, w_first;
  bool trunc_bad = false;
  const double thr = kSpikeDrop;
  if (M >= 2) {
    double2 v = zdiv(fv[M - 2], pl[M - 2]);
    double2 w = zdiv(zneg(msl[M - 2]), pl[M - 2]);
    V[(M - 2) * C + c] = to_cx(v);
    W[(M - 2) * C + c] = to_cx(w);
    if (M - 2 >= f.trunc && hypot(v.x, v.y) > thr) trunc_bad = true;
    v_last = v;
    w_last = w;
    for (int i = M - 3; i >= 0; --i) {
      v = zdiv(zsub(fv[i], zmul(msl[i], v)), pl[i]);
      w = zdiv(zneg(zmul(msl[i], w)), pl[i]);
      V[i * C + c] = to_cx(v);
      W[i * C + c] = to_cx(w);
      if (i >= f.trunc && hypot(v.x, v.y) > thr) trunc_bad = true;
      if (i < M - 1 - f.trunc && hypot(w.x, w.y) > thr) trunc_bad = true;
    }
    v_first = v;
    w_first = w;
  } else {
    v_last = z2(1, 0);
    w_last = z2(0, 0);
    v_first = z2(0, 0);
    w_first = z2(1, 0);
  }
  if (trunc_bad && f.err != nullptr) atomicOr(f.err, (int)kDevSpikeTruncation);
  // Reduced C-unknown tridiagonal system on the separators.
  fsm[3 * C + c] = v_first;
  fsm[4 * C + c] = w_first;
  __syncthreads();
  const double2 vf_n = (c < C - 1) ? fsm[3 * C + c + 1] : z2(0, 0);
  const double2 wf_n = (c < C - 1) ? fsm[4 * C + c + 1] : z2(0, 0);
  double2 ra = zmul(me_a, v_last);
  double2 rd = zadd(me_d, zadd(zmul(me_a, w_last), c < C - 1 ? zmul(me_c, vf_n) : z2(0, 0)));
  double2 rc = c < C - 1 ? zmul(me_c, wf_n) : z2(0, 0);
  LR[0 * C + c] = to_cx(me_a);
  LR[1 * C + c] = to_cx(c < C - 1 ? me_c : z2(0, 0));
  double amax = 0.0;  // largest PCR coefficient of this chunk
  for (int l = 0; l < f.levels; ++l) {
    const int s = 1 << l;
    fsm[c] = ra;
    fsm[C + c] = rd;
    fsm[2 * C + c] = rc;
    __syncthreads();
    const bool hm = c >= s, hp = c + s < C;
    const double2 ra_m = hm ? fsm[c - s] : z2(0, 0), rd_m = hm ? fsm[C + c - s] : z2(1, 0),
                  rc_m = hm ? fsm[2 * C + c - s] : z2(0, 0);
    const double2 ra_p = hp ? fsm[c + s] : z2(0, 0), rd_p = hp ? fsm[C + c + s] : z2(1, 0),
                  rc_p = hp ? fsm[2 * C + c + s] : z2(0, 0);
    __syncthreads();
    const double2 al = hm ? zneg(zdiv(ra, rd_m)) : z2(0, 0);
    const double2 ga = hp ? zneg(zdiv(rc, rd_p)) : z2(0, 0);
    const double2 nra = zmul(al, ra_m), nrc = zmul(ga, rc_p);
    rd = zadd(rd, zadd(zmul(al, rc_m), zmul(ga, ra_p)));
    ra = nra;
    rc = nrc;
    LR[rec_alpha(f.levels, l) * C + c] = to_cx(al);
    LR[rec_gamma(f.levels, l) * C + c] = to_cx(ga);
    amax = fmax(amax, fmax(hypot(al.x, al.y), hypot(ga.x, ga.y)));
  }
  // non-negative floats order like their bit patterns
  if (f.coupling != nullptr) atomicMax(f.coupling, __float_as_uint((float)fmin(amax, 3.0e38)));
  LR[rec_rde(f.levels) * C + c] = to_cx(zdiv(z2(1.0 - rd.x, -rd.y), rd));
}

// --------------------------------------------------------------------------
// March
// --------------------------------------------------------------------------




// U <- (I + P_s) U with P's boundary-row specials.
template <int M, bool ALIGNED>
__device__ __forceinline__ void cn2d_rhs(cx (&U)[M], const cx *__restrict__ QD, int lane,
                                         const MarchParams &p) {
  const cx zero = czero();
  const cx left = shfl_up2(U[M - 1], 1);
  const cx right = shfl_down2(U[0], 1);
  cx prev = (lane == 0) ? zero : left;
  const cx rlast = (lane == 31) ? zero : right;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const cx cur = U[i];
    const cx nxt = (i < M - 1) ? U[(i + 1) < M ? i + 1 : i] : rlast;
    cx r = cfma(QD[i * 32 + lane], cur, cur);
    if constexpr (ALIGNED) {
      r = cfma(p.sp.p_o, cadd(prev, nxt), r);
      if (i == 0 && lane == 0) r = cfma(p.sp.d_sup0, nxt, r);
      if ((M >= 2 ? (i == 1) : (i == 0)) && lane == (M >= 2 ? 0 : 1)) r = cfma(p.sp.d_sub1, prev, r);
      if ((M >= 2 ? (i == M - 2) : (i == 0)) && lane == (M >= 2 ? 31 : 30)) r = cfma(p.sp.d_supN2, nxt, r);
      if (i == M - 1 && lane == 31) r = cfma(p.sp.d_subN1, prev, r);
    } else {
      const int g = lane * M + i;
      const cx psub = (g == p.N - 1) ? p.sp.subN1 : ((g == 1) ? p.sp.sub1 : p.sp.p_o);
      const cx psup = (g == 0) ? p.sp.sup0 : ((g == p.N - 2) ? p.sp.supN2 : p.sp.p_o);
      r = cfma(psub, prev, r);
      r = cfma(psup, nxt, r);
      if (g >= p.N) r = zero;
    }
    prev = cur;
    U[i] = r;
  }
}

// U <- M_s^{-1} U (partitioned solve with the slice's factor set F).
template <int M, bool ALIGNED>
__device__ __forceinline__ void cn2d_solve(cx (&U)[M], const cx *__restrict__ F, int lane,
                                           const MarchParams &p) {
  const cx *LF = F + M * 32, *EP = F + 2 * M * 32, *V = F + 3 * M * 32, *W = F + 4 * M * 32,
               *LR = F + 5 * M * 32;
  if constexpr (M >= 2) {
#pragma unroll
    for (int i = 1; i <= M - 2; ++i) U[i] = cfnma(LF[i * 32 + lane], U[i - 1], U[i]);
    {
      const cx t = U[M - 2];
      U[M - 2] = cfma(t, EP[(M - 2) * 32 + lane], t);
    }
    const cx m_o = mkcx(-p.sp.p_o.x, -p.sp.p_o.y);
#pragma unroll
    for (int i = M - 3; i >= 0; --i) {
      cx msup = m_o;
      if (i == 0 && lane == 0) msup = mkcx(-p.sp.sup0.x, -p.sp.sup0.y);
      if constexpr (!ALIGNED) {
        if (lane * M + i == p.N - 2) msup = mkcx(-p.sp.supN2.x, -p.sp.supN2.y);
      }
      const cx t = cfnma(msup, U[i + 1], U[i]);
      U[i] = cfma(t, EP[i * 32 + lane], t);
    }
  }
  cx rho;
  if constexpr (M >= 2) {
    const cx y0n = shfl_down2(U[0], 1);
    rho = cfnma(LR[kRecMA * 32 + lane], U[M - 2], U[M - 1]);
    rho = cfnma(LR[kRecMC * 32 + lane], y0n, rho);
  } else {
    rho = U[0];
  }
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    const int s = 1 << l;
    const cx up = shfl_up2(rho, s), dn = shfl_down2(rho, s);
    const cx r2 = cfma(LR[(kRecAlpha + l) * 32 + lane], up, rho);
    rho = cfma(LR[(kRecGamma + l) * 32 + lane], dn, r2);
  }
  const cx x = cfma(rho, LR[kRecRDE * 32 + lane], rho);
  const cx xp = shfl_up2(x, 1);
  if constexpr (M >= 2) {
#pragma unroll
    for (int i = 0; i <= M - 2; ++i) U[i] = cfma(W[i * 32 + lane], x, cfma(V[i * 32 + lane], xp, U[i]));
  }
  U[M - 1] = x;
}

template <int M>
__device__ __forceinline__ void add_natural(cx (&U)[M], const cx *__restrict__ src, int lane, int N) {
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int g = lane * M + i;
    if (g < N) U[i] = cadd(U[i], src[g]);
  }
}

template <int M, bool ALIGNED, bool LAGGED>
__global__ void __launch_bounds__(kMarchWarps * 32, 1) cn2d_march_kernel(const MarchParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int probe = blockIdx.x * kMarchWarps + warp;
  const bool active = probe < p.P;
  const size_t sb = p.slice_bytes;
  cx *bufs = reinterpret_cast<cx *>(smem);
  cx *gacc = reinterpret_cast<cx *>(smem + 2 * sb);  // [2][M][33]
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + 2 * sb + 2 * M * 33 * sizeof(cx));
  const bool do_grad = LAGGED && (p.grad_c != nullptr);
  const size_t slice_f2 = sb / sizeof(cx);

  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_mbar_init();
  }
  if (do_grad)
    for (int e = tid; e < 2 * M * 33; e += blockDim.x) gacc[e] = czero();
  __syncthreads();

  auto slice_of = [&](int t) { return p.backward ? (p.L + 1 - t) : t; };
  if (tid == 0) {
    mbar_arrive_expect_tx(&mbar[1], (uint32_t)sb);
    bulk_g2s(bufs + slice_f2, p.factors + (size_t)(slice_of(p.t0) - 1) * sb, (uint32_t)sb, &mbar[1]);
  }

  cx U[M];
#pragma unroll
  for (int i = 0; i < M; ++i) U[i] = czero();
  if (active && p.state_in != nullptr) {
    const cx *src = p.state_in + (size_t)probe * p.Npad;
#pragma unroll
    for (int i = 0; i < M; ++i) U[i] = src[i * 32 + lane];
  } else if (active && p.probes != nullptr && p.t0 == 1) {
    add_natural<M>(U, p.probes + (size_t)probe * p.N, lane, p.N);
  }
  if (active && p.u_store != nullptr && store_index(p, p.t0 - 1) >= 0) {
    cx *dst = p.u_store + ((size_t)probe * p.store_slices + store_index(p, p.t0 - 1)) * p.Npad;
#pragma unroll
    for (int i = 0; i < M; ++i) dst[i * 32 + lane] = U[i];
  }

  uint32_t phase = 0;
  bool ok = mbar_wait_bounded(&mbar[1], 0, p.err);
  phase ^= 2u;
  if (__syncthreads_or(!ok)) {
    // Give the copy that timed out a second bounded chance to land before the
    // CTA's shared memory is released.
    if (tid == 0) mbar_wait_bounded(&mbar[1], 0, nullptr);
    __syncthreads();
    return;
  }

  for (int t = p.t0; t <= p.t1; ++t) {
    const int cb = (t - p.t0 + 1) & 1;
    const int s = slice_of(t);
    if (tid == 0 && t < p.t1) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&mbar[cb ^ 1], (uint32_t)sb);
      bulk_g2s(bufs + (cb ^ 1) * slice_f2, p.factors + (size_t)(slice_of(t + 1) - 1) * sb, (uint32_t)sb,
               &mbar[cb ^ 1]);
    }
    const cx *F = bufs + cb * slice_f2;
    if (active) {
      if constexpr (!LAGGED) cn2d_rhs<M, ALIGNED>(U, F, lane, p);
      if (p.src_shared != nullptr) add_natural<M>(U, p.src_shared + (size_t)(t - 1) * p.N, lane, p.N);
      if (p.src_probe != nullptr) {
        const int col = p.src_rev ? (p.L - t) : (t - 1);
        add_natural<M>(U, p.src_probe + ((size_t)probe * p.L + col) * p.N, lane, p.N);
      }
      if (t == 1 && p.src_exit != nullptr) add_natural<M>(U, p.src_exit + (size_t)probe * p.N, lane, p.N);
      cn2d_solve<M, ALIGNED>(U, F, lane, p);
      if (p.u_store != nullptr && store_index(p, t) >= 0) {
        cx *dst = p.u_store + ((size_t)probe * p.store_slices + store_index(p, t)) * p.Npad;
#pragma unroll
        for (int i = 0; i < M; ++i) dst[i * 32 + lane] = U[i];
      }
      if (t == p.L && p.exit_out != nullptr) {
        cx *dst = p.exit_out + (size_t)probe * p.N;
#pragma unroll
        for (int i = 0; i < M; ++i) {
          const int g = lane * M + i;
          if (g < p.N) dst[g] = U[i];
        }
      }
      if (do_grad) {
        const cx *ua = p.u_fwd + ((size_t)probe * p.ufwd_slices + (s - p.ufwd_base)) * p.Npad;
        const cx *ub = ua - p.Npad;
        cx *ga = gacc + cb * M * 33;
#pragma unroll
        for (int i = 0; i < M; ++i) {
          const cx w = cadd(ua[i * 32 + lane], ub[i * 32 + lane]);
          const cx v = cmulc(U[i], w);
          atomicAdd(&ga[i * 33 + lane].x, v.x);
          atomicAdd(&ga[i * 33 + lane].y, v.y);
        }
      }
      if constexpr (LAGGED) cn2d_rhs<M, ALIGNED>(U, F, lane, p);
    }
    bool good = true;
    if (t < p.t1) {
      good = mbar_wait_bounded(&mbar[cb ^ 1], (phase >> (cb ^ 1)) & 1u, p.err);
      phase ^= (1u << (cb ^ 1));
    }
    if (__syncthreads_or(!good)) {
      // The copy waited for is the only one in flight: drain it (bounded).
      if (tid == 0) mbar_wait_bounded(&mbar[cb ^ 1], ((phase >> (cb ^ 1)) & 1u) ^ 1u, nullptr);
      __syncthreads();
      return;
    }
    if (do_grad) {
      // gradient buffer in the chunked layout: row k*M + i at offset i*32 + k
      cx *ga = gacc + cb * M * 33;
      cx *dst = p.grad_c + (size_t)(s - 1) * p.Npad;
      for (int e = tid; e < p.Npad; e += blockDim.x) {
        const int i = e / 32, k = e % 32;
        const cx v = ga[i * 33 + k];
        red_add_cx(&dst[e], v);
        ga[i * 33 + k] = czero();
      }
    }
  }
  if (active && p.state_out != nullptr) {
    cx *dst = p.state_out + (size_t)probe * p.Npad;
#pragma unroll
    for (int i = 0; i < M; ++i) dst[i * 32 + lane] = U[i];
  }
}

// --------------------------------------------------------------------------
// Layout and gradient helpers
// --------------------------------------------------------------------------
__global__ void cn2d_unchunk_kernel(const cx *__restrict__ st, cx *__restrict__ out, int P, int N, int nz,
                                    int M, int C, int pair) {
  const size_t Npad = (size_t)C * M;
  const size_t total = (size_t)P * N * nz;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int t = (int)(idx % nz);
    const size_t pg = idx / nz;
    const int g = (int)(pg % N);
    const size_t pp = pg / N;
    const int i = g % M, k = g / M;
    const size_t off = pair ? ((size_t)(i >> 1) * C + k) * 2 + (i & 1) : (size_t)i * C + k;
    out[idx] = st[(pp * nz + t) * Npad + off];
  }
}

struct GradParams {
  int N, L, nz, n_obj, empty_px, exact, is_delta, dtype;
  int t0, nt;  // node columns [t0, t0 + nt) are mapped
  int M, C, pair, Npad;
  double k, dz;
  const cx *gc;
  const void *n;
  cx *gn;
};

__global__ void cn2d_grad_to_n_kernel(const GradParams q) {
  const size_t total = (size_t)q.n_obj * q.nt;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int t = q.t0 + (int)(e % q.nt);
    const int x = (int)(e / q.nt);
    const size_t idx = (size_t)x * q.nz + t;
    const int g = x + q.empty_px;
    const int i = g % q.M, k = g / q.M;
    const size_t off = q.pair ? ((size_t)(i >> 1) * q.C + k) * 2 + (i & 1) : (size_t)i * q.C + k;
    double2 acc = z2(0, 0);
    if (t >= 1) {
      const cx a = q.gc[(size_t)(t - 1) * q.Npad + off];
      acc = zadd(acc, z2(a.x, a.y));
    }
    if (t <= q.L - 1) {
      const cx b = q.gc[(size_t)t * q.Npad + off];
      acc = zadd(acc, z2(b.x, b.y));
    }
    // dc/dn = (dz/4) coef'(n); coef' = k/i  or (k/i) n
    double2 d = z2(0.0, -0.25 * q.dz * q.k);
    if (q.exact) {
      double2 nv;
      if (q.dtype == TP_C128) nv = static_cast<const double2 *>(q.n)[idx];
      else {
        float2 f = static_cast<const float2 *>(q.n)[idx];
        nv = z2(f.x, f.y);
      }
      if (q.is_delta) nv.x += 1.0;
      d = zmul(d, nv);
    }
    const double2 r = zmul(zconj(d), acc);
    q.gn[idx] = to_cx(r);
  }
}

// Device error word (timeouts of bounded waits); read by tp_device_status.
__device__ int g_device_error;

static SymbolCache g_device_error_addr;

int *device_error_ptr() {
  void *p = nullptr;
  if (symbol_address(&g_device_error, g_device_error_addr, &p) != TP_OK) return nullptr;
  return static_cast<int *>(p);
}

// --------------------------------------------------------------------------
// Host launchers
// --------------------------------------------------------------------------
static inline double2 hz(const double v[2]) { return make_double2(v[0], v[1]); }

static int validate_op(const tp_cn2d_op *op) {
  if (op == nullptr) return set_error(TP_ERR_INVALID, "op is NULL");
  if (op->n < 4) return set_error(TP_ERR_INVALID, "N=%d must be >= 4", op->n);
  Partition pt;
  if (partition_for(op->n, &pt) != TP_OK) return TP_ERR_UNSUPPORTED;
  if (op->nz < 2) return set_error(TP_ERR_INVALID, "nz=%d must be >= 2", op->nz);
  if (op->empty_px < 0 || op->n_obj != op->n - 2 * op->empty_px)
    return set_error(TP_ERR_INVALID, "n_obj=%d must equal N - 2*empty_px (N=%d, empty_px=%d)", op->n_obj, op->n,
                     op->empty_px);
  return TP_OK;
}

static void mode_transform(int mode, double *sigma, int *conj_t) {
  *sigma = (mode == TP_MODE_REVERSE) ? -1.0 : 1.0;
  *conj_t = (mode == TP_MODE_ADJOINT || mode == TP_MODE_ADJOINT_EXACT) ? 1 : 0;
}

// P's off-diagonal entries (host mirror of p_sub / p_sup).
static Spec make_spec(const tp_cn2d_op *op, int mode) {
  double sigma;
  int ct;
  mode_transform(mode, &sigma, &ct);
  auto f = [&](const double v[2], bool conj) {
    return mkcx((rx)(sigma * v[0]), (rx)(sigma * (conj ? -v[1] : v[1])));
  };
  Spec s;
  s.p_o = f(op->k_off, ct);
  if (!ct) {
    s.sup0 = f(op->k_01, false);   // P[0,1] = K[0,1]
    s.subN1 = f(op->k_nm, false);  // P[N-1,N-2] = K[N-1,N-2]
    s.sub1 = s.p_o;
    s.supN2 = s.p_o;
  } else {
    s.sub1 = f(op->k_01, true);    // P[1,0] = conj(K[0,1])
    s.supN2 = f(op->k_nm, true);   // P[N-2,N-1] = conj(K[N-1,N-2])
    s.sup0 = s.p_o;
    s.subN1 = s.p_o;
  }
  auto d = [&](cx a) { return mkcx(a.x - s.p_o.x, a.y - s.p_o.y); };
  s.d_sup0 = d(s.sup0);
  s.d_sub1 = d(s.sub1);
  s.d_supN2 = d(s.supN2);
  s.d_subN1 = d(s.subN1);
  return s;
}

template <int M, bool ALIGNED, bool LAGGED>
static int launch_march_t(const MarchParams &mp, cudaStream_t st) {
  auto kern = cn2d_march_kernel<M, ALIGNED, LAGGED>;
  const size_t smem = 2 * mp.slice_bytes + 2 * (size_t)M * 33 * sizeof(cx) + 2 * sizeof(uint64_t);
  TP_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (mp.P + kMarchWarps - 1) / kMarchWarps;
  kern<<<grid, kMarchWarps * 32, smem, st>>>(mp);
  return check_cuda(cudaGetLastError(), "cn2d_march_kernel launch");
}

template <int M>
static int launch_march_m(const MarchParams &mp, bool aligned, bool lagged, cudaStream_t st) {
  if (aligned) return lagged ? launch_march_t<M, true, true>(mp, st) : launch_march_t<M, true, false>(mp, st);
  return lagged ? launch_march_t<M, false, true>(mp, st) : launch_march_t<M, false, false>(mp, st);
}

static int launch_march(int M, const MarchParams &mp, bool aligned, bool lagged, cudaStream_t st) {
  switch (M) {
#define TP_CASE(m) \
  case m:          \
    return launch_march_m<m>(mp, aligned, lagged, st);
    TP_CASE(1)
    TP_CASE(2)
    TP_CASE(3)
    TP_CASE(4)
    TP_CASE(6)
    TP_CASE(8)
    TP_CASE(12)
    TP_CASE(16)
    TP_CASE(24)
    TP_CASE(32)
    TP_CASE(48)
    TP_CASE(64)
#undef TP_CASE
    default:
      return set_error(TP_ERR_UNSUPPORTED, "no kernel for %d rows per lane", M);
  }
}

}  // namespace tp

using namespace tp;

extern "C" int tp_cn2d_layout(int32_t n, int32_t *chunks, int32_t *rows_per_chunk, int32_t *npad) {
  Partition pt;
  int rc = partition_for(n, &pt);
  if (rc) return rc;
  if (chunks) *chunks = pt.C;
  if (rows_per_chunk) *rows_per_chunk = pt.M;
  if (npad) *npad = pt.C * pt.M;
  return TP_OK;
}

extern "C" size_t tp_cn2d_factor_bytes(int32_t n, int32_t nz) {
  Partition pt;
  if (nz < 2 || partition_for(n, &pt) != TP_OK) return 0;
  return slice_bytes(pt) * (size_t)(nz - 1) + kFactorTailBytes;
}

// Factorise slices [s_begin, s_end] (1-based, inclusive) of the factor set.
static int factor_slices(const tp_cn2d_op *op, const void *n_field, int32_t n_dtype, int32_t mode, void *factors,
                         size_t factors_bytes, int s_begin, int s_end, tp_stream_t stream) {
  int rc = validate_op(op);
  if (rc) return rc;
  if (n_field == nullptr || factors == nullptr) return set_error(TP_ERR_INVALID, "n_field/factors is NULL");
  if (n_dtype != TP_C128 && n_dtype != TP_C64) return set_error(TP_ERR_INVALID, "bad n_dtype %d", n_dtype);
  if (mode < TP_MODE_FORWARD || mode > TP_MODE_ADJOINT_EXACT) return set_error(TP_ERR_INVALID, "bad mode %d", mode);
  const size_t need = tp_cn2d_factor_bytes(op->n, op->nz);
  if (factors_bytes < need)
    return set_error(TP_ERR_WORKSPACE, "factor workspace %zu B < required %zu B", factors_bytes, need);
  if ((reinterpret_cast<uintptr_t>(factors) & 255u) != 0)
    return set_error(TP_ERR_INVALID, "factor workspace must be 256-byte aligned");
  Partition pt;
  rc = partition_for(op->n, &pt);
  if (rc) return rc;
  int *err = device_error_ptr();
  if (err == nullptr) return set_error(TP_ERR_CUDA, "cannot resolve the device error word");
  FactorParams f{};
  f.N = op->n;
  f.L = op->nz - 1;
  f.C = pt.C;
  f.M = pt.M;
  f.levels = pt.levels;
  f.nrec = pt.nrec;
  f.trunc = pt.team ? team_spike_rows(op, pt.M) : pt.M - 1;
  f.nz = op->nz;
  f.n_obj = op->n_obj;
  f.empty_px = op->empty_px;
  f.exact = op->exact_ref_coeff;
  f.is_delta = op->field_is_delta;
  f.dtype = n_dtype;
  mode_transform(mode, &f.sigma, &f.conj_t);
  f.k = op->k;
  f.dz = op->dz;
  f.k_off = hz(op->k_off);
  f.k_diag = hz(op->k_diag);
  f.k_d0 = hz(op->k_d0);
  f.k_dn = hz(op->k_dn);
  f.k_01 = hz(op->k_01);
  f.k_nm = hz(op->k_nm);
  f.n = n_field;
  f.factors = static_cast<char *>(factors);
  f.slice_bytes = slice_bytes(pt);
  f.coupling = reinterpret_cast<unsigned *>(f.factors + (size_t)f.L * f.slice_bytes);
  f.err = err;
  if (s_begin < 1 || s_end > f.L || s_begin > s_end)
    return set_error(TP_ERR_INVALID, "slice range [%d, %d] outside [1, %d]", s_begin, s_end, f.L);
  f.sl0 = s_begin - 1;
  // the PCR coupling bound is a running maximum over the slices factorised
  // since the last reset, which the range starting at slice 1 performs
  if (s_begin == 1)
    TP_CHECK_CUDA(cudaMemsetAsync(f.coupling, 0, sizeof(unsigned), reinterpret_cast<cudaStream_t>(stream)));
  const size_t smem = 5 * (size_t)pt.C * sizeof(double2);
  cn2d_factor_kernel<<<s_end - s_begin + 1, pt.C, smem, reinterpret_cast<cudaStream_t>(stream)>>>(f);
  return check_cuda(cudaGetLastError(), "cn2d_factor_kernel launch");
}

extern "C" int tp_cn2d_factor(const tp_cn2d_op *op, const void *n_field, int32_t n_dtype, int32_t mode,
                              void *factors, size_t factors_bytes, tp_stream_t stream) {
  if (op == nullptr) return set_error(TP_ERR_INVALID, "op is NULL");
  return factor_slices(op, n_field, n_dtype, mode, factors, factors_bytes, 1, op->nz - 1, stream);
}

extern "C" int tp_cn2d_factor_range(const tp_cn2d_op *op, const void *n_field, int32_t n_dtype, int32_t mode,
                                    void *factors, size_t factors_bytes, int32_t slice_begin, int32_t slice_end,
                                    tp_stream_t stream) {
  if (op == nullptr) return set_error(TP_ERR_INVALID, "op is NULL");
  return factor_slices(op, n_field, n_dtype, mode, factors, factors_bytes, slice_begin, slice_end, stream);
}

extern "C" int tp_copy_columns(void *dst, const void *src, int64_t rows, int64_t row_bytes, int64_t byte_begin,
                               int64_t byte_count, tp_stream_t stream) {
  if (dst == nullptr || src == nullptr || rows < 1 || row_bytes < 1 || byte_begin < 0 || byte_count < 1 ||
      byte_begin + byte_count > row_bytes)
    return set_error(TP_ERR_INVALID, "bad tp_copy_columns arguments");
  char *d = static_cast<char *>(dst) + byte_begin;
  const char *s = static_cast<const char *>(src) + byte_begin;
  return check_cuda(cudaMemcpy2DAsync(d, (size_t)row_bytes, s, (size_t)row_bytes, (size_t)byte_count, (size_t)rows,
                                      cudaMemcpyDefault, reinterpret_cast<cudaStream_t>(stream)),
                    "tp_copy_columns");
}

extern "C" int tp_cn2d_march(const tp_cn2d_op *op, const void *factors, const tp_cn2d_march_args *a,
                             tp_stream_t stream) {
  int rc = validate_op(op);
  if (rc) return rc;
  if (a == nullptr || factors == nullptr) return set_error(TP_ERR_INVALID, "args/factors is NULL");
  if (a->num_probes < 1) return set_error(TP_ERR_INVALID, "num_probes=%d", a->num_probes);
  if (a->mode < TP_MODE_FORWARD || a->mode > TP_MODE_ADJOINT_EXACT)
    return set_error(TP_ERR_INVALID, "bad mode %d", a->mode);
  if ((reinterpret_cast<uintptr_t>(factors) & 255u) != 0)
    return set_error(TP_ERR_INVALID, "factor workspace must be 256-byte aligned");
  const bool lagged = a->mode == TP_MODE_ADJOINT_EXACT;
  if ((a->grad_c != nullptr) != (a->u_fwd != nullptr))
    return set_error(TP_ERR_INVALID, "grad_c and u_fwd must be given together");
  if (a->grad_c != nullptr && !lagged)
    return set_error(TP_ERR_INVALID, "the fused gradient needs mode TP_MODE_ADJOINT_EXACT");
  Partition pt;
  rc = partition_for(op->n, &pt);
  if (rc) return rc;
  int *err = device_error_ptr();
  if (err == nullptr) return set_error(TP_ERR_CUDA, "cannot resolve the device error word");
  MarchParams mp{};
  mp.N = op->n;
  mp.L = op->nz - 1;
  mp.nz = op->nz;
  mp.P = a->num_probes;
  mp.Npad = pt.C * pt.M;
  mp.backward = (a->mode != TP_MODE_FORWARD) ? 1 : 0;
  mp.flip_out = (a->mode == TP_MODE_ADJOINT) ? 1 : 0;
  mp.src_rev = (a->mode == TP_MODE_ADJOINT || a->mode == TP_MODE_ADJOINT_EXACT) ? 1 : 0;
  mp.trunc = pt.team ? team_spike_rows(op, pt.M) : pt.M - 1;
  mp.slice_bytes = slice_bytes(pt);
  mp.factors = static_cast<const char *>(factors);
  mp.sp = make_spec(op, a->mode);
  mp.probes = static_cast<const cx *>(a->probes);
  mp.src_shared = static_cast<const cx *>(a->src_shared);
  mp.src_probe = static_cast<const cx *>(a->src_probe);
  mp.src_exit = static_cast<const cx *>(a->src_exit);
  mp.u_store = static_cast<cx *>(a->u_store);
  mp.exit_out = static_cast<cx *>(a->exit_out);
  mp.u_fwd = static_cast<const cx *>(a->u_fwd);
  mp.grad_c = static_cast<cx *>(a->grad_c);
  mp.coupling = reinterpret_cast<const unsigned *>(mp.factors + (size_t)mp.L * mp.slice_bytes);
  mp.err = err;
  mp.t0 = a->t_begin > 0 ? a->t_begin : 1;
  mp.t1 = a->t_end > 0 ? a->t_end : mp.L;
  if (mp.t0 > mp.t1 || mp.t1 > mp.L) return set_error(TP_ERR_INVALID, "bad step range [%d, %d] (L=%d)", mp.t0, mp.t1, mp.L);
  if (mp.flip_out && (mp.t0 != 1 || mp.t1 != mp.L) && a->u_store != nullptr)
    return set_error(TP_ERR_INVALID, "the flipped ADJOINT store needs the full step range");
  mp.state_in = static_cast<const cx *>(a->state_in);
  mp.state_out = static_cast<cx *>(a->state_out);
  mp.store_slices = a->store_slices > 0 ? a->store_slices : op->nz;
  mp.store_every = a->store_every;
  mp.store_base = a->store_base;
  mp.ufwd_slices = a->ufwd_slices > 0 ? a->ufwd_slices : op->nz;
  mp.ufwd_base = a->ufwd_base;
  mp.store_sums = a->store_sums;
  if (a->store_sums != 0) {
    if (a->store_sums != 1) return set_error(TP_ERR_INVALID, "store_sums=%d (0 or 1)", a->store_sums);
    if (a->mode != TP_MODE_FORWARD && a->mode != TP_MODE_ADJOINT_EXACT)
      return set_error(TP_ERR_INVALID, "store_sums needs mode FORWARD or ADJOINT_EXACT");
    if (a->mode == TP_MODE_FORWARD && a->store_every > 1)
      return set_error(TP_ERR_INVALID, "store_sums cannot keep checkpoints (store_every=%d)", a->store_every);
    if (!pt.team)
      return set_error(TP_ERR_UNSUPPORTED, "store_sums needs the team path (N in {512, 1024, 2048}), N=%d", op->n);
  }
  if (pt.team) {
    if (op->k_off[0] != 0.0 || op->k_01[0] != 0.0 || op->k_nm[0] != 0.0)
      return set_error(TP_ERR_UNSUPPORTED,
                       "N=%d uses the team kernels, which need purely imaginary off-diagonals of K "
                       "(mu = i dz/(4 k dx^2))", op->n);
    // 16-byte row-pair vectors and whole-slice bulk copies (stores, loads, reductions)
    const void *vec[] = {a->u_store, a->u_fwd, a->grad_c, a->state_in, a->state_out};
    for (const void *v : vec)
      if (v != nullptr && (reinterpret_cast<uintptr_t>(v) & 15u) != 0)
        return set_error(TP_ERR_INVALID, "the team path needs 16-byte aligned u_store, u_fwd, grad_c, state_in, state_out");
    return launch_team_march(pt, mp, lagged, reinterpret_cast<cudaStream_t>(stream));
  }
  return launch_march(pt.M, mp, op->n == pt.C * pt.M, lagged, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int tp_cn2d_unchunk(const tp_cn2d_op *op, int32_t num_probes, const void *u_store, void *u_out,
                               tp_stream_t stream) {
  int rc = validate_op(op);
  if (rc) return rc;
  if (u_store == nullptr || u_out == nullptr || num_probes < 1) return set_error(TP_ERR_INVALID, "bad unchunk args");
  Partition pt;
  rc = partition_for(op->n, &pt);
  if (rc) return rc;
  cn2d_unchunk_kernel<<<1184, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      static_cast<const cx *>(u_store), static_cast<cx *>(u_out), num_probes, op->n, op->nz, pt.M, pt.C, pt.team);
  return check_cuda(cudaGetLastError(), "cn2d_unchunk_kernel launch");
}

static int grad_to_n_nodes(const tp_cn2d_op *op, const void *grad_c, const void *n_field, int32_t n_dtype,
                           void *grad_n, int node_begin, int node_end, tp_stream_t stream) {
  int rc = validate_op(op);
  if (rc) return rc;
  if (grad_c == nullptr || grad_n == nullptr) return set_error(TP_ERR_INVALID, "grad_c/grad_n is NULL");
  if (op->exact_ref_coeff && n_field == nullptr) return set_error(TP_ERR_INVALID, "exact_ref_coeff needs n_field");
  Partition pt;
  rc = partition_for(op->n, &pt);
  if (rc) return rc;
  GradParams q{};
  q.M = pt.M;
  q.C = pt.C;
  q.pair = pt.team;
  q.Npad = pt.C * pt.M;
  q.N = op->n;
  q.L = op->nz - 1;
  q.nz = op->nz;
  q.n_obj = op->n_obj;
  q.empty_px = op->empty_px;
  q.exact = op->exact_ref_coeff;
  q.is_delta = op->field_is_delta;
  q.dtype = n_dtype;
  q.k = op->k;
  q.dz = op->dz;
  q.gc = static_cast<const cx *>(grad_c);
  q.n = n_field;
  q.gn = static_cast<cx *>(grad_n);
  if (node_begin < 0 || node_end >= op->nz || node_begin > node_end)
    return set_error(TP_ERR_INVALID, "node range [%d, %d] outside [0, %d]", node_begin, node_end, op->nz - 1);
  q.t0 = node_begin;
  q.nt = node_end - node_begin + 1;
  cn2d_grad_to_n_kernel<<<592, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(q);
  return check_cuda(cudaGetLastError(), "cn2d_grad_to_n_kernel launch");
}

extern "C" int tp_cn2d_grad_to_n(const tp_cn2d_op *op, const void *grad_c, const void *n_field, int32_t n_dtype,
                                 void *grad_n, tp_stream_t stream) {
  if (op == nullptr) return set_error(TP_ERR_INVALID, "op is NULL");
  return grad_to_n_nodes(op, grad_c, n_field, n_dtype, grad_n, 0, op->nz - 1, stream);
}

extern "C" int tp_cn2d_grad_to_n_range(const tp_cn2d_op *op, const void *grad_c, const void *n_field,
                                       int32_t n_dtype, void *grad_n, int32_t node_begin, int32_t node_end,
                                       tp_stream_t stream) {
  if (op == nullptr) return set_error(TP_ERR_INVALID, "op is NULL");
  return grad_to_n_nodes(op, grad_c, n_field, n_dtype, grad_n, node_begin, node_end, stream);
}

extern "C" int tp_device_status(tp_stream_t stream, int32_t *code) {
  int *err = device_error_ptr();
  if (err == nullptr) return set_error(TP_ERR_CUDA, "cannot resolve the device error word");
  int h = 0;
  TP_CHECK_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, reinterpret_cast<cudaStream_t>(stream)));
  TP_CHECK_CUDA(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)));
  if (code) *code = h;
  if (h != 0) {
    const int zero = 0;
    TP_CHECK_CUDA(cudaMemcpy(err, &zero, sizeof(int), cudaMemcpyHostToDevice));
    if (h & kDevSpikeTruncation)
      return set_error(TP_ERR_UNSUPPORTED,
                       "the factorised matrices have slowly decaying spikes beyond the kept rows (code %d): "
                       "results of the team path are inaccurate for this operator", h);
    return set_error(TP_ERR_TIMEOUT, "a device-side bounded wait timed out (code %d)", h);
  }
  return TP_OK;
}
