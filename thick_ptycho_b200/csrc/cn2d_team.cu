// Team path of the 2D Crank–Nicolson march: N in {512, 1024, 2048}.
//
// A team of 4 warps (128 threads) marches a group of Q probes; a CTA holds TM
// teams that share the staged factor slice (so an SM runs 4*TM warps while
// holding one copy of the factors) and synchronise among themselves with
// named barriers.  Thread c of a team owns chunk c (M = N/128 consecutive
// rows) of every probe of its group, so
// each factor value read from shared memory serves Q probes and the Q
// recurrences of a thread are independent (instruction-level parallelism
// where the warp path has one dependent chain).  The 128 separators of each
// probe form a tridiagonal system solved by 7 levels of parallel cyclic
// reduction through shared memory.  Only the first and last T rows of the
// spike vectors are staged (they decay geometrically; T is chosen from the
// operator and verified when factorising).
//
// Exact-adjoint gradient: each probe's contribution lambda*conj(u_s+u_{s-1})
// is added to the chunked gradient buffer.  In the Cayley-form kernel the
// forward half sums arrive by bulk loads into shared memory, each team
// writes its contributions over them, and the CTA sums its teams before one
// 16-byte vector reduction per row pair (a quarter of the global reductions
// of one per probe); the two-slice kernel adds each probe's contribution
// with its own vector reductions.
#include "cn2d_internal.cuh"
#include <stdio.h>
#include <stdlib.h>

#include "tp_errors.h"

namespace tp {

constexpr int kTeamThreads = kTeamChunks;  // threads per team: one per chunk
constexpr int kTeamLevels = 7;

// Barrier among the 128 threads of one team (ids 1..TM; 0 is __syncthreads).
__device__ __forceinline__ void team_sync(int team) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + team), "r"(kTeamThreads) : "memory");
}
// fused a*b + c in the march's real type
__device__ __forceinline__ float rfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return fma(a, b, c); }

// b * i * z for real b (the off-diagonal of P is purely imaginary: i*dz/(4k dx^2)).
__device__ __forceinline__ cx imul_acc(rx b, cx z, cx acc) {
  return mkcx(rfma(-b, z.y, acc.x), rfma(b, z.x, acc.y));
}

// Chunked team layout: rows are stored in pairs, so thread c's rows 2j, 2j+1
// are one 16-byte vector at offset (j*C + c)*2 of a slice.
__device__ __forceinline__ void store_pairs(cx *dst, const cx *U, int M, int c) {
#pragma unroll 8
  for (int j = 0; j < M / 2; ++j)
    reinterpret_cast<cx2 *>(dst)[j * kTeamChunks + c] = mkcx2(U[2 * j], U[2 * j + 1]);
}

// Load thread c's M rows of one stored slice (row pairs).
template <int M>
__device__ __forceinline__ void load_pairs(cx (&dst)[M], const cx *slice, int c) {
  const cx2 *src = reinterpret_cast<const cx2 *>(slice) + c;
#pragma unroll
  for (int j = 0; j < M / 2; ++j) {
    const cx2 v = src[j * kTeamChunks];
    dst[2 * j] = mkcx(v.x, v.y);
    dst[2 * j + 1] = mkcx(v.z, v.w);
  }
}

// Shared-memory bytes of one staged factor slice.  The Cayley-form kernels
// never apply the right-hand-side stencil, so they stage LF|EP without the
// QD rows (qd = false).
__host__ __device__ inline size_t team_slice_smem(int M, int T, bool qd = true) {
  return (size_t)((qd ? 3 : 2) * M + 2 * T + 3 + 2 * kTeamLevels) * kTeamChunks * sizeof(cx);
}

// Exchange rows per probe: Y0, R0, R1, XS, and for the stencil (qd) XL, XF.
__host__ __device__ constexpr int team_xrows(bool qd) { return qd ? 6 : 4; }

// Shared memory of a team kernel: the factor double buffer, the exchange
// rows, for the staged kernels (stg; never the two-slice exact adjoint, qd)
// one staging slice per probe, and the mbarriers (factor double buffer, one
// per team).
size_t team_smem_bytes(const Partition &pt, int trunc, int Q, int TM, bool qd, bool stg) {
  const size_t slice = (size_t)pt.M * kTeamChunks * sizeof(cx);
  const size_t stage = (qd || !stg) ? 0 : (size_t)TM * Q * slice;
  return 2 * team_slice_smem(pt.M, trunc, qd) + (size_t)team_xrows(qd) * TM * Q * kTeamChunks * sizeof(cx) +
         stage + (2 + (size_t)TM) * sizeof(uint64_t);
}

// Issue the bulk copies of one slice's factor set ([QD|]LF|EP, V head, W tail, records).
__device__ __forceinline__ void team_issue(cx *dst, const char *slice, int M, int T, uint64_t *bar, bool qd) {
  constexpr int C = kTeamChunks;
  const uint32_t row = C * sizeof(cx);
  const uint32_t b_main = (qd ? 3 : 2) * M * row, b_sp = T * row, b_rec = (3 + 2 * kTeamLevels) * row;
  mbar_arrive_expect_tx(bar, b_main + 2 * b_sp + b_rec);
  char *d = reinterpret_cast<char *>(dst);
  bulk_g2s(d, slice + (qd ? 0 : (size_t)M * row), b_main, bar);
  bulk_g2s(d + b_main, slice + (size_t)3 * M * row, b_sp, bar);
  bulk_g2s(d + b_main + b_sp, slice + (size_t)(4 * M + (M - 1 - T)) * row, b_sp, bar);
  bulk_g2s(d + b_main + 2 * b_sp, slice + (size_t)5 * M * row, b_rec, bar);
}

// U <- (I + P_s) U for the Q probes (boundary rows: chunk 0 rows 0,1 and
// chunk C-1 rows M-2, M-1).
template <int M, int Q>
__device__ __forceinline__ void team_rhs(cx (&U)[Q][M], const cx *__restrict__ QD, cx *XL, cx *XF,
                                         int c, int team, const Spec &sp) {
  constexpr int C = kTeamChunks;
  const cx zero = czero();
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    XL[q * C + c] = U[q][M - 1];
    XF[q * C + c] = U[q][0];
  }
  team_sync(team);
  cx prev[Q], right[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    prev[q] = (c > 0) ? XL[q * C + c - 1] : zero;
    right[q] = (c < C - 1) ? XF[q * C + c + 1] : zero;
  }
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const cx qd = QD[i * C + c];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const cx cur = U[q][i];
      const cx nxt = (i < M - 1) ? U[q][(i + 1) < M ? i + 1 : i] : right[q];
      cx r = cfma(qd, cur, cur);
      r = imul_acc(sp.p_o.y, cadd(prev[q], nxt), r);
      if (i == 0 && c == 0) r = cfma(sp.d_sup0, nxt, r);
      if (i == 1 && c == 0) r = cfma(sp.d_sub1, prev[q], r);
      if (i == M - 2 && c == C - 1) r = cfma(sp.d_supN2, nxt, r);
      if (i == M - 1 && c == C - 1) r = cfma(sp.d_subN1, prev[q], r);
      prev[q] = cur;
      U[q][i] = r;
    }
  }
}

// U <- M_s^{-1} U with the staged factor slice F (T spike rows staged: a
// compile-time count, so the spike corrections touch only those rows; QD:
// the slice starts with the QD rows; WAITR: the caller stages bulk stores).
template <int M, int Q, int T, bool QD, bool WAITR>
__device__ __forceinline__ void team_solve(cx (&U)[Q][M], const cx *__restrict__ F, cx *Y0,
                                           cx *R0, cx *R1, cx *XS, int c, int team, const Spec &sp,
                                           bool pcr) {
  constexpr int C = kTeamChunks;
  const cx zero = czero();
  const cx *LF = F + (QD ? M * C : 0), *EP = LF + M * C, *VH = EP + M * C, *WT = VH + T * C, *LR = WT + T * C;
#pragma unroll
  for (int i = 1; i <= M - 2; ++i) {
    const cx lf = LF[i * C + c];
#pragma unroll
    for (int q = 0; q < Q; ++q) U[q][i] = cfnma(lf, U[q][i - 1], U[q][i]);
  }
  {
    const cx ep = EP[(M - 2) * C + c];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const cx t = U[q][M - 2];
      U[q][M - 2] = cfma(t, ep, t);
    }
  }
#pragma unroll
  for (int i = M - 3; i >= 0; --i) {
    const cx ep = EP[i * C + c];
    // t = U[i] - M[i,i+1] U[i+1] = U[i] + P[i,i+1] U[i+1]; P[0,1] is the only special entry here.
    const rx bsup = (i == 0 && c == 0) ? sp.sup0.y : sp.p_o.y;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const cx t = imul_acc(bsup, U[q][i + 1], U[q][i]);
      U[q][i] = cfma(t, ep, t);
    }
  }
  // The staging slice that is written after this solve may still be read by
  // the bulk store issued from it in the previous step: its issuing thread
  // waits for that read before the exchange barrier below, which every
  // thread of the team passes before it writes the staging slice again (the
  // wait is executed by all threads, without a branch; it returns at once
  // in threads with no bulk copies in flight).
  if constexpr (WAITR) bulk_wait_read();
  cx x[Q], xp[Q];
  constexpr int kRd = 2 + 2 * kTeamLevels;  // record row of the reduced diagonal
  if (!pcr) {
    // The factorisation found every separator coupling below kPcrSkipBound,
    // so the reduced system is diagonal to far beneath fp32 round-off:
    // x_c = rho_c / rd_c with rho_c = z_c - mc_c y0_{c+1}.  One exchange
    // publishes each chunk's first row y0 and partial residual z; thread c
    // then forms its own separator and recomputes its left neighbour's from
    // the neighbour's records (the same operations, so the same bits), which
    // saves the second exchange and its barrier.
    const cx ma = LR[0 * C + c], mc = LR[1 * C + c];
    cx zc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      zc[q] = cfnma(ma, U[q][M - 2], U[q][M - 1]);
      Y0[q * C + c] = U[q][0];
      R0[q * C + c] = zc[q];
    }
    team_sync(team);
    const cx rde = LR[kRd * C + c];
    const cx mcl = c > 0 ? LR[1 * C + c - 1] : zero, rdel = c > 0 ? LR[kRd * C + c - 1] : zero;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const cx y0n = (c < C - 1) ? Y0[q * C + c + 1] : zero;
      const cx r = cfnma(mc, y0n, zc[q]);
      x[q] = cfma(r, rde, r);
      if (c > 0) {
        const cx rl = cfnma(mcl, U[q][0], R0[q * C + c - 1]);
        xp[q] = cfma(rl, rdel, rl);
      } else {
        xp[q] = zero;
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) Y0[q * C + c] = U[q][0];
    team_sync(team);
    cx rho[Q];
    {
      const cx ma = LR[0 * C + c], mc = LR[1 * C + c];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const cx y0n = (c < C - 1) ? Y0[q * C + c + 1] : zero;
        rho[q] = cfnma(mc, y0n, cfnma(ma, U[q][M - 2], U[q][M - 1]));
      }
    }
    // PCR on the separators (7 levels through shared memory)
#pragma unroll
    for (int l = 0; l < kTeamLevels; ++l) {
      const int s = 1 << l;
      cx *Rb = (l & 1) ? R1 : R0;
#pragma unroll
      for (int q = 0; q < Q; ++q) Rb[q * C + c] = rho[q];
      team_sync(team);
      const cx al = LR[(2 + l) * C + c], ga = LR[(2 + kTeamLevels + l) * C + c];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const cx up = (c >= s) ? Rb[q * C + c - s] : zero;
        const cx dn = (c + s < C) ? Rb[q * C + c + s] : zero;
        rho[q] = cfma(ga, dn, cfma(al, up, rho[q]));
      }
    }
    const cx rde = LR[kRd * C + c];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      x[q] = cfma(rho[q], rde, rho[q]);
      XS[q * C + c] = x[q];
    }
    team_sync(team);
#pragma unroll
    for (int q = 0; q < Q; ++q) xp[q] = (c > 0) ? XS[q * C + c - 1] : zero;
  }
  constexpr int wlo = M - 1 - T;
#pragma unroll
  for (int i = 0; i <= M - 2; ++i) {
    if (i < T) {
      const cx v = VH[i * C + c];
#pragma unroll
      for (int q = 0; q < Q; ++q) U[q][i] = cfma(v, xp[q], U[q][i]);
    }
    if (i >= wlo) {
      const cx w = WT[(i - wlo) * C + c];
#pragma unroll
      for (int q = 0; q < Q; ++q) U[q][i] = cfma(w, x[q], U[q][i]);
    }
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) U[q][M - 1] = x[q];
}

// Forward store through the staging slices: thread c writes its row pairs of
// the Q probes (conflict-free 16-byte shared stores), and after the team
// barrier thread 0 copies each probe's slice to store slice sidx with one
// bulk store.  The staging slices are written again only after the next
// solve's exchange barrier, before which thread 0 waits for the copy's read.
template <int M, int Q>
__device__ __forceinline__ void store_staged(const cx (&U)[Q][M], cx2 *stg, const MarchParams &p, int p0,
                                             int sidx, int c, int team) {
  constexpr int C = kTeamChunks;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (p0 + q >= p.P) continue;
#pragma unroll
    for (int j = 0; j < M / 2; ++j)
      stg[(q * (M / 2) + j) * C + c] =
          mkcx2(U[q][2 * j], U[q][2 * j + 1]);
  }
  fence_proxy_async_smem();
  team_sync(team);
  if (c == 0) {
#pragma unroll
    for (int q = 0; q < Q; ++q)
      if (p0 + q < p.P)
        bulk_s2g(p.u_store + ((size_t)(p0 + q) * p.store_slices + sidx) * p.Npad, stg + (size_t)q * (M / 2) * C,
                 M * C * sizeof(cx));
    bulk_commit();
  }
}

// Exact-adjoint gradient of one team and step: the team's Q staging slices
// hold this step's forward half pair sums (u_s + u_{s-1})/2 of its probes,
// bulk-loaded ahead of the solve; each row pair's contributions
// lambda conj(half sum), summed over the Q probes in registers (zero for
// padded probes), replace the first slice in place, so that after the
// end-of-step barrier the CTA's teams can be summed (and doubled: the pair
// sum is twice the half sum) before the gradient row is updated
// (grad_sum_flush).
template <int M, int Q>
__device__ __forceinline__ void grad_contrib(const cx (&U)[Q][M], cx2 *stg, int nvalid, int c) {
  constexpr int C = kTeamChunks;
#pragma unroll
  for (int j = 0; j < M / 2; ++j) {
    cx2 w = mkcx2(czero(), czero());
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (q >= nvalid) continue;
      const cx2 v = stg[(q * (M / 2) + j) * C + c];
      const cx a = cmulc(U[q][2 * j], mkcx(v.x, v.y));
      const cx b = cmulc(U[q][2 * j + 1], mkcx(v.z, v.w));
      w = mkcx2(mkcx(w.x + a.x, w.y + a.y), mkcx(w.z + b.x, w.w + b.y));
    }
    stg[j * C + c] = w;
  }
}

// Sum the TM teams' contribution slices (each team's first staging slice),
// double the sum (half sums to pair sums) and add it to gradient row `row`
// (chunked row pairs) with 16-byte vector reductions: one reduction per row
// pair and CTA instead of one per probe.  Every thread of the CTA takes its
// share of the row pairs; the slices are complete after a CTA barrier and
// free for the next bulk loads after the next one.
template <int M, int Q, int TM>
__device__ __forceinline__ void grad_sum_flush(const cx2 *stage, cx *row, int tid) {
  constexpr int E = (M / 2) * kTeamChunks, NT = TM * kTeamThreads;
  cx2 *g = reinterpret_cast<cx2 *>(row);
#pragma unroll
  for (int e = tid; e < E; e += NT) {
    cx2 v = stage[e];
#pragma unroll
    for (int m = 1; m < TM; ++m) {
      const cx2 w = stage[m * Q * E + e];  // team m's first slice
      v = mkcx2(mkcx(v.x + w.x, v.y + w.y), mkcx(v.z + w.z, v.w + w.w));
    }
    red_add_cx2(g + e, mkcx2(mkcx(2 * v.x, 2 * v.y), mkcx(2 * v.z, 2 * v.w)));
  }
  // the slices are next written by bulk loads (async proxy)
  fence_proxy_async_smem();
}

// TS: spike rows staged per slice (>= the rows the factorisation found
// significant).  LAGGED: exact-adjoint order (solve, gradient, then the
// right-hand side of the same slice).  SUMS (LAGGED only): that step in Cayley form, with u_fwd
// (when given) holding the half pair sums (u_s + u_{s-1})/2 written by a
// forward march with store_sums, so one forward slice is read per step and
// the registers of the second serve the Cayley step.
//
// STG: whole-slice global traffic goes through one staging slice per probe
// in shared memory (never in the two-slice exact adjoint; the host selects it
// where it fits beside the factor double buffer, i.e. all but the 15-spike-row
// factor sets, which keep direct per-thread stores and loads): the forward
// stores its slices with bulk stores, and the exact adjoint's gradient has
// its half-sum slice bulk-loaded at the start of the step, ahead of the
// solve (no registers hold data in flight), and its contribution summed
// over the CTA's teams before it reaches global memory.
template <int M, int Q, int TM, bool LAGGED, bool SUMS, int TS, bool STG>
__global__ void __launch_bounds__(kTeamThreads *TM, 1) cn2d_team_kernel(const MarchParams p) {
  static_assert(LAGGED || !SUMS, "SUMS selects the exact-adjoint Cayley step");
  static_assert(!LAGGED || Q == 1 || (SUMS && STG), "exact adjoint: several probes per thread only staged");
  constexpr bool QD = LAGGED && !SUMS;     // only the two-slice exact adjoint applies the stencil
  constexpr bool STAGE = !QD && STG;              // staging slices in shared memory
  constexpr bool GSTAGE = LAGGED && SUMS && STG;  // the gradient goes through them
  constexpr int C = kTeamChunks;
  constexpr uint32_t NB = M * C * sizeof(cx);  // bytes of one probe's slice
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x;
  const int team = tid / kTeamThreads;
  const int c = tid % kTeamThreads;
  constexpr int T = TS;  // the host sets p.trunc = TS
  const size_t ss = p.smem_slice_bytes;
  cx *bufs = reinterpret_cast<cx *>(smem);
  constexpr int XR = team_xrows(QD);
  cx *xb = reinterpret_cast<cx *>(smem + 2 * ss) + (size_t)team * XR * Q * C;
  cx *XL = QD ? xb : nullptr, *XF = QD ? xb + Q * C : nullptr;  // stencil rows (QD only)
  cx *Y0 = xb + (QD ? 2 : 0) * Q * C, *R0 = Y0 + Q * C, *R1 = R0 + Q * C, *XS = R1 + Q * C;
  cx2 *stage = reinterpret_cast<cx2 *>(smem + 2 * ss + (size_t)TM * XR * Q * C * sizeof(cx));
  cx2 *stg = stage + (size_t)team * Q * (M / 2) * C;  // this team's Q staging slices
  uint64_t *mbar = reinterpret_cast<uint64_t *>(reinterpret_cast<unsigned char *>(stage) +
                                                (STAGE ? (size_t)TM * Q * NB : 0));
  uint64_t *gbar = mbar + 2;  // one per team: its half-sum slice
  const bool do_grad = LAGGED && (p.grad_c != nullptr);
  const size_t ssf = ss / sizeof(cx);
  const int p0 = (blockIdx.x * TM + team) * Q;
  const bool pcr = p.coupling == nullptr || __uint_as_float(__ldg(p.coupling)) >= kPcrSkipBound;

  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
#pragma unroll
    for (int m = 0; m < TM; ++m) mbar_init(&gbar[m], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto slice_of = [&](int t) { return p.backward ? (p.L + 1 - t) : t; };
  if (tid == 0)
    team_issue(bufs + ssf, p.factors + (size_t)(slice_of(p.t0) - 1) * p.slice_bytes, M, T, &mbar[1], QD);

  cx U[Q][M];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
#pragma unroll
    for (int i = 0; i < M; ++i) U[q][i] = czero();
    if (p0 + q >= p.P) continue;
    if (p.state_in != nullptr) {
      const cx2 *src = reinterpret_cast<const cx2 *>(p.state_in + (size_t)(p0 + q) * p.Npad) + c;
#pragma unroll
      for (int j = 0; j < M / 2; ++j) {
        const cx2 v = src[j * C];
        U[q][2 * j] = mkcx(v.x, v.y);
        U[q][2 * j + 1] = mkcx(v.z, v.w);
      }
    } else if (p.probes != nullptr && p.t0 == 1) {
      const cx *src = p.probes + (size_t)(p0 + q) * p.N + c * M;
#pragma unroll
      for (int i = 0; i < M; ++i) U[q][i] = src[i];
    }
  }
  if (p.u_store != nullptr && !p.store_sums && store_index(p, p.t0 - 1) >= 0) {
    const int idx = store_index(p, p.t0 - 1);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (p0 + q >= p.P) continue;
      store_pairs(p.u_store + ((size_t)(p0 + q) * p.store_slices + idx) * p.Npad, U[q], M, c);
    }
  }

  // Two-slice gradient (QD): the forward slice u_s of the current step is
  // kept from the previous step (u_prev); only u_{s-1} is read, issued at the
  // start of the step so that its latency overlaps the solve.
  cx u_prev[Q][M], u_new[Q][M];
  if constexpr (QD) {
    if (do_grad) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int pq = (p0 + q < p.P) ? p0 + q : p.P - 1;
        load_pairs<M>(u_prev[q], p.u_fwd + ((size_t)pq * p.ufwd_slices + (slice_of(p.t0) - p.ufwd_base)) * p.Npad, c);
      }
    }
  }

  uint32_t phase = 0;
  {
    const bool ok = mbar_wait_bounded(&mbar[1], 0, p.err);
    phase ^= 2u;
    if (__syncthreads_or(!ok)) {
      if (tid == 0) mbar_wait_bounded(&mbar[1], 0, nullptr);
      __syncthreads();
      return;
    }
  }

  // Half-sum slices of the staged gradient: thread 0 of the team loads the
  // slice of step t into the team's staging slice at the start of step t,
  // once the previous step's contributions have been summed out of it.
  // g_pending / g_pend_par track a load that thread 0 has not yet seen
  // complete, so that an early return waits for it.
  const int nvalid = p.P - p0 < Q ? p.P - p0 : Q;  // probes of this team (<= 0: padding)
  const bool gvalid = nvalid > 0;
  uint32_t gphase = 0, g_pend_par = 0;
  bool g_pending = false;
  auto load_half_sums = [&](int t) {  // thread 0 of the team: step t's slices of its probes
    mbar_arrive_expect_tx(&gbar[team], (uint32_t)nvalid * NB);
#pragma unroll
    for (int q = 0; q < Q; ++q)
      if (q < nvalid)
        bulk_g2s(stg + (size_t)q * (M / 2) * C,
                 p.u_fwd + ((size_t)(p0 + q) * p.ufwd_slices + (slice_of(t) - p.ufwd_base)) * p.Npad, NB,
                 &gbar[team]);
    g_pending = true;
    g_pend_par = gphase;
  };
  if constexpr (GSTAGE) {
    if (do_grad && c == 0 && gvalid) load_half_sums(p.t0);
  }

  for (int t = p.t0; t <= p.t1; ++t) {
    const int cb = (t - p.t0 + 1) & 1;
    const int s = slice_of(t);
    if constexpr (GSTAGE) {
      // the previous step's contributions are complete (end-of-step
      // barrier): sum them into the gradient, then reload the slices
      if (do_grad && t > p.t0) {
        grad_sum_flush<M, Q, TM>(stage, p.grad_c + (size_t)(slice_of(t - 1) - 1) * p.Npad, tid);
        __syncthreads();
        if (c == 0 && gvalid) load_half_sums(t);
      }
    }
    if (tid == 0 && t < p.t1) {
      fence_proxy_async_smem();
      team_issue(bufs + (cb ^ 1) * ssf, p.factors + (size_t)(slice_of(t + 1) - 1) * p.slice_bytes, M, T,
                 &mbar[cb ^ 1], QD);
    }
    const cx *F = bufs + cb * ssf;
    if constexpr (!GSTAGE) {
      // unstaged gradient: this step's forward slice (QD: u_{s-1}; SUMS: the
      // half sum), issued before the solve so that its latency overlaps it
      if (do_grad) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const int pq = (p0 + q < p.P) ? p0 + q : p.P - 1;
          const int ix = SUMS ? s - p.ufwd_base : s - 1 - p.ufwd_base;
          load_pairs<M>(u_new[q], p.u_fwd + ((size_t)pq * p.ufwd_slices + ix) * p.Npad, c);
        }
      }
    }
    // Forward and reference-adjoint steps use the Cayley form of the step:
    // with M = I - P, (I + P) = 2I - M commutes with M^{-1}, so
    // M^{-1}((I + P) u + b) = 2 M^{-1}(u + b/2) - u.  The right-hand-side
    // stencil and its neighbour exchange drop out; the step keeps u in
    // registers and ends with one fused multiply-subtract per row.  The
    // exact-adjoint step (I + P) M^{-1} v = 2 M^{-1} v - v (SUMS) keeps the
    // solve's input v = u + b instead.  In the forward step the solve result
    // x = M^{-1}(u_{t-1} + b/2) is exactly (u_t + u_{t-1})/2, the half pair
    // sum the gradient contracts with: store_sums stores x itself.
    cx u_old[Q][M];
    if constexpr (!LAGGED) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int i = 0; i < M; ++i) u_old[q][i] = U[q][i];
    }
    const rx sw = LAGGED ? rx(1) : rx(0.5);  // source weight
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (p0 + q >= p.P) continue;
      const int g0 = c * M;
      if (p.src_shared != nullptr) {
        const cx *src = p.src_shared + (size_t)(t - 1) * p.N + g0;
#pragma unroll
        for (int i = 0; i < M; ++i) U[q][i] = caxpy(sw, src[i], U[q][i]);
      }
      if (p.src_probe != nullptr) {
        const int col = p.src_rev ? (p.L - t) : (t - 1);
        const cx *src = p.src_probe + ((size_t)(p0 + q) * p.L + col) * p.N + g0;
#pragma unroll
        for (int i = 0; i < M; ++i) U[q][i] = caxpy(sw, src[i], U[q][i]);
      }
      if (t == 1 && p.src_exit != nullptr) {
        const cx *src = p.src_exit + (size_t)(p0 + q) * p.N + g0;
#pragma unroll
        for (int i = 0; i < M; ++i) U[q][i] = caxpy(sw, src[i], U[q][i]);
      }
    }
    if constexpr (SUMS) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int i = 0; i < M; ++i) u_old[q][i] = U[q][i];
    }
    team_solve<M, Q, T, QD, STAGE && !LAGGED>(U, F, Y0, R0, R1, XS, c, team, p.sp, pcr);
    const int sidx = p.u_store != nullptr ? store_index(p, t) : -1;
    auto store_direct = [&]() {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        if (p0 + q >= p.P) continue;
        store_pairs(p.u_store + ((size_t)(p0 + q) * p.store_slices + sidx) * p.Npad, U[q], M, c);
      }
    };
    if constexpr (!LAGGED) {
      if (p.store_sums && sidx >= 0) {
        if constexpr (STAGE) store_staged<M, Q>(U, stg, p, p0, sidx, c, team);
        else store_direct();
      }
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int i = 0; i < M; ++i)
          U[q][i] = mkcx(rfma(rx(2), U[q][i].x, -u_old[q][i].x), rfma(rx(2), U[q][i].y, -u_old[q][i].y));
      if (!p.store_sums && sidx >= 0) {
        if constexpr (STAGE) store_staged<M, Q>(U, stg, p, p0, sidx, c, team);
        else store_direct();
      }
    } else {
      if (sidx >= 0) store_direct();
    }
    if (t == p.L && p.exit_out != nullptr) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        if (p0 + q >= p.P) continue;
        cx *dst = p.exit_out + (size_t)(p0 + q) * p.N + c * M;
#pragma unroll
        for (int i = 0; i < M; ++i) dst[i] = U[q][i];
      }
    }
    bool good = true;
    if (do_grad) {
      if constexpr (GSTAGE) {
        bool okg = true;
        if (gvalid) okg = mbar_wait_bounded(&gbar[team], gphase, p.err);
        if (okg) g_pending = false;
        gphase ^= 1u;
        good = okg;
        grad_contrib<M, Q>(U, stg, nvalid, c);
      } else {
        cx2 *gdst = reinterpret_cast<cx2 *>(p.grad_c + (size_t)(s - 1) * p.Npad) + c;
#pragma unroll
        for (int j = 0; j < M / 2; ++j) {
          cx2 ga = mkcx2(czero(), czero());
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            if (p0 + q >= p.P) continue;  // padded probes contribute nothing
            cx wa, wb;
            if constexpr (SUMS) {
              wa = u_new[q][2 * j];
              wb = u_new[q][2 * j + 1];
            } else {
              wa = cadd(u_prev[q][2 * j], u_new[q][2 * j]);
              wb = cadd(u_prev[q][2 * j + 1], u_new[q][2 * j + 1]);
            }
            const cx a = cmulc(U[q][2 * j], wa);
            const cx b = cmulc(U[q][2 * j + 1], wb);
            ga.x += a.x;
            ga.y += a.y;
            ga.z += b.x;
            ga.w += b.y;
          }
          if constexpr (SUMS) ga = mkcx2(mkcx(2 * ga.x, 2 * ga.y), mkcx(2 * ga.z, 2 * ga.w));  // half sums
          red_add_cx2(gdst + j * C, ga);
        }
        if constexpr (!SUMS) {
#pragma unroll
          for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int i = 0; i < M; ++i) u_prev[q][i] = u_new[q][i];
        }
      }
    }
    if constexpr (SUMS) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int i = 0; i < M; ++i)
          U[q][i] = mkcx(rfma(rx(2), U[q][i].x, -u_old[q][i].x), rfma(rx(2), U[q][i].y, -u_old[q][i].y));
    } else if constexpr (LAGGED) {
      team_rhs<M, Q>(U, F, XL, XF, c, team, p.sp);
    }
    if (t < p.t1) {
      const bool okf = mbar_wait_bounded(&mbar[cb ^ 1], (phase >> (cb ^ 1)) & 1u, p.err);
      good = good && okf;
      phase ^= (1u << (cb ^ 1));
    }
    if (__syncthreads_or(!good)) {
      if (tid == 0) mbar_wait_bounded(&mbar[cb ^ 1], ((phase >> (cb ^ 1)) & 1u) ^ 1u, nullptr);
      if constexpr (STAGE) {
        if (c == 0) {
          if (g_pending) mbar_wait_bounded(&gbar[team], g_pend_par, nullptr);
          bulk_wait();
        }
      }
      __syncthreads();
      return;
    }
  }
  if constexpr (GSTAGE) {
    if (do_grad) grad_sum_flush<M, Q, TM>(stage, p.grad_c + (size_t)(slice_of(p.t1) - 1) * p.Npad, tid);
  }
  if (p.state_out != nullptr) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (p0 + q >= p.P) continue;
      store_pairs(p.state_out + (size_t)(p0 + q) * p.Npad, U[q], M, c);
    }
  }
  if constexpr (STAGE) {
    if (c == 0) bulk_wait();
  }
}

template <int M, int Q, int TM, bool LAGGED, bool SUMS, int TS, bool STG>
static int launch_team_t(const Partition &pt, MarchParams &mp, cudaStream_t st) {
  auto kern = cn2d_team_kernel<M, Q, TM, LAGGED, SUMS, TS, STG>;
  if (mp.trunc != TS) return set_error(TP_ERR_INVALID, "team march staged %d spike rows, kernel has %d", mp.trunc, TS);
  constexpr bool QD = LAGGED && !SUMS;
  mp.smem_slice_bytes = team_slice_smem(M, TS, QD);
  const size_t smem = team_smem_bytes(pt, mp.trunc, Q, TM, QD, STG);
  TP_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (mp.P + Q * TM - 1) / (Q * TM);
  kern<<<grid, kTeamThreads * TM, smem, st>>>(mp);
  return check_cuda(cudaGetLastError(), "cn2d_team_kernel launch");
}

template <int M, bool LAGGED, bool SUMS, int TS, bool STG>
static int launch_team_qt(const Partition &pt, MarchParams &mp, int Q, int TM, cudaStream_t st) {
  if (TM == 1 && Q == 1) return launch_team_t<M, 1, 1, LAGGED, SUMS, TS, STG>(pt, mp, st);
  if (TM == 2 && Q == 1) return launch_team_t<M, 1, 2, LAGGED, SUMS, TS, STG>(pt, mp, st);
  if (TM == 4 && Q == 1) return launch_team_t<M, 1, 4, LAGGED, SUMS, TS, STG>(pt, mp, st);
  if constexpr (!LAGGED || (SUMS && STG)) {
    if (TM == 2 && Q == 2) return launch_team_t<M, 2, 2, LAGGED, SUMS, TS, STG>(pt, mp, st);
  }
  return set_error(TP_ERR_UNSUPPORTED, "no team kernel for Q=%d, TM=%d", Q, TM);
}

// Exact adjoint in Cayley form unless a gradient reads plain forward slices
// (two per step: not enough registers for the Cayley state as well).  The
// staged variants exist for the Cayley-form kernels only.
template <int M, int TS>
static int launch_team_m(const Partition &pt, MarchParams &mp, bool lagged, bool sums, bool stg, int Q, int TM,
                         cudaStream_t st) {
  if (!lagged)
    return stg ? launch_team_qt<M, false, false, TS, true>(pt, mp, Q, TM, st)
               : launch_team_qt<M, false, false, TS, false>(pt, mp, Q, TM, st);
  if (sums)
    return stg ? launch_team_qt<M, true, true, TS, true>(pt, mp, Q, TM, st)
               : launch_team_qt<M, true, true, TS, false>(pt, mp, Q, TM, st);
  return launch_team_qt<M, true, false, TS, false>(pt, mp, Q, TM, st);
}

// (teams per CTA, probes per thread) for K probes per CTA: one probe per
// thread (K teams) unless overridden.  With the Cayley step 4 teams x 1 probe
// time 2.75 ms per forward march at N = 2048 x 1023 slices x 512 probes
// against 2.84 ms for 2 x 2.
static void team_shape(int K, int *TM, int *Q, const char *var = "TPCUDA_TEAM_SHAPE") {
  const char *env = getenv(var);  // "TM,Q" override for tuning sweeps
  if (env != nullptr && sscanf(env, "%d,%d", TM, Q) == 2 && *TM * *Q == K) return;
  *TM = K;
  *Q = 1;
}

int launch_team_march(const Partition &pt, MarchParams &mp, bool lagged, cudaStream_t st) {
  // Spike rows staged: a compile-time count >= the rows the factorisation
  // keeps (the factor set holds all M rows; extra rows only add accuracy).
  if (pt.M == 16) mp.trunc = mp.trunc <= 8 ? 8 : 15;
  else mp.trunc = pt.M - 1;
  mp.smem_slice_bytes = team_slice_smem(pt.M, mp.trunc);
  int dev = 0, sms = 148, max_smem = 232448;
  TP_CHECK_CUDA(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const bool sums = lagged && (mp.u_fwd == nullptr || mp.store_sums);
  const bool qd = lagged && !sums;
  // Probes per CTA: one CTA per SM (the factor double buffer fills most of
  // an SM's shared memory), so K = ceil(P / SMs) rounded up to 1, 2 or 4.
  int K = 1;
  while (K < 4 && (mp.P + K - 1) / K > sms) K *= 2;
  int TM, Q;
  if (lagged) {
    // one probe per thread: the kept and prefetched forward slices need 2M
    // complex registers per probe on top of the state; the staged Cayley
    // form keeps none and may take a tuning override
    TM = K;
    Q = 1;
    if (sums) team_shape(K, &TM, &Q, "TPCUDA_ADJ_SHAPE");
  } else {
    team_shape(K, &TM, &Q);
  }
  // Staged global traffic where the staging slices fit beside the factor
  // double buffer at this shape; otherwise the direct path at this shape
  // (fewer teams per CTA would mean more CTAs than SMs).
  bool stg = !qd && team_smem_bytes(pt, mp.trunc, Q, TM, qd, true) <= (size_t)max_smem;
  if (lagged && Q > 1 && !stg) {  // several probes per thread need the staged gradient
    TM = K;
    Q = 1;
    stg = !qd && team_smem_bytes(pt, mp.trunc, Q, TM, qd, true) <= (size_t)max_smem;
  }
  while (team_smem_bytes(pt, mp.trunc, Q, TM, qd, stg) > (size_t)max_smem && TM * Q > 1) {
    if (TM > 1) TM /= 2;
    else Q /= 2;
  }
  if (team_smem_bytes(pt, mp.trunc, Q, TM, qd, stg) > (size_t)max_smem)
    return set_error(TP_ERR_UNSUPPORTED, "team march needs %zu B of shared memory (> %d)",
                     team_smem_bytes(pt, mp.trunc, Q, TM, qd, stg), max_smem);
  switch (pt.M) {
    case 4:
      return launch_team_m<4, 3>(pt, mp, lagged, sums, stg, Q, TM, st);
    case 8:
      return launch_team_m<8, 7>(pt, mp, lagged, sums, stg, Q, TM, st);
    case 16:
      return mp.trunc == 8 ? launch_team_m<16, 8>(pt, mp, lagged, sums, stg, Q, TM, st)
                           : launch_team_m<16, 15>(pt, mp, lagged, sums, stg, Q, TM, st);
    default:
      return set_error(TP_ERR_UNSUPPORTED, "no team kernel for %d rows per chunk", pt.M);
  }
}

}  // namespace tp
