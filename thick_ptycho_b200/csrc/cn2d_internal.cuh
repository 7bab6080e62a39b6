// Internal declarations shared by the 2D Crank–Nicolson translation units.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "tp_common.cuh"
#include "tpcuda.h"

namespace tp {

// The matrix rows are cut into C chunks of M rows (N_pad = C*M); chunk k's
// row i is matrix row k*M + i.  Two kernel families:
//   warp path  (C = 32):  one warp per probe, any 4 <= N <= 2048;
//   team path  (C = 128): a 4-warp CTA per group of Q probes, N in {512, 1024, 2048}.
constexpr int kWarpChunks = 32;
constexpr int kTeamChunks = 128;
constexpr int kMaxRowsPerLane = 64;

struct Partition {
  int C;      // chunks
  int M;      // rows per chunk
  int team;   // 1 = team path
  int levels; // log2(C): PCR levels of the reduced system
  int nrec;   // per-chunk reduced-system records: MA, MC, alpha[levels], gamma[levels], RDE
};

__host__ __device__ inline int rec_alpha(int levels, int l) { return 2 + l; }
__host__ __device__ inline int rec_gamma(int levels, int l) { return 2 + levels + l; }
__host__ __device__ inline int rec_rde(int levels) { return 2 + 2 * levels; }

// Global factor set of one slice: QD, LF, EP, V, W ([M][C] complex values
// each) then the records ([nrec][C]), padded to 256 bytes.  The workspace of a
// factorisation holds L slices and then kFactorTailBytes: the largest PCR
// coefficient of all slices (float bits), which the team march reads.
__host__ __device__ inline size_t slice_bytes(const Partition &pt) {
  size_t b = (size_t)(5 * pt.M + pt.nrec) * pt.C * sizeof(cx);
  return (b + 255) & ~size_t(255);
}

constexpr size_t kFactorTailBytes = 256;
// Below this bound the reduced (separator) system is diagonal to far beneath
// the state's round-off and the team march skips its PCR levels; spike
// entries below kSpikeDrop are not staged.  Both scale with the precision of
// the build, so that in the complex128 check build the approximations stay
// beneath fp64 round-off too.
#ifdef TP_C128_CHECK
constexpr float kPcrSkipBound = 1e-17f;
constexpr double kSpikeDrop = 1e-17;
#else
constexpr float kPcrSkipBound = 1e-12f;
constexpr double kSpikeDrop = 1e-9;
#endif

int partition_for(int n, Partition *pt);  // TP_OK or an error code

// Device error codes (bit flags) recorded instead of trapping.
enum DeviceErrorBits : int { kDevSpikeTruncation = 2 };

struct FactorParams {
  int N, L, nz, n_obj, empty_px, exact, is_delta, dtype;
  int sl0;  // first slice (0-based) of this launch; CTA b factorises slice sl0 + b
  int C, M, levels, nrec;
  int trunc;  // spike rows the march keeps (V rows [0,T), W rows [M-1-T, M-1))
  double sigma;
  int conj_t;
  double k, dz;
  double2 k_off, k_diag, k_d0, k_dn, k_01, k_nm;
  const void *n;
  char *factors;
  size_t slice_bytes;
  unsigned *coupling;  // max |alpha|, |gamma| of the PCR records (float bits), atomically maxed
  int *err;
};

// P's off-diagonals: interior value and the four boundary entries (+ deltas).
struct Spec {
  cx p_o;
  cx sup0, sub1, supN2, subN1;
  cx d_sup0, d_sub1, d_supN2, d_subN1;
};

struct MarchParams {
  int N, L, nz, P, Npad;
  int backward, flip_out, src_rev;
  int trunc;                 // team path: spike rows kept in shared memory
  size_t slice_bytes;        // global factor-set stride
  size_t smem_slice_bytes;   // team path: shared-memory slice size
  const char *factors;
  Spec sp;
  const cx *probes, *src_shared, *src_probe, *src_exit;
  cx *u_store, *exit_out;
  const cx *u_fwd;
  cx *grad_c;
  const unsigned *coupling;     // the factor set's PCR coupling bound (float bits), or NULL
  int *err;
  int t0, t1;                   // step range
  const cx *state_in;           // chunked (P, Npad) or null
  cx *state_out;
  int store_slices, store_every, store_base;
  int ufwd_slices, ufwd_base;
  int store_sums;               // FORWARD: u_store gets u_t + u_{t-1}; ADJOINT_EXACT: u_fwd holds them
};

// Index in u_store of the state after step t (t0-1 = the initial state), or -1.
__host__ __device__ inline int store_index(const MarchParams &p, int t) {
  int idx;
  if (p.store_every > 1) {
    if (t % p.store_every != 0) return -1;
    idx = t / p.store_every;
  } else {
    idx = p.flip_out ? (p.L - t) : (t - p.store_base);
  }
  return (idx >= 0 && idx < p.store_slices) ? idx : -1;
}

// Spike rows kept by the team path for operator `op` with M rows per chunk:
// the inverse of a diagonally dominant tridiagonal matrix decays like rho^d,
// rho = (d0 - sqrt(d0^2 - 4 b^2)) / (2 b) with b the off-diagonal and d0 the
// diagonal magnitude of the free-space matrix; keep rows until rho^T is
// below kSpikeDrop (plus one).  The factor kernel verifies the choice on the actual matrices.
int team_spike_rows(const tp_cn2d_op *op, int M);

// Team-path launcher (cn2d_team.cu).
int launch_team_march(const Partition &pt, MarchParams &mp, bool lagged, cudaStream_t st);
size_t team_smem_bytes(const Partition &pt, int trunc, int Q, int TM, bool qd, bool stg);

}  // namespace tp
