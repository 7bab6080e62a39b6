/*
 * tpcuda.h — C ABI of libtpcuda.so, the sm_100a implementation of the
 * thick_ptycho paraxial finite-difference (PWE) hot path.
 *
 * Every entry point returns an int status (TP_OK = 0); on failure
 * tp_last_error_string() describes the last error of the calling thread.
 * Pointers are device pointers unless stated otherwise; complex numbers are
 * interleaved (re, im) pairs: float2 for complex64, double2 for complex128.
 * All work is enqueued on the caller's stream; no entry point synchronises
 * except where stated, and none allocates device memory: the caller passes
 * workspaces sized by the *_bytes() queries.
 *
 * libtpcuda_c128.so, the complex128 check build, exports the tp_cn2d_* and
 * tp_cn3d_* entry points with the same signatures and every complex buffer
 * (state, operator diagonals, stores, sources, workspaces' vectors)
 * complex128; its *_bytes() queries size for that.  Its 3D march has no
 * learned correction (precond = 2 returns TP_ERR_UNSUPPORTED).
 *
 * Step equation (reference iterative_lu.py:185-193, operator_matrices.py:36-72):
 *   (A - C_j) u_j = (B + C_j) u_{j-1} + b_j,  A = I - K, B = I + K,
 *   K = scaled tridiagonal second difference with boundary-row edits,
 *   C_j = diag((dz/2) * 0.5 * (coef(n[:, j-1]) + coef(n[:, j]))),
 *   coef(n) = (k/i)(n - 1)  or  (k/2i)(n^2 - 1)  (exact_ref_coeff)
 *   (reference base_simulation_space.py:315-383).
 */
#ifndef TPCUDA_H
#define TPCUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TP_API __attribute__((visibility("default")))
#else
#define TP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *tp_stream_t; /* = cudaStream_t */

enum tp_status {
  TP_OK = 0,
  TP_ERR_INVALID = 1,   /* bad argument (size, null pointer, mode) */
  TP_ERR_UNSUPPORTED = 2,
  TP_ERR_CUDA = 3,      /* a CUDA runtime call failed */
  TP_ERR_TIMEOUT = 4,   /* a device-side bounded wait gave up */
  TP_ERR_WORKSPACE = 5  /* workspace too small */
};

/* Propagation modes (reference iterative_lu.py:90-133, 185-197). */
enum tp_mode {
  TP_MODE_FORWARD = 0,       /* (A - C_j) u_j = (B + C_j) u_{j-1} + b      */
  TP_MODE_ADJOINT = 1,       /* reference adjoint: (A - C_s)^H, (B + C_s)^H,
                                s = L+1-j, output flipped along z          */
  TP_MODE_REVERSE = 2,       /* A<->B swapped, C negated, slices reversed   */
  TP_MODE_ADJOINT_EXACT = 3  /* exact discrete adjoint of FORWARD:
                                (A - C_s)^H l_s = e_s + (B + C_{s+1})^H l_{s+1} */
};

/* Dtype of the refractive-index array handed to tp_cn2d_factor. */
enum tp_dtype { TP_C128 = 0, TP_C64 = 1 };

/*
 * The 2D step operator: K's interior entries and its boundary-row edits.
 * Replaces the reference's sparse A_step/B_step (operator_matrices.py:47-72,
 * boundary_conditions.py:57-94) and the C_j coefficients
 * (base_simulation_space.py:315-383).  Complex values are (re, im).
 */
typedef struct tp_cn2d_op {
  int32_t n;               /* transverse rows N (block_size), 4 <= N <= 2048 */
  int32_t nz;              /* z nodes; L = nz - 1 steps                     */
  int32_t n_obj;           /* rows of the object array (N - 2*empty_px)      */
  int32_t empty_px;        /* zero padding of the object coefficient         */
  int32_t exact_ref_coeff; /* coef = (k/2i)(n^2-1) instead of (k/i)(n-1)     */
  int32_t field_is_delta;  /* the index array holds n - 1 instead of n       */
  double k;                /* wavenumber 2*pi/lambda                         */
  double dz;               /* z step                                         */
  double k_off[2];         /* interior off-diagonal of K (mu_x)              */
  double k_diag[2];        /* interior diagonal of K (-2 mu_x)               */
  double k_d0[2];          /* K[0,0]                                          */
  double k_dn[2];          /* K[N-1,N-1]                                      */
  double k_01[2];          /* K[0,1]                                          */
  double k_nm[2];          /* K[N-1,N-2]                                      */
} tp_cn2d_op;

/* Arguments of one batched march over all probes. */
typedef struct tp_cn2d_march_args {
  int32_t num_probes;        /* P                                             */
  int32_t mode;              /* tp_mode; must match the factor set            */
  const void *probes;        /* float2 (P, N) initial fields, or NULL (zero)  */
  const void *src_shared;    /* float2 (L, N) probe-independent source, row t-1
                                used at step t (exact test boundary data,
                                reference boundary_condition_test.py:109-114),
                                or NULL                                       */
  const void *src_probe;     /* float2 (P, L, N) per-probe source (the
                                reference's rhs_block transposed to slice-major;
                                slice t-1 at step t, or L-t for the adjoint
                                modes), or NULL                               */
  const void *src_exit;      /* float2 (P, N) source applied at the first step
                                only (exit-wave error for the adjoints), or NULL */
  void *u_store;             /* float2 (P, nz, Npad) full field in the chunked
                                layout (see tp_cn2d_layout), or NULL    */
  void *exit_out;            /* float2 (P, N) last-step field, or NULL        */
  const void *u_fwd;         /* ADJOINT_EXACT + gradient: forward full field
                                (chunked, as written by a FORWARD march)      */
  void *grad_c;              /* ADJOINT_EXACT: float2 (L, Npad) accumulator of
                                sum_p lambda_s * conj(u_s + u_{s-1}) in the
                                chunked layout of tp_cn2d_layout; the caller
                                zeroes it; row s-1 holds slice s               */
  /* Partial marches (checkpointed gradients).  All zero = one march over all
   * L steps storing every slice at its own index. */
  int32_t t_begin, t_end;    /* step range [t_begin, t_end], 1-based; 0 = 1 / L */
  const void *state_in;      /* float2 (P, Npad) chunked state before t_begin
                                (overrides probes), or NULL                   */
  void *state_out;           /* float2 (P, Npad) chunked state after t_end (for
                                ADJOINT_EXACT: the next step's right-hand side),
                                or NULL                                        */
  int32_t store_slices;      /* slices per probe in u_store (0 = nz)          */
  int32_t store_every;       /* 0 or 1: state after step t at index t - store_base;
                                S > 1: only when t % S == 0, at index t / S    */
  int32_t store_base;
  int32_t ufwd_slices;       /* slices per probe in u_fwd (0 = nz)             */
  int32_t ufwd_base;         /* u_fwd index of forward slice s is s - ufwd_base */
  int32_t store_sums;        /* 0, or 1 (N in {512, 1024, 2048} only): FORWARD
                                stores the half pair sums (u_t + u_{t-1})/2 the
                                gradient contracts with instead of u_t (the
                                initial state is not stored; needs
                                store_every <= 1); ADJOINT_EXACT reads u_fwd as
                                such sums (one slice per step instead of two) */
} tp_cn2d_march_args;

/* Partition of N rows into `chunks` chunks of `rows_per_chunk` rows (padded
 * row count Npad = chunks * rows_per_chunk).  Chunked full fields store row
 * k*rows_per_chunk + i of a slice at offset i*chunks + k when chunks == 32,
 * and in row pairs, at offset ((i/2)*chunks + k)*2 + i%2, when chunks == 128
 * (N in {512, 1024, 2048}; these sizes need purely imaginary off-diagonals
 * of K, which every paraxial operator has). */
TP_API int tp_cn2d_layout(int32_t n, int32_t *chunks, int32_t *rows_per_chunk, int32_t *npad);

/* Bytes of the per-slice factor workspace for (N, nz). */
TP_API size_t tp_cn2d_factor_bytes(int32_t n, int32_t nz);

/*
 * Factorise every slice's LHS (the reference's _build_lu_factors,
 * iterative_lu.py:103-133, and the per-mode matrix choice of :90-128) into
 * the caller's workspace.  `n_field` is the refractive index, shape
 * (n_obj, nz), row-major, dtype `n_dtype`.
 */
TP_API int tp_cn2d_factor(const tp_cn2d_op *op, const void *n_field, int32_t n_dtype, int32_t mode,
                   void *factors, size_t factors_bytes, tp_stream_t stream);

/* The same for slices [slice_begin, slice_end] only (1-based, inclusive;
 * slice s reads index columns s-1 and s), so that factorisation can follow
 * the index field onto the device column block by column block.  The range
 * starting at slice 1 resets the factor set's PCR coupling bound, which later
 * ranges raise: factorise the ranges in increasing order and march a range
 * only after it is factorised.  (No reference counterpart: a pipelining
 * form of tp_cn2d_factor.) */
TP_API int tp_cn2d_factor_range(const tp_cn2d_op *op, const void *n_field, int32_t n_dtype, int32_t mode,
                                void *factors, size_t factors_bytes, int32_t slice_begin, int32_t slice_end,
                                tp_stream_t stream);

/* Asynchronous copy of bytes [byte_begin, byte_begin + byte_count) of each of
 * `rows` rows of `row_bytes` bytes between equally laid-out arrays (host or
 * device, pinned host memory for asynchrony): a column block of a row-major
 * array, e.g. the z nodes of the index field a factorisation range needs. */
TP_API int tp_copy_columns(void *dst, const void *src, int64_t rows, int64_t row_bytes, int64_t byte_begin,
                           int64_t byte_count, tp_stream_t stream);

/*
 * March all probes through the slices with a factor set of the same mode
 * (the reference's per-probe loop iterative_lu.py:138-197 and the serial
 * probe loop base/base_solver.py:124-143, batched).
 */
TP_API int tp_cn2d_march(const tp_cn2d_op *op, const void *factors, const tp_cn2d_march_args *args,
                  tp_stream_t stream);

/*
 * Map the per-step gradient sum_p lambda_s conj(u_s + u_{s-1}) (L, Npad,
 * chunked layout as written by tp_cn2d_march) onto the
 * refractive-index nodes (n_obj, nz) (torch convention d/dRe + i d/dIm):
 * g_n[x, t] = conj((dz/4) coef'(n[x,t])) * (g_c[t] + g_c[t+1]).
 * `n_field` is needed only when exact_ref_coeff is set (else may be NULL).
 * grad_n is float2 (n_obj, nz), row-major, overwritten.
 */
TP_API int tp_cn2d_grad_to_n(const tp_cn2d_op *op, const void *grad_c, const void *n_field, int32_t n_dtype,
                      void *grad_n, tp_stream_t stream);
/* The same for node columns [node_begin, node_end] only (node t reads slices
 * t and t + 1 of grad_c), so that finished columns can be mapped and copied
 * off while the adjoint march still runs on the earlier slices.  (No
 * reference counterpart.) */
TP_API int tp_cn2d_grad_to_n_range(const tp_cn2d_op *op, const void *grad_c, const void *n_field, int32_t n_dtype,
                                   void *grad_n, int32_t node_begin, int32_t node_end, tp_stream_t stream);

/* Gather a chunked full field (P, nz, Npad) into the reference layout
 * (P, N, nz) complex64. */
TP_API int tp_cn2d_unchunk(const tp_cn2d_op *op, int32_t num_probes, const void *u_store, void *u_out,
                    tp_stream_t stream);

/*
 * tp_cn2d_factor + tp_cn2d_march in one call that allocates nothing: the
 * factor set lives in a 32 MiB file-scope device array instead of a caller
 * workspace.  This entry point has no counterpart in the reference.  It is
 * for callers that cannot allocate device memory: a host that owns the whole
 * device budget as a pre-reserved pool and passes only input and output
 * buffers, or a latency-bounded loop where cudaMalloc (which may synchronise
 * the device) is not allowed.  Problems whose tp_cn2d_factor_bytes exceeds
 * 32 MiB return TP_ERR_WORKSPACE.  Every GPU that loads the library holds the
 * array until exit; calls share it, so calls that overlap on the GPU race.
 * The first call on a device resolves the array's address
 * (cudaGetSymbolAddress) and should come before any stream capture.
 */
TP_API int tp_cn2d_march_noalloc(const tp_cn2d_op *op, const void *n_field, int32_t n_dtype,
                                 const tp_cn2d_march_args *args, tp_stream_t stream);

/*
 * The reference's NLCG pieces on stored chunked fields (P, nz, Npad) of a
 * FORWARD march (u_store) and a reference ADJOINT march (lam_store), with its
 * constant gradient operator grad_A = -(diag(G) + subdiag(G)), G = (dz/2)(k/i)
 * (forward_model.py:128-153).  Both need exact_ref_coeff = 0 and empty_px = 0.
 */
/* compute_grad_least_squares (pwe_reconstructor.py:100-164): grad_re, grad_im
 * float32 (L*N), z-major like the reference's vector form; overwritten. */
TP_API int tp_cn2d_ref_gradient(const tp_cn2d_op *op, int32_t num_probes, const void *u_store,
                                const void *lam_store, float *grad_re, float *grad_im, tp_stream_t stream);
/* The per-probe source grad_A @ u_p of compute_alphak (pwe_reconstructor.py:
 * 166-219) as float2 (P, L, N), the src_probe layout of tp_cn2d_march. */
TP_API int tp_cn2d_alpha_source(const tp_cn2d_op *op, int32_t num_probes, const void *u_store, void *src,
                                tp_stream_t stream);

/* ---------------------------------------------------------------- FFT heads
 * Shared-memory mixed-radix FFTs: n = 2^a 3^b 5^c, n <= 4096; rows of n
 * complex64 values, numpy conventions (forward unnormalised, inverse 1/n). */

/* Batched 1D FFT of `batch` rows (in may equal out). Replaces numpy.fft.fft /
 * ifft of base/base_solver.py:234-242 and base_reconstructor.py:191,205. */
TP_API int tp_fft1d(int32_t n, int32_t batch, const void *in, void *out, int32_t inverse, tp_stream_t stream);

/* Far-field intensities |FFT(exit)|^2 (float32, unnormalised, no shift):
 * base/base_solver.py:234-242 without the Poisson noise. */
TP_API int tp_farfield_intensity(int32_t n, int32_t batch, const void *exit_waves, float *intensity,
                                 tp_stream_t stream);

/* Amplitude loss sum (|F e| - a)^2 of exit waves e (batch, n) against the
 * measured amplitudes a = sqrt(I) (float32), and its gradient w.r.t. e in
 * torch's convention, F^H[2(|Fe| - a) Fe/|Fe|] = 2n (e - P_GS(e)) with P_GS
 * the reference's modulus projection (base_reconstructor.py:171-207).
 * *loss_out is accumulated (the caller zeroes it). */
TP_API int tp_amplitude_residual(int32_t n, int32_t batch, const void *exit_waves, const float *amplitude,
                                 void *grad_out, double *loss_out, tp_stream_t stream);

/* ----------------------------------------------------------- multislice
 * Angular-spectrum multislice of forward_model/multislice/ms_solver.py:49-159:
 * u_{z+1} = IFFT(H . FFT(T_z u_z)), T_z = exp(i k (n[:,z] - n_medium) dz),
 * H = exp(i (k_z - k) dz), k_z = sqrt(max(k^2 - k_x^2, 0)). */
typedef struct tp_ms2d_op {
  int32_t n;             /* transverse points, 2^a 3^b 5^c <= 4096 */
  int32_t nz;            /* z nodes (L = nz - 1 steps) */
  double k, dx, dz;
  double n_medium[2];    /* background index (re, im) */
} tp_ms2d_op;

/* Transmission table T (L, n) complex64 from the index n (n, nz), dtype TP_C128/TP_C64. */
TP_API int tp_ms2d_transmission(const tp_ms2d_op *op, const void *n_field, int32_t n_dtype, void *trans,
                                tp_stream_t stream);
/* March P probes (P, n); u_store (P, nz, n) or NULL; exit_out (P, n) or NULL. */
TP_API int tp_ms2d_march(const tp_ms2d_op *op, const void *trans, const void *probes, int32_t num_probes,
                         void *u_store, void *exit_out, tp_stream_t stream);
/* Adjoint march from the exit-wave gradient src_exit (P, n) with the forward
 * field u_fwd (P, nz, n); accumulates grad_t (L, n) += sum_p conj(T_z u_z) g_z,
 * g_z = IFFT(conj(H) FFT(lambda_{z+1})).  d loss/d n[:, z] = conj(i k dz) grad_t[z]. */
TP_API int tp_ms2d_backward(const tp_ms2d_op *op, const void *trans, const void *u_fwd, const void *src_exit,
                            int32_t num_probes, void *grad_t, tp_stream_t stream);

/* Multislice 3PIE reconstruction (reconstruction/ms_reconstructor.py:40-190):
 * `iters` epochs over the probes in scan order, each probe's forward march,
 * modulus constraint and slice-by-slice back-propagation update applied to
 * the estimate in place (sequential, as the reference; one CTA).
 * data: float (P, n) far-field intensities when phase_retrieval != 0, else
 * float2 (P, n) known exit waves.  n_est: double2 (n, nz) row-major, the
 * starting estimate in, the result out.  loss: double (iters), the rms of
 * (corrected - modelled) exit waves per epoch.  Workspace:
 * tp_ms2d_3pie_workspace_bytes(n, nz). */
TP_API size_t tp_ms2d_3pie_workspace_bytes(int32_t n, int32_t nz);
TP_API int tp_ms2d_3pie(const tp_ms2d_op *op, const void *probes, int32_t num_probes, const void *data,
                        int32_t phase_retrieval, int32_t iters, double alpha_obj, void *n_est, double *loss,
                        void *workspace, size_t workspace_bytes, tp_stream_t stream);

/* ------------------------------------------------ PiT space-time solve
 * The full-system form of the 2D march (full_pint.py:71-275,
 * _pint_utils.py:27-205): the L = nz - 1 steps as one block-bidiagonal
 * system M u = b, M = diag(A - C_j) - subdiag(B + C_j), b = [B u_0 + rhs_0,
 * rhs_1, ...] (the probe enters through B alone, as in the reference's
 * full-system solvers), solved by restarted GMRES right-preconditioned with
 * the alpha-circulant R = Gamma^-1 F blockdiag((A - w_j B)^-1) F* Gamma of the
 * free-space A, B, in its flexible form (u = u_0 + Z s with z_j = R v_j).
 * All probes' Krylov spaces are built together.
 * Replaces PWEFullPinTSolver._solve_single_probe_impl for the forward mode. */
typedef struct tp_pit_args {
  int32_t num_probes;      /* P                                                */
  int32_t restart;         /* Krylov vectors per cycle (0 = 20, scipy's
                              default), <= 64                                  */
  int32_t max_cycles;      /* restart cycles (0 = 1000)                        */
  int32_t mode;            /* TP_MODE_FORWARD, or TP_MODE_ADJOINT: the
                              reference's adjoint system (full_pint.py:140-166)
                              - blocks A^H - C'_j, -(B^H + C'_j) with
                              C' = conj(C) flipped along z, the forward
                              preconditioner, b = rhs (+ B u_0 with the forward
                              B), u not flipped                               */
  double alpha;            /* circulant parameter (0 = 1e-2, the reference's)  */
  double rtol, atol;       /* stop at ||b - M u|| <= max(atol, rtol ||b||)
                              (0 = 1e-5 / 1e-8, the reference's gmres call)    */
  const void *probes;      /* float2 (P, N) initial fields u_0, or NULL         */
  const void *rhs;         /* float2 (P, nz-1, N) added to b (slice-major), or
                              NULL                                             */
  void *u;                 /* float2 (P, nz-1, N): u_1 .. u_L, the initial
                              guess in (zeros for none), the solution out      */
  int32_t *iters;          /* host (P) or NULL: Arnoldi steps per probe          */
  double *resid;           /* host (P) or NULL: final ||b - M u|| per probe      */
} tp_pit_args;

/* Workspace bytes of tp_pit_solve (0 if unsupported). */
TP_API size_t tp_pit_workspace_bytes(int32_t n, int32_t nz, int32_t num_probes, int32_t restart);
/* Solve for every probe; op as for tp_cn2d_factor (its K and object fields);
 * n_field (n_obj, nz) of dtype n_dtype.  nz - 1 <= 2048.  Synchronises the
 * stream (the GMRES control flow runs on the host). */
TP_API int tp_pit_solve(const tp_cn2d_op *op, const void *n_field, int32_t n_dtype, const tp_pit_args *args,
                        void *workspace, size_t workspace_bytes, tp_stream_t stream);

/* ---------------------------------------------------- 3D multislice
 * The propagator of tp_ms2d_* on an (n1, n2) transverse grid (the
 * reference's multislice solver is 2D only, ms_solver.py:28-31):
 * u_{z+1} = IFFT2(H . FFT2(T_z u_z)), H = exp(i (k_z - k) dz),
 * k_z = sqrt(max(k^2 - k1^2 - k2^2, 0)), k1 = 2 pi fftfreq(n1, d1),
 * k2 = 2 pi fftfreq(n2, d2).  Element (a, b) of a slice is at a * n2 + b
 * (the C-order flattening of the reference's (nx, ny) arrays); the index
 * field is (n1 * n2, nz). */
typedef struct tp_ms3d_op {
  int32_t n1, n2;        /* transverse grid, each 2^a 3^b 5^c <= 4096 */
  int32_t nz;            /* z nodes (L = nz - 1 steps) */
  int32_t reserved;
  double k, d1, d2, dz;
  double n_medium[2];    /* background index (re, im) */
} tp_ms3d_op;

/* Workspace of tp_ms3d_march / tp_ms3d_backward for P probes (the field and
 * spectrum work buffers, (H - 1)/N and the twiddles). */
TP_API size_t tp_ms3d_workspace_bytes(int32_t n1, int32_t n2, int32_t num_probes);
/* Transmission table T - 1, (L, n1 * n2) complex64, from the index field. */
TP_API int tp_ms3d_transmission(const tp_ms3d_op *op, const void *n_field, int32_t n_dtype, void *trans,
                                tp_stream_t stream);
/* March P probes (P, n1 * n2); u_store (P, nz, n1 * n2) or NULL; exit_out
 * (P, n1 * n2) or NULL.  Two kernels per slice (row pass, column pass). */
TP_API int tp_ms3d_march(const tp_ms3d_op *op, const void *trans, const void *probes, int32_t num_probes,
                         void *u_store, void *exit_out, void *workspace, size_t workspace_bytes,
                         tp_stream_t stream);
/* Adjoint march from src_exit (P, n1 * n2) with the forward field u_fwd
 * (P, nz, n1 * n2): grad_t (L, n1 * n2) += sum_p conj(T_z u_z) g_z,
 * g_z = IFFT2(conj(H) FFT2(lambda_{z+1})); d loss/d n[:, z] = conj(i k dz) grad_t[z]. */
TP_API int tp_ms3d_backward(const tp_ms3d_op *op, const void *trans, const void *u_fwd, const void *src_exit,
                            int32_t num_probes, void *grad_t, void *workspace, size_t workspace_bytes,
                            tp_stream_t stream);

/* ------------------------------------------------------------------- 3D
 * 3D problems (2D transverse, N = nf*nb rows, index i = b*nf + f, the
 * flattening of kron(I_y, A_x) in operator_matrices.py:75-99): each slice is
 * solved by FFT-preconditioned BiCGStab in delta form (see cn3d.cu), batched
 * over probes, fp64 inner products.  Replaces the per-slice SuperLU of the 2D
 * operator (iterative_lu.py:103-133) and the per-probe march (:138-197). */
struct tp_cnn_model;

typedef struct tp_cn3d_op {
  int32_t nf, nb, nz;        /* fast / block transverse sizes, z nodes          */
  int32_t exact_ref_coeff;   /* coef = (k/2i)(n^2-1) instead of (k/i)(n-1)       */
  int32_t field_is_delta;    /* the index array holds n - 1                     */
  int32_t reserved;
  double k, dz;
  double mu_x[2], mu_y[2];   /* interior couplings of K (preconditioner symbol) */
  const void *kc, *kw, *ke, *ks, *kn;  /* device float2 (N) diagonals of K:
                                (K x)_i = c x_i + w x_{i-1} + e x_{i+1}
                                        + s x_{i-nf} + n x_{i+nf}               */
} tp_cn3d_op;

typedef struct tp_cn3d_march_args {
  int32_t num_probes, mode;  /* tp_mode                                          */
  int32_t max_iter;          /* BiCGStab iterations per solve (0 = 20)           */
  int32_t precond;           /* 1: periodic FFT preconditioner (when nf, nb are
                                2^a 3^b 5^c and tile), 0: none, 2: the FFT
                                preconditioner with the learned per-pixel
                                correction of `model` (not REVERSE)             */
  int32_t host_check;        /* 1: stop iterating a step once all its probes
                                converged (on the device when the march runs as
                                a graph, else by a stream synchronisation per
                                iteration); 0: always max_iter iterations, step
                                by step                                          */
  int32_t launch;            /* 0: one CUDA graph per march, whose step and
                                iteration loops are conditional WHILE nodes (no
                                host round trip), except on a capturing stream
                                or with training pairs; 1: step by step          */
  double tol;                /* relative residual per solve (0 = 1e-6)           */
  const void *probes;        /* float2 (P, N) initial fields, or NULL            */
  const void *src_shared;    /* float2 (L, N) probe-independent source by step   */
  const void *src_exit;      /* float2 (P, N) source at the first step, or NULL  */
  void *u_store;             /* float2 (P, nz, N) or NULL                        */
  void *exit_out;            /* float2 (P, N) or NULL                            */
  const void *u_fwd;         /* ADJOINT_EXACT gradient: forward field (P, nz, N) */
  void *grad_c;              /* ADJOINT_EXACT: float2 (L, N) accumulator of
                                sum_p lambda_s conj(u_s + u_{s-1}); caller zeroes */
  int32_t *stats;            /* device int32[5]: total iterations, solves, solves
                                whose true residual exceeded 10 tol, largest
                                iteration count (accumulated), and [4] = 1 when
                                the march ran as one graph (0 step by step);
                                or NULL.  A caller of the learned form re-runs
                                the march with precond = 1 when stats[2] grew
                                (fallback) */
  const struct tp_cnn_model *model;  /* precond == 2: the network            */
  void *learned_ws;          /* precond == 2: tp_cn3d_learned_ws_bytes, 256-B aligned */
  size_t learned_ws_bytes;
  /* Training pairs (no counterpart in the reference): at every step t with
   * t % train_every == 0, index k = t/train_every - 1 receives a vector x and
   * z0 = M0^{-1} v with (I - P_s) x = v, M0^{-1} the plain FFT preconditioner
   * (train_z0 and train_sol, (P, N) each), and the object diagonal
   * sigma*T(c_s) of the slice (train_diag, (N)).  train_kind 0: v is the
   * step's right-hand side and x its converged update; 1: x is uniform
   * complex white noise (a counter hash of step, probe and row) and
   * v = (I - P_s) x exactly. */
  void *train_z0, *train_sol, *train_diag;
  int32_t train_every;       /* 0 = no training pairs                           */
  int32_t train_kind;
  int32_t learned_reuse;     /* precond == 2: 1 = the learned workspace already
                                holds the filters of this index field and model
                                (from the previous march with it, e.g. the
                                forward before the adjoint): the network is not
                                run again                                       */
  int32_t kernels;           /* kernel choice, the same arithmetic either way
                                (0 = automatic).  Bit 0: the preconditioner's
                                transforms always by the shared-memory Stockham
                                kernels (automatic: register four-step kernels
                                where nf = nb is 64, 128, 192 or 256).  Bit 1:
                                the stencil kernels (right-hand side, matvecs,
                                finish) always with per-thread loads
                                (automatic: inputs staged by tensor-memory
                                copies where nf is 64, 128, 192 or 256 and nb
                                is even; complex64 build).  Bit 2: the learned
                                filter by register shuffles (automatic: rows
                                staged by bulk copies where nf is 64, 128, 192
                                or 256).                                        */
} tp_cn3d_march_args;

TP_API size_t tp_cn3d_workspace_bytes(int32_t n_total, int32_t num_probes);
/* Learned-form workspace: the CNN activations of 64 slices, the filters of
 * all nz - 1 slices (13 complex64 taps per pixel) and P plain-preconditioned
 * vectors. */
TP_API size_t tp_cn3d_learned_ws_bytes(int32_t nf, int32_t nb, int32_t nz, int32_t num_probes);
TP_API int tp_cn3d_march(const tp_cn3d_op *op, const void *n_field, int32_t n_dtype, const tp_cn3d_march_args *args,
                         void *workspace, size_t workspace_bytes, tp_stream_t stream);

/* ------------------------------------------------ learned 3D preconditioner
 * The reference has no learned component; these entry points are this
 * library's own addition to the 3D path (a learned correction of the FFT
 * preconditioner).
 * A four-layer 3x3 CNN (bf16 weights, fp32 accumulation on the tcgen05
 * tensor cores) maps the object diagonal d of one slice to a 13-tap complex
 * filter per pixel; the learned preconditioner is y = z + sum_t F_t(x) z(x + o_t)
 * with z the plain FFT-preconditioned vector, taps o_t = (0,0), (0,-1), (0,1),
 * (-1,0), (1,0), (-1,-1), (-1,1), (1,-1), (1,1), (0,-2), (0,2), (-2,0), (2,0)
 * as (row, column) offsets of the nb x nf image (vector index b*nf + f).
 *
 * Activations use a padded-linear bf16 layout (one-pixel zero border around
 * each image, images back to back, channels in chunks of 8); buffers sized by
 * tp_cnn_act_bytes must be zeroed once before first use (only interior pixels
 * are ever written).  Weights of a layer with cin inputs and 32 outputs:
 * bf16 [9 taps (row-major 3x3)][cin/8][32][8]. */
typedef struct tp_cnn_model {
  const void *w[4];     /* layers 16->32, 32->32, 32->32, 32->32 (26 used)   */
  const float *b[4];    /* fp32 biases (32 each) or NULL                      */
  float kappa;          /* scale of the d features                            */
  float out_scale;      /* the filter is out_scale * (last layer + bias)      */
} tp_cnn_model;

enum tp_conv_epilogue {
  TP_CONV_RELU = 0,     /* out = relu(conv + b), bf16 32 channels             */
  TP_CONV_MASK = 1,     /* out = conv * (aux > 0) (ReLU backward), bf16       */
  TP_CONV_FILTER = 2    /* out = out_scale (conv + b) as float2 (13, batch*nf*nb) */
};

TP_API size_t tp_cnn_act_bytes(int32_t nf, int32_t nb, int32_t batch, int32_t channels);
/* 16 feature channels of `batch` diagonals d (float2 (batch, nf*nb)). */
TP_API int tp_cnn_features(int32_t nf, int32_t nb, int32_t batch, const void *diag, float kappa, void *feat,
                           tp_stream_t stream);
/* One 3x3 layer, cin in {16, 32} (TP_CONV_RELU) or 32 (MASK, FILTER). */
TP_API int tp_conv3x3_bf16(int32_t nf, int32_t nb, int32_t batch, int32_t cin, int32_t epilogue, const void *in,
                           const void *weights, const float *bias, const void *aux, void *out, float out_scale,
                           tp_stream_t stream);
/* dw[tap][c][o] += sum_q x[q+o_tap][c] dy[q][o] (fp32 (9, cin, 32)); db[o] += sum_q dy[q][o] (db may be NULL). */
TP_API int tp_conv3x3_wgrad(int32_t nf, int32_t nb, int32_t batch, int32_t cin, const void *x, const void *dy,
                            float *dw, float *db, tp_stream_t stream);
/* y_v = z_v + sum_t F_t z_v(x + o_t) for nvec vectors (nvec, nf*nb) float2;
 * vector v uses filter image v / per_image (per_image = 0: image 0 for all);
 * conj != 0 applies conj(F) (the adjoint modes). */
TP_API int tp_cnn_filter_apply(int32_t nf, int32_t nb, int32_t nvec, int32_t per_image, int32_t conj,
                               const void *filt, const void *z, void *y, tp_stream_t stream);
/* Last-layer gradient (bf16, 32 channels, padded-linear) of
 * sum_v |y_v - t_v|^2 s_v given e_v = s_v (y_v - t_v):
 * 2 out_scale conj(z_v(x+o_t)) e_v(x) summed over the per_image vectors of
 * each of the nimg filter images. */
TP_API int tp_cnn_filter_grad(int32_t nf, int32_t nb, int32_t nimg, int32_t per_image, const void *z, const void *e,
                              float out_scale, void *dy, tp_stream_t stream);
/* Whole forward (features, 4 layers) of `batch` diagonals into the filter. */
TP_API size_t tp_cnn_forward_ws_bytes(int32_t nf, int32_t nb, int32_t batch);
TP_API int tp_cnn_forward(int32_t nf, int32_t nb, int32_t batch, const tp_cnn_model *model, const void *diag,
                          void *ws, size_t ws_bytes, void *filt, tp_stream_t stream);

/* Synchronise `stream` and report device-side failures of earlier launches
 * (a bounded wait that gave up).  Returns TP_ERR_TIMEOUT and clears the flag
 * when one was recorded; *code receives the raw device code (0 = none). */
TP_API int tp_device_status(tp_stream_t stream, int32_t *code);

/* Message of the last failed call on this thread ("" if none). */
TP_API const char *tp_last_error_string(void);

/* Library version (major*10000 + minor*100 + patch). */
TP_API int tp_version(void);

#ifdef __cplusplus
}
#endif
#endif /* TPCUDA_H */
