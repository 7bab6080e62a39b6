// Shared-memory mixed-radix (8, 4, 2, 3, 5) Stockham FFT for one CTA.
//
// A transform of length n = 2^a 3^b 5^c lives in shared memory; each pass of
// radix R reads R values with stride n/R, applies the twiddles
// W_{Ns R}^{r k} (k = j mod Ns, Ns = product of the previous radices), does
// an R-point DFT in registers and writes them with stride Ns (autosort, so
// the result is in natural order without a bit-reversal pass).  Twiddles
// W_n^t = exp(-2 pi i t / n) are computed once per CTA in fp64 into shared
// memory.  Both directions are unnormalised (the inverse is n times
// numpy.fft.ifft); callers fold the 1/n into an adjacent multiply.
#pragma once

#include "tp_common.cuh"

namespace tp {

constexpr int kFftMaxPasses = 12;
constexpr int kFftMaxN = 4096;

struct FftPlan {
  int n;
  int npass;
  int radix[kFftMaxPasses];
};

// Host: radices of n (8s first, then 4, 2, 3, 5); npass = 0 if unsupported.
inline FftPlan make_fft_plan(int n) {
  FftPlan p{};
  p.n = n;
  int m = n, k = 0;
  if (n < 1 || n > kFftMaxN) return p;
  while (m % 8 == 0 && k < kFftMaxPasses) { p.radix[k++] = 8; m /= 8; }
  while (m % 4 == 0 && k < kFftMaxPasses) { p.radix[k++] = 4; m /= 4; }
  while (m % 2 == 0 && k < kFftMaxPasses) { p.radix[k++] = 2; m /= 2; }
  while (m % 3 == 0 && k < kFftMaxPasses) { p.radix[k++] = 3; m /= 3; }
  while (m % 5 == 0 && k < kFftMaxPasses) { p.radix[k++] = 5; m /= 5; }
  p.npass = (m == 1) ? k : 0;
  return p;
}

__device__ __forceinline__ void fft_twiddles(cx *tw, int n, int tid, int nth) {
  for (int t = tid; t < n; t += nth) {
    double s, c;
    sincospi(-2.0 * (double)t / (double)n, &s, &c);
    tw[t] = mkcx((rx)c, (rx)s);
  }
}

// R-point DFT in place (sign = -1 forward, +1 inverse).
template <int R>
__device__ __forceinline__ void dft_small(cx (&v)[8], rx sign);

template <>
__device__ __forceinline__ void dft_small<2>(cx (&v)[8], rx) {
  const cx a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

// multiply by sign*i
__device__ __forceinline__ cx mul_si(cx z, rx sign) { return mkcx(-sign * z.y, sign * z.x); }

template <>
__device__ __forceinline__ void dft_small<4>(cx (&v)[8], rx sign) {
  const cx a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
  const cx b0 = cadd(v[1], v[3]), b1 = mul_si(csub(v[1], v[3]), sign);
  v[0] = cadd(a0, b0);
  v[2] = csub(a0, b0);
  v[1] = cadd(a1, b1);
  v[3] = csub(a1, b1);
}

template <>
__device__ __forceinline__ void dft_small<8>(cx (&v)[8], rx sign) {
  const rx h = TP_R(0.70710678118654752440);  // 1/sqrt(2)
  cx e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  // 4-point DFTs of the even and odd samples
  cx a0 = cadd(e[0], e[2]), a1 = csub(e[0], e[2]), b0 = cadd(e[1], e[3]), b1 = mul_si(csub(e[1], e[3]), sign);
  e[0] = cadd(a0, b0); e[2] = csub(a0, b0); e[1] = cadd(a1, b1); e[3] = csub(a1, b1);
  a0 = cadd(o[0], o[2]); a1 = csub(o[0], o[2]); b0 = cadd(o[1], o[3]); b1 = mul_si(csub(o[1], o[3]), sign);
  o[0] = cadd(a0, b0); o[2] = csub(a0, b0); o[1] = cadd(a1, b1); o[3] = csub(a1, b1);
  // twiddles W8^k = exp(sign * i * pi k / 4)
  const cx w1 = mkcx(h, sign * h), w3 = mkcx(-h, sign * h);
  o[1] = cmul(o[1], w1);
  o[2] = mul_si(o[2], sign);
  o[3] = cmul(o[3], w3);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cadd(e[k], o[k]);
    v[k + 4] = csub(e[k], o[k]);
  }
}

// 4-point DFT of (a0, a1, a2, a3) in place, X_m = sum_r a_r exp(sign 2 pi i r m / 4).
__device__ __forceinline__ void dft4_inplace(cx &a0, cx &a1, cx &a2, cx &a3, rx sign) {
  const cx s02 = cadd(a0, a2), d02 = csub(a0, a2), s13 = cadd(a1, a3);
  const cx jd13 = mul_si(csub(a1, a3), sign);
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, jd13);
  a3 = csub(d02, jd13);
}

// 16-point DFT as 4 x 4: with n = 4 n1 + n2 and m = k1 + 4 k2,
// X_m = sum_n2 W16^{n2 k1} W4^{n2 k2} sum_n1 x_{4 n1 + n2} W4^{n1 k1}:
// DFT-4 over n1 for every n2, twiddles W16^{n2 k1}, DFT-4 over n2 for every
// k1, then the 4 x 4 transpose of the output order.
__device__ __forceinline__ void dft16(cx (&v)[16], rx sign) {
  // cos and sin of 2 pi m / 16, m = 0..9 (the twiddle exponents n2 k1 used)
  constexpr rx kc[10] = {TP_R(1.0), TP_R(0.92387953251128675613), TP_R(0.70710678118654752440), TP_R(0.38268343236508977173), TP_R(0.0),
                            -TP_R(0.38268343236508977173), -TP_R(0.70710678118654752440), -TP_R(0.92387953251128675613), -TP_R(1.0),
                            -TP_R(0.92387953251128675613)};
  constexpr rx ks[10] = {TP_R(0.0), TP_R(0.38268343236508977173), TP_R(0.70710678118654752440), TP_R(0.92387953251128675613), TP_R(1.0),
                            TP_R(0.92387953251128675613), TP_R(0.70710678118654752440), TP_R(0.38268343236508977173), TP_R(0.0),
                            -TP_R(0.38268343236508977173)};
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) dft4_inplace(v[n2], v[4 + n2], v[8 + n2], v[12 + n2], sign);
  // now v[4 k1 + n2] holds the inner DFT for (n2, k1)
#pragma unroll
  for (int k1 = 1; k1 < 4; ++k1)
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2) {
      const int m = n2 * k1;
      v[4 * k1 + n2] = cmul(v[4 * k1 + n2], mkcx(kc[m], sign * ks[m]));
    }
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4_inplace(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3], sign);
  // v[4 k1 + k2] holds X_{k1 + 4 k2}: transpose
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = r + 1; c < 4; ++c) {
      const cx t = v[4 * r + c];
      v[4 * r + c] = v[4 * c + r];
      v[4 * c + r] = t;
    }
}

template <>
__device__ __forceinline__ void dft_small<3>(cx (&v)[8], rx sign) {
  const rx s3 = TP_R(0.86602540378443864676);  // sin(2 pi / 3)
  const cx t = cadd(v[1], v[2]);
  const cx d = mul_si(csub(v[1], v[2]), sign * s3);
  const cx m = mkcx(v[0].x - TP_R(0.5) * t.x, v[0].y - TP_R(0.5) * t.y);
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, d);
  v[2] = csub(m, d);
}

template <>
__device__ __forceinline__ void dft_small<5>(cx (&v)[8], rx sign) {
  const rx c1 = TP_R(0.30901699437494742410), c2 = -TP_R(0.80901699437494742410);  // cos(2pi/5), cos(4pi/5)
  const rx s1 = TP_R(0.95105651629515357212), s2 = TP_R(0.58778525229247312917);   // sin(2pi/5), sin(4pi/5)
  const cx a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  const cx a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  const cx x0 = v[0];
  const cx m1 = mkcx(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
  const cx m2 = mkcx(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
  const cx n1 = mul_si(mkcx(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), sign);
  const cx n2 = mul_si(mkcx(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), sign);
  v[0] = cadd(x0, cadd(a1, a2));
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

template <int R>
__device__ __forceinline__ void fft_pass(const cx *a, cx *b, int n, int Ns, const cx *tw, rx sign,
                                         int nb, int tid, int nth) {
  const int T = n / R;
  const int step = n / (Ns * R);
  for (int w = tid; w < nb * T; w += nth) {
    const int bi = w / T, j = w - bi * T;
    const cx *src = a + bi * n;
    cx *dst = b + bi * n;
    const int k = j % Ns;
    cx v[8];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[j + r * T];
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const cx t = tw[(r * k * step) % n];
      v[r] = cmul(v[r], mkcx(t.x, sign < 0 ? t.y : -t.y));
    }
    dft_small<R>(v, sign);
    const int idx = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[idx + r * Ns] = v[r];
  }
}

// ------------------------------------------------------ fixed-size plans
// The same passes with the length and the radix sequence known at compile
// time, so that every index division and modulo is by a constant.  Used by
// the 3D preconditioner for the common transverse sizes.
template <int N, int Ns, int R>
__device__ __forceinline__ void fft_pass_fixed(const cx *a, cx *b, const cx *tw, rx sign, int nb, int tid,
                                               int nth) {
  constexpr int T = N / R;
  constexpr int step = N / (Ns * R);
  for (int w = tid; w < nb * T; w += nth) {
    const int bi = w / T, j = w - bi * T;
    const cx *src = a + bi * N;
    cx *dst = b + bi * N;
    const int k = j % Ns;
    cx v[R > 8 ? 16 : 8];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[j + r * T];
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const cx t = tw[(r * k * step) % N];
      v[r] = cmul(v[r], mkcx(t.x, sign < 0 ? t.y : -t.y));
    }
    if constexpr (R == 16) dft16(v, sign);
    else dft_small<R>(v, sign);
    const int idx = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[idx + r * Ns] = v[r];
  }
}

template <int N, int Ns, int R, int... Rest>
__device__ __forceinline__ cx *fft_run_fixed(cx *a, cx *b, const cx *tw, rx sign, int nb, int tid,
                                                 int nth) {
  fft_pass_fixed<N, Ns, R>(a, b, tw, sign, nb, tid, nth);
  __syncthreads();
  if constexpr (sizeof...(Rest) == 0) {
    return b;
  } else {
    return fft_run_fixed<N, Ns * R, Rest...>(b, a, tw, sign, nb, tid, nth);
  }
}

// Padded shared-memory layout of the fixed-size transforms: element i of a
// transform sits at i + i/8 (one spare slot per 8 elements) and transform bi
// starts at bi * S, S = N + N/8 + 1.  The Stockham writes of the early passes
// (stride R elements) and column transposes (stride S) then spread over the
// shared-memory banks instead of hitting a few of them.
template <int N>
struct FftPad {
  static constexpr int S = N + N / 8 + 1;
};
__device__ __forceinline__ int fft_pad(int i) { return i + (i >> 3); }

template <int N, int Ns, int R>
__device__ __forceinline__ void fft_pass_padded(const cx *a, cx *b, const cx *tw, rx sign, int nb, int tid,
                                                int nth) {
  constexpr int T = N / R;
  constexpr int step = N / (Ns * R);
  constexpr int S = FftPad<N>::S;
  for (int w = tid; w < nb * T; w += nth) {
    const int bi = w / T, j = w - bi * T;
    const cx *src = a + bi * S;
    cx *dst = b + bi * S;
    const int k = j % Ns;
    cx v[R > 8 ? 16 : 8];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[fft_pad(j + r * T)];
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const cx t = tw[(r * k * step) % N];
      v[r] = cmul(v[r], mkcx(t.x, sign < 0 ? t.y : -t.y));
    }
    if constexpr (R == 16) dft16(v, sign);
    else dft_small<R>(v, sign);
    const int idx = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[fft_pad(idx + r * Ns)] = v[r];
  }
}

template <int N, int Ns, int R, int... Rest>
__device__ __forceinline__ cx *fft_run_padded(cx *a, cx *b, const cx *tw, rx sign, int nb, int tid,
                                                  int nth) {
  fft_pass_padded<N, Ns, R>(a, b, tw, sign, nb, tid, nth);
  __syncthreads();
  if constexpr (sizeof...(Rest) == 0) {
    return b;
  } else {
    return fft_run_padded<N, Ns * R, Rest...>(b, a, tw, sign, nb, tid, nth);
  }
}

// Lengths with a compile-time plan (radix 16 for 128 and 256, else 8s first,
// then 4, 2, 3).
// (fft_block_fixed also has a 2048 plan, 16 * 16 * 8, for callers that select
// it themselves; the padded layout and the callers of fft_fixed_size do not.)
__host__ __device__ constexpr bool fft_fixed_size(int n) {
  return n == 32 || n == 64 || n == 128 || n == 192 || n == 256 || n == 512;
}

template <int N>
__device__ __forceinline__ cx *fft_block_fixed(cx *a, cx *b, const cx *tw, bool inverse, int nb,
                                                   int tid, int nth) {
  const rx sign = inverse ? TP_R(1.0) : -TP_R(1.0);
  if constexpr (N == 32) return fft_run_fixed<32, 1, 8, 4>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 64) return fft_run_fixed<64, 1, 8, 8>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 128) return fft_run_fixed<128, 1, 8, 16>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 192) return fft_run_fixed<192, 1, 8, 8, 3>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 256) return fft_run_fixed<256, 1, 16, 16>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 2048) return fft_run_fixed<2048, 1, 16, 16, 8>(a, b, tw, sign, nb, tid, nth);
  else return fft_run_fixed<512, 1, 8, 8, 8>(a, b, tw, sign, nb, tid, nth);
}

// The fixed-size transforms in the padded layout (FftPad).
template <int N>
__device__ __forceinline__ cx *fft_block_padded(cx *a, cx *b, const cx *tw, bool inverse, int nb,
                                                    int tid, int nth) {
  const rx sign = inverse ? TP_R(1.0) : -TP_R(1.0);
  if constexpr (N == 32) return fft_run_padded<32, 1, 8, 4>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 64) return fft_run_padded<64, 1, 8, 8>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 128) return fft_run_padded<128, 1, 8, 16>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 192) return fft_run_padded<192, 1, 8, 8, 3>(a, b, tw, sign, nb, tid, nth);
  else if constexpr (N == 256) return fft_run_padded<256, 1, 16, 16>(a, b, tw, sign, nb, tid, nth);
  else return fft_run_padded<512, 1, 8, 8, 8>(a, b, tw, sign, nb, tid, nth);
}

// nb transforms of length pl.n stored back to back in `a` (scratch `b` of
// the same size).  Returns the buffer holding the result (a or b).  Ends
// with __syncthreads().
__device__ __forceinline__ cx *fft_block(cx *a, cx *b, const FftPlan &pl, const cx *tw, bool inverse,
                                             int nb, int tid, int nth) {
  const rx sign = inverse ? TP_R(1.0) : -TP_R(1.0);
  int Ns = 1;
  for (int ps = 0; ps < pl.npass; ++ps) {
    const int R = pl.radix[ps];
    switch (R) {
      case 8: fft_pass<8>(a, b, pl.n, Ns, tw, sign, nb, tid, nth); break;
      case 4: fft_pass<4>(a, b, pl.n, Ns, tw, sign, nb, tid, nth); break;
      case 2: fft_pass<2>(a, b, pl.n, Ns, tw, sign, nb, tid, nth); break;
      case 3: fft_pass<3>(a, b, pl.n, Ns, tw, sign, nb, tid, nth); break;
      default: fft_pass<5>(a, b, pl.n, Ns, tw, sign, nb, tid, nth); break;
    }
    __syncthreads();
    cx *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// FFT of `rows` transforms of length n in shared memory: the compile-time
// plan in the padded layout when N > 0, else the runtime plan `pl`
// (unpadded).  Whole-CTA call.
template <int N>
__device__ __forceinline__ cx *fft_rows(cx *a, cx *b, const FftPlan &pl, const cx *tw, bool inverse,
                                            int rows) {
  if constexpr (N > 0) return fft_block_padded<N>(a, b, tw, inverse, rows, threadIdx.x, blockDim.x);
  else return fft_block(a, b, pl, tw, inverse, rows, threadIdx.x, blockDim.x);
}

// Shared-memory slot of element i of transform bi (length n).
template <int N>
__device__ __forceinline__ int fslot(int bi, int i, int n) {
  if constexpr (N > 0) return bi * FftPad<N>::S + fft_pad(i);
  else return bi * n + i;
}
// Shared-memory slots per transform.
template <int N>
__host__ __device__ constexpr int fstride(int n) {
  if constexpr (N > 0) return FftPad<N>::S;
  else return n;
}

__device__ __forceinline__ void load_twiddles(cx *tw, const cx *__restrict__ twg, int n) {
  for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twg[t];
}

// ------------------------------------------------ register four-step transforms
// A transform of length N = R1 * R2 with the short DFTs held in registers:
// with n = R2 n1 + n2 and k = k1 + R1 k2,
//   X[k1 + R1 k2] = sum_n2 W_R2^{n2 k2} W_N^{n2 k1} sum_n1 x[R2 n1 + n2] W_R1^{n1 k1}.
// Stage A (one thread per n2): the R1-point DFT over n1 in registers, the
// twiddles W_N^{n2 k1}, one write to shared memory; stage C (one thread per
// k1): one read, the R2-point DFT over n2, giving X[k1 + R1 k2].  An element
// passes through shared memory once (one write, one read) instead of once per
// Stockham pass plus the staging copies.  The inverse runs the stages in the
// opposite order with conjugate twiddles.  The twiddle table is padded like
// the transpose: W_N^{n2 k1} at k1 * (R2 + 1) + n2, so that both stages read
// it without bank conflicts.

// 12-point DFT as 4 x 3 (n = 3 n1 + n2, k = k1 + 4 k2), natural order in and out.
__device__ __forceinline__ void dft12(cx (&v)[16], rx sign) {
  const rx s3 = TP_R(0.86602540378443864676);  // sin(pi / 3)
  cx y[12];
#pragma unroll
  for (int n2 = 0; n2 < 3; ++n2) {
    cx a0 = v[n2], a1 = v[3 + n2], a2 = v[6 + n2], a3 = v[9 + n2];
    dft4_inplace(a0, a1, a2, a3, sign);
    y[4 * n2] = a0;
    y[4 * n2 + 1] = a1;
    y[4 * n2 + 2] = a2;
    y[4 * n2 + 3] = a3;
  }
  // W12^m = exp(sign 2 pi i m / 12) for m = n2 k1 in {1, 2, 3, 2, 4, 6}
  const cx w1 = mkcx(s3, sign * TP_R(0.5)), w2 = mkcx(TP_R(0.5), sign * s3), w3 = mkcx(TP_R(0.0), sign);
  const cx w4 = mkcx(-TP_R(0.5), sign * s3), w6 = mkcx(-TP_R(1.0), TP_R(0.0));
  y[5] = cmul(y[5], w1);
  y[6] = cmul(y[6], w2);
  y[7] = cmul(y[7], w3);
  y[9] = cmul(y[9], w2);
  y[10] = cmul(y[10], w4);
  y[11] = cmul(y[11], w6);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    const cx a = y[k1], b = y[4 + k1], c = y[8 + k1];
    const cx t = cadd(b, c);
    const cx d = mul_si(csub(b, c), sign * s3);
    const cx m = mkcx(a.x - TP_R(0.5) * t.x, a.y - TP_R(0.5) * t.y);
    v[k1] = cadd(a, t);
    v[k1 + 4] = cadd(m, d);
    v[k1 + 8] = csub(m, d);
  }
}

// R-point DFT (R = 4, 8, 12, 16) of v[0..R) in registers, natural order in and out.
template <int R>
__device__ __forceinline__ void dft_reg(cx (&v)[16], rx sign) {
  static_assert(R == 4 || R == 8 || R == 12 || R == 16, "dft_reg: unsupported length");
  if constexpr (R == 16) {
    dft16(v, sign);
  } else if constexpr (R == 12) {
    dft12(v, sign);
  } else if constexpr (R == 8) {
    cx w[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) w[j] = v[j];
    dft_small<8>(w, sign);
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = w[j];
  } else {
    dft4_inplace(v[0], v[1], v[2], v[3], sign);
  }
}

// Factors of the lengths with a four-step plan (R1 >= R2, both <= 16).
__host__ __device__ constexpr int four_r1(int n) { return n == 64 ? 8 : 16; }
__host__ __device__ constexpr int four_r2(int n) { return n / four_r1(n); }
__host__ __device__ constexpr bool four_step_size(int n) { return n == 64 || n == 128 || n == 192 || n == 256; }
// Entries of the padded twiddle table.
__host__ __device__ constexpr int four_tw_len(int n) { return four_r1(n) * (four_r2(n) + 1); }

}  // namespace tp
