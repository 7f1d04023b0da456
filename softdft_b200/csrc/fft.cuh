// fft.cuh -- CTA-wide DCT-II / inverse-DCT-II of P real points through one
// complex FFT of M = P/2 points held in shared memory, several transforms at
// a time.
//
// The reference convolves every field on a mirrored, doubled grid of 2P
// points with complex FFTs (src/iDFT/coordinate_system/Cartesian/process_fourier.jl:15-49,
// utilities/apply_mirroring.jl:1-23).  For the half-sample-even extension
// x_ext = [x_0..x_{P-1}, x_{P-1}..x_0] the 2P-point FFT is
//     X[k] = 2 e^{i pi k / 2P} C[k],   C[k] = sum_n x_n cos(pi k (2n+1) / 2P),
// so multiplying by a real even weight W and inverting is exactly
//     y = iDCT2(W C),   iDCT2(E)[m] = (1/P) [E_0 + 2 sum_{k>=1} E_k cos(pi k (2m+1) / 2P)].
// Odd (vector) weights map to the same pair with a reversed coefficient index
// and a (-1)^m sign (see objective.cuh).  DCT-II of P points is computed with
// Makhoul's reordering and a real FFT of P points, i.e. a complex FFT of P/2
// points (J. Makhoul, IEEE TASSP 28(1), 1980).
//
// Shared memory holds TB transform buffers of M complex values each, padded by
// one slot every 8 (index i lives at i + i/8) so that the strided accesses of
// the butterfly passes fall on different banks.  Forward: the load scatters into
// bit-reversed order and radix-8/4/2 decimation-in-time passes (three radix-2
// stages per pass, in registers) leave natural order.  Inverse: radix-8/4/2
// decimation-in-frequency passes take natural order and leave bit-reversed
// order, undone by the gather of the store.  A length M that is not a power of
// two runs mixed-radix passes instead (radices 4, 2, 3, 5, 7 and primes up to
// kMaxGenRadix) with a digit-reversed load and store.  The DCT twiddle step only couples
// Z[k] and Z[M-k], so a convolution is: load, FFT, one in-place pair pass that
// also applies the weight, IFFT, store.
//
// Batched entry points run nT <= TB independent transforms in the same passes
// (transform t uses buffer t); the functors take the transform index.
#pragma once

#include "common.cuh"

// SDFT_FFT_GEN selects the transform passes a translation unit carries: 0 for
// power-of-two M, 1 for a general M (see kernels.cuh)
#ifndef SDFT_FFT_GEN
#error "define SDFT_FFT_GEN (0: power-of-two FFT lengths, 1: general lengths) before including fft.cuh"
#endif

namespace sdft {
namespace {  // internal linkage: each kernel build (kernels.cuh) has its own copy

__device__ __forceinline__ int brev_bits(int m, int L) {
  return L == 0 ? 0 : (int)(__brev((unsigned)m) >> (32 - L));
}

// C = double2 (FP64) or float2 (the mixed-precision propagator convolutions)
template <class C>
struct FftCtxT {
  C* z;              // TB buffers of `stride` slots
  int stride;        // M + M/8
  int P, M, L, H;    // H = M/2
  int nrad;          // general length: mixed-radix passes over rad[0 .. nrad-1]
  const int* rad;
  const int* __restrict__ slot;  // general length: digit-reversed slot of natural index m
  const C* __restrict__ tw;   // [M/2] e^{-2 pi i k / M} ([M] for a general length)
  const C* __restrict__ twP;  // [M+1] e^{-2 pi i k / P}
  const C* __restrict__ twD;  // [M+1] e^{-i pi k / 2P}
  int blue;                   // general length: Bluestein transform (a prime factor above kMaxGenRadix)
  int LB, lLB;                // Bluestein convolution length 2^lLB >= 2M - 1
  const C* __restrict__ bw;   // [M] chirp e^{-i pi n^2 / M}
  const C* __restrict__ bB;   // [LB] chirp filter spectrum / LB, bit-reversed order
  const C* __restrict__ btw;  // [LB/2] e^{-2 pi i k / LB}
};
using FftCtx = FftCtxT<double2>;

__device__ __forceinline__ FftCtx make_fft(double2* z, const DReq& r) {
  FftCtx c;
  c.z = z;
  c.M = r.M;
  c.L = r.L;
  c.P = r.NPt;
  c.H = r.M >> 1;
  c.stride = fft_buffer_len(r.M);
  c.nrad = r.nrad;
  c.rad = r.rad;
  c.slot = r.slot;
  c.tw = r.tw;
  c.twP = r.twP;
  c.twD = r.twD;
  c.blue = r.blue;
  c.LB = r.LB;
  c.lLB = r.lLB;
  c.bw = r.bw;
  c.bB = r.bB;
  c.btw = r.btw;
  if (r.blue) c.stride = fft_buffer_len(r.LB);
  return c;
}

// FP32 transform buffers over the same shared memory
__device__ __forceinline__ FftCtxT<float2> make_fft32(double2* z, const DReq& r) {
  FftCtxT<float2> c;
  c.z = reinterpret_cast<float2*>(z);
  c.M = r.M;
  c.L = r.L;
  c.P = r.NPt;
  c.H = r.M >> 1;
  c.stride = fft_buffer_len(r.M);
  c.nrad = r.nrad;
  c.rad = r.rad;
  c.slot = r.slot;
  c.tw = r.tw32;
  c.twP = r.twP32;
  c.twD = r.twD32;
  c.blue = r.blue;
  c.LB = r.LB;
  c.lLB = r.lLB;
  c.bw = r.bw32;
  c.bB = r.bB32;
  c.btw = r.btw32;
  if (r.blue) c.stride = fft_buffer_len(r.LB);
  return c;
}

// The loops below come in two instantiations: G = false for power-of-two M
// (bit reversal, shifts), G = true for a general M (digit-reversal table,
// divisions); the entry points instantiate the one SDFT_FFT_GEN selects.

// buffer slot of natural complex index m
template <bool G, class C>
__device__ __forceinline__ int fslot(const FftCtxT<C>& c, int m) {
  if constexpr (G)
    return __ldg(&c.slot[m]);
  else
    return brev_bits(m, c.L);
}

// transform index of item it, n items per transform (n = 2^ln when !G)
template <bool G>
__device__ __forceinline__ int item_t(int it, int n, int ln) {
  if constexpr (G)
    return it / n;
  else
    return it >> ln;
}

// position of real sample K in the packed complex buffer: (slot, component)
template <bool G, class C>
__device__ __forceinline__ void dct_slot(const FftCtxT<C>& c, int K, int* pos, int* comp) {
  int q = (K & 1) ? (c.P - 1 - (K >> 1)) : (K >> 1);  // Makhoul reorder v[q]
  *pos = fslot<G>(c, q >> 1);
  *comp = q & 1;
}

template <bool G, class F>
__device__ __forceinline__ void load_b(const FftCtx& c, int nT, F f) {
  const int lp = c.L + 1;  // log2 P
  for (int it = threadIdx.x; it < nT * c.P; it += blockDim.x) {
    const int t = item_t<G>(it, c.P, lp), K = it - t * c.P;
    int pos, comp;
    dct_slot<G>(c, K, &pos, &comp);
    reinterpret_cast<double*>(c.z + (size_t)t * c.stride + fpad(pos))[comp] = f(t, K);
  }
}

template <bool G, class S>
__device__ __forceinline__ void store_b(const FftCtx& c, int nT, double scale, S st) {
  const int lp = c.L + 1;
  for (int it = threadIdx.x; it < nT * c.P; it += blockDim.x) {
    const int t = item_t<G>(it, c.P, lp), K = it - t * c.P;
    int pos, comp;
    dct_slot<G>(c, K, &pos, &comp);
    st(t, K, reinterpret_cast<const double*>(c.z + (size_t)t * c.stride + fpad(pos))[comp] * scale);
  }
}

// ---- grid-point pairs: the (K, K+1) samples of a transform moved together ----
// Pair kp covers K = 2 kp (Makhoul index q = kp) and K + 1 (q = P - 1 - kp);
// the functors read and write both samples with 16-byte accesses.  Each round
// of a thread handles two pairs whose global loads are issued first.
__device__ __forceinline__ double2 ldcg2(const double* p) { return __ldcg(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ void stcg2(double* p, double2 v) { __stcg(reinterpret_cast<double2*>(p), v); }
__device__ __forceinline__ float2 ldcg2(const float* p) { return __ldcg(reinterpret_cast<const float2*>(p)); }
// L1-cached pair loads (ld.global.ca) for arrays that one CTA reads repeatedly
// after writing them earlier in the same kernel: the SM's L1 sees its own writes
__device__ __forceinline__ double2 ldca2(const double* p) { return __ldca(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ float2 ldca2(const float* p) { return __ldca(reinterpret_cast<const float2*>(p)); }
__device__ __forceinline__ void stcg2(float* p, float2 v) { __stcg(reinterpret_cast<float2*>(p), v); }

template <bool G, class C, class V>
__device__ __forceinline__ void put_pair(const FftCtxT<C>& c, int t, int kp, V v) {
  using R = typename Cx<C>::R;
  R* zb = reinterpret_cast<R*>(c.z + (size_t)t * c.stride);
  const int q1 = c.P - 1 - kp;
  zb[2 * fpad(fslot<G>(c, kp >> 1)) + (kp & 1)] = (R)v.x;
  zb[2 * fpad(fslot<G>(c, q1 >> 1)) + (q1 & 1)] = (R)v.y;
}
template <bool G, class C>
__device__ __forceinline__ C get_pair(const FftCtxT<C>& c, int t, int kp) {
  using R = typename Cx<C>::R;
  const R* zb = reinterpret_cast<const R*>(c.z + (size_t)t * c.stride);
  const int q1 = c.P - 1 - kp;
  return Cx<C>::make(zb[2 * fpad(fslot<G>(c, kp >> 1)) + (kp & 1)], zb[2 * fpad(fslot<G>(c, q1 >> 1)) + (q1 & 1)]);
}

// f2(t, K) -> (f(K), f(K+1)) for even K
template <bool G, class C, class F2>
__device__ __forceinline__ void load_b2(const FftCtxT<C>& c, int nT, F2 f2) {
  const int lm = c.L, M = c.M;
  const int total = nT * M;
  for (int b0 = threadIdx.x; b0 < total; b0 += 2 * blockDim.x) {
    const int i1 = b0 + blockDim.x;
    const int t0 = item_t<G>(b0, M, lm), k0 = b0 - t0 * M;
    const int t1 = item_t<G>(i1, M, lm), k1 = i1 - t1 * M;
    const auto v0 = f2(t0, k0 << 1);
    auto v1 = v0;
    if (i1 < total) v1 = f2(t1, k1 << 1);
    put_pair<G>(c, t0, k0, v0);
    if (i1 < total) put_pair<G>(c, t1, k1, v1);
  }
}

// put2(t, K, (y_K, y_K+1) * scale, pre2(t, K)) for even K; pre2 holds the loads
template <bool G, class C, class A2, class S2>
__device__ __forceinline__ void store_b2(const FftCtxT<C>& c, int nT, typename Cx<C>::R scale, A2 pre2, S2 put2) {
  const int lm = c.L, M = c.M;
  const int total = nT * M;
  for (int b0 = threadIdx.x; b0 < total; b0 += 2 * blockDim.x) {
    const int i1 = b0 + blockDim.x;
    const int t0 = item_t<G>(b0, M, lm), K0 = (b0 - t0 * M) << 1;
    C y0 = get_pair<G>(c, t0, K0 >> 1);
    const auto a0 = pre2(t0, K0);
    C y1 = y0;
    auto a1 = a0;
    const int t1 = item_t<G>(i1, M, lm), K1 = (i1 - t1 * M) << 1;
    if (i1 < total) {
      y1 = get_pair<G>(c, t1, K1 >> 1);
      a1 = pre2(t1, K1);
    }
    y0.x *= scale;
    y0.y *= scale;
    put2(t0, K0, y0, a0);
    if (i1 < total) {
      y1.x *= scale;
      y1.y *= scale;
      put2(t1, K1, y1, a1);
    }
  }
}

template <class C>
__device__ __forceinline__ void bfly(C& a, C& b, C w) {  // DIT: (a + wb, a - wb)
  const C wb = cmul(b, w);
  b = sub2(a, wb);
  a = add2(a, wb);
}
template <class C>
__device__ __forceinline__ void bfly_dif(C& a, C& b, C w) {  // DIF: (a + b, (a - b) w)
  const C d = sub2(a, b);
  a = add2(a, b);
  b = cmul(d, w);
}

// ---- general length M --------------------------------------------------------
// M = r_0 r_1 ... r_{s-1} with radices 4, 2, 3, 5, 7, 11, 13 and primes up to
// kMaxGenRadix.  Forward: in-place decimation in time over stages of growing
// span m = r_0 ... r_{i-1}; the butterfly (group g, offset j < m) takes
// x_q = z[g m r + j + q m] w_{m r}^{j q} (q < r) and writes its r-point DFT back to
// the same slots.  Its input order is the mixed-radix digit reversal: natural
// index n = d_0 M/r_0 + d_1 M/(r_0 r_1) + ... sits in slot d_0 + r_0 (d_1 + r_1 (...)),
// which the host tabulates as slot[n].  Inverse: the stages in reverse order as
// decimation in frequency (r-point inverse DFT, then the conjugate twiddles),
// natural order in, the same digit-reversed order out.  Roots of unity come
// from tw[k] = e^{-2 pi i k / M}: w_r^e = tw[e M / r].

// r-point DFT of an odd prime r in registers: x_q and x_{r-q} are paired,
// S_q = x_q + x_{r-q}, D_q = x_q - x_{r-q}, and for l = 1 .. (r-1)/2
//   X_l, X_{r-l} = A_l -+ i B_l,  A_l = x_0 + sum_q S_q cos(2 pi q l / r),
//   B_l = sum_q D_q sin(2 pi q l / r)   (signs swapped for the inverse),
// real weights only, a quarter of the multiplies of the plain sum
template <class C, int R>
__device__ __forceinline__ void dft_odd_prime(C* x, const C* __restrict__ tw, int step, bool inv) {
  using T = typename Cx<C>::R;
  constexpr int H = (R - 1) / 2;
  T cs[H + 1], sn[H + 1];
#pragma unroll
  for (int e = 1; e <= H; e++) {
    const C w = __ldg(&tw[e * step]);  // e^{-2 pi i e / r}
    cs[e] = w.x;
    sn[e] = -w.y;
  }
  C S[H], D[H];
#pragma unroll
  for (int q = 1; q <= H; q++) {
    S[q - 1] = add2(x[q], x[R - q]);
    D[q - 1] = sub2(x[q], x[R - q]);
  }
  C X0 = x[0];
#pragma unroll
  for (int q = 0; q < H; q++) X0 = add2(X0, S[q]);
#pragma unroll
  for (int l = 1; l <= H; l++) {
    C A = x[0], B = Cx<C>::make((T)0, (T)0);
#pragma unroll
    for (int q = 1; q <= H; q++) {
      const int e = (q * l) % R;
      const T cv = e <= H ? cs[e] : cs[R - e];
      const T sv = e <= H ? sn[e] : -sn[R - e];
      A = add2(A, scl2(S[q - 1], cv));
      B = add2(B, scl2(D[q - 1], sv));
    }
    const C iB = inv ? Cx<C>::make(-B.y, B.x) : Cx<C>::make(B.y, -B.x);  // +i B (inverse), -i B (forward)
    x[l] = add2(A, iB);
    x[R - l] = sub2(A, iB);
  }
  x[0] = X0;
}

// r-point DFT in registers (inv: conjugate roots), compile-time r
template <class C, int R>
__device__ __forceinline__ void dft_fixed(C* x, const C* __restrict__ tw, int step, bool inv) {
  if constexpr (R == 2) {
    const C a = x[0], b = x[1];
    x[0] = add2(a, b);
    x[1] = sub2(a, b);
  } else if constexpr (R == 4) {
    const C s02 = add2(x[0], x[2]), d02 = sub2(x[0], x[2]);
    const C s13 = add2(x[1], x[3]), d13 = sub2(x[1], x[3]);
    const C jd = inv ? Cx<C>::make(-d13.y, d13.x) : Cx<C>::make(d13.y, -d13.x);  // (+-i) d13
    x[0] = add2(s02, s13);
    x[2] = sub2(s02, s13);
    x[1] = add2(d02, jd);
    x[3] = sub2(d02, jd);
  } else {
    dft_odd_prime<C, R>(x, tw, step, inv);
  }
}

// the same paired DFT for an odd prime r known only at run time (r <= kMaxGenRadix)
template <class C>
__device__ __noinline__ void dft_any(C* x, int R, const C* __restrict__ tw, int step, bool inv) {
  using T = typename Cx<C>::R;
  constexpr int HM = (kMaxGenRadix - 1) / 2;
  const int H = (R - 1) / 2;
  C S[HM], D[HM];
  C X0 = x[0];
  for (int q = 1; q <= H; q++) {
    S[q - 1] = add2(x[q], x[R - q]);
    D[q - 1] = sub2(x[q], x[R - q]);
    X0 = add2(X0, S[q - 1]);
  }
  for (int l = 1; l <= H; l++) {
    C A = x[0], B = Cx<C>::make((T)0, (T)0);
    int e = 0;  // (q l) mod R
    for (int q = 1; q <= H; q++) {
      e += l;
      if (e >= R) e -= R;
      const C w = __ldg(&tw[e * step]);  // cos = w.x, sin = -w.y
      A = add2(A, scl2(S[q - 1], w.x));
      B = add2(B, scl2(D[q - 1], -w.y));
    }
    const C iB = inv ? Cx<C>::make(-B.y, B.x) : Cx<C>::make(B.y, -B.x);
    x[l] = add2(A, iB);
    x[R - l] = sub2(A, iB);
  }
  x[0] = X0;
}

// one stage of radix R (R = 0: run-time radix rr) and span m; DIT forward or DIF inverse
template <class C, int R>
__device__ __forceinline__ void gen_stage(const FftCtxT<C>& c, int nT, int m, int rr, bool inv) {
  constexpr int NX = R > 0 ? R : kMaxGenRadix;
  const int r = R > 0 ? R : rr;
  const int M = c.M, nb = M / r, tws = M / (m * r), step = M / r;
  for (int it = threadIdx.x; it < nT * nb; it += blockDim.x) {
    const int t = it / nb, b = it - t * nb;
    const int j = b % m, base = (b - j) * r + j;
    C* zb = c.z + (size_t)t * c.stride;
    C x[NX];
#pragma unroll
    for (int q = 0; q < NX; q++)
      if (q < r) x[q] = zb[fpad(base + q * m)];
    if (!inv) {
#pragma unroll
      for (int q = 1; q < NX; q++)
        if (q < r) x[q] = cmul(x[q], __ldg(&c.tw[j * q * tws]));
    }
    if (R > 0)
      dft_fixed<C, (R > 0 ? R : 2)>(x, c.tw, step, inv);
    else
      dft_any(x, r, c.tw, step, inv);
    if (inv) {
#pragma unroll
      for (int q = 1; q < NX; q++)
        if (q < r) x[q] = cmul(x[q], conj2(__ldg(&c.tw[j * q * tws])));
    }
#pragma unroll
    for (int q = 0; q < NX; q++)
      if (q < r) zb[fpad(base + q * m)] = x[q];
  }
}

template <class C>
__device__ __forceinline__ void gen_stage_any_radix(const FftCtxT<C>& c, int nT, int m, int r, bool inv) {
  switch (r) {
    case 2: gen_stage<C, 2>(c, nT, m, 2, inv); break;
    case 3: gen_stage<C, 3>(c, nT, m, 3, inv); break;
    case 4: gen_stage<C, 4>(c, nT, m, 4, inv); break;
    case 5: gen_stage<C, 5>(c, nT, m, 5, inv); break;
    case 7: gen_stage<C, 7>(c, nT, m, 7, inv); break;
    case 11: gen_stage<C, 11>(c, nT, m, 11, inv); break;
    case 13: gen_stage<C, 13>(c, nT, m, 13, inv); break;
    default: gen_stage<C, 0>(c, nT, m, r, inv); break;
  }
}

// general-length forward FFT: digit-reversed input -> natural output
template <class C>
__device__ __noinline__ void fft_gen_fwd(const FftCtxT<C> c, int nT) {
  int m = 1;
  for (int s = 0; s < c.nrad; s++) {
    const int r = c.rad[s];
    __syncthreads();
    gen_stage_any_radix(c, nT, m, r, false);
    m *= r;
  }
  __syncthreads();
}

// general-length inverse FFT (unscaled): natural input -> digit-reversed output
template <class C>
__device__ __noinline__ void fft_gen_inv(const FftCtxT<C> c, int nT) {
  int m = c.M;
  for (int s = c.nrad - 1; s >= 0; s--) {
    const int r = c.rad[s];
    m /= r;
    __syncthreads();
    gen_stage_any_radix(c, nT, m, r, true);
  }
  __syncthreads();
}

// ---- power-of-two pass sets over nT buffers of N = 2^lN points ----------------
// DIT: bit-reversed input -> natural output; DIF: natural input -> bit-reversed
// output.  tw[k] = e^{-2 pi i k / N} (k < N/2); CONJ uses the conjugate roots (an
// unscaled inverse transform).  Three radix-2 stages per pass (radix-8), a
// radix-4 or radix-2 pass takes the remainder of lN.
template <class C, bool CONJ>
__device__ __forceinline__ C tw_at(const C* __restrict__ tw, int k) {
  const C w = __ldg(&tw[k]);
  return CONJ ? conj2(w) : w;
}

template <class C, bool CONJ>
__device__ __forceinline__ void pow2_dit(C* z, int stride, int nT, int N, int L, const C* __restrict__ tw) {
  for (int s = 0; s < L;) {
    const int rr = min(3, L - s);
    const int h = 1 << s;
    __syncthreads();
    if (rr == 3) {
      const int per = N >> 3, lper = L - 3;
      for (int it = threadIdx.x; it < nT * per; it += blockDim.x) {
        const int t = it >> lper, u = it & (per - 1);
        C* zb = z + (size_t)t * stride;
        const int p = u & (h - 1);
        const int base = ((u >> s) << (s + 3)) + p;
        C x[8];
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = zb[fpad(base + j * h)];
        const C w1 = tw_at<C, CONJ>(tw, p << (L - 1 - s));
#pragma unroll
        for (int m = 0; m < 4; m++) bfly(x[2 * m], x[2 * m + 1], w1);
        const C w2a = tw_at<C, CONJ>(tw, p << (L - 2 - s));
        const C w2b = tw_at<C, CONJ>(tw, (p + h) << (L - 2 - s));
        bfly(x[0], x[2], w2a);
        bfly(x[1], x[3], w2b);
        bfly(x[4], x[6], w2a);
        bfly(x[5], x[7], w2b);
#pragma unroll
        for (int j = 0; j < 4; j++) bfly(x[j], x[j + 4], tw_at<C, CONJ>(tw, (p + j * h) << (L - 3 - s)));
#pragma unroll
        for (int j = 0; j < 8; j++) zb[fpad(base + j * h)] = x[j];
      }
    } else if (rr == 2) {
      const int per = N >> 2, lper = L - 2;
      for (int it = threadIdx.x; it < nT * per; it += blockDim.x) {
        const int t = it >> lper, u = it & (per - 1);
        C* zb = z + (size_t)t * stride;
        const int p = u & (h - 1);
        const int base = ((u >> s) << (s + 2)) + p;
        C x[4];
#pragma unroll
        for (int j = 0; j < 4; j++) x[j] = zb[fpad(base + j * h)];
        const C w1 = tw_at<C, CONJ>(tw, p << (L - 1 - s));
        bfly(x[0], x[1], w1);
        bfly(x[2], x[3], w1);
        bfly(x[0], x[2], tw_at<C, CONJ>(tw, p << (L - 2 - s)));
        bfly(x[1], x[3], tw_at<C, CONJ>(tw, (p + h) << (L - 2 - s)));
#pragma unroll
        for (int j = 0; j < 4; j++) zb[fpad(base + j * h)] = x[j];
      }
    } else {
      const int per = N >> 1, lper = L - 1;
      for (int it = threadIdx.x; it < nT * per; it += blockDim.x) {
        const int t = it >> lper, u = it & (per - 1);
        C* zb = z + (size_t)t * stride;
        const int p = u & (h - 1);
        const int base = ((u >> s) << (s + 1)) + p;
        C a = zb[fpad(base)], b = zb[fpad(base + h)];
        bfly(a, b, tw_at<C, CONJ>(tw, p << (L - 1 - s)));
        zb[fpad(base)] = a;
        zb[fpad(base + h)] = b;
      }
    }
    s += rr;
  }
  __syncthreads();
}

template <class C, bool CONJ>
__device__ __forceinline__ void pow2_dif(C* z, int stride, int nT, int N, int L, const C* __restrict__ tw) {
  for (int top = L; top > 0;) {
    const int rr = min(3, top);
    const int s0 = top - rr;
    const int h = 1 << s0;
    __syncthreads();
    if (rr == 3) {
      const int per = N >> 3, lper = L - 3;
      for (int it = threadIdx.x; it < nT * per; it += blockDim.x) {
        const int t = it >> lper, u = it & (per - 1);
        C* zb = z + (size_t)t * stride;
        const int p = u & (h - 1);
        const int base = ((u >> s0) << (s0 + 3)) + p;
        C x[8];
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = zb[fpad(base + j * h)];
#pragma unroll
        for (int j = 0; j < 4; j++) bfly_dif(x[j], x[j + 4], tw_at<C, CONJ>(tw, (p + j * h) << (L - 3 - s0)));
        const C w2a = tw_at<C, CONJ>(tw, p << (L - 2 - s0));
        const C w2b = tw_at<C, CONJ>(tw, (p + h) << (L - 2 - s0));
        bfly_dif(x[0], x[2], w2a);
        bfly_dif(x[1], x[3], w2b);
        bfly_dif(x[4], x[6], w2a);
        bfly_dif(x[5], x[7], w2b);
        const C w1 = tw_at<C, CONJ>(tw, p << (L - 1 - s0));
#pragma unroll
        for (int m = 0; m < 4; m++) bfly_dif(x[2 * m], x[2 * m + 1], w1);
#pragma unroll
        for (int j = 0; j < 8; j++) zb[fpad(base + j * h)] = x[j];
      }
    } else if (rr == 2) {
      const int per = N >> 2, lper = L - 2;
      for (int it = threadIdx.x; it < nT * per; it += blockDim.x) {
        const int t = it >> lper, u = it & (per - 1);
        C* zb = z + (size_t)t * stride;
        const int p = u & (h - 1);
        const int base = ((u >> s0) << (s0 + 2)) + p;
        C x[4];
#pragma unroll
        for (int j = 0; j < 4; j++) x[j] = zb[fpad(base + j * h)];
        bfly_dif(x[0], x[2], tw_at<C, CONJ>(tw, p << (L - 2 - s0)));
        bfly_dif(x[1], x[3], tw_at<C, CONJ>(tw, (p + h) << (L - 2 - s0)));
        const C w1 = tw_at<C, CONJ>(tw, p << (L - 1 - s0));
        bfly_dif(x[0], x[1], w1);
        bfly_dif(x[2], x[3], w1);
#pragma unroll
        for (int j = 0; j < 4; j++) zb[fpad(base + j * h)] = x[j];
      }
    } else {
      const int per = N >> 1, lper = L - 1;
      for (int it = threadIdx.x; it < nT * per; it += blockDim.x) {
        const int t = it >> lper, u = it & (per - 1);
        C* zb = z + (size_t)t * stride;
        const int p = u & (h - 1);
        const int base = ((u >> s0) << (s0 + 1)) + p;
        C a = zb[fpad(base)], b = zb[fpad(base + h)];
        bfly_dif(a, b, tw_at<C, CONJ>(tw, p << (L - 1 - s0)));
        zb[fpad(base)] = a;
        zb[fpad(base + h)] = b;
      }
    }
    top = s0;
  }
  __syncthreads();
}

// ---- Bluestein (chirp-z) transform for lengths with a large prime factor ----
// X[k] = sum_n x_n W^{nk}, W = e^{-2 pi i / M}, through nk = (n^2 + k^2 - (k-n)^2) / 2:
// X[k] = w_k sum_n (x_n w_n) conj(w_{k-n}),  w_n = e^{-i pi n^2 / M}
// (L. Bluestein, IEEE Trans. Audio Electroacoust. 18(4), 1970).  The sum is a
// cyclic convolution of length L = 2^lL >= 2M - 1: the chirped input, zero
// padded, goes through a DIF pass set (natural -> bit-reversed), is multiplied by
// the spectrum of the chirp filter (host table bB, bit-reversed order, divided by
// L), and comes back through a DIT pass set with the conjugate roots (bit-reversed
// -> natural).  The inverse DFT is conj(DFT(conj x)).  Input and output are in
// natural order in buffer slots [0, M).
template <class C>
__device__ void bluestein_b(const FftCtxT<C>& c, int nT, bool inverse) {
  const int M = c.M, LB = c.LB;
  __syncthreads();
  for (int it = threadIdx.x; it < nT * LB; it += blockDim.x) {
    const int t = it >> c.lLB, m = it & (LB - 1);
    C* zb = c.z + (size_t)t * c.stride;
    C v = Cx<C>::make(0, 0);
    if (m < M) {
      v = zb[fpad(m)];
      if (inverse) v = conj2(v);
      v = cmul(v, __ldg(&c.bw[m]));
    }
    zb[fpad(m)] = v;
  }
  pow2_dif<C, false>(c.z, c.stride, nT, LB, c.lLB, c.btw);
  for (int it = threadIdx.x; it < nT * LB; it += blockDim.x) {
    const int t = it >> c.lLB, j = it & (LB - 1);
    C* zb = c.z + (size_t)t * c.stride;
    zb[fpad(j)] = cmul(zb[fpad(j)], __ldg(&c.bB[j]));
  }
  pow2_dit<C, true>(c.z, c.stride, nT, LB, c.lLB, c.btw);
  for (int it = threadIdx.x; it < nT * M; it += blockDim.x) {
    const int t = it / M, k = it - t * M;
    C* zb = c.z + (size_t)t * c.stride;
    C v = cmul(zb[fpad(k)], __ldg(&c.bw[k]));
    zb[fpad(k)] = inverse ? conj2(v) : v;
  }
  __syncthreads();
}

// forward FFT of nT buffers: bit-reversed (digit-reversed) input -> natural output
template <class C>
__device__ __forceinline__ void fft_fwd_b(const FftCtxT<C>& c, int nT) {
  if constexpr (SDFT_FFT_GEN != 0) {
    if (c.blue) {
      bluestein_b(c, nT, false);
      return;
    }
    fft_gen_fwd(c, nT);
    return;
  }
  pow2_dit<C, false>(c.z, c.stride, nT, c.M, c.L, c.tw);
}

// inverse FFT of nT buffers (unscaled): natural input -> bit-reversed (digit-reversed) output
template <class C>
__device__ __forceinline__ void fft_inv_b(const FftCtxT<C>& c, int nT) {
  if constexpr (SDFT_FFT_GEN != 0) {
    if (c.blue) {
      bluestein_b(c, nT, true);
      return;
    }
    fft_gen_inv(c, nT);
    return;
  }
  pow2_dif<C, true>(c.z, c.stride, nT, c.M, c.L, c.tw);
}

// ---- pair step ------------------------------------------------------------
// From Z[k], Z[M-k] (natural order, after the forward FFT) to the four DCT-II
// coefficients C[k], C[P-k], C[M-k], C[M+k] (0 < k < M/2).
template <class R>
struct QuadT {
  R c0, c1, c2, c3;  // indices k, P-k, M-k, M+k
};
using Quad = QuadT<double>;

template <class C>
__device__ __forceinline__ QuadT<typename Cx<C>::R> pair_forward(C A, C B, C wk, C dk, C dk2) {
  using R = typename Cx<C>::R;
  const R half = (R)0.5;
  C Ze = scl2(add2(A, conj2(B)), half);
  C D = sub2(A, conj2(B));
  C Zo = Cx<C>::make(half * D.y, -half * D.x);  // -i D / 2
  C wZo = cmul(wk, Zo);
  C Vk = add2(Ze, wZo);
  C Vk2 = conj2(sub2(Ze, wZo));
  C tk = cmul(dk, Vk);
  C tk2 = cmul(dk2, Vk2);
  QuadT<R> q;
  q.c0 = tk.x;
  q.c1 = -tk.y;
  q.c2 = tk2.x;
  q.c3 = -tk2.y;
  return q;
}

// inverse of pair_forward: coefficients E[k], E[P-k], E[M-k], E[M+k] -> Z'[k], Z'[M-k]
template <class C>
__device__ __forceinline__ void pair_inverse(const QuadT<typename Cx<C>::R>& e, C wk, C dk, C dk2, C* Zk, C* Zk2) {
  using R = typename Cx<C>::R;
  const R half = (R)0.5;
  C Vk = cmul(conj2(dk), Cx<C>::make(e.c0, -e.c1));
  C Vk2 = cmul(conj2(dk2), Cx<C>::make(e.c2, -e.c3));
  C Ze = scl2(add2(Vk, conj2(Vk2)), half);
  C Zo = scl2(cmul(sub2(Vk, conj2(Vk2)), conj2(wk)), half);
  *Zk = Cx<C>::make(Ze.x - Zo.y, Ze.y + Zo.x);
  *Zk2 = Cx<C>::make(Ze.x + Zo.y, -Ze.y + Zo.x);
}

// k = 0: C[0] and C[M] (C[P] does not exist)
template <class C, class R>
__device__ __forceinline__ void zero_forward(C A, C dM, R* c0, R* cM) {
  R V0 = A.x + A.y;
  R VM = A.x - A.y;
  *c0 = V0;
  *cM = VM * dM.x;
}
template <class C>
__device__ __forceinline__ C zero_inverse(typename Cx<C>::R e0, typename Cx<C>::R eM, C dM) {
  using R = typename Cx<C>::R;
  const R half = (R)0.5;
  C VM = cmul(conj2(dM), Cx<C>::make(eM, -eM));
  C Ze = scl2(add2(Cx<C>::make(e0, (R)0), conj2(VM)), half);
  C Zo = scl2(sub2(Cx<C>::make(e0, (R)0), conj2(VM)), half);
  return Cx<C>::make(Ze.x - Zo.y, Ze.y + Zo.x);
}
// k = M/2: C[M/2], C[P-M/2]
template <class C, class R>
__device__ __forceinline__ void mid_forward(C A, C dh, R* ch, R* cPh) {
  C t = cmul(dh, conj2(A));
  *ch = t.x;
  *cPh = -t.y;
}
template <class C>
__device__ __forceinline__ C mid_inverse(typename Cx<C>::R eh, typename Cx<C>::R ePh, C dh) {
  C V = cmul(conj2(dh), Cx<C>::make(eh, -ePh));
  return conj2(V);
}

// pair items: it -> (t, k) with k in [0, (M+1)/2); k = 0 also handles k = H = M/2
// when M is even (odd M has no middle coefficient pair)
#define SDFT_PAIR_LOOP(c, nT)                                           \
  const int lH_ = (c).L - 1, cnt_ = ((c).M + 1) >> 1;                   \
  for (int it = threadIdx.x; it < (nT) * cnt_; it += blockDim.x) {     \
    const int t = item_t<GEN>(it, cnt_, lH_), k = it - t * cnt_;        \
    auto* zb = (c).z + (size_t)t * (c).stride;

// ---- odd P (general build): two real transforms per complex FFT -------------
// Transforms 2b and 2b+1 share buffer b as the real and the imaginary part of
// one complex FFT of M = P points of their Makhoul sequences, Z = V_{2b} + i V_{2b+1};
// each V is Hermitian, so V_{2b}[k] = (Z[k] + conj Z[P-k]) / 2 and
// V_{2b+1}[k] = -i (Z[k] - conj Z[P-k]) / 2.  Per transform, C[0] = Re V[0],
// C[k] = Re(d_k V[k]) and C[P-k] = Re(d_{P-k} conj V[k]) with d_k = e^{-i pi k / 2P}
// (twD).  The inverse builds V'[0] = E[0] and V'[k] = conj(d_k) (E[k] - i E[P-k])
// per transform, Z'[k] = V'_{2b}[k] + i V'_{2b+1}[k] and
// Z'[P-k] = conj V'_{2b}[k] + i conj V'_{2b+1}[k]; the real and imaginary parts of
// the unscaled inverse FFT, divided by P, are the two outputs.  A lone last
// transform (odd nT) has a zero partner.  The grid-point pairs (K, K+1) run over
// the padded stride P + 1: the pad sample K + 1 = P is not loaded and is stored as 0.
__device__ __forceinline__ int makhoul_q(int K, int P) { return (K & 1) ? (P - 1 - (K >> 1)) : (K >> 1); }

// component t & 1 of buffer t >> 1 at slot s
template <class C>
__device__ __forceinline__ typename Cx<C>::R& odd_part(const FftCtxT<C>& c, int t, int s) {
  using R = typename Cx<C>::R;
  return reinterpret_cast<R*>(c.z + (size_t)(t >> 1) * c.stride + fpad(s))[t & 1];
}

template <class F>
__device__ __forceinline__ void load_b_odd(const FftCtx& c, int nT, F f) {
  const int nT2 = (nT + 1) & ~1;
  for (int it = threadIdx.x; it < nT2 * c.P; it += blockDim.x) {
    const int t = it / c.P, K = it - t * c.P;
    odd_part(c, t, fslot<true>(c, makhoul_q(K, c.P))) = t < nT ? f(t, K) : 0.0;
  }
}

template <class S>
__device__ __forceinline__ void store_b_odd(const FftCtx& c, int nT, double scale, S st) {
  for (int it = threadIdx.x; it < nT * c.P; it += blockDim.x) {
    const int t = it / c.P, K = it - t * c.P;
    st(t, K, odd_part(c, t, fslot<true>(c, makhoul_q(K, c.P))) * scale);
  }
}

template <class C, class F2>
__device__ __forceinline__ void load_b2_odd(const FftCtxT<C>& c, int nT, F2 f2) {
  using R = typename Cx<C>::R;
  const int np = (c.P + 1) >> 1, nT2 = (nT + 1) & ~1;
  for (int b = threadIdx.x; b < nT2 * np; b += blockDim.x) {
    const int t = b / np, kp = b - t * np, K = 2 * kp;
    R v0 = (R)0, v1 = (R)0;
    if (t < nT) {
      const auto v = f2(t, K);
      v0 = (R)v.x;
      v1 = (R)v.y;
    }
    odd_part(c, t, fslot<true>(c, kp)) = v0;
    if (K + 1 < c.P) odd_part(c, t, fslot<true>(c, c.P - 1 - kp)) = v1;
  }
}

template <class C, class A2, class S2>
__device__ __forceinline__ void store_b2_odd(const FftCtxT<C>& c, int nT, typename Cx<C>::R scale, A2 pre2, S2 put2) {
  using R = typename Cx<C>::R;
  const int np = (c.P + 1) >> 1;
  for (int b = threadIdx.x; b < nT * np; b += blockDim.x) {
    const int t = b / np, kp = b - t * np, K = 2 * kp;
    const R y0 = odd_part(c, t, fslot<true>(c, kp));
    const R y1 = (K + 1 < c.P) ? odd_part(c, t, fslot<true>(c, c.P - 1 - kp)) : (R)0;
    const auto a = pre2(t, K);
    put2(t, K, Cx<C>::make(y0 * scale, y1 * scale), a);
  }
}

// the two Hermitian spectra packed in Z[k], Z[P-k] (k >= 1)
template <class C>
__device__ __forceinline__ void odd_unpack(C A, C B, C* V0, C* V1) {
  using R = typename Cx<C>::R;
  const R h = (R)0.5;
  const C S = add2(A, conj2(B)), D = sub2(A, conj2(B));
  *V0 = scl2(S, h);
  *V1 = Cx<C>::make(h * D.y, -h * D.x);  // -i D / 2
}
// Z'[k], Z'[P-k] from the two inverse spectra
template <class C>
__device__ __forceinline__ void odd_pack(C W0, C W1, C* Zk, C* Zpk) {
  *Zk = Cx<C>::make(W0.x - W1.y, W0.y + W1.x);
  *Zpk = Cx<C>::make(W0.x + W1.y, -W0.y + W1.x);
}
// C[k], C[P-k] of one spectrum; V'[k] from E[k], E[P-k]
template <class C>
__device__ __forceinline__ void odd_forward(C V, C dk, C dpk, typename Cx<C>::R* ck, typename Cx<C>::R* cpk) {
  *ck = cmul(dk, V).x;
  *cpk = cmul(dpk, conj2(V)).x;
}
template <class C>
__device__ __forceinline__ C odd_inverse(typename Cx<C>::R ek, typename Cx<C>::R epk, C dk) {
  return cmul(conj2(dk), Cx<C>::make(ek, -epk));
}

template <class F, class E>
__device__ __forceinline__ void dct2_forward_odd(const FftCtx& c, int nT, F f, E emit) {
  const int P = c.P, cnt = (P + 1) >> 1, nb = (nT + 1) >> 1;
  __syncthreads();
  load_b_odd(c, nT, f);
  fft_fwd_b(c, nb);
  for (int it = threadIdx.x; it < nb * cnt; it += blockDim.x) {
    const int b = it / cnt, k = it - b * cnt, t0 = 2 * b, t1 = t0 + 1;
    const double2* zb = c.z + (size_t)b * c.stride;
    if (k == 0) {
      emit(t0, 0, zb[0].x);
      if (t1 < nT) emit(t1, 0, zb[0].y);
    } else {
      double2 V0, V1;
      odd_unpack(zb[fpad(k)], zb[fpad(P - k)], &V0, &V1);
      const double2 dk = __ldg(&c.twD[k]), dpk = __ldg(&c.twD[P - k]);
      double ck, cpk;
      odd_forward(V0, dk, dpk, &ck, &cpk);
      emit(t0, k, ck);
      emit(t0, P - k, cpk);
      if (t1 < nT) {
        odd_forward(V1, dk, dpk, &ck, &cpk);
        emit(t1, k, ck);
        emit(t1, P - k, cpk);
      }
    }
  }
  __syncthreads();
}

template <class G, class S>
__device__ __forceinline__ void dct2_inverse_odd(const FftCtx& c, int nT, G get, S store) {
  const int P = c.P, cnt = (P + 1) >> 1, nb = (nT + 1) >> 1;
  __syncthreads();
  for (int it = threadIdx.x; it < nb * cnt; it += blockDim.x) {
    const int b = it / cnt, k = it - b * cnt, t0 = 2 * b, t1 = t0 + 1;
    double2* zb = c.z + (size_t)b * c.stride;
    if (k == 0) {
      zb[0] = make_double2(get(t0, 0), t1 < nT ? get(t1, 0) : 0.0);
    } else {
      const double2 dk = __ldg(&c.twD[k]);
      const double2 W0 = odd_inverse(get(t0, k), get(t0, P - k), dk);
      const double2 W1 = t1 < nT ? odd_inverse(get(t1, k), get(t1, P - k), dk) : make_double2(0.0, 0.0);
      odd_pack(W0, W1, &zb[fpad(k)], &zb[fpad(P - k)]);
    }
  }
  fft_inv_b(c, nb);
  store_b_odd(c, nT, 1.0 / (double)P, store);
  __syncthreads();
}

template <class F, class W, class S>
__device__ __forceinline__ void dct2_convolve_odd(const FftCtx& c, int nT, F f, W wgt, S store) {
  const int P = c.P, cnt = (P + 1) >> 1, nb = (nT + 1) >> 1;
  __syncthreads();
  load_b_odd(c, nT, f);
  fft_fwd_b(c, nb);
  for (int it = threadIdx.x; it < nb * cnt; it += blockDim.x) {
    const int b = it / cnt, k = it - b * cnt, t0 = 2 * b, t1 = t0 + 1;
    double2* zb = c.z + (size_t)b * c.stride;
    if (k == 0) {
      const double2 A = zb[0];
      zb[0] = make_double2(A.x * wgt(t0, 0), t1 < nT ? A.y * wgt(t1, 0) : 0.0);
    } else {
      double2 V0, V1;
      odd_unpack(zb[fpad(k)], zb[fpad(P - k)], &V0, &V1);
      const double2 dk = __ldg(&c.twD[k]), dpk = __ldg(&c.twD[P - k]);
      double ck, cpk;
      odd_forward(V0, dk, dpk, &ck, &cpk);
      const double2 W0 = odd_inverse(ck * wgt(t0, k), cpk * wgt(t0, P - k), dk);
      double2 W1 = make_double2(0.0, 0.0);
      if (t1 < nT) {
        odd_forward(V1, dk, dpk, &ck, &cpk);
        W1 = odd_inverse(ck * wgt(t1, k), cpk * wgt(t1, P - k), dk);
      }
      odd_pack(W0, W1, &zb[fpad(k)], &zb[fpad(P - k)]);
    }
  }
  fft_inv_b(c, nb);
  store_b_odd(c, nT, 1.0 / (double)P, store);
  __syncthreads();
}

template <class C, class F2, class W, class A2, class S2>
__device__ __forceinline__ void dct2_convolve_b2_odd(const FftCtxT<C>& c, int nT, F2 f2, W wgt, A2 pre2, S2 put2) {
  using R = typename Cx<C>::R;
  const int P = c.P, cnt = (P + 1) >> 1, nb = (nT + 1) >> 1;
  __syncthreads();
  load_b2_odd(c, nT, f2);
  fft_fwd_b(c, nb);
  for (int it = threadIdx.x; it < nb * cnt; it += blockDim.x) {
    const int b = it / cnt, k = it - b * cnt, t0 = 2 * b, t1 = t0 + 1;
    C* zb = c.z + (size_t)b * c.stride;
    if (k == 0) {
      const C A = zb[0];
      zb[0] = Cx<C>::make(A.x * (R)wgt(t0, 0), t1 < nT ? A.y * (R)wgt(t1, 0) : (R)0);
    } else {
      C V0, V1;
      odd_unpack(zb[fpad(k)], zb[fpad(P - k)], &V0, &V1);
      const C dk = __ldg(&c.twD[k]), dpk = __ldg(&c.twD[P - k]);
      R ck, cpk;
      odd_forward(V0, dk, dpk, &ck, &cpk);
      const C W0 = odd_inverse(ck * (R)wgt(t0, k), cpk * (R)wgt(t0, P - k), dk);
      C W1 = Cx<C>::make((R)0, (R)0);
      if (t1 < nT) {
        odd_forward(V1, dk, dpk, &ck, &cpk);
        W1 = odd_inverse(ck * (R)wgt(t1, k), cpk * (R)wgt(t1, P - k), dk);
      }
      odd_pack(W0, W1, &zb[fpad(k)], &zb[fpad(P - k)]);
    }
  }
  fft_inv_b(c, nb);
  store_b2_odd(c, nT, (R)1 / (R)P, pre2, put2);
  __syncthreads();
}

// ---- whole transforms ------------------------------------------------------

// C[q] for q in [0, P): forward DCT-II of f(t, .); emit(t, q, C[q])
template <bool GEN, class F, class E>
__device__ __forceinline__ void dct2_forward_b_impl(const FftCtx& c, int nT, F f, E emit) {
  const int P = c.P, M = c.M, H = c.H;
  __syncthreads();
  load_b<GEN>(c, nT, f);
  fft_fwd_b(c, nT);
  SDFT_PAIR_LOOP(c, nT)
  if (k == 0) {
    double c0, cM;
    zero_forward(zb[0], __ldg(&c.twD[M]), &c0, &cM);
    emit(t, 0, c0);
    emit(t, M, cM);
    if (!(M & 1)) {
      double ch, cPh;
      mid_forward(zb[fpad(H)], __ldg(&c.twD[H]), &ch, &cPh);
      emit(t, H, ch);
      emit(t, P - H, cPh);
    }
  } else {
    Quad q = pair_forward(zb[fpad(k)], zb[fpad(M - k)], __ldg(&c.twP[k]), __ldg(&c.twD[k]), __ldg(&c.twD[M - k]));
    emit(t, k, q.c0);
    emit(t, P - k, q.c1);
    emit(t, M - k, q.c2);
    emit(t, M + k, q.c3);
  }
}
__syncthreads();
}

template <class F, class E>
__device__ __forceinline__ void dct2_forward_b(const FftCtx& c, int nT, F f, E emit) {
  if constexpr (SDFT_FFT_GEN != 0) {
    if (c.P & 1) {
      dct2_forward_odd(c, nT, f, emit);
      return;
    }
  }
  dct2_forward_b_impl<(SDFT_FFT_GEN != 0)>(c, nT, f, emit);
}

// y = iDCT2(E_t), E_t[q] = get(t, q); store(t, K, y[K])
template <bool GEN, class G, class S>
__device__ __forceinline__ void dct2_inverse_b_impl(const FftCtx& c, int nT, G get, S store) {
  const int P = c.P, M = c.M, H = c.H;
  __syncthreads();
  SDFT_PAIR_LOOP(c, nT)
  if (k == 0) {
    zb[0] = zero_inverse(get(t, 0), get(t, M), __ldg(&c.twD[M]));
    if (!(M & 1)) zb[fpad(H)] = mid_inverse(get(t, H), get(t, P - H), __ldg(&c.twD[H]));
  } else {
    Quad e;
    e.c0 = get(t, k);
    e.c1 = get(t, P - k);
    e.c2 = get(t, M - k);
    e.c3 = get(t, M + k);
    double2 a, b;
    pair_inverse(e, __ldg(&c.twP[k]), __ldg(&c.twD[k]), __ldg(&c.twD[M - k]), &a, &b);
    zb[fpad(k)] = a;
    zb[fpad(M - k)] = b;
  }
}
fft_inv_b(c, nT);
store_b<GEN>(c, nT, 1.0 / (double)M, store);
__syncthreads();
}

template <class G, class S>
__device__ __forceinline__ void dct2_inverse_b(const FftCtx& c, int nT, G get, S store) {
  if constexpr (SDFT_FFT_GEN != 0) {
    if (c.P & 1) {
      dct2_inverse_odd(c, nT, get, store);
      return;
    }
  }
  dct2_inverse_b_impl<(SDFT_FFT_GEN != 0)>(c, nT, get, store);
}

// y = iDCT2(W_t .* DCT2(f_t)); W_t[q] = wgt(t, q); store(t, K, y[K])
template <bool GEN, class F, class W, class S>
__device__ __forceinline__ void dct2_convolve_b_impl(const FftCtx& c, int nT, F f, W wgt, S store) {
  const int P = c.P, M = c.M, H = c.H;
  __syncthreads();
  load_b<GEN>(c, nT, f);
  fft_fwd_b(c, nT);
  SDFT_PAIR_LOOP(c, nT)
  if (k == 0) {
    const double2 dM = __ldg(&c.twD[M]);
    double c0, cM;
    zero_forward(zb[0], dM, &c0, &cM);
    zb[0] = zero_inverse(c0 * wgt(t, 0), cM * wgt(t, M), dM);
    if (!(M & 1)) {
      const double2 dh = __ldg(&c.twD[H]);
      double ch, cPh;
      mid_forward(zb[fpad(H)], dh, &ch, &cPh);
      zb[fpad(H)] = mid_inverse(ch * wgt(t, H), cPh * wgt(t, P - H), dh);
    }
  } else {
    const double2 wk = __ldg(&c.twP[k]), dk = __ldg(&c.twD[k]), dk2 = __ldg(&c.twD[M - k]);
    Quad q = pair_forward(zb[fpad(k)], zb[fpad(M - k)], wk, dk, dk2);
    q.c0 *= wgt(t, k);
    q.c1 *= wgt(t, P - k);
    q.c2 *= wgt(t, M - k);
    q.c3 *= wgt(t, M + k);
    double2 a, b;
    pair_inverse(q, wk, dk, dk2, &a, &b);
    zb[fpad(k)] = a;
    zb[fpad(M - k)] = b;
  }
}
fft_inv_b(c, nT);
store_b<GEN>(c, nT, 1.0 / (double)M, store);
__syncthreads();
}

template <class F, class W, class S>
__device__ __forceinline__ void dct2_convolve_b(const FftCtx& c, int nT, F f, W wgt, S store) {
  if constexpr (SDFT_FFT_GEN != 0) {
    if (c.P & 1) {
      dct2_convolve_odd(c, nT, f, wgt, store);
      return;
    }
  }
  dct2_convolve_b_impl<(SDFT_FFT_GEN != 0)>(c, nT, f, wgt, store);
}

// the same convolution with grid-point pair functors (load_b2 / store_b2), in
// the precision of the context (FP64, or FP32 for mixed-precision propagators)
template <bool GEN, class C, class F2, class W, class A2, class S2>
__device__ __forceinline__ void dct2_convolve_b2_impl(const FftCtxT<C>& c, int nT, F2 f2, W wgt, A2 pre2, S2 put2) {
  using R = typename Cx<C>::R;
  const int P = c.P, M = c.M, H = c.H;
  __syncthreads();
  load_b2<GEN>(c, nT, f2);
  fft_fwd_b(c, nT);
  SDFT_PAIR_LOOP(c, nT)
  if (k == 0) {
    const C dM = __ldg(&c.twD[M]);
    R c0, cM;
    zero_forward(zb[0], dM, &c0, &cM);
    zb[0] = zero_inverse(c0 * (R)wgt(t, 0), cM * (R)wgt(t, M), dM);
    if (!(M & 1)) {
      const C dh = __ldg(&c.twD[H]);
      R ch, cPh;
      mid_forward(zb[fpad(H)], dh, &ch, &cPh);
      zb[fpad(H)] = mid_inverse(ch * (R)wgt(t, H), cPh * (R)wgt(t, P - H), dh);
    }
  } else {
    const C wk = __ldg(&c.twP[k]), dk = __ldg(&c.twD[k]), dk2 = __ldg(&c.twD[M - k]);
    QuadT<R> q = pair_forward(zb[fpad(k)], zb[fpad(M - k)], wk, dk, dk2);
    q.c0 *= (R)wgt(t, k);
    q.c1 *= (R)wgt(t, P - k);
    q.c2 *= (R)wgt(t, M - k);
    q.c3 *= (R)wgt(t, M + k);
    C a, b;
    pair_inverse(q, wk, dk, dk2, &a, &b);
    zb[fpad(k)] = a;
    zb[fpad(M - k)] = b;
  }
}
fft_inv_b(c, nT);
store_b2<GEN>(c, nT, (R)1 / (R)M, pre2, put2);
__syncthreads();
}

template <class C, class F2, class W, class A2, class S2>
__device__ __forceinline__ void dct2_convolve_b2(const FftCtxT<C>& c, int nT, F2 f2, W wgt, A2 pre2, S2 put2) {
  if constexpr (SDFT_FFT_GEN != 0) {
    if (c.P & 1) {
      dct2_convolve_b2_odd(c, nT, f2, wgt, pre2, put2);
      return;
    }
  }
  dct2_convolve_b2_impl<(SDFT_FFT_GEN != 0)>(c, nT, f2, wgt, pre2, put2);
}

// ---- grid-pair-major convolution driver (even P) ------------------------------
// The same convolution of nT transforms, with load and store phases organised
// by grid-point pair instead of by transform: loadkp(kp, put) issues every load
// that pair kp needs for all nT transforms before it calls put(t, (f_K, f_K+1));
// storekp(kp, get) receives get(t) = (y_K, y_K+1) for every transform.  A
// thread owns the same pairs in both phases, so whatever the store phase keeps
// per pair (a running maximum, sums over transforms) needs no exchange, and the
// loads of all nT transforms are in flight together.
template <bool GEN, class C, class LK, class W, class SK>
__device__ __forceinline__ void dct2_convolve_kpair_impl(const FftCtxT<C>& c, int nT, LK loadkp, W wgt, SK storekp) {
  using R = typename Cx<C>::R;
  const int P = c.P, M = c.M, H = c.H;
  __syncthreads();
  for (int kp = threadIdx.x; kp < M; kp += blockDim.x)
    loadkp(kp, [&](int t, double2 v) { put_pair<GEN>(c, t, kp, v); });
  fft_fwd_b(c, nT);
  SDFT_PAIR_LOOP(c, nT)
  if (k == 0) {
    const C dM = __ldg(&c.twD[M]);
    R c0, cM;
    zero_forward(zb[0], dM, &c0, &cM);
    zb[0] = zero_inverse(c0 * (R)wgt(t, 0), cM * (R)wgt(t, M), dM);
    if (!(M & 1)) {
      const C dh = __ldg(&c.twD[H]);
      R ch, cPh;
      mid_forward(zb[fpad(H)], dh, &ch, &cPh);
      zb[fpad(H)] = mid_inverse(ch * (R)wgt(t, H), cPh * (R)wgt(t, P - H), dh);
    }
  } else {
    const R w0 = (R)wgt(t, k), w1 = (R)wgt(t, P - k), w2 = (R)wgt(t, M - k), w3 = (R)wgt(t, M + k);
    const C wk = __ldg(&c.twP[k]), dk = __ldg(&c.twD[k]), dk2 = __ldg(&c.twD[M - k]);
    QuadT<R> q = pair_forward(zb[fpad(k)], zb[fpad(M - k)], wk, dk, dk2);
    q.c0 *= w0;
    q.c1 *= w1;
    q.c2 *= w2;
    q.c3 *= w3;
    C a, b;
    pair_inverse(q, wk, dk, dk2, &a, &b);
    zb[fpad(k)] = a;
    zb[fpad(M - k)] = b;
  }
}
fft_inv_b(c, nT);
const R scale = (R)1 / (R)M;
for (int kp = threadIdx.x; kp < M; kp += blockDim.x)
  storekp(kp, [&](int t) {
    C y = get_pair<GEN>(c, t, kp);
    y.x *= scale;
    y.y *= scale;
    return y;
  });
__syncthreads();
}

template <class C, class LK, class W, class SK>
__device__ __forceinline__ void dct2_convolve_kpair(const FftCtxT<C>& c, int nT, LK loadkp, W wgt, SK storekp) {
  dct2_convolve_kpair_impl<(SDFT_FFT_GEN != 0)>(c, nT, loadkp, wgt, storekp);
}

// ---- grid-pair-major forward and inverse transforms (any P) -------------------
// The batched forward DCT-II and inverse DCT-II with the grid-side phase
// organised by grid-point pair, as dct2_convolve_kpair: loadkp(kp, put) calls
// put(t, (f_K, f_K+1)) for every transform t, storekp(kp, get) reads
// get(t) = (y_K, y_K+1).  Pairs run over kp < ceil(P/2); on an odd grid the last
// pair's second sample is the pad point beyond the grid (read by loadkp, never
// transformed, given as 0 by get).  The coefficient side keeps the per-index
// functors of dct2_forward_b / dct2_inverse_b.
template <bool GEN, class LK>
__device__ __forceinline__ void load_kpair(const FftCtx& c, int nT, LK loadkp) {
  if (GEN && (c.P & 1)) {  // odd P: transforms 2b, 2b+1 are the real and imaginary parts of buffer b
    const int np = (c.P + 1) >> 1;
    for (int kp = threadIdx.x; kp < np; kp += blockDim.x) {
      const bool two = 2 * kp + 1 < c.P;
      const int s0 = fslot<true>(c, kp), s1 = two ? fslot<true>(c, c.P - 1 - kp) : 0;
      loadkp(kp, [&](int t, double2 v) {
        odd_part(c, t, s0) = v.x;
        if (two) odd_part(c, t, s1) = v.y;
      });
      if (nT & 1) {  // a lone last transform has a zero partner
        odd_part(c, nT, s0) = 0.0;
        if (two) odd_part(c, nT, s1) = 0.0;
      }
    }
    return;
  }
  for (int kp = threadIdx.x; kp < c.M; kp += blockDim.x)
    loadkp(kp, [&](int t, double2 v) { put_pair<GEN>(c, t, kp, v); });
}

template <bool GEN, class SK>
__device__ __forceinline__ void store_kpair(const FftCtx& c, double scale, SK storekp) {
  if (GEN && (c.P & 1)) {
    const int np = (c.P + 1) >> 1;
    for (int kp = threadIdx.x; kp < np; kp += blockDim.x) {
      const bool two = 2 * kp + 1 < c.P;
      const int s0 = fslot<true>(c, kp), s1 = two ? fslot<true>(c, c.P - 1 - kp) : 0;
      storekp(kp, [&](int t) {
        return make_double2(odd_part(c, t, s0) * scale, two ? odd_part(c, t, s1) * scale : 0.0);
      });
    }
    return;
  }
  for (int kp = threadIdx.x; kp < c.M; kp += blockDim.x)
    storekp(kp, [&](int t) {
      double2 y = get_pair<GEN>(c, t, kp);
      y.x *= scale;
      y.y *= scale;
      return y;
    });
}

// C[q] for q in [0, P): forward DCT-II; emit(t, q, C[q]) as dct2_forward_b
template <class LK, class E>
__device__ __forceinline__ void dct2_forward_kp(const FftCtx& c, int nT, LK loadkp, E emit) {
  constexpr bool GEN = SDFT_FFT_GEN != 0;
  const int P = c.P, M = c.M, H = c.H;
  __syncthreads();
  load_kpair<GEN>(c, nT, loadkp);
  if (GEN && (P & 1)) {
    const int cnt = (P + 1) >> 1, nb = (nT + 1) >> 1;
    fft_fwd_b(c, nb);
    for (int it = threadIdx.x; it < nb * cnt; it += blockDim.x) {
      const int b = it / cnt, k = it - b * cnt, t0 = 2 * b, t1 = t0 + 1;
      const double2* zb = c.z + (size_t)b * c.stride;
      if (k == 0) {
        emit(t0, 0, zb[0].x);
        if (t1 < nT) emit(t1, 0, zb[0].y);
      } else {
        double2 V0, V1;
        odd_unpack(zb[fpad(k)], zb[fpad(P - k)], &V0, &V1);
        const double2 dk = __ldg(&c.twD[k]), dpk = __ldg(&c.twD[P - k]);
        double ck, cpk;
        odd_forward(V0, dk, dpk, &ck, &cpk);
        emit(t0, k, ck);
        emit(t0, P - k, cpk);
        if (t1 < nT) {
          odd_forward(V1, dk, dpk, &ck, &cpk);
          emit(t1, k, ck);
          emit(t1, P - k, cpk);
        }
      }
    }
    __syncthreads();
    return;
  }
  fft_fwd_b(c, nT);
  const int lH = c.L - 1, cnt = (M + 1) >> 1;
  for (int it = threadIdx.x; it < nT * cnt; it += blockDim.x) {
    const int t = item_t<GEN>(it, cnt, lH), k = it - t * cnt;
    const double2* zb = c.z + (size_t)t * c.stride;
    if (k == 0) {
      double c0, cM;
      zero_forward(zb[0], __ldg(&c.twD[M]), &c0, &cM);
      emit(t, 0, c0);
      emit(t, M, cM);
      if (!(M & 1)) {
        double ch, cPh;
        mid_forward(zb[fpad(H)], __ldg(&c.twD[H]), &ch, &cPh);
        emit(t, H, ch);
        emit(t, P - H, cPh);
      }
    } else {
      Quad q = pair_forward(zb[fpad(k)], zb[fpad(M - k)], __ldg(&c.twP[k]), __ldg(&c.twD[k]), __ldg(&c.twD[M - k]));
      emit(t, k, q.c0);
      emit(t, P - k, q.c1);
      emit(t, M - k, q.c2);
      emit(t, M + k, q.c3);
    }
  }
  __syncthreads();
}

// y_t = iDCT2(E_t), E_t[q] = get(t, q) as dct2_inverse_b; pair-major store
template <class G, class SK>
__device__ __forceinline__ void dct2_inverse_kp(const FftCtx& c, int nT, G get, SK storekp) {
  constexpr bool GEN = SDFT_FFT_GEN != 0;
  const int P = c.P, M = c.M, H = c.H;
  __syncthreads();
  if (GEN && (P & 1)) {
    const int cnt = (P + 1) >> 1, nb = (nT + 1) >> 1;
    for (int it = threadIdx.x; it < nb * cnt; it += blockDim.x) {
      const int b = it / cnt, k = it - b * cnt, t0 = 2 * b, t1 = t0 + 1;
      double2* zb = c.z + (size_t)b * c.stride;
      if (k == 0) {
        zb[0] = make_double2(get(t0, 0), t1 < nT ? get(t1, 0) : 0.0);
      } else {
        const double2 dk = __ldg(&c.twD[k]);
        const double2 W0 = odd_inverse(get(t0, k), get(t0, P - k), dk);
        const double2 W1 = t1 < nT ? odd_inverse(get(t1, k), get(t1, P - k), dk) : make_double2(0.0, 0.0);
        odd_pack(W0, W1, &zb[fpad(k)], &zb[fpad(P - k)]);
      }
    }
    fft_inv_b(c, nb);
    store_kpair<GEN>(c, 1.0 / (double)P, storekp);
    __syncthreads();
    return;
  }
  const int lH = c.L - 1, cnt = (M + 1) >> 1;
  for (int it = threadIdx.x; it < nT * cnt; it += blockDim.x) {
    const int t = item_t<GEN>(it, cnt, lH), k = it - t * cnt;
    double2* zb = c.z + (size_t)t * c.stride;
    if (k == 0) {
      zb[0] = zero_inverse(get(t, 0), get(t, M), __ldg(&c.twD[M]));
      if (!(M & 1)) zb[fpad(H)] = mid_inverse(get(t, H), get(t, P - H), __ldg(&c.twD[H]));
    } else {
      Quad e;
      e.c0 = get(t, k);
      e.c1 = get(t, P - k);
      e.c2 = get(t, M - k);
      e.c3 = get(t, M + k);
      double2 a, b;
      pair_inverse(e, __ldg(&c.twP[k]), __ldg(&c.twD[k]), __ldg(&c.twD[M - k]), &a, &b);
      zb[fpad(k)] = a;
      zb[fpad(M - k)] = b;
    }
  }
  fft_inv_b(c, nT);
  store_kpair<GEN>(c, 1.0 / (double)M, storekp);
  __syncthreads();
}

#undef SDFT_PAIR_LOOP

// ---- single-transform wrappers -----------------------------------------
template <class F, class E>
__device__ __forceinline__ void dct2_forward(const FftCtx& c, F f, E emit) {
  dct2_forward_b(
      c, 1, [&](int, int K) { return f(K); }, [&](int, int q, double v) { emit(q, v); });
}
template <class G, class S>
__device__ __forceinline__ void dct2_inverse(const FftCtx& c, G get, S store) {
  dct2_inverse_b(
      c, 1, [&](int, int q) { return get(q); }, [&](int, int K, double y) { store(K, y); });
}

}  // namespace
}  // namespace sdft
