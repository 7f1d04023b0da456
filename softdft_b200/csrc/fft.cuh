// fft.cuh -- CTA-wide DCT-II / inverse-DCT-II of P real points through one
// complex FFT of M = P/2 points held in shared memory.
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
// Shared buffer: z[M] double2.  Forward: the load scatters into bit-reversed
// order, a radix-2 decimation-in-time FFT leaves z in natural order.  Inverse:
// a decimation-in-frequency IFFT takes natural order and leaves bit-reversed
// order, undone by the gather of the store.  No permutation pass is needed.
//
// Every butterfly of the pair step (k, M-k) only touches Z[k] and Z[M-k], so a
// whole convolution is: load, FFT, one in-place pair pass, IFFT, store.
#pragma once

#include "common.cuh"

namespace sdft {

__device__ __forceinline__ int brev_bits(int m, int L) {
  return L == 0 ? 0 : (int)(__brev((unsigned)m) >> (32 - L));
}

// position of real sample K in the packed complex buffer: (bit-reversed index, component)
__device__ __forceinline__ void dct_slot(int K, int P, int L, int* pos, int* comp) {
  int q = (K & 1) ? (P - 1 - (K >> 1)) : (K >> 1);  // Makhoul reorder v[q]
  *pos = brev_bits(q >> 1, L);
  *comp = q & 1;
}

// z <- (bit-reversed) packed reorder of x, x[K] = f(K)
template <class F>
__device__ __forceinline__ void dct_load(double2* z, int P, int L, F f) {
  double* zd = reinterpret_cast<double*>(z);
  for (int K = threadIdx.x; K < P; K += blockDim.x) {
    int pos, comp;
    dct_slot(K, P, L, &pos, &comp);
    zd[2 * pos + comp] = f(K);
  }
}

// radix-2 DIT on bit-reversed input -> natural output (forward, e^{-i})
__device__ __forceinline__ void fft_dit(double2* z, int M, int L, const double2* __restrict__ tw) {
  const int half_n = M >> 1;
  for (int s = 0; s < L; s++) {
    __syncthreads();
    const int h = 1 << s;
    for (int b = threadIdx.x; b < half_n; b += blockDim.x) {
      int pos = b & (h - 1);
      int i = ((b >> s) << (s + 1)) + pos;
      int j = i + h;
      double2 w = __ldg(&tw[pos << (L - 1 - s)]);
      double2 a = z[i];
      double2 c = cmul(z[j], w);
      z[i] = add2(a, c);
      z[j] = sub2(a, c);
    }
  }
  __syncthreads();
}

// radix-2 DIF inverse on natural input -> bit-reversed output (e^{+i}, unscaled)
__device__ __forceinline__ void ifft_dif(double2* z, int M, int L, const double2* __restrict__ tw) {
  const int half_n = M >> 1;
  for (int s = L - 1; s >= 0; s--) {
    __syncthreads();
    const int h = 1 << s;
    for (int b = threadIdx.x; b < half_n; b += blockDim.x) {
      int pos = b & (h - 1);
      int i = ((b >> s) << (s + 1)) + pos;
      int j = i + h;
      double2 w = conj2(__ldg(&tw[pos << (L - 1 - s)]));
      double2 a = z[i];
      double2 c = z[j];
      z[i] = add2(a, c);
      z[j] = cmul(sub2(a, c), w);
    }
  }
  __syncthreads();
}

// y[K] = scale * iDCT2 sample K; g(K, y)
template <class G>
__device__ __forceinline__ void dct_store(const double2* z, int P, int L, double scale, G g) {
  const double* zd = reinterpret_cast<const double*>(z);
  for (int K = threadIdx.x; K < P; K += blockDim.x) {
    int pos, comp;
    dct_slot(K, P, L, &pos, &comp);
    g(K, zd[2 * pos + comp] * scale);
  }
}

// ---- pair step ------------------------------------------------------------
// From Z[k], Z[M-k] (natural order, after the forward FFT) to the four DCT-II
// coefficients C[k], C[P-k], C[M-k], C[M+k] (0 < k < M/2).
struct Quad {
  double c0, c1, c2, c3;  // indices k, P-k, M-k, M+k
};

__device__ __forceinline__ Quad pair_forward(double2 A, double2 B, double2 wk, double2 dk, double2 dk2) {
  double2 Ze = scl2(add2(A, conj2(B)), 0.5);
  double2 D = sub2(A, conj2(B));
  double2 Zo = make_double2(0.5 * D.y, -0.5 * D.x);  // -i D / 2
  double2 wZo = cmul(wk, Zo);
  double2 Vk = add2(Ze, wZo);
  double2 Vk2 = conj2(sub2(Ze, wZo));
  double2 tk = cmul(dk, Vk);
  double2 tk2 = cmul(dk2, Vk2);
  Quad q;
  q.c0 = tk.x;
  q.c1 = -tk.y;
  q.c2 = tk2.x;
  q.c3 = -tk2.y;
  return q;
}

// inverse of pair_forward: coefficients E[k], E[P-k], E[M-k], E[M+k] -> Z'[k], Z'[M-k]
__device__ __forceinline__ void pair_inverse(const Quad& e, double2 wk, double2 dk, double2 dk2, double2* Zk,
                                             double2* Zk2) {
  double2 Vk = cmul(conj2(dk), make_double2(e.c0, -e.c1));
  double2 Vk2 = cmul(conj2(dk2), make_double2(e.c2, -e.c3));
  double2 Ze = scl2(add2(Vk, conj2(Vk2)), 0.5);
  double2 Zo = scl2(cmul(sub2(Vk, conj2(Vk2)), conj2(wk)), 0.5);
  *Zk = make_double2(Ze.x - Zo.y, Ze.y + Zo.x);
  *Zk2 = make_double2(Ze.x + Zo.y, -Ze.y + Zo.x);
}

// k = 0: C[0] and C[M] (C[P] does not exist)
__device__ __forceinline__ void zero_forward(double2 A, double2 dM, double* c0, double* cM) {
  double V0 = A.x + A.y;
  double VM = A.x - A.y;
  *c0 = V0;
  *cM = VM * dM.x;
}
__device__ __forceinline__ double2 zero_inverse(double e0, double eM, double2 dM) {
  double2 VM = cmul(conj2(dM), make_double2(eM, -eM));
  double2 Ze = scl2(add2(make_double2(e0, 0.0), conj2(VM)), 0.5);
  double2 Zo = scl2(sub2(make_double2(e0, 0.0), conj2(VM)), 0.5);
  return make_double2(Ze.x - Zo.y, Ze.y + Zo.x);
}
// k = M/2: C[M/2], C[P-M/2]
__device__ __forceinline__ void mid_forward(double2 A, double2 dh, double* ch, double* cPh) {
  double2 t = cmul(dh, conj2(A));
  *ch = t.x;
  *cPh = -t.y;
}
__device__ __forceinline__ double2 mid_inverse(double eh, double ePh, double2 dh) {
  double2 V = cmul(conj2(dh), make_double2(eh, -ePh));
  return conj2(V);
}

// ---- whole transforms ------------------------------------------------------

// C[q] for q in [0, P): forward DCT-II of f; emit(q, C[q]) for every q (C[P] is not emitted).
template <class F, class E>
__device__ __forceinline__ void dct2_forward(double2* z, const DReq& r, F f, E emit) {
  const int P = r.NP, M = r.M, L = r.L;
  __syncthreads();
  dct_load(z, P, L, f);
  fft_dit(z, M, L, r.tw);
  const int H = M >> 1;
  for (int k = threadIdx.x; k <= H; k += blockDim.x) {
    if (k == 0) {
      double c0, cM;
      zero_forward(z[0], __ldg(&r.twD[M]), &c0, &cM);
      emit(0, c0);
      emit(M, cM);
    } else if (k == H) {
      double ch, cPh;
      mid_forward(z[H], __ldg(&r.twD[H]), &ch, &cPh);
      emit(H, ch);
      emit(P - H, cPh);
    } else {
      Quad q = pair_forward(z[k], z[M - k], __ldg(&r.twP[k]), __ldg(&r.twD[k]), __ldg(&r.twD[M - k]));
      emit(k, q.c0);
      emit(P - k, q.c1);
      emit(M - k, q.c2);
      emit(M + k, q.c3);
    }
  }
  __syncthreads();
}

// y = iDCT2(E), E[q] = get(q) for q in [0, P); store(K, y[K])
template <class G, class S>
__device__ __forceinline__ void dct2_inverse(double2* z, const DReq& r, G get, S store) {
  const int P = r.NP, M = r.M, L = r.L;
  const int H = M >> 1;
  __syncthreads();
  for (int k = threadIdx.x; k <= H; k += blockDim.x) {
    if (k == 0) {
      z[0] = zero_inverse(get(0), get(M), __ldg(&r.twD[M]));
    } else if (k == H) {
      z[H] = mid_inverse(get(H), get(P - H), __ldg(&r.twD[H]));
    } else {
      Quad e;
      e.c0 = get(k);
      e.c1 = get(P - k);
      e.c2 = get(M - k);
      e.c3 = get(M + k);
      double2 a, b;
      pair_inverse(e, __ldg(&r.twP[k]), __ldg(&r.twD[k]), __ldg(&r.twD[M - k]), &a, &b);
      z[k] = a;
      z[M - k] = b;
    }
  }
  ifft_dif(z, M, r.L, r.tw);
  dct_store(z, P, L, 1.0 / (double)M, store);
  __syncthreads();
}

// y = iDCT2(W .* DCT2(f)); W[q] = wgt(q); store(K, y[K])
template <class F, class W, class S>
__device__ __forceinline__ void dct2_convolve(double2* z, const DReq& r, F f, W wgt, S store) {
  const int P = r.NP, M = r.M, L = r.L;
  const int H = M >> 1;
  __syncthreads();
  dct_load(z, P, L, f);
  fft_dit(z, M, L, r.tw);
  for (int k = threadIdx.x; k <= H; k += blockDim.x) {
    if (k == 0) {
      double2 dM = __ldg(&r.twD[M]);
      double c0, cM;
      zero_forward(z[0], dM, &c0, &cM);
      z[0] = zero_inverse(c0 * wgt(0), cM * wgt(M), dM);
    } else if (k == H) {
      double2 dh = __ldg(&r.twD[H]);
      double ch, cPh;
      mid_forward(z[H], dh, &ch, &cPh);
      z[H] = mid_inverse(ch * wgt(H), cPh * wgt(P - H), dh);
    } else {
      double2 wk = __ldg(&r.twP[k]), dk = __ldg(&r.twD[k]), dk2 = __ldg(&r.twD[M - k]);
      Quad q = pair_forward(z[k], z[M - k], wk, dk, dk2);
      q.c0 *= wgt(k);
      q.c1 *= wgt(P - k);
      q.c2 *= wgt(M - k);
      q.c3 *= wgt(M + k);
      double2 a, b;
      pair_inverse(q, wk, dk, dk2, &a, &b);
      z[k] = a;
      z[M - k] = b;
    }
  }
  ifft_dif(z, M, L, r.tw);
  dct_store(z, P, L, 1.0 / (double)M, store);
  __syncthreads();
}

}  // namespace sdft
