// objective.cuh -- one evaluation of the fixed-point map G(x) by one CTA.
//
// Restates objective_dft (src/iDFT/evaluation/objective/objective_dft.jl:17-30):
//   lambda       get_onebody_potential!      eval_spatial_density.jl:138-149
//   chains       compute_child_propagators   freely_jointed/child_propagators.jl:1-162
//                compute_parent_propagators  freely_jointed/parent_propagators.jl:1-142
//                handle_fixed                freely_jointed/handle_fixed.jl:1-120
//                accumulate_densities!       freely_jointed/accumulate_densities.jl:95-184
//   beads        update_spatial_structures!  functions/update_spatial_structures.jl:1-34
//   rho_hat      calc_rho_beads/bonds_hat!   fourier_transforms/calc_rho_hat.jl:17-97
//   functionals  TPT1mfmt / mfmt            functionals/excluded_volume/{TPT1mfmt,mfmt}.jl
//                TPT1msa / msa              functionals/electrostaticcorrelations/{TPT1msa,msa}.jl
//   mu, lng      eval_mu_functionals         functions/eval_mu_functional.jl:1-52
//   Psi, PsiC    solve_coulomb               coulomb/models/coulomb.jl:84-125, coulomb/neutrality_shift.jl
// All convolutions run in DCT-II coefficient space (fft.cuh).  Linear chains
// (parent of segment g is g-1) with an optional grafted segment 0.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace sdft {
namespace {  // internal linkage: each kernel build (kernels.cuh) has its own copy

struct Shared {
  double2* z;   // TB transform buffers (fft.cuh)
  double* red;  // 1024 doubles
};

__device__ __forceinline__ const double* xs_mu(const DReq& r, const double* x) { return x; }
__device__ __forceinline__ const double* xs_lng(const DReq& r, const double* x) { return x + (size_t)r.NP * r.NB; }
__device__ __forceinline__ const double* xs_psi(const DReq& r, const double* x) {
  return x + (size_t)r.NP * (r.NB + 2 * r.MB);
}
__device__ __forceinline__ size_t off_psic(const DReq& r) { return (size_t)r.NP * (r.NB + 2 * r.MB + 1); }
// grid points: odd grids (their stride NP is one more) only run in the general
// build, so the power-of-two build reads the stride itself
__device__ __forceinline__ int grid_points(const DReq& r) { return SDFT_FFT_GEN ? r.NPt : r.NP; }

__device__ __forceinline__ double dist2_grid(int K, int c, double dz) {
  double d = (double)(K - c) * dz;
  return d * d;
}

// ---------------------------------------------------------------------------
// lambda_K = mu_ex_K + (Psi + PsiC) z + Ext + dmuH
// ---------------------------------------------------------------------------
// lambda and e^{-lambda}; each thread takes four elements a round, every load of
// the round issued before the first use
__device__ void stage_lambda(const DReq& r) {
  constexpr int U = 4;
  const int P = r.NP, total = r.NB * P, bd = blockDim.x;
  const double* mu = xs_mu(r, r.x);
  const double* psi = xs_psi(r, r.x);
  const double psic = r.x[off_psic(r)];
  for (int i0 = threadIdx.x; i0 < total; i0 += U * bd) {
    double m[U], ps[U], ex[U];
#pragma unroll
    for (int k = 0; k < U; k++) {
      const int idx = i0 + k * bd;
      if (idx >= total) continue;
      const int K = idx - (idx / P) * P;
      m[k] = mu[idx];
      ps[k] = psi[K];
      ex[k] = r.Ext[idx];
    }
#pragma unroll
    for (int k = 0; k < U; k++) {
      const int idx = i0 + k * bd;
      if (idx >= total) continue;
      const int j = idx / P;
      const double p = ps[k] + psic;
      const double lam = m[k] + p * r.z[j] + ex[k] + r.dmu[j];
      r.lambda[idx] = lam;
      r.elam[idx] = exp(-lam);
    }
  }
  __syncthreads();
}

// Bond-end factors of the propagator convolutions for the current x, one pair
// of fields per bond end (b, e) with bead j = bonds[2b + e]:
//   Fin  = e^{-lambda_j + lng_{b,e}/2} trapez_j   (the input factor of a
//          convolution towards the bead at this end, child_propagators.jl:118-133)
//   Fout = e^{lng_{b,e}/2}                          (the output factor at this end)
// computed once per evaluation instead of once per (segment, state pair).
// In an FP32 evaluation the factors are also written as floats, the input
// factors divided by one power of two 2^sc and the output factors by one 2^so
// that bring their maxima below 1 (e^{-lambda} and e^{lng/2} can exceed the
// float range far from the solution); sc and so go to scal[1] and scal[2], and
// every FP32 convolution step adds sc + so to the carried propagator exponent
// (its outputs are the true propagators times 2^-(sc+so); the grafted
// segment's local sums are shifted to match).
__device__ void stage_bond_factors(const DReq& r, Shared sh, bool fp32) {
  constexpr int U = 4;  // elements a round per thread, loads issued before the first use
  const int P = r.NP, nbe = 2 * r.MB, total = nbe * P, bd = blockDim.x, Pt = grid_points(r);
  const double* lng = xs_lng(r, r.x);
  double mx = 0.0, mo = 0.0;  // largest input factor and output factor e^{lng/2}
  for (int i0 = threadIdx.x; i0 < total; i0 += U * bd) {
    double l[U], lam[U], tr[U];
#pragma unroll
    for (int k = 0; k < U; k++) {
      const int idx = i0 + k * bd;
      if (idx >= total) continue;
      const int be = idx / P, K = idx - be * P;
      const int j = r.bonds[be];
      l[k] = lng[idx];
      lam[k] = r.lambda[(size_t)j * P + K];
      tr[k] = r.trapez[(size_t)j * P + K];
    }
#pragma unroll
    for (int k = 0; k < U; k++) {
      const int idx = i0 + k * bd;
      if (idx >= total) continue;
      const int K = idx - (idx / P) * P;
      const double fin = exp(-lam[k] + l[k] / 2.0) * tr[k];
      const double fo = exp(l[k] / 2.0);
      r.fbe[idx] = fin;
      r.fbe[(size_t)nbe * P + idx] = fo;
      if (K < Pt && isfinite(fin)) mx = fmax(mx, fin);
      if (K < Pt && isfinite(fo)) mo = fmax(mo, fo);
    }
  }
  if (fp32 && r.fbe32) {
    block_max2(&mx, &mo, sh.red);
    int sc = 0, so = 0;
    if (mx > 0.0) frexp(mx, &sc);
    if (mo > 0.0) frexp(mo, &so);
    for (int idx = threadIdx.x; idx < nbe * P; idx += blockDim.x) {
      r.fbe32[idx] = (float)ldexp(r.fbe[idx], -sc);
      r.fbe32[(size_t)nbe * P + idx] = (float)ldexp(r.fbe[(size_t)nbe * P + idx], -so);
    }
    if (threadIdx.x == 0) {
      r.scal[1] = (double)sc;
      r.scal[2] = (double)so;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// chain propagators
//
// Per-segment renormalisation: the reference scales propagators only by
// `normative`, so products over ~100+ segments underflow and the density
// prefactor e^{mu_species} overflows.  When the largest entry of a segment's
// propagators leaves [2^-400, 2^400] the entries are divided by the power of two
// 2^e that brings the maximum into [0.5, 1) -- an exact scaling -- and e is
// carried (expo); otherwise e = 0 and the arithmetic is the reference's.
// ---------------------------------------------------------------------------
// precision of the propagator stage: R = double (FP64) or float (mixed)
template <class R>
__device__ __forceinline__ FftCtxT<double2> fft_ctx_sel(double2* z, const DReq& r, double*) {
  return make_fft(z, r);
}
template <class R>
__device__ __forceinline__ FftCtxT<float2> fft_ctx_sel(double2* z, const DReq& r, float*) {
  return make_fft32(z, r);
}
template <class R>
__device__ __forceinline__ auto fft_ctx(double2* z, const DReq& r) {
  return fft_ctx_sel<R>(z, r, (R*)nullptr);
}
__device__ __forceinline__ const double* bond_factors(const DReq& r, double*) { return r.fbe; }
__device__ __forceinline__ const float* bond_factors(const DReq& r, float*) { return r.fbe32; }
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2((double)v.x, (double)v.y); }

// fp32_bounds: the propagators feed FP32 convolutions (mixed precision) and
// are kept in [2^-30, 2^30], so that the FP32 inputs (factors <= 1 times
// propagator sums) stay far from the float range; FP64 keeps [2^-400, 2^400].
// P is the stride, Pt the number of grid points (the maximum ignores the pad
// point of odd grids)
__device__ int renormalise_block(double* a, int count_per_K, int P, int Pt, double* red, bool fp32_bounds) {
  const double lo = fp32_bounds ? 0x1p-30 : 0x1p-400, hi = fp32_bounds ? 0x1p30 : 0x1p400;
  double mx = 0.0;
  for (int K = threadIdx.x; K < Pt; K += blockDim.x)
    for (int q = 0; q < count_per_K; q++) mx = fmax(mx, fabs(a[(size_t)q * P + K]));
  mx = block_max(mx, red);
  if (!(mx > 0.0) || !isfinite(mx)) return 0;
  if (mx >= lo && mx <= hi) return 0;
  int e;
  frexp(mx, &e);
  for (int K = threadIdx.x; K < P; K += blockDim.x)
    for (int q = 0; q < count_per_K; q++) a[(size_t)q * P + K] = ldexp(a[(size_t)q * P + K], -e);
  __syncthreads();
  return e;
}

template <class R>
__device__ bool chain_child(const DReq& r, const DSpecies& s, Shared sh) {
  const int P = r.NP, S = s.S, N = s.n_seg;
  double* const gC = s.gC;
  // FP32: the factors are stored divided by 2^sc (inputs) and 2^so (outputs), stage_bond_factors
  const int sc = sizeof(R) == 4 ? (int)r.scal[1] + (int)r.scal[2] : 0;
  bool scaled = false;
  int e_child = 0;  // exponent carried by gC of segment p + 1 (the leaf carries none)
  const double* lng = xs_lng(r, r.x);
  const double inv_norm = 1.0 / s.normative;
  const auto fc = fft_ctx<R>(sh.z, r);
  for (int p = N - 2; p >= 0; p--) {
    const int c = p + 1;
    const int nc = s.nst[c];
    const int npair = s.nst[p] * nc;
    if (p == 0 && s.fixed >= 0) {
      for (int pi = 0; pi < npair; pi++) {
        const int ii = pi / nc, jj = pi - ii * nc;
        const int si = s.states[p * S + ii], sj = s.states[c * S + jj];
        const int bond = s.bnd[(p * S + ii) * S + jj];
        const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
        double* out = gC + ((size_t)(p * S + ii) * S + jj) * P;
        const double* lam_j = r.lambda + (size_t)sj * P;
        const double* lng_pj = lng + (size_t)(bond * 2 + pair_j) * P;
        const double* lng_pi = lng + (size_t)(bond * 2 + pair_i) * P;
        const double* tr_j = r.trapez + (size_t)sj * P;
        const double* gcc = (c < N - 1) ? gC + ((size_t)(c * S + jj) * S) * P : nullptr;
        // parent grafted, child free: local sum within sigma_ij (child_propagators.jl:91-116)
        const int Kp = s.fixed;
        const double Dij = (r.sig[si] + r.sig[sj]) / 2.0;
        const double Dij2 = Dij * Dij;
        const double renorm = 2.0 * Dij;
        const double el = exp(lng_pi[Kp] / 2.0);
        double acc = 0.0;
        for (int K1 = threadIdx.x; K1 < grid_points(r); K1 += blockDim.x) {
          double d2 = dist2_grid(K1, Kp, r.dz);
          if (d2 <= Dij2) {
            double f = exp(-lam_j[K1] + lng_pj[K1] / 2.0);
            if (gcc) {
              double t = 0.0;
              for (int q = 0; q < S; q++) t += gcc[(size_t)q * P + K1];
              f *= t;
            }
            double t = fabs(f) * el * r.dz * tr_j[K1] / renorm;
            if (fabs(d2 - Dij2) <= 1e-6) t /= 2.0;
            acc += t / s.normative;
          }
        }
        acc = block_sum(acc, sh.red);
        if (sc) acc = ldexp(acc, -sc);
        for (int K = threadIdx.x; K < P; K += blockDim.x) out[K] = (K == Kp) ? acc : 0.0;
      }
    } else {
      const R* fin = bond_factors(r, (R*)nullptr);
      const R* fout = fin + (size_t)2 * r.MB * P;
      for (int g0 = 0; g0 < npair; g0 += r.TB) {
        const int nT = min(r.TB, npair - g0);
        const R* in_t[kMaxTB];
        const R* out_f[kMaxTB];
        const double* gcc_t[kMaxTB];
        const double* wb_t[kMaxTB];
        double* out_t[kMaxTB];
        for (int t = 0; t < nT; t++) {
          const int pi = g0 + t, ii = pi / nc, jj = pi - ii * nc;
          const int si = s.states[p * S + ii], sj = s.states[c * S + jj];
          const int bond = s.bnd[(p * S + ii) * S + jj];
          const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
          out_t[t] = gC + ((size_t)(p * S + ii) * S + jj) * P;
          in_t[t] = fin + (size_t)(bond * 2 + pair_j) * P;
          out_f[t] = fout + (size_t)(bond * 2 + pair_i) * P;
          gcc_t[t] = (c < N - 1) ? gC + ((size_t)(c * S + jj) * S) * P : nullptr;
          wb_t[t] = r.Wbond + (size_t)bond * P;
        }
        dct2_convolve_b2(
            fc, nT,
            [&](int t, int K) {
              const auto fin = ldcg2(in_t[t] + K);
              double2 f = make_double2(fin.x, fin.y);
              if (gcc_t[t]) {
                double2 q2 = make_double2(0.0, 0.0);
                for (int q = 0; q < S; q++) {
                  const double2 v = ldcg2(gcc_t[t] + (size_t)q * P + K);
                  q2.x += v.x;
                  q2.y += v.y;
                }
                f.x *= q2.x;
                f.y *= q2.y;
              }
              return f;
            },
            [&](int t, int q) { return __ldg(&wb_t[t][q]); },
            [&](int t, int K) { return ldcg2(out_f[t] + K); },
            [&](int t, int K, auto y, auto fo) {
              stcg2(out_t[t] + K, make_double2(fabs((double)y.x) * (double)fo.x * inv_norm,
                                               fabs((double)y.y) * (double)fo.y * inv_norm));
            });
      }
    }
    if (s.fixed >= 0) {  // max-distance mask (child_propagators.jl:147-157)
      const double md2 = s.md[p] * s.md[p];
      __syncthreads();
      for (int K = threadIdx.x; K < P; K += blockDim.x)
        if (dist2_grid(K, s.fixed, r.dz) > md2)
          for (int q = 0; q < S * S; q++) gC[((size_t)p * S * S + q) * P + K] = 0.0;
    }
    __syncthreads();
    const int e = renormalise_block(gC + (size_t)p * S * S * P, S * S, P, grid_points(r), sh.red, sizeof(R) == 4);
    e_child += e + sc;
    scaled |= (e + sc) != 0;
    if (threadIdx.x == 0) s.expo[p] = e_child;
  }
  if (threadIdx.x == 0) s.expo[N - 1] = 0;
  __syncthreads();
  return scaled;
}

template <class R>
__device__ bool chain_parent(const DReq& r, const DSpecies& s, Shared sh) {
  const int P = r.NP, S = s.S, N = s.n_seg;
  double* const gP = s.gP;
  // FP32: the factors are stored divided by 2^sc (inputs) and 2^so (outputs), stage_bond_factors
  const int sc = sizeof(R) == 4 ? (int)r.scal[1] + (int)r.scal[2] : 0;
  bool scaled = false;
  int e_parent = 0;  // exponent carried by gP of segment c - 1 (the root carries none)
  if (threadIdx.x == 0) s.expo[N] = 0;
  const double* lng = xs_lng(r, r.x);
  const double inv_norm = 1.0 / s.normative;
  // root: base case gP[K, 1, idx_i, root] = 1 (only the graft point when fixed)
  for (int K = threadIdx.x; K < P; K += blockDim.x) {
    for (int ii = 0; ii < S; ii++)
      for (int jj = 0; jj < S; jj++) {
        double v = 0.0;
        if (jj == 0 && ii < s.nst[0]) v = (s.fixed < 0 || K == s.fixed) ? 1.0 : 0.0;
        gP[((size_t)ii * S + jj) * P + K] = v;
      }
  }
  __syncthreads();
  const auto fc = fft_ctx<R>(sh.z, r);
  for (int c = 1; c < N; c++) {
    const int p = c - 1;
    // base case then the parent loop overwrites slot jj < nst[p]
    for (int K = threadIdx.x; K < P; K += blockDim.x)
      for (int ii = 0; ii < S; ii++)
        for (int jj = 0; jj < S; jj++)
          gP[((size_t)(c * S + ii) * S + jj) * P + K] = (jj == 0 && ii < s.nst[c]) ? 1.0 : 0.0;
    __syncthreads();
    const int np_ = s.nst[p];
    const int npair = s.nst[c] * np_;
    if (p == 0 && s.fixed >= 0) {
      for (int pi = 0; pi < npair; pi++) {
        const int ii = pi / np_, jj = pi - ii * np_;
        const int si = s.states[c * S + ii], sj = s.states[p * S + jj];
        const int bond = s.bnd[(p * S + jj) * S + ii];
        const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
        double* out = gP + ((size_t)(c * S + ii) * S + jj) * P;
        const double* lng_pj = lng + (size_t)(bond * 2 + pair_j) * P;
        const double* lng_pi = lng + (size_t)(bond * 2 + pair_i) * P;
        const double* gpp = gP + ((size_t)(p * S + jj) * S) * P;
        // parent grafted (parent_propagators.jl:72-94)
        const int Kp = s.fixed;
        const double Dij = (r.sig[si] + r.sig[sj]) / 2.0;
        const double Dij2 = Dij * Dij;
        const double renorm = 2.0 * Dij;
        double tq = 0.0;
        for (int q = 0; q < S; q++) tq += gpp[(size_t)q * P + Kp];
        const double f = exp(-r.lambda[(size_t)sj * P + Kp] + lng_pj[Kp] / 2.0) * tq;
        for (int K1 = threadIdx.x; K1 < grid_points(r); K1 += blockDim.x) {
          double d2 = dist2_grid(K1, Kp, r.dz);
          if (d2 <= Dij2) {
            double v = fabs(f) * exp(lng_pi[K1] / 2.0) / renorm / s.normative;
            if (fabs(d2 - Dij2) <= 1e-6) v /= 2.0;
            out[K1] = sc ? ldexp(v, -sc) : v;
          }
        }
        __syncthreads();
      }
    } else {
      const R* fin = bond_factors(r, (R*)nullptr);
      const R* fout = fin + (size_t)2 * r.MB * P;
      for (int g0 = 0; g0 < npair; g0 += r.TB) {
        const int nT = min(r.TB, npair - g0);
        const R* in_t[kMaxTB];
        const R* out_f[kMaxTB];
        const double* gpp_t[kMaxTB];
        const double* wb_t[kMaxTB];
        double* out_t[kMaxTB];
        for (int t = 0; t < nT; t++) {
          const int pi = g0 + t, ii = pi / np_, jj = pi - ii * np_;
          const int si = s.states[c * S + ii], sj = s.states[p * S + jj];
          const int bond = s.bnd[(p * S + jj) * S + ii];
          const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
          out_t[t] = gP + ((size_t)(c * S + ii) * S + jj) * P;
          in_t[t] = fin + (size_t)(bond * 2 + pair_j) * P;
          out_f[t] = fout + (size_t)(bond * 2 + pair_i) * P;
          gpp_t[t] = gP + ((size_t)(p * S + jj) * S) * P;
          wb_t[t] = r.Wbond + (size_t)bond * P;
        }
        dct2_convolve_b2(
            fc, nT,
            [&](int t, int K) {
              double2 q2 = make_double2(0.0, 0.0);
              for (int q = 0; q < S; q++) {
                const double2 v = ldcg2(gpp_t[t] + (size_t)q * P + K);
                q2.x += v.x;
                q2.y += v.y;
              }
              const auto in = ldcg2(in_t[t] + K);
              return make_double2((double)in.x * q2.x, (double)in.y * q2.y);
            },
            [&](int t, int q) { return __ldg(&wb_t[t][q]); },
            [&](int t, int K) { return ldcg2(out_f[t] + K); },
            [&](int t, int K, auto y, auto fo) {
              stcg2(out_t[t] + K, make_double2(fabs((double)y.x) * (double)fo.x * inv_norm,
                                               fabs((double)y.y) * (double)fo.y * inv_norm));
            });
      }
    }
    if (s.fixed >= 0) {
      const double md2 = s.md[c] * s.md[c];
      __syncthreads();
      for (int K = threadIdx.x; K < P; K += blockDim.x)
        if (dist2_grid(K, s.fixed, r.dz) > md2)
          for (int q = 0; q < S * S; q++) gP[((size_t)c * S * S + q) * P + K] = 0.0;
    }
    __syncthreads();
    const int e = renormalise_block(gP + (size_t)c * S * S * P, S * S, P, grid_points(r), sh.red, sizeof(R) == 4);
    e_parent += e + sc;
    scaled |= (e + sc) != 0;
    if (threadIdx.x == 0) s.expo[N + c] = e_parent;
  }
  __syncthreads();
  return scaled;
}

// ---------------------------------------------------------------------------
// Both recursions of a linear chain in one loop (even grids).  The child
// recursion (child_propagators.jl:118-141) runs from the leaf to the root and
// the parent recursion (parent_propagators.jl:96-122) from the root to the leaf;
// neither reads the other, so step t computes gC of segment p = N-2-t and gP of
// segment c = t+1 together: up to 2 S^2 transforms share each FFT pass, and a
// chain of N segments takes N-1 steps of passes instead of 2(N-1).  The
// arithmetic per entry is that of chain_child / chain_parent: input
// Fin * sum_q g[prev][j][q], the filtered bond-kernel convolution, output
// |y| Fout / normative, the max-distance mask of grafted species, the grafted
// segment's local sums, and per-segment power-of-two renormalisation with the
// same exponent bookkeeping (expo[p] child, expo[N + c] parent).
// ---------------------------------------------------------------------------
struct FuseT {             // one transform of a fused chain step (shared memory)
  const void* fin;         // input bond-end factor (R)
  const void* fout;        // output bond-end factor (R)
  const void* src;         // S slots of the previous segment's propagator (R), summed; nullptr: the base case 1
  const double* w;         // filtered bond kernel in C-space
  void* out;               // propagator slot written (R)
  int sweep;               // 0: child recursion, 1: parent recursion
  int pad;
};
constexpr int kFuseOffset = 64;  // FuseT table position in Shared::red (doubles), after the reduction slots

// exponent of the power of two that brings mx into [0.5, 1) when mx leaves
// [2^-400, 2^400] ([2^-30, 2^30] for FP32 propagator convolutions); else 0
__device__ __forceinline__ int renorm_exponent(double mx, bool fp32_bounds) {
  const double lo = fp32_bounds ? 0x1p-30 : 0x1p-400, hi = fp32_bounds ? 0x1p30 : 0x1p400;
  if (!(mx > 0.0) || !isfinite(mx)) return 0;
  if (mx >= lo && mx <= hi) return 0;
  int e;
  frexp(mx, &e);
  return e;
}

template <class T>
__device__ void rescale_segment(T* a, int count_per_K, int P, int e) {
  for (int K = threadIdx.x; K < P; K += blockDim.x)
    for (int q = 0; q < count_per_K; q++) a[(size_t)q * P + K] = (T)ldexp((double)a[(size_t)q * P + K], -e);
}

template <class R, int SM>
__device__ bool chain_sweeps(const DReq& r, const DSpecies& s, Shared sh) {
  using R2 = decltype(ldcg2((const R*)nullptr));
  const int P = r.NP, S = s.S, N = s.n_seg;
  // propagators are stored in the precision of the step (FP32 in a mixed evaluation)
  R* const gC = reinterpret_cast<R*>(s.gC);
  R* const gP = reinterpret_cast<R*>(s.gP);
  // FP32: the factors are stored divided by 2^sc (inputs) and 2^so (outputs), stage_bond_factors
  const int sc = sizeof(R) == 4 ? (int)r.scal[1] + (int)r.scal[2] : 0;
  const bool fp32 = sizeof(R) == 4;
  const double* lng = xs_lng(r, r.x);
  const double inv_norm = 1.0 / s.normative;
  const R* fin = bond_factors(r, (R*)nullptr);
  const R* fout = fin + (size_t)2 * r.MB * P;
  FuseT* fd = reinterpret_cast<FuseT*>(sh.red + kFuseOffset);
  const auto fc = fft_ctx<R>(sh.z, r);
  bool scaled = false;
  int eC = 0, eP = 0;  // exponents carried by gC of segment p + 1 and gP of segment c - 1
  // root base case of the parent recursion: gP[0][i][0] = 1 (only at the graft point when fixed)
  for (int K = threadIdx.x; K < P; K += blockDim.x)
    for (int ii = 0; ii < S; ii++)
      for (int jj = 0; jj < S; jj++)
        gP[((size_t)ii * S + jj) * P + K] =
            (R)((jj == 0 && ii < s.nst[0] && (s.fixed < 0 || K == s.fixed)) ? 1.0 : 0.0);
  if (threadIdx.x == 0) {
    s.expo[N - 1] = 0;
    s.expo[N] = 0;
  }
  for (int t = 0; t < N - 1; t++) {
    const int p = N - 2 - t, c = p + 1;  // child recursion: gC[p] from gC[c]
    const int c2 = t + 1, p2 = t;        // parent recursion: gP[c2] from gP[p2]
    const bool child_local = p == 0 && s.fixed >= 0;
    const bool parent_local = p2 == 0 && s.fixed >= 0;
    const int ncC = s.nst[c], npP = s.nst[p2];
    const int nC = child_local ? 0 : s.nst[p] * ncC;
    const int nP = parent_local ? 0 : s.nst[c2] * npP;
    const int nT = nC + nP;
    __syncthreads();  // the previous step's table and outputs are complete
    if (threadIdx.x < nT) {
      FuseT d;
      const int q = threadIdx.x;
      if (q < nC) {  // child pair (ii of p, jj of c)
        const int ii = q / ncC, jj = q - ii * ncC;
        const int si = s.states[p * S + ii], sj = s.states[c * S + jj];
        const int bond = s.bnd[(p * S + ii) * S + jj];
        const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
        d.fin = fin + (size_t)(bond * 2 + pair_j) * P;
        d.fout = fout + (size_t)(bond * 2 + pair_i) * P;
        d.src = c < N - 1 ? gC + ((size_t)(c * S + jj) * S) * P : nullptr;
        d.w = r.Wbond + (size_t)bond * P;
        d.out = gC + ((size_t)(p * S + ii) * S + jj) * P;
        d.sweep = 0;
      } else {  // parent pair (ii of c2, jj of p2)
        const int qq = q - nC, ii = qq / npP, jj = qq - ii * npP;
        const int si = s.states[c2 * S + ii], sj = s.states[p2 * S + jj];
        const int bond = s.bnd[(p2 * S + jj) * S + ii];
        const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
        d.fin = fin + (size_t)(bond * 2 + pair_j) * P;
        d.fout = fout + (size_t)(bond * 2 + pair_i) * P;
        d.src = gP + ((size_t)(p2 * S + jj) * S) * P;
        d.w = r.Wbond + (size_t)bond * P;
        d.out = gP + ((size_t)(c2 * S + ii) * S + jj) * P;
        d.sweep = 1;
      }
      d.pad = 0;
      fd[q] = d;
    }
    double mxC = 0.0, mxP = 0.0;  // largest output of each recursion at this step (this thread)
    // grafted segment 0 as the child's parent: local sums within sigma_ij (child_propagators.jl:91-116)
    if (child_local) {
      const int Kp = s.fixed;
      for (int pi = 0; pi < s.nst[p] * ncC; pi++) {
        const int ii = pi / ncC, jj = pi - ii * ncC;
        const int si = s.states[p * S + ii], sj = s.states[c * S + jj];
        const int bond = s.bnd[(p * S + ii) * S + jj];
        const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
        const double* lam_j = r.lambda + (size_t)sj * P;
        const double* lng_pj = lng + (size_t)(bond * 2 + pair_j) * P;
        const double* lng_pi = lng + (size_t)(bond * 2 + pair_i) * P;
        const double* tr_j = r.trapez + (size_t)sj * P;
        const R* gcc = (c < N - 1) ? gC + ((size_t)(c * S + jj) * S) * P : nullptr;
        const double Dij = (r.sig[si] + r.sig[sj]) / 2.0;
        const double Dij2 = Dij * Dij;
        const double renorm = 2.0 * Dij;
        const double el = exp(lng_pi[Kp] / 2.0);
        double acc = 0.0;
        for (int K1 = threadIdx.x; K1 < P; K1 += blockDim.x) {
          const double d2 = dist2_grid(K1, Kp, r.dz);
          if (d2 <= Dij2) {
            double f = exp(-lam_j[K1] + lng_pj[K1] / 2.0);
            if (gcc) {
              double tq = 0.0;
              for (int q = 0; q < S; q++) tq += (double)gcc[(size_t)q * P + K1];
              f *= tq;
            }
            double v = fabs(f) * el * r.dz * tr_j[K1] / renorm;
            if (fabs(d2 - Dij2) <= 1e-6) v /= 2.0;
            acc += v / s.normative;
          }
        }
        acc = block_sum(acc, sh.red);
        if (sc) acc = ldexp(acc, -sc);
        R* out = gC + ((size_t)(p * S + ii) * S + jj) * P;
        // the max-distance mask of segment 0 keeps only the graft point
        const double md2 = s.md[p] * s.md[p];
        for (int K = threadIdx.x; K < P; K += blockDim.x)
          out[K] = (R)((K == Kp && dist2_grid(K, Kp, r.dz) <= md2) ? acc : 0.0);
        mxC = fmax(mxC, fabs(acc));
      }
    }
    // grafted segment 0 as the parent: local writes within sigma_ij (parent_propagators.jl:72-94)
    if (parent_local) {
      const int Kp = s.fixed;
      for (int pi = 0; pi < s.nst[c2] * npP; pi++) {
        const int ii = pi / npP, jj = pi - ii * npP;
        const int si = s.states[c2 * S + ii], sj = s.states[p2 * S + jj];
        const int bond = s.bnd[(p2 * S + jj) * S + ii];
        const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
        const double* lng_pj = lng + (size_t)(bond * 2 + pair_j) * P;
        const double* lng_pi = lng + (size_t)(bond * 2 + pair_i) * P;
        const R* gpp = gP + ((size_t)(p2 * S + jj) * S) * P;
        const double Dij = (r.sig[si] + r.sig[sj]) / 2.0;
        const double Dij2 = Dij * Dij;
        const double renorm = 2.0 * Dij;
        double tq = 0.0;
        for (int q = 0; q < S; q++) tq += (double)gpp[(size_t)q * P + Kp];
        const double f = exp(-r.lambda[(size_t)sj * P + Kp] + lng_pj[Kp] / 2.0) * tq;
        const double md2 = s.md[c2] * s.md[c2];
        const double base = jj == 0 ? 1.0 : 0.0;  // the base case left where no bond reaches
        R* out = gP + ((size_t)(c2 * S + ii) * S + jj) * P;
        for (int K1 = threadIdx.x; K1 < P; K1 += blockDim.x) {
          const double d2 = dist2_grid(K1, Kp, r.dz);
          double v = base;
          if (d2 <= Dij2) {
            v = fabs(f) * exp(lng_pi[K1] / 2.0) / renorm / s.normative;
            if (fabs(d2 - Dij2) <= 1e-6) v /= 2.0;
            if (sc) v = ldexp(v, -sc);
          }
          if (d2 > md2) v = 0.0;
          out[K1] = (R)v;
          mxP = fmax(mxP, fabs(v));
        }
      }
    }
    // the convolutions of both recursions, TB transforms per pass set
    const double mdC = s.fixed >= 0 ? s.md[p] * s.md[p] : 0.0;
    const double mdP = s.fixed >= 0 ? s.md[c2] * s.md[c2] : 0.0;
    for (int g0 = 0; g0 < nT; g0 += r.TB) {
      const int nb = min(r.TB, nT - g0);
      dct2_convolve_kpair(
          fc, nb,
          [&](int kp, auto put) {
            const int K = 2 * kp;
            double2 f[kMaxTB];
#pragma unroll
            for (int u = 0; u < kMaxTB; u++)
              if (u < nb) {
                const FuseT& d = fd[g0 + u];
                // the bond-end factors (4 MB P values) exceed L1 beside the
                // twiddles and bond kernels that every pass rereads: L2 only
                const R2 fv = ldcg2(reinterpret_cast<const R*>(d.fin) + K);
                f[u] = make_double2((double)fv.x, (double)fv.y);
                if (d.src) {
                  double2 q2 = make_double2(0.0, 0.0);
#pragma unroll
                  for (int q = 0; q < SM; q++)
                    if (q < S) {
                      const R2 v = ldcg2(reinterpret_cast<const R*>(d.src) + (size_t)q * P + K);
                      q2.x += v.x;
                      q2.y += v.y;
                    }
                  f[u].x *= q2.x;
                  f[u].y *= q2.y;
                }
              }
#pragma unroll
            for (int u = 0; u < kMaxTB; u++)
              if (u < nb) put(u, f[u]);
          },
          [&](int u, int q) { return __ldg(&fd[g0 + u].w[q]); },
          [&](int kp, auto get) {
            const int K = 2 * kp;
            R2 fo[kMaxTB];
#pragma unroll
            for (int u = 0; u < kMaxTB; u++)
              if (u < nb) fo[u] = ldcg2(reinterpret_cast<const R*>(fd[g0 + u].fout) + K);
            const bool cut = s.fixed >= 0;
#pragma unroll
            for (int u = 0; u < kMaxTB; u++)
              if (u < nb) {
                const FuseT& d = fd[g0 + u];
                const auto y = get(u);
                double2 v = make_double2(fabs((double)y.x) * (double)fo[u].x * inv_norm,
                                         fabs((double)y.y) * (double)fo[u].y * inv_norm);
                if (cut) {  // max-distance mask (child_propagators.jl:147-157)
                  const double md2 = d.sweep ? mdP : mdC;
                  if (dist2_grid(K, s.fixed, r.dz) > md2) v.x = 0.0;
                  if (dist2_grid(K + 1, s.fixed, r.dz) > md2) v.y = 0.0;
                }
                R2 st;
                st.x = (R)v.x;
                st.y = (R)v.y;
                stcg2(reinterpret_cast<R*>(d.out) + K, st);
                const double m = fmax(fabs(v.x), fabs(v.y));
                if (d.sweep) mxP = fmax(mxP, m);
                else mxC = fmax(mxC, m);
              }
          });
    }
    // per-segment renormalisation of both new segments
    block_max2(&mxC, &mxP, sh.red);
    const int ec = renorm_exponent(mxC, fp32), ep = renorm_exponent(mxP, fp32);
    if (ec) rescale_segment(gC + (size_t)p * S * S * P, S * S, P, ec);
    if (ep) rescale_segment(gP + (size_t)c2 * S * S * P, S * S, P, ep);
    eC += ec + sc;
    eP += ep + sc;
    scaled |= (ec + sc) != 0 || (ep + sc) != 0;
    if (threadIdx.x == 0) {
      s.expo[p] = eC;
      s.expo[N + c2] = eP;
    }
  }
  __syncthreads();
  return scaled;
}

// handle_fixed (handle_fixed.jl:1-120): chain normalisation; false on lambda <= 0
template <class R>
__device__ bool chain_norm(const DReq& r, DSpecies& s, Shared sh, double* norm_out) {
  const int P = r.NP, S = s.S, N = s.n_seg;
  const R* gP = reinterpret_cast<const R*>(s.gP);
  const R* gC = reinterpret_cast<const R*>(s.gC);
  double lam, norm;
  if (s.fixed >= 0) {
    norm = s.fixed_density;
    s.mu_species = 0.0;
    const int parent = 1;  // first free segment
    double acc = 0.0;
    for (int K = threadIdx.x; K < grid_points(r); K += blockDim.x) {
      for (int ii = 0; ii < s.nst[parent]; ii++) {
        const int si = s.states[parent * S + ii];
        double sp = 0.0;
        for (int q = 0; q < S; q++) sp += gP[((size_t)(parent * S + ii) * S + q) * P + K];
        double contr = exp(-r.lambda[(size_t)si * P + K]) * sp;
        double temp;
        if (parent < N - 1) {
          temp = 0.0;
          for (int jj = 0; jj < s.nst[parent + 1]; jj++) temp += gC[((size_t)(parent * S + ii) * S + jj) * P + K];
        } else {
          temp = (ii == 0) ? 1.0 : 0.0;  // leaf base case read as gC[K, :, idx_i, 1, parent]
        }
        acc += contr * temp * r.trapez[(size_t)si * P + K] * r.dz;
      }
    }
    lam = block_sum(acc, sh.red);
  } else {
    lam = 1.0;
    norm = s.norm_free;
  }
  if (!isfinite(lam) || lam <= 0.0) return false;
  norm *= 1.0 / lam;
  s.lambda_fixed = lam / s.norm_free;
  *norm_out = norm;
  return true;
}

// ln of the density prefactor of segment g with renormalised propagators:
// norm e^{mu} 2^{eP_g + eC_g}; free chains norm = normative^(N-1), grafted
// chains norm = density / lambda with lambda carrying 2^{eP_1 + eC_1}
__device__ __forceinline__ double log_prefactor(const DSpecies& s, double norm, int g) {
  const int N = s.n_seg;
  const int sg = s.expo[N + g] + (g < N - 1 ? s.expo[g] : 0);
  if (s.fixed >= 0) {
    const int s1 = s.expo[N + 1] + (1 < N - 1 ? s.expo[1] : 0);
    return log(norm) + s.mu_species + (double)(sg - s1) * 0.6931471805599453;
  }
  return s.mu_species + (double)(N - 1) * log(s.normative) + (double)sg * 0.6931471805599453;
}

// accumulate_densities! for one species: rho_seg and both bond ends
template <class R>
__device__ void chain_accumulate(const DReq& r, const DSpecies& s, double norm, bool scaled) {
  const int P = r.NP, S = s.S, N = s.n_seg;
  const R* gP = reinterpret_cast<const R*>(s.gP);
  const R* gC = reinterpret_cast<const R*>(s.gC);
  const double mu = s.mu_species;
  for (int K = threadIdx.x; K < P; K += blockDim.x) {
    for (int g = 0; g < N; g++) {
      const double lp = scaled ? log_prefactor(s, norm, g) : 0.0;
      for (int ii = 0; ii < s.nst[g]; ii++) {
        const int si = s.states[g * S + ii];
        double sp;
        if (N > 1) {
          sp = 0.0;
          for (int q = 0; q < S; q++) sp += gP[((size_t)(g * S + ii) * S + q) * P + K];
        } else {
          sp = (s.fixed < 0 || K == s.fixed) ? 1.0 : 0.0;
        }
        const double contr = scaled ? exp(lp - r.lambda[(size_t)si * P + K]) * sp
                                    : norm * exp(mu - r.lambda[(size_t)si * P + K]) * sp;
        double temp;
        if (g < N - 1) {
          temp = 0.0;
          for (int jj = 0; jj < s.nst[g + 1]; jj++) {
            const int bond = s.bnd[(g * S + ii) * S + jj];
            const double t2 = gC[((size_t)(g * S + ii) * S + jj) * P + K];
            r.rho_bonds[(size_t)(bond * 2 + 0) * P + K] += contr * t2;
            temp += t2;
          }
        } else {
          temp = 1.0;
        }
        s.rho_seg[(size_t)(g * S + ii) * P + K] += contr * temp;
      }
    }
    for (int c = 1; c < N; c++) {
      const double lp = scaled ? log_prefactor(s, norm, c) : 0.0;
      for (int ii = 0; ii < s.nst[c]; ii++) {
        const int si = s.states[c * S + ii];
        double contr = scaled ? exp(lp - r.lambda[(size_t)si * P + K]) : norm * exp(mu - r.lambda[(size_t)si * P + K]);
        if (c < N - 1) {
          double t = 0.0;
          for (int q = 0; q < S; q++) t += gC[((size_t)(c * S + ii) * S + q) * P + K];
          contr *= t;
        }
        for (int jj = 0; jj < s.nst[c - 1]; jj++) {
          const int bond = s.bnd[((c - 1) * S + jj) * S + ii];
          r.rho_bonds[(size_t)(bond * 2 + 1) * P + K] += contr * gP[((size_t)(c * S + ii) * S + jj) * P + K];
        }
      }
    }
  }
  __syncthreads();
}

// a[idx] += v for a register array (idx < N): unrolled select, no local memory
template <int N>
__device__ __forceinline__ void acc_add(double* a, int idx, double v) {
#pragma unroll
  for (int q = 0; q < N; q++)
    if (q == idx) a[q] += v;
}

// accumulate_densities! of one species with its bond-end and bead densities
// summed in registers (species-local slots, BR bond slots, ER bead slots) and
// added to rho_bonds / rho_beads once per grid point, instead of one global
// read-modify-write per segment.  Each point's sums run over (segment, state,
// child state) in the reference's order.  The segment prefactor uses
// e^{-lambda} of the evaluation: norm e^{mu} e^{-lambda_K} (unscaled), or
// e^{lp} e^{-lambda_K} with lp the log prefactor of the renormalised
// propagators (e^{lp - lambda_K} directly when |lp| > 600).  Also adds the
// species to the bead densities (update_spatial_structures.jl:1-34).
template <int BR, int ER, class R>
__device__ __noinline__ void accumulate_regs(const DReq& r, const DSpecies& s, double norm, bool scaled,
                                             const R* __restrict__ gP, const R* __restrict__ gC,
                                             const double* __restrict__ elam, const double* __restrict__ lam,
                                             const int* __restrict__ states, const int* __restrict__ nst,
                                             const int* __restrict__ bslot, const int* __restrict__ eslot,
                                             double* __restrict__ rho_seg, double* __restrict__ rho_bonds,
                                             double* __restrict__ rho_beads) {
  const int P = r.NP, S = s.S, N = s.n_seg;
  const double pref = norm * exp(s.mu_species);
  for (int K = threadIdx.x; K < P; K += blockDim.x) {
    double a0[BR], a1[BR], ab[ER];
#pragma unroll
    for (int q = 0; q < BR; q++) a0[q] = a1[q] = 0.0;
#pragma unroll
    for (int q = 0; q < ER; q++) ab[q] = 0.0;
    for (int g = 0; g < N; g++) {
      double lp = 0.0, elp = pref;
      bool direct = false;
      if (scaled) {
        lp = log_prefactor(s, norm, g);
        direct = fabs(lp) > 600.0;
        elp = exp(lp);
      }
      const int nn = g < N - 1 ? nst[g + 1] : 0;
      for (int ii = 0; ii < nst[g]; ii++) {
        const int si = states[g * S + ii];
        double sp;
        if (N > 1) {
          sp = 0.0;
          for (int q = 0; q < S; q++) sp += gP[((size_t)(g * S + ii) * S + q) * P + K];
        } else {
          sp = (s.fixed < 0 || K == s.fixed) ? 1.0 : 0.0;
        }
        const double contr = direct ? exp(lp - lam[(size_t)si * P + K]) * sp : elp * elam[(size_t)si * P + K] * sp;
        double temp;
        if (nn) {
          temp = 0.0;
          for (int jj = 0; jj < nn; jj++) {
            const double t2 = gC[((size_t)(g * S + ii) * S + jj) * P + K];
            acc_add<BR>(a0, bslot[(g * S + ii) * S + jj], contr * t2);
            temp += t2;
          }
        } else {
          temp = 1.0;
        }
        const double v = contr * temp;
        rho_seg[(size_t)(g * S + ii) * P + K] = v;
        if (g == 0 && s.fixed >= 0) {
          if (K == s.fixed) acc_add<ER>(ab, eslot[g * S + ii], v / r.dz / r.trapez[(size_t)si * P + K]);
        } else {
          acc_add<ER>(ab, eslot[g * S + ii], v);
        }
      }
    }
    for (int c = 1; c < N; c++) {
      double lp = 0.0, elp = pref;
      bool direct = false;
      if (scaled) {
        lp = log_prefactor(s, norm, c);
        direct = fabs(lp) > 600.0;
        elp = exp(lp);
      }
      for (int ii = 0; ii < nst[c]; ii++) {
        const int si = states[c * S + ii];
        double contr = direct ? exp(lp - lam[(size_t)si * P + K]) : elp * elam[(size_t)si * P + K];
        if (c < N - 1) {
          double t = 0.0;
          for (int q = 0; q < S; q++) t += gC[((size_t)(c * S + ii) * S + q) * P + K];
          contr *= t;
        }
        for (int jj = 0; jj < nst[c - 1]; jj++)
          acc_add<BR>(a1, bslot[((c - 1) * S + jj) * S + ii], contr * gP[((size_t)(c * S + ii) * S + jj) * P + K]);
      }
    }
#pragma unroll
    for (int q = 0; q < BR; q++)
      if (q < s.nbslot) {
        const int b = s.bslot_bond[q];
        rho_bonds[(size_t)(b * 2 + 0) * P + K] += a0[q];
        rho_bonds[(size_t)(b * 2 + 1) * P + K] += a1[q];
      }
#pragma unroll
    for (int q = 0; q < ER; q++)
      if (q < s.neslot) rho_beads[(size_t)s.eslot_bead[q] * P + K] += ab[q];
  }
  __syncthreads();
}

// accumulate_regs for chains with at most two states per segment, on grid-point
// pairs (K, K+1) with 16-byte loads, software-pipelined over the segment
// states: the loads of the next (segment, state) are issued before the
// current one is combined, so two steps' memory latencies overlap.  Same sums
// in the same order as accumulate_regs.
struct AccStep {
  double2 el, p0, p1, c0, c1;
};

template <int BR, int ER, class R>
__device__ __noinline__ void accumulate_pairs(const DReq& r, const DSpecies& s, double norm, bool scaled) {
  const int P = r.NP, S = s.S, N = s.n_seg;
  const double pref = norm * exp(s.mu_species);
  const R* __restrict__ gP = reinterpret_cast<const R*>(s.gP);
  const R* __restrict__ gC = reinterpret_cast<const R*>(s.gC);
  const double* __restrict__ elam = r.elam;
  const int* __restrict__ states = s.states;
  const int* __restrict__ nst = s.nst;
  const int* __restrict__ bslot = s.bslot;
  const int* __restrict__ eslot = s.eslot;
  auto seg_pref = [&](int g, double* lp, bool* direct) {
    if (!scaled) {
      *lp = 0.0;
      *direct = false;
      return pref;
    }
    *lp = log_prefactor(s, norm, g);
    *direct = fabs(*lp) > 600.0;
    return exp(*lp);
  };
  for (int kp = threadIdx.x; kp < P / 2; kp += blockDim.x) {
    const int K = 2 * kp;
    double2 a0[BR], a1[BR], ab[ER];
#pragma unroll
    for (int q = 0; q < BR; q++) a0[q] = a1[q] = make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < ER; q++) ab[q] = make_double2(0.0, 0.0);
    // segment densities and bond end 0: steps (g, ii) in order
    auto load1 = [&](int g, int ii, AccStep& d) {
      const int si = states[g * S + ii];
      d.el = ldcg2(elam + (size_t)si * P + K);
      if (N > 1) {
        d.p0 = to_d2(ldcg2(gP + ((size_t)(g * S + ii) * S) * P + K));
        if (S > 1) d.p1 = to_d2(ldcg2(gP + ((size_t)(g * S + ii) * S + 1) * P + K));
      }
      const int nn = g < N - 1 ? nst[g + 1] : 0;
      if (nn > 0) d.c0 = to_d2(ldcg2(gC + ((size_t)(g * S + ii) * S) * P + K));
      if (nn > 1) d.c1 = to_d2(ldcg2(gC + ((size_t)(g * S + ii) * S + 1) * P + K));
    };
    {
      int g = 0, ii = 0;
      AccStep cur, nxt;
      load1(0, 0, cur);
      while (g < N) {
        int g2 = g, ii2 = ii + 1;
        if (ii2 == nst[g2]) {
          g2++;
          ii2 = 0;
        }
        if (g2 < N) load1(g2, ii2, nxt);
        // combine (g, ii)
        double lp;
        bool direct;
        const double elp = seg_pref(g, &lp, &direct);
        const int si = states[g * S + ii];
        double2 sp;
        if (N > 1) {
          sp.x = 0.0 + cur.p0.x;
          sp.y = 0.0 + cur.p0.y;
          if (S > 1) {
            sp.x += cur.p1.x;
            sp.y += cur.p1.y;
          }
        } else {
          sp.x = (s.fixed < 0 || K == s.fixed) ? 1.0 : 0.0;
          sp.y = (s.fixed < 0 || K + 1 == s.fixed) ? 1.0 : 0.0;
        }
        double2 contr;
        if (direct) {
          contr.x = exp(lp - r.lambda[(size_t)si * P + K]) * sp.x;
          contr.y = exp(lp - r.lambda[(size_t)si * P + K + 1]) * sp.y;
        } else {
          contr.x = elp * cur.el.x * sp.x;
          contr.y = elp * cur.el.y * sp.y;
        }
        const int nn = g < N - 1 ? nst[g + 1] : 0;
        double2 temp;
        if (nn) {
          temp = make_double2(0.0, 0.0);
          const int b0 = bslot[(g * S + ii) * S];
#pragma unroll
          for (int q = 0; q < BR; q++)
            if (q == b0) {
              a0[q].x += contr.x * cur.c0.x;
              a0[q].y += contr.y * cur.c0.y;
            }
          temp.x += cur.c0.x;
          temp.y += cur.c0.y;
          if (nn > 1) {
            const int b1 = bslot[(g * S + ii) * S + 1];
#pragma unroll
            for (int q = 0; q < BR; q++)
              if (q == b1) {
                a0[q].x += contr.x * cur.c1.x;
                a0[q].y += contr.y * cur.c1.y;
              }
            temp.x += cur.c1.x;
            temp.y += cur.c1.y;
          }
        } else {
          temp = make_double2(1.0, 1.0);
        }
        const double2 v = make_double2(contr.x * temp.x, contr.y * temp.y);
        stcg2(s.rho_seg + (size_t)(g * S + ii) * P + K, v);
        const int e = eslot[g * S + ii];
        if (g == 0 && s.fixed >= 0) {
#pragma unroll
          for (int q = 0; q < ER; q++)
            if (q == e) {
              if (K == s.fixed) ab[q].x += v.x / r.dz / r.trapez[(size_t)si * P + K];
              if (K + 1 == s.fixed) ab[q].y += v.y / r.dz / r.trapez[(size_t)si * P + K + 1];
            }
        } else {
#pragma unroll
          for (int q = 0; q < ER; q++)
            if (q == e) {
              ab[q].x += v.x;
              ab[q].y += v.y;
            }
        }
        cur = nxt;
        g = g2;
        ii = ii2;
      }
    }
    // bond end 1: steps (c, ii), c >= 1
    auto load2 = [&](int c, int ii, AccStep& d) {
      const int si = states[c * S + ii];
      d.el = ldcg2(elam + (size_t)si * P + K);
      if (c < N - 1) {
        d.c0 = to_d2(ldcg2(gC + ((size_t)(c * S + ii) * S) * P + K));
        if (S > 1) d.c1 = to_d2(ldcg2(gC + ((size_t)(c * S + ii) * S + 1) * P + K));
      }
      const int np_ = nst[c - 1];
      d.p0 = to_d2(ldcg2(gP + ((size_t)(c * S + ii) * S) * P + K));
      if (np_ > 1) d.p1 = to_d2(ldcg2(gP + ((size_t)(c * S + ii) * S + 1) * P + K));
    };
    if (N > 1) {
      int c = 1, ii = 0;
      AccStep cur, nxt;
      load2(1, 0, cur);
      while (c < N) {
        int c2 = c, ii2 = ii + 1;
        if (ii2 == nst[c2]) {
          c2++;
          ii2 = 0;
        }
        if (c2 < N) load2(c2, ii2, nxt);
        double lp;
        bool direct;
        const double elp = seg_pref(c, &lp, &direct);
        const int si = states[c * S + ii];
        double2 contr;
        if (direct) {
          contr.x = exp(lp - r.lambda[(size_t)si * P + K]);
          contr.y = exp(lp - r.lambda[(size_t)si * P + K + 1]);
        } else {
          contr.x = elp * cur.el.x;
          contr.y = elp * cur.el.y;
        }
        if (c < N - 1) {
          double2 t = make_double2(0.0 + cur.c0.x, 0.0 + cur.c0.y);
          if (S > 1) {
            t.x += cur.c1.x;
            t.y += cur.c1.y;
          }
          contr.x *= t.x;
          contr.y *= t.y;
        }
        const int np_ = nst[c - 1];
        const int b0 = bslot[((c - 1) * S) * S + ii];
#pragma unroll
        for (int q = 0; q < BR; q++)
          if (q == b0) {
            a1[q].x += contr.x * cur.p0.x;
            a1[q].y += contr.y * cur.p0.y;
          }
        if (np_ > 1) {
          const int b1 = bslot[((c - 1) * S + 1) * S + ii];
#pragma unroll
          for (int q = 0; q < BR; q++)
            if (q == b1) {
              a1[q].x += contr.x * cur.p1.x;
              a1[q].y += contr.y * cur.p1.y;
            }
        }
        cur = nxt;
        c = c2;
        ii = ii2;
      }
    }
#pragma unroll
    for (int q = 0; q < BR; q++)
      if (q < s.nbslot) {
        const int b = s.bslot_bond[q];
        double* r0 = r.rho_bonds + (size_t)(b * 2 + 0) * P + K;
        double* r1 = r.rho_bonds + (size_t)(b * 2 + 1) * P + K;
        const double2 o0 = ldcg2(r0), o1 = ldcg2(r1);
        stcg2(r0, make_double2(o0.x + a0[q].x, o0.y + a0[q].y));
        stcg2(r1, make_double2(o1.x + a1[q].x, o1.y + a1[q].y));
      }
#pragma unroll
    for (int q = 0; q < ER; q++)
      if (q < s.neslot) {
        double* rb = r.rho_beads + (size_t)s.eslot_bead[q] * P + K;
        const double2 o = ldcg2(rb);
        stcg2(rb, make_double2(o.x + ab[q].x, o.y + ab[q].y));
      }
  }
  __syncthreads();
}

// accumulate_pairs with its two loops merged: at step (g, ii) the segment
// density, the bond end 0 of segment g and the bond end 1 of segment g (as the
// child c = g of the second loop) read the same e^{-lambda}, gP and gC slots, so
// one pass over the (segment, state) steps serves all three, and each thread
// carries KP grid-point pairs through the steps together, the loads of the next
// step issued before the current one is combined.  Every sum runs in the order
// of accumulate_pairs (a0 and ab over (g, ii), a1 over (c, ii) with c >= 1).
template <int BR, int ER, class R, int KP>
__device__ __noinline__ void accumulate_merged(const DReq& r, const DSpecies& s, double norm, bool scaled) {
  const int P = r.NP, S = s.S, N = s.n_seg;
  const double pref = norm * exp(s.mu_species);
  const R* __restrict__ gP = reinterpret_cast<const R*>(s.gP);
  const R* __restrict__ gC = reinterpret_cast<const R*>(s.gC);
  const double* __restrict__ elam = r.elam;
  const int* __restrict__ states = s.states;
  const int* __restrict__ nst = s.nst;
  const int* __restrict__ bslot = s.bslot;
  const int* __restrict__ eslot = s.eslot;
  auto seg_pref = [&](int g, double* lp, bool* direct) {
    if (!scaled) {
      *lp = 0.0;
      *direct = false;
      return pref;
    }
    *lp = log_prefactor(s, norm, g);
    *direct = fabs(*lp) > 600.0;
    return exp(*lp);
  };
  const int bd = blockDim.x;
  for (int kp0 = threadIdx.x; kp0 < P / 2; kp0 += KP * bd) {
    int Ks[KP];
    bool on[KP];
#pragma unroll
    for (int v = 0; v < KP; v++) {
      Ks[v] = 2 * (kp0 + v * bd);
      on[v] = Ks[v] < P;
    }
    double2 a0[KP][BR], a1[KP][BR], ab[KP][ER];
#pragma unroll
    for (int v = 0; v < KP; v++) {
#pragma unroll
      for (int q = 0; q < BR; q++) a0[v][q] = a1[v][q] = make_double2(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < ER; q++) ab[v][q] = make_double2(0.0, 0.0);
    }
    auto load = [&](int g, int ii, AccStep* d) {
      const int si = states[g * S + ii];
#pragma unroll
      for (int v = 0; v < KP; v++) {
        if (!on[v]) continue;
        const int K = Ks[v];
        d[v].el = ldcg2(elam + (size_t)si * P + K);
        if (N > 1) {
          d[v].p0 = to_d2(ldcg2(gP + ((size_t)(g * S + ii) * S) * P + K));
          if (S > 1) d[v].p1 = to_d2(ldcg2(gP + ((size_t)(g * S + ii) * S + 1) * P + K));
        }
        if (g < N - 1) {
          d[v].c0 = to_d2(ldcg2(gC + ((size_t)(g * S + ii) * S) * P + K));
          if (S > 1) d[v].c1 = to_d2(ldcg2(gC + ((size_t)(g * S + ii) * S + 1) * P + K));
        }
      }
    };
    AccStep cur[KP], nxt[KP];
    int g = 0, ii = 0;
    load(0, 0, cur);
    while (g < N) {
      int g2 = g, ii2 = ii + 1;
      if (ii2 == nst[g2]) {
        g2++;
        ii2 = 0;
      }
      if (g2 < N) load(g2, ii2, nxt);
      double lp;
      bool direct;
      const double elp = seg_pref(g, &lp, &direct);
      const int si = states[g * S + ii];
      const int nn = g < N - 1 ? nst[g + 1] : 0;
      const int b0 = nn > 0 ? bslot[(g * S + ii) * S] : -1;
      const int b1 = nn > 1 ? bslot[(g * S + ii) * S + 1] : -1;
      const int e = eslot[g * S + ii];
      const int np_ = g > 0 ? nst[g - 1] : 0;
      const int c0s = g > 0 ? bslot[((g - 1) * S) * S + ii] : -1;
      const int c1s = np_ > 1 ? bslot[((g - 1) * S + 1) * S + ii] : -1;
#pragma unroll
      for (int v = 0; v < KP; v++) {
        if (!on[v]) continue;
        const int K = Ks[v];
        const AccStep& d = cur[v];
        // segment density and bond end 0 (the first loop of accumulate_pairs)
        double2 sp;
        if (N > 1) {
          sp.x = 0.0 + d.p0.x;
          sp.y = 0.0 + d.p0.y;
          if (S > 1) {
            sp.x += d.p1.x;
            sp.y += d.p1.y;
          }
        } else {
          sp.x = (s.fixed < 0 || K == s.fixed) ? 1.0 : 0.0;
          sp.y = (s.fixed < 0 || K + 1 == s.fixed) ? 1.0 : 0.0;
        }
        double2 base;  // the prefactor times e^{-lambda} at K, K+1
        if (direct) {
          base.x = exp(lp - r.lambda[(size_t)si * P + K]);
          base.y = exp(lp - r.lambda[(size_t)si * P + K + 1]);
        } else {
          base.x = elp * d.el.x;
          base.y = elp * d.el.y;
        }
        const double2 contr = direct ? make_double2(base.x * sp.x, base.y * sp.y)
                                     : make_double2(elp * d.el.x * sp.x, elp * d.el.y * sp.y);
        double2 temp;
        if (nn) {
          temp = make_double2(0.0, 0.0);
#pragma unroll
          for (int q = 0; q < BR; q++)
            if (q == b0) {
              a0[v][q].x += contr.x * d.c0.x;
              a0[v][q].y += contr.y * d.c0.y;
            }
          temp.x += d.c0.x;
          temp.y += d.c0.y;
          if (nn > 1) {
#pragma unroll
            for (int q = 0; q < BR; q++)
              if (q == b1) {
                a0[v][q].x += contr.x * d.c1.x;
                a0[v][q].y += contr.y * d.c1.y;
              }
            temp.x += d.c1.x;
            temp.y += d.c1.y;
          }
        } else {
          temp = make_double2(1.0, 1.0);
        }
        const double2 val = make_double2(contr.x * temp.x, contr.y * temp.y);
        stcg2(s.rho_seg + (size_t)(g * S + ii) * P + K, val);
        if (g == 0 && s.fixed >= 0) {
#pragma unroll
          for (int q = 0; q < ER; q++)
            if (q == e) {
              if (K == s.fixed) ab[v][q].x += val.x / r.dz / r.trapez[(size_t)si * P + K];
              if (K + 1 == s.fixed) ab[v][q].y += val.y / r.dz / r.trapez[(size_t)si * P + K + 1];
            }
        } else {
#pragma unroll
          for (int q = 0; q < ER; q++)
            if (q == e) {
              ab[v][q].x += val.x;
              ab[v][q].y += val.y;
            }
        }
        // bond end 1 of segment g as the child (the second loop of accumulate_pairs)
        if (g >= 1) {
          double2 c1v = base;
          if (g < N - 1) {
            double2 t = make_double2(0.0 + d.c0.x, 0.0 + d.c0.y);
            if (S > 1) {
              t.x += d.c1.x;
              t.y += d.c1.y;
            }
            c1v.x *= t.x;
            c1v.y *= t.y;
          }
#pragma unroll
          for (int q = 0; q < BR; q++)
            if (q == c0s) {
              a1[v][q].x += c1v.x * d.p0.x;
              a1[v][q].y += c1v.y * d.p0.y;
            }
          if (np_ > 1) {
#pragma unroll
            for (int q = 0; q < BR; q++)
              if (q == c1s) {
                a1[v][q].x += c1v.x * d.p1.x;
                a1[v][q].y += c1v.y * d.p1.y;
              }
          }
        }
      }
#pragma unroll
      for (int v = 0; v < KP; v++) cur[v] = nxt[v];
      g = g2;
      ii = ii2;
    }
#pragma unroll
    for (int v = 0; v < KP; v++) {
      if (!on[v]) continue;
      const int K = Ks[v];
#pragma unroll
      for (int q = 0; q < BR; q++)
        if (q < s.nbslot) {
          const int b = s.bslot_bond[q];
          double* r0 = r.rho_bonds + (size_t)(b * 2 + 0) * P + K;
          double* r1 = r.rho_bonds + (size_t)(b * 2 + 1) * P + K;
          const double2 o0 = ldcg2(r0), o1 = ldcg2(r1);
          stcg2(r0, make_double2(o0.x + a0[v][q].x, o0.y + a0[v][q].y));
          stcg2(r1, make_double2(o1.x + a1[v][q].x, o1.y + a1[v][q].y));
        }
#pragma unroll
      for (int q = 0; q < ER; q++)
        if (q < s.neslot) {
          double* rb = r.rho_beads + (size_t)s.eslot_bead[q] * P + K;
          const double2 o = ldcg2(rb);
          stcg2(rb, make_double2(o.x + ab[v][q].x, o.y + ab[v][q].y));
        }
    }
  }
  __syncthreads();
}

// accumulate_densities! for long grids, segment-outer: each (segment, state)
// step streams its slices over the grid on point pairs, two pairs per round
// with every load of the round issued first, and adds into rho_bonds /
// rho_beads in place.  Per grid point the sums run over the steps in the
// reference's order; two updates of one address are a whole grid sweep apart.
// Chains with at most two states per segment.
template <class R>
__device__ __noinline__ void accumulate_stream(const DReq& r, const DSpecies& s, double norm, bool scaled) {
  const int P = r.NP, S = s.S, N = s.n_seg, P2 = P / 2;
  const double pref = norm * exp(s.mu_species);
  const int bd = blockDim.x;
  for (int g = 0; g < N; g++) {
    double lp = 0.0, elp = pref;
    bool direct = false;
    if (scaled) {
      lp = log_prefactor(s, norm, g);
      direct = fabs(lp) > 600.0;
      elp = exp(lp);
    }
    const int nn = g < N - 1 ? s.nst[g + 1] : 0;
    for (int ii = 0; ii < s.nst[g]; ii++) {
      const int si = s.states[g * S + ii];
      const double* el = r.elam + (size_t)si * P;
      const R* gp = N > 1 ? reinterpret_cast<const R*>(s.gP) + (size_t)(g * S + ii) * S * P : nullptr;
      const R* gc = reinterpret_cast<const R*>(s.gC) + (size_t)(g * S + ii) * S * P;
      double* rb0 = nn > 0 ? r.rho_bonds + (size_t)(s.bnd[(g * S + ii) * S] * 2) * P : nullptr;
      double* rb1 = nn > 1 ? r.rho_bonds + (size_t)(s.bnd[(g * S + ii) * S + 1] * 2) * P : nullptr;
      double* rs = s.rho_seg + (size_t)(g * S + ii) * P;
      double* rbd = r.rho_beads + (size_t)si * P;
      const bool graft = g == 0 && s.fixed >= 0;
      for (int k0 = threadIdx.x; k0 < P2; k0 += 2 * bd) {
        AccStep d[2];
        double2 o0[2], o1[2], ob[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int K = 2 * (k0 + u * bd);
          if (K < P) {
            d[u].el = ldcg2(el + K);
            if (gp) {
              d[u].p0 = to_d2(ldcg2(gp + K));
              if (S > 1) d[u].p1 = to_d2(ldcg2(gp + P + K));
            }
            if (nn > 0) {
              d[u].c0 = to_d2(ldcg2(gc + K));
              o0[u] = ldcg2(rb0 + K);
            }
            if (nn > 1) {
              d[u].c1 = to_d2(ldcg2(gc + P + K));
              o1[u] = ldcg2(rb1 + K);
            }
            ob[u] = ldcg2(rbd + K);
          }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int K = 2 * (k0 + u * bd);
          if (K >= P) continue;
          double2 sp;
          if (gp) {
            sp.x = 0.0 + d[u].p0.x;
            sp.y = 0.0 + d[u].p0.y;
            if (S > 1) {
              sp.x += d[u].p1.x;
              sp.y += d[u].p1.y;
            }
          } else {
            sp.x = (s.fixed < 0 || K == s.fixed) ? 1.0 : 0.0;
            sp.y = (s.fixed < 0 || K + 1 == s.fixed) ? 1.0 : 0.0;
          }
          double2 contr;
          if (direct) {
            contr.x = exp(lp - r.lambda[(size_t)si * P + K]) * sp.x;
            contr.y = exp(lp - r.lambda[(size_t)si * P + K + 1]) * sp.y;
          } else {
            contr.x = elp * d[u].el.x * sp.x;
            contr.y = elp * d[u].el.y * sp.y;
          }
          double2 temp = make_double2(1.0, 1.0);
          if (nn > 0) {
            temp = make_double2(0.0 + d[u].c0.x, 0.0 + d[u].c0.y);
            stcg2(rb0 + K, make_double2(o0[u].x + contr.x * d[u].c0.x, o0[u].y + contr.y * d[u].c0.y));
          }
          if (nn > 1) {
            temp.x += d[u].c1.x;
            temp.y += d[u].c1.y;
            stcg2(rb1 + K, make_double2(o1[u].x + contr.x * d[u].c1.x, o1[u].y + contr.y * d[u].c1.y));
          }
          const double2 v = make_double2(contr.x * temp.x, contr.y * temp.y);
          stcg2(rs + K, v);
          if (graft) {
            double2 b = ob[u];
            if (K == s.fixed) b.x += v.x / r.dz / r.trapez[(size_t)si * P + K];
            if (K + 1 == s.fixed) b.y += v.y / r.dz / r.trapez[(size_t)si * P + K + 1];
            stcg2(rbd + K, b);
          } else {
            stcg2(rbd + K, make_double2(ob[u].x + v.x, ob[u].y + v.y));
          }
        }
      }
      __syncthreads();
    }
  }
  for (int c = 1; c < N; c++) {
    double lp = 0.0, elp = pref;
    bool direct = false;
    if (scaled) {
      lp = log_prefactor(s, norm, c);
      direct = fabs(lp) > 600.0;
      elp = exp(lp);
    }
    const int np_ = s.nst[c - 1];
    for (int ii = 0; ii < s.nst[c]; ii++) {
      const int si = s.states[c * S + ii];
      const double* el = r.elam + (size_t)si * P;
      const R* gc = c < N - 1 ? reinterpret_cast<const R*>(s.gC) + (size_t)(c * S + ii) * S * P : nullptr;
      const R* gp = reinterpret_cast<const R*>(s.gP) + (size_t)(c * S + ii) * S * P;
      double* rb0 = r.rho_bonds + (size_t)(s.bnd[((c - 1) * S) * S + ii] * 2 + 1) * P;
      double* rb1 = np_ > 1 ? r.rho_bonds + (size_t)(s.bnd[((c - 1) * S + 1) * S + ii] * 2 + 1) * P : nullptr;
      for (int k0 = threadIdx.x; k0 < P2; k0 += 2 * bd) {
        AccStep d[2];
        double2 o0[2], o1[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int K = 2 * (k0 + u * bd);
          if (K < P) {
            d[u].el = ldcg2(el + K);
            if (gc) {
              d[u].c0 = to_d2(ldcg2(gc + K));
              if (S > 1) d[u].c1 = to_d2(ldcg2(gc + P + K));
            }
            d[u].p0 = to_d2(ldcg2(gp + K));
            o0[u] = ldcg2(rb0 + K);
            if (np_ > 1) {
              d[u].p1 = to_d2(ldcg2(gp + P + K));
              o1[u] = ldcg2(rb1 + K);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int K = 2 * (k0 + u * bd);
          if (K >= P) continue;
          double2 contr;
          if (direct) {
            contr.x = exp(lp - r.lambda[(size_t)si * P + K]);
            contr.y = exp(lp - r.lambda[(size_t)si * P + K + 1]);
          } else {
            contr.x = elp * d[u].el.x;
            contr.y = elp * d[u].el.y;
          }
          if (gc) {
            double2 t = make_double2(0.0 + d[u].c0.x, 0.0 + d[u].c0.y);
            if (S > 1) {
              t.x += d[u].c1.x;
              t.y += d[u].c1.y;
            }
            contr.x *= t.x;
            contr.y *= t.y;
          }
          stcg2(rb0 + K, make_double2(o0[u].x + contr.x * d[u].p0.x, o0[u].y + contr.y * d[u].p0.y));
          if (np_ > 1) stcg2(rb1 + K, make_double2(o1[u].x + contr.x * d[u].p1.x, o1[u].y + contr.y * d[u].p1.y));
        }
      }
      __syncthreads();
    }
  }
  __syncthreads();
}

// true when the species went through accumulate_regs (its bead densities are added)
template <class R>
__device__ __forceinline__ bool accumulate_fast(const DReq& r, const DSpecies& s, double norm, bool scaled) {
  if (s.S <= 2 && s.n_seg > 1 && (r.NP >= 4096 || s.nbslot > 4 || s.neslot > 4)) {
    accumulate_stream<R>(r, s, norm, scaled);
    return true;
  }
  if (s.S <= 2 && s.nbslot <= 4 && s.neslot <= 2) {
    accumulate_merged<4, 2, R, 1>(r, s, norm, scaled);
    return true;
  }
  if (s.S <= 2 && s.nbslot <= 4 && s.neslot <= 4) {
    accumulate_merged<4, 4, R, 1>(r, s, norm, scaled);
    return true;
  }
  if (s.nbslot <= 4 && s.neslot <= 4) {
    accumulate_regs<4, 4, R>(r, s, norm, scaled, reinterpret_cast<const R*>(s.gP), reinterpret_cast<const R*>(s.gC), r.elam, r.lambda, s.states, s.nst, s.bslot, s.eslot, s.rho_seg,
                          r.rho_bonds, r.rho_beads);
    return true;
  }
  if (s.nbslot <= 16 && s.neslot <= 8) {
    accumulate_regs<16, 8, R>(r, s, norm, scaled, reinterpret_cast<const R*>(s.gP), reinterpret_cast<const R*>(s.gC), r.elam, r.lambda, s.states, s.nst, s.bslot, s.eslot, s.rho_seg,
                           r.rho_bonds, r.rho_beads);
    return true;
  }
  return false;
}

// eval_spatial_density! + update_spatial_structures!; false on a normalisation error
// ---------------------------------------------------------------------------
// branched chains: the level walks of child_propagators.jl:53-141 and
// parent_propagators.jl:54-122 and the tree branches of handle_fixed.jl:41-73
// and accumulate_densities.jl:95-184, for any tree whose segments have at most
// S children, in FP64 and without renormalisation (the reference's
// arithmetic).  The propagators are indexed as the reference's arrays:
// gC[g][i][c][j] (state i of g, child slot c, state j of that child) and
// gP[g][i][j] (state i of g, state j of its parent).  Two index quirks of the
// reference are kept: the other-children factor of a parent propagator reads
// gC[p][oc][idx_j] with the slots exchanged (parent_propagators.jl:150), and the
// grafted normalisation of a leaf reads gC[p][0][idx_i] (handle_fixed.jl:55); the
// host refuses the trees for which these indices leave the arrays, where the
// reference fails too.  accumulate_densities keeps the last child's sum (the
// reference assigns temp inside its loop over children).  Only segment 0 (the
// root) can be grafted in a 1D slit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ size_t tgc(const DSpecies& s, int P, int g, int i, int c, int j) {
  return ((((size_t)g * s.S + i) * s.C + c) * s.S + j) * P;
}
__device__ __forceinline__ size_t tgp(const DSpecies& s, int P, int g, int i, int j) {
  return (((size_t)g * s.S + i) * s.S + j) * P;
}
// sum over the child states of gC[g][i][c][:] at K (sum_gC_states)
__device__ __forceinline__ double tgc_sum(const DSpecies& s, int P, int K, int g, int i, int c) {
  double t = 0.0;
  for (int j = 0; j < s.S; j++) t += s.gC[tgc(s, P, g, i, c, j) + K];
  return t;
}
__device__ __forceinline__ int bond_of(const DReq& r, int a, int b) {
  const int lo = min(a, b), hi = max(a, b);
  for (int u = 0; u < r.MB; u++)
    if (r.bonds[2 * u] == lo && r.bonds[2 * u + 1] == hi) return u;
  return -1;
}
// max-path-distance mask of a grafted species: entries of segment g farther
// from the graft point than its path distance are zeroed (child_propagators.jl:147-157)
__device__ void tree_mask(const DReq& r, const DSpecies& s, double* a, int count_per_K, double md) {
  const int P = r.NP, Pt = grid_points(r);
  const double md2 = md * md;
  for (int K = threadIdx.x; K < Pt; K += blockDim.x)
    if (dist2_grid(K, s.fixed, r.dz) > md2)
      for (int q = 0; q < count_per_K; q++) a[(size_t)q * P + K] = 0.0;
}

__device__ void tree_child(const DReq& r, const DSpecies& s, Shared sh) {
  const int P = r.NP, Pt = grid_points(r), S = s.S, C = s.C, N = s.n_seg;
  const double* lng = xs_lng(r, r.x);
  const double* fin = r.fbe;
  const double* fout = r.fbe + (size_t)2 * r.MB * P;
  const double inv_norm = 1.0 / s.normative;
  const FftCtx fc = make_fft(sh.z, r);
  for (size_t q = threadIdx.x; q < (size_t)N * S * C * S * P; q += blockDim.x) s.gC[q] = 0.0;
  __syncthreads();
  for (int o = N - 1; o >= 0; o--) {
    const int p = s.order[o];
    const bool graft = p == 0 && s.fixed >= 0;
    for (int ii = 0; ii < s.nst[p]; ii++) {  // base case gC[p][i][0][0] = 1
      double* b = s.gC + tgc(s, P, p, ii, 0, 0);
      if (graft) {
        if (threadIdx.x == 0) b[s.fixed] = 1.0;
      } else {
        for (int K = threadIdx.x; K < Pt; K += blockDim.x) b[K] = 1.0;
      }
    }
    __syncthreads();
    for (int ic = 0; ic < s.nch[p]; ic++) {
      const int c = s.child[p * C + ic];
      for (int ii = 0; ii < s.nst[p]; ii++)
        for (int jj = 0; jj < s.nst[c]; jj++) {
          const int si = s.states[p * S + ii], sj = s.states[c * S + jj];
          const int bond = bond_of(r, si, sj);
          const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
          double* out = s.gC + tgc(s, P, p, ii, ic, jj);
          if (graft) {  // grafted parent, free child: local sum within sigma_ij (child_propagators.jl:91-116)
            const int Kp = s.fixed;
            const double Dij = (r.sig[si] + r.sig[sj]) / 2.0, Dij2 = Dij * Dij, renorm = 2.0 * Dij;
            const double* lng_pj = lng + (size_t)(bond * 2 + pair_j) * P;
            const double el = exp(lng[(size_t)(bond * 2 + pair_i) * P + Kp] / 2.0);
            double acc = 0.0;
            for (int K1 = threadIdx.x; K1 < Pt; K1 += blockDim.x) {
              const double d2 = dist2_grid(K1, Kp, r.dz);
              if (d2 <= Dij2) {
                double f = exp(-r.lambda[(size_t)sj * P + K1] + lng_pj[K1] / 2.0);
                for (int gc = 0; gc < s.nch[c]; gc++) f *= tgc_sum(s, P, K1, c, jj, gc);
                double t = fabs(f) * el * r.dz * r.trapez[(size_t)sj * P + K1] / renorm;
                if (fabs(d2 - Dij2) <= 1e-6) t /= 2.0;
                acc += t / s.normative;
              }
            }
            acc = block_sum(acc, sh.red);
            if (threadIdx.x == 0) out[Kp] = acc;
            __syncthreads();
          } else {  // convolution with the bond kernel (child_propagators.jl:118-141)
            const double* fj = fin + (size_t)(bond * 2 + pair_j) * P;
            const double* fo = fout + (size_t)(bond * 2 + pair_i) * P;
            dct2_convolve_b(
                fc, 1,
                [&](int, int K) {
                  double f = fj[K];
                  for (int gc = 0; gc < s.nch[c]; gc++) f *= tgc_sum(s, P, K, c, jj, gc);
                  return f;
                },
                [&](int, int k) { return __ldg(&r.Wbond[(size_t)bond * P + k]); },
                [&](int, int K, double y) { out[K] = fabs(y) * fo[K] * inv_norm; });
          }
        }
    }
    if (s.fixed >= 0) tree_mask(r, s, s.gC + tgc(s, P, p, 0, 0, 0), S * C * S, s.md[p]);
    __syncthreads();
  }
}

__device__ void tree_parent(const DReq& r, const DSpecies& s, Shared sh) {
  const int P = r.NP, Pt = grid_points(r), S = s.S, C = s.C, N = s.n_seg;
  const double* lng = xs_lng(r, r.x);
  const double* fin = r.fbe;
  const double* fout = r.fbe + (size_t)2 * r.MB * P;
  const double inv_norm = 1.0 / s.normative;
  const FftCtx fc = make_fft(sh.z, r);
  for (size_t q = threadIdx.x; q < (size_t)N * S * S * P; q += blockDim.x) s.gP[q] = 0.0;
  __syncthreads();
  for (int o = 0; o < N; o++) {
    const int c = s.order[o];
    for (int ii = 0; ii < s.nst[c]; ii++) {  // base case gP[c][i][0] = 1
      double* b = s.gP + tgp(s, P, c, ii, 0);
      if (c == 0 && s.fixed >= 0) {
        if (threadIdx.x == 0) b[s.fixed] = 1.0;
      } else {
        for (int K = threadIdx.x; K < Pt; K += blockDim.x) b[K] = 1.0;
      }
    }
    __syncthreads();
    const int p = s.parent[c];
    if (p >= 0) {
      for (int ii = 0; ii < s.nst[c]; ii++)
        for (int jj = 0; jj < s.nst[p]; jj++) {
          const int si = s.states[c * S + ii], sj = s.states[p * S + jj];
          const int bond = bond_of(r, si, sj);
          const int pair_i = si <= sj ? 0 : 1, pair_j = 1 - pair_i;
          double* out = s.gP + tgp(s, P, c, ii, jj);
          // f_parent without the trapezoid weight (parent_propagators.jl:144-153)
          auto fpar = [&](int K) {
            double sp = 0.0;
            for (int q = 0; q < S; q++) sp += s.gP[tgp(s, P, p, jj, q) + K];
            double f = sp;
            for (int oc = 0; oc < s.nch[p]; oc++)
              if (s.child[p * C + oc] != c) f *= tgc_sum(s, P, K, p, oc, jj);  // slots exchanged, as the reference
            return f;
          };
          if (p == 0 && s.fixed >= 0) {  // grafted parent: local write within sigma_ij (parent_propagators.jl:72-94)
            const int Kp = s.fixed;
            const double Dij = (r.sig[si] + r.sig[sj]) / 2.0, Dij2 = Dij * Dij, renorm = 2.0 * Dij;
            const double f = exp(-r.lambda[(size_t)sj * P + Kp] + lng[(size_t)(bond * 2 + pair_j) * P + Kp] / 2.0) *
                             fpar(Kp);
            const double* lng_pi = lng + (size_t)(bond * 2 + pair_i) * P;
            for (int K1 = threadIdx.x; K1 < Pt; K1 += blockDim.x) {
              const double d2 = dist2_grid(K1, Kp, r.dz);
              if (d2 <= Dij2) {
                double v = fabs(f) * exp(lng_pi[K1] / 2.0) / renorm * inv_norm;
                if (fabs(d2 - Dij2) <= 1e-6) v /= 2.0;
                out[K1] = v;
              }
            }
          } else {
            const double* fj = fin + (size_t)(bond * 2 + pair_j) * P;
            const double* fo = fout + (size_t)(bond * 2 + pair_i) * P;
            dct2_convolve_b(
                fc, 1, [&](int, int K) { return fj[K] * fpar(K); },
                [&](int, int k) { return __ldg(&r.Wbond[(size_t)bond * P + k]); },
                [&](int, int K, double y) { out[K] = fabs(y) * fo[K] * inv_norm; });
          }
          __syncthreads();
        }
    }
    if (s.fixed >= 0) tree_mask(r, s, s.gP + tgp(s, P, c, 0, 0), S * S, s.md[c]);
    __syncthreads();
  }
}

// handle_fixed.jl:41-73 and :105-112 for a tree
__device__ bool tree_norm(const DReq& r, DSpecies& s, Shared sh, double* norm_out) {
  const int P = r.NP, Pt = grid_points(r), S = s.S, C = s.C;
  double lam, norm;
  if (s.fixed >= 0) {
    norm = s.fixed_density;
    s.mu_species = 0.0;
    const int p = 1;  // the first free segment
    double acc = 0.0;
    for (int K = threadIdx.x; K < Pt; K += blockDim.x)
      for (int ii = 0; ii < s.nst[p]; ii++) {
        const int si = s.states[p * S + ii];
        double sp = 0.0;
        for (int q = 0; q < S; q++) sp += s.gP[tgp(s, P, p, ii, q) + K];
        const double contr = exp(-r.lambda[(size_t)si * P + K]) * sp;
        double temp;
        if (s.nch[p] == 0) {
          temp = tgc_sum(s, P, K, p, 0, ii);  // gC[K, :, idx_i, 1, parent] (handle_fixed.jl:55)
        } else {
          temp = 0.0;
          for (int ic = 0; ic < s.nch[p]; ic++) {
            const int c = s.child[p * C + ic];
            double t1 = 0.0;
            for (int jj = 0; jj < s.nst[c]; jj++) {
              double t2 = s.gC[tgc(s, P, p, ii, ic, jj) + K];
              for (int oc = 0; oc < s.nch[p]; oc++)
                if (oc != ic) t2 *= tgc_sum(s, P, K, p, ii, oc);
              t1 += t2;
            }
            temp = t1;
          }
        }
        acc += contr * temp * r.trapez[(size_t)si * P + K] * r.dz;
      }
    lam = block_sum(acc, sh.red);
  } else {
    lam = 1.0;
    norm = s.norm_free;
  }
  if (!isfinite(lam) || lam <= 0.0) return false;
  norm *= 1.0 / lam;
  s.lambda_fixed = lam / s.norm_free;
  *norm_out = norm;
  return true;
}

// accumulate_densities.jl:95-184 for a tree: segment densities and both bond ends
__device__ void tree_accumulate(const DReq& r, const DSpecies& s, double norm, bool scaled) {
  const int P = r.NP, Pt = grid_points(r), S = s.S, C = s.C, N = s.n_seg;
  const double mu = s.mu_species;
  for (int K = threadIdx.x; K < Pt; K += blockDim.x) {
    for (int g = 0; g < N; g++) {
      const double lp = scaled ? log_prefactor(s, norm, g) : 0.0;
      for (int ii = 0; ii < s.nst[g]; ii++) {
        const int si = s.states[g * S + ii];
        double sp = 0.0;
        for (int q = 0; q < S; q++) sp += s.gP[tgp(s, P, g, ii, q) + K];
        const double contr = scaled ? exp(lp - r.lambda[(size_t)si * P + K]) * sp
                                    : norm * exp(mu - r.lambda[(size_t)si * P + K]) * sp;
        double temp;
        if (s.nch[g] == 0) {
          temp = tgc_sum(s, P, K, g, ii, 0);
        } else {
          temp = 0.0;
          for (int ic = 0; ic < s.nch[g]; ic++) {
            const int c = s.child[g * C + ic];
            double t1 = 0.0;
            for (int jj = 0; jj < s.nst[c]; jj++) {
              const int bond = bond_of(r, si, s.states[c * S + jj]);
              double t2 = s.gC[tgc(s, P, g, ii, ic, jj) + K];
              for (int oc = 0; oc < s.nch[g]; oc++)
                if (oc != ic) t2 *= tgc_sum(s, P, K, g, ii, oc);
              r.rho_bonds[(size_t)(bond * 2 + 0) * P + K] += contr * t2;
              t1 += t2;
            }
            temp = t1;  // the last child's sum, as the reference
          }
        }
        s.rho_seg[(size_t)(g * S + ii) * P + K] += contr * temp;
      }
    }
    for (int c = 0; c < N; c++) {
      const int p = s.parent[c];
      if (p < 0) continue;
      const double lp = scaled ? log_prefactor(s, norm, c) : 0.0;
      for (int ii = 0; ii < s.nst[c]; ii++) {
        const int si = s.states[c * S + ii];
        double contr = scaled ? exp(lp - r.lambda[(size_t)si * P + K]) : norm * exp(mu - r.lambda[(size_t)si * P + K]);
        for (int gc = 0; gc < s.nch[c]; gc++) contr *= tgc_sum(s, P, K, c, ii, gc);
        for (int jj = 0; jj < s.nst[p]; jj++) {
          const int bond = bond_of(r, si, s.states[p * S + jj]);
          r.rho_bonds[(size_t)(bond * 2 + 1) * P + K] += contr * s.gP[tgp(s, P, c, ii, jj) + K];
        }
      }
    }
  }
  __syncthreads();
}

// one branched species: propagators, normalisation and densities (kept out of
// line so that the linear-chain path of stage_densities carries none of it)
__device__ __noinline__ bool tree_species(const DReq& r, int u, Shared sh) {
  DSpecies s = r.sp[u];
  tree_child(r, s, sh);
  tree_parent(r, s, sh);
  double norm;
  if (!tree_norm(r, s, sh, &norm)) return false;
  if (threadIdx.x == 0) {
    DSpecies* w = const_cast<DSpecies*>(&r.sp[u]);
    w->mu_species = s.mu_species;
    w->lambda_fixed = s.lambda_fixed;
  }
  // the reference's prefactor norm e^{mu - lambda} overflows beyond e^709
  const bool scaled = fabs(s.mu_species) + (double)(s.n_seg - 1) * fabs(log(s.normative)) > 600.0;
  tree_accumulate(r, s, norm, scaled);
  return true;
}

template <class R, bool TREES>
__device__ __noinline__ bool stage_densities(const DReq& r, Shared sh, int* bad_species) {
  const int P = r.NP;
  unsigned fast_mask = 0;  // species whose bead densities accumulate_regs added
  for (int u = 0; u < r.NS; u++) {
    const DSpecies& s = r.sp[u];
    for (size_t q = threadIdx.x; q < (size_t)s.n_seg * s.S * P; q += blockDim.x) s.rho_seg[q] = 0.0;
  }
  for (size_t q = threadIdx.x; q < (size_t)r.MB * 2 * P; q += blockDim.x) r.rho_bonds[q] = 0.0;
  for (size_t q = threadIdx.x; q < (size_t)r.NB * P; q += blockDim.x) r.rho_beads[q] = 0.0;
  __syncthreads();
  for (int u = 0; u < r.NS; u++) {
    DSpecies s = r.sp[u];
    bool scaled = false;
    if (TREES && s.tree) {  // branched topology: FP64 level walks
      if (!tree_species(r, u, sh)) {
        *bad_species = u;
        return false;
      }
      continue;
    }
    if (s.n_seg > 1) {
      if (grid_points(r) == P) {  // even grids: both recursions in one loop
        scaled |= s.S <= 2 ? chain_sweeps<R, 2>(r, s, sh) : chain_sweeps<R, kMaxStates>(r, s, sh);
      } else {
        scaled |= chain_child<R>(r, s, sh);
        scaled |= chain_parent<R>(r, s, sh);
      }
    }
    // the even-grid fused sweep stores the propagators in the precision of the
    // step (FP32 in a mixed evaluation); the odd-grid recursions in FP64
    const bool f32 = sizeof(R) == 4 && s.n_seg > 1 && grid_points(r) == P;
    double norm;
    bool ok = f32 ? chain_norm<float>(r, s, sh, &norm) : chain_norm<double>(r, s, sh, &norm);
    if (!ok) {
      *bad_species = u;
      return false;
    }
    if (threadIdx.x == 0) {
      DSpecies* w = const_cast<DSpecies*>(&r.sp[u]);
      w->mu_species = s.mu_species;
      w->lambda_fixed = s.lambda_fixed;
    }
    // the reference's prefactor norm e^{mu - lambda} overflows beyond e^709
    if (fabs(s.mu_species) + (double)(s.n_seg - 1) * fabs(log(s.normative)) > 600.0) scaled = true;
    if (f32 ? accumulate_fast<float>(r, s, norm, scaled) : accumulate_fast<double>(r, s, norm, scaled))
      fast_mask |= 1u << u;
    else if (f32)
      chain_accumulate<float>(r, s, norm, scaled);
    else
      chain_accumulate<double>(r, s, norm, scaled);
  }
  // update_spatial_structures! for the species accumulated without register slots
  if (fast_mask != (1u << r.NS) - 1u) {
    for (int K = threadIdx.x; K < P; K += blockDim.x) {
      for (int u = 0; u < r.NS; u++) {
        if (fast_mask & (1u << u)) continue;
        const DSpecies& s = r.sp[u];
        for (int g = 0; g < s.n_seg; g++)
          for (int ii = 0; ii < s.nst[g]; ii++) {
            const int st = s.states[g * s.S + ii];
            const double v = s.rho_seg[(size_t)(g * s.S + ii) * P + K];
            if (g == 0 && s.fixed >= 0) {
              if (K == s.fixed) r.rho_beads[(size_t)st * P + K] += v / r.dz / r.trapez[(size_t)st * P + K];
            } else {
              r.rho_beads[(size_t)st * P + K] += v;
            }
          }
      }
    }
  }
  __syncthreads();
  return true;
}

// ---------------------------------------------------------------------------
// rho_hat (DCT-II of rho * trapez)
// ---------------------------------------------------------------------------
__device__ void stage_rho_hat(const DReq& r, Shared sh) {
  const int P = r.NP;
  const FftCtx fc = make_fft(sh.z, r);
  const int ntot = r.NB + 2 * r.MB;
  // transform q: bead densities (q < NB) or bond-end densities, times the trapezoid weight of their bead
  auto rho_of = [&](int q) { return q < r.NB ? r.rho_beads + (size_t)q * P : r.rho_bonds + (size_t)(q - r.NB) * P; };
  auto tr_of = [&](int q) { return r.trapez + (size_t)(q < r.NB ? q : r.bonds[q - r.NB]) * P; };
  for (int g0 = 0; g0 < ntot; g0 += r.TB) {
    const int nT = min(r.TB, ntot - g0);
    dct2_forward_kp(
        fc, nT,
        [&](int kp, auto put) {
          const int K = 2 * kp;
          double2 a[kMaxTB], b[kMaxTB];
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) {
              a[u] = ldcg2(rho_of(g0 + u) + K);
              b[u] = ldcg2(tr_of(g0 + u) + K);
            }
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) put(u, make_double2(a[u].x * b[u].x, a[u].y * b[u].y));
        },
        [&](int t, int q, double v) {
          const int w = g0 + t;
          (w < r.NB ? r.Cb + (size_t)w * P : r.Cbond + (size_t)(w - r.NB) * P)[q] = v;
        });
  }
}

// ---------------------------------------------------------------------------
// White-Bear FMT (+TPT1): point-wise derivative of iLST mfmt.jl:210-244 and
// TPT1mfmt.jl:311-374 on the true grid
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mfmt_deriv_pt(double n0, double n1, double n2, double n3, double nV1, double nV2,
                                              double* d) {
  const double om = 1.0 - n3;
  const double l1 = log(om);
  const double i1 = 1.0 / om;
  const double i3 = 1.0 / n3;
  const double i36 = 1.0 / (36.0 * kPi);
  const double dot12 = nV1 * nV2, dot22 = nV2 * nV2;
  d[0] = -l1;
  d[1] = n2 * i1;
  d[2] = n1 * i1 + (n2 * n2 - dot22) * 3.0 * i36 * i3 * (l1 * i3 + i1 * i1);
  d[3] = n0 * i1 + (n1 * n2 - dot12) * (i1 * i1) -
         (l1 * (i3 * i3 * i3) * 2.0 * i36 + (i3 * i3) * i1 * i36 + (1.0 - 3.0 * n3) * (i3 * i3) * i36 * (i1 * i1 * i1)) *
             (n2 * n2 * n2 - 3.0 * n2 * dot22);
  d[4] = -nV2 * i1;
  d[5] = -nV1 * i1 - (l1 * i3 + i1 * i1) * n2 * nV2 * i3 * 6.0 * i36;
}

// scalar weighted densities n0..n3, nV1, nV2 into wa[0..6P); bond weighted
// densities into wb.  |.| is taken per bead type before the bead sum, as in
// TPT1mfmt.jl:79-89, so each bead's two transforms go to their own scratch
// arrays (wd) and are summed afterwards in bead order.
__device__ void fmt_weighted(const DReq& r, Shared sh, bool tpt1) {
  const int P = r.NP, NB = r.NB, MB = r.MB;
  const FftCtx fc = make_fft(sh.z, r);
  double* n0 = r.wa;
  double* n1 = r.wa + (size_t)1 * P;
  double* n2 = r.wa + (size_t)2 * P;
  double* n3 = r.wa + (size_t)3 * P;
  double* nV1 = r.wa + (size_t)4 * P;
  double* nV2 = r.wa + (size_t)5 * P;
  const int ns = 2 * NB;  // (bead j, weight m) -> wd[(2j+m) P]
  for (int g0 = 0; g0 < ns; g0 += r.TB) {
    const int nT = min(r.TB, ns - g0);
    dct2_inverse_kp(
        fc, nT,
        [&](int t, int q) {
          const int jm = g0 + t, j = jm >> 1, m = jm & 1;
          return r.Cb[(size_t)j * P + q] * r.Wfmt[((size_t)j * 3 + m) * P + q];
        },
        [&](int kp, auto get) {
          const int K = 2 * kp;
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) {
              const double2 y = get(u);
              stcg2(r.wd + (size_t)(g0 + u) * P + K, make_double2(fabs(y.x), fabs(y.y)));
            }
        });
  }
  for (int K = threadIdx.x; K < P; K += blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    for (int j = 0; j < NB; j++) {
      const double s = r.sig[j];
      const double a = r.wd[(size_t)(2 * j) * P + K];
      a0 += a / (kPi * (s * s));
      a1 += a / (2 * kPi * s);
      a2 += a;
      a3 += r.wd[(size_t)(2 * j + 1) * P + K];
    }
    n0[K] = a0;
    n1[K] = a1;
    n2[K] = a2;
    n3[K] = a3;
  }
  // vector weighted densities: odd output of the odd weight; the bead sum is linear
  for (int g0 = 0; g0 < 2; g0 += r.TB) {
    const int nT = min(r.TB, 2 - g0);
    dct2_inverse_kp(
        fc, nT,
        [&](int t, int q) {
          if (q == 0) return 0.0;
          const int k = grid_points(r) - q;  // coefficient reversal over the grid points (not the stride)
          double s = 0.0;
          for (int j = 0; j < NB; j++) {
            double c = r.Cb[(size_t)j * P + k] * r.Wfmt[((size_t)j * 3 + 2) * P + k];
            s += g0 + t == 0 ? c / (2 * kPi * r.sig[j]) : c;
          }
          return s;
        },
        [&](int kp, auto get) {
          const int K = 2 * kp;  // (K even, K + 1 odd): the odd output takes (-y_K, y_K+1)
#pragma unroll
          for (int u = 0; u < 2; u++)
            if (u < nT) {
              const double2 y = get(u);
              stcg2((g0 + u == 0 ? nV1 : nV2) + K, make_double2(-y.x, y.y));
            }
        });
  }
  // bond weighted densities (TPT1mfmt.jl:106-133)
  if (tpt1) {
    const int nb2 = 2 * MB;
    for (int g0 = 0; g0 < nb2; g0 += r.TB) {
      const int nT = min(r.TB, nb2 - g0);
      dct2_inverse_kp(
          fc, nT,
          [&](int t, int q) {
            const int be = g0 + t, i = r.bonds[be];
            return r.Cbond[(size_t)be * P + q] * r.Wfmt[((size_t)i * 3 + 0) * P + q] / (r.sig[i] * r.sig[i]) / kPi;
          },
          [&](int kp, auto get) {
            const int K = 2 * kp;
#pragma unroll
            for (int u = 0; u < kMaxTB; u++)
              if (u < nT) {
                const double2 y = get(u);
                stcg2(r.wb + (size_t)(g0 + u) * P + K, make_double2(fabs(y.x), fabs(y.y)));
              }
          });
    }
  }
}

__device__ void stage_fmt(const DReq& r, Shared sh, bool tpt1) {
  const int P = r.NP, NB = r.NB, MB = r.MB;
  const FftCtx fc = make_fft(sh.z, r);
  double* n0 = r.wa;
  double* n1 = r.wa + (size_t)1 * P;
  double* n2 = r.wa + (size_t)2 * P;
  double* n3 = r.wa + (size_t)3 * P;
  double* nV1 = r.wa + (size_t)4 * P;
  double* nV2 = r.wa + (size_t)5 * P;
  fmt_weighted(r, sh, tpt1);
  __syncthreads();
  // point-wise derivative; fields D0..D5 and ln y_HS per bond
  double* D = r.wc;
  double* lny = r.wc + (size_t)6 * P;
  for (int K = threadIdx.x; K < P; K += blockDim.x) {
    double a0 = n0[K], a1 = n1[K], a2 = n2[K], a3 = n3[K], v1 = nV1[K], v2 = nV2[K];
    if (a3 > 0.95) {
      const double fac = 0.95 / a3;
      a0 *= fac; a1 *= fac; a2 *= fac; a3 *= fac; v1 *= fac; v2 *= fac;
    }
    double d[6];
    if (a3 > 1e-10) {
      mfmt_deriv_pt(a0, a1, a2, a3, v1, v2, d);
      if (tpt1) {
        double Xi = 1.0 - (v2 * v2) / (a2 * a2);
        if (Xi < 0.0) Xi = 0.0;
        const double i1 = 1.0 / (1.0 - a3);
        const double term2 = a2 * Xi / 4.0 * (i1 * i1);
        const double term3 = (a2 * a2) * Xi / 72.0 * (i1 * i1 * i1);
        for (int u = 0; u < MB; u++) {
          const int bi = r.bonds[2 * u], bj = r.bonds[2 * u + 1];
          const double sij = (r.sig[bi] + r.sig[bj]) / 2;
          const double tau = r.sig[bi] * r.sig[bj] / sij;
          const double y = i1 + term2 * tau + term3 * (tau * tau);
          const double dl2 = (tau / 4.0 * (i1 * i1) + a2 * (tau * tau) * (i1 * i1 * i1) / 36.0) / y;
          const double dl3 =
              ((i1 * i1) + a2 * Xi / 2.0 * (i1 * i1 * i1) * tau + (a2 * a2) * Xi / 24.0 * ((i1 * i1) * (i1 * i1)) * (tau * tau)) / y;
          const double rb = r.wb[(size_t)(u * 2) * P + K] + r.wb[(size_t)(u * 2 + 1) * P + K];
          d[2] -= 0.5 * rb * dl2;
          d[3] -= 0.5 * rb * dl3;
          const double dlv = -v2 * (tau / (2.0 * a2) * (i1 * i1) + (tau * tau) / 36.0 * (i1 * i1 * i1)) / y;
          d[5] -= 0.5 * rb * dlv;
          lny[(size_t)u * P + K] = log(y);
        }
      }
    } else {
      for (int q = 0; q < 6; q++) d[q] = 0.0;
      if (tpt1)
        for (int u = 0; u < MB; u++) lny[(size_t)u * P + K] = 0.0;
    }
    for (int q = 0; q < 6; q++) D[(size_t)q * P + K] = d[q];
  }
  __syncthreads();
  // forward transforms: even D0..D3, odd D4, D5 (DST-II through (-1)^K and reversal)
  double* CD = r.wa;  // 6 coefficient arrays (weighted densities are dead now)
  if (threadIdx.x == 0) {
    CD[(size_t)4 * P] = 0.0;
    CD[(size_t)5 * P] = 0.0;
  }
  for (int g0 = 0; g0 < 6; g0 += r.TB) {
    const int nT = min(r.TB, 6 - g0);
    dct2_forward_kp(
        fc, nT,
        [&](int kp, auto put) {
          const int K = 2 * kp;
          double2 v[kMaxTB];
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) v[u] = ldcg2(D + (size_t)(g0 + u) * P + K);
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) put(u, g0 + u >= 4 ? make_double2(v[u].x, -v[u].y) : v[u]);  // odd weights: (-1)^K
        },
        [&](int t, int k, double v) {
          const int q = g0 + t;
          if (q < 4) CD[(size_t)q * P + k] = v;
          else if (k > 0) CD[(size_t)q * P + (grid_points(r) - k)] = v;
        });
  }
  // mu_ex coefficients (accumulate_mu_ex!, TPT1mfmt.jl:244-283)
  for (int idx = threadIdx.x; idx < NB * P; idx += blockDim.x) {
    const int j = idx / P, k = idx - j * P;
    const double s = r.sig[j];
    const double W1 = r.Wfmt[((size_t)j * 3 + 0) * P + k];
    const double W2 = r.Wfmt[((size_t)j * 3 + 1) * P + k];
    const double W3 = r.Wfmt[((size_t)j * 3 + 2) * P + k];
    const double c1 = CD[k] / (kPi * (s * s)) + CD[(size_t)P + k] / (2 * kPi * s) + CD[(size_t)2 * P + k];
    const double c2 = CD[(size_t)3 * P + k];
    const double c3 = CD[(size_t)4 * P + k] / (2 * kPi * s) + CD[(size_t)5 * P + k];
    r.Cmu[idx] += c1 * W1 + c2 * W2 - c3 * W3;
  }
  __syncthreads();
  // ln g coefficients (accumulate_lng!, TPT1mfmt.jl:286-313)
  if (tpt1) {
    for (int g0 = 0; g0 < MB; g0 += r.TB) {
      const int nT = min(r.TB, MB - g0);
      dct2_forward_kp(
          fc, nT,
          [&](int kp, auto put) {
            const int K = 2 * kp;
            double2 v[kMaxTB];
#pragma unroll
            for (int u = 0; u < kMaxTB; u++)
              if (u < nT) v[u] = ldcg2(lny + (size_t)(g0 + u) * P + K);
#pragma unroll
            for (int u = 0; u < kMaxTB; u++)
              if (u < nT) put(u, v[u]);
          },
          [&](int t, int k, double c) {
            const int u = g0 + t;
            const int ia = r.bonds[2 * u], ib = r.bonds[2 * u + 1];
            r.Clng[(size_t)(u * 2) * P + k] += c * (r.Wfmt[((size_t)ia * 3) * P + k] / (kPi * (r.sig[ia] * r.sig[ia])));
            r.Clng[(size_t)(u * 2 + 1) * P + k] += c * (r.Wfmt[((size_t)ib * 3) * P + k] / (kPi * (r.sig[ib] * r.sig[ib])));
          });
    }
  }
}

// ---------------------------------------------------------------------------
// MSA (+TPT1): Gamma by the damped fixed point of iLST msa.jl:181-230
// ---------------------------------------------------------------------------
struct MsaGamma {
  double G, eta, H;
};

__device__ __forceinline__ MsaGamma gamma_msa_pt(const double* rho, const double* sig, const double* Z, int nb,
                                                 double lB) {
  const double tol = 1e-10;
  double s = 0.0;
  for (int j = 0; j < nb; j++) s += rho[j] * Z[j] * Z[j];
  const double kappa = sqrt(4.0 * kPi * lB * s);
  MsaGamma out;
  if (kappa < tol) {
    out.G = kappa / 2.0;
    out.eta = 0.0;
    out.H = 2.0 / kPi;
    return out;
  }
  double sr = 0.0, srs = 0.0, s3 = 0.0;
  for (int j = 0; j < nb; j++) {
    sr += rho[j] * sig[j];
    srs += rho[j];
    s3 += rho[j] * sig[j] * sig[j] * sig[j];
  }
  const double sig_eff = sr / srs;
  const double xx = sig_eff * sqrt(4.0 * kPi * lB * s);
  double G = (sqrt(1.0 + 2.0 * xx) - 1.0) / (2.0 * sig_eff);
  const double term2 = 2.0 / kPi * (1.0 - kPi / 6.0 * s3);
  double eta = 0.0, H = 0.0;
  for (int it = 1;; it++) {
    double hs = 0.0, es = 0.0;
    for (int j = 0; j < nb; j++) {
      hs += rho[j] * sig[j] * sig[j] * sig[j] / (1.0 + G * sig[j]);
      es += rho[j] * Z[j] * sig[j] / (1.0 + G * sig[j]);
    }
    H = hs + term2;
    eta = es / H;
    double gs = 0.0;
    for (int j = 0; j < nb; j++) {
      const double a = Z[j] - eta * sig[j] * sig[j];
      gs += rho[j] * a * a / (1.0 + G * sig[j]) / (1.0 + G * sig[j]);
    }
    const double G1 = sqrt(kPi * lB * gs);
    const double Gn = 0.9 * G + 0.1 * G1;
    if (fabs(G1 - G) < tol || it >= 1000) {
      G = Gn;
      break;
    }
    G = Gn;
  }
  out.G = G;
  out.eta = eta;
  out.H = H;
  return out;
}

// The same damped iteration with the bead sums taken per diameter group: with
// c_g = sum rho_j, b_g = sum rho_j z_j, a_g = sum rho_j z_j^2 over the beads of
// diameter s_g,
//   sum_j rho_j s_j^3 / (1 + G s_j)          = sum_g c_g s_g^3 / (1 + G s_g)
//   sum_j rho_j z_j s_j / (1 + G s_j)        = sum_g b_g s_g / (1 + G s_g)
//   sum_j rho_j (z_j - eta s_j^2)^2 / (1 + G s_j)^2
//                        = sum_g (a_g - 2 eta s_g^2 b_g + eta^2 s_g^4 c_g) / (1 + G s_g)^2,
// so an iteration costs O(groups) instead of O(beads) (equal up to rounding).
constexpr int kMaxGroups = 4;

__device__ __forceinline__ MsaGamma gamma_msa_grouped(const DReq& r, const double* rho) {
  const int nb = r.NB;
  const double lB = r.lB;
  const double tol = 1e-10;
  double s = 0.0, sr = 0.0, srs = 0.0, s3 = 0.0;
  double cg[kMaxGroups], bg[kMaxGroups], ag[kMaxGroups], sg[kMaxGroups];
#pragma unroll
  for (int q = 0; q < kMaxGroups; q++) {
    cg[q] = bg[q] = ag[q] = 0.0;
    sg[q] = q < r.ngrp ? r.grp_sig[q] : 0.0;
  }
  for (int j = 0; j < nb; j++) {
    const double rj = rho[j], zj = r.z[j], sj = r.sig[j];
    const int gj = r.grp[j];
    s += rj * zj * zj;
    sr += rj * sj;
    srs += rj;
    s3 += rj * sj * sj * sj;
#pragma unroll
    for (int q = 0; q < kMaxGroups; q++)
      if (q == gj) {
        cg[q] += rj;
        bg[q] += rj * zj;
        ag[q] += rj * zj * zj;
      }
  }
  const double kappa = sqrt(4.0 * kPi * lB * s);
  MsaGamma out;
  if (kappa < tol) {
    out.G = kappa / 2.0;
    out.eta = 0.0;
    out.H = 2.0 / kPi;
    return out;
  }
  const double sig_eff = sr / srs;
  const double xx = sig_eff * sqrt(4.0 * kPi * lB * s);
  double G = (sqrt(1.0 + 2.0 * xx) - 1.0) / (2.0 * sig_eff);
  const double term2 = 2.0 / kPi * (1.0 - kPi / 6.0 * s3);
  double eta = 0.0, H = 0.0;
  for (int it = 1;; it++) {
    double hs = 0.0, es = 0.0, inv[kMaxGroups];
#pragma unroll
    for (int q = 0; q < kMaxGroups; q++)
      if (q < r.ngrp) {
        inv[q] = 1.0 / (1.0 + G * sg[q]);
        hs += cg[q] * sg[q] * sg[q] * sg[q] * inv[q];
        es += bg[q] * sg[q] * inv[q];
      }
    H = hs + term2;
    eta = es / H;
    double gs = 0.0;
#pragma unroll
    for (int q = 0; q < kMaxGroups; q++)
      if (q < r.ngrp) {
        const double s2 = sg[q] * sg[q];
        gs += (ag[q] - 2.0 * eta * s2 * bg[q] + eta * eta * s2 * s2 * cg[q]) * (inv[q] * inv[q]);
      }
    const double G1 = sqrt(kPi * lB * gs);
    const double Gn = 0.9 * G + 0.1 * G1;
    if (fabs(G1 - G) < tol || it >= 1000) {
      G = Gn;
      break;
    }
    G = Gn;
  }
  out.G = G;
  out.eta = eta;
  out.H = H;
  return out;
}

// Gamma at one point: grouped when the diameters fall into few groups
__device__ __forceinline__ MsaGamma gamma_msa_point(const DReq& r, const double* rho) {
  if (r.ngrp <= kMaxGroups) return gamma_msa_grouped(r, rho);
  return gamma_msa_pt(rho, r.sig, r.z, r.NB, r.lB);
}

__device__ void msa_weighted(const DReq& r, Shared sh, bool tpt1) {
  const int P = r.NP, NB = r.NB, MB = r.MB;
  const FftCtx fc = make_fft(sh.z, r);
  const int ntot = NB + (tpt1 ? 2 * MB : 0);
  for (int g0 = 0; g0 < ntot; g0 += r.TB) {
    const int nT = min(r.TB, ntot - g0);
    dct2_inverse_kp(
        fc, nT,
        [&](int t, int q) {
          const int w = g0 + t;
          if (w < NB) return r.Cb[(size_t)w * P + q] * r.Wmsa[(size_t)w * P + q];
          const int be = w - NB;
          return r.Cbond[(size_t)be * P + q] * r.Wmsa[(size_t)r.bonds[be] * P + q];
        },
        [&](int kp, auto get) {
          const int K = 2 * kp;
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) {
              const int w = g0 + u;
              const double2 y = get(u);
              stcg2((w < NB ? r.wa + (size_t)w * P : r.wb + (size_t)(w - NB) * P) + K, make_double2(fabs(y.x), fabs(y.y)));
            }
        });
  }
}

// Gamma, eta, H of every grid point into out[0..3P) from the MSA weighted
// densities wa.  With a single diameter group (all beads of one size) each
// thread iterates four points in lock-step, so that their dependent
// divide/square-root chains overlap; the per-point arithmetic is exactly that
// of gamma_msa_grouped, and a point's value is frozen once its own stopping
// test fires.
constexpr int kGammaLanes = 4;

__device__ __noinline__ void msa_gamma_pass(const DReq& r, double* out) {
  const int P = r.NP, Pt = grid_points(r), nb = r.NB;  // stride, grid points
  if (r.ngrp != 1) {
    for (int K = threadIdx.x; K < Pt; K += blockDim.x) {
      double rho[kMaxBeads];
      for (int j = 0; j < nb; j++) rho[j] = r.wa[(size_t)j * P + K];
      const MsaGamma gm = gamma_msa_point(r, rho);
      out[K] = gm.G;
      out[(size_t)P + K] = gm.eta;
      out[(size_t)2 * P + K] = gm.H;
    }
    __syncthreads();
    return;
  }
  const double lB = r.lB, tol = 1e-10, sg = r.grp_sig[0];
  const int bd = blockDim.x;
  for (int K0 = threadIdx.x; K0 < Pt; K0 += kGammaLanes * bd) {
    double G[kGammaLanes], eta[kGammaLanes], H[kGammaLanes], cg[kGammaLanes], bg[kGammaLanes], ag[kGammaLanes],
        term2[kGammaLanes];
    bool live[kGammaLanes];
#pragma unroll
    for (int u = 0; u < kGammaLanes; u++) {
      const int K = K0 + u * bd;
      live[u] = false;
      G[u] = eta[u] = H[u] = 0.0;
      cg[u] = bg[u] = ag[u] = term2[u] = 0.0;
      if (K >= Pt) continue;
      double s = 0.0, sr = 0.0, srs = 0.0, s3 = 0.0;
      for (int j = 0; j < nb; j++) {
        const double rj = r.wa[(size_t)j * P + K], zj = r.z[j], sj = r.sig[j];
        s += rj * zj * zj;
        sr += rj * sj;
        srs += rj;
        s3 += rj * sj * sj * sj;
        cg[u] += rj;
        bg[u] += rj * zj;
        ag[u] += rj * zj * zj;
      }
      const double kappa = sqrt(4.0 * kPi * lB * s);
      if (kappa < tol) {
        G[u] = kappa / 2.0;
        eta[u] = 0.0;
        H[u] = 2.0 / kPi;
        continue;
      }
      const double sig_eff = sr / srs;
      const double xx = sig_eff * sqrt(4.0 * kPi * lB * s);
      G[u] = (sqrt(1.0 + 2.0 * xx) - 1.0) / (2.0 * sig_eff);
      term2[u] = 2.0 / kPi * (1.0 - kPi / 6.0 * s3);
      live[u] = true;
    }
    for (int it = 1;; it++) {
      bool any = false;
#pragma unroll
      for (int u = 0; u < kGammaLanes; u++) {
        if (!live[u]) continue;
        const double inv = 1.0 / (1.0 + G[u] * sg);
        const double hs = 0.0 + cg[u] * sg * sg * sg * inv;
        const double es = 0.0 + bg[u] * sg * inv;
        H[u] = hs + term2[u];
        eta[u] = es / H[u];
        const double s2 = sg * sg;
        const double gs = 0.0 + (ag[u] - 2.0 * eta[u] * s2 * bg[u] + eta[u] * eta[u] * s2 * s2 * cg[u]) * (inv * inv);
        const double G1 = sqrt(kPi * lB * gs);
        const double Gn = 0.9 * G[u] + 0.1 * G1;
        if (fabs(G1 - G[u]) < tol || it >= 1000) live[u] = false;
        G[u] = Gn;
        any |= live[u];
      }
      if (!any) break;
    }
#pragma unroll
    for (int u = 0; u < kGammaLanes; u++) {
      const int K = K0 + u * bd;
      if (K < Pt) {
        out[K] = G[u];
        out[(size_t)P + K] = eta[u];
        out[(size_t)2 * P + K] = H[u];
      }
    }
  }
  __syncthreads();
}

__device__ void stage_msa(const DReq& r, Shared sh, bool tpt1) {
  const int P = r.NP, NB = r.NB, MB = r.MB;
  const FftCtx fc = make_fft(sh.z, r);
  msa_weighted(r, sh, tpt1);
  __syncthreads();
  msa_gamma_pass(r, r.wd);  // wd is free between the FMT stage and the next evaluation
  // point-wise derivative (TPT1msa.jl:129-156 -> iLST TPT1msa.jl:200-282).  The
  // per-bead denominators 1 + G sigma_j, their reciprocals and the per-bond
  // sums of the bond weighted densities are formed once per point; every use
  // below is the same expression as before, so the values are unchanged.
  const double* sig = r.sig;
  const double* Z = r.z;
  const double lB = r.lB;
  for (int K = threadIdx.x; K < P; K += blockDim.x) {
    double rho[kMaxBeads], dphi[kMaxBeads], og[kMaxBeads], inv[kMaxBeads];
    for (int j = 0; j < NB; j++) rho[j] = r.wa[(size_t)j * P + K];
    const double G = r.wd[K], eta = r.wd[(size_t)P + K], H = r.wd[(size_t)2 * P + K];
    for (int j = 0; j < NB; j++) {
      og[j] = 1.0 + G * sig[j];
      inv[j] = 1.0 / og[j];
    }
    double us = 0.0;
    for (int j = 0; j < NB; j++) us += rho[j] * sig[j] * sig[j] * ((Z[j] - eta * sig[j] * sig[j]) / og[j] + Z[j]);
    us = -kPi / 6 * us;
    for (int j = 0; j < NB; j++)
      dphi[j] = -lB * (G * (Z[j] * Z[j]) / og[j] +
                       eta * sig[j] * ((2.0 * Z[j] - eta * (sig[j] * sig[j])) / og[j] + eta * (sig[j] * sig[j]) / 3.0) +
                       Z[j] * us);
    if (tpt1) {
      double* lngo = r.wc + (size_t)NB * P;
      if (G == 0.0) {
        for (int u = 0; u < MB; u++) {
          const int i = r.bonds[2 * u], j = r.bonds[2 * u + 1];
          lngo[(size_t)u * P + K] = -lB / ((sig[i] + sig[j]) / 2.0) * Z[i] * Z[j];
        }
      } else {
        for (int u = 0; u < MB; u++) {
          const int i = r.bonds[2 * u], j = r.bonds[2 * u + 1];
          const double sij = (sig[i] + sig[j]) / 2.0;
          const double Xi = (Z[i] - eta * (sig[i] * sig[i])) / og[i];
          const double Xj = (Z[j] - eta * (sig[j] * sig[j])) / og[j];
          lngo[(size_t)u * P + K] = -lB / sij * Xi * Xj;
        }
        double dfG = 0.0, dfe = 0.0, deG = 0.0, dHG = 0.0;
        for (int w = 0; w < NB; w++) {
          const double a = Z[w] - eta * sig[w] * sig[w];
          dfG += rho[w] * sig[w] * a * a / og[w] / og[w] / og[w];
          dfe += rho[w] * sig[w] * sig[w] * a / og[w] / og[w];
          deG += rho[w] * Z[w] * sig[w] * sig[w] / og[w] / og[w];
          dHG += rho[w] * sig[w] * sig[w] * sig[w] * sig[w] / og[w] / og[w];
        }
        dfG = -2.0 * kPi * lB * dfG;
        dfe = -2.0 * kPi * lB * dfe;
        deG = -1.0 / H * deG;
        const double deH = -eta / H;
        dHG = -dHG;
        const double detaG = deG + deH * dHG;
        const double denom = 1.0 / (2.0 * G - dfe * detaG - dfG);
        double rbu[kMaxBonds];
        for (int u = 0; u < MB; u++) rbu[u] = r.wb[(size_t)(u * 2) * P + K] + r.wb[(size_t)(u * 2 + 1) * P + K];
        for (int w = 0; w < NB; w++) {
          const double Xw = (Z[w] - eta * (sig[w] * sig[w])) * inv[w];
          const double dfr = kPi * lB * (Xw * Xw);
          const double der = sig[w] / H * Z[w] * inv[w];
          const double dHr = (sig[w] * sig[w] * sig[w]) * (inv[w] - 1.0 / 3.0);
          const double dGr = (dfr + dfe * (der + dfe * deH * dHr)) * denom;
          const double detar = detaG * dGr;
          for (int u = 0; u < MB; u++) {
            const int i = r.bonds[2 * u], j = r.bonds[2 * u + 1];
            const double sij = (sig[i] + sig[j]) / 2.0;
            const double ii = inv[i];
            const double Xi = (Z[i] - eta * (sig[i] * sig[i])) * ii;
            const double dXi = -((sig[i] * sig[i]) * ii * detar + sig[i] * Xi * ii * dGr);
            const double ij = inv[j];
            const double Xj = (Z[j] - eta * (sig[j] * sig[j])) * ij;
            const double dXj = -((sig[j] * sig[j]) * ij * detar + sig[j] * Xj * ij * dGr);
            dphi[w] += rbu[u] / 2.0 * lB / sij * (dXi * Xj + Xi * dXj);
          }
        }
      }
    }
    for (int j = 0; j < NB; j++) r.wc[(size_t)j * P + K] = dphi[j];
  }
  __syncthreads();
  const int nf = NB + (tpt1 ? MB : 0);
  for (int g0 = 0; g0 < nf; g0 += r.TB) {
    const int nT = min(r.TB, nf - g0);
    dct2_forward_kp(
        fc, nT,
        [&](int kp, auto put) {
          const int K = 2 * kp;
          double2 v[kMaxTB];
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) v[u] = ldcg2(r.wc + (size_t)(g0 + u) * P + K);
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) put(u, v[u]);
        },
        [&](int t, int k, double c) {
          const int w = g0 + t;
          if (w < NB) {
            r.Cmu[(size_t)w * P + k] += c * r.Wmsa[(size_t)w * P + k];
          } else {
            const int u = w - NB;
            r.Clng[(size_t)(u * 2) * P + k] += c * r.Wmsa[(size_t)r.bonds[2 * u] * P + k];
            r.Clng[(size_t)(u * 2 + 1) * P + k] += c * r.Wmsa[(size_t)r.bonds[2 * u + 1] * P + k];
          }
        });
  }
}

// ---------------------------------------------------------------------------
// neutrality shift (neutrality_shift.jl:1-99) -> PsiC increment
// ---------------------------------------------------------------------------
__device__ double stage_neutrality(const DReq& r, Shared sh) {
  const int P = r.NP, NS = r.NS;
  // per species: N_u and sum_seg N z (partial sums per thread, one vector reduction)
  double part[2 * 16];
  for (int u = 0; u < 2 * NS; u++) part[u] = 0.0;
  for (int u = 0; u < NS; u++) {
    const DSpecies& s = r.sp[u];
    for (int g = 0; g < s.n_seg; g++)
      for (int ii = 0; ii < s.nst[g]; ii++) {
        const int st = s.states[g * s.S + ii];
        const double* rs = s.rho_seg + (size_t)(g * s.S + ii) * P;
        double nn = 0.0;
        if (g == 0 && s.fixed >= 0) {
          if (threadIdx.x == 0) nn = rs[s.fixed];
        } else {
          for (int K = threadIdx.x; K < grid_points(r); K += blockDim.x) nn += rs[K] * r.trapez[(size_t)st * P + K] * r.dz;
        }
        part[2 * u] += nn;
        part[2 * u + 1] += nn * r.z[st];
      }
  }
  block_sum_vec<32>(part, 2 * NS, sh.red);
  double psi1 = 0.0;
  if (threadIdx.x == 0) {
    double num[16], chg[16];
    double Qtot = r.total_charge;
    for (int u = 0; u < NS; u++) {
      const DSpecies& s = r.sp[u];
      num[u] = part[2 * u] / (double)s.n_seg;
      chg[u] = num[u] <= 0.0 ? 0.0 : part[2 * u + 1] / num[u];
      bool fam = false;
      for (int g = 0; g < s.n_seg; g++) fam |= s.nst[g] > 1;
      if (fam || s.fixed >= 0) {
        Qtot += num[u] * chg[u];
        chg[u] = 0.0;
      }
    }
    double acc = 0.0;
    for (int u = 0; u < NS; u++) acc += num[u] * chg[u];
    double err = fabs(Qtot + acc);
    double Cstar = exp(-psi1);
    int iter = 1;
    while (err > 1e-10) {
      double fx = Qtot, fx1 = 0.0;
      for (int i = 0; i < NS; i++) {
        const double t = pow(Cstar, chg[i]) * num[i] * chg[i];
        fx += t;
        fx1 -= t * chg[i];
      }
      err = fabs(fx);
      if (fabs(fx1) < 1e-10) break;
      const double del = fmax(1.0, fabs(fx / fx1));
      psi1 -= fx / (fx1 * del);
      Cstar = exp(-psi1);
      iter++;
      if (iter > 1000) break;
    }
    sh.red[0] = psi1;
  }
  __syncthreads();
  psi1 = sh.red[0];
  __syncthreads();
  return psi1;
}

// ---------------------------------------------------------------------------
// full G(x): writes r.g; returns false on a normalisation error
// ---------------------------------------------------------------------------
// fp32: the propagator stage in FP32 (mixed precision), everything else FP64
__device__ bool objective(const DReq& r, Shared sh, bool fp32 = false) {
  const int P = r.NP;
  stage_lambda(r);
  stage_bond_factors(r, sh, fp32);
  int bad = -1;
  // requests with branched species run the instantiation that carries the tree path
  const bool ok = r.has_tree ? stage_densities<double, true>(r, sh, &bad)
                             : (fp32 ? stage_densities<float, false>(r, sh, &bad) : stage_densities<double, false>(r, sh, &bad));
  if (!ok) return false;
  stage_rho_hat(r, sh);
  for (size_t q = threadIdx.x; q < (size_t)r.NB * P; q += blockDim.x) r.Cmu[q] = 0.0;
  for (size_t q = threadIdx.x; q < (size_t)r.MB * 2 * P; q += blockDim.x) r.Clng[q] = 0.0;
  __syncthreads();
  if (r.funcs & 0x1) stage_fmt(r, sh, false);
  if (r.funcs & 0x2) stage_fmt(r, sh, true);
  if (r.funcs & 0x4) stage_msa(r, sh, false);
  if (r.funcs & 0x8) stage_msa(r, sh, true);
  double* g = r.g;
  const FftCtx fc = make_fft(sh.z, r);
  // mu_ex (NB), ln g (2 MB) and Psi (1): independent inverse transforms
  const int nout = r.NB + 2 * r.MB + 1;
  for (int g0 = 0; g0 < nout; g0 += r.TB) {
    const int nT = min(r.TB, nout - g0);
    dct2_inverse_kp(
        fc, nT,
        [&](int t, int k) {
          const int w = g0 + t;
          if (w < r.NB) return r.Cmu[(size_t)w * P + k];
          if (w < r.NB + 2 * r.MB) return r.Clng[(size_t)(w - r.NB) * P + k];
          // Poisson (solve_poisson_eq): (surf + sum_j z_j rho_hat_j) * w_coul
          double f = r.Csurf[k];
          for (int j = 0; j < r.NB; j++) f += r.Cb[(size_t)j * P + k] * r.z[j];
          return f * r.Wcoul[k];
        },
        [&](int kp, auto get) {
          const int K = 2 * kp;
#pragma unroll
          for (int u = 0; u < kMaxTB; u++)
            if (u < nT) stcg2(g + (size_t)(g0 + u) * P + K, get(u));
        });
  }
  const double shift = stage_neutrality(r, sh);
  if (threadIdx.x == 0) g[off_psic(r)] = r.x[off_psic(r)] + shift;
  // the pad point of odd grids is not an unknown: G(x) keeps it at 0 there, as x does
  if (SDFT_FFT_GEN && r.NPt != P)
    for (int w = threadIdx.x; w < nout; w += blockDim.x) g[(size_t)w * P + r.NPt] = 0.0;
  __syncthreads();
  return true;
}

}  // namespace
}  // namespace sdft
