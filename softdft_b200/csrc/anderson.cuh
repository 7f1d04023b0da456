// anderson.cuh -- Anderson mixing driver of one request, run by its CTA.
//
// Restates solver_function(::AndersonMixing, ...)
// (src/NonlinearSolvers/fixed_point/AndersonMixing.jl:56-169): ring-buffer
// history col = (iter-1) mod m of x and G(x)-x, err = max|G(x)-x| floored at
// 1e-20, amix = min(mixing_max, damping/err), Picard x <- (1-a)x + aG while
// iter < m or (err > switch_tole and still Picard), else the least-squares
// step of IterativeSolvers.lsqr! warm-started from the previous coefficients:
//   x <- x + dX lambda + amix (g + dG lambda),  min || dG lambda + g ||.
// LSQR is the published Paige-Saunders recurrence (ACM TOMS 8(1), 1982) with
// atol = btol = sqrt(eps), conlim = 1/sqrt(eps), maxiter = max(n, m-1); its
// n-vectors live in global memory and its (m-1)-vectors in every thread's
// registers (all threads run the same scalar recurrence on CTA-reduced values).
#pragma once

#include "common.cuh"

namespace sdft {
namespace {  // internal linkage: each kernel build (kernels.cuh) has its own copy

struct AndersonState {
  int use_picard;
  double lam[kMaxAnderson];
};

// columns j != col of the history, ascending
__device__ __forceinline__ int hist_col(int c, int col) { return c < col ? c : c + 1; }

// One sweep over q of  w_q = a_q . v + coef * u_q  (a_q[c] = G_hist[j_c][q] - g_k[q]),
// storing w, and accumulating ||w||^2 (acc[NC]) and A^T w (acc[c]).  Element
// pairs move as 16-byte loads (every history column starts on a 256-byte
// boundary; the last element of an odd n is handled alone) and each thread
// keeps U pairs in flight, every load of a round issued before the first use;
// the history columns, g_k and u are distinct arrays.
template <int NC>
__device__ __forceinline__ void lsqr_pass(const double* __restrict__ gk, const double* const* hc, double* __restrict__ u,
                                          long long n, int nc, const double* v, double coef, double* acc) {
  constexpr int U = 2;  // element pairs in flight per thread (more spill at the 128-register cap)
  const long long n2 = n >> 1;
  const double2* __restrict__ gk2 = reinterpret_cast<const double2*>(gk);
  double2* __restrict__ u2 = reinterpret_cast<double2*>(u);
  const int bd = blockDim.x;
  for (long long p0 = threadIdx.x; p0 < n2; p0 += U * bd) {
    double2 g[U], uu[U], h[U][NC];
    bool on[U];
#pragma unroll
    for (int k = 0; k < U; k++) {
      const long long pk = p0 + (long long)k * bd;
      on[k] = pk < n2;
      if (!on[k]) continue;
      g[k] = __ldcg(gk2 + pk);
      uu[k] = __ldcg(u2 + pk);
#pragma unroll
      for (int c = 0; c < NC; c++)
        if (c < nc) h[k][c] = __ldcg(reinterpret_cast<const double2*>(hc[c]) + pk);
    }
#pragma unroll
    for (int k = 0; k < U; k++) {
      if (!on[k]) continue;
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const double gq = e ? g[k].y : g[k].x;
        const double uq = e ? uu[k].y : uu[k].x;
        double aq[NC];
        double av = 0.0;
#pragma unroll
        for (int c = 0; c < NC; c++)
          if (c < nc) {
            aq[c] = (e ? h[k][c].y : h[k][c].x) - gq;
            av += aq[c] * v[c];
          }
        const double wq = coef * uq + av;
        if (e) uu[k].y = wq;
        else uu[k].x = wq;
        acc[NC] += wq * wq;
#pragma unroll
        for (int c = 0; c < NC; c++)
          if (c < nc) acc[c] += aq[c] * wq;
      }
      __stcg(u2 + p0 + (long long)k * bd, uu[k]);
    }
  }
  if ((n & 1) && threadIdx.x == 0) {  // the last element of an odd length
    const long long q = n - 1;
    const double gq = gk[q];
    double aq[NC];
    double av = 0.0;
#pragma unroll
    for (int c = 0; c < NC; c++)
      if (c < nc) {
        aq[c] = hc[c][q] - gq;
        av += aq[c] * v[c];
      }
    const double wq = coef * u[q] + av;
    u[q] = wq;
    acc[NC] += wq * wq;
#pragma unroll
    for (int c = 0; c < NC; c++)
      if (c < nc) acc[c] += aq[c] * wq;
  }
}

// Streams element pairs p = tid, tid + bd, ... < n2 through shared memory: each
// thread copies its own pairs of up to A arrays (src(a) gives array a as double2,
// nullptr: not read) into its own stage slots with cp.async, D pairs ahead, and
// body(p, slots) reads them back as slots[a * blockDim.x].  A thread reads only
// what it copied, so no barrier is needed, and the copies of the next D pairs
// are in flight while the current one is combined (plain loads hold registers
// until their first use, which caps them at about two pairs a thread here).
// stage: D * A * blockDim.x double2 slots.
template <int A, int D, class Src, class Body>
__device__ __forceinline__ void staged_pairs(long long n2, double2* stage, Src src, Body body) {
  const int bd = blockDim.x, tid = threadIdx.x;
  auto issue = [&](long long p, int s) {
    if (p < n2) {
      double2* b = stage + (size_t)s * A * bd + tid;
#pragma unroll
      for (int a = 0; a < A; a++) {
        const double2* g = src(a);
        if (g) cp_async16(b + (size_t)a * bd, g + p);
      }
    }
    cp_async_commit();  // an empty group past the end keeps the group count uniform
  };
#pragma unroll
  for (int s = 0; s < D; s++) issue(tid + (long long)s * bd, s);
  int s = 0;
  for (long long p = tid; p < n2; p += bd) {
    cp_async_wait<D - 1>();
    body(p, static_cast<const double2*>(stage + (size_t)s * A * bd + tid));
    // the slots of stage s were read and used by body
    issue(p + (long long)D * bd, s);
    s = s + 1 == D ? 0 : s + 1;
  }
  cp_async_wait<0>();
}

// lsqr_pass with its operands streamed through shared memory (staged_pairs):
// slots g_k, u, the history columns
template <int NC, int D>
__device__ __forceinline__ void lsqr_pass_staged(const double* __restrict__ gk, const double* const* hc,
                                                 double* __restrict__ u, long long n, int nc, const double* v,
                                                 double coef, double* acc, double2* stage) {
  const long long n2 = n >> 1;
  double2* u2 = reinterpret_cast<double2*>(u);
  const int bd = blockDim.x;
  staged_pairs<NC + 2, D>(
      n2, stage,
      [&](int a) -> const double2* {
        if (a == 0) return reinterpret_cast<const double2*>(gk);
        if (a == 1) return u2;
        return a - 2 < nc ? reinterpret_cast<const double2*>(hc[a - 2]) : nullptr;
      },
      [&](long long p, const double2* b) {
        const double2 g = b[0];
        double2 uu = b[bd];
        double2 h[NC];
#pragma unroll
        for (int c = 0; c < NC; c++)
          if (c < nc) h[c] = b[(size_t)(2 + c) * bd];
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const double gq = e ? g.y : g.x;
          const double uq = e ? uu.y : uu.x;
          double aq[NC];
          double av = 0.0;
#pragma unroll
          for (int c = 0; c < NC; c++)
            if (c < nc) {
              aq[c] = (e ? h[c].y : h[c].x) - gq;
              av += aq[c] * v[c];
            }
          const double wq = coef * uq + av;
          if (e) uu.y = wq;
          else uu.x = wq;
          acc[NC] += wq * wq;
#pragma unroll
          for (int c = 0; c < NC; c++)
            if (c < nc) acc[c] += aq[c] * wq;
        }
        __stcg(u2 + p, uu);
      });
  if ((n & 1) && threadIdx.x == 0) {  // the last element of an odd length
    const long long q = n - 1;
    const double gq = gk[q];
    double aq[NC];
    double av = 0.0;
#pragma unroll
    for (int c = 0; c < NC; c++)
      if (c < nc) {
        aq[c] = hc[c][q] - gq;
        av += aq[c] * v[c];
      }
    const double wq = coef * u[q] + av;
    u[q] = wq;
    acc[NC] += wq * wq;
#pragma unroll
    for (int c = 0; c < NC; c++)
      if (c < nc) acc[c] += aq[c] * wq;
  }
}

// u = b - A x with b = -g_k and A[:, c] = G_hist[j_c] - g_k, its squared norm
// (acc[NC]) and A^T u (acc[c]).  Thread t takes the elements t, t + bd, t + 2 bd,
// ... in that order, U of them per round with every load issued before the first
// use; the order of every sum is that of one element per round.
template <int NC>
__device__ __forceinline__ void lsqr_init_pass(const double* __restrict__ gk, const double* const* hc,
                                               double* __restrict__ u, long long n, int nc, const double* x,
                                               double* acc) {
  constexpr int U = 4;
  const int bd = blockDim.x;
  for (long long q0 = threadIdx.x; q0 < n; q0 += (long long)U * bd) {
    double g[U], h[U][NC];
#pragma unroll
    for (int k = 0; k < U; k++) {
      const long long q = q0 + (long long)k * bd;
      if (q >= n) continue;
      g[k] = __ldcg(gk + q);
#pragma unroll
      for (int c = 0; c < NC; c++)
        if (c < nc) h[k][c] = __ldcg(hc[c] + q);
    }
#pragma unroll
    for (int k = 0; k < U; k++) {
      const long long q = q0 + (long long)k * bd;
      if (q >= n) continue;
      const double gq = g[k];
      double aq[NC];
      double ax = 0.0;
#pragma unroll
      for (int c = 0; c < NC; c++)
        if (c < nc) {
          aq[c] = h[k][c] - gq;
          ax += aq[c] * x[c];
        }
      const double uq = -gq - ax;
      __stcg(u + q, uq);
      acc[NC] += uq * uq;
#pragma unroll
      for (int c = 0; c < NC; c++)
        if (c < nc) acc[c] += aq[c] * uq;
    }
  }
}

// One sweep over the history serves each LSQR iteration: the next vector
// w = A v - alpha u is stored unnormalised (u_true = uscale * u_stored) while
// ||w||^2 and A^T w are accumulated in the same pass; A^T u_{i+1} = A^T w / beta
// follows once beta = ||w|| is known.  The recurrence is LSQR's own; only the
// order of the divisions by beta differs.  NC bounds the column count at
// compile time so that the per-thread column values stay in registers.
template <int NC>
__device__ __noinline__ void lsqr_sweep_device(const DReq& r, int nc, int col, double* lam, double* red,
                                              double2* stage, size_t stage_bytes) {
  const long long n = r.n, hs = r.hstride;
  const double* gk = r.hg + (size_t)col * hs;
  const double* hc[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) hc[c] = c < nc ? r.hg + (size_t)hist_col(c, col) * hs : gk;
  double* u = r.lsq_u;
  const double eps = 2.220446049250313e-16;
  const double atol = sqrt(eps), btol = sqrt(eps), conlim = 1.0 / sqrt(eps);
  const long long maxiter = n > nc ? n : nc;
  const double ctol = conlim > 0 ? 1.0 / conlim : 0.0;
  double v[NC], w[NC], acc[NC + 1], x[NC];
  // pipeline depth of the staged passes that the shared-memory stage holds
  const size_t per_stage = (size_t)(NC + 2) * blockDim.x * sizeof(double2);
  const int depth = stage_bytes >= 3 * per_stage ? 3 : stage_bytes >= 2 * per_stage ? 2 : 0;
#pragma unroll
  for (int c = 0; c < NC; c++) x[c] = c < nc ? lam[c] : 0.0;
  // u = b - A x with b = -g_k and A[:, c] = G_hist[j_c] - g_k; ||u||^2 and A^T u
#pragma unroll
  for (int c = 0; c <= NC; c++) acc[c] = 0.0;
  lsqr_init_pass<NC>(gk, hc, u, n, nc, x, acc);
  block_sum_vec<NC + 1>(acc, NC + 1, red);
  double beta = sqrt(acc[NC]);
  double uscale = beta > 0 ? 1.0 / beta : 1.0;
  double alpha = 0.0;
#pragma unroll
  for (int c = 0; c < NC; c++) v[c] = 0.0;
  if (beta > 0) {
    double a2 = 0.0;
#pragma unroll
    for (int c = 0; c < NC; c++)
      if (c < nc) {
        v[c] = acc[c] / beta;
        a2 += v[c] * v[c];
      }
    alpha = sqrt(a2);
  }
  if (alpha > 0)
#pragma unroll
    for (int c = 0; c < NC; c++) v[c] /= alpha;
#pragma unroll
  for (int c = 0; c < NC; c++) w[c] = v[c];
  double arnorm = alpha * beta;
  if (arnorm == 0) return;
  double anorm = 0, ddnorm = 0, res2 = 0, xxnorm = 0, zz = 0, sn2 = 0, cs2 = -1.0;
  double rhobar = alpha, phibar = beta;
  const double bnorm = beta;
  long long itn = 0;
  int istop = 0;
  while (itn < maxiter && istop == 0) {
    itn++;
    // w = A v - alpha u (unnormalised), its norm and A^T w in one sweep
    const double coef = alpha * uscale;
#pragma unroll
    for (int c = 0; c <= NC; c++) acc[c] = 0.0;
    if (depth == 3) lsqr_pass_staged<NC, 3>(gk, hc, u, n, nc, v, -coef, acc, stage);
    else if (depth == 2) lsqr_pass_staged<NC, 2>(gk, hc, u, n, nc, v, -coef, acc, stage);
    else lsqr_pass<NC>(gk, hc, u, n, nc, v, -coef, acc);
    block_sum_vec<NC + 1>(acc, NC + 1, red);
    beta = sqrt(acc[NC]);
    if (beta > 0) {
      uscale = 1.0 / beta;
      anorm = sqrt(anorm * anorm + alpha * alpha + beta * beta);
      double a2 = 0.0;
#pragma unroll
      for (int c = 0; c < NC; c++)
        if (c < nc) {
          v[c] = -beta * v[c] + acc[c] / beta;
          a2 += v[c] * v[c];
        }
      alpha = sqrt(a2);
      if (alpha > 0)
#pragma unroll
        for (int c = 0; c < NC; c++) v[c] /= alpha;
    }
    const double rhobar1 = rhobar, psi = 0.0;
    const double rho = sqrt(rhobar1 * rhobar1 + beta * beta);
    const double cs = rhobar1 / rho, sn = beta / rho;
    const double theta = sn * alpha;
    rhobar = -cs * alpha;
    const double phi = cs * phibar;
    phibar = sn * phibar;
    const double tau = sn * phi;
    const double t1 = phi / rho, t2 = -theta / rho;
    double dk2 = 0.0;
#pragma unroll
    for (int c = 0; c < NC; c++)
      if (c < nc) {
        const double dk = w[c] / rho;
        dk2 += dk * dk;
        x[c] += t1 * w[c];
        w[c] = v[c] + t2 * w[c];
      }
    ddnorm += dk2;
    const double delta = sn2 * rho, gambar = -cs2 * rho, rhs = phi - delta * zz;
    const double zbar = rhs / gambar;
    const double xnorm = sqrt(xxnorm + zbar * zbar);
    const double gamma = sqrt(gambar * gambar + theta * theta);
    cs2 = gambar / gamma;
    sn2 = theta / gamma;
    zz = rhs / gamma;
    xxnorm += zz * zz;
    const double acond = anorm * sqrt(ddnorm);
    const double res1 = phibar * phibar;
    res2 += psi * psi;
    const double rnorm = sqrt(res1 + res2);
    arnorm = alpha * fabs(tau);
    const double test1 = rnorm / bnorm;
    const double test2 = (anorm * rnorm != 0) ? arnorm / (anorm * rnorm) : INFINITY;
    const double test3 = acond != 0 ? 1.0 / acond : INFINITY;
    const double t1b = test1 / (1.0 + anorm * xnorm / bnorm);
    const double rtol = btol + atol * anorm * xnorm / bnorm;
    if (itn >= maxiter) istop = 7;
    if (1.0 + test3 <= 1.0) istop = 6;
    if (1.0 + test2 <= 1.0) istop = 5;
    if (1.0 + t1b <= 1.0) istop = 4;
    if (test3 <= ctol) istop = 3;
    if (test2 <= atol) istop = 2;
    if (test1 <= rtol) istop = 1;
  }
#pragma unroll
  for (int c = 0; c < NC; c++)
    if (c < nc) lam[c] = x[c];
}

__device__ void lsqr_device(const DReq& r, int m, int col, double* lam, double* red, double2* stage,
                            size_t stage_bytes) {
  const int nc = m - 1;
  if (nc <= 4) lsqr_sweep_device<4>(r, nc, col, lam, red, stage, stage_bytes);
  else if (nc <= 9) lsqr_sweep_device<9>(r, nc, col, lam, red, stage, stage_bytes);
  else lsqr_sweep_device<kMaxAnderson - 1>(r, nc, col, lam, red, stage, stage_bytes);
}

// x <- X_k + dX lambda + amix (g_k + dG lambda) over element pairs (AndersonMixing.jl:144),
// the sums over the history columns j != col in ascending order as the reference's
// matrix-vector products; NC bounds the column count so that the column values stay
// in registers
template <int NC>
__device__ __noinline__ void anderson_mix(const DReq& r, int nc, int col, const double* lam, double amix) {
  const long long n = r.n, hs = r.hstride, n2 = n >> 1;
  const double* __restrict__ hxc = r.hx + (size_t)col * hs;
  const double* __restrict__ hgc = r.hg + (size_t)col * hs;
  const double* hxj[NC];
  const double* hgj[NC];
  double lm[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) {
    const int j = c < nc ? hist_col(c, col) : col;
    hxj[c] = r.hx + (size_t)j * hs;
    hgj[c] = r.hg + (size_t)j * hs;
    lm[c] = c < nc ? lam[c] : 0.0;
  }
  double* __restrict__ x = r.x;
  auto mix = [&](double xq, double gq, const double* hxq, const double* hgq) {
    double sx = 0.0, sg = 0.0;
#pragma unroll
    for (int c = 0; c < NC; c++)
      if (c < nc) {
        sx += (hxq[c] - xq) * lm[c];
        sg += (hgq[c] - gq) * lm[c];
      }
    return xq + sx + amix * (gq + sg);
  };
  for (long long p = threadIdx.x; p < n2; p += blockDim.x) {
    const double2 xk = __ldcg(reinterpret_cast<const double2*>(hxc) + p);
    const double2 gk = __ldcg(reinterpret_cast<const double2*>(hgc) + p);
    double2 hx2[NC], hg2[NC];
#pragma unroll
    for (int c = 0; c < NC; c++)
      if (c < nc) {
        hx2[c] = __ldcg(reinterpret_cast<const double2*>(hxj[c]) + p);
        hg2[c] = __ldcg(reinterpret_cast<const double2*>(hgj[c]) + p);
      }
    double ax[NC], ag[NC], bx[NC], bg[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
      ax[c] = c < nc ? hx2[c].x : 0.0;
      ag[c] = c < nc ? hg2[c].x : 0.0;
      bx[c] = c < nc ? hx2[c].y : 0.0;
      bg[c] = c < nc ? hg2[c].y : 0.0;
    }
    __stcg(reinterpret_cast<double2*>(x) + p, make_double2(mix(xk.x, gk.x, ax, ag), mix(xk.y, gk.y, bx, bg)));
  }
  if ((n & 1) && threadIdx.x == 0) {  // the last element of an odd length
    const long long q = n - 1;
    double ax[NC], ag[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
      ax[c] = c < nc ? hxj[c][q] : 0.0;
      ag[c] = c < nc ? hgj[c][q] : 0.0;
    }
    x[q] = mix(hxc[q], hgc[q], ax, ag);
  }
}

// One Anderson update after r.g = G(x).  Returns ST_RUNNING, ST_OK (converged
// after this update) or ST_NONFINITE.  stage: shared memory free during the
// update (the transform buffers), stage_bytes of it; 0 when there is none.
__device__ int anderson_step(const DReq& r, const SolveCfg& cfg, int iter, AndersonState& st, double* red,
                             double2* stage, size_t stage_bytes, double* err_out) {
  const long long n = r.n, hs = r.hstride, n2 = n >> 1;
  const int m = cfg.anderm;
  const int col = (iter - 1) % m;
  double* __restrict__ hxc = r.hx + (size_t)col * hs;
  double* __restrict__ hgc = r.hg + (size_t)col * hs;
  const double* __restrict__ xv = r.x;
  const double* __restrict__ gv = r.g;
  double mx = 0.0;
  int bad = 0;
  // ring-buffer column col: x and G(x) - x (AndersonMixing.jl:102-111), element
  // pairs, streamed through the stage when it holds four rounds (the maximum and
  // the finite test do not depend on the order)
  auto column = [&](long long p, double2 xq, double2 g2) {
    const double2 gq = make_double2(g2.x - xq.x, g2.y - xq.y);
    __stcg(reinterpret_cast<double2*>(hxc) + p, xq);
    __stcg(reinterpret_cast<double2*>(hgc) + p, gq);
    const double a0 = fabs(gq.x), a1 = fabs(gq.y);
    if (!isfinite(a0) || !isfinite(a1)) bad = 1;
    mx = fmax(mx, fmax(a0, a1));
  };
  if (stage_bytes >= (size_t)4 * 2 * blockDim.x * sizeof(double2)) {
    const int bd = blockDim.x;
    staged_pairs<2, 4>(
        n2, stage,
        [&](int a) { return reinterpret_cast<const double2*>(a == 0 ? xv : gv); },
        [&](long long p, const double2* b) { column(p, b[0], b[bd]); });
  } else {
    for (long long p = threadIdx.x; p < n2; p += blockDim.x)
      column(p, __ldcg(reinterpret_cast<const double2*>(xv) + p), __ldcg(reinterpret_cast<const double2*>(gv) + p));
  }
  if ((n & 1) && threadIdx.x == 0) {
    const long long q = n - 1;
    const double xq = xv[q], gq = gv[q] - xq;
    hxc[q] = xq;
    hgc[q] = gq;
    const double a = fabs(gq);
    if (!isfinite(a)) bad = 1;
    mx = fmax(mx, a);
  }
  const double nb = block_sum((double)bad, red);
  mx = block_max(mx, red);
  if (nb > 0) {
    *err_out = mx;
    return ST_NONFINITE;
  }
  const double err = mx > 1e-20 ? mx : 1e-20;
  *err_out = err;
  const double amix = fmin(cfg.mixing_max, cfg.damping / err);
  if (iter < m || (err > cfg.switch_tole && st.use_picard)) {
    const double c1 = 1.0 - amix, c2 = amix;
    double* __restrict__ x = r.x;
    auto picard = [&](long long p, double2 xq, double2 gq) {
      __stcg(reinterpret_cast<double2*>(x) + p, make_double2(c1 * xq.x + c2 * gq.x, c1 * xq.y + c2 * gq.y));
    };
    if (stage_bytes >= (size_t)4 * 2 * blockDim.x * sizeof(double2)) {
      const int bd = blockDim.x;
      staged_pairs<2, 4>(
          n2, stage,
          [&](int a) { return reinterpret_cast<const double2*>(a == 0 ? x : gv); },
          [&](long long p, const double2* b) { picard(p, b[0], b[bd]); });
    } else {
      for (long long p = threadIdx.x; p < n2; p += blockDim.x)
        picard(p, __ldcg(reinterpret_cast<const double2*>(x) + p), __ldcg(reinterpret_cast<const double2*>(gv) + p));
    }
    if ((n & 1) && threadIdx.x == 0) x[n - 1] = c1 * x[n - 1] + c2 * gv[n - 1];
  } else {
    st.use_picard = 0;
    lsqr_device(r, m, col, st.lam, red, stage, stage_bytes);
    const int nc = m - 1;
    if (nc <= 4) anderson_mix<4>(r, nc, col, st.lam, amix);
    else if (nc <= 9) anderson_mix<9>(r, nc, col, st.lam, amix);
    else anderson_mix<kMaxAnderson - 1>(r, nc, col, st.lam, amix);
  }
  __syncthreads();
  return err < cfg.tole ? ST_OK : ST_RUNNING;
}

}  // namespace
}  // namespace sdft
