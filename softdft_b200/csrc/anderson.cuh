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

struct SolveCfg {
  int max_iters;
  int anderm;
  double damping, mixing_max, switch_tole, tole;
};

struct AndersonState {
  int use_picard;
  double lam[kMaxAnderson];
};

// columns j != col of the history, ascending
__device__ __forceinline__ int hist_col(int c, int col) { return c < col ? c : c + 1; }

__device__ void lsqr_device(const DReq& r, int m, int col, double* lam, double* red) {
  const long long n = r.n;
  const int nc = m - 1;
  const double* gk = r.hg + (size_t)col * n;
  double* u = r.lsq_u;
  const double eps = 2.220446049250313e-16;
  const double atol = sqrt(eps), btol = sqrt(eps), conlim = 1.0 / sqrt(eps);
  const long long maxiter = n > nc ? n : nc;
  const double ctol = conlim > 0 ? 1.0 / conlim : 0.0;
  double v[kMaxAnderson], w[kMaxAnderson], tmp[kMaxAnderson];
  // u = b - A x, b = -g_k,  A[:, c] = G_hist[j_c] - g_k
  double ss = 0.0;
  for (long long q = threadIdx.x; q < n; q += blockDim.x) {
    const double gq = gk[q];
    double ax = 0.0;
    for (int c = 0; c < nc; c++) ax += (r.hg[(size_t)hist_col(c, col) * n + q] - gq) * lam[c];
    const double uq = -gq - ax;
    u[q] = uq;
    ss += uq * uq;
  }
  double beta = sqrt(block_sum(ss, red));
  double alpha = 0.0;
  for (int c = 0; c < nc; c++) v[c] = 0.0;
  if (beta > 0) {
    for (int c = 0; c < nc; c++) tmp[c] = 0.0;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) {
      const double uq = u[q] / beta;
      u[q] = uq;
      const double gq = gk[q];
      for (int c = 0; c < nc; c++) tmp[c] += (r.hg[(size_t)hist_col(c, col) * n + q] - gq) * uq;
    }
    block_sum_vec<kMaxAnderson>(tmp, nc, red);
    double a2 = 0.0;
    for (int c = 0; c < nc; c++) {
      v[c] = tmp[c];
      a2 += v[c] * v[c];
    }
    alpha = sqrt(a2);
  }
  if (alpha > 0)
    for (int c = 0; c < nc; c++) v[c] /= alpha;
  for (int c = 0; c < nc; c++) w[c] = v[c];
  double arnorm = alpha * beta;
  if (arnorm == 0) return;
  double anorm = 0, ddnorm = 0, res2 = 0, xxnorm = 0, zz = 0, sn2 = 0, cs2 = -1.0;
  double rhobar = alpha, phibar = beta;
  const double bnorm = beta;
  long long itn = 0;
  int istop = 0;
  while (itn < maxiter && istop == 0) {
    itn++;
    // u = A v - alpha u
    ss = 0.0;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) {
      const double gq = gk[q];
      double av = 0.0;
      for (int c = 0; c < nc; c++) av += (r.hg[(size_t)hist_col(c, col) * n + q] - gq) * v[c];
      const double uq = -alpha * u[q] + av;
      u[q] = uq;
      ss += uq * uq;
    }
    beta = sqrt(block_sum(ss, red));
    if (beta > 0) {
      anorm = sqrt(anorm * anorm + alpha * alpha + beta * beta);
      for (int c = 0; c < nc; c++) tmp[c] = 0.0;
      for (long long q = threadIdx.x; q < n; q += blockDim.x) {
        const double uq = u[q] / beta;
        u[q] = uq;
        const double gq = gk[q];
        for (int c = 0; c < nc; c++) tmp[c] += (r.hg[(size_t)hist_col(c, col) * n + q] - gq) * uq;
      }
      block_sum_vec<kMaxAnderson>(tmp, nc, red);
      double a2 = 0.0;
      for (int c = 0; c < nc; c++) {
        v[c] = -beta * v[c] + tmp[c];
        a2 += v[c] * v[c];
      }
      alpha = sqrt(a2);
      if (alpha > 0)
        for (int c = 0; c < nc; c++) v[c] /= alpha;
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
    for (int c = 0; c < nc; c++) {
      const double dk = w[c] / rho;
      dk2 += dk * dk;
      lam[c] += t1 * w[c];
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
}

// One Anderson update after r.g = G(x).  Returns ST_RUNNING, ST_OK (converged
// after this update) or ST_NONFINITE.
__device__ int anderson_step(const DReq& r, const SolveCfg& cfg, int iter, AndersonState& st, double* red,
                             double* err_out) {
  const long long n = r.n;
  const int m = cfg.anderm;
  const int col = (iter - 1) % m;
  double* hxc = r.hx + (size_t)col * n;
  double* hgc = r.hg + (size_t)col * n;
  double mx = 0.0;
  int bad = 0;
  for (long long q = threadIdx.x; q < n; q += blockDim.x) {
    const double xq = r.x[q];
    const double gq = r.g[q] - xq;
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
    for (long long q = threadIdx.x; q < n; q += blockDim.x) r.x[q] = c1 * r.x[q] + c2 * r.g[q];
  } else {
    st.use_picard = 0;
    lsqr_device(r, m, col, st.lam, red);
    const int nc = m - 1;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) {
      const double xq = hxc[q], gq = hgc[q];
      double sx = 0.0, sg = 0.0;
      for (int c = 0; c < nc; c++) {
        const int j = hist_col(c, col);
        sx += (r.hx[(size_t)j * n + q] - xq) * st.lam[c];
        sg += (r.hg[(size_t)j * n + q] - gq) * st.lam[c];
      }
      r.x[q] = xq + sx + amix * (gq + sg);
    }
  }
  __syncthreads();
  return err < cfg.tole ? ST_OK : ST_RUNNING;
}

}  // namespace sdft
