// omega.cuh -- grand potential and chains per species of the current state.
//
// grand_potential (src/iDFT/evaluation/analysis/grand_potential.jl:4-28):
//   Omega = [ sum_K f_ex(K)  -  sum rho_beads mu_ex trapez  +  sum rho_bonds lng / 2 ] dz
//           - sum_u N_u,
// with f_ex the point-wise free energy of each functional on the true grid
// (TPT1mfmt.jl:163-186, TPT1msa.jl:103-126, mfmt.jl, msa.jl; no trapez weight)
// computed from the densities of the last G(x) evaluation, mu_ex and lng from
// the current x, and N_u from get_num_species (num_species.jl:1-38).
#pragma once

#include "objective.cuh"

namespace sdft {
namespace {  // internal linkage: each kernel build (kernels.cuh) has its own copy

// out[0] = Omega, out[1 + u] = N_u
__device__ void grand_potential(const DReq& r, Shared sh, double* out) {
  const int P = r.NP, NB = r.NB, MB = r.MB;
  double fe = 0.0;
  for (int pass = 0; pass < 2; pass++) {
    const bool tpt1 = pass == 1;
    if (!(r.funcs & (tpt1 ? 0x2 : 0x1))) continue;
    fmt_weighted(r, sh, tpt1);
    double acc = 0.0;
    for (int K = threadIdx.x; K < grid_points(r); K += blockDim.x) {
      double n0 = r.wa[K], n1 = r.wa[(size_t)P + K], n2 = r.wa[(size_t)2 * P + K], n3 = r.wa[(size_t)3 * P + K];
      double v1 = r.wa[(size_t)4 * P + K], v2 = r.wa[(size_t)5 * P + K];
      if (n3 > 0.95) {
        const double fac = 0.95 / n3;
        n0 *= fac; n1 *= fac; n2 *= fac; n3 *= fac; v1 *= fac; v2 *= fac;
      }
      const double om = 1.0 - n3;
      const double lt = log(om);
      const double inv_denom = 1.0 / (36.0 * kPi * (n3 * n3) * (om * om));
      double f = -n0 * lt + (n1 * n2 - v1 * v2) / om + (n2 * n2 * n2 - 3.0 * n2 * (v2 * v2)) * (n3 + (om * om) * lt) * inv_denom;
      if (tpt1) {
        const double Xi = 1.0 - (v2 * v2) / (n2 * n2);
        const double i1 = 1.0 / (1.0 - n3);
        const double term2 = n2 * Xi / 4.0 * (i1 * i1);
        const double term3 = (n2 * n2) * Xi / 72.0 * (i1 * i1 * i1);
        for (int u = 0; u < MB; u++) {
          const int bi = r.bonds[2 * u], bj = r.bonds[2 * u + 1];
          const double sij = (r.sig[bi] + r.sig[bj]) / 2;
          const double tau = r.sig[bi] * r.sig[bj] / sij;
          const double y = i1 + term2 * tau + term3 * (tau * tau);
          f -= 0.5 * (r.wb[(size_t)(u * 2) * P + K] + r.wb[(size_t)(u * 2 + 1) * P + K]) * log(y);
        }
      }
      acc += f;
    }
    fe += block_sum(acc, sh.red);
  }
  for (int pass = 0; pass < 2; pass++) {
    const bool tpt1 = pass == 1;
    if (!(r.funcs & (tpt1 ? 0x8 : 0x4))) continue;
    msa_weighted(r, sh, tpt1);
    __syncthreads();
    double acc = 0.0;
    for (int K = threadIdx.x; K < grid_points(r); K += blockDim.x) {
      double rho[kMaxBeads];
      for (int j = 0; j < NB; j++) rho[j] = r.wa[(size_t)j * P + K];
      const MsaGamma gm = gamma_msa_point(r, rho);
      double s = 0.0;
      for (int j = 0; j < NB; j++) s += rho[j] * r.z[j] * (r.z[j] * gm.G + gm.eta * r.sig[j]) / (1.0 + gm.G * r.sig[j]);
      double f = (gm.G * gm.G * gm.G) / (3.0 * kPi) - r.lB * s;
      if (tpt1)
        for (int u = 0; u < MB; u++) {
          const int i = r.bonds[2 * u], j = r.bonds[2 * u + 1];
          const double sij = (r.sig[i] + r.sig[j]) / 2.0;
          const double Xi = (r.z[i] - gm.eta * (r.sig[i] * r.sig[i])) / (1.0 + gm.G * r.sig[i]);
          const double Xj = (r.z[j] - gm.eta * (r.sig[j] * r.sig[j])) / (1.0 + gm.G * r.sig[j]);
          f -= 0.5 * (r.wb[(size_t)(u * 2) * P + K] + r.wb[(size_t)(u * 2 + 1) * P + K]) * (-r.lB / sij * Xi * Xj);
        }
      acc += f;
    }
    fe += block_sum(acc, sh.red);
  }
  // - rho mu_ex trapez + rho_bonds lng / 2, on the current unknowns
  const double* mu = r.x;
  const double* lng = r.x + (size_t)P * NB;
  double a1 = 0.0, a2 = 0.0;
  for (size_t q = threadIdx.x; q < (size_t)NB * P; q += blockDim.x)
    if ((int)(q % P) < grid_points(r)) a1 += r.rho_beads[q] * mu[q] * r.trapez[q];
  for (size_t q = threadIdx.x; q < (size_t)2 * MB * P; q += blockDim.x)
    if ((int)(q % P) < grid_points(r)) a2 += r.rho_bonds[q] * lng[q] / 2.0;
  a1 = block_sum(a1, sh.red);
  a2 = block_sum(a2, sh.red);
  double om = ((fe - a1) + a2) * r.dz;
  // chains per species
  double part[16];
  for (int u = 0; u < r.NS; u++) {
    const DSpecies& s = r.sp[u];
    double acc = 0.0;
    for (int g = 0; g < s.n_seg; g++)
      for (int ii = 0; ii < s.nst[g]; ii++) {
        const int st = s.states[g * s.S + ii];
        const double* rs = s.rho_seg + (size_t)(g * s.S + ii) * P;
        if (g == 0 && s.fixed >= 0) {
          if (threadIdx.x == 0) acc += rs[s.fixed] / (double)s.n_seg;
        } else {
          double nn = 0.0;
          for (int K = threadIdx.x; K < grid_points(r); K += blockDim.x) nn += rs[K] * r.trapez[(size_t)st * P + K] * r.dz;
          acc += nn / (double)s.n_seg;
        }
      }
    part[u] = acc;
  }
  block_sum_vec<16>(part, r.NS, sh.red);
  if (threadIdx.x == 0) {
    for (int u = 0; u < r.NS; u++) {
      om -= part[u];
      out[1 + u] = part[u];
    }
    out[0] = om;
  }
  __syncthreads();
}

}  // namespace
}  // namespace sdft
