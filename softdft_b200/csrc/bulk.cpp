// bulk.cpp -- host evaluation of the bulk (iLST) state for the C ABI.
//
// One call evaluates, for given species densities and the current bulk excess
// chemical potentials / bond contact logarithms, the two expensive steps of the
// bulk residual (src/iLST/evaluation/objective/residual_bulkstate.jl:26-35):
//   * eval_bulk_density! (eval_bulk_density.jl:9-22): segment, bead and
//     bond-end densities from the bulk freely-jointed propagators of every
//     species (species_model/freely_jointed/child_propagators.jl:22-62,
//     parent_propagators.jl:27-73, partition_function.jl:21-53,
//     accumulate_densities.jl), monomer beads by their state sums
//     (species_model/monomerbead/*.jl); chains whose propagator products leave
//     the double range are evaluated with log-domain propagators;
//   * bulk_chemical_potential (bulk_chemical_potential.jl:9-25): ideal term,
//     White-Bear FMT (free_energy/excluded_volume/mfmt.jl:275-299), TPT1-FMT
//     (TPT1mfmt.jl:399-444), MSA with the damped Gamma fixed point
//     (free_energy/electrostaticcorrelations/msa.jl:147-230) and TPT1-MSA
//     (TPT1msa.jl:200-282), then mu_species -= ln Xi.
// The solver loops around it (AndersonResidual) stay with the caller.
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include "../../include/softdft.h"

namespace {

constexpr double kPiB = 3.14159265358979323846;
const double kNegInf = -std::numeric_limits<double>::infinity();

struct Tree {
  int n, S, C;  // segments, max states, max children
  const int32_t* nst;
  const int32_t* states;
  const int32_t* parent;
  const int32_t* nch;
  const int32_t* children;
  const int32_t* level_ptr;
  const int32_t* level_segs;
  int n_levels;
  int st(int seg, int i) const { return states[(size_t)seg * S + i]; }
  int ch(int seg, int k) const { return children[(size_t)seg * C + k]; }
};

struct Ctx {
  const sdft_bulk_system* sys;
  const double* mu;
  const double* lng;
  int bond(int a, int b) const {
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    for (int u = 0; u < sys->mb; u++)
      if (sys->bond_types[2 * u] == lo && sys->bond_types[2 * u + 1] == hi) return u;
    return -1;
  }
};

double lse(const double* v, int n) {
  double m = kNegInf;
  for (int i = 0; i < n; i++) m = std::fmax(m, v[i]);
  if (!std::isfinite(m)) return m;
  double s = 0.0;
  for (int i = 0; i < n; i++) s += std::exp(v[i] - m);
  return m + std::log(s);
}

// gC[((ij * C + ic) * S + ii) * n + p], gP[(ij * S + ii) * n + c] as in the reference's (S, C, S, n) / (S, S, n)
struct Props {
  int n, S, C;
  std::vector<double> gC, gP;
  double& c(int ij, int ic, int ii, int p) { return gC[(((size_t)ij * C + ic) * S + ii) * n + p]; }
  double& pp(int ij, int ii, int c_) { return gP[((size_t)ij * S + ii) * n + c_]; }
  double csum(int ic, int ii, int p) {
    double s = 0.0;
    for (int q = 0; q < S; q++) s += c(q, ic, ii, p);
    return s;
  }
  double psum(int ii, int p) {
    double s = 0.0;
    for (int q = 0; q < S; q++) s += pp(q, ii, p);
    return s;
  }
};

// linear-domain propagators and Xi (child_propagators.jl:22-62, parent_propagators.jl:27-73,
// partition_function.jl:21-53); log_domain: the same recursions on logarithms
double fj_propagators(const Ctx& x, const Tree& t, Props& g, bool log_domain) {
  const double* dm = x.sys->delta_muH;
  const int n = t.n, S = t.S, C = t.C;
  g.n = n;
  g.S = S;
  g.C = C;
  const double zero = log_domain ? kNegInf : 0.0;
  g.gC.assign((size_t)S * C * S * n, zero);
  g.gP.assign((size_t)S * S * n, zero);
  std::vector<double> tmp(S);
  auto csum = [&](int ic, int ii, int p) {
    if (!log_domain) return g.csum(ic, ii, p);
    for (int q = 0; q < S; q++) tmp[q] = g.c(q, ic, ii, p);
    return lse(tmp.data(), S);
  };
  auto psum = [&](int ii, int p) {
    if (!log_domain) return g.psum(ii, p);
    for (int q = 0; q < S; q++) tmp[q] = g.pp(q, ii, p);
    return lse(tmp.data(), S);
  };
  for (int L = t.n_levels - 1; L >= 0; L--)
    for (int k = t.level_ptr[L]; k < t.level_ptr[L + 1]; k++) {
      const int p = t.level_segs[k];
      for (int ii = 0; ii < t.nst[p]; ii++) {
        g.c(0, 0, ii, p) = log_domain ? 0.0 : 1.0;
        for (int ic = 0; ic < t.nch[p]; ic++) {
          const int c = t.ch(p, ic);
          for (int ij = 0; ij < t.nst[c]; ij++) {
            const int sj = t.st(c, ij);
            const int b = x.bond(t.st(p, ii), sj);
            if (log_domain) {
              double val = -dm[sj] - x.mu[sj] + x.lng[b];
              for (int igc = 0; igc < t.nch[c]; igc++) val += csum(igc, ij, c);
              g.c(ij, ic, ii, p) = val;
            } else {
              double val = std::exp(-dm[sj] - x.mu[sj] + x.lng[b]);
              for (int igc = 0; igc < t.nch[c]; igc++) val *= g.csum(igc, ij, c);
              g.c(ij, ic, ii, p) = val;
            }
          }
        }
      }
    }
  for (int L = 0; L < t.n_levels; L++)
    for (int k = t.level_ptr[L]; k < t.level_ptr[L + 1]; k++) {
      const int c = t.level_segs[k];
      for (int ij = 0; ij < t.nst[c]; ij++) {
        g.pp(0, ij, c) = log_domain ? 0.0 : 1.0;
        const int p = t.parent[c];
        if (p < 0) continue;
        for (int ii = 0; ii < t.nst[p]; ii++) {
          const int si = t.st(p, ii);
          const int b = x.bond(si, t.st(c, ij));
          if (log_domain) {
            double val = -dm[si] - x.mu[si] + x.lng[b] + psum(ii, p);
            for (int ioc = 0; ioc < t.nch[p]; ioc++)
              if (t.ch(p, ioc) != c) val += csum(ioc, ii, p);
            g.pp(ii, ij, c) = val;
          } else {
            double val = std::exp(-dm[si] - x.mu[si] + x.lng[b]);
            val *= g.psum(ii, p);
            for (int ioc = 0; ioc < t.nch[p]; ioc++)
              if (t.ch(p, ioc) != c) val *= g.csum(ioc, ii, p);
            g.pp(ii, ij, c) = val;
          }
        }
      }
    }
  if (log_domain) {
    std::vector<double> terms;
    for (int ii = 0; ii < t.nst[0]; ii++) {
      const int si = t.st(0, ii);
      double v = -(x.mu[si] + dm[si]) + psum(ii, 0);
      for (int ic = 0; ic < t.nch[0]; ic++) v += csum(ic, ii, 0);
      terms.push_back(v);
    }
    return lse(terms.data(), (int)terms.size());
  }
  double Xi = 0.0;
  for (int ii = 0; ii < t.nst[0]; ii++) {
    const int si = t.st(0, ii);
    double v = std::exp(-(x.mu[si] + dm[si])) * g.psum(ii, 0);
    for (int ic = 0; ic < t.nch[0]; ic++) v *= g.csum(ic, ii, 0);
    Xi += v;
  }
  return Xi;
}

bool all_finite(const std::vector<double>& v) {
  for (double a : v)
    if (!std::isfinite(a)) return false;
  return true;
}

// ---- functionals --------------------------------------------------------------
void mfmt_deriv(double n0, double n1, double n2, double n3, double d[4]) {
  const double om = 1.0 - n3, l1 = std::log(om), i1 = 1.0 / om, i3 = 1.0 / n3, i36 = 1.0 / (36.0 * kPiB);
  d[0] = -l1;
  d[1] = n2 * i1;
  d[2] = n1 * i1 + std::pow(n2, 2) * 3.0 * i36 * i3 * (l1 * i3 + std::pow(i1, 2));
  d[3] = (n0 * i1 + (n1 * n2) * std::pow(i1, 2) -
          (l1 * std::pow(i3, 3) * 2.0 * i36 + std::pow(i3, 2) * i1 * i36 +
           (1.0 - 3.0 * n3) * std::pow(i3, 2) * i36 * std::pow(i1, 3)) *
              std::pow(n2, 3));
}

struct Gam {
  double G, eta, H;
};

Gam gamma_msa(const double* rho, const double* sig, const double* Z, int nb, double lB) {
  const double tol = 1e-10;
  double s = 0.0;
  for (int j = 0; j < nb; j++) s += rho[j] * Z[j] * Z[j];
  const double kappa = std::sqrt(4.0 * kPiB * lB * s);
  if (kappa < tol) return {kappa / 2.0, 0.0, 2.0 / kPiB};
  double sr = 0.0, srs = 0.0, s3 = 0.0;
  for (int j = 0; j < nb; j++) {
    sr += rho[j] * sig[j];
    srs += rho[j];
    s3 += rho[j] * std::pow(sig[j], 3);
  }
  const double sig_eff = sr / srs;
  const double xx = sig_eff * std::sqrt(4.0 * kPiB * lB * s);
  double G = (std::sqrt(1.0 + 2.0 * xx) - 1.0) / (2.0 * sig_eff);
  const double term2 = 2.0 / kPiB * (1.0 - kPiB / 6.0 * s3);
  double H = 0.0, eta = 0.0;
  for (int it = 1;; it++) {
    double hs = 0.0, es = 0.0, gs = 0.0;
    for (int j = 0; j < nb; j++) hs += rho[j] * std::pow(sig[j], 3) / (1.0 + G * sig[j]);
    H = hs + term2;
    for (int j = 0; j < nb; j++) es += rho[j] * Z[j] * sig[j] / (1.0 + G * sig[j]);
    eta = es / H;
    for (int j = 0; j < nb; j++)
      gs += rho[j] * std::pow(Z[j] - eta * sig[j] * sig[j], 2) / std::pow(1.0 + G * sig[j], 2);
    const double G1 = std::sqrt(kPiB * lB * gs);
    const double Gn = 0.9 * G + 0.1 * G1;
    if (std::fabs(G1 - G) < tol || it >= 1000) {
      G = Gn;
      break;
    }
    G = Gn;
  }
  return {G, eta, H};
}

void msa_deriv(const double* rho, const double* sig, const double* Z, int nb, double lB, double* out) {
  const Gam g = gamma_msa(rho, sig, Z, nb, lB);
  double us = 0.0;
  for (int j = 0; j < nb; j++)
    us += rho[j] * sig[j] * sig[j] * ((Z[j] - g.eta * sig[j] * sig[j]) / (1.0 + g.G * sig[j]) + Z[j]);
  const double u_star = -kPiB / 6 * us;
  for (int j = 0; j < nb; j++)
    out[j] = -lB * (g.G * std::pow(Z[j], 2) / (1.0 + g.G * sig[j]) +
                    g.eta * sig[j] * ((2.0 * Z[j] - g.eta * std::pow(sig[j], 2)) / (1.0 + g.G * sig[j]) +
                                      g.eta * std::pow(sig[j], 2) / 3.0) +
                    Z[j] * u_star);
}

void tpt1msa_deriv(const sdft_bulk_system* sy, const double* bonds2, const double* rho, double* dphi, double* lng) {
  const int nb = sy->nb, mb = sy->mb;
  const double *sig = sy->diameter, *Z = sy->valence, lB = sy->bjerrum_length;
  msa_deriv(rho, sig, Z, nb, lB, dphi);
  const Gam g = gamma_msa(rho, sig, Z, nb, lB);
  const double G = g.G, eta = g.eta, H = g.H;
  if (G == 0.0) {
    for (int u = 0; u < mb; u++) {
      const int i = sy->bond_types[2 * u], j = sy->bond_types[2 * u + 1];
      lng[u] = -lB / ((sig[i] + sig[j]) / 2.0) * Z[i] * Z[j];
    }
    return;
  }
  for (int u = 0; u < mb; u++) {
    const int i = sy->bond_types[2 * u], j = sy->bond_types[2 * u + 1];
    const double sij = (sig[i] + sig[j]) / 2.0;
    const double Xi = (Z[i] - eta * std::pow(sig[i], 2)) / (1.0 + G * sig[i]);
    const double Xj = (Z[j] - eta * std::pow(sig[j], 2)) / (1.0 + G * sig[j]);
    lng[u] = -lB / sij * Xi * Xj;
  }
  double dfG = 0.0, dfe = 0.0, deG = 0.0, dHG = 0.0;
  for (int w = 0; w < nb; w++) {
    const double opg = 1.0 + G * sig[w];
    dfG += rho[w] * sig[w] * std::pow(Z[w] - eta * sig[w] * sig[w], 2) / std::pow(opg, 3);
    dfe += rho[w] * sig[w] * sig[w] * (Z[w] - eta * sig[w] * sig[w]) / std::pow(opg, 2);
    deG += rho[w] * Z[w] * sig[w] * sig[w] / std::pow(opg, 2);
    dHG += rho[w] * std::pow(sig[w], 4) / std::pow(opg, 2);
  }
  dfG = -2.0 * kPiB * lB * dfG;
  dfe = -2.0 * kPiB * lB * dfe;
  deG = -1.0 / H * deG;
  const double deH = -eta / H;
  dHG = -dHG;
  const double detaG = deG + deH * dHG;
  const double denom = 1.0 / (2.0 * G - dfe * detaG - dfG);
  for (int w = 0; w < nb; w++) {
    const double inv = 1.0 / (1.0 + G * sig[w]);
    const double Xw = (Z[w] - eta * std::pow(sig[w], 2)) * inv;
    const double dfr = kPiB * lB * std::pow(Xw, 2);
    const double der = sig[w] / H * Z[w] * inv;
    const double dHr = std::pow(sig[w], 3) * (inv - 1.0 / 3.0);
    const double dGr = (dfr + dfe * (der + dfe * deH * dHr)) * denom;
    const double detar = detaG * dGr;
    for (int u = 0; u < mb; u++) {
      const int i = sy->bond_types[2 * u], j = sy->bond_types[2 * u + 1];
      const double sij = (sig[i] + sig[j]) / 2.0;
      const double ii = 1.0 / (1.0 + G * sig[i]);
      const double Xi = (Z[i] - eta * std::pow(sig[i], 2)) * ii;
      const double dXi = -(std::pow(sig[i], 2) * ii * detar + sig[i] * Xi * ii * dGr);
      const double ij = 1.0 / (1.0 + G * sig[j]);
      const double Xj = (Z[j] - eta * std::pow(sig[j], 2)) * ij;
      const double dXj = -(std::pow(sig[j], 2) * ij * detar + sig[j] * Xj * ij * dGr);
      dphi[w] += (bonds2[u] + bonds2[mb + u]) / 2.0 * lB / sij * (dXi * Xj + Xi * dXj);
    }
  }
}

void weighted_bulk(const sdft_bulk_system* sy, const double* rho, double n[4]) {
  const double* sig = sy->diameter;
  n[0] = n[1] = n[2] = n[3] = 0.0;
  for (int j = 0; j < sy->nb; j++) {
    n[0] += rho[j];
    n[1] += rho[j] * sig[j] / 2;
    n[2] += rho[j] * kPiB * std::pow(sig[j], 2);
    n[3] += rho[j] * kPiB * std::pow(sig[j], 3) / 6;
  }
}

void tpt1mfmt_deriv(const sdft_bulk_system* sy, const double* bonds2, const double* rho, double* mu, double* lng) {
  const double* sig = sy->diameter;
  const int mb = sy->mb;
  double n[4], d[4];
  weighted_bulk(sy, rho, n);
  mfmt_deriv(n[0], n[1], n[2], n[3], d);
  const double i1 = 1.0 / (1.0 - n[3]);
  const double term2 = n[2] / 4.0 * std::pow(i1, 2);
  const double term3 = std::pow(n[2], 2) / 72.0 * std::pow(i1, 3);
  for (int u = 0; u < mb; u++) {
    const int i = sy->bond_types[2 * u], j = sy->bond_types[2 * u + 1];
    const double sij = (sig[i] + sig[j]) / 2;
    const double tau = sig[i] * sig[j] / sij;
    const double y = i1 + term2 * tau + term3 * std::pow(tau, 2);
    const double dl2 = (tau / 4.0 * std::pow(i1, 2) + n[2] * std::pow(tau, 2) * std::pow(i1, 3) / 36.0) / y;
    const double dl3 = (std::pow(i1, 2) + n[2] / 2.0 * std::pow(i1, 3) * tau +
                        std::pow(n[2], 2) / 24.0 * std::pow(i1, 4) * std::pow(tau, 2)) / y;
    d[2] -= 0.5 * (bonds2[u] + bonds2[mb + u]) * dl2;
    d[3] -= 0.5 * (bonds2[u] + bonds2[mb + u]) * dl3;
    lng[u] = std::log(y);
  }
  for (int j = 0; j < sy->nb; j++)
    mu[j] = d[0] + d[1] * sig[j] / 2 + d[2] * kPiB * std::pow(sig[j], 2) + d[3] * kPiB * std::pow(sig[j], 3) / 6;
}

Tree tree_of(const sdft_bulk_species& s) {
  Tree t;
  t.n = s.n_seg;
  t.S = s.max_states;
  t.C = s.max_children > 0 ? s.max_children : 1;
  t.nst = s.n_states;
  t.states = s.states;
  t.parent = s.parent;
  t.nch = s.n_children;
  t.children = s.children;
  t.level_ptr = s.level_ptr;
  t.level_segs = s.level_segs;
  t.n_levels = s.n_levels;
  return t;
}

}  // namespace

extern "C" int sdft_bulk_eval(const sdft_bulk_system* sy, const double* rho_species, const double* mu_ex_in,
                              const double* lng_in, double* rho_segments, double* rho_beads, double* rho_bonds,
                              double* mu_species, double* mu_ex, double* lng, double* Xi_out) {
  if (!sy || !rho_species || !mu_ex_in || !rho_beads || !mu_species || !mu_ex || !Xi_out) return SDFT_ERR_ARG;
  const int nb = sy->nb, mb = sy->mb, ns = sy->ns;
  const double* dm = sy->delta_muH;
  Ctx x{sy, mu_ex_in, lng_in};
  for (int j = 0; j < nb; j++) rho_beads[j] = 0.0;
  for (int q = 0; q < 2 * mb; q++) rho_bonds[q] = 0.0;
  std::vector<double> Xi(ns, 0.0);
  Props g;
  // ---- eval_bulk_density!
  size_t seg_off = 0;
  for (int u = 0; u < ns; u++) {
    const sdft_bulk_species& sp = sy->species[u];
    const Tree t = tree_of(sp);
    double* seg = rho_segments + seg_off;  // [S * n] as (state, segment)
    seg_off += (size_t)t.S * t.n;
    for (int q = 0; q < t.S * t.n; q++) seg[q] = 0.0;
    auto SEG = [&](int ii, int si) -> double& { return seg[(size_t)si * t.S + ii]; };
    const double rs = rho_species[u];
    if (sp.monomerbead) {
      double X = 0.0;
      for (int ii = 0; ii < t.nst[0]; ii++) X += std::exp(-mu_ex_in[t.st(0, ii)] - dm[t.st(0, ii)]);
      Xi[u] = X;
      for (int si = 0; si < t.n; si++)
        for (int ii = 0; ii < t.nst[si]; ii++) {
          const int s_i = t.st(si, ii);
          const double val = rs / X * std::exp(-mu_ex_in[s_i] - dm[s_i]);
          rho_beads[s_i] += val;
          SEG(ii, si) += val;
        }
      continue;
    }
    const double X = fj_propagators(x, t, g, false);
    if (!(std::isfinite(X) && X > 0 && all_finite(g.gC) && all_finite(g.gP) && rs > 0)) {
      if (!(rs > 0)) {
        Xi[u] = X;
        continue;
      }
      // log-domain accumulation
      const double lXi = fj_propagators(x, t, g, true);
      Xi[u] = lXi < 700 ? std::exp(lXi) : std::numeric_limits<double>::infinity();
      std::vector<double> tmp(std::max(t.S, 1)), terms;
      for (int si = 0; si < t.n; si++)
        for (int ii = 0; ii < t.nst[si]; ii++) {
          const int s_i = t.st(si, ii);
          const double lam = mu_ex_in[s_i] + dm[s_i];
          for (int q = 0; q < t.S; q++) tmp[q] = g.pp(q, ii, si);
          const double lpref = std::log(rs) - lam + lse(tmp.data(), t.S) - lXi;
          double lcc = 0.0;
          if (t.nch[si] > 0) {
            const int child = t.ch(si, 0);
            terms.clear();
            for (int ij = 0; ij < t.nst[child]; ij++) {
              double v = g.c(ij, 0, ii, si);
              for (int ioc = 0; ioc < t.nch[si]; ioc++)
                if (t.ch(si, ioc) != child) {
                  for (int q = 0; q < t.S; q++) tmp[q] = g.c(q, ioc, ii, si);
                  v += lse(tmp.data(), t.S);
                }
              terms.push_back(v);
            }
            lcc = lse(terms.data(), (int)terms.size());
          }
          const double lval = lpref + lcc;
          const double val = std::exp(lval);
          SEG(ii, si) = val;
          rho_beads[s_i] += val;
          for (int ic = 0; ic < t.nch[si]; ic++) {
            for (int q = 0; q < t.S; q++) tmp[q] = g.c(q, ic, ii, si);
            const double lQ = lse(tmp.data(), t.S);
            const int c = t.ch(si, ic);
            for (int ij = 0; ij < t.nst[c]; ij++) {
              const double f = std::exp(lval + g.c(ij, ic, ii, si) - lQ);
              const int b = x.bond(s_i, t.st(c, ij));
              rho_bonds[b] += f;
              rho_bonds[mb + b] += f;
            }
          }
        }
      continue;
    }
    Xi[u] = X;
    for (int si = 0; si < t.n; si++)
      for (int ii = 0; ii < t.nst[si]; ii++) {
        const int s_i = t.st(si, ii);
        const double lam = mu_ex_in[s_i] + dm[s_i];
        const double pref = rs * std::exp(-lam) * g.psum(ii, si) / X;
        double cc = 1.0;
        if (t.nch[si] > 0) {
          const int child = t.ch(si, 0);
          cc = 0.0;
          for (int ij = 0; ij < t.nst[child]; ij++) {
            double v = g.c(ij, 0, ii, si);
            for (int ioc = 0; ioc < t.nch[si]; ioc++)
              if (t.ch(si, ioc) != child) v *= g.csum(ioc, ii, si);
            cc += v;
          }
        }
        const double val = pref * cc;
        SEG(ii, si) = val;
        rho_beads[s_i] += val;
        for (int ic = 0; ic < t.nch[si]; ic++) {
          const double Qc = g.csum(ic, ii, si);
          const int c = t.ch(si, ic);
          for (int ij = 0; ij < t.nst[c]; ij++) {
            const double f = val * g.c(ij, ic, ii, si) / Qc;
            const int b = x.bond(s_i, t.st(c, ij));
            rho_bonds[b] += f;
            rho_bonds[mb + b] += f;
          }
        }
      }
  }
  // ---- bulk_chemical_potential
  for (int u = 0; u < ns; u++) mu_species[u] = 0.0;
  for (int j = 0; j < nb; j++) mu_ex[j] = 0.0;
  for (int q = 0; q < mb; q++) lng[q] = 0.0;
  std::vector<double> tmu(nb), tl(mb);
  if (sy->models & SDFT_BULK_IDEAL)
    for (int u = 0; u < ns; u++)
      mu_species[u] += rho_species[u] > 1e-100 ? std::log(std::fmax(rho_species[u], 1e-300)) : -1e20;
  if (sy->models & SDFT_BULK_MFMT) {
    // bulk_chemical_potential.jl's own weighted sums (n2 = rho sig sig pi, n3 = rho sig^3 pi / 6)
    double n[4] = {0.0, 0.0, 0.0, 0.0}, d[4];
    for (int j = 0; j < nb; j++) {
      const double sj = sy->diameter[j];
      n[0] += rho_beads[j];
      n[1] += rho_beads[j] * sj / 2;
      n[2] += rho_beads[j] * sj * sj * kPiB;
      n[3] += rho_beads[j] * std::pow(sj, 3) * kPiB / 6;
    }
    mfmt_deriv(n[0], n[1], n[2], n[3], d);
    const double* sig = sy->diameter;
    for (int j = 0; j < nb; j++)
      mu_ex[j] += d[0] + d[1] * sig[j] / 2 + d[2] * kPiB * std::pow(sig[j], 2) + d[3] * kPiB * std::pow(sig[j], 3) / 6;
  }
  if (sy->models & SDFT_BULK_TPT1MFMT) {
    tpt1mfmt_deriv(sy, rho_bonds, rho_beads, tmu.data(), tl.data());
    for (int j = 0; j < nb; j++) mu_ex[j] += tmu[j];
    for (int q = 0; q < mb; q++) lng[q] += tl[q];
  }
  if (sy->models & SDFT_BULK_MSA) {
    msa_deriv(rho_beads, sy->diameter, sy->valence, nb, sy->bjerrum_length, tmu.data());
    for (int j = 0; j < nb; j++) mu_ex[j] += tmu[j];
  }
  if (sy->models & SDFT_BULK_TPT1MSA) {
    tpt1msa_deriv(sy, rho_bonds, rho_beads, tmu.data(), tl.data());
    for (int j = 0; j < nb; j++) mu_ex[j] += tmu[j];
    for (int q = 0; q < mb; q++) lng[q] += tl[q];
  }
  // mu_species -= ln Xi at the new mu_ex / lng
  Ctx x2{sy, mu_ex, lng};
  for (int u = 0; u < ns; u++) {
    const sdft_bulk_species& sp = sy->species[u];
    const Tree t = tree_of(sp);
    double lxi;
    if (sp.monomerbead) {
      double X = 0.0;
      for (int ii = 0; ii < t.nst[0]; ii++) X += std::exp(-mu_ex[t.st(0, ii)] - dm[t.st(0, ii)]);
      lxi = std::log(X);
      Xi[u] = X;
    } else {
      const double X = fj_propagators(x2, t, g, false);
      if (std::isfinite(X) && X > 0) lxi = std::log(X);
      else lxi = fj_propagators(x2, t, g, true);
      Xi[u] = lxi < 700 ? std::exp(lxi) : std::numeric_limits<double>::infinity();
    }
    mu_species[u] -= lxi;
  }
  for (int u = 0; u < ns; u++) Xi_out[u] = Xi[u];
  return SDFT_OK;
}
