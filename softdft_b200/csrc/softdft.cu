// softdft.cu -- the C ABI of include/softdft.h (host side).
//
// The kernels live in kernels.cuh (built by kernels_pow2.cu and kernels_gen.cu);
// this file validates descriptors, lays out each request's device memory,
// builds the grid fields and k-space weights of setup_iDFT
// (src/iDFT/setup/setup_iDFT.jl:9-30) from the plain-C descriptor, and runs the
// single, batched and serving solves.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <new>
#include <stdexcept>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/softdft.h"
#include "common.cuh"

using namespace sdft;

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
static thread_local double g_batch_ms = 0.0;
static thread_local int g_batch_launches = 0;
static thread_local std::vector<double> g_batch_latency;

static int set_err(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
// the same record for the host-only translation units (input.cpp)
int sdft_record_error(int code, const std::string& msg) { return set_err(code, msg); }

#define CUDA_TRY(expr)                                                                 \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return set_err(SDFT_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

static int tb_for(int M);
static size_t smem_bytes(int M);

struct SpeciesHost {
  int n_seg, S, fixed;
  bool tree = false;             // branched topology
  int C = 1;                     // most children of a segment
  std::vector<int> parent, nch, child, order;
  std::vector<int> states, nst, bnd, bslot, bslot_bond, eslot, eslot_bead;
  std::vector<double> md;
  double fixed_density, mu_species, normative, norm_free;
};

namespace {

double kvec(int k, int N, double DR) {
  if (k <= N / 2) return 2.0 * kPi * (double)k / ((double)N * DR);
  return -2.0 * kPi * (double)(N - k) / ((double)N * DR);
}
double w_delta(int k, int N, double DR, double b) {  // delta_func.jl
  if (k == 0) return 4.0 * kPi * (b * b);
  double kv = kvec(k, N, DR), d = std::sqrt(kv * kv);
  return 4.0 * kPi * b * std::sin(b * d) / d;
}
double w_step(int k, int N, double DR, double b) {  // step_func.jl
  if (k == 0) return (4.0 / 3.0) * kPi * (b * b * b);
  double kv = kvec(k, N, DR), d = std::sqrt(kv * kv);
  return 4.0 * kPi * (std::sin(b * d) - b * d * std::cos(b * d)) / (d * d * d);
}
double w_vec(int k, int N, double DR, double b) {  // vectored_delta_func.jl
  if (k == 0) return 0.0;
  double kv = kvec(k, N, DR), d = std::sqrt(kv * kv);
  return -4.0 * kPi * (std::sin(b * d) - b * d * std::cos(b * d)) / (d * d * d) * kv;
}
double w_coul(int k, int N, double DR, double BJ) {  // coul_func_fft.jl
  if (k == 0) return 0.0;
  double kv = kvec(k, N, DR);
  return 2.0 * kPi * BJ / ((1.0 - std::cos(kv * DR)) / (DR * DR));
}
double filter_k(int k, int N, double dz) {  // apply_filter.jl
  double kc = 0.5 * (kPi / dz);
  int nn = k > N / 2 ? k - N : k;
  double kd = 2.0 * kPi * (double)nn / ((double)N * dz);
  double t = std::sqrt(kd * kd) / kc;
  double t2 = t * t;
  return std::exp(-(t2 * t2));
}
double2 cis(long double a) { return make_double2((double)cosl(a), (double)sinl(a)); }

// in-place forward DFT X[k] = sum_m x_m e^{-2 pi i k m / n} of a power-of-two
// length, radix-2 decimation in time in long double (host tables only)
void fft_host(std::vector<std::complex<long double>>& a) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; i++) {  // bit-reversal permutation
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  const long double pi = 3.14159265358979323846264338327950288L;
  for (size_t len = 2; len <= n; len <<= 1) {
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; k++) {
        const std::complex<long double> w = std::polar(1.0L, -2.0L * pi * (long double)k / (long double)len);
        const std::complex<long double> u = a[i + k], v = a[i + k + len / 2] * w;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
  }
}
int jround(double x) { return (int)std::nearbyint(x); }

struct Layout {
  size_t off = 0;
  template <class T>
  size_t take(size_t count) {
    size_t o = (off + 255) & ~(size_t)255;
    off = o + count * sizeof(T);
    return o;
  }
};

int bond_lookup(const std::vector<int>& bonds, int a, int b) {
  int lo = std::min(a, b), hi = std::max(a, b);
  for (size_t u = 0; u < bonds.size() / 2; u++)
    if (bonds[2 * u] == lo && bonds[2 * u + 1] == hi) return (int)u;
  return -1;
}

// Everything a request needs on the device, derived from the descriptor once:
// validated species, the byte layout of one device block and the host-built
// tables.  sdft_request_create places it in its own allocation (with Anderson
// history), sdft_objective_noalloc in the library's static scratch array.
struct Plan {
  int P = 0, M = 0, L = 0, NB = 0, MB = 0, NS = 0;
  int Pt = 0;                    // grid points; P is the stride of per-point arrays (Pt + 1 for odd Pt)
  long long n_caller = 0;        // unknowns in the caller's layout (rows of Pt points)
  bool gen = false;              // M is not a power of two: mixed-radix FFT
  std::vector<int> rad;          // general length: radices, M = their product
  std::vector<int> slot;         // general length: [M] digit-reversed slot of natural index m
  long long n = 0;
  long long hstride = 0;  // column stride of the Anderson histories (n rounded up to 32)
  bool history = false;
  std::vector<int> bonds;
  std::vector<SpeciesHost> sp;
  std::vector<int> grp;          // [NB] diameter group of each bead type
  std::vector<double> grp_sig;   // [ngrp] group diameters
  // layout
  size_t o_sig = 0, o_z = 0, o_dmu = 0, o_bonds = 0, o_grp = 0, o_grp_sig = 0, o_sp = 0;
  std::vector<size_t> o_states, o_nst, o_bnd, o_md, o_gC, o_gP, o_rho, o_expo, o_bslot, o_bslot_bond, o_eslot, o_eslot_bead;
  std::vector<size_t> o_parent, o_nch, o_child, o_order;
  size_t o_Ext = 0, o_tr = 0, o_Csurf = 0, o_Wbond = 0, o_Wfmt = 0, o_Wmsa = 0, o_Wcoul = 0, o_tw = 0, o_twP = 0, o_twD = 0;
  size_t o_tw32 = 0, o_twP32 = 0, o_twD32 = 0, o_fbe32 = 0, o_slot_tab = 0;
  int prec = SDFT_PREC_FP64;
  size_t o_x = 0, o_g = 0, o_lam = 0, o_rb = 0, o_rbo = 0, o_Cb = 0, o_Cbond = 0, o_Cmu = 0, o_Clng = 0;
  size_t o_wa = 0, o_wb = 0, o_wc = 0, o_wd = 0, o_fbe = 0, o_elam = 0;
  size_t o_hx = 0, o_hg = 0, o_u = 0;
  size_t o_status = 0, o_iters = 0, o_err = 0, o_scal = 0, o_dreq = 0, o_slot = 0, o_out = 0;
  size_t bytes = 0;
  // host tables
  std::vector<double> Ext, tr, Csurf, Wbond, Wfmt, Wmsa, Wcoul, x0;
  std::vector<double2> tw, twP, twD;
  std::vector<float2> tw32, twP32, twD32;
  // Bluestein transform: a length with a prime factor above kMaxGenRadix
  bool blue = false;
  int LB = 0, lLB = 0;   // convolution length 2^lLB >= 2M - 1
  int BL = 0;            // points of a transform buffer: M, or LB under Bluestein
  std::vector<double2> bw, bB, btw;
  std::vector<float2> bw32, bB32, btw32;
  size_t o_bw = 0, o_bB = 0, o_btw = 0, o_bw32 = 0, o_bB32 = 0, o_btw32 = 0;
};

// radices of a general-length FFT of M points (4s, then 2, 3, 5, 7 and larger
// primes up to kMaxGenRadix); false when M has a larger prime factor
static bool fft_radices(int M, std::vector<int>& rad) {
  rad.clear();
  int m = M;
  while (m % 4 == 0) {
    rad.push_back(4);
    m /= 4;
  }
  if (m % 2 == 0) {
    rad.push_back(2);
    m /= 2;
  }
  for (int p = 3; p <= kMaxGenRadix && m > 1; p += 2)
    while (m % p == 0) {
      rad.push_back(p);
      m /= p;
    }
  return m == 1 && (int)rad.size() <= kMaxRadices;
}

// slot[n] = buffer position of natural index n at the input of the
// decimation-in-time passes: n = d_0 M/r_0 + d_1 M/(r_0 r_1) + ... sits at
// d_0 + r_0 (d_1 + r_1 (d_2 + ...))
static void fft_digit_slots(int M, const std::vector<int>& rad, std::vector<int>& slot) {
  slot.assign(M, 0);
  for (int pos = 0; pos < M; pos++) {
    int p = pos, n = 0, span = M;
    for (int r : rad) {
      const int dgt = p % r;
      p /= r;
      span /= r;
      n += dgt * span;
    }
    slot[n] = pos;
  }
}

// validation of the descriptor (the device solve's supported subset) and the
// per-species host data
// grid size: even NP runs the DCT through a complex FFT of NP/2 points, odd NP
// through one of NP points on real data, with every per-point device array
// padded to the even stride NP + 1 (the pad point lies beyond the grid)
static int plan_grid(int Pt, Plan& pl) {
  if (Pt < 16) return set_err(SDFT_ERR_UNSUPPORTED, "the device solve needs NP >= 16 (got " + std::to_string(Pt) + ")");
  if (Pt > (1 << 20))  // far above the one-CTA limit below; keeps NP + 1 and the sizes in range
    return set_err(SDFT_ERR_UNSUPPORTED, "NP = " + std::to_string(Pt) + " needs more shared memory than a CTA has");
  const bool odd = (Pt & 1) != 0;
  const int P = odd ? Pt + 1 : Pt;
  const int Mf = odd ? Pt : Pt / 2;
  // a length with a prime factor above kMaxGenRadix runs Bluestein's chirp
  // convolution of length LB = 2^lLB >= 2M - 1
  pl.blue = !fft_radices(Mf, pl.rad);
  pl.LB = pl.lLB = 0;
  if (pl.blue) {
    pl.rad.clear();
    while ((1 << pl.lLB) < 2 * Mf - 1) pl.lLB++;
    pl.LB = 1 << pl.lLB;
  }
  pl.gen = pl.blue || (Mf & (Mf - 1)) != 0;
  pl.BL = pl.blue ? pl.LB : Mf;
  if (smem_bytes(pl.BL) > kMaxSmemBytes)
    return set_err(SDFT_ERR_UNSUPPORTED, "NP = " + std::to_string(Pt) + " needs more shared memory than a CTA has" +
                                             (pl.blue ? " (Bluestein transform of " + std::to_string(pl.LB) + " points)" : ""));
  pl.P = P;
  pl.Pt = Pt;
  pl.M = Mf;
  pl.L = 0;
  while ((1 << pl.L) < pl.M) pl.L++;
  return SDFT_OK;
}

int plan_species(const sdft_system_desc* d, Plan& pl) {
  int rc = plan_grid(d->np, pl);
  if (rc) return rc;
  const int P = pl.P, Pt = pl.Pt;
  if (d->nb < 1 || d->nb > kMaxBeads) return set_err(SDFT_ERR_UNSUPPORTED, "bead types must be in [1, 32]");
  if (d->mb < 0 || d->mb > kMaxBonds) return set_err(SDFT_ERR_UNSUPPORTED, "bond types must be in [0, 64]");
  if (d->n_species < 1 || d->n_species > 16) return set_err(SDFT_ERR_UNSUPPORTED, "species must be in [1, 16]");
  if (!(d->bin_width > 0) || !std::isfinite(d->bin_width)) return set_err(SDFT_ERR_ARG, "bin_width must be positive and finite");
  if (!std::isfinite(d->length)) return set_err(SDFT_ERR_ARG, "length must be finite");
  if (d->functionals & ~0xFu) return set_err(SDFT_ERR_ARG, "unknown functional bits");
  for (int j = 0; j < d->nb; j++)
    if (!std::isfinite(d->diameter[j])) return set_err(SDFT_ERR_ARG, "bead diameters must be finite");
  for (int u = 0; u < 2 * d->mb; u++)  // the wall and bond tables index diameters by these
    if (d->bond_types[u] < 0 || d->bond_types[u] >= d->nb) return set_err(SDFT_ERR_ARG, "bond_types entry out of range");
  pl.NB = d->nb;
  pl.MB = d->mb;
  pl.NS = d->n_species;
  pl.n = (long long)P * (pl.NB + 2 * pl.MB + 1) + 1;
  pl.hstride = (pl.n + 31) / 32 * 32;
  pl.n_caller = (long long)Pt * (pl.NB + 2 * pl.MB + 1) + 1;
  pl.bonds.assign(d->bond_types, d->bond_types + 2 * pl.MB);
  const int NB = pl.NB;
  for (int u = 0; u < pl.NS; u++) {
    const sdft_species_desc& s = d->species[u];
    SpeciesHost h;
    h.n_seg = s.n_seg;
    h.S = s.max_states;
    if (h.n_seg < 1 || h.S < 1 || h.S > kMaxStates)
      return set_err(SDFT_ERR_UNSUPPORTED, "segments >= 1 and 1 <= states <= 4 per segment are required");
    for (int g = 0; g < h.n_seg; g++) {
      if ((g == 0) != (s.parent[g] < 0) || s.parent[g] >= g)
        return set_err(SDFT_ERR_ARG, "segment 0 must be the root and parents must precede their children");
      if (s.parent[g] != g - 1) h.tree = true;
      if (s.n_states[g] < 1 || s.n_states[g] > h.S) return set_err(SDFT_ERR_ARG, "n_states out of range");
    }
    h.parent.assign(s.parent, s.parent + h.n_seg);
    h.nch.assign(h.n_seg, 0);
    for (int g = 1; g < h.n_seg; g++) h.nch[h.parent[g]]++;
    h.C = 1;
    for (int g = 0; g < h.n_seg; g++) h.C = std::max(h.C, h.nch[g]);
    h.child.assign((size_t)h.n_seg * h.C, -1);
    {
      std::vector<int> cnt(h.n_seg, 0), depth(h.n_seg, 0);
      for (int g = 1; g < h.n_seg; g++) {
        h.child[(size_t)h.parent[g] * h.C + cnt[h.parent[g]]++] = g;
        depth[g] = depth[h.parent[g]] + 1;
      }
      // levels by depth from the root, ascending segment index within a level (parse_topology.jl:41-44)
      h.order.clear();
      const int maxd = *std::max_element(depth.begin(), depth.end());
      for (int l = 0; l <= maxd; l++)
        for (int g = 0; g < h.n_seg; g++)
          if (depth[g] == l) h.order.push_back(g);
    }
    h.nst.assign(s.n_states, s.n_states + h.n_seg);
    h.states.assign(s.states, s.states + (size_t)h.n_seg * h.S);
    h.fixed = -1;
    if (s.fixed_coord) {
      for (int g = 1; g < h.n_seg; g++)
        if (s.fixed_coord[g] >= 0) return set_err(SDFT_ERR_UNSUPPORTED, "only segment 0 can be fixed in a 1D slit");
      h.fixed = s.fixed_coord[0];
    }
    if (h.fixed >= 0) {
      if (h.fixed >= Pt || h.n_seg < 2 || !s.max_distance)
        return set_err(SDFT_ERR_ARG, "fixed segment needs a grid point, a free segment and max_distance");
      if (h.n_seg == 2 && h.nst[1] > 1) return set_err(SDFT_ERR_UNSUPPORTED, "grafted dimer with a multi-state free segment");
      h.md.resize(h.n_seg);
      for (int g = 0; g < h.n_seg; g++) h.md[g] = s.max_distance[(size_t)g * h.n_seg + 0];
    } else {
      h.md.assign(h.n_seg, 0.0);
    }
    for (int g = 0; g < h.n_seg; g++)
      for (int i = 0; i < h.nst[g]; i++) {
        int st = h.states[(size_t)g * h.S + i];
        if (st < 0 || st >= NB) return set_err(SDFT_ERR_ARG, "state bead type out of range");
        if (g > 0)
          for (int j = 0; j < h.nst[h.parent[g]]; j++)
            if (bond_lookup(pl.bonds, st, h.states[(size_t)h.parent[g] * h.S + j]) < 0)
              return set_err(SDFT_ERR_ARG, "bond missing from bond_types");
      }
    if (h.tree) {
      // the reference reads gC[p][oc][idx_j] for the other children of p and, for
      // a grafted species whose first free segment is a leaf, gC[1][0][idx_i]:
      // trees for which these leave the arrays fail there, and are refused here
      for (int g = 0; g < h.n_seg; g++)
        if (h.nch[g] >= 2 && (h.nch[g] > h.S || h.nst[g] > h.C))
          return set_err(SDFT_ERR_UNSUPPORTED, "branched topology index out of range (children or states of a branch point)");
      if (h.fixed >= 0 && h.nch[1] == 0 && h.nst[1] > h.C)
        return set_err(SDFT_ERR_UNSUPPORTED, "branched topology index out of range (leaf next to the graft)");
    }
    // bond type between state i of segment g and state j of segment g + 1 (linear chains)
    h.bnd.assign((size_t)h.n_seg * h.S * h.S, -1);
    for (int g = 0; !h.tree && g + 1 < h.n_seg; g++)
      for (int i = 0; i < h.nst[g]; i++)
        for (int j = 0; j < h.nst[g + 1]; j++)
          h.bnd[((size_t)g * h.S + i) * h.S + j] =
              bond_lookup(pl.bonds, h.states[(size_t)g * h.S + i], h.states[(size_t)(g + 1) * h.S + j]);
    // species-local slots of the bond types and bead types the species touches
    h.bslot.assign(h.bnd.size(), -1);
    for (size_t q = 0; q < h.bnd.size(); q++) {
      if (h.bnd[q] < 0) continue;
      int slot = -1;
      for (size_t t = 0; t < h.bslot_bond.size(); t++)
        if (h.bslot_bond[t] == h.bnd[q]) slot = (int)t;
      if (slot < 0) {
        slot = (int)h.bslot_bond.size();
        h.bslot_bond.push_back(h.bnd[q]);
      }
      h.bslot[q] = slot;
    }
    h.eslot.assign(h.states.size(), -1);
    for (int g = 0; g < h.n_seg; g++)
      for (int i = 0; i < h.nst[g]; i++) {
        const int b = h.states[(size_t)g * h.S + i];
        int slot = -1;
        for (size_t t = 0; t < h.eslot_bead.size(); t++)
          if (h.eslot_bead[t] == b) slot = (int)t;
        if (slot < 0) {
          slot = (int)h.eslot_bead.size();
          h.eslot_bead.push_back(b);
        }
        h.eslot[(size_t)g * h.S + i] = slot;
      }
    h.fixed_density = s.fixed_density;
    h.mu_species = s.mu_species;
    // normative (child_propagators.jl:41-50): levels are visited leaves first
    double nv = 1.0;
    for (int g = h.n_seg - 1; g >= 0; g--) {
      double t = 0.0;
      for (int i = 0; i < h.nst[g]; i++) t += std::exp(-d->delta_muH[h.states[(size_t)g * h.S + i]]);
      nv *= std::pow(t, 1.0 / (double)h.n_seg);
    }
    h.normative = nv;
    h.norm_free = std::pow(nv, (double)(h.n_seg - 1));
    pl.sp.push_back(h);
  }
  // bead types of equal diameter share the MSA screening sums
  pl.grp.assign(NB, 0);
  pl.grp_sig.clear();
  for (int j = 0; j < NB; j++) {
    int g = -1;
    for (size_t q = 0; q < pl.grp_sig.size(); q++)
      if (pl.grp_sig[q] == d->diameter[j]) g = (int)q;
    if (g < 0) {
      g = (int)pl.grp_sig.size();
      pl.grp_sig.push_back(d->diameter[j]);
    }
    pl.grp[j] = g;
  }
  return SDFT_OK;
}

void plan_layout(Plan& pl, bool history) {
  const int P = pl.P, NB = pl.NB, MB = pl.MB, NS = pl.NS, M = pl.M;
  pl.history = history;
  const int nwa = std::max(NB, 6), nwc = std::max(NB + MB, 6 + MB);
  Layout lay;
  pl.o_sig = lay.take<double>(NB);
  pl.o_z = lay.take<double>(NB);
  pl.o_dmu = lay.take<double>(NB);
  pl.o_bonds = lay.take<int>(2 * MB + 2);
  pl.o_grp = lay.take<int>(NB);
  pl.o_grp_sig = lay.take<double>(NB);
  pl.o_sp = lay.take<DSpecies>(NS);
  pl.o_states.resize(NS);
  pl.o_nst.resize(NS);
  pl.o_bnd.resize(NS);
  pl.o_md.resize(NS);
  pl.o_gC.resize(NS);
  pl.o_gP.resize(NS);
  pl.o_rho.resize(NS);
  pl.o_expo.resize(NS);
  pl.o_bslot.resize(NS);
  pl.o_bslot_bond.resize(NS);
  pl.o_eslot.resize(NS);
  pl.o_eslot_bead.resize(NS);
  pl.o_parent.resize(NS);
  pl.o_nch.resize(NS);
  pl.o_child.resize(NS);
  pl.o_order.resize(NS);
  for (int u = 0; u < NS; u++) {
    const SpeciesHost& h = pl.sp[u];
    pl.o_states[u] = lay.take<int>(h.states.size());
    pl.o_nst[u] = lay.take<int>(h.nst.size());
    pl.o_bnd[u] = lay.take<int>(h.bnd.size());
    pl.o_md[u] = lay.take<double>(h.md.size());
    size_t gsz = h.n_seg > 1 ? (size_t)h.n_seg * h.S * h.S * P : 0;
    pl.o_gC[u] = lay.take<double>(gsz * (size_t)h.C);
    pl.o_gP[u] = lay.take<double>(gsz);
    pl.o_parent[u] = lay.take<int>(h.parent.size());
    pl.o_nch[u] = lay.take<int>(h.nch.size());
    pl.o_child[u] = lay.take<int>(h.child.size());
    pl.o_order[u] = lay.take<int>(h.order.size());
    pl.o_rho[u] = lay.take<double>((size_t)h.n_seg * h.S * P);
    pl.o_expo[u] = lay.take<int>((size_t)2 * h.n_seg);
    pl.o_bslot[u] = lay.take<int>(h.bslot.size());
    pl.o_bslot_bond[u] = lay.take<int>(h.bslot_bond.size() + 1);
    pl.o_eslot[u] = lay.take<int>(h.eslot.size());
    pl.o_eslot_bead[u] = lay.take<int>(h.eslot_bead.size() + 1);
  }
  pl.o_Ext = lay.take<double>((size_t)NB * P);
  pl.o_tr = lay.take<double>((size_t)NB * P);
  pl.o_Csurf = lay.take<double>(P);
  pl.o_Wbond = lay.take<double>((size_t)MB * P + 1);
  pl.o_Wfmt = lay.take<double>((size_t)NB * 3 * P);
  pl.o_Wmsa = lay.take<double>((size_t)NB * P);
  pl.o_Wcoul = lay.take<double>(P);
  const size_t ntw = pl.gen ? (size_t)M : (size_t)(M / 2 + 1);
  pl.o_tw = lay.take<double2>(ntw);
  pl.o_slot_tab = pl.gen ? lay.take<int>(M) : 0;
  pl.o_twP = lay.take<double2>(M + 1);
  pl.o_twD = lay.take<double2>(M + 1);
  if (pl.blue) {
    pl.o_bw = lay.take<double2>(M);
    pl.o_bB = lay.take<double2>(pl.LB);
    pl.o_btw = lay.take<double2>(pl.LB / 2 + 1);
    if (pl.prec == SDFT_PREC_MIXED) {
      pl.o_bw32 = lay.take<float2>(M);
      pl.o_bB32 = lay.take<float2>(pl.LB);
      pl.o_btw32 = lay.take<float2>(pl.LB / 2 + 1);
    }
  }
  if (pl.prec == SDFT_PREC_MIXED) {
    pl.o_tw32 = lay.take<float2>(ntw);
    pl.o_twP32 = lay.take<float2>(M + 1);
    pl.o_twD32 = lay.take<float2>(M + 1);
    pl.o_fbe32 = lay.take<float>((size_t)4 * MB * P + 1);
  }
  if (history) {
    pl.o_x = lay.take<double>(pl.n);
    pl.o_g = lay.take<double>(pl.n);
  }
  pl.o_lam = lay.take<double>((size_t)NB * P);
  pl.o_rb = lay.take<double>((size_t)NB * P);
  pl.o_rbo = lay.take<double>((size_t)MB * 2 * P + 1);
  pl.o_Cb = lay.take<double>((size_t)NB * P);
  pl.o_Cbond = lay.take<double>((size_t)MB * 2 * P + 1);
  pl.o_Cmu = lay.take<double>((size_t)NB * P);
  pl.o_Clng = lay.take<double>((size_t)MB * 2 * P + 1);
  pl.o_wa = lay.take<double>((size_t)nwa * P);
  pl.o_wb = lay.take<double>((size_t)MB * 2 * P + 1);
  pl.o_wc = lay.take<double>((size_t)nwc * P);
  pl.o_wd = lay.take<double>((size_t)2 * NB * P);
  pl.o_fbe = lay.take<double>((size_t)4 * MB * P + 1);
  pl.o_elam = lay.take<double>((size_t)NB * P);
  if (history) {
    pl.o_hx = lay.take<double>((size_t)kMaxAnderson * pl.hstride);
    pl.o_hg = lay.take<double>((size_t)kMaxAnderson * pl.hstride);
    pl.o_u = lay.take<double>(pl.n);
  }
  pl.o_status = lay.take<int>(4);
  pl.o_iters = lay.take<int>(4);
  pl.o_err = lay.take<double>(4);
  pl.o_scal = lay.take<double>(8);
  pl.o_dreq = lay.take<DReq>(1);
  if (history) {
    pl.o_slot = lay.take<SolveSlot>(1);
    pl.o_out = lay.take<double>(1 + NS);
  }
  pl.bytes = lay.off;
}

void plan_tables(const sdft_system_desc* d, Plan& pl) {
  const int P = pl.P, Pt = pl.Pt, NB = pl.NB, MB = pl.MB, M = pl.M, NPS = 2 * Pt;
  pl.Ext.assign((size_t)NB * P, 0.0);
  pl.tr.assign((size_t)NB * P, 1.0);
  if (P != Pt)  // the pad point of odd grids: excluded and unweighted
    for (int j = 0; j < NB; j++) {
      pl.Ext[(size_t)j * P + Pt] = 1.0e20;
      pl.tr[(size_t)j * P + Pt] = 0.0;
    }
  if (d->hard_walls) {  // hard_walls.jl:6-46
    for (int K = 0; K < Pt; K++) {
      int idx = K + 1;
      for (int j = 0; j < NB; j++) {
        double dd = d->diameter[j];
        int lo = jround((0.0 + dd / 2.0) / d->bin_width) + 1;
        int hi = jround((d->length - dd / 2.0) / d->bin_width) + 1;
        size_t qq = (size_t)j * P + K;
        if (idx < lo) {
          pl.Ext[qq] += 1.0e20;
          pl.tr[qq] = 1.0;
        } else if (idx == lo) {
          pl.tr[qq] = 0.5;
        }
        if (idx > hi) {
          pl.Ext[qq] += 1.0e20;
          pl.tr[qq] = 1.0;
        } else if (idx == hi) {
          pl.tr[qq] = 0.5;
        }
      }
    }
  }
  std::vector<double> surf(Pt, 0.0);
  pl.Csurf.assign(P, 0.0);
  if (d->charged_walls) {  // charged_walls.jl:7-57
    double pos[2] = {0.0, d->length};
    for (int w = 0; w < 2; w++) {
      int gp = jround(pos[w] / d->bin_width) + 1;
      if (gp >= 1 && gp <= Pt) surf[gp - 1] += d->wall_charge[w] * (1.0 / d->bin_width);
    }
    for (int k = 0; k < Pt; k++) {
      long double acc = 0.0L;
      for (int K = 0; K < Pt; K++)
        if (surf[K] != 0.0) acc += (long double)surf[K] * cosl(3.14159265358979323846264338327950288L * k * (2 * K + 1) / (2.0L * Pt));
      pl.Csurf[k] = (double)acc;
    }
  }
  pl.Wbond.assign((size_t)MB * P + 1, 0.0);
  pl.Wfmt.assign((size_t)NB * 3 * P, 0.0);
  pl.Wmsa.assign((size_t)NB * P, 0.0);
  pl.Wcoul.assign(P, 0.0);
  for (int u = 0; u < MB; u++) {
    double sij = (d->diameter[pl.bonds[2 * u]] + d->diameter[pl.bonds[2 * u + 1]]) / 2.0;
    for (int k = 0; k < Pt; k++)
      pl.Wbond[(size_t)u * P + k] = filter_k(k, NPS, d->bin_width) * (w_delta(k, NPS, d->bin_width, sij) / (4.0 * kPi * (sij * sij)));
  }
  for (int j = 0; j < NB; j++) {
    double b = d->diameter[j] / 2.0;
    for (int k = 0; k < Pt; k++) {
      pl.Wfmt[((size_t)j * 3 + 0) * P + k] = w_delta(k, NPS, d->bin_width, b);
      pl.Wfmt[((size_t)j * 3 + 1) * P + k] = w_step(k, NPS, d->bin_width, b);
      pl.Wfmt[((size_t)j * 3 + 2) * P + k] = w_vec(k, NPS, d->bin_width, b);
      pl.Wmsa[(size_t)j * P + k] = w_delta(k, NPS, d->bin_width, b) / (4.0 * kPi * (b * b));
    }
  }
  for (int k = 0; k < Pt; k++) pl.Wcoul[k] = w_coul(k, NPS, d->bin_width, d->bjerrum_length);
  const long double PI_L = 3.14159265358979323846264338327950288L;
  pl.tw.resize(pl.gen ? M : M / 2 + 1);
  pl.twP.resize(M + 1);
  pl.twD.resize(M + 1);
  for (size_t k = 0; k < pl.tw.size(); k++) pl.tw[k] = cis(-2.0L * PI_L * (long double)k / M);
  if (pl.blue) {  // natural order in and out; the chirp tables
    pl.slot.resize(M);
    for (int m = 0; m < M; m++) pl.slot[m] = m;
    const int LB = pl.LB;
    pl.bw.resize(M);
    for (int m = 0; m < M; m++) {
      const long long q = ((long long)m * m) % (2LL * M);  // e^{-i pi m^2 / M} with the argument reduced mod 2 pi
      pl.bw[m] = cis(-PI_L * (long double)q / M);
    }
    // filter b[m] = conj(w_m) for |m| < M on the cyclic grid of LB points, and its DFT
    std::vector<std::complex<long double>> b(LB, 0.0L);
    for (int m = 0; m < M; m++) {
      const long long q = ((long long)m * m) % (2LL * M);
      const std::complex<long double> v = std::polar(1.0L, PI_L * (long double)q / M);
      b[m] = v;
      if (m) b[LB - m] = v;
    }
    fft_host(b);
    pl.bB.resize(LB);
    for (int j = 0; j < LB; j++) {
      int k = 0;
      for (int bit = 0; bit < pl.lLB; bit++) k |= ((j >> bit) & 1) << (pl.lLB - 1 - bit);
      const std::complex<long double> v = b[k] / (long double)LB;
      pl.bB[j] = make_double2((double)v.real(), (double)v.imag());
    }
    pl.btw.resize(LB / 2 + 1);
    for (int k = 0; k <= LB / 2; k++) pl.btw[k] = cis(-2.0L * PI_L * k / LB);
  } else if (pl.gen) {
    fft_digit_slots(M, pl.rad, pl.slot);
  }
  for (int k = 0; k <= M; k++) pl.twP[k] = cis(-2.0L * PI_L * k / Pt);
  for (int k = 0; k <= M; k++) pl.twD[k] = cis(-PI_L * k / (2.0L * Pt));
  if (pl.prec == SDFT_PREC_MIXED) {
    auto f2 = [](double2 v) { return make_float2((float)v.x, (float)v.y); };
    pl.tw32.resize(pl.tw.size());
    pl.twP32.resize(pl.twP.size());
    pl.twD32.resize(pl.twD.size());
    for (size_t k = 0; k < pl.tw.size(); k++) pl.tw32[k] = f2(pl.tw[k]);
    for (size_t k = 0; k < pl.twP.size(); k++) pl.twP32[k] = f2(pl.twP[k]);
    for (size_t k = 0; k < pl.twD.size(); k++) pl.twD32[k] = f2(pl.twD[k]);
    if (pl.blue) {
      pl.bw32.resize(pl.bw.size());
      pl.bB32.resize(pl.bB.size());
      pl.btw32.resize(pl.btw.size());
      for (size_t k = 0; k < pl.bw.size(); k++) pl.bw32[k] = f2(pl.bw[k]);
      for (size_t k = 0; k < pl.bB.size(); k++) pl.bB32[k] = f2(pl.bB[k]);
      for (size_t k = 0; k < pl.btw.size(); k++) pl.btw32[k] = f2(pl.btw[k]);
    }
  }
  if (pl.history) {
    pl.x0.assign(pl.n, 0.0);
    for (int j = 0; j < NB; j++)
      for (int K = 0; K < Pt; K++) pl.x0[(size_t)j * P + K] = d->mu_ex_bulk[j];
    for (int u = 0; u < MB; u++)
      for (int e2 = 0; e2 < 2; e2++)
        for (int K = 0; K < Pt; K++) pl.x0[(size_t)P * NB + (size_t)(u * 2 + e2) * P + K] = d->lng_bulk[u];
  }
}

// device descriptor of a plan placed at `base`; x and g given for the no-alloc form
DReq plan_bind(const sdft_system_desc* d, const Plan& pl, char* base, double* x, double* g, std::vector<DSpecies>& dsp) {
  auto at = [&](size_t o) { return (void*)(base + o); };
  dsp.assign(pl.NS, DSpecies{});
  for (int u = 0; u < pl.NS; u++) {
    const SpeciesHost& h = pl.sp[u];
    DSpecies& s = dsp[u];
    s.n_seg = h.n_seg;
    s.S = h.S;
    s.fixed = h.fixed;
    s.states = (const int*)at(pl.o_states[u]);
    s.nst = (const int*)at(pl.o_nst[u]);
    s.bnd = (const int*)at(pl.o_bnd[u]);
    s.md = (const double*)at(pl.o_md[u]);
    s.fixed_density = h.fixed_density;
    s.mu_species = h.mu_species;
    s.normative = h.normative;
    s.norm_free = h.norm_free;
    s.lambda_fixed = 1.0;
    s.gC = h.n_seg > 1 ? (double*)at(pl.o_gC[u]) : nullptr;
    s.gP = h.n_seg > 1 ? (double*)at(pl.o_gP[u]) : nullptr;
    s.rho_seg = (double*)at(pl.o_rho[u]);
    s.expo = (int*)at(pl.o_expo[u]);
    s.bslot = (const int*)at(pl.o_bslot[u]);
    s.bslot_bond = (const int*)at(pl.o_bslot_bond[u]);
    s.eslot = (const int*)at(pl.o_eslot[u]);
    s.eslot_bead = (const int*)at(pl.o_eslot_bead[u]);
    s.nbslot = (int)h.bslot_bond.size();
    s.neslot = (int)h.eslot_bead.size();
    s.tree = h.tree ? 1 : 0;
    s.C = h.C;
    s.parent = (const int*)at(pl.o_parent[u]);
    s.nch = (const int*)at(pl.o_nch[u]);
    s.child = (const int*)at(pl.o_child[u]);
    s.order = (const int*)at(pl.o_order[u]);
  }
  DReq r{};
  r.NP = pl.P;
  r.NPt = pl.Pt;
  r.M = pl.M;
  r.L = pl.L;
  r.NB = pl.NB;
  r.MB = pl.MB;
  r.NS = pl.NS;
  r.funcs = (int)d->functionals;
  // odd grids pack two real transforms into each buffer
  r.TB = pl.P != pl.Pt ? std::min(kMaxTB, 2 * tb_for(pl.BL)) : tb_for(pl.BL);
  r.ngrp = (int)pl.grp_sig.size();
  r.prec = pl.prec;
  r.dz = d->bin_width;
  r.lB = d->bjerrum_length;
  r.total_charge = d->charged_walls ? d->wall_charge[0] + d->wall_charge[1] : 0.0;
  r.n = pl.n;
  r.hstride = pl.hstride;
  r.zbytes = (long long)(smem_bytes(pl.BL) - sizeof(double) * kRedDoubles);
  r.sig = (const double*)at(pl.o_sig);
  r.z = (const double*)at(pl.o_z);
  r.dmu = (const double*)at(pl.o_dmu);
  r.bonds = (const int*)at(pl.o_bonds);
  r.grp = (const int*)at(pl.o_grp);
  r.grp_sig = (const double*)at(pl.o_grp_sig);
  r.sp = (const DSpecies*)at(pl.o_sp);
  r.Ext = (const double*)at(pl.o_Ext);
  r.trapez = (const double*)at(pl.o_tr);
  r.Csurf = (const double*)at(pl.o_Csurf);
  r.Wbond = (const double*)at(pl.o_Wbond);
  r.Wfmt = (const double*)at(pl.o_Wfmt);
  r.Wmsa = (const double*)at(pl.o_Wmsa);
  r.Wcoul = (const double*)at(pl.o_Wcoul);
  r.tw = (const double2*)at(pl.o_tw);
  r.gen = pl.gen ? 1 : 0;
  r.has_tree = 0;
  for (const SpeciesHost& h : pl.sp) r.has_tree |= h.tree ? 1 : 0;
  r.nrad = pl.gen ? (int)pl.rad.size() : 0;
  for (int i = 0; i < r.nrad; i++) r.rad[i] = pl.rad[i];
  r.slot = pl.gen ? (const int*)at(pl.o_slot_tab) : nullptr;
  r.blue = pl.blue ? 1 : 0;
  r.LB = pl.LB;
  r.lLB = pl.lLB;
  r.bw = pl.blue ? (const double2*)at(pl.o_bw) : nullptr;
  r.bB = pl.blue ? (const double2*)at(pl.o_bB) : nullptr;
  r.btw = pl.blue ? (const double2*)at(pl.o_btw) : nullptr;
  r.bw32 = pl.blue && pl.o_bw32 ? (const float2*)at(pl.o_bw32) : nullptr;
  r.bB32 = pl.blue && pl.o_bB32 ? (const float2*)at(pl.o_bB32) : nullptr;
  r.btw32 = pl.blue && pl.o_btw32 ? (const float2*)at(pl.o_btw32) : nullptr;
  r.twP = (const double2*)at(pl.o_twP);
  r.twD = (const double2*)at(pl.o_twD);
  const bool mixed = pl.prec == SDFT_PREC_MIXED;
  r.tw32 = mixed ? (const float2*)at(pl.o_tw32) : nullptr;
  r.twP32 = mixed ? (const float2*)at(pl.o_twP32) : nullptr;
  r.twD32 = mixed ? (const float2*)at(pl.o_twD32) : nullptr;
  r.fbe32 = mixed ? (float*)at(pl.o_fbe32) : nullptr;
  r.x = pl.history ? (double*)at(pl.o_x) : x;
  r.g = pl.history ? (double*)at(pl.o_g) : g;
  r.lambda = (double*)at(pl.o_lam);
  r.rho_beads = (double*)at(pl.o_rb);
  r.rho_bonds = (double*)at(pl.o_rbo);
  r.Cb = (double*)at(pl.o_Cb);
  r.Cbond = (double*)at(pl.o_Cbond);
  r.Cmu = (double*)at(pl.o_Cmu);
  r.Clng = (double*)at(pl.o_Clng);
  r.wa = (double*)at(pl.o_wa);
  r.wb = (double*)at(pl.o_wb);
  r.wc = (double*)at(pl.o_wc);
  r.wd = (double*)at(pl.o_wd);
  r.fbe = (double*)at(pl.o_fbe);
  r.elam = (double*)at(pl.o_elam);
  r.hx = pl.history ? (double*)at(pl.o_hx) : nullptr;
  r.hg = pl.history ? (double*)at(pl.o_hg) : nullptr;
  r.lsq_u = pl.history ? (double*)at(pl.o_u) : nullptr;
  r.status = (int*)at(pl.o_status);
  r.iters = (int*)at(pl.o_iters);
  r.err = (double*)at(pl.o_err);
  r.scal = (double*)at(pl.o_scal);
  return r;
}

// copies the tables and the descriptor of a bound plan; stream-ordered
cudaError_t plan_upload(const sdft_system_desc* d, const Plan& pl, char* base, const DReq& r,
                        const std::vector<DSpecies>& dsp, cudaStream_t stream) {
  const int NB = pl.NB, MB = pl.MB, P = pl.P;
  cudaError_t ce = cudaSuccess;
  auto up = [&](size_t o, const void* src, size_t nbytes) {
    if (ce == cudaSuccess && nbytes) ce = cudaMemcpyAsync(base + o, src, nbytes, cudaMemcpyHostToDevice, stream);
  };
  up(pl.o_sig, d->diameter, sizeof(double) * NB);
  up(pl.o_z, d->valence, sizeof(double) * NB);
  up(pl.o_dmu, d->delta_muH, sizeof(double) * NB);
  up(pl.o_bonds, pl.bonds.data(), sizeof(int) * 2 * MB);
  up(pl.o_grp, pl.grp.data(), sizeof(int) * NB);
  up(pl.o_grp_sig, pl.grp_sig.data(), sizeof(double) * pl.grp_sig.size());
  for (int u = 0; u < pl.NS; u++) {
    const SpeciesHost& h = pl.sp[u];
    up(pl.o_states[u], h.states.data(), sizeof(int) * h.states.size());
    up(pl.o_nst[u], h.nst.data(), sizeof(int) * h.nst.size());
    up(pl.o_bnd[u], h.bnd.data(), sizeof(int) * h.bnd.size());
    up(pl.o_md[u], h.md.data(), sizeof(double) * h.md.size());
    up(pl.o_parent[u], h.parent.data(), sizeof(int) * h.parent.size());
    up(pl.o_nch[u], h.nch.data(), sizeof(int) * h.nch.size());
    up(pl.o_child[u], h.child.data(), sizeof(int) * h.child.size());
    up(pl.o_order[u], h.order.data(), sizeof(int) * h.order.size());
    up(pl.o_bslot[u], h.bslot.data(), sizeof(int) * h.bslot.size());
    up(pl.o_bslot_bond[u], h.bslot_bond.data(), sizeof(int) * h.bslot_bond.size());
    up(pl.o_eslot[u], h.eslot.data(), sizeof(int) * h.eslot.size());
    up(pl.o_eslot_bead[u], h.eslot_bead.data(), sizeof(int) * h.eslot_bead.size());
  }
  up(pl.o_sp, dsp.data(), sizeof(DSpecies) * pl.NS);
  up(pl.o_Ext, pl.Ext.data(), sizeof(double) * pl.Ext.size());
  up(pl.o_tr, pl.tr.data(), sizeof(double) * pl.tr.size());
  up(pl.o_Csurf, pl.Csurf.data(), sizeof(double) * P);
  up(pl.o_Wbond, pl.Wbond.data(), sizeof(double) * pl.Wbond.size());
  up(pl.o_Wfmt, pl.Wfmt.data(), sizeof(double) * pl.Wfmt.size());
  up(pl.o_Wmsa, pl.Wmsa.data(), sizeof(double) * pl.Wmsa.size());
  up(pl.o_Wcoul, pl.Wcoul.data(), sizeof(double) * P);
  up(pl.o_tw, pl.tw.data(), sizeof(double2) * pl.tw.size());
  if (pl.gen) up(pl.o_slot_tab, pl.slot.data(), sizeof(int) * pl.slot.size());
  if (pl.blue) {
    up(pl.o_bw, pl.bw.data(), sizeof(double2) * pl.bw.size());
    up(pl.o_bB, pl.bB.data(), sizeof(double2) * pl.bB.size());
    up(pl.o_btw, pl.btw.data(), sizeof(double2) * pl.btw.size());
    if (pl.o_bw32) {
      up(pl.o_bw32, pl.bw32.data(), sizeof(float2) * pl.bw32.size());
      up(pl.o_bB32, pl.bB32.data(), sizeof(float2) * pl.bB32.size());
      up(pl.o_btw32, pl.btw32.data(), sizeof(float2) * pl.btw32.size());
    }
  }
  up(pl.o_twP, pl.twP.data(), sizeof(double2) * pl.twP.size());
  up(pl.o_twD, pl.twD.data(), sizeof(double2) * pl.twD.size());
  if (pl.prec == SDFT_PREC_MIXED) {
    up(pl.o_tw32, pl.tw32.data(), sizeof(float2) * pl.tw32.size());
    up(pl.o_twP32, pl.twP32.data(), sizeof(float2) * pl.twP32.size());
    up(pl.o_twD32, pl.twD32.data(), sizeof(float2) * pl.twD32.size());
  }
  if (pl.history) up(pl.o_x, pl.x0.data(), sizeof(double) * pl.n);
  up(pl.o_dreq, &r, sizeof(DReq));
  return ce;
}

}  // namespace

// ---- device blocks of destroyed requests ----
// Kept for later requests instead of going back through cudaFree, which
// synchronises the whole device (a server that retires and admits requests at
// every step would stall the GPU once per request); cudaMalloc can synchronise
// too.  Keyed by device; a request takes the smallest cached block that holds it
// with at most a quarter to spare.
namespace {
struct BlockCache {
  std::mutex mu;
  std::map<int, std::multimap<size_t, char*>> blocks;  // device -> (bytes, block)
};
BlockCache& block_cache() {
  static BlockCache c;
  return c;
}
bool block_fits(size_t have, size_t need) { return have >= need && have - need <= need / 4; }
// a cached block of dev for need bytes (its size in *got), or nullptr; take=false only looks
char* cache_find(int dev, size_t need, size_t* got, bool take) {
  BlockCache& c = block_cache();
  std::lock_guard<std::mutex> g(c.mu);
  auto& m = c.blocks[dev];
  auto it = m.lower_bound(need);
  if (it == m.end() || !block_fits(it->first, need)) return nullptr;
  char* p = it->second;
  if (got) *got = it->first;
  if (take) m.erase(it);
  return p;
}
void cache_put(int dev, char* p, size_t bytes) {
  BlockCache& c = block_cache();
  std::lock_guard<std::mutex> g(c.mu);
  c.blocks[dev].emplace(bytes, p);
}
// frees the cached blocks of dev (the current device); returns their bytes
size_t cache_release(int dev) {
  BlockCache& c = block_cache();
  std::lock_guard<std::mutex> g(c.mu);
  size_t total = 0;
  auto& m = c.blocks[dev];
  for (auto& kv : m) {
    cudaFree(kv.second);
    total += kv.first;
  }
  m.clear();
  return total;
}
}  // namespace

struct sdft_request {
  int device = 0;
  cudaStream_t stream = nullptr;
  int precision = SDFT_PREC_FP64;
  int NP = 0, M = 0, L = 0, NB = 0, MB = 0, NS = 0;
  int BL = 0;             // points of a transform buffer (M, or the Bluestein length)
  int NPt = 0;            // grid points (NP: stride of the device arrays)
  long long n = 0;
  long long n_caller = 0;  // unknowns in the caller's layout
  std::vector<SpeciesHost> sp;
  char* dmem = nullptr;
  size_t bytes = 0;
  size_t dbytes = 0;       // size of the device block (a cached block may be larger than bytes)
  DReq h{};            // host copy of the device descriptor
  DReq* dreq = nullptr;
  SolveSlot* dslot = nullptr;
  double* dout = nullptr;  // omega + num species
  // solver state after the last solve (checkpoint / resume): iteration count,
  // Picard flag, residual and LSQR warm start; the ring buffers stay in hx / hg
  SolveSlot slot{};
  int slot_m = 0;  // depth of the ring buffers in use (0: fresh)
  // a prepared request (sdft_request_prepare) holds its plan and the descriptor
  // values the upload reads until it is placed on the device
  std::unique_ptr<Plan> pending;
  sdft_system_desc pdesc{};
  std::vector<double> pdia, pval, pdmu;
};

// the state of a solve that has not started (AndersonMixing.jl:80-90)
static SolveSlot fresh_slot() {
  SolveSlot s{};
  s.iter = 0;
  s.status = ST_RUNNING;
  s.use_picard = 1;
  s.err = 1.0;
  return s;
}

extern "C" int32_t sdft_abi_version(void) { return SDFT_ABI_VERSION; }
extern "C" const char* sdft_last_error(void) { return g_err.c_str(); }

extern "C" int sdft_device_count(int32_t* count) {
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    *count = 0;
    return set_err(SDFT_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  *count = c;
  return SDFT_OK;
}

extern "C" void sdft_numerics_default(sdft_numerics* o) {
  o->max_iters = 100000;
  o->anderm = 5;
  o->damping = 0.5;
  o->mixing_max = 1.0;
  o->switch_tole = 1e-3;
  o->tole = 1e-6;
  o->mixed_switch = 0.0;
}

// device placement of a request: one allocation for the plan, its tables
// uploaded and the initial guess in x; the request's stream exists already
static int request_place(sdft_request* q, const sdft_system_desc* d, Plan& pl) {
  size_t got = 0;
  q->dmem = cache_find(q->device, pl.bytes, &got, true);
  if (q->dmem) {
    q->dbytes = got;
  } else {
    cudaError_t e = cudaMalloc(&q->dmem, pl.bytes);
    if (e != cudaSuccess) {  // give the cached blocks back to the driver and try once more
      cudaGetLastError();    // the failed allocation leaves no sticky error
      cache_release(q->device);
      e = cudaMalloc(&q->dmem, pl.bytes);
    }
    if (e != cudaSuccess) {
      q->dmem = nullptr;
      cudaGetLastError();
      return set_err(SDFT_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    q->dbytes = pl.bytes;
  }
  cudaError_t ce = cudaMemsetAsync(q->dmem, 0, pl.bytes, q->stream);
  std::vector<DSpecies> dsp;
  q->h = plan_bind(d, pl, q->dmem, nullptr, nullptr, dsp);
  q->dreq = (DReq*)(q->dmem + pl.o_dreq);
  q->dslot = (SolveSlot*)(q->dmem + pl.o_slot);
  q->dout = (double*)(q->dmem + pl.o_out);
  if (ce == cudaSuccess) ce = plan_upload(d, pl, q->dmem, q->h, dsp, q->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(q->stream);
  if (ce != cudaSuccess) {
    cudaFree(q->dmem);
    q->dmem = nullptr;
    return set_err(SDFT_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(ce));
  }
  return SDFT_OK;
}

// validated plan and host tables of a request, with its stream; no device memory
static int request_plan(const sdft_system_desc* d, int32_t precision, std::unique_ptr<sdft_request>& q,
                        std::unique_ptr<Plan>& pl) {
  if (d->abi_version != SDFT_ABI_VERSION) return set_err(SDFT_ERR_ARG, "ABI version mismatch");
  if (precision != SDFT_PREC_FP64 && precision != SDFT_PREC_MIXED) return set_err(SDFT_ERR_ARG, "unknown precision");
  pl.reset(new Plan());
  pl->prec = precision;
  int rc = plan_species(d, *pl);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(SDFT_ERR_CUDA, "no CUDA device");
  plan_layout(*pl, true);
  plan_tables(d, *pl);
  q.reset(new sdft_request());
  cudaGetDevice(&q->device);
  q->precision = precision;
  q->NP = pl->P;
  q->NPt = pl->Pt;
  q->n_caller = pl->n_caller;
  q->M = pl->M;
  q->BL = pl->BL;
  q->L = pl->L;
  q->NB = pl->NB;
  q->MB = pl->MB;
  q->NS = pl->NS;
  q->n = pl->n;
  q->sp = pl->sp;
  q->bytes = pl->bytes;
  cudaError_t e = cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    q->stream = nullptr;
    return set_err(SDFT_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  return SDFT_OK;
}

int request_create(const sdft_system_desc* d, int32_t precision, sdft_handle* out) {
  if (!d || !out) return set_err(SDFT_ERR_ARG, "null argument");
  *out = nullptr;
  std::unique_ptr<sdft_request> q;
  std::unique_ptr<Plan> pl;
  int rc = request_plan(d, precision, q, pl);
  if (rc == SDFT_OK) rc = request_place(q.get(), d, *pl);
  if (rc) {
    if (q && q->stream) cudaStreamDestroy(q->stream);
    return rc;
  }
  *out = q.release();
  return SDFT_OK;
}

// sdft_request_prepare: the plan and the descriptor values its upload reads are
// kept in the handle; the device memory is taken by request_ensure
int request_prepare(const sdft_system_desc* d, int32_t precision, sdft_handle* out) {
  if (!d || !out) return set_err(SDFT_ERR_ARG, "null argument");
  *out = nullptr;
  std::unique_ptr<sdft_request> q;
  std::unique_ptr<Plan> pl;
  int rc = request_plan(d, precision, q, pl);
  if (rc) {
    if (q && q->stream) cudaStreamDestroy(q->stream);
    return rc;
  }
  const int NB = pl->NB;
  q->pdia.assign(d->diameter, d->diameter + NB);
  q->pval.assign(d->valence, d->valence + NB);
  q->pdmu.assign(d->delta_muH, d->delta_muH + NB);
  q->pdesc = *d;  // scalars; the arrays that plan_bind / plan_upload read are the copies above
  q->pdesc.diameter = q->pdia.data();
  q->pdesc.valence = q->pval.data();
  q->pdesc.delta_muH = q->pdmu.data();
  q->pdesc.species = nullptr;
  q->pdesc.bond_types = nullptr;
  q->pdesc.mu_ex_bulk = nullptr;
  q->pdesc.lng_bulk = nullptr;
  q->pending = std::move(pl);
  *out = q.release();
  return SDFT_OK;
}

// a prepared request takes its device memory now; SDFT_ERR_OOM leaves it prepared
static int request_ensure(sdft_handle h) {
  if (!h->pending) return SDFT_OK;
  int rc = request_place(h, &h->pdesc, *h->pending);
  if (rc) return rc;
  h->pending.reset();
  h->pdia.clear();
  h->pval.clear();
  h->pdmu.clear();
  return SDFT_OK;
}

// host tables are sized by the descriptor; a failed host allocation is a status, not an exception across the C ABI
extern "C" int sdft_request_create(const sdft_system_desc* d, int32_t precision, sdft_handle* out) {
  try {
    return request_create(d, precision, out);
  } catch (const std::bad_alloc&) {
    return set_err(SDFT_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return set_err(SDFT_ERR_ARG, e.what());
  }
}

extern "C" int sdft_request_prepare(const sdft_system_desc* d, int32_t precision, sdft_handle* out) {
  try {
    return request_prepare(d, precision, out);
  } catch (const std::bad_alloc&) {
    return set_err(SDFT_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return set_err(SDFT_ERR_ARG, e.what());
  }
}

extern "C" int sdft_request_destroy(sdft_handle h) {
  if (!h) return SDFT_OK;
  // the request's own work is complete (batch solves and server steps
  // synchronise their streams before they return): its block is idle
  const cudaError_t e = cudaStreamSynchronize(h->stream);
  if (h->dmem) {
    if (e == cudaSuccess) cache_put(h->device, h->dmem, h->dbytes);
    else cudaFree(h->dmem);
  }
  cudaStreamDestroy(h->stream);
  delete h;
  return SDFT_OK;
}

extern "C" int sdft_release_cached_memory(int64_t* bytes) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return set_err(SDFT_ERR_CUDA, "no CUDA device");
  }
  const size_t b = cache_release(dev);
  if (bytes) *bytes = (int64_t)b;
  return SDFT_OK;
}

extern "C" int sdft_request_resident(sdft_handle h, int32_t* per_device) {
  if (!h || !per_device) return set_err(SDFT_ERR_ARG, "null argument");
  int ctas = 0, sms = 0;
  CUDA_TRY(h->h.gen || (h->pending && h->pending->gen) ? occupancy_solve_gen(smem_bytes(h->BL), &ctas)
                                                      : occupancy_solve_pow2(smem_bytes(h->BL), &ctas));
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
  *per_device = ctas * sms;
  return SDFT_OK;
}

extern "C" int sdft_grid_supported(int32_t np) {
  Plan pl;
  return plan_grid(np, pl);
}

extern "C" int sdft_request_sizes(sdft_handle h, int64_t* n_unknowns, int64_t* device_bytes) {
  if (!h) return set_err(SDFT_ERR_ARG, "null handle");
  if (n_unknowns) *n_unknowns = h->n_caller;
  if (device_bytes) *device_bytes = (int64_t)h->bytes;
  return SDFT_OK;
}

// transform buffers per CTA: up to kMaxTB within kTransformBudget, so that the
// solve kernel's occupancy target (kSolveCtasPerSm CTAs) fits an SM's shared
// memory; one buffer of fft_buffer_len(M) complex values minimum
static int tb_for(int M) {
  const size_t buf = sizeof(double2) * (size_t)fft_buffer_len(M);
  size_t tb = kTransformBudget / buf;
  if (tb < 1) tb = 1;
  if (tb > (size_t)kMaxTB) tb = kMaxTB;
  return (int)tb;
}
static size_t smem_bytes(int M) {
  return sizeof(double) * kRedDoubles + sizeof(double2) * (size_t)fft_buffer_len(M) * (size_t)tb_for(M);
}

// launches of the kernel build that matches the request (power-of-two or general FFT length)
static cudaError_t launch_objective(bool gen, const DReq* reqs, size_t smem, cudaStream_t s) {
  return gen ? launch_objective_gen(reqs, 1, smem, s) : launch_objective_pow2(reqs, 1, smem, s);
}
static cudaError_t launch_omega(bool gen, const DReq* reqs, double* out, size_t smem, cudaStream_t s) {
  return gen ? launch_omega_gen(reqs, out, smem, s) : launch_omega_pow2(reqs, out, smem, s);
}
// a batch: one launch of each build that has requests in it; *launches counts
// them.  With both kinds present the general build runs on a second stream that
// forks from and joins back into s, so the two launches share the GPU (each
// writes only the slots of its own requests).
static cudaError_t launch_solve(bool any_pow2, bool any_gen, const DReq* reqs, SolveSlot* slots, const SolveCfg& cfg,
                                int max_chunk, int n, size_t smem, cudaStream_t s, int* launches) {
  if (!(any_pow2 && any_gen)) {
    cudaError_t e = any_gen ? launch_solve_gen(reqs, slots, cfg, max_chunk, n, smem, s)
                            : launch_solve_pow2(reqs, slots, cfg, max_chunk, n, smem, s);
    if (e == cudaSuccess) (*launches)++;
    return e;
  }
  cudaStream_t s2 = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(fork, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, fork, 0);
  if (e == cudaSuccess) e = launch_solve_pow2(reqs, slots, cfg, max_chunk, n, smem, s);
  if (e == cudaSuccess) e = launch_solve_gen(reqs, slots, cfg, max_chunk, n, smem, s2);
  if (e == cudaSuccess) e = cudaEventRecord(join, s2);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, join, 0);
  if (e == cudaSuccess) *launches += 2;
  if (join) cudaEventDestroy(join);
  if (fork) cudaEventDestroy(fork);
  if (s2) cudaStreamDestroy(s2);
  return e;
}

// `rows` fields of NPt points between the caller's packed layout and the device
// layout of stride NP (equal for even grids; the pad point of odd grids is not copied)
static cudaError_t rows_copy(const sdft_request* h, double* dst, const double* src, size_t rows, cudaMemcpyKind kind) {
  const size_t Pt = h->NPt, P = h->NP;
  if (P == Pt) return cudaMemcpyAsync(dst, src, sizeof(double) * P * rows, kind, h->stream);
  const bool to_dev = kind == cudaMemcpyHostToDevice;
  return cudaMemcpy2DAsync(dst, sizeof(double) * (to_dev ? P : Pt), src, sizeof(double) * (to_dev ? Pt : P),
                           sizeof(double) * Pt, rows, kind, h->stream);
}

extern "C" int sdft_set_state(sdft_handle h, const double* mu_ex_K, const double* lng_K, const double* Psi,
                              const double* PsiC) {
  if (!h) return set_err(SDFT_ERR_ARG, "null handle");
  if (int rc_ = request_ensure(h)) return rc_;
  const size_t P = h->NP;
  double* x = h->h.x;
  const cudaMemcpyKind H2D = cudaMemcpyHostToDevice;
  if (mu_ex_K) CUDA_TRY(rows_copy(h, x, mu_ex_K, h->NB, H2D));
  if (lng_K && h->MB) CUDA_TRY(rows_copy(h, x + P * h->NB, lng_K, 2 * h->MB, H2D));
  if (Psi) CUDA_TRY(rows_copy(h, x + P * (h->NB + 2 * h->MB), Psi, 1, H2D));
  if (PsiC)
    CUDA_TRY(cudaMemcpyAsync(x + P * (h->NB + 2 * h->MB + 1), PsiC, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return SDFT_OK;
}

static int copy_vec_out(sdft_handle h, const double* dv, double* mu_ex_K, double* lng_K, double* Psi, double* PsiC) {
  const size_t P = h->NP;
  const cudaMemcpyKind D2H = cudaMemcpyDeviceToHost;
  if (mu_ex_K) CUDA_TRY(rows_copy(h, mu_ex_K, dv, h->NB, D2H));
  if (lng_K && h->MB) CUDA_TRY(rows_copy(h, lng_K, dv + P * h->NB, 2 * h->MB, D2H));
  if (Psi) CUDA_TRY(rows_copy(h, Psi, dv + P * (h->NB + 2 * h->MB), 1, D2H));
  if (PsiC)
    CUDA_TRY(cudaMemcpyAsync(PsiC, dv + P * (h->NB + 2 * h->MB + 1), sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return SDFT_OK;
}

extern "C" int sdft_get_state(sdft_handle h, double* mu_ex_K, double* lng_K, double* Psi, double* PsiC) {
  if (!h) return set_err(SDFT_ERR_ARG, "null handle");
  if (int rc_ = request_ensure(h)) return rc_;
  return copy_vec_out(h, h->h.x, mu_ex_K, lng_K, Psi, PsiC);
}

extern "C" int sdft_objective(sdft_handle h, double* mu_ex_K, double* lng_K, double* Psi, double* PsiC) {
  if (!h) return set_err(SDFT_ERR_ARG, "null handle");
  if (int rc_ = request_ensure(h)) return rc_;
  size_t sm = smem_bytes(h->BL);
  CUDA_TRY(launch_objective(h->h.gen != 0, h->dreq, sm, h->stream));
  int st = 0;
  CUDA_TRY(cudaMemcpyAsync(&st, h->h.status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (st == ST_NORM) return set_err(SDFT_ERR_NORM, "Normalization error: lambda <= 0 or not finite");
  return copy_vec_out(h, h->h.g, mu_ex_K, lng_K, Psi, PsiC);
}

// Mixed precision: a request evaluates G(x) with FP32 convolutions and
// propagators while the max-norm residual of the previous iteration is above
// the switch, then in FP64 to the tolerance, so the converged state is the FP64
// fixed point.  One FP32 evaluation differs from the FP64 one by 4e-8..1.4e-6
// (max-norm relative to max|G| on the test systems); the Anderson history must
// not be dominated by that noise, hence a switch well above it.
static double mixed_switch(const sdft_numerics* num) {
  const double s = num->mixed_switch > 0.0 ? num->mixed_switch : 1e-2;
  return std::max(s, 10.0 * num->tole);
}

static int validate_numerics(const sdft_numerics* num) {
  if (!num) return set_err(SDFT_ERR_ARG, "null numerics");
  if (num->anderm < 2 || num->anderm > kMaxAnderson) return set_err(SDFT_ERR_UNSUPPORTED, "anderm must be in [2, 16]");
  if (num->max_iters < 1) return set_err(SDFT_ERR_ARG, "max_iters must be >= 1");
  return SDFT_OK;
}

// chunked persistent solve of a batch of requests that share one stream
static int run_batch(sdft_handle* hs, int32_t n, const sdft_numerics* num, int32_t* iters, double* errs, int32_t* status,
                     bool resume = false) {
  int rc = validate_numerics(num);
  if (rc) return rc;
  for (int i = 0; i < n; i++)
    if ((rc = request_ensure(hs[i]))) return rc;
  if (resume)
    for (int i = 0; i < n; i++)
      if (hs[i]->slot_m != 0 && hs[i]->slot_m != num->anderm)
        return set_err(SDFT_ERR_ARG, "anderm differs from the solver state's");
  cudaStream_t stream = hs[0]->stream;
  size_t sm = 0;
  bool any_pow2 = false, any_gen = false;
  for (int i = 0; i < n; i++) {
    sm = std::max(sm, smem_bytes(hs[i]->BL));
    (hs[i]->h.gen ? any_gen : any_pow2) = true;
  }
  // device arrays and events of this batch, released on every return path
  struct BatchRes {
    cudaStream_t stream;
    DReq* dreqs = nullptr;
    SolveSlot* dslots = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~BatchRes() {
      if (dreqs) cudaFreeAsync(dreqs, stream);
      if (dslots) cudaFreeAsync(dslots, stream);
      if (ev0) cudaEventDestroy(ev0);
      if (ev1) cudaEventDestroy(ev1);
      if (dreqs || dslots) cudaStreamSynchronize(stream);
    }
  } res{stream};
  CUDA_TRY(cudaMallocAsync(&res.dreqs, sizeof(DReq) * n, stream));
  CUDA_TRY(cudaMallocAsync(&res.dslots, sizeof(SolveSlot) * n, stream));
  DReq* const dreqs = res.dreqs;
  SolveSlot* const dslots = res.dslots;
  std::vector<DReq> hreq(n);
  std::vector<SolveSlot> slots(n);
  for (int i = 0; i < n; i++) {
    hreq[i] = hs[i]->h;
    SolveSlot s = fresh_slot();
    if (resume && hs[i]->slot_m) {
      s = hs[i]->slot;
      s.status = ST_RUNNING;
    }
    slots[i] = s;
  }
  // requests on other streams must be idle before the batch stream uses them
  for (int i = 0; i < n; i++)
    if (hs[i]->stream != stream) CUDA_TRY(cudaStreamSynchronize(hs[i]->stream));
  CUDA_TRY(cudaMemcpyAsync(dreqs, hreq.data(), sizeof(DReq) * n, cudaMemcpyHostToDevice, stream));
  CUDA_TRY(cudaMemcpyAsync(dslots, slots.data(), sizeof(SolveSlot) * n, cudaMemcpyHostToDevice, stream));
  SolveCfg cfg;
  cfg.max_iters = num->max_iters;
  cfg.anderm = num->anderm;
  cfg.damping = num->damping;
  cfg.mixing_max = num->mixing_max;
  cfg.switch_tole = num->switch_tole;
  cfg.tole = num->tole;
  cfg.mixed_switch = mixed_switch(num);
  // bounded launches: each runs at most `chunk` iterations per request, the
  // host re-launches until every request has converged, failed or hit max_iters
  const int chunk = 1024;
  CUDA_TRY(cudaEventCreate(&res.ev0));
  CUDA_TRY(cudaEventCreate(&res.ev1));
  cudaEvent_t const ev0 = res.ev0, ev1 = res.ev1;
  double dev_ms = 0.0;
  int launches = 0;
  for (;;) {
    CUDA_TRY(cudaEventRecord(ev0, stream));
    CUDA_TRY(launch_solve(any_pow2, any_gen, dreqs, dslots, cfg, chunk, n, sm, stream, &launches));
    CUDA_TRY(cudaEventRecord(ev1, stream));
    CUDA_TRY(cudaMemcpyAsync(slots.data(), dslots, sizeof(SolveSlot) * n, cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
    dev_ms += ms;
    bool running = false;
    for (int i = 0; i < n; i++) running |= slots[i].status == ST_RUNNING;
    if (!running) break;
  }
  g_batch_ms = dev_ms;
  g_batch_launches = launches;
  g_batch_latency.assign(n, 0.0);
  for (int i = 0; i < n; i++) g_batch_latency[i] = (double)(slots[i].t1 - slots[i].t0) * 1e-6;
  int worst = SDFT_OK;
  for (int i = 0; i < n; i++) {
    hs[i]->slot = slots[i];
    hs[i]->slot_m = num->anderm;
    if (iters) iters[i] = slots[i].iter;
    if (errs) errs[i] = slots[i].err;
    int r = slots[i].status == ST_OK ? SDFT_OK
            : slots[i].status == ST_MAX_ITERS ? SDFT_MAX_ITERS
            : slots[i].status == ST_NORM ? SDFT_ERR_NORM
                                         : SDFT_ERR_NONFINITE;
    if (status) status[i] = r;
    if (r > worst) worst = r;
  }
  return worst;
}

static int solve_one(sdft_handle h, const sdft_numerics* num, int32_t* iters, double* err, bool resume) {
  if (!h) return set_err(SDFT_ERR_ARG, "null handle");
  int32_t it = 0, st = 0;
  double e = 0.0;
  int rc = run_batch(&h, 1, num, &it, &e, &st, resume);
  if (rc == SDFT_ERR_ARG || rc == SDFT_ERR_UNSUPPORTED) return rc;
  if (iters) *iters = it;
  if (err) *err = e;
  if (rc == SDFT_ERR_CUDA) return rc;
  if (st == SDFT_ERR_NORM) return set_err(SDFT_ERR_NORM, "Normalization error: lambda <= 0 or not finite");
  if (st == SDFT_ERR_NONFINITE) return set_err(SDFT_ERR_NONFINITE, "non-finite fixed-point residual");
  return st;
}

extern "C" int sdft_solve(sdft_handle h, const sdft_numerics* num, int32_t* iters, double* err) {
  return solve_one(h, num, iters, err, false);
}

extern "C" int sdft_solve_resume(sdft_handle h, const sdft_numerics* num, int32_t* iters, double* err) {
  return solve_one(h, num, iters, err, true);
}

// one caller-layout vector (mu_ex_K | lng_K | Psi | PsiC, NPt points per row)
// to or from a device vector of stride NP
static int vec_in(sdft_handle h, double* dv, const double* src) {
  const size_t P = h->NP, Pt = h->NPt, rows = (size_t)h->NB + 2 * h->MB + 1;
  CUDA_TRY(rows_copy(h, dv, src, rows, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpyAsync(dv + P * rows, src + Pt * rows, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  return SDFT_OK;
}
static int vec_out(sdft_handle h, const double* dv, double* dst) {
  const size_t P = h->NP, Pt = h->NPt, rows = (size_t)h->NB + 2 * h->MB + 1;
  CUDA_TRY(rows_copy(h, dst, dv, rows, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpyAsync(dst + Pt * rows, dv + P * rows, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return SDFT_OK;
}

extern "C" int sdft_get_solver_state(sdft_handle h, sdft_solver_state* st, double* hist_x, double* hist_g) {
  if (!h || !st) return set_err(SDFT_ERR_ARG, "null argument");
  if (int rc_ = request_ensure(h)) return rc_;
  const SolveSlot& s = h->slot_m ? h->slot : fresh_slot();
  std::memset(st, 0, sizeof(*st));
  st->anderm = h->slot_m;
  st->iter = s.iter;
  st->use_picard = s.use_picard;
  st->err = s.err;
  for (int c = 0; c + 1 < h->slot_m && c < 15; c++) st->lambdas[c] = s.lam[c];
  for (int c = 0; c < h->slot_m; c++) {
    if (hist_x) {
      int rc = vec_out(h, h->h.hx + (size_t)c * h->h.hstride, hist_x + (size_t)c * h->n_caller);
      if (rc) return rc;
    }
    if (hist_g) {
      int rc = vec_out(h, h->h.hg + (size_t)c * h->h.hstride, hist_g + (size_t)c * h->n_caller);
      if (rc) return rc;
    }
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return SDFT_OK;
}

extern "C" int sdft_set_solver_state(sdft_handle h, const sdft_solver_state* st, const double* hist_x,
                                     const double* hist_g) {
  if (!h || !st) return set_err(SDFT_ERR_ARG, "null argument");
  if (int rc_ = request_ensure(h)) return rc_;
  if (st->anderm < 2 || st->anderm > kMaxAnderson) return set_err(SDFT_ERR_ARG, "anderm must be in [2, 16]");
  if (st->iter < 0) return set_err(SDFT_ERR_ARG, "negative iteration count");
  SolveSlot s = fresh_slot();
  s.iter = st->iter;
  s.use_picard = st->use_picard ? 1 : 0;
  s.err = st->err;
  for (int c = 0; c + 1 < st->anderm; c++) s.lam[c] = st->lambdas[c];
  // the columns hold stride-NP vectors; the pad point of odd grids stays 0
  CUDA_TRY(cudaMemsetAsync(h->h.hx, 0, sizeof(double) * (size_t)kMaxAnderson * h->h.hstride, h->stream));
  CUDA_TRY(cudaMemsetAsync(h->h.hg, 0, sizeof(double) * (size_t)kMaxAnderson * h->h.hstride, h->stream));
  for (int c = 0; c < st->anderm; c++) {
    if (hist_x) {
      int rc = vec_in(h, h->h.hx + (size_t)c * h->h.hstride, hist_x + (size_t)c * h->n_caller);
      if (rc) return rc;
    }
    if (hist_g) {
      int rc = vec_in(h, h->h.hg + (size_t)c * h->h.hstride, hist_g + (size_t)c * h->n_caller);
      if (rc) return rc;
    }
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->slot = s;
  h->slot_m = st->anderm;
  return SDFT_OK;
}

extern "C" int sdft_anderson_step(sdft_handle h, const sdft_numerics* num, const double* g_mu_ex_K,
                                  const double* g_lng_K, const double* g_Psi, const double* g_PsiC, double* err) {
  if (!h) return set_err(SDFT_ERR_ARG, "null handle");
  if (int rc_ = request_ensure(h)) return rc_;
  int rc = validate_numerics(num);
  if (rc) return rc;
  if (!g_mu_ex_K || (h->MB && !g_lng_K) || !g_Psi || !g_PsiC) return set_err(SDFT_ERR_ARG, "null G(x) component");
  if (h->slot_m != 0 && h->slot_m != num->anderm) return set_err(SDFT_ERR_ARG, "anderm differs from the solver state's");
  const size_t P = h->NP;
  double* g = h->h.g;
  const cudaMemcpyKind H2D = cudaMemcpyHostToDevice;
  CUDA_TRY(rows_copy(h, g, g_mu_ex_K, h->NB, H2D));
  if (h->MB) CUDA_TRY(rows_copy(h, g + P * h->NB, g_lng_K, 2 * h->MB, H2D));
  CUDA_TRY(rows_copy(h, g + P * (h->NB + 2 * h->MB), g_Psi, 1, H2D));
  CUDA_TRY(cudaMemcpyAsync(g + P * (h->NB + 2 * h->MB + 1), g_PsiC, sizeof(double), H2D, h->stream));
  SolveSlot s = h->slot_m ? h->slot : fresh_slot();
  s.status = ST_RUNNING;
  CUDA_TRY(cudaMemcpyAsync(h->dslot, &s, sizeof(SolveSlot), H2D, h->stream));
  SolveCfg cfg;
  cfg.max_iters = num->max_iters;
  cfg.anderm = num->anderm;
  cfg.damping = num->damping;
  cfg.mixing_max = num->mixing_max;
  cfg.switch_tole = num->switch_tole;
  cfg.tole = num->tole;
  cfg.mixed_switch = mixed_switch(num);
  CUDA_TRY(h->h.gen ? launch_anderson_gen(h->dreq, h->dslot, cfg, h->stream)
                    : launch_anderson_pow2(h->dreq, h->dslot, cfg, h->stream));
  CUDA_TRY(cudaMemcpyAsync(&s, h->dslot, sizeof(SolveSlot), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->slot = s;
  h->slot_m = num->anderm;
  if (err) *err = s.err;
  if (s.status == ST_NONFINITE) return set_err(SDFT_ERR_NONFINITE, "non-finite fixed-point residual");
  return SDFT_OK;
}

extern "C" int sdft_solve_batch(sdft_handle* hs, int32_t n, const sdft_numerics* num, int32_t* iters, double* errs,
                                int32_t* status) {
  if (!hs || n < 1) return set_err(SDFT_ERR_ARG, "empty batch");
  for (int i = 0; i < n; i++)
    if (!hs[i]) return set_err(SDFT_ERR_ARG, "null handle in batch");
  return run_batch(hs, n, num, iters, errs, status);
}

extern "C" int sdft_last_batch_stats(double* device_ms, int32_t* launches, double* latency_ms, int32_t n) {
  if (device_ms) *device_ms = g_batch_ms;
  if (launches) *launches = g_batch_launches;
  if (latency_ms)
    for (int i = 0; i < n && i < (int)g_batch_latency.size(); i++) latency_ms[i] = g_batch_latency[i];
  return SDFT_OK;
}

// ---------------------------------------------------------------------------
// serving loop: continuous batching over persistent solver slots
//
// Requests are queued with sdft_server_submit and admitted, first in first
// out, into free slots while the slot count and the device-byte budget allow.
// Each sdft_server_step runs one launch of sdft_k_solve over the slots, at
// most `iters` Anderson iterations per request, then retires the requests that
// converged or failed; requests submitted meanwhile join at the next step.  A
// request's fields, history and solver scalars stay on the device between
// launches, so its result does not depend on the other requests in the mix.
// ---------------------------------------------------------------------------
struct sdft_server {
  sdft_numerics num{};
  int max_slots = 0;
  long long max_bytes = 0;
  cudaStream_t stream = nullptr;
  DReq* dreqs = nullptr;
  SolveSlot* dslots = nullptr;
  std::vector<DReq> hreq;
  std::vector<SolveSlot> hslot;
  std::vector<sdft_handle> owner;   // per slot, null when free
  std::vector<long long> tag;
  std::deque<std::pair<sdft_handle, long long>> queue;
  long long bytes_active = 0;
  long long reserve = 0;  // device bytes admission leaves free (requests placed at admission)
  int active = 0;
  // pipelined stepping: a step returns once its launch is queued; the launch's
  // slot states come back into pin (pinned, so that the copy is asynchronous)
  // and are collected at the next step
  bool pipeline = false;
  bool inflight = false;
  int hi_launched = 0;
  SolveSlot* pin = nullptr;
  struct Done {
    long long tag;
    int status, iters;
    double err, device_ms;
  };
  std::deque<Done> done;
};

static int slot_status_to_rc(int st) {
  return st == ST_OK ? SDFT_OK : st == ST_MAX_ITERS ? SDFT_MAX_ITERS : st == ST_NORM ? SDFT_ERR_NORM : SDFT_ERR_NONFINITE;
}

extern "C" int sdft_server_create(const sdft_numerics* num, int32_t max_slots, int64_t max_bytes, sdft_server_t* out) {
  if (!out) return set_err(SDFT_ERR_ARG, "null argument");
  *out = nullptr;
  int rc = validate_numerics(num);
  if (rc) return rc;
  if (max_slots < 1 || max_slots > 65535) return set_err(SDFT_ERR_ARG, "max_slots must be in [1, 65535]");
  auto* sv = new sdft_server();
  sv->num = *num;
  sv->max_slots = max_slots;
  sv->max_bytes = max_bytes;
  cudaError_t e = cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&sv->dreqs, sizeof(DReq) * max_slots);
  if (e == cudaSuccess) e = cudaMalloc(&sv->dslots, sizeof(SolveSlot) * max_slots);
  if (e == cudaSuccess) e = cudaMallocHost(&sv->pin, sizeof(SolveSlot) * max_slots);
  if (e != cudaSuccess) {
    if (sv->dreqs) cudaFree(sv->dreqs);
    if (sv->dslots) cudaFree(sv->dslots);
    if (sv->stream) cudaStreamDestroy(sv->stream);
    delete sv;
    return set_err(SDFT_ERR_OOM, std::string("server allocation: ") + cudaGetErrorString(e));
  }
  sv->hreq.assign(max_slots, DReq{});
  SolveSlot idle{};
  idle.status = -1;  // not ST_RUNNING: the kernel skips the slot
  sv->hslot.assign(max_slots, idle);
  sv->owner.assign(max_slots, nullptr);
  sv->tag.assign(max_slots, 0);
  *out = sv;
  return SDFT_OK;
}

extern "C" int sdft_server_destroy(sdft_server_t sv) {
  if (!sv) return SDFT_OK;
  cudaStreamSynchronize(sv->stream);
  cudaFree(sv->dreqs);
  cudaFree(sv->dslots);
  cudaFreeHost(sv->pin);
  cudaStreamDestroy(sv->stream);
  delete sv;
  return SDFT_OK;
}

extern "C" int sdft_server_submit(sdft_server_t sv, sdft_handle h, int64_t tag) {
  if (!sv || !h) return set_err(SDFT_ERR_ARG, "null argument");
  if (sv->max_bytes > 0 && (long long)h->bytes > sv->max_bytes)
    return set_err(SDFT_ERR_ARG, "request needs more device memory than the server budget");
  sv->queue.emplace_back(h, tag);
  return SDFT_OK;
}

// waits for the launch in flight and retires the requests that finished in it
static int server_collect(sdft_server* sv) {
  if (!sv->inflight) return SDFT_OK;
  sv->inflight = false;
  CUDA_TRY(cudaStreamSynchronize(sv->stream));
  const int hi = sv->hi_launched;
  std::memcpy(sv->hslot.data(), sv->pin, sizeof(SolveSlot) * hi);
  for (int i = 0; i < hi; i++) {
    if (!sv->owner[i] || sv->hslot[i].status == ST_RUNNING) continue;
    sdft_server::Done d;
    d.tag = sv->tag[i];
    d.status = slot_status_to_rc(sv->hslot[i].status);
    d.iters = sv->hslot[i].iter;
    d.err = sv->hslot[i].err;
    d.device_ms = (double)(sv->hslot[i].t1 - sv->hslot[i].t0) * 1e-6;
    sv->done.push_back(d);
    sv->bytes_active -= (long long)sv->owner[i]->bytes;
    sv->owner[i] = nullptr;
    sv->hslot[i].status = -1;
    sv->active--;
  }
  return SDFT_OK;
}

extern "C" int sdft_server_set_pipeline(sdft_server_t sv, int32_t on) {
  if (!sv) return set_err(SDFT_ERR_ARG, "null server");
  if (!on) {
    const int rc = server_collect(sv);
    if (rc) return rc;
  }
  sv->pipeline = on != 0;
  return SDFT_OK;
}

extern "C" int sdft_server_step(sdft_server_t sv, int32_t iters, int32_t* active, int32_t* queued) {
  if (!sv) return set_err(SDFT_ERR_ARG, "null server");
  if (iters < 1) return set_err(SDFT_ERR_ARG, "iters must be >= 1");
  // the previous launch of a pipelined server finishes first
  int rc0 = server_collect(sv);
  if (rc0) return rc0;
  // admission: FIFO into free slots within the byte budget; a prepared request
  // (sdft_request_prepare) is placed on the device here, once the free device
  // memory less the reserve covers it, else it waits for retirements
  int slot = 0;
  while (!sv->queue.empty()) {
    while (slot < sv->max_slots && sv->owner[slot]) slot++;
    if (slot >= sv->max_slots) break;
    sdft_handle h = sv->queue.front().first;
    const long long tag = sv->queue.front().second;
    if (sv->max_bytes > 0 && sv->bytes_active + (long long)h->bytes > sv->max_bytes) break;
    if (h->pending && !cache_find(h->device, h->bytes, nullptr, false)) {
      // a cached block would take no free device memory; a new one must leave the reserve
      size_t fr = 0, tot = 0;
      CUDA_TRY(cudaMemGetInfo(&fr, &tot));
      if ((long long)fr - (long long)h->bytes < sv->reserve) break;
    }
    if (h->pending) {
      const int rc = request_ensure(h);
      if (rc == SDFT_ERR_OOM) break;  // another allocation took the memory: retry at the next step
      if (rc) {                       // the request cannot be placed: it completes with that status
        sv->done.push_back(sdft_server::Done{tag, rc, 0, 0.0, 0.0});
        sv->queue.pop_front();
        continue;
      }
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));  // the request's own uploads are complete
    const int i = slot;
    sv->owner[i] = h;
    sv->tag[i] = tag;
    sv->queue.pop_front();
    sv->hreq[i] = h->h;
    SolveSlot s{};
    s.iter = 0;
    s.status = ST_RUNNING;
    s.use_picard = 1;
    s.err = 1.0;
    sv->hslot[i] = s;
    sv->bytes_active += (long long)h->bytes;
    sv->active++;
  }
  int hi = 0;
  size_t sm = 0;
  bool any_pow2 = false, any_gen = false;
  for (int i = 0; i < sv->max_slots; i++)
    if (sv->owner[i]) {
      hi = i + 1;
      sm = std::max(sm, smem_bytes(sv->owner[i]->BL));
      (sv->owner[i]->h.gen ? any_gen : any_pow2) = true;
    }
  if (hi > 0) {
    CUDA_TRY(cudaMemcpyAsync(sv->dreqs, sv->hreq.data(), sizeof(DReq) * hi, cudaMemcpyHostToDevice, sv->stream));
    CUDA_TRY(cudaMemcpyAsync(sv->dslots, sv->hslot.data(), sizeof(SolveSlot) * hi, cudaMemcpyHostToDevice, sv->stream));
    SolveCfg cfg;
    cfg.max_iters = sv->num.max_iters;
    cfg.anderm = sv->num.anderm;
    cfg.damping = sv->num.damping;
    cfg.mixing_max = sv->num.mixing_max;
    cfg.switch_tole = sv->num.switch_tole;
    cfg.tole = sv->num.tole;
    cfg.mixed_switch = mixed_switch(&sv->num);
    int launched = 0;
    CUDA_TRY(launch_solve(any_pow2, any_gen, sv->dreqs, sv->dslots, cfg, iters, hi, sm, sv->stream, &launched));
    CUDA_TRY(cudaMemcpyAsync(sv->pin, sv->dslots, sizeof(SolveSlot) * hi, cudaMemcpyDeviceToHost, sv->stream));
    sv->hi_launched = hi;
    sv->inflight = true;
    if (!sv->pipeline) {  // retire now; a pipelined server retires at the next step
      const int rc = server_collect(sv);
      if (rc) return rc;
    }
  }
  if (active) *active = sv->active;
  if (queued) *queued = (int32_t)sv->queue.size();
  return SDFT_OK;
}

extern "C" int sdft_server_set_reserve(sdft_server_t sv, int64_t reserve_bytes) {
  if (!sv) return set_err(SDFT_ERR_ARG, "null server");
  if (reserve_bytes < 0) return set_err(SDFT_ERR_ARG, "reserve must be >= 0");
  sv->reserve = reserve_bytes;
  return SDFT_OK;
}

extern "C" int sdft_server_poll(sdft_server_t sv, int64_t* tags, int32_t* status, int32_t* iters, double* errs,
                                double* device_ms, int32_t max, int32_t* n) {
  if (!sv || !n) return set_err(SDFT_ERR_ARG, "null argument");
  int k = 0;
  while (k < max && !sv->done.empty()) {
    const auto& d = sv->done.front();
    if (tags) tags[k] = d.tag;
    if (status) status[k] = d.status;
    if (iters) iters[k] = d.iters;
    if (errs) errs[k] = d.err;
    if (device_ms) device_ms[k] = d.device_ms;
    sv->done.pop_front();
    k++;
  }
  *n = k;
  return SDFT_OK;
}

extern "C" int sdft_get_densities(sdft_handle h, double* const* rho_segments, double* rho_beads_K, double* rho_bonds_K) {
  if (!h) return set_err(SDFT_ERR_ARG, "null handle");
  if (int rc_ = request_ensure(h)) return rc_;
  if (rho_segments) {
    std::vector<DSpecies> dsp(h->NS);
    CUDA_TRY(cudaMemcpyAsync(dsp.data(), h->h.sp, sizeof(DSpecies) * h->NS, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int u = 0; u < h->NS; u++)
      if (rho_segments[u])
        CUDA_TRY(rows_copy(h, rho_segments[u], dsp[u].rho_seg, (size_t)h->sp[u].S * h->sp[u].n_seg, cudaMemcpyDeviceToHost));
  }
  if (rho_beads_K) CUDA_TRY(rows_copy(h, rho_beads_K, h->h.rho_beads, h->NB, cudaMemcpyDeviceToHost));
  if (rho_bonds_K && h->MB) CUDA_TRY(rows_copy(h, rho_bonds_K, h->h.rho_bonds, 2 * h->MB, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return SDFT_OK;
}

static int run_omega(sdft_handle h, std::vector<double>& out) {
  size_t sm = smem_bytes(h->BL);
  CUDA_TRY(launch_omega(h->h.gen != 0, h->dreq, h->dout, sm, h->stream));
  out.assign(1 + h->NS, 0.0);
  CUDA_TRY(cudaMemcpyAsync(out.data(), h->dout, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return SDFT_OK;
}

extern "C" int sdft_grand_potential(sdft_handle h, double* omega) {
  if (!h || !omega) return set_err(SDFT_ERR_ARG, "null argument");
  if (int rc_ = request_ensure(h)) return rc_;
  std::vector<double> out;
  int rc = run_omega(h, out);
  if (rc) return rc;
  *omega = out[0];
  return SDFT_OK;
}

extern "C" int sdft_num_species(sdft_handle h, double* num_species) {
  if (!h || !num_species) return set_err(SDFT_ERR_ARG, "null argument");
  if (int rc_ = request_ensure(h)) return rc_;
  std::vector<double> out;
  int rc = run_omega(h, out);
  if (rc) return rc;
  for (int u = 0; u < h->NS; u++) num_species[u] = out[1 + u];
  return SDFT_OK;
}

// ---------------------------------------------------------------------------
// G(x) without device allocation (sdft_objective_noalloc)
//
// Some callers cannot call cudaMalloc: their device memory belongs to another
// allocator (a framework's caching pool, or a budget reserved once at start-up)
// that must stay the only owner, or they cannot afford the implicit device
// synchronisation a cudaMalloc may cause while other work is in flight.  This
// entry point evaluates G(x) with every intermediate array in one static device
// array of SDFT_NOALLOC_SCRATCH_BYTES; the caller passes x and G(x) as its own
// device arrays.  The array exists on every GPU that loads the library, until
// the process exits.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char sdft_noalloc_scratch[SDFT_NOALLOC_SCRATCH_BYTES];

namespace {
// device address of the scratch array in the current device's context, looked
// up on every call: a cached address would dangle after cudaDeviceReset (the
// module, and the array with it, is loaded again at another address)
int noalloc_scratch_address(void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, sdft_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return set_err(SDFT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  *out = p;
  return SDFT_OK;
}
}  // namespace

namespace {
int objective_noalloc(const sdft_system_desc* d, const double* x_dev, double* g_dev, void* stream_ptr) {
  if (!d || !x_dev || !g_dev) return set_err(SDFT_ERR_ARG, "null argument");
  if (d->abi_version != SDFT_ABI_VERSION) return set_err(SDFT_ERR_ARG, "ABI version mismatch");
  // G(x) is written as 16-byte grid-point pairs
  if (reinterpret_cast<uintptr_t>(g_dev) % 16 != 0 || reinterpret_cast<uintptr_t>(x_dev) % 8 != 0)
    return set_err(SDFT_ERR_ARG, "x_dev must be 8-byte and g_dev 16-byte aligned");
  Plan pl;
  int rc = plan_species(d, pl);
  if (rc) return rc;
  if (pl.P != pl.Pt)  // x and G(x) are the caller's arrays in the packed layout
    return set_err(SDFT_ERR_UNSUPPORTED, "sdft_objective_noalloc needs an even NP (got " + std::to_string(pl.Pt) + ")");
  // layout inside the scratch array (no Anderson history: G(x) only)
  plan_layout(pl, false);
  if (pl.bytes > (size_t)SDFT_NOALLOC_SCRATCH_BYTES)
    return set_err(SDFT_ERR_ARG, "system needs " + std::to_string(pl.bytes) + " bytes of scratch; sdft_objective_noalloc holds " +
                                     std::to_string((size_t)SDFT_NOALLOC_SCRATCH_BYTES));
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_ptr);
  void* base_v = nullptr;
  rc = noalloc_scratch_address(&base_v);
  if (rc) return rc;
  char* base = static_cast<char*>(base_v);
  plan_tables(d, pl);
  std::vector<DSpecies> dsp;
  DReq r = plan_bind(d, pl, base, const_cast<double*>(x_dev), g_dev, dsp);  // x is read only in G(x)
  // the array keeps the previous call's contents: clear the region this call uses
  CUDA_TRY(cudaMemsetAsync(base, 0, pl.bytes, stream));
  CUDA_TRY(plan_upload(d, pl, base, r, dsp, stream));
  size_t sm = smem_bytes(pl.BL);
  CUDA_TRY(launch_objective(pl.gen, (const DReq*)(base + pl.o_dreq), sm, stream));
  int st = 0;
  CUDA_TRY(cudaMemcpyAsync(&st, r.status, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CUDA_TRY(cudaStreamSynchronize(stream));
  if (st == ST_NORM) return set_err(SDFT_ERR_NORM, "Normalization error: lambda <= 0 or not finite");
  return SDFT_OK;
}
}  // namespace

extern "C" int sdft_objective_noalloc(const sdft_system_desc* d, const double* x_dev, double* g_dev, void* stream_ptr) {
  try {
    return objective_noalloc(d, x_dev, g_dev, stream_ptr);
  } catch (const std::bad_alloc&) {
    return set_err(SDFT_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return set_err(SDFT_ERR_ARG, e.what());
  }
}
