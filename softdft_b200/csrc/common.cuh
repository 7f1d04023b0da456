// common.cuh -- device-side request layout shared by every stage of the solve.
//
// One request (one inhomogeneous system) is owned by one CTA for the whole
// solve.  Grid arrays use the reference's column-major layout with the grid
// index K fastest (src/iDFT/setup/setup_steps/process_fields.jl:20-59):
//   x      = [ mu_ex_K (NB x NP) | lng_K (MB x 2 x NP) | Psi (NP) | PsiC ]
//   lambda = (NB x NP), Ext/trapez = (NB x NP), rho_beads = (NB x NP),
//   rho_bonds = (MB x 2 x NP), rho_seg_u = (n_seg x S x NP).
// Every mirrored-grid convolution of the reference is carried in DCT-II
// coefficient space ("C-space"): P real coefficients per field, see fft.cuh.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sdft {

#ifndef SDFT_THREADS
#define SDFT_THREADS 256
#endif
constexpr int kThreads = SDFT_THREADS;  // CTA size of the solve kernels
constexpr int kMaxStates = 4;        // per-segment state families the device supports
constexpr int kMaxBeads = 32;        // bead types
constexpr int kMaxBonds = 64;        // bond types
constexpr int kMaxAnderson = 16;     // Anderson depth m
constexpr int kMaxTB = 8;            // transforms in flight per CTA
constexpr int kMaxRadices = 24;      // stages of a general-length FFT
constexpr int kMaxGenRadix = 61;     // largest prime factor of a general-length FFT
constexpr double kPi = 3.14159265358979323846;

// status codes written by the kernels (mirror sdft_status)
enum : int {
  ST_OK = 0,
  ST_MAX_ITERS = 1,
  ST_NORM = 6,
  ST_NONFINITE = 7,
  ST_RUNNING = 100,
};

struct DSpecies {
  int n_seg;          // segments N_u
  int S;              // state slots per segment
  int fixed;          // grid index of the grafted segment 0, -1 if free
  int tree;           // 1: branched topology (general level walks, arrays below)
  const int* states;  // [n_seg * S] bead type per (segment, slot), -1 padding
  const int* nst;     // [n_seg] states per segment
  const int* bnd;     // [(g * S + i) * S + j] bond type between state i of segment g and state j of g+1, -1 if none
  const double* md;   // [n_seg] max path distance from segment g to segment 0 (fixed species)
  double fixed_density;
  double mu_species;  // bulk chemical potential (set to 0 for grafted species each evaluation)
  double normative;   // prod_g (sum_states e^-dmuH)^(1/N)  (child_propagators.jl:41-50)
  double norm_free;   // normative^(N-1): chain normalisation of a free species (handle_fixed.jl:105-108)
  double lambda_fixed;
  double* gC;         // [(g * S + i) * S + j] * P + K : parent g state i, child g+1 state j
  double* gP;         // [(g * S + i) * S + j] * P + K : child g state i, parent g-1 state j
  double* rho_seg;    // [(g * S + i) * P + K]
  int* expo;          // [2 * n_seg]: power-of-two exponent carried by gC of g, then by gP of g
  // species-local slots for register accumulation of bond-end and bead densities
  const int* bslot;       // [(g * S + i) * S + j] slot of bond bnd[...] among the species' bonds
  const int* bslot_bond;  // [nbslot] bond type of each slot
  const int* eslot;       // [g * S + i] slot of bead type states[g * S + i] among the species' beads
  const int* eslot_bead;  // [neslot] bead type of each slot
  int nbslot, neslot;
  // branched topologies: gC is [(g * S + i) * C + c) * S + j] * P + K (child slot c)
  int C;                  // most children of a segment
  int pad1;
  const int* parent;      // [n_seg] parent segment, -1 for the root
  const int* nch;         // [n_seg] children per segment
  const int* child;       // [n_seg * C] children of each segment
  const int* order;       // [n_seg] segments by level from the root (ascending index within a level)
};

struct DReq {
  // sizes
  int NP, M, L;       // stride of per-point arrays, FFT length, log2(M) (power-of-two M)
  int NPt;            // grid points: NP for even grids, NP - 1 for odd ones (the last point pads)
  int gen;            // 1: M is not a power of two (mixed-radix tables below)
  int has_tree;       // 1: a species has a branched topology
  int nrad;           // general length: number of radices
  int rad[kMaxRadices];  // general length: radices r_0 .. r_{nrad-1}, M = their product
  int NB, MB, NS;
  int funcs;          // SDFT_FUNC_* bits
  int TB;             // transform buffers in shared memory for this launch (1..kMaxTB)
  int ngrp;           // distinct bead diameters
  int prec;           // 0: FP64; 1: FP32 propagators while the residual is above the switch
  double dz, lB, total_charge;
  long long n;        // Anderson unknowns
  long long hstride;  // column stride of the Anderson histories: n rounded up to 32 (256-byte columns)
  long long zbytes;   // shared memory of the transform buffers (free while the Anderson update runs)
  // per-bead / per-bond constants
  const double* sig;  // [NB]
  const double* z;    // [NB]
  const double* dmu;  // [NB]
  const int* bonds;   // [MB * 2]
  const int* grp;     // [NB] index of the bead's diameter in grp_sig
  const double* grp_sig;  // [ngrp] distinct diameters
  const DSpecies* sp; // [NS]
  // fixed fields
  const double* Ext;      // [NB * P]
  const double* trapez;   // [NB * P]
  const double* Csurf;    // [P] DCT-II of the mirrored surface charge
  // C-space weights, k = 0..P-1 (index k of the reference's 2P-point FFT grid)
  const double* Wbond;    // [MB * P] filtered bond kernel: w_b(k) * exp(-(k/kc)^4)
  const double* Wfmt;     // [NB * 3 * P] delta shell, step, vector (odd) weights at R = sigma/2
  const double* Wmsa;     // [NB * P]
  const double* Wcoul;    // [P]
  // FFT tables
  const double2* tw;      // [M/2] e^{-2 pi i k / M} ([M] for a general length)
  const int* slot;        // general length: [M] digit-reversed slot of natural index m
  const double2* twP;     // [M+1] e^{-2 pi i k / P}
  const double2* twD;     // [M+1] e^{-i pi k / (2P)}
  const float2* tw32;     // FP32 copies of tw, twP, twD (mixed precision)
  const float2* twP32;
  const float2* twD32;
  // Bluestein transform (general length with a prime factor above kMaxGenRadix)
  int blue;               // 1: the length-M DFTs run as chirp convolutions of length LB
  int LB, lLB;            // LB = 2^lLB >= 2M - 1 (the transform buffers hold LB points)
  const double2* bw;      // [M] chirp e^{-i pi n^2 / M}
  const double2* bB;      // [LB] spectrum of the chirp filter / LB, bit-reversed order
  const double2* btw;     // [LB/2 + 1] e^{-2 pi i k / LB}
  const float2* bw32;     // FP32 copies (mixed precision)
  const float2* bB32;
  const float2* btw32;
  // state
  double* x;              // [n] unknowns
  double* g;              // [n] G(x) of the last evaluation
  double* lambda;         // [NB * P]
  double* rho_beads;      // [NB * P]
  double* rho_bonds;      // [MB * 2 * P]
  double* Cb;             // [NB * P]      DCT-II of rho_beads * trapez
  double* Cbond;          // [MB * 2 * P]  DCT-II of rho_bonds * trapez(end bead)
  double* Cmu;            // [NB * P]      accumulated mu_ex coefficients
  double* Clng;           // [MB * 2 * P]  accumulated ln g coefficients
  double* wa;             // [max(NB, 6) * P] scratch (weighted densities, derivatives)
  double* wb;             // [MB * 2 * P]  scratch (bond weighted densities)
  double* wc;             // [max(NB, 6 + MB) * P] scratch (derivative fields)
  double* wd;             // [2 * NB * P] scratch (per-bead FMT weighted densities)
  double* elam;           // [NB * P] e^{-lambda} of the current x
  float* fbe32;           // [4 * MB * P] FP32 copy of fbe (mixed precision)
  double* fbe;            // [4 * MB * P] bond-end factors of the current x: e^{-lambda_j + lng/2} trapez_j, then e^{lng/2}
  // Anderson
  double* hx;             // [m * n] history of x
  double* hg;             // [m * n] history of G(x) - x
  double* lsq_u;          // [n] LSQR work vector
  // results
  int* status;            // [1]
  int* iters;             // [1]
  double* err;            // [1]
  double* scal;           // [8] scalars: 0 PsiC shift, 1.. reserved
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 sub2(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 scl2(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// the same for FP32 complex values (mixed-precision propagators)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conj2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 scl2(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// real type and constructor of a complex type
template <class C>
struct Cx;
template <>
struct Cx<double2> {
  using R = double;
  static __device__ __forceinline__ double2 make(double x, double y) { return make_double2(x, y); }
};
template <>
struct Cx<float2> {
  using R = float;
  static __device__ __forceinline__ float2 make(float x, float y) { return make_float2(x, y); }
};

// ---------------------------------------------------------------------------
// CTA reductions (warp shuffles + one shared slot per warp)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// returns the CTA-wide sum to every thread; red must hold >= 32 doubles
__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  const int nw = blockDim.x >> 5;
  for (int i = 0; i < nw; i++) t += red[i];
  return t;
}

__device__ __forceinline__ double block_max(double v, double* red) {
  v = warp_max(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = red[0];
  const int nw = blockDim.x >> 5;
  for (int i = 1; i < nw; i++) t = fmax(t, red[i]);
  return t;
}

// the maxima of two values over the CTA (one barrier pair)
__device__ __forceinline__ void block_max2(double* a, double* b, double* red) {
  double x = warp_max(*a), y = warp_max(*b);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
    red[w] = x;
    red[32 + w] = y;
  }
  __syncthreads();
  x = red[0];
  y = red[32];
  for (int i = 1; i < nw; i++) {
    x = fmax(x, red[i]);
    y = fmax(y, red[32 + i]);
  }
  *a = x;
  *b = y;
}

// 16-byte asynchronous global -> shared copies, completed per thread by commit
// groups (cp.async.cg: cached in L2 only, as __ldcg); both addresses 16-byte aligned
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's commit groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// k sums at once (k <= 16): vals[k] in/out
template <int KMAX>
__device__ __forceinline__ void block_sum_vec(double* vals, int k, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int q = 0; q < k; q++) vals[q] = warp_sum(vals[q]);
  __syncthreads();
  if (lane == 0)
    for (int q = 0; q < k; q++) red[q * 32 + w] = vals[q];
  __syncthreads();
  for (int q = 0; q < k; q++) {
    double t = 0.0;
    for (int i = 0; i < nw; i++) t += red[q * 32 + i];
    vals[q] = t;
  }
}

// ---- solve configuration and per-request solver state (host and device) ----
struct SolveCfg {
  int max_iters;
  int anderm;
  double damping, mixing_max, switch_tole, tole;
  double mixed_switch;  // residual below which a mixed-precision request evaluates in FP64
};

struct SolveSlot {       // per-request solver state kept across launches
  int iter;
  int status;
  int use_picard;
  int pad;
  double err;
  unsigned long long t0, t1;  // %globaltimer (ns) at the first and the last iteration
  double lam[kMaxAnderson];
};

constexpr int kRedDoubles = 1024;              // reduction scratch ahead of the transform buffers
// Occupancy target of the solve kernel: CTAs resident per SM.  It sets the
// register cap (65536 / (256 CTAs)) through __launch_bounds__ and the shared
// memory each CTA may use for transform buffers (an SM holds 228 KB).
#ifndef SDFT_SOLVE_CTAS
#define SDFT_SOLVE_CTAS 2
#endif
constexpr int kSolveCtasPerSm = SDFT_SOLVE_CTAS;
constexpr size_t kTransformBudget = kSolveCtasPerSm >= 3 ? 64 * 1024 : 96 * 1024;
constexpr size_t kMaxSmemBytes = 227 * 1024;   // dynamic shared memory a CTA may opt into

// Padded position of complex index i in a transform buffer: one spare slot
// after every 8 and after every 64 values.  The strided radix passes then meet
// no bank conflicts, and the bit-reversed slots that the Makhoul reorder
// writes and reads spread over the banks (with one spare per 8 alone, the 16
// slots a warp touches there fall on two bank groups).
__host__ __device__ constexpr int fpad(int i) { return i + (i >> 3) + (i >> 6); }
// slots of a transform buffer of n complex values
__host__ __device__ constexpr int fft_buffer_len(int n) { return n > 0 ? fpad(n - 1) + 1 : 0; }
// ---- kernel launches ----
// The kernels are compiled twice (kernels_pow2.cu, kernels_gen.cu): once with
// the power-of-two FFT passes and once with the general-length ones, so that
// neither build carries the other's code.  A launch runs one CTA per request
// and skips the requests of the other kind.
cudaError_t launch_objective_pow2(const DReq* reqs, int n, size_t smem, cudaStream_t s);
cudaError_t launch_solve_pow2(const DReq* reqs, SolveSlot* slots, SolveCfg cfg, int max_chunk, int n, size_t smem,
                              cudaStream_t s);
cudaError_t launch_omega_pow2(const DReq* reqs, double* out, size_t smem, cudaStream_t s);
cudaError_t launch_anderson_pow2(const DReq* reqs, SolveSlot* slots, SolveCfg cfg, cudaStream_t s);
cudaError_t occupancy_solve_pow2(size_t smem, int* ctas_per_sm);
cudaError_t occupancy_solve_gen(size_t smem, int* ctas_per_sm);
cudaError_t launch_anderson_gen(const DReq* reqs, SolveSlot* slots, SolveCfg cfg, cudaStream_t s);
cudaError_t launch_objective_gen(const DReq* reqs, int n, size_t smem, cudaStream_t s);
cudaError_t launch_solve_gen(const DReq* reqs, SolveSlot* slots, SolveCfg cfg, int max_chunk, int n, size_t smem,
                             cudaStream_t s);
cudaError_t launch_omega_gen(const DReq* reqs, double* out, size_t smem, cudaStream_t s);

}  // namespace sdft
