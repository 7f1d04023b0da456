/*
 * softdft.h -- C ABI of the B200 iDFT self-consistent solve.
 *
 * The library replaces the bodies of the reference's inhomogeneous solve loop:
 *   solver_dft(dft_system)                 src/iDFT/evaluation/objective/solver_dft.jl:5-25
 *   solver_function(::AndersonMixing, ...) src/NonlinearSolvers/fixed_point/AndersonMixing.jl:56-169
 *   objective_dft(problem_data)            src/iDFT/evaluation/objective/objective_dft.jl:6-30
 *   grand_potential(dft_system)            src/iDFT/evaluation/analysis/grand_potential.jl:4-28
 *   get_num_species(...)                   src/iDFT/evaluation/analysis/num_species.jl:1-38
 * Setup (input.yaml, molecular system, bulk iLST state, geometry) stays on the
 * host; the host fills a sdft_system_desc and the library builds every grid
 * field, k-space weight and FFT plan on the device.
 *
 * Conventions
 *  - Plain C types only.  Input pointers are borrowed for the duration of the
 *    call; the library copies what it needs.  Output pointers are caller-owned
 *    host memory.
 *  - Grid arrays use the reference's column-major layout with the grid index
 *    fastest:  mu_ex_K[K + NP*j]          (NP, NB)
 *              lng_K[K + NP*(e + 2*b)]    (NP, 2, MB)   e = bond end 0/1
 *              Psi[K]                     (NP)
 *              rho_segments_u[K + NP*(s + S_u*g)]  (NP, S_u, N_u)
 *  - Indices (bead types, bonds, segments, grid points) are 0-based.
 *  - Every function returns an sdft_status; sdft_last_error() gives the text of
 *    the most recent failure on the calling thread.  SDFT_MAX_ITERS is returned
 *    by the solve when max_iters is reached; it is not an error (the reference
 *    returns normally in that case) and the state is valid.
 *  - Handles are independent; each owns one CUDA stream.  A handle must not be
 *    used from two threads at once.
 */
#ifndef SOFTDFT_H
#define SOFTDFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDFT_ABI_VERSION 2

typedef enum sdft_status {
  SDFT_OK = 0,
  SDFT_MAX_ITERS = 1,        /* solve stopped at max_iters (state valid) */
  SDFT_ERR_ARG = 2,          /* invalid descriptor or argument */
  SDFT_ERR_UNSUPPORTED = 3,  /* feature outside the device solve */
  SDFT_ERR_CUDA = 4,         /* CUDA runtime error or no device */
  SDFT_ERR_OOM = 5,          /* device or host memory exhausted / admission refused */
  SDFT_ERR_NORM = 6,         /* chain normalisation lambda <= 0 or not finite */
  SDFT_ERR_NONFINITE = 7,    /* NaN/Inf in the fixed-point residual */
  SDFT_ERR_TIMEOUT = 8       /* reserved: no call of this version waits on the device
                                without a bound, so none returns it */
} sdft_status;

/* functional set (bitmask): the `model:` list of input.yaml minus `ideal`;
 * registry src/iDFT/functionals/Abstract_Types/functional_registry.jl:53-70 */
#define SDFT_FUNC_MFMT      0x1u   /* White-Bear FMT                 functionals/excluded_volume/mfmt.jl */
#define SDFT_FUNC_TPT1MFMT  0x2u   /* White-Bear FMT + TPT1 bonding  functionals/excluded_volume/TPT1mfmt.jl */
#define SDFT_FUNC_MSA       0x4u   /* MSA electrostatic correlations functionals/electrostaticcorrelations/msa.jl */
#define SDFT_FUNC_TPT1MSA   0x8u   /* MSA + TPT1 bonding             functionals/electrostaticcorrelations/TPT1msa.jl */

/* arithmetic of the solve */
#define SDFT_PREC_FP64   0   /* every stage in FP64 (the plain form) */
#define SDFT_PREC_MIXED  1   /* FP32 convolutions/propagators; FP64 Anderson,
                                state sums, functional pointwise terms, residual */

/* One species (configuration): src/molecular_system/structures/ConfigurationStruct.jl:41-47
 * plus its fixed (grafted) segments, src/iDFT/structures/FixedSpecies.jl:20-39. */
typedef struct sdft_species_desc {
  int32_t n_seg;                 /* segments N_u */
  int32_t max_states;            /* S_u = max over segments of the state count */
  const int32_t* parent;         /* [n_seg] parent segment, -1 for the root (segment 0) */
  const int32_t* n_states;       /* [n_seg] states of each segment */
  const int32_t* states;         /* [n_seg*max_states] bead type of (segment, state slot) */
  const int32_t* fixed_coord;    /* [n_seg] 0-based grid index of a fixed segment, -1 if free; may be NULL */
  double fixed_density;          /* grafting density (chains per unit area) */
  const double* max_distance;    /* [n_seg*n_seg] row-major path-length matrix; may be NULL without fixed segments */
  double mu_species;             /* bulk chemical potential of the species */
} sdft_species_desc;

/* One inhomogeneous system (request). */
typedef struct sdft_system_desc {
  int32_t abi_version;           /* SDFT_ABI_VERSION */
  int32_t np;                    /* grid points NP = cld(H, dz) + 1 */
  double bin_width;              /* dz */
  double length;                 /* slit width H (wall positions 0 and H) */
  int32_t hard_walls;            /* nonzero: hard walls at 0 and H */
  int32_t charged_walls;         /* nonzero: surface charges at 0 and H */
  double wall_charge[2];         /* (qL, qR), e per area */
  double bjerrum_length;         /* in units of the length scale */
  int32_t nb;                    /* bead types */
  const double* diameter;        /* [nb] */
  const double* valence;         /* [nb] */
  const double* delta_muH;       /* [nb] */
  int32_t mb;                    /* bond types */
  const int32_t* bond_types;     /* [mb*2] (min, max) bead-type pairs */
  int32_t n_species;
  const sdft_species_desc* species;
  uint32_t functionals;          /* SDFT_FUNC_* */
  const double* mu_ex_bulk;      /* [nb] bulk excess chemical potential (initial guess) */
  const double* lng_bulk;        /* [mb] bulk ln g (initial guess) */
} sdft_system_desc;

/* Anderson controls: numerical section of input.yaml,
 * src/NonlinearSolvers/fixed_point/AndersonMixing.jl:74-79 */
typedef struct sdft_numerics {
  int32_t max_iters;             /* default 100000 */
  int32_t anderm;                /* history depth m, default 5 */
  double damping;                /* default 0.5 */
  double mixing_max;             /* default 1.0 */
  double switch_tole;            /* default 1e-3 */
  double tole;                   /* default 1e-6 */
  double mixed_switch;           /* SDFT_PREC_MIXED requests evaluate with FP32 propagators while
                                    the residual is above this, then in FP64 (0: the default 1e-2;
                                    never below 10 * tole).  No reference counterpart. */
} sdft_numerics;

typedef struct sdft_request* sdft_handle;

/* Library / device */
int32_t sdft_abi_version(void);
const char* sdft_last_error(void);
int sdft_device_count(int32_t* count);
void sdft_numerics_default(sdft_numerics* out);

/* Request lifecycle.  Builds Ext, trapez, k-space weights, the surface charge
 * spectrum and the initial guess of process_guess
 * (src/iDFT/setup/setup_steps/process_guess.jl:5-54) on the device. */
int sdft_request_create(const sdft_system_desc* desc, int32_t precision, sdft_handle* out);
int sdft_request_destroy(sdft_handle h);
/* Device memory of destroyed requests is cached by the library for later
 * requests of a size it covers (a cudaFree synchronises the whole device, and a
 * server retires and admits requests at every step).  A request takes the
 * smallest cached block of its device that holds it with at most a quarter to
 * spare; a failed device allocation releases the device's cache and is tried
 * once more.  sdft_release_cached_memory returns the cached blocks of the
 * current device to the driver and *bytes (may be NULL) says how many bytes
 * that was.  No reference counterpart (Julia's GC owns the reference's
 * arrays). */
int sdft_release_cached_memory(int64_t* bytes);
/* A request without device memory yet: the descriptor is validated and the
 * host tables are built as by sdft_request_create, and the handle keeps them;
 * the device memory (sdft_request_sizes' device_bytes) is taken when the
 * request is first used, or by a server when it admits the request.  No
 * reference counterpart (the reference holds one system per process). */
int sdft_request_prepare(const sdft_system_desc* desc, int32_t precision, sdft_handle* out);
/* sizes: n = NP*(NB + 2*MB + 1) + 1 (Anderson vector length) */
int sdft_request_sizes(sdft_handle h, int64_t* n_unknowns, int64_t* device_bytes);
/* How many requests of this one's shape (grid, transform buffers) the device
 * runs at once: resident solve CTAs per SM times the SM count.  A batch or a
 * server of that many requests fills the GPU in one wave.  No reference
 * counterpart. */
int sdft_request_resident(sdft_handle h, int32_t* per_device);
/* SDFT_OK when the device solve runs a grid of np points, else
 * SDFT_ERR_UNSUPPORTED with the reason in sdft_last_error().  No reference
 * counterpart (FFTW plans any length): the device transform takes np >= 16
 * whose FFT length M (np/2 for even np, np for odd np) fits one CTA's shared
 * memory: mixed radix when M has no prime factor above 61 (M up to 12288),
 * else Bluestein's chirp convolution of 2^k >= 2M - 1 points (M up to 4096).
 * Host-only: needs no GPU. */
int sdft_grid_supported(int32_t np);

/* Unknowns x = (mu_ex_K, lng_K, Psi, PsiC), solver_dft.jl:13 */
int sdft_set_state(sdft_handle h, const double* mu_ex_K, const double* lng_K,
                   const double* Psi, const double* PsiC);
int sdft_get_state(sdft_handle h, double* mu_ex_K, double* lng_K, double* Psi, double* PsiC);

/* One fixed-point map evaluation G(x) (objective_dft), without changing x.
 * Any output pointer may be NULL. */
int sdft_objective(sdft_handle h, double* mu_ex_K, double* lng_K, double* Psi, double* PsiC);

/* Anderson-mixing solve from the current state; x is updated in place. */
int sdft_solve(sdft_handle h, const sdft_numerics* num, int32_t* iters, double* err);

/* Solver state of a request: what the Anderson driver carries from one
 * iteration to the next in solver_function(::AndersonMixing, ...)
 * (AndersonMixing.jl:80-168): the iteration count, the Picard flag, the last
 * max-norm residual, the LSQR warm start `lambdas` (:88, :142) and the ring
 * buffers X and G of depth m (:81-84; G holds the residuals G(x) - x).  The
 * reference keeps these in locals of one call; here they persist in the request
 * so that a solve can stop and continue (checkpoint / resume), move to another
 * handle of the same system, or start from a given history. */
typedef struct sdft_solver_state {
  int32_t anderm;                /* depth m of the ring buffers */
  int32_t iter;                  /* iterations done (0: fresh) */
  int32_t use_picard;            /* 1 while the Picard phase lasts */
  int32_t reserved;              /* 0 */
  double err;                    /* max-norm residual of the last iteration */
  double lambdas[15];            /* LSQR coefficients of the last Anderson step (anderm - 1 used) */
} sdft_solver_state;

/* Read / replace the solver state.  hist_x and hist_g hold anderm columns of
 * n_unknowns doubles (ring slot c at offset c * n_unknowns, each column in the
 * layout mu_ex_K | lng_K | Psi | PsiC of sdft_get_state); either may be NULL
 * (set: zero columns).  Before any solve the state is fresh (iter 0). */
int sdft_get_solver_state(sdft_handle h, sdft_solver_state* st, double* hist_x, double* hist_g);
int sdft_set_solver_state(sdft_handle h, const sdft_solver_state* st, const double* hist_x, const double* hist_g);
/* Continue the Anderson solve from the stored solver state (the end of the last
 * solve, or sdft_set_solver_state) up to num->max_iters iterations in total;
 * num->anderm must equal the state's.  sdft_solve starts from a fresh state,
 * as a call of solver_function does. */
int sdft_solve_resume(sdft_handle h, const sdft_numerics* num, int32_t* iters, double* err);
/* One iteration of the Anderson driver with G(x) given by the caller (the
 * layout of sdft_objective's outputs) instead of evaluated on the device: the
 * loop body of AndersonMixing.jl:98-160 after `cur = objective_function(...)`.
 * It updates x and the solver state; *err receives the max-norm residual
 * |G(x) - x| of this iteration.  A caller that evaluates its own objective can
 * drive the device mixer with it, as solver_function takes any objective. */
int sdft_anderson_step(sdft_handle h, const sdft_numerics* num, const double* g_mu_ex_K, const double* g_lng_K,
                       const double* g_Psi, const double* g_PsiC, double* err);

/* Densities of the last G(x) evaluation.  rho_segments: array of n_species host
 * pointers (entries may be NULL).  Any argument may be NULL. */
int sdft_get_densities(sdft_handle h, double* const* rho_segments, double* rho_beads_K,
                       double* rho_bonds_K);

/* Grand potential (grand_potential.jl:4-28) from the current x and the densities
 * of the last evaluation; chains per species (num_species.jl:1-38). */
int sdft_grand_potential(sdft_handle h, double* omega);
int sdft_num_species(sdft_handle h, double* num_species);

/* Batched solve: every request of the batch runs in one launch (one persistent
 * CTA per request).  status[i] receives the per-request sdft_status. */
int sdft_solve_batch(sdft_handle* hs, int32_t n, const sdft_numerics* num,
                     int32_t* iters, double* errs, int32_t* status);

/* Device statistics of the calling thread's most recent sdft_solve /
 * sdft_solve_batch: CUDA-event time of its kernel launches on the launch
 * stream (ms), number of kernel launches, and per request the device time
 * from its first to its last iteration (%globaltimer, ms; n entries).
 * No reference counterpart: measurement support for the batched solve. */
int sdft_last_batch_stats(double* device_ms, int32_t* launches, double* latency_ms, int32_t n);

/* Serving loop with continuous batching.  No reference counterpart: the
 * reference solves one request per process (iDFT.jl); these entry points keep
 * many requests resident on the GPU and admit new ones as slots free up.
 *
 * sdft_server_create: all requests of the server share `num`; at most
 *   max_slots requests are active at a time and, when max_bytes > 0, the sum of
 *   their device footprints (sdft_request_sizes) stays within max_bytes.
 * sdft_server_submit: queue a request (it starts from its current state); the
 *   handle must stay alive until its completion has been polled.  A prepared
 *   request (sdft_request_prepare) is placed on the device only at admission,
 *   and only while the device's free memory less the server's reserve covers
 *   it: admission then follows the free HBM.  A finished request keeps its
 *   device memory until the caller destroys the handle, so a stream driver
 *   reads each result and destroys the request to make room for the queue.
 * sdft_server_set_reserve: device bytes that admission leaves free (default 0).
 * sdft_server_step: admit queued requests (first in, first out), run every
 *   active request for at most `iters` Anderson iterations in one launch, retire
 *   the finished ones; returns the counts still active and still queued.
 * sdft_server_poll: completions since the last poll (tag, sdft_status,
 *   iterations, final residual, device ms from first to last iteration). */
typedef struct sdft_server* sdft_server_t;
int sdft_server_create(const sdft_numerics* num, int32_t max_slots, int64_t max_bytes, sdft_server_t* out);
int sdft_server_destroy(sdft_server_t server);
int sdft_server_submit(sdft_server_t server, sdft_handle h, int64_t tag);
int sdft_server_step(sdft_server_t server, int32_t iters, int32_t* active, int32_t* queued);
int sdft_server_poll(sdft_server_t server, int64_t* tags, int32_t* status, int32_t* iters, double* errs,
                     double* device_ms, int32_t max, int32_t* n);
int sdft_server_set_reserve(sdft_server_t server, int64_t reserve_bytes);
/* sdft_server_set_pipeline: with on != 0, sdft_server_step returns once its
 * launch is queued, and the requests that finish in that launch are retired
 * (and reported by sdft_server_poll) at the next sdft_server_step, so that the
 * caller's host work between steps (preparing arrivals, reading results back)
 * overlaps the GPU.  A request's state does not depend on the mode.  Off by
 * default; turning it off collects the launch in flight. */
int sdft_server_set_pipeline(sdft_server_t server, int32_t on);

/* ---- bulk (iLST) state evaluation on the host --------------------------------
 * One evaluation of the bulk residual's expensive steps, for the host solve of
 * the bulk state that seeds every request (src/iLST/evaluation/objective/
 * residual_bulkstate.jl:26-35): eval_bulk_density! (eval_bulk_density.jl:9-22
 * with the freely-jointed / monomer-bead accumulate_densities!) followed by
 * bulk_chemical_potential (bulk_chemical_potential.jl:9-25).  Topologies are
 * general trees: per segment its parent (-1 for the root), children, and the
 * segments grouped by level (root level first). */
#define SDFT_BULK_IDEAL     1u
#define SDFT_BULK_MFMT      2u
#define SDFT_BULK_TPT1MFMT  4u
#define SDFT_BULK_MSA       8u
#define SDFT_BULK_TPT1MSA  16u

typedef struct sdft_bulk_species {
  int32_t n_seg, max_states, max_children, n_levels;
  int32_t monomerbead;           /* 1: monomer-bead model (state sum of segment 0) */
  const int32_t* n_states;       /* [n_seg] */
  const int32_t* states;         /* [n_seg * max_states] bead type of each state */
  const int32_t* parent;         /* [n_seg] */
  const int32_t* n_children;     /* [n_seg] */
  const int32_t* children;       /* [n_seg * max_children] */
  const int32_t* level_ptr;      /* [n_levels + 1] */
  const int32_t* level_segs;     /* [n_seg] */
} sdft_bulk_species;

typedef struct sdft_bulk_system {
  int32_t nb, mb, ns;
  uint32_t models;               /* SDFT_BULK_* bits */
  const double* diameter;        /* [nb] */
  const double* valence;         /* [nb] */
  const double* delta_muH;       /* [nb] */
  const int32_t* bond_types;     /* [2 * mb] sorted pairs */
  const sdft_bulk_species* species; /* [ns] */
  double bjerrum_length;
} sdft_bulk_system;

/* Inputs: species densities [ns], mu_ex [nb] and lng [mb] of the previous
 * evaluation.  Outputs: segment densities (per species max_states x n_seg,
 * state index fastest, species after species), bead densities [nb], bond-end
 * densities [2 x mb] (row-major), mu_species [ns], the new mu_ex [nb] and lng
 * [mb], and the partition functions Xi [ns].  Host only; no device call. */
int sdft_bulk_eval(const sdft_bulk_system* sys, const double* rho_species, const double* mu_ex_in,
                   const double* lng_in, double* rho_segments, double* rho_beads, double* rho_bonds,
                   double* mu_species, double* mu_ex, double* lng, double* xi);

/* input.yaml to a request on the host, without a Julia or Python host.  No
 * single reference counterpart: this is the host pipeline of iDFT
 * (src/iDFT/iDFT.jl:24-40: YAML.load_file, iLST, geometry_system, setup_iDFT),
 * i.e. the molecular system (src/molecular_system/setup/setup_molsys.jl:48-75),
 * the bulk solve (src/iLST/evaluation/objective/solver_bulkstate.jl:31-104) and
 * the 1D slit with its fixed segments, restated in C++.
 * sdft_input_from_yaml: parses the text and builds the descriptor; errors come
 *   back as SDFT_ERR_ARG / SDFT_ERR_UNSUPPORTED with the reference's message in
 *   sdft_last_error().  Host only.  The reader takes the YAML the reference's
 *   inputs use (block and flow collections, plain and quoted scalars, comments,
 *   YAML.jl's exponent floats); a repeated key takes its last value, as in
 *   YAML.jl; tags, anchors, aliases and block scalars are refused with the line.
 * sdft_input_descriptor: the descriptor for sdft_request_create; it stays valid
 *   until sdft_input_destroy.
 * sdft_input_numerics: the numerical section with the defaults of
 *   AndersonMixing.jl:74-79.
 * sdft_input_bulk_stats: iterations and max-norm residual of the bulk solve. */
typedef struct sdft_input sdft_input;
int sdft_input_from_yaml(const char* yaml_text, sdft_input** out);
const sdft_system_desc* sdft_input_descriptor(const sdft_input* in);
int sdft_input_numerics(const sdft_input* in, sdft_numerics* out);
int sdft_input_bulk_stats(const sdft_input* in, int32_t* iterations, double* residual);
int sdft_input_destroy(sdft_input* in);

/* Bytes of the static device array behind sdft_objective_noalloc (16 MiB). */
#define SDFT_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)

/* One G(x) evaluation that allocates no device memory.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc, because their device
 * memory belongs to another allocator (a framework's caching pool, or a budget
 * reserved once at start-up) or because they cannot afford the implicit device
 * synchronisation a cudaMalloc may cause while other work is in flight.
 *  - x_dev, g_dev: the caller's device arrays of n = NP*(NB+2*MB+1)+1 doubles in
 *    the layout of sdft_objective (x read, G(x) written); g_dev 16-byte aligned
 *    (as cudaMalloc returns), x_dev 8-byte aligned, else SDFT_ERR_ARG.
 *  - Every other array (grid fields, weights, propagators, densities, spectra)
 *    lives in one static device array of SDFT_NOALLOC_SCRATCH_BYTES that each GPU
 *    loading the library holds until the process exits.  A system whose working
 *    set exceeds it is rejected with SDFT_ERR_ARG and a message giving both sizes
 *    (the plain slit, NP = 1024 with a 20-segment chain, needs about 3 MB).
 *  - Every call looks up the array's address in the current device's context
 *    (cudaGetSymbolAddress), uploads the system's tables from host memory and
 *    waits for its stream, so it cannot be called on a stream that is being
 *    captured into a CUDA graph.
 *  - All calls share the array and it keeps the last call's contents; each call
 *    clears the part it uses.  Calls that overlap on the GPU (other streams or
 *    host threads) race on it.
 *  - stream: a cudaStream_t, NULL for the default stream; the call waits for its
 *    own work on that stream before returning. */
int sdft_objective_noalloc(const sdft_system_desc* desc, const double* x_dev, double* g_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SOFTDFT_H */
