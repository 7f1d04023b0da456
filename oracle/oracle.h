/*
 * oracle.h -- CPU FP64 restatement of the reference's iDFT solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the device solve
 * in libsoftdft: the parity tests, the smoke check and the timed CPU baseline
 * of bench.py link it.  Nothing in the product path calls it.
 *
 * Parity status: UNPINNED.  The reference is Julia; no Julia toolchain exists on
 * either machine and the reference ships no tests, fixtures or golden vectors.
 * The restatement follows the cited reference lines and is checked against
 * physics known-answer tests (bulk fixed point, ideal-chain limit, charge
 * neutrality, analytic weight integrals) in tests/.
 *
 * It takes the same sdft_system_desc as the device library and keeps the
 * reference's algorithm: every convolution is a complex FFT of the mirrored,
 * doubled grid NP* = 2*NP (src/iDFT/coordinate_system/Cartesian/process_fourier.jl:15-49).
 */
#ifndef SDFT_ORACLE_H
#define SDFT_ORACLE_H

#include "../include/softdft.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_sys oracle_sys;

int oracle_create(const sdft_system_desc* desc, oracle_sys** out);
void oracle_destroy(oracle_sys* o);
const char* oracle_last_error(void);
int64_t oracle_n_unknowns(const oracle_sys* o);

/* x = (mu_ex_K, lng_K, Psi, PsiC) flattened in the solver_dft order */
int oracle_set_x(oracle_sys* o, const double* x);
int oracle_get_x(const oracle_sys* o, double* x);
/* G(x) -> g (same flattening); x unchanged */
int oracle_objective(oracle_sys* o, double* g);
/* Anderson solve from the current x */
int oracle_solve(oracle_sys* o, const sdft_numerics* num, int32_t* iters, double* err);
int oracle_solve_trace(oracle_sys* o, const sdft_numerics* num, int32_t* iters, double* err,
                       double* err_trace, int32_t trace_len);

/* Anderson driver state (sdft_solver_state of softdft.h; hist_x / hist_g hold
 * anderm columns of n_unknowns in the flattening of x): read it after a solve,
 * set it to seed one, continue a solve from it, or take one driver iteration
 * with a given G(x) instead of evaluating it */
int oracle_get_solver_state(const oracle_sys* o, sdft_solver_state* st, double* hist_x, double* hist_g);
int oracle_set_solver_state(oracle_sys* o, const sdft_solver_state* st, const double* hist_x, const double* hist_g);
int oracle_solve_resume(oracle_sys* o, const sdft_numerics* num, int32_t* iters, double* err);
int oracle_anderson_step(oracle_sys* o, const sdft_numerics* num, const double* g, double* err);

int oracle_get_densities(const oracle_sys* o, double* const* rho_segments, double* rho_beads,
                         double* rho_bonds);
int oracle_grand_potential(oracle_sys* o, double* omega);
int oracle_num_species(const oracle_sys* o, double* num);
/* Ext and trapez (NP x NB), for tests */
int oracle_get_fields(const oracle_sys* o, double* ext, double* trapez);

/* batch.c: independent solves spread over host threads (threads <= 0: all cores) */
int oracle_solve_many(oracle_sys** sys, int32_t n, const sdft_numerics* num, int32_t* iters, double* errs,
                      int32_t* status, int32_t threads);
int oracle_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
