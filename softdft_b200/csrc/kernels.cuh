// kernels.cuh -- the solve kernels and their host launch wrappers.
//
// One CTA owns one request for a whole solve (k_solve): every stage of
// objective_dft and the Anderson update run back to back in that CTA, with the
// FFT workspace in shared memory and the request's fields in HBM/L2.  A batch
// is one launch with one CTA per request; requests of different sizes share the
// launch.
//
// This file is compiled twice, with SDFT_FFT_GEN = 0 (kernels_pow2.cu: grids
// whose FFT length M = NP/2 is a power of two) and SDFT_FFT_GEN = 1
// (kernels_gen.cu: any other M).  The kernels of the general build carry the
// suffix _gen; each build's CTAs return at once for requests of the other kind,
// so a mixed batch is one launch of each build over the same request array.
#pragma once

#include "anderson.cuh"
#include "common.cuh"
#include "objective.cuh"
#include "omega.cuh"

#if SDFT_FFT_GEN
#define SDFT_KNAME(x) x##_gen
#else
#define SDFT_KNAME(x) x
#endif
#define SDFT_KLAUNCH(x) SDFT_KLAUNCH2(x, SDFT_FFT_GEN)
#define SDFT_KLAUNCH2(x, g) SDFT_KLAUNCH3(x, g)
#define SDFT_KLAUNCH3(x, g) SDFT_KLAUNCH_##g(x)
#define SDFT_KLAUNCH_0(x) x##_pow2
#define SDFT_KLAUNCH_1(x) x##_gen

using namespace sdft;

__device__ __forceinline__ Shared make_shared(double* smem) {
  Shared sh;
  sh.red = smem;
  sh.z = reinterpret_cast<double2*>(smem + kRedDoubles);
  return sh;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

extern "C" __global__ void __launch_bounds__(kThreads) SDFT_KNAME(sdft_k_objective)(const DReq* reqs) {
  extern __shared__ double smem[];
  const DReq& r = reqs[blockIdx.x];
  if (r.gen != SDFT_FFT_GEN) return;
  Shared sh = make_shared(smem);
  bool ok = objective(r, sh, r.prec == 1);
  if (threadIdx.x == 0) *r.status = ok ? ST_OK : ST_NORM;
}

extern "C" __global__ void __launch_bounds__(kThreads, kSolveCtasPerSm)
    SDFT_KNAME(sdft_k_solve)(const DReq* reqs, SolveSlot* slots, SolveCfg cfg, int max_chunk) {
  extern __shared__ double smem[];
  const DReq& r = reqs[blockIdx.x];
  SolveSlot* sl = &slots[blockIdx.x];
  Shared sh = make_shared(smem);
  if (sl->status != ST_RUNNING || r.gen != SDFT_FFT_GEN) return;
  if (threadIdx.x == 0 && sl->iter == 0) sl->t0 = global_ns();
  AndersonState st;
  st.use_picard = sl->use_picard;
  for (int c = 0; c < kMaxAnderson; c++) st.lam[c] = sl->lam[c];
  // the request's transform buffers, free while the Anderson update runs
  const size_t zbytes = (size_t)r.zbytes;
  int iter = sl->iter;
  int status = ST_RUNNING;
  double err = sl->err;
  for (int step = 0; step < max_chunk && iter < cfg.max_iters; step++) {
    iter++;
    // mixed precision: FP32 propagators once the driver has left its Picard
    // phase (the first least-squares history is built from FP64 evaluations)
    // and while the residual is above the switch
    if (!objective(r, sh, r.prec == 1 && !st.use_picard && err > cfg.mixed_switch)) {
      status = ST_NORM;
      break;
    }
    int s = anderson_step(r, cfg, iter, st, sh.red, sh.z, zbytes, &err);
    if (s != ST_RUNNING) {
      status = s;
      break;
    }
  }
  if (status == ST_RUNNING && iter >= cfg.max_iters) status = ST_MAX_ITERS;
  if (threadIdx.x == 0) {
    sl->iter = iter;
    sl->status = status;
    sl->use_picard = st.use_picard;
    sl->err = err;
    sl->t1 = global_ns();
    for (int c = 0; c < kMaxAnderson; c++) sl->lam[c] = st.lam[c];
    *r.status = status;
    *r.iters = iter;
    *r.err = err;
  }
}

// one iteration of the Anderson driver with r.g = G(x) supplied by the caller
extern "C" __global__ void __launch_bounds__(kThreads) SDFT_KNAME(sdft_k_anderson)(const DReq* reqs, SolveSlot* slots,
                                                                                  SolveCfg cfg) {
  extern __shared__ double smem[];
  const DReq& r = reqs[blockIdx.x];
  SolveSlot* sl = &slots[blockIdx.x];
  if (r.gen != SDFT_FFT_GEN) return;
  AndersonState st;
  st.use_picard = sl->use_picard;
  for (int c = 0; c < kMaxAnderson; c++) st.lam[c] = sl->lam[c];
  const int iter = sl->iter + 1;
  double err = sl->err;
  const int s = anderson_step(r, cfg, iter, st, smem, nullptr, 0, &err);  // launched without transform buffers
  if (threadIdx.x == 0) {
    sl->iter = iter;
    sl->status = s;
    sl->use_picard = st.use_picard;
    sl->err = err;
    for (int c = 0; c < kMaxAnderson; c++) sl->lam[c] = st.lam[c];
  }
}

extern "C" __global__ void __launch_bounds__(kThreads) SDFT_KNAME(sdft_k_omega)(const DReq* reqs, double* out) {
  extern __shared__ double smem[];
  const DReq& r = reqs[blockIdx.x];
  if (r.gen != SDFT_FFT_GEN) return;
  Shared sh = make_shared(smem);
  grand_potential(r, sh, out);
}

// ---- host launch wrappers ----
namespace sdft {

static cudaError_t allow_smem(const void* fn, size_t smem) {
  if (smem > 48 * 1024) return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaSuccess;
}

cudaError_t SDFT_KLAUNCH(launch_objective)(const DReq* reqs, int n, size_t smem, cudaStream_t s) {
  cudaError_t e = allow_smem((const void*)SDFT_KNAME(sdft_k_objective), smem);
  if (e != cudaSuccess) return e;
  SDFT_KNAME(sdft_k_objective)<<<n, kThreads, smem, s>>>(reqs);
  return cudaGetLastError();
}

cudaError_t SDFT_KLAUNCH(launch_solve)(const DReq* reqs, SolveSlot* slots, SolveCfg cfg, int max_chunk, int n,
                                       size_t smem, cudaStream_t s) {
  cudaError_t e = allow_smem((const void*)SDFT_KNAME(sdft_k_solve), smem);
  if (e != cudaSuccess) return e;
  SDFT_KNAME(sdft_k_solve)<<<n, kThreads, smem, s>>>(reqs, slots, cfg, max_chunk);
  return cudaGetLastError();
}

cudaError_t SDFT_KLAUNCH(occupancy_solve)(size_t smem, int* ctas_per_sm) {
  cudaError_t e = allow_smem((const void*)SDFT_KNAME(sdft_k_solve), smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, SDFT_KNAME(sdft_k_solve), kThreads, smem);
}

cudaError_t SDFT_KLAUNCH(launch_anderson)(const DReq* reqs, SolveSlot* slots, SolveCfg cfg, cudaStream_t s) {
  SDFT_KNAME(sdft_k_anderson)<<<1, kThreads, sizeof(double) * kRedDoubles, s>>>(reqs, slots, cfg);
  return cudaGetLastError();
}

cudaError_t SDFT_KLAUNCH(launch_omega)(const DReq* reqs, double* out, size_t smem, cudaStream_t s) {
  cudaError_t e = allow_smem((const void*)SDFT_KNAME(sdft_k_omega), smem);
  if (e != cudaSuccess) return e;
  SDFT_KNAME(sdft_k_omega)<<<1, kThreads, smem, s>>>(reqs, out);
  return cudaGetLastError();
}

}  // namespace sdft
