/*
 * batch.c -- thread pool that runs independent oracle solves on the host
 * cores (TEST INFRASTRUCTURE: the timed CPU baseline of the batched
 * workloads).  Each solve is single-threaded, as the reference is; requests
 * are independent, so they are spread over threads.
 */
#include "oracle.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <unistd.h>

typedef struct {
  oracle_sys** sys;
  int32_t n;
  const sdft_numerics* num;
  int32_t *iters, *status;
  double* errs;
  atomic_int next;
} job_t;

static void* worker(void* arg) {
  job_t* j = (job_t*)arg;
  for (;;) {
    int i = atomic_fetch_add(&j->next, 1);
    if (i >= j->n) break;
    j->status[i] = oracle_solve(j->sys[i], j->num, &j->iters[i], &j->errs[i]);
  }
  return NULL;
}

int oracle_max_threads(void) {
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

int oracle_solve_many(oracle_sys** sys, int32_t n, const sdft_numerics* num, int32_t* iters, double* errs,
                      int32_t* status, int32_t threads) {
  if (threads <= 0) threads = oracle_max_threads();
  if (threads > n) threads = n;
  job_t job = {sys, n, num, iters, status, errs, 0};
  atomic_init(&job.next, 0);
  pthread_t* th = malloc(sizeof(pthread_t) * (size_t)(threads > 0 ? threads : 1));
  int started = 0;
  for (int t = 0; t < threads; t++)
    if (pthread_create(&th[t], NULL, worker, &job) == 0) started++;
  if (started == 0) worker(&job);
  for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
  free(th);
  return 0;
}
