/*
 * oracle.c -- CPU FP64 restatement of the reference's iDFT solve.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for libsoftdft (parity tests, smoke
 * check, timed CPU baseline).  Parity status: UNPINNED (the Julia reference
 * cannot run here and ships no golden vectors); see oracle.h.
 *
 * Each function names the reference lines it restates (paths relative to the
 * reference project).  Indices are 0-based; the reference is 1-based.
 * Layouts follow the reference's column-major arrays with the grid index
 * fastest.  Convolutions use the reference's algorithm: mirror the true grid
 * into a doubled grid of NPS = 2*NP points, complex FFT, multiply by the
 * sampled analytic weight, inverse FFT (scaled by 1/NPS), real part.
 */
#include "oracle.h"

#include <complex.h>
#include <fenv.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PI 3.14159265358979323846

static _Thread_local char g_err[512];

static int fail(int code, const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return code;
}

const char* oracle_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------ */
/* FFT: iterative radix-2 for powers of two, Bluestein chirp-z otherwise.    */
/* Forward is unnormalised e^{-2 pi i k n / N}; inverse is scaled by 1/N,   */
/* matching FFTW's fft!/ifft! used through plan_fft!/plan_ifft!              */
/* (src/iDFT/coordinate_system/Cartesian/process_fourier.jl:39-40).         */
/* ------------------------------------------------------------------------ */
typedef struct fft_plan {
  int n;
  int pow2;
  int m;                 /* working radix-2 length (n or the Bluestein length) */
  double complex* tw;    /* m/2 twiddles e^{-2 pi i k / m} */
  double complex* chirp; /* n: e^{-i pi k^2 / n}        (Bluestein) */
  double complex* bhat;  /* m: FFT of the conjugate chirp (Bluestein) */
  double complex* work;  /* m */
} fft_plan;

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void fft_radix2(double complex* a, int m, const double complex* tw, int inverse) {
  for (int i = 1, j = 0; i < m; i++) {
    int bit = m >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double complex t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
  for (int len = 2; len <= m; len <<= 1) {
    int half = len >> 1, step = m / len;
    for (int i = 0; i < m; i += len) {
      for (int k = 0; k < half; k++) {
        double complex w = tw[k * step];
        if (inverse) w = conj(w);
        double complex u = a[i + k], v = a[i + k + half] * w;
        a[i + k] = u + v;
        a[i + k + half] = u - v;
      }
    }
  }
}

static int fft_plan_init(fft_plan* p, int n) {
  memset(p, 0, sizeof *p);
  p->n = n;
  p->pow2 = is_pow2(n);
  if (p->pow2) {
    p->m = n;
  } else {
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
  }
  p->tw = malloc(sizeof(double complex) * (size_t)(p->m / 2 + 1));
  p->work = malloc(sizeof(double complex) * (size_t)p->m);
  if (!p->tw || !p->work) return -1;
  for (int k = 0; k < p->m / 2; k++) {
    double a = -2.0 * PI * (double)k / (double)p->m;
    p->tw[k] = cos(a) + I * sin(a);
  }
  if (!p->pow2) {
    p->chirp = malloc(sizeof(double complex) * (size_t)n);
    p->bhat = calloc((size_t)p->m, sizeof(double complex));
    if (!p->chirp || !p->bhat) return -1;
    for (int k = 0; k < n; k++) {
      long long k2 = ((long long)k * k) % (2LL * n); /* exact phase reduction */
      double a = -PI * (double)k2 / (double)n;
      p->chirp[k] = cos(a) + I * sin(a);
    }
    p->bhat[0] = conj(p->chirp[0]);
    for (int k = 1; k < n; k++) p->bhat[k] = p->bhat[p->m - k] = conj(p->chirp[k]);
    fft_radix2(p->bhat, p->m, p->tw, 0);
  }
  return 0;
}

static void fft_plan_free(fft_plan* p) {
  free(p->tw);
  free(p->chirp);
  free(p->bhat);
  free(p->work);
}

/* in place; inverse includes the 1/n scaling */
static void fft_exec(fft_plan* p, double complex* a, int inverse) {
  int n = p->n;
  if (p->pow2) {
    fft_radix2(a, n, p->tw, inverse);
  } else {
    double complex* w = p->work;
    for (int k = 0; k < n; k++) {
      double complex c = inverse ? conj(p->chirp[k]) : p->chirp[k];
      w[k] = a[k] * c;
    }
    for (int k = n; k < p->m; k++) w[k] = 0;
    fft_radix2(w, p->m, p->tw, 0);
    if (inverse) {
      /* the inverse chirp transform uses conj(bhat) in the time domain, i.e.
         bhat of the conjugated chirp; conj(FFT(conj(b)))[k] = FFT(b)[-k] */
      for (int k = 0; k < p->m; k++) w[k] *= conj(p->bhat[(p->m - k) % p->m]);
    } else {
      for (int k = 0; k < p->m; k++) w[k] *= p->bhat[k];
    }
    fft_radix2(w, p->m, p->tw, 1);
    double sm = 1.0 / (double)p->m;
    for (int k = 0; k < n; k++) {
      double complex c = inverse ? conj(p->chirp[k]) : p->chirp[k];
      a[k] = w[k] * sm * c;
    }
  }
  if (inverse) {
    double s = 1.0 / (double)n;
    for (int k = 0; k < n; k++) a[k] *= s;
  }
}

/* ------------------------------------------------------------------------ */
/* system                                                                   */
/* ------------------------------------------------------------------------ */
typedef struct species_t {
  int n_seg, S, C;
  int* parent;
  int* n_states;
  int* states;          /* [seg*S + idx] */
  int* n_children;
  int* children;        /* [seg*C + idx] */
  int n_levels;
  int* level_start;     /* [n_levels+1] */
  int* level_seg;       /* segments grouped by level, ascending index */
  int* fixed;           /* [seg] grid index or -1 */
  int any_fixed;
  double fixed_density;
  double* max_distance; /* [n_seg*n_seg] */
  double mu_species;
  double lambda_fixed;
  double* rho_seg;      /* [(seg*S + idx)*NP + K] */
  double* gC;           /* (K, j, c, i, seg) */
  double* gP;           /* (K, j, i, seg) */
  int linear;           /* parent of segment g is g-1 */
  int* eC;              /* [seg] power-of-two exponent carried by the stored gC of seg */
  int* eP;              /* [seg] the same for gP */
  int scaled;           /* some exponent of this evaluation is non-zero */
} species_t;

struct oracle_sys {
  int NP, NPS, NB, MB, NS;
  double dz, H, lB;
  int hard, charged;
  double qw[2];
  double total_charge;
  double *sig, *z, *dmu;
  int* bonds;
  unsigned funcs;
  species_t* sp;
  int64_t n;
  double* x;            /* current unknowns */
  double *lambda, *Ext, *trapez;
  double *rho_beads, *rho_bonds;
  double complex *rho_beads_hat, *rho_bonds_hat, *mu_ex_hat, *lng_hat, *surf_hat, *f_hat;
  double* w_bond;       /* [u*NPS + k] */
  double* w_fmt;        /* [(j*3 + m)*NPS + k], m = 0 delta, 1 step, 2 vector */
  double* w_msa;        /* [j*NPS + k] */
  double* w_coul;
  double* filter;
  fft_plan plan;
  /* scratch */
  double *nai, *wtb, *dphi, *lngK, *wtrho;
  /* Anderson driver state kept between calls (checkpoint / resume): the ring
     buffers X (unknowns) and G (residuals G(x) - x) of depth hm, the
     iteration count, the Picard flag, the last residual and the LSQR warm start */
  double *hX, *hG;
  int hm;
  int32_t s_iter, s_use_picard;
  double s_err;
  double s_lam[64];
};

#define IDX_MU(o, K, j) ((size_t)(j) * (o)->NP + (K))
#define IDX_LNG(o, K, e, u) (((size_t)(u) * 2 + (e)) * (o)->NP + (K))

static double* x_mu(oracle_sys* o, double* x) { (void)o; return x; }
static double* x_lng(oracle_sys* o, double* x) { return x + (size_t)o->NP * o->NB; }
static double* x_psi(oracle_sys* o, double* x) { return x + (size_t)o->NP * (o->NB + 2 * o->MB); }
static double* x_psic(oracle_sys* o, double* x) { return x + (size_t)o->NP * (o->NB + 2 * o->MB + 1); }

static size_t gC_idx(const oracle_sys* o, const species_t* s, int K, int j, int c, int i, int seg) {
  return ((((size_t)seg * s->S + i) * s->C + c) * s->S + j) * o->NP + K;
}
static size_t gP_idx(const oracle_sys* o, const species_t* s, int K, int j, int i, int seg) {
  return (((size_t)seg * s->S + i) * s->S + j) * o->NP + K;
}

/* ------------------------------------------------------------------------ */
/* k-space weights: src/iDFT/coordinate_system/Cartesian/fourier_transforms */
/* ------------------------------------------------------------------------ */
static double kvec(int k, int N, double DR) {
  /* delta_func.jl:13-21: jv <= div(N,2) -> positive branch */
  if (k <= N / 2) return 2.0 * PI * (double)k / ((double)N * DR);
  return -2.0 * PI * (double)(N - k) / ((double)N * DR);
}

static void delta_func_fft(double* w, int N, double DR, double b) { /* delta_func.jl:1-31 */
  w[0] = 4.0 * PI * (b * b);
  for (int k = 1; k < N; k++) {
    double kv = kvec(k, N, DR);
    double d = sqrt(kv * kv);
    w[k] = 4.0 * PI * b * sin(b * d) / d;
  }
}

static void step_func_fft(double* w, int N, double DR, double b) { /* step_func.jl:1-35 */
  w[0] = (4.0 / 3.0) * PI * (b * b * b);
  for (int k = 1; k < N; k++) {
    double kv = kvec(k, N, DR);
    double d = sqrt(kv * kv);
    w[k] = 4.0 * PI * (sin(b * d) - b * d * cos(b * d)) / (d * d * d);
  }
}

static void vector_delta_func_fft(double* w, int N, double DR, double b) { /* vectored_delta_func.jl:1-44 */
  w[0] = 0.0;
  for (int k = 1; k < N; k++) {
    double kv = kvec(k, N, DR);
    double d = sqrt(kv * kv);
    w[k] = -4.0 * PI * (sin(b * d) - b * d * cos(b * d)) / (d * d * d) * kv;
  }
}

static void coul_func_fft(double* w, int N, double DR, double BJ) { /* coul_func_fft.jl:1-29 */
  w[0] = 0.0;
  for (int k = 1; k < N; k++) {
    double kv = kvec(k, N, DR);
    double t = (1.0 - cos(kv * DR)) / (DR * DR);
    w[k] = 2.0 * PI * BJ / t;
  }
}

static void make_filter(double* f, int N, double dz) { /* utilities/apply_filter.jl:15-41 */
  double kc = 0.5 * (PI / dz);
  for (int k = 0; k < N; k++) {
    int nn = k;
    if (nn > N / 2) nn -= N;
    double kd = 2.0 * PI * (double)nn / ((double)N * dz);
    double kk = sqrt(kd * kd);
    double t = kk / kc;
    double t2 = t * t;
    f[k] = exp(-(t2 * t2));
  }
}

/* apply_mirroring.jl:1-23 with the partner index NPS-1-K of mirrored.jl:50-53 */
static void mirror(const oracle_sys* o, double complex* f) {
  for (int K = 0; K < o->NP; K++) f[o->NPS - 1 - K] = f[K];
}

static int jround(double x) { return (int)nearbyint(x); } /* round(Int, x): ties to even */

/* external_fields/hard_walls.jl:6-46 and charged_walls.jl:7-57 */
static void eval_external_field(oracle_sys* o) {
  int NP = o->NP;
  for (size_t i = 0; i < (size_t)NP * o->NB; i++) {
    o->Ext[i] = 0.0;
    o->trapez[i] = 1.0;
  }
  for (int k = 0; k < o->NPS; k++) o->surf_hat[k] = 0.0;
  if (o->hard) {
    double lo_w = 0.0, hi_w = o->H;
    for (int K = 0; K < NP; K++) {
      int idx = K + 1;
      for (int j = 0; j < o->NB; j++) {
        double d = o->sig[j];
        int lo = jround((lo_w + d / 2.0) / o->dz) + 1;
        int hi = jround((hi_w - d / 2.0) / o->dz) + 1;
        size_t q = IDX_MU(o, K, j);
        if (idx < lo) {
          o->Ext[q] += 1.0e20;
          o->trapez[q] = 1.0;
        } else if (idx == lo) {
          o->trapez[q] = 0.5;
        }
        if (idx > hi) {
          o->Ext[q] += 1.0e20;
          o->trapez[q] = 1.0;
        } else if (idx == hi) {
          o->trapez[q] = 0.5;
        }
      }
    }
  }
  if (o->charged) {
    double pos[2] = {0.0, o->H};
    for (int K = 0; K < NP; K++) {
      for (int w = 0; w < 2; w++) {
        int gp = jround(pos[w] / o->dz) + 1;
        if (K + 1 == gp) o->surf_hat[K] += o->qw[w] * (1.0 / o->dz);
      }
    }
    mirror(o, o->surf_hat);
  }
  fft_exec(&o->plan, o->surf_hat, 0);
}

/* ------------------------------------------------------------------------ */
/* create / destroy                                                          */
/* ------------------------------------------------------------------------ */
static void species_free(species_t* s) {
  free(s->parent); free(s->n_states); free(s->states); free(s->n_children); free(s->children);
  free(s->level_start); free(s->level_seg); free(s->fixed); free(s->max_distance);
  free(s->rho_seg); free(s->gC); free(s->gP); free(s->eC); free(s->eP);
}

void oracle_destroy(oracle_sys* o) {
  if (!o) return;
  if (o->sp) {
    for (int u = 0; u < o->NS; u++) species_free(&o->sp[u]);
    free(o->sp);
  }
  free(o->sig); free(o->z); free(o->dmu); free(o->bonds); free(o->x);
  free(o->lambda); free(o->Ext); free(o->trapez); free(o->rho_beads); free(o->rho_bonds);
  free(o->rho_beads_hat); free(o->rho_bonds_hat); free(o->mu_ex_hat); free(o->lng_hat);
  free(o->surf_hat); free(o->f_hat); free(o->w_bond); free(o->w_fmt); free(o->w_msa);
  free(o->w_coul); free(o->filter); free(o->nai); free(o->wtb); free(o->dphi); free(o->lngK);
  free(o->wtrho);
  free(o->hX); free(o->hG);
  fft_plan_free(&o->plan);
  free(o);
}

int64_t oracle_n_unknowns(const oracle_sys* o) { return o->n; }

static int bond_index(const oracle_sys* o, int a, int b) {
  int lo = a < b ? a : b, hi = a < b ? b : a;
  for (int u = 0; u < o->MB; u++)
    if (o->bonds[2 * u] == lo && o->bonds[2 * u + 1] == hi) return u;
  return -1;
}

int oracle_create(const sdft_system_desc* d, oracle_sys** out) {
  if (!d || !out) return fail(SDFT_ERR_ARG, "null argument");
  if (d->abi_version != SDFT_ABI_VERSION) return fail(SDFT_ERR_ARG, "ABI version mismatch");
  if (d->np < 2 || d->nb < 1 || d->n_species < 1 || d->bin_width <= 0)
    return fail(SDFT_ERR_ARG, "invalid grid or species counts");
  oracle_sys* o = calloc(1, sizeof *o);
  if (!o) return fail(SDFT_ERR_OOM, "out of memory");
  o->NP = d->np;
  o->NPS = 2 * d->np;
  o->NB = d->nb;
  o->MB = d->mb;
  o->NS = d->n_species;
  o->dz = d->bin_width;
  o->H = d->length;
  o->lB = d->bjerrum_length;
  o->hard = d->hard_walls != 0;
  o->charged = d->charged_walls != 0;
  o->qw[0] = d->wall_charge[0];
  o->qw[1] = d->wall_charge[1];
  o->total_charge = o->charged ? d->wall_charge[0] + d->wall_charge[1] : 0.0;
  o->funcs = d->functionals;
  int NP = o->NP, NPS = o->NPS, NB = o->NB, MB = o->MB;
  o->sig = malloc(sizeof(double) * NB);
  o->z = malloc(sizeof(double) * NB);
  o->dmu = malloc(sizeof(double) * NB);
  o->bonds = malloc(sizeof(int) * (2 * MB + 2));
  memcpy(o->sig, d->diameter, sizeof(double) * NB);
  memcpy(o->z, d->valence, sizeof(double) * NB);
  memcpy(o->dmu, d->delta_muH, sizeof(double) * NB);
  for (int u = 0; u < 2 * MB; u++) o->bonds[u] = d->bond_types[u];
  o->n = (int64_t)NP * (NB + 2 * MB + 1) + 1;
  o->x = calloc((size_t)o->n, sizeof(double));
  o->lambda = calloc((size_t)NP * NB, sizeof(double));
  o->Ext = calloc((size_t)NP * NB, sizeof(double));
  o->trapez = calloc((size_t)NP * NB, sizeof(double));
  o->rho_beads = calloc((size_t)NP * NB, sizeof(double));
  o->rho_bonds = calloc((size_t)NP * 2 * MB + 1, sizeof(double));
  o->rho_beads_hat = calloc((size_t)NPS * NB, sizeof(double complex));
  o->rho_bonds_hat = calloc((size_t)NPS * 2 * MB + 1, sizeof(double complex));
  o->mu_ex_hat = calloc((size_t)NPS * NB, sizeof(double complex));
  o->lng_hat = calloc((size_t)NPS * 2 * MB + 1, sizeof(double complex));
  o->surf_hat = calloc((size_t)NPS, sizeof(double complex));
  o->f_hat = calloc((size_t)NPS, sizeof(double complex));
  o->w_bond = calloc((size_t)NPS * MB + 1, sizeof(double));
  o->w_fmt = calloc((size_t)NPS * 3 * NB, sizeof(double));
  o->w_msa = calloc((size_t)NPS * NB, sizeof(double));
  o->w_coul = calloc((size_t)NPS, sizeof(double));
  o->filter = calloc((size_t)NPS, sizeof(double));
  o->nai = calloc((size_t)NPS * 3 * NB, sizeof(double));
  o->wtb = calloc((size_t)NPS * 2 * MB + 1, sizeof(double));
  o->dphi = calloc((size_t)NPS * 3 * NB, sizeof(double));
  o->lngK = calloc((size_t)NPS * 2 * MB + 1, sizeof(double));
  o->wtrho = calloc((size_t)NPS * NB, sizeof(double));
  if (!o->x || !o->filter || !o->wtrho || fft_plan_init(&o->plan, NPS) != 0) {
    oracle_destroy(o);
    return fail(SDFT_ERR_OOM, "out of memory");
  }
  /* species */
  o->sp = calloc((size_t)o->NS, sizeof(species_t));
  for (int u = 0; u < o->NS; u++) {
    const sdft_species_desc* sd = &d->species[u];
    species_t* s = &o->sp[u];
    int n = sd->n_seg, S = sd->max_states;
    if (n < 1 || S < 1) { oracle_destroy(o); return fail(SDFT_ERR_ARG, "species with no segments or states"); }
    s->n_seg = n;
    s->S = S;
    s->parent = malloc(sizeof(int) * n);
    s->n_states = malloc(sizeof(int) * n);
    s->states = malloc(sizeof(int) * n * S);
    s->n_children = calloc((size_t)n, sizeof(int));
    s->fixed = malloc(sizeof(int) * n);
    for (int g = 0; g < n; g++) {
      s->parent[g] = sd->parent[g];
      s->n_states[g] = sd->n_states[g];
      for (int i = 0; i < S; i++) s->states[g * S + i] = sd->states[g * S + i];
      s->fixed[g] = sd->fixed_coord ? sd->fixed_coord[g] : -1;
      if (s->fixed[g] >= 0) s->any_fixed = 1;
      if (g == 0 && s->parent[g] != -1) { oracle_destroy(o); return fail(SDFT_ERR_ARG, "segment 0 must be the root"); }
      if (g > 0 && (s->parent[g] < 0 || s->parent[g] >= g)) { oracle_destroy(o); return fail(SDFT_ERR_ARG, "parents must precede children"); }
    }
    for (int g = 1; g < n; g++) s->n_children[s->parent[g]]++;
    int C = 1;
    for (int g = 0; g < n; g++) C = s->n_children[g] > C ? s->n_children[g] : C;
    s->C = C;
    s->children = malloc(sizeof(int) * n * C);
    int* cnt = calloc((size_t)n, sizeof(int));
    for (int g = 1; g < n; g++) {
      int p = s->parent[g];
      s->children[p * C + cnt[p]++] = g;
    }
    free(cnt);
    /* levels = depth (parse_topology.jl:41-44) */
    int* depth = malloc(sizeof(int) * n);
    int maxd = 0;
    for (int g = 0; g < n; g++) {
      depth[g] = g == 0 ? 0 : depth[s->parent[g]] + 1;
      maxd = depth[g] > maxd ? depth[g] : maxd;
    }
    s->n_levels = maxd + 1;
    s->level_start = calloc((size_t)s->n_levels + 1, sizeof(int));
    s->level_seg = malloc(sizeof(int) * n);
    for (int g = 0; g < n; g++) s->level_start[depth[g] + 1]++;
    for (int l = 0; l < s->n_levels; l++) s->level_start[l + 1] += s->level_start[l];
    int* fill = calloc((size_t)s->n_levels, sizeof(int));
    for (int g = 0; g < n; g++) s->level_seg[s->level_start[depth[g]] + fill[depth[g]]++] = g;
    free(fill);
    free(depth);
    s->fixed_density = sd->fixed_density;
    s->mu_species = sd->mu_species;
    s->lambda_fixed = 1.0;
    if (s->any_fixed) {
      if (!sd->max_distance) { oracle_destroy(o); return fail(SDFT_ERR_ARG, "fixed segments need max_distance"); }
      s->max_distance = malloc(sizeof(double) * n * n);
      memcpy(s->max_distance, sd->max_distance, sizeof(double) * n * n);
      if (s->fixed[0] < 0) { oracle_destroy(o); return fail(SDFT_ERR_UNSUPPORTED, "only segment 0 can be fixed"); }
      for (int g = 1; g < n; g++)
        if (s->fixed[g] >= 0) { oracle_destroy(o); return fail(SDFT_ERR_UNSUPPORTED, "only segment 0 can be fixed"); }
      if (n < 2) { oracle_destroy(o); return fail(SDFT_ERR_UNSUPPORTED, "a fixed species needs a free segment"); }
    }
    s->linear = 1;
    for (int g = 1; g < n; g++) s->linear &= s->parent[g] == g - 1;
    s->eC = calloc((size_t)n, sizeof(int));
    s->eP = calloc((size_t)n, sizeof(int));
    s->rho_seg = calloc((size_t)NP * S * n, sizeof(double));
    s->gC = calloc((size_t)NP * S * C * S * n, sizeof(double));
    s->gP = calloc((size_t)NP * S * S * n, sizeof(double));
    if (!s->rho_seg || !s->gC || !s->gP) { oracle_destroy(o); return fail(SDFT_ERR_OOM, "out of memory"); }
    for (int g = 0; g < n; g++) {
      if (g > 0)
        for (int i = 0; i < s->n_states[g]; i++)
          for (int j = 0; j < s->n_states[s->parent[g]]; j++)
            if (bond_index(o, s->states[g * S + i], s->states[s->parent[g] * S + j]) < 0) {
              oracle_destroy(o);
              return fail(SDFT_ERR_ARG, "bond missing from bond_types");
            }
    }
  }
  /* weights (process_propagators.jl:13-34, TPT1mfmt.jl:20-64, TPT1msa.jl:20-46, coulomb.jl:37-46) */
  double* tmp = malloc(sizeof(double) * NPS);
  for (int u = 0; u < MB; u++) {
    double sij = (o->sig[o->bonds[2 * u]] + o->sig[o->bonds[2 * u + 1]]) / 2.0;
    delta_func_fft(tmp, NPS, o->dz, sij);
    for (int k = 0; k < NPS; k++) o->w_bond[(size_t)u * NPS + k] = tmp[k] / (4.0 * PI * (sij * sij));
  }
  for (int j = 0; j < NB; j++) {
    double b = o->sig[j] / 2.0;
    delta_func_fft(o->w_fmt + ((size_t)j * 3 + 0) * NPS, NPS, o->dz, b);
    step_func_fft(o->w_fmt + ((size_t)j * 3 + 1) * NPS, NPS, o->dz, b);
    vector_delta_func_fft(o->w_fmt + ((size_t)j * 3 + 2) * NPS, NPS, o->dz, b);
    delta_func_fft(tmp, NPS, o->dz, b);
    for (int k = 0; k < NPS; k++) o->w_msa[(size_t)j * NPS + k] = tmp[k] / (4.0 * PI * (b * b));
  }
  free(tmp);
  coul_func_fft(o->w_coul, NPS, o->dz, o->lB);
  make_filter(o->filter, NPS, o->dz);
  eval_external_field(o);
  /* process_guess.jl:47-64: mu_ex_K = bulk mu_ex, lng_K = bulk lng, Psi = PsiC = 0 */
  for (int j = 0; j < NB; j++)
    for (int K = 0; K < NP; K++) o->x[IDX_MU(o, K, j)] = d->mu_ex_bulk[j];
  for (int u = 0; u < MB; u++)
    for (int e = 0; e < 2; e++)
      for (int K = 0; K < NP; K++) x_lng(o, o->x)[IDX_LNG(o, K, e, u) - 0] = d->lng_bulk[u];
  *out = o;
  return SDFT_OK;
}

int oracle_set_x(oracle_sys* o, const double* x) {
  memcpy(o->x, x, sizeof(double) * (size_t)o->n);
  return SDFT_OK;
}

int oracle_get_x(const oracle_sys* o, double* x) {
  memcpy(x, o->x, sizeof(double) * (size_t)o->n);
  return SDFT_OK;
}

int oracle_get_fields(const oracle_sys* o, double* ext, double* trapez) {
  if (ext) memcpy(ext, o->Ext, sizeof(double) * (size_t)o->NP * o->NB);
  if (trapez) memcpy(trapez, o->trapez, sizeof(double) * (size_t)o->NP * o->NB);
  return SDFT_OK;
}

/* ------------------------------------------------------------------------ */
/* propagators: species_model/freely_jointed (child, parent, handle_fixed, accumulate) */
/* ------------------------------------------------------------------------ */
static double normative_of(const oracle_sys* o, const species_t* s) {
  /* child_propagators.jl:41-50: prod over segments of (sum_states e^-dmuH)^(1/N) */
  double nv = 1.0;
  for (int l = s->n_levels - 1; l >= 0; l--) {
    for (int q = s->level_start[l]; q < s->level_start[l + 1]; q++) {
      int p = s->level_seg[q];
      double t = 0.0;
      for (int i = 0; i < s->n_states[p]; i++) t += exp(-o->dmu[s->states[p * s->S + i]]);
      nv *= pow(t, 1.0 / (double)s->n_seg);
    }
  }
  return nv;
}

/* get_bond_info (child_propagators.jl:204-215): bond, and which end each state is */
static void bond_info(const oracle_sys* o, int si, int sj, int* bond, int* pair_i, int* pair_j) {
  if (si <= sj) { *pair_i = 0; *pair_j = 1; }
  else { *pair_i = 1; *pair_j = 0; }
  *bond = bond_index(o, si, sj);
}

static double dist2(int K, int coord, double dz) {
  double d = (double)(K - coord) * dz;
  return d * d;
}

static double sum_gC_states(const oracle_sys* o, const species_t* s, int K, int c, int i, int seg) {
  double t = 0.0;
  for (int j = 0; j < s->S; j++) t += s->gC[gC_idx(o, s, K, j, c, i, seg)];
  return t;
}

/* calc_f_hat_child! (child_propagators.jl:187-193) */
static double f_child(const oracle_sys* o, const species_t* s, int K, int child, int idx_j, int state_j,
                      int pair_j, int bond) {
  const double* lng = o->x + (size_t)o->NP * o->NB;
  double f = exp(-o->lambda[IDX_MU(o, K, state_j)] + lng[IDX_LNG(o, K, pair_j, bond)] / 2.0);
  for (int gc = 0; gc < s->n_children[child]; gc++) f *= sum_gC_states(o, s, K, gc, idx_j, child);
  return f;
}

/* calc_f_hat_parent! (parent_propagators.jl:144-153), including its index quirk:
   the other-children factor reads gC[K, :, idx_j, oc, parent] (child-index and
   parent-state slots swapped) */
static int f_parent(const oracle_sys* o, const species_t* s, int K, int parent, int child, int idx_j,
                    int state_j, int pair_j, int bond, double* out) {
  const double* lng = o->x + (size_t)o->NP * o->NB;
  double f = exp(-o->lambda[IDX_MU(o, K, state_j)] + lng[IDX_LNG(o, K, pair_j, bond)] / 2.0);
  double sp = 0.0;
  for (int jj = 0; jj < s->S; jj++) sp += s->gP[gP_idx(o, s, K, jj, idx_j, parent)];
  f *= sp;
  for (int oc = 0; oc < s->n_children[parent]; oc++) {
    if (s->children[parent * s->C + oc] == child) continue;
    if (idx_j >= s->C || oc >= s->S) return fail(SDFT_ERR_UNSUPPORTED, "branched topology index out of range");
    f *= sum_gC_states(o, s, K, idx_j, oc, parent);
  }
  *out = f;
  return SDFT_OK;
}

static double get_renorm(double Dij) { return 2.0 * Dij; } /* 1D: child_propagators.jl:218-226 */

/* mirrored FFT convolution with the filtered bond kernel (child_propagators.jl:118-141) */
static void convolve_bond(oracle_sys* o, int bond) {
  mirror(o, o->f_hat);
  fft_exec(&o->plan, o->f_hat, 0);
  for (int k = 0; k < o->NPS; k++) o->f_hat[k] *= o->filter[k];
  for (int k = 0; k < o->NPS; k++) o->f_hat[k] *= o->w_bond[(size_t)bond * o->NPS + k];
  fft_exec(&o->plan, o->f_hat, 1);
}

/* Per-segment renormalisation (linear chains).  The reference scales chain
   propagators only by `normative`; products over ~100+ segments underflow
   (e^-700) and the density prefactor e^{mu_species} overflows.  When the largest
   propagator entry of a segment leaves [2^-400, 2^400] the segment's entries are
   divided by the power of two 2^e that brings the maximum into [0.5, 1) (an
   exact scaling) and e is carried; otherwise e = 0 and the arithmetic is the
   reference's.  Returns e. */
static int renormalise(double* a, size_t count) {
  double mx = 0.0;
  for (size_t q = 0; q < count; q++) mx = fmax(mx, fabs(a[q]));
  if (!(mx > 0.0) || !isfinite(mx)) return 0;
  if (mx >= 0x1p-400 && mx <= 0x1p400) return 0;
  int e;
  frexp(mx, &e);
  for (size_t q = 0; q < count; q++) a[q] = ldexp(a[q], -e);
  return e;
}

static void compute_child_propagators(oracle_sys* o, species_t* s) {
  int NP = o->NP, S = s->S;
  const double* lng = o->x + (size_t)NP * o->NB;
  double normative = normative_of(o, s);
  memset(s->gC, 0, sizeof(double) * (size_t)NP * S * s->C * S * s->n_seg);
  memset(s->eC, 0, sizeof(int) * (size_t)s->n_seg);
  for (int l = s->n_levels - 1; l >= 0; l--) {
    for (int q = s->level_start[l]; q < s->level_start[l + 1]; q++) {
      int parent = s->level_seg[q];
      for (int idx_i = 0; idx_i < s->n_states[parent]; idx_i++) {
        int state_i = s->states[parent * S + idx_i];
        if (s->fixed[parent] >= 0) {
          s->gC[gC_idx(o, s, s->fixed[parent], 0, 0, idx_i, parent)] = 1.0;
        } else {
          for (int K = 0; K < NP; K++) s->gC[gC_idx(o, s, K, 0, 0, idx_i, parent)] = 1.0;
        }
        for (int idx_c = 0; idx_c < s->n_children[parent]; idx_c++) {
          int child = s->children[parent * s->C + idx_c];
          for (int idx_j = 0; idx_j < s->n_states[child]; idx_j++) {
            int state_j = s->states[child * S + idx_j];
            int bond, pair_i, pair_j;
            bond_info(o, state_i, state_j, &bond, &pair_i, &pair_j);
            double Dij = (o->sig[state_i] + o->sig[state_j]) / 2.0;
            double renorm = get_renorm(Dij);
            double Dij2 = Dij * Dij;
            for (int k = 0; k < o->NPS; k++) o->f_hat[k] = 0.0;
            if (s->fixed[parent] >= 0) {
              int Kp = s->fixed[parent];
              size_t gi = gC_idx(o, s, Kp, idx_j, idx_c, idx_i, parent);
              if (s->fixed[child] >= 0) {
                int Kc = s->fixed[child];
                double f = f_child(o, s, Kc, child, idx_j, state_j, pair_j, bond);
                s->gC[gi] = fabs(f) * exp(lng[IDX_LNG(o, Kp, pair_i, bond)] / 2.0) / renorm / o->dz / normative;
              } else {
                s->gC[gi] = 0.0;
                for (int K1 = 0; K1 < NP; K1++) {
                  double d2 = dist2(K1, Kp, o->dz);
                  if (d2 <= Dij2) {
                    double f = f_child(o, s, K1, child, idx_j, state_j, pair_j, bond);
                    double t = fabs(f) * exp(lng[IDX_LNG(o, Kp, pair_i, bond)] / 2.0) * o->dz *
                               o->trapez[IDX_MU(o, K1, state_j)] / renorm;
                    if (fabs(d2 - Dij2) <= 1e-6) t /= 2.0;
                    s->gC[gi] += t / normative;
                  }
                }
              }
            } else if (s->fixed[child] >= 0) {
              int Kc = s->fixed[child];
              double f = f_child(o, s, Kc, child, idx_j, state_j, pair_j, bond);
              for (int K1 = 0; K1 < NP; K1++) {
                double d2 = dist2(K1, Kc, o->dz);
                if (d2 <= Dij2) {
                  size_t gi = gC_idx(o, s, K1, idx_j, idx_c, idx_i, parent);
                  s->gC[gi] = fabs(f) * exp(lng[IDX_LNG(o, K1, pair_i, bond)] / 2.0) / renorm / normative;
                  if (fabs(d2 - Dij2) <= 1e-6) s->gC[gi] /= 2.0;
                }
              }
            } else {
              for (int K = 0; K < NP; K++) {
                double f = f_child(o, s, K, child, idx_j, state_j, pair_j, bond);
                o->f_hat[K] = f * o->trapez[IDX_MU(o, K, state_j)];
              }
              convolve_bond(o, bond);
              for (int K = 0; K < NP; K++)
                s->gC[gC_idx(o, s, K, idx_j, idx_c, idx_i, parent)] =
                    fabs(creal(o->f_hat[K])) * exp(lng[IDX_LNG(o, K, pair_i, bond)] / 2.0) / normative;
            }
          }
        }
      }
      /* max-path-distance mask around fixed segments (child_propagators.jl:147-157) */
      for (int seg = 0; seg < s->n_seg; seg++) {
        if (s->fixed[seg] < 0) continue;
        double md = s->max_distance[(size_t)parent * s->n_seg + seg];
        double md2 = md * md;
        for (int K1 = 0; K1 < NP; K1++) {
          if (dist2(K1, s->fixed[seg], o->dz) > md2) {
            for (int i = 0; i < S; i++)
              for (int c = 0; c < s->C; c++)
                for (int j = 0; j < S; j++) s->gC[gC_idx(o, s, K1, j, c, i, parent)] = 0.0;
          }
        }
      }
      if (s->linear && s->n_children[parent] > 0) {
        int e = renormalise(s->gC + gC_idx(o, s, 0, 0, 0, 0, parent), (size_t)NP * S * s->C * S);
        s->eC[parent] = e + s->eC[parent + 1];
        if (e) s->scaled = 1;
      }
    }
  }
}

static int compute_parent_propagators(oracle_sys* o, species_t* s) {
  int NP = o->NP, S = s->S;
  const double* lng = o->x + (size_t)NP * o->NB;
  double normative = normative_of(o, s);
  memset(s->gP, 0, sizeof(double) * (size_t)NP * S * S * s->n_seg);
  memset(s->eP, 0, sizeof(int) * (size_t)s->n_seg);
  for (int l = 0; l < s->n_levels; l++) {
    for (int q = s->level_start[l]; q < s->level_start[l + 1]; q++) {
      int child = s->level_seg[q];
      for (int idx_i = 0; idx_i < s->n_states[child]; idx_i++) {
        int state_i = s->states[child * S + idx_i];
        if (s->fixed[child] >= 0) {
          s->gP[gP_idx(o, s, s->fixed[child], 0, idx_i, child)] = 1.0;
        } else {
          for (int K = 0; K < NP; K++) s->gP[gP_idx(o, s, K, 0, idx_i, child)] = 1.0;
        }
        int parent = s->parent[child];
        if (parent < 0) continue;
        for (int idx_j = 0; idx_j < s->n_states[parent]; idx_j++) {
          int state_j = s->states[parent * S + idx_j];
          int bond, pair_i, pair_j;
          bond_info(o, state_i, state_j, &bond, &pair_i, &pair_j);
          double Dij = (o->sig[state_i] + o->sig[state_j]) / 2.0;
          double Dij2 = Dij * Dij;
          double renorm = get_renorm(Dij);
          for (int k = 0; k < o->NPS; k++) o->f_hat[k] = 0.0;
          if (s->fixed[parent] >= 0) {
            int Kp = s->fixed[parent];
            double f;
            int rc = f_parent(o, s, Kp, parent, child, idx_j, state_j, pair_j, bond, &f);
            if (rc) return rc;
            for (int K1 = 0; K1 < NP; K1++) {
              double d2 = dist2(K1, Kp, o->dz);
              if (d2 <= Dij2) {
                size_t gi = gP_idx(o, s, K1, idx_j, idx_i, child);
                s->gP[gi] = fabs(f) * exp(lng[IDX_LNG(o, K1, pair_i, bond)] / 2.0) / renorm / normative;
                if (fabs(d2 - Dij2) <= 1e-6) s->gP[gi] /= 2.0;
              }
            }
          } else {
            for (int K = 0; K < NP; K++) {
              double f;
              int rc = f_parent(o, s, K, parent, child, idx_j, state_j, pair_j, bond, &f);
              if (rc) return rc;
              o->f_hat[K] = f * o->trapez[IDX_MU(o, K, state_j)];
            }
            convolve_bond(o, bond);
            for (int K = 0; K < NP; K++)
              s->gP[gP_idx(o, s, K, idx_j, idx_i, child)] =
                  fabs(creal(o->f_hat[K])) * exp(lng[IDX_LNG(o, K, pair_i, bond)] / 2.0) / normative;
          }
        }
      }
      for (int seg = 0; seg < s->n_seg; seg++) { /* parent_propagators.jl:127-138 */
        if (s->fixed[seg] < 0) continue;
        double md = s->max_distance[(size_t)child * s->n_seg + seg];
        double md2 = md * md;
        for (int K1 = 0; K1 < NP; K1++)
          if (dist2(K1, s->fixed[seg], o->dz) > md2)
            for (int i = 0; i < S; i++)
              for (int j = 0; j < S; j++) s->gP[gP_idx(o, s, K1, j, i, child)] = 0.0;
      }
      if (s->linear && child > 0) {
        int e = renormalise(s->gP + gP_idx(o, s, 0, 0, 0, child), (size_t)NP * S * S);
        s->eP[child] = e + s->eP[child - 1];
        if (e) s->scaled = 1;
      }
    }
  }
  return SDFT_OK;
}

/* handle_fixed.jl:1-120 -> norm; sets the species' mu to 0 when grafted.  With
   renormalised propagators lambda is computed from the scaled segment-1 entries;
   the carried exponent enters accumulate_densities through log_prefactor. */
static int handle_fixed(oracle_sys* o, species_t* s, double* norm_out) {
  int NP = o->NP, S = s->S;
  double normative = normative_of(o, s);
  double lam, norm;
  if (s->any_fixed) {
    norm = s->fixed_density;
    s->mu_species = 0.0;
    lam = 0.0;
    int parent = -1;
    for (int g = 0; g < s->n_seg; g++)
      if (s->fixed[g] < 0) { parent = g; break; }
    if (parent < 0) return fail(SDFT_ERR_ARG, "No non-fixed segment available for lambda normalization.");
    for (int K = 0; K < NP; K++) {
      for (int idx_i = 0; idx_i < s->n_states[parent]; idx_i++) {
        int state_i = s->states[parent * S + idx_i];
        double sp = 0.0;
        for (int jj = 0; jj < S; jj++) sp += s->gP[gP_idx(o, s, K, jj, idx_i, parent)];
        double contr = exp(-o->lambda[IDX_MU(o, K, state_i)]) * sp;
        double temp;
        if (s->n_children[parent] == 0) {
          /* handle_fixed.jl:55 reads gC[K, :, idx_i, 1, parent] */
          if (idx_i >= s->C) return fail(SDFT_ERR_UNSUPPORTED, "leaf normalisation index out of range");
          temp = sum_gC_states(o, s, K, idx_i, 0, parent);
        } else {
          temp = 0.0;
          for (int idx_c = 0; idx_c < s->n_children[parent]; idx_c++) {
            int child = s->children[parent * s->C + idx_c];
            double t1 = 0.0;
            for (int idx_j = 0; idx_j < s->n_states[child]; idx_j++) {
              double t2 = s->gC[gC_idx(o, s, K, idx_j, idx_c, idx_i, parent)];
              for (int oc = 0; oc < s->n_children[parent]; oc++)
                if (oc != idx_c) t2 *= sum_gC_states(o, s, K, oc, idx_i, parent);
              t1 += t2;
            }
            temp = t1;
          }
        }
        lam += contr * temp * o->trapez[IDX_MU(o, K, state_i)] * o->dz;
      }
    }
  } else {
    lam = 1.0;
    norm = pow(normative, (double)(s->n_seg - 1));
  }
  if (!isfinite(lam) || lam <= 0) return fail(SDFT_ERR_NORM, "Normalization error: lambda <= 0 or not finite");
  norm *= 1.0 / lam;
  lam /= pow(normative, (double)(s->n_seg - 1));
  s->lambda_fixed = lam;
  *norm_out = norm;
  return SDFT_OK;
}

/* ln of the density prefactor of segment g when propagators were renormalised:
   norm e^{mu} 2^{eP_g + eC_g} (free chains: norm = normative^(N-1); grafted:
   norm = density / lambda with lambda carrying 2^{eP_1 + eC_1}) */
static double log_prefactor(const species_t* s, double norm, double normative, int g) {
  int sg = s->eP[g] + (g < s->n_seg - 1 ? s->eC[g] : 0);
  if (s->any_fixed) {
    int s1 = s->eP[1] + (1 < s->n_seg - 1 ? s->eC[1] : 0);
    return log(norm) + s->mu_species + (double)(sg - s1) * 0.6931471805599453;
  }
  return s->mu_species + (double)(s->n_seg - 1) * log(normative) + (double)sg * 0.6931471805599453;
}

/* accumulate_densities! (accumulate_densities.jl:95-184) */
static void accumulate_densities(oracle_sys* o, species_t* s, double norm) {
  int NP = o->NP, S = s->S;
  double mu = s->mu_species;
  double normative = normative_of(o, s);
  for (int parent = 0; parent < s->n_seg; parent++) {
    for (int idx_i = 0; idx_i < s->n_states[parent]; idx_i++) {
      int state_i = s->states[parent * S + idx_i];
      double lp = s->scaled ? log_prefactor(s, norm, normative, parent) : 0.0;
      for (int K = 0; K < NP; K++) {
        double sp = 0.0;
        for (int jj = 0; jj < S; jj++) sp += s->gP[gP_idx(o, s, K, jj, idx_i, parent)];
        double contr = s->scaled ? exp(lp - o->lambda[IDX_MU(o, K, state_i)]) * sp
                                 : norm * exp(mu - o->lambda[IDX_MU(o, K, state_i)]) * sp;
        double temp;
        if (s->n_children[parent] == 0) {
          temp = sum_gC_states(o, s, K, 0, idx_i, parent);
        } else {
          temp = 0.0;
          for (int idx_c = 0; idx_c < s->n_children[parent]; idx_c++) {
            int child = s->children[parent * s->C + idx_c];
            double t1 = 0.0;
            for (int idx_j = 0; idx_j < s->n_states[child]; idx_j++) {
              int state_j = s->states[child * S + idx_j];
              int bond = bond_index(o, state_i, state_j);
              double t2 = s->gC[gC_idx(o, s, K, idx_j, idx_c, idx_i, parent)];
              for (int oc = 0; oc < s->n_children[parent]; oc++)
                if (oc != idx_c) t2 *= sum_gC_states(o, s, K, oc, idx_i, parent);
              o->rho_bonds[IDX_LNG(o, K, 0, bond)] += contr * t2;
              t1 += t2;
            }
            temp = t1;
          }
        }
        s->rho_seg[((size_t)parent * S + idx_i) * NP + K] += contr * temp;
      }
    }
  }
  for (int child = 0; child < s->n_seg; child++) {
    int parent = s->parent[child];
    if (parent < 0) continue;
    for (int idx_i = 0; idx_i < s->n_states[child]; idx_i++) {
      int state_i = s->states[child * S + idx_i];
      double lp = s->scaled ? log_prefactor(s, norm, normative, child) : 0.0;
      for (int K = 0; K < NP; K++) {
        double contr = s->scaled ? exp(lp - o->lambda[IDX_MU(o, K, state_i)])
                                 : norm * exp(mu - o->lambda[IDX_MU(o, K, state_i)]);
        for (int gc = 0; gc < s->n_children[child]; gc++) contr *= sum_gC_states(o, s, K, gc, idx_i, child);
        for (int idx_j = 0; idx_j < s->n_states[parent]; idx_j++) {
          int state_j = s->states[parent * S + idx_j];
          int bond = bond_index(o, state_i, state_j);
          o->rho_bonds[IDX_LNG(o, K, 1, bond)] += contr * s->gP[gP_idx(o, s, K, idx_j, idx_i, child)];
        }
      }
    }
  }
}

/* eval_spatial_density! (eval_spatial_density.jl:123-149) */
static int eval_spatial_density(oracle_sys* o) {
  int NP = o->NP;
  const double* mu_ex = o->x;
  const double* psi = x_psi(o, o->x);
  double psic = *x_psic(o, o->x);
  for (int u = 0; u < o->NS; u++)
    memset(o->sp[u].rho_seg, 0, sizeof(double) * (size_t)NP * o->sp[u].S * o->sp[u].n_seg);
  memset(o->rho_bonds, 0, sizeof(double) * (size_t)NP * 2 * o->MB);
  for (int K = 0; K < NP; K++) {
    double p = psi[K] + psic;
    for (int j = 0; j < o->NB; j++)
      o->lambda[IDX_MU(o, K, j)] = mu_ex[IDX_MU(o, K, j)] + p * o->z[j] + o->Ext[IDX_MU(o, K, j)] + o->dmu[j];
  }
  for (int u = 0; u < o->NS; u++) {
    species_t* s = &o->sp[u];
    s->scaled = 0;
    compute_child_propagators(o, s);
    int rc = compute_parent_propagators(o, s);
    if (rc) return rc;
    double norm;
    rc = handle_fixed(o, s, &norm);
    if (rc) return rc;
    /* the reference's prefactor norm e^{mu - lambda} overflows beyond e^709 */
    if (fabs(s->mu_species) + (double)(s->n_seg - 1) * fabs(log(normative_of(o, s))) > 600.0) s->scaled = 1;
    accumulate_densities(o, s, norm);
  }
  return SDFT_OK;
}

/* update_spatial_structures! (update_spatial_structures.jl:1-34) */
static void update_spatial_structures(oracle_sys* o) {
  int NP = o->NP;
  memset(o->rho_beads, 0, sizeof(double) * (size_t)NP * o->NB);
  for (int u = 0; u < o->NS; u++) {
    species_t* s = &o->sp[u];
    for (int g = 0; g < s->n_seg; g++) {
      for (int i = 0; i < s->n_states[g]; i++) {
        int st = s->states[g * s->S + i];
        const double* r = s->rho_seg + ((size_t)g * s->S + i) * NP;
        if (s->fixed[g] >= 0) {
          /* the reference reads coordinates[1][seg] for every fixed segment */
          int K = s->fixed[0];
          o->rho_beads[IDX_MU(o, K, st)] += r[K] / o->dz / o->trapez[IDX_MU(o, K, st)];
        } else {
          for (int K = 0; K < NP; K++) o->rho_beads[IDX_MU(o, K, st)] += r[K];
        }
      }
    }
  }
}

/* calc_rho_hat.jl:17-97 */
static void eval_rho_hat(oracle_sys* o) {
  int NP = o->NP, NPS = o->NPS;
  for (int j = 0; j < o->NB; j++) {
    for (int k = 0; k < NPS; k++) o->f_hat[k] = 0.0;
    for (int K = 0; K < NP; K++) o->f_hat[K] = o->rho_beads[IDX_MU(o, K, j)] * o->trapez[IDX_MU(o, K, j)];
    mirror(o, o->f_hat);
    fft_exec(&o->plan, o->f_hat, 0);
    memcpy(o->rho_beads_hat + (size_t)j * NPS, o->f_hat, sizeof(double complex) * NPS);
  }
  for (int u = 0; u < o->MB; u++) {
    for (int e = 0; e < 2; e++) {
      int bead = o->bonds[2 * u + e];
      for (int k = 0; k < NPS; k++) o->f_hat[k] = 0.0;
      for (int K = 0; K < NP; K++)
        o->f_hat[K] = o->rho_bonds[IDX_LNG(o, K, e, u)] * o->trapez[IDX_MU(o, K, bead)];
      mirror(o, o->f_hat);
      fft_exec(&o->plan, o->f_hat, 0);
      memcpy(o->rho_bonds_hat + ((size_t)u * 2 + e) * NPS, o->f_hat, sizeof(double complex) * NPS);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* pointwise functional formulas: src/iLST/free_energy (mfmt, msa, TPT1 variants)   */
/* ------------------------------------------------------------------------ */
/* compute_mfmt_deriv! (iLST/free_energy/excluded_volume/mfmt.jl:210-244); 1D:
   only vector component 1 is non-zero.  d[0..3] scalars, d[4] = dPhi/dnV1_x,
   d[5] = dPhi/dnV2_x */
static void mfmt_deriv(double n0, double n1, double n2, double n3, double nV1, double nV2, double* d) {
  double om = 1.0 - n3;
  double l1 = log(om);
  double i1 = 1.0 / om;
  double i3 = 1.0 / n3;
  double i36 = 1.0 / (36.0 * PI);
  double dot12 = nV1 * nV2, dot22 = nV2 * nV2;
  d[0] = -l1;
  d[1] = n2 * i1;
  d[2] = n1 * i1 + (n2 * n2 - dot22) * 3.0 * i36 * i3 * (l1 * i3 + i1 * i1);
  d[3] = n0 * i1 + (n1 * n2 - dot12) * (i1 * i1) -
         (l1 * (i3 * i3 * i3) * 2.0 * i36 + (i3 * i3) * i1 * i36 + (1.0 - 3.0 * n3) * (i3 * i3) * i36 * (i1 * i1 * i1)) *
             (n2 * n2 * n2 - 3.0 * n2 * dot22);
  d[4] = -nV2 * i1;
  d[5] = -nV1 * i1 - (l1 * i3 + i1 * i1) * n2 * nV2 * i3 * 6.0 * i36;
}

/* free_energy_mfmt (inhomogeneous, iLST mfmt.jl:103-117) */
static double free_energy_mfmt(double n0, double n1, double n2, double n3, double nV1, double nV2) {
  double om = 1.0 - n3;
  double lt = log(om);
  double inv_denom = 1.0 / (36.0 * PI * (n3 * n3) * (om * om));
  double dot12 = nV1 * nV2, dot22 = nV2 * nV2;
  return -n0 * lt + (n1 * n2 - dot12) / om + (n2 * n2 * n2 - 3.0 * n2 * dot22) * (n3 + (om * om) * lt) * inv_denom;
}

/* Gamma_msa (iLST/free_energy/electrostaticcorrelations/msa.jl:181-230) */
static int gamma_msa(const double* rho, const double* sig, const double* Z, int nb, double lB, double* G_,
                     double* eta_, double* H_) {
  const double tol = 1e-10;
  double s = 0.0;
  for (int j = 0; j < nb; j++) s += rho[j] * Z[j] * Z[j];
  double kappa = sqrt(4.0 * PI * lB * s);
  double G, eta, H, G1 = 0.0;
  if (kappa < tol) {
    *G_ = kappa / 2.0;
    *eta_ = 0.0;
    *H_ = 2.0 / PI;
    return 0;
  }
  double sr = 0.0, srs = 0.0, s3 = 0.0;
  for (int j = 0; j < nb; j++) {
    sr += rho[j] * sig[j];
    srs += rho[j];
    s3 += rho[j] * sig[j] * sig[j] * sig[j];
  }
  double sig_eff = sr / srs;
  double xx = sig_eff * sqrt(4.0 * PI * lB * s);
  G = (sqrt(1.0 + 2.0 * xx) - 1.0) / (2.0 * sig_eff);
  double term2 = 2.0 / PI * (1.0 - PI / 6.0 * s3);
  int it = 0;
  for (;;) {
    double hs = 0.0, es = 0.0;
    for (int j = 0; j < nb; j++) {
      hs += rho[j] * sig[j] * sig[j] * sig[j] / (1.0 + G * sig[j]);
      es += rho[j] * Z[j] * sig[j] / (1.0 + G * sig[j]);
    }
    H = hs + term2;
    eta = es / H;
    double gs = 0.0;
    for (int j = 0; j < nb; j++) {
      double a = Z[j] - eta * sig[j] * sig[j];
      gs += rho[j] * a * a / (1.0 + G * sig[j]) / (1.0 + G * sig[j]);
    }
    G1 = sqrt(PI * lB * gs);
    double Gn = 0.9 * G + 0.1 * G1;
    it++;
    if (fabs(G1 - G) < tol || it >= 1000) {
      G = Gn;
      break;
    }
    G = Gn;
  }
  *G_ = G;
  *eta_ = eta;
  *H_ = H;
  return it;
}

/* compute_msa_deriv! (msa.jl:147-155) for a given (G, eta) */
static void msa_deriv(const double* rho, const double* sig, const double* Z, int nb, double lB, double G,
                      double eta, double* dphi) {
  double us = 0.0;
  for (int j = 0; j < nb; j++)
    us += rho[j] * sig[j] * sig[j] * ((Z[j] - eta * sig[j] * sig[j]) / (1.0 + G * sig[j]) + Z[j]);
  us = -PI / 6 * us;
  for (int j = 0; j < nb; j++) {
    dphi[j] = -lB * (G * (Z[j] * Z[j]) / (1.0 + G * sig[j]) +
                     eta * sig[j] * ((2.0 * Z[j] - eta * (sig[j] * sig[j])) / (1.0 + G * sig[j]) + eta * (sig[j] * sig[j]) / 3.0) +
                     Z[j] * us);
  }
}

static double free_energy_msa(const double* rho, const double* sig, const double* Z, int nb, double lB) {
  double G, eta, H;
  gamma_msa(rho, sig, Z, nb, lB, &G, &eta, &H);
  double s = 0.0;
  for (int j = 0; j < nb; j++) s += rho[j] * Z[j] * (Z[j] * G + eta * sig[j]) / (1.0 + G * sig[j]);
  return (G * G * G) / (3.0 * PI) - lB * s;
}

/* compute_TPT1msa_deriv! (TPT1msa.jl:200-282); bonds2[(u*2+e)] */
static void tpt1msa_deriv(const oracle_sys* o, const double* rho, const double* bonds2, double* dphi, double* lng) {
  int nb = o->NB, mb = o->MB;
  const double *sig = o->sig, *Z = o->z;
  double lB = o->lB;
  double G, eta, H;
  gamma_msa(rho, sig, Z, nb, lB, &G, &eta, &H);
  msa_deriv(rho, sig, Z, nb, lB, G, eta, dphi);
  if (G == 0.0) { /* isapprox(G, 0.0) with default tolerances */
    for (int u = 0; u < mb; u++) {
      int i = o->bonds[2 * u], j = o->bonds[2 * u + 1];
      double sij = (sig[i] + sig[j]) / 2.0;
      lng[u] = -lB / sij * Z[i] * Z[j];
    }
    return;
  }
  for (int u = 0; u < mb; u++) {
    int i = o->bonds[2 * u], j = o->bonds[2 * u + 1];
    double sij = (sig[i] + sig[j]) / 2.0;
    double Xi = (Z[i] - eta * (sig[i] * sig[i])) / (1.0 + G * sig[i]);
    double Xj = (Z[j] - eta * (sig[j] * sig[j])) / (1.0 + G * sig[j]);
    lng[u] = -lB / sij * Xi * Xj;
  }
  double dfG = 0.0, dfe = 0.0, deG = 0.0, dHG = 0.0;
  for (int w = 0; w < nb; w++) {
    double a = Z[w] - eta * sig[w] * sig[w];
    double og = 1.0 + G * sig[w];
    dfG += rho[w] * sig[w] * a * a / og / og / og;
    dfe += rho[w] * sig[w] * sig[w] * a / og / og;
    deG += rho[w] * Z[w] * sig[w] * sig[w] / og / og;
    dHG += rho[w] * sig[w] * sig[w] * sig[w] * sig[w] / og / og;
  }
  dfG = -2.0 * PI * lB * dfG;
  dfe = -2.0 * PI * lB * dfe;
  deG = -1.0 / H * deG;
  double deH = -eta / H;
  dHG = -dHG;
  double detaG = deG + deH * dHG;
  double denom = 1.0 / (2.0 * G - dfe * detaG - dfG);
  for (int w = 0; w < nb; w++) {
    double inv = 1.0 / (1.0 + G * sig[w]);
    double Xw = (Z[w] - eta * (sig[w] * sig[w])) * inv;
    double dfr = PI * lB * (Xw * Xw);
    double der = sig[w] / H * Z[w] * inv;
    double dHr = (sig[w] * sig[w] * sig[w]) * (inv - 1.0 / 3.0);
    double dGr = (dfr + dfe * (der + dfe * deH * dHr)) * denom;
    double detar = detaG * dGr;
    for (int u = 0; u < mb; u++) {
      int i = o->bonds[2 * u], j = o->bonds[2 * u + 1];
      double sij = (sig[i] + sig[j]) / 2.0;
      double ii = 1.0 / (1.0 + G * sig[i]);
      double Xi = (Z[i] - eta * (sig[i] * sig[i])) * ii;
      double dXi = -((sig[i] * sig[i]) * ii * detar + sig[i] * Xi * ii * dGr);
      double ij = 1.0 / (1.0 + G * sig[j]);
      double Xj = (Z[j] - eta * (sig[j] * sig[j])) * ij;
      double dXj = -((sig[j] * sig[j]) * ij * detar + sig[j] * Xj * ij * dGr);
      dphi[w] += (bonds2[2 * u] + bonds2[2 * u + 1]) / 2.0 * lB / sij * (dXi * Xj + Xi * dXj);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* functionals: src/iDFT/functionals                                         */
/* ------------------------------------------------------------------------ */
static void inv_fft_real(oracle_sys* o, const double complex* a, const double* w, double complex wfac, int take_abs,
                         double* out) {
  for (int k = 0; k < o->NPS; k++) o->f_hat[k] = a[k] * (w[k] * wfac);
  fft_exec(&o->plan, o->f_hat, 1);
  for (int k = 0; k < o->NPS; k++) out[k] = take_abs ? fabs(creal(o->f_hat[k])) : creal(o->f_hat[k]);
}

/* nai (NPS, 3, NB): m=0 n2-type, 1 n3-type, 2 vector (TPT1mfmt.jl:67-103) */
static void fmt_bead_weighted(oracle_sys* o) {
  size_t NPS = (size_t)o->NPS;
  for (int j = 0; j < o->NB; j++) {
    for (int m = 0; m < 2; m++)
      inv_fft_real(o, o->rho_beads_hat + j * NPS, o->w_fmt + ((size_t)j * 3 + m) * NPS, 1.0, 1,
                   o->nai + ((size_t)j * 3 + m) * NPS);
    inv_fft_real(o, o->rho_beads_hat + j * NPS, o->w_fmt + ((size_t)j * 3 + 2) * NPS, I, 0,
                 o->nai + ((size_t)j * 3 + 2) * NPS);
  }
}

/* point-wise weighted densities with the n3 cap of TPT1mfmt.jl:135-160 */
static void fmt_point(const oracle_sys* o, int Ks, double* n0, double* n1, double* n2, double* n3, double* nV1,
                      double* nV2, double* n3sum) {
  size_t NPS = (size_t)o->NPS;
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0, v1 = 0, v2 = 0;
  for (int j = 0; j < o->NB; j++) {
    double s = o->sig[j];
    double w1 = o->nai[((size_t)j * 3 + 0) * NPS + Ks];
    double w2 = o->nai[((size_t)j * 3 + 1) * NPS + Ks];
    double w3 = o->nai[((size_t)j * 3 + 2) * NPS + Ks];
    a0 += w1 / (PI * (s * s));
    a1 += w1 / (2 * PI * s);
    a2 += w1;
    a3 += w2;
    v1 += w3 / (2 * PI * s);
    v2 += w3;
  }
  if (a3 > 0.95) {
    double fac = 0.95 / a3;
    a0 *= fac; a1 *= fac; a2 *= fac; a3 *= fac; v1 *= fac; v2 *= fac;
  }
  *n0 = a0; *n1 = a1; *n2 = a2; *n3 = a3; *nV1 = v1; *nV2 = v2;
  *n3sum = a3;
}

static void fmt_functional(oracle_sys* o, int tpt1) {
  int NPS = o->NPS, NB = o->NB, MB = o->MB;
  fmt_bead_weighted(o);
  if (tpt1) { /* bond weighted densities (TPT1mfmt.jl:106-133) */
    for (int u = 0; u < MB; u++)
      for (int e = 0; e < 2; e++) {
        int i = o->bonds[2 * u + e];
        double sc = 1.0 / (o->sig[i] * o->sig[i]) / PI;
        for (int k = 0; k < NPS; k++)
          o->f_hat[k] = o->rho_bonds_hat[((size_t)u * 2 + e) * NPS + k] * (o->w_fmt[((size_t)i * 3) * NPS + k] / (o->sig[i] * o->sig[i]) / PI);
        (void)sc;
        fft_exec(&o->plan, o->f_hat, 1);
        for (int k = 0; k < NPS; k++) o->wtb[((size_t)u * 2 + e) * NPS + k] = fabs(creal(o->f_hat[k]));
      }
  }
  /* point-wise derivative over the whole doubled grid (TPT1mfmt.jl:197-241) */
  double d[6];
  double* lngp = malloc(sizeof(double) * (MB + 1));
  for (int Ks = 0; Ks < NPS; Ks++) {
    double n0, n1, n2, n3, nV1, nV2, n3s;
    fmt_point(o, Ks, &n0, &n1, &n2, &n3, &nV1, &nV2, &n3s);
    for (int u = 0; u < MB; u++) lngp[u] = 0.0;
    if (n3s > 1e-10) {
      mfmt_deriv(n0, n1, n2, n3, nV1, nV2, d);
      if (tpt1) {
        double Xi = 1.0 - (nV2 * nV2) / (n2 * n2);
        if (Xi < 0.0) Xi = 0.0;
        double i1 = 1.0 / (1.0 - n3);
        double term2 = n2 * Xi / 4.0 * (i1 * i1);
        double term3 = (n2 * n2) * Xi / 72.0 * (i1 * i1 * i1);
        for (int u = 0; u < MB; u++) {
          int bi = o->bonds[2 * u], bj = o->bonds[2 * u + 1];
          double sij = (o->sig[bi] + o->sig[bj]) / 2;
          double tau = o->sig[bi] * o->sig[bj] / sij;
          double y = i1 + term2 * tau + term3 * (tau * tau);
          double dl2 = (tau / 4.0 * (i1 * i1) + n2 * (tau * tau) * (i1 * i1 * i1) / 36.0) / y;
          double dl3 = ((i1 * i1) + n2 * Xi / 2.0 * (i1 * i1 * i1) * tau +
                        (n2 * n2) * Xi / 24.0 * ((i1 * i1) * (i1 * i1)) * (tau * tau)) / y;
          double rb = o->wtb[((size_t)u * 2 + 0) * NPS + Ks] + o->wtb[((size_t)u * 2 + 1) * NPS + Ks];
          d[2] -= 0.5 * rb * dl2;
          d[3] -= 0.5 * rb * dl3;
          double dlv = -nV2 * (tau / (2.0 * n2) * (i1 * i1) + (tau * tau) / 36.0 * (i1 * i1 * i1)) / y;
          d[5] -= 0.5 * rb * dlv;
          lngp[u] = log(y);
        }
      }
    } else {
      for (int q = 0; q < 6; q++) d[q] = 0.0;
    }
    for (int j = 0; j < NB; j++) {
      double s = o->sig[j];
      o->dphi[((size_t)j * 3 + 0) * NPS + Ks] = d[0] / (PI * (s * s)) + d[1] / (2 * PI * s) + d[2];
      o->dphi[((size_t)j * 3 + 1) * NPS + Ks] = d[3];
      o->dphi[((size_t)j * 3 + 2) * NPS + Ks] = d[4] / (2 * PI * s) + d[5];
    }
    if (tpt1)
      for (int u = 0; u < MB; u++) {
        o->lngK[((size_t)u * 2 + 0) * NPS + Ks] = lngp[u];
        o->lngK[((size_t)u * 2 + 1) * NPS + Ks] = lngp[u];
      }
  }
  free(lngp);
  /* accumulate_mu_ex! (TPT1mfmt.jl:244-283) */
  for (int j = 0; j < NB; j++) {
    for (int m = 0; m < 3; m++) {
      for (int k = 0; k < NPS; k++) o->f_hat[k] = o->dphi[((size_t)j * 3 + m) * NPS + k];
      fft_exec(&o->plan, o->f_hat, 0);
      const double* w = o->w_fmt + ((size_t)j * 3 + m) * NPS;
      double complex fac = m < 2 ? 1.0 : -I;
      for (int k = 0; k < NPS; k++) o->mu_ex_hat[(size_t)j * NPS + k] += o->f_hat[k] * (fac * w[k]);
    }
  }
  if (tpt1) /* accumulate_lng! (TPT1mfmt.jl:286-313) */
    for (int u = 0; u < MB; u++)
      for (int e = 0; e < 2; e++) {
        int i = o->bonds[2 * u + e];
        for (int k = 0; k < NPS; k++) o->f_hat[k] = o->lngK[((size_t)u * 2 + e) * NPS + k];
        fft_exec(&o->plan, o->f_hat, 0);
        for (int k = 0; k < NPS; k++)
          o->lng_hat[((size_t)u * 2 + e) * NPS + k] +=
              o->f_hat[k] * (o->w_fmt[((size_t)i * 3) * NPS + k] / (PI * (o->sig[i] * o->sig[i])));
      }
}

static void msa_weighted(oracle_sys* o, int tpt1) {
  size_t NPS = (size_t)o->NPS;
  for (int j = 0; j < o->NB; j++)
    inv_fft_real(o, o->rho_beads_hat + j * NPS, o->w_msa + j * NPS, 1.0, 1, o->wtrho + j * NPS);
  if (tpt1)
    for (int u = 0; u < o->MB; u++)
      for (int e = 0; e < 2; e++) {
        int i = o->bonds[2 * u + e];
        inv_fft_real(o, o->rho_bonds_hat + ((size_t)u * 2 + e) * NPS, o->w_msa + i * NPS, 1.0, 1,
                     o->wtb + ((size_t)u * 2 + e) * NPS);
      }
}

static void msa_functional(oracle_sys* o, int tpt1) {
  int NPS = o->NPS, NB = o->NB, MB = o->MB;
  msa_weighted(o, tpt1);
  double* rho = malloc(sizeof(double) * NB);
  double* b2 = malloc(sizeof(double) * (2 * MB + 1));
  double* dp = malloc(sizeof(double) * NB);
  double* lg = malloc(sizeof(double) * (MB + 1));
  for (int Ks = 0; Ks < NPS; Ks++) {
    for (int j = 0; j < NB; j++) rho[j] = o->wtrho[(size_t)j * NPS + Ks];
    if (tpt1) {
      for (int q = 0; q < 2 * MB; q++) b2[q] = o->wtb[(size_t)q * NPS + Ks];
      tpt1msa_deriv(o, rho, b2, dp, lg);
      for (int u = 0; u < MB; u++) {
        o->lngK[((size_t)u * 2 + 0) * NPS + Ks] = lg[u];
        o->lngK[((size_t)u * 2 + 1) * NPS + Ks] = lg[u];
      }
    } else {
      double G, eta, H;
      gamma_msa(rho, o->sig, o->z, NB, o->lB, &G, &eta, &H);
      msa_deriv(rho, o->sig, o->z, NB, o->lB, G, eta, dp);
    }
    for (int j = 0; j < NB; j++) o->dphi[(size_t)j * NPS + Ks] = dp[j];
  }
  free(rho); free(b2); free(dp); free(lg);
  for (int j = 0; j < NB; j++) { /* accumulate_mu_ex! (TPT1msa.jl:159-175) */
    for (int k = 0; k < NPS; k++) o->f_hat[k] = o->dphi[(size_t)j * NPS + k];
    fft_exec(&o->plan, o->f_hat, 0);
    for (int k = 0; k < NPS; k++) o->mu_ex_hat[(size_t)j * NPS + k] += o->f_hat[k] * o->w_msa[(size_t)j * NPS + k];
  }
  if (tpt1) /* accumulate_lng! (TPT1msa.jl:178-205) */
    for (int u = 0; u < MB; u++)
      for (int e = 0; e < 2; e++) {
        int i = o->bonds[2 * u + e];
        for (int k = 0; k < NPS; k++) o->f_hat[k] = o->lngK[((size_t)u * 2 + e) * NPS + k];
        fft_exec(&o->plan, o->f_hat, 0);
        for (int k = 0; k < NPS; k++)
          o->lng_hat[((size_t)u * 2 + e) * NPS + k] += o->f_hat[k] * o->w_msa[(size_t)i * NPS + k];
      }
}

/* eval_mu_functionals (eval_mu_functional.jl:1-52) -> new mu_ex_K, lng_K */
static void eval_mu_functionals(oracle_sys* o, double* g) {
  int NP = o->NP, NPS = o->NPS;
  memset(o->mu_ex_hat, 0, sizeof(double complex) * (size_t)NPS * o->NB);
  memset(o->lng_hat, 0, sizeof(double complex) * (size_t)NPS * 2 * o->MB);
  if (o->funcs & SDFT_FUNC_MFMT) fmt_functional(o, 0);
  if (o->funcs & SDFT_FUNC_TPT1MFMT) fmt_functional(o, 1);
  if (o->funcs & SDFT_FUNC_MSA) msa_functional(o, 0);
  if (o->funcs & SDFT_FUNC_TPT1MSA) msa_functional(o, 1);
  for (int j = 0; j < o->NB; j++) {
    memcpy(o->f_hat, o->mu_ex_hat + (size_t)j * NPS, sizeof(double complex) * NPS);
    fft_exec(&o->plan, o->f_hat, 1);
    for (int K = 0; K < NP; K++) g[IDX_MU(o, K, j)] = creal(o->f_hat[K]);
  }
  double* gl = x_lng(o, g);
  for (int u = 0; u < o->MB; u++)
    for (int e = 0; e < 2; e++) {
      memcpy(o->f_hat, o->lng_hat + ((size_t)u * 2 + e) * NPS, sizeof(double complex) * NPS);
      fft_exec(&o->plan, o->f_hat, 1);
      for (int K = 0; K < NP; K++) gl[IDX_LNG(o, K, e, u)] = creal(o->f_hat[K]);
    }
}

/* solve_poisson_eq (coulomb.jl:96-125) */
static void solve_poisson(oracle_sys* o, double* psi_out) {
  int NPS = o->NPS;
  for (int k = 0; k < NPS; k++) o->f_hat[k] = o->surf_hat[k];
  for (int j = 0; j < o->NB; j++)
    for (int k = 0; k < NPS; k++) o->f_hat[k] += o->rho_beads_hat[(size_t)j * NPS + k] * o->z[j];
  for (int k = 0; k < NPS; k++) o->f_hat[k] *= o->w_coul[k];
  fft_exec(&o->plan, o->f_hat, 1);
  for (int K = 0; K < o->NP; K++) psi_out[K] = creal(o->f_hat[K]);
}

/* compute_neutrality_shift (neutrality_shift.jl:1-99) */
static double neutrality_shift(oracle_sys* o) {
  int NP = o->NP;
  double Qtot = o->total_charge;
  int NS = o->NS;
  double* num = calloc((size_t)NS, sizeof(double));
  double* chg = calloc((size_t)NS, sizeof(double));
  for (int u = 0; u < NS; u++) {
    species_t* s = &o->sp[u];
    for (int g = 0; g < s->n_seg; g++)
      for (int i = 0; i < s->n_states[g]; i++) {
        int st = s->states[g * s->S + i];
        const double* r = s->rho_seg + ((size_t)g * s->S + i) * NP;
        double nn;
        if (s->fixed[g] >= 0) {
          nn = r[s->fixed[0]];
        } else {
          nn = 0.0;
          for (int K = 0; K < NP; K++) nn += r[K] * o->trapez[IDX_MU(o, K, st)] * o->dz;
        }
        num[u] += nn;
        chg[u] += nn * o->z[st];
      }
    num[u] /= (double)s->n_seg;
    if (num[u] <= 0.0) chg[u] = 0.0;
    else chg[u] /= num[u];
  }
  for (int u = 0; u < NS; u++) {
    species_t* s = &o->sp[u];
    int has_fam = 0;
    for (int g = 0; g < s->n_seg; g++) has_fam |= s->n_states[g] > 1;
    if (has_fam || s->any_fixed) {
      Qtot += num[u] * chg[u];
      chg[u] = 0.0;
    }
  }
  double acc = 0.0;
  for (int u = 0; u < NS; u++) acc += num[u] * chg[u];
  double err = fabs(Qtot + acc);
  double tol = 1e-10, psi1 = 0.0, Cstar = exp(-psi1);
  int iter = 1;
  while (err > tol) {
    double fx = Qtot, fx1 = 0.0;
    for (int i = 0; i < NS; i++) {
      double t = pow(Cstar, chg[i]) * num[i] * chg[i];
      fx += t;
      fx1 -= t * chg[i];
    }
    err = fabs(fx);
    if (fabs(fx1) < 1e-10) break;
    double del = fmax(1.0, fabs(fx / fx1));
    psi1 -= fx / (fx1 * del);
    Cstar = exp(-psi1);
    iter++;
    if (iter > 1000) break;
  }
  free(num);
  free(chg);
  return psi1;
}

int oracle_objective(oracle_sys* o, double* g) {
  int rc = eval_spatial_density(o);
  if (rc) return rc;
  update_spatial_structures(o);
  eval_rho_hat(o);
  eval_mu_functionals(o, g);
  solve_poisson(o, x_psi(o, g));
  *x_psic(o, g) = *x_psic(o, o->x) + neutrality_shift(o);
  return SDFT_OK;
}

/* ------------------------------------------------------------------------ */
/* LSQR (Paige & Saunders 1982) with IterativeSolvers' defaults, warm start  */
/* ------------------------------------------------------------------------ */
static double nrm2(const double* a, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; i++) s += a[i] * a[i];
  return sqrt(s);
}

/* A is column-major m x nc (columns contiguous) */
static void lsqr(const double* A, int64_t m, int nc, const double* b, double* x, double* u, double* tmpm) {
  const double eps = 2.220446049250313e-16;
  double atol = sqrt(eps), btol = sqrt(eps), conlim = 1.0 / sqrt(eps);
  int64_t maxiter = m > nc ? m : nc;
  double ctol = conlim > 0 ? 1.0 / conlim : 0.0;
  double v[64], w[64], tmpn[64];
  for (int64_t r = 0; r < m; r++) {
    double ax = 0.0;
    for (int c = 0; c < nc; c++) ax += A[(size_t)c * m + r] * x[c];
    u[r] = b[r] - ax;
  }
  double alpha = 0.0, beta = nrm2(u, m);
  for (int c = 0; c < nc; c++) v[c] = 0.0;
  if (beta > 0) {
    for (int64_t r = 0; r < m; r++) u[r] /= beta;
    for (int c = 0; c < nc; c++) {
      double s = 0.0;
      for (int64_t r = 0; r < m; r++) s += A[(size_t)c * m + r] * u[r];
      v[c] = s;
    }
    alpha = nrm2(v, nc);
  }
  if (alpha > 0)
    for (int c = 0; c < nc; c++) v[c] /= alpha;
  for (int c = 0; c < nc; c++) w[c] = v[c];
  double arnorm = alpha * beta;
  if (arnorm == 0) return;
  double anorm = 0, acond = 0, ddnorm = 0, res2 = 0, xxnorm = 0, z = 0, sn2 = 0, cs2 = -1.0;
  double rhobar = alpha, phibar = beta, bnorm = beta;
  int64_t itn = 0;
  int istop = 0;
  while (itn < maxiter && istop == 0) {
    itn++;
    for (int64_t r = 0; r < m; r++) {
      double av = 0.0;
      for (int c = 0; c < nc; c++) av += A[(size_t)c * m + r] * v[c];
      tmpm[r] = av;
    }
    for (int64_t r = 0; r < m; r++) u[r] = -alpha * u[r] + tmpm[r];
    beta = nrm2(u, m);
    if (beta > 0) {
      for (int64_t r = 0; r < m; r++) u[r] /= beta;
      anorm = sqrt(anorm * anorm + alpha * alpha + beta * beta);
      for (int c = 0; c < nc; c++) {
        double s = 0.0;
        for (int64_t r = 0; r < m; r++) s += A[(size_t)c * m + r] * u[r];
        tmpn[c] = s;
      }
      for (int c = 0; c < nc; c++) v[c] = -beta * v[c] + tmpn[c];
      alpha = nrm2(v, nc);
      if (alpha > 0)
        for (int c = 0; c < nc; c++) v[c] /= alpha;
    }
    double rhobar1 = rhobar, psi = 0.0;
    double rho = sqrt(rhobar1 * rhobar1 + beta * beta);
    double cs = rhobar1 / rho, sn = beta / rho;
    double theta = sn * alpha;
    rhobar = -cs * alpha;
    double phi = cs * phibar;
    phibar = sn * phibar;
    double tau = sn * phi;
    double t1 = phi / rho, t2 = -theta / rho;
    double dk2 = 0.0;
    for (int c = 0; c < nc; c++) {
      double dk = w[c] / rho;
      dk2 += dk * dk;
      x[c] += t1 * w[c];
      w[c] = v[c] + t2 * w[c];
    }
    ddnorm += dk2;
    double delta = sn2 * rho, gambar = -cs2 * rho, rhs = phi - delta * z;
    double zbar = rhs / gambar;
    double xnorm = sqrt(xxnorm + zbar * zbar);
    double gamma = sqrt(gambar * gambar + theta * theta);
    cs2 = gambar / gamma;
    sn2 = theta / gamma;
    z = rhs / gamma;
    xxnorm += z * z;
    acond = anorm * sqrt(ddnorm);
    double res1 = phibar * phibar;
    res2 += psi * psi;
    double rnorm = sqrt(res1 + res2);
    arnorm = alpha * fabs(tau);
    double test1 = rnorm / bnorm;
    double test2 = (anorm * rnorm != 0) ? arnorm / (anorm * rnorm) : INFINITY;
    double test3 = acond != 0 ? 1.0 / acond : INFINITY;
    double t1b = test1 / (1.0 + anorm * xnorm / bnorm);
    double rtol = btol + atol * anorm * xnorm / bnorm;
    if (itn >= maxiter) istop = 7;
    if (1.0 + test3 <= 1.0) istop = 6;
    if (1.0 + test2 <= 1.0) istop = 5;
    if (1.0 + t1b <= 1.0) istop = 4;
    if (test3 <= ctol) istop = 3;
    if (test2 <= atol) istop = 2;
    if (test1 <= rtol) istop = 1;
  }
}

/* ring buffers of depth m, reallocated when m changes; 0 or an error status */
static int anderson_buffers(oracle_sys* o, int m) {
  if (o->hm == m && o->hX && o->hG) return SDFT_OK;
  free(o->hX); free(o->hG);
  o->hX = calloc((size_t)o->n * m, sizeof(double));
  o->hG = calloc((size_t)o->n * m, sizeof(double));
  o->hm = m;
  if (!o->hX || !o->hG) {
    free(o->hX); free(o->hG);
    o->hX = o->hG = NULL;
    o->hm = 0;
    return fail(SDFT_ERR_OOM, "out of memory");
  }
  return SDFT_OK;
}

static void anderson_reset(oracle_sys* o) {
  o->s_iter = 0;
  o->s_use_picard = 1;
  o->s_err = 1.0;
  memset(o->s_lam, 0, sizeof(o->s_lam));
}

/* One pass of the loop body of solver_function(::AndersonMixing, ...)
 * (AndersonMixing.jl:98-160) with cur = G(x) already evaluated: ring-buffer
 * column col = mod(iter - 1, m) (:102), residual, amix (:112-114), Picard step
 * (:123-125) or the least-squares step (:127-145).  Returns 0, or
 * SDFT_ERR_NONFINITE. */
static int anderson_update(oracle_sys* o, const sdft_numerics* num, const double* cur, double* tX, double* tG,
                           double* Xk, double* Gk, double* rhs, double* u, double* tmpm) {
  const int64_t n = o->n;
  const int m = o->hm;
  const int iter = ++o->s_iter;
  const int col = (iter - 1) % m;
  double* X = o->hX;
  double* G = o->hG;
  memcpy(Xk, o->x, sizeof(double) * n);
  double mx = 0.0;
  int finite = 1;
  for (int64_t k = 0; k < n; k++) {
    Gk[k] = cur[k] - Xk[k];
    X[(size_t)col * n + k] = Xk[k];
    G[(size_t)col * n + k] = Gk[k];
    double a = fabs(Gk[k]);
    if (!(a == a) || a == INFINITY) finite = 0;
    if (a > mx) mx = a;
  }
  if (!finite) {
    o->s_err = mx;
    return fail(SDFT_ERR_NONFINITE, "non-finite fixed-point residual");
  }
  double err = mx > 1e-20 ? mx : 1e-20;
  o->s_err = err;
  double amix = fmin(num->mixing_max, num->damping / err);
  if (iter < m || (err > num->switch_tole && o->s_use_picard)) {
    double c1 = 1.0 - amix, c2 = amix;
    for (int64_t k = 0; k < n; k++) o->x[k] = c1 * o->x[k] + c2 * cur[k];
  } else {
    o->s_use_picard = 0;
    int i = 0;
    for (int j = 0; j < m; j++) {
      if (j == col) continue;
      for (int64_t k = 0; k < n; k++) {
        tX[(size_t)i * n + k] = X[(size_t)j * n + k] - Xk[k];
        tG[(size_t)i * n + k] = G[(size_t)j * n + k] - Gk[k];
      }
      i++;
    }
    for (int64_t k = 0; k < n; k++) rhs[k] = -Gk[k];
    lsqr(tG, n, m - 1, rhs, o->s_lam, u, tmpm);
    for (int64_t k = 0; k < n; k++) {
      double sx = 0.0, sg = 0.0;
      for (int c = 0; c < m - 1; c++) {
        sx += tX[(size_t)c * n + k] * o->s_lam[c];
        sg += tG[(size_t)c * n + k] * o->s_lam[c];
      }
      double r = Xk[k] + sx + amix * (Gk[k] + sg);
      o->x[k] = 0.0 * Xk[k] + 1.0 * r;
    }
  }
  return SDFT_OK;
}

/* work vectors of one Anderson update */
typedef struct {
  double *cur, *tX, *tG, *Xk, *Gk, *rhs, *u, *tmpm;
} anderson_work;

static void work_free(anderson_work* w) {
  free(w->cur); free(w->tX); free(w->tG); free(w->Xk); free(w->Gk); free(w->rhs); free(w->u); free(w->tmpm);
}

static int work_alloc(anderson_work* w, int64_t n, int m) {
  w->cur = malloc(sizeof(double) * n);
  w->tX = calloc((size_t)n * (m - 1), sizeof(double));
  w->tG = calloc((size_t)n * (m - 1), sizeof(double));
  w->Xk = malloc(sizeof(double) * n);
  w->Gk = malloc(sizeof(double) * n);
  w->rhs = malloc(sizeof(double) * n);
  w->u = malloc(sizeof(double) * n);
  w->tmpm = malloc(sizeof(double) * n);
  if (!w->cur || !w->tX || !w->tG || !w->Xk || !w->Gk || !w->rhs || !w->u || !w->tmpm) {
    work_free(w);
    return fail(SDFT_ERR_OOM, "out of memory");
  }
  return SDFT_OK;
}

/* solver_function(::AndersonMixing, ...) (AndersonMixing.jl:56-169), continuing
 * from the state in o (iteration count, Picard flag, ring buffers, warm start) */
static int solve_loop(oracle_sys* o, const sdft_numerics* num, int32_t* iters, double* err_out, double* trace,
                      int32_t trace_len) {
  int m = num->anderm;
  if (m < 2 || m > 60) return fail(SDFT_ERR_ARG, "anderm must be in [2, 60]");
  if (o->hm != m) return fail(SDFT_ERR_ARG, "anderm differs from the solver state's");
  anderson_work w;
  int rc = work_alloc(&w, o->n, m);
  if (rc) return rc;
  while (o->s_iter < num->max_iters) {
    rc = oracle_objective(o, w.cur);
    if (rc) break;
    rc = anderson_update(o, num, w.cur, w.tX, w.tG, w.Xk, w.Gk, w.rhs, w.u, w.tmpm);
    if (rc) break;
    if (trace && o->s_iter <= trace_len) trace[o->s_iter - 1] = o->s_err;
    if (o->s_err < num->tole) break;
  }
  *iters = o->s_iter;
  *err_out = o->s_err;
  work_free(&w);
  if (rc) return rc;
  return (o->s_err < num->tole) ? SDFT_OK : SDFT_MAX_ITERS;
}

int oracle_solve_trace(oracle_sys* o, const sdft_numerics* num, int32_t* iters, double* err_out,
                       double* trace, int32_t trace_len) {
  int m = num->anderm;
  if (m < 2 || m > 60) return fail(SDFT_ERR_ARG, "anderm must be in [2, 60]");
  int rc = anderson_buffers(o, m);
  if (rc) return rc;
  memset(o->hX, 0, sizeof(double) * (size_t)o->n * m);
  memset(o->hG, 0, sizeof(double) * (size_t)o->n * m);
  anderson_reset(o);
  return solve_loop(o, num, iters, err_out, trace, trace_len);
}

int oracle_solve(oracle_sys* o, const sdft_numerics* num, int32_t* iters, double* err) {
  return oracle_solve_trace(o, num, iters, err, NULL, 0);
}

int oracle_solve_resume(oracle_sys* o, const sdft_numerics* num, int32_t* iters, double* err) {
  if (!o->hX) return fail(SDFT_ERR_ARG, "no solver state to resume");
  return solve_loop(o, num, iters, err, NULL, 0);
}

int oracle_get_solver_state(const oracle_sys* o, sdft_solver_state* st, double* hist_x, double* hist_g) {
  if (!o->hX) return fail(SDFT_ERR_ARG, "no solver state");
  memset(st, 0, sizeof(*st));
  st->anderm = o->hm;
  st->iter = o->s_iter;
  st->use_picard = o->s_use_picard;
  st->err = o->s_err;
  for (int c = 0; c < o->hm - 1 && c < 15; c++) st->lambdas[c] = o->s_lam[c];
  if (hist_x) memcpy(hist_x, o->hX, sizeof(double) * (size_t)o->n * o->hm);
  if (hist_g) memcpy(hist_g, o->hG, sizeof(double) * (size_t)o->n * o->hm);
  return SDFT_OK;
}

int oracle_set_solver_state(oracle_sys* o, const sdft_solver_state* st, const double* hist_x, const double* hist_g) {
  if (st->anderm < 2 || st->anderm > 16) return fail(SDFT_ERR_ARG, "anderm must be in [2, 16]");
  int rc = anderson_buffers(o, st->anderm);
  if (rc) return rc;
  anderson_reset(o);
  o->s_iter = st->iter;
  o->s_use_picard = st->use_picard;
  o->s_err = st->err;
  for (int c = 0; c < st->anderm - 1; c++) o->s_lam[c] = st->lambdas[c];
  size_t bytes = sizeof(double) * (size_t)o->n * st->anderm;
  if (hist_x) memcpy(o->hX, hist_x, bytes); else memset(o->hX, 0, bytes);
  if (hist_g) memcpy(o->hG, hist_g, bytes); else memset(o->hG, 0, bytes);
  return SDFT_OK;
}

int oracle_anderson_step(oracle_sys* o, const sdft_numerics* num, const double* g, double* err) {
  if (!o->hX || o->hm != num->anderm) return fail(SDFT_ERR_ARG, "anderm differs from the solver state's");
  anderson_work w;
  int rc = work_alloc(&w, o->n, num->anderm);
  if (rc) return rc;
  memcpy(w.cur, g, sizeof(double) * o->n);
  rc = anderson_update(o, num, w.cur, w.tX, w.tG, w.Xk, w.Gk, w.rhs, w.u, w.tmpm);
  *err = o->s_err;
  work_free(&w);
  return rc;
}

int oracle_get_densities(const oracle_sys* o, double* const* rho_segments, double* rho_beads, double* rho_bonds) {
  if (rho_segments)
    for (int u = 0; u < o->NS; u++)
      if (rho_segments[u])
        memcpy(rho_segments[u], o->sp[u].rho_seg, sizeof(double) * (size_t)o->NP * o->sp[u].S * o->sp[u].n_seg);
  if (rho_beads) memcpy(rho_beads, o->rho_beads, sizeof(double) * (size_t)o->NP * o->NB);
  if (rho_bonds) memcpy(rho_bonds, o->rho_bonds, sizeof(double) * (size_t)o->NP * 2 * o->MB);
  return SDFT_OK;
}

/* get_num_species (num_species.jl:1-38) */
int oracle_num_species(const oracle_sys* o, double* out) {
  int NP = o->NP;
  for (int u = 0; u < o->NS; u++) {
    const species_t* s = &o->sp[u];
    double acc = 0.0;
    for (int g = 0; g < s->n_seg; g++)
      for (int i = 0; i < s->n_states[g]; i++) {
        int st = s->states[g * s->S + i];
        const double* r = s->rho_seg + ((size_t)g * s->S + i) * NP;
        double nn;
        if (s->fixed[g] >= 0) {
          nn = r[s->fixed[0]];
        } else {
          nn = 0.0;
          for (int K = 0; K < NP; K++) nn += r[K] * o->trapez[IDX_MU(o, K, st)] * o->dz;
        }
        acc += nn / (double)s->n_seg;
      }
    out[u] = acc;
  }
  return SDFT_OK;
}

/* eval_fe_functional of each functional on the true domain
   (TPT1mfmt.jl:163-186, TPT1msa.jl:103-126, mfmt.jl, msa.jl) */
static double functional_free_energy(oracle_sys* o) {
  int NP = o->NP, NPS = o->NPS, NB = o->NB, MB = o->MB;
  double fe = 0.0;
  if (o->funcs & (SDFT_FUNC_MFMT | SDFT_FUNC_TPT1MFMT)) {
    for (int pass = 0; pass < 2; pass++) {
      int tpt1 = pass == 1;
      if (!(o->funcs & (tpt1 ? SDFT_FUNC_TPT1MFMT : SDFT_FUNC_MFMT))) continue;
      fmt_bead_weighted(o);
      if (tpt1)
        for (int u = 0; u < MB; u++)
          for (int e = 0; e < 2; e++) {
            int i = o->bonds[2 * u + e];
            for (int k = 0; k < NPS; k++)
              o->f_hat[k] = o->rho_bonds_hat[((size_t)u * 2 + e) * NPS + k] *
                            (o->w_fmt[((size_t)i * 3) * NPS + k] / (o->sig[i] * o->sig[i]) / PI);
            fft_exec(&o->plan, o->f_hat, 1);
            for (int k = 0; k < NPS; k++) o->wtb[((size_t)u * 2 + e) * NPS + k] = fabs(creal(o->f_hat[k]));
          }
      for (int K = 0; K < NP; K++) {
        double n0, n1, n2, n3, nV1, nV2, n3s;
        fmt_point(o, K, &n0, &n1, &n2, &n3, &nV1, &nV2, &n3s);
        double f = free_energy_mfmt(n0, n1, n2, n3, nV1, nV2);
        if (tpt1) {
          double Xi = 1.0 - (nV2 * nV2) / (n2 * n2);
          double i1 = 1.0 / (1.0 - n3);
          double term2 = n2 * Xi / 4.0 * (i1 * i1);
          double term3 = (n2 * n2) * Xi / 72.0 * (i1 * i1 * i1);
          for (int u = 0; u < MB; u++) {
            int bi = o->bonds[2 * u], bj = o->bonds[2 * u + 1];
            double sij = (o->sig[bi] + o->sig[bj]) / 2;
            double tau = o->sig[bi] * o->sig[bj] / sij;
            double y = i1 + term2 * tau + term3 * (tau * tau);
            f -= 0.5 * (o->wtb[((size_t)u * 2) * NPS + K] + o->wtb[((size_t)u * 2 + 1) * NPS + K]) * log(y);
          }
        }
        fe += f;
      }
    }
  }
  for (int pass = 0; pass < 2; pass++) {
    int tpt1 = pass == 1;
    if (!(o->funcs & (tpt1 ? SDFT_FUNC_TPT1MSA : SDFT_FUNC_MSA))) continue;
    msa_weighted(o, tpt1);
    double* rho = malloc(sizeof(double) * NB);
    for (int K = 0; K < NP; K++) {
      for (int j = 0; j < NB; j++) rho[j] = o->wtrho[(size_t)j * NPS + K];
      double f = free_energy_msa(rho, o->sig, o->z, NB, o->lB);
      if (tpt1) {
        double G, eta, H;
        gamma_msa(rho, o->sig, o->z, NB, o->lB, &G, &eta, &H);
        for (int u = 0; u < MB; u++) {
          int i = o->bonds[2 * u], j = o->bonds[2 * u + 1];
          double sij = (o->sig[i] + o->sig[j]) / 2.0;
          double Xi = (o->z[i] - eta * (o->sig[i] * o->sig[i])) / (1.0 + G * o->sig[i]);
          double Xj = (o->z[j] - eta * (o->sig[j] * o->sig[j])) / (1.0 + G * o->sig[j]);
          double lng = -o->lB / sij * Xi * Xj;
          f -= 0.5 * (o->wtb[((size_t)u * 2) * NPS + K] + o->wtb[((size_t)u * 2 + 1) * NPS + K]) * lng;
        }
      }
      fe += f;
    }
    free(rho);
  }
  return fe;
}

/* grand_potential (grand_potential.jl:4-28) */
int oracle_grand_potential(oracle_sys* o, double* omega) {
  int NP = o->NP;
  double om = functional_free_energy(o);
  const double* mu = o->x;
  const double* lng = x_lng(o, o->x);
  for (size_t q = 0; q < (size_t)NP * o->NB; q++) om -= o->rho_beads[q] * mu[q] * o->trapez[q];
  for (size_t q = 0; q < (size_t)NP * 2 * o->MB; q++) om += o->rho_bonds[q] * lng[q] / 2.0;
  om *= o->dz;
  double* ns = malloc(sizeof(double) * o->NS);
  oracle_num_species(o, ns);
  for (int u = 0; u < o->NS; u++) om -= ns[u];
  free(ns);
  *omega = om;
  return SDFT_OK;
}
