/*
 * oracle.c -- CPU restatement of calaman_G's matrix-exponential path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU library and the timed CPU
 * baseline. Never linked into the product. See oracle.h for the per-function
 * citations of the calaman_G sources this restates.
 *
 * Build: oracle/Makefile (gcc -O3 -std=c11 -fcx-limited-range, pthreads).
 * -std=c11 keeps floating-point contraction off, so the arithmetic is plain
 * IEEE double with a fixed evaluation order.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ---- a tiny static-partition parallel-for over pthreads ----------------- */

static int g_threads = 1;

void oracle_set_threads(int nthreads) { g_threads = nthreads < 1 ? 1 : nthreads; }
int oracle_get_threads(void) { return g_threads; }

typedef void (*range_fn)(void *ctx, int begin, int end);

typedef struct {
  range_fn fn;
  void *ctx;
  int begin, end;
} par_task;

static void *par_trampoline(void *arg) {
  par_task *t = (par_task *)arg;
  t->fn(t->ctx, t->begin, t->end);
  return NULL;
}

/* Run fn over [0, count) split into contiguous chunks, one per worker.
 * `serial` forces a single chunk (small problems are not worth a spawn). */
static void oracle_parallel_for(int count, int serial, range_fn fn, void *ctx) {
  int nt = g_threads;
  if (serial || nt <= 1 || count < 2) {
    fn(ctx, 0, count);
    return;
  }
  if (nt > count) nt = count;
  par_task *tasks = (par_task *)malloc(sizeof(par_task) * (size_t)nt);
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
  if (!tasks || !th) {
    free(tasks);
    free(th);
    fn(ctx, 0, count);
    return;
  }
  for (int t = 0; t < nt; ++t) {
    tasks[t].fn = fn;
    tasks[t].ctx = ctx;
    tasks[t].begin = (int)(((long long)count * t) / nt);
    tasks[t].end = (int)(((long long)count * (t + 1)) / nt);
  }
  int spawned = 1;
  for (int t = 1; t < nt; ++t, ++spawned) {
    if (pthread_create(&th[t], NULL, par_trampoline, &tasks[t]) != 0) break;
  }
  /* any task that could not get a thread runs here */
  for (int t = spawned; t < nt; ++t) fn(ctx, tasks[t].begin, tasks[t].end);
  fn(ctx, tasks[0].begin, tasks[0].end);
  for (int t = 1; t < spawned; ++t) pthread_join(th[t], NULL);
  free(tasks);
  free(th);
}

/* ---- Pade tables: b_j = (2m-j)! m! / ((2m)! j! (m-j)!) --------------------
 * The diagonal Pade coefficients of exp, normalised to b_0 = 1 (Higham 2005,
 * eq. 2.2; the same table as src/expm/expm_bridge.h:58-91). Spelled as exact
 * rationals; tests/test_oracle.py re-derives each one from the factorial
 * formula in exact arithmetic. */
static const double kB3[4] = {1.0, 1.0 / 2.0, 1.0 / 10.0, 1.0 / 120.0};
static const double kB5[6] = {1.0, 1.0 / 2.0, 1.0 / 9.0, 1.0 / 72.0, 1.0 / 1008.0, 1.0 / 30240.0};
static const double kB7[8] = {1.0,          1.0 / 2.0,     3.0 / 26.0,     5.0 / 312.0,
                              5.0 / 3432.0, 1.0 / 11440.0, 1.0 / 308880.0, 1.0 / 17297280.0};
static const double kB9[10] = {1.0,           1.0 / 2.0,         2.0 / 17.0,
                               7.0 / 408.0,   7.0 / 4080.0,      1.0 / 8160.0,
                               1.0 / 159120.0, 1.0 / 4455360.0,  1.0 / 196035840.0,
                               1.0 / 17643225600.0};
static const double kB13[14] = {1.0,
                                1.0 / 2.0,
                                3.0 / 25.0,
                                11.0 / 600.0,
                                11.0 / 5520.0,
                                3.0 / 18400.0,
                                1.0 / 96600.0,
                                1.0 / 1932000.0,
                                1.0 / 48944000.0,
                                1.0 / 1585785600.0,
                                1.0 / 67395888000.0,
                                1.0 / 3953892096000.0,
                                1.0 / 355850288640000.0,
                                1.0 / 64764752532480000.0};

const double *oracle_pade_coeffs(int m) {
  switch (m) {
  case 3: return kB3;
  case 5: return kB5;
  case 7: return kB7;
  case 9: return kB9;
  case 13: return kB13;
  default: return NULL;
  }
}

/* src/expm/expm_bridge.h:122-130 */
int oracle_pade_num_powers(int m) { return (m == 13) ? 3 : (m - 1) / 2; }
int oracle_pade_num_gemms(int m) { return oracle_pade_num_powers(m) + 1 + ((m == 13) ? 2 : 0); }

/* ---- theta_m and the plan, src/expm/plan.cppm:51-130 ---------------------
 * theta_m = the largest x with sum_{k>=2m+1} |h_k| x^(k-1) <= u, h(x) =
 * log(exp(-x) r_m(x)), for u = 2^-53 (double) and 2^-24 (single). The single
 * column is used as its float-rounded value, as a float computation sees it.
 * tests/golden/make_golden.py re-derives both columns by exact rational series
 * arithmetic and bisection; the fixture pins these constants. */
double oracle_pade_theta(int m, int single_theta) {
  if (single_theta) {
    switch (m) {
    case 3: return (double)4.258730034897931e-1f;
    case 5: return (double)1.880152698533769f;
    case 7: return (double)3.925724846433284f;
    case 9: return (double)6.249156334514102f;
    case 13: return (double)1.124873763647540e1f;
    default: return 0.0;
    }
  }
  switch (m) {
  case 3: return 1.495585217958292e-2;
  case 5: return 2.539398330063232e-1;
  case 7: return 9.504178996162932e-1;
  case 9: return 2.097847961257067;
  case 13: return 5.371920351148152;
  default: return 0.0;
  }
}

oracle_expm_plan_t oracle_expm_plan(double norm1, int single_theta) {
  static const int degrees[5] = {3, 5, 7, 9, 13};
  for (int i = 0; i < 5; ++i) {
    if (norm1 <= oracle_pade_theta(degrees[i], single_theta)) {
      oracle_expm_plan_t p = {degrees[i], 0, oracle_pade_num_gemms(degrees[i])};
      return p;
    }
  }
  const double theta = oracle_pade_theta(13, single_theta);
  int s = (int)ceil(log2(norm1 / theta));
  if (s < 0) s = 0;
  oracle_expm_plan_t p = {13, s, oracle_pade_num_gemms(13) + s};
  return p;
}

/* ---- Paterson-Stockmeyer plan, src/paterson_stockmeyer/interface.cppm:117-210 */
int oracle_ps_cost(int degree, int s) {
  if (s < 1 || degree < 1) return 0;
  const int r = degree / s;
  const int max_power = (r >= 1) ? s : degree;
  const int num_powers = (max_power >= 2) ? (max_power - 1) : 0;
  return num_powers + r;
}

int oracle_ps_block_size(int degree) {
  if (degree < 1) return 1;
  int best_s = 1, best = oracle_ps_cost(degree, 1);
  for (int s = 2; s <= degree + 1; ++s) {
    const int c = oracle_ps_cost(degree, s);
    if (c < best) {
      best = c;
      best_s = s;
    }
  }
  return best_s;
}

oracle_ps_plan_t oracle_ps_plan(int degree, int s_requested) {
  oracle_ps_plan_t p = {1, 0, 0, 0, 0};
  if (degree < 0) return p;
  int s = (s_requested > 0) ? s_requested : oracle_ps_block_size(degree);
  if (s > degree + 1) s = degree + 1;
  if (s < 1) s = 1;
  p.s = s;
  p.r = degree / s;
  const int max_power = (p.r >= 1) ? s : degree;
  p.num_powers = (max_power >= 2) ? (max_power - 1) : 0;
  p.num_blocks = p.num_powers + ((p.r >= 1) ? 1 : 0);
  p.num_gemms = p.num_powers + p.r;
  return p;
}

/* ---- the two element types ------------------------------------------- */
#define T double
#define SUF d
#define IS_CPLX 0
#include "oracle_impl.inc"
#undef T
#undef SUF
#undef IS_CPLX

#define T double complex
#define SUF z
#define IS_CPLX 1
#include "oracle_impl.inc"
#undef T
#undef SUF
#undef IS_CPLX

#define R float
#define SUF s
#include "oracle_lacn2.inc"
#undef R
#undef SUF

#define R double
#define SUF d
#include "oracle_lacn2.inc"
#undef R
#undef SUF

void oracle_gemm_d(int m, int n, int k, double alpha, const double *A, int lda, const double *B,
                   int ldb, double beta, double *C, int ldc) {
  gemm_impl_d(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

void oracle_gemm_z(int m, int n, int k, const double *alpha, const double *A, int lda,
                   const double *B, int ldb, const double *beta, double *C, int ldc) {
  const double complex a = alpha[0] + I * alpha[1];
  const double complex b = beta[0] + I * beta[1];
  gemm_impl_z(m, n, k, a, (const double complex *)A, lda, (const double complex *)B, ldb, b,
              (double complex *)C, ldc);
}

/* ---- Paterson-Stockmeyer evaluation ----------------------------------------
 * src/paterson_stockmeyer/interface.cppm:329-422 (power bank A^k = A^(k-1) A,
 * outer Horner over X = A^s with the block written first and the product
 * accumulated on top with beta = 1, parity chosen so the last step lands in P),
 * block build src/paterson_stockmeyer/paterson_stockmeyer.cu:51-85. */
static void ps_build_block(double *B, int ldb, int n, const double *A, int lda,
                           const double *powers, size_t stride, const double *c, int terms) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double acc = (i == j) ? c[0] : 0.0;
      if (terms > 1) acc = c[1] * A[i + (size_t)j * lda] + acc;
      for (int k = 2; k < terms; ++k) acc = c[k] * powers[(size_t)(k - 2) * stride + i + (size_t)j * n] + acc;
      B[i + (size_t)j * ldb] = acc;
    }
}

int oracle_paterson_stockmeyer_d(int n, const double *coeffs, int degree, const double *A, int lda,
                                 double *P, int ldp, int s_requested) {
  if (n < 1 || degree < 0 || lda < n || ldp < n || s_requested < 0) return -1;
  if (!coeffs || !A || !P) return -1;
  const oracle_ps_plan_t plan = oracle_ps_plan(degree, s_requested);
  const size_t nn = (size_t)n * n;
  const size_t stride = nn;
  double *powers = plan.num_powers > 0 ? (double *)malloc(sizeof(double) * nn * plan.num_powers) : NULL;
  double *scratch = plan.r >= 1 ? (double *)malloc(sizeof(double) * nn) : NULL;
  for (int k = 2; k <= plan.num_powers + 1; ++k) {
    const double *left = (k == 2) ? A : powers + (size_t)(k - 3) * stride;
    const int ldl = (k == 2) ? lda : n;
    gemm_impl_d(n, n, n, 1.0, left, ldl, A, lda, 0.0, powers + (size_t)(k - 2) * stride, n);
  }
  const double *X = plan.r < 1 ? NULL : (plan.s >= 2 ? powers + (size_t)(plan.s - 2) * stride : A);
  const int ldx = (plan.s >= 2) ? n : lda;
  double *buf[2] = {P, scratch};
  const int ld[2] = {ldp, n};
  int cur = (plan.r % 2 == 0) ? 0 : 1;
#define TERMS(j) ((degree - (j) * plan.s + 1) < plan.s ? (degree - (j) * plan.s + 1) : plan.s)
  ps_build_block(buf[cur], ld[cur], n, A, lda, powers, stride, coeffs + (size_t)plan.r * plan.s,
                 TERMS(plan.r));
  for (int j = plan.r - 1; j >= 0; --j) {
    const int next = 1 - cur;
    ps_build_block(buf[next], ld[next], n, A, lda, powers, stride, coeffs + (size_t)j * plan.s,
                   TERMS(j));
    gemm_impl_d(n, n, n, 1.0, buf[cur], ld[cur], X, ldx, 1.0, buf[next], ld[next]);
    cur = next;
  }
#undef TERMS
  free(powers);
  free(scratch);
  return 0;
}

/* ---- Horner evaluation, src/horner/interface.cppm:156-194 ------------------ */
int oracle_horner_d(int n, const double *coeffs, int degree, const double *A, int lda, double *P,
                    int ldp) {
  if (n < 1 || degree < 0 || lda < n || ldp < n) return -1;
  if (!coeffs || !A || !P) return -1;
  double *work = degree > 0 ? (double *)malloc(sizeof(double) * (size_t)n * n) : NULL;
  double *buf[2] = {P, work};
  const int ld[2] = {ldp, n};
  int cur = (degree % 2 == 0) ? 0 : 1;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) buf[cur][i + (size_t)j * ld[cur]] = (i == j) ? coeffs[degree] : 0.0;
  for (int k = degree - 1; k >= 0; --k) {
    const int next = 1 - cur;
    gemm_impl_d(n, n, n, 1.0, buf[cur], ld[cur], A, lda, 0.0, buf[next], ld[next]);
    cur = next;
    for (int i = 0; i < n; ++i) buf[cur][i * ((size_t)ld[cur] + 1)] += coeffs[k];
  }
  free(work);
  return 0;
}
