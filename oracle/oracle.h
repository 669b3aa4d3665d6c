/*
 * oracle.h -- CPU restatement of calaman_G's matrix-exponential path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker the GPU path is
 * compared against (and the timed CPU baseline); it is never linked into, or
 * called by, the product library. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it.
 *
 * Everything is computed in FP64 (real double or complex double), whatever
 * precision the GPU tier runs in. For the single-precision tiers the caller
 * asks for the single-precision theta ladder (`single_theta` = 1), so the
 * oracle chooses the same (m, s) the float path chooses and then evaluates that
 * plan in double.
 *
 * What each function restates (paths relative to the calaman_G project):
 *   oracle_pade_theta / oracle_expm_plan   src/expm/plan.cppm:51-130
 *   oracle_pade_coeffs, num_powers/gemms  src/expm/expm_bridge.h:58-130
 *   oracle_norm1_{d,z}                    src/expm/norm1.cppm:45-56,
 *                                         src/expm/expm.cu:188-245 (true modulus,
 *                                         NaN-sticky max)
 *   oracle_pade_{d,z}                     src/expm/pade.cppm:77-191
 *   oracle_expm_{d,z}                     src/expm/expm.cppm:87-174
 *   oracle_ps_* / oracle_paterson_stockmeyer_d
 *                                         src/paterson_stockmeyer/interface.cppm:117-422,
 *                                         src/paterson_stockmeyer/paterson_stockmeyer.cu:51-85
 *   oracle_horner_d                       src/horner/interface.cppm:156-194,
 *                                         src/horner/horner.cu:39-67
 *   oracle_lacn2_{s,d}                    src/lapack/lacn2/interface.cppm:104-200
 *                                         (LAPACK xLACN2, 3.10+ sign test)
 *   oracle_getrf/getrs_{d,z}              LAPACK xGETRF/xGETRS semantics (the
 *                                         reference reaches cuSOLVER through
 *                                         WarpWraps, src/expm/pade.cppm:186-188):
 *                                         partial pivoting, first maximal
 *                                         |Re|+|Im| (LAPACK IxAMAX) as the pivot.
 *
 * Parity pinning: tests/test_oracle.py checks these functions against the
 * reference's own known answers (theta table, Pade coefficients, plan ladders,
 * PS cost table, buffer sizes, closed forms exp(0)=I, exp(diag), nilpotent
 * series, exp(A)exp(-A)=I, exp(A)=exp(A/2)^2, the degree ladder against r_13,
 * PS against the power series) and against tests/golden/ fixtures.
 *
 * Matrices are column-major. Complex values are interleaved (re, im) doubles,
 * i.e. C99 `double complex`.
 */
#ifndef CALAMAN_ORACLE_H
#define CALAMAN_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int m;
  int s;
  int num_gemms;
} oracle_expm_plan_t;

typedef struct {
  int s;
  int r;
  int num_powers;
  int num_blocks;
  int num_gemms;
} oracle_ps_plan_t;

/* Worker threads used by the GEMM / LU loops (1 = serial). Results do not
 * depend on the count: every output element is owned by one thread and summed
 * in a fixed order. */
void oracle_set_threads(int nthreads);
int oracle_get_threads(void);

/* ---- plan / tables ---------------------------------------------------- */
double oracle_pade_theta(int m, int single_theta);
oracle_expm_plan_t oracle_expm_plan(double norm1, int single_theta);
const double *oracle_pade_coeffs(int m); /* NULL off the ladder */
int oracle_pade_num_powers(int m);
int oracle_pade_num_gemms(int m);

int oracle_ps_cost(int degree, int s);
int oracle_ps_block_size(int degree);
oracle_ps_plan_t oracle_ps_plan(int degree, int s_requested);

/* ---- real double ------------------------------------------------------ */
double oracle_norm1_d(int n, const double *A, int lda);
void oracle_gemm_d(int m, int n, int k, double alpha, const double *A, int lda,
                   const double *B, int ldb, double beta, double *C, int ldc);
int oracle_getrf_d(int n, double *A, int lda, int *ipiv);
/* scaling half of ?gebal (src/lapack/gebal/gebal.cu:175-310); A overwritten
 * with D^-1 A D, scale = diag(D) */
int oracle_gebal_scale_d(int n, double *A, int lda, double *scale, int max_sweeps, int *sweeps);
int oracle_gebal_scale_z(int n, double *A, int lda, double *scale, int max_sweeps, int *sweeps);
int oracle_getrs_d(int n, int nrhs, const double *LU, int lda, const int *ipiv,
                   double *B, int ldb);
/* returns 0, or -1 for an invalid argument; *info gets the getrf info code */
int oracle_pade_d(int m, int n, const double *A, int lda, double *R, int ldr, int *info);
/* returns 0, -1 invalid argument, -2 non-finite norm */
int oracle_expm_d(int n, const double *A, int lda, double *E, int lde, int single_theta,
                  oracle_expm_plan_t *plan, int *info);

/* ---- complex double (interleaved re,im) -------------------------------- */
double oracle_norm1_z(int n, const double *A, int lda);
void oracle_gemm_z(int m, int n, int k, const double *alpha, const double *A, int lda,
                   const double *B, int ldb, const double *beta, double *C, int ldc);
int oracle_getrf_z(int n, double *A, int lda, int *ipiv);
int oracle_getrs_z(int n, int nrhs, const double *LU, int lda, const int *ipiv,
                   double *B, int ldb);
int oracle_pade_z(int m, int n, const double *A, int lda, double *R, int ldr, int *info);
int oracle_expm_z(int n, const double *A, int lda, double *E, int lde, int single_theta,
                  oracle_expm_plan_t *plan, int *info);

/* ---- matrix polynomials (real double) ---------------------------------- */
/* coeffs ascending: coeffs[k] multiplies A^k. Returns 0 or -1 (bad argument). */
int oracle_paterson_stockmeyer_d(int n, const double *coeffs, int degree, const double *A,
                                 int lda, double *P, int ldp, int s_requested);
int oracle_horner_d(int n, const double *coeffs, int degree, const double *A, int lda,
                    double *P, int ldp);

/* ---- 1-norm estimator by reverse communication (LAPACK xLACN2) --------
 * Start with *kase = 0; on a return with kase 1 (2) overwrite x with A x
 * (A^T x) and call again. kase 0 on return: *est <= ||A||_1, v = A w with
 * est = ||v||_1 / ||w||_1. isgn: n ints kept across calls; isave: 3 ints,
 * 1-based. Returns 0, or -1 for a bad argument or state. */
int oracle_lacn2_s(int n, float *v, float *x, int *isgn, float *est, int *kase, int *isave);
int oracle_lacn2_d(int n, double *v, double *x, int *isgn, double *est, int *kase, int *isave);

#ifdef __cplusplus
}
#endif

#endif /* CALAMAN_ORACLE_H */
