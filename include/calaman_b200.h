/*
 * calaman_b200.h -- C ABI of the B200-native matrix-exponential library.
 *
 * A drop-in for calaman_G's `calaman.expm`, `calaman.paterson_stockmeyer` and
 * `calaman.horner` C++23 modules. Every entry point below names the reference
 * interface it replaces (paths relative to the calaman_G project). The
 * reference's template functions are split into one symbol per element type:
 *   _s float   _d double   _c complex float (interleaved)   _z complex double
 * horner / paterson_stockmeyer exist for _s and _d only, as in the reference
 * (src/horner/instantiations.cpp, src/paterson_stockmeyer/instantiations.cpp).
 *
 * Conventions kept from the reference:
 *   - Column-major matrices; every leading dimension >= n.
 *   - The caller owns every buffer, including the workspace, which must be
 *     256-byte aligned and sized by the matching *_bufferSize query. The
 *     library allocates no device memory on these paths.
 *   - Only the n x n block of an output is written; padding rows between n
 *     and the leading dimension are left untouched.
 *   - Everything is stream ordered. expm synchronises its stream once (to
 *     read the 1-norm); pade, horner and paterson_stockmeyer never do.
 *   - Errors come back as calamanStatus_t {domain, code}: argument errors are
 *     rejected before any device work. expm/pade return INVALID_VALUE for bad
 *     arguments or a non-finite norm and ALLOC_FAILED for a short workspace;
 *     horner/paterson_stockmeyer return NOT_INITIALIZED for every argument
 *     error (src/expm/expm.cppm:94-102,122-124,
 *     src/paterson_stockmeyer/interface.cppm:333-345,
 *     src/horner/interface.cppm:160-164).
 *
 * The handle plays both roles of the reference's wwrblasHandle_t and
 * wwrsolverDnHandle_t: it carries the stream and the pointer mode.
 * Complex arguments are passed as pointers to interleaved (re, im) pairs.
 */
#ifndef CALAMAN_B200_H
#define CALAMAN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status (src/error_handling/error_handling.cppm:88-187) ------------ */
typedef enum {
  CALAMAN_DOMAIN_BLAS = 0,
  CALAMAN_DOMAIN_SOLVER = 1,
  CALAMAN_DOMAIN_RUNTIME = 2
} calamanErrorDomain_t;

/* BLAS-domain codes, numerically those of the CUDA backend's blas status. */
enum {
  CALAMAN_STATUS_SUCCESS = 0,
  CALAMAN_STATUS_NOT_INITIALIZED = 1,
  CALAMAN_STATUS_ALLOC_FAILED = 3,
  CALAMAN_STATUS_INVALID_VALUE = 7,
  CALAMAN_STATUS_ARCH_MISMATCH = 8,
  CALAMAN_STATUS_EXECUTION_FAILED = 13,
  CALAMAN_STATUS_INTERNAL_ERROR = 14,
  CALAMAN_STATUS_NOT_SUPPORTED = 15
};

typedef struct {
  int32_t domain; /* calamanErrorDomain_t */
  int32_t code;   /* 0 = success in every domain */
} calamanStatus_t;

/* ---- handle (replaces wwrblasHandle_t / wwrsolverDnHandle_t) ----------- */
typedef struct calamanContext *calamanHandle_t;
typedef calamanHandle_t calamanBlasHandle_t;
typedef calamanHandle_t calamanSolverHandle_t;
typedef void *calamanStream_t; /* a cudaStream_t */

enum { CALAMAN_POINTER_MODE_HOST = 0, CALAMAN_POINTER_MODE_DEVICE = 1 };

/* wwrblasFillMode_t: which triangle of a symmetric / Hermitian matrix is read
 * (numerically the CUDA backend's values). */
enum { CALAMAN_FILL_MODE_LOWER = 0, CALAMAN_FILL_MODE_UPPER = 1 };

/* wwrblasCreate / wwrsolverDnCreate: binds the current device, stream 0. */
calamanStatus_t calamanCreate(calamanHandle_t *handle);
calamanStatus_t calamanDestroy(calamanHandle_t handle);
/* wwrblasSetStream / wwrblasGetStream */
calamanStatus_t calamanSetStream(calamanHandle_t handle, calamanStream_t stream);
calamanStatus_t calamanGetStream(calamanHandle_t handle, calamanStream_t *stream);
/* wwrblasSetPointerMode / GetPointerMode; expm and pade save and restore it
 * (src/expm/expm.cppm:107-115). */
calamanStatus_t calamanSetPointerMode(calamanHandle_t handle, int mode);
calamanStatus_t calamanGetPointerMode(calamanHandle_t handle, int *mode);

/* Library version string and the sm_ target it was compiled for. */
const char *calamanGetVersion(void);

/* ---- plan (src/expm/plan.cppm:51-130) --------------------------------- */
typedef struct {
  int m;         /* Pade degree in {3, 5, 7, 9, 13} */
  int s;         /* squarings: the matrix is evaluated at A / 2^s */
  int num_gemms; /* matrix products the evaluation issues */
} calamanExpmPlan_t;

/* pade_theta<T>(m): backward-error threshold, 0 off the ladder. _s/_c use
 * the u = 2^-24 column, _d/_z the u = 2^-53 column. */
float calaman_pade_theta_s(int m);
double calaman_pade_theta_d(int m);
/* expm_plan<T>(norm1) */
calamanExpmPlan_t calaman_expm_plan_s(float norm1);
calamanExpmPlan_t calaman_expm_plan_d(double norm1);
/* pade_num_powers / pade_num_gemms (src/expm/expm_bridge.h:122-130) */
int calaman_pade_num_powers(int m);
int calaman_pade_num_gemms(int m);

/* ---- workspace queries (src/expm/buffer_size.cppm:47-97) --------------- */
calamanStatus_t calaman_expm_bufferSize_s(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_bufferSize_d(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_bufferSize_c(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_bufferSize_z(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_pade_bufferSize_s(calamanSolverHandle_t h, int m, int n, size_t *bytes);
calamanStatus_t calaman_pade_bufferSize_d(calamanSolverHandle_t h, int m, int n, size_t *bytes);
calamanStatus_t calaman_pade_bufferSize_c(calamanSolverHandle_t h, int m, int n, size_t *bytes);
calamanStatus_t calaman_pade_bufferSize_z(calamanSolverHandle_t h, int m, int n, size_t *bytes);

/* ---- expm (src/expm/expm.cppm:87-174) ----------------------------------
 * exp(A) by scaling and squaring with a diagonal Pade approximant (Higham
 * 2005, Algorithm 2.3). d_info: device array of 2 ints ([0] LU info, [1]
 * solve info). plan may be NULL. Synchronises `stream` once.
 * The _s/_c tiers run their dense products as split-BF16 tensor-core GEMMs
 * with FP32 accumulation; the 1-norm is always accumulated in FP64. */
calamanStatus_t calaman_expm_s(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                               calamanStream_t stream, int n, const float *d_A, int lda,
                               float *d_expA, int lde, void *d_work, size_t lwork_bytes,
                               int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_d(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                               calamanStream_t stream, int n, const double *d_A, int lda,
                               double *d_expA, int lde, void *d_work, size_t lwork_bytes,
                               int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_c(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                               calamanStream_t stream, int n, const void *d_A, int lda,
                               void *d_expA, int lde, void *d_work, size_t lwork_bytes,
                               int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_z(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                               calamanStream_t stream, int n, const void *d_A, int lda,
                               void *d_expA, int lde, void *d_work, size_t lwork_bytes,
                               int *d_info, calamanExpmPlan_t *plan);

/* ---- expm_vjp: the adjoint of expm --------------------------------------
 * New entry point: calaman_G has no derivative of expm. For a real loss
 * L(E), E = expm(A), d_G = dL/dE, writes d_gradA = dL/dA = L(A^H, G): the
 * Frechet derivative, at A^H in direction G, of the function expm evaluates
 * for A (r_m(X / 2^s)^(2^s) with (m, s) = expm_plan(||A||_1), returned in
 * *plan). A^T for the real types; the convention of torch.matrix_exp's
 * backward; equal to the upper-right n x n block of expm([[A^H, G], [0, A^H]]).
 * d_expA (may be NULL) receives expm(A) from the same evaluation. d_gradA may
 * overlap d_A or d_G. d_info: 2 ints as for expm. Synchronises `stream` once.
 * Work for m = 13: 19 + 3 s GEMMs, one LU, two n-RHS solves. */
calamanStatus_t calaman_expm_vjp_bufferSize_s(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_vjp_bufferSize_d(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_vjp_bufferSize_c(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_vjp_bufferSize_z(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_vjp_s(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                   calamanStream_t stream, int n, const float *d_A, int lda,
                                   const float *d_G, int ldg, float *d_gradA, int ldga,
                                   float *d_expA, int lde, void *d_work, size_t lwork_bytes,
                                   int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_vjp_d(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                   calamanStream_t stream, int n, const double *d_A, int lda,
                                   const double *d_G, int ldg, double *d_gradA, int ldga,
                                   double *d_expA, int lde, void *d_work, size_t lwork_bytes,
                                   int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_vjp_c(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                   calamanStream_t stream, int n, const void *d_A, int lda,
                                   const void *d_G, int ldg, void *d_gradA, int ldga,
                                   void *d_expA, int lde, void *d_work, size_t lwork_bytes,
                                   int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_vjp_z(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                   calamanStream_t stream, int n, const void *d_A, int lda,
                                   const void *d_G, int ldg, void *d_gradA, int ldga,
                                   void *d_expA, int lde, void *d_work, size_t lwork_bytes,
                                   int *d_info, calamanExpmPlan_t *plan);

/* ---- expm_batched: many small matrices in one call ----------------------
 * New entry point: calaman_G evaluates one matrix per call. exp(A_i) for
 * i < batch, every matrix with its own n_i (1 <= n_i <= 256; larger returns
 * CALAMAN_STATUS_NOT_SUPPORTED -- use calaman_expm_* for those), leading
 * dimensions and its own plan (m_i, s_i) = expm_plan(||A_i||_1), exactly the
 * plan calaman_expm_* picks for that matrix. h_n, h_lda, h_lde are host arrays;
 * h_A / h_expA are host arrays of device pointers. d_info: 2 * batch device
 * ints ([2i] LU info of matrix i, [2i + 1] solve info). h_plans (host, may be
 * NULL) receives every plan. Synchronises `stream` once (one readback of all
 * norms); a non-finite norm anywhere fails the whole call with
 * INVALID_VALUE before any output is written. The _s tier evaluates matrices
 * with s_i = 0 in FP32 and those with s_i > 0 wholly in FP64. When a batch
 * holds both, the FP64 ones run on a second stream that the blas handle
 * creates on first use (non-blocking, forked from and joined back to `stream`
 * within the call, released by calamanDestroy). */
calamanStatus_t calaman_expm_batched_bufferSize_s(calamanSolverHandle_t h, int batch,
                                                  const int *h_n, size_t *bytes);
calamanStatus_t calaman_expm_batched_bufferSize_d(calamanSolverHandle_t h, int batch,
                                                  const int *h_n, size_t *bytes);
calamanStatus_t calaman_expm_batched_s(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                       calamanStream_t stream, int batch, const int *h_n,
                                       const float *const *h_A, const int *h_lda,
                                       float *const *h_expA, const int *h_lde, void *d_work,
                                       size_t lwork_bytes, int *d_info, calamanExpmPlan_t *h_plans);
calamanStatus_t calaman_expm_batched_d(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                       calamanStream_t stream, int batch, const int *h_n,
                                       const double *const *h_A, const int *h_lda,
                                       double *const *h_expA, const int *h_lde, void *d_work,
                                       size_t lwork_bytes, int *d_info, calamanExpmPlan_t *h_plans);

/* ---- expm_vjp_batched: the adjoint over many small pairs ------------------
 * New entry point (no counterpart in the reference). calaman_expm_vjp_* for
 * every pair (A_i, G_i) of a batch, n_i <= 256 (larger: NOT_SUPPORTED), each
 * with its own plan (m_i, s_i) = expm_plan(||A_i||_1). Host arrays as for
 * calaman_expm_batched_*; h_expA may be NULL, or hold NULL entries, where
 * expm(A_i) is not wanted (h_lde is then only read where it is). d_info: 2 *
 * batch device ints. The _s tier evaluates pairs with s_i = 0 in FP32 and
 * pairs with s_i > 0 in FP64, like calaman_expm_batched_s. Synchronises
 * `stream` once. */
calamanStatus_t calaman_expm_vjp_batched_bufferSize_s(calamanSolverHandle_t h, int batch,
                                                      const int *h_n, size_t *bytes);
calamanStatus_t calaman_expm_vjp_batched_bufferSize_d(calamanSolverHandle_t h, int batch,
                                                      const int *h_n, size_t *bytes);
calamanStatus_t calaman_expm_vjp_batched_s(
    calamanBlasHandle_t blas, calamanSolverHandle_t solver, calamanStream_t stream, int batch,
    const int *h_n, const float *const *h_A, const int *h_lda, const float *const *h_G,
    const int *h_ldg, float *const *h_gradA, const int *h_ldga, float *const *h_expA,
    const int *h_lde, void *d_work, size_t lwork_bytes, int *d_info, calamanExpmPlan_t *h_plans);
calamanStatus_t calaman_expm_vjp_batched_d(
    calamanBlasHandle_t blas, calamanSolverHandle_t solver, calamanStream_t stream, int batch,
    const int *h_n, const double *const *h_A, const int *h_lda, const double *const *h_G,
    const int *h_ldg, double *const *h_gradA, const int *h_ldga, double *const *h_expA,
    const int *h_lde, void *d_work, size_t lwork_bytes, int *d_info, calamanExpmPlan_t *h_plans);

/* ---- balancing: the scaling half of gebal, and the balanced expm ---------
 * calaman_gebal_*: src/lapack/gebal/interface.cppm:100-255 (calaman::gebal).
 * job: 0 None, 1 Permute, 2 Scale, 3 Both (GebalJob order); only None and
 * Scale are built (Permute/Both return NOT_SUPPORTED). Overwrites A with
 * B = D^-1 A D (Parlett-Reinsch, powers of two, exact), d_scale (real, n) =
 * diag(D); *ilo = 1, *ihi = n. d_work: calaman_gebal_bufferSize ints.
 * max_sweeps <= 0 selects the default cap (1000); *sweeps (may be NULL)
 * receives the sweeps run. Synchronises `stream` once per sweep.
 * calaman_expm_balanced_*: new entry point composing the reference's
 * documented recipe (src/expm/README.md:100-122): exp(A) = D exp(B) D^-1.
 * Same arguments and results as calaman_expm_*; *plan is the plan of B. */
calamanStatus_t calaman_gebal_bufferSize(int n, int *lwork_ints);
calamanStatus_t calaman_gebal_s(calamanStream_t stream, int job, int n, float *d_A, int lda, int *ilo,
                                int *ihi, float *d_scale, int *d_work, int max_sweeps, int *sweeps);
calamanStatus_t calaman_gebal_d(calamanStream_t stream, int job, int n, double *d_A, int lda, int *ilo,
                                int *ihi, double *d_scale, int *d_work, int max_sweeps, int *sweeps);
calamanStatus_t calaman_gebal_c(calamanStream_t stream, int job, int n, void *d_A, int lda, int *ilo,
                                int *ihi, float *d_scale, int *d_work, int max_sweeps, int *sweeps);
calamanStatus_t calaman_gebal_z(calamanStream_t stream, int job, int n, void *d_A, int lda, int *ilo,
                                int *ihi, double *d_scale, int *d_work, int max_sweeps, int *sweeps);
calamanStatus_t calaman_expm_balanced_bufferSize_s(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_balanced_bufferSize_d(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_balanced_bufferSize_c(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_balanced_bufferSize_z(calamanSolverHandle_t h, int n, size_t *bytes);
calamanStatus_t calaman_expm_balanced_s(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                        calamanStream_t stream, int n, const float *d_A, int lda,
                                        float *d_expA, int lde, void *d_work, size_t lwork_bytes,
                                        int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_balanced_d(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                        calamanStream_t stream, int n, const double *d_A, int lda,
                                        double *d_expA, int lde, void *d_work, size_t lwork_bytes,
                                        int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_balanced_c(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                        calamanStream_t stream, int n, const void *d_A, int lda,
                                        void *d_expA, int lde, void *d_work, size_t lwork_bytes,
                                        int *d_info, calamanExpmPlan_t *plan);
calamanStatus_t calaman_expm_balanced_z(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                        calamanStream_t stream, int n, const void *d_A, int lda,
                                        void *d_expA, int lde, void *d_work, size_t lwork_bytes,
                                        int *d_info, calamanExpmPlan_t *plan);

/* ---- expm_herm: exp(A) for symmetric / Hermitian A by eigendecomposition --
 * src/expm/expm_herm.cppm:70-199 (calaman::expm_herm_bufferSize, expm_herm).
 * Reads only the `uplo` triangle of A (CALAMAN_FILL_MODE_*); exp(A) =
 * U diag(exp(w)) U^H from the library's own eigensolver. Never synchronises.
 * d_info: ONE device int, 0 on success (n + 1 if the eigensolver could not
 * complete). INVALID_VALUE for n < 1, n > 46340, lda/lde < n, a null
 * workspace or a bad uplo; ALLOC_FAILED for a short workspace. The single
 * tiers are solved in FP64 and rounded. */
calamanStatus_t calaman_expm_herm_bufferSize_s(calamanSolverHandle_t h, int uplo, int n, size_t *bytes);
calamanStatus_t calaman_expm_herm_bufferSize_d(calamanSolverHandle_t h, int uplo, int n, size_t *bytes);
calamanStatus_t calaman_expm_herm_bufferSize_c(calamanSolverHandle_t h, int uplo, int n, size_t *bytes);
calamanStatus_t calaman_expm_herm_bufferSize_z(calamanSolverHandle_t h, int uplo, int n, size_t *bytes);
calamanStatus_t calaman_expm_herm_s(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                    calamanStream_t stream, int uplo, int n, const float *d_A, int lda,
                                    float *d_expA, int lde, void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_expm_herm_d(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                    calamanStream_t stream, int uplo, int n, const double *d_A, int lda,
                                    double *d_expA, int lde, void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_expm_herm_c(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                    calamanStream_t stream, int uplo, int n, const void *d_A, int lda,
                                    void *d_expA, int lde, void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_expm_herm_z(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                                    calamanStream_t stream, int uplo, int n, const void *d_A, int lda,
                                    void *d_expA, int lde, void *d_work, size_t lwork_bytes, int *d_info);

/* ---- heevd: the symmetric / Hermitian eigensolver behind expm_herm -------
 * The reference's expm_herm calls the vendor syevd / heevd through WarpWraps
 * (src/expm/expm_herm.cppm:176-182); this is the library's own, with that
 * call's meaning: eigenvalues ascending into d_w (real, n), eigenvectors
 * overwrite A (columns, lda), only the `uplo` triangle is read. Tridiagonal
 * reduction, divide and conquer, compact-WY back-transformation, all on the
 * device; never synchronises. d_info: one device int as for expm_herm. */
calamanStatus_t calaman_heevd_bufferSize_s(int uplo, int n, size_t *bytes);
calamanStatus_t calaman_heevd_bufferSize_d(int uplo, int n, size_t *bytes);
calamanStatus_t calaman_heevd_bufferSize_c(int uplo, int n, size_t *bytes);
calamanStatus_t calaman_heevd_bufferSize_z(int uplo, int n, size_t *bytes);
calamanStatus_t calaman_heevd_s(calamanStream_t stream, int uplo, int n, float *d_A, int lda, float *d_w,
                                void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_heevd_d(calamanStream_t stream, int uplo, int n, double *d_A, int lda, double *d_w,
                                void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_heevd_c(calamanStream_t stream, int uplo, int n, void *d_A, int lda, float *d_w,
                                void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_heevd_z(calamanStream_t stream, int uplo, int n, void *d_A, int lda, double *d_w,
                                void *d_work, size_t lwork_bytes, int *d_info);

/* ---- geodesic trial points of the cg_unitary line searches ---------------
 * The rotation half of calaman::cg_detail::sample_derivative
 * (src/cg_unitary/geodesic_search.cppm:338-420): for j = 1 .. num_samples-1,
 * d_Wout block j-1 (n x n, packed, ld n) = exp(j * step * H) * W, with H in
 * u(n) (skew-Hermitian; skew-symmetric for the real tiers) and W n x n (ldw).
 * Sample 0 is W itself and is not written. Only H's lower triangle (and the
 * imaginary part of its diagonal) is read. The reference forms R_1 =
 * expm(step H) and R_j = R_{j-1} R_1; here exp(t H) comes from one Hermitian
 * eigensolve of i H and every trial point from one wide product, no error
 * growing along j. 1 <= num_samples <= 64. Never synchronises; d_info: ONE
 * device int as for expm_herm. INVALID_VALUE / ALLOC_FAILED as expm. */
calamanStatus_t calaman_geodesic_points_bufferSize_s(calamanSolverHandle_t h, int n, int num_samples, size_t *bytes);
calamanStatus_t calaman_geodesic_points_bufferSize_d(calamanSolverHandle_t h, int n, int num_samples, size_t *bytes);
calamanStatus_t calaman_geodesic_points_bufferSize_c(calamanSolverHandle_t h, int n, int num_samples, size_t *bytes);
calamanStatus_t calaman_geodesic_points_bufferSize_z(calamanSolverHandle_t h, int n, int num_samples, size_t *bytes);
calamanStatus_t calaman_geodesic_points_s(calamanBlasHandle_t blas, calamanSolverHandle_t solver, calamanStream_t stream,
                                          int n, const float *d_W, int ldw, const float *d_H, int ldh, double step,
                                          int num_samples, float *d_Wout, void *d_work, size_t lwork_bytes,
                                          int *d_info);
calamanStatus_t calaman_geodesic_points_d(calamanBlasHandle_t blas, calamanSolverHandle_t solver, calamanStream_t stream,
                                          int n, const double *d_W, int ldw, const double *d_H, int ldh, double step,
                                          int num_samples, double *d_Wout, void *d_work, size_t lwork_bytes,
                                          int *d_info);
calamanStatus_t calaman_geodesic_points_c(calamanBlasHandle_t blas, calamanSolverHandle_t solver, calamanStream_t stream,
                                          int n, const void *d_W, int ldw, const void *d_H, int ldh, double step,
                                          int num_samples, void *d_Wout, void *d_work, size_t lwork_bytes,
                                          int *d_info);
calamanStatus_t calaman_geodesic_points_z(calamanBlasHandle_t blas, calamanSolverHandle_t solver, calamanStream_t stream,
                                          int n, const void *d_W, int ldw, const void *d_H, int ldh, double step,
                                          int num_samples, void *d_Wout, void *d_work, size_t lwork_bytes,
                                          int *d_info);

/* ---- lacn2: 1-norm estimate by reverse communication (LAPACK xLACN2) ----
 * src/lapack/lacn2/interface.cppm:85-200 (calaman::lacn2_bufferSize,
 * calaman::lacn2). Real only (s/d), as the reference. Start with *kase = 0;
 * on a return with *kase 1 (2) overwrite d_x with A x (A^T x), ordered on
 * the handle's stream, and call again with everything else unchanged; *kase
 * 0 on return: *est <= ||A||_1 and d_v = A w with est = ||v||_1 / ||w||_1.
 * est, kase and isave[3] are host state (isave 1-based, as the reference's
 * std::array<int, 3>); d_work holds ISGN and must be the same buffer, of at
 * least calaman_lacn2_bufferSize_*(n) bytes, on every call of one run.
 * Synchronises the handle's stream at most once per call. INVALID_VALUE for
 * n < 1, a null pointer, a bad state or a short workspace. */
size_t calaman_lacn2_bufferSize_s(int n);
size_t calaman_lacn2_bufferSize_d(int n);
calamanStatus_t calaman_lacn2_s(calamanBlasHandle_t blas, int n, float *d_v, float *d_x, void *d_work,
                                size_t work_bytes, float *est, int *kase, int *isave);
calamanStatus_t calaman_lacn2_d(calamanBlasHandle_t blas, int n, double *d_v, double *d_x, void *d_work,
                                size_t work_bytes, double *est, int *kase, int *isave);

/* ---- expm without a caller workspace ----------------------------------
 * No counterpart in the reference: calaman_G's expm always takes a caller
 * workspace. For callers that cannot call cudaMalloc (code hosted by a
 * framework that owns every device allocation, loops that must not allocate
 * once running, FFI or plugin callers without a device allocator), this runs
 * calaman_expm_d on a 4 MiB workspace held in a static device array of the
 * library, for n <= 256; larger n returns CALAMAN_STATUS_NOT_SUPPORTED. The
 * array is resident on every GPU that loads the library until exit. Its
 * address is looked up on the first call made on each device: make that
 * first call before any stream capture. The address is kept for the life of
 * the process, so cudaDeviceReset after that first call is not supported.
 * All calls share the array, so calls
 * that overlap on the GPU race on it: serialise them. Nothing in it needs to
 * start at zero; it keeps the last call's data. Same results, status codes
 * and single stream synchronisation as calaman_expm_d. */
calamanStatus_t calaman_expm_noalloc_d(calamanBlasHandle_t blas, calamanStream_t stream, int n,
                                       const double *d_A, int lda, double *d_expA, int lde,
                                       int *d_info, calamanExpmPlan_t *plan);

/* ---- pade (src/expm/pade.cppm:77-191) ----------------------------------
 * Unscaled r_m(A) = q_m(A)^-1 p_m(A); never synchronises. */
calamanStatus_t calaman_pade_s(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                               calamanStream_t stream, int m, int n, const float *d_A, int lda,
                               float *d_r, int ldr, void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_pade_d(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                               calamanStream_t stream, int m, int n, const double *d_A, int lda,
                               double *d_r, int ldr, void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_pade_c(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                               calamanStream_t stream, int m, int n, const void *d_A, int lda,
                               void *d_r, int ldr, void *d_work, size_t lwork_bytes, int *d_info);
calamanStatus_t calaman_pade_z(calamanBlasHandle_t blas, calamanSolverHandle_t solver,
                               calamanStream_t stream, int m, int n, const void *d_A, int lda,
                               void *d_r, int ldr, void *d_work, size_t lwork_bytes, int *d_info);

/* ---- matrix_norm1 (src/expm/norm1.cppm:45-56) --------------------------
 * Maximum absolute column sum (true complex modulus), NaN if any element is
 * NaN. d_colsum: device scratch of n reals of the element's real type; it
 * receives the column sums and, in [0], the maximum. Synchronises `stream`.
 * Returns NaN (and writes nothing) for n < 1 or a null pointer. */
float calaman_matrix_norm1_s(calamanStream_t stream, int n, const float *d_A, int lda,
                             float *d_colsum);
double calaman_matrix_norm1_d(calamanStream_t stream, int n, const double *d_A, int lda,
                              double *d_colsum);
float calaman_matrix_norm1_c(calamanStream_t stream, int n, const void *d_A, int lda,
                             float *d_colsum);
double calaman_matrix_norm1_z(calamanStream_t stream, int n, const void *d_A, int lda,
                              double *d_colsum);

/* ---- horner (src/horner/interface.cppm:104-194) ------------------------ */
size_t calaman_horner_bufferSize_s(int n);
size_t calaman_horner_bufferSize_d(int n);
/* P = sum_{k=0}^{degree} c_k A^k by Horner's rule; coefficients on the
 * DEVICE, ascending. d_work may be NULL when degree == 0. */
calamanStatus_t calaman_horner_s(calamanBlasHandle_t handle, int n, const float *d_coeffs,
                                 int degree, const float *d_A, int lda, float *d_P, int ldp,
                                 void *d_work, size_t work_bytes);
calamanStatus_t calaman_horner_d(calamanBlasHandle_t handle, int n, const double *d_coeffs,
                                 int degree, const double *d_A, int lda, double *d_P, int ldp,
                                 void *d_work, size_t work_bytes);

/* ---- paterson_stockmeyer (src/paterson_stockmeyer/interface.cppm:117-422) */
typedef struct {
  int s;          /* block size actually used */
  int r;          /* Horner steps over X = A^s: floor(degree / s) */
  int num_powers; /* powers held at once: A^2 .. A^(num_powers+1) */
  int num_blocks; /* n x n workspace blocks */
  int num_gemms;  /* matrix products issued */
} calamanPatersonStockmeyerPlan_t;

int calaman_paterson_stockmeyer_cost(int degree, int s);
int calaman_paterson_stockmeyer_block_size(int degree);
calamanPatersonStockmeyerPlan_t calaman_paterson_stockmeyer_plan(int degree, int s_requested);
size_t calaman_paterson_stockmeyer_power_stride_s(int n);
size_t calaman_paterson_stockmeyer_power_stride_d(int n);
size_t calaman_paterson_stockmeyer_bufferSize_s(int n, int degree, int s_requested);
size_t calaman_paterson_stockmeyer_bufferSize_d(int n, int degree, int s_requested);
calamanStatus_t calaman_paterson_stockmeyer_s(calamanBlasHandle_t handle, int n,
                                              const float *d_coeffs, int degree, const float *d_A,
                                              int lda, float *d_P, int ldp, void *d_work,
                                              size_t work_bytes, int s_requested);
calamanStatus_t calaman_paterson_stockmeyer_d(calamanBlasHandle_t handle, int n,
                                              const double *d_coeffs, int degree,
                                              const double *d_A, int lda, double *d_P, int ldp,
                                              void *d_work, size_t work_bytes, int s_requested);

/* ---- building blocks and instrumentation ------------------------------
 * No counterpart in the reference's modules: calaman_G takes its matrix
 * products from WarpWraps' wwr::gemm (cuBLAS). Exposed so callers (and the
 * benchmark) can run the same tensor-core GEMM the path uses.
 * C = alpha A B + beta C, no transposes, column-major, real alpha/beta; for
 * _c/_z the pointers are interleaved complex. beta == 0 never reads C. */
calamanStatus_t calaman_gemm_s(calamanStream_t stream, int m, int n, int k, double alpha,
                               const float *A, int lda, const float *B, int ldb, double beta,
                               float *C, int ldc);
calamanStatus_t calaman_gemm_d(calamanStream_t stream, int m, int n, int k, double alpha,
                               const double *A, int lda, const double *B, int ldb, double beta,
                               double *C, int ldc);
calamanStatus_t calaman_gemm_c(calamanStream_t stream, int m, int n, int k, double alpha,
                               const void *A, int lda, const void *B, int ldb, double beta,
                               void *C, int ldc);
calamanStatus_t calaman_gemm_z(calamanStream_t stream, int m, int n, int k, double alpha,
                               const void *A, int lda, const void *B, int ldb, double beta,
                               void *C, int ldc);

/* FP32 GEMM on the tcgen05 tensor cores: every operand element is split into
 * bf16 parts (x = h + m + l) and the product accumulates, in FP32 TMEM, the
 * part products the precision level keeps: terms = 3 (h and m parts, ~16-bit
 * operands) or 6 (h, m and l parts, ~24-bit operands, about FP32 accuracy).
 * This is how the _s tier of expm/pade runs its dense products; `work` holds
 * the operand parts (calaman_gemm_bf16x_bufferSize bytes, 256-byte aligned). */
calamanStatus_t calaman_gemm_bf16x_bufferSize(int m, int n, int k, int terms, size_t *bytes);
calamanStatus_t calaman_gemm_bf16x_s(calamanStream_t stream, int m, int n, int k, double alpha,
                                     const float *A, int lda, const float *B, int ldb, double beta,
                                     float *C, int ldc, int terms, void *work, size_t work_bytes);
/* How the handle's FP64 / complex128 calls (expm, pade, expm_vjp,
 * expm_balanced and their squarings) run their n x n products: -1 (default)
 * on the INT8 tensor cores by the Ozaki scheme with 7 digits when n >= 1536,
 * where that measured faster, and on the FP64 tensor cores otherwise; 0
 * always on the FP64 tensor cores; 2..8 always emulated with that many digits
 * (n >= 128). The workspace queries take the same handle: size the workspace
 * after setting this. Batched calls always use the FP64 tensor cores. */
calamanStatus_t calamanSetDoubleEmulation(calamanHandle_t handle, int digits);
calamanStatus_t calamanGetDoubleEmulation(calamanHandle_t handle, int *digits);
/* Complex64 C = alpha A B + beta C on the tensor cores as split-BF16 part
 * products: one real product of twice the rows and depth,
 * [Cr; Ci] = [[Ar, -Ai]; [Ai, Ar]] [Br; Bi]. This is how the _c tier of
 * expm/pade runs its dense products (the reference's wwr::gemm for complex
 * float, src/expm/pade.cppm:115-136). */
calamanStatus_t calaman_gemm_bf16x_bufferSize_c(int m, int n, int k, int terms, size_t *bytes);
calamanStatus_t calaman_gemm_bf16x_c(calamanStream_t stream, int m, int n, int k, double alpha, const void *A,
                                     int lda, const void *B, int ldb, double beta, void *C, int ldc, int terms,
                                     void *work, size_t work_bytes);
/* A device workspace attached to the handle (cublasSetWorkspace's role;
 * 256-byte aligned; NULL and 0 detach it). horner_s and paterson_stockmeyer_s,
 * whose own workspaces are sized as the reference's, run their products on the
 * tensor cores when the attached workspace holds at least
 * calaman_poly_tensor_workspace_s(n) bytes, and on the SIMT cores otherwise.
 * The caller keeps it alive while calls that may use it run. */
calamanStatus_t calamanSetWorkspace(calamanHandle_t handle, void *d_work, size_t bytes);
size_t calaman_poly_tensor_workspace_s(int n);
/* The split level the handle's _s expm/pade calls use (default 6). */
calamanStatus_t calamanSetFloatSplit(calamanHandle_t handle, int terms);
calamanStatus_t calamanGetFloatSplit(calamanHandle_t handle, int *terms);

/* FP64 / complex128 GEMM C = alpha A B + beta C (column-major, no transposes,
 * real alpha and beta) on the INT8 tensor cores by the Ozaki splitting scheme:
 * each row of A and each column of B is scaled by the power of two of its
 * largest magnitude and cut into `digits` signed 7-bit digits; the digit
 * products of total weight < digits are summed exactly in int32 and combined
 * in FP64. Error about 2^(-7 digits) relative to |A||B| row by column
 * (digits = 7: 49 bits, FP64-grade for the expm path). Stands in for the
 * reference's wwr::gemm FP64 products (src/expm/pade.cppm:115-136,162,176,180;
 * src/expm/expm.cppm:160-165) where it is faster than the FP64 tensor cores.
 * digits in 2..8, k (2k for _z) small enough that digits * 127^2 * k < 2^31.
 * `work` holds the digit planes (calaman_gemm_ozaki_bufferSize bytes, 256-byte
 * aligned); its first word receives a nonzero code if a bounded wait of the
 * kernel ran out. Never synchronises. */
calamanStatus_t calaman_gemm_ozaki_bufferSize(int m, int n, int k, int is_complex, int digits,
                                              size_t *bytes);
calamanStatus_t calaman_gemm_ozaki_d(calamanStream_t stream, int m, int n, int k, double alpha,
                                     const double *A, int lda, const double *B, int ldb, double beta,
                                     double *C, int ldc, int digits, void *work, size_t work_bytes);
calamanStatus_t calaman_gemm_ozaki_z(calamanStream_t stream, int m, int n, int k, double alpha,
                                     const void *A, int lda, const void *B, int ldb, double beta,
                                     void *C, int ldc, int digits, void *work, size_t work_bytes);
/* Self-test of the tensor-core kernels' bounded waits: runs the Ozaki GEMM
 * kernel once (128^3) with its producer issuing no copy and every wait limited
 * to `spin` tries, so that the waits run out; synchronises and returns in *code
 * the error code the kernel recorded (nonzero: the kernel gave up and unwound
 * instead of hanging). `work`: at least 1 MiB of device memory. */
calamanStatus_t calaman_gemm_ozaki_wait_check(calamanStream_t stream, long long spin, void *work,
                                              size_t work_bytes, int *code);

/* The batched tier's schedule and launch mode (no counterpart: the reference
 * evaluates one matrix per call). A batched call whose configuration (sizes,
 * plans, pointers, schedule) repeats the previous call's is captured once as a
 * CUDA graph of its kernels and replayed from then on (on by default; off
 * while kernel timing is on). The schedule gives, per size bucket
 * b = ceil(n / 16) (index 1..16 of a 17-int array), the CTA size of the
 * per-matrix LU (64, 128 or 256 threads, >= 16 b), and the smallest n whose
 * FP32 products run on the tensor cores. calamanTuneBatched measures it on the
 * current device with `count` float32 matrices per size (scratch:
 * calamanTuneBatched_bufferSize(count) bytes), keeps it in the handle and
 * returns it; the built-in default is the table it measured on a B200. */
calamanStatus_t calamanSetBatchedGraphs(calamanHandle_t handle, int enable);
/* calaman_expm_{s,d,c,z} and calaman_expm_vjp_{s,d,c,z} likewise (no
 * counterpart in the reference, whose expm launches its kernels one by one):
 * everything after the 1-norm readback depends only on the size, the plan, the
 * pointers, the stream and the handle's settings, so a call that repeats the
 * previous call of its entry and type in all of them replays a captured CUDA
 * graph of those launches (on by default; off while kernel timing is on, on
 * the legacy default streams, and in calaman_expm_noalloc_d). `cached`: the
 * entry and type pairs with a graph held. */
calamanStatus_t calamanSetExpmGraphs(calamanHandle_t handle, int enable);
calamanStatus_t calamanGetExpmGraphs(calamanHandle_t handle, int *enabled, int *cached);
calamanStatus_t calamanGetBatchedGraphs(calamanHandle_t handle, int *enabled, int *cached);
calamanStatus_t calamanSetBatchedTuning(calamanHandle_t handle, const int *lu_threads, int fp32_tc_min_n);
calamanStatus_t calamanGetBatchedTuning(calamanHandle_t handle, int *lu_threads, int *fp32_tc_min_n);
size_t calamanTuneBatched_bufferSize(int count);
calamanStatus_t calamanTuneBatched(calamanHandle_t handle, int count, void *d_work, size_t work_bytes,
                                   int *lu_threads, int *fp32_tc_min_n);

/* Self-test of the grid barrier of the one-launch tridiagonal reduction
 * (expm_herm / heevd): a two-CTA launch in which one CTA never arrives, so the
 * other's wait runs out after `limit` polls; synchronises and returns in *code
 * the failure flag the barrier set (1: it gave up instead of hanging). `work`:
 * at least 256 bytes of device memory. No counterpart in the reference. */
calamanStatus_t calaman_grid_barrier_wait_check(calamanStream_t stream, unsigned limit, void *work,
                                                size_t work_bytes, int *code);

/* LU with partial pivoting and the n-right-hand-side solve that pade() runs on
 * q_m(A) (the reference calls the solver library's getrf/getrs through
 * WarpWraps, src/expm/pade.cppm:186-188). LAPACK semantics: P A = L U, pivot
 * = first entry of largest |Re|+|Im|. `scratch` is calaman_getrf_bufferSize
 * device bytes; it begins with the n pivot rows (0-based, int) and must be
 * passed unchanged to getrs. getrs reads B and writes X (no aliasing).
 * d_info: getrf writes the first zero pivot (1-based) or 0; getrs writes 0. */
calamanStatus_t calaman_getrf_bufferSize(int n, size_t *bytes);
calamanStatus_t calaman_getrf_s(calamanStream_t stream, int n, float *A, int lda, void *scratch,
                                int *d_info);
calamanStatus_t calaman_getrf_d(calamanStream_t stream, int n, double *A, int lda, void *scratch,
                                int *d_info);
calamanStatus_t calaman_getrf_c(calamanStream_t stream, int n, void *A, int lda, void *scratch,
                                int *d_info);
calamanStatus_t calaman_getrf_z(calamanStream_t stream, int n, void *A, int lda, void *scratch,
                                int *d_info);
calamanStatus_t calaman_getrs_s(calamanStream_t stream, int n, int nrhs, const float *LU, int lda,
                                const void *scratch, const float *B, int ldb, float *X, int ldx,
                                int *d_info);
calamanStatus_t calaman_getrs_d(calamanStream_t stream, int n, int nrhs, const double *LU, int lda,
                                const void *scratch, const double *B, int ldb, double *X, int ldx,
                                int *d_info);
calamanStatus_t calaman_getrs_c(calamanStream_t stream, int n, int nrhs, const void *LU, int lda,
                                const void *scratch, const void *B, int ldb, void *X, int ldx,
                                int *d_info);
calamanStatus_t calaman_getrs_z(calamanStream_t stream, int n, int nrhs, const void *LU, int lda,
                                const void *scratch, const void *B, int ldb, void *X, int ldx,
                                int *d_info);

/* Total kernel launches this library has issued in the process. */
unsigned long long calamanGetLaunchCount(void);

/* Per-handle CUDA-event timing of the dense products (every GEMM launch the
 * handle's calls issue, including those inside the LU and the solves).
 * Enabling clears the record; reading synchronises on the last event. */
typedef struct {
  long long gemm_launches;
  double gemm_ms;        /* summed device time of those launches */
  double gemm_flops;     /* algorithmic flops: 2mnk real, 8mnk complex */
} calamanKernelTiming_t;
calamanStatus_t calamanSetKernelTiming(calamanHandle_t handle, int enable);
calamanStatus_t calamanGetKernelTiming(calamanHandle_t handle, calamanKernelTiming_t *out);

#ifdef __cplusplus
}
#endif

#endif /* CALAMAN_B200_H */
