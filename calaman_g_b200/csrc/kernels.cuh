// kernels.cuh -- launchers of every device kernel, shared by the host drivers.
//
// Each launcher enqueues on `stream`, returns the launch's cudaError_t, and
// never synchronises. Matrices are column-major.
#pragma once

#include "common.cuh"

namespace clm {

// ---- 1-norm ---------------------------------------------------------------
// Fused column |.|-sums (FP64 accumulation, true complex modulus) and the
// NaN-sticky max over them, written to *d_norm (one double). d_colsum, if not
// null, receives the per-column sums (as doubles). d_norm is reset inside.
template <typename T>
cudaError_t launch_norm1(cudaStream_t s, int n, const T *A, int lda, double *d_colsum,
                         double *d_norm);

// The reference's two-step form for the public matrix_norm1 (src/expm/norm1.cppm:45-56):
// column sums into d_colsum (element real type), then the max in place at d_colsum[0].
template <typename T, typename R>
cudaError_t launch_colsums_then_max(cudaStream_t s, int n, const T *A, int lda, R *d_colsum);

// ---- Pade elementwise steps (src/expm/expm.cu:74-162) ---------------------
// V = cv0 I + sum_k cv[k+1] P_k,  W = cw0 I + sum_k cw[k+1] P_k  (ld = n)
template <typename T>
cudaError_t launch_pade_even_odd(cudaStream_t s, int n, int np, const T *P1, const T *P2,
                                 const T *P3, const T *P4, const double *cv, const double *cw,
                                 T *V, T *W);
// P = V + U (into ldp), Q = V - U (ld n; may alias V)
template <typename T>
cudaError_t launch_pade_split(cudaStream_t s, int n, const T *U, const T *V, T *P, int ldp, T *Q);

// B = f * A (f = 1 is a copy); n x n, arbitrary leading dimensions.
template <typename T>
cudaError_t launch_scale_copy(cudaStream_t s, int n, double f, const T *A, int lda, T *B, int ldb);

// B = (To) A: precision conversion of an n x n matrix (float <-> double,
// complex64 <-> complex128).
template <typename Ti, typename To>
cudaError_t launch_convert(cudaStream_t s, int n, const Ti *A, int lda, To *B, int ldb);

// ---- matrix polynomials -----------------------------------------------------
// B_j = c0 I + c1 A + sum_{k>=2} c_k A^k, coefficients on the device
// (src/paterson_stockmeyer/paterson_stockmeyer.cu:51-85)
template <typename T>
cudaError_t launch_ps_build_block(cudaStream_t s, T *B, int ldb, int n, const T *A, int lda,
                                  const T *powers, std::size_t stride, const T *coeffs, int terms);
// P = alpha I, and P_ii += alpha (src/horner/horner.cu:39-67)
template <typename T>
cudaError_t launch_set_scaled_identity(cudaStream_t s, T *P, int n, int ldp, const T *d_alpha);
template <typename T>
cudaError_t launch_add_scaled_identity(cudaStream_t s, T *P, int n, int ldp, const T *d_alpha);

// ---- GEMM -----------------------------------------------------------------
// C = alpha * A * B + beta * C, all non-transposed, column-major. alpha and
// beta are real host scalars (the path uses 1, -1, 0). beta == 0 never reads C.
template <typename T>
cudaError_t gemm_nn(cudaStream_t s, int M, int N, int K, double alpha, const T *A, int lda,
                    const T *B, int ldb, double beta, T *C, int ldc);

// The same product with K split into slices computed in parallel (blockIdx.z)
// into `partial` (slices * M * N elements, ld M) and summed in slice order:
// for skinny products whose few output tiles would leave most SMs idle.
// At most max_splits slices of a 64-multiple of K; FP64 types only.
template <typename T>
cudaError_t gemm_nn_splitk(cudaStream_t s, int M, int N, int K, double alpha, const T *A, int lda, const T *B,
                           int ldb, double beta, T *C, int ldc, T *partial, int max_splits);

// FP32 / complex64 GEMM on the tcgen05 tensor cores as split-BF16 part
// products (terms = 3 or 6), accumulated in FP32 TMEM; needs
// tc_gemm_workspace_bytes of scratch (cplx: for the complex product).
std::size_t tc_gemm_workspace_bytes(int M, int N, int K, int terms, bool cplx = false);
cudaError_t tc_gemm_f32(cudaStream_t s, int M, int N, int K, double alpha, const float *A, int lda,
                        const float *B, int ldb, double beta, float *C, int ldc, void *ws,
                        std::size_t ws_bytes, int terms);
cudaError_t tc_gemm_c64(cudaStream_t s, int M, int N, int K, double alpha, const float2 *A, int lda,
                        const float2 *B, int ldb, double beta, float2 *C, int ldc, void *ws,
                        std::size_t ws_bytes, int terms);

// FP64 / complex128 GEMM on the INT8 tensor cores by the Ozaki splitting
// scheme (oz_gemm.cu): `ks` signed 7-bit digits per operand element (row
// scaling of A, column scaling of B), digit pairs of total weight < ks, exact
// int32 level sums; needs oz_gemm_workspace_bytes of scratch. spin: tries of
// every bounded wait (0: the default limit); skip_loads: test-only, the
// producer issues no copy so that the waits run out and the kernel returns its
// error code in the first workspace word.
std::size_t oz_gemm_workspace_bytes(int M, int N, int K, bool cplx, int ks);
bool oz_gemm_supported(int K, bool cplx, int ks);
template <typename T>
cudaError_t oz_gemm(cudaStream_t s, int M, int N, int K, double alpha, const T *A, int lda, const T *B,
                    int ldb, double beta, T *C, int ldc, void *ws, std::size_t ws_bytes, int ks,
                    long long spin = 0, int skip_loads = 0);

// ---- LU with partial pivoting and the n-RHS solve -------------------------
// Scratch the LU needs beyond the matrix: ipiv (n ints), perm (n ints) and a
// small swap map; bytes for an n x n factorisation.
std::size_t lu_scratch_bytes(int n);

// Factor A (n x n, lda) in place: P A = L U. info_dev[0] receives the first
// zero pivot (1-based) or 0. `scratch` is lu_scratch_bytes(n) device bytes.
template <typename T>
cudaError_t getrf(cudaStream_t s, int n, T *A, int lda, void *scratch, int *info_dev);

// While a NoLookAheadScope is open on a host thread, getrf on that thread
// factors every panel on the caller's stream instead of overlapping the next
// panel on the library's auxiliary stream, so it creates no stream or event.
extern thread_local bool tl_no_lookahead;
struct NoLookAheadScope {
  bool saved;
  NoLookAheadScope() : saved(tl_no_lookahead) { tl_no_lookahead = true; }
  ~NoLookAheadScope() { tl_no_lookahead = saved; }
};

// Solve A X = B with the factors from getrf: B (n x nrhs, ldb) is read, X is
// written to (ldx); B and X may not alias. info_dev[0] = 0.
template <typename T>
cudaError_t getrs(cudaStream_t s, int n, int nrhs, const T *LU, int lda, const void *scratch,
                  const T *B, int ldb, T *X, int ldx, int *info_dev);

// B = f op(A) for an rows x cols matrix A: op is the transpose, conjugated
// when `conj` (complex types); B is cols x rows. A and B may not alias.
template <typename T>
cudaError_t launch_transpose(cudaStream_t s, int rows, int cols, double f, const T *A, int lda, T *B,
                             int ldb, bool conj);

}  // namespace clm
