// balance.cu -- diagonal balancing (the scaling half of ?gebal) and the
// balanced expm, D exp(D^-1 A D) D^-1.
//
// gebal (src/lapack/gebal/interface.cppm:100-255, sweep kernel
// src/lapack/gebal/gebal.cu:175-310) balances with the Parlett-Reinsch
// iteration: index by index (Gauss-Seidel -- index i is scaled before i + 1
// measures its norms), the off-diagonal 1-norms c of column i and r of row i
// are driven towards each other by a power-of-two factor f, accepted only for
// a 5% drop of c + r and within LAPACK's overflow guards; sweeps repeat until
// one changes nothing. Factors are powers of two, so B = D^-1 A D is exact and
// D B D^-1 reproduces A bit for bit. Only the scaling job is built: it is the
// half that lowers the 1-norm, i.e. removes squarings from expm
// (src/expm/README.md:100-122); the permutation half is NOT_SUPPORTED here.
//
// One sweep runs in one CTA of kBalThreads threads: the O(n) measurements of an
// index are split over the threads (thread t takes j = t, t + kBalThreads, ...,
// the warp sums by a xor butterfly, the warp partials in warp order -- the
// oracle repeats this order, so FP64 results match it bit for bit), and the
// decision is evaluated by every thread on identical inputs.
#include <cfloat>
#include <cmath>
#include <vector>

#include "expm_common.cuh"

namespace clm {
namespace {

constexpr int kBalThreads = 512;
constexpr int kGebalMaxSweeps = 1000;  // the reference's default cap

template <typename R>
struct BalLimits {
  R sfmin1, sfmax1, sfmin2, sfmax2;
};

template <typename R>
BalLimits<R> bal_limits() {
  const R eps = sizeof(R) == 4 ? (R)FLT_EPSILON : (R)DBL_EPSILON;
  const R tiny = sizeof(R) == 4 ? (R)FLT_MIN : (R)DBL_MIN;
  const R s1 = tiny / eps, s2 = s1 * (R)2;
  return BalLimits<R>{s1, (R)1 / s1, s2, (R)1 / s2};
}

template <typename T>
__device__ __forceinline__ typename elem<T>::real mag1(T x);
template <> __device__ __forceinline__ float mag1<float>(float x) { return fabsf(x); }
template <> __device__ __forceinline__ double mag1<double>(double x) { return fabs(x); }
template <> __device__ __forceinline__ float mag1<float2>(float2 x) { return fabsf(x.x) + fabsf(x.y); }
template <> __device__ __forceinline__ double mag1<double2>(double2 x) { return fabs(x.x) + fabs(x.y); }

template <typename R>
__device__ __forceinline__ R warp_sum(R v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename R>
__device__ __forceinline__ R warp_max(R v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// The radix-2 balancing decision of LAPACK xGEBAL for one index, from its
// off-diagonal column and row 1-norms c, r and the largest magnitudes ca, ra
// of its column and row (Parlett and Reinsch 1969; LAPACK's DGEBAL, scaling
// job). Two passes over powers of two, each step exact:
//   grow:   while the column side is below half the row side (c < r / 2) and
//           no scaled quantity reaches the guards, double the column side and
//           halve the row side (f *= 2);
//   shrink: while half the column side is still at least the row side, halve
//           the column side and double the row side (f /= 2), under the same
//           guards.
// f is taken when it shrinks c + r below 0.95 of its old value and the
// accumulated scale d_i f stays inside [sfmin1, sfmax1].
template <typename R>
__device__ __forceinline__ bool balance_step(R c, R r, R ca, R ra, R scale_i, const BalLimits<R> &lim,
                                             R *factor) {
  *factor = (R)1;
  if (c == (R)0 || r == (R)0 || !isfinite(c + r + ca + ra)) return false;
  const R before = c + r;
  R f = 1, half_r = r / 2;
  while (c < half_r && fmax(fmax(f, c), ca) < lim.sfmax2 && fmin(fmin(r, half_r), ra) > lim.sfmin2) {
    f *= 2;
    c *= 2;
    ca *= 2;
    r /= 2;
    half_r /= 2;
    ra /= 2;
  }
  R half_c = c / 2;
  while (half_c >= r && fmax(r, ra) < lim.sfmax2 && fmin(fmin(f, c), fmin(half_c, ca)) > lim.sfmin2) {
    f /= 2;
    c /= 2;
    half_c /= 2;
    ca /= 2;
    r *= 2;
    ra *= 2;
  }
  if (!(c + r < (R)0.95 * before)) return false;
  if (f < (R)1 && scale_i < (R)1 && f * scale_i <= lim.sfmin1) return false;
  if (f > (R)1 && scale_i > (R)1 && scale_i >= lim.sfmax1 / f) return false;
  *factor = f;
  return true;
}

// One Parlett-Reinsch sweep over every index (scaling job: the window is the
// whole matrix). noconv[0] is set when any index was rescaled.
template <typename T>
__global__ void __launch_bounds__(kBalThreads)
    gebal_sweep_kernel(int n, T *__restrict__ A, int lda, typename elem<T>::real *__restrict__ dsc,
                       int *__restrict__ noconv, BalLimits<typename elem<T>::real> lim) {
  using R = typename elem<T>::real;
  constexpr int W = kBalThreads / 32;
  __shared__ R part[4][W];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int i = 0; i < n; ++i) {
    R c = 0, r = 0, ca = 0, ra = 0;
    for (int j = t; j < n; j += kBalThreads) {
      const R ac = mag1(A[(std::size_t)i * lda + j]);  // A(j, i)
      const R ar = mag1(A[(std::size_t)j * lda + i]);  // A(i, j)
      if (j != i) {
        c += ac;
        r += ar;
      }
      ca = fmax(ca, ac);
      ra = fmax(ra, ar);
    }
    c = warp_sum(c);
    r = warp_sum(r);
    ca = warp_max(ca);
    ra = warp_max(ra);
    if (lane == 0) {
      part[0][warp] = c;
      part[1][warp] = r;
      part[2][warp] = ca;
      part[3][warp] = ra;
    }
    __syncthreads();
    c = part[0][0];
    r = part[1][0];
    ca = part[2][0];
    ra = part[3][0];
    for (int w = 1; w < W; ++w) {
      c += part[0][w];
      r += part[1][w];
      ca = fmax(ca, part[2][w]);
      ra = fmax(ra, part[3][w]);
    }
    // the decision, on identical inputs in every thread
    R f = 1;
    const bool accept = balance_step(c, r, ca, ra, dsc[i], lim, &f);
    __syncthreads();  // every read of this index is done
    if (accept) {     // row i by 1/f, then column i by f (A(i,i) is touched by both)
      const R inv = (R)1 / f;
      for (int j = t; j < n; j += kBalThreads) A[(std::size_t)j * lda + i] = scale(A[(std::size_t)j * lda + i], inv);
    }
    __syncthreads();
    if (accept) {
      for (int j = t; j < n; j += kBalThreads) A[(std::size_t)i * lda + j] = scale(A[(std::size_t)i * lda + j], f);
      if (t == 0) {
        dsc[i] *= f;
        *noconv = 1;
      }
    }
    __syncthreads();
  }
}

template <typename R>
__global__ void fill_ones_kernel(int n, R *x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = (R)1;
}

// E(i, j) *= d_i / d_j: exp(A) = D exp(B) D^-1 (powers of two: exact)
template <typename T>
__global__ void unbalance_kernel(int n, const typename elem<T>::real *__restrict__ d, T *__restrict__ E,
                                 int lde) {
  using R = typename elem<T>::real;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const R di = d[row];
  for (int col = blockIdx.y; col < n; col += gridDim.y) {
    T &e = E[(std::size_t)col * lde + row];
    e = scale(scale(e, di), (R)1 / d[col]);
  }
}

enum { kJobNone = 0, kJobPermute = 1, kJobScale = 2, kJobBoth = 3 };

template <typename T>
calamanStatus_t gebal_run(cudaStream_t st, int job, int n, T *A, int lda, int *ilo, int *ihi,
                          typename elem<T>::real *d_scale, int *d_work, int max_sweeps, int *sweeps_out) {
  using R = typename elem<T>::real;
  if (n < 0 || lda < (n > 1 ? n : 1) || A == nullptr || d_scale == nullptr || ilo == nullptr ||
      ihi == nullptr || job < kJobNone || job > kJobBoth)
    return runtime_status(cudaErrorInvalidValue);
  if (job == kJobPermute || job == kJobBoth) return blas_status(CALAMAN_STATUS_NOT_SUPPORTED);
  *ilo = 1;
  *ihi = n;
  if (sweeps_out) *sweeps_out = 0;
  if (n == 0) return ok_status();
  if (d_work == nullptr) return runtime_status(cudaErrorInvalidValue);
  fill_ones_kernel<R><<<(n + 255) / 256, 256, 0, st>>>(n, d_scale);
  CLM_CUDA(launched());
  if (job == kJobNone) return ok_status();
  const BalLimits<R> lim = bal_limits<R>();
  int swept = 0;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    CLM_CUDA(cudaMemsetAsync(d_work, 0, sizeof(int), st));
    gebal_sweep_kernel<T><<<1, kBalThreads, 0, st>>>(n, A, lda, d_scale, d_work, lim);
    CLM_CUDA(launched());
    int noconv = 0;
    CLM_CUDA(cudaMemcpyAsync(&noconv, d_work, sizeof(int), cudaMemcpyDeviceToHost, st));
    CLM_CUDA(cudaStreamSynchronize(st));
    ++swept;
    if (noconv == 0) break;
  }
  if (sweeps_out) *sweeps_out = swept;
  return ok_status();
}

// balanced expm workspace: [B (n x n) | d (n reals) | flag | expm workspace]
template <typename T>
struct BalWs {
  T *B = nullptr;
  typename elem<T>::real *d = nullptr;
  int *flag = nullptr;
  void *expm = nullptr;
  std::size_t carve(void *base, int n) {
    Layout L(base);
    B = L.take<T>((std::size_t)n * n);
    d = L.take<typename elem<T>::real>(n);
    flag = L.take<int>(1);
    expm = L.cursor();
    return L.used;
  }
};

}  // namespace

// the expm entry of driver.cu for the balanced composition
template <typename T>
calamanStatus_t expm_entry(calamanHandle_t blas, calamanStream_t stream, int n, const T *A, int lda, T *E,
                           int lde, void *work, std::size_t lwork, int *d_info, calamanExpmPlan_t *plan);
template <typename T>
std::size_t expm_workspace_bytes(calamanHandle_t h, int n);

namespace {

template <typename T>
std::size_t balanced_bytes(calamanHandle_t h, int n) {
  BalWs<T> w;
  return w.carve(nullptr, n) + expm_workspace_bytes<T>(h, n);
}

template <typename T>
calamanStatus_t expm_balanced_api(calamanHandle_t blas, calamanStream_t stream, int n, const T *A, int lda,
                                  T *E, int lde, void *work, std::size_t lwork, int *d_info,
                                  calamanExpmPlan_t *plan) {
  if (n < 1 || n > kMaxDim || lda < n || lde < n || work == nullptr)
    return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  if (lwork < balanced_bytes<T>(blas, n)) return blas_status(CALAMAN_STATUS_ALLOC_FAILED);
  if (A == nullptr || E == nullptr || d_info == nullptr) return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  BalWs<T> ws;
  ws.carve(work, n);
  CLM_CUDA(launch_scale_copy<T>(st, n, 1.0, A, lda, ws.B, n));
  int ilo = 0, ihi = 0;
  CLM_TRY(gebal_run<T>(st, kJobScale, n, ws.B, n, &ilo, &ihi, ws.d, ws.flag, kGebalMaxSweeps, nullptr));
  CLM_TRY(expm_entry<T>(blas, stream, n, ws.B, n, E, lde, ws.expm, lwork - (std::size_t)((char *)ws.expm - (char *)work),
                        d_info, plan));
  const int gy = n < 65535 ? n : 65535;
  unbalance_kernel<T><<<dim3((n + 255) / 256, gy), 256, 0, st>>>(n, ws.d, E, lde);
  CLM_CUDA(launched());
  return ok_status();
}

}  // namespace
}  // namespace clm

using namespace clm;

extern "C" {

calamanStatus_t calaman_gebal_bufferSize(int n, int *lwork_ints) {
  if (n < 0 || lwork_ints == nullptr) return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  *lwork_ints = 1;
  return ok_status();
}

#define CLM_BAL_API(SUF, T, R, PT, CPT)                                                               \
  calamanStatus_t calaman_gebal_##SUF(calamanStream_t stream, int job, int n, PT A, int lda, int *ilo, \
                                      int *ihi, R *d_scale, int *d_work, int max_sweeps,               \
                                      int *sweeps) {                                                  \
    return gebal_run<T>(static_cast<cudaStream_t>(stream), job, n, reinterpret_cast<T *>(A), lda, ilo, \
                        ihi, d_scale, d_work, max_sweeps > 0 ? max_sweeps : kGebalMaxSweeps, sweeps);  \
  }                                                                                                    \
  calamanStatus_t calaman_expm_balanced_bufferSize_##SUF(calamanSolverHandle_t h, int n, size_t *bytes) { \
    if (n < 1 || n > kMaxDim || bytes == nullptr) return blas_status(CALAMAN_STATUS_INVALID_VALUE);     \
    *bytes = balanced_bytes<T>(h, n);                                                                  \
    return ok_status();                                                                                \
  }                                                                                                    \
  calamanStatus_t calaman_expm_balanced_##SUF(calamanBlasHandle_t blas, calamanSolverHandle_t,         \
                                              calamanStream_t stream, int n, CPT A, int lda, PT E,     \
                                              int lde, void *work, size_t lwork, int *d_info,          \
                                              calamanExpmPlan_t *plan) {                               \
    return expm_balanced_api<T>(blas, stream, n, reinterpret_cast<const T *>(A), lda,                 \
                                reinterpret_cast<T *>(E), lde, work, lwork, d_info, plan);             \
  }
CLM_BAL_API(s, float, float, float *, const float *)
CLM_BAL_API(d, double, double, double *, const double *)
CLM_BAL_API(c, float2, float, void *, const void *)
CLM_BAL_API(z, double2, double, void *, const void *)
#undef CLM_BAL_API

}  // extern "C"
