// lacn2.cu -- the 1-norm estimator by reverse communication (Hager's method
// with Higham's refinements, LAPACK's xLACN2), real s/d.
//
// calaman::lacn2 (src/lapack/lacn2/interface.cppm:104-200) keeps LAPACK's
// state machine on the host (kase, isave 1-based, est) and ISGN in the
// caller's workspace; each call returns with kase 1 (2) for the caller to
// overwrite x with A x (A^T x), until kase 0 leaves est <= ||A||_1 and v = A w.
// The same machine runs here. Each state's device work is one fused pass over
// x plus, for multi-block sizes, one pass over the block partials:
//   state 1  est = sum |x|, then x = isgn = sign(x)            (one pass)
//   state 2  j = argmax |x|, then x = e_j
//   state 3  v = x, est = sum |v|, changed = any sign(x) != isgn (one pass)
//   state 4  j = argmax |x| with x(jlast) and x(j) read back
//   state 5  sum |x|, v = x when the alternating-sign estimate wins
// and the host reads the few scalars it branches on with one synchronisation
// per call (the reference reads them back by up to three).
//
// Sums are taken in double for both tiers and in a fixed order for a given n
// (each thread strides its block's range, warps combine by a xor butterfly,
// warps and blocks in index order), so a run is deterministic. The argmax is
// reference BLAS IxAMAX: the first index of the largest |x_i|, an entry taking
// the lead only when strictly larger (a NaN never does, unless it is x_1). The
// sign test is LAPACK 3.10's x_i >= 0 -> +1, so -0 gives +1 and NaN -1.
#include <cmath>

#include "common.cuh"

namespace clm {
namespace {

constexpr int kLcThreads = 256;
constexpr int kLcPerBlock = 8192;  // elements one block takes before a second is added
constexpr int kLcMaxBlocks = 2 * 148;

enum : int { kLcAsum = 1, kLcArgmax = 2, kLcChanged = 4, kLcCopyV = 8, kLcSign = 16 };

// One block's share of a reduction.
struct LcPart {
  double sum;
  double amax;  // -1: no non-NaN entry seen
  int idx;      // 0-based index of amax
  int changed;
};

// What the host reads back (fits the handle's four pinned doubles).
template <typename R>
struct LcResult {
  double asum;
  R xlast;
  R xnew;
  int imax;  // 1-based
  int changed;
};
static_assert(sizeof(LcResult<double>) <= 4 * sizeof(double), "read-back slot");

struct LcWs {
  int *isgn;
  LcPart *part;
  void *res;
};

template <typename R>
LcWs carve_lc(void *base, int n, std::size_t *bytes) {
  Layout L(base);
  LcWs w;
  w.isgn = L.take<int>(n < 1 ? 1 : n);
  w.part = L.take<LcPart>(kLcMaxBlocks);
  w.res = L.take<LcResult<R>>(1);
  if (bytes) *bytes = L.used;
  return w;
}

__device__ __forceinline__ bool lc_better(double a, int i, double b, int j) {
  return a > b || (a == b && i < j);
}

// Combine (sum, amax, idx, changed) over the block; the result is valid in
// thread 0. Fixed tree: xor butterfly in each warp, warps in index order.
__device__ LcPart lc_block_reduce(LcPart p) {
  __shared__ LcPart sh[kLcThreads / 32];
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const double s = __shfl_xor_sync(0xffffffffu, p.sum, o);
    const double a = __shfl_xor_sync(0xffffffffu, p.amax, o);
    const int i = __shfl_xor_sync(0xffffffffu, p.idx, o);
    const int c = __shfl_xor_sync(0xffffffffu, p.changed, o);
    p.sum += s;  // IEEE addition commutes: both lanes form the same value
    if (lc_better(a, i, p.amax, p.idx)) {
      p.amax = a;
      p.idx = i;
    }
    p.changed |= c;
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sh[warp] = p;
  __syncthreads();
  if (threadIdx.x == 0) {
    p = sh[0];
    for (int w = 1; w < kLcThreads / 32; ++w) {
      p.sum += sh[w].sum;
      if (lc_better(sh[w].amax, sh[w].idx, p.amax, p.idx)) {
        p.amax = sh[w].amax;
        p.idx = sh[w].idx;
      }
      p.changed |= sh[w].changed;
    }
  }
  return p;
}

template <typename R>
__device__ void lc_finish(LcPart p, int n, const R *__restrict__ x, int jlast, LcResult<R> *res) {
  LcResult<R> r;
  r.asum = p.sum;
  // IxAMAX: x_1 leads unless a later entry is strictly larger; a NaN x_1
  // is never overtaken, and all-NaN x gives 1
  const bool first_nan = isnan((double)x[0]);
  r.imax = (first_nan || p.amax < 0.0) ? 1 : p.idx + 1;
  r.changed = p.changed;
  r.xlast = jlast > 0 ? x[jlast - 1] : (R)0;
  r.xnew = x[r.imax - 1];
  *res = r;
}

// One pass over x for the requested modes. With one block the block writes
// the result itself; otherwise each block leaves its partial.
template <typename R, int kMode>
__global__ void __launch_bounds__(kLcThreads)
    lc_pass_kernel(int n, R *__restrict__ x, R *__restrict__ v, int *__restrict__ isgn,
                   LcPart *__restrict__ part, LcResult<R> *__restrict__ res, int jlast) {
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int lo = blockIdx.x * per;
  const int hi = min(n, lo + per);
  LcPart p{0.0, -1.0, 0x7fffffff, 0};
  for (int i = lo + threadIdx.x; i < hi; i += kLcThreads) {
    const R xi = x[i];
    const double a = fabs((double)xi);
    if (kMode & kLcAsum) p.sum += a;
    if ((kMode & kLcArgmax) && a > p.amax) {  // strictly larger: first index, NaN skipped
      p.amax = a;
      p.idx = i;
    }
    const int s = xi >= (R)0 ? 1 : -1;
    if (kMode & kLcChanged) p.changed |= (s != isgn[i]);
    if (kMode & kLcCopyV) v[i] = xi;
    if (kMode & kLcSign) {
      x[i] = (R)s;
      isgn[i] = s;
    }
  }
  p = lc_block_reduce(p);
  if (threadIdx.x == 0) {
    if (gridDim.x == 1) {
      lc_finish<R>(p, n, x, jlast, res);
    } else {
      part[blockIdx.x] = p;
    }
  }
}

// Combine the block partials in block order.
template <typename R>
__global__ void __launch_bounds__(kLcThreads)
    lc_final_kernel(int n, int nparts, const LcPart *__restrict__ part, const R *__restrict__ x, int jlast,
                    LcResult<R> *__restrict__ res) {
  LcPart p{0.0, -1.0, 0x7fffffff, 0};
  for (int b = threadIdx.x; b < nparts; b += kLcThreads) {
    const LcPart q = part[b];
    p.sum += q.sum;
    if (lc_better(q.amax, q.idx, p.amax, p.idx)) {
      p.amax = q.amax;
      p.idx = q.idx;
    }
    p.changed |= q.changed;
  }
  p = lc_block_reduce(p);
  if (threadIdx.x == 0) lc_finish<R>(p, n, x, jlast, res);
}

enum : int { kLcFill = 0, kLcUnit = 1, kLcAlt = 2, kLcSignOnly = 3, kLcCopy = 4 };

// The elementwise vectors of the state machine.
template <typename R, int kWhat>
__global__ void lc_vec_kernel(int n, R *__restrict__ x, R *__restrict__ v, int *__restrict__ isgn, int j1) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (kWhat == kLcFill) {
      x[i] = (R)1 / (R)n;
    } else if (kWhat == kLcUnit) {
      x[i] = (i == j1 - 1) ? (R)1 : (R)0;
    } else if (kWhat == kLcAlt) {
      // LAPACK: x_i = (-1)^(i-1) (1 + (i-1)/(n-1)), 1-based
      const R mag = (R)1 + (R)i / (R)(n - 1);
      x[i] = (i & 1) ? -mag : mag;
    } else if (kWhat == kLcSignOnly) {
      const int s = x[i] >= (R)0 ? 1 : -1;
      x[i] = (R)s;
      isgn[i] = s;
    } else {
      v[i] = x[i];
    }
  }
}

int lc_blocks(int n) {
  const int b = (n + kLcPerBlock - 1) / kLcPerBlock;
  return b < 1 ? 1 : (b > kLcMaxBlocks ? kLcMaxBlocks : b);
}

int vec_blocks(int n) {
  const int b = (n + kLcThreads - 1) / kLcThreads;
  return b < 1 ? 1 : (b > 8 * 148 ? 8 * 148 : b);
}

template <typename R, int kWhat>
cudaError_t lc_vec(cudaStream_t st, int n, R *x, R *v, int *isgn, int j1) {
  lc_vec_kernel<R, kWhat><<<vec_blocks(n), kLcThreads, 0, st>>>(n, x, v, isgn, j1);
  return launched();
}

// One reduction pass (plus the partials' combine when more than one block),
// then the read-back of its result: the call's single synchronisation.
template <typename R, int kMode>
cudaError_t lc_reduce(calamanHandle_t h, cudaStream_t st, int n, R *x, R *v, const LcWs &w, int jlast,
                      LcResult<R> *out) {
  const int nb = lc_blocks(n);
  auto *res = static_cast<LcResult<R> *>(w.res);
  lc_pass_kernel<R, kMode><<<nb, kLcThreads, 0, st>>>(n, x, v, w.isgn, w.part, res, jlast);
  cudaError_t e = launched();
  if (e != cudaSuccess) return e;
  if (nb > 1) {
    lc_final_kernel<R><<<1, kLcThreads, 0, st>>>(n, nb, w.part, x, jlast, res);
    if ((e = launched()) != cudaSuccess) return e;
  }
  void *host = (h && h->h_pinned) ? static_cast<void *>(h->h_pinned) : static_cast<void *>(out);
  if ((e = cudaMemcpyAsync(host, res, sizeof(LcResult<R>), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if (host != out) *out = *static_cast<const LcResult<R> *>(host);
  return cudaSuccess;
}

template <typename R>
calamanStatus_t lacn2_api(calamanHandle_t h, int n, R *v, R *x, void *work, std::size_t bytes, R *est,
                          int *kase, int *isave) {
  constexpr int kItmax = 5;
  if (n < 1 || v == nullptr || x == nullptr || work == nullptr || est == nullptr || kase == nullptr ||
      isave == nullptr || (*kase != 0 && (isave[0] < 1 || isave[0] > 5)))
    return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  std::size_t need = 0;
  carve_lc<R>(nullptr, n, &need);
  if (bytes < need) return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  const LcWs w = carve_lc<R>(work, n, nullptr);
  const cudaStream_t st = h ? h->stream : nullptr;
  LcResult<R> r{};

  auto to_unit = [&]() -> calamanStatus_t {  // label 50: x = e_j, ask for A x
    CLM_CUDA((lc_vec<R, kLcUnit>(st, n, x, v, w.isgn, isave[1])));
    *kase = 1;
    isave[0] = 3;
    return ok_status();
  };
  auto to_final = [&]() -> calamanStatus_t {  // label 120: alternating signs, ask for A x
    CLM_CUDA((lc_vec<R, kLcAlt>(st, n, x, v, w.isgn, 0)));
    *kase = 1;
    isave[0] = 5;
    return ok_status();
  };

  if (*kase == 0) {
    CLM_CUDA((lc_vec<R, kLcFill>(st, n, x, v, w.isgn, 0)));
    *kase = 1;
    isave[0] = 1;
    return ok_status();
  }
  switch (isave[0]) {
    case 1:  // label 20: x = A (e / n)
      if (n == 1) {
        CLM_CUDA((lc_reduce<R, kLcAsum | kLcCopyV>(h, st, n, x, v, w, 0, &r)));
        *est = (R)r.asum;
        *kase = 0;
        return ok_status();
      }
      CLM_CUDA((lc_reduce<R, kLcAsum | kLcSign>(h, st, n, x, v, w, 0, &r)));
      *est = (R)r.asum;
      *kase = 2;
      isave[0] = 2;
      return ok_status();
    case 2:  // label 40: x = A^T sign, first column guess
      CLM_CUDA((lc_reduce<R, kLcArgmax>(h, st, n, x, v, w, 0, &r)));
      isave[1] = r.imax;
      isave[2] = 2;
      return to_unit();
    case 3: {  // label 70: x = A e_j
      CLM_CUDA((lc_reduce<R, kLcAsum | kLcChanged | kLcCopyV>(h, st, n, x, v, w, 0, &r)));
      const R estold = *est;
      *est = (R)r.asum;
      // a repeated sign vector means convergence, a non-increasing est cycling
      if (!r.changed || *est <= estold) return to_final();
      CLM_CUDA((lc_vec<R, kLcSignOnly>(st, n, x, v, w.isgn, 0)));
      *kase = 2;
      isave[0] = 4;
      return ok_status();
    }
    case 4: {  // label 110: x = A^T sign, next column guess
      const int jlast = isave[1];
      if (jlast < 1 || jlast > n) return blas_status(CALAMAN_STATUS_INVALID_VALUE);
      CLM_CUDA((lc_reduce<R, kLcArgmax>(h, st, n, x, v, w, jlast, &r)));
      isave[1] = r.imax;
      if (r.xlast != std::fabs(r.xnew) && isave[2] < kItmax) {
        ++isave[2];
        return to_unit();
      }
      return to_final();
    }
    default: {  // label 140: x = A altsgn
      CLM_CUDA((lc_reduce<R, kLcAsum>(h, st, n, x, v, w, 0, &r)));
      const R temp = (R)2 * ((R)r.asum / (R)(3 * n));
      if (temp > *est) {
        CLM_CUDA((lc_vec<R, kLcCopy>(st, n, x, v, w.isgn, 0)));
        *est = temp;
      }
      *kase = 0;
      return ok_status();
    }
  }
}

}  // namespace
}  // namespace clm

using namespace clm;

extern "C" {

size_t calaman_lacn2_bufferSize_s(int n) {
  std::size_t b = 0;
  carve_lc<float>(nullptr, n, &b);
  return b;
}
size_t calaman_lacn2_bufferSize_d(int n) {
  std::size_t b = 0;
  carve_lc<double>(nullptr, n, &b);
  return b;
}
calamanStatus_t calaman_lacn2_s(calamanBlasHandle_t blas, int n, float *d_v, float *d_x, void *d_work,
                                size_t work_bytes, float *est, int *kase, int *isave) {
  return lacn2_api<float>(blas, n, d_v, d_x, d_work, work_bytes, est, kase, isave);
}
calamanStatus_t calaman_lacn2_d(calamanBlasHandle_t blas, int n, double *d_v, double *d_x, void *d_work,
                                size_t work_bytes, double *est, int *kase, int *isave) {
  return lacn2_api<double>(blas, n, d_v, d_x, d_work, work_bytes, est, kase, isave);
}

}  // extern "C"
