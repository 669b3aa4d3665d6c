// herm.cu -- exp(A) for a symmetric / Hermitian A by eigendecomposition, and
// the eigensolver behind it.
//
// calaman::expm_herm (src/expm/expm_herm.cppm:97-199) forms A = U diag(w) U^H
// with the wrapped syevd / heevd, scales the eigenvector columns by exp(w_j)
// (herm_exp_scale, src/expm/expm.cu:170-184,289-297) and re-forms
// exp(A) = M U^H with one GEMM. It reads only the `uplo` triangle, never
// synchronises, and reports the eigensolver's status in one device int.
//
// The eigensolver here is this library's own, built for the GPU in four
// stages that never return to the host:
//
//  1. Tridiagonal reduction (LAPACK xHETD2's Householder sequence,
//     H_k = I - tau_k v_k v_k^H, Q^H A Q = T with real off-diagonal) in ONE
//     cooperative launch: every CTA owns the columns c = blockIdx.x (mod
//     grid) of the full Hermitian working copy (kept in L2 for the sizes the
//     path meets) and each step k is two grid barriers -- (a) every CTA reads
//     column k, forms the reflector redundantly (so no broadcast is needed)
//     and, in the same pass, the dot products of its columns with it (the
//     Hermitian product p = tau A22 v, column-wise); (b) after the p's are
//     published, every CTA forms alpha = -1/2 tau p^H v and applies the rank-2
//     update A22 -= v w^H + w v^H to its own columns. Barriers spin on an
//     acquire load with an iteration limit; one that runs out sets an error
//     word and every CTA returns.
//  2. Divide and conquer on the real symmetric tridiagonal (Cuppen's
//     tearing with Gu-Eisenstat eigenvectors, the method of LAPACK xSTEDC),
//     bottom-up from 1 x 1 leaves in FP64: per level, one launch per step over
//     all merges of the level -- deflation (LAPACK xLAED2's two tests, small
//     z component and close poles by a Givens rotation), the secular
//     equation roots (safeguarded two-pole rational iteration, differences
//     d_i - lambda_j kept relative to the nearer pole), the Gu-Eisenstat
//     z-hat that makes the computed roots exact for a nearby problem, the
//     normalised vectors placed at their eigenvalue's rank, and the product
//     Q_new = Q_old U (DMMA GEMM per merge, or a shared-memory kernel for
//     the small merges of the low levels).
//  3. Back-transformation U = Q Z by blocks of 64 reflectors in compact WY
//     form (I - V T V^H, T from the Gram matrix V^H V), three GEMMs a block.
//  4. (expm_herm) M = U diag(exp(w)), exp(A) = M U^H.
//
// FP32 / complex64 inputs are promoted and solved in FP64 (their results are
// rounded back at the end). The input is scaled into the safe range first,
// as LAPACK xHEEVD does (max |a_ij| outside [sqrt(smlnum), sqrt(bignum)]),
// and the tridiagonal by its max-norm, as xSTEDC does.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "kernels.cuh"
#include "expm_common.cuh"

namespace clm {
namespace {

// ---- element helpers (FP64 compute types: double, double2) ----------------
__device__ __forceinline__ double cj(double x) { return x; }
__device__ __forceinline__ double2 cj(double2 x) { return make_double2(x.x, -x.y); }
__device__ __forceinline__ double re(double x) { return x; }
__device__ __forceinline__ double re(double2 x) { return x.x; }
__device__ __forceinline__ double abs2(double x) { return x * x; }
__device__ __forceinline__ double abs2(double2 x) { return x.x * x.x + x.y * x.y; }
__device__ __forceinline__ double sub_(double a, double b) { return a - b; }
__device__ __forceinline__ double2 sub_(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C from_re(double r);
template <> __device__ __forceinline__ double from_re<double>(double r) { return r; }
template <> __device__ __forceinline__ double2 from_re<double2>(double r) { return make_double2(r, 0.0); }

__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }
__device__ __forceinline__ double2 ldcg(const double2 *p) { return __ldcg(p); }

__device__ __forceinline__ double shfl_xor(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ double2 shfl_xor(double2 v, int o) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}
// max with NaN sticky (a NaN operand wins)
__device__ __forceinline__ double max_nan(double a, double b) { return (a > b || a != a) ? a : b; }
__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = max_nan(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <typename V>
__device__ __forceinline__ V warp_sum(V v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = add(v, shfl_xor(v, o));
  return v;
}
// Sum over the block, returned to every thread (same order everywhere).
template <typename V, int kWarps>
__device__ __forceinline__ V block_sum(V v, V *red) {
  static_assert(kWarps <= 32, "one partial per lane");
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  V t{};
  if ((threadIdx.x & 31) < kWarps) t = red[threadIdx.x & 31];
  return warp_sum(t);  // every warp forms the same total from the same partials
}

// ---- bounded grid barrier ---------------------------------------------------
constexpr unsigned kSpinLimit = 1u << 24;  // x ~100 ns sleeps: seconds, then give up

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// All CTAs of the (co-resident, cooperatively launched) grid meet here. The
// counter only grows: barrier e is passed when it reaches e * gridDim.x.
// Returns false (for every thread of the CTA) when the wait ran out or another
// CTA reported a failure; the caller then returns.
__device__ __forceinline__ void red_add_release(unsigned *p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The arrival is a release (it publishes every write the CTA made before the
// block barrier), the polls are acquires (later reads of the CTA see every
// CTA's published writes).
__device__ bool grid_sync(unsigned *count, int *err, unsigned &epoch, int *s_ok, unsigned limit = kSpinLimit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    ++epoch;
    const unsigned target = epoch * gridDim.x;
    red_add_release(count, 1u);
    int ok = 1;
    unsigned spins = 0;
    while (ld_acquire(count) < target) {
      if (++spins > limit || *(volatile int *)err) {
        ok = 0;
        break;
      }
      __nanosleep(20);
    }
    if (!ok) atomicExch(err, 1);
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// Self-test of the barrier's bound: CTA 1 never arrives, so CTA 0's wait runs
// out after `limit` polls, records the failure in *err and returns.
__global__ void grid_sync_check_kernel(unsigned *count, int *err, unsigned limit) {
  __shared__ int s_ok;
  unsigned epoch = 0;
  if (blockIdx.x != 0) return;
  grid_sync(count, err, epoch, &s_ok, limit);
}

// ---- stage 0: range scaling and the Hermitian working copy -----------------
template <typename T>
__global__ void herm_maxabs_kernel(int n, const T *__restrict__ A, int lda, int upper,
                                   unsigned long long *__restrict__ amax) {
  double m = 0.0;
  const long long total = (long long)n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    if (upper ? (i <= j) : (i >= j)) {
      m = max_nan(modulus(A[(std::size_t)j * lda + i]), m);
    }
  }
  // non-negative doubles (and NaN above +inf) order like their bit patterns
  m = warp_max_d(m);
  if ((threadIdx.x & 31) == 0) atomicMax(amax, (unsigned long long)__double_as_longlong(m));
}

// sigma: the factor that brings max |a_ij| into [sqrt(smlnum), sqrt(bignum)]
// (LAPACK xHEEVD), 1 when it is there already or zero.
__device__ __forceinline__ double herm_sigma(const unsigned long long *amax) {
  const double anrm = __longlong_as_double((long long)*amax);
  const double smlnum = DBL_MIN / DBL_EPSILON;
  const double rmin = sqrt(smlnum), rmax = sqrt(1.0 / smlnum);
  if (anrm > 0.0 && anrm < rmin) return rmin / anrm;
  if (anrm > rmax) return rmax / anrm;
  return 1.0;
}

__device__ __forceinline__ double2 to_c2(float x) { return make_double2((double)x, 0.0); }
__device__ __forceinline__ double2 to_c2(double x) { return make_double2(x, 0.0); }
__device__ __forceinline__ double2 to_c2(float2 x) { return make_double2(x.x, x.y); }
__device__ __forceinline__ double2 to_c2(double2 x) { return x; }
__device__ __forceinline__ double to_c(float x) { return (double)x; }
__device__ __forceinline__ double to_c(double x) { return x; }
__device__ __forceinline__ double2 to_c(float2 x) { return make_double2(x.x, x.y); }
__device__ __forceinline__ double2 to_c(double2 x) { return x; }

// W (n x n, ld n, FP64) = sigma * the Hermitian matrix whose `uplo` triangle
// is A's; the diagonal keeps its real part only.
template <typename T, typename C>
__global__ void herm_fill_kernel(int n, const T *__restrict__ A, int lda, int upper,
                                 const unsigned long long *__restrict__ amax, C *__restrict__ W) {
  const double sg = herm_sigma(amax);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    const bool stored = upper ? (i <= j) : (i >= j);
    C v = stored ? to_c(A[(std::size_t)j * lda + i]) : cj(to_c(A[(std::size_t)i * lda + j]));
    if (i == j) v = from_re<C>(re(v));
    W[(std::size_t)j * n + i] = scale(v, sg);
  }
}

// ---- stage 1: tridiagonal reduction, one cooperative launch ----------------
constexpr int kTrdThreads = 1024;
constexpr int kTrdWarps = kTrdThreads / 32;
constexpr int kTrdMaxGrid = 160;  // CTAs of the reduction: one per SM at most
constexpr int kTrdVecs = 5;       // pivot, v, next v, p, w (n each)

template <typename C>
struct TrdArgs {
  int n;
  C *W;
  double *d, *e;
  C *tau, *vsc, *p;
  C *vec;  // per-CTA vectors (4 n each) when they do not stay in shared memory
  unsigned *bar;
  int *err;
};

// xLARFG: H^H [alpha; x] = [beta; 0], beta real, H = I - tau v v^H with
// v = [1; scl x]. Real: tau = 0 when x = 0; complex: when x = 0 and alpha
// is real.
__device__ __forceinline__ void reflector(double alpha, double xnorm2, double &tau, double &scl,
                                          double &beta) {
  if (xnorm2 == 0.0) {
    tau = 0.0;
    scl = 0.0;
    beta = alpha;
    return;
  }
  beta = -copysign(sqrt(alpha * alpha + xnorm2), alpha);
  tau = (beta - alpha) / beta;
  scl = 1.0 / (alpha - beta);
}
__device__ __forceinline__ void reflector(double2 alpha, double xnorm2, double2 &tau, double2 &scl,
                                          double &beta) {
  if (xnorm2 == 0.0 && alpha.y == 0.0) {
    tau = make_double2(0.0, 0.0);
    scl = make_double2(0.0, 0.0);
    beta = alpha.x;
    return;
  }
  beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
  // two independent reciprocals instead of a chain of divisions:
  // tau = (beta - alpha) / beta, scl = 1 / (alpha - beta) = conj(d) / |d|^2
  const double rb = 1.0 / beta;
  const double dr = alpha.x - beta, di = alpha.y;
  const double rd = 1.0 / (dr * dr + di * di);
  tau = make_double2((beta - alpha.x) * rb, -alpha.y * rb);
  scl = make_double2(dr * rd, -di * rd);
}

// One grid barrier per column, and one pass over the CTA's own columns per
// column. After the barrier of step k every CTA holds, identically, the pivot
// column k+1 brought up to date (the value its owner published, minus step
// k's rank-2 correction), forms reflector k+1 itself, and then sweeps its own
// columns once: each element gets step k's update and, still in registers,
// enters the dot product with v_{k+1} that is its share of step k+1's
// Hermitian product. Only that product p has to cross CTAs (double-buffered,
// so a CTA one step ahead never overwrites what a slower one still reads).
//   prologue: reflector 0, p^(0) = tau_0 A v_0 over the own columns;
//   step k: barrier; gather p^(k) and the published column k+1;
//     alpha_h = -1/2 tau_k p^H v_k, w = p + alpha_h v_k;
//     pivot k+1 = old column k+1 - v_k conj(w_{k+1}) - w conj(v_{k+1});
//     reflector k+1; own columns c >= k+2 -= v_k conj(w_c) + w conj(v_k,c)
//     fused with p^(k+1)_c = tau_{k+1} conj(col_c) . v_{k+1};
//     the owner of column k+2 publishes it.
// Column k+1 is never updated in place at step k (every CTA derives it), so
// reading its published value races with nothing. kRes keeps the CTA's own
// columns and the five vectors in shared memory; otherwise the columns stay
// in W (L2) and the vectors in a per-CTA global scratch.
template <typename C, bool kRes>
__device__ __forceinline__ C trd_ld(const C *p) {
  if constexpr (kRes) return *p;
  else return ldcg(p);
}

template <typename C, bool kRes>
__global__ void __launch_bounds__(kTrdThreads, 1) hetrd_kernel(TrdArgs<C> a) {
  extern __shared__ __align__(16) unsigned char trd_smem[];
  __shared__ C red_c[kTrdWarps];
  __shared__ double red_d[kTrdWarps];
  __shared__ int s_ok;
  const int n = a.n, G = gridDim.x, b = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ncmax = (n + G - 1) / G;
  C *acc = reinterpret_cast<C *>(trd_smem);  // max(ncmax, kTrdWarps) partial dots
  C *xv, *res = nullptr;
  if constexpr (kRes) {
    xv = acc + (ncmax > kTrdWarps ? ncmax : kTrdWarps);
    res = xv + kTrdVecs * (std::size_t)n;  // own column j at res + j n
  } else {
    xv = a.vec + (std::size_t)b * kTrdVecs * n;
  }
  C *vv = xv + n, *vn = vv + n, *pv = vn + n, *wv = pv + n;
  const C zero = from_re<C>(0.0), one = from_re<C>(1.0);
  if constexpr (kRes) {
    for (int j = 0; j < ncmax; ++j) {
      const int c = b + j * G;
      if (c >= n) break;
      for (int r = tid; r < n; r += kTrdThreads) res[(std::size_t)j * n + r] = ldcg(a.W + (std::size_t)c * n + r);
    }
  }
  for (int i = tid; i < n; i += kTrdThreads) xv[i] = ldcg(a.W + i);  // the first pivot, column 0
  __syncthreads();
  // own columns c >= first, as (index of the first, count, warps per column)
  auto own = [&](int first, int &c0, int &nc, int &j0, int &wpc) {
    c0 = first + ((b - first) % G + G) % G;
    nc = c0 < n ? (n - 1 - c0) / G + 1 : 0;
    j0 = (c0 - b) / G;
    wpc = nc > 0 && nc < kTrdWarps ? kTrdWarps / nc : 1;
  };
  auto column = [&](int c0, int j0, int j) -> C * {
    if constexpr (kRes) return res + (std::size_t)(j0 + j) * n;
    else return a.W + (std::size_t)(c0 + j * G) * n;
  };
  C tau = zero, scl = zero;
  if (n > 1) {
    // prologue: reflector 0 and p^(0) = tau_0 conj(col_c) . v_0, own c >= 1
    double nrm = 0.0;
    for (int i = 2 + tid; i < n; i += kTrdThreads) nrm += abs2(xv[i]);
    double beta;
    reflector(xv[1], block_sum<double, kTrdWarps>(nrm, red_d), tau, scl, beta);
    for (int i = 1 + tid; i < n; i += kTrdThreads) vv[i] = (i == 1) ? one : mul(scl, xv[i]);
    if (b == 0 && tid == 0) {
      a.d[0] = re(xv[0]);
      a.e[0] = beta;
      a.tau[0] = tau;
      a.vsc[0] = scl;
    }
    __syncthreads();
    int c0, nc, j0, wpc;
    own(1, c0, nc, j0, wpc);
    for (int jw = warp; jw < nc * wpc; jw += kTrdWarps) {
      const int j = jw / wpc, sub = jw - j * wpc;
      const C *col = column(c0, j0, j);
      C sacc = zero;
#pragma unroll 4
      for (int i = 1 + lane + 32 * sub; i < n; i += 32 * wpc) sacc = fmac(cj(trd_ld<C, kRes>(col + i)), vv[i], sacc);
      sacc = warp_sum(sacc);
      if (lane == 0) acc[jw] = sacc;
    }
    __syncthreads();
    for (int j = tid; j < nc; j += kTrdThreads) {
      C dot = acc[j * wpc];
      for (int sub = 1; sub < wpc; ++sub) dot = add(dot, acc[j * wpc + sub]);
      a.p[c0 + j * G] = mul(tau, dot);
    }
  }
  unsigned epoch = 0;
  for (int k = 0; k + 1 < n; ++k) {
    if (!grid_sync(a.bar, a.err, epoch, &s_ok)) return;
    const C *pk = a.p + (std::size_t)(k & 1) * n;
    C *pn = a.p + (std::size_t)((k + 1) & 1) * n;
    // the pivot column k is read by nobody else now: store it for the back-transform
    if (b == 0)
      for (int i = k + 1 + tid; i < n; i += kTrdThreads) a.W[(std::size_t)k * n + i] = xv[i];
    // gather p^(k) and the published column k+1
    C part = zero;
    for (int i = k + 1 + tid; i < n; i += kTrdThreads) {
      const C pi = ldcg(pk + i);
      pv[i] = pi;
      wv[i] = ldcg(a.W + (std::size_t)(k + 1) * n + i);
      part = fmac(cj(pi), vv[i], part);
    }
    const C phv = block_sum<C, kTrdWarps>(part, red_c);  // also orders the CTA-0 store above
    const C ah = scale(mul(tau, phv), -0.5);
    const C cw1 = cj(add(pv[k + 1], ah));  // conj(w_{k+1}); v_{k+1} = 1
    double nrm = 0.0;
    for (int i = k + 1 + tid; i < n; i += kTrdThreads) {
      const C wi = fmac(ah, vv[i], pv[i]);
      C x = sub_(wv[i], add(mul(vv[i], cw1), wi));
      if (i == k + 1) x = from_re<C>(re(x));
      xv[i] = x;
      wv[i] = wi;
      if (i >= k + 3) nrm += abs2(x);
    }
    const double xnorm2 = block_sum<double, kTrdWarps>(nrm, red_d);  // xv, wv complete
    const bool more = k + 2 < n;  // a reflector k+1 exists
    C taun = zero, scln = zero;
    if (more) {
      double beta;
      reflector(xv[k + 2], xnorm2, taun, scln, beta);
      for (int i = k + 2 + tid; i < n; i += kTrdThreads) vn[i] = (i == k + 2) ? one : mul(scln, xv[i]);
      if (b == 0 && tid == 0) {
        a.d[k + 1] = re(xv[k + 1]);
        a.e[k + 1] = beta;
        a.tau[k + 1] = taun;
        a.vsc[k + 1] = scln;
      }
    }
    __syncthreads();
    // own columns c >= k+2: update (rows k+1..) fused with the next dot (rows k+2..)
    {
      int c0, nc, j0, wpc;
      own(k + 2, c0, nc, j0, wpc);
      for (int jw = warp; jw < nc * wpc; jw += kTrdWarps) {
        const int j = jw / wpc, sub = jw - j * wpc;
        const int c = c0 + j * G;
        C *col = column(c0, j0, j);
        const C cvc = cj(vv[c]), cwc = cj(wv[c]);
        C sacc = zero;
#pragma unroll 4
        for (int i = k + 1 + lane + 32 * sub; i < n; i += 32 * wpc) {
          C y = sub_(trd_ld<C, kRes>(col + i), add(mul(vv[i], cwc), mul(wv[i], cvc)));
          if (i == c) y = from_re<C>(re(y));
          col[i] = y;
          if (i >= k + 2) sacc = fmac(cj(y), vn[i], sacc);
        }
        sacc = warp_sum(sacc);
        if (lane == 0) acc[jw] = sacc;
      }
      __syncthreads();
      if (more)
        for (int j = tid; j < nc; j += kTrdThreads) {
          C dot = acc[j * wpc];
          for (int sub = 1; sub < wpc; ++sub) dot = add(dot, acc[j * wpc + sub]);
          pn[c0 + j * G] = mul(taun, dot);
        }
    }
    if constexpr (kRes) {
      // the owner of column k+2 publishes it (rows k+2..) for the next step
      if (more && (k + 2) % G == b) {
        const C *src = res + (std::size_t)((k + 2 - b) / G) * n;
        for (int r = k + 2 + tid; r < n; r += kTrdThreads) a.W[(std::size_t)(k + 2) * n + r] = src[r];
      }
    }
    C *t = vv;
    vv = vn;
    vn = t;
    tau = taun;
    scl = scln;
  }
  if (b == 0 && tid == 0) a.d[n - 1] = re(xv[n - 1]);
}

// ---- stage 2: divide and conquer on the tridiagonal (FP64) -----------------
struct DcWs {
  double *Za, *Zb, *DEL, *UF;
  double *lamA, *lamB, *dd, *ee;
  double *srt_d, *srt_z, *nd_d, *nd_z, *df_d, *rot_c, *rot_s, *nd_lam, *zh;
  int *srt_c, *nd_c, *df_c, *rot_a, *rot_b, *cnt;
  double *sc;  // [0] the tridiagonal's scale
};

constexpr int kDcThreads = 256;
constexpr int kDcScanSmem = 4096;  // merges up to this size scan in shared memory

// dd = (T's diagonal - the tearing corrections) / sc, ee = e / sc, sc = max
// |T_ij| (xSTEDC's scaling); leaves: lamA = dd, Za = I (Za, Zb zeroed before).
__global__ void __launch_bounds__(1024) dc_init_kernel(int n, const double *__restrict__ d,
                                                       const double *__restrict__ e, DcWs w) {
  __shared__ double red[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    m = fmax(m, fabs(d[i]));
    if (i + 1 < n) m = fmax(m, fabs(e[i]));
  }
  m = warp_max_d(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t = fmax(t, red[i]);
    red[0] = t > 0.0 ? t : 1.0;
  }
  __syncthreads();
  const double sc = red[0];
  if (threadIdx.x == 0) w.sc[0] = sc;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double v = d[i] / sc;
    if (i > 0) v -= fabs(e[i - 1] / sc);
    if (i + 1 < n) v -= fabs(e[i] / sc);
    w.dd[i] = v;
    w.lamA[i] = v;
    w.ee[i] = i + 1 < n ? e[i] / sc : 0.0;
    w.Za[(std::size_t)i * n + i] = 1.0;
  }
}

struct DcLevel {
  int n, b;  // half size; merges q start at b0 = 2bq, left n1 = b, right n2 = min(b, n - b0 - b)
  int scan_smem;  // 1: the deflation scan stages its merge in dynamic shared memory
  const double *lam;  // this level's input eigenvalues (ascending per block)
  double *lam_out;
  double *Z;  // input eigenvectors (block diagonal)
};

__device__ __forceinline__ void merge_dims(const DcLevel &L, int q, int &b0, int &n1, int &m) {
  b0 = 2 * L.b * q;
  n1 = L.b;
  m = n1 + min(L.b, L.n - b0 - L.b);
}
__device__ __forceinline__ std::size_t merge_off(const DcLevel &L, int b0) {
  return (std::size_t)b0 * (2 * L.b);  // the merge's m x m scratch (ld m) in DEL / UF
}

// Lower bound: elements of the sorted x[0, len) strictly below v (or <= v).
__device__ __forceinline__ int count_below(const double *x, int len, double v, bool or_equal) {
  int lo = 0, hi = len;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const bool go = or_equal ? (x[mid] <= v) : (x[mid] < v);
    if (go) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// z, the merged order and the deflation scan (xLAED2's two tests).
__global__ void __launch_bounds__(kDcThreads) dc_deflate_kernel(DcLevel L, DcWs w) {
  extern __shared__ double dsm[];  // [2 * m] when m <= kDcScanSmem
  __shared__ double red[2][kDcThreads / 32];
  const int q = blockIdx.x;
  int b0, n1, m;
  merge_dims(L, q, b0, n1, m);
  const int n = L.n;
  const double beta = w.ee[b0 + n1 - 1];
  const double rho = 2.0 * fabs(beta);
  const double sgn = beta < 0.0 ? -1.0 : 1.0;
  const double *lam = L.lam + b0;
  double dmax = 0.0, zmax = 0.0;
  for (int i = threadIdx.x; i < m; i += kDcThreads) {
    const double x = lam[i];
    double z;
    int pos;
    if (i < n1) {
      z = L.Z[(std::size_t)(b0 + i) * n + (b0 + n1 - 1)];
      pos = i + count_below(lam + n1, m - n1, x, false);
    } else {
      z = sgn * L.Z[(std::size_t)(b0 + i) * n + (b0 + n1)];
      pos = (i - n1) + count_below(lam, n1, x, true);
    }
    z *= 0.70710678118654752440;  // the two unit rows make |z| = sqrt(2)
    w.srt_d[b0 + pos] = x;
    w.srt_z[b0 + pos] = z;
    w.srt_c[b0 + pos] = i;
    dmax = fmax(dmax, fabs(x));
    zmax = fmax(zmax, fabs(z));
  }
  dmax = warp_max_d(dmax);
  zmax = warp_max_d(zmax);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = dmax;
    red[1][threadIdx.x >> 5] = zmax;
  }
  __syncthreads();
  const bool in_smem = L.scan_smem != 0;
  double *sd = in_smem ? dsm : w.srt_d + b0;
  double *sz = in_smem ? dsm + m : w.srt_z + b0;
  if (in_smem) {
    for (int i = threadIdx.x; i < m; i += kDcThreads) {
      dsm[i] = w.srt_d[b0 + i];
      dsm[m + i] = w.srt_z[b0 + i];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  for (int i = 1; i < kDcThreads / 32; ++i) {
    dmax = fmax(dmax, red[0][i]);
    zmax = fmax(zmax, red[1][i]);
  }
  const double tol = 8.0 * DBL_EPSILON * fmax(dmax, zmax);
  const int *sc_ = w.srt_c + b0;
  double *ndd = w.nd_d + b0, *ndz = w.nd_z + b0, *dfd = w.df_d + b0;
  int *ndc = w.nd_c + b0, *dfc = w.df_c + b0;
  int k = 0, ndf = 0, nr = 0;
  if (rho * zmax <= tol) {
    for (int j = 0; j < m; ++j) {
      dfd[ndf] = sd[j];
      dfc[ndf++] = sc_[j];
    }
  } else {
    int prev = -1;
    for (int j = 0; j < m; ++j) {
      const double zj = sz[j];
      if (rho * fabs(zj) <= tol) {
        dfd[ndf] = sd[j];
        dfc[ndf++] = sc_[j];
        continue;
      }
      if (prev < 0) {
        prev = j;
        continue;
      }
      const double zp = sz[prev];
      const double t = sd[j] - sd[prev];
      const double tt = zj * zj + zp * zp;  // |t c s| <= tol with c = zj/tau, s = -zp/tau
      if (fabs(t * zj * zp) <= tol * tt) {
        // close poles: rotate columns (prev, j) so z_prev = 0 and deflate prev
        const double tau = sqrt(tt);
        const double c = zj / tau, s = -zp / tau;
        sz[j] = tau;
        sz[prev] = 0.0;
        w.rot_a[b0 + nr] = sc_[prev];
        w.rot_b[b0 + nr] = sc_[j];
        w.rot_c[b0 + nr] = c;
        w.rot_s[b0 + nr] = s;
        ++nr;
        const double dp = sd[prev], dn = sd[j];
        sd[prev] = dp * c * c + dn * s * s;
        sd[j] = dp * s * s + dn * c * c;
        dfd[ndf] = sd[prev];
        dfc[ndf++] = sc_[prev];
      } else {
        ndd[k] = sd[prev];
        ndz[k] = sz[prev];
        ndc[k++] = sc_[prev];
      }
      prev = j;
    }
    if (prev >= 0) {
      ndd[k] = sd[prev];
      ndz[k] = sz[prev];
      ndc[k++] = sc_[prev];
    }
  }
  w.cnt[3 * q] = k;
  w.cnt[3 * q + 1] = ndf;
  w.cnt[3 * q + 2] = nr;
}

// Apply the deflation rotations, in order, to the merge's block of Z (each
// thread one row).
__global__ void __launch_bounds__(kDcThreads) dc_rotate_kernel(DcLevel L, DcWs w) {
  const int q = blockIdx.y;
  int b0, n1, m;
  merge_dims(L, q, b0, n1, m);
  const int r = blockIdx.x * kDcThreads + threadIdx.x;
  const int nr = w.cnt[3 * q + 2];
  if (r >= m || nr == 0) return;
  double *Z = L.Z + (std::size_t)b0 * L.n + b0 + r;  // Z(b0 + r, b0 + col) = Z[col * n]
  for (int t = 0; t < nr; ++t) {
    const int ca = w.rot_a[b0 + t], cb = w.rot_b[b0 + t];
    // a NaN input can leave merged-order slots unwritten (equal ranks), so a
    // column index read back through them is checked before it addresses memory
    if ((unsigned)ca >= (unsigned)m || (unsigned)cb >= (unsigned)m) continue;
    const double c = w.rot_c[b0 + t], s = w.rot_s[b0 + t];
    const double xa = Z[(std::size_t)ca * L.n], xb = Z[(std::size_t)cb * L.n];
    Z[(std::size_t)ca * L.n] = c * xa + s * xb;
    Z[(std::size_t)cb * L.n] = c * xb - s * xa;
  }
}

// Root j of 1/rho + sum_i z_i^2 / (d_i - lambda) = 0 (d ascending, rho > 0):
// lambda_j in (d_j, d_{j+1}), the last in (d_{k-1}, d_{k-1} + rho |z|^2).
// The unknown is tau = lambda - d_K with K the nearer pole, so every
// difference d_i - lambda = (d_i - d_K) - tau keeps full relative accuracy.
// Each step fits psi (poles i <= j) and phi (poles i > j) by c + s/(d - x)
// through value and slope and takes the root of the fitted two-pole
// equation, falling back to bisection of the bracket. One warp per root: the
// lanes share the sums (every lane ends with the same totals, so the
// iteration is warp-uniform).
constexpr int kSecWarps = 4;
__global__ void __launch_bounds__(32 * kSecWarps) dc_secular_kernel(DcLevel L, DcWs w) {
  const int q = blockIdx.y;
  int b0, n1, m;
  merge_dims(L, q, b0, n1, m);
  const int j = blockIdx.x * kSecWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int k = w.cnt[3 * q];
  if (j >= k) return;
  const double *dv = w.nd_d + b0, *zv = w.nd_z + b0;
  const double rho = 2.0 * fabs(w.ee[b0 + n1 - 1]);
  double *del = w.DEL + merge_off(L, b0) + (std::size_t)j * m;
  const double rinv = 1.0 / rho;
  int K = j;
  double lo, hi;
  if (j + 1 < k) {
    const double gap = dv[j + 1] - dv[j];
    const double mid = 0.5 * gap;
    double g = 0.0;
    for (int i = lane; i < k; i += 32) g += zv[i] * zv[i] / ((dv[i] - dv[j]) - mid);
    g = rinv + warp_sum(g);
    if (g >= 0.0) {
      K = j;
      lo = 0.0;
      hi = mid;
    } else {
      K = j + 1;  // tau relative to d_{j+1}: (d_j - d_{j+1}) + mid = -mid
      lo = -mid;
      hi = 0.0;
    }
  } else {
    double zz = 0.0;
    for (int i = lane; i < k; i += 32) zz += zv[i] * zv[i];
    lo = 0.0;
    hi = rho * warp_sum(zz);
  }
  const double dK = dv[K];
  const double dj = dv[j] - dK;                           // pole j relative to the origin
  const double dj1 = (j + 1 < k) ? dv[j + 1] - dK : 0.0;  // pole j+1 (unused for the last root)
  double tau = 0.5 * (lo + hi);
  for (int it = 0; it < 100; ++it) {
    double psi = 0.0, phi = 0.0, dpsi = 0.0, dphi = 0.0;
    for (int i = lane; i < k; i += 32) {
      const double dl = (dv[i] - dK) - tau;
      const double t = zv[i] / dl;
      if (i <= j) {
        psi += zv[i] * t;
        dpsi += t * t;
      } else {
        phi += zv[i] * t;
        dphi += t * t;
      }
    }
    psi = warp_sum(psi);
    phi = warp_sum(phi);
    dpsi = warp_sum(dpsi);
    dphi = warp_sum(dphi);
    const double g = rinv + psi + phi;
    if (g == 0.0) break;
    if (g < 0.0) lo = tau;
    else hi = tau;
    const double tolg = 8.0 * DBL_EPSILON * (rinv + fabs(psi) + fabs(phi) + fabs(tau) * (dpsi + dphi));
    if (fabs(g) <= tolg) break;
    if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi))) break;
    // two-pole model through (psi, dpsi) at pole dj and (phi, dphi) at dj1
    const double Dj = dj - tau;
    double next;
    if (j + 1 < k) {
      const double Dj1 = dj1 - tau;
      const double sj = dpsi * Dj * Dj, sj1 = dphi * Dj1 * Dj1;
      const double Cm = rinv + (psi - dpsi * Dj) + (phi - dphi * Dj1);
      // Cm + sj/(dj - x) + sj1/(dj1 - x) = 0; with u = x - tau:
      // Cm (Dj - u)(Dj1 - u) + sj (Dj1 - u) + sj1 (Dj - u) = 0
      const double qa = Cm, qb = -(Cm * (Dj + Dj1) + sj + sj1), qc = Cm * Dj * Dj1 + sj * Dj1 + sj1 * Dj;
      double u = NAN;
      if (qa == 0.0) {
        if (qb != 0.0) u = -qc / qb;
      } else {
        const double disc = fmax(qb * qb - 4.0 * qa * qc, 0.0);
        const double qq = -0.5 * (qb + copysign(sqrt(disc), qb));
        const double u1 = qq / qa, u2 = qq != 0.0 ? qc / qq : NAN;
        const double x1 = tau + u1, x2 = tau + u2;
        const bool in1 = x1 > lo && x1 < hi, in2 = x2 > lo && x2 < hi;
        u = in1 ? u1 : (in2 ? u2 : NAN);
      }
      next = tau + u;
    } else {
      const double sj = dpsi * Dj * Dj;
      const double Cm = rinv + (psi - dpsi * Dj) + phi;
      next = Cm > 0.0 ? dj + sj / Cm : NAN;  // Cm + sj/(dj - x) = 0
    }
    tau = (next > lo && next < hi) ? next : 0.5 * (lo + hi);
  }
  for (int i = lane; i < k; i += 32) del[i] = (dv[i] - dK) - tau;
  if (lane == 0) w.nd_lam[b0 + j] = dK + tau;
}

// Gu-Eisenstat: zhat_i^2 = (lambda_i - d_i)/rho * prod_{j != i} (lambda_j - d_i)/(d_j - d_i),
// the z for which the computed roots are exact; sign from z. One warp per i
// (lane partial products, then a xor-butterfly product).
__global__ void __launch_bounds__(32 * kSecWarps) dc_zhat_kernel(DcLevel L, DcWs w) {
  const int q = blockIdx.y;
  int b0, n1, m;
  merge_dims(L, q, b0, n1, m);
  const int i = blockIdx.x * kSecWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int k = w.cnt[3 * q];
  if (i >= k) return;
  const double *dv = w.nd_d + b0;
  const double rho = 2.0 * fabs(w.ee[b0 + n1 - 1]);
  const double *del = w.DEL + merge_off(L, b0);
  double prod = 1.0;
  for (int j = lane; j < k; j += 32)
    prod *= (j == i) ? -del[(std::size_t)i * m + i] / rho : -del[(std::size_t)j * m + i] / (dv[j] - dv[i]);
#pragma unroll
  for (int o = 16; o; o >>= 1) prod *= __shfl_xor_sync(0xffffffffu, prod, o);
  if (lane == 0) w.zh[b0 + i] = copysign(sqrt(fmax(prod, 0.0)), w.nd_z[b0 + i]);
}

// Place every eigenpair of the merge at its eigenvalue's rank: the
// nondeflated vectors u_t(i) = zhat_i / (d_i - lambda_t), normalised, into
// row nd_c[i] of UF's column rank(t); a deflated column c gets a unit entry.
// Ties rank deflated values first, then by list order. One warp per pair.
__global__ void __launch_bounds__(kDcThreads) dc_vectors_kernel(DcLevel L, DcWs w) {
  const int q = blockIdx.y;
  int b0, n1, m;
  merge_dims(L, q, b0, n1, m);
  const int item = blockIdx.x * (kDcThreads / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int k = w.cnt[3 * q], ndf = w.cnt[3 * q + 1];
  if (item >= k + ndf) return;
  const double *dfd = w.df_d + b0;
  double *UF = w.UF + merge_off(L, b0);
  if (item < k) {
    const int t = item;
    const double lam = w.nd_lam[b0 + t];
    int below = 0;
    for (int u = lane; u < ndf; u += 32) below += dfd[u] <= lam;
    below = __reduce_add_sync(0xffffffffu, below);
    const int pos = t + below;
    const double *del = w.DEL + merge_off(L, b0) + (std::size_t)t * m;
    double ss = 0.0;
    for (int i = lane; i < k; i += 32) {
      const double v = w.zh[b0 + i] / del[i];
      ss += v * v;
    }
    ss = warp_sum(ss);
    const double inv = 1.0 / sqrt(ss);
    for (int i = lane; i < k; i += 32) {
      const int col = w.nd_c[b0 + i];  // in range unless a NaN input broke the merge order
      if ((unsigned)col < (unsigned)m) UF[(std::size_t)pos * m + col] = w.zh[b0 + i] / del[i] * inv;
    }
    if (lane == 0) L.lam_out[b0 + pos] = lam;
  } else {
    const int u = item - k;
    const double x = dfd[u];
    int below = 0;
    for (int v = lane; v < ndf; v += 32) below += (dfd[v] < x) || (dfd[v] == x && v < u);
    below = __reduce_add_sync(0xffffffffu, below);
    if (lane == 0) {
      const int pos = below + count_below(w.nd_lam + b0, k, x, false);
      const int col = w.df_c[b0 + u];
      if ((unsigned)col < (unsigned)m) UF[(std::size_t)pos * m + col] = 1.0;
      L.lam_out[b0 + pos] = x;
    }
  }
}

// Small merges (m <= 64): Zout block = Z block x UF in shared memory, one CTA
// per merge.
constexpr int kDcSmallM = 64;
__global__ void __launch_bounds__(kDcThreads) dc_small_gemm_kernel(DcLevel L, DcWs w, double *Zout) {
  extern __shared__ double gsm[];  // [2 m m], m <= kDcSmallM
  const int q = blockIdx.x;
  int b0, n1, m;
  merge_dims(L, q, b0, n1, m);
  double *As = gsm, *Bs = gsm + m * m;
  const int n = L.n;
  const double *UF = w.UF + merge_off(L, b0);
  for (int idx = threadIdx.x; idx < m * m; idx += kDcThreads) {
    const int r = idx % m, c = idx / m;
    As[idx] = L.Z[(std::size_t)(b0 + c) * n + b0 + r];
    Bs[idx] = UF[idx];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < m * m; idx += kDcThreads) {
    const int r = idx % m, c = idx / m;
    double s = 0.0;
    for (int l = 0; l < m; ++l) s = fma(As[l * m + r], Bs[c * m + l], s);
    Zout[(std::size_t)(b0 + c) * n + b0 + r] = s;
  }
}

// A block without a partner at this level moves to the output buffers as is.
__global__ void dc_carry_kernel(int n, int b0, const double *__restrict__ Zin, const double *__restrict__ lam,
                                double *__restrict__ Zout, double *__restrict__ lam_out) {
  const int m = n - b0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < m * m; idx += gridDim.x * blockDim.x) {
    const int r = idx % m, c = idx / m;
    Zout[(std::size_t)(b0 + c) * n + b0 + r] = Zin[(std::size_t)(b0 + c) * n + b0 + r];
    if (c == 0) lam_out[b0 + r] = lam[b0 + r];
  }
}

__global__ void dc_unscale_kernel(int n, const double *__restrict__ lam, const double *__restrict__ sc,
                                  double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = lam[i] * sc[0];
}

// Eigenvalues (ascending) into lam_final and eigenvectors of the tridiagonal
// (d, e) into *Zfinal (one of w.Za / w.Zb).
cudaError_t stedc_run(cudaStream_t s, int n, const double *d, const double *e, DcWs &w, double *lam_final,
                      double **Zfinal) {
  cudaError_t err;
  const std::size_t nn = (std::size_t)n * n;
  if ((err = cudaFuncSetAttribute(dc_deflate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  2 * kDcScanSmem * (int)sizeof(double))) != cudaSuccess)
    return err;
  if ((err = cudaFuncSetAttribute(dc_small_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  2 * kDcSmallM * kDcSmallM * (int)sizeof(double))) != cudaSuccess)
    return err;
  if ((err = cudaMemsetAsync(w.Za, 0, nn * sizeof(double), s)) != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(w.Zb, 0, nn * sizeof(double), s)) != cudaSuccess) return err;
  dc_init_kernel<<<1, 1024, 0, s>>>(n, d, e, w);
  if ((err = launched()) != cudaSuccess) return err;
  double *Zin = w.Za, *Zout = w.Zb, *lin = w.lamA, *lout = w.lamB;
  for (int b = 1; b < n; b *= 2) {
    const int nm = (n - b + 2 * b - 1) / (2 * b);  // merges: b0 = 2bq with b0 + b < n
    const int mmax = 2 * b < n ? 2 * b : n;
    const int m_scan = mmax <= kDcScanSmem ? mmax : 0;
    DcLevel L{n, b, m_scan > 0, lin, lout, Zin};
    if ((err = cudaMemsetAsync(w.UF, 0, nn * sizeof(double), s)) != cudaSuccess) return err;
    dc_deflate_kernel<<<nm, kDcThreads, 2 * m_scan * sizeof(double), s>>>(L, w);
    if ((err = launched()) != cudaSuccess) return err;
    dc_rotate_kernel<<<dim3((mmax + kDcThreads - 1) / kDcThreads, nm), kDcThreads, 0, s>>>(L, w);
    if ((err = launched()) != cudaSuccess) return err;
    dc_secular_kernel<<<dim3((mmax + kSecWarps - 1) / kSecWarps, nm), 32 * kSecWarps, 0, s>>>(L, w);
    if ((err = launched()) != cudaSuccess) return err;
    dc_zhat_kernel<<<dim3((mmax + kSecWarps - 1) / kSecWarps, nm), 32 * kSecWarps, 0, s>>>(L, w);
    if ((err = launched()) != cudaSuccess) return err;
    dc_vectors_kernel<<<dim3((mmax + kDcThreads / 32 - 1) / (kDcThreads / 32), nm), kDcThreads, 0, s>>>(L, w);
    if ((err = launched()) != cudaSuccess) return err;
    if (mmax <= kDcSmallM) {
      dc_small_gemm_kernel<<<nm, kDcThreads, 2 * (std::size_t)mmax * mmax * sizeof(double), s>>>(L, w, Zout);
      if ((err = launched()) != cudaSuccess) return err;
    } else {
      for (int q = 0; q < nm; ++q) {
        const int b0 = 2 * b * q;
        const int m = b + (b < n - b0 - b ? b : n - b0 - b);
        const double *A = Zin + (std::size_t)b0 * n + b0;
        const double *B = w.UF + (std::size_t)b0 * (2 * b);
        if ((err = gemm_nn<double>(s, m, m, m, 1.0, A, n, B, m, 0.0, Zout + (std::size_t)b0 * n + b0, n)) !=
            cudaSuccess)
          return err;
      }
    }
    const int b0c = 2 * b * nm;
    if (b0c < n) {
      dc_carry_kernel<<<64, 256, 0, s>>>(n, b0c, Zin, lin, Zout, lout);
      if ((err = launched()) != cudaSuccess) return err;
    }
    double *tz = Zin;
    Zin = Zout;
    Zout = tz;
    double *tl = lin;
    lin = lout;
    lout = tl;
  }
  dc_unscale_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, lin, w.sc, lam_final);
  if ((err = launched()) != cudaSuccess) return err;
  *Zfinal = Zin;
  return cudaSuccess;
}

// ---- stage 3: back-transformation U = Q Z (compact WY blocks) --------------
constexpr int kWyBlock = 64;

// All blocks' V (mrows x kb, ld mrows) and V^H (kb x mrows, ld kb), packed
// block after block: block bi starts at 64 (bi (n-1) - 64 bi (bi-1) / 2).
__host__ __device__ __forceinline__ std::size_t wy_off(int n, int bi) {
  return (std::size_t)kWyBlock * ((std::size_t)bi * (n - 1) - (std::size_t)kWyBlock * bi * (bi - 1) / 2);
}

template <typename C>
__global__ void wy_build_kernel(int n, const C *__restrict__ W, const C *__restrict__ tau, const C *__restrict__ vsc,
                                C *__restrict__ Vall, C *__restrict__ VHall) {
  const int bi = blockIdx.z, j0 = bi * kWyBlock;
  const int kb = min(kWyBlock, n - 1 - j0), mrows = n - j0 - 1;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y;
  if (r >= mrows || jj >= kb) return;
  C *V = Vall + wy_off(n, bi);
  C *VH = VHall + wy_off(n, bi);
  const int j = j0 + jj, row = j0 + 1 + r;
  C v = from_re<C>(0.0);
  if (!is_zero(tau[j])) {
    if (row == j + 1) v = from_re<C>(1.0);
    else if (row > j + 1) v = mul(vsc[j], W[(std::size_t)j * n + row]);
  }
  V[(std::size_t)jj * mrows + r] = v;
  VH[(std::size_t)r * kb + jj] = cj(v);
}

// T (kb x kb, upper triangular) of every block (one CTA each) with
// H_j0 ... H_{j0+kb-1} = I - V T V^H: T(i,i) = tau_i,
// T(0:i, i) = -tau_i T(0:i, 0:i) G(0:i, i), G = V^H V. G and T live in
// shared memory (2 kb^2 elements); thread r owns row r.
template <typename C>
__global__ void wy_t_kernel(int n, const C *__restrict__ tau, const C *__restrict__ Gall, C *__restrict__ Tall) {
  extern __shared__ __align__(16) unsigned char wy_smem[];
  const int bi = blockIdx.x, j0 = bi * kWyBlock;
  const int kb = min(kWyBlock, n - 1 - j0);
  const C *G = Gall + (std::size_t)bi * kWyBlock * kWyBlock;
  C *T = Tall + (std::size_t)bi * kWyBlock * kWyBlock;
  C *Gs = reinterpret_cast<C *>(wy_smem);
  C *Ts = Gs + kb * kb;
  const int r = threadIdx.x;
  for (int idx = r; idx < kb * kb; idx += blockDim.x) {
    Gs[idx] = G[idx];
    Ts[idx] = from_re<C>(0.0);
  }
  __syncthreads();
  for (int i = 0; i < kb; ++i) {
    if (r < i) {
      C sacc = from_re<C>(0.0);
      for (int l = r; l < i; ++l) sacc = fmac(Ts[l * kb + r], Gs[i * kb + l], sacc);
      Ts[i * kb + r] = neg(mul(tau[j0 + i], sacc));  // column i: no thread reads it in this pass
    } else if (r == i) {
      Ts[i * kb + i] = tau[j0 + i];
    }
    __syncthreads();
  }
  for (int idx = r; idx < kb * kb; idx += blockDim.x) T[idx] = Ts[idx];
}

constexpr int kSplitMax = 16;  // K slices of the skinny back-transform products

template <typename C>
struct BtWs {
  C *Vall, *VHall;  // aliases of the divide-and-conquer scratch (free by then)
  C *G, *T, *Wm, *Wm2, *part;
};

__global__ void real_to_c_kernel(std::size_t count, const double *__restrict__ Z, double *__restrict__ U) {
  for (std::size_t i = blockIdx.x * (std::size_t)blockDim.x + threadIdx.x; i < count;
       i += (std::size_t)gridDim.x * blockDim.x)
    U[i] = Z[i];
}
__global__ void real_to_c_kernel(std::size_t count, const double *__restrict__ Z, double2 *__restrict__ U) {
  for (std::size_t i = blockIdx.x * (std::size_t)blockDim.x + threadIdx.x; i < count;
       i += (std::size_t)gridDim.x * blockDim.x)
    U[i] = make_double2(Z[i], 0.0);
}

template <typename C>
cudaError_t back_transform(cudaStream_t s, int n, const C *W, const C *tau, const C *vsc, const double *Z, C *U,
                           const BtWs<C> &bt) {
  cudaError_t err;
  const std::size_t nn = (std::size_t)n * n;
  real_to_c_kernel<<<(int)std::min<std::size_t>((nn + 255) / 256, 8 * 148), 256, 0, s>>>(nn, Z, U);
  if ((err = launched()) != cudaSuccess) return err;
  if (n < 2) return cudaSuccess;
  const int nblk = (n - 1 + kWyBlock - 1) / kWyBlock;
  // every block's V, V^H, Gram matrix and T first: none depends on U
  wy_build_kernel<C><<<dim3((n + 126) / 128, kWyBlock, nblk), 128, 0, s>>>(n, W, tau, vsc, bt.Vall, bt.VHall);
  if ((err = launched()) != cudaSuccess) return err;
  for (int bi = 0; bi < nblk; ++bi) {
    const int j0 = bi * kWyBlock, kb = std::min(kWyBlock, n - 1 - j0), mrows = n - j0 - 1;
    const C *V = bt.Vall + wy_off(n, bi), *VH = bt.VHall + wy_off(n, bi);
    if ((err = gemm_nn_splitk<C>(s, kb, kb, mrows, 1.0, VH, kb, V, mrows, 0.0,
                                 bt.G + (std::size_t)bi * kWyBlock * kWyBlock, kb, bt.part, kSplitMax)) !=
        cudaSuccess)
      return err;
  }
  if ((err = cudaFuncSetAttribute(wy_t_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  2 * kWyBlock * kWyBlock * (int)sizeof(C))) != cudaSuccess)
    return err;
  wy_t_kernel<C><<<nblk, kWyBlock, 2 * (std::size_t)kWyBlock * kWyBlock * sizeof(C), s>>>(n, tau, bt.G, bt.T);
  if ((err = launched()) != cudaSuccess) return err;
  // U = (I - V_0 T_0 V_0^H) ... (I - V_last T_last V_last^H) Z, the last block first
  for (int bi = nblk - 1; bi >= 0; --bi) {
    const int j0 = bi * kWyBlock, kb = std::min(kWyBlock, n - 1 - j0), mrows = n - j0 - 1;
    const C *V = bt.Vall + wy_off(n, bi), *VH = bt.VHall + wy_off(n, bi);
    const C *T = bt.T + (std::size_t)bi * kWyBlock * kWyBlock;
    C *Us = U + j0 + 1;
    if ((err = gemm_nn_splitk<C>(s, kb, n, mrows, 1.0, VH, kb, Us, n, 0.0, bt.Wm, kb, bt.part, kSplitMax)) !=
        cudaSuccess)
      return err;
    if ((err = gemm_nn<C>(s, kb, n, kb, 1.0, T, kb, bt.Wm, kb, 0.0, bt.Wm2, kb)) != cudaSuccess) return err;
    if ((err = gemm_nn<C>(s, mrows, n, kb, -1.0, V, mrows, bt.Wm2, kb, 1.0, Us, n)) != cudaSuccess) return err;
  }
  return cudaSuccess;
}

// ---- workspace ---------------------------------------------------------------
template <typename C>
struct HermWs {
  C *W, *U, *M, *tau, *vsc, *p, *vec;
  double *d, *e, *lam;
  DcWs dc;
  BtWs<C> bt;
  unsigned *bar;
  int *err;
  unsigned long long *amax;
};

template <typename C>
HermWs<C> carve_herm(void *base, int n, bool want_expm, std::size_t *bytes) {
  Layout L(base);
  const std::size_t nn = (std::size_t)n * n, nv = (std::size_t)(n < 1 ? 1 : n);
  HermWs<C> w{};
  w.W = L.take<C>(nn);
  w.U = L.take<C>(nn);
  w.M = want_expm ? L.take<C>(nn) : nullptr;
  w.tau = L.take<C>(nv);
  w.vsc = L.take<C>(nv);
  w.p = L.take<C>(2 * nv);
  w.vec = L.take<C>(kTrdVecs * nv * kTrdMaxGrid);
  w.d = L.take<double>(nv);
  w.e = L.take<double>(nv);
  w.lam = L.take<double>(nv);
  DcWs &c = w.dc;
  c.Za = L.take<double>(nn);
  c.Zb = L.take<double>(nn);
  c.DEL = L.take<double>(nn);
  c.UF = L.take<double>(nn);
  double **dv[] = {&c.lamA, &c.lamB, &c.dd, &c.ee, &c.srt_d, &c.srt_z, &c.nd_d, &c.nd_z,
                   &c.df_d, &c.rot_c, &c.rot_s, &c.nd_lam, &c.zh};
  for (double **p : dv) *p = L.take<double>(nv);
  int **iv[] = {&c.srt_c, &c.nd_c, &c.df_c, &c.rot_a, &c.rot_b};
  for (int **p : iv) *p = L.take<int>(nv);
  c.cnt = L.take<int>(3 * nv);
  c.sc = L.take<double>(1);
  const std::size_t nb = kWyBlock, nblk = (nv + nb - 1) / nb;
  // V and V^H of all blocks (about n^2 / 2 elements each) reuse Za|Zb and
  // DEL|UF: the back-transform starts by copying Z out of them
  w.bt.Vall = reinterpret_cast<C *>(c.Za);
  w.bt.VHall = reinterpret_cast<C *>(c.DEL);
  w.bt.G = L.take<C>(nblk * nb * nb);
  w.bt.T = L.take<C>(nblk * nb * nb);
  w.bt.Wm = L.take<C>(nv * nb);
  w.bt.Wm2 = L.take<C>(nv * nb);
  w.bt.part = L.take<C>(kSplitMax * nv * nb);
  w.bar = L.take<unsigned>(1);
  w.err = L.take<int>(1);
  w.amax = L.take<unsigned long long>(1);
  if (bytes) *bytes = L.used;
  return w;
}

__global__ void herm_status_kernel(int n, const int *__restrict__ err, int *__restrict__ info) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *info = *err ? n + 1 : 0;
}

constexpr std::size_t kTrdResidentBytes = 220 * 1024;

template <typename C, bool kRes>
cudaError_t launch_hetrd(cudaStream_t s, int G, std::size_t smem, int n, HermWs<C> &w) {
  cudaError_t err;
  int per_sm = 0;
  if ((err = cudaFuncSetAttribute(hetrd_kernel<C, kRes>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
      cudaSuccess)
    return err;
  if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hetrd_kernel<C, kRes>, kTrdThreads, smem)) !=
      cudaSuccess)
    return err;
  if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
  TrdArgs<C> ta{n, w.W, w.d, w.e, w.tau, w.vsc, w.p, w.vec, w.bar, w.err};
  void *args[] = {&ta};
  if ((err = cudaLaunchCooperativeKernel((const void *)hetrd_kernel<C, kRes>, dim3(G), dim3(kTrdThreads), args, smem,
                                         s)) != cudaSuccess)
    return err;
  return launched();
}

// Eigenvalues (FP64, ascending, of the scaled matrix) into w.lam and
// eigenvectors (compute type, ld n) into w.U.
template <typename T, typename C>
cudaError_t heev_run(cudaStream_t s, int upper, int n, const T *A, int lda, HermWs<C> &w) {
  cudaError_t err;
  if ((err = cudaMemsetAsync(w.bar, 0, sizeof(unsigned), s)) != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(w.err, 0, sizeof(int), s)) != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(w.amax, 0, sizeof(unsigned long long), s)) != cudaSuccess) return err;
  const long long total = (long long)n * n;
  const int mb = (int)std::min<long long>((total + 255) / 256, 4 * 148);
  herm_maxabs_kernel<T><<<mb, 256, 0, s>>>(n, A, lda, upper, w.amax);
  if ((err = launched()) != cudaSuccess) return err;
  herm_fill_kernel<T, C><<<dim3((n + 127) / 128, std::min(n, 1024)), 128, 0, s>>>(n, A, lda, upper, w.amax, w.W);
  if ((err = launched()) != cudaSuccess) return err;
  // tridiagonal reduction: one cooperative launch
  const int G = std::max(1, std::min(std::min(sm_count(), kTrdMaxGrid), (n + 7) / 8));
  const std::size_t ncmax = (std::size_t)((n + G - 1) / G);
  const std::size_t base = std::max<std::size_t>(ncmax, kTrdWarps) * sizeof(C);
  const std::size_t resident = base + (ncmax + kTrdVecs) * (std::size_t)n * sizeof(C);
  const bool use_res = resident <= kTrdResidentBytes;
  if ((err = use_res ? launch_hetrd<C, true>(s, G, resident, n, w) : launch_hetrd<C, false>(s, G, base, n, w)) !=
      cudaSuccess)
    return err;
  double *Z = nullptr;
  if ((err = stedc_run(s, n, w.d, w.e, w.dc, w.lam, &Z)) != cudaSuccess) return err;
  return back_transform<C>(s, n, w.W, w.tau, w.vsc, Z, w.U, w.bt);
}

// M(:, j) = U(:, j) exp(lam_j / sigma)
template <typename C>
__global__ void herm_exp_scale_kernel(int n, const C *__restrict__ U, const double *__restrict__ lam,
                                      const unsigned long long *__restrict__ amax, C *__restrict__ M) {
  const double sg = herm_sigma(amax);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = blockIdx.y; j < n; j += gridDim.y)
    M[(std::size_t)j * n + i] = scale(U[(std::size_t)j * n + i], exp(lam[j] / sg));
}

template <typename R>
__global__ void herm_w_out_kernel(int n, const double *__restrict__ lam, const unsigned long long *__restrict__ amax,
                                  R *__restrict__ out) {
  const double sg = herm_sigma(amax);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (R)(lam[i] / sg);
}

template <typename T> struct compute_of { using type = double; };
template <> struct compute_of<float2> { using type = double2; };
template <> struct compute_of<double2> { using type = double2; };

template <typename T>
std::size_t herm_bytes(int n, bool want_expm) {
  using C = typename compute_of<T>::type;
  std::size_t b = 0;
  carve_herm<C>(nullptr, n, want_expm, &b);
  return b;
}

template <typename T>
calamanStatus_t expm_herm_api(calamanHandle_t blas, calamanStream_t stream, int uplo, int n, const T *A, int lda,
                              T *E, int lde, void *work, std::size_t lwork, int *d_info) {
  using C = typename compute_of<T>::type;
  if (n < 1 || n > kMaxDim || lda < n || lde < n || work == nullptr || A == nullptr || E == nullptr ||
      d_info == nullptr || (uplo != CALAMAN_FILL_MODE_LOWER && uplo != CALAMAN_FILL_MODE_UPPER))
    return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  std::size_t need = 0;
  carve_herm<C>(nullptr, n, true, &need);
  if (lwork < need) return blas_status(CALAMAN_STATUS_ALLOC_FAILED);
  HermWs<C> w = carve_herm<C>(work, n, true, nullptr);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  TimerScope timing(timer_of(blas));
  CLM_CUDA((heev_run<T, C>(s, uplo == CALAMAN_FILL_MODE_UPPER, n, A, lda, w)));
  herm_exp_scale_kernel<C><<<dim3((n + 127) / 128, std::min(n, 1024)), 128, 0, s>>>(n, w.U, w.lam, w.amax, w.M);
  CLM_CUDA(launched());
  C *UH = w.W;  // the reflectors are spent
  CLM_CUDA(launch_transpose<C>(s, n, n, 1.0, w.U, n, UH, n, true));
  if constexpr (std::is_same<T, C>::value) {
    CLM_CUDA(gemm_nn<C>(s, n, n, n, 1.0, w.M, n, UH, n, 0.0, E, lde));
  } else {
    C *tmp = w.U;
    CLM_CUDA(gemm_nn<C>(s, n, n, n, 1.0, w.M, n, UH, n, 0.0, tmp, n));
    CLM_CUDA((launch_convert<C, T>(s, n, tmp, n, E, lde)));
  }
  herm_status_kernel<<<1, 32, 0, s>>>(n, w.err, d_info);
  CLM_CUDA(launched());
  return ok_status();
}

// The eigensolver alone: A (uplo triangle) is overwritten by the eigenvectors,
// d_w receives the eigenvalues ascending (cuSOLVER xSYEVD / xHEEVD with
// vectors, the calls the reference's expm_herm makes through WarpWraps).
template <typename T>
calamanStatus_t heevd_api(calamanStream_t stream, int uplo, int n, T *A, int lda, typename elem<T>::real *d_w,
                          void *work, std::size_t lwork, int *d_info) {
  using C = typename compute_of<T>::type;
  using R = typename elem<T>::real;
  if (n < 1 || n > kMaxDim || lda < n || work == nullptr || A == nullptr || d_w == nullptr || d_info == nullptr ||
      (uplo != CALAMAN_FILL_MODE_LOWER && uplo != CALAMAN_FILL_MODE_UPPER))
    return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  std::size_t need = 0;
  carve_herm<C>(nullptr, n, false, &need);
  if (lwork < need) return blas_status(CALAMAN_STATUS_ALLOC_FAILED);
  HermWs<C> w = carve_herm<C>(work, n, false, nullptr);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  CLM_CUDA((heev_run<T, C>(s, uplo == CALAMAN_FILL_MODE_UPPER, n, A, lda, w)));
  herm_w_out_kernel<R><<<(n + 255) / 256, 256, 0, s>>>(n, w.lam, w.amax, d_w);
  CLM_CUDA(launched());
  if constexpr (std::is_same<T, C>::value) {
    CLM_CUDA(launch_scale_copy<C>(s, n, 1.0, w.U, n, A, lda));
  } else {
    CLM_CUDA((launch_convert<C, T>(s, n, w.U, n, A, lda)));
  }
  herm_status_kernel<<<1, 32, 0, s>>>(n, w.err, d_info);
  CLM_CUDA(launched());
  return ok_status();
}

// ---- geodesic trial points: W_j = exp(j step H) W ---------------------------
// The sampling sweep of the cg_unitary line searches
// (src/cg_unitary/geodesic_search.cppm:338-420) evaluates the cost gradient at
// W_j = exp(j mu H) W, j = 1 .. N-1, H in u(n) (skew-Hermitian), and forms the
// rotations as R_1 = expm(mu H), R_j = R_{j-1} R_1 -- N-2 dependent products,
// then N-1 more for R_j W. Here H = -i Hh with Hh = i H Hermitian, so
// exp(t H) = U diag(exp(-i t w)) U^H from ONE Hermitian eigensolve, and all
// trial points come out of one wide product:
//   [W_1 | ... | W_{N-1}] = U [D_1 Y | ... | D_{N-1} Y],  Y = U^H W,
// D_j = diag(exp(-i j mu w)): no error accumulates along j, and the N-1
// products become one GEMM with N-1 times the columns. Real tiers (H skew-
// symmetric, W orthogonal) run through the complex path and keep real parts.

// Wt = i H, Hermitian, from H's lower triangle (its strictly upper part is not
// read); the diagonal keeps i H_jj's real part.
template <typename T>
__global__ void geo_fill_kernel(int n, const T *__restrict__ H, int ldh, double2 *__restrict__ Wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    const double2 h = i >= j ? to_c2(H[(std::size_t)j * ldh + i]) : cj(to_c2(H[(std::size_t)i * ldh + j]));
    // lower entry i H_ij; the mirrored upper entry is conj(i H_ji) = -i conj(H_ji)
    double2 v = i >= j ? make_double2(-h.y, h.x) : make_double2(h.y, -h.x);
    if (i == j) v.y = 0.0;
    Wt[(std::size_t)j * n + i] = v;
  }
}

template <typename T>
__global__ void geo_load_kernel(int n, const T *__restrict__ W, int ldw, double2 *__restrict__ Wc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = blockIdx.y; j < n; j += gridDim.y) Wc[(std::size_t)j * n + i] = to_c2(W[(std::size_t)j * ldw + i]);
}

// B (n x (N-1) n): block j-1 = D_j Y, D_j = diag(exp(-i j mu w_r)), w = lam / sigma
__global__ void geo_phase_kernel(int n, int nsteps, double mu, const double *__restrict__ lam,
                                 const unsigned long long *__restrict__ amax, const double2 *__restrict__ Y,
                                 double2 *__restrict__ B) {
  const double sg = herm_sigma(amax);
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const double wr = lam[r] / sg;
  for (int col = blockIdx.y; col < nsteps * n; col += gridDim.y) {
    const int j = col / n + 1, c = col - (j - 1) * n;
    double sn, cs;
    sincos(-(double)j * mu * wr, &sn, &cs);
    B[(std::size_t)col * n + r] = mul(make_double2(cs, sn), Y[(std::size_t)c * n + r]);
  }
}

template <typename T>
__global__ void geo_real_out_kernel(std::size_t count, const double2 *__restrict__ Z, T *__restrict__ out) {
  for (std::size_t i = blockIdx.x * (std::size_t)blockDim.x + threadIdx.x; i < count;
       i += (std::size_t)gridDim.x * blockDim.x)
    out[i] = (T)Z[i].x;
}
template <typename T>
__global__ void geo_cplx_out_kernel(std::size_t count, const double2 *__restrict__ Z, T *__restrict__ out) {
  for (std::size_t i = blockIdx.x * (std::size_t)blockDim.x + threadIdx.x; i < count;
       i += (std::size_t)gridDim.x * blockDim.x) {
    T v;
    v.x = Z[i].x;
    v.y = Z[i].y;
    out[i] = v;
  }
}

constexpr int kGeoMaxSamples = 64;

struct GeoWs {
  HermWs<double2> h;
  double2 *Hh, *Wc, *Y, *B, *Out;
};

GeoWs carve_geo(void *base, int n, int num_samples, bool direct_out, std::size_t *bytes) {
  Layout L(base);
  GeoWs g;
  const std::size_t nn = (std::size_t)n * n, ns = (std::size_t)(num_samples > 1 ? num_samples - 1 : 1);
  g.Hh = L.take<double2>(nn);
  g.Wc = L.take<double2>(nn);
  g.Y = L.take<double2>(nn);
  g.B = L.take<double2>(ns * nn);
  g.Out = direct_out ? nullptr : L.take<double2>(ns * nn);
  std::size_t hb = 0;
  g.h = carve_herm<double2>(L.cursor(), n, false, &hb);
  if (bytes) *bytes = L.used + hb;
  return g;
}

template <typename T>
calamanStatus_t geodesic_api(calamanHandle_t blas, calamanStream_t stream, int n, const T *W, int ldw, const T *H,
                             int ldh, double mu, int num_samples, T *Wout, void *work, std::size_t lwork,
                             int *d_info) {
  constexpr bool kDirect = std::is_same<T, double2>::value;
  if (n < 1 || n > kMaxDim || ldw < n || ldh < n || W == nullptr || H == nullptr || work == nullptr ||
      d_info == nullptr || num_samples < 1 || num_samples > kGeoMaxSamples || !std::isfinite(mu) ||
      (num_samples > 1 && Wout == nullptr))
    return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  std::size_t need = 0;
  carve_geo(nullptr, n, num_samples, kDirect, &need);
  if (lwork < need) return blas_status(CALAMAN_STATUS_ALLOC_FAILED);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  CLM_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int), s));
  if (num_samples == 1) return ok_status();  // sample 0 is W itself
  GeoWs g = carve_geo(work, n, num_samples, kDirect, nullptr);
  TimerScope timing(timer_of(blas));
  const dim3 grid2((n + 127) / 128, std::min(n, 1024));
  geo_fill_kernel<T><<<grid2, 128, 0, s>>>(n, H, ldh, g.Hh);
  CLM_CUDA(launched());
  geo_load_kernel<T><<<grid2, 128, 0, s>>>(n, W, ldw, g.Wc);
  CLM_CUDA(launched());
  CLM_CUDA((heev_run<double2, double2>(s, 0, n, g.Hh, n, g.h)));  // Hh = U diag(lam / sigma) U^H
  double2 *UH = g.h.W;                                              // the reflectors are spent
  CLM_CUDA(launch_transpose<double2>(s, n, n, 1.0, g.h.U, n, UH, n, true));
  CLM_CUDA(gemm_nn<double2>(s, n, n, n, 1.0, UH, n, g.Wc, n, 0.0, g.Y, n));
  const int steps = num_samples - 1;
  geo_phase_kernel<<<dim3((n + 127) / 128, std::min(steps * n, 4096)), 128, 0, s>>>(n, steps, mu, g.h.lam, g.h.amax,
                                                                                   g.Y, g.B);
  CLM_CUDA(launched());
  double2 *out = kDirect ? reinterpret_cast<double2 *>(Wout) : g.Out;
  CLM_CUDA(gemm_nn<double2>(s, n, steps * n, n, 1.0, g.h.U, n, g.B, n, 0.0, out, n));
  if constexpr (!kDirect) {
    const std::size_t count = (std::size_t)steps * n * n;
    const int blocks = (int)std::min<std::size_t>((count + 255) / 256, 8 * 148);
    if constexpr (elem<T>::complex) geo_cplx_out_kernel<T><<<blocks, 256, 0, s>>>(count, out, Wout);
    else geo_real_out_kernel<T><<<blocks, 256, 0, s>>>(count, out, Wout);
    CLM_CUDA(launched());
  }
  herm_status_kernel<<<1, 32, 0, s>>>(n, g.h.err, d_info);
  CLM_CUDA(launched());
  return ok_status();
}

template <typename T>
std::size_t geodesic_bytes(int n, int num_samples) {
  std::size_t b = 0;
  carve_geo(nullptr, n, num_samples, std::is_same<T, double2>::value, &b);
  return b;
}

}  // namespace
}  // namespace clm

using namespace clm;

extern "C" {

calamanStatus_t calaman_grid_barrier_wait_check(calamanStream_t stream, unsigned limit, void *work,
                                                size_t work_bytes, int *code) {
  if (work == nullptr || code == nullptr || limit < 1) return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  if (work_bytes < 256) return blas_status(CALAMAN_STATUS_ALLOC_FAILED);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned *count = static_cast<unsigned *>(work);
  int *err = reinterpret_cast<int *>(static_cast<char *>(work) + 128);
  CLM_CUDA(cudaMemsetAsync(work, 0, 256, st));
  grid_sync_check_kernel<<<2, 64, 0, st>>>(count, err, limit);
  CLM_CUDA(launched());
  int h = 0;
  CLM_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CLM_CUDA(cudaStreamSynchronize(st));
  *code = h;
  return ok_status();
}

#define CLM_HERM_API(SUF, T, R, PT, CPT)                                                                    \
  calamanStatus_t calaman_expm_herm_bufferSize_##SUF(calamanSolverHandle_t, int uplo, int n, size_t *bytes) { \
    if (n < 1 || n > kMaxDim || bytes == nullptr ||                                                         \
        (uplo != CALAMAN_FILL_MODE_LOWER && uplo != CALAMAN_FILL_MODE_UPPER))                               \
      return blas_status(CALAMAN_STATUS_INVALID_VALUE);                                                     \
    *bytes = herm_bytes<T>(n, true);                                                                        \
    return ok_status();                                                                                     \
  }                                                                                                         \
  calamanStatus_t calaman_expm_herm_##SUF(calamanBlasHandle_t blas, calamanSolverHandle_t,                  \
                                          calamanStream_t stream, int uplo, int n, CPT A, int lda, PT E,     \
                                          int lde, void *work, size_t lwork, int *d_info) {                 \
    return expm_herm_api<T>(blas, stream, uplo, n, reinterpret_cast<const T *>(A), lda,                     \
                            reinterpret_cast<T *>(E), lde, work, lwork, d_info);                            \
  }                                                                                                         \
  calamanStatus_t calaman_heevd_bufferSize_##SUF(int uplo, int n, size_t *bytes) {                          \
    if (n < 1 || n > kMaxDim || bytes == nullptr ||                                                         \
        (uplo != CALAMAN_FILL_MODE_LOWER && uplo != CALAMAN_FILL_MODE_UPPER))                               \
      return blas_status(CALAMAN_STATUS_INVALID_VALUE);                                                     \
    *bytes = herm_bytes<T>(n, false);                                                                       \
    return ok_status();                                                                                     \
  }                                                                                                         \
  calamanStatus_t calaman_heevd_##SUF(calamanStream_t stream, int uplo, int n, PT A, int lda, R *d_w,        \
                                      void *work, size_t lwork, int *d_info) {                              \
    return heevd_api<T>(stream, uplo, n, reinterpret_cast<T *>(A), lda, d_w, work, lwork, d_info);          \
  }
#define CLM_GEO_API(SUF, T, PT, CPT)                                                                         \
  calamanStatus_t calaman_geodesic_points_bufferSize_##SUF(calamanSolverHandle_t, int n, int num_samples,      \
                                                           size_t *bytes) {                                    \
    if (n < 1 || n > kMaxDim || num_samples < 1 || num_samples > kGeoMaxSamples || bytes == nullptr)            \
      return blas_status(CALAMAN_STATUS_INVALID_VALUE);                                                        \
    *bytes = geodesic_bytes<T>(n, num_samples);                                                                \
    return ok_status();                                                                                        \
  }                                                                                                            \
  calamanStatus_t calaman_geodesic_points_##SUF(calamanBlasHandle_t blas, calamanSolverHandle_t,               \
                                                calamanStream_t stream, int n, CPT W, int ldw, CPT H, int ldh,  \
                                                double step, int num_samples, PT Wout, void *work,             \
                                                size_t lwork, int *d_info) {                                   \
    return geodesic_api<T>(blas, stream, n, reinterpret_cast<const T *>(W), ldw, reinterpret_cast<const T *>(H), \
                           ldh, step, num_samples, reinterpret_cast<T *>(Wout), work, lwork, d_info);          \
  }
CLM_GEO_API(s, float, float *, const float *)
CLM_GEO_API(d, double, double *, const double *)
CLM_GEO_API(c, float2, void *, const void *)
CLM_GEO_API(z, double2, void *, const void *)
#undef CLM_GEO_API

CLM_HERM_API(s, float, float, float *, const float *)
CLM_HERM_API(d, double, double, double *, const double *)
CLM_HERM_API(c, float2, float, void *, const void *)
CLM_HERM_API(z, double2, double, void *, const void *)
#undef CLM_HERM_API

}  // extern "C"
