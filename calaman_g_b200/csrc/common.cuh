// common.cuh -- element types, complex arithmetic, status plumbing and launch
// helpers shared by every translation unit of the B200 matrix-exponential
// library.
//
// Four element types, as in calaman_G (src/expm/README.md:16-18): float,
// double, float2 (complex64) and double2 (complex128), interleaved (re, im),
// column-major matrices.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cmath>
#include <vector>

#include "../../include/calaman_b200.h"

namespace clm {

// ---------------------------------------------------------------------------
// Element traits
// ---------------------------------------------------------------------------
template <typename T> struct elem;

template <> struct elem<float> {
  using real = float;
  static constexpr bool complex = false;
  static constexpr bool single = true;
  __host__ __device__ static float zero() { return 0.f; }
  __host__ __device__ static float one() { return 1.f; }
  __host__ __device__ static float from_real(double x) { return (float)x; }
};
template <> struct elem<double> {
  using real = double;
  static constexpr bool complex = false;
  static constexpr bool single = false;
  __host__ __device__ static double zero() { return 0.0; }
  __host__ __device__ static double one() { return 1.0; }
  __host__ __device__ static double from_real(double x) { return x; }
};
template <> struct elem<float2> {
  using real = float;
  static constexpr bool complex = true;
  static constexpr bool single = true;
  __host__ __device__ static float2 zero() { return make_float2(0.f, 0.f); }
  __host__ __device__ static float2 one() { return make_float2(1.f, 0.f); }
  __host__ __device__ static float2 from_real(double x) { return make_float2((float)x, 0.f); }
};
template <> struct elem<double2> {
  using real = double;
  static constexpr bool complex = true;
  static constexpr bool single = false;
  __host__ __device__ static double2 zero() { return make_double2(0.0, 0.0); }
  __host__ __device__ static double2 one() { return make_double2(1.0, 0.0); }
  __host__ __device__ static double2 from_real(double x) { return make_double2(x, 0.0); }
};

// ---------------------------------------------------------------------------
// Arithmetic on the four types (real scalars are the common case; complex is
// spelled out so nothing depends on cuComplex's helpers).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ float add(float a, float b) { return a + b; }
__host__ __device__ __forceinline__ double add(double a, double b) { return a + b; }
__host__ __device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

__host__ __device__ __forceinline__ float sub(float a, float b) { return a - b; }
__host__ __device__ __forceinline__ double sub(double a, double b) { return a - b; }
__host__ __device__ __forceinline__ float2 sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

__host__ __device__ __forceinline__ float mul(float a, float b) { return a * b; }
__host__ __device__ __forceinline__ double mul(double a, double b) { return a * b; }
__host__ __device__ __forceinline__ float2 mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// a*b + c
__device__ __forceinline__ float fmac(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmac(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float2 fmac(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(-a.y, b.y, fmaf(a.x, b.x, c.x)), fmaf(a.y, b.x, fmaf(a.x, b.y, c.y)));
}
__device__ __forceinline__ double2 fmac(double2 a, double2 b, double2 c) {
  return make_double2(fma(-a.y, b.y, fma(a.x, b.x, c.x)), fma(a.y, b.x, fma(a.x, b.y, c.y)));
}

// real scalar r times element x, plus c
__device__ __forceinline__ float rfma(float r, float x, float c) { return fmaf(r, x, c); }
__device__ __forceinline__ double rfma(double r, double x, double c) { return fma(r, x, c); }
__device__ __forceinline__ float2 rfma(float r, float2 x, float2 c) { return make_float2(fmaf(r, x.x, c.x), fmaf(r, x.y, c.y)); }
__device__ __forceinline__ double2 rfma(double r, double2 x, double2 c) { return make_double2(fma(r, x.x, c.x), fma(r, x.y, c.y)); }

__host__ __device__ __forceinline__ float scale(float x, float r) { return x * r; }
__host__ __device__ __forceinline__ double scale(double x, double r) { return x * r; }
__host__ __device__ __forceinline__ float2 scale(float2 x, float r) { return make_float2(x.x * r, x.y * r); }
__host__ __device__ __forceinline__ double2 scale(double2 x, double r) { return make_double2(x.x * r, x.y * r); }

__host__ __device__ __forceinline__ float add_real(float x, float r) { return x + r; }
__host__ __device__ __forceinline__ double add_real(double x, double r) { return x + r; }
__host__ __device__ __forceinline__ float2 add_real(float2 x, float r) { return make_float2(x.x + r, x.y); }
__host__ __device__ __forceinline__ double2 add_real(double2 x, double r) { return make_double2(x.x + r, x.y); }

__host__ __device__ __forceinline__ float neg(float a) { return -a; }
__host__ __device__ __forceinline__ double neg(double a) { return -a; }
__host__ __device__ __forceinline__ float2 neg(float2 a) { return make_float2(-a.x, -a.y); }
__host__ __device__ __forceinline__ double2 neg(double2 a) { return make_double2(-a.x, -a.y); }

// Division a / b; complex division by Smith's scaled algorithm (Smith 1962).
__device__ __forceinline__ float divide(float a, float b) { return a / b; }
__device__ __forceinline__ double divide(double a, double b) { return a / b; }
template <typename C, typename R>
__device__ __forceinline__ C cdiv_smith(C a, C b) {
  C q;
  if (fabs((double)b.x) >= fabs((double)b.y)) {
    const R r = b.y / b.x;
    const R d = b.x + b.y * r;
    q.x = (a.x + a.y * r) / d;
    q.y = (a.y - a.x * r) / d;
  } else {
    const R r = b.x / b.y;
    const R d = b.y + b.x * r;
    q.x = (a.x * r + a.y) / d;
    q.y = (a.y * r - a.x) / d;
  }
  return q;
}
__device__ __forceinline__ float2 divide(float2 a, float2 b) { return cdiv_smith<float2, float>(a, b); }
__device__ __forceinline__ double2 divide(double2 a, double2 b) { return cdiv_smith<double2, double>(a, b); }

// |x|: true modulus (the induced 1-norm, src/expm/expm.cu:188-191)
__device__ __forceinline__ double modulus(float x) { return fabs((double)x); }
__device__ __forceinline__ double modulus(double x) { return fabs(x); }
__device__ __forceinline__ double modulus(float2 x) { return hypot((double)x.x, (double)x.y); }
__device__ __forceinline__ double modulus(double2 x) { return hypot(x.x, x.y); }

// |Re|+|Im|: how partial pivoting ranks candidates (LAPACK IxAMAX).
__device__ __forceinline__ double abs1(float x) { return fabs((double)x); }
__device__ __forceinline__ double abs1(double x) { return fabs(x); }
__device__ __forceinline__ double abs1(float2 x) { return fabs((double)x.x) + fabs((double)x.y); }
__device__ __forceinline__ double abs1(double2 x) { return fabs(x.x) + fabs(x.y); }

__host__ __device__ __forceinline__ bool is_zero(float x) { return x == 0.f; }
__host__ __device__ __forceinline__ bool is_zero(double x) { return x == 0.0; }
__host__ __device__ __forceinline__ bool is_zero(float2 x) { return x.x == 0.f && x.y == 0.f; }
__host__ __device__ __forceinline__ bool is_zero(double2 x) { return x.x == 0.0 && x.y == 0.0; }

// ---------------------------------------------------------------------------
// Status helpers
// ---------------------------------------------------------------------------
inline calamanStatus_t ok_status() { return calamanStatus_t{CALAMAN_DOMAIN_BLAS, CALAMAN_STATUS_SUCCESS}; }
inline calamanStatus_t blas_status(int code) { return calamanStatus_t{CALAMAN_DOMAIN_BLAS, code}; }
inline calamanStatus_t runtime_status(cudaError_t e) { return calamanStatus_t{CALAMAN_DOMAIN_RUNTIME, (int)e}; }
inline bool is_ok(calamanStatus_t s) { return s.code == 0; }

#define CLM_TRY(expr)                                   \
  do {                                                  \
    const calamanStatus_t clm_st_ = (expr);             \
    if (clm_st_.code != 0) return clm_st_;              \
  } while (0)

// A launch or runtime call: surface its error in the runtime domain.
#define CLM_CUDA(expr)                                  \
  do {                                                  \
    const cudaError_t clm_e_ = (expr);                  \
    if (clm_e_ != cudaSuccess) return ::clm::runtime_status(clm_e_); \
  } while (0)

#define CLM_LAUNCHED() CLM_CUDA(cudaGetLastError())

inline std::size_t align_up(std::size_t x, std::size_t a) { return (x + a - 1) / a * a; }

// Workspace carving: positional, 256-byte-aligned regions (the same contract
// as calaman_G's WorkspaceLayout, src/common/workspace.cppm:69-159). A null
// base sizes without carving.
struct Layout {
  char *base;
  std::size_t used = 0;
  explicit Layout(void *b) : base(static_cast<char *>(b)) {}
  template <typename U> U *take(std::size_t count) {
    U *p = base ? reinterpret_cast<U *>(base + used) : nullptr;
    used += align_up(count * sizeof(U), 256);
    return p;
  }
  void *cursor() const { return base ? base + used : nullptr; }
};

// Number of SMs on the current device (cached per device).
int sm_count();

// Every launcher bumps this process-wide counter (calamanGetLaunchCount).
void note_launch(unsigned n = 1);
unsigned long long g_launch_count();
// After a <<<>>> launch: count it and return the launch error.
inline cudaError_t launched() {
  note_launch(1);
  return cudaGetLastError();
}

// CUDA-event timing of GEMM launches, active while a handle with timing
// enabled is inside one of its calls (set per thread by TimerScope).
struct KernelTimer {
  bool enabled = false;
  std::vector<cudaEvent_t> pool;  // reused event objects
  std::size_t used = 0;           // events handed out since the last read
  std::vector<cudaEvent_t> starts, stops;  // one pair per recorded launch
  std::vector<double> flops;               // algorithmic flops of that launch
  cudaEvent_t take();
};
extern thread_local KernelTimer *tl_timer;

struct TimerScope {
  KernelTimer *saved;
  explicit TimerScope(KernelTimer *t) : saved(tl_timer) { tl_timer = (t && t->enabled) ? t : nullptr; }
  ~TimerScope() { tl_timer = saved; }
};

// Device scratch for the split-BF16 tensor-core FP32 GEMM, lent by a driver
// for the duration of one call (the FP32 products inside the LU and the solves
// included). Without it, FP32 products take the SIMT kernel.
struct GemmScratch {
  void *ptr = nullptr;
  std::size_t bytes = 0;
  int terms = 6;  // 3 or 6 bf16 part products
  // FP64 / complex128 products emulated on the INT8 tensor cores (oz_gemm):
  // digit planes, digits per operand, and the smallest M, N and K that take
  // that path (smaller products stay on the FP64 tensor cores)
  void *oz = nullptr;
  std::size_t oz_bytes = 0;
  int oz_digits = 0;
  int oz_min_dim = 0;
};
extern thread_local GemmScratch *tl_gemm_scratch;
struct GemmScratchScope {
  GemmScratch *saved;
  explicit GemmScratchScope(GemmScratch *g) : saved(tl_gemm_scratch) { tl_gemm_scratch = g; }
  ~GemmScratchScope() { tl_gemm_scratch = saved; }
};

}  // namespace clm

namespace clm {

// ---- pivot search: CTA-wide argmax of |x| with the first index on ties ------
// A candidate magnitude v >= 0 is keyed by its IEEE-754 bits, which order
// non-negative doubles exactly as their values; rows that are not candidates
// (and NaN magnitudes, which partial pivoting never selects) carry key 0 and
// index INT_MAX. The warp stage is three redux.sync reductions (high word, low
// word among the high word's winners, smallest index among the key's winners).
struct ArgMax {
  unsigned long long key;
  int idx;
};

__device__ __forceinline__ ArgMax argmax_key(double v, int idx, bool candidate) {
  if (!candidate || !(v >= 0.0)) return ArgMax{0ull, 0x7fffffff};
  return ArgMax{(unsigned long long)__double_as_longlong(v), idx};
}

__device__ __forceinline__ ArgMax warp_argmax(ArgMax a) {
  const unsigned full = 0xffffffffu;
  const unsigned hi = (unsigned)(a.key >> 32), lo = (unsigned)a.key;
  const unsigned mhi = __reduce_max_sync(full, hi);
  const unsigned mlo = __reduce_max_sync(full, hi == mhi ? lo : 0u);
  const bool win = hi == mhi && lo == mlo;
  const unsigned midx = __reduce_min_sync(full, win ? (unsigned)a.idx : 0x7fffffffu);
  return ArgMax{((unsigned long long)mhi << 32) | mlo, (int)midx};
}

// The two stages of cta_argmax, for callers that overlap work with the
// cross-warp exchange (the warp winner may start on its row meanwhile).
__device__ __forceinline__ void cta_argmax_publish(const ArgMax &w, unsigned long long *red_key, int *red_idx) {
  if ((threadIdx.x & 31) == 0) {
    red_key[threadIdx.x >> 5] = w.key;
    red_idx[threadIdx.x >> 5] = w.idx;
  }
}
__device__ __forceinline__ ArgMax cta_argmax_collect(const unsigned long long *red_key, const int *red_idx) {
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const ArgMax b = lane < nwarps ? ArgMax{red_key[lane], red_idx[lane]} : ArgMax{0ull, 0x7fffffff};
  return warp_argmax(b);
}
// As cta_argmax_collect, and wwarp = the warp whose entry won (meaningful
// when the winner's index is a real row: rows are unique across warps).
__device__ __forceinline__ ArgMax cta_argmax_collect_at(const unsigned long long *red_key, const int *red_idx,
                                                        int &wwarp) {
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const ArgMax b = lane < nwarps ? ArgMax{red_key[lane], red_idx[lane]} : ArgMax{0ull, 0x7fffffff};
  const ArgMax m = warp_argmax(b);
  wwarp = __ffs(__ballot_sync(0xffffffffu, lane < nwarps && b.idx == m.idx)) - 1;
  return m;
}

// CTA-wide: every thread passes its own candidate and receives the winner.
// red_key / red_idx: shared arrays of blockDim.x / 32 entries. Contains one
// __syncthreads; the caller separates consecutive calls by another barrier.
__device__ __forceinline__ ArgMax cta_argmax(ArgMax a, unsigned long long *red_key, int *red_idx) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  a = warp_argmax(a);
  if (lane == 0) {
    red_key[warp] = a.key;
    red_idx[warp] = a.idx;
  }
  __syncthreads();
  ArgMax b = lane < nwarps ? ArgMax{red_key[lane], red_idx[lane]} : ArgMax{0ull, 0x7fffffff};
  return warp_argmax(b);
}

// Per-size schedule of the batched tier (size buckets b = ceil(n / 16), n <= 256):
// the CTA size of the per-matrix LU (>= n) and the smallest n whose FP32
// products run on the tensor cores (smaller ones on the SIMT kernel). The
// defaults are the table calamanTuneBatched measured on a B200;
// calamanTuneBatched re-measures it on the caller's device.
struct BatchedTuning {
  int lu_threads[17];
  int fp32_tc_min_n;
};
inline BatchedTuning default_batched_tuning() {
  BatchedTuning t{};
  for (int b = 0; b <= 16; ++b) t.lu_threads[b] = 16 * b <= 64 ? 64 : 16 * b <= 128 ? 128 : 256;
  // measured on a B200 (calamanTuneBatched, 512 float32 matrices per size):
  // the SIMT kernel is faster for the products of n <= 64, the tensor cores above
  t.fp32_tc_min_n = 65;
  return t;
}

// A batched call's launches captured as a CUDA graph, replayed while the
// call's configuration (sizes, plans, pointers, schedule) is unchanged.
struct BatchedGraph {
  unsigned long long key = 0;   // configuration of the cached graph
  unsigned long long seen = 0;  // configuration of the last call (captured when it repeats)
  void *exec = nullptr;         // cudaGraphExec_t
  unsigned launches = 0;        // kernels in the graph (counted again at every replay)
};

}  // namespace clm

// The opaque handle behind calamanHandle_t.
struct calamanContext {
  cudaStream_t stream = nullptr;
  int pointer_mode = CALAMAN_POINTER_MODE_HOST;
  int device = 0;
  int sm_count = 0;
  double *h_pinned = nullptr;  // pinned host slots for the 1-norm readback
  int split_terms = 6;         // bf16 part products per FP32 product (3 or 6)
  int fp64_digits = -1;        // FP64 products: -1 by size, 0 FP64 tensor cores, else Ozaki digits
  void *work = nullptr;        // caller-attached device workspace (calamanSetWorkspace)
  std::size_t work_bytes = 0;
  clm::BatchedTuning tune = clm::default_batched_tuning();
  int graphs = 1;              // batched calls replay a captured CUDA graph of their launches
  clm::BatchedGraph graph[2];  // per batched tier: [0] float, [1] double
  int expm_graphs = 1;         // calaman_expm_* replays its launches after the norm readback
  clm::BatchedGraph single[4]; // per expm type: [0] float, [1] double, [2] complex64, [3] complex128
  clm::BatchedGraph vjp[4];    // per expm_vjp type, the same order
  // second stream of the batched mixed tiers (the FP64 matrices run on it
  // beside the FP32 ones) and the fork / join events, created on first use
  cudaStream_t side = nullptr;
  cudaEvent_t side_fork = nullptr, side_join = nullptr;
  clm::KernelTimer timer;
};
