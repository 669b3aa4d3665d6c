// tc_gemm.cu -- FP32 GEMM as split-BF16 products on the 5th-generation tensor
// cores (tcgen05, TMEM accumulators, TMA-fed shared memory), for the single-
// precision tiers of the matrix-exponential path.
//
// C = alpha * A B + beta * C with A (M x K), B (K x N), C column-major FP32.
// Each operand element x is split into bf16 parts
//     h = bf16(x), m = bf16(x - h), l = bf16(x - h - m)
// and the product is the sum of the part products the precision level keeps,
// smallest first, all accumulated into one FP32 accumulator in TMEM:
//     x3: (m,h) (h,m) (h,h)                          ~16-bit operands
//     x6: (l,h) (h,l) (m,m) (m,h) (h,m) (h,h)         ~24-bit operands
// Complex64 products are one real product of twice the rows and twice the
// depth, [Cr; Ci] = [[Ar, -Ai]; [Ai, Ar]] [Br; Bi]: the split kernels read the
// interleaved operands in that block form and the epilogue writes rows < M to
// the real and rows >= M to the imaginary halves of C.
// The parts are written once per operand by split kernels into a K-major
// layout (rows of Kpad bf16, zero padded to the tile grid), so the GEMM's
// producer warp reads every operand tile with one TMA copy, 128-byte swizzled.
//
// Kernel structure (one CTA per 128 x 256 output tile, 10 warps):
//   warp 0      TMA producer: a 4-stage (or, for products of few k-blocks,
//               2-stage, two CTAs per SM) ring of (A 128x64, B 256x64) tiles
//   warp 1      TMEM allocator and MMA issuer (one elected thread issues
//               tcgen05.mma 128x256x16, commits each stage back to the ring)
//   warps 2..9  epilogue, two warps per TMEM lane quarter: tcgen05.ld 32 lanes
//               x 32 columns at a time, alpha/beta, coalesced column-major
//               stores
// Every mbarrier wait is bounded; a wait that runs out records an error code
// and the CTA unwinds (draining its own TMA copies, freeing its TMEM).
#include <cuda.h>
#include <cuda_bf16.h>

#include <type_traits>

#include "kernels.cuh"
#include "tcgen05.cuh"

namespace clm {

namespace {

using namespace tc;

constexpr int TM = 128;       // UMMA M (TMEM lanes)
constexpr int TN = 256;       // UMMA N (TMEM columns)
constexpr int TK = 64;        // k-block: one 128-byte swizzle atom of bf16
constexpr int UK = 16;        // UMMA K for 16-bit inputs
constexpr int kThreads = 320;   // producer, MMA issuer, 8 epilogue warps
constexpr int kA = TM * TK * 2;  // bytes of one A stage
constexpr int kB = TN * TK * 2;  // bytes of one B stage

struct TcParams {
  int M, N, nkb;        // nkb: k-blocks per part product (Kpad / TK); M: rows of the real product
  int Mc;               // complex: rows of the caller's C (rows >= Mc are imaginary parts), else 0
  int Mpad, Npad;       // rows of one A part / one B part in the part buffers
  int nterms;
  int pa[9], pb[9];     // part index of A and of B for every term
  float alpha, beta;
  float *C;
  int ldc;
  int *err;
};

// Instruction descriptor: bf16 x bf16 -> f32, both K-major, M = TM, N = TN.
constexpr uint32_t kIdesc = idesc_bf16_f32(TM, TN);

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t acc) {
  mma_f16(tmem_d, a, b, kIdesc, acc);
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) { mma_commit(bar); }
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) { return smem_desc_sw128(addr); }

// Element (m, n) of the real product in the caller's C, as a float index.
__device__ __forceinline__ std::size_t c_index(const TcParams &p, int m, int n) {
  if (p.Mc == 0) return (std::size_t)n * p.ldc + m;
  const bool im = m >= p.Mc;
  return 2 * ((std::size_t)n * p.ldc + (im ? m - p.Mc : m)) + (im ? 1 : 0);
}

// STAGES: depth of the TMA ring; MINB: CTAs per SM the kernel is built for
// (the two-stage variant fits two CTAs on an SM, for products with few
// k-blocks, where the epilogue's traffic dominates).
template <int STAGES, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    tc_split_gemm_kernel(const __grid_constant__ CUtensorMap map_a,
                         const __grid_constant__ CUtensorMap map_b, const TcParams prm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte alignment for the 128-byte swizzle atoms
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char *sA = base;
  unsigned char *sB = base + STAGES * kA;
  uint64_t *full = reinterpret_cast<uint64_t *>(sB + STAGES * kB);
  uint64_t *empty = full + STAGES;
  uint64_t *acc_full = empty + STAGES;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_full + 1);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  const int total = prm.nterms * prm.nkb;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {  // TMEM: 256 columns x 128 lanes of f32
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     saddr(tmem_slot)),
                 "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    asm volatile("tcgen05.fence::before_thread_sync;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer ----
    int issued = 0;
    for (int it = 0; it < total; ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)((it / STAGES) & 1);
      if (!mbar_wait(&empty[s], ph ^ 1u) || *(volatile int *)abort_flag) {
        record_error(prm.err, 1);
        *(volatile int *)abort_flag = 1;
        break;
      }
      const int t = it / prm.nkb, kb = it - t * prm.nkb;
      mbar_expect_tx(&full[s], kA + kB);
      tma_load_2d(sA + s * kA, &map_a, &full[s], kb * TK, prm.pa[t] * prm.Mpad + m0);
      tma_load_2d(sB + s * kB, &map_b, &full[s], kb * TK, prm.pb[t] * prm.Npad + n0);
      issued = it + 1;
    }
    // drain: the copies this thread issued must land before the CTA exits
    for (int it = issued - STAGES > 0 ? issued - STAGES : 0; it < issued; ++it)
      mbar_wait(&full[it % STAGES], (uint32_t)((it / STAGES) & 1));
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    bool ok = true;
    for (int it = 0; it < total; ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)((it / STAGES) & 1);
      if (!mbar_wait(&full[s], ph) || *(volatile int *)abort_flag) {
        record_error(prm.err, 2);
        *(volatile int *)abort_flag = 1;
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = saddr(sA + s * kA), b0 = saddr(sB + s * kB);
#pragma unroll
      for (int k = 0; k < TK / UK; ++k)  // +32 bytes per 16-element k step inside the atom
        umma(tmem, smem_desc(a0 + k * 32), smem_desc(b0 + k * 32), (it > 0 || k > 0) ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    if (!ok) *(volatile int *)abort_flag = 1;
    // The commit tracks every MMA issued above, so it is made on the abort
    // path too; this thread then waits for it, so no MMA still reads shared
    // memory or writes TMEM when the CTA frees its TMEM and exits.
    umma_commit(acc_full);
    if (!mbar_wait(acc_full, 0)) record_error(prm.err, 4);
  } else if (warp >= 2) {
    // ---- epilogue: two warps per TMEM lane quarter, 128 columns each ----
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int half = (warp - 2) >> 2;
    // bounded wait for the accumulator; gives up early once the CTA aborted
    bool ok = false;
    for (long long i = 0; i < kSpinLimit; ++i) {
      if (mbar_try_wait(acc_full, 0)) {
        ok = true;
        break;
      }
      if ((i & 1023) == 1023 && *(volatile int *)abort_flag) break;
    }
    if (!ok && !*(volatile int *)abort_flag) record_error(prm.err, 3);
    if (ok && !*(volatile int *)abort_flag) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int m = m0 + q * 32 + lane;
      for (int c0 = half * (TN / 2); c0 < (half + 1) * (TN / 2); c0 += 32) {
        if (n0 + c0 >= prm.N) break;
        uint32_t v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
        if (m < prm.M) {
          // the 32 old C values of this chunk are loaded before any store
          float old[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int n = n0 + c0 + j;
            old[j] = (prm.beta != 0.f && n < prm.N) ? prm.C[c_index(prm, m, n)] : 0.f;
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int n = n0 + c0 + j;
            if (n < prm.N) {
              const float x = prm.alpha * __uint_as_float(v[j]);
              prm.C[c_index(prm, m, n)] = (prm.beta == 0.f) ? x : fmaf(prm.beta, old[j], x);
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
  }
}

// ---- operand split kernels --------------------------------------------------
__device__ __forceinline__ void split3(float x, __nv_bfloat16 &h, __nv_bfloat16 &m, __nv_bfloat16 &l) {
  h = __float2bfloat16_rn(x);
  const float r = x - __bfloat162float(h);
  m = __float2bfloat16_rn(r);
  l = __float2bfloat16_rn(r - __bfloat162float(m));
}

// Element (m, k) of the real A operand: A itself, or for complex (Mc > 0,
// Kc = the complex depth) the block [[Ar, -Ai]; [Ai, Ar]].
template <typename T>
__device__ __forceinline__ float a_at(const T *A, int lda, int Mc, int Kc, int m, int k) {
  if constexpr (std::is_same<T, float2>::value) {
    const bool lo = m < Mc, left = k < Kc;
    const float2 z = A[(std::size_t)(left ? k : k - Kc) * lda + (lo ? m : m - Mc)];
    return lo ? (left ? z.x : -z.y) : (left ? z.y : z.x);
  } else {
    return A[(std::size_t)k * lda + m];
  }
}

// A (M x K real rows; column-major, lda) -> parts[p][row][k], rows of Kpad,
// Mpad rows per part; the transpose goes through a 32 x 33 shared tile.
template <typename T>
__global__ void split_a_kernel(int M, int K, const T *__restrict__ A, int lda, int Mc, int Kc, int Mpad,
                               int Kpad, int nparts, __nv_bfloat16 *__restrict__ parts) {
  __shared__ float tile[32][33];
  const int mb = blockIdx.x * 32, kb = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int r = ty; r < 32; r += 8) {  // read: consecutive m along tx
    const int m = mb + tx, k = kb + r;
    tile[r][tx] = (m < M && k < K) ? a_at<T>(A, lda, Mc, Kc, m, k) : 0.f;
  }
  __syncthreads();
  const std::size_t part_stride = (std::size_t)Mpad * Kpad;
  for (int r = ty; r < 32; r += 8) {  // write: consecutive k along tx
    const int m = mb + r, k = kb + tx;
    if (m < Mpad && k < Kpad) {
      __nv_bfloat16 h, mm, l;
      split3(tile[tx][r], h, mm, l);
      const std::size_t at = (std::size_t)m * Kpad + k;
      parts[at] = h;
      parts[part_stride + at] = mm;
      if (nparts > 2) parts[2 * part_stride + at] = l;
    }
  }
}

// B (K x N real; column-major, ldb; for complex [Br; Bi] with Kc the complex
// depth) -> parts[p][col][k]: already K-contiguous.
template <typename T>
__global__ void split_b_kernel(int K, int N, const T *__restrict__ B, int ldb, int Kc, int Npad,
                               int Kpad, int nparts, __nv_bfloat16 *__restrict__ parts) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Kpad) return;
  const std::size_t part_stride = (std::size_t)Npad * Kpad;
  for (int n = blockIdx.y; n < Npad; n += gridDim.y) {
    float x = 0.f;
    if (k < K && n < N) {
      if constexpr (std::is_same<T, float2>::value) {
        const float2 z = B[(std::size_t)n * ldb + (k < Kc ? k : k - Kc)];
        x = k < Kc ? z.x : z.y;
      } else {
        x = B[(std::size_t)n * ldb + k];
      }
    }
    __nv_bfloat16 h, m, l;
    split3(x, h, m, l);
    const std::size_t at = (std::size_t)n * Kpad + k;
    parts[at] = h;
    parts[part_stride + at] = m;
    if (nparts > 2) parts[2 * part_stride + at] = l;
  }
}

// ---- host side ----------------------------------------------------------------
// A row-major bf16 matrix of `rows` x `cols` (cols contiguous), boxes of box_rows x 64.
bool make_map(CUtensorMap *map, void *ptr, long long rows, long long cols, int box_rows) {
  return make_rowmajor_map_sw128(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, rows, cols * 2, box_rows);
}

struct SplitLayout {
  int Mpad, Npad, Kpad;
  std::size_t a_bytes, b_bytes, total;
};
SplitLayout split_layout(int M, int N, int K, int nparts) {
  SplitLayout L;
  L.Mpad = (M + TM - 1) / TM * TM;
  L.Npad = (N + TN - 1) / TN * TN;
  L.Kpad = (K + TK - 1) / TK * TK;
  L.a_bytes = align_up((std::size_t)nparts * L.Mpad * L.Kpad * 2, 256);
  L.b_bytes = align_up((std::size_t)nparts * L.Npad * L.Kpad * 2, 256);
  L.total = 256 + L.a_bytes + L.b_bytes;  // [error word | A parts | B parts]
  return L;
}

}  // namespace

EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  if (fn == nullptr) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

bool make_rowmajor_map_sw128(CUtensorMap *map, CUtensorMapDataType type, int elem_bytes, void *ptr,
                             long long rows, long long row_bytes, int box_rows) {
  EncodeTiledFn fn = tensor_map_encoder();
  if (fn == nullptr || row_bytes % 16 != 0 || row_bytes < 128) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)(row_bytes / elem_bytes), (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)(128 / elem_bytes), (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, type, 2, ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

std::size_t tc_gemm_workspace_bytes(int M, int N, int K, int terms, bool cplx) {
  return split_layout(cplx ? 2 * M : M, N, cplx ? 2 * K : K, terms == 3 ? 2 : 3).total;
}

namespace {
template <typename T>
cudaError_t tc_gemm_run(cudaStream_t s, int Mc, int N, int Kc, double alpha, const T *A, int lda, const T *B,
                        int ldb, double beta, float *C, int ldc, void *ws, std::size_t ws_bytes, int terms) {
  constexpr bool cplx = std::is_same<T, float2>::value;
  if (Mc <= 0 || N <= 0) return cudaSuccess;
  const int M = cplx ? 2 * Mc : Mc, K = cplx ? 2 * Kc : Kc;  // the real product
  const int nparts = terms == 3 ? 2 : 3;
  const SplitLayout L = split_layout(M, N, K > 0 ? K : 1, nparts);
  if (ws == nullptr || ws_bytes < L.total) return cudaErrorInvalidValue;
  char *w = static_cast<char *>(ws);
  int *err = reinterpret_cast<int *>(w);
  auto *pa = reinterpret_cast<__nv_bfloat16 *>(w + 256);
  auto *pb = reinterpret_cast<__nv_bfloat16 *>(w + 256 + L.a_bytes);

  cudaError_t e;
  split_a_kernel<T><<<dim3(L.Mpad / 32, L.Kpad / 32), 256, 0, s>>>(M, K, A, lda, Mc, Kc, L.Mpad, L.Kpad, nparts,
                                                                   pa);
  if ((e = launched()) != cudaSuccess) return e;
  {
    const int gy = L.Npad < 65535 ? L.Npad : 65535;
    split_b_kernel<T><<<dim3((L.Kpad + 255) / 256, gy), 256, 0, s>>>(K, N, B, ldb, Kc, L.Npad, L.Kpad, nparts,
                                                                     pb);
    if ((e = launched()) != cudaSuccess) return e;
  }

  CUtensorMap ma, mb;
  if (!make_map(&ma, pa, (long long)nparts * L.Mpad, L.Kpad, TM)) return cudaErrorNotSupported;
  if (!make_map(&mb, pb, (long long)nparts * L.Npad, L.Kpad, TN)) return cudaErrorNotSupported;

  TcParams p = {};
  p.M = M;
  p.Mc = cplx ? Mc : 0;
  p.N = N;
  p.nkb = L.Kpad / TK;
  p.Mpad = L.Mpad;
  p.Npad = L.Npad;
  if (terms == 3) {
    const int A3[3] = {1, 0, 0}, B3[3] = {0, 1, 0};
    p.nterms = 3;
    for (int t = 0; t < 3; ++t) p.pa[t] = A3[t], p.pb[t] = B3[t];
  } else {
    const int A6[6] = {2, 0, 1, 1, 0, 0}, B6[6] = {0, 2, 1, 0, 1, 0};
    p.nterms = 6;
    for (int t = 0; t < 6; ++t) p.pa[t] = A6[t], p.pb[t] = B6[t];
  }
  p.alpha = (float)alpha;
  p.beta = (float)beta;
  p.C = C;
  p.ldc = ldc;
  p.err = err;

  // few k-blocks (the LU's K = 32 / 64 updates): two stages, two CTAs per SM
  const bool shallow = p.nterms * p.nkb <= 12;
  auto kern = shallow ? tc_split_gemm_kernel<2, 2> : tc_split_gemm_kernel<4, 1>;
  const int smem = (shallow ? 2 : 4) * (kA + kB) + 1024 + 256;
  static bool configured[2] = {false, false};
  if (!configured[shallow]) {
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
      return e;
    configured[shallow] = true;
  }
  kern<<<dim3(L.Mpad / TM, L.Npad / TN), kThreads, smem, s>>>(ma, mb, p);
  return launched();
}
}  // namespace

cudaError_t tc_gemm_f32(cudaStream_t s, int M, int N, int K, double alpha, const float *A, int lda,
                        const float *B, int ldb, double beta, float *C, int ldc, void *ws,
                        std::size_t ws_bytes, int terms) {
  return tc_gemm_run<float>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, ws, ws_bytes, terms);
}

cudaError_t tc_gemm_c64(cudaStream_t s, int M, int N, int K, double alpha, const float2 *A, int lda,
                        const float2 *B, int ldb, double beta, float2 *C, int ldc, void *ws,
                        std::size_t ws_bytes, int terms) {
  return tc_gemm_run<float2>(s, M, N, K, alpha, A, lda, B, ldb, beta, reinterpret_cast<float *>(C), ldc, ws,
                             ws_bytes, terms);
}

}  // namespace clm
