// oz_gemm.cu -- FP64 and complex128 GEMM on the INT8 tensor cores
// (tcgen05.mma kind::i8, s32 accumulators in TMEM) by the Ozaki splitting
// scheme, for the double-precision tiers of the matrix-exponential path.
//
// C = alpha A B + beta C, column-major, alpha and beta real. Every row r of A
// is scaled by 2^-ea[r], ea[r] the binary exponent of the row's largest
// magnitude, every column c of B by 2^-eb[c]; the scaled values lie in
// (-1, 1) and are cut into ks signed 7-bit digits by truncation, each digit in
// [-127, 127]:
//     A[r,k] = 2^ea[r] sum_{i<ks} a_i[r,k] 2^(-7(i+1))  + |rest| < 2^(ea[r]-7ks)
// The product keeps the digit pairs of total weight i + j < ks, level by
// level:
//     S_l = sum_{i+j=l} a_i b_j              (exact in int32 on the tensor cores)
//     C[r,c] = 2^(ea[r]+eb[c]-14) sum_{l<ks} 2^(-7l) S_l[r,c]   (FP64)
// so the error is about 2^(-7ks) relative to |A| |B| row by column (ks = 7:
// 49 bits). Complex products are one real product of twice the rows and twice
// the depth, [Cr; Ci] = [[Ar, -Ai]; [Ai, Ar]] [Br; Bi], rows r and M + r
// sharing one exponent and the two halves of column c of B' one exponent.
//
// Square products (M = N = K) split off both diagonals first, X = Dx + Yx,
// Z = Dz + Yz: the digits cut only the off-diagonal parts (their rows and
// columns scaled by their own maxima) and the epilogue adds the rest exactly
// in FP64 by a pass after the GEMM, X Z = Yx Yz + Dx Z + X Dz - Dx Dz. The
// expm path's operands are
// often close to a multiple of I plus a small part (W, the quotient before its
// squarings, the powers of a skew-Hermitian matrix), whose diagonal would
// otherwise set every row's scale and cost the off-diagonal entries ~10 bits.
//
// Digits are written once per operand by slicing kernels into K-major int8
// buffers (rows of Kp bytes, zero padded to the tile grid), so the GEMM's
// producer reads every operand tile with one TMA copy, 128-byte swizzled.
//
// GEMM kernel (one CTA per 128 x 128 output tile, 10 warps):
//   warp 0      TMA producer: a 4-stage ring of (A 128 x 128, B 128 x 128)
//               int8 tiles, level by level, digit pair by digit pair
//   warp 1      TMEM allocator (two 128-column s32 accumulators) and MMA
//               issuer: one elected thread issues tcgen05.mma 128x128x32,
//               level l into accumulator l % 2
//   warps 2..9  epilogue: drain level l's accumulator (tcgen05.ld) into FP64
//               registers while the MMAs of level l + 1 run into the other,
//               then scale and store; two warps per TMEM lane quarter, 64
//               columns each
// Every mbarrier wait is bounded and gives up early once the CTA has aborted;
// an abort records an error code in the workspace and the CTA unwinds only
// after its own TMA copies and MMAs have completed.
#include <cuda.h>

#include <type_traits>

#include "kernels.cuh"
#include "tcgen05.cuh"

namespace clm {

namespace {

using namespace tc;

constexpr int OTM = 128;            // UMMA M (TMEM lanes)
constexpr int OTN = 128;            // UMMA N (TMEM columns per accumulator)
constexpr int OTK = 128;            // k-block: one 128-byte swizzle atom of int8
constexpr int OUK = 32;             // UMMA K for 8-bit inputs
constexpr int OSTAGES = 6;
constexpr int kOzThreads = 320;
constexpr int kOzEpiWarps = 8;
constexpr int kOA = OTM * OTK;      // bytes of one A stage
constexpr int kOB = OTN * OTK;      // bytes of one B stage
constexpr uint32_t kOzIdesc = idesc_s8_s32(OTM, OTN);

struct OzParams {
  int Mrows, N;        // rows of A (2M for complex) and columns of the output
  int M;               // rows of the caller's C (complex: rows >= M are imaginary parts)
  int nkb;             // k-blocks of the (real) depth
  int ks;              // digits per operand
  int Mrp, Np;         // rows of one A digit plane / one B digit plane
  const unsigned long long *amax;  // per row of A: bits of the largest magnitude
  const unsigned long long *bmax;  // per column of B
  double alpha, beta;
  double *C;           // as doubles; complex: interleaved (re, im)
  int ldc;             // in elements of the caller's type
  int cplx;
  int *err;
  long long spin;      // bounded-wait tries (kSpinLimit in normal use)
  int skip_loads;      // 1: the producer issues no copy (exercises the abort path)
};

// Bounded wait that also gives up once the CTA's abort flag is raised.
__device__ __forceinline__ bool wait_or_abort(uint64_t *bar, uint32_t parity, const int *abort_flag,
                                              long long limit) {
  for (long long i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255 && *(volatile const int *)abort_flag) return false;
  }
  return false;
}

__device__ __forceinline__ int exp_of_bits(unsigned long long bits) {
  int e = 0;
  frexp(__longlong_as_double((long long)bits), &e);
  return e;
}

// Exact int32 -> double through the 1.5 * 2^52 bias.
__device__ __forceinline__ double i32_to_f64(uint32_t v) {
  const long long bias = 0x4338000000000000ll;
  return __longlong_as_double(bias + (long long)(int)v) - 6755399441055744.0;
}

__global__ void __launch_bounds__(kOzThreads, 1)
    oz_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                   const OzParams prm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char *sA = base;
  unsigned char *sB = base + OSTAGES * kOA;
  uint64_t *full = reinterpret_cast<uint64_t *>(sB + OSTAGES * kOB);
  uint64_t *empty = full + OSTAGES;
  uint64_t *acc_full = empty + OSTAGES;  // [2]
  uint64_t *acc_empty = acc_full + 2;    // [2]
  uint64_t *mma_done = acc_empty + 2;
  int *col_exp = reinterpret_cast<int *>(mma_done + 1);  // [OTN]
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(col_exp + OTN);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * OTM, n0 = blockIdx.y * OTN;
  const int ks = prm.ks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < OSTAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kOzEpiWarps);
    }
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < OTN) {
    const int c = n0 + threadIdx.x;
    col_exp[threadIdx.x] = c < prm.N ? exp_of_bits(prm.bmax[c]) : 0;
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 2 * OTN);
    fence_before();
  }
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer: level l, digit pair (i, l - i), k-block kb ----
    int it = 0, issued = 0;
    bool ok = true;
    for (int l = 0; l < ks && ok; ++l)
      for (int i = 0; i <= l && ok; ++i)
        for (int kb = 0; kb < prm.nkb; ++kb, ++it) {
          const int s = it % OSTAGES;
          const uint32_t ph = (uint32_t)((it / OSTAGES) & 1);
          if (!wait_or_abort(&empty[s], ph ^ 1u, abort_flag, prm.spin)) {
            record_error(prm.err, 1);
            *(volatile int *)abort_flag = 1;
            ok = false;
            break;
          }
          if (prm.skip_loads) continue;
          mbar_expect_tx(&full[s], kOA + kOB);
          tma_load_2d(sA + s * kOA, &map_a, &full[s], kb * OTK, i * prm.Mrp + m0);
          tma_load_2d(sB + s * kOB, &map_b, &full[s], kb * OTK, (l - i) * prm.Np + n0);
          issued = it + 1;
        }
    // drain: the copies this thread issued land before the CTA exits
    for (int j = issued - OSTAGES > 0 ? issued - OSTAGES : 0; j < issued; ++j)
      mbar_wait(&full[j % OSTAGES], (uint32_t)((j / OSTAGES) & 1), prm.spin);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    int it = 0;
    bool ok = true;
    for (int l = 0; l < ks && ok; ++l) {
      const int b = l & 1;
      const uint32_t use = (uint32_t)(l >> 1);
      if (!wait_or_abort(&acc_empty[b], (use & 1u) ^ 1u, abort_flag, prm.spin)) {
        record_error(prm.err, 2);
        ok = false;
        break;
      }
      fence_after();
      const uint32_t d = tmem + (uint32_t)(b * OTN);
      for (int i = 0; i <= l && ok; ++i)
        for (int kb = 0; kb < prm.nkb; ++kb, ++it) {
          const int s = it % OSTAGES;
          const uint32_t ph = (uint32_t)((it / OSTAGES) & 1);
          if (!wait_or_abort(&full[s], ph, abort_flag, prm.spin)) {
            record_error(prm.err, 2);
            ok = false;
            break;
          }
          fence_after();
          const uint32_t a0 = saddr(sA + s * kOA), b0 = saddr(sB + s * kOB);
#pragma unroll
          for (int k = 0; k < OTK / OUK; ++k)  // +32 bytes per 32-element k step inside the atom
            mma_i8(d, smem_desc_sw128(a0 + k * 32), smem_desc_sw128(b0 + k * 32), kOzIdesc,
                   (i > 0 || kb > 0 || k > 0) ? 1u : 0u);
          mma_commit(&empty[s]);
        }
      if (ok) mma_commit(&acc_full[b]);
    }
    if (!ok) *(volatile int *)abort_flag = 1;
    // tracks every MMA issued above: nothing reads shared memory or writes
    // TMEM once this wait has passed
    mma_commit(mma_done);
    if (!mbar_wait(mma_done, 0, prm.spin)) record_error(prm.err, 4);
  } else if (warp >= 2) {
    // ---- epilogue ----
    const int q = warp & 3;                 // TMEM lane quarter this warp may access
    const int half = (warp - 2) >> 2;       // columns [64 half, 64 half + 64) of the tile
    const int row = m0 + q * 32 + lane;
    const bool live = row < prm.Mrows;
    const int er = live ? exp_of_bits(prm.amax[row]) - 14 : 0;
    const bool imag = prm.cplx && row >= prm.M;
    const int r = imag ? row - prm.M : row;
    double acc[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) acc[j] = 0.0;
    bool ok = true;
    for (int l = 0; l < ks; ++l) {
      const int b = l & 1;
      if (!wait_or_abort(&acc_full[b], (uint32_t)((l >> 1) & 1), abort_flag, prm.spin)) {
        if (!*(volatile int *)abort_flag) record_error(prm.err, 3);
        *(volatile int *)abort_flag = 1;
        ok = false;
        break;
      }
      fence_after();
      const double w = ldexp(1.0, -7 * l);
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * OTN + half * 64);
      uint32_t v[32];
      tmem_ld32(taddr, v);
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[j] = fma(i32_to_f64(v[j]), w, acc[j]);
      tmem_ld32(taddr + 32, v);
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[32 + j] = fma(i32_to_f64(v[j]), w, acc[32 + j]);
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
    }
    if (ok && live) {
      // element (r, c) of C as a double; complex: its real or imaginary half
      const std::size_t step = prm.cplx ? 2 * (std::size_t)prm.ldc : (std::size_t)prm.ldc;
      double *cbase = prm.C + (prm.cplx ? 2 * (std::size_t)r + (imag ? 1 : 0) : (std::size_t)r) +
                      (std::size_t)(n0 + half * 64) * step;
      // four columns at a time: their old values are all loaded before the
      // first of their stores
#pragma unroll
      for (int j0 = 0; j0 < 64; j0 += 4) {
        double old[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int c = n0 + half * 64 + j0 + j;
          old[j] = (prm.beta != 0.0 && c < prm.N) ? cbase[(j0 + j) * step] : 0.0;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cl = half * 64 + j0 + j, c = n0 + cl;
          if (c < prm.N) {
            const double x = prm.alpha * scalbn(acc[j0 + j], er + col_exp[cl]);
            cbase[(j0 + j) * step] = prm.beta == 0.0 ? x : fma(prm.beta, old[j], x);
          }
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 1) {
    fence_after();
    tmem_dealloc(tmem, 2 * OTN);
  }
}

// ---- operand maxima -----------------------------------------------------------
// Largest |A[r,k]| over k for every row r of the caller's A (complex: the
// larger of |Re| and |Im|), as the bits of a non-negative double. Block:
// 32 rows x 32 k-lanes, the k-lanes reduced through shared memory.
template <typename T>
__global__ void __launch_bounds__(1024) oz_row_max_kernel(int M, int K, const T *__restrict__ A, int lda,
                                                          int diag, unsigned long long *__restrict__ amax) {
  __shared__ double red[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + tx;
  double m = 0.0;
  if (r < M)
    for (int k = ty; k < K; k += 32) {
      const T x = A[(std::size_t)k * lda + r];
      double v;
      if constexpr (elem<T>::complex) v = fmax(fabs((double)x.x), fabs((double)x.y));
      else v = fabs((double)x);
      m = fmax(m, (diag && k == r) ? 0.0 : v);
    }
  red[ty][tx] = m;
  __syncthreads();
  if (ty == 0 && r < M) {
    for (int j = 1; j < 32; ++j) m = fmax(m, red[j][tx]);
    const unsigned long long bits = (unsigned long long)__double_as_longlong(m);
    amax[r] = bits;
    if constexpr (elem<T>::complex) amax[M + r] = bits;
  }
}

// Largest |B[k,c]| over k for every column c (complex: |Re| and |Im|): one
// warp per column.
template <typename T>
__global__ void __launch_bounds__(256) oz_col_max_kernel(int K, int N, const T *__restrict__ B, int ldb,
                                                         int diag, unsigned long long *__restrict__ bmax) {
  const int c = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= N) return;
  double m = 0.0;
  for (int k = lane; k < K; k += 32) {
    const T x = B[(std::size_t)c * ldb + k];
    double v;
    if constexpr (elem<T>::complex) v = fmax(fabs((double)x.x), fabs((double)x.y));
    else v = fabs((double)x);
    m = fmax(m, (diag && k == c) ? 0.0 : v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) bmax[c] = (unsigned long long)__double_as_longlong(m);
}

// The ks digits of 16 consecutive values x[0..15] scaled by 2^(7 - e),
// packed little-endian into 16 bytes per digit plane.
template <int KS>
__device__ __forceinline__ void digits16(const double (&x)[16], int e, uint4 (&out)[KS]) {
  uint32_t w[KS][4];
#pragma unroll
  for (int i = 0; i < KS; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[i][q] = 0u;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    double y = ldexp(x[j], 7 - e);  // |y| < 128
#pragma unroll
    for (int i = 0; i < KS; ++i) {
      const double d = trunc(y);
      w[i][j >> 2] |= ((uint32_t)(int)d & 0xffu) << (8 * (j & 3));
      y = (y - d) * 128.0;
    }
  }
#pragma unroll
  for (int i = 0; i < KS; ++i) out[i] = make_uint4(w[i][0], w[i][1], w[i][2], w[i][3]);
}

// Element (r, k) of the real A operand: A itself, or for complex the block
// [[Ar, -Ai]; [Ai, Ar]] of 2M rows and 2K columns.
template <typename T>
__device__ __forceinline__ double a_elem(const T *A, int lda, int M, int K, int r, int k, int diag) {
  if constexpr (elem<T>::complex) {
    const bool lo = r < M, left = k < K;
    if (diag && (lo ? r : r - M) == (left ? k : k - K)) return 0.0;
    const T x = A[(std::size_t)(left ? k : k - K) * lda + (lo ? r : r - M)];
    return lo ? (left ? (double)x.x : -(double)x.y) : (left ? (double)x.y : (double)x.x);
  } else {
    if (diag && r == k) return 0.0;
    return (double)A[(std::size_t)k * lda + r];
  }
}

// A digits: planes [ks][Mrp][Kp] of int8, row r = row r of the real A operand.
// Block: 64 rows x 64 k through a shared tile (coalesced reads along rows),
// each thread then cuts 16 consecutive k of one row.
template <typename T, int KS>
__global__ void __launch_bounds__(256) oz_slice_a_kernel(int M, int K, const T *__restrict__ A, int lda,
                                                         int Mrows, int Kr, int Mrp, int Kp, int diag,
                                                         const unsigned long long *__restrict__ amax,
                                                         int8_t *__restrict__ digits) {
  __shared__ double tile[64][65];
  const int r0 = blockIdx.x * 64, k0 = blockIdx.y * 64;
  const int t = threadIdx.x;
  for (int idx = t; idx < 64 * 64; idx += 256) {
    const int rr = idx & 63, kk = idx >> 6;
    const int r = r0 + rr, k = k0 + kk;
    tile[kk][rr] = (r < Mrows && k < Kr) ? a_elem<T>(A, lda, M, K, r, k, diag) : 0.0;
  }
  __syncthreads();
  const int rr = t >> 2, kg = (t & 3) * 16;
  const int r = r0 + rr;
  double x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = tile[kg + j][rr];
  const int e = r < Mrows ? exp_of_bits(amax[r]) : 0;
  uint4 d[KS];
  digits16<KS>(x, e, d);
  const std::size_t plane = (std::size_t)Mrp * Kp;
  int8_t *dst = digits + (std::size_t)r * Kp + k0 + kg;
#pragma unroll
  for (int i = 0; i < KS; ++i) *reinterpret_cast<uint4 *>(dst + i * plane) = d[i];
}

// B digits: planes [ks][Np][Kp], row c = column c of the real B operand (for
// complex, [Br; Bi]); each thread cuts 16 consecutive k of one column.
template <typename T, int KS>
__global__ void __launch_bounds__(128) oz_slice_b_kernel(int K, int N, const T *__restrict__ B, int ldb,
                                                         int Kr, int Np, int Kp, int diag,
                                                         const unsigned long long *__restrict__ bmax,
                                                         int8_t *__restrict__ digits) {
  const int c = blockIdx.y;
  const int k0 = (blockIdx.x * 128 + threadIdx.x) * 16;
  if (k0 >= Kp) return;
  double x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int k = k0 + j;
    double v = 0.0;
    if (c < N && k < Kr && !(diag && (k < K ? k : k - K) == c)) {
      if constexpr (elem<T>::complex) {
        const T z = B[(std::size_t)c * ldb + (k < K ? k : k - K)];
        v = k < K ? (double)z.x : (double)z.y;
      } else {
        v = (double)B[(std::size_t)c * ldb + k];
      }
    }
    x[j] = v;
  }
  const int e = c < N ? exp_of_bits(bmax[c]) : 0;
  uint4 d[KS];
  digits16<KS>(x, e, d);
  const std::size_t plane = (std::size_t)Np * Kp;
  int8_t *dst = digits + (std::size_t)c * Kp + k0;
#pragma unroll
  for (int i = 0; i < KS; ++i) *reinterpret_cast<uint4 *>(dst + i * plane) = d[i];
}

// After the emulated product of the off-diagonal parts of a square product:
// C += alpha (Dx Z + X Dz - Dx Dz), Dx = diag(X), Dz = diag(Z). Coalesced
// along rows, one element per thread.
template <typename T>
__global__ void __launch_bounds__(256) oz_diag_terms_kernel(int n, double alpha, const T *__restrict__ X, int ldx,
                                                            const T *__restrict__ Z, int ldz, T *__restrict__ C,
                                                            int ldc) {
  const int r = blockIdx.x * 256 + threadIdx.x, c = blockIdx.y;
  if (r >= n) return;
  const T dx = X[(std::size_t)r * ldx + r], dz = Z[(std::size_t)c * ldz + c];
  T t = add(mul(dx, Z[(std::size_t)c * ldz + r]), mul(X[(std::size_t)c * ldx + r], dz));
  if (r == c) t = sub(t, mul(dx, dz));
  T &out = C[(std::size_t)c * ldc + r];
  out = add(out, scale(t, alpha));
}

struct OzLayout {
  int Mrows, Kr, Mrp, Np, Kp;
  std::size_t amax_off, bmax_off, a_off, b_off, total;
};
OzLayout oz_layout(int M, int N, int K, bool cplx, int ks) {
  OzLayout L;
  L.Mrows = cplx ? 2 * M : M;
  L.Kr = cplx ? 2 * K : K;
  L.Mrp = (L.Mrows + OTM - 1) / OTM * OTM;
  L.Np = (N + OTN - 1) / OTN * OTN;
  L.Kp = (L.Kr + OTK - 1) / OTK * OTK;
  std::size_t at = 256;  // error word
  L.amax_off = at;
  at += align_up((std::size_t)L.Mrows * 8, 256);
  L.bmax_off = at;
  at += align_up((std::size_t)N * 8, 256);
  L.a_off = at;
  at += align_up((std::size_t)ks * L.Mrp * L.Kp, 256);
  L.b_off = at;
  at += align_up((std::size_t)ks * L.Np * L.Kp, 256);
  L.total = at;
  return L;
}

template <typename T, int KS>
cudaError_t slice_operands(cudaStream_t s, int M, int N, int K, const T *A, int lda, const T *B, int ldb,
                           int diag, const OzLayout &L, char *w) {
  auto *amax = reinterpret_cast<unsigned long long *>(w + L.amax_off);
  auto *bmax = reinterpret_cast<unsigned long long *>(w + L.bmax_off);
  auto *da = reinterpret_cast<int8_t *>(w + L.a_off);
  auto *db = reinterpret_cast<int8_t *>(w + L.b_off);
  cudaError_t e;
  oz_row_max_kernel<T><<<(M + 31) / 32, 1024, 0, s>>>(M, K, A, lda, diag, amax);
  if ((e = launched()) != cudaSuccess) return e;
  oz_col_max_kernel<T><<<(N + 7) / 8, 256, 0, s>>>(K, N, B, ldb, diag, bmax);
  if ((e = launched()) != cudaSuccess) return e;
  oz_slice_a_kernel<T, KS><<<dim3(L.Mrp / 64, L.Kp / 64), 256, 0, s>>>(M, K, A, lda, L.Mrows, L.Kr, L.Mrp,
                                                                       L.Kp, diag, amax, da);
  if ((e = launched()) != cudaSuccess) return e;
  oz_slice_b_kernel<T, KS><<<dim3((L.Kp / 16 + 127) / 128, L.Np), 128, 0, s>>>(K, N, B, ldb, L.Kr, L.Np, L.Kp,
                                                                               diag, bmax, db);
  return launched();
}

constexpr int kOzSmem = OSTAGES * (kOA + kOB) + 1024 + 256 + OTN * 4 + 64;

}  // namespace

std::size_t oz_gemm_workspace_bytes(int M, int N, int K, bool cplx, int ks) {
  return oz_layout(M, N, K > 0 ? K : 1, cplx, ks).total;
}

bool oz_gemm_supported(int K, bool cplx, int ks) {
  // the level sums stay exact in int32: (ks) digit pairs x 127^2 x depth
  const double depth = cplx ? 2.0 * K : (double)K;
  return ks >= 2 && ks <= 8 && (double)ks * 127.0 * 127.0 * depth < 2147483647.0;
}

template <typename T>
cudaError_t oz_gemm(cudaStream_t s, int M, int N, int K, double alpha, const T *A, int lda, const T *B,
                    int ldb, double beta, T *C, int ldc, void *ws, std::size_t ws_bytes, int ks,
                    long long spin, int skip_loads) {
  static_assert(std::is_same<T, double>::value || std::is_same<T, double2>::value, "FP64 types only");
  constexpr bool cplx = elem<T>::complex;
  if (M <= 0 || N <= 0) return cudaSuccess;
  if (!oz_gemm_supported(K, cplx, ks)) return cudaErrorInvalidValue;
  const OzLayout L = oz_layout(M, N, K > 0 ? K : 1, cplx, ks);
  if (ws == nullptr || ws_bytes < L.total) return cudaErrorInvalidValue;
  char *w = static_cast<char *>(ws);
  const int diag = (M == N && N == K) ? 1 : 0;
  cudaError_t e;
  switch (ks) {
  case 2: e = slice_operands<T, 2>(s, M, N, K, A, lda, B, ldb, diag, L, w); break;
  case 3: e = slice_operands<T, 3>(s, M, N, K, A, lda, B, ldb, diag, L, w); break;
  case 4: e = slice_operands<T, 4>(s, M, N, K, A, lda, B, ldb, diag, L, w); break;
  case 5: e = slice_operands<T, 5>(s, M, N, K, A, lda, B, ldb, diag, L, w); break;
  case 6: e = slice_operands<T, 6>(s, M, N, K, A, lda, B, ldb, diag, L, w); break;
  case 7: e = slice_operands<T, 7>(s, M, N, K, A, lda, B, ldb, diag, L, w); break;
  default: e = slice_operands<T, 8>(s, M, N, K, A, lda, B, ldb, diag, L, w); break;
  }
  if (e != cudaSuccess) return e;

  CUtensorMap ma, mb;
  if (!make_rowmajor_map_sw128(&ma, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, w + L.a_off, (long long)ks * L.Mrp, L.Kp,
                               OTM))
    return cudaErrorNotSupported;
  if (!make_rowmajor_map_sw128(&mb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, w + L.b_off, (long long)ks * L.Np, L.Kp,
                               OTN))
    return cudaErrorNotSupported;

  OzParams p = {};
  p.Mrows = L.Mrows;
  p.N = N;
  p.M = M;
  p.nkb = L.Kp / OTK;
  p.ks = ks;
  p.Mrp = L.Mrp;
  p.Np = L.Np;
  p.amax = reinterpret_cast<const unsigned long long *>(w + L.amax_off);
  p.bmax = reinterpret_cast<const unsigned long long *>(w + L.bmax_off);
  p.alpha = alpha;
  p.beta = beta;
  p.C = reinterpret_cast<double *>(C);
  p.ldc = ldc;
  p.cplx = cplx ? 1 : 0;
  p.err = reinterpret_cast<int *>(w);
  p.spin = spin > 0 ? spin : kSpinLimit;
  p.skip_loads = skip_loads;

  static bool configured = false;
  if (!configured) {
    if ((e = cudaFuncSetAttribute(oz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzSmem)) !=
        cudaSuccess)
      return e;
    configured = true;
  }
  oz_gemm_kernel<<<dim3(L.Mrp / OTM, L.Np / OTN), kOzThreads, kOzSmem, s>>>(ma, mb, p);
  if ((e = launched()) != cudaSuccess || !diag) return e;
  oz_diag_terms_kernel<T><<<dim3((M + 255) / 256, N), 256, 0, s>>>(M, alpha, A, lda, B, ldb, C, ldc);
  return launched();
}

template cudaError_t oz_gemm<double>(cudaStream_t, int, int, int, double, const double *, int, const double *,
                                     int, double, double *, int, void *, std::size_t, int, long long, int);
template cudaError_t oz_gemm<double2>(cudaStream_t, int, int, int, double, const double2 *, int,
                                      const double2 *, int, double, double2 *, int, void *, std::size_t, int,
                                      long long, int);

}  // namespace clm
