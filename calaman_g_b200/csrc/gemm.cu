// gemm.cu -- C = alpha A B + beta C (NN, column-major) for the four element
// types of the path.
//
//   double   : FP64 tensor-core tiles (mma.sync m16n8k8 .f64, "DMMA"); tcgen05
//              has no f64 kind, so this is the FP64 tensor path on sm_100a.
//   double2  : complex128 as four real DMMA products per tile
//              (Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br), operands read once
//              as interleaved 16-byte pairs.
//   float / float2 : register-tiled FP32 SIMT kernel (the plain single tier).
//
// Operands are staged global -> shared by cp.async in a multi-stage ring; all
// edges (M, N, K not multiples of the tile) are zero-filled by the copy's
// src-size operand, so any shape and any leading dimension is legal.
#include <algorithm>
#include "dmma.cuh"

namespace clm {

namespace {

// ---------------------------------------------------------------------------
// Real FP64: CTA tile BM x BN x 16, warp tile WM x WN built from 16x8 DMMAs.
// Shared layout: sA[k][m] (row stride BM+4 doubles), sB[n][k] (stride 20);
// both strides are 4 mod 16 doubles, which makes every 8-byte fragment load
// of a half-warp hit 16 distinct bank pairs.
// ---------------------------------------------------------------------------
template <int BM, int BN, int WM, int WN, int STAGES, bool V16>
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32)
    dgemm_nn_kernel(int M, int N, int K, double alpha, const double *__restrict__ A, int lda,
                    const double *__restrict__ B, int ldb, double beta, double *__restrict__ C,
                    int ldc, int kslice, long long cstride) {
  // split K: slice blockIdx.z takes K rows [z kslice, (z+1) kslice) into C + z cstride
  {
    const int kz0 = blockIdx.z * kslice;
    K = min(K - kz0, kslice);
    A += (std::size_t)kz0 * lda;
    B += kz0;
    C += (std::size_t)blockIdx.z * cstride;
  }
  constexpr int BK = 16;
  constexpr int NT = (BM / WM) * (BN / WN) * 32;
  constexpr int SA = BM + 4;
  constexpr int SB = BK + 4;
  constexpr int MI = WM / 16;
  constexpr int NI = WN / 8;
  extern __shared__ __align__(16) double smem_d[];
  double *sA = smem_d;                       // [STAGES][BK][SA]
  double *sB = smem_d + STAGES * BK * SA;    // [STAGES][BN][SB]

  const int m0 = blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp % (BM / WM)) * WM;
  const int wn0 = (warp / (BM / WM)) * WN;

  auto load_tile = [&](int stage, int kt) {
    const int k0 = kt * BK;
    double *a = sA + stage * BK * SA;
    double *b = sB + stage * BN * SB;
    if (V16) {
      constexpr int CA = BK * BM / 2;
#pragma unroll
      for (int c = tid; c < CA; c += NT) {
        const int kk = c / (BM / 2), mm = (c % (BM / 2)) * 2;
        const int gm = m0 + mm, gk = k0 + kk;
        int bytes = (gk < K) ? (M - gm) * 8 : 0;
        bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
        const double *src = bytes ? A + (std::size_t)gk * lda + gm : A;
        cp_async16(a + kk * SA + mm, src, bytes);
      }
      constexpr int CB = BN * BK / 2;
#pragma unroll
      for (int c = tid; c < CB; c += NT) {
        const int nn = c / (BK / 2), kk = (c % (BK / 2)) * 2;
        const int gn = n0 + nn, gk = k0 + kk;
        int bytes = (gn < N) ? (K - gk) * 8 : 0;
        bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
        const double *src = bytes ? B + (std::size_t)gn * ldb + gk : B;
        cp_async16(b + nn * SB + kk, src, bytes);
      }
    } else {
      constexpr int CA = BK * BM;
#pragma unroll 4
      for (int c = tid; c < CA; c += NT) {
        const int kk = c / BM, mm = c % BM;
        const int gm = m0 + mm, gk = k0 + kk;
        const int bytes = (gk < K && gm < M) ? 8 : 0;
        cp_async8(a + kk * SA + mm, bytes ? A + (std::size_t)gk * lda + gm : A, bytes);
      }
      constexpr int CB = BN * BK;
#pragma unroll 4
      for (int c = tid; c < CB; c += NT) {
        const int nn = c / BK, kk = c % BK;
        const int gn = n0 + nn, gk = k0 + kk;
        const int bytes = (gn < N && gk < K) ? 8 : 0;
        cp_async8(b + nn * SB + kk, bytes ? B + (std::size_t)gn * ldb + gk : B, bytes);
      }
    }
  };

  double acc[MI][NI][4];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

  const int KT = (K + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) load_tile(s, s);
    cp_commit();
  }

  for (int kt = 0; kt < KT; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if (nk < KT) load_tile(nk % STAGES, nk);
      cp_commit();
    }
    const double *a = sA + (kt % STAGES) * BK * SA;
    const double *b = sB + (kt % STAGES) * BN * SB;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 8) {
      double af[MI][4], bf[NI][2];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const int m = wm0 + i * 16 + g;
        af[i][0] = a[(kk + t) * SA + m];
        af[i][1] = a[(kk + t) * SA + m + 8];
        af[i][2] = a[(kk + t + 4) * SA + m];
        af[i][3] = a[(kk + t + 4) * SA + m + 8];
      }
#pragma unroll
      for (int j = 0; j < NI; ++j) {
        const int nn = wn0 + j * 8 + g;
        bf[j][0] = b[nn * SB + kk + t];
        bf[j][1] = b[nn * SB + kk + t + 4];
      }
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NI; ++j) dmma16x8x8(acc[i][j], af[i], bf[j]);
    }
  }
  cp_wait<0>();

  // epilogue: C = alpha acc + beta C (beta == 0 never reads C). Per row
  // block, every old C value is loaded before the first store, so the loads
  // are in flight together instead of one round trip per element.
#pragma unroll
  for (int i = 0; i < MI; ++i) {
    double old[NI][4];
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = m0 + wm0 + i * 16 + g + ((r & 2) ? 8 : 0);
        const int n = n0 + wn0 + j * 8 + 2 * t + (r & 1);
        old[j][r] = (beta != 0.0 && m < M && n < N) ? C[(std::size_t)n * ldc + m] : 0.0;
      }
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = m0 + wm0 + i * 16 + g + ((r & 2) ? 8 : 0);
        const int n = n0 + wn0 + j * 8 + 2 * t + (r & 1);
        if (m < M && n < N) {
          const double v = alpha * acc[i][j][r];
          C[(std::size_t)n * ldc + m] = (beta == 0.0) ? v : fma(beta, old[j][r], v);
        }
      }
  }
}

// ---------------------------------------------------------------------------
// Complex128: CTA tile BM x BN x 16 complex, interleaved (re, im) in shared
// memory; each fragment element is one 16-byte load. Row strides BM+2 and 20
// (complex units) are 2 and 4 mod 8, so a quarter-warp's 16-byte loads hit
// 8 distinct bank quads.
// ---------------------------------------------------------------------------
// kGauss: three real products per complex product instead of four (Gauss /
// "3M": t1 = Ar Br, t2 = Ai Bi, t3 = (Ar + Ai)(Br + Bi); Re = t1 - t2,
// Im = t3 - t1 - t2). The kernel is bound by the FP64 tensor pipe, so a quarter
// of its DMMAs go; the imaginary part's rounding error grows to
// ~eps (|Ar| + |Ai|)(|Br| + |Bi|) per term, the same order as the real part's.
template <int BM, int BN, int WM, int WN, int STAGES, bool kGauss = false>
__global__ void __launch_bounds__((BM / WM) * (BN / WN) * 32)
    zgemm_nn_kernel(int M, int N, int K, double alpha, const double2 *__restrict__ A, int lda,
                    const double2 *__restrict__ B, int ldb, double beta, double2 *__restrict__ C,
                    int ldc, int kslice, long long cstride) {
  {
    const int kz0 = blockIdx.z * kslice;
    K = min(K - kz0, kslice);
    A += (std::size_t)kz0 * lda;
    B += kz0;
    C += (std::size_t)blockIdx.z * cstride;
  }
  constexpr int BK = 16;
  constexpr int NT = (BM / WM) * (BN / WN) * 32;
  constexpr int SA = BM + 2;
  constexpr int SB = BK + 4;
  constexpr int MI = WM / 16;
  constexpr int NI = WN / 8;
  extern __shared__ __align__(16) double2 smem_z[];
  double2 *sA = smem_z;
  double2 *sB = smem_z + STAGES * BK * SA;

  const int m0 = blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp % (BM / WM)) * WM;
  const int wn0 = (warp / (BM / WM)) * WN;

  auto load_tile = [&](int stage, int kt) {
    const int k0 = kt * BK;
    double2 *a = sA + stage * BK * SA;
    double2 *b = sB + stage * BN * SB;
    constexpr int CA = BK * BM;
#pragma unroll
    for (int c = tid; c < CA; c += NT) {
      const int kk = c / BM, mm = c % BM;
      const int gm = m0 + mm, gk = k0 + kk;
      const int bytes = (gk < K && gm < M) ? 16 : 0;
      cp_async16(a + kk * SA + mm, bytes ? A + (std::size_t)gk * lda + gm : A, bytes);
    }
    constexpr int CB = BN * BK;
#pragma unroll
    for (int c = tid; c < CB; c += NT) {
      const int nn = c / BK, kk = c % BK;
      const int gn = n0 + nn, gk = k0 + kk;
      const int bytes = (gn < N && gk < K) ? 16 : 0;
      cp_async16(b + nn * SB + kk, bytes ? B + (std::size_t)gn * ldb + gk : B, bytes);
    }
  };

  // 4M: re, im accumulate Re and Im directly; 3M (kGauss): re = t1, im = t2, t3
  double re[MI][NI][4], im[MI][NI][4], t3[kGauss ? MI : 1][kGauss ? NI : 1][4];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) re[i][j][r] = im[i][j][r] = 0.0;
  if constexpr (kGauss) {
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NI; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) t3[i][j][r] = 0.0;
  }

  const int KT = (K + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) load_tile(s, s);
    cp_commit();
  }
  for (int kt = 0; kt < KT; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if (nk < KT) load_tile(nk % STAGES, nk);
      cp_commit();
    }
    const double2 *a = sA + (kt % STAGES) * BK * SA;
    const double2 *b = sB + (kt % STAGES) * BN * SB;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 8) {
      double ar[MI][4], ai[MI][4], an[MI][4], br[NI][2], bi[NI][2];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const int m = wm0 + i * 16 + g;
        const double2 x0 = a[(kk + t) * SA + m];
        const double2 x1 = a[(kk + t) * SA + m + 8];
        const double2 x2 = a[(kk + t + 4) * SA + m];
        const double2 x3 = a[(kk + t + 4) * SA + m + 8];
        ar[i][0] = x0.x; ai[i][0] = x0.y;
        ar[i][1] = x1.x; ai[i][1] = x1.y;
        ar[i][2] = x2.x; ai[i][2] = x2.y;
        ar[i][3] = x3.x; ai[i][3] = x3.y;
#pragma unroll
        for (int r = 0; r < 4; ++r) an[i][r] = -ai[i][r];
      }
#pragma unroll
      for (int j = 0; j < NI; ++j) {
        const int nn = wn0 + j * 8 + g;
        const double2 y0 = b[nn * SB + kk + t];
        const double2 y1 = b[nn * SB + kk + t + 4];
        br[j][0] = y0.x; bi[j][0] = y0.y;
        br[j][1] = y1.x; bi[j][1] = y1.y;
      }
      if constexpr (kGauss) {
        double as[MI][4], bs[NI][2];
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
          for (int r = 0; r < 4; ++r) as[i][r] = ar[i][r] + ai[i][r];
#pragma unroll
        for (int j = 0; j < NI; ++j)
#pragma unroll
          for (int r = 0; r < 2; ++r) bs[j][r] = br[j][r] + bi[j][r];
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
          for (int j = 0; j < NI; ++j) {
            dmma16x8x8(re[i][j], ar[i], br[j]);
            dmma16x8x8(im[i][j], ai[i], bi[j]);
            dmma16x8x8(t3[i][j], as[i], bs[j]);
          }
      } else {
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
          for (int j = 0; j < NI; ++j) {
            dmma16x8x8(re[i][j], ar[i], br[j]);
            dmma16x8x8(re[i][j], an[i], bi[j]);
            dmma16x8x8(im[i][j], ar[i], bi[j]);
            dmma16x8x8(im[i][j], ai[i], br[j]);
          }
      }
    }
  }
  cp_wait<0>();
  if constexpr (kGauss) {
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NI; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const double t1 = re[i][j][r], t2 = im[i][j][r];
          re[i][j][r] = t1 - t2;
          im[i][j][r] = t3[i][j][r] - t1 - t2;
        }
  }

  // epilogue: all old C values of a row block are loaded before any store
#pragma unroll
  for (int i = 0; i < MI; ++i) {
    double2 old[NI][4];
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = m0 + wm0 + i * 16 + g + ((r & 2) ? 8 : 0);
        const int n = n0 + wn0 + j * 8 + 2 * t + (r & 1);
        old[j][r] = (beta != 0.0 && m < M && n < N) ? C[(std::size_t)n * ldc + m] : make_double2(0.0, 0.0);
      }
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = m0 + wm0 + i * 16 + g + ((r & 2) ? 8 : 0);
        const int n = n0 + wn0 + j * 8 + 2 * t + (r & 1);
        if (m < M && n < N) {
          double2 v = make_double2(alpha * re[i][j][r], alpha * im[i][j][r]);
          if (beta != 0.0) {
            v.x = fma(beta, old[j][r].x, v.x);
            v.y = fma(beta, old[j][r].y, v.y);
          }
          C[(std::size_t)n * ldc + m] = v;
        }
      }
  }
}

// ---------------------------------------------------------------------------
// FP32 SIMT (float, complex64): 64 x 64 CTA tile, 16-deep k slices, 256
// threads each owning a 4 x 4 micro-tile (rows ty + 16 i, cols tx + 16 j).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
    simt_gemm_nn_kernel(int M, int N, int K, double alpha, const T *__restrict__ A, int lda,
                        const T *__restrict__ B, int ldb, double beta, T *__restrict__ C, int ldc) {
  using R = typename elem<T>::real;
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ T sA[2][BK][BM];
  __shared__ T sB[2][BK][BN + 1];
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = elem<T>::zero();

  auto load = [&](int buf, int k0) {
#pragma unroll
    for (int c = tid; c < BK * BM; c += 256) {
      const int kk = c / BM, mm = c % BM;
      const int gm = m0 + mm, gk = k0 + kk;
      sA[buf][kk][mm] = (gm < M && gk < K) ? A[(std::size_t)gk * lda + gm] : elem<T>::zero();
    }
#pragma unroll
    for (int c = tid; c < BK * BN; c += 256) {
      const int nn = c / BK, kk = c % BK;
      const int gn = n0 + nn, gk = k0 + kk;
      sB[buf][kk][nn] = (gn < N && gk < K) ? B[(std::size_t)gn * ldb + gk] : elem<T>::zero();
    }
  };
  const int KT = (K + BK - 1) / BK;
  load(0, 0);
  __syncthreads();
  for (int kt = 0; kt < KT; ++kt) {
    const int cur = kt & 1;
    if (kt + 1 < KT) load(cur ^ 1, (kt + 1) * BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sA[cur][kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sB[cur][kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmac(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  T old[4][4];  // every old C value in flight before the first store
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
      old[i][j] = (beta != 0.0 && m < M && n < N) ? C[(std::size_t)n * ldc + m] : elem<T>::zero();
    }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
      if (m < M && n < N) {
        T v = scale(acc[i][j], (R)alpha);
        if (beta != 0.0) v = add(v, scale(old[i][j], (R)beta));
        C[(std::size_t)n * ldc + m] = v;
      }
    }
}

template <int BM, int BN, int WM, int WN, int STAGES, bool V16>
cudaError_t run_dgemm(cudaStream_t s, int M, int N, int K, double alpha, const double *A, int lda,
                      const double *B, int ldb, double beta, double *C, int ldc, int splits = 1,
                      int kslice = 0, long long cstride = 0) {
  constexpr int NT = (BM / WM) * (BN / WN) * 32;
  constexpr int smem = STAGES * (16 * (BM + 4) + BN * 20) * (int)sizeof(double);
  auto kern = dgemm_nn_kernel<BM, BN, WM, WN, STAGES, V16>;
  static bool configured = false;  // attribute is per-function, process-wide
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, splits);
  kern<<<grid, NT, smem, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, splits > 1 ? kslice : K,
                              cstride);
  return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, int STAGES, bool kGauss = true>
cudaError_t run_zgemm(cudaStream_t s, int M, int N, int K, double alpha, const double2 *A, int lda,
                      const double2 *B, int ldb, double beta, double2 *C, int ldc, int splits = 1,
                      int kslice = 0, long long cstride = 0) {
  constexpr int NT = (BM / WM) * (BN / WN) * 32;
  constexpr int smem = STAGES * (16 * (BM + 2) + BN * 20) * (int)sizeof(double2);
  auto kern = zgemm_nn_kernel<BM, BN, WM, WN, STAGES, kGauss>;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, splits);
  kern<<<grid, NT, smem, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, splits > 1 ? kslice : K,
                              cstride);
  return cudaGetLastError();
}

inline bool aligned16(const void *p) { return (reinterpret_cast<std::uintptr_t>(p) & 15u) == 0; }

// Launch through `run`, bracketed by CUDA events when a timer is active.
template <typename F>
cudaError_t timed_launch(cudaStream_t s, double flops, F &&run, bool count = true) {
  KernelTimer *t = tl_timer;
  if (count) note_launch();
  if (t == nullptr) return run();
  cudaEvent_t a = t->take(), b = t->take();
  if (a == nullptr || b == nullptr) return run();
  cudaEventRecord(a, s);
  const cudaError_t e = run();
  cudaEventRecord(b, s);
  t->starts.push_back(a);
  t->stops.push_back(b);
  t->flops.push_back(flops);
  return e;
}

inline double real_flops(int M, int N, int K) { return 2.0 * M * (double)N * K; }

}  // namespace

// The emulated path, when the driver lent digit-plane scratch and the product
// is large enough (GemmScratch::oz_min_dim in every dimension).
template <typename T>
bool use_oz(int M, int N, int K) {
  const GemmScratch *g = tl_gemm_scratch;
  return g && g->oz && g->oz_digits > 0 && M >= g->oz_min_dim && N >= g->oz_min_dim &&
         K >= g->oz_min_dim && oz_gemm_supported(K, elem<T>::complex, g->oz_digits) &&
         oz_gemm_workspace_bytes(M, N, K, elem<T>::complex, g->oz_digits) <= g->oz_bytes;
}

template <>
cudaError_t gemm_nn<double>(cudaStream_t s, int M, int N, int K, double alpha, const double *A,
                            int lda, const double *B, int ldb, double beta, double *C, int ldc) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  if (use_oz<double>(M, N, K)) {
    const GemmScratch *g = tl_gemm_scratch;
    return timed_launch(
        s, real_flops(M, N, K),
        [&] { return oz_gemm<double>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, g->oz, g->oz_bytes,
                                     g->oz_digits); },
        /*count=*/false);  // its kernels count themselves
  }
  const bool v16 = aligned16(A) && aligned16(B) && (lda % 2 == 0) && (ldb % 2 == 0);
  // 64 x 64 tiles (measured faster than 128 x 128 at 2048^3 and 4096^3: 558
  // vs 658 us, 4.27 vs 4.53 ms); up to two waves of them, 32 x 32 tiles put
  // four times the CTAs on the SMs
  const long long tiles64 = (long long)((M + 63) / 64) * ((N + 63) / 64);
  return timed_launch(s, real_flops(M, N, K), [&] {
    if (tiles64 <= 2 * 148) {
      return v16 ? run_dgemm<32, 32, 16, 16, 4, true>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
                 : run_dgemm<32, 32, 16, 16, 4, false>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    }
    return v16 ? run_dgemm<64, 64, 32, 32, 4, true>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
               : run_dgemm<64, 64, 32, 32, 4, false>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  });
}

template <>
cudaError_t gemm_nn<double2>(cudaStream_t s, int M, int N, int K, double alpha, const double2 *A,
                             int lda, const double2 *B, int ldb, double beta, double2 *C, int ldc) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  if (use_oz<double2>(M, N, K)) {
    const GemmScratch *g = tl_gemm_scratch;
    return timed_launch(
        s, 4.0 * real_flops(M, N, K),
        [&] { return oz_gemm<double2>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, g->oz, g->oz_bytes,
                                      g->oz_digits); },
        /*count=*/false);
  }
  const long long tiles64 = (long long)((M + 63) / 64) * ((N + 63) / 64);
  return timed_launch(s, 4.0 * real_flops(M, N, K), [&] {
    // up to two waves of 64 x 64 tiles (n <= 1024 square, skinny products):
    // 32 x 32 tiles, four times the CTAs, spread the last wave (1024^3: 1.73
    // waves -> 6.9, 278 -> 235 us)
    if (tiles64 <= 2 * 148)
      return run_zgemm<32, 32, 16, 16, 3>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    return run_zgemm<64, 64, 32, 16, 3>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  });
}

// Thin products (fewer than 64 rows or columns: the LU's look-ahead update of
// the next panel's 32 columns, the last blocks of the triangular solves) fill
// few tensor-core tiles; they run on the SIMT kernel, one launch instead of two
// split kernels and a tcgen05 GEMM (float32 4096 expm 34.3 -> 36.4 expm/s, the
// same error against the FP64 oracle).
inline bool thin_product(int M, int N) { return M < 64 || N < 64; }

template <>
cudaError_t gemm_nn<float>(cudaStream_t s, int M, int N, int K, double alpha, const float *A,
                           int lda, const float *B, int ldb, double beta, float *C, int ldc) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  GemmScratch *g = tl_gemm_scratch;
  if (g && K > 0 && g->ptr && !thin_product(M, N) && tc_gemm_workspace_bytes(M, N, K, g->terms) <= g->bytes) {
    return timed_launch(
        s, real_flops(M, N, K),
        [&] { return tc_gemm_f32(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, g->ptr, g->bytes, g->terms); },
        /*count=*/false);  // its split and GEMM kernels count themselves
  }
  return timed_launch(s, real_flops(M, N, K), [&] {
    dim3 grid((M + 63) / 64, (N + 63) / 64);
    simt_gemm_nn_kernel<float><<<grid, 256, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    return cudaGetLastError();
  });
}

template <>
cudaError_t gemm_nn<float2>(cudaStream_t s, int M, int N, int K, double alpha, const float2 *A,
                            int lda, const float2 *B, int ldb, double beta, float2 *C, int ldc) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  GemmScratch *g = tl_gemm_scratch;
  if (g && K > 0 && g->ptr && !thin_product(M, N) && tc_gemm_workspace_bytes(M, N, K, g->terms, true) <= g->bytes) {
    return timed_launch(
        s, 4.0 * real_flops(M, N, K),
        [&] { return tc_gemm_c64(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, g->ptr, g->bytes, g->terms); },
        /*count=*/false);
  }
  return timed_launch(s, 4.0 * real_flops(M, N, K), [&] {
    dim3 grid((M + 63) / 64, (N + 63) / 64);
    simt_gemm_nn_kernel<float2><<<grid, 256, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    return cudaGetLastError();
  });
}

// ---- split-K: the skinny products (few output tiles, long K) ----------------
namespace {
template <typename T>
__global__ void splitk_reduce_kernel(int M, int N, int splits, const T *__restrict__ part, double alpha,
                                     double beta, T *__restrict__ C, int ldc) {
  const long long total = (long long)M * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    T acc = part[idx];
    for (int z = 1; z < splits; ++z) acc = add(acc, part[(std::size_t)z * total + idx]);  // slice order
    const int i = (int)(idx % M), j = (int)(idx / M);
    T &c = C[(std::size_t)j * ldc + i];
    c = beta == 0.0 ? scale(acc, alpha) : rfma(alpha, acc, scale(c, beta));
  }
}

// Slices of 64-multiple K so that tiles x slices fills two waves of SMs.
int splitk_slices(int M, int N, int K, int max_splits, int *kslice) {
  const long long tiles = (long long)((M + 63) / 64) * ((N + 63) / 64);
  long long want = (2LL * sm_count() + tiles - 1) / tiles;
  want = std::min<long long>(want, max_splits);
  want = std::min<long long>(want, std::max(1, K / 64));
  if (want < 1) want = 1;
  int ks = (int)((K + want - 1) / want);
  ks = (ks + 63) / 64 * 64;
  *kslice = ks;
  return (K + ks - 1) / ks;
}
}  // namespace

template <>
cudaError_t gemm_nn_splitk<double>(cudaStream_t s, int M, int N, int K, double alpha, const double *A, int lda,
                                   const double *B, int ldb, double beta, double *C, int ldc, double *partial,
                                   int max_splits) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  int ks = 0;
  const int sp = splitk_slices(M, N, K, max_splits, &ks);
  if (sp <= 1) return gemm_nn<double>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  const bool v16 = aligned16(A) && aligned16(B) && (lda % 2 == 0) && (ldb % 2 == 0);
  cudaError_t e = timed_launch(s, real_flops(M, N, K), [&] {
    return v16 ? run_dgemm<64, 64, 32, 32, 4, true>(s, M, N, K, 1.0, A, lda, B, ldb, 0.0, partial, M, sp, ks,
                                                     (long long)M * N)
               : run_dgemm<64, 64, 32, 32, 4, false>(s, M, N, K, 1.0, A, lda, B, ldb, 0.0, partial, M, sp, ks,
                                                      (long long)M * N);
  });
  if (e != cudaSuccess) return e;
  splitk_reduce_kernel<double><<<std::min(((long long)M * N + 255) / 256, 4LL * 148), 256, 0, s>>>(
      M, N, sp, partial, alpha, beta, C, ldc);
  return launched();
}

template <>
cudaError_t gemm_nn_splitk<double2>(cudaStream_t s, int M, int N, int K, double alpha, const double2 *A,
                                    int lda, const double2 *B, int ldb, double beta, double2 *C, int ldc,
                                    double2 *partial, int max_splits) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  int ks = 0;
  const int sp = splitk_slices(M, N, K, max_splits, &ks);
  if (sp <= 1) return gemm_nn<double2>(s, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  cudaError_t e = timed_launch(s, 4.0 * real_flops(M, N, K), [&] {
    return run_zgemm<64, 64, 32, 16, 3>(s, M, N, K, 1.0, A, lda, B, ldb, 0.0, partial, M, sp, ks,
                                         (long long)M * N);
  });
  if (e != cudaSuccess) return e;
  splitk_reduce_kernel<double2><<<std::min(((long long)M * N + 255) / 256, 4LL * 148), 256, 0, s>>>(
      M, N, sp, partial, alpha, beta, C, ldc);
  return launched();
}

}  // namespace clm
