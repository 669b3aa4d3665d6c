// elementwise.cu -- the HBM-bound kernels of the path: the 1-norm, the fused
// Pade combinations, the numerator/denominator split, scaling/copies, the
// Paterson-Stockmeyer block build and Horner's identity updates.
//
// Layout: column-major; the 2-D launch maps blockIdx.y to a column and the x
// dimension to rows, so consecutive threads touch consecutive addresses and no
// integer division is needed to recover (row, col).
#include "kernels.cuh"

namespace clm {

namespace {

constexpr int kRowThreads = 256;

inline dim3 grid_2d(int rows, int cols) {
  const int gx = (rows + kRowThreads - 1) / kRowThreads;
  const int gy = cols < 65535 ? cols : 65535;
  return dim3(gx, gy, 1);
}

// ---- 1-norm: one warp per column, FP64 sums, NaN-sticky max by atomicMax on
// the bit pattern of a non-negative double (monotone for +0 .. +Inf; a NaN is
// canonicalised to the positive quiet NaN, whose pattern exceeds +Inf).
template <typename T>
__global__ void norm1_kernel(int n, const T *__restrict__ A, int lda, double *__restrict__ colsum,
                             unsigned long long *__restrict__ norm_bits) {
  const int warps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int col = blockIdx.x * warps + (threadIdx.x >> 5); col < n; col += gridDim.x * warps) {
    const T *c = A + (std::size_t)col * lda;
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += modulus(c[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      if (colsum) colsum[col] = s;
      const unsigned long long bits =
          isnan(s) ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(s);
      atomicMax(norm_bits, bits);
    }
  }
}

template <typename T, typename R>
__global__ void colsum_kernel(int n, const T *__restrict__ A, int lda, R *__restrict__ colsum) {
  const int warps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int col = blockIdx.x * warps + (threadIdx.x >> 5); col < n; col += gridDim.x * warps) {
    const T *c = A + (std::size_t)col * lda;
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += modulus(c[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) colsum[col] = (R)s;
  }
}

// Single-block NaN-propagating max in place at v[0] (src/expm/expm.cu:212-245).
template <typename R>
__global__ void max_inplace_kernel(int n, R *v) {
  __shared__ R sm[32];
  R best = R(0);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const R x = v[i];
    if (x > best || isnan(x)) {
      if (!isnan(best)) best = x;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const R y = __shfl_xor_sync(0xffffffffu, best, o);
    if (y > best || isnan(y)) {
      if (!isnan(best)) best = y;
    }
  }
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int w = blockDim.x >> 5;
    best = threadIdx.x < w ? sm[threadIdx.x] : R(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const R y = __shfl_xor_sync(0xffffffffu, best, o);
      if (y > best || isnan(y)) {
        if (!isnan(best)) best = y;
      }
    }
    if (threadIdx.x == 0) v[0] = best;
  }
}

// ---- Pade even/odd: every power read once, both combinations written ------
template <typename T, int NP>
__global__ void pade_even_odd_kernel(int n, const T *__restrict__ P1, const T *__restrict__ P2,
                                     const T *__restrict__ P3, const T *__restrict__ P4,
                                     double cv0, double cv1, double cv2, double cv3, double cv4,
                                     double cw0, double cw1, double cw2, double cw3, double cw4,
                                     T *__restrict__ V, T *__restrict__ W) {
  using R = typename elem<T>::real;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  for (int col = blockIdx.y; col < n; col += gridDim.y) {
    const std::size_t idx = (std::size_t)col * n + row;
    T v = elem<T>::zero(), w = elem<T>::zero();
    const T x1 = P1[idx];
    v = rfma((R)cv1, x1, v);
    w = rfma((R)cw1, x1, w);
    if (NP >= 2) {
      const T x = P2[idx];
      v = rfma((R)cv2, x, v);
      w = rfma((R)cw2, x, w);
    }
    if (NP >= 3) {
      const T x = P3[idx];
      v = rfma((R)cv3, x, v);
      w = rfma((R)cw3, x, w);
    }
    if (NP >= 4) {
      const T x = P4[idx];
      v = rfma((R)cv4, x, v);
      w = rfma((R)cw4, x, w);
    }
    if (row == col) {
      v = add_real(v, (R)cv0);
      w = add_real(w, (R)cw0);
    }
    V[idx] = v;
    W[idx] = w;
  }
}

template <typename T>
__global__ void pade_split_kernel(int n, const T *__restrict__ U, const T *V, T *__restrict__ P,
                                  int ldp, T *Q) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  for (int col = blockIdx.y; col < n; col += gridDim.y) {
    const std::size_t idx = (std::size_t)col * n + row;
    const T u = U[idx];
    const T v = V[idx];  // read before the (possibly aliasing) write of Q
    P[(std::size_t)col * ldp + row] = add(v, u);
    Q[idx] = sub(v, u);
  }
}

template <typename T>
__global__ void scale_copy_kernel(int n, double f, const T *__restrict__ A, int lda,
                                  T *__restrict__ B, int ldb) {
  using R = typename elem<T>::real;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  for (int col = blockIdx.y; col < n; col += gridDim.y) {
    const T a = A[(std::size_t)col * lda + row];
    B[(std::size_t)col * ldb + row] = (f == 1.0) ? a : scale(a, (R)f);
  }
}

__device__ __forceinline__ double cvt(float x, double *) { return (double)x; }
__device__ __forceinline__ float cvt(double x, float *) { return (float)x; }
__device__ __forceinline__ double2 cvt(float2 x, double2 *) { return make_double2(x.x, x.y); }
__device__ __forceinline__ float2 cvt(double2 x, float2 *) { return make_float2((float)x.x, (float)x.y); }

template <typename Ti, typename To>
__global__ void convert_kernel(int n, const Ti *__restrict__ A, int lda, To *__restrict__ B, int ldb) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  for (int col = blockIdx.y; col < n; col += gridDim.y)
    B[(std::size_t)col * ldb + row] = cvt(A[(std::size_t)col * lda + row], (To *)nullptr);
}

template <typename T>
__global__ void ps_build_block_kernel(T *__restrict__ B, int ldb, int n, const T *__restrict__ A,
                                      int lda, const T *__restrict__ powers, std::size_t stride,
                                      const T *__restrict__ c, int terms) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  for (int col = blockIdx.y; col < n; col += gridDim.y) {
    T acc = (row == col) ? c[0] : elem<T>::zero();
    if (terms > 1) acc = fmac(c[1], A[(std::size_t)col * lda + row], acc);
    for (int k = 2; k < terms; ++k)
      acc = fmac(c[k], powers[(std::size_t)(k - 2) * stride + (std::size_t)col * n + row], acc);
    B[(std::size_t)col * ldb + row] = acc;
  }
}

template <typename T>
__global__ void set_scaled_identity_kernel(T *__restrict__ P, int n, int ldp,
                                           const T *__restrict__ alpha) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const T a = *alpha;
  for (int col = blockIdx.y; col < n; col += gridDim.y)
    P[(std::size_t)col * ldp + row] = (row == col) ? a : elem<T>::zero();
}

template <typename T>
__global__ void add_scaled_identity_kernel(T *__restrict__ P, int n, int ldp,
                                           const T *__restrict__ alpha) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const std::size_t at = (std::size_t)i * ((std::size_t)ldp + 1);
  P[at] = add(P[at], *alpha);
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
template <typename T>
cudaError_t launch_norm1(cudaStream_t s, int n, const T *A, int lda, double *d_colsum,
                         double *d_norm) {
  if (n < 1) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(d_norm, 0, sizeof(double), s);
  if (e != cudaSuccess) return e;
  const int warps = 8;
  int blocks = (n + warps - 1) / warps;
  const int cap = 148 * 16;
  if (blocks > cap) blocks = cap;
  norm1_kernel<T><<<blocks, warps * 32, 0, s>>>(n, A, lda, d_colsum,
                                                reinterpret_cast<unsigned long long *>(d_norm));
  return launched();
}

template <typename T, typename R>
cudaError_t launch_colsums_then_max(cudaStream_t s, int n, const T *A, int lda, R *d_colsum) {
  if (n < 1) return cudaSuccess;
  const int warps = 8;
  int blocks = (n + warps - 1) / warps;
  if (blocks > 148 * 16) blocks = 148 * 16;
  colsum_kernel<T, R><<<blocks, warps * 32, 0, s>>>(n, A, lda, d_colsum);
  cudaError_t e = launched();
  if (e != cudaSuccess) return e;
  max_inplace_kernel<R><<<1, 256, 0, s>>>(n, d_colsum);
  return launched();
}

template <typename T>
cudaError_t launch_pade_even_odd(cudaStream_t s, int n, int np, const T *P1, const T *P2,
                                 const T *P3, const T *P4, const double *cv, const double *cw,
                                 T *V, T *W) {
  if (n < 1) return cudaSuccess;
  const dim3 g = grid_2d(n, n);
  switch (np) {
#define CLM_EO(NPV)                                                                             \
  case NPV:                                                                                     \
    pade_even_odd_kernel<T, NPV><<<g, kRowThreads, 0, s>>>(n, P1, P2, P3, P4, cv[0], cv[1],    \
                                                           cv[2], cv[3], cv[4], cw[0], cw[1],  \
                                                           cw[2], cw[3], cw[4], V, W);         \
    break;
    CLM_EO(1)
    CLM_EO(2)
    CLM_EO(3)
    CLM_EO(4)
#undef CLM_EO
  default:
    return cudaErrorInvalidValue;
  }
  return launched();
}

template <typename T>
cudaError_t launch_pade_split(cudaStream_t s, int n, const T *U, const T *V, T *P, int ldp, T *Q) {
  if (n < 1) return cudaSuccess;
  pade_split_kernel<T><<<grid_2d(n, n), kRowThreads, 0, s>>>(n, U, V, P, ldp, Q);
  return launched();
}

template <typename T>
cudaError_t launch_scale_copy(cudaStream_t s, int n, double f, const T *A, int lda, T *B, int ldb) {
  if (n < 1) return cudaSuccess;
  scale_copy_kernel<T><<<grid_2d(n, n), kRowThreads, 0, s>>>(n, f, A, lda, B, ldb);
  return launched();
}

__device__ __forceinline__ float conj_if(float x, bool) { return x; }
__device__ __forceinline__ double conj_if(double x, bool) { return x; }
__device__ __forceinline__ float2 conj_if(float2 x, bool c) { return c ? make_float2(x.x, -x.y) : x; }
__device__ __forceinline__ double2 conj_if(double2 x, bool c) { return c ? make_double2(x.x, -x.y) : x; }

// B (cols x rows) = f A^T or f A^H, through a 32 x 33 shared tile so both the
// read and the write are coalesced.
template <typename T>
__global__ void transpose_kernel(int rows, int cols, double f, const T *__restrict__ A, int lda,
                                 T *__restrict__ B, int ldb, bool conj) {
  using R = typename elem<T>::real;
  __shared__ T tile[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int j = ty; j < 32; j += 8) {
    const int r = r0 + tx, c = c0 + j;
    if (r < rows && c < cols) tile[j][tx] = A[(std::size_t)c * lda + r];
  }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {
    const int c = c0 + tx, r = r0 + j;  // B(c, r) = f op(A(r, c))
    if (r < rows && c < cols) B[(std::size_t)r * ldb + c] = scale(conj_if(tile[tx][j], conj), (R)f);
  }
}

template <typename T>
cudaError_t launch_transpose(cudaStream_t s, int rows, int cols, double f, const T *A, int lda, T *B,
                             int ldb, bool conj) {
  if (rows < 1 || cols < 1) return cudaSuccess;
  // rows, cols <= 46340, so both grid extents stay far below their limits
  transpose_kernel<T><<<dim3((rows + 31) / 32, (cols + 31) / 32), 256, 0, s>>>(rows, cols, f, A, lda, B,
                                                                              ldb, conj);
  return launched();
}

#define CLM_INST_T(T) \
  template cudaError_t launch_transpose<T>(cudaStream_t, int, int, double, const T *, int, T *, int, bool);
CLM_INST_T(float)
CLM_INST_T(double)
CLM_INST_T(float2)
CLM_INST_T(double2)
#undef CLM_INST_T

template <typename Ti, typename To>
cudaError_t launch_convert(cudaStream_t s, int n, const Ti *A, int lda, To *B, int ldb) {
  if (n < 1) return cudaSuccess;
  convert_kernel<Ti, To><<<grid_2d(n, n), kRowThreads, 0, s>>>(n, A, lda, B, ldb);
  return launched();
}
template cudaError_t launch_convert<float, double>(cudaStream_t, int, const float *, int, double *, int);
template cudaError_t launch_convert<double, float>(cudaStream_t, int, const double *, int, float *, int);
template cudaError_t launch_convert<float2, double2>(cudaStream_t, int, const float2 *, int, double2 *, int);
template cudaError_t launch_convert<double2, float2>(cudaStream_t, int, const double2 *, int, float2 *, int);

template <typename T>
cudaError_t launch_ps_build_block(cudaStream_t s, T *B, int ldb, int n, const T *A, int lda,
                                  const T *powers, std::size_t stride, const T *coeffs, int terms) {
  if (n < 1 || terms < 1) return cudaSuccess;
  ps_build_block_kernel<T><<<grid_2d(n, n), kRowThreads, 0, s>>>(B, ldb, n, A, lda, powers, stride,
                                                                  coeffs, terms);
  return launched();
}

template <typename T>
cudaError_t launch_set_scaled_identity(cudaStream_t s, T *P, int n, int ldp, const T *d_alpha) {
  if (n < 1) return cudaSuccess;
  set_scaled_identity_kernel<T><<<grid_2d(n, n), kRowThreads, 0, s>>>(P, n, ldp, d_alpha);
  return launched();
}

template <typename T>
cudaError_t launch_add_scaled_identity(cudaStream_t s, T *P, int n, int ldp, const T *d_alpha) {
  if (n < 1) return cudaSuccess;
  add_scaled_identity_kernel<T><<<(n + 255) / 256, 256, 0, s>>>(P, n, ldp, d_alpha);
  return launched();
}

// ---- explicit instantiations ------------------------------------------------
#define CLM_INST_ALL(T)                                                                          \
  template cudaError_t launch_norm1<T>(cudaStream_t, int, const T *, int, double *, double *);  \
  template cudaError_t launch_pade_even_odd<T>(cudaStream_t, int, int, const T *, const T *,    \
                                               const T *, const T *, const double *,            \
                                               const double *, T *, T *);                       \
  template cudaError_t launch_pade_split<T>(cudaStream_t, int, const T *, const T *, T *, int,  \
                                            T *);                                               \
  template cudaError_t launch_scale_copy<T>(cudaStream_t, int, double, const T *, int, T *, int);
CLM_INST_ALL(float)
CLM_INST_ALL(double)
CLM_INST_ALL(float2)
CLM_INST_ALL(double2)
#undef CLM_INST_ALL

template cudaError_t launch_colsums_then_max<float, float>(cudaStream_t, int, const float *, int, float *);
template cudaError_t launch_colsums_then_max<double, double>(cudaStream_t, int, const double *, int, double *);
template cudaError_t launch_colsums_then_max<float2, float>(cudaStream_t, int, const float2 *, int, float *);
template cudaError_t launch_colsums_then_max<double2, double>(cudaStream_t, int, const double2 *, int, double *);

#define CLM_INST_POLY(T)                                                                         \
  template cudaError_t launch_ps_build_block<T>(cudaStream_t, T *, int, int, const T *, int,    \
                                                const T *, std::size_t, const T *, int);        \
  template cudaError_t launch_set_scaled_identity<T>(cudaStream_t, T *, int, int, const T *);   \
  template cudaError_t launch_add_scaled_identity<T>(cudaStream_t, T *, int, int, const T *);
CLM_INST_POLY(float)
CLM_INST_POLY(double)
#undef CLM_INST_POLY

}  // namespace clm
