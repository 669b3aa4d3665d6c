// lu.cu -- LU with partial pivoting (xGETRF semantics) and the n-right-hand-
// side solve (xGETRS, no transpose) for the Pade denominator q_m(A), written
// for sm_100a without cuSOLVER (the reference reaches cuSOLVER through
// WarpWraps: src/expm/pade.cppm:186-188).
//
// Blocked right-looking factorisation, panel width kb <= 64:
//   1. panel: one thread-block CLUSTER (<= 8 CTAs) holds the h x kb panel in
//      the CTAs' shared memory, rows split across the CTAs. Each column costs
//      one cluster barrier: every CTA publishes its local pivot candidate (and
//      that candidate's whole row) into a double-buffered slot, the barrier
//      makes the slots visible, and every CTA then reads all candidates over
//      distributed shared memory, agrees on the global pivot (largest
//      |Re|+|Im|, first index on ties -- LAPACK IxAMAX), swaps, scales and
//      applies the rank-1 update to its own rows.
//   2. swap + TRSM: one warp per column outside the panel applies the panel's
//      row permutation (a compact gather of <= 2 kb rows) and, right of the
//      panel, solves with the unit-lower L11 in registers.
//   3. trailing update: A22 -= L21 U12 on the tensor-core GEMM.
// The solve gathers the right-hand side through the accumulated row
// permutation and runs blocked forward / backward substitution (diagonal
// blocks per warp, off-diagonal blocks on the GEMM).
#include <cooperative_groups.h>
#include <climits>

#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace clm {

namespace {

constexpr int kMaxKb = 64;
constexpr int kPanelThreads = 512;
constexpr int kMaxCluster = 8;
constexpr std::size_t kPanelSmemBudget = 180 * 1024;  // bytes of panel per CTA

// scratch: ipiv[n] | perm[n] | map_pos[2*kMaxKb] | map_src[2*kMaxKb] | map_count
struct LuScratch {
  int *ipiv, *perm, *map_pos, *map_src, *map_count;
};
inline LuScratch carve_lu(void *base, int n) {
  Layout L(base);
  LuScratch s;
  s.ipiv = L.take<int>(n);
  s.perm = L.take<int>(n);
  s.map_pos = L.take<int>(2 * kMaxKb);
  s.map_src = L.take<int>(2 * kMaxKb);
  s.map_count = L.take<int>(1);
  return s;
}

__host__ __device__ inline std::size_t align16(std::size_t x) { return (x + 15) & ~std::size_t(15); }

// Offsets of the panel kernel's shared-memory regions (host and device agree).
struct PanelSmem {
  std::size_t S, slot_row, slot_diag, pivrow, oldrow, slot_val, slot_idx, red_val, red_idx, plist,
      scal, map_pos, map_org, total;
};
template <typename T>
__host__ __device__ inline PanelSmem panel_smem(int rpc, int kb) {
  PanelSmem o;
  std::size_t at = 0;
  o.S = at; at = align16(at + sizeof(T) * (std::size_t)rpc * kb);
  o.slot_row = at; at = align16(at + sizeof(T) * 2 * kb);
  o.slot_diag = at; at = align16(at + sizeof(T) * 2 * kb);
  o.pivrow = at; at = align16(at + sizeof(T) * kb);
  o.oldrow = at; at = align16(at + sizeof(T) * kb);
  o.slot_val = at; at = align16(at + sizeof(double) * 2);
  o.slot_idx = at; at = align16(at + sizeof(int) * 2);
  o.red_val = at; at = align16(at + sizeof(double) * (kPanelThreads / 32));
  o.red_idx = at; at = align16(at + sizeof(int) * (kPanelThreads / 32));
  o.plist = at; at = align16(at + sizeof(int) * kb);
  o.scal = at; at = align16(at + sizeof(double) * 4);
  o.map_pos = at; at = align16(at + sizeof(int) * 2 * kb);
  o.map_org = at; at = align16(at + sizeof(int) * 2 * kb);
  o.total = at;
  return o;
}

template <typename T> __device__ __forceinline__ T shfl(T v, int src);
template <> __device__ __forceinline__ float shfl<float>(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <> __device__ __forceinline__ double shfl<double>(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <> __device__ __forceinline__ float2 shfl<float2>(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
template <> __device__ __forceinline__ double2 shfl<double2>(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// (value, index) max with the first index winning ties
__device__ __forceinline__ void argmax_merge(double &v, int &i, double ov, int oi) {
  if (ov > v || (ov == v && oi < i)) {
    v = ov;
    i = oi;
  }
}

template <typename T>
__global__ void __launch_bounds__(kPanelThreads)
    lu_panel_kernel(int n, T *__restrict__ A, int lda, int k, int kb, int rpc, int *__restrict__ ipiv,
                    int *__restrict__ perm, int *__restrict__ g_map_pos, int *__restrict__ g_map_src,
                    int *__restrict__ g_map_count, int *__restrict__ info) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int ncta = (int)cluster.num_blocks();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int h = n - k;
  const int r0 = rank * rpc;
  int rows_here = h - r0;
  rows_here = rows_here < 0 ? 0 : (rows_here > rpc ? rpc : rows_here);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const PanelSmem o = panel_smem<T>(rpc, kb);
  T *S = reinterpret_cast<T *>(smem_raw + o.S);
  T *slot_row = reinterpret_cast<T *>(smem_raw + o.slot_row);
  T *slot_diag = reinterpret_cast<T *>(smem_raw + o.slot_diag);
  T *pivrow = reinterpret_cast<T *>(smem_raw + o.pivrow);
  T *oldrow = reinterpret_cast<T *>(smem_raw + o.oldrow);
  double *slot_val = reinterpret_cast<double *>(smem_raw + o.slot_val);
  int *slot_idx = reinterpret_cast<int *>(smem_raw + o.slot_idx);
  double *red_val = reinterpret_cast<double *>(smem_raw + o.red_val);
  int *red_idx = reinterpret_cast<int *>(smem_raw + o.red_idx);
  int *plist = reinterpret_cast<int *>(smem_raw + o.plist);
  double *scal = reinterpret_cast<double *>(smem_raw + o.scal);
  int *spiv = reinterpret_cast<int *>(scal + 2);  // [0] = p, [1] = first zero pivot

  // ---- stage the panel rows this CTA owns ----
  for (int idx = tid; idx < rows_here * kb; idx += kPanelThreads) {
    const int li = idx % rows_here, c = idx / rows_here;
    S[(std::size_t)c * rpc + li] = A[(std::size_t)(k + c) * lda + (k + r0 + li)];
  }
  if (tid == 0) spiv[1] = -1;
  __syncthreads();

  for (int j = 0; j < kb; ++j) {
    const int par = j & 1;
    // ---- local pivot candidate over rows >= j ----
    double bv = -1.0;
    int bi = INT_MAX;
    for (int li = tid; li < rows_here; li += kPanelThreads) {
      const int gi = r0 + li;
      if (gi >= j) argmax_merge(bv, bi, abs1(S[(std::size_t)j * rpc + li]), gi);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      argmax_merge(bv, bi, ov, oi);
    }
    if (lane == 0) {
      red_val[warp] = bv;
      red_idx[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
      bv = lane < kPanelThreads / 32 ? red_val[lane] : -1.0;
      bi = lane < kPanelThreads / 32 ? red_idx[lane] : INT_MAX;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        argmax_merge(bv, bi, ov, oi);
      }
      if (lane == 0) {
        slot_val[par] = bv;
        slot_idx[par] = bi;
      }
    }
    __syncthreads();
    // ---- publish the candidate's row and, if owned here, row j ----
    if (tid < kb) {
      const int cand = slot_idx[par];
      if (cand != INT_MAX) slot_row[par * kb + tid] = S[(std::size_t)tid * rpc + (cand - r0)];
      if (j >= r0 && j < r0 + rows_here) slot_diag[par * kb + tid] = S[(std::size_t)tid * rpc + (j - r0)];
    }
    cluster.sync();

    // ---- agree on the global pivot ----
    if (warp == 0) {
      double v = -1.0;
      int i = INT_MAX;
      if (lane < ncta) {
        v = cluster.map_shared_rank(slot_val, lane)[par];
        i = cluster.map_shared_rank(slot_idx, lane)[par];
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i, off);
        argmax_merge(v, i, ov, oi);
      }
      if (lane == 0) {
        spiv[0] = i;
        scal[0] = v;
      }
    }
    __syncthreads();
    const int p = spiv[0];
    const int owner_p = p / rpc, owner_j = j / rpc;
    if (tid < kb) {
      pivrow[tid] = cluster.map_shared_rank(slot_row, owner_p)[par * kb + tid];
      if (rank == owner_p && p != j)
        oldrow[tid] = cluster.map_shared_rank(slot_diag, owner_j)[par * kb + tid];
    }
    __syncthreads();
    if (tid < kb) {
      if (rank == owner_j) S[(std::size_t)tid * rpc + (j - r0)] = pivrow[tid];
      if (rank == owner_p && p != j) S[(std::size_t)tid * rpc + (p - r0)] = oldrow[tid];
    }
    if (tid == 0) {
      plist[j] = p;
      if (scal[0] == 0.0 && spiv[1] < 0) spiv[1] = j;
    }
    __syncthreads();
    // ---- scale the column below the pivot ----
    const T piv = pivrow[j];
    if (!is_zero(piv)) {
      for (int li = tid; li < rows_here; li += kPanelThreads)
        if (r0 + li > j) S[(std::size_t)j * rpc + li] = divide(S[(std::size_t)j * rpc + li], piv);
    }
    __syncthreads();
    // ---- rank-1 update of the columns right of j, rows below j ----
    const int w = kb - j - 1;
    if (w > 0 && rows_here > 0) {
      const int total = rows_here * w;
      for (int idx = tid; idx < total; idx += kPanelThreads) {
        const int li = idx % rows_here;
        const int c = j + 1 + idx / rows_here;
        if (r0 + li > j) {
          T &x = S[(std::size_t)c * rpc + li];
          x = sub(x, mul(S[(std::size_t)j * rpc + li], pivrow[c]));
        }
      }
    }
    __syncthreads();
  }

  // ---- write the factored panel back ----
  for (int idx = tid; idx < rows_here * kb; idx += kPanelThreads) {
    const int li = idx % rows_here, c = idx / rows_here;
    A[(std::size_t)(k + c) * lda + (k + r0 + li)] = S[(std::size_t)c * rpc + li];
  }

  if (rank != 0) {
    cluster.sync();  // keep every CTA's shared memory alive until rank 0 is done reading
    return;
  }
  if (tid < kb) ipiv[k + tid] = k + plist[tid];
  if (tid == 0 && spiv[1] >= 0 && info[0] == 0) info[0] = k + spiv[1] + 1;

  // ---- compact row map of the panel's swaps (warp 0 of rank 0) ----
  // entries 0..kb-1 are rows k..k+kb-1 in order; extra rows the swaps reached
  // are appended. After replaying the swaps, row pos[e] holds old row org[e].
  int *mpos = reinterpret_cast<int *>(smem_raw + o.map_pos);
  int *morg = reinterpret_cast<int *>(smem_raw + o.map_org);
  if (warp == 0) {
    for (int e = lane; e < kb; e += 32) {
      mpos[e] = k + e;
      morg[e] = k + e;
    }
    __syncwarp();
    int count = kb;
    for (int j = 0; j < kb; ++j) {
      const int b = plist[j];
      int bidx;
      if (b < kb) {
        bidx = b;
      } else {
        bidx = -1;
        for (int base = kb; base < count; base += 32) {
          const int e = base + lane;
          const unsigned hit = __ballot_sync(0xffffffffu, e < count && mpos[e] == k + b);
          if (hit) {
            bidx = base + __ffs(hit) - 1;
            break;
          }
        }
        if (bidx < 0) {
          bidx = count;
          if (lane == 0) {
            mpos[count] = k + b;
            morg[count] = k + b;
          }
          ++count;
        }
      }
      __syncwarp();
      if (lane == 0 && bidx != j) {
        const int t = morg[j];
        morg[j] = morg[bidx];
        morg[bidx] = t;
      }
      __syncwarp();
    }
    int pv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = lane + 32 * q;
      if (e < count) {
        g_map_pos[e] = mpos[e];
        g_map_src[e] = morg[e];
        pv[q] = perm[morg[e]];
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = lane + 32 * q;
      if (e < count) perm[mpos[e]] = pv[q];
    }
    if (lane == 0) *g_map_count = count;
  }
  cluster.sync();
}

// ---- swap + TRSM for the columns outside the panel: one warp per column ----
template <typename T>
__global__ void __launch_bounds__(256)
    lu_swap_trsm_kernel(int n, T *__restrict__ A, int lda, int k, int kb,
                        const int *__restrict__ map_pos, const int *__restrict__ map_src,
                        const int *__restrict__ map_count) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *L = reinterpret_cast<T *>(smem_raw);  // kb x kb, column-major
  const int warps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  const int ci = blockIdx.x * warps + (threadIdx.x >> 5);
  const bool block_needs_L = (int)(blockIdx.x + 1) * warps > k;  // holds a right-of-panel column
  if (block_needs_L) {
    for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x)
      L[idx] = A[(std::size_t)(k + idx / kb) * lda + (k + idx % kb)];
  }
  __syncthreads();
  if (ci >= n - kb) return;
  const int c = ci < k ? ci : ci + kb;
  T *col = A + (std::size_t)c * lda;
  const int cnt = *map_count;
  T v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = lane + 32 * q;
    v[q] = e < cnt ? col[map_src[e]] : elem<T>::zero();
  }
  __syncwarp();
  if (c < k) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = lane + 32 * q;
      if (e < cnt) col[map_pos[e]] = v[q];
    }
    return;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = lane + 32 * q;
    if (e >= kb && e < cnt) col[map_pos[e]] = v[q];
  }
  T x0 = v[0], x1 = v[1];  // rows k+lane, k+lane+32
  for (int l = 0; l < kb; ++l) {
    const T xl = shfl(l < 32 ? x0 : x1, l & 31);
    if (lane > l && lane < kb) x0 = sub(x0, mul(L[l * kb + lane], xl));
    if (lane + 32 > l && lane + 32 < kb) x1 = sub(x1, mul(L[l * kb + lane + 32], xl));
  }
  if (lane < kb) col[k + lane] = x0;
  if (lane + 32 < kb) col[k + lane + 32] = x1;
}

__global__ void iota_kernel(int n, int *p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}

// X(i, c) = B(perm[i], c)
template <typename T>
__global__ void gather_rows_kernel(int n, int nrhs, const int *__restrict__ perm,
                                   const T *__restrict__ B, int ldb, T *__restrict__ X, int ldx) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int src = perm[row];
  for (int c = blockIdx.y; c < nrhs; c += gridDim.y)
    X[(std::size_t)c * ldx + row] = B[(std::size_t)c * ldb + src];
}

// Diagonal-block triangular solve on rows [k, k+kb) of X, one warp per RHS
// column. LOWER: unit lower (forward); else non-unit upper (backward).
template <typename T, bool LOWER>
__global__ void __launch_bounds__(256)
    trsm_diag_kernel(int nrhs, const T *__restrict__ LU, int lda, int k, int kb, T *__restrict__ X,
                     int ldx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *D = reinterpret_cast<T *>(smem_raw);
  for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x)
    D[idx] = LU[(std::size_t)(k + idx / kb) * lda + (k + idx % kb)];
  __syncthreads();
  const int warps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * warps + (threadIdx.x >> 5);
  if (c >= nrhs) return;
  T *col = X + (std::size_t)c * ldx + k;
  T x0 = lane < kb ? col[lane] : elem<T>::zero();
  T x1 = lane + 32 < kb ? col[lane + 32] : elem<T>::zero();
  if (LOWER) {
    for (int l = 0; l < kb; ++l) {
      const T xl = shfl(l < 32 ? x0 : x1, l & 31);
      if (lane > l && lane < kb) x0 = sub(x0, mul(D[l * kb + lane], xl));
      if (lane + 32 > l && lane + 32 < kb) x1 = sub(x1, mul(D[l * kb + lane + 32], xl));
    }
  } else {
    for (int l = kb - 1; l >= 0; --l) {
      if (l < 32) {
        if (lane == l) x0 = divide(x0, D[l * kb + l]);
      } else {
        if (lane + 32 == l) x1 = divide(x1, D[l * kb + l]);
      }
      const T xl = shfl(l < 32 ? x0 : x1, l & 31);
      if (lane < l) x0 = sub(x0, mul(D[l * kb + lane], xl));
      if (lane + 32 < l) x1 = sub(x1, mul(D[l * kb + lane + 32], xl));
    }
  }
  if (lane < kb) col[lane] = x0;
  if (lane + 32 < kb) col[lane + 32] = x1;
}

// Panel width for an n x n factorisation: the widest kb <= 64 whose full-height
// panel fits in kMaxCluster CTAs' shared memory.
template <typename T>
int choose_kb(int n) {
  int kb = kMaxKb;
  while (kb > 1 && (std::size_t)n * kb * sizeof(T) > kPanelSmemBudget * kMaxCluster) kb /= 2;
  return kb;
}

template <typename T>
cudaError_t launch_panel(cudaStream_t s, int n, T *A, int lda, int k, int kb, const LuScratch &sc,
                         int *info) {
  const int h = n - k;
  int ncta = (int)(((std::size_t)h * kb * sizeof(T) + kPanelSmemBudget - 1) / kPanelSmemBudget);
  if (ncta < 1) ncta = 1;
  if (ncta > kMaxCluster) ncta = kMaxCluster;
  if (ncta > h) ncta = h;
  const int rpc = (h + ncta - 1) / ncta;
  const PanelSmem o = panel_smem<T>(rpc, kb);
  auto kern = lu_panel_kernel<T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o.total);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ncta, 1, 1);
  cfg.blockDim = dim3(kPanelThreads, 1, 1);
  cfg.dynamicSmemBytes = o.total;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ncta;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, kern, n, A, lda, k, kb, rpc, sc.ipiv, sc.perm, sc.map_pos,
                            sc.map_src, sc.map_count, info);
}

}  // namespace

std::size_t lu_scratch_bytes(int n) {
  Layout L(nullptr);
  L.take<int>(n < 1 ? 1 : n);  // ipiv
  L.take<int>(n < 1 ? 1 : n);  // perm
  L.take<int>(2 * kMaxKb);     // map_pos
  L.take<int>(2 * kMaxKb);     // map_src
  L.take<int>(1);              // map_count
  return L.used;
}

template <typename T>
cudaError_t getrf(cudaStream_t s, int n, T *A, int lda, void *scratch, int *info_dev) {
  if (n < 1) return cudaSuccess;
  const LuScratch sc = carve_lu(scratch, n);
  cudaError_t e = cudaMemsetAsync(info_dev, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  iota_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, sc.perm);
  if ((e = launched()) != cudaSuccess) return e;
  const int kbn = choose_kb<T>(n);
  for (int k = 0; k < n; k += kbn) {
    const int kb = (k + kbn < n) ? kbn : n - k;
    if ((e = launch_panel<T>(s, n, A, lda, k, kb, sc, info_dev)) != cudaSuccess) return e;
    const int others = n - kb;
    if (others > 0) {
      const int warps = 8;
      const std::size_t smem = sizeof(T) * (std::size_t)kb * kb;
      auto kern = lu_swap_trsm_kernel<T>;
      if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
      kern<<<(others + warps - 1) / warps, warps * 32, smem, s>>>(n, A, lda, k, kb, sc.map_pos,
                                                                 sc.map_src, sc.map_count);
      if ((e = launched()) != cudaSuccess) return e;
    }
    const int rest = n - (k + kb);
    if (rest > 0) {
      e = gemm_nn<T>(s, rest, rest, kb, -1.0, A + (std::size_t)k * lda + (k + kb), lda,
                     A + (std::size_t)(k + kb) * lda + k, lda, 1.0,
                     A + (std::size_t)(k + kb) * lda + (k + kb), lda);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

template <typename T>
cudaError_t getrs(cudaStream_t s, int n, int nrhs, const T *LU, int lda, const void *scratch,
                  const T *B, int ldb, T *X, int ldx, int *info_dev) {
  if (n < 1 || nrhs < 1) return cudaSuccess;
  const LuScratch sc = carve_lu(const_cast<void *>(scratch), n);
  cudaError_t e = cudaMemsetAsync(info_dev, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  {
    const int gy = nrhs < 65535 ? nrhs : 65535;
    gather_rows_kernel<T><<<dim3((n + 255) / 256, gy), 256, 0, s>>>(n, nrhs, sc.perm, B, ldb, X, ldx);
    if ((e = launched()) != cudaSuccess) return e;
  }
  constexpr int NB = 64;
  const int warps = 8;
  const std::size_t smem = sizeof(T) * NB * NB;
  auto kl = trsm_diag_kernel<T, true>;
  auto ku = trsm_diag_kernel<T, false>;
  if ((e = cudaFuncSetAttribute(kl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(ku, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) return e;
  const int blocks = (nrhs + warps - 1) / warps;
  for (int k = 0; k < n; k += NB) {
    const int kb = (k + NB < n) ? NB : n - k;
    kl<<<blocks, warps * 32, sizeof(T) * kb * kb, s>>>(nrhs, LU, lda, k, kb, X, ldx);
    if ((e = launched()) != cudaSuccess) return e;
    if (k + kb < n) {
      e = gemm_nn<T>(s, n - (k + kb), nrhs, kb, -1.0, LU + (std::size_t)k * lda + (k + kb), lda,
                     X + k, ldx, 1.0, X + (k + kb), ldx);
      if (e != cudaSuccess) return e;
    }
  }
  const int last = ((n - 1) / NB) * NB;
  for (int k = last; k >= 0; k -= NB) {
    const int kb = (k + NB < n) ? NB : n - k;
    ku<<<blocks, warps * 32, sizeof(T) * kb * kb, s>>>(nrhs, LU, lda, k, kb, X, ldx);
    if ((e = launched()) != cudaSuccess) return e;
    if (k > 0) {
      e = gemm_nn<T>(s, k, nrhs, kb, -1.0, LU + (std::size_t)k * lda, lda, X + k, ldx, 1.0, X, ldx);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

#define CLM_INST_LU(T)                                                                            \
  template cudaError_t getrf<T>(cudaStream_t, int, T *, int, void *, int *);                     \
  template cudaError_t getrs<T>(cudaStream_t, int, int, const T *, int, const void *, const T *, \
                                int, T *, int, int *);
CLM_INST_LU(float)
CLM_INST_LU(double)
CLM_INST_LU(float2)
CLM_INST_LU(double2)
#undef CLM_INST_LU

}  // namespace clm
