// lu.cu -- LU with partial pivoting (xGETRF semantics) and the n-right-hand-
// side solve (xGETRS, no transpose) for the Pade denominator q_m(A), written
// for sm_100a without cuSOLVER (the reference reaches cuSOLVER through
// WarpWraps: src/expm/pade.cppm:186-188).
//
// Blocked right-looking factorisation, panel width kb <= 64:
//   1. panel: one thread-block CLUSTER (<= 8 CTAs) holds the h x kb panel in
//      the CTAs' shared memory, rows split across the CTAs. Per pivot column:
//        - every CTA reduces its local pivot candidate (largest |Re|+|Im|,
//          first index on ties -- LAPACK IxAMAX) and publishes it, with the
//          candidate's whole row, into a double-buffered slot;
//        - ONE cluster barrier;
//        - every CTA fetches all candidates and their rows (and row j) over
//          distributed shared memory in a single round trip, and agrees on
//          the pivot without further communication;
//        - one fused pass swaps, scales by the pivot's reciprocal (as xGETF2
//          does above the safe minimum), applies the rank-1 update to its own
//          rows and already forms the NEXT column's local candidate.
//      That is two CTA barriers and one cluster barrier per column.
//   2. swap + TRSM: one warp per column outside the panel applies the panel's
//      row permutation (a compact gather of <= 2 kb rows) and, right of the
//      panel, solves with the unit-lower L11 held in shared memory.
//   3. trailing update: A22 -= L21 U12 on the tensor-core GEMM.
// The solve gathers the right-hand side through the accumulated row
// permutation and runs blocked forward / backward substitution (diagonal
// blocks per warp, off-diagonal blocks on the GEMM).
#include <cooperative_groups.h>
#include <cfloat>
#include <climits>
#include <type_traits>

#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace clm {

namespace {

constexpr int kMaxKb = 64;
constexpr int kPanelThreads = 512;
constexpr int kMaxCluster = 8;
constexpr std::size_t kPanelSmemBudget = 176 * 1024;  // bytes of panel per CTA

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
  std::size_t S, slot_row, slot_diag, cand, oldrow, slot_rcp, cand_rcp, slot_val, slot_idx,
      cand_val, cand_idx, red_val, red_idx, plist, flags, map_pos, map_org, total;
};
template <typename T>
__host__ __device__ inline PanelSmem panel_smem(int rpc, int kb) {
  PanelSmem o;
  std::size_t at = 0;
  o.S = at; at = align16(at + sizeof(T) * (std::size_t)rpc * kb);
  o.slot_row = at; at = align16(at + sizeof(T) * 2 * kb);
  o.slot_diag = at; at = align16(at + sizeof(T) * 2 * kb);
  o.cand = at; at = align16(at + sizeof(T) * kMaxCluster * kb);
  o.oldrow = at; at = align16(at + sizeof(T) * kb);
  o.slot_rcp = at; at = align16(at + sizeof(T) * 2);
  o.cand_rcp = at; at = align16(at + sizeof(T) * kMaxCluster);
  o.slot_val = at; at = align16(at + sizeof(double) * 2);
  o.slot_idx = at; at = align16(at + sizeof(int) * 2);
  o.cand_val = at; at = align16(at + sizeof(double) * kMaxCluster);
  o.cand_idx = at; at = align16(at + sizeof(int) * kMaxCluster);
  o.red_val = at; at = align16(at + sizeof(double) * (kPanelThreads / 32));
  o.red_idx = at; at = align16(at + sizeof(int) * (kPanelThreads / 32));
  o.plist = at; at = align16(at + sizeof(int) * kb);
  o.flags = at; at = align16(at + sizeof(int) * 4);
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

// one element global -> shared, asynchronously (4, 8 or 16 bytes)
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (sizeof(T) == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
  } else if constexpr (sizeof(T) == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
  }
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::);
}

template <typename T> __device__ __forceinline__ double safe_min();
template <> __device__ __forceinline__ double safe_min<float>() { return FLT_MIN; }
template <> __device__ __forceinline__ double safe_min<double>() { return DBL_MIN; }
template <> __device__ __forceinline__ double safe_min<float2>() { return FLT_MIN; }
template <> __device__ __forceinline__ double safe_min<double2>() { return DBL_MIN; }

__device__ __noinline__ void panel_finish(cg::cluster_group &cluster, int rank, int k, int kb,
                                          const int *plist, const int *flags, int *mpos, int *morg,
                                          int *__restrict__ ipiv, int *__restrict__ perm,
                                          int *__restrict__ g_map_pos, int *__restrict__ g_map_src,
                                          int *__restrict__ g_map_count, int *__restrict__ info);

template <typename T>
__global__ void __launch_bounds__(kPanelThreads)
    lu_panel_kernel(int n, T *__restrict__ A, int lda, int k, int kb, int rpc, int *__restrict__ ipiv,
                    int *__restrict__ perm, int *__restrict__ g_map_pos, int *__restrict__ g_map_src,
                    int *__restrict__ g_map_count, int *__restrict__ info) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int ncta = (int)cluster.num_blocks();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nt = blockDim.x;  // a multiple of 32, at most kPanelThreads
  const int h = n - k;
  const int r0 = rank * rpc;
  int rows_here = h - r0;
  rows_here = rows_here < 0 ? 0 : (rows_here > rpc ? rpc : rows_here);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const PanelSmem o = panel_smem<T>(rpc, kb);
  T *S = reinterpret_cast<T *>(smem_raw + o.S);
  T *slot_row = reinterpret_cast<T *>(smem_raw + o.slot_row);
  T *slot_diag = reinterpret_cast<T *>(smem_raw + o.slot_diag);
  T *cand = reinterpret_cast<T *>(smem_raw + o.cand);
  T *oldrow = reinterpret_cast<T *>(smem_raw + o.oldrow);
  double *slot_val = reinterpret_cast<double *>(smem_raw + o.slot_val);
  int *slot_idx = reinterpret_cast<int *>(smem_raw + o.slot_idx);
  double *cand_val = reinterpret_cast<double *>(smem_raw + o.cand_val);
  int *cand_idx = reinterpret_cast<int *>(smem_raw + o.cand_idx);
  double *red_val = reinterpret_cast<double *>(smem_raw + o.red_val);
  int *red_idx = reinterpret_cast<int *>(smem_raw + o.red_idx);
  int *plist = reinterpret_cast<int *>(smem_raw + o.plist);
  int *flags = reinterpret_cast<int *>(smem_raw + o.flags);  // [0] first zero pivot

  // Work split of the fused pass: ncph adjacent lanes share a row, each taking
  // every ncph-th column, so a row's readers of column j sit in one warp and a
  // __syncwarp orders them before column j is overwritten.
  int ncph = 1;
  while (ncph * 2 <= 32 && ncph * 2 * rpc <= nt) ncph *= 2;
  const int RT = nt / ncph;  // rows covered per sweep
  const int my_c = tid % ncph, my_r = tid / ncph;
  const int iters = (rpc + RT - 1) / RT;  // uniform across the CTA

  // ---- stage the panel rows this CTA owns (all copies in flight at once) ----
  for (int idx = tid; idx < rows_here * kb; idx += nt) {
    const int li = idx % rows_here, c = idx / rows_here;
    cp_async_elem(&S[(std::size_t)c * rpc + li], &A[(std::size_t)(k + c) * lda + (k + r0 + li)]);
  }
  cp_async_wait_all();
  if (tid == 0) flags[0] = -1;
  __syncthreads();

  // local candidate for column 0 (the lane whose phase owns column 0)
  double bv = -1.0;
  int bi = INT_MAX;
  if (my_c == 0)
    for (int li = my_r; li < rows_here; li += RT) argmax_merge(bv, bi, abs1(S[li]), r0 + li);

  for (int j = 0; j < kb; ++j) {
    const int par = j & 1;
    const int owner_j = j / rpc;
    // ---- (1) CTA-wide candidate, published with its row ----
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
      double v = lane < nt / 32 ? red_val[lane] : -1.0;
      int i = lane < nt / 32 ? red_idx[lane] : INT_MAX;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i, off);
        argmax_merge(v, i, ov, oi);
      }
      if (lane == 0) {
        slot_val[par] = v;
        slot_idx[par] = i;
      }
      for (int c = lane; c < kb; c += 32) {
        if (i != INT_MAX) slot_row[par * kb + c] = S[(std::size_t)c * rpc + (i - r0)];
        if (rank == owner_j) slot_diag[par * kb + c] = S[(std::size_t)c * rpc + (j - r0)];
      }
    }
    cluster.sync();

    // ---- (2) one DSMEM round trip: every candidate, its row, and row j ----
    for (int t = tid; t < ncta * kb + kb + ncta; t += nt) {
      if (t < ncta * kb) {
        const int q = t / kb, c = t % kb;
        cand[q * kb + c] = cluster.map_shared_rank(slot_row, q)[par * kb + c];
      } else if (t < ncta * kb + kb) {
        const int c = t - ncta * kb;
        oldrow[c] = cluster.map_shared_rank(slot_diag, owner_j)[par * kb + c];
      } else {
        const int q = t - ncta * kb - kb;
        cand_val[q] = cluster.map_shared_rank(slot_val, q)[par];
        cand_idx[q] = cluster.map_shared_rank(slot_idx, q)[par];
      }
    }
    __syncthreads();

    // ---- (3) the pivot, agreed by every warp from the same data ----
    double pv = lane < ncta ? cand_val[lane] : -1.0;
    int p = lane < ncta ? cand_idx[lane] : INT_MAX;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {  // full butterfly: every lane ends with the winner
      const double ov = __shfl_xor_sync(0xffffffffu, pv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, p, off);
      argmax_merge(pv, p, ov, oi);
    }
    if (p == INT_MAX || p < j) {  // no comparable candidate (NaN column): keep row j
      p = j;
      pv = 0.0;
    }
    const T *pivrow = (p == j) ? oldrow : cand + (p / rpc) * kb;
    const T piv = pivrow[j];
    const bool singular = is_zero(piv);
    const bool use_recip = abs1(piv) >= safe_min<T>();
    const T rpiv = (use_recip && !singular) ? divide(elem<T>::one(), piv) : elem<T>::one();
    auto scale_by_pivot = [&](T x) -> T {
      return singular ? x : (use_recip ? mul(x, rpiv) : divide(x, piv));
    };
    if (tid == 0) {
      plist[j] = p;
      if (pv == 0.0 && flags[0] < 0) flags[0] = j;
    }

    // ---- (4a) the two rows that move, one element per thread: position j
    //      receives the pivot row, position p the old row j (updated) ----
    bv = -1.0;
    bi = INT_MAX;
    const int nextc = j + 1;
    const bool own_j = rank == owner_j;
    const bool own_p = p != j && rank == p / rpc;
    for (int t = tid; t < 2 * kb; t += nt) {
      if (t < kb) {
        if (own_j) S[(std::size_t)t * rpc + (j - r0)] = pivrow[t];
      } else if (own_p) {
        const int c = t - kb;
        const T lp = scale_by_pivot(oldrow[j]);
        T v;
        if (c < j) v = oldrow[c];
        else if (c == j) v = lp;
        else v = sub(oldrow[c], mul(lp, pivrow[c]));
        S[(std::size_t)c * rpc + (p - r0)] = v;
        if (c == nextc) argmax_merge(bv, bi, abs1(v), p);
      }
    }

    // ---- (4b) every other row below j: scale, rank-1 update, next candidate ----
    for (int it = 0; it < iters; ++it) {
      const int li = my_r + it * RT;
      const int gi = r0 + li;
      const bool row_ok = li < rows_here && gi > j && gi != p;
      T xj = elem<T>::zero();
      if (row_ok) xj = S[(std::size_t)j * rpc + li];
      __syncwarp();  // every lane of this row has read column j
      if (!row_ok) continue;
      T *row = S + li;
      const T l = scale_by_pivot(xj);
      // first column >= j in this lane's phase (ncph is a power of two)
      int c = j + ((my_c - j) & (ncph - 1));
      if (c == j) {
        row[(std::size_t)j * rpc] = l;
        c += ncph;
      }
      // four columns at a time, all loads issued before the stores
      for (; c < kb; c += 4 * ncph) {
        T x[4], pr[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int cc = c + u * ncph;
          if (cc < kb) {
            x[u] = row[(std::size_t)cc * rpc];
            pr[u] = pivrow[cc];
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int cc = c + u * ncph;
          if (cc < kb) row[(std::size_t)cc * rpc] = sub(x[u], mul(l, pr[u]));
        }
      }
      // this lane's share of the next column's candidate
      if (nextc < kb && ((nextc - my_c) & (ncph - 1)) == 0)
        argmax_merge(bv, bi, abs1(row[(std::size_t)nextc * rpc]), gi);
    }
  }

  // ---- write the factored panel back ----
  __syncthreads();
  for (int idx = tid; idx < rows_here * kb; idx += nt) {
    const int li = idx % rows_here, c = idx / rows_here;
    A[(std::size_t)(k + c) * lda + (k + r0 + li)] = S[(std::size_t)c * rpc + li];
  }

  panel_finish(cluster, rank, k, kb, plist, flags, reinterpret_cast<int *>(smem_raw + o.map_pos),
               reinterpret_cast<int *>(smem_raw + o.map_org), ipiv, perm, g_map_pos, g_map_src,
               g_map_count, info);
}

// Epilogue shared by both panel kernels: the pivot vector, LAPACK's info, the
// compact row map the swap kernel replays, and the accumulated permutation.
// Ends with the cluster barrier that keeps every CTA's shared memory alive
// until the last remote read of it has completed.
__device__ __noinline__ void panel_finish(cg::cluster_group &cluster, int rank, int k, int kb,
                                          const int *plist, const int *flags, int *mpos, int *morg,
                                          int *__restrict__ ipiv, int *__restrict__ perm,
                                          int *__restrict__ g_map_pos, int *__restrict__ g_map_src,
                                          int *__restrict__ g_map_count, int *__restrict__ info) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (rank != 0) {
    cluster.sync();
    return;
  }
  if (tid < kb) ipiv[k + tid] = k + plist[tid];
  if (tid == 0 && flags[0] >= 0 && info[0] == 0) info[0] = k + flags[0] + 1;

  // ---- compact row map of the panel's swaps (warp 0 of rank 0) ----
  // entries 0..kb-1 are rows k..k+kb-1 in order; extra rows the swaps reached
  // are appended. After replaying the swaps, row pos[e] holds old row org[e].
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

// ---------------------------------------------------------------------------
// Register-resident panel: the algorithm of lu_panel_kernel with each row of
// the panel held in the registers of NCPH adjacent lanes (lane phase q keeps
// columns q, q + NCPH, ...), so the rank-1 update costs no shared-memory
// traffic; only the pivot row is broadcast from shared memory. The CTA whose
// candidate wins already publishes the pivot's reciprocal with the row, so
// the division is done once, by one thread, while the row is being copied.
// Used when the rows of a CTA fit its NT / NCPH lanes.
// ---------------------------------------------------------------------------
template <typename T, int KB, int NCPH, int NT>
__global__ void __launch_bounds__(NT)
    lu_panel_reg_kernel(int n, T *__restrict__ A, int lda, int k, int kb, int rpc,
                        int *__restrict__ ipiv, int *__restrict__ perm, int *__restrict__ g_map_pos,
                        int *__restrict__ g_map_src, int *__restrict__ g_map_count,
                        int *__restrict__ info) {
  constexpr int CPL = KB / NCPH;  // columns per lane
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int ncta = (int)cluster.num_blocks();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int h = n - k;
  const int r0 = rank * rpc;
  int rows_here = h - r0;
  rows_here = rows_here < 0 ? 0 : (rows_here > rpc ? rpc : rows_here);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const PanelSmem o = panel_smem<T>(0, KB);
  T *slot_row = reinterpret_cast<T *>(smem_raw + o.slot_row);    // [2][KB]
  T *slot_diag = reinterpret_cast<T *>(smem_raw + o.slot_diag);  // [2][KB]
  T *cand = reinterpret_cast<T *>(smem_raw + o.cand);            // [kMaxCluster][KB]
  T *oldrow = reinterpret_cast<T *>(smem_raw + o.oldrow);
  T *slot_rcp = reinterpret_cast<T *>(smem_raw + o.slot_rcp);
  T *cand_rcp = reinterpret_cast<T *>(smem_raw + o.cand_rcp);
  double *slot_val = reinterpret_cast<double *>(smem_raw + o.slot_val);
  int *slot_idx = reinterpret_cast<int *>(smem_raw + o.slot_idx);
  double *cand_val = reinterpret_cast<double *>(smem_raw + o.cand_val);
  int *cand_idx = reinterpret_cast<int *>(smem_raw + o.cand_idx);
  double *red_val = reinterpret_cast<double *>(smem_raw + o.red_val);
  int *red_idx = reinterpret_cast<int *>(smem_raw + o.red_idx);
  int *plist = reinterpret_cast<int *>(smem_raw + o.plist);
  int *flags = reinterpret_cast<int *>(smem_raw + o.flags);

  const int phase = tid % NCPH;
  const int li = tid / NCPH;  // this lane's row within the CTA
  const bool has_row = li < rows_here;
  const int gi = r0 + li;     // panel-relative row
  const int group0 = lane & ~(NCPH - 1);

  // ---- stage: this lane's columns of its row ----
  T r[CPL];
#pragma unroll
  for (int u = 0; u < CPL; ++u) {
    const int c = phase + u * NCPH;
    r[u] = (has_row && c < kb) ? A[(std::size_t)(k + c) * lda + (k + gi)] : elem<T>::zero();
  }
  if (tid == 0) flags[0] = -1;

  // candidate for column 0: the phase-0 lane of every row
  double bv = -1.0;
  int bi = INT_MAX;
  if (has_row && phase == 0) argmax_merge(bv, bi, abs1(r[0]), gi);

  for (int j = 0; j < kb; ++j) {
    const int par = j & 1;
    const int owner_j = j / rpc;
    const int jphase = j % NCPH, ju = j / NCPH;
    // ---- (1) CTA-wide candidate; the lanes holding it publish its row ----
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
    double cv = lane < nwarps ? red_val[lane] : -1.0;
    int ci = lane < nwarps ? red_idx[lane] : INT_MAX;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, cv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, ci, off);
      argmax_merge(cv, ci, ov, oi);
    }
    if (tid == 0) {
      slot_val[par] = cv;
      slot_idx[par] = ci;
    }
    if (has_row && (gi == ci || gi == j)) {
#pragma unroll
      for (int u = 0; u < CPL; ++u) {
        const int c = phase + u * NCPH;
        if (c < kb) {
          if (gi == ci) slot_row[par * KB + c] = r[u];
          if (gi == j) slot_diag[par * KB + c] = r[u];
        }
      }
      if (gi == ci && phase == jphase) {  // one division per column, off the other lanes' path
        T x = elem<T>::zero();
#pragma unroll
        for (int u = 0; u < CPL; ++u)
          if (u == ju) x = r[u];
        slot_rcp[par] = is_zero(x) ? elem<T>::one() : divide(elem<T>::one(), x);
      }
    }
    cluster.sync();

    // ---- (2) one DSMEM round trip: every candidate, its row, and row j ----
    for (int t = tid; t < (kMaxCluster + 1) * KB + kMaxCluster; t += blockDim.x) {
      if (t < kMaxCluster * KB) {
        const int q = t / KB, c = t % KB;  // KB is a power of two
        if (q < ncta && c < kb) cand[q * KB + c] = cluster.map_shared_rank(slot_row, q)[par * KB + c];
      } else if (t < (kMaxCluster + 1) * KB) {
        const int c = t - kMaxCluster * KB;
        if (c < kb) oldrow[c] = cluster.map_shared_rank(slot_diag, owner_j)[par * KB + c];
      } else {
        const int q = t - (kMaxCluster + 1) * KB;
        if (q < ncta) {
          cand_val[q] = cluster.map_shared_rank(slot_val, q)[par];
          cand_idx[q] = cluster.map_shared_rank(slot_idx, q)[par];
          cand_rcp[q] = cluster.map_shared_rank(slot_rcp, q)[par];
        }
      }
    }
    __syncthreads();

    // ---- (3) the pivot ----
    double pv = lane < ncta ? cand_val[lane] : -1.0;
    int p = lane < ncta ? cand_idx[lane] : INT_MAX;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, pv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, p, off);
      argmax_merge(pv, p, ov, oi);
    }
    bool forced = false;
    if (p == INT_MAX || p < j) {  // no comparable candidate (NaN column): keep row j
      p = j;
      pv = 0.0;
      forced = true;
    }
    const int powner = p / rpc;
    const T *pivrow = (p == j) ? oldrow : cand + powner * KB;
    const T piv = pivrow[j];
    const bool singular = forced || is_zero(piv);
    const bool use_recip = abs1(piv) >= safe_min<T>();
    const T rpiv = cand_rcp[powner];
    if (tid == 0) {
      plist[j] = p;
      if (pv == 0.0 && flags[0] < 0) flags[0] = j;
    }

    // ---- (4) swap, scale, rank-1 update, next candidate: all in registers ----
    T xj_mine = elem<T>::zero();
#pragma unroll
    for (int u = 0; u < CPL; ++u)
      if (u == ju) xj_mine = r[u];
    T xj = shfl(xj_mine, group0 + jphase);
    bv = -1.0;
    bi = INT_MAX;
    if (has_row && gi >= j) {
      if (gi == j) {  // position j receives the pivot row
#pragma unroll
        for (int u = 0; u < CPL; ++u) {
          const int c = phase + u * NCPH;
          if (c < kb) r[u] = pivrow[c];
        }
      } else {
        if (gi == p) {  // position p receives the old row j
          xj = oldrow[j];
#pragma unroll
          for (int u = 0; u < CPL; ++u) {
            const int c = phase + u * NCPH;
            if (c < kb) r[u] = oldrow[c];
          }
        }
        const T l = singular ? xj : (use_recip ? mul(xj, rpiv) : divide(xj, piv));
#pragma unroll
        for (int u = 0; u < CPL; ++u) {
          const int c = phase + u * NCPH;
          if (c == j) r[u] = l;
          else if (c > j && c < kb) r[u] = sub(r[u], mul(l, pivrow[c]));
        }
        if (j + 1 < kb && phase == (j + 1) % NCPH) {
          const int nu = (j + 1) / NCPH;
          T xn = elem<T>::zero();
#pragma unroll
          for (int u = 0; u < CPL; ++u)
            if (u == nu) xn = r[u];
          argmax_merge(bv, bi, abs1(xn), gi);
        }
      }
    }
  }

  // ---- write the factored panel back ----
#pragma unroll
  for (int u = 0; u < CPL; ++u) {
    const int c = phase + u * NCPH;
    if (has_row && c < kb) A[(std::size_t)(k + c) * lda + (k + gi)] = r[u];
  }
  __syncthreads();
  panel_finish(cluster, rank, k, kb, plist, flags, reinterpret_cast<int *>(smem_raw + o.map_pos),
               reinterpret_cast<int *>(smem_raw + o.map_org), ipiv, perm, g_map_pos, g_map_src,
               g_map_count, info);
}

// Load the kb x kb diagonal block A[k:k+kb, k:k+kb] into shared memory (D[l kb + i]
// = A(k + i, k + l)): a warp per column, 16-byte copies when every column of
// the block starts 16-byte aligned, else one element per copy. (The per-element
// form with an index division per element set the time of the 128-row float32
// solve blocks: 16k copies per CTA.)
template <typename T>
__device__ __forceinline__ void load_diag_block(T *D, const T *A, int lda, int k, int kb) {
  constexpr int V = 16 / sizeof(T);  // elements per 16-byte copy
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  const T *base = A + (std::size_t)k * lda + k;
  if (V > 1 && kb % V == 0 && lda % V == 0 && (reinterpret_cast<std::uintptr_t>(base) & 15) == 0) {
    for (int l = threadIdx.x >> 5; l < kb; l += warps)
      for (int i = lane * V; i < kb; i += 32 * V) {
        const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(&D[l * kb + i]));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(&base[(std::size_t)l * lda + i]));
      }
  } else {
    for (int l = threadIdx.x >> 5; l < kb; l += warps)
      for (int i = lane; i < kb; i += 32) cp_async_elem(&D[l * kb + i], &base[(std::size_t)l * lda + i]);
  }
  cp_async_wait_all();
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
  if (block_needs_L) load_diag_block(L, A, lda, k, kb);
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

// The same solve for a full block (kb = 32 VPL): the steps run in runs of 32
// whose pivot rows sit in one register of every lane (x[vo]), so the lane
// selection and most bound checks are static; each row still takes the
// updates in the same order, so the results are those of the general kernel.
template <typename T, bool LOWER, int VPL>
__global__ void __launch_bounds__(256)
    trsm_diag_full_kernel(int nrhs, const T *__restrict__ LU, int lda, int k, T *__restrict__ X, int ldx) {
  constexpr int kb = 32 * VPL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *D = reinterpret_cast<T *>(smem_raw);
  T *rdiag = D + kb * kb;
  load_diag_block(D, LU, lda, k, kb);
  __syncthreads();
  if (!LOWER && threadIdx.x < kb) {
    const T d = D[threadIdx.x * kb + threadIdx.x];
    rdiag[threadIdx.x] = divide(elem<T>::one(), d);
  }
  __syncthreads();
  const int warps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * warps + (threadIdx.x >> 5);
  if (c >= nrhs) return;
  T *col = X + (std::size_t)c * ldx + k;
  T x[VPL];
#pragma unroll
  for (int v = 0; v < VPL; ++v) x[v] = col[lane + 32 * v];
  if (LOWER) {
#pragma unroll
    for (int vo = 0; vo < VPL; ++vo) {
#pragma unroll 4
      for (int ll = 0; ll < 32; ++ll) {
        const int l = 32 * vo + ll;
        const T xl = shfl(x[vo], ll);
        if (lane > ll) x[vo] = sub(x[vo], mul(D[l * kb + lane + 32 * vo], xl));
#pragma unroll
        for (int v = vo + 1; v < VPL; ++v) x[v] = sub(x[v], mul(D[l * kb + lane + 32 * v], xl));
      }
    }
  } else {
#pragma unroll
    for (int vo = VPL - 1; vo >= 0; --vo) {
#pragma unroll 4
      for (int ll = 31; ll >= 0; --ll) {
        const int l = 32 * vo + ll;
        const T xl = mul(shfl(x[vo], ll), rdiag[l]);
        if (lane == ll) x[vo] = xl;
        if (lane < ll) x[vo] = sub(x[vo], mul(D[l * kb + lane + 32 * vo], xl));
#pragma unroll
        for (int v = 0; v < vo; ++v) x[v] = sub(x[v], mul(D[l * kb + lane + 32 * v], xl));
      }
    }
  }
#pragma unroll
  for (int v = 0; v < VPL; ++v) col[lane + 32 * v] = x[v];
}

// Diagonal-block triangular solve on rows [k, k+kb) of X (kb <= 32 VPL), one
// warp per RHS column, lane l keeping rows l, l + 32, ... LOWER: unit lower
// (forward); else non-unit upper (backward), whose diagonal reciprocals are
// formed once per block, off the dependent chain.
template <typename T, bool LOWER, int VPL>
__global__ void __launch_bounds__(256)
    trsm_diag_kernel(int nrhs, const T *__restrict__ LU, int lda, int k, int kb, T *__restrict__ X,
                     int ldx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *D = reinterpret_cast<T *>(smem_raw);
  T *rdiag = D + kb * kb;
  load_diag_block(D, LU, lda, k, kb);
  __syncthreads();
  if (!LOWER && threadIdx.x < kb) {
    const T d = D[threadIdx.x * kb + threadIdx.x];
    rdiag[threadIdx.x] = divide(elem<T>::one(), d);
  }
  __syncthreads();
  const int warps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * warps + (threadIdx.x >> 5);
  if (c >= nrhs) return;
  T *col = X + (std::size_t)c * ldx + k;
  T x[VPL];
#pragma unroll
  for (int v = 0; v < VPL; ++v) x[v] = lane + 32 * v < kb ? col[lane + 32 * v] : elem<T>::zero();
  if (LOWER) {
    for (int l = 0; l < kb; ++l) {
      T src = x[0];
#pragma unroll
      for (int v = 1; v < VPL; ++v)
        if ((l >> 5) == v) src = x[v];
      const T xl = shfl(src, l & 31);
#pragma unroll
      for (int v = 0; v < VPL; ++v)
        if (lane + 32 * v > l && lane + 32 * v < kb) x[v] = sub(x[v], mul(D[l * kb + lane + 32 * v], xl));
    }
  } else {
    for (int l = kb - 1; l >= 0; --l) {
      T src = x[0];
#pragma unroll
      for (int v = 1; v < VPL; ++v)
        if ((l >> 5) == v) src = x[v];
      const T xl = mul(shfl(src, l & 31), rdiag[l]);
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        if (lane + 32 * v == l) x[v] = xl;
        if (lane + 32 * v < l) x[v] = sub(x[v], mul(D[l * kb + lane + 32 * v], xl));
      }
    }
  }
#pragma unroll
  for (int v = 0; v < VPL; ++v)
    if (lane + 32 * v < kb) col[lane + 32 * v] = x[v];
}

// ---------------------------------------------------------------------------
// One-CTA panel, two levels: the h x kb panel (kb <= 64) stays in global
// memory (L2) and is factored in sub-panels of KBS columns; a sub-panel's rows
// live in registers (thread t keeps rows t, t + NT, ... -- RPT of them), so a
// pivot column costs one CTA-wide argmax and one or two barriers, with no cluster
// barrier and no distributed shared memory. After each sub-panel the CTA
// applies its swaps to the panel's other columns, solves the sub-panel's
// U12 rows with the unit-lower L11, and updates the rest of the panel.
// ---------------------------------------------------------------------------
constexpr int kCtaChunk = 8;  // columns per register chunk of the in-panel update

template <typename T>
__device__ __forceinline__ void lds_vec8(const T *src, T (&dst)[kCtaChunk]) {
  // 8 consecutive elements as 16-byte shared loads (src 16-byte aligned)
  union {
    float4 v[kCtaChunk * sizeof(T) / 16];
    T e[kCtaChunk];
  } u;
  const float4 *s4 = reinterpret_cast<const float4 *>(src);
#pragma unroll
  for (int i = 0; i < (int)(kCtaChunk * sizeof(T) / 16); ++i) u.v[i] = s4[i];
#pragma unroll
  for (int i = 0; i < kCtaChunk; ++i) dst[i] = u.e[i];
}

// kRotate: the rotating-register column loop (measured faster for complex128
// and float32 panels: C2 +3 %, C3 +4 %); otherwise the fully unrolled one
// (faster for float64: the wider sub-panels make the rotation and the masked
// update cost more than the smaller code saves).
template <typename T> constexpr bool panel_rotates() {
  return std::is_same<T, double2>::value || std::is_same<T, float>::value;
}

// One pivot step's search and row exchange. The pivot is the largest
// |Re| + |Im| of column col among rows >= a, first index on ties; the owner of
// row a publishes that row into slot kRowA (after the warps' slots). kOneBarrier: every warp's winner
// publishes its whole row into the warp's slot before the single barrier, and
// after it every thread agrees on the pivot p and reads the pivot row from its
// slot (the caller alternates buffers by step: a slot is rewritten two steps
// later, after every reader has passed the intervening barrier). Otherwise the
// CTA argmax (one barrier) comes first and the pivot's owner alone publishes
// its row into slot 0 before a second barrier; measured faster with one row
// per thread (float64, 256 rows: 2.5 %), slower with two or more. Returns the
// slot of the pivot row. forced: no comparable candidate (NaN column), p = a.
template <typename T, int KBS, int RPT, bool kOneBarrier, int kRowA>
__device__ __forceinline__ int panel_pivot(const T (&r)[RPT][KBS], int col, int a, int h, T (*wrow)[KBS],
                                           unsigned long long *red_key, int *red_idx, int &p, bool &forced,
                                           double &pv) {
  const int tid = threadIdx.x, NT = blockDim.x;
  double bv = -1.0;
  int bi = INT_MAX;
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int gi = tid + q * NT;
    if (gi >= a && gi < h) argmax_merge(bv, bi, abs1(r[q][col]), gi);
  }
  if constexpr (kOneBarrier) {
    const int lane = tid & 31, warp = tid >> 5;
    const ArgMax wa = warp_argmax(argmax_key(bv, bi, bi != INT_MAX));
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int gi = tid + q * NT;
      if (gi == a) {
#pragma unroll
        for (int c = 0; c < KBS; ++c) wrow[kRowA][c] = r[q][c];
      }
      if (gi == wa.idx) {
#pragma unroll
        for (int c = 0; c < KBS; ++c) wrow[warp][c] = r[q][c];
      }
    }
    if (lane == 0) {
      red_key[warp] = wa.key;
      red_idx[warp] = wa.idx;
    }
    __syncthreads();
    int wp;
    const ArgMax am = cta_argmax_collect_at(red_key, red_idx, wp);
    pv = __longlong_as_double((long long)am.key);
    p = am.idx;
    forced = false;
    if (p >= h || p < a) {
      p = a;
      pv = 0.0;
      forced = true;
    }
    return forced ? kRowA : wp;
  } else {
    const ArgMax am = cta_argmax(argmax_key(bv, bi, bi != INT_MAX), red_key, red_idx);
    pv = __longlong_as_double((long long)am.key);
    p = am.idx;
    forced = false;
    if (p >= h || p < a) {
      p = a;
      pv = 0.0;
      forced = true;
    }
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int gi = tid + q * NT;
      if (gi == a) {
#pragma unroll
        for (int c = 0; c < KBS; ++c) wrow[kRowA][c] = r[q][c];
      }
      if (gi == p) {
#pragma unroll
        for (int c = 0; c < KBS; ++c) wrow[0][c] = r[q][c];
      }
    }
    __syncthreads();
    return 0;
  }
}

template <typename T, int KBS, int RPT, int MAXT = 512, bool kRotate = panel_rotates<T>()>
__global__ void __launch_bounds__(MAXT, 1)
    lu_panel_cta_kernel(int n, T *__restrict__ A, int lda, int k, int kb, int *__restrict__ ipiv,
                        int *__restrict__ perm, int *__restrict__ g_map_pos, int *__restrict__ g_map_src,
                        int *__restrict__ g_map_count, int *__restrict__ info) {
  cg::cluster_group cluster = cg::this_cluster();  // launched as a cluster of one
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NT = blockDim.x, nwarps = NT >> 5;
  const int h = n - k;
  T *P = A + (std::size_t)k * lda + k;  // the panel: P[c * lda + i], i < h, c < kb
  // per pivot step, alternating: slots 0..kW-1 each warp winner's row, slot
  // kW row a before the exchange
  constexpr int kW = MAXT / 32;  // warps at most (MAXT threads)
  __shared__ __align__(16) T wrow[2][kW + 1][KBS];
  __shared__ T l11[KBS][KBS + 1];
  __shared__ __align__(16) T u12[KBS][kMaxKb];
  __shared__ unsigned long long red_key[2][kW];
  __shared__ int red_idx[2][kW];
  __shared__ int plist[kMaxKb];
  __shared__ int flags[1];
  __shared__ int mpos[2 * kMaxKb], morg[2 * kMaxKb];
  __shared__ int src_top[KBS], disp_row[KBS], disp_src[KBS], ndisp[1];

  if (tid == 0) flags[0] = -1;
  T r[RPT][KBS];
  for (int sb = 0; sb < kb; sb += KBS) {
    const int w = min(KBS, kb - sb);
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int gi = tid + q * NT;
#pragma unroll
      for (int c = 0; c < KBS; ++c)
        r[q][c] = (gi >= sb && gi < h && c < w) ? P[(std::size_t)(sb + c) * lda + gi] : elem<T>::zero();
    }
    if constexpr (kRotate) {
    // ---- factor the sub-panel, one pivot column at a time. Each row's
    // registers rotate one place left after every step, so the pivot column
    // is always r[q][0] and every step runs the same (rolled) code with
    // static register indices; finished columns ride at the back of the row
    // (still swapped with it) and the update is masked to the unfinished
    // positions. After KBS steps (idle ones past w) the row is back in
    // column order. ----
#pragma unroll 1
    for (int j = 0; j < KBS; ++j) {
      if (j < w) {
        const int a = sb + j, buf = j & 1;
        int p;
        bool forced;
        double pv;
        const int ps = panel_pivot<T, KBS, RPT, (RPT > 1), kW>(r, 0, a, h, wrow[buf], red_key[buf], red_idx[buf], p, forced, pv);
        const T *prow = wrow[buf][ps];
        if (tid == 0) {
          plist[a] = p;
          if (pv == 0.0 && flags[0] < 0) flags[0] = a;
        }
        const T piv = prow[0];
        const bool singular = forced || is_zero(piv);
        const bool use_recip = abs1(piv) >= safe_min<T>();
        const T rpiv = singular ? elem<T>::one() : divide(elem<T>::one(), piv);
        const int lim = w - j;  // positions 1 .. lim-1 hold unfinished columns
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
          const int gi = tid + q * NT;
          if (gi < a || gi >= h) continue;
          if (gi == a) {
            if (p != a) {
#pragma unroll
              for (int c = 0; c < KBS; ++c) r[q][c] = prow[c];
            }
            continue;
          }
          if (gi == p) {
#pragma unroll
            for (int c = 0; c < KBS; ++c) r[q][c] = wrow[buf][kW][c];
          }
          const T l = singular ? r[q][0] : (use_recip ? mul(r[q][0], rpiv) : divide(r[q][0], piv));
          r[q][0] = l;
#pragma unroll
          for (int c = 1; c < KBS; ++c)
            if (c < lim) r[q][c] = sub(r[q][c], mul(l, prow[c]));
        }
      }
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const T t0 = r[q][0];
#pragma unroll
        for (int c = 0; c + 1 < KBS; ++c) r[q][c] = r[q][c + 1];
        r[q][KBS - 1] = t0;
      }
    }
    } else {
    // ---- factor the sub-panel, one pivot column at a time ----
#pragma unroll
    for (int j = 0; j < KBS; ++j) {
      if (j >= w) break;
      const int a = sb + j, buf = j & 1;
      int p;
      bool forced;
      double pv;
      const int ps = panel_pivot<T, KBS, RPT, (RPT > 1), kW>(r, j, a, h, wrow[buf], red_key[buf], red_idx[buf], p, forced, pv);
      const T *prow = wrow[buf][ps];
      if (tid == 0) {
        plist[a] = p;
        if (pv == 0.0 && flags[0] < 0) flags[0] = a;
      }
      const T piv = prow[j];
      const bool singular = forced || is_zero(piv);
      const bool use_recip = abs1(piv) >= safe_min<T>();
      const T rpiv = singular ? elem<T>::one() : divide(elem<T>::one(), piv);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int gi = tid + q * NT;
        if (gi < a || gi >= h) continue;
        if (gi == a) {
          if (p != a) {
#pragma unroll
            for (int c = 0; c < KBS; ++c) r[q][c] = prow[c];
          }
          continue;
        }
        if (gi == p) {
#pragma unroll
          for (int c = 0; c < KBS; ++c) r[q][c] = wrow[buf][kW][c];
        }
        const T l = singular ? r[q][j] : (use_recip ? mul(r[q][j], rpiv) : divide(r[q][j], piv));
        r[q][j] = l;
#pragma unroll
        for (int c = j + 1; c < KBS; ++c)
          if (c < w) r[q][c] = sub(r[q][c], mul(l, prow[c]));
      }
    }
    }
    // ---- sub-panel back to memory, L11 to shared memory ----
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int gi = tid + q * NT;
      if (gi >= sb && gi < h) {
#pragma unroll
        for (int c = 0; c < KBS; ++c)
          if (c < w) P[(std::size_t)(sb + c) * lda + gi] = r[q][c];
      }
      if (gi >= sb && gi < sb + w) {
#pragma unroll
        for (int c = 0; c < KBS; ++c) l11[gi - sb][c] = r[q][c];
      }
    }
    // ---- where the sub-panel's swaps moved rows: position sb + j now holds
    // old row src_top[j]; a row d below the block holds old top-block row
    // disp_src[e] (rows below only ever receive rows of the top block) ----
    // (every lane follows one final position back through the swaps, in
    // reverse order, to the row it came from)
    if (warp == 0) {
      const int e = lane;
      int x = -1;
      if (e < w) x = sb + e;                                                      // a top-block position
      else if (e < 2 * w && plist[sb + e - w] >= sb + w) x = plist[sb + e - w];  // a displaced row
      if (x >= 0) {
        const int fin = x;
        for (int j = w - 1; j >= 0; --j) {
          const int pj = plist[sb + j];
          if (x == sb + j) x = pj;
          else if (x == pj) x = sb + j;
        }
        if (e < w) src_top[e] = x;
        else {
          disp_row[e - w] = fin;
          disp_src[e - w] = x;
        }
      } else if (e >= w && e < 2 * w) {
        disp_row[e - w] = -1;
      }
      if (lane == 0) ndisp[0] = w;
    }
    __syncthreads();
    // ---- the panel's other columns: swap, and right of the sub-panel solve
    // the top block with L11 (U12 rows into shared memory) ----
    if (tid < kb - w) {
      const int c = tid < sb ? tid : tid + w;
      T *col = P + (std::size_t)c * lda;
      T top[KBS], x[KBS];
#pragma unroll
      for (int j = 0; j < KBS; ++j) top[j] = j < w ? col[sb + j] : elem<T>::zero();
#pragma unroll
      for (int j = 0; j < KBS; ++j) {
        x[j] = elem<T>::zero();
        if (j < w) {
          const int src = src_top[j];
          if (src >= sb + w) x[j] = col[src];
          else {
#pragma unroll
            for (int q = 0; q < KBS; ++q)
              if (q == src - sb) x[j] = top[q];
          }
        }
      }
      for (int e = 0; e < ndisp[0]; ++e) {
        if (disp_row[e] < 0) continue;
        const int srcq = disp_src[e] - sb;
        T v = elem<T>::zero();
#pragma unroll
        for (int q = 0; q < KBS; ++q)
          if (q == srcq) v = top[q];
        col[disp_row[e]] = v;
      }
      if (c >= sb + w) {
#pragma unroll
        for (int j = 1; j < KBS; ++j)
#pragma unroll
          for (int q = 0; q < j; ++q)
            if (j < w) x[j] = sub(x[j], mul(l11[j][q], x[q]));
#pragma unroll
        for (int j = 0; j < KBS; ++j)
          if (j < w) u12[j][c] = x[j];
      }
#pragma unroll
      for (int j = 0; j < KBS; ++j)
        if (j < w) col[sb + j] = x[j];
    }
    __syncthreads();
    // ---- update the rest of the panel: rows below the block, columns right
    // of the sub-panel (the multipliers are reloaded from the written-back
    // sub-panel, so no panel registers stay live through the column phase) ----
    const int c0 = sb + w;
    if (c0 < kb) {
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int gi = tid + q * NT;
        if (gi < c0 || gi >= h) continue;
#pragma unroll
        for (int j = 0; j < KBS; ++j) r[q][j] = j < w ? P[(std::size_t)(sb + j) * lda + gi] : elem<T>::zero();
        for (int c = c0; c < kb; c += kCtaChunk) {
          T v[kCtaChunk];
#pragma unroll
          for (int u = 0; u < kCtaChunk; ++u)
            v[u] = c + u < kb ? P[(std::size_t)(c + u) * lda + gi] : elem<T>::zero();
#pragma unroll
          for (int j = 0; j < KBS; ++j) {
            T b[kCtaChunk];
            lds_vec8(&u12[j][c], b);
#pragma unroll
            for (int u = 0; u < kCtaChunk; ++u) v[u] = sub(v[u], mul(r[q][j], b[u]));
          }
#pragma unroll
          for (int u = 0; u < kCtaChunk; ++u)
            if (c + u < kb) P[(std::size_t)(c + u) * lda + gi] = v[u];
        }
      }
    }
    __syncthreads();
  }
  panel_finish(cluster, 0, k, kb, plist, flags, mpos, morg, ipiv, perm, g_map_pos, g_map_src, g_map_count,
               info);
}

// One-CTA panel configurations by height: RPT rows per thread for heights up
// to 512 RPT (512 threads), sub-panel width KBS (64 registers of sub-panel per
// thread at most), outer panel width KB. Heights 2049..4096 take RPT8 rows per
// thread on NT8 threads: float32 runs 1024 threads of 4 rows there (64
// registers, a few spilled), measured 5 % faster on the float32 4096 expm than
// 512 threads of 8 rows; float64 1024 x 2 rows at heights up to 2048, and
// complex128 1024 x 1 row (sub-panels of 4) at 1024, measured slower. Panels
// of 16 columns for float32, float64 and complex128: with the expm's launches
// replayed as a graph, more and narrower panels cost less than a second
// sub-panel's rest-of-panel update on the one SM (float64 256 expm +15 %,
// complex128 1024 +4 %, float32 4096 +3 %; 8 columns: float32 4096 -20 %).
template <typename T> struct CtaPanel;
template <> struct CtaPanel<double2> {
  static constexpr int KBS1 = 8, KBS2 = 8, KBS4 = 4, KBS8 = 0, RPT8 = 8, NT8 = 512, KB = 16;
};
template <> struct CtaPanel<double> {
  static constexpr int KBS1 = 16, KBS2 = 16, KBS4 = 8, KBS8 = 4, RPT8 = 8, NT8 = 512, KB = 16;
};
template <> struct CtaPanel<float2> {
  static constexpr int KBS1 = 16, KBS2 = 16, KBS4 = 8, KBS8 = 4, RPT8 = 8, NT8 = 512, KB = 32;
};
template <> struct CtaPanel<float> {  // 32 wide: the in-panel SIMT update costs h kb^2 / 2 per panel
  static constexpr int KBS1 = 16, KBS2 = 16, KBS4 = 16, KBS8 = 8, RPT8 = 4, NT8 = 1024, KB = 16;
};

// Panel width of the one-CTA path for an n x n factorisation, 0 if n is too
// tall for it.
template <typename T>
int cta_panel_kb(int n) {
  const int kbs = n <= 512 ? CtaPanel<T>::KBS1 : n <= 1024 ? CtaPanel<T>::KBS2
                : n <= 2048 ? CtaPanel<T>::KBS4 : n <= 4096 ? CtaPanel<T>::KBS8 : 0;
  return kbs > 0 ? CtaPanel<T>::KB : 0;
}

// Register-panel configurations: KB columns, NCPH lanes per row, NT threads
// per CTA (so NT / NCPH rows per CTA). Each lane keeps KB / NCPH elements,
// 64 (RegPanel) or 128 (RegPanelWide, more rows per CTA) 32-bit registers.
template <typename T> struct RegPanel;
template <> struct RegPanel<double2> { static constexpr int KB = 32, NCPH = 4, NT = 512, kRows = NT / NCPH; };
template <> struct RegPanel<double> { static constexpr int KB = 64, NCPH = 4, NT = 512, kRows = NT / NCPH; };
template <> struct RegPanel<float2> { static constexpr int KB = 64, NCPH = 4, NT = 512, kRows = NT / NCPH; };
template <> struct RegPanel<float> { static constexpr int KB = 64, NCPH = 2, NT = 512, kRows = NT / NCPH; };
template <typename T> struct RegPanelWide;
template <> struct RegPanelWide<double2> { static constexpr int KB = 32, NCPH = 1, NT = 256, kRows = NT / NCPH; };
template <> struct RegPanelWide<double> { static constexpr int KB = 64, NCPH = 1, NT = 256, kRows = NT / NCPH; };
template <> struct RegPanelWide<float2> { static constexpr int KB = 64, NCPH = 1, NT = 256, kRows = NT / NCPH; };
template <> struct RegPanelWide<float> { static constexpr int KB = 64, NCPH = 1, NT = 512, kRows = NT / NCPH; };

// Panel width of the outer blocking: complex128 panels are 32 wide so a row's
// register share stays at 64 registers.
template <typename T> constexpr int panel_width() { return RegPanel<T>::KB; }

// Panel width for an n x n factorisation: the widest kb <= 64 whose full-height
// panel fits in kMaxCluster CTAs' shared memory.
template <typename T>
int choose_kb(int n) {
  int kb = panel_width<T>();
  while (kb > 1 && (std::size_t)n * kb * sizeof(T) > kPanelSmemBudget * kMaxCluster) kb /= 2;
  return kb;
}


inline cudaLaunchAttribute cluster_attr(int ncta) {
  cudaLaunchAttribute a;
  a.id = cudaLaunchAttributeClusterDimension;
  a.val.clusterDim.x = ncta;
  a.val.clusterDim.y = 1;
  a.val.clusterDim.z = 1;
  return a;
}

template <typename T, int KB, int NCPH, int NT>
cudaError_t launch_reg_panel(cudaStream_t s, int n, T *A, int lda, int k, int kb, const LuScratch &sc,
                             int *info) {
  constexpr int kRows = NT / NCPH;
  const int h = n - k;
  const int ncta = (h + kRows - 1) / kRows;
  const int rpc = (h + ncta - 1) / ncta;
  const PanelSmem o = panel_smem<T>(0, KB);
  auto kern = lu_panel_reg_kernel<T, KB, NCPH, NT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)o.total);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ncta, 1, 1);
  int nt = ((rpc * NCPH + 31) / 32) * 32;
  if (nt < 64) nt = 64;
  cfg.blockDim = dim3(nt, 1, 1);
  cfg.dynamicSmemBytes = o.total;
  cfg.stream = s;
  cudaLaunchAttribute attr[1] = {cluster_attr(ncta)};
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, kern, n, A, lda, k, kb, rpc, sc.ipiv, sc.perm, sc.map_pos,
                            sc.map_src, sc.map_count, info);
}

template <typename T, int KBS, int RPT, int MAXT = 512>
cudaError_t launch_cta_panel_cfg(cudaStream_t s, int n, T *A, int lda, int k, int kb, const LuScratch &sc,
                                 int *info) {
  const int h = n - k;
  int nt = (h + RPT - 1) / RPT;
  nt = ((nt + 31) / 32) * 32;
  if (nt < 64) nt = 64;  // >= kb - KBS column threads
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(1, 1, 1);
  cfg.blockDim = dim3(nt, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1] = {cluster_attr(1)};
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, lu_panel_cta_kernel<T, KBS, RPT, MAXT>, n, A, lda, k, kb, sc.ipiv, sc.perm,
                            sc.map_pos, sc.map_src, sc.map_count, info);
}

// The one-CTA panel for a step of an n x n factorisation (kb = cta_panel_kb).
template <typename T>
cudaError_t launch_cta_panel(cudaStream_t s, int n, T *A, int lda, int k, int kb, const LuScratch &sc,
                             int *info) {
  using C = CtaPanel<T>;
  if (n <= 512) {
    if constexpr (C::KBS1 > 0) return launch_cta_panel_cfg<T, C::KBS1, 1>(s, n, A, lda, k, kb, sc, info);
  } else if (n <= 1024) {
    if constexpr (C::KBS2 > 0) return launch_cta_panel_cfg<T, C::KBS2, 2>(s, n, A, lda, k, kb, sc, info);
  } else if (n <= 2048) {
    if constexpr (C::KBS4 > 0) return launch_cta_panel_cfg<T, C::KBS4, 4>(s, n, A, lda, k, kb, sc, info);
  } else {
    if constexpr (C::KBS8 > 0)
      return launch_cta_panel_cfg<T, C::KBS8, C::RPT8, C::NT8>(s, n, A, lda, k, kb, sc, info);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_panel(cudaStream_t s, int n, T *A, int lda, int k, int kb, const LuScratch &sc,
                         int *info) {
  const int h = n - k;
  if (kb <= RegPanel<T>::KB && h <= kMaxCluster * RegPanel<T>::kRows) {
    return launch_reg_panel<T, RegPanel<T>::KB, RegPanel<T>::NCPH, RegPanel<T>::NT>(s, n, A, lda, k, kb, sc, info);
  }
  if (kb <= RegPanel<T>::KB && h <= kMaxCluster * RegPanelWide<T>::kRows) {
    return launch_reg_panel<T, RegPanelWide<T>::KB, RegPanelWide<T>::NCPH, RegPanelWide<T>::NT>(s, n, A, lda, k, kb, sc, info);
  }
  // enough CTAs for the panel to fit, and for every row to get >= 2 lanes of
  // the fused pass when the cluster allows it (<= 256 rows per CTA)
  int ncta = (int)(((std::size_t)h * kb * sizeof(T) + kPanelSmemBudget - 1) / kPanelSmemBudget);
  const int by_rows = (h + 255) / 256;
  if (ncta < by_rows) ncta = by_rows;
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
  // threads: enough lanes for every row x column phase, in whole warps
  int ncph = 1;
  while (ncph * 2 <= 32 && ncph * 2 * rpc <= kPanelThreads) ncph *= 2;
  int nt = ((rpc * ncph + 31) / 32) * 32;
  if (nt > kPanelThreads) nt = kPanelThreads;
  if (nt < 64) nt = 64;
  cfg.blockDim = dim3(nt, 1, 1);
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

// Look-ahead resources of the calling host thread on the current device: a
// high-priority auxiliary stream on which the next panel is factored while the
// caller's stream runs the wide trailing update, and the two events that order
// them.
struct LookAhead {
  int device = -1;
  cudaStream_t aux = nullptr;
  cudaEvent_t ready = nullptr, done = nullptr;
};
thread_local LookAhead tl_lookahead;
thread_local bool tl_no_lookahead = false;

cudaError_t lookahead(LookAhead *&out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  LookAhead &la = tl_lookahead;
  if (la.device != dev) {
    if (la.aux) {  // a different device than last time: release the old set
      cudaStreamDestroy(la.aux);
      cudaEventDestroy(la.ready);
      cudaEventDestroy(la.done);
      la = LookAhead{};
    }
    int lo = 0, hi = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&lo, &hi)) != cudaSuccess) return e;
    if ((e = cudaStreamCreateWithPriority(&la.aux, cudaStreamNonBlocking, hi)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&la.ready, cudaEventDisableTiming)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&la.done, cudaEventDisableTiming)) != cudaSuccess) return e;
    la.device = dev;
  }
  out = &la;
  return cudaSuccess;
}

// Blocked right-looking factorisation with a one-panel look-ahead: after the
// swaps and U12 solve of panel k, the next panel's columns are updated first
// (a narrow GEMM); panel k+1 is then factored on the auxiliary stream while
// the caller's stream updates the columns beyond it, and panel k+1's swaps wait
// for both.
template <typename T>
cudaError_t getrf(cudaStream_t s, int n, T *A, int lda, void *scratch, int *info_dev) {
  if (n < 1) return cudaSuccess;
  const LuScratch sc = carve_lu(scratch, n);
  cudaError_t e = cudaMemsetAsync(info_dev, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  iota_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, sc.perm);
  if ((e = launched()) != cudaSuccess) return e;
  const int kb_cta = cta_panel_kb<T>(n);
  const int kbn = kb_cta > 0 ? kb_cta : choose_kb<T>(n);
  auto swap_kern = lu_swap_trsm_kernel<T>;
  const std::size_t swap_smem = sizeof(T) * (std::size_t)kbn * kbn;
  if ((e = cudaFuncSetAttribute(swap_kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)swap_smem)) !=
      cudaSuccess)
    return e;
  // only matrices of more than one panel use the look-ahead stream, and not
  // while a NoLookAheadScope is open on this thread (then every panel runs on s)
  const bool ahead = n > kbn && !tl_no_lookahead;
  LookAhead *la = nullptr;
  if (ahead && (e = lookahead(la)) != cudaSuccess) return e;
  auto panel = [&](cudaStream_t st, int k, int kb) {
    return kb_cta > 0 ? launch_cta_panel<T>(st, n, A, lda, k, kb, sc, info_dev)
                      : launch_panel<T>(st, n, A, lda, k, kb, sc, info_dev);
  };
  if ((e = panel(s, 0, kbn < n ? kbn : n)) != cudaSuccess) return e;
  for (int k = 0; k < n; k += kbn) {
    const int kb = (k + kbn < n) ? kbn : n - k;
    if (ahead && k > 0 && (e = cudaStreamWaitEvent(s, la->done, 0)) != cudaSuccess) return e;  // panel k
    const int others = n - kb;
    if (others > 0) {
      const int warps = 8;
      swap_kern<<<(others + warps - 1) / warps, warps * 32, sizeof(T) * (std::size_t)kb * kb, s>>>(
          n, A, lda, k, kb, sc.map_pos, sc.map_src, sc.map_count);
      if ((e = launched()) != cudaSuccess) return e;
    }
    const int rest = n - (k + kb);
    if (rest > 0) {
      const int kb2 = rest < kbn ? rest : kbn;  // the next panel's width
      const T *L21 = A + (std::size_t)k * lda + (k + kb);
      // next panel's columns first
      e = gemm_nn<T>(s, rest, kb2, kb, -1.0, L21, lda, A + (std::size_t)(k + kb) * lda + k, lda, 1.0,
                     A + (std::size_t)(k + kb) * lda + (k + kb), lda);
      if (e != cudaSuccess) return e;
      if (ahead) {
        if ((e = cudaEventRecord(la->ready, s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(la->aux, la->ready, 0)) != cudaSuccess) return e;
        if ((e = panel(la->aux, k + kb, kb2)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(la->done, la->aux)) != cudaSuccess) return e;
      } else if ((e = panel(s, k + kb, kb2)) != cudaSuccess) {  // disjoint from the wide update
        return e;
      }
      // the wide update, concurrent with that panel
      if (rest > kb2) {
        e = gemm_nn<T>(s, rest, rest - kb2, kb, -1.0, L21, lda, A + (std::size_t)(k + kb + kb2) * lda + k, lda,
                       1.0, A + (std::size_t)(k + kb + kb2) * lda + (k + kb), lda);
        if (e != cudaSuccess) return e;
      }
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
  // Diagonal blocks of 64 rows; float32 systems above 1024 take 128 (half as
  // many passes of the off-diagonal updates over the right-hand side: float32
  // 4096 expm +3 %; float64 2048 measured 8 % slower with 128)
  const bool wide = std::is_same<T, float>::value && n > 1024;
  const int NB = wide ? 128 : 64;
  const int warps = 8;
  const std::size_t smem = sizeof(T) * (NB * NB + NB);
  auto kl = wide ? trsm_diag_kernel<T, true, 4> : trsm_diag_kernel<T, true, 2>;
  auto ku = wide ? trsm_diag_kernel<T, false, 4> : trsm_diag_kernel<T, false, 2>;
  // full blocks (every one but a ragged last) take the static-lane kernel
  auto fl = wide ? trsm_diag_full_kernel<T, true, 4> : trsm_diag_full_kernel<T, true, 2>;
  auto fu = wide ? trsm_diag_full_kernel<T, false, 4> : trsm_diag_full_kernel<T, false, 2>;
  for (auto kern : {kl, ku})
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
      return e;
  for (auto kern : {fl, fu})
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
      return e;
  const int blocks = (nrhs + warps - 1) / warps;
  for (int k = 0; k < n; k += NB) {
    const int kb = (k + NB < n) ? NB : n - k;
    if (kb == NB) fl<<<blocks, warps * 32, sizeof(T) * (kb * kb + kb), s>>>(nrhs, LU, lda, k, X, ldx);
    else kl<<<blocks, warps * 32, sizeof(T) * (kb * kb + kb), s>>>(nrhs, LU, lda, k, kb, X, ldx);
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
    if (kb == NB) fu<<<blocks, warps * 32, sizeof(T) * (kb * kb + kb), s>>>(nrhs, LU, lda, k, X, ldx);
    else ku<<<blocks, warps * 32, sizeof(T) * (kb * kb + kb), s>>>(nrhs, LU, lda, k, kb, X, ldx);
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
