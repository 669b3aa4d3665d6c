// dmma.cuh -- the FP64 tensor-core tile (mma.sync m16n8k8 .f64) and the
// cp.async helpers that stage its operands; shared by the single-matrix GEMMs
// and the grouped GEMM of the batched tier.
#pragma once

#include "kernels.cuh"

namespace clm {
namespace {

// ---- cp.async helpers -------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// 16-byte copy with zero fill past src_bytes (0, 8 or 16)
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D = A B + D on a 16x8x8 FP64 tile. Fragment ownership (g = lane>>2,
// t = lane&3): A a0=(g,t) a1=(g+8,t) a2=(g,t+4) a3=(g+8,t+4); B b0=(t,g)
// b1=(t+4,g); C c0=(g,2t) c1=(g,2t+1) c2=(g+8,2t) c3=(g+8,2t+1).
__device__ __forceinline__ void dmma16x8x8(double (&d)[4], const double (&a)[4],
                                           const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

}  // namespace
}  // namespace clm
