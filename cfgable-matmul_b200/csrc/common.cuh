// common.cuh -- small device helpers shared by the kernels of libcfgmm.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace cfgmm {

// 8-byte asynchronous global->shared copy.  When `valid` is false nothing is
// read from `src` (src-size 0) and the 8 destination bytes are zero-filled.
__device__ __forceinline__ void cp_async_8(void* smem_dst, const void* gmem_src, bool valid) {
  const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  const int src_size = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(gmem_src),
               "r"(src_size)
               : "memory");
}

// 16-byte asynchronous copy (L2 only), zero-filled when `valid` is false.
__device__ __forceinline__ void cp_async_16(void* smem_dst, const void* gmem_src, bool valid) {
  const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  const int src_size = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(gmem_src),
               "r"(src_size)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// FP64 tensor-core MMA, D(16x8) += A(16x4) * B(4x8), row.col fragments:
//   lane = 4*g + q:  a0 = A[g][q], a1 = A[g+8][q], b0 = B[q][g],
//   d0,d1 = D[g][2q, 2q+1], d2,d3 = D[g+8][2q, 2q+1].
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// FP64 tensor-core MMA, D(16x8) += A(16x8) * B(8x8), row.col fragments:
//   a0 = A[g][q], a1 = A[g+8][q], a2 = A[g][q+4], a3 = A[g+8][q+4],
//   b0 = B[q][g], b1 = B[q+4][g], d as in dmma_16x8x4.
__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], double a0, double a1, double a2,
                                            double a3, double b0, double b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// Offset (in doubles) of element (row, col) of a shared-memory tile whose rows
// hold `kRowDoubles` doubles (a multiple of 16), with the 16-byte chunks of
// each row XOR-swizzled.  A 16-byte fragment load of a warp (lane = 4g + q
// reads row r0 + g, chunk c0 + q, r0 % 8 == 0) is served in four phases of 8
// lanes = rows {2p, 2p+1}; the XOR key ((r&1)<<2 | (r>>1)&3) sends those two
// rows to disjoint halves of the 8 bank groups, so every phase is one
// conflict-free wavefront.
__device__ __forceinline__ int swz_key(int row) { return ((row & 1) << 2) | ((row >> 1) & 3); }

template <int kRowDoubles>
__device__ __forceinline__ int swz(int row, int col) {
  return row * kRowDoubles + (((col >> 1) ^ swz_key(row)) << 1) + (col & 1);
}

}  // namespace cfgmm
