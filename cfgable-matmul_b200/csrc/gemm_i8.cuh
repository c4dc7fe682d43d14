// gemm_i8.cuh -- internal interface of the batched INT8 tcgen05 GEMM with a
// modular-residue epilogue (gemm_i8.cu).
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace cfgmm {

constexpr int kMaxModuli = 16;

struct GemmI8Args {
  int rows_a;      // rows of each A plane (M)
  int rows_b;      // rows of each B plane (N)
  int k;           // contraction length (<= 65536: exact INT32 sums)
  int nmod;        // number of planes / moduli
  int8_t* out;     // residues [nmod][rows_a][ldr]
  size_t ldr;      // row stride of `out` (multiple of 16)
  int mod[kMaxModuli];
  float inv[kMaxModuli];
};

// Tile geometry (A rows per tile, B rows per tile, K bytes per stage).
int gemm_i8_tile_rows_a();
int gemm_i8_tile_rows_b();
int gemm_i8_k_block();

// tmA / tmB: 3-D tensor maps over INT8 planes (K, rows, nmod), 128-byte
// swizzle, boxes (128, 128, 1) and (128, 256, 1).
cudaError_t gemm_i8_mod(const CUtensorMap& tmA, const CUtensorMap& tmB, const GemmI8Args& args,
                        cudaStream_t stream);

// Sticky per-device error word of the kernel (0 = ok; else the code of the
// wait that timed out).  reset enqueues a clear; read is synchronous.
cudaError_t gemm_i8_reset_error(cudaStream_t stream);
cudaError_t gemm_i8_read_error(int* code);

}  // namespace cfgmm
