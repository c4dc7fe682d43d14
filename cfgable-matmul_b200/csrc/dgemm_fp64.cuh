// dgemm_fp64.cuh -- internal launcher of the FP64 tensor-core DGEMM.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cfgmm {

// C[i*ldc+j] += sum_p opA(i,p) opB(p,j) on `stream`; device pointers.
cudaError_t dgemm_fp64(double* c, const double* a, const double* b, int m, int n, int k,
                       size_t lda, size_t ldb, size_t ldc, bool transa, bool transb,
                       cudaStream_t stream);

// Masked GEMM (src/impl_matmul_non0tab.rs:210-306): B is not transposed;
// element (p, j) of B takes part only when tab[p * ldtab + j / blk] != 0.
cudaError_t dgemm_fp64_non0tab(double* c, const double* a, const double* b, int m, int n, int k,
                               size_t lda, size_t ldb, size_t ldc, bool transa,
                               const uint8_t* tab, size_t ldtab, int blk, cudaStream_t stream);

// Fock-build contraction of one density set on `stream`: V[u*ldv + v] +=
// sum over g with tab[u][g/blk] and tab[v][g/blk] of ao_lhs[u][g] w[g]
// ao_rhs[v][g].  `workspace` holds fock_fp64_workspace(nao, ngrid) bytes,
// 256-byte aligned; pack_rhs = false reuses the right operand and activity map
// left there by a previous call with the same ao_rhs and mask.
size_t fock_fp64_workspace(int nao, int ngrid);
cudaError_t fock_fp64(double* v, size_t ldv, const double* w, const double* ao_lhs,
                      const double* ao_rhs, size_t stride_grid, int nao, int ngrid,
                      const uint8_t* tab, size_t ldtab, int blk, bool pack_rhs, void* workspace,
                      cudaStream_t stream);

// Sticky error word of the TMA form's bounded waits (0 = none).
cudaError_t dgemm_reset_error(cudaStream_t stream);
cudaError_t dgemm_read_error(int* code);

}  // namespace cfgmm
