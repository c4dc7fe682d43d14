// dgemm_fp64.cuh -- internal launcher of the FP64 tensor-core DGEMM.
#pragma once
#include <cuda_runtime.h>

namespace cfgmm {

// C[i*ldc+j] += sum_p opA(i,p) opB(p,j) on `stream`; device pointers.
cudaError_t dgemm_fp64(double* c, const double* a, const double* b, int m, int n, int k,
                       size_t lda, size_t ldb, size_t ldc, bool transa, bool transb,
                       cudaStream_t stream);

}  // namespace cfgmm
