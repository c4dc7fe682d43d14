// aodmao2rho_split.cuh -- internal launcher of the split-precision (INT8
// tcgen05, slice-form Ozaki) masked AO-DM-AO contraction.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cfgmm {

// Device scratch (bytes) of the split contraction: active lists, work list,
// D digits (8 bytes per element of D), phi digit tiles, partial sums.
size_t aodmao2rho_split_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk);

// Same contract as aodmao2rho_fp64; nao <= 16384 keeps the INT32 level sums exact.
cudaError_t aodmao2rho_split(double* rhos, const double* dms, const double* ao_lhs,
                             const double* ao_rhs, size_t stride_ao, size_t stride_grid, int nao,
                             int ngrid, int nset, const uint8_t* tab, size_t ldtab, int blk,
                             void* workspace, cudaStream_t stream);

// Sticky per-device error word of the split kernel's bounded waits.
cudaError_t aodmao2rho_split_reset_error(cudaStream_t stream);
cudaError_t aodmao2rho_split_read_error(int* code);

}  // namespace cfgmm
