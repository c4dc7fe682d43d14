// aodmao2rho_fp64.cuh -- internal launcher of the FP64 masked AO-DM-AO contraction.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cfgmm {

// Device scratch (bytes) the contraction needs for the given problem: the
// per-block active AO lists, their counts and the per-row-tile partial sums.
size_t aodmao2rho_fp64_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk);

// rhos[s*stride_grid+g] += ... (see cfgmm.h) on `stream`; device pointers,
// `workspace` holds aodmao2rho_fp64_workspace(...) bytes, 256-byte aligned.
cudaError_t aodmao2rho_fp64(double* rhos, const double* dms, const double* ao_lhs,
                            const double* ao_rhs, size_t stride_ao, size_t stride_grid, int nao,
                            int ngrid, int nset, const uint8_t* tab, size_t ldtab, int blk,
                            void* workspace, cudaStream_t stream);

// Builds the per-block active AO lists: lists[b*nao + i] = i-th u (ascending)
// with tab[u*ldtab + b] != 0, counts[b] = their number.
cudaError_t aodm_block_lists_launch(const uint8_t* tab, size_t ldtab, int nao, int nblk,
                                    int* lists, int* counts, cudaStream_t stream);

}  // namespace cfgmm
