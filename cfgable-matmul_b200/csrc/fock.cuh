// fock.cuh -- the Fock-build contraction on the per-block compacted AO lists.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace cfgmm {

// Device scratch (bytes) of fock_compact_fp64: active lists, work list, counters.
size_t fock_compact_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk);

// vs[s*stride_ao^2 + u*stride_ao + v] += sum over g with tab[u][g/blk] and
// tab[v][g/blk] of ao_lhs[u][g] * ws[s*stride_grid + g] * ao_rhs[v][g], for
// s < nset, on `stream`; device pointers; `workspace` holds
// fock_compact_workspace(...) bytes, 256-byte aligned.
cudaError_t fock_compact_fp64(double* vs, const double* ws, const double* ao_lhs,
                              const double* ao_rhs, size_t stride_ao, size_t stride_grid,
                              int nao, int ngrid, int nset, const uint8_t* tab, size_t ldtab,
                              int blk, void* workspace, cudaStream_t stream);

}  // namespace cfgmm
