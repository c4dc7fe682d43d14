// ao_eval.cuh -- internal interface of the device AO evaluator.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cfgmm {

// phi of every shell at every point (and, when bmax != null, the per-(shell,
// block) maxima of |phi|, zeroed first); see ao_eval.cu for the functions.
cudaError_t eval_ao(double* ao, size_t stride_grid, const double* pts, int ngrid, const double* sxyz,
                    const int* sl, const double* salpha, const double* snorm, const int* srow,
                    int nshell, double* bmax, int blksize, cudaStream_t stream);

// Mask from the maxima (> thr) and phi zeroed outside it.
cudaError_t mask_ao(double* ao, size_t stride_grid, int ngrid, const int* sl, const int* srow,
                    int nshell, const double* bmax, double thr, uint8_t* tab, size_t ldtab,
                    int blksize, cudaStream_t stream);

}  // namespace cfgmm
