// f32.cuh -- element-type conversions of the f32 entry points (f32.cu).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace cfgmm {

// dst[i] = double(src[i]) for i < n (exact).
cudaError_t widen_f32(const float* src, double* dst, size_t n, cudaStream_t stream);
// dst[i] = float(src[i]) for i < n (round to nearest even).
cudaError_t narrow_f64(const double* src, float* dst, size_t n, cudaStream_t stream);

}  // namespace cfgmm
