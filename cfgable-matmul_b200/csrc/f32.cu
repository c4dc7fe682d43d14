// f32.cu -- conversions behind the f32 forms of the two paths.
//
// The reference's MatmulLoops is generic over the element type (structs.rs:3-13)
// with f64 implementations only (structs.rs:19-20); the f32 entry points of the
// C ABI take f32 operands, widen them exactly to f64 in device scratch, run the
// f64 kernels (DMMA, or the Ozaki split with the moduli that 26-bit operands
// need) and round the accumulated result back to f32 once.  These kernels are
// the widening and narrowing passes: one read and one write of each array,
// vectorised where the base pointers allow, grid-stride over the SMs.
#include "f32.cuh"

#include <cstdint>

namespace cfgmm {
namespace {

__global__ void __launch_bounds__(256) widen_kernel(const float* __restrict__ src,
                                                    double* __restrict__ dst, size_t n) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  const bool vec = (reinterpret_cast<uintptr_t>(src) % 16 == 0) &&
                   (reinterpret_cast<uintptr_t>(dst) % 16 == 0);
  if (vec) {
    const size_t n4 = n / 4;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += stride) {
      const float4 v = reinterpret_cast<const float4*>(src)[i];
      reinterpret_cast<double2*>(dst)[2 * i] = make_double2(v.x, v.y);
      reinterpret_cast<double2*>(dst)[2 * i + 1] = make_double2(v.z, v.w);
    }
    for (size_t i = 4 * n4 + size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
      dst[i] = double(src[i]);
  } else {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
      dst[i] = double(src[i]);
  }
}

__global__ void __launch_bounds__(256) narrow_kernel(const double* __restrict__ src,
                                                     float* __restrict__ dst, size_t n) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    dst[i] = __double2float_rn(src[i]);
}

unsigned grid_for(size_t n) {
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t want = (n + 1023) / 1024;
  const size_t cap = size_t(nsm) * 8;
  return unsigned(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

cudaError_t widen_f32(const float* src, double* dst, size_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  widen_kernel<<<grid_for(n), 256, 0, stream>>>(src, dst, n);
  return cudaGetLastError();
}

cudaError_t narrow_f64(const double* src, float* dst, size_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  narrow_kernel<<<grid_for(n), 256, 0, stream>>>(src, dst, n);
  return cudaGetLastError();
}

}  // namespace cfgmm
