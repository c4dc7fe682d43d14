// peaks.cu -- measured compute peaks used as roofline denominators by bench.py
// (libcfgmm_peaks.so, not part of the product ABI).
//
// The driver-measured peaks cover HBM copy bandwidth and cuBLAS bf16 only;
// the paths here compute in FP64 (DMMA) and INT8, so their ceilings are
// measured the same way: register-resident loops of independent instructions
// on every SM, timed with CUDA events after a warm-up launch.
#include <cuda_runtime.h>
#include <cstdint>

namespace {

constexpr int kChains = 8;  // independent accumulators per warp

template <int kChains>
__global__ void __launch_bounds__(256) dmma_loop(double* out, int iters, double seed) {
  const int lane = threadIdx.x & 31;
  double a0 = seed + lane * 1e-3, a1 = seed - lane * 1e-3, b0 = 1.0 + lane * 1e-6;
  double acc[kChains][4];
#pragma unroll
  for (int c = 0; c < kChains; ++c)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[c][e] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c)
      asm volatile(
          "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
          "{%0,%1,%2,%3};\n"
          : "+d"(acc[c][0]), "+d"(acc[c][1]), "+d"(acc[c][2]), "+d"(acc[c][3])
          : "d"(a0), "d"(a1), "d"(b0));
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c][0] + acc[c][1] + acc[c][2] + acc[c][3];
  if (s == 12345.678) out[0] = s;  // keeps the loop live; never true in practice
}

__global__ void __launch_bounds__(256) dfma_loop(double* out, int iters, double seed) {
  double x[kChains];
  const double m = 1.0 + threadIdx.x * 1e-9;
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = seed + c;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], m, 1e-12);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 12345.678) out[0] = s;
}

template <class F>
double time_kernel(F launch, double flops) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -1.0;
  launch();  // warm-up
  cudaEventRecord(e0);
  launch();
  cudaEventRecord(e1);
  if (cudaEventSynchronize(e1) != cudaSuccess) return -1.0;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
  return flops / (ms * 1e-3) / 1e12;
}

int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

}  // namespace

extern "C" {

// FP64 tensor-core (DMMA m16n8k4) throughput in TFLOP/s; < 0 on error.
double cfgmm_peak_dmma_tflops(int iters, int ctas_per_sm) {
  double* out = nullptr;
  if (cudaMalloc(&out, 8) != cudaSuccess) return -1.0;
  const int grid = sm_count() * ctas_per_sm;
  const double flops = double(grid) * 8 /*warps*/ * iters * kChains * 2.0 * 16 * 8 * 4;
  double r = time_kernel([&] { dmma_loop<kChains><<<grid, 256>>>(out, iters, 0.5); }, flops);
  cudaFree(out);
  return r;
}

// DMMA throughput with `chains` (4, 8 or 16) independent accumulators per warp,
// `warps` (1..8) warps per CTA and `ctas_per_sm` CTAs per SM: how much
// parallelism the FP64 tensor pipe needs.
double cfgmm_peak_dmma_sweep(int iters, int ctas_per_sm, int warps, int chains) {
  double* out = nullptr;
  if (warps < 1 || warps > 8 || cudaMalloc(&out, 8) != cudaSuccess) return -1.0;
  const int grid = sm_count() * ctas_per_sm;
  const double flops = double(grid) * warps * iters * chains * 2.0 * 16 * 8 * 4;
  double r = -1.0;
  if (chains == 4)
    r = time_kernel([&] { dmma_loop<4><<<grid, 32 * warps>>>(out, iters, 0.5); }, flops);
  else if (chains == 8)
    r = time_kernel([&] { dmma_loop<8><<<grid, 32 * warps>>>(out, iters, 0.5); }, flops);
  else if (chains == 16)
    r = time_kernel([&] { dmma_loop<16><<<grid, 32 * warps>>>(out, iters, 0.5); }, flops);
  cudaFree(out);
  return r;
}

// FP64 FMA-pipe (DFMA) throughput in TFLOP/s; < 0 on error.
double cfgmm_peak_dfma_tflops(int iters, int ctas_per_sm) {
  double* out = nullptr;
  if (cudaMalloc(&out, 8) != cudaSuccess) return -1.0;
  const int grid = sm_count() * ctas_per_sm;
  const double flops = double(grid) * 256 * iters * kChains * 2.0;
  double r = time_kernel([&] { dfma_loop<<<grid, 256>>>(out, iters, 0.5); }, flops);
  cudaFree(out);
  return r;
}

}  // extern "C"
