// peaks.cu -- measured compute peaks used as roofline denominators by bench.py
// (libcfgmm_peaks.so, not part of the product ABI).
//
// The driver-measured peaks cover HBM copy bandwidth and cuBLAS bf16 only;
// the paths here compute in FP64 (DMMA) and INT8, so their ceilings are
// measured the same way: register-resident loops of independent instructions
// on every SM, timed with CUDA events after a warm-up launch.
#include <cuda_runtime.h>
#include <cstdint>

#include "../tcgen05.cuh"

namespace {

constexpr int kChains = 8;  // independent accumulators per warp

// The same loop with the m16n8k8 shape (twice the work per instruction).
template <int kChains>
__global__ void __launch_bounds__(256) dmma8_loop(double* out, int iters, double seed) {
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
          "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
          "{%8,%9}, {%0,%1,%2,%3};\n"
          : "+d"(acc[c][0]), "+d"(acc[c][1]), "+d"(acc[c][2]), "+d"(acc[c][3])
          : "d"(a0), "d"(a1), "d"(a1), "d"(a0), "d"(b0), "d"(b0));
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c][0] + acc[c][1] + acc[c][2] + acc[c][3];
  if (s == 12345.678) out[0] = s;  // keeps the loop live; never true in practice
}

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

__device__ int g_peak_err;

// tcgen05.mma kind::i8, M=128 N=256 K=32, issued back to back by one thread
// on operands resident in shared memory (zeros), accumulating in TMEM.
__global__ void __launch_bounds__(128, 1) i8_mma_loop(int iters) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint8_t* sA = smem;                // 128 x 128 B
  uint8_t* sB = smem + 16384;        // 256 x 128 B
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 49152);
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + 49160);
  for (int i = threadIdx.x; i < 49152 / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    cfgmm::tc::mbar_init(bar, 1);
    cfgmm::tc::mbar_fence_init();
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (threadIdx.x < 32) {
    cfgmm::tc::tmem_alloc(slot, 256);
    cfgmm::tc::tmem_relinquish();
  }
  cfgmm::tc::fence_before_sync();
  __syncthreads();
  cfgmm::tc::fence_after_sync();
  const uint32_t tmem = *slot;
  if (threadIdx.x == 0) {
    const uint32_t idesc = cfgmm::tc::idesc_i8(128, 256);
    const uint32_t a0 = cfgmm::tc::smem_u32(sA), b0 = cfgmm::tc::smem_u32(sB);
    for (int it = 0; it < iters; ++it)
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        cfgmm::tc::mma_i8(tmem, cfgmm::tc::smem_desc_k128(a0 + 32 * ks),
                          cfgmm::tc::smem_desc_k128(b0 + 32 * ks), idesc, it > 0 || ks > 0);
    cfgmm::tc::mma_commit(bar);
    cfgmm::tc::mbar_wait(bar, 0, &g_peak_err, 1, true);
  }
  cfgmm::tc::fence_before_sync();
  __syncthreads();
  cfgmm::tc::fence_after_sync();
  if (threadIdx.x < 32) cfgmm::tc::tmem_dealloc(tmem, 256);
}

}  // namespace

extern "C" {

// INT8 tensor-core (tcgen05.mma kind::i8) throughput in TOP/s; < 0 on error.
double cfgmm_peak_i8_tops(int iters) {
  const int smem = 49152 + 1024 + 64;
  if (cudaFuncSetAttribute(i8_mma_loop, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess)
    return -1.0;
  const int grid = sm_count();
  const double ops = double(grid) * iters * 4 * 2.0 * 128 * 256 * 32;
  double r = time_kernel([&] { i8_mma_loop<<<grid, 128, smem>>>(iters); }, ops);
  int code = 0;
  cudaMemcpyFromSymbol(&code, g_peak_err, sizeof(int));
  return code ? -2.0 : r;
}

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

// Sustained DMMA throughput: back-to-back launches of the same loop for about
// `seconds`, TFLOP/s over the second half (the clock settles under the power
// cap while it runs).  For kernels timed inside a long step.
double cfgmm_peak_dmma_sustained(double seconds) {
  double* out = nullptr;
  if (cudaMalloc(&out, 8) != cudaSuccess) return -1.0;
  const int grid = sm_count() * 2;
  const int iters = 20000;
  const double flops = double(grid) * 8 * iters * kChains * 2.0 * 16 * 8 * 4;
  const double burst = time_kernel([&] { dmma_loop<kChains><<<grid, 256>>>(out, iters, 0.5); },
                                   flops);
  if (burst <= 0) {
    cudaFree(out);
    return -1.0;
  }
  const double launch_s = flops / (burst * 1e12);
  const int n = int(seconds / launch_s) + 2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int i = 0; i < n / 2; ++i) dmma_loop<kChains><<<grid, 256>>>(out, iters, 0.5);
  cudaEventRecord(e0);
  for (int i = n / 2; i < n; ++i) dmma_loop<kChains><<<grid, 256>>>(out, iters, 0.5);
  cudaEventRecord(e1);
  double r = -1.0;
  if (cudaEventSynchronize(e1) == cudaSuccess) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    r = flops * (n - n / 2) / (ms * 1e-3) / 1e12;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return r;
}

// m16n8k8 DMMA throughput, same parameters as cfgmm_peak_dmma_sweep.
double cfgmm_peak_dmma8_sweep(int iters, int ctas_per_sm, int warps, int chains) {
  double* out = nullptr;
  if (warps < 1 || warps > 8 || cudaMalloc(&out, 8) != cudaSuccess) return -1.0;
  const int grid = sm_count() * ctas_per_sm;
  const double flops = double(grid) * warps * iters * chains * 2.0 * 16 * 8 * 8;
  double r = -1.0;
  if (chains == 4)
    r = time_kernel([&] { dmma8_loop<4><<<grid, 32 * warps>>>(out, iters, 0.5); }, flops);
  else if (chains == 8)
    r = time_kernel([&] { dmma8_loop<8><<<grid, 32 * warps>>>(out, iters, 0.5); }, flops);
  else if (chains == 16)
    r = time_kernel([&] { dmma8_loop<16><<<grid, 32 * warps>>>(out, iters, 0.5); }, flops);
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
