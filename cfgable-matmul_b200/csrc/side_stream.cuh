// A second stream beside the caller's, for independent preparation kernels
// that overlap (one chain bound by DRAM, the other by instruction issue).
#pragma once

#include <cuda_runtime.h>

namespace cfgmm {

// A non-blocking stream and its fork / join events per host thread and device,
// made on first use and kept for the life of the thread (per thread, so that
// calls from several threads never record over one another's fork event).
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

// The calling thread's side stream on the current device, or nullptr when one
// cannot be made (callers then stay on their own stream).
const SideStream* side_stream();

// side->s waits for the work enqueued on `stream` so far.
inline cudaError_t side_fork(const SideStream* side, cudaStream_t stream) {
  cudaError_t err = cudaEventRecord(side->fork, stream);
  return err != cudaSuccess ? err : cudaStreamWaitEvent(side->s, side->fork, 0);
}

// `stream` waits for the work enqueued on side->s so far.
inline cudaError_t side_join(const SideStream* side, cudaStream_t stream) {
  cudaError_t err = cudaEventRecord(side->join, side->s);
  return err != cudaSuccess ? err : cudaStreamWaitEvent(stream, side->join, 0);
}

}  // namespace cfgmm
