// A second stream beside the caller's, for independent preparation kernels
// that overlap (one chain bound by DRAM, the other by instruction issue).
#pragma once

#include <cuda_runtime.h>

namespace cfgmm {

// A non-blocking stream and its fork / join events per host thread and device,
// made on first use and destroyed when the thread exits (per thread, so that
// calls from several threads never record over one another's fork event).
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  SideStream() = default;
  SideStream(const SideStream&) = delete;
  SideStream& operator=(const SideStream&) = delete;
  // At thread exit.  After a device reset or once the CUDA runtime is being
  // torn down the handles may be stale; the calls then return an error, which
  // is ignored (there is nothing left to release).
  ~SideStream() {
    if (join) cudaEventDestroy(join);
    if (fork) cudaEventDestroy(fork);
    if (s) cudaStreamDestroy(s);
    cudaGetLastError();
  }
};

// The calling thread's side stream on the current device, or nullptr when one
// cannot be made (callers then stay on their own stream).  high_priority: a
// separate stream at the device's greatest priority, whose pending CTAs the
// block scheduler serves before those of default-priority streams.
const SideStream* side_stream(bool high_priority = false);

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

// Forks the side stream off `stream` and joins it back on every exit from the
// scope, so an error return between the two never leaves side-stream work
// unordered against the caller's stream (which would break a stream capture,
// or let the caller free scratch that side-stream kernels still write).
// `side` may be null: then nothing is forked and `stream()` is the caller's.
class SideScope {
 public:
  SideScope(const SideStream* side, cudaStream_t stream) : side_(side), stream_(stream) {}
  SideScope(const SideScope&) = delete;
  SideScope& operator=(const SideScope&) = delete;
  ~SideScope() {
    if (forked_) side_join(side_, stream_);
  }
  // Forks; on failure the side stream is not used and work stays on `stream`.
  cudaError_t fork() {
    if (!side_) return cudaSuccess;
    cudaError_t err = side_fork(side_, stream_);
    forked_ = err == cudaSuccess;
    return err;
  }
  // The stream the side chain is enqueued on.
  cudaStream_t stream() const { return forked_ ? side_->s : stream_; }
  // Joins now and reports the join's status.
  cudaError_t join() {
    if (!forked_) return cudaSuccess;
    forked_ = false;
    return side_join(side_, stream_);
  }

 private:
  const SideStream* side_;
  cudaStream_t stream_;
  bool forked_ = false;
};

}  // namespace cfgmm
