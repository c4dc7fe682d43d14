// aodmao2rho_noalloc.cu -- the masked AO-DM-AO contraction for callers that
// cannot allocate device memory.
//
// Who needs this: a host that has handed all of a GPU's memory to its own
// pool or arena (a serving process that reserves HBM up front, an embedding
// runtime whose memory manager owns the device), and code that must not call
// cudaMalloc / cudaFree inside a time-critical loop because those calls can
// synchronise the whole device.  cfgmm_aodmao2rho_dev needs scratch for the
// per-block active AO lists and the per-row-tile partial sums and takes it
// from the stream-ordered allocator; this variant takes it from one
// fixed-size array in the library's own device memory instead, so it
// allocates nothing.  The caller still provides every input and output.
//
// The array (CFGMM_NOALLOC_SCRATCH_BYTES, 32 MiB) is part of the library's
// device image: every GPU on which the library is loaded holds it until the
// process exits.  Problems whose scratch would not fit are refused with
// CFGMM_ERR_INVALID_ARGUMENT and a message giving the size they need.
//
// The first call on a device loads the library's device image there and looks
// up the array's device address; make that first call before any stream
// capture.  Every later call looks the address up again (a lookup in the
// runtime's table, no allocation), so a device reset and a new context between
// two calls can never leave a stale address behind.
//
// All calls share the one array and it keeps whatever the previous call left
// in it.  Nothing in it needs to start at zero: the list kernel writes every
// count and list entry the later kernels read, the work-list kernel writes the
// work items and resets the work counters before the main kernel draws from
// them, and the main kernel writes every partial sum the reduction reads.  Two calls whose work overlaps on the
// GPU (different streams, or different host threads without ordering) race on
// the array and may return wrong results; the caller must order them.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "../../include/cfgmm.h"
#include "aodmao2rho_fp64.cuh"

namespace cfgmm {
void set_last_error(const std::string& msg);
int check_aodm_dev(const void* rhos, const void* dms, const void* ao_lhs, const void* ao_rhs,
                   size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
                   const uint8_t* tab, size_t ldtab, size_t blksize);
}

namespace {

// Host code must never hand `g_noalloc_scratch` itself to a kernel: on the
// host the name only stands in for the symbol.  Its device address comes from
// cudaGetSymbolAddress with the calling device current, below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[CFGMM_NOALLOC_SCRATCH_BYTES];

int fail(int status, const std::string& msg) {
  cfgmm::set_last_error(msg);
  return status;
}

int cuda_fail(cudaError_t err, const char* where) {
  return fail(err == cudaErrorNoDevice ? CFGMM_ERR_NO_DEVICE : CFGMM_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) +
                  ")");
}

// Device address of the current device's copy of the scratch array, in the
// current context.  Not cached: a cached address would outlive a device reset.
int scratch_address(void** out) {
  void* p = nullptr;
  cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (err != cudaSuccess) return cuda_fail(err, "cudaGetSymbolAddress(scratch)");
  if (!p) return fail(CFGMM_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
  *out = p;
  return CFGMM_OK;
}

}  // namespace

extern "C" int cfgmm_aodmao2rho_dev_noalloc(double* rhos, const double* dms, const double* ao_lhs,
                                            const double* ao_rhs, size_t stride_ao,
                                            size_t stride_grid, size_t nao, size_t ngrid,
                                            size_t nset, const uint8_t* tab, size_t ldtab,
                                            size_t blksize, void* stream) {
  cfgmm::set_last_error("");
  // the same checks, in the same order, as cfgmm_aodmao2rho_dev
  int rc = cfgmm::check_aodm_dev(rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, nao, ngrid,
                                 nset, tab, ldtab, blksize);
  if (rc != CFGMM_OK) return rc;
  if (nao == 0 || ngrid == 0 || nset == 0) return CFGMM_OK;
  const size_t need = cfgmm::aodmao2rho_fp64_workspace(nao, ngrid, nset, blksize);
  if (need > size_t(CFGMM_NOALLOC_SCRATCH_BYTES)) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "problem needs %zu bytes of scratch; the no-allocation entry point has %zu "
                  "(use cfgmm_aodmao2rho_dev)",
                  need, size_t(CFGMM_NOALLOC_SCRATCH_BYTES));
    return fail(CFGMM_ERR_INVALID_ARGUMENT, msg);
  }
  int ndev = 0;
  cudaError_t err = cudaGetDeviceCount(&ndev);
  if (err != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(CFGMM_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  void* ws = nullptr;
  if ((rc = scratch_address(&ws)) != CFGMM_OK) return rc;
  err = cfgmm::aodmao2rho_fp64(rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, int(nao),
                               int(ngrid), int(nset), tab, ldtab, int(blksize), ws,
                               static_cast<cudaStream_t>(stream));
  if (err != cudaSuccess) return cuda_fail(err, "aodmao2rho_fp64");
  return CFGMM_OK;
}
