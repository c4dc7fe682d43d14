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
// All calls share the one array and it keeps whatever the previous call left
// in it.  Nothing in it needs to start at zero: the list kernel writes every
// count and list entry the later kernels read, the work-list kernel writes the
// work items and resets the work counters before the main kernel draws from
// them, and the main kernel writes every partial sum the reduction reads.  Two calls whose work overlaps on the
// GPU (different streams, or different host threads without ordering) race on
// the array and may return wrong results; the caller must order them.
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/cfgmm.h"
#include "aodmao2rho_fp64.cuh"

namespace cfgmm {
void set_last_error(const std::string& msg);
}

namespace {

// Host code must never hand `g_noalloc_scratch` itself to a kernel: on the
// host the name only stands in for the symbol.  Its device address comes from
// cudaGetSymbolAddress, once per device, below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[CFGMM_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};

int fail(int status, const std::string& msg) {
  cfgmm::set_last_error(msg);
  return status;
}

int cuda_fail(cudaError_t err, const char* where) {
  return fail(err == cudaErrorNoDevice ? CFGMM_ERR_NO_DEVICE : CFGMM_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) +
                  ")");
}

// Device address of this device's copy of the scratch array.  Set up on the
// first call made with `dev` current; later calls reuse the cached address.
int scratch_address(int dev, void** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(CFGMM_ERR_INVALID_ARGUMENT, "device index");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess) return cuda_fail(err, "cudaGetSymbolAddress(scratch)");
    if (!p) return fail(CFGMM_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return CFGMM_OK;
}

bool fits_int(size_t v) { return v <= size_t(INT_MAX) - 4096; }

}  // namespace

extern "C" int cfgmm_aodmao2rho_dev_noalloc(double* rhos, const double* dms, const double* ao_lhs,
                                            const double* ao_rhs, size_t stride_ao,
                                            size_t stride_grid, size_t nao, size_t ngrid,
                                            size_t nset, const uint8_t* tab, size_t ldtab,
                                            size_t blksize, void* stream) {
  cfgmm::set_last_error("");
  if (blksize == 0) return fail(CFGMM_ERR_INVALID_ARGUMENT, "BLKSIZE must be at least 1");
  if (nao == 0 || ngrid == 0 || nset == 0) return CFGMM_OK;
  if (!fits_int(nao) || !fits_int(ngrid) || !fits_int(nset) || !fits_int(blksize))
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "nao, ngrid, nset and BLKSIZE must be below 2^31");
  if (stride_grid < ngrid)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "stride_grid < ngrid: rows of rho would overlap");
  if (!rhos || !dms || !ao_lhs || !ao_rhs || !tab)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  const size_t need = cfgmm::aodmao2rho_fp64_workspace(nao, ngrid, nset, blksize);
  if (need > size_t(CFGMM_NOALLOC_SCRATCH_BYTES)) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "problem needs %zu bytes of scratch; the no-allocation entry point has %zu "
                  "(use cfgmm_aodmao2rho_dev)",
                  need, size_t(CFGMM_NOALLOC_SCRATCH_BYTES));
    return fail(CFGMM_ERR_INVALID_ARGUMENT, msg);
  }
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return cuda_fail(err, "cudaGetDevice");
  void* ws = nullptr;
  int rc = scratch_address(dev, &ws);
  if (rc != CFGMM_OK) return rc;
  err = cfgmm::aodmao2rho_fp64(rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, int(nao),
                               int(ngrid), int(nset), tab, ldtab, int(blksize), ws,
                               static_cast<cudaStream_t>(stream));
  if (err != cudaSuccess) return cuda_fail(err, "aodmao2rho_fp64");
  return CFGMM_OK;
}
