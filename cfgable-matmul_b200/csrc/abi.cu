// abi.cu -- the extern "C" boundary of libcfgmm.so (declared in include/cfgmm.h).
//
// Host-side duties only: argument validation that reproduces the reference's
// panics as status codes, per-device workspaces and streams, host<->device
// staging for the host-pointer entry points, and dispatch to the kernels.
// Validation happens before any CUDA call, so a rejected call never touches a
// device or an output buffer.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cfgmm.h"
#include "aodmao2rho_fp64.cuh"
#include "aodmao2rho_split.cuh"
#include "ao_eval.cuh"
#include "dgemm_fp64.cuh"
#include "f32.cuh"
#include "fock.cuh"
#include "server.cuh"
#include "gemm_i8.cuh"
#include "ozaki.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t err, const char* where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorName(err) + " (" +
                 cudaGetErrorString(err) + ")";
  if (err == cudaErrorMemoryAllocation) return CFGMM_ERR_OUT_OF_MEMORY;
  if (err == cudaErrorNoDevice || err == cudaErrorInsufficientDriver) return CFGMM_ERR_NO_DEVICE;
  return CFGMM_ERR_CUDA;
}

#define CFGMM_CUDA(call)                                   \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);    \
  } while (0)

// ---------------------------------------------------------------------------
// extents: number of elements a Rust slice must hold for the index range read
// or written (0 when nothing is accessed).
// ---------------------------------------------------------------------------
bool mul_ok(size_t a, size_t b, size_t* out) { return !__builtin_mul_overflow(a, b, out); }
bool add_ok(size_t a, size_t b, size_t* out) { return !__builtin_add_overflow(a, b, out); }

// rows x cols with row stride ld: (rows-1)*ld + cols
bool extent2(size_t rows, size_t cols, size_t ld, size_t* out) {
  if (rows == 0 || cols == 0) { *out = 0; return true; }
  size_t t;
  return mul_ok(rows - 1, ld, &t) && add_ok(t, cols, out);
}

// Kernels index with 32-bit ints and round sizes up to their tiles.
bool fits_int(size_t v) { return v <= size_t(INT_MAX) - 4096; }

// ---------------------------------------------------------------------------
// per-device state for the host-pointer entry points
// ---------------------------------------------------------------------------
// Most blocks of a large host-pointer GEMM (see gemm_host_blocked).
constexpr size_t kHostBlocks = 8;

struct DeviceState {
  std::mutex mu;
  cudaStream_t stream = nullptr;
  // second copy stream and its events: C's upload overlaps the split
  // DGEMM's residues and INT8 GEMM (C is first read by the reconstruction)
  cudaStream_t copy = nullptr;
  cudaEvent_t ab_done = nullptr, c_ready = nullptr;
  // blocked host GEMM: uploads on `copy`, compute on `stream`, downloads on
  // `down`, one pair of events per block
  cudaStream_t down = nullptr;
  cudaEvent_t up[kHostBlocks] = {}, done[kHostBlocks] = {};
  void* buf = nullptr;
  size_t cap = 0;
};

std::mutex g_devices_mu;
std::vector<std::unique_ptr<DeviceState>> g_devices;

// Once per device and process: keep memory freed with cudaFreeAsync in the
// device's default pool, so the stream-ordered scratch of repeated _dev calls
// is reused instead of being returned to the driver at every synchronisation.
void init_device_once(int dev) {
  static std::mutex mu;
  static std::vector<bool> done;
  std::lock_guard<std::mutex> lk(mu);
  if (done.size() <= size_t(dev)) done.resize(dev + 1, false);
  if (done[dev]) return;
  done[dev] = true;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
}

int current_device(int* dev) {
  int n = 0;
  cudaError_t err = cudaGetDeviceCount(&n);
  if (err != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(CFGMM_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  CFGMM_CUDA(cudaGetDevice(dev));
  init_device_once(*dev);
  return CFGMM_OK;
}

DeviceState* device_state(int dev) {
  std::lock_guard<std::mutex> lk(g_devices_mu);
  if (g_devices.size() <= size_t(dev)) g_devices.resize(dev + 1);
  if (!g_devices[dev]) g_devices[dev].reset(new DeviceState);
  return g_devices[dev].get();
}

// Creates the copy stream and events of the overlapped C upload (caller holds st->mu).
int ensure_copy_stream(DeviceState* st) {
  if (!st->copy) CFGMM_CUDA(cudaStreamCreateWithFlags(&st->copy, cudaStreamNonBlocking));
  if (!st->ab_done) CFGMM_CUDA(cudaEventCreateWithFlags(&st->ab_done, cudaEventDisableTiming));
  if (!st->c_ready) CFGMM_CUDA(cudaEventCreateWithFlags(&st->c_ready, cudaEventDisableTiming));
  return CFGMM_OK;
}

// The download stream and block events of the blocked host GEMM (caller holds st->mu).
int ensure_block_pipeline(DeviceState* st) {
  int rc = ensure_copy_stream(st);
  if (rc != CFGMM_OK) return rc;
  if (!st->down) CFGMM_CUDA(cudaStreamCreateWithFlags(&st->down, cudaStreamNonBlocking));
  for (size_t i = 0; i < kHostBlocks; ++i) {
    if (!st->up[i]) CFGMM_CUDA(cudaEventCreateWithFlags(&st->up[i], cudaEventDisableTiming));
    if (!st->done[i]) CFGMM_CUDA(cudaEventCreateWithFlags(&st->done[i], cudaEventDisableTiming));
  }
  return CFGMM_OK;
}

// Grows the device's staging buffer to at least `bytes` (caller holds st->mu).
int reserve(DeviceState* st, size_t bytes) {
  if (!st->stream) CFGMM_CUDA(cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking));
  if (st->cap >= bytes) return CFGMM_OK;
  if (st->buf) {
    CFGMM_CUDA(cudaFree(st->buf));
    st->buf = nullptr;
    st->cap = 0;
  }
  CFGMM_CUDA(cudaMalloc(&st->buf, bytes));
  st->cap = bytes;
  return CFGMM_OK;
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// ---------------------------------------------------------------------------
// DGEMM
// ---------------------------------------------------------------------------
struct GemmExtents {
  size_t a, b, c;
};

// Element counts only (any element type): pointers are checked for null.
int check_gemm(const void* c, size_t c_len, const void* a, size_t a_len, const void* b,
               size_t b_len, size_t m, size_t n, size_t k, size_t lda, size_t ldb, size_t ldc,
               bool ta, bool tb, GemmExtents* ex) {
  if (m == 0 || n == 0 || k == 0) {
    *ex = {0, 0, 0};
    return CFGMM_OK;
  }
  if (!fits_int(m) || !fits_int(n) || !fits_int(k))
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "m, n and k must each be below 2^31");
  if (ldc < n)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "ldc < n: rows of C would overlap");
  bool ok = (ta ? extent2(k, m, lda, &ex->a) : extent2(m, k, lda, &ex->a)) &&
            (tb ? extent2(n, k, ldb, &ex->b) : extent2(k, n, ldb, &ex->b)) &&
            extent2(m, n, ldc, &ex->c);
  if (!ok) return fail(CFGMM_ERR_INVALID_ARGUMENT, "index range overflows usize");
  if (a_len < ex->a || b_len < ex->b || c_len < ex->c) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "slice too short (a %zu < %zu, b %zu < %zu or c %zu < %zu): the reference "
                  "panics here",
                  a_len, ex->a, b_len, ex->b, c_len, ex->c);
    return fail(CFGMM_ERR_INVALID_ARGUMENT, msg);
  }
  if (!a || !b || !c) return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  return CFGMM_OK;
}

int check_precision(int precision) {
  if (precision == CFGMM_PREC_FP64 || precision == CFGMM_PREC_OZAKI_INT8) return CFGMM_OK;
  return fail(CFGMM_ERR_INVALID_ARGUMENT, "unknown precision");
}

int check_split_gemm(size_t k) {
  if (k > size_t(cfgmm::kOzakiMaxK))
    return fail(CFGMM_ERR_UNIMPLEMENTED,
                "CFGMM_PREC_OZAKI_INT8 supports k <= 65536 (exact INT32 accumulation)");
  return CFGMM_OK;
}

// Reads the sticky error words of the tcgen05 kernels after a synchronised call.
int check_device_waits() {
  int code = 0, code2 = 0, code3 = 0, code4 = 0;
  CFGMM_CUDA(cfgmm::gemm_i8_read_error(&code));
  CFGMM_CUDA(cfgmm::aodmao2rho_split_read_error(&code2));
  CFGMM_CUDA(cfgmm::dgemm_read_error(&code3));
  CFGMM_CUDA(cfgmm::aodm_read_error(&code4));
  if (code == 0) code = code2;
  if (code == 0) code = code3;
  if (code == 0) code = code4;
  if (code != 0) {
    // reported once: the words start over for the next call
    cudaError_t e = cfgmm::gemm_i8_reset_error(nullptr);
    if (e == cudaSuccess) e = cfgmm::aodmao2rho_split_reset_error(nullptr);
    if (e == cudaSuccess) e = cfgmm::dgemm_reset_error(nullptr);
    if (e == cudaSuccess) e = cfgmm::aodm_reset_error(nullptr);
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "resetting the device wait words");
    char msg[128];
    std::snprintf(msg, sizeof(msg), "a tensor-core pipeline wait timed out (code %d)", code);
    return fail(CFGMM_ERR_TIMEOUT, msg);
  }
  return CFGMM_OK;
}

// Mask of the masked GEMM: tab[p * ldtab + j / blk] for p < k, j < n.
struct GemmMask {
  const uint8_t* tab;  // null: plain GEMM
  size_t tab_len, ldtab, blk;
};

int check_mask(const GemmMask& mk, size_t n, size_t k, uint8_t transb, size_t* tab_extent) {
  *tab_extent = 0;
  if (!mk.tab && mk.tab_len == 0 && mk.blk == 0) return CFGMM_OK;  // plain GEMM
  // impl_matmul_non0tab.rs:228-230: transb panics before anything else
  if (transb)
    return fail(CFGMM_ERR_UNIMPLEMENTED,
                "transb=true is not implemented for the masked GEMM (as in the reference)");
  if (mk.blk == 0) return fail(CFGMM_ERR_INVALID_ARGUMENT, "BLKSIZE must be at least 1");
  if (n == 0 || k == 0) return CFGMM_OK;
  if (!fits_int(mk.blk)) return fail(CFGMM_ERR_INVALID_ARGUMENT, "BLKSIZE must be below 2^31");
  if (!extent2(k, (n + mk.blk - 1) / mk.blk, mk.ldtab, tab_extent))
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "index range overflows usize");
  if (mk.tab_len < *tab_extent) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "slice too short (tab %zu < %zu): the reference panics here",
                  mk.tab_len, *tab_extent);
    return fail(CFGMM_ERR_INVALID_ARGUMENT, msg);
  }
  if (!mk.tab) return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  return CFGMM_OK;
}

// A large host-pointer GEMM in kHostBlocks blocks, so that the PCIe transfers
// of one block overlap the work and the transfers of the others (the link
// carries both directions at once): one operand goes up whole first, then each
// block's part of the other operand and of C go up on the copy stream, the
// block is computed on the compute stream and its part of C comes back on the
// download stream.  In split precision, and for the masked GEMM (its mask runs
// along the columns of B and goes up whole), the transfers bound the call: 5 blocks
// of rows of C and op(A) that shrink (30, 25, 20, 15, 10 %), so that the last
// block's work and download, which nothing overlaps, are the smallest; B goes
// up first and its residues are formed once.  In FP64 the work bounds the
// call: 8 equal blocks of columns of C and op(B), A going up first (186 MB
// instead of 505 MB at the headline shape), so that the work starts early and
// each block's upload takes about as long as the previous block's work.  The device buffers keep the host layouts; every element of C is
// computed from the same row of op(A) and column of op(B) as in one call.
int gemm_host_blocked(DeviceState* st, double* c, const double* a, const double* b, size_t m,
                      size_t n, size_t k, size_t lda, size_t ldb, size_t ldc, bool transa,
                      bool transb, bool split, int nmod, double* da, double* db, double* dc,
                      void* ws, bool by_rows, const uint8_t* tab, uint8_t* dt, size_t tab_ext,
                      size_t ldtab, size_t blk_mask) {
  int rc = ensure_block_pipeline(st);
  if (rc != CFGMM_OK) return rc;
  const size_t extent = by_rows ? m : n;
  static constexpr double kSplitShare[5] = {0.30, 0.25, 0.20, 0.15, 0.10};
  const size_t nblocks = by_rows ? 5 : kHostBlocks;
  size_t bound[kHostBlocks + 1] = {0};
  double acc = 0.0;
  for (size_t i = 0; i < nblocks; ++i) {
    acc += by_rows ? kSplitShare[i] : 1.0 / double(nblocks);
    bound[i + 1] =
        i + 1 == nblocks ? extent : std::min(extent, size_t(acc * double(extent) + 0.5));
  }
  const size_t ea = transa ? (k - 1) * lda + m : (m - 1) * lda + k;
  const size_t eb = transb ? (n - 1) * ldb + k : (k - 1) * ldb + n;
  cudaError_t err = cudaSuccess;
  if (split) err = cfgmm::gemm_i8_reset_error(st->stream);
  if (err == cudaSuccess)
    err = by_rows ? cudaMemcpyAsync(db, b, eb * 8, cudaMemcpyHostToDevice, st->copy)
                  : cudaMemcpyAsync(da, a, ea * 8, cudaMemcpyHostToDevice, st->copy);
  if (err == cudaSuccess && dt)  // the mask of the masked GEMM, whole
    err = cudaMemcpyAsync(dt, tab, tab_ext, cudaMemcpyHostToDevice, st->copy);
  size_t done_blocks = 0;
  for (size_t blk = 0; err == cudaSuccess && blk < nblocks; ++blk) {
    const size_t x0 = bound[blk], xk = bound[blk + 1] - x0;
    if (xk == 0) continue;
    // the block of C: rows x0.. (by_rows) or columns x0..; pointers into the
    // device copies, which keep the host layouts
    const size_t i0 = by_rows ? x0 : 0, mk = by_rows ? xk : m;
    const size_t j0 = by_rows ? 0 : x0, nk = by_rows ? n : xk;
    if (by_rows)  // rows of op(A): columns of A when transposed
      err = transa ? cudaMemcpy2DAsync(da + i0, lda * 8, a + i0, lda * 8, mk * 8, k,
                                       cudaMemcpyHostToDevice, st->copy)
                   : cudaMemcpy2DAsync(da + i0 * lda, lda * 8, a + i0 * lda, lda * 8, k * 8, mk,
                                       cudaMemcpyHostToDevice, st->copy);
    else  // columns of op(B): rows of B when transposed
      err = transb ? cudaMemcpy2DAsync(db + j0 * ldb, ldb * 8, b + j0 * ldb, ldb * 8, k * 8, nk,
                                       cudaMemcpyHostToDevice, st->copy)
                   : cudaMemcpy2DAsync(db + j0, ldb * 8, b + j0, ldb * 8, nk * 8, k,
                                       cudaMemcpyHostToDevice, st->copy);
    double* dck = dc + i0 * ldc + j0;
    if (err == cudaSuccess)
      err = cudaMemcpy2DAsync(dck, ldc * 8, c + i0 * ldc + j0, ldc * 8, nk * 8, mk,
                              cudaMemcpyHostToDevice, st->copy);
    if (err == cudaSuccess) err = cudaEventRecord(st->up[blk], st->copy);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(st->stream, st->up[blk], 0);
    const double* dak = transa ? da + i0 : da + i0 * lda;
    const double* dbk = transb ? db + j0 * ldb : db + j0;
    if (err == cudaSuccess)
      err = split ? cfgmm::ozaki_dgemm(dck, dak, dbk, int(mk), int(nk), int(k), lda, ldb, ldc,
                                       transa, transb, nmod, ws, st->stream, nullptr, dt, ldtab,
                                       int(blk_mask), nullptr, int(m), int(n), false,
                                       done_blocks > 0)
            : dt ? cfgmm::dgemm_fp64_non0tab(dck, dak, dbk, int(mk), int(nk), int(k), lda, ldb,
                                             ldc, transa, dt, ldtab, int(blk_mask), st->stream)
                 : cfgmm::dgemm_fp64(dck, dak, dbk, int(mk), int(nk), int(k), lda, ldb, ldc,
                                     transa, transb, st->stream);
    if (err == cudaSuccess) err = cudaEventRecord(st->done[blk], st->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(st->down, st->done[blk], 0);
    if (err == cudaSuccess)
      err = cudaMemcpy2DAsync(c + i0 * ldc + j0, ldc * 8, dck, ldc * 8, nk * 8, mk,
                              cudaMemcpyDeviceToHost, st->down);
    ++done_blocks;
  }
  // every stream drained before the staging buffer can be reused
  const cudaError_t e1 = cudaStreamSynchronize(st->copy);
  const cudaError_t e2 = cudaStreamSynchronize(st->stream);
  const cudaError_t e3 = cudaStreamSynchronize(st->down);
  if (err == cudaSuccess) err = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
  if (err != cudaSuccess) return cuda_fail(err, "blocked host GEMM");
  return check_device_waits();
}

int gemm_host(double* c, size_t c_len, const double* a, size_t a_len, const double* b,
              size_t b_len, size_t m, size_t n, size_t k, size_t lda, size_t ldb, size_t ldc,
              uint8_t transa, uint8_t transb, int precision,
              GemmMask mk = GemmMask{nullptr, 0, 0, 0}) {
  g_last_error.clear();
  const bool masked = mk.tab || mk.tab_len || mk.blk;
  size_t tab_ext = 0;
  int rc = check_mask(mk, n, k, transb, &tab_ext);
  if (rc != CFGMM_OK) return rc;
  GemmExtents ex;
  rc = check_gemm(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa != 0,
                  transb != 0, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  if (ex.c == 0) return CFGMM_OK;
  const bool split = precision == CFGMM_PREC_OZAKI_INT8;
  if (split && (rc = check_split_gemm(k)) != CFGMM_OK) return rc;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  DeviceState* st = device_state(dev);
  std::lock_guard<std::mutex> lk(st->mu);
  const int nmod = split ? cfgmm::ozaki_default_moduli(int(k)) : 0;
  const size_t oa = 0, ob = align256(ex.a * 8), oc = ob + align256(ex.b * 8);
  const size_t ot = oc + align256(ex.c * 8);
  const size_t ows = ot + align256(tab_ext);
  const size_t wsb = split ? cfgmm::ozaki_dgemm_workspace(int(m), int(n), int(k), nmod) : 0;
  if ((rc = reserve(st, ows + wsb)) != CFGMM_OK) return rc;
  char* base = static_cast<char*>(st->buf);
  double* da = reinterpret_cast<double*>(base + oa);
  double* db = reinterpret_cast<double*>(base + ob);
  double* dc = reinterpret_cast<double*>(base + oc);
  uint8_t* dt = masked ? reinterpret_cast<uint8_t*>(base + ot) : nullptr;
  // masked products block by rows (the mask runs along B's columns and is
  // needed whole); unmasked FP64 ones by columns
  const bool by_rows = split || masked;
  if (ex.c * 8 >= (size_t(64) << 20) && (by_rows ? m : n) >= 512)
    return gemm_host_blocked(st, c, a, b, m, n, k, lda, ldb, ldc, transa != 0, transb != 0, split,
                             nmod, da, db, dc, base + ows, by_rows, mk.tab, dt, tab_ext,
                             mk.ldtab, mk.blk);
  CFGMM_CUDA(cudaMemcpyAsync(da, a, ex.a * 8, cudaMemcpyHostToDevice, st->stream));
  CFGMM_CUDA(cudaMemcpyAsync(db, b, ex.b * 8, cudaMemcpyHostToDevice, st->stream));
  if (masked) CFGMM_CUDA(cudaMemcpyAsync(dt, mk.tab, tab_ext, cudaMemcpyHostToDevice, st->stream));
  if (split) {
    // C goes up on the copy stream once A and B are in, while the residues
    // and the INT8 GEMM run; the reconstruction waits for it
    if ((rc = ensure_copy_stream(st)) != CFGMM_OK) return rc;
    CFGMM_CUDA(cudaEventRecord(st->ab_done, st->stream));
    CFGMM_CUDA(cudaStreamWaitEvent(st->copy, st->ab_done, 0));
    CFGMM_CUDA(cudaMemcpyAsync(dc, c, ex.c * 8, cudaMemcpyHostToDevice, st->copy));
    CFGMM_CUDA(cudaEventRecord(st->c_ready, st->copy));
    cudaError_t err = cfgmm::gemm_i8_reset_error(st->stream);
    if (err == cudaSuccess)
      err = cfgmm::ozaki_dgemm(dc, da, db, int(m), int(n), int(k), lda, ldb, ldc, transa != 0,
                               transb != 0, nmod, base + ows, st->stream, nullptr, dt, mk.ldtab,
                               int(mk.blk), st->c_ready);
    // C is complete before it goes back, whichever path ozaki_dgemm took
    if (err == cudaSuccess) err = cudaStreamWaitEvent(st->stream, st->c_ready, 0);
    if (err != cudaSuccess) {
      cudaStreamSynchronize(st->copy);  // the staging buffer is not reused under a live copy
      return cuda_fail(err, "ozaki_dgemm");
    }
  } else if (masked) {
    CFGMM_CUDA(cudaMemcpyAsync(dc, c, ex.c * 8, cudaMemcpyHostToDevice, st->stream));
    CFGMM_CUDA(cfgmm::dgemm_fp64_non0tab(dc, da, db, int(m), int(n), int(k), lda, ldb, ldc,
                                         transa != 0, dt, mk.ldtab, int(mk.blk), st->stream));
  } else {
    CFGMM_CUDA(cudaMemcpyAsync(dc, c, ex.c * 8, cudaMemcpyHostToDevice, st->stream));
    CFGMM_CUDA(cfgmm::dgemm_fp64(dc, da, db, int(m), int(n), int(k), lda, ldb, ldc, transa != 0,
                                 transb != 0, st->stream));
  }
  CFGMM_CUDA(cudaMemcpyAsync(c, dc, ex.c * 8, cudaMemcpyDeviceToHost, st->stream));
  CFGMM_CUDA(cudaStreamSynchronize(st->stream));
  return check_device_waits();
}

// ---------------------------------------------------------------------------
// AO-DM-AO
// ---------------------------------------------------------------------------
struct AodmExtents {
  size_t rhos, dms, ao, tab;
};

int check_aodm(const void* rhos, size_t rhos_len, const void* dms, size_t dms_len,
               const void* ao_lhs, size_t ao_lhs_len, const void* ao_rhs, size_t ao_rhs_len,
               size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
               const uint8_t* tab, size_t tab_len, size_t ldtab, size_t blksize,
               AodmExtents* ex) {
  if (blksize == 0)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "BLKSIZE must be at least 1");
  if (nao == 0 || ngrid == 0 || nset == 0) {
    *ex = {0, 0, 0, 0};
    return CFGMM_OK;
  }
  if (!fits_int(nao) || !fits_int(ngrid) || !fits_int(nset) || !fits_int(blksize))
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "nao, ngrid, nset and BLKSIZE must be below 2^31");
  if (stride_grid < ngrid)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "stride_grid < ngrid: rows of rho would overlap");
  const size_t nblk = (ngrid + blksize - 1) / blksize;
  size_t dm_stride, t;
  bool ok = extent2(nset, ngrid, stride_grid, &ex->rhos) && extent2(nao, ngrid, stride_grid, &ex->ao) &&
            extent2(nao, nblk, ldtab, &ex->tab) && mul_ok(stride_ao, stride_ao, &dm_stride) &&
            extent2(nao, nao, stride_ao, &t) && mul_ok(nset - 1, dm_stride, &ex->dms) &&
            add_ok(ex->dms, t, &ex->dms);
  if (!ok) return fail(CFGMM_ERR_INVALID_ARGUMENT, "index range overflows usize");
  if (rhos_len < ex->rhos || dms_len < ex->dms || ao_lhs_len < ex->ao || ao_rhs_len < ex->ao ||
      tab_len < ex->tab) {
    char msg[320];
    std::snprintf(msg, sizeof(msg),
                  "slice too short (rhos %zu/%zu, dms %zu/%zu, ao_lhs %zu/%zu, ao_rhs %zu/%zu, "
                  "tab %zu/%zu): the reference panics here",
                  rhos_len, ex->rhos, dms_len, ex->dms, ao_lhs_len, ex->ao, ao_rhs_len, ex->ao,
                  tab_len, ex->tab);
    return fail(CFGMM_ERR_INVALID_ARGUMENT, msg);
  }
  if (!rhos || !dms || !ao_lhs || !ao_rhs || !tab)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  return CFGMM_OK;
}

// The status of a finished AO-DM-AO run: a timed-out pipeline wait of either kernel family.
int aodm_device_status(bool split) {
  if (split) return check_device_waits();
  int code = 0;
  CFGMM_CUDA(cfgmm::aodm_read_error(&code));
  if (code != 0) {
    char msg[128];
    std::snprintf(msg, sizeof(msg), "a pipeline wait of the FP64 kernel timed out (code %d)", code);
    return fail(CFGMM_ERR_TIMEOUT, msg);
  }
  return CFGMM_OK;
}

// A host-pointer AO-DM-AO contraction whose phi tables exceed 64 MB, in 4
// blocks of whole grid blocks so that the PCIe transfers of one block overlap
// the work and the transfers of the others: D, the mask and rho go up first,
// then each block's columns of phi go up on the copy stream, the block is
// contracted on the compute stream and its columns of rho come back on the
// download stream.  Every grid block is contracted exactly as in one call (its
// rho depends only on its own phi columns, D and its mask column).
int aodm_host_blocked(DeviceState* st, double* rhos, const double* dms, const double* ao_lhs,
                      const double* ao_rhs, size_t stride_ao, size_t stride_grid, size_t nao,
                      size_t ngrid, size_t nset, const uint8_t* tab, size_t ldtab,
                      size_t blksize, bool split, const AodmExtents& ex, double* d_dms,
                      double* d_lhs, double* d_rhs, uint8_t* d_tab, double* d_rho, void* ws) {
  int rc = ensure_block_pipeline(st);
  if (rc != CFGMM_OK) return rc;
  constexpr size_t kBlocks = 4;
  const size_t nblk = (ngrid + blksize - 1) / blksize;
  size_t bound[kBlocks + 1] = {0};
  for (size_t i = 1; i <= kBlocks; ++i) bound[i] = std::min(ngrid, (nblk * i / kBlocks) * blksize);
  bound[kBlocks] = ngrid;
  const bool same_ao = d_lhs == d_rhs;
  cudaError_t err = split ? cfgmm::aodmao2rho_split_reset_error(st->stream) : cudaSuccess;
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d_dms, dms, ex.dms * 8, cudaMemcpyHostToDevice, st->copy);
  if (err == cudaSuccess) err = cudaMemcpyAsync(d_tab, tab, ex.tab, cudaMemcpyHostToDevice, st->copy);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d_rho, rhos, ex.rhos * 8, cudaMemcpyHostToDevice, st->copy);
  for (size_t blk = 0; err == cudaSuccess && blk < kBlocks; ++blk) {
    const size_t g0 = bound[blk], gk = bound[blk + 1] - g0;
    if (gk == 0) continue;
    err = cudaMemcpy2DAsync(d_lhs + g0, stride_grid * 8, ao_lhs + g0, stride_grid * 8, gk * 8, nao,
                            cudaMemcpyHostToDevice, st->copy);
    if (err == cudaSuccess && !same_ao)
      err = cudaMemcpy2DAsync(d_rhs + g0, stride_grid * 8, ao_rhs + g0, stride_grid * 8, gk * 8,
                              nao, cudaMemcpyHostToDevice, st->copy);
    if (err == cudaSuccess) err = cudaEventRecord(st->up[blk], st->copy);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(st->stream, st->up[blk], 0);
    const size_t b0 = g0 / blksize;
    if (err == cudaSuccess)
      err = split ? cfgmm::aodmao2rho_split(d_rho + g0, d_dms, d_lhs + g0, d_rhs + g0, stride_ao,
                                            stride_grid, int(nao), int(gk), int(nset), d_tab + b0,
                                            ldtab, int(blksize), ws, st->stream)
                  : cfgmm::aodmao2rho_fp64(d_rho + g0, d_dms, d_lhs + g0, d_rhs + g0, stride_ao,
                                           stride_grid, int(nao), int(gk), int(nset), d_tab + b0,
                                           ldtab, int(blksize), ws, st->stream);
    if (err == cudaSuccess) err = cudaEventRecord(st->done[blk], st->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(st->down, st->done[blk], 0);
    if (err == cudaSuccess)
      err = cudaMemcpy2DAsync(rhos + g0, stride_grid * 8, d_rho + g0, stride_grid * 8, gk * 8, nset,
                              cudaMemcpyDeviceToHost, st->down);
  }
  // every stream drained before the staging buffer can be reused
  const cudaError_t e1 = cudaStreamSynchronize(st->copy);
  const cudaError_t e2 = cudaStreamSynchronize(st->stream);
  const cudaError_t e3 = cudaStreamSynchronize(st->down);
  if (err == cudaSuccess) err = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
  if (err != cudaSuccess) return cuda_fail(err, "blocked AO-DM-AO");
  return aodm_device_status(split);
}

int aodm_host(double* rhos, size_t rhos_len, const double* dms, size_t dms_len,
              const double* ao_lhs, size_t ao_lhs_len, const double* ao_rhs, size_t ao_rhs_len,
              size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
              const uint8_t* tab, size_t tab_len, size_t ldtab, size_t blksize, int precision) {
  g_last_error.clear();
  AodmExtents ex;
  int rc = check_aodm(rhos, rhos_len, dms, dms_len, ao_lhs, ao_lhs_len, ao_rhs, ao_rhs_len,
                      stride_ao, stride_grid, nao, ngrid, nset, tab, tab_len, ldtab, blksize, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  const bool split = precision == CFGMM_PREC_OZAKI_INT8;
  if (split && nao > 16384)
    return fail(CFGMM_ERR_UNIMPLEMENTED, "split-precision AO-DM-AO supports nao <= 16384");
  if (ex.rhos == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  DeviceState* st = device_state(dev);
  std::lock_guard<std::mutex> lk(st->mu);
  // ao_lhs and ao_rhs are usually the same table (rho = phi^T D phi): stage once.
  const bool same_ao = ao_lhs == ao_rhs;
  const size_t o_dms = 0;
  const size_t o_lhs = o_dms + align256(ex.dms * 8);
  const size_t o_rhs = o_lhs + align256(ex.ao * 8);
  const size_t o_tab = o_rhs + (same_ao ? 0 : align256(ex.ao * 8));
  const size_t o_rho = o_tab + align256(ex.tab);
  const size_t o_ws = o_rho + align256(ex.rhos * 8);
  const size_t ws = split ? cfgmm::aodmao2rho_split_workspace(nao, ngrid, nset, blksize)
                          : cfgmm::aodmao2rho_fp64_workspace(nao, ngrid, nset, blksize);
  if ((rc = reserve(st, o_ws + ws)) != CFGMM_OK) return rc;
  char* base = static_cast<char*>(st->buf);
  double* d_dms = reinterpret_cast<double*>(base + o_dms);
  double* d_lhs = reinterpret_cast<double*>(base + o_lhs);
  double* d_rhs = reinterpret_cast<double*>(base + o_rhs);
  uint8_t* d_tab = reinterpret_cast<uint8_t*>(base + o_tab);
  double* d_rho = reinterpret_cast<double*>(base + o_rho);
  if (ex.ao * 8 >= (size_t(64) << 20) && ngrid >= 4 * blksize)
    return aodm_host_blocked(st, rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, nao, ngrid,
                             nset, tab, ldtab, blksize, split, ex, d_dms, d_lhs,
                             same_ao ? d_lhs : d_rhs, d_tab, d_rho, base + o_ws);
  CFGMM_CUDA(cudaMemcpyAsync(d_dms, dms, ex.dms * 8, cudaMemcpyHostToDevice, st->stream));
  CFGMM_CUDA(cudaMemcpyAsync(d_lhs, ao_lhs, ex.ao * 8, cudaMemcpyHostToDevice, st->stream));
  if (!same_ao)
    CFGMM_CUDA(cudaMemcpyAsync(d_rhs, ao_rhs, ex.ao * 8, cudaMemcpyHostToDevice, st->stream));
  CFGMM_CUDA(cudaMemcpyAsync(d_tab, tab, ex.tab, cudaMemcpyHostToDevice, st->stream));
  CFGMM_CUDA(cudaMemcpyAsync(d_rho, rhos, ex.rhos * 8, cudaMemcpyHostToDevice, st->stream));
  if (split) {
    CFGMM_CUDA(cfgmm::aodmao2rho_split_reset_error(st->stream));
    CFGMM_CUDA(cfgmm::aodmao2rho_split(d_rho, d_dms, d_lhs, same_ao ? d_lhs : d_rhs, stride_ao,
                                       stride_grid, int(nao), int(ngrid), int(nset), d_tab, ldtab,
                                       int(blksize), base + o_ws, st->stream));
  } else {
    CFGMM_CUDA(cfgmm::aodmao2rho_fp64(d_rho, d_dms, d_lhs, same_ao ? d_lhs : d_rhs, stride_ao,
                                      stride_grid, int(nao), int(ngrid), int(nset), d_tab, ldtab,
                                      int(blksize), base + o_ws, st->stream));
  }
  CFGMM_CUDA(cudaMemcpyAsync(rhos, d_rho, ex.rhos * 8, cudaMemcpyDeviceToHost, st->stream));
  CFGMM_CUDA(cudaStreamSynchronize(st->stream));
  if (split) return check_device_waits();
  int code = 0;
  CFGMM_CUDA(cfgmm::aodm_read_error(&code));
  if (code != 0) {
    char msg[128];
    std::snprintf(msg, sizeof(msg), "a pipeline wait of the FP64 kernel timed out (code %d)", code);
    return fail(CFGMM_ERR_TIMEOUT, msg);
  }
  return CFGMM_OK;
}

// ---------------------------------------------------------------------------
// Fock-build contraction (the transpose of AO-DM-AO): V_s += phi_lhs diag(w_s) phi_rhs^T
// over the AO pairs active in each block.  Same layouts as AO-DM-AO, with the
// weights w in rho's place and V in D's place.
// ---------------------------------------------------------------------------
int check_fock(double* vs, size_t vs_len, const double* ws, size_t ws_len, const double* ao_lhs,
               size_t ao_lhs_len, const double* ao_rhs, size_t ao_rhs_len, size_t stride_ao,
               size_t stride_grid, size_t nao, size_t ngrid, size_t nset, const uint8_t* tab,
               size_t tab_len, size_t ldtab, size_t blksize, AodmExtents* ex) {
  if (nao > 0 && stride_ao < nao)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "stride_ao < nao: rows of V would overlap");
  // w has rho's shape and V has D's: the AO-DM-AO checks cover both
  const int rc = check_aodm(const_cast<double*>(ws), ws_len, vs, vs_len, ao_lhs, ao_lhs_len,
                            ao_rhs, ao_rhs_len, stride_ao, stride_grid, nao, ngrid, nset, tab,
                            tab_len, ldtab, blksize, ex);
  if (rc != CFGMM_OK && g_last_error.find("slice too short") == 0)
    g_last_error = "slice too short (in the names of this message, rhos = w and dms = V)" +
                   g_last_error.substr(std::string("slice too short").size());
  return rc;
}

// The compacted form (fock.cu) unless CFGMM_FOCK_DENSE=1 selects the dense
// product with K-step skipping (dgemm_fp64.cu).
bool fock_dense() {
  static const bool on = [] {
    const char* e = std::getenv("CFGMM_FOCK_DENSE");
    return e && e[0] == '1';
  }();
  return on;
}

size_t fock_workspace(size_t nao, size_t ngrid, size_t nset, size_t blksize) {
  return fock_dense() ? cfgmm::fock_fp64_workspace(int(nao), int(ngrid))
                      : cfgmm::fock_compact_workspace(nao, ngrid, nset, blksize);
}

int fock_run(double* d_v, const double* d_w, const double* d_lhs, const double* d_rhs,
             size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
             const uint8_t* d_tab, size_t ldtab, size_t blksize, void* ws, cudaStream_t s) {
  if (!fock_dense()) {
    CFGMM_CUDA(cfgmm::fock_compact_fp64(d_v, d_w, d_lhs, d_rhs, stride_ao, stride_grid,
                                        int(nao), int(ngrid), int(nset), d_tab, ldtab,
                                        int(blksize), ws, s));
    return CFGMM_OK;
  }
  CFGMM_CUDA(cfgmm::dgemm_reset_error(s));
  for (size_t set = 0; set < nset; ++set)
    CFGMM_CUDA(cfgmm::fock_fp64(d_v + set * stride_ao * stride_ao, stride_ao,
                                d_w + set * stride_grid, d_lhs, d_rhs, stride_grid, int(nao),
                                int(ngrid), d_tab, ldtab, int(blksize), set == 0, ws, s));
  return CFGMM_OK;
}

int fock_host(double* vs, size_t vs_len, const double* ws, size_t ws_len, const double* ao_lhs,
              size_t ao_lhs_len, const double* ao_rhs, size_t ao_rhs_len, size_t stride_ao,
              size_t stride_grid, size_t nao, size_t ngrid, size_t nset, const uint8_t* tab,
              size_t tab_len, size_t ldtab, size_t blksize) {
  g_last_error.clear();
  AodmExtents ex;
  int rc = check_fock(vs, vs_len, ws, ws_len, ao_lhs, ao_lhs_len, ao_rhs, ao_rhs_len, stride_ao,
                      stride_grid, nao, ngrid, nset, tab, tab_len, ldtab, blksize, &ex);
  if (rc != CFGMM_OK) return rc;
  if (ex.rhos == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  DeviceState* st = device_state(dev);
  std::lock_guard<std::mutex> lk(st->mu);
  const bool same_ao = ao_lhs == ao_rhs;
  const size_t o_w = 0;
  const size_t o_lhs = o_w + align256(ex.rhos * 8);
  const size_t o_rhs = o_lhs + align256(ex.ao * 8);
  const size_t o_tab = o_rhs + (same_ao ? 0 : align256(ex.ao * 8));
  const size_t o_v = o_tab + align256(ex.tab);
  const size_t o_ws = o_v + align256(ex.dms * 8);
  if ((rc = reserve(st, o_ws + fock_workspace(nao, ngrid, nset, blksize))) != CFGMM_OK) return rc;
  char* base = static_cast<char*>(st->buf);
  double* d_w = reinterpret_cast<double*>(base + o_w);
  double* d_lhs = reinterpret_cast<double*>(base + o_lhs);
  double* d_rhs = reinterpret_cast<double*>(base + o_rhs);
  uint8_t* d_tab = reinterpret_cast<uint8_t*>(base + o_tab);
  double* d_v = reinterpret_cast<double*>(base + o_v);
  CFGMM_CUDA(cudaMemcpyAsync(d_w, ws, ex.rhos * 8, cudaMemcpyHostToDevice, st->stream));
  CFGMM_CUDA(cudaMemcpyAsync(d_lhs, ao_lhs, ex.ao * 8, cudaMemcpyHostToDevice, st->stream));
  if (!same_ao)
    CFGMM_CUDA(cudaMemcpyAsync(d_rhs, ao_rhs, ex.ao * 8, cudaMemcpyHostToDevice, st->stream));
  CFGMM_CUDA(cudaMemcpyAsync(d_tab, tab, ex.tab, cudaMemcpyHostToDevice, st->stream));
  CFGMM_CUDA(cudaMemcpyAsync(d_v, vs, ex.dms * 8, cudaMemcpyHostToDevice, st->stream));
  if ((rc = fock_run(d_v, d_w, d_lhs, same_ao ? d_lhs : d_rhs, stride_ao, stride_grid, nao, ngrid,
                     nset, d_tab, ldtab, blksize, base + o_ws, st->stream)) != CFGMM_OK)
    return rc;
  CFGMM_CUDA(cudaMemcpyAsync(vs, d_v, ex.dms * 8, cudaMemcpyDeviceToHost, st->stream));
  CFGMM_CUDA(cudaStreamSynchronize(st->stream));
  return check_device_waits();
}

// ---------------------------------------------------------------------------
// f32 forms: operands widened exactly to f64 in stream-ordered scratch, the f64
// kernels, the result rounded back to f32 once.
// ---------------------------------------------------------------------------
struct StreamScratch {
  cudaStream_t s;
  std::vector<void*> blocks;
  explicit StreamScratch(cudaStream_t st) : s(st) {}
  ~StreamScratch() {
    for (void* q : blocks) cudaFreeAsync(q, s);
  }
  cudaError_t get(void** out, size_t bytes) {
    const cudaError_t e = cudaMallocAsync(out, bytes > 0 ? bytes : 1, s);
    if (e == cudaSuccess) blocks.push_back(*out);
    return e;
  }
};

constexpr int kF32OperandBits = 26;  // f32 mantissa (24 bits) and two guard bits

int matmul_f32_run(float* c, const float* a, const float* b, size_t m, size_t n, size_t k,
                   size_t lda, size_t ldb, size_t ldc, bool ta, bool tb, const GemmExtents& ex,
                   int precision, cudaStream_t s) {
  StreamScratch sc(s);
  double *da = nullptr, *db = nullptr, *dc = nullptr;
  CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&da), ex.a * 8));
  CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&db), ex.b * 8));
  CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&dc), ex.c * 8));
  CFGMM_CUDA(cfgmm::widen_f32(a, da, ex.a, s));
  CFGMM_CUDA(cfgmm::widen_f32(b, db, ex.b, s));
  CFGMM_CUDA(cfgmm::widen_f32(c, dc, ex.c, s));
  if (precision == CFGMM_PREC_OZAKI_INT8) {
    const int nmod = cfgmm::ozaki_moduli_for_bits(int(k), kF32OperandBits);
    void* ws = nullptr;
    CFGMM_CUDA(sc.get(&ws, cfgmm::ozaki_dgemm_workspace(int(m), int(n), int(k), nmod)));
    CFGMM_CUDA(cfgmm::ozaki_dgemm(dc, da, db, int(m), int(n), int(k), lda, ldb, ldc, ta, tb, nmod,
                                  ws, s));
  } else {
    CFGMM_CUDA(cfgmm::dgemm_fp64(dc, da, db, int(m), int(n), int(k), lda, ldb, ldc, ta, tb, s));
  }
  CFGMM_CUDA(cfgmm::narrow_f64(dc, c, ex.c, s));
  return CFGMM_OK;
}

int aodm_f32_run(float* rhos, const float* dms, const float* ao_lhs, const float* ao_rhs,
                 size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
                 const uint8_t* tab, size_t ldtab, size_t blksize, const AodmExtents& ex,
                 int precision, cudaStream_t s) {
  StreamScratch sc(s);
  const bool same_ao = ao_lhs == ao_rhs;
  double *d_rho = nullptr, *d_dms = nullptr, *d_lhs = nullptr, *d_rhs = nullptr;
  CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_rho), ex.rhos * 8));
  CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_dms), ex.dms * 8));
  CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_lhs), ex.ao * 8));
  if (!same_ao) CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_rhs), ex.ao * 8));
  CFGMM_CUDA(cfgmm::widen_f32(rhos, d_rho, ex.rhos, s));
  CFGMM_CUDA(cfgmm::widen_f32(dms, d_dms, ex.dms, s));
  CFGMM_CUDA(cfgmm::widen_f32(ao_lhs, d_lhs, ex.ao, s));
  if (!same_ao) CFGMM_CUDA(cfgmm::widen_f32(ao_rhs, d_rhs, ex.ao, s));
  const bool split = precision == CFGMM_PREC_OZAKI_INT8;
  void* ws = nullptr;
  CFGMM_CUDA(sc.get(&ws, split ? cfgmm::aodmao2rho_split_workspace(nao, ngrid, nset, blksize)
                               : cfgmm::aodmao2rho_fp64_workspace(nao, ngrid, nset, blksize)));
  const double* rhs = same_ao ? d_lhs : d_rhs;
  CFGMM_CUDA(split ? cfgmm::aodmao2rho_split(d_rho, d_dms, d_lhs, rhs, stride_ao, stride_grid,
                                             int(nao), int(ngrid), int(nset), tab, ldtab,
                                             int(blksize), ws, s)
                   : cfgmm::aodmao2rho_fp64(d_rho, d_dms, d_lhs, rhs, stride_ao, stride_grid,
                                            int(nao), int(ngrid), int(nset), tab, ldtab,
                                            int(blksize), ws, s));
  CFGMM_CUDA(cfgmm::narrow_f64(d_rho, rhos, ex.rhos, s));
  return CFGMM_OK;
}

}  // namespace

namespace cfgmm {
// Lets entry points defined in other translation units report a detail
// message through cfgmm_last_error().
void set_last_error(const std::string& msg) { g_last_error = msg; }

// The argument checks of cfgmm_aodmao2rho_dev (device pointers: no slice
// lengths, so every length is unbounded) for entry points in other
// translation units; sets the detail message on failure.
int check_aodm_dev(const void* rhos, const void* dms, const void* ao_lhs, const void* ao_rhs,
                   size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
                   const uint8_t* tab, size_t ldtab, size_t blksize) {
  AodmExtents ex;
  return check_aodm(rhos, SIZE_MAX, dms, SIZE_MAX, ao_lhs, SIZE_MAX, ao_rhs, SIZE_MAX, stride_ao,
                    stride_grid, nao, ngrid, nset, tab, SIZE_MAX, ldtab, blksize, &ex);
}
}  // namespace cfgmm

extern "C" {

const char* cfgmm_status_string(int status) {
  switch (status) {
    case CFGMM_OK: return "success";
    case CFGMM_ERR_INVALID_ARGUMENT: return "invalid argument (the reference would panic)";
    case CFGMM_ERR_UNIMPLEMENTED: return "not implemented (the reference's unimplemented!)";
    case CFGMM_ERR_CUDA: return "CUDA runtime error";
    case CFGMM_ERR_NO_DEVICE: return "no CUDA device";
    case CFGMM_ERR_OUT_OF_MEMORY: return "device out of memory";
    case CFGMM_ERR_TIMEOUT: return "device-side wait timed out";
    case CFGMM_ERR_BUSY: return "busy: request refused";
    default: return "unknown status";
  }
}

const char* cfgmm_last_error(void) { return g_last_error.c_str(); }

int cfgmm_version(void) { return 100; }

int cfgmm_matmul_loop_parallel_mnk_pack_a(double* c, size_t c_len, const double* a, size_t a_len,
                                          const double* b, size_t b_len, size_t m, size_t n,
                                          size_t k, size_t lda, size_t ldb, size_t ldc,
                                          uint8_t transa, uint8_t transb) {
  return gemm_host(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa, transb,
                   CFGMM_PREC_FP64);
}

int cfgmm_matmul_anyway_full(double* c, size_t c_len, const double* a, size_t a_len,
                             const double* b, size_t b_len, size_t m, size_t n, size_t k,
                             size_t lda, size_t ldb, size_t ldc, uint8_t transa, uint8_t transb) {
  return gemm_host(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa, transb,
                   CFGMM_PREC_FP64);
}

int cfgmm_matmul_loop_macro_mb(double* c, size_t c_len, const double* a, size_t a_len,
                               const double* b, size_t b_len, size_t m, size_t n, size_t k,
                               size_t lda, size_t ldb, size_t ldc, uint8_t transa,
                               uint8_t transb) {
  return gemm_host(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa, transb,
                   CFGMM_PREC_FP64);
}

int cfgmm_matmul_ex(double* c, size_t c_len, const double* a, size_t a_len, const double* b,
                    size_t b_len, size_t m, size_t n, size_t k, size_t lda, size_t ldb,
                    size_t ldc, uint8_t transa, uint8_t transb, int precision) {
  return gemm_host(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa, transb,
                   precision);
}

int cfgmm_matmul_dev(double* c, const double* a, const double* b, size_t m, size_t n, size_t k,
                     size_t lda, size_t ldb, size_t ldc, uint8_t transa, uint8_t transb,
                     int precision, void* stream) {
  g_last_error.clear();
  GemmExtents ex;
  int rc = check_gemm(c, SIZE_MAX, a, SIZE_MAX, b, SIZE_MAX, m, n, k, lda, ldb, ldc, transa != 0,
                      transb != 0, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  if (ex.c == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == CFGMM_PREC_OZAKI_INT8) {
    if ((rc = check_split_gemm(k)) != CFGMM_OK) return rc;
    const int nmod = cfgmm::ozaki_default_moduli(int(k));
    void* ws = nullptr;
    CFGMM_CUDA(cudaMallocAsync(&ws, cfgmm::ozaki_dgemm_workspace(int(m), int(n), int(k), nmod), s));
    cudaError_t err = cfgmm::ozaki_dgemm(c, a, b, int(m), int(n), int(k), lda, ldb, ldc,
                                         transa != 0, transb != 0, nmod, ws, s);
    cudaError_t err2 = cudaFreeAsync(ws, s);
    if (err != cudaSuccess) return cuda_fail(err, "ozaki_dgemm");
    if (err2 != cudaSuccess) return cuda_fail(err2, "cudaFreeAsync");
    return CFGMM_OK;
  }
  CFGMM_CUDA(cfgmm::dgemm_fp64(c, a, b, int(m), int(n), int(k), lda, ldb, ldc, transa != 0,
                               transb != 0, s));
  return CFGMM_OK;
}

int cfgmm_matmul_anyway_full_non0tab(double* c, size_t c_len, const double* a, size_t a_len,
                                     const double* b, size_t b_len, size_t m, size_t n, size_t k,
                                     size_t lda, size_t ldb, size_t ldc, uint8_t transa,
                                     uint8_t transb, const uint8_t* tab, size_t tab_len,
                                     size_t ldtab) {
  return gemm_host(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa, transb,
                   CFGMM_PREC_FP64, GemmMask{tab, tab_len, ldtab, 48});
}

int cfgmm_matmul_loop_parallel_mnk_pack_a_non0tab(double* c, size_t c_len, const double* a,
                                                  size_t a_len, const double* b, size_t b_len,
                                                  size_t m, size_t n, size_t k, size_t lda,
                                                  size_t ldb, size_t ldc, uint8_t transa,
                                                  uint8_t transb, const uint8_t* tab,
                                                  size_t tab_len, size_t ldtab, size_t blksize) {
  return gemm_host(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa, transb,
                   CFGMM_PREC_FP64, GemmMask{tab, tab_len, ldtab, blksize});
}

int cfgmm_matmul_non0tab_ex(double* c, size_t c_len, const double* a, size_t a_len,
                            const double* b, size_t b_len, size_t m, size_t n, size_t k,
                            size_t lda, size_t ldb, size_t ldc, uint8_t transa, uint8_t transb,
                            const uint8_t* tab, size_t tab_len, size_t ldtab, size_t blksize,
                            int precision) {
  return gemm_host(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa, transb,
                   precision, GemmMask{tab, tab_len, ldtab, blksize});
}

int cfgmm_matmul_non0tab_dev(double* c, const double* a, const double* b, size_t m, size_t n,
                             size_t k, size_t lda, size_t ldb, size_t ldc, uint8_t transa,
                             uint8_t transb, const uint8_t* tab, size_t ldtab, size_t blksize,
                             int precision, void* stream) {
  g_last_error.clear();
  size_t tab_ext = 0;
  int rc = check_mask(GemmMask{tab, SIZE_MAX, ldtab, blksize}, n, k, transb, &tab_ext);
  if (rc != CFGMM_OK) return rc;
  GemmExtents ex;
  rc = check_gemm(c, SIZE_MAX, a, SIZE_MAX, b, SIZE_MAX, m, n, k, lda, ldb, ldc, transa != 0,
                  false, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  if (ex.c == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == CFGMM_PREC_OZAKI_INT8) {
    if ((rc = check_split_gemm(k)) != CFGMM_OK) return rc;
    const int nmod = cfgmm::ozaki_default_moduli(int(k));
    void* ws = nullptr;
    CFGMM_CUDA(cudaMallocAsync(&ws, cfgmm::ozaki_dgemm_workspace(int(m), int(n), int(k), nmod), s));
    cudaError_t err = cfgmm::ozaki_dgemm(c, a, b, int(m), int(n), int(k), lda, ldb, ldc,
                                         transa != 0, false, nmod, ws, s, nullptr, tab, ldtab,
                                         int(blksize));
    cudaError_t err2 = cudaFreeAsync(ws, s);
    if (err != cudaSuccess) return cuda_fail(err, "ozaki_dgemm (masked)");
    if (err2 != cudaSuccess) return cuda_fail(err2, "cudaFreeAsync");
    return CFGMM_OK;
  }
  CFGMM_CUDA(cfgmm::dgemm_fp64_non0tab(c, a, b, int(m), int(n), int(k), lda, ldb, ldc,
                                       transa != 0, tab, ldtab, int(blksize), s));
  return CFGMM_OK;
}

int cfgmm_matmul_dev_timed(double* c, const double* a, const double* b, size_t m, size_t n,
                           size_t k, size_t lda, size_t ldb, size_t ldc, uint8_t transa,
                           uint8_t transb, int precision, void* stream, void* const* events,
                           int nevents) {
  g_last_error.clear();
  const int need = precision == CFGMM_PREC_OZAKI_INT8 ? 4 : 2;
  if (!events || nevents != need)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "events: 2 for FP64, 4 for OZAKI_INT8");
  GemmExtents ex;
  int rc = check_gemm(c, SIZE_MAX, a, SIZE_MAX, b, SIZE_MAX, m, n, k, lda, ldb, ldc, transa != 0,
                      transb != 0, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  if (ex.c == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const cudaEvent_t* ev = reinterpret_cast<const cudaEvent_t*>(events);
  if (precision == CFGMM_PREC_OZAKI_INT8) {
    if ((rc = check_split_gemm(k)) != CFGMM_OK) return rc;
    const int nmod = cfgmm::ozaki_default_moduli(int(k));
    void* ws = nullptr;
    CFGMM_CUDA(cudaMallocAsync(&ws, cfgmm::ozaki_dgemm_workspace(int(m), int(n), int(k), nmod), s));
    cudaError_t err = cfgmm::ozaki_dgemm(c, a, b, int(m), int(n), int(k), lda, ldb, ldc,
                                         transa != 0, transb != 0, nmod, ws, s, ev);
    cudaError_t err2 = cudaFreeAsync(ws, s);
    if (err != cudaSuccess) return cuda_fail(err, "ozaki_dgemm");
    if (err2 != cudaSuccess) return cuda_fail(err2, "cudaFreeAsync");
    return CFGMM_OK;
  }
  CFGMM_CUDA(cudaEventRecord(ev[0], s));
  CFGMM_CUDA(cfgmm::dgemm_fp64(c, a, b, int(m), int(n), int(k), lda, ldb, ldc, transa != 0,
                               transb != 0, s));
  CFGMM_CUDA(cudaEventRecord(ev[1], s));
  return CFGMM_OK;
}

int cfgmm_split_moduli(size_t k) { return cfgmm::ozaki_default_moduli(int(k > 65536 ? 65536 : k)); }

int cfgmm_test_arm_wait_timeout(int precision, double wait_ms) {
  g_last_error.clear();
  int rc = check_precision(precision);
  if (rc != CFGMM_OK) return rc;
  if (!(wait_ms >= 1.0 && wait_ms <= 2000.0))
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "wait_ms must lie in [1, 2000]");
  cfgmm::arm_wait_injection(precision == CFGMM_PREC_OZAKI_INT8 ? 1 : 0,
                            static_cast<unsigned long long>(wait_ms * 1e6));
  return CFGMM_OK;
}

int cfgmm_device_check(void) {
  g_last_error.clear();
  int dev;
  int rc = current_device(&dev);
  if (rc != CFGMM_OK) return rc;
  CFGMM_CUDA(cudaDeviceSynchronize());
  return check_device_waits();
}

int cfgmm_aodmao2rho_loop_parallel(double* rhos, size_t rhos_len, const double* dms,
                                   size_t dms_len, const double* ao_lhs, size_t ao_lhs_len,
                                   const double* ao_rhs, size_t ao_rhs_len, size_t stride_ao,
                                   size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
                                   const uint8_t* tab, size_t tab_len, size_t ldtab,
                                   size_t blksize) {
  return aodm_host(rhos, rhos_len, dms, dms_len, ao_lhs, ao_lhs_len, ao_rhs, ao_rhs_len,
                   stride_ao, stride_grid, nao, ngrid, nset, tab, tab_len, ldtab, blksize,
                   CFGMM_PREC_FP64);
}

int cfgmm_aodmao2rho_anyway(double* rhos, size_t rhos_len, const double* dms, size_t dms_len,
                            const double* ao_lhs, size_t ao_lhs_len, const double* ao_rhs,
                            size_t ao_rhs_len, size_t stride_ao, size_t stride_grid, size_t nao,
                            size_t ngrid, size_t nset, const uint8_t* tab, size_t tab_len,
                            size_t ldtab) {
  return aodm_host(rhos, rhos_len, dms, dms_len, ao_lhs, ao_lhs_len, ao_rhs, ao_rhs_len,
                   stride_ao, stride_grid, nao, ngrid, nset, tab, tab_len, ldtab, 48,
                   CFGMM_PREC_FP64);
}

int cfgmm_aodmao2rho_ex(double* rhos, size_t rhos_len, const double* dms, size_t dms_len,
                        const double* ao_lhs, size_t ao_lhs_len, const double* ao_rhs,
                        size_t ao_rhs_len, size_t stride_ao, size_t stride_grid, size_t nao,
                        size_t ngrid, size_t nset, const uint8_t* tab, size_t tab_len,
                        size_t ldtab, size_t blksize, int precision) {
  return aodm_host(rhos, rhos_len, dms, dms_len, ao_lhs, ao_lhs_len, ao_rhs, ao_rhs_len,
                   stride_ao, stride_grid, nao, ngrid, nset, tab, tab_len, ldtab, blksize,
                   precision);
}

int cfgmm_aodmao2rho_dev(double* rhos, const double* dms, const double* ao_lhs,
                         const double* ao_rhs, size_t stride_ao, size_t stride_grid, size_t nao,
                         size_t ngrid, size_t nset, const uint8_t* tab, size_t ldtab,
                         size_t blksize, int precision, void* stream) {
  g_last_error.clear();
  AodmExtents ex;
  int rc = check_aodm(rhos, SIZE_MAX, dms, SIZE_MAX, ao_lhs, SIZE_MAX, ao_rhs, SIZE_MAX,
                      stride_ao, stride_grid, nao, ngrid, nset, tab, SIZE_MAX, ldtab, blksize, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  const bool split = precision == CFGMM_PREC_OZAKI_INT8;
  if (split && nao > 16384)
    return fail(CFGMM_ERR_UNIMPLEMENTED, "split-precision AO-DM-AO supports nao <= 16384");
  if (ex.rhos == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Stream-ordered scratch: safe against concurrent calls on other streams.
  void* ws = nullptr;
  const size_t bytes = split ? cfgmm::aodmao2rho_split_workspace(nao, ngrid, nset, blksize)
                             : cfgmm::aodmao2rho_fp64_workspace(nao, ngrid, nset, blksize);
  CFGMM_CUDA(cudaMallocAsync(&ws, bytes, s));
  cudaError_t err =
      split ? cfgmm::aodmao2rho_split(rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, int(nao),
                                      int(ngrid), int(nset), tab, ldtab, int(blksize), ws, s)
            : cfgmm::aodmao2rho_fp64(rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, int(nao),
                                     int(ngrid), int(nset), tab, ldtab, int(blksize), ws, s);
  cudaError_t err2 = cudaFreeAsync(ws, s);
  if (err != cudaSuccess) return cuda_fail(err, "aodmao2rho_fp64");
  if (err2 != cudaSuccess) return cuda_fail(err2, "cudaFreeAsync");
  return CFGMM_OK;
}

int cfgmm_eval_ao_dev(double* ao, size_t stride_grid, const double* points, size_t ngrid,
                      const double* shell_xyz, const int* shell_l, const double* shell_alpha,
                      const double* shell_norm, const int* shell_row, size_t nshell,
                      double* shell_block_max, size_t blksize, void* stream) {
  g_last_error.clear();
  if (ngrid == 0 || nshell == 0) return CFGMM_OK;
  if (!ao || !points || !shell_xyz || !shell_l || !shell_alpha || !shell_norm || !shell_row)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  if (stride_grid < ngrid || !fits_int(ngrid) || nshell > 65535 || blksize == 0 ||
      !fits_int(blksize))
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "invalid sizes");
  int dev;
  int rc = current_device(&dev);
  if (rc != CFGMM_OK) return rc;
  CFGMM_CUDA(cfgmm::eval_ao(ao, stride_grid, points, int(ngrid), shell_xyz, shell_l, shell_alpha,
                            shell_norm, shell_row, int(nshell), shell_block_max, int(blksize),
                            static_cast<cudaStream_t>(stream)));
  return CFGMM_OK;
}

int cfgmm_mask_ao_dev(double* ao, size_t stride_grid, size_t ngrid, const int* shell_l,
                      const int* shell_row, size_t nshell, const double* shell_block_max,
                      double threshold, uint8_t* tab, size_t ldtab, size_t blksize, void* stream) {
  g_last_error.clear();
  if (ngrid == 0 || nshell == 0) return CFGMM_OK;
  if (!ao || !shell_l || !shell_row || !shell_block_max || !tab)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "null pointer");
  if (stride_grid < ngrid || !fits_int(ngrid) || nshell > 65535 || blksize == 0 ||
      !fits_int(blksize) || ldtab < (ngrid + blksize - 1) / blksize)
    return fail(CFGMM_ERR_INVALID_ARGUMENT, "invalid sizes");
  int dev;
  int rc = current_device(&dev);
  if (rc != CFGMM_OK) return rc;
  CFGMM_CUDA(cfgmm::mask_ao(ao, stride_grid, int(ngrid), shell_l, shell_row, int(nshell),
                            shell_block_max, threshold, tab, ldtab, int(blksize),
                            static_cast<cudaStream_t>(stream)));
  return CFGMM_OK;
}

int cfgmm_aodm_fock(double* vs, size_t vs_len, const double* ws, size_t ws_len,
                    const double* ao_lhs, size_t ao_lhs_len, const double* ao_rhs,
                    size_t ao_rhs_len, size_t stride_ao, size_t stride_grid, size_t nao,
                    size_t ngrid, size_t nset, const uint8_t* tab, size_t tab_len, size_t ldtab,
                    size_t blksize) {
  return fock_host(vs, vs_len, ws, ws_len, ao_lhs, ao_lhs_len, ao_rhs, ao_rhs_len, stride_ao,
                   stride_grid, nao, ngrid, nset, tab, tab_len, ldtab, blksize);
}

int cfgmm_aodm_fock_dev(double* vs, const double* ws, const double* ao_lhs, const double* ao_rhs,
                        size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid,
                        size_t nset, const uint8_t* tab, size_t ldtab, size_t blksize,
                        void* stream) {
  g_last_error.clear();
  AodmExtents ex;
  int rc = check_fock(vs, SIZE_MAX, ws, SIZE_MAX, ao_lhs, SIZE_MAX, ao_rhs, SIZE_MAX, stride_ao,
                      stride_grid, nao, ngrid, nset, tab, SIZE_MAX, ldtab, blksize, &ex);
  if (rc != CFGMM_OK) return rc;
  if (ex.rhos == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  void* work = nullptr;
  CFGMM_CUDA(cudaMallocAsync(&work, fock_workspace(nao, ngrid, nset, blksize), s));
  rc = fock_run(vs, ws, ao_lhs, ao_rhs, stride_ao, stride_grid, nao, ngrid, nset, tab, ldtab,
                blksize, work, s);
  const cudaError_t e2 = cudaFreeAsync(work, s);
  if (rc != CFGMM_OK) return rc;
  if (e2 != cudaSuccess) return cuda_fail(e2, "cudaFreeAsync");
  return CFGMM_OK;
}

int cfgmm_matmul_f32(float* c, size_t c_len, const float* a, size_t a_len, const float* b,
                     size_t b_len, size_t m, size_t n, size_t k, size_t lda, size_t ldb,
                     size_t ldc, uint8_t transa, uint8_t transb, int precision) {
  g_last_error.clear();
  GemmExtents ex;
  int rc = check_gemm(c, c_len, a, a_len, b, b_len, m, n, k, lda, ldb, ldc, transa != 0,
                      transb != 0, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  if (ex.c == 0) return CFGMM_OK;
  if (precision == CFGMM_PREC_OZAKI_INT8 && (rc = check_split_gemm(k)) != CFGMM_OK) return rc;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  DeviceState* st = device_state(dev);
  std::lock_guard<std::mutex> lk(st->mu);
  cudaStream_t s = st->stream;
  {
    StreamScratch sc(s);
    float *da = nullptr, *db = nullptr, *dc = nullptr;
    CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&da), ex.a * 4));
    CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&db), ex.b * 4));
    CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&dc), ex.c * 4));
    CFGMM_CUDA(cudaMemcpyAsync(da, a, ex.a * 4, cudaMemcpyHostToDevice, s));
    CFGMM_CUDA(cudaMemcpyAsync(db, b, ex.b * 4, cudaMemcpyHostToDevice, s));
    CFGMM_CUDA(cudaMemcpyAsync(dc, c, ex.c * 4, cudaMemcpyHostToDevice, s));
    if (precision == CFGMM_PREC_OZAKI_INT8) CFGMM_CUDA(cfgmm::gemm_i8_reset_error(s));
    if ((rc = matmul_f32_run(dc, da, db, m, n, k, lda, ldb, ldc, transa != 0, transb != 0, ex,
                             precision, s)) != CFGMM_OK)
      return rc;
    CFGMM_CUDA(cudaMemcpyAsync(c, dc, ex.c * 4, cudaMemcpyDeviceToHost, s));
  }
  CFGMM_CUDA(cudaStreamSynchronize(s));
  return check_device_waits();
}

int cfgmm_matmul_f32_dev(float* c, const float* a, const float* b, size_t m, size_t n, size_t k,
                         size_t lda, size_t ldb, size_t ldc, uint8_t transa, uint8_t transb,
                         int precision, void* stream) {
  g_last_error.clear();
  GemmExtents ex;
  int rc = check_gemm(c, SIZE_MAX, a, SIZE_MAX, b, SIZE_MAX, m, n, k, lda, ldb, ldc, transa != 0,
                      transb != 0, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  if (ex.c == 0) return CFGMM_OK;
  if (precision == CFGMM_PREC_OZAKI_INT8 && (rc = check_split_gemm(k)) != CFGMM_OK) return rc;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  return matmul_f32_run(c, a, b, m, n, k, lda, ldb, ldc, transa != 0, transb != 0, ex, precision,
                        static_cast<cudaStream_t>(stream));
}

int cfgmm_aodmao2rho_f32(float* rhos, size_t rhos_len, const float* dms, size_t dms_len,
                         const float* ao_lhs, size_t ao_lhs_len, const float* ao_rhs,
                         size_t ao_rhs_len, size_t stride_ao, size_t stride_grid, size_t nao,
                         size_t ngrid, size_t nset, const uint8_t* tab, size_t tab_len,
                         size_t ldtab, size_t blksize, int precision) {
  g_last_error.clear();
  AodmExtents ex;
  int rc = check_aodm(rhos, rhos_len, dms, dms_len, ao_lhs, ao_lhs_len, ao_rhs, ao_rhs_len,
                      stride_ao, stride_grid, nao, ngrid, nset, tab, tab_len, ldtab, blksize, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  const bool split = precision == CFGMM_PREC_OZAKI_INT8;
  if (split && nao > 16384)
    return fail(CFGMM_ERR_UNIMPLEMENTED, "split-precision AO-DM-AO supports nao <= 16384");
  if (ex.rhos == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  DeviceState* st = device_state(dev);
  std::lock_guard<std::mutex> lk(st->mu);
  cudaStream_t s = st->stream;
  const bool same_ao = ao_lhs == ao_rhs;
  {
    StreamScratch sc(s);
    float *d_rho = nullptr, *d_dms = nullptr, *d_lhs = nullptr, *d_rhs = nullptr;
    uint8_t* d_tab = nullptr;
    CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_rho), ex.rhos * 4));
    CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_dms), ex.dms * 4));
    CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_lhs), ex.ao * 4));
    if (!same_ao) CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_rhs), ex.ao * 4));
    CFGMM_CUDA(sc.get(reinterpret_cast<void**>(&d_tab), ex.tab));
    CFGMM_CUDA(cudaMemcpyAsync(d_rho, rhos, ex.rhos * 4, cudaMemcpyHostToDevice, s));
    CFGMM_CUDA(cudaMemcpyAsync(d_dms, dms, ex.dms * 4, cudaMemcpyHostToDevice, s));
    CFGMM_CUDA(cudaMemcpyAsync(d_lhs, ao_lhs, ex.ao * 4, cudaMemcpyHostToDevice, s));
    if (!same_ao)
      CFGMM_CUDA(cudaMemcpyAsync(d_rhs, ao_rhs, ex.ao * 4, cudaMemcpyHostToDevice, s));
    CFGMM_CUDA(cudaMemcpyAsync(d_tab, tab, ex.tab, cudaMemcpyHostToDevice, s));
    if (split) CFGMM_CUDA(cfgmm::aodmao2rho_split_reset_error(s));
    if ((rc = aodm_f32_run(d_rho, d_dms, d_lhs, same_ao ? d_lhs : d_rhs, stride_ao, stride_grid,
                           nao, ngrid, nset, d_tab, ldtab, blksize, ex, precision, s)) !=
        CFGMM_OK)
      return rc;
    CFGMM_CUDA(cudaMemcpyAsync(rhos, d_rho, ex.rhos * 4, cudaMemcpyDeviceToHost, s));
  }
  CFGMM_CUDA(cudaStreamSynchronize(s));
  if (split) return check_device_waits();
  int code = 0;
  CFGMM_CUDA(cfgmm::aodm_read_error(&code));
  if (code != 0) return fail(CFGMM_ERR_TIMEOUT, "a pipeline wait of the FP64 kernel timed out");
  return CFGMM_OK;
}

int cfgmm_aodmao2rho_f32_dev(float* rhos, const float* dms, const float* ao_lhs,
                             const float* ao_rhs, size_t stride_ao, size_t stride_grid,
                             size_t nao, size_t ngrid, size_t nset, const uint8_t* tab,
                             size_t ldtab, size_t blksize, int precision, void* stream) {
  g_last_error.clear();
  AodmExtents ex;
  int rc = check_aodm(rhos, SIZE_MAX, dms, SIZE_MAX, ao_lhs, SIZE_MAX, ao_rhs, SIZE_MAX,
                      stride_ao, stride_grid, nao, ngrid, nset, tab, SIZE_MAX, ldtab, blksize, &ex);
  if (rc != CFGMM_OK) return rc;
  if ((rc = check_precision(precision)) != CFGMM_OK) return rc;
  if (precision == CFGMM_PREC_OZAKI_INT8 && nao > 16384)
    return fail(CFGMM_ERR_UNIMPLEMENTED, "split-precision AO-DM-AO supports nao <= 16384");
  if (ex.rhos == 0) return CFGMM_OK;
  int dev;
  if ((rc = current_device(&dev)) != CFGMM_OK) return rc;
  return aodm_f32_run(rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, nao, ngrid, nset, tab,
                      ldtab, blksize, ex, precision, static_cast<cudaStream_t>(stream));
}

int cfgmm_release_workspace(void) {
  g_last_error.clear();
  int dev;
  int rc = current_device(&dev);
  if (rc != CFGMM_OK) return rc;
  DeviceState* st = device_state(dev);
  std::lock_guard<std::mutex> lk(st->mu);
  if (st->buf) CFGMM_CUDA(cudaFree(st->buf));
  st->buf = nullptr;
  st->cap = 0;
  cfgmm::release_pinned_staging();
  return CFGMM_OK;
}

}  // extern "C"
