/*
 * cfgmm.h -- C ABI of libcfgmm.so, a B200 (sm_100a) implementation of the two
 * data-parallel hot paths of cfgable-matmul:
 *
 *   1. the row-major blocked DGEMM   C += op(A) * op(B)
 *   2. the non0tab-masked AO-DM-AO density contraction
 *        rho[s][g] += sum_{u,v active in g's block} ao_lhs[u][g] * D_s[u][v] * ao_rhs[v][g]
 *
 * Every entry point keeps the argument order and meaning of the Rust function
 * it replaces (cited per declaration, paths relative to the reference crate
 * root).  A Rust `&[T]` / `&mut [T]` slice is passed as (pointer, length); a
 * Rust `bool` is one byte holding 0 or 1, and `&[bool]` is `const uint8_t*`
 * (any nonzero byte counts as true).  `usize` is `size_t`.
 *
 * Semantics shared by every entry point:
 *   - Outputs are ACCUMULATED into (C += ..., rho += ...), exactly as in the
 *     reference (impl_matmul.rs:31-46, impl_aodmao2rho.rs:77-92); the caller
 *     zero-fills when it wants a plain product.
 *   - Host-pointer entry points are synchronous and blocking, like the
 *     reference's calls: inputs are copied to the current CUDA device, the
 *     kernels run, the output is copied back, and the call returns.
 *   - `_dev` entry points take device pointers and a cudaStream_t (passed as
 *     void*, NULL = the legacy default stream) and only enqueue work; they do
 *     not synchronize.
 *   - Where the reference panics (a slice shorter than the index range it
 *     reads or writes, `unimplemented!`, a failed `assert!`), the call returns
 *     a negative status instead and touches no output.
 *   - Zero-sized problems (m, n or k == 0; nao, ngrid or nset == 0) are valid
 *     and leave the output unchanged, as in the reference.
 *   - Calls are thread-safe: per-device workspaces are guarded internally.
 *   - There is no CPU fallback.  Without a usable CUDA device a call returns
 *     CFGMM_ERR_NO_DEVICE.
 */
#ifndef CFGMM_H
#define CFGMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define CFGMM_OK                    0
#define CFGMM_ERR_INVALID_ARGUMENT (-1) /* reference would panic: slice too short, bad BLKSIZE, null */
#define CFGMM_ERR_UNIMPLEMENTED    (-2) /* reference `unimplemented!` (masked GEMM with transb) */
#define CFGMM_ERR_CUDA             (-3) /* CUDA runtime error; see cfgmm_last_error() */
#define CFGMM_ERR_NO_DEVICE        (-4) /* no CUDA device visible */
#define CFGMM_ERR_OUT_OF_MEMORY    (-5) /* device allocation failed */
#define CFGMM_ERR_TIMEOUT          (-6) /* a bounded device-side wait gave up */
#define CFGMM_ERR_BUSY             (-7) /* serving queue full / request refused by the HBM budget */

/* ---- arithmetic of a call ---------------------------------------------- */
#define CFGMM_PREC_FP64        0 /* FP64 tensor-core (DMMA) kernels */
#define CFGMM_PREC_OZAKI_INT8  1 /* Ozaki-style INT8 split-precision kernels (tcgen05) */

/* Short English description of a status code. */
const char* cfgmm_status_string(int status);
/* Detail of the last error raised on the calling thread ("" when none). */
const char* cfgmm_last_error(void);
/* Library version, major * 10000 + minor * 100 + patch. */
int cfgmm_version(void);

/* ======================================================================== */
/* 1. DGEMM  C[i*ldc + j] += sum_p opA(i,p) * opB(p,j)                      */
/*    opA(i,p) = transa ? a[p*lda + i] : a[i*lda + p]                       */
/*    opB(p,j) = transb ? b[j*ldb + p] : b[p*ldb + j]                       */
/* ======================================================================== */

/* Replaces MatmulLoops::<T,MC,KC,NC,MR,NR_LANE,LANE>::matmul_loop_parallel_mnk_pack_a
 * (src/impl_matmul.rs:155-167 signature, 155-231 body).  The CPU const
 * generics have no meaning on the GPU: tiles are chosen by the library. */
int cfgmm_matmul_loop_parallel_mnk_pack_a(double* c, size_t c_len, const double* a, size_t a_len,
                                          const double* b, size_t b_len, size_t m, size_t n,
                                          size_t k, size_t lda, size_t ldb, size_t ldc,
                                          uint8_t transa, uint8_t transb);

/* Replaces matmul_anyway_full (src/impl_matmul.rs:234-248): the same call with
 * the reference's fixed Zen4 tuning; here identical to the entry point above. */
int cfgmm_matmul_anyway_full(double* c, size_t c_len, const double* a, size_t a_len,
                             const double* b, size_t b_len, size_t m, size_t n, size_t k,
                             size_t lda, size_t ldb, size_t ldc, uint8_t transa, uint8_t transb);

/* Replaces MatmulLoops::<f64,MC,KC,NC,MR,NR_LANE,LANE,MB>::matmul_loop_macro_mb as
 * README.md:22-31 documents it (the function is named there but absent from
 * the crate's sources).  Same semantics as matmul_loop_parallel_mnk_pack_a. */
int cfgmm_matmul_loop_macro_mb(double* c, size_t c_len, const double* a, size_t a_len,
                               const double* b, size_t b_len, size_t m, size_t n, size_t k,
                               size_t lda, size_t ldb, size_t ldc, uint8_t transa,
                               uint8_t transb);

/* Host-pointer DGEMM with an explicit arithmetic (CFGMM_PREC_*).  With
 * CFGMM_PREC_FP64 this is cfgmm_matmul_anyway_full. */
int cfgmm_matmul_ex(double* c, size_t c_len, const double* a, size_t a_len, const double* b,
                    size_t b_len, size_t m, size_t n, size_t k, size_t lda, size_t ldb,
                    size_t ldc, uint8_t transa, uint8_t transb, int precision);

/* Device-pointer DGEMM, enqueued on `stream` (cudaStream_t).  Same index
 * semantics as above; the caller guarantees the extents. */
int cfgmm_matmul_dev(double* c, const double* a, const double* b, size_t m, size_t n, size_t k,
                     size_t lda, size_t ldb, size_t ldc, uint8_t transa, uint8_t transb,
                     int precision, void* stream);

/* ---- masked GEMM: C[i*ldc + j] += sum_{p: tab[p*ldtab + j/BLK]} opA(i,p) * b[p*ldb + j] ----
 * Element (p, j) of B takes part only when its (row, column block) flag is
 * set, whatever B holds there (impl_matmul_non0tab.rs:196-207).  B cannot be
 * transposed: transb != 0 returns CFGMM_ERR_UNIMPLEMENTED, as the reference's
 * `unimplemented!` (impl_matmul_non0tab.rs:181-183, 228-230). */

/* Replaces matmul_anyway_full_non0tab (src/impl_matmul_non0tab.rs:308-326): BLKSIZE 48. */
int cfgmm_matmul_anyway_full_non0tab(double* c, size_t c_len, const double* a, size_t a_len,
                                     const double* b, size_t b_len, size_t m, size_t n, size_t k,
                                     size_t lda, size_t ldb, size_t ldc, uint8_t transa,
                                     uint8_t transb, const uint8_t* tab, size_t tab_len,
                                     size_t ldtab);

/* Replaces MatmulLoops::matmul_loop_parallel_mnk_pack_a_non0tab::<BLKSIZE>
 * (src/impl_matmul_non0tab.rs:210-306); any blksize >= 1. */
int cfgmm_matmul_loop_parallel_mnk_pack_a_non0tab(double* c, size_t c_len, const double* a,
                                                  size_t a_len, const double* b, size_t b_len,
                                                  size_t m, size_t n, size_t k, size_t lda,
                                                  size_t ldb, size_t ldc, uint8_t transa,
                                                  uint8_t transb, const uint8_t* tab,
                                                  size_t tab_len, size_t ldtab, size_t blksize);

/* Host-pointer masked GEMM with an explicit arithmetic (CFGMM_PREC_*). */
int cfgmm_matmul_non0tab_ex(double* c, size_t c_len, const double* a, size_t a_len,
                            const double* b, size_t b_len, size_t m, size_t n, size_t k,
                            size_t lda, size_t ldb, size_t ldc, uint8_t transa, uint8_t transb,
                            const uint8_t* tab, size_t tab_len, size_t ldtab, size_t blksize,
                            int precision);

/* Device-pointer masked GEMM enqueued on `stream`; `tab` is a device pointer. */
int cfgmm_matmul_non0tab_dev(double* c, const double* a, const double* b, size_t m, size_t n,
                             size_t k, size_t lda, size_t ldb, size_t ldc, uint8_t transa,
                             uint8_t transb, const uint8_t* tab, size_t ldtab, size_t blksize,
                             int precision, void* stream);

/* No counterpart in the reference: benchmark instrumentation.  The device-
 * pointer DGEMM with CUDA events (cudaEvent_t, passed as void*) recorded on
 * `stream` at its phase boundaries: FP64 -- events[0] before and events[1]
 * after the GEMM kernel (nevents = 2); OZAKI_INT8 -- before the residue
 * preparation, after it, after the INT8 GEMM, after the reconstruction
 * (nevents = 4). */
int cfgmm_matmul_dev_timed(double* c, const double* a, const double* b, size_t m, size_t n,
                           size_t k, size_t lda, size_t ldb, size_t ldc, uint8_t transa,
                           uint8_t transb, int precision, void* stream, void* const* events,
                           int nevents);

/* No counterpart in the reference: the number of INT8 moduli (GEMM passes)
 * the split-precision path uses for contraction length k.  The environment
 * variable CFGMM_OZAKI_MODULI (2..16) overrides the default, which keeps at
 * least 46 bits of every operand relative to its row / column maximum. */
int cfgmm_split_moduli(size_t k);

/* No counterpart in the reference: synchronises the current device and
 * reports CFGMM_ERR_TIMEOUT if a tensor-core pipeline wait of an earlier
 * asynchronous (_dev) call gave up; CFGMM_OK otherwise.  A timeout is reported
 * once: the device's wait words are cleared when it is. */
int cfgmm_device_check(void);

/* No counterpart in the reference: the test hook of the device-side failure
 * detection.  Arms the calling thread's NEXT masked AO-DM-AO contraction in
 * `precision` (CFGMM_PREC_FP64: the pipelined FP64 kernel; OZAKI_INT8: the
 * split pair kernel -- the form of contractions from 1024 AOs and 8192 points
 * on, or of every one under CFGMM_SPLIT_FORM=pair) so that one producer never
 * publishes the first pipeline stage and every wait in the kernel gives up
 * after `wait_ms` (1..2000) milliseconds instead of 2 s.  The waiting warp
 * records a timeout, every warp leaves, copies in flight land, tensor memory
 * is freed and the kernel returns: the call (a host-pointer one) or the next
 * cfgmm_device_check (after a _dev one) returns CFGMM_ERR_TIMEOUT, and the
 * calls after it run normally.  Nothing faults or hangs; the results of the
 * armed call are not defined. */
int cfgmm_test_arm_wait_timeout(int precision, double wait_ms);

/* ======================================================================== */
/* 2. Masked AO-DM-AO contraction                                           */
/*    rhos[s*stride_grid + g] += sum_{u,v: tab[u*ldtab + g/BLK] && tab[v*ldtab + g/BLK]}
 *        ao_lhs[u*stride_grid + g] * dms[s*stride_ao^2 + u*stride_ao + v] * ao_rhs[v*stride_grid + g]
 *    for s < nset, g < ngrid; strides = [stride_ao, stride_grid], shape = [nao, ngrid].
 *    Masked (AO, block) entries are skipped whatever ao_lhs/ao_rhs hold there
 *    (impl_aodmao2rho.rs:128-151).                                         */
/* ======================================================================== */

/* Replaces MatmulLoops::aodmao2rho_loop_parallel::<BLKSIZE>
 * (src/impl_aodmao2rho.rs:171-181 signature, 171-244 body); BLKSIZE is the
 * `blksize` argument.  Any blksize >= 1 is accepted (the reference's own
 * constraints, BLKSIZE % 16 == 0 and NC % BLKSIZE == 0, stem from its CPU
 * tiling and do not apply). */
int cfgmm_aodmao2rho_loop_parallel(double* rhos, size_t rhos_len, const double* dms,
                                   size_t dms_len, const double* ao_lhs, size_t ao_lhs_len,
                                   const double* ao_rhs, size_t ao_rhs_len, size_t stride_ao,
                                   size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
                                   const uint8_t* tab, size_t tab_len, size_t ldtab,
                                   size_t blksize);

/* Replaces aodmao2rho_anyway (src/impl_aodmao2rho.rs:247-261): BLKSIZE 48. */
int cfgmm_aodmao2rho_anyway(double* rhos, size_t rhos_len, const double* dms, size_t dms_len,
                            const double* ao_lhs, size_t ao_lhs_len, const double* ao_rhs,
                            size_t ao_rhs_len, size_t stride_ao, size_t stride_grid, size_t nao,
                            size_t ngrid, size_t nset, const uint8_t* tab, size_t tab_len,
                            size_t ldtab);

/* Host-pointer contraction with an explicit arithmetic (CFGMM_PREC_*). */
int cfgmm_aodmao2rho_ex(double* rhos, size_t rhos_len, const double* dms, size_t dms_len,
                        const double* ao_lhs, size_t ao_lhs_len, const double* ao_rhs,
                        size_t ao_rhs_len, size_t stride_ao, size_t stride_grid, size_t nao,
                        size_t ngrid, size_t nset, const uint8_t* tab, size_t tab_len,
                        size_t ldtab, size_t blksize, int precision);

/* Device-pointer contraction enqueued on `stream`; `tab` is a device pointer. */
int cfgmm_aodmao2rho_dev(double* rhos, const double* dms, const double* ao_lhs,
                         const double* ao_rhs, size_t stride_ao, size_t stride_grid, size_t nao,
                         size_t ngrid, size_t nset, const uint8_t* tab, size_t ldtab,
                         size_t blksize, int precision, void* stream);

/* No counterpart in the reference: an addition for callers that cannot
 * allocate device memory -- a host that has given all of the GPU's memory to
 * its own pool or arena, or code that must not call cudaMalloc/cudaFree (which
 * can synchronise the whole device) inside a time-critical loop.
 * Same arguments and result as cfgmm_aodmao2rho_dev with CFGMM_PREC_FP64, but
 * the scratch it needs (per-block active AO lists, per-row-tile partial sums)
 * lives in one fixed array of CFGMM_NOALLOC_SCRATCH_BYTES inside the library's
 * device image, which every GPU that loads the library holds until exit; the
 * call itself allocates nothing.  A problem whose scratch does not fit is
 * refused with CFGMM_ERR_INVALID_ARGUMENT (the message gives the size it
 * needs).  The first call on a device looks up that device's copy of the
 * array; make that first call before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race and must be ordered by the caller. */
#define CFGMM_NOALLOC_SCRATCH_BYTES (32u << 20)
int cfgmm_aodmao2rho_dev_noalloc(double* rhos, const double* dms, const double* ao_lhs,
                                 const double* ao_rhs, size_t stride_ao, size_t stride_grid,
                                 size_t nao, size_t ngrid, size_t nset, const uint8_t* tab,
                                 size_t ldtab, size_t blksize, void* stream);

/* ---- the step after the contraction: the Fock-build (V) contraction ------
 * No counterpart in the reference (its DFT callers build V themselves); the
 * transpose of AO-DM-AO with the same layouts and mask:
 *   vs[s*stride_ao^2 + u*stride_ao + v] += sum over g with tab[u][g/BLK] and
 *       tab[v][g/BLK] of ao_lhs[u][g] * ws[s*stride_grid + g] * ao_rhs[v][g]
 * for s < nset, u, v < nao (stride_ao >= nao).  Outputs are accumulated into.
 * FP64 on the tensor cores over the per-block compacted AO lists: only the
 * masked products are formed, and when ao_lhs and ao_rhs are the same array
 * each symmetric pair of products is formed once and added to V[u][v] and
 * V[v][u].  V is accumulated with FP64 atomics, so its last bits depend on the
 * order in which blocks finish.  Setting CFGMM_FOCK_DENSE=1 in the environment
 * selects the dense product over packed operands instead.  Slices too short,
 * BLKSIZE 0 or overlapping V rows are rejected as in the AO-DM-AO calls. */
int cfgmm_aodm_fock(double* vs, size_t vs_len, const double* ws, size_t ws_len,
                    const double* ao_lhs, size_t ao_lhs_len, const double* ao_rhs,
                    size_t ao_rhs_len, size_t stride_ao, size_t stride_grid, size_t nao,
                    size_t ngrid, size_t nset, const uint8_t* tab, size_t tab_len, size_t ldtab,
                    size_t blksize);
int cfgmm_aodm_fock_dev(double* vs, const double* ws, const double* ao_lhs, const double* ao_rhs,
                        size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid,
                        size_t nset, const uint8_t* tab, size_t ldtab, size_t blksize,
                        void* stream);

/* ---- f32 forms of the two paths (MatmulLoops<f32, ...>) -------------------
 * The reference's MatmulLoops is generic over T (src/structs.rs:3-13) but
 * implements f64 only (src/structs.rs:19-20); these are its f32 instantiations
 * with the arguments, layouts, mask and accumulate-into semantics of the f64
 * calls above (cfgmm_matmul_ex, cfgmm_aodmao2rho_ex and their _dev forms).
 * Operands are widened exactly to f64 on the device, the f64 kernels run
 * (CFGMM_PREC_FP64 on DMMA; CFGMM_PREC_OZAKI_INT8 with the moduli that 26-bit
 * operands need, fewer than for f64 data) and each output element is rounded
 * back to f32 once. */
int cfgmm_matmul_f32(float* c, size_t c_len, const float* a, size_t a_len, const float* b,
                     size_t b_len, size_t m, size_t n, size_t k, size_t lda, size_t ldb,
                     size_t ldc, uint8_t transa, uint8_t transb, int precision);
int cfgmm_matmul_f32_dev(float* c, const float* a, const float* b, size_t m, size_t n, size_t k,
                         size_t lda, size_t ldb, size_t ldc, uint8_t transa, uint8_t transb,
                         int precision, void* stream);
int cfgmm_aodmao2rho_f32(float* rhos, size_t rhos_len, const float* dms, size_t dms_len,
                         const float* ao_lhs, size_t ao_lhs_len, const float* ao_rhs,
                         size_t ao_rhs_len, size_t stride_ao, size_t stride_grid, size_t nao,
                         size_t ngrid, size_t nset, const uint8_t* tab, size_t tab_len,
                         size_t ldtab, size_t blksize, int precision);
int cfgmm_aodmao2rho_f32_dev(float* rhos, const float* dms, const float* ao_lhs,
                             const float* ao_rhs, size_t stride_ao, size_t stride_grid,
                             size_t nao, size_t ngrid, size_t nset, const uint8_t* tab,
                             size_t ldtab, size_t blksize, int precision, void* stream);

/* ---- batched plans: many grid batches of one molecule in one launch ------
 * No counterpart in the reference (whose callers batch grids themselves,
 * impl_matmul.rs:354-355): a plan holds device pointers to every batch's phi
 * tables, mask and rho plus the density matrices shared by all batches.  It
 * builds the active lists and one global work list once, picks the kernel's
 * tile configuration with an autotuner (timed on the problem, cached in
 * CFGMM_AUTOTUNE_CACHE), and captures the run in a CUDA graph.  phi and the
 * masks must not change while the plan lives; the contents of `dms` may (an
 * SCF step); each run accumulates into every batch's rho. */
typedef struct cfgmm_aodm_batch {
  double* rhos;            /* (nset, stride_grid), device */
  const double* ao_lhs;    /* (nao, stride_grid), device */
  const double* ao_rhs;    /* (nao, stride_grid), device */
  const uint8_t* tab;      /* (nao, ldtab), device */
  size_t stride_grid, ngrid, ldtab;
  size_t nset;             /* uses density matrices 0 .. nset-1 (<= the plan's nset_max) */
} cfgmm_aodm_batch;

typedef struct cfgmm_aodm_plan cfgmm_aodm_plan;

#define CFGMM_PLAN_NO_GRAPH 1 /* run with plain launches instead of a CUDA graph */
#define CFGMM_PLAN_NO_TUNE  2 /* skip the autotuner: default tiles */

int cfgmm_aodm_plan_create(cfgmm_aodm_plan** plan, const cfgmm_aodm_batch* batches, size_t nbatch,
                           const double* dms, size_t stride_ao, size_t nao, size_t nset_max,
                           size_t blksize, int precision, int flags, void* stream);
int cfgmm_aodm_plan_run(cfgmm_aodm_plan* plan, void* stream);
/* JSON description: precision, batch and item counts, algorithmic flops of
 * one run (sum over batches, matrices and blocks of (2|I_b|^2 + 2|I_b|)|b|),
 * chosen tiles, autotuner timings. */
const char* cfgmm_aodm_plan_info(const cfgmm_aodm_plan* plan);
int cfgmm_aodm_plan_destroy(cfgmm_aodm_plan* plan);

/* ---- the step before the contraction: AOs on the grid, on the device ------
 * No counterpart in the reference (its callers tabulate phi themselves).
 * phi[shell_row[sh] + f][g] = shell_norm[sh] exp(-shell_alpha[sh] r^2) Y_f(x,y,z)
 * for the 2*shell_l[sh]+1 real solid harmonics Y_f (l <= 3, unnormalised
 * polynomials), (x,y,z) = points[g] - shell_xyz[sh], r^2 = x^2+y^2+z^2.
 * All arrays are device arrays; points and shell_xyz are (n, 3); nshell <=
 * 65535 and shell_l[sh] in 0..3 (checked by neither call: device data).  With
 * shell_block_max != NULL also writes max |phi| per (shell, block of blksize
 * points), a (nshell, ceil(ngrid/blksize)) array. */
int cfgmm_eval_ao_dev(double* ao, size_t stride_grid, const double* points, size_t ngrid,
                      const double* shell_xyz, const int* shell_l, const double* shell_alpha,
                      const double* shell_norm, const int* shell_row, size_t nshell,
                      double* shell_block_max, size_t blksize, void* stream);

/* The mask of the contraction from those maxima: tab[row][b] = 1 for every row
 * of shell sh when shell_block_max[sh][b] > threshold, else 0 with phi zeroed
 * on that (row, block). */
int cfgmm_mask_ao_dev(double* ao, size_t stride_grid, size_t ngrid, const int* shell_l,
                      const int* shell_row, size_t nshell, const double* shell_block_max,
                      double threshold, uint8_t* tab, size_t ldtab, size_t blksize, void* stream);

/* Releases the calling device's cached workspaces (they are otherwise kept
 * and reused across calls until process exit), and the servers' idle pinned
 * host staging buffers, which are kept for the process and reused across
 * servers. */
int cfgmm_release_workspace(void);

/* ---- serving: density requests from many molecules, continuous batching ----
 * No counterpart in the reference (a library of blocking calls).  A server
 * owns a worker thread and `nslots` CUDA streams on the current device.
 * Molecules are opened once; their phi, mask, D and rho buffers and batched
 * plan stay on the device while they have work, within `hbm_budget` bytes
 * (the server's own buffers plus an upper bound of each plan; a device
 * molecule's caller-owned phi and mask are counted too).  Requests are taken
 * in arrival order as slots and memory free up; idle molecules are evicted,
 * least recently used first, to admit others (their host or shell data is
 * uploaded or evaluated again on their next request).  Requests of one
 * molecule run in submission order; requests of different molecules overlap.
 * A result does not depend on the other requests in flight.
 * All calls are thread-safe. */
typedef struct cfgmm_server cfgmm_server;

typedef struct cfgmm_request_stats {
  double queue_ms;   /* submit -> start on the GPU */
  double device_ms;  /* the contraction on the GPU (CUDA events) */
  double total_ms;   /* submit -> rho in the caller's buffer */
  double flops;      /* sum_s sum_b (2|I_b|^2 + 2|I_b|)|b| of the request */
} cfgmm_request_stats;

int cfgmm_server_create(cfgmm_server** server, size_t hbm_budget, int nslots, int precision,
                        size_t blksize);
/* Finishes every submitted request, then frees everything. */
int cfgmm_server_destroy(cfgmm_server* server);

/* A molecule from phi (nao, ngrid) and mask (nao, ldtab), row-major, stride
 * ngrid.  on_device = 0: host arrays, read on each admission (keep them until
 * close); 1: the caller's device arrays, used in place.  ao_rhs NULL = ao_lhs.
 * Fails with CFGMM_ERR_OUT_OF_MEMORY when one molecule exceeds the budget. */
int cfgmm_server_open(cfgmm_server* server, const double* ao_lhs, const double* ao_rhs,
                      const uint8_t* tab, size_t nao, size_t ngrid, size_t ldtab,
                      size_t nset_max, int on_device, uint64_t* molecule);
/* A molecule from Gaussian shells on a grid (host arrays, copied): phi as
 * cfgmm_eval_ao_dev computes it (AO rows in shell order), and the mask keeping
 * the `density` fraction (0 < density <= 1) of (shell, block) tiles with the
 * largest max |phi|, phi zeroed outside it.  Evaluated on the device on
 * admission; phi never crosses PCIe. */
int cfgmm_server_open_shells(cfgmm_server* server, const double* points, size_t ngrid,
                             const double* shell_xyz, const int* shell_l,
                             const double* shell_alpha, const double* shell_norm, size_t nshell,
                             double density, size_t nset_max, uint64_t* molecule);
/* No more requests for the molecule; its memory is freed once they finish. */
int cfgmm_server_close(cfgmm_server* server, uint64_t molecule);

/* rhos (nset, ngrid), host = the contraction of the molecule's phi with dms
 * (nset, nao, nao), host, nset <= nset_max (rhos is overwritten, not
 * accumulated into).  dms is copied before the call returns; rhos must stay
 * valid until the ticket is waited for.  Every ticket must be waited for. */
int cfgmm_server_submit(cfgmm_server* server, uint64_t molecule, const double* dms, size_t nset,
                        double* rhos, uint64_t* ticket);
/* The same with D and rho on the device (an SCF loop kept on the GPU): dms
 * (nset, nao, nao) is read once the work enqueued on `stream` so far is done
 * and must stay unchanged until the ticket is waited for; rhos (nset, ngrid)
 * is overwritten by a device copy, complete when the wait returns.  No host
 * staging and no PCIe traffic for the request. */
int cfgmm_server_submit_dev(cfgmm_server* server, uint64_t molecule, const double* dms,
                            size_t nset, double* rhos, void* stream, uint64_t* ticket);
/* Waits for a request (timeout_s < 0: no limit; CFGMM_ERR_TIMEOUT leaves the
 * ticket valid) and returns its status; stats may be NULL. */
int cfgmm_server_wait(cfgmm_server* server, uint64_t ticket, double timeout_s,
                      cfgmm_request_stats* stats);
/* JSON: completed/failed counts, molecules resident, evictions, budget, used
 * and peak bytes, flops of the completed requests, p50/p99 latency (total,
 * queue, device) in ms, molecule load and plan build times, the sum of the
 * requests' device spans (device_ms_total) and the most requests in flight at
 * once (max_inflight). */
const char* cfgmm_server_stats(cfgmm_server* server);

#ifdef __cplusplus
}
#endif

#endif /* CFGMM_H */
