// aodmao2rho_fp64.cuh -- internal interface of the FP64 masked AO-DM-AO contraction.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace cfgmm {

// One grid batch: its phi tables, rho, active lists and point count.
struct AodmBatch {
  const double* ao_lhs;
  const double* ao_rhs;
  double* rhos;            // (nset, stride_grid)
  const int* lists;        // [nblk][nao] active AOs per block
  const int* counts;       // [nblk]
  size_t stride_grid;
  int ngrid;
  int nset;                // density matrices used by this batch (<= nset_max)
  long long partial_off;   // first partial-sum slot of this batch
  int rhs_tma;             // pipelined form: ao_rhs rows by TMA (its map is valid), else cp.async
};

// Kernel arguments: density matrices shared by all batches, and either a
// device array of batch descriptors or one descriptor by value.
struct AodmArgs {
  const double* dms;
  size_t stride_ao, dm_stride;  // dm_stride = stride_ao^2
  int nao, blk, gsub;           // gsub = 64-point tiles per grid block
  int max_utiles;               // partial slots per (batch, block tile)
  int nset_max;
  const AodmBatch* batches;     // null: use `one`
  const CUtensorMap* rhs_maps;  // with batches: ao_rhs gather map of each batch (pipelined form)
  AodmBatch one;
  const int4* items;            // work list: (batch, block tile, row tile, 0)
  int* counters;                // [ngroups] work counters, the item total, the asymmetry flag
  int ngroups;
  const int* asym;              // null, or counters + ngroups + 1: 0 when every D_s is symmetric
  double* partial;              // [slot][nset_max][64]
  unsigned long long wait_ns;   // bound of the pipelined kernel's waits (0: the default 2 s)
  int inject;                   // test hook: the pipelined kernel's first stage is never published
};

// Test hook of the failure detection (cfgmm_test_arm_wait_timeout): arms the
// calling thread's next contraction of `kind` (0: the FP64 pipelined kernel,
// 1: the split pair kernel) to run with waits bounded by `wait_ns` and one
// producer that never publishes its first stage.  take_wait_injection returns
// whether the next launch of `kind` is armed (and disarms it).
void arm_wait_injection(int kind, unsigned long long wait_ns);
bool take_wait_injection(int kind, unsigned long long* wait_ns);

// Tile configuration of the main kernel (the autotuner's search space):
// `ns` density matrices share one ao_rhs tile (1..3), `tk` compacted AOs per
// pipeline stage of form 3 (16 or 32), or tk = 0 for the pipelined form
// (which then takes the ao_rhs maps from AodmArgs::rhs_maps).
struct AodmConfig {
  int ns;
  int tk;
};

AodmConfig aodm_default_config(int nset);
int aodm_groups(const AodmConfig& cfg, int nset_max);
int aodm_row_tile();    // compacted rows per work item (64)
int aodm_point_tile();  // grid points per work item (64)

// Device scratch (bytes) the single-call contraction needs: the per-block
// active AO lists, their counts, the work list and the partial sums.
size_t aodmao2rho_fp64_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk);

// rhos[s*stride_grid+g] += ... (see cfgmm.h) on `stream`; device pointers,
// `workspace` holds aodmao2rho_fp64_workspace(...) bytes, 256-byte aligned.
cudaError_t aodmao2rho_fp64(double* rhos, const double* dms, const double* ao_lhs,
                            const double* ao_rhs, size_t stride_ao, size_t stride_grid, int nao,
                            int ngrid, int nset, const uint8_t* tab, size_t ldtab, int blk,
                            void* workspace, cudaStream_t stream);

// Builds the per-block active AO lists: lists[b*nao + i] = i-th u (ascending)
// with tab[u*ldtab + b] != 0, counts[b] = their number.
cudaError_t aodm_block_lists_launch(const uint8_t* tab, size_t ldtab, int nao, int nblk,
                                    int* lists, int* counts, cudaStream_t stream);

// Work list of one grid batch: items[i] = (0, block tile, row tile of 64 active
// AOs, 0) in block order; counters[0..ncounters) = 0, counters[ncounters] = the
// item count, counters[ncounters + 1] = 0.
cudaError_t aodm_build_items_launch(const int* counts, int nblk, int gsub, int4* items,
                                    int* counters, int ncounters, cudaStream_t stream);

// Pieces of a batched run: counter reset, the persistent kernel, and the
// reduction over (batch, block tile) pairs (rpairs null: batch 0, bg = index).
cudaError_t aodm_launch_reset(int* counters, int ngroups, cudaStream_t stream);
// attrs_only: set the kernel's attributes (before a stream capture), no launch
cudaError_t aodm_launch_main(const AodmArgs& a, const AodmConfig& cfg, cudaStream_t stream,
                             bool attrs_only = false);
cudaError_t aodm_launch_reduce(const AodmArgs& a, const int2* rpairs, int npairs,
                               cudaStream_t stream);

// Pipelined form of the main kernel (warp-specialised; ao_rhs rows by TMA
// gather4 where AodmBatch::rhs_tma is set, by the producers' cp.async
// otherwise).  aodm_rhs_map builds the gather map of one ao_rhs table and
// returns false where TMA does not apply (base or row pitch not 16-byte
// aligned, odd BLKSIZE).  `map` is used when a.batches is null, a.rhs_maps
// (a 64-byte aligned device array, one map per batch) otherwise.
// aodm_pipe_enabled() is false when CFGMM_AODM_PIPE=0 (form 3 then runs).
bool aodm_pipe_enabled();
bool aodm_rhs_map(CUtensorMap* map, const double* ao_rhs, size_t stride_grid, int nao, int ngrid,
                  int blk);
cudaError_t aodm_launch_pipe(const AodmArgs& a, int ns, const CUtensorMap& map,
                             cudaStream_t stream, bool attrs_only = false);
// Code of the first timed-out wait of the pipelined kernel since the last
// call's setup kernel (0: none).
cudaError_t aodm_read_error(int* code);
cudaError_t aodm_reset_error(cudaStream_t stream);

// Symmetric-D mode of the pipelined form: aodm_launch_sym_check sets
// *asym = 1 unless every D_s (s < nset) equals its transpose bit for bit
// (*asym is zeroed by the setup kernels).  With a.asym pointing at the flag and
// the flag 0, row tile a of a block contracts only the compacted columns from
// its own first one on, rho += 2 phi_a^T (D'_aa phi_a + D_{a,>a} phi_>a) with
// D'_aa the upper triangle of the diagonal tile and half its diagonal: about
// half the D gather and the FLOPs.  aodm_sym_enabled() is false when
// CFGMM_AODM_SYM=0.
bool aodm_sym_enabled();
cudaError_t aodm_launch_sym_check(const double* dms, size_t stride_ao, int nao, int nset,
                                  int* asym, cudaStream_t stream);

}  // namespace cfgmm
