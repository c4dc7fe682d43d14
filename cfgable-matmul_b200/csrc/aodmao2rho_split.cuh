// aodmao2rho_split.cuh -- internal launcher of the split-precision (INT8
// tcgen05, slice-form Ozaki) masked AO-DM-AO contraction.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "side_stream.cuh"

namespace cfgmm {

// One grid batch of the split contraction (device pointers).
struct SplitBatch {
  const double* ao_lhs;
  double* rhos;             // (nset, stride_grid)
  const int* lists;         // [nblk][nao] active AOs per block
  const int* counts;        // [nblk]
  const int* cbase;         // [nbg] first phi digit chunk of each 64-point tile
  const int* sigma;         // [ngrid] point scales
  size_t stride_grid;
  int ngrid;
  int nset;                 // density matrices used by this batch
  long long partial_off;    // first partial-sum group of this batch
};

// Arguments of the persistent kernel and the reduction.
struct SplitArgs {
  const uint2* dsl;         // D digits [s][u][v], 8 bytes each
  const int* tau;           // row scales [s][u]
  const uint8_t* phisl;     // phi digit tiles of every batch
  const SplitBatch* batches;  // device array, or null: `one`
  SplitBatch one;
  const int4* items;        // (tile, row tile, s, batch); s < 0: per-matrix list
  const int* total;         // [0] items to run, [1] tiles per matrix (s < 0 lists)
  double* partial;          // [group][64]
  int nao, blk, gsub, max_ut;
  const int* asym;          // null, or a flag that is 0 when every D_s is symmetric: then row
                            // tile a contracts only the compacted columns from its own on
                            // (the diagonal tile's strict upper triangle and half diagonal,
                            // times 2), as in the FP64 kernel's symmetric mode
};

// Device scratch (bytes) of the split contraction: active lists, work list,
// D digits (8 bytes per element of D), phi digit tiles, partial sums.
size_t aodmao2rho_split_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk);

// Same contract as aodmao2rho_fp64; nao <= 16384 keeps the INT32 level sums exact.
cudaError_t aodmao2rho_split(double* rhos, const double* dms, const double* ao_lhs,
                             const double* ao_rhs, size_t stride_ao, size_t stride_grid, int nao,
                             int ngrid, int nset, const uint8_t* tab, size_t ldtab, int blk,
                             void* workspace, cudaStream_t stream);

// Pieces of a batched run (the plan keeps phi digits across runs):
//   split_prepare_d   D digits and row scales of nset matrices;
//   split_prepare_phi point scales and phi digit tiles of one batch (pmax:
//                     ngrid 8-byte scratch; cbase: device chunk offsets);
//   split_launch_main / split_launch_reduce  the contraction and its reduction
//                     over (batch, 64-point tile) pairs.
// With asym non-null and *asym == 0 (symmetric mode) the diagonal entries'
// digits are those of D_uu / 2.
cudaError_t split_prepare_d(const double* dms, size_t stride_ao, int nao, int nset, uint2* dsl,
                            int* tau, cudaStream_t stream, const int* asym = nullptr);
cudaError_t split_prepare_phi(const double* ao_rhs, size_t stride_grid, const int* lists,
                              const int* counts, const int* cbase, int nao, int ngrid, int blk,
                              unsigned long long* pmax, int* sigma, uint8_t* phisl,
                              cudaStream_t stream);
// stages: pipeline depth split_min_stages()..5 (shallower requests run at the
// minimum), 0 = default (CFGMM_SPLIT_STAGES or 3);
// attrs_only: set the kernel's attributes (before a stream capture), no launch
cudaError_t split_launch_main(const SplitArgs& a, cudaStream_t stream, int stages = 0,
                              bool attrs_only = false);
cudaError_t split_launch_reduce(const SplitArgs& a, const int2* pairs, int npairs,
                                cudaStream_t stream);
int split_min_stages();    // shallowest pipeline of the main kernel (3)
int split_row_tile();      // rows per work item (128)
int split_point_tile();    // points per work item (64)
int split_chunk();         // compacted AOs per chunk (32)
size_t split_chunk_bytes();  // bytes of one chunk's phi digit tiles
int split_epi_parts();     // partial-sum groups per (tile, row tile, matrix)

// ---- the pair form: two grid block tiles with alike active lists per item ----
// (aodmao2rho_split_pair.cu)  NSL = 7 digits (about 2^-51 of
// sum_v |D_uv||phi_vg|) or 6 (about 2^-43, fewer MMAs and larger tiles).

// One grid batch of the pair form (device pointers).
struct PairBatch {
  const double* ao_lhs;
  double* rhos;        // (nset, stride_grid)
  const int* sigma;    // [ngrid] point scales
  size_t stride_grid;
  int ngrid;
  int nset;
};

// Arguments of the pair form's persistent kernel and reduction.
struct PairArgs {
  const uint2* dsl;       // D digits [s][u][v], 8 bytes each
  const int* tau;         // row scales [s][u]
  const uint2* dhalf;     // digits of D_uu / 2 [s][u] (the symmetric mode's diagonal)
  const uint8_t* phisl;   // phi digit tiles [chunk][NSL][128 x 32]
  const int4* items;      // (pair, row tile, s, batch)
  const int* total;       // [0] items
  const int4* pairs;      // (lo tile, hi tile or -1, batch, 0), tiles local to the batch
  const int* ucount;      // [pair] union size
  const int* ulist;       // [pair][nao] union AOs, ascending
  const uint8_t* uflag;   // [pair][nao] bit 0 / 1: active in the lo / hi tile's block
  const int* cbase;       // [pair] first phi chunk
  const PairBatch* batches;  // device array, or null: `one`
  PairBatch one;
  double* partial;        // [poff[pair] + row tile][nset_max][128]
  const int* poff;        // [pair] first partial row tile, or null: pair * max_t
  int nao, blk, gsub, max_t, nset_max;
  const int* asym;        // null, or 0 when every D_s is symmetric (half contraction)
  int* counter;           // work items drawn so far (zeroed before each launch)
  unsigned long long wait_ns;  // bound of every wait in the kernel (0: the default 2 s)
  int inject;             // test hook: nonzero = the first phi stage is never published
};

// Device pointers of the preparation of one batch (pairing, unions, work
// list, phi tiles); see split_pair_prepare_batch.
struct PairPrep {
  const uint8_t* tab;
  size_t ldtab;
  const double* ao_rhs;
  size_t stride_grid;
  int nao, ngrid, blk, nset, nsl, batch, pair0, chunk0;
  const int* lists;       // [nblk][nao] active AOs of each block, built
  const int* counts;      // [nblk]
  uint32_t* bits;         // scratch [nbg][ceil(nao/32)]
  int* cnt;               // scratch [nbg]
  unsigned long long* key;  // scratch [nbg]
  int *order, *cand, *ncand, *partner, *pos, *choice;  // scratch
  int4* pairs;            // out: pairs pair0 ..
  int* npairs;            // out: [0] pairs of this batch
  int* ulist;             // out: [pair][nao]
  uint8_t* uflag;         // out: [pair][nao]
  int* ucount;            // out: [pair]
  int* cbase;             // out: [pair]
  int* cpair;             // out: the pair of each of the batch's chunks [nbg * ceil(nao/32)]
  int4* items;            // out: appended at *total
  int* total;             // in/out: items so far
  int* chunks_end;        // out: chunk0 + this batch's chunks
  int* sigma;             // out: [ngrid]
  unsigned long long* pmax;  // scratch [ngrid]
  uint8_t* phisl;         // out: phi tiles from chunk0
};

size_t aodmao2rho_split_pair_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk,
                                       int nsl);
// The single-call contraction in the pair form (same contract as
// aodmao2rho_split); inject / wait_ns: test hooks (0 = off / the default bound).
cudaError_t aodmao2rho_split_pair(double* rhos, const double* dms, const double* ao_lhs,
                                  const double* ao_rhs, size_t stride_ao, size_t stride_grid,
                                  int nao, int ngrid, int nset, const uint8_t* tab, size_t ldtab,
                                  int blk, int nsl, void* workspace, cudaStream_t stream,
                                  int inject = 0, unsigned long long wait_ns = 0);
// The preparation of one grid batch whose block lists are built: point scales
// (from the block lists), pairing and work list (from the mask), phi tiles
// (from both); prepare_batch runs the three in that order on one stream.
cudaError_t split_pair_prepare_scales(const PairPrep& q, cudaStream_t stream);
// signatures = false: pair_lists_and_signatures has made them (with the
// block lists, from one read of the mask)
cudaError_t split_pair_prepare_pairs(const PairPrep& q, cudaStream_t stream,
                                     bool signatures = true);
cudaError_t split_pair_lists_and_signatures(const PairPrep& q, int* lists, int* counts,
                                            cudaStream_t stream);
cudaError_t split_pair_prepare_tiles(const PairPrep& q, cudaStream_t stream);
cudaError_t split_pair_prepare_batch(const PairPrep& q, cudaStream_t stream);
// poff[pi]: the first partial row of pair pi (pairs from 0, npairs on the
// device), poff[npairs] their total; one launch, no host round trip.
cudaError_t split_pair_partial_offsets(const int* ucount, const int* npairs, int tn, int* poff,
                                       cudaStream_t stream);
// D digits of every row (dsl, tau, and dhalf: the digits of D_uu / 2 for the
// symmetric mode's diagonal) and, when asym is non-null (zeroed by the
// caller), the bitwise symmetry check of every D, in one launch.
cudaError_t split_pair_prepare_d(const double* dms, size_t stride_ao, int nao, int nset, int nsl,
                                 uint2* dsl, int* tau, uint2* dhalf, int* asym,
                                 cudaStream_t stream);
int split_pair_stages();  // the pair kernel's pipeline depth
// partial sums per (row tile, DM) of a pair: one per gather group and point
int split_pair_partial_points();
// stages: ignored (the pair form's pipeline depth is fixed: split_pair_stages())
cudaError_t split_pair_launch_main(const PairArgs& a, int nsl, cudaStream_t stream,
                                   bool attrs_only = false, int stages = 0);
cudaError_t split_pair_launch_reduce(const PairArgs& a, int nsl, const int* npairs, int pair0,
                                     int max_pairs, cudaStream_t stream);
// Whether a single call (points = ngrid) or a plan (points = all batches'
// points) runs the pair form: CFGMM_SPLIT_FORM=pair / =row, else the pair
// form from kPairMinAos AOs and kPairMinPoints points on (below that the
// pairing and tile building cost more than the pairs save).
constexpr size_t kPairMinAos = 1024, kPairMinPoints = 8192;
bool split_pair_form(size_t nao, size_t points);
int split_pair_row_tile(int nsl);  // D rows per item (the MMA N): 80 (6 digits), 64 (7)
int split_pair_digits();           // digit count (CFGMM_SPLIT_DIGITS, default 7), read per call
cudaError_t aodmao2rho_split_pair_reset_error(cudaStream_t stream);
cudaError_t aodmao2rho_split_pair_read_error(int* code);

// Sticky per-device error word of the split kernel's bounded waits.
cudaError_t aodmao2rho_split_reset_error(cudaStream_t stream);
cudaError_t aodmao2rho_split_read_error(int* code);

}  // namespace cfgmm
