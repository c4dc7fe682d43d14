// gemm_i8.cu -- batched INT8 GEMM on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, accumulators in TMEM) whose epilogue reduces each
// exact INT32 result modulo the batch's modulus: the workhorse of the
// Ozaki-scheme split-precision paths.
//
//   for l < nmod:  R[l][i][j] = (sum_p A[l][i][p] * B[l][j][p]) mods m_l
//
// A[l] (rows x K) and B[l] (cols x K) are signed INT8, K-major, read by TMA
// through 3-D tensor maps (K, rows, l) with 128-byte swizzling; out-of-range
// rows and K are zero-filled by TMA.  "mods" is the symmetric residue in
// [-(m>>1), (m-1)>>1], stored as int8 in R[l] (rows x ldr).
//
// Structure: a persistent kernel, one CTA (6 warps) per SM, walks the tiles
// (l, 128-row block, 256-column block) in a grouped order.
//   warp 0  TMA producer: 4-stage ring of (A 128x128 B, B 256x128 B) tiles.
//   warp 1  owns TMEM (512 columns = two 128x256 INT32 accumulators) and
//           issues the MMAs (M=128, N=256, K=32, 4 per stage) from one thread.
//   warps 2-5 epilogue: tcgen05.ld the accumulator of the previous tile while
//           the MMAs of the next one run, reduce mod m_l, store int8.
// Every mbarrier wait is bounded (tcgen05.cuh); on a timeout the kernel
// records an error code, drains what it issued, frees TMEM and exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdlib>

#include "gemm_i8.cuh"
#include "tcgen05.cuh"

namespace cfgmm {
namespace {

constexpr int BM = 128, BN = 256, BK = 128, STAGES = 4, KSTEPS = BK / 32;
constexpr int THREADS = 192;
constexpr int GROUP_M = 16;
constexpr uint32_t A_STAGE = BM * BK, B_STAGE = BN * BK;  // bytes
constexpr uint32_t STAGE_BYTES = A_STAGE + B_STAGE;
constexpr uint32_t TMEM_COLS = 512;
constexpr size_t SMEM_BYTES = size_t(STAGES) * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;

__device__ int g_gemm_i8_error;  // sticky per-device error word (0 = ok)

struct TileIdx {
  int l, m0, n0;
};

__device__ __forceinline__ TileIdx tile_of(int t, int tiles_m, int tiles_n) {
  const int per_l = tiles_m * tiles_n;
  TileIdx r;
  r.l = t / per_l;
  const int u = t % per_l;
  const int per_group = GROUP_M * tiles_n;
  const int group = u / per_group;
  const int first_m = group * GROUP_M;
  const int gsz = min(tiles_m - first_m, GROUP_M);
  const int in_group = u % per_group;
  r.m0 = (first_m + in_group % gsz) * BM;
  r.n0 = (in_group / gsz) * BN;
  return r;
}

__global__ void __launch_bounds__(THREADS, 1)
gemm_i8_mod_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   GemmI8Args p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + STAGES * A_STAGE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* full = bars;              // [STAGES]  TMA -> MMA
  uint64_t* empty = bars + STAGES;    // [STAGES]  MMA -> TMA
  uint64_t* tfull = bars + 2 * STAGES;      // [2]  MMA -> epilogue
  uint64_t* tempty = bars + 2 * STAGES + 2;  // [2]  epilogue -> MMA
  uint64_t* drain = bars + 2 * STAGES + 4;   // MMA completion at teardown
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 5);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* err = &g_gemm_i8_error;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&tfull[b], 1);
      tc::mbar_init(&tempty[b], 4);
    }
    tc::mbar_init(drain, 1);
    tc::mbar_fence_init();
    tc::prefetch_tensormap(&tmA);
    tc::prefetch_tensormap(&tmB);
  }
  if (warp == 1) {
    tc::tmem_alloc(tmem_slot, TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem_base = *tmem_slot;

  const int tiles_m = (p.rows_a + BM - 1) / BM;
  const int tiles_n = (p.rows_b + BN - 1) / BN;
  const int ntiles = tiles_m * tiles_n * p.nmod;
  const int kblocks = (p.k + BK - 1) / BK;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int stage = 0;
      uint32_t uses[STAGES] = {0, 0, 0, 0};
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const TileIdx ti = tile_of(t, tiles_m, tiles_n);
        for (int kb = 0; kb < kblocks; ++kb) {
          if (uses[stage] > 0 && !tc::mbar_wait(&empty[stage], (uses[stage] - 1) & 1, err, 1)) {
            ok = false;
            break;
          }
          tc::mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
          tc::tma_load_3d(sA + stage * A_STAGE, &tmA, &full[stage], kb * BK, ti.m0, ti.l);
          tc::tma_load_3d(sB + stage * B_STAGE, &tmB, &full[stage], kb * BK, ti.n0, ti.l);
          ++uses[stage];
          stage = (stage + 1) % STAGES;
        }
      }
      // teardown: let every armed stage land before the CTA can exit
      for (int s = 0; s < STAGES; ++s)
        if (uses[s] > 0) tc::mbar_wait(&full[s], (uses[s] - 1) & 1, err, 2, true);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_i8(BM, BN);
      int stage = 0;
      uint32_t fuse[STAGES] = {0, 0, 0, 0};
      uint32_t buse[2] = {0, 0};
      int buf = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        if (buse[buf] > 0 && !tc::mbar_wait(&tempty[buf], (buse[buf] - 1) & 1, err, 3)) break;
        tc::fence_after_sync();
        const uint32_t dtmem = tmem_base + uint32_t(buf * BN);
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!tc::mbar_wait(&full[stage], fuse[stage] & 1, err, 4)) {
            ok = false;
            break;
          }
          ++fuse[stage];
          tc::fence_after_sync();
          const uint32_t a0 = tc::smem_u32(sA + stage * A_STAGE);
          const uint32_t b0 = tc::smem_u32(sB + stage * B_STAGE);
#pragma unroll
          for (int ks = 0; ks < KSTEPS; ++ks)
            tc::mma_i8(dtmem, tc::smem_desc_k128(a0 + 32 * ks), tc::smem_desc_k128(b0 + 32 * ks),
                       idesc, kb > 0 || ks > 0);
          tc::mma_commit(&empty[stage]);
          stage = (stage + 1) % STAGES;
        }
        if (!ok) break;
        tc::mma_commit(&tfull[buf]);
        ++buse[buf];
        buf ^= 1;
      }
      // teardown: wait until every issued MMA has completed
      tc::mma_commit(drain);
      tc::mbar_wait(drain, 0, err, 5, true);
    }
  } else {
    // ---------------- epilogue (warps 2..5) ----------------
    const int quarter = warp & 3;  // TMEM lanes this warp may access
    const uint32_t lane_off = uint32_t(32 * quarter) << 16;
    uint32_t buse[2] = {0, 0};
    int buf = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const TileIdx ti = tile_of(t, tiles_m, tiles_n);
      if (!tc::mbar_wait(&tfull[buf], buse[buf] & 1, err, 6)) break;
      ++buse[buf];
      tc::fence_after_sync();
      const int m = p.mod[ti.l];
      const float inv = p.inv[ti.l];
      const int hi = (m - 1) >> 1, lo = -(m >> 1);
      const int row = ti.m0 + 32 * quarter + lane;
      int8_t* out = p.out + (size_t(ti.l) * p.rows_a + row) * p.ldr;
#pragma unroll 1
      for (int c = 0; c < BN; c += 32) {
        uint32_t v[32];
        tc::tmem_ld_32x32b_x32(tmem_base + uint32_t(buf * BN + c) + lane_off, v);
        tc::tmem_ld_wait();
        uint32_t packed[8];
#pragma unroll
        for (int w = 0; w < 8; ++w) {
          uint32_t word = 0;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int a = int(v[4 * w + e]);
            const int q = __float2int_rn(__int2float_rn(a) * inv);
            int r = a - q * m;  // q is within 2 of the exact quotient for |a| < 2^30
            if (r > hi) r -= m;
            if (r > hi) r -= m;
            if (r < lo) r += m;
            if (r < lo) r += m;
            word |= (uint32_t(r) & 0xffu) << (8 * e);
          }
          packed[w] = word;
        }
        const int col = ti.n0 + c;
        if (row < p.rows_a && col < p.rows_b) {
          if (col + 32 <= p.rows_b) {
            uint4* dst = reinterpret_cast<uint4*>(out + col);
            dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
          } else {
            for (int e = 0; e < p.rows_b - col; ++e)
              out[col + e] = int8_t((packed[e >> 2] >> (8 * (e & 3))) & 0xffu);
          }
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&tempty[buf]);
      buf ^= 1;
    }
  }

  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 1) tc::tmem_dealloc(tmem_base, TMEM_COLS);
}

// ---------------------------------------------------------------------------
// Pair form: a cluster of two CTAs computes 256 x 256 tiles with
// tcgen05.mma.cta_group::2 (M = 256, N = 256, K = 32).  CTA r (its rank in the
// cluster) loads rows 128r.. of the A tile and columns 128r.. of the B tile,
// holds accumulator rows 128r.. in its own TMEM and stores them, so each SM
// reads 8 KB of operands per MMA from shared memory instead of 12 KB.  One
// thread of CTA 0 issues the MMAs; its stage barrier counts the TMA bytes of
// both CTAs, the MMA commits arrive on both CTAs' barriers, and the epilogue
// warps of both CTAs release an accumulator on CTA 0's barrier.  Every role
// leaves its loop on a bounded wait's timeout and meets the other CTA at the
// final cluster barrier.
// ---------------------------------------------------------------------------
constexpr int P_BM = 256, P_BN = 256, P_STAGES = 6;
constexpr uint32_t P_A_STAGE = (P_BM / 2) * BK, P_B_STAGE = (P_BN / 2) * BK;  // per CTA
constexpr uint32_t P_STAGE_BYTES = P_A_STAGE + P_B_STAGE;
constexpr size_t P_SMEM_BYTES = size_t(P_STAGES) * P_STAGE_BYTES + 1024 + 256;

__device__ __forceinline__ TileIdx pair_tile_of(int t, int tiles_m, int tiles_n) {
  const int per_l = tiles_m * tiles_n;
  TileIdx r;
  r.l = t / per_l;
  const int u = t % per_l;
  const int per_group = GROUP_M * tiles_n;
  const int group = u / per_group;
  const int first_m = group * GROUP_M;
  const int gsz = min(tiles_m - first_m, GROUP_M);
  const int in_group = u % per_group;
  r.m0 = (first_m + in_group % gsz) * P_BM;
  r.n0 = (in_group / gsz) * P_BN;
  return r;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1)
gemm_i8_mod_pair_kernel(const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB, GemmI8Args p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + P_STAGES * P_A_STAGE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + P_STAGES * P_STAGE_BYTES);
  uint64_t* full = bars;                      // [P_STAGES] TMA -> MMA (CTA 0's counts both)
  uint64_t* empty = bars + P_STAGES;          // [P_STAGES] MMA -> each CTA's producer
  uint64_t* tfull = bars + 2 * P_STAGES;      // [2] MMA -> each CTA's epilogue
  uint64_t* tempty = bars + 2 * P_STAGES + 2;  // [2] (CTA 0's) 8 epilogue warps -> MMA
  uint64_t* drain = bars + 2 * P_STAGES + 4;   // MMA completion at teardown (CTA 0)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * P_STAGES + 5);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = tc::cluster_ctarank();
  int* err = &g_gemm_i8_error;

  if (threadIdx.x == 0) {
    for (int s = 0; s < P_STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&tfull[b], 1);
      tc::mbar_init(&tempty[b], 8);
    }
    tc::mbar_init(drain, 1);
    tc::mbar_fence_init();
    tc::prefetch_tensormap(&tmA);
    tc::prefetch_tensormap(&tmB);
  }
  if (warp == 1) {
    tc::tmem_alloc_pair(tmem_slot, TMEM_COLS);
    tc::tmem_relinquish_pair();
  }
  tc::fence_before_sync();
  tc::cluster_sync();  // both CTAs' barriers initialised, TMEM allocated
  tc::fence_after_sync();
  const uint32_t tmem_base = *tmem_slot;

  const int tiles_m = (p.rows_a + P_BM - 1) / P_BM;
  const int tiles_n = (p.rows_b + P_BN - 1) / P_BN;
  const int ntiles = tiles_m * tiles_n * p.nmod;
  const int kblocks = (p.k + BK - 1) / BK;
  const int cid = int(blockIdx.x >> 1), nclusters = int(gridDim.x >> 1);

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      const uint32_t full0 = tc::mapa_shared(tc::smem_u32(full), 0);  // CTA 0's full[0]
      int stage = 0;
      uint32_t uses[P_STAGES] = {0, 0, 0, 0, 0, 0};
      bool ok = true;
      for (int t = cid; t < ntiles && ok; t += nclusters) {
        const TileIdx ti = pair_tile_of(t, tiles_m, tiles_n);
        for (int kb = 0; kb < kblocks; ++kb) {
          if (uses[stage] > 0 && !tc::mbar_wait(&empty[stage], (uses[stage] - 1) & 1, err, 21)) {
            ok = false;
            break;
          }
          if (rank == 0) tc::mbar_arrive_expect_tx(&full[stage], 2 * P_STAGE_BYTES);
          const uint32_t fb = full0 + uint32_t(stage) * 8u;
          tc::tma_load_3d_pair(sA + stage * P_A_STAGE, &tmA, fb, kb * BK,
                               ti.m0 + int(rank) * (P_BM / 2), ti.l);
          tc::tma_load_3d_pair(sB + stage * P_B_STAGE, &tmB, fb, kb * BK,
                               ti.n0 + int(rank) * (P_BN / 2), ti.l);
          ++uses[stage];
          stage = (stage + 1) % P_STAGES;
        }
      }
      // teardown: CTA 0's stage barriers count both CTAs' bytes
      if (rank == 0)
        for (int s = 0; s < P_STAGES; ++s)
          if (uses[s] > 0) tc::mbar_wait(&full[s], (uses[s] - 1) & 1, err, 22, true);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (CTA 0) ----------------
    if (rank == 0 && lane == 0) {
      const uint32_t idesc = tc::idesc_i8(P_BM, P_BN);
      int stage = 0;
      uint32_t fuse[P_STAGES] = {0, 0, 0, 0, 0, 0};
      uint32_t buse[2] = {0, 0};
      int buf = 0;
      bool ok = true;
      for (int t = cid; t < ntiles && ok; t += nclusters) {
        if (buse[buf] > 0 &&
            !tc::mbar_wait_cluster(&tempty[buf], (buse[buf] - 1) & 1, err, 23))
          break;
        tc::fence_after_sync();
        const uint32_t dtmem = tmem_base + uint32_t(buf * P_BN);
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!tc::mbar_wait_cluster(&full[stage], fuse[stage] & 1, err, 24)) {
            ok = false;
            break;
          }
          ++fuse[stage];
          tc::fence_after_sync();
          const uint32_t a0 = tc::smem_u32(sA + stage * P_A_STAGE);
          const uint32_t b0 = tc::smem_u32(sB + stage * P_B_STAGE);
#pragma unroll
          for (int ks = 0; ks < KSTEPS; ++ks)
            tc::mma_i8_pair(dtmem, tc::smem_desc_k128(a0 + 32 * ks),
                            tc::smem_desc_k128(b0 + 32 * ks), idesc, kb > 0 || ks > 0);
          tc::mma_commit_pair(&empty[stage]);
          stage = (stage + 1) % P_STAGES;
        }
        if (!ok) break;
        tc::mma_commit_pair(&tfull[buf]);
        ++buse[buf];
        buf ^= 1;
      }
      // teardown: every issued MMA has completed
      tc::mma_commit_pair_local(drain);
      tc::mbar_wait(drain, 0, err, 25, true);
    }
  } else {
    // ---------------- epilogue (warps 2..5, both CTAs) ----------------
    const int quarter = warp & 3;  // TMEM lanes this warp may access
    const uint32_t lane_off = uint32_t(32 * quarter) << 16;
    const uint32_t tempty0 = tc::mapa_shared(tc::smem_u32(tempty), 0);  // CTA 0's tempty[0]
    uint32_t buse[2] = {0, 0};
    int buf = 0;
    for (int t = cid; t < ntiles; t += nclusters) {
      const TileIdx ti = pair_tile_of(t, tiles_m, tiles_n);
      if (!tc::mbar_wait_cluster(&tfull[buf], buse[buf] & 1, err, 26)) break;
      ++buse[buf];
      tc::fence_after_sync();
      const int m = p.mod[ti.l];
      const float inv = p.inv[ti.l];
      const int hi = (m - 1) >> 1, lo = -(m >> 1);
      const int row = ti.m0 + int(rank) * (P_BM / 2) + 32 * quarter + lane;
      int8_t* out = p.out + (size_t(ti.l) * p.rows_a + row) * p.ldr;
#pragma unroll 1
      for (int c = 0; c < P_BN; c += 32) {
        uint32_t v[32];
        tc::tmem_ld_32x32b_x32(tmem_base + uint32_t(buf * P_BN + c) + lane_off, v);
        tc::tmem_ld_wait();
        uint32_t packed[8];
#pragma unroll
        for (int w = 0; w < 8; ++w) {
          uint32_t word = 0;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int a = int(v[4 * w + e]);
            const int q = __float2int_rn(__int2float_rn(a) * inv);
            int r = a - q * m;  // q is within 2 of the exact quotient for |a| < 2^30
            if (r > hi) r -= m;
            if (r > hi) r -= m;
            if (r < lo) r += m;
            if (r < lo) r += m;
            word |= (uint32_t(r) & 0xffu) << (8 * e);
          }
          packed[w] = word;
        }
        const int col = ti.n0 + c;
        if (row < p.rows_a && col < p.rows_b) {
          if (col + 32 <= p.rows_b) {
            uint4* dst = reinterpret_cast<uint4*>(out + col);
            dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
          } else {
            for (int e = 0; e < p.rows_b - col; ++e)
              out[col + e] = int8_t((packed[e >> 2] >> (8 * (e & 3))) & 0xffu);
          }
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive_cluster(tempty0 + uint32_t(buf) * 8u);
      buf ^= 1;
    }
  }

  tc::fence_before_sync();
  tc::cluster_sync();  // the pair's MMAs and remote arrivals are done on both sides
  tc::fence_after_sync();
  if (warp == 1) tc::tmem_dealloc_pair(tmem_base, TMEM_COLS);
}

// The pair form is used unless CFGMM_GEMM_PAIR=0.
bool pair_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("CFGMM_GEMM_PAIR");
    return !(e && e[0] == '0');
  }();
  return on;
}

}  // namespace

int gemm_i8_tile_rows_a() { return BM; }
int gemm_i8_tile_rows_b() { return pair_enabled() ? P_BN / 2 : BN; }
int gemm_i8_k_block() { return BK; }

cudaError_t gemm_i8_mod(const CUtensorMap& tmA, const CUtensorMap& tmB, const GemmI8Args& args,
                        cudaStream_t stream) {
  if (pair_enabled()) {
    cudaError_t err = cudaFuncSetAttribute(gemm_i8_mod_pair_kernel,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(P_SMEM_BYTES));
    if (err != cudaSuccess) return err;
    const long long tiles = (long long)((args.rows_a + P_BM - 1) / P_BM) *
                            ((args.rows_b + P_BN - 1) / P_BN) * args.nmod;
    if (tiles <= 0) return cudaSuccess;
    // as many pairs as can be resident at once (a persistent kernel)
    static int max_clusters = [] {
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(2, 1, 1);
      cfg.blockDim = dim3(THREADS, 1, 1);
      cfg.dynamicSmemBytes = P_SMEM_BYTES;
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, gemm_i8_mod_pair_kernel, &cfg) != cudaSuccess)
        n = 0;
      return n;
    }();
    if (max_clusters <= 0) return cudaErrorLaunchOutOfResources;
    const long long clusters = tiles < max_clusters ? tiles : max_clusters;
    gemm_i8_mod_pair_kernel<<<unsigned(2 * clusters), THREADS, P_SMEM_BYTES, stream>>>(tmA, tmB,
                                                                                     args);
    return cudaGetLastError();
  }
  cudaError_t err = cudaFuncSetAttribute(gemm_i8_mod_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(SMEM_BYTES));
  if (err != cudaSuccess) return err;
  int dev = 0, nsm = 0;
  if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
  if ((err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return err;
  const long long tiles = (long long)((args.rows_a + BM - 1) / BM) *
                          ((args.rows_b + BN - 1) / BN) * args.nmod;
  if (tiles <= 0) return cudaSuccess;
  const int grid = int(tiles < nsm ? tiles : nsm);
  gemm_i8_mod_kernel<<<grid, THREADS, SMEM_BYTES, stream>>>(tmA, tmB, args);
  return cudaGetLastError();
}

cudaError_t gemm_i8_reset_error(cudaStream_t stream) {
  static const int zero = 0;
  return cudaMemcpyToSymbolAsync(g_gemm_i8_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice,
                                 stream);
}

cudaError_t gemm_i8_read_error(int* code) {
  return cudaMemcpyFromSymbol(code, g_gemm_i8_error, sizeof(int));
}

}  // namespace cfgmm
