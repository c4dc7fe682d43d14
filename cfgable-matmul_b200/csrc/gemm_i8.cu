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

#include "gemm_i8.cuh"
#include "tcgen05.cuh"

namespace cfgmm {
namespace {

constexpr int BM = 128, BN = 256, BK = 128, STAGES = 4, KSTEPS = BK / 32;
constexpr int THREADS = 192;
constexpr int GROUP_M = 8;
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

}  // namespace

int gemm_i8_tile_rows_a() { return BM; }
int gemm_i8_tile_rows_b() { return BN; }
int gemm_i8_k_block() { return BK; }

cudaError_t gemm_i8_mod(const CUtensorMap& tmA, const CUtensorMap& tmB, const GemmI8Args& args,
                        cudaStream_t stream) {
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
