// dgemm_fp64.cu -- C += op(A) * op(B) in FP64 on the B200 FP64 tensor cores.
//
// Semantics follow MatmulLoops::matmul_loop_parallel_mnk_pack_a
// (src/impl_matmul.rs:155-231): row-major operands, opA(i,p) = transa ?
// a[p*lda+i] : a[i*lda+p], opB(p,j) = transb ? b[j*ldb+p] : b[p*ldb+j], and the
// product is ACCUMULATED into C (impl_matmul.rs:31-46).
//
// Design (B200-first, not a translation of the CPU loops):
//   * FP64 has no tcgen05 kind, so the math is the FP64 tensor-core MMA
//     (DMMA, mma.sync m16n8k4 f64), fed from shared memory.
//   * CTA tile 128x128, K step 32, 8 warps in a 2x4 grid (warp tile 64x32,
//     4x4 m16n8k8 DMMA tiles, 64 FP64 accumulators per thread), 3-stage
//     cp.async ring (192 KB shared memory, one CTA per SM).
//   * Every operand tile is stored "K-contiguous" in shared memory
//     (As[m][k], Bs[n][k]) whatever transa/transb are: the global->shared
//     copies do the transposition, with the thread->element map chosen so that
//     global reads stay coalesced for each transpose case.
//   * 8-byte cp.async keeps any lda/ldb (odd ld, as in the 3527x6581x9583
//     workload) and any base alignment legal; out-of-range elements are
//     zero-filled, so edge tiles need no separate path.  Each thread's copy
//     pointers are computed once and bumped per K step, and the copies of the
//     next stage are spread between the DMMA groups of the current one, so
//     the tensor pipe keeps issuing while they go out.
//   * The k index inside each 8-wide group is permuted (thread q of a quad
//     holds k = 2q and 2q+1 as MMA k-slots q and q+4), so each fragment load
//     is one 16-byte shared-memory load; the same permutation is applied to A
//     and B, which leaves the sum unchanged up to FP64 rounding order.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "common.cuh"
#include "dgemm_fp64.cuh"
#include "tcgen05.cuh"

namespace cfgmm {
namespace {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, THREADS = 256, GROUP_M = 8;
constexpr int TILE_DOUBLES = BM * BK;  // As or Bs per stage (BM == BN)
constexpr size_t SMEM_BYTES = size_t(STAGES) * 2 * TILE_DOUBLES * sizeof(double);
constexpr int CPT = TILE_DOUBLES / THREADS;  // copies per thread per operand tile (16)

// One thread's share of the copies of one 128 x BK operand tile into shared
// memory as S[r][k] (r = row of op(X): m for A, n for B).
//   kRowsContig: element (r,k) at x[r*ld + k] (k contiguous).  The thread copies
//     k = tid % 32 of rows tid/32 + 8i: a warp reads 256 contiguous bytes.
//   otherwise:   element (r,k) at x[k*ld + r] (r contiguous).  The thread copies
//     r = tid % 128 of k = tid/128 + 2i: a warp reads 256 contiguous bytes.
// Column mask of the masked GEMM (impl_matmul_non0tab.rs:196-207): element
// (p, j) of B takes part only when tab[p * ldtab + j / blk] != 0.
struct ColMask {
  const uint8_t* tab;  // null: no mask
  size_t ldtab;
  int blk;
};

template <bool kRowsContig>
struct TileCopier {
  const double* src;     // element i = 0 of the current K step
  size_t step_i;         // distance between consecutive elements i
  size_t step_k;         // advance per K step
  int dst0;              // shared offset of element 0 within a stage
  unsigned row_ok;       // bit i: element i's row is inside the matrix
  int kpos;              // k of element 0 relative to the K step
  int key;               // swizzle key of the thread's row (kRowsContig = false)
  const uint8_t* mcol;   // mask column of the thread's row (masked B only), else null
  size_t mstride;        // mask row stride (ldtab)

  __device__ __forceinline__ void init(const double* x, size_t ld, int r0, int rmax, int tid,
                                       ColMask mask = ColMask{nullptr, 0, 1}) {
    mcol = nullptr;
    mstride = 0;
    if (kRowsContig) {
      const int k = tid & 31, rb = tid >> 5;
      src = x + size_t(r0 + rb) * ld + k;
      step_i = 8 * ld;
      step_k = BK;
      dst0 = swz<BK>(rb, k);
      row_ok = 0;
#pragma unroll
      for (int i = 0; i < CPT; ++i) row_ok |= unsigned(r0 + rb + 8 * i < rmax) << i;
      kpos = k;
    } else {
      const int r = tid & 127, kb = tid >> 7;
      src = x + size_t(kb) * ld + (r0 + r);
      step_i = 2 * ld;
      step_k = size_t(BK) * ld;
      key = swz_key(r);
      dst0 = r * BK + kb;
      row_ok = (r0 + r < rmax) ? 0xffffu : 0u;
      kpos = kb;
      if (mask.tab && r0 + r < rmax) {
        mcol = mask.tab + (r0 + r) / mask.blk + size_t(kb) * mask.ldtab;
        mstride = mask.ldtab;
      }
    }
  }

  // Issues elements [i0, i0 + n) of K step `kt` into stage buffer S.
  template <int i0, int n>
  __device__ __forceinline__ void issue(double* S, int kt, int kmax) const {
    const double* base = src + size_t(kt) * step_k;
    const int krem = kmax - kt * BK - kpos;  // element ok while its k offset < krem
#pragma unroll
    for (int i = i0; i < i0 + n; ++i) {
      bool ok;
      int dst;
      if (kRowsContig) {
        ok = ((row_ok >> i) & 1u) && krem > 0;
        dst = dst0 + i * 8 * BK;  // rows +8i keep the same swizzle key
      } else {
        ok = row_ok && 2 * i < krem;
        dst = dst0 + ((i ^ key) << 1);  // k = kb + 2i: chunk i, half kb
        if (mcol && ok) ok = mcol[(size_t(kt) * BK + 2 * i) * mstride] != 0;
      }
      cp_async_8(S + dst, ok ? base + size_t(i) * step_i : src, ok);
    }
  }
};

// The tiles of a last, partial wave of CTAs may be split along K: block
// full + j (j < tail * splits) computes K steps [s*ktiles/splits, (s+1)*ktiles/splits)
// of tile full + j / splits (s = j % splits) and stores its partial tile in
// ws[j]; splits == 0 means no split.
struct TailSplit {
  int full, splits;
  double* ws;  // [tail * splits][BM * BN]
};

template <bool TA, bool TB>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_fp64_kernel(double* __restrict__ c, const double* __restrict__ a,
                  const double* __restrict__ b, int m, int n, int k, size_t lda, size_t ldb,
                  size_t ldc, ColMask mask, TailSplit tail) {
  extern __shared__ __align__(128) double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * TILE_DOUBLES;

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warp grid
  const int g = lane >> 2, q = lane & 3;

  // 1-D grid in groups of GROUP_M tile rows: CTAs running together share the
  // B panels of a group and the A panels of its rows in L2.
  const int tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  const bool split = tail.splits > 0 && int(blockIdx.x) >= tail.full;
  const int job = split ? int(blockIdx.x) - tail.full : 0;
  const int tile = split ? tail.full + job / tail.splits : int(blockIdx.x);
  const int per_group = GROUP_M * tiles_n;
  const int group = tile / per_group;
  const int first_m = group * GROUP_M;
  const int gsz = min(tiles_m - first_m, GROUP_M);
  const int in_group = tile % per_group;
  const int m0 = (first_m + in_group % gsz) * BM;
  const int n0 = (in_group / gsz) * BN;
  const int kall = (k + BK - 1) / BK;
  const int sidx = split ? job % tail.splits : 0;
  const int kt0 = split ? int((long long)sidx * kall / tail.splits) : 0;
  const int kt1 = split ? int((long long)(sidx + 1) * kall / tail.splits) : kall;

  // A: rows m, k contiguous unless transposed.  B: rows n, k contiguous only
  // when transposed (b[j*ldb + p]).
  TileCopier<!TA> ca;
  TileCopier<TB> cb;
  ca.init(a, lda, m0, m, tid);
  cb.init(b, ldb, n0, n, tid, mask);  // the mask only applies to a non-transposed B

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (kt0 + s < kt1) {
      ca.template issue<0, CPT>(As + s * TILE_DOUBLES, kt0 + s, k);
      cb.template issue<0, CPT>(Bs + s * TILE_DOUBLES, kt0 + s, k);
    }
    cp_async_commit();
  }

  for (int kt = kt0; kt < kt1; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int nk = kt + STAGES - 1;  // K step whose copies go out during this one
    const bool pre = nk < kt1;
    double* An = As + ((nk - kt0) % STAGES) * TILE_DOUBLES;
    double* Bn = Bs + ((nk - kt0) % STAGES) * TILE_DOUBLES;

    const double* A_s = As + ((kt - kt0) % STAGES) * TILE_DOUBLES;
    const double* B_s = Bs + ((kt - kt0) % STAGES) * TILE_DOUBLES;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 8) {
      double2 av[4][2], bv[4];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int r = wm * 64 + mt * 16 + g;
        av[mt][0] = *reinterpret_cast<const double2*>(A_s + swz<BK>(r, kk + 2 * q));
        av[mt][1] = *reinterpret_cast<const double2*>(A_s + swz<BK>(r + 8, kk + 2 * q));
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int r = wn * 32 + nt * 8 + g;
        bv[nt] = *reinterpret_cast<const double2*>(B_s + swz<BK>(r, kk + 2 * q));
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
          dmma_16x8x8(acc[mt][nt], av[mt][0].x, av[mt][1].x, av[mt][0].y, av[mt][1].y, bv[nt].x,
                      bv[nt].y);
      // a quarter of the next stage's copies after each group of 16 DMMAs
      if (pre) {
        if (kk == 0) ca.template issue<0, CPT / 2>(An, nk, k);
        if (kk == 8) ca.template issue<CPT / 2, CPT / 2>(An, nk, k);
        if (kk == 16) cb.template issue<0, CPT / 2>(Bn, nk, k);
        if (kk == 24) cb.template issue<CPT / 2, CPT / 2>(Bn, nk, k);
      }
    }
    cp_async_commit();
  }
  cp_async_wait<0>();

  if (split) {  // the partial tile, dense 128 x 128, to the workspace
    double* w = tail.ws + size_t(job) * (BM * BN);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = wm * 64 + mt * 16 + g + 8 * h;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
          *reinterpret_cast<double2*>(w + r * BN + wn * 32 + nt * 8 + 2 * q) =
              make_double2(acc[mt][nt][2 * h], acc[mt][nt][2 * h + 1]);
      }
    return;
  }

  // Epilogue: C += acc, element-wise bounds checks.
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = m0 + wm * 64 + mt * 16 + g + 8 * h;
      if (row >= m) continue;
      double* crow = c + size_t(row) * ldc;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int col = n0 + wn * 32 + nt * 8 + 2 * q;
        if (col < n) crow[col] += acc[mt][nt][2 * h];
        if (col + 1 < n) crow[col + 1] += acc[mt][nt][2 * h + 1];
      }
    }
}

// ---------------------------------------------------------------------------
// Second form, for large products: A and B packed once into K-contiguous,
// 16-byte-aligned buffers (the mask of the masked GEMM applied while packing),
// tiles staged by TMA (two 128 x 16-double boxes per operand per K step, 128-
// byte swizzle) issued by one thread, so the warps only load fragments and
// issue DMMAs.  Same tile order, warp layout, k permutation, epilogue and K
// split of the last wave as the first form.
// ---------------------------------------------------------------------------
__device__ int g_dgemm_error;

constexpr uint32_t BOX_BYTES = 128 * 16 * 8;      // 16 KB: 128 rows x 16 doubles
constexpr uint32_t OP_BYTES = 2 * BOX_BYTES;      // one operand tile, 128 x 32
constexpr uint32_t TSTAGE = 2 * OP_BYTES;         // A and B
constexpr size_t TMA_SMEM = size_t(STAGES) * TSTAGE + 1024 + 64;

// Double offset of element (r, kp) (kp < 32) in a 128 x 32 operand tile laid
// down by two TMA boxes with 128-byte swizzle: 16-byte chunk (kp % 16) / 2 of
// row r sits at chunk position ((kp % 16) / 2) ^ (r % 8).
__device__ __forceinline__ int tma_off(int r, int kp) {
  return (kp >> 4) * (128 * 16) + r * 16 + ((((kp & 15) >> 1) ^ (r & 7)) << 1) + (kp & 1);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%3, %4}], [%2];" ::"r"(tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(tc::smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}

__global__ void __launch_bounds__(THREADS, 1)
dgemm_tma_kernel(double* __restrict__ c, int m, int n, int k, size_t ldc,
                 const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 TailSplit tail) {
  extern __shared__ uint8_t tsmem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tsmem_raw) + 1023) &
                                           ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + STAGES * TSTAGE);
  int* err = &g_dgemm_error;

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warp grid
  const int g = lane >> 2, q = lane & 3;

  const int tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  const bool split = tail.splits > 0 && int(blockIdx.x) >= tail.full;
  const int job = split ? int(blockIdx.x) - tail.full : 0;
  const int tile = split ? tail.full + job / tail.splits : int(blockIdx.x);
  const int per_group = GROUP_M * tiles_n;
  const int group = tile / per_group;
  const int first_m = group * GROUP_M;
  const int gsz = min(tiles_m - first_m, GROUP_M);
  const int in_group = tile % per_group;
  const int m0 = (first_m + in_group % gsz) * BM;
  const int n0 = (in_group / gsz) * BN;
  const int kall = (k + BK - 1) / BK;
  const int sidx = split ? job % tail.splits : 0;
  const int kt0 = split ? int((long long)sidx * kall / tail.splits) : 0;
  const int kt1 = split ? int((long long)(sidx + 1) * kall / tail.splits) : kall;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) tc::mbar_init(&full[s], 1);
    tc::mbar_fence_init();
    tc::prefetch_tensormap(&tmA);
    tc::prefetch_tensormap(&tmB);
  }
  __syncthreads();
  auto issue = [&](int kt) {  // thread 0: both operand tiles of K step kt
    const int s = (kt - kt0) % STAGES;
    uint8_t* st = sm + s * TSTAGE;
    tc::mbar_arrive_expect_tx(&full[s], TSTAGE);
    tma_load_2d(st, &tmA, &full[s], kt * BK, m0);
    tma_load_2d(st + BOX_BYTES, &tmA, &full[s], kt * BK + 16, m0);
    tma_load_2d(st + OP_BYTES, &tmB, &full[s], kt * BK, n0);
    tma_load_2d(st + OP_BYTES + BOX_BYTES, &tmB, &full[s], kt * BK + 16, n0);
  };
  if (tid == 0)
    for (int kt = kt0; kt < min(kt1, kt0 + STAGES - 1); ++kt) issue(kt);

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

  bool ok = true;
  int kfail = kt1;
  for (int kt = kt0; kt < kt1 && ok; ++kt) {
    __syncthreads();  // every warp is done with step kt-1: its stage can be refilled
    if (tid == 0 && kt + STAGES - 1 < kt1) issue(kt + STAGES - 1);
    const int s = (kt - kt0) % STAGES;
    if (!tc::mbar_wait(&full[s], ((kt - kt0) / STAGES) & 1, err, 51)) {
      ok = false;
      kfail = kt;
      break;
    }
    const double* A_s = reinterpret_cast<const double*>(sm + s * TSTAGE);
    const double* B_s = reinterpret_cast<const double*>(sm + s * TSTAGE + OP_BYTES);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 8) {
      double2 av[4][2], bv[4];
#pragma unroll
      // k pair of this lane: the step at kk % 16 == 0 reads the even 16-byte
      // chunks of the box row, the next one the odd chunks, so that after the
      // swizzle (chunk ^ row % 8) the 8 lanes of a quarter warp (rows g, g^1)
      // hit 8 different chunks.  A and B use the same order of k.
      const int kp = (kk & 16) + 4 * q + ((kk >> 2) & 2);
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int r = wm * 64 + mt * 16 + g;
        av[mt][0] = *reinterpret_cast<const double2*>(A_s + tma_off(r, kp));
        av[mt][1] = *reinterpret_cast<const double2*>(A_s + tma_off(r + 8, kp));
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int r = wn * 32 + nt * 8 + g;
        bv[nt] = *reinterpret_cast<const double2*>(B_s + tma_off(r, kp));
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
          dmma_16x8x8(acc[mt][nt], av[mt][0].x, av[mt][1].x, av[mt][0].y, av[mt][1].y, bv[nt].x,
                      bv[nt].y);
    }
  }
  if (!ok) {  // the copies issued for steps kfail .. kfail+STAGES-1 land before the CTA exits
    if (tid == 0)
      for (int kt = kfail; kt < min(kt1, kfail + STAGES); ++kt) {
        const int s2 = (kt - kt0) % STAGES;
        tc::mbar_wait(&full[s2], ((kt - kt0) / STAGES) & 1, err, 52, true);
      }
    return;
  }

  if (split) {  // the partial tile, dense 128 x 128, to the workspace
    double* w = tail.ws + size_t(job) * (BM * BN);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = wm * 64 + mt * 16 + g + 8 * h;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
          *reinterpret_cast<double2*>(w + r * BN + wn * 32 + nt * 8 + 2 * q) =
              make_double2(acc[mt][nt][2 * h], acc[mt][nt][2 * h + 1]);
      }
    return;
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = m0 + wm * 64 + mt * 16 + g + 8 * h;
      if (row >= m) continue;
      double* crow = c + size_t(row) * ldc;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int col = n0 + wn * 32 + nt * 8 + 2 * q;
        if (col < n) crow[col] += acc[mt][nt][2 * h];
        if (col + 1 < n) crow[col + 1] += acc[mt][nt][2 * h + 1];
      }
    }
}

// The TMA kernel with K-step activity maps (act_m: [tiles_m][ksteps], act_n:
// [tiles_n][ksteps], nonzero = the tile has a nonzero operand row in that K
// step): a CTA runs only the K steps active for both of its tiles.  No K split.
__global__ void __launch_bounds__(THREADS, 1)
dgemm_tma_act_kernel(double* __restrict__ c, int m, int n, int k, size_t ldc,
                     const __grid_constant__ CUtensorMap tmA,
                     const __grid_constant__ CUtensorMap tmB, const uint8_t* __restrict__ act_m,
                     const uint8_t* __restrict__ act_n) {
  const TailSplit tail{0, 0, nullptr};
  extern __shared__ uint8_t tsmem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tsmem_raw) + 1023) &
                                           ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + STAGES * TSTAGE);
  int* err = &g_dgemm_error;

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warp grid
  const int g = lane >> 2, q = lane & 3;

  const int tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  const bool split = tail.splits > 0 && int(blockIdx.x) >= tail.full;
  const int job = split ? int(blockIdx.x) - tail.full : 0;
  const int tile = split ? tail.full + job / tail.splits : int(blockIdx.x);
  const int per_group = GROUP_M * tiles_n;
  const int group = tile / per_group;
  const int first_m = group * GROUP_M;
  const int gsz = min(tiles_m - first_m, GROUP_M);
  const int in_group = tile % per_group;
  const int m0 = (first_m + in_group % gsz) * BM;
  const int n0 = (in_group / gsz) * BN;
  const int kall = (k + BK - 1) / BK;
  const int sidx = split ? job % tail.splits : 0;
  const int kt0 = split ? int((long long)sidx * kall / tail.splits) : 0;
  const int kt1 = split ? int((long long)(sidx + 1) * kall / tail.splits) : kall;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) tc::mbar_init(&full[s], 1);
    tc::mbar_fence_init();
    tc::prefetch_tensormap(&tmA);
    tc::prefetch_tensormap(&tmB);
  }
  __syncthreads();
  const uint8_t* am = act_m + size_t(m0 / BM) * kall;
  const uint8_t* an = act_n + size_t(n0 / BN) * kall;
  auto next = [&](int kt) {  // first K step >= kt that this CTA runs
    while (kt < kt1 && !(am[kt] && an[kt])) ++kt;
    return kt;
  };
  auto issue = [&](int kt, int s) {  // thread 0: both operand tiles of K step kt into stage s
    uint8_t* st = sm + s * TSTAGE;
    tc::mbar_arrive_expect_tx(&full[s], TSTAGE);
    tma_load_2d(st, &tmA, &full[s], kt * BK, m0);
    tma_load_2d(st + BOX_BYTES, &tmA, &full[s], kt * BK + 16, m0);
    tma_load_2d(st + OP_BYTES, &tmB, &full[s], kt * BK, n0);
    tma_load_2d(st + OP_BYTES + BOX_BYTES, &tmB, &full[s], kt * BK + 16, n0);
  };
  // steps are consumed in order: the i-th one issued goes to stage i % STAGES
  int kiss = next(kt0), nissued = 0;
  for (; nissued < STAGES - 1 && kiss < kt1; ++nissued, kiss = next(kiss + 1))
    if (tid == 0) issue(kiss, nissued % STAGES);

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

  bool ok = true;
  int ncons = 0;
  for (int kt = next(kt0); kt < kt1; kt = next(kt + 1), ++ncons) {
    __syncthreads();  // every warp is done with the previous step: its stage can be refilled
    if (kiss < kt1) {
      if (tid == 0) issue(kiss, nissued % STAGES);
      ++nissued;
      kiss = next(kiss + 1);
    }
    const int s = ncons % STAGES;
    if (!tc::mbar_wait(&full[s], (ncons / STAGES) & 1, err, 51)) {
      ok = false;
      break;
    }
    const double* A_s = reinterpret_cast<const double*>(sm + s * TSTAGE);
    const double* B_s = reinterpret_cast<const double*>(sm + s * TSTAGE + OP_BYTES);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 8) {
      double2 av[4][2], bv[4];
#pragma unroll
      // k pair of this lane: the step at kk % 16 == 0 reads the even 16-byte
      // chunks of the box row, the next one the odd chunks, so that after the
      // swizzle (chunk ^ row % 8) the 8 lanes of a quarter warp (rows g, g^1)
      // hit 8 different chunks.  A and B use the same order of k.
      const int kp = (kk & 16) + 4 * q + ((kk >> 2) & 2);
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int r = wm * 64 + mt * 16 + g;
        av[mt][0] = *reinterpret_cast<const double2*>(A_s + tma_off(r, kp));
        av[mt][1] = *reinterpret_cast<const double2*>(A_s + tma_off(r + 8, kp));
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int r = wn * 32 + nt * 8 + g;
        bv[nt] = *reinterpret_cast<const double2*>(B_s + tma_off(r, kp));
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
          dmma_16x8x8(acc[mt][nt], av[mt][0].x, av[mt][1].x, av[mt][0].y, av[mt][1].y, bv[nt].x,
                      bv[nt].y);
    }
  }
  if (!ok) {  // the copies issued and not consumed land before the CTA exits
    if (tid == 0)
      for (int i = ncons; i < nissued; ++i)
        tc::mbar_wait(&full[i % STAGES], (i / STAGES) & 1, err, 52, true);
    return;
  }

  if (split) {  // the partial tile, dense 128 x 128, to the workspace
    double* w = tail.ws + size_t(job) * (BM * BN);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = wm * 64 + mt * 16 + g + 8 * h;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
          *reinterpret_cast<double2*>(w + r * BN + wn * 32 + nt * 8 + 2 * q) =
              make_double2(acc[mt][nt][2 * h], acc[mt][nt][2 * h + 1]);
      }
    return;
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = m0 + wm * 64 + mt * 16 + g + 8 * h;
      if (row >= m) continue;
      double* crow = c + size_t(row) * ldc;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int col = n0 + wn * 32 + nt * 8 + 2 * q;
        if (col < n) crow[col] += acc[mt][nt][2 * h];
        if (col + 1 < n) crow[col + 1] += acc[mt][nt][2 * h + 1];
      }
    }
}

// dst[r][kk] = src[r * ld + kk] (kk < k), 0 for k <= kk < kpad: rows of a
// K-contiguous operand.  A warp per row, 256 columns per block.
__global__ void __launch_bounds__(256)
pack_rows(double* __restrict__ dst, const double* __restrict__ src, size_t ld, int rows, int k,
          int kpad) {
  const int r = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (r >= rows) return;
  const double* srow = src + size_t(r) * ld;
  double* drow = dst + size_t(r) * kpad;
  for (int j = threadIdx.x & 31; j < 256; j += 32) {
    const int kk = blockIdx.x * 256 + j;
    if (kk < kpad) drow[kk] = kk < k ? srow[kk] : 0.0;
  }
}

// dst[j][p] = src[p * ld + j] for p < k (0 for k <= p < kpad), j < cols: the
// transpose into a K-contiguous operand, through a 32 x 32 shared tile.  With
// a mask, element (p, j) is zero unless tab[p * ldtab + j / blk].
__global__ void __launch_bounds__(256)
pack_transpose(double* __restrict__ dst, const double* __restrict__ src, size_t ld, int cols,
               int k, int kpad, const uint8_t* __restrict__ tab, size_t ldtab, int blk) {
  __shared__ double t[32][33];
  const int j0 = blockIdx.x * 32, p0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
#pragma unroll
  for (int i = 0; i < 32; i += 8) {
    const int p = p0 + ty + i, j = j0 + tx;
    double v = 0.0;
    if (p < k && j < cols) {
      v = src[size_t(p) * ld + j];
      if (tab && !tab[size_t(p) * ldtab + j / blk]) v = 0.0;
    }
    t[ty + i][tx] = v;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 32; i += 8) {
    const int j = j0 + ty + i, p = p0 + tx;
    if (j < cols && p < kpad) dst[size_t(j) * kpad + p] = t[tx][ty + i];
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &qr) ==
            cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

// 2-D map of a packed operand: rows x kpad doubles, 128 x 16 boxes, 128-byte swizzle.
bool make_operand_map(CUtensorMap* map, const double* base, int rows, int kpad) {
  auto enc = encode_fn();
  if (!enc) return false;
  cuuint64_t dims[2] = {cuuint64_t(kpad), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(kpad) * sizeof(double)};
  cuuint32_t box[2] = {16, 128};
  cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C[tile] += the splits' partial tiles, added in split order (deterministic).
__global__ void __launch_bounds__(256)
dgemm_tail_reduce(double* __restrict__ c, const double* __restrict__ ws, int m, int n,
                  size_t ldc, int full, int splits) {
  const int tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  const int tile = full + blockIdx.x;
  const int per_group = GROUP_M * tiles_n;
  const int group = tile / per_group;
  const int first_m = group * GROUP_M;
  const int gsz = min(tiles_m - first_m, GROUP_M);
  const int in_group = tile % per_group;
  const int m0 = (first_m + in_group % gsz) * BM;
  const int n0 = (in_group / gsz) * BN;
  const double* w = ws + size_t(blockIdx.x) * splits * (BM * BN);
  for (int e = threadIdx.x; e < BM * BN; e += 256) {
    const int r = e / BN, cc = e % BN;
    if (m0 + r >= m || n0 + cc >= n) continue;
    double v = 0.0;
    for (int s2 = 0; s2 < splits; ++s2) v += w[size_t(s2) * (BM * BN) + e];
    double* dst = c + size_t(m0 + r) * ldc + n0 + cc;
    *dst += v;
  }
}

int sm_count() {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nsm;
}

template <bool TA, bool TB>
cudaError_t launch_t(double* c, const double* a, const double* b, int m, int n, int k,
                     size_t lda, size_t ldb, size_t ldc, ColMask mask, cudaStream_t stream) {
  auto kern = dgemm_fp64_kernel<TA, TB>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(SMEM_BYTES));
  if (err != cudaSuccess) return err;
  const long long tiles = (long long)((m + BM - 1) / BM) * ((n + BN - 1) / BN);
  if (tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  // One CTA per SM: a last wave of `tail` < nsm tiles leaves SMs idle, so its
  // tiles are split along K (at least 4 K steps per split) over them.
  const int nsm = sm_count();
  const int kall = (k + BK - 1) / BK;
  TailSplit ts{0, 0, nullptr};
  if (nsm > 0 && tiles > nsm && tiles % nsm != 0) {
    const int tail = int(tiles % nsm);
    const int splits = std::min(nsm / tail, kall / 4);
    if (splits >= 2) {
      ts.full = int(tiles - tail);
      ts.splits = splits;
      err = cudaMallocAsync(reinterpret_cast<void**>(&ts.ws),
                            size_t(tail) * splits * BM * BN * sizeof(double), stream);
      if (err != cudaSuccess) return err;
    }
  }
  const long long grid = ts.splits ? ts.full + (tiles - ts.full) * ts.splits : tiles;
  kern<<<unsigned(grid), THREADS, SMEM_BYTES, stream>>>(c, a, b, m, n, k, lda, ldb, ldc, mask,
                                                         ts);
  err = cudaGetLastError();
  if (ts.splits) {
    if (err == cudaSuccess) {
      dgemm_tail_reduce<<<unsigned(tiles - ts.full), 256, 0, stream>>>(c, ts.ws, m, n, ldc,
                                                                       ts.full, ts.splits);
      err = cudaGetLastError();
    }
    const cudaError_t e2 = cudaFreeAsync(ts.ws, stream);
    if (err == cudaSuccess) err = e2;
  }
  return err;
}

// The TMA form: pack A and B, build their tensor maps, run, release.
cudaError_t launch_packed(double* c, const double* a, const double* b, int m, int n, int k,
                          size_t lda, size_t ldb, size_t ldc, bool transa, bool transb,
                          ColMask mask, cudaStream_t stream) {
  const int kpad = (k + 7) / 8 * 8;
  double* ws = nullptr;
  cudaError_t err = cudaMallocAsync(reinterpret_cast<void**>(&ws),
                                    (size_t(m) + n) * kpad * sizeof(double), stream);
  if (err != cudaSuccess) return err;
  double* ap = ws;
  double* bp = ws + size_t(m) * kpad;
  if (!transa)
    pack_rows<<<dim3((kpad + 255) / 256, (m + 7) / 8), 256, 0, stream>>>(ap, a, lda, m, k, kpad);
  else
    pack_transpose<<<dim3((m + 31) / 32, (kpad + 31) / 32), 256, 0, stream>>>(
        ap, a, lda, m, k, kpad, nullptr, 0, 1);
  if (transb)
    pack_rows<<<dim3((kpad + 255) / 256, (n + 7) / 8), 256, 0, stream>>>(bp, b, ldb, n, k, kpad);
  else
    pack_transpose<<<dim3((n + 31) / 32, (kpad + 31) / 32), 256, 0, stream>>>(
        bp, b, ldb, n, k, kpad, mask.tab, mask.ldtab, mask.blk);
  err = cudaGetLastError();
  CUtensorMap tmA, tmB;
  if (err == cudaSuccess &&
      (!make_operand_map(&tmA, ap, m, kpad) || !make_operand_map(&tmB, bp, n, kpad)))
    err = cudaErrorInvalidValue;
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(dgemm_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(TMA_SMEM));
  const long long tiles = (long long)((m + BM - 1) / BM) * ((n + BN - 1) / BN);
  const int nsm = sm_count();
  const int kall = (k + BK - 1) / BK;
  TailSplit ts{0, 0, nullptr};
  if (err == cudaSuccess && nsm > 0 && tiles > nsm && tiles % nsm != 0) {
    const int tail = int(tiles % nsm);
    const int splits = std::min(nsm / tail, kall / 4);
    if (splits >= 2) {
      ts.full = int(tiles - tail);
      ts.splits = splits;
      err = cudaMallocAsync(reinterpret_cast<void**>(&ts.ws),
                            size_t(tail) * splits * BM * BN * sizeof(double), stream);
      if (err != cudaSuccess) ts.splits = 0;
    }
  }
  if (err == cudaSuccess) {
    const long long grid = ts.splits ? ts.full + (tiles - ts.full) * ts.splits : tiles;
    dgemm_tma_kernel<<<unsigned(grid), THREADS, TMA_SMEM, stream>>>(c, m, n, k, ldc, tmA, tmB, ts);
    err = cudaGetLastError();
    if (err == cudaSuccess && ts.splits) {
      dgemm_tail_reduce<<<unsigned(tiles - ts.full), 256, 0, stream>>>(c, ts.ws, m, n, ldc,
                                                                       ts.full, ts.splits);
      err = cudaGetLastError();
    }
  }
  if (ts.ws) cudaFreeAsync(ts.ws, stream);
  const cudaError_t e2 = cudaFreeAsync(ws, stream);
  return err != cudaSuccess ? err : e2;
}

// ---------------------------------------------------------------------------
// Fock-build contraction V[u][v] += sum_g phi_lhs[u][g] w[g] phi_rhs[v][g] over
// the u, v active in g's block: a product of the masked (and, on the left,
// weighted) operands packed K-contiguous, K = grid points, run by the TMA
// kernel with its K-step activity maps.
// ---------------------------------------------------------------------------
// dst[u][g] = tab[u][g / blk] ? src[u][g] * (w ? w[g] : 1) : 0 for g < ngrid, 0
// up to kpad.  A warp per row, 256 points per block.
__global__ void __launch_bounds__(256)
pack_masked(double* __restrict__ dst, const double* __restrict__ src, size_t ld, int rows,
            int ngrid, int kpad, const uint8_t* __restrict__ tab, size_t ldtab, int blk,
            const double* __restrict__ w) {
  const int r = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (r >= rows) return;
  const double* srow = src + size_t(r) * ld;
  const uint8_t* trow = tab + size_t(r) * ldtab;
  double* drow = dst + size_t(r) * kpad;
  for (int j = threadIdx.x & 31; j < 256; j += 32) {
    const int g = blockIdx.x * 256 + j;
    if (g >= kpad) continue;
    double v = 0.0;
    if (g < ngrid && trow[g / blk]) v = w ? srow[g] * w[g] : srow[g];
    drow[g] = v;
  }
}

// act[t][kt] = some AO of 128-row tile t is active in a block that K step kt
// (points 32kt .. 32kt+31) touches.
__global__ void __launch_bounds__(256)
tile_activity(uint8_t* __restrict__ act, const uint8_t* __restrict__ tab, size_t ldtab, int nao,
              int ngrid, int blk, int ksteps) {
  const int t = blockIdx.y;
  for (int kt = blockIdx.x * 256 + threadIdx.x; kt < ksteps; kt += gridDim.x * 256) {
    const int g0 = kt * BK, g1 = min(ngrid, g0 + BK) - 1;
    const int b0 = g0 / blk, b1 = g1 / blk;
    uint8_t any = 0;
    for (int u = t * BM; u < min(nao, t * BM + BM) && !any; ++u)
      for (int b = b0; b <= b1; ++b) any |= tab[size_t(u) * ldtab + b];
    act[size_t(t) * ksteps + kt] = any ? 1 : 0;
  }
}

}  // namespace

size_t fock_fp64_workspace(int nao, int ngrid) {
  const size_t kpad = (size_t(ngrid) + 7) / 8 * 8;
  const size_t tiles = (size_t(nao) + BM - 1) / BM, ksteps = (size_t(ngrid) + BK - 1) / BK;
  return 2 * size_t(nao) * kpad * sizeof(double) + (tiles * ksteps + 255) / 256 * 256 + 256;
}

cudaError_t fock_fp64(double* v, size_t ldv, const double* w, const double* ao_lhs,
                      const double* ao_rhs, size_t stride_grid, int nao, int ngrid,
                      const uint8_t* tab, size_t ldtab, int blk, bool pack_rhs, void* workspace,
                      cudaStream_t stream) {
  if (nao <= 0 || ngrid <= 0) return cudaSuccess;
  const int kpad = (ngrid + 7) / 8 * 8;
  const int ksteps = (ngrid + BK - 1) / BK;
  const int tiles = (nao + BM - 1) / BM;
  double* ap = static_cast<double*>(workspace);
  double* bp = ap + size_t(nao) * kpad;
  uint8_t* act = reinterpret_cast<uint8_t*>(bp + size_t(nao) * kpad);
  const dim3 pgrid((kpad + 255) / 256, (nao + 7) / 8);
  pack_masked<<<pgrid, 256, 0, stream>>>(ap, ao_lhs, stride_grid, nao, ngrid, kpad, tab, ldtab,
                                         blk, w);
  if (pack_rhs) {  // the right operand and the activity map change only with phi and the mask
    pack_masked<<<pgrid, 256, 0, stream>>>(bp, ao_rhs, stride_grid, nao, ngrid, kpad, tab, ldtab,
                                           blk, nullptr);
    tile_activity<<<dim3((ksteps + 255) / 256, tiles), 256, 0, stream>>>(act, tab, ldtab, nao,
                                                                         ngrid, blk, ksteps);
  }
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  CUtensorMap tmA, tmB;
  if (!make_operand_map(&tmA, ap, nao, kpad) || !make_operand_map(&tmB, bp, nao, kpad))
    return cudaErrorInvalidValue;
  if ((err = cudaFuncSetAttribute(dgemm_tma_act_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, int(TMA_SMEM))) !=
      cudaSuccess)
    return err;
  const long long ntiles = (long long)tiles * tiles;
  dgemm_tma_act_kernel<<<unsigned(ntiles), THREADS, TMA_SMEM, stream>>>(v, nao, nao, ngrid, ldv,
                                                                        tmA, tmB, act, act);
  return cudaGetLastError();
}

namespace {

// Products from this many flops on use the packed TMA form (the packing costs
// one pass over A and B); CFGMM_DGEMM_PACK_MIN_FLOPS overrides, < 0 disables.
bool use_packed(int m, int n, int k) {
  static const double min_flops = [] {
    const char* e = std::getenv("CFGMM_DGEMM_PACK_MIN_FLOPS");
    return e ? std::atof(e) : 2e9;
  }();
  return min_flops >= 0 && 2.0 * m * n * k >= min_flops && k >= 2 * BK;
}

}  // namespace

cudaError_t dgemm_fp64(double* c, const double* a, const double* b, int m, int n, int k,
                       size_t lda, size_t ldb, size_t ldc, bool transa, bool transb,
                       cudaStream_t stream) {
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  const ColMask none{nullptr, 0, 1};
  if (use_packed(m, n, k))
    return launch_packed(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, none, stream);
  if (!transa && !transb)
    return launch_t<false, false>(c, a, b, m, n, k, lda, ldb, ldc, none, stream);
  if (!transa && transb)
    return launch_t<false, true>(c, a, b, m, n, k, lda, ldb, ldc, none, stream);
  if (transa && !transb)
    return launch_t<true, false>(c, a, b, m, n, k, lda, ldb, ldc, none, stream);
  return launch_t<true, true>(c, a, b, m, n, k, lda, ldb, ldc, none, stream);
}

cudaError_t dgemm_fp64_non0tab(double* c, const double* a, const double* b, int m, int n, int k,
                               size_t lda, size_t ldb, size_t ldc, bool transa,
                               const uint8_t* tab, size_t ldtab, int blk, cudaStream_t stream) {
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  const ColMask mask{tab, ldtab, blk};
  if (use_packed(m, n, k))
    return launch_packed(c, a, b, m, n, k, lda, ldb, ldc, transa, false, mask, stream);
  if (!transa) return launch_t<false, false>(c, a, b, m, n, k, lda, ldb, ldc, mask, stream);
  return launch_t<true, false>(c, a, b, m, n, k, lda, ldb, ldc, mask, stream);
}

cudaError_t dgemm_reset_error(cudaStream_t stream) {
  static const int zero = 0;
  return cudaMemcpyToSymbolAsync(g_dgemm_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice,
                                 stream);
}

cudaError_t dgemm_read_error(int* code) {
  return cudaMemcpyFromSymbol(code, g_dgemm_error, sizeof(int));
}

}  // namespace cfgmm
