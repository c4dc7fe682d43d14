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
//   * CTA tile 128x128, K step 16, 8 warps in a 2x4 grid (warp tile 64x32,
//     4x4 MMA tiles, 64 FP64 accumulators per thread), 4-stage cp.async ring.
//   * Every operand tile is stored "K-contiguous" in shared memory
//     (As[m][k], Bs[n][k]) whatever transa/transb are: the global->shared
//     copies do the transposition, with the thread->element map chosen so that
//     global reads stay coalesced for each transpose case.
//   * 8-byte cp.async keeps any lda/ldb (odd ld, as in the 3527x6581x9583
//     workload) and any base alignment legal; out-of-range elements are
//     zero-filled, so edge tiles need no separate path.
//   * The k index inside each 8-wide group is permuted (thread q of a quad
//     holds k = 2q and 2q+1), so each fragment load is one 16-byte
//     shared-memory load; the same permutation is applied to A and B, which
//     leaves the sum unchanged up to FP64 rounding order.
#include "common.cuh"
#include "dgemm_fp64.cuh"

namespace cfgmm {
namespace {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 4, THREADS = 256, GROUP_M = 8;
constexpr int TILE_DOUBLES = BM * BK;  // As or Bs per stage (BM == BN)
constexpr size_t SMEM_BYTES = size_t(STAGES) * 2 * TILE_DOUBLES * sizeof(double);

// Copies one BMxBK tile of op(X) (X = A, or B viewed as its transpose) into
// shared memory as S[r][k], r < 128 rows of op(X) ("m" for A, "n" for B).
//   kRowsContig: X's rows are the 128-dim (element (r,k) at x[r*ld + k], k
//   contiguous); otherwise element (r,k) is at x[k*ld + r], r contiguous.
template <bool kRowsContig>
__device__ __forceinline__ void load_tile(double* S, const double* x, size_t ld, int r0, int k0,
                                          int rmax, int kmax, int tid) {
  if (kRowsContig) {
    // 16 threads sweep the 16 contiguous k of one row: 128-byte segments.
    const int k = tid & 15;
    const int rb = tid >> 4;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = rb + 16 * i;
      const bool ok = (r0 + r < rmax) && (k0 + k < kmax);
      const double* src = ok ? x + size_t(r0 + r) * ld + (k0 + k) : x;
      cp_async_8(S + swz<BK>(r, k), src, ok);
    }
  } else {
    // 128 threads sweep the 128 contiguous r of one k: 1-KB segments.
    const int r = tid & 127;
    const int kb = tid >> 7;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = kb + 2 * i;
      const bool ok = (r0 + r < rmax) && (k0 + k < kmax);
      const double* src = ok ? x + size_t(k0 + k) * ld + (r0 + r) : x;
      cp_async_8(S + swz<BK>(r, k), src, ok);
    }
  }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_fp64_kernel(double* __restrict__ c, const double* __restrict__ a,
                  const double* __restrict__ b, int m, int n, int k, size_t lda, size_t ldb,
                  size_t ldc) {
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
  const int per_group = GROUP_M * tiles_n;
  const int group = blockIdx.x / per_group;
  const int first_m = group * GROUP_M;
  const int gsz = min(tiles_m - first_m, GROUP_M);
  const int in_group = blockIdx.x % per_group;
  const int m0 = (first_m + in_group % gsz) * BM;
  const int n0 = (in_group / gsz) * BN;
  const int ktiles = (k + BK - 1) / BK;

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

  // A: rows m, k contiguous unless transposed.  B: rows n, k contiguous only
  // when transposed (b[j*ldb + p]).
  auto issue = [&](int kt) {
    const int st = kt % STAGES;
    load_tile<!TA>(As + st * TILE_DOUBLES, a, lda, m0, kt * BK, m, k, tid);
    load_tile<TB>(Bs + st * TILE_DOUBLES, b, ldb, n0, kt * BK, n, k, tid);
  };

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) issue(s);
    cp_async_commit();
  }

  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    if (kt + STAGES - 1 < ktiles) issue(kt + STAGES - 1);
    cp_async_commit();

    const double* A_s = As + (kt % STAGES) * TILE_DOUBLES;
    const double* B_s = Bs + (kt % STAGES) * TILE_DOUBLES;
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
        for (int nt = 0; nt < 4; ++nt) {
          dmma_16x8x4(acc[mt][nt], av[mt][0].x, av[mt][1].x, bv[nt].x);
          dmma_16x8x4(acc[mt][nt], av[mt][0].y, av[mt][1].y, bv[nt].y);
        }
    }
  }
  cp_async_wait<0>();

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

template <bool TA, bool TB>
cudaError_t launch_t(double* c, const double* a, const double* b, int m, int n, int k,
                     size_t lda, size_t ldb, size_t ldc, cudaStream_t stream) {
  auto kern = dgemm_fp64_kernel<TA, TB>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(SMEM_BYTES));
  if (err != cudaSuccess) return err;
  const long long tiles = (long long)((m + BM - 1) / BM) * ((n + BN - 1) / BN);
  if (tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  kern<<<unsigned(tiles), THREADS, SMEM_BYTES, stream>>>(c, a, b, m, n, k, lda, ldb, ldc);
  return cudaGetLastError();
}

}  // namespace

cudaError_t dgemm_fp64(double* c, const double* a, const double* b, int m, int n, int k,
                       size_t lda, size_t ldb, size_t ldc, bool transa, bool transb,
                       cudaStream_t stream) {
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  if (!transa && !transb) return launch_t<false, false>(c, a, b, m, n, k, lda, ldb, ldc, stream);
  if (!transa && transb) return launch_t<false, true>(c, a, b, m, n, k, lda, ldb, ldc, stream);
  if (transa && !transb) return launch_t<true, false>(c, a, b, m, n, k, lda, ldb, ldc, stream);
  return launch_t<true, true>(c, a, b, m, n, k, lda, ldb, ldc, stream);
}

}  // namespace cfgmm
