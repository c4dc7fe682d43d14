// aodmao2rho_split.cu -- the masked AO-DM-AO contraction in split precision
// on the INT8 tensor cores (tcgen05.mma kind::i8), by the slice form of the
// Ozaki scheme (Ozaki, Ogita, Oishi and Rump 2012), restated here:
//
//   Every row u of D_s is scaled by 2^tau_u and every grid point g of phi by
//   2^sigma_g so that the scaled values are below 2^6 in magnitude; each is
//   then written as seven signed digits  x' = sum_{j<7} x_j 2^(-7j)  with
//   x_0 in [-64, 64] and x_j in [-64, 64] (round to nearest at every step), 48
//   bits in all.  The products of the digits of D and phi whose levels add up
//   to L = i + j <= 6 are summed EXACTLY in one INT32 accumulator per level:
//     S_L[u][g] = sum_{i+j=L} sum_v d_i(u,v) p_j(v,g)        (28 INT8 MMAs)
//   and X[u][g] = 2^-(tau_u + sigma_g) sum_L 2^(-7L) S_L[u][g] in FP64.  The
//   dropped levels L >= 7 weigh at most 2^-49 of the scaled products, so X
//   carries about 46 bits relative to sum_v |D_uv| |phi_vg|.
//
// The contraction itself follows aodmao2rho_loop_parallel
// (src/impl_aodmao2rho.rs:171-244): per grid block b the active list I(b) of
// AOs (the reference's compaction, impl_matmul_non0tab.rs:118-129) is built on
// the device, X = D_s[I,I] phi[I, tile] is formed over the compacted lists,
// and rho[s][g] += sum_{u in I} phi[u][g] X[u][g].
//
// Kernels:
//   split_d_slices    one CTA per row of D_s: row scale, 7 digits per element
//                     stored as 8 bytes, so the gather of one element is one
//                     8-byte load -- the same traffic as the FP64 kernel.
//   split_phi_sigma / split_phi_slices   per (block, 64-point tile): point
//                     scales and the digit tiles of phi[I(b), tile], written
//                     chunk by chunk (32 compacted AOs) directly in the UMMA
//                     32-byte-swizzled K-major layout, so one bulk copy moves
//                     the 7 digit tiles of a chunk into shared memory.
//   split_build       work list (block tile, 128-row tile of I(b), DM) and
//                     chunk offsets.
//   split_main        persistent, 6 warps: warps 0-3 gather the D digits of
//                     128 rows x 32 compacted columns (thread = row), transpose
//                     the bytes into 7 swizzled A tiles and later run the
//                     epilogue; warp 5 bulk-loads the phi digit tiles; warp 4
//                     issues the 28 MMAs of a chunk (M=128, N=64, K=32) into 7
//                     TMEM level accumulators (448 of 512 columns).  The
//                     epilogue rebuilds X in FP64, weights it with phi and
//                     reduces over the 128 rows; X never leaves the SM.
//   split_reduce      adds the row-tile partial sums in a fixed order.
// Every mbarrier wait is bounded (tcgen05.cuh).
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "aodmao2rho_fp64.cuh"
#include "aodmao2rho_split.cuh"
#include "tcgen05.cuh"

namespace cfgmm {
namespace {

constexpr int TU = 128;   // compacted rows per item (TMEM lanes)
constexpr int TG = 64;    // grid points per item
constexpr int TK = 32;    // compacted columns per chunk (one INT8 MMA K step)
constexpr int NSL = 7;    // digits per value
constexpr int STAGES = 4;
constexpr uint32_t A_SLICE = TU * TK;        // 4096 B
constexpr uint32_t B_SLICE = TG * TK;        // 2048 B
constexpr uint32_t A_STAGE = NSL * A_SLICE;  // 28672 B
constexpr uint32_t B_STAGE = NSL * B_SLICE;  // 14336 B
constexpr uint32_t STAGE = A_STAGE + B_STAGE;
constexpr int THREADS = 192;
constexpr int kBadExp = INT_MAX;  // scale of a row / point holding Inf or NaN

__device__ int g_split_error;

__device__ __forceinline__ int exp_for(double amax) {  // 2^6 > amax * 2^exp
  if (!(amax <= 1.7976931348623157e308)) return kBadExp;
  if (amax == 0.0) return 0;
  int E;
  frexp(amax, &E);
  return 6 - E;
}

// x (|x| < 2^6 after scaling) -> 7 signed digits, x = sum_j d_j 2^(-7j) + O(2^-49).
__device__ __forceinline__ void digits(double x, int (&d)[NSL]) {
  double r = x;
#pragma unroll
  for (int j = 0; j < NSL; ++j) {
    const double t = rint(r);
    d[j] = int(t);
    r = (r - t) * 128.0;  // exact
  }
}

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  return (uint32_t(a) & 0xffu) | ((uint32_t(b) & 0xffu) << 8) | ((uint32_t(c) & 0xffu) << 16) |
         ((uint32_t(d) & 0xffu) << 24);
}

// ---------------------------------------------------------------------------
// D digits: dsl[s][u][v] = 8 bytes (digits 0..6, 0), tau[s][u]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
split_d_slices(const double* __restrict__ dms, size_t stride_ao, size_t dm_stride, int nao,
               uint2* __restrict__ dsl, int* __restrict__ tau) {
  const int row = blockIdx.x;  // s * nao + u
  const int s = row / nao, u = row % nao;
  const double* d = dms + size_t(s) * dm_stride + size_t(u) * stride_ao;
  double mx = 0.0;
  bool bad = false;
  for (int v = threadIdx.x; v < nao; v += 256) {
    const double a = fabs(d[v]);
    bad |= !(a <= 1.7976931348623157e308);
    mx = fmax(mx, a);
  }
  __shared__ double red[8];
  __shared__ int badw[8];
  __shared__ int e_s;
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    bad |= __shfl_xor_sync(0xffffffffu, int(bad), o) != 0;
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = mx;
    badw[threadIdx.x >> 5] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    int b = 0;
    for (int w = 0; w < 8; ++w) {
      m = fmax(m, red[w]);
      b |= badw[w];
    }
    e_s = b ? kBadExp : exp_for(m);
    tau[row] = e_s;
  }
  __syncthreads();
  const int e = e_s;
  uint2* out = dsl + size_t(row) * nao;
  for (int v = threadIdx.x; v < nao; v += 256) {
    int dg[NSL] = {0, 0, 0, 0, 0, 0, 0};
    if (e != kBadExp) digits(ldexp(d[v], e), dg);
    out[v] = make_uint2(pack4(dg[0], dg[1], dg[2], dg[3]), pack4(dg[4], dg[5], dg[6], 0));
  }
}

// ---------------------------------------------------------------------------
// phi scales: sigma[g] for the 64 points of each (block, tile)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(64)
split_phi_sigma(const double* __restrict__ ao, size_t stride_grid, const int* __restrict__ lists,
                const int* __restrict__ counts, int nao, int ngrid, int blk, int gsub,
                int* __restrict__ sigma) {
  const int bg = blockIdx.x;
  const int b = bg / gsub, gt = bg % gsub;
  const int g0 = b * blk + gt * TG;
  const int gend = min(min((b + 1) * blk, ngrid), g0 + TG);
  const int g = g0 + threadIdx.x;
  if (g >= gend) return;
  const int nb = counts[b];
  const int* I = lists + size_t(b) * nao;
  double mx = 0.0;
  bool bad = false;
  for (int i = 0; i < nb; ++i) {
    const double a = fabs(ao[size_t(I[i]) * stride_grid + g]);
    bad |= !(a <= 1.7976931348623157e308);
    mx = fmax(mx, a);
  }
  sigma[g] = bad ? kBadExp : exp_for(mx);
}

// phi digit tiles: for chunk c of (block tile bg), digit j: a 64 x 32-byte
// K-major tile (row = point, byte = compacted AO within the chunk) in the
// 32-byte-swizzled layout, at phisl + ((cbase[bg] + c) * 7 + j) * 2048.
__global__ void __launch_bounds__(256)
split_phi_slices(const double* __restrict__ ao, size_t stride_grid,
                 const int* __restrict__ lists, const int* __restrict__ counts,
                 const int* __restrict__ cbase, const int* __restrict__ sigma, int nao, int ngrid,
                 int blk, int gsub, uint8_t* __restrict__ phisl) {
  const int bg = blockIdx.x;
  const int b = bg / gsub, gt = bg % gsub;
  const int g0 = b * blk + gt * TG;
  const int gend = min(min((b + 1) * blk, ngrid), g0 + TG);
  const int nb = counts[b];
  const int kc = (nb + TK - 1) / TK;
  const int* I = lists + size_t(b) * nao;
  uint8_t* base = phisl + size_t(cbase[bg]) * NSL * B_SLICE;
  // units: (chunk c, point row g, quad q of 4 compacted AOs): kc * 64 * 8
  for (int unit = threadIdx.x; unit < kc * TG * 8; unit += 256) {
    const int c = unit / (TG * 8);
    const int rem = unit % (TG * 8);
    const int gr = rem >> 3, q = rem & 7;
    const int g = g0 + gr;
    const int e = (g < gend) ? sigma[g] : 0;
    int dg[4][NSL];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int i = c * TK + q * 4 + t;
#pragma unroll
      for (int j = 0; j < NSL; ++j) dg[t][j] = 0;
      if (g < gend && i < nb && e != kBadExp)
        digits(ldexp(ao[size_t(I[i]) * stride_grid + g], e), dg[t]);
    }
    uint8_t* tile0 = base + size_t(c) * NSL * B_SLICE;
    const uint32_t off = tc::sw32_offset(uint32_t(gr), uint32_t(q >> 2)) + uint32_t(q & 3) * 4;
#pragma unroll
    for (int j = 0; j < NSL; ++j)
      *reinterpret_cast<uint32_t*>(tile0 + j * B_SLICE + off) =
          pack4(dg[0][j], dg[1][j], dg[2][j], dg[3][j]);
  }
}

// ---------------------------------------------------------------------------
// work list: cbase[bg] (prefix of chunk counts), items (bg, utile, s), total
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
split_build(const int* __restrict__ counts, int nbg, int gsub, int nset, int max_ut,
            int* __restrict__ cbase, int4* __restrict__ items, int* __restrict__ total) {
  __shared__ int warp_c[32], warp_i[32];
  __shared__ int base_c, base_i;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) base_c = base_i = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nbg; b0 += 1024) {
    const int bg = b0 + tid;
    const int nb = (bg < nbg) ? counts[bg / gsub] : 0;
    const int kc = (nb + TK - 1) / TK;
    const int nut = (nb + TU - 1) / TU;
    int ic = kc, ii = nut;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int tc_ = __shfl_up_sync(0xffffffffu, ic, o);
      const int ti = __shfl_up_sync(0xffffffffu, ii, o);
      if (lane >= o) {
        ic += tc_;
        ii += ti;
      }
    }
    if (lane == 31) {
      warp_c[warp] = ic;
      warp_i[warp] = ii;
    }
    __syncthreads();
    int bc = base_c, bi = base_i;
    for (int w = 0; w < warp; ++w) {
      bc += warp_c[w];
      bi += warp_i[w];
    }
    bc += ic - kc;
    bi += ii - nut;
    if (bg < nbg) {
      cbase[bg] = bc;
      for (int u = 0; u < nut; ++u) items[bi + u] = make_int4(bg, u, 0, 0);
    }
    __syncthreads();
    if (tid == 0) {
      for (int w = 0; w < 32; ++w) {
        base_c += warp_c[w];
        base_i += warp_i[w];
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    cbase[nbg] = base_c;
    total[0] = base_i * nset;  // items are (tile item, set): set-major order
    total[1] = base_i;
  }
}

// ---------------------------------------------------------------------------
// main kernel
// ---------------------------------------------------------------------------
struct MainArgs {
  const uint2* dsl;
  const int* tau;
  const uint8_t* phisl;
  const int* sigma;
  const double* ao_lhs;
  const int* lists;
  const int* counts;
  const int* cbase;
  const int4* items;
  const int* total;  // [0] items x sets, [1] items per set
  double* partial;   // [(bg * max_ut + ut) * nset + s][TG]
  size_t stride_grid;
  int nao, ngrid, nset, blk, gsub, max_ut;
};

// 4x4 byte transpose: out_i holds byte i of w0..w3 (w_t in byte t).
__device__ __forceinline__ void transpose4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3,
                                           uint32_t& o0, uint32_t& o1, uint32_t& o2,
                                           uint32_t& o3) {
  const uint32_t a = __byte_perm(w0, w1, 0x5140);  // w0.b0 w1.b0 w0.b1 w1.b1
  const uint32_t b = __byte_perm(w0, w1, 0x7362);  // w0.b2 w1.b2 w0.b3 w1.b3
  const uint32_t c = __byte_perm(w2, w3, 0x5140);
  const uint32_t d = __byte_perm(w2, w3, 0x7362);
  o0 = __byte_perm(a, c, 0x5410);
  o1 = __byte_perm(a, c, 0x7632);
  o2 = __byte_perm(b, d, 0x5410);
  o3 = __byte_perm(b, d, 0x7632);
}

__global__ void __launch_bounds__(THREADS, 1) split_main(MainArgs p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE);
  uint64_t* full_a = bars;
  uint64_t* full_b = bars + STAGES;
  uint64_t* empty = bars + 2 * STAGES;
  uint64_t* acc_full = bars + 3 * STAGES;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 3);
  __shared__ double red[4][TG];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* err = &g_split_error;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full_a[s], 128);
      tc::mbar_init(&full_b[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(acc_full, 1);
    tc::mbar_init(acc_empty, 128);
    tc::mbar_init(drain, 1);
    tc::mbar_fence_init();
  }
  if (warp == 4) {
    tc::tmem_alloc(tmem_slot, 512);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const int total = p.total[0], per_set = p.total[1];

  if (warp < 4) {
    // ---------------- gather D digits, then the epilogue ----------------
    const int tid = threadIdx.x;  // tile row
    uint32_t uses[STAGES] = {0, 0, 0, 0};
    int stage = 0;
    uint32_t nitem = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++nitem) {
      const int s = t / per_set;
      const int4 it = p.items[t % per_set];
      const int bg = it.x, ut = it.y;
      const int b = bg / p.gsub, gt = bg % p.gsub;
      const int nb = p.counts[b];
      const int kc = (nb + TK - 1) / TK;
      const int* I = p.lists + size_t(b) * p.nao;
      const int row = ut * TU + tid;
      const bool rvalid = row < nb;
      const int iu = rvalid ? I[row] : 0;
      const uint2* drow = p.dsl + (size_t(s) * p.nao + iu) * p.nao;
      for (int c = 0; c < kc; ++c) {
        if (uses[stage] > 0 && !tc::mbar_wait(&empty[stage], (uses[stage] - 1) & 1, err, 11)) {
          ok = false;
          break;
        }
        uint2 w[TK];
#pragma unroll
        for (int j = 0; j < TK; ++j) {
          const int k = c * TK + j;
          const int iv = (k < nb) ? __ldg(I + k) : -1;
          w[j] = (rvalid && iv >= 0) ? __ldg(drow + iv) : make_uint2(0u, 0u);
        }
        uint8_t* As = smem + stage * STAGE;
#pragma unroll
        for (int h = 0; h < 2; ++h) {  // 16-byte halves of the row (16 columns each)
          uint32_t o[NSL][4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {  // 4 columns per 32-bit word
            const int j0 = h * 16 + q * 4;
            uint32_t x0, x1, x2, x3, y0, y1, y2, y3;
            transpose4(w[j0].x, w[j0 + 1].x, w[j0 + 2].x, w[j0 + 3].x, x0, x1, x2, x3);
            transpose4(w[j0].y, w[j0 + 1].y, w[j0 + 2].y, w[j0 + 3].y, y0, y1, y2, y3);
            o[0][q] = x0;
            o[1][q] = x1;
            o[2][q] = x2;
            o[3][q] = x3;
            o[4][q] = y0;
            o[5][q] = y1;
            o[6][q] = y2;
          }
          const uint32_t off = tc::sw32_offset(uint32_t(tid), uint32_t(h));
#pragma unroll
          for (int sl = 0; sl < NSL; ++sl)
            *reinterpret_cast<uint4*>(As + sl * A_SLICE + off) =
                make_uint4(o[sl][0], o[sl][1], o[sl][2], o[sl][3]);
        }
        tc::fence_proxy_async_smem();
        tc::mbar_arrive(&full_a[stage]);
        ++uses[stage];
        stage = (stage + 1) % STAGES;
      }
      if (!ok) break;
      // ---- epilogue: rho partial over the 128 rows of this item ----
      if (!tc::mbar_wait(acc_full, nitem & 1, err, 12)) break;
      tc::fence_after_sync();
      const int g0 = b * p.blk + gt * TG;
      const int gw = min(min((b + 1) * p.blk, p.ngrid), g0 + TG) - g0;
      const int tu = p.tau[size_t(s) * p.nao + iu];
      const double* lrow = p.ao_lhs + size_t(iu) * p.stride_grid + g0;
      const uint32_t trow = tmem + (uint32_t(32 * warp) << 16);
#pragma unroll 1
      for (int cc = 0; cc < TG; cc += 16) {
        uint32_t v[NSL][16];
#pragma unroll
        for (int L = 0; L < NSL; ++L) tc::tmem_ld_32x32b_x16(trow + uint32_t(L * TG + cc), v[L]);
        tc::tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int gl = cc + j;
          double contrib = 0.0;
          if (rvalid && gl < gw) {
            double x = double(int(v[NSL - 1][j]));
#pragma unroll
            for (int L = NSL - 2; L >= 0; --L) x = fma(x, 0.0078125, double(int(v[L][j])));
            const int sg = p.sigma[g0 + gl];
            contrib = (tu == kBadExp || sg == kBadExp)
                          ? __longlong_as_double(0x7ff8000000000000LL)
                          : ldexp(x, -(tu + sg)) * lrow[gl];
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
          if (lane == 0) red[warp][gl] = contrib;
        }
      }
      tc::fence_before_sync();
      tc::mbar_arrive(acc_empty);  // the MMA warp may overwrite the accumulators
      asm volatile("bar.sync 1, 128;" ::: "memory");
      if (tid < TG) {
        const size_t slot = (size_t(bg) * p.max_ut + ut) * p.nset + s;
        p.partial[slot * TG + tid] = red[0][tid] + red[1][tid] + red[2][tid] + red[3][tid];
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
    }
  } else if (warp == 4) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_i8(TU, TG);
      uint32_t fuse[STAGES] = {0, 0, 0, 0};
      int stage = 0;
      uint32_t nitem = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++nitem) {
        const int4 it = p.items[t % per_set];
        const int nb = p.counts[it.x / p.gsub];
        const int kc = (nb + TK - 1) / TK;
        if (nitem > 0 && !tc::mbar_wait(acc_empty, (nitem - 1) & 1, err, 13)) break;
        tc::fence_after_sync();
        for (int c = 0; c < kc; ++c) {
          if (!tc::mbar_wait(&full_a[stage], fuse[stage] & 1, err, 14) ||
              !tc::mbar_wait(&full_b[stage], fuse[stage] & 1, err, 15)) {
            ok = false;
            break;
          }
          ++fuse[stage];
          tc::fence_after_sync();
          const uint32_t a0 = tc::smem_u32(smem + stage * STAGE);
          const uint32_t b0 = a0 + A_STAGE;
#pragma unroll
          for (int L = 0; L < NSL; ++L)
#pragma unroll
            for (int i = 0; i <= L; ++i)
              tc::mma_i8(tmem + uint32_t(L * TG), tc::smem_desc_k32(a0 + i * A_SLICE),
                         tc::smem_desc_k32(b0 + (L - i) * B_SLICE), idesc, c > 0 || i > 0);
          tc::mma_commit(&empty[stage]);
          stage = (stage + 1) % STAGES;
        }
        if (!ok) break;
        tc::mma_commit(acc_full);
      }
      tc::mma_commit(drain);
      tc::mbar_wait(drain, 0, err, 16, true);
    }
  } else {
    // ---------------- phi digit tiles: bulk loads ----------------
    if (lane == 0) {
      uint32_t uses[STAGES] = {0, 0, 0, 0};
      int stage = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
        const int4 it = p.items[t % per_set];
        const int nb = p.counts[it.x / p.gsub];
        const int kc = (nb + TK - 1) / TK;
        const uint8_t* src = p.phisl + size_t(p.cbase[it.x]) * B_STAGE;
        for (int c = 0; c < kc; ++c) {
          if (uses[stage] > 0 && !tc::mbar_wait(&empty[stage], (uses[stage] - 1) & 1, err, 17)) {
            ok = false;
            break;
          }
          tc::mbar_arrive_expect_tx(&full_b[stage], B_STAGE);
          tc::bulk_load(smem + stage * STAGE + A_STAGE, src + size_t(c) * B_STAGE, B_STAGE,
                        &full_b[stage]);
          ++uses[stage];
          stage = (stage + 1) % STAGES;
        }
      }
      for (int s = 0; s < STAGES; ++s)
        if (uses[s] > 0) tc::mbar_wait(&full_b[s], (uses[s] - 1) & 1, err, 18, true);
    }
  }

  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 4) tc::tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------------------
// deterministic reduction of the row-tile partials into rho
// ---------------------------------------------------------------------------
__global__ void split_reduce(double* __restrict__ rhos, const double* __restrict__ partial,
                             const int* __restrict__ counts, size_t stride_grid, int ngrid,
                             int nset, int blk, int gsub, int max_ut, int nbg) {
  const int bg = blockIdx.x;
  if (bg >= nbg) return;
  const int b = bg / gsub, gt = bg % gsub;
  const int nt = (counts[b] + TU - 1) / TU;
  if (nt == 0) return;  // fully masked block: rho untouched
  const int g0 = b * blk + gt * TG;
  const int gend = min(min((b + 1) * blk, ngrid), g0 + TG);
  for (int t = threadIdx.x; t < nset * TG; t += blockDim.x) {
    const int s = t / TG, j = t % TG;
    if (g0 + j >= gend) continue;
    double v = 0.0;
    for (int u = 0; u < nt; ++u) v += partial[((size_t(bg) * max_ut + u) * nset + s) * TG + j];
    double* r = rhos + size_t(s) * stride_grid + g0 + j;
    *r = v + *r;
  }
}

size_t a256(size_t v) { return (v + 255) / 256 * 256; }

struct Layout {
  size_t lists, counts, cbase, items, total, dsl, tau, sigma, phisl, partial, bytes;
};

Layout layout(size_t nao, size_t ngrid, size_t nset, size_t blk) {
  const size_t nblk = (ngrid + blk - 1) / blk;
  const size_t gsub = (blk + TG - 1) / TG;
  const size_t nbg = nblk * gsub;
  const size_t max_ut = (nao + TU - 1) / TU;
  const size_t max_kc = (nao + TK - 1) / TK;
  Layout L;
  L.lists = 0;
  L.counts = L.lists + a256(nblk * nao * sizeof(int));
  L.cbase = L.counts + a256(nblk * sizeof(int));
  L.items = L.cbase + a256((nbg + 1) * sizeof(int));
  L.total = L.items + a256(nbg * max_ut * sizeof(int4));
  L.dsl = L.total + 256;
  L.tau = L.dsl + a256(nset * nao * nao * 8);
  L.sigma = L.tau + a256(nset * nao * sizeof(int));
  L.phisl = L.sigma + a256(ngrid * sizeof(int));
  L.partial = L.phisl + a256(nbg * max_kc * B_STAGE);
  L.bytes = L.partial + nbg * max_ut * nset * TG * sizeof(double);
  return L;
}

}  // namespace

size_t aodmao2rho_split_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk) {
  return layout(nao, ngrid, nset, blk).bytes;
}

cudaError_t aodmao2rho_split(double* rhos, const double* dms, const double* ao_lhs,
                             const double* ao_rhs, size_t stride_ao, size_t stride_grid, int nao,
                             int ngrid, int nset, const uint8_t* tab, size_t ldtab, int blk,
                             void* workspace, cudaStream_t stream) {
  if (nao <= 0 || ngrid <= 0 || nset <= 0) return cudaSuccess;
  const int nblk = (ngrid + blk - 1) / blk;
  const int gsub = (blk + TG - 1) / TG;
  const int nbg = nblk * gsub;
  const int max_ut = (nao + TU - 1) / TU;
  const Layout L = layout(nao, ngrid, nset, blk);
  char* ws = static_cast<char*>(workspace);
  int* lists = reinterpret_cast<int*>(ws + L.lists);
  int* counts = reinterpret_cast<int*>(ws + L.counts);
  int* cbase = reinterpret_cast<int*>(ws + L.cbase);
  int4* items = reinterpret_cast<int4*>(ws + L.items);
  int* total = reinterpret_cast<int*>(ws + L.total);
  uint2* dsl = reinterpret_cast<uint2*>(ws + L.dsl);
  int* tau = reinterpret_cast<int*>(ws + L.tau);
  int* sigma = reinterpret_cast<int*>(ws + L.sigma);
  uint8_t* phisl = reinterpret_cast<uint8_t*>(ws + L.phisl);
  double* partial = reinterpret_cast<double*>(ws + L.partial);

  cudaError_t err = aodm_block_lists_launch(tab, ldtab, nao, nblk, lists, counts, stream);
  if (err != cudaSuccess) return err;
  split_build<<<1, 1024, 0, stream>>>(counts, nbg, gsub, nset, max_ut, cbase, items, total);
  split_d_slices<<<nset * nao, 256, 0, stream>>>(dms, stride_ao, stride_ao * stride_ao, nao, dsl,
                                                 tau);
  split_phi_sigma<<<nbg, TG, 0, stream>>>(ao_rhs, stride_grid, lists, counts, nao, ngrid, blk,
                                          gsub, sigma);
  split_phi_slices<<<nbg, 256, 0, stream>>>(ao_rhs, stride_grid, lists, counts, cbase, sigma, nao,
                                            ngrid, blk, gsub, phisl);
  if ((err = cudaGetLastError()) != cudaSuccess) return err;

  MainArgs a;
  a.dsl = dsl;
  a.tau = tau;
  a.phisl = phisl;
  a.sigma = sigma;
  a.ao_lhs = ao_lhs;
  a.lists = lists;
  a.counts = counts;
  a.cbase = cbase;
  a.items = items;
  a.total = total;
  a.partial = partial;
  a.stride_grid = stride_grid;
  a.nao = nao;
  a.ngrid = ngrid;
  a.nset = nset;
  a.blk = blk;
  a.gsub = gsub;
  a.max_ut = max_ut;
  constexpr size_t smem = size_t(STAGES) * STAGE + 1024 + 256;
  if ((err = cudaFuncSetAttribute(split_main, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem))) != cudaSuccess)
    return err;
  int dev = 0, nsm = 0;
  if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
  if ((err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return err;
  split_main<<<nsm, THREADS, smem, stream>>>(a);
  if ((err = cudaGetLastError()) != cudaSuccess) return err;
  split_reduce<<<nbg, 128, 0, stream>>>(rhos, partial, counts, stride_grid, ngrid, nset, blk, gsub,
                                        max_ut, nbg);
  return cudaGetLastError();
}

cudaError_t aodmao2rho_split_reset_error(cudaStream_t stream) {
  static const int zero = 0;
  return cudaMemcpyToSymbolAsync(g_split_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice,
                                 stream);
}

cudaError_t aodmao2rho_split_read_error(int* code) {
  return cudaMemcpyFromSymbol(code, g_split_error, sizeof(int));
}

}  // namespace cfgmm
