// aodmao2rho_split.cu -- the masked AO-DM-AO contraction in split precision
// on the INT8 tensor cores (tcgen05.mma kind::i8), by the slice form of the
// Ozaki scheme (Ozaki, Ogita, Oishi and Rump 2012), restated here:
//
//   Every row u of D_s is scaled by 2^tau_u and every grid point g of phi by
//   2^sigma_g so that the scaled values are below 2^6 in magnitude; each is
//   then written as seven signed base-256 digits  x' = sum_{j<7} x_j 2^(-8j)
//   with x_0 in [-64, 64] and x_j in [-128, 127], read off the bytes of the
//   integer round(x' 2^48) (digits_packed below).  The products of the
//   digits of D and phi whose levels add up to L = i + j <= 6 are summed
//   EXACTLY in one INT32 accumulator per level:
//     S_L[u][g] = sum_{i+j=L} sum_v d_i(u,v) p_j(v,g)        (28 INT8 MMAs)
//   and X[u][g] = 2^-(tau_u + sigma_g) sum_L 2^(-8L) S_L[u][g] in FP64.  The
//   dropped levels L >= 7 weigh at most 6 * 2^-54 of the largest scaled
//   product and the digit remainders 2^-55 each, so X carries about 51 bits
//   relative to sum_v |D_uv| |phi_vg|.  |S_L| <= 7 * 2^14 * nao keeps the
//   INT32 sums exact for nao <= 16384.
//
// The contraction itself follows aodmao2rho_loop_parallel
// (src/impl_aodmao2rho.rs:171-244): per grid block b the active list I(b) of
// AOs (the reference's compaction, impl_matmul_non0tab.rs:118-129) is built on
// the device, X = D_s[I,I] phi[I, tile] is formed over the compacted lists,
// and rho[s][g] += sum_{u in I} phi[u][g] X[u][g].
//
// Kernels:
//   split_d_slices    a warp per row of D_s: row scale, 7 digits per element
//                     stored as 8 bytes, so the gather of one element is one
//                     8-byte load -- the same traffic as the FP64 kernel.
//   split_phi_max     per (64-point tile, slab of 64 active AOs): max |phi|
//                     per point, combined by atomic max.
//   split_phi_digits  per (64-point tile, chunk of 32 active AOs): point
//                     scales and the digit tiles of phi[I(b), tile], staged in
//                     shared memory and written out in the UMMA
//                     32-byte-swizzled K-major layout, so one bulk copy moves
//                     the 7 digit tiles of a chunk into shared memory.
//   split_build       work list (block tile, 128-row tile of I(b), DM) and
//                     chunk offsets.
//   split_main        persistent, 14 warps: warps 0-11 gather the D digits of
//                     128 rows x 32 compacted columns in three groups of four
//                     that take turns by chunk (a lane loads 8 bytes; lanes
//                     along a row read consecutive columns; two shuffle rounds
//                     turn the 8-byte elements into digit planes, stored
//                     without bank conflicts) and later run the epilogue;
//                     warp 12 issues the 28 MMAs of a chunk (M=128, N=64, K=32)
//                     into 7 TMEM level accumulators (448 columns), grouped by
//                     D digit so that each D plane is read once and reused
//                     from the tensor core's collector buffer; warp 13
//                     bulk-loads the phi digit tiles.  The epilogue rebuilds X
//                     in FP64, weights it with phi and reduces over the rows
//                     of each warp; X never leaves the SM.
//   split_reduce      adds the (row tile, warp) partial sums in a fixed order.
// Every mbarrier wait is bounded (tcgen05.cuh).
#include <cuda_runtime.h>

#include <climits>
#include <cstdlib>
#include <cstdint>

#include "aodmao2rho_fp64.cuh"
#include "aodmao2rho_split.cuh"
#include "side_stream.cuh"
#include "tcgen05.cuh"

namespace cfgmm {
namespace {

constexpr int TU = 128;   // compacted rows per item (TMEM lanes)
constexpr int TG = 64;    // grid points per item
constexpr int TK = 32;    // compacted columns per chunk (one INT8 MMA K step)
constexpr int NSL = 7;    // digits per value
constexpr int kDefaultStages = 3;  // pipeline depth (CFGMM_SPLIT_STAGES overrides: 3..5)
constexpr uint32_t A_SLICE = TU * TK;        // 4096 B
constexpr uint32_t B_SLICE = TG * TK;        // 2048 B
constexpr uint32_t A_STAGE = NSL * A_SLICE;  // 28672 B
constexpr uint32_t B_STAGE = NSL * B_SLICE;  // 14336 B
constexpr uint32_t STAGE = A_STAGE + B_STAGE;
constexpr int NGROUPS = 3;                    // gather groups of four warps (128 rows each)
constexpr int GATHER_WARPS = 4 * NGROUPS;
// points of an item's epilogue per group: multiples of 8 (the TMEM load width)
constexpr int EPI_SPAN = (TG / NGROUPS + 7) / 8 * 8;
static_assert(EPI_SPAN <= 32 && NGROUPS * EPI_SPAN >= TG, "a lane holds one point scale");
// A group's consecutive chunks of an item are NGROUPS apart in the stage
// sequence, and its wait for a stage names the phase by parity only: with at
// least NGROUPS stages the phase before the awaited one has completed by then
// (the group's own previous wait saw a later MMA finish), so a parity wait
// cannot pass a phase early.  Across items the epilogue's accumulator wait
// orders every MMA of the previous item first.
constexpr int kMinStages = NGROUPS;
static_assert(kDefaultStages >= kMinStages, "default pipeline too shallow for the groups");
constexpr int THREADS = 32 * (GATHER_WARPS + 2);
constexpr int EPI_PARTS = 4;                  // partial sums per item (one per row quarter)
constexpr int kBadExp = INT_MAX;  // scale of a row / point holding Inf or NaN

__device__ int g_split_error;

__device__ __forceinline__ int exp_for(double amax) {  // 2^6 > amax * 2^exp
  if (!(amax <= 1.7976931348623157e308)) return kBadExp;
  if (amax == 0.0) return 0;
  int E;
  frexp(amax, &E);
  return 6 - E;
}

// 2^k for k in [-1022, 1023].
__device__ __forceinline__ double pow2(int k) {
  return __longlong_as_double(static_cast<long long>(k + 1023) << 52);
}

// The 7 digits of x * 2^e (|x * 2^e| < 2^6) packed as bytes 0..6 (byte 7 = 0).
// X = round(x * 2^(e+48)) is an integer below 2^54 in magnitude; adding
// 0x808080808080 = 128 * sum_{j<6} 256^j makes every low byte u_j of the sum
// the unsigned form of a balanced digit u_j - 128 in [-128, 127] (flipping
// bit 7 of the byte turns it into that signed byte), and leaves
// floor((X + 0x808080808080) / 2^48) in [-64, 64] as the leading digit:
//   X = d_0 256^6 + sum_{j=1..6} d_j 256^(6-j),  x 2^e = sum_j d_j 2^(-8j) + r 2^-48,
// |r| <= 1/2.  The scaling by 2^(e+48) is done in two exact halves.
__device__ __forceinline__ uint2 digits_packed(double x, int e) {
  const int k = e + 48;
  const int k1 = k / 2;
  const long long X = __double2ll_rn(x * pow2(k1) * pow2(k - k1));
  const unsigned long long Z =
      static_cast<unsigned long long>(X + 0x808080808080LL) ^ 0x808080808080ULL;
  const uint32_t lo = static_cast<uint32_t>(Z);        // d6 d5 d4 d3
  const uint32_t hi = static_cast<uint32_t>(Z >> 32);  // d2 d1 d0 (sign byte)
  return make_uint2(__byte_perm(hi, lo, 0x7012), __byte_perm(lo, 0u, 0x4012));
}

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

// ---------------------------------------------------------------------------
// D digits: dsl[s][u][v] = 8 bytes (digits 0..6, 0), tau[s][u]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
split_d_slices(const double* __restrict__ dms, size_t stride_ao, size_t dm_stride, int nao,
               int nrows, uint2* __restrict__ dsl, int* __restrict__ tau,
               const int* __restrict__ asym) {
  const int row = blockIdx.x * 8 + (threadIdx.x >> 5);  // s * nao + u, a warp per row
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const bool half_diag = asym != nullptr && *asym == 0;
  const int s = row / nao, u = row % nao;
  const double* d = dms + size_t(s) * dm_stride + size_t(u) * stride_ao;
  double mx = 0.0;
  bool bad = false;
#pragma unroll 4
  for (int v = lane; v < nao; v += 32) {
    const double a = fabs(d[v]);
    bad |= !(a <= 1.7976931348623157e308);
    mx = fmax(mx, a);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    bad |= __shfl_xor_sync(0xffffffffu, int(bad), o) != 0;
  }
  const int e = bad ? kBadExp : exp_for(mx);
  if (lane == 0) tau[row] = e;
  uint2* out = dsl + size_t(row) * nao;
#pragma unroll 4
  for (int v = lane; v < nao; v += 32)
    out[v] = e != kBadExp ? digits_packed(half_diag && v == u ? 0.5 * d[v] : d[v], e)
                          : make_uint2(0u, 0u);
}

// ---------------------------------------------------------------------------
// phi, step 1: pmax[g] = max |phi[u][g]| over the active AOs u of g's block
// (+Inf when one of them is Inf or NaN).  CTA (block tile, slab of 64
// compacted AOs): 64 points x 4 row groups, then one atomic max per point on
// the bit pattern (non-negative doubles order like their bits); pmax starts at 0.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
split_phi_max(const double* __restrict__ ao, size_t stride_grid, const int* __restrict__ lists,
              const int* __restrict__ counts, int nao, int ngrid, int blk, int gsub,
              unsigned long long* __restrict__ pmax) {
  const int bg = blockIdx.x, slab = blockIdx.y;
  const int b = bg / gsub, gt = bg % gsub;
  const int nb = counts[b];
  const int i0 = slab * 64;
  if (i0 >= nb) return;
  const int g0 = b * blk + gt * TG;
  const int gend = min(min((b + 1) * blk, ngrid), g0 + TG);
  const int* I = lists + size_t(b) * nao;
  const int gr = threadIdx.x & (TG - 1), rg = threadIdx.x >> 6;
  const int g = g0 + gr;
  __shared__ double red[4][TG];
  double mx = 0.0;
  if (g < gend) {
    bool bad = false;
    const int iend = min(nb, i0 + 64);
#pragma unroll 4
    for (int i = i0 + rg; i < iend; i += 4) {
      const double a = fabs(ao[size_t(__ldg(I + i)) * stride_grid + g]);
      bad |= !(a <= 1.7976931348623157e308);
      mx = fmax(mx, a);
    }
    if (bad) mx = __longlong_as_double(0x7ff0000000000000LL);
  }
  red[rg][gr] = mx;
  __syncthreads();
  if (threadIdx.x < TG && g < gend) {
    const double m = fmax(fmax(red[0][gr], red[1][gr]), fmax(red[2][gr], red[3][gr]));
    atomicMax(pmax + g, static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

// ---------------------------------------------------------------------------
// phi, step 2: sigma[g] and, for chunk c of (block tile bg) and digit j, a
// 64 x 32-byte K-major tile (row = point, byte = compacted AO within the
// chunk) in the 32-byte-swizzled layout, at phisl + ((cbase[bg] + c) * 7 + j) * 2048.
// CTA (block tile, chunk).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
split_phi_digits(const double* __restrict__ ao, size_t stride_grid, const int* __restrict__ lists,
                 const int* __restrict__ counts, const int* __restrict__ cbase,
                 const unsigned long long* __restrict__ pmax, int nao, int ngrid, int blk,
                 int gsub, int* __restrict__ sigma, uint8_t* __restrict__ phisl) {
  const int bg = blockIdx.x, c = blockIdx.y;
  const int b = bg / gsub, gt = bg % gsub;
  const int nb = counts[b];
  if (c * TK >= nb) return;
  // staged digit words [digit][quad of 4 AOs][point], rows padded to 68 words
  // so that the read-out below is free of bank conflicts
  __shared__ uint32_t stage[NSL][8][TG + 4];
  const int g0 = b * blk + gt * TG;
  const int gend = min(min((b + 1) * blk, ngrid), g0 + TG);
  const int* I = lists + size_t(b) * nao;
  const int gr = threadIdx.x & (TG - 1), rg = threadIdx.x >> 6;
  const int g = g0 + gr;
  const bool gok = g < gend;
  const int e = gok ? exp_for(__longlong_as_double(static_cast<long long>(pmax[g]))) : 0;
  if (c == 0 && rg == 0 && gok) sigma[g] = e;
#pragma unroll
  for (int hq = 0; hq < 2; ++hq) {
    const int q = rg + 4 * hq;  // quad of 4 compacted AOs
    uint2 w[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int i = c * TK + q * 4 + t;
      w[t] = (gok && i < nb && e != kBadExp)
                 ? digits_packed(ao[size_t(__ldg(I + i)) * stride_grid + g], e)
                 : make_uint2(0u, 0u);
    }
    uint32_t o[8];
    transpose4(w[0].x, w[1].x, w[2].x, w[3].x, o[0], o[1], o[2], o[3]);
    transpose4(w[0].y, w[1].y, w[2].y, w[3].y, o[4], o[5], o[6], o[7]);
#pragma unroll
    for (int j = 0; j < NSL; ++j) stage[j][q][gr] = o[j];
  }
  __syncthreads();
  // write-out: (digit, point row, 16-byte half) vectors, consecutive threads
  // covering consecutive rows -> coalesced 16-byte stores
  uint8_t* tile0 = phisl + (size_t(cbase[bg]) + c) * B_STAGE;
  for (int v = threadIdx.x; v < NSL * TG * 2; v += 256) {
    const int h = v & 1, r = (v >> 1) & (TG - 1), j = v >> 7;
    const uint4 w = make_uint4(stage[j][4 * h][r], stage[j][4 * h + 1][r], stage[j][4 * h + 2][r],
                               stage[j][4 * h + 3][r]);
    *reinterpret_cast<uint4*>(tile0 + j * B_SLICE + tc::sw32_offset(uint32_t(r), uint32_t(h))) = w;
  }
}

// ---------------------------------------------------------------------------
// work list: cbase[bg] (prefix of chunk counts), items (bg, utile, -1, 0), total
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
      for (int u = 0; u < nut; ++u) items[bi + u] = make_int4(bg, u, -1, 0);
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

// Work item t: (64-point tile bg, 128-row tile ut, density matrix s, batch).
// Items with s < 0 come from a list of per_set tiles run once per matrix.
__device__ __forceinline__ int4 item_at(const SplitArgs& p, int t, int per_set) {
  if (p.items[0].z >= 0) return p.items[t];
  int4 it = p.items[t % per_set];
  it.z = t / per_set;
  return it;
}

__device__ __forceinline__ const SplitBatch& batch_of(const SplitArgs& p, int w) {
  return p.batches ? p.batches[w] : p.one;
}

// Byte selector that assembles, from `keep` (bytes 0..3) and `recv` (4..7) of
// the gather's second shuffle round, the digit word of 4 consecutive columns:
// column qd comes from keep.b0, qd^2 from keep.b2, qd^1 from recv.b0 and qd^3
// from recv.b2 (the second digit plane of the lane: +1 on every nibble).
__device__ __forceinline__ uint32_t gather_selector(int qd) {
  uint32_t sel = 0;
#pragma unroll
  for (int col = 0; col < 4; ++col) {
    const uint32_t src = col == qd ? 0u : col == (qd ^ 2) ? 2u : col == (qd ^ 1) ? 4u : 6u;
    sel |= src << (4 * col);
  }
  return sel;
}

template <int STAGES>
__global__ void __launch_bounds__(THREADS, 1) split_main(SplitArgs p) {
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

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* err = &g_split_error;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full_a[s], 4);  // one arrival per warp of a gather group
      tc::mbar_init(&full_b[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(acc_full, 1);
    tc::mbar_init(acc_empty, GATHER_WARPS);
    tc::mbar_init(drain, 1);
    tc::mbar_fence_init();
  }
  if (warp == GATHER_WARPS) {
    tc::tmem_alloc(tmem_slot, 512);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const int total = p.total[0], per_set = p.total[1];
  const bool sym = p.asym != nullptr && *p.asym == 0;

  if (warp < GATHER_WARPS) {
    // ---------------- gather D digits, then the epilogue ----------------
    // Group grp takes the chunks c = grp, grp+NGROUPS, ... of every item; warp wq
    // of the group fills tile rows 32wq .. 32wq+31, four rows per step.
    // Lane (qd, ri, hh) = lane bits (4:3, 2:1, 0) loads, for row 4*step+ri,
    // the columns 16hh + 4k + qd (k = 0..3) and ends up holding digit planes
    // 2qd and 2qd+1 of the 16-byte half hh of that row (plane 7 is the zero
    // padding byte and is not stored).
    const int grp = warp >> 2, wq = warp & 3;
    const int qd = lane >> 3, ri = (lane >> 1) & 3, hh = lane & 1;
    const bool b1 = (qd & 2) != 0, b0 = (qd & 1) != 0;
    const uint32_t sel_a = gather_selector(qd), sel_b = sel_a + 0x1111u;
    // 16-byte loads of phi_lhs when every row segment starts 16-byte aligned
    uint32_t seq0 = 0;  // CTA-wide sequence number of the item's first chunk
    uint32_t nitem = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++nitem) {
      const int4 it = item_at(p, t, per_set);
      const int bg = it.x, ut = it.y, s = it.z;
      const SplitBatch& B = batch_of(p, it.w);
      const int b = bg / p.gsub, gt = bg % p.gsub;
      const int nb = B.counts[b];
      const int kc = (nb + TK - 1) / TK;
      const int kc0 = sym ? ut * (TU / TK) : 0;  // symmetric D: from the tile's own columns on
      const int* I = B.lists + size_t(b) * p.nao;
      const uint2* dset = p.dsl + size_t(s) * p.nao * p.nao;
      int iu[8];
#pragma unroll
      for (int st = 0; st < 8; ++st) {
        const int row = ut * TU + 32 * wq + 4 * st + ri;
        iu[st] = row < nb ? __ldg(I + row) : -1;
      }
      // what the epilogue of this item reads is requested now, while the
      // chunks run: the row's AO index and scale, the point scale of this
      // lane, and the phi_lhs row segment (into L2)
      const int g0 = b * p.blk + gt * TG;
      const int gw = min(min((b + 1) * p.blk, B.ngrid), g0 + TG) - g0;
      const int erow = ut * TU + 32 * wq + lane;
      const bool ev = erow < nb;
      const int eu = ev ? __ldg(I + erow) : 0;
      const int tu = p.tau[size_t(s) * p.nao + eu];
      // the group's epilogue points ep0 .. ep1-1; lane l holds the scale of point ep0 + l
      const int ep0 = grp * EPI_SPAN, ep1 = min(TG, ep0 + EPI_SPAN);
      const int sg_lane = ep0 + lane < min(ep1, gw) ? B.sigma[g0 + ep0 + lane] : 0;
      const double* lrow = B.ao_lhs + size_t(eu) * B.stride_grid + g0;
      if (ev && ep0 < gw) {
        const char* pf = reinterpret_cast<const char*>(lrow + ep0);
        const char* pe = reinterpret_cast<const char*>(lrow + min(gw, ep1));
        for (const char* q = pf; q < pe; q += 128)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(q));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(pe - 8));
      }
      for (int c = kc0 + grp; c < kc; c += NGROUPS) {
        const uint32_t seq = seq0 + uint32_t(c - kc0);
        const int stg = int(seq % STAGES);
        const uint32_t use = seq / STAGES;
        // the loads go out first; the stage has to be free only for the stores
        int iv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int kk = c * TK + 16 * hh + 4 * k + qd;
          iv[k] = kk < nb ? __ldg(I + kk) : -1;
        }
        // symmetric D, diagonal tile: the strict lower triangle (column before
        // row in the compacted order) is left out; elsewhere nothing is
        const int lower_lim = sym && c < kc0 + TU / TK ? c * TK - ut * TU : TU;
        uint2 w[8][4];
#pragma unroll
        for (int st = 0; st < 8; ++st)
#pragma unroll
          for (int k = 0; k < 4; ++k)
            w[st][k] = (iu[st] >= 0 && iv[k] >= 0 &&
                        lower_lim + 16 * hh + 4 * k + qd >= 32 * wq + 4 * st + ri)
                           ? __ldg(dset + size_t(iu[st]) * p.nao + iv[k])
                           : make_uint2(0u, 0u);
        if (use > 0 && !tc::mbar_wait(&empty[stg], (use - 1) & 1, err, 11)) {
          ok = false;
          break;
        }
        uint8_t* As = smem + stg * STAGE;
#pragma unroll
        for (int st = 0; st < 8; ++st) {
          uint32_t wa[4], wb[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            // round 1 (lanes qd, qd^2): keep digits 0-3 (b1 = 0) or 4-7 (b1 = 1)
            const uint32_t x = b1 ? w[st][k].y : w[st][k].x;
            const uint32_t y = __shfl_xor_sync(0xffffffffu, b1 ? w[st][k].x : w[st][k].y, 16);
            // round 2 (lanes qd, qd^1): keep two of those four digits
            const uint32_t lo = __byte_perm(x, y, 0x5410), hi = __byte_perm(x, y, 0x7632);
            const uint32_t keep = b0 ? hi : lo;
            const uint32_t recv = __shfl_xor_sync(0xffffffffu, b0 ? lo : hi, 8);
            wa[k] = __byte_perm(keep, recv, sel_a);
            wb[k] = __byte_perm(keep, recv, sel_b);
          }
          const uint32_t off = tc::sw32_offset(uint32_t(32 * wq + 4 * st + ri), uint32_t(hh));
          *reinterpret_cast<uint4*>(As + (2 * qd) * A_SLICE + off) =
              make_uint4(wa[0], wa[1], wa[2], wa[3]);
          if (qd < 3)
            *reinterpret_cast<uint4*>(As + (2 * qd + 1) * A_SLICE + off) =
                make_uint4(wb[0], wb[1], wb[2], wb[3]);
        }
        tc::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&full_a[stg]);
      }
      seq0 += uint32_t(kc - kc0);
      if (!ok) break;
      // ---- epilogue: group grp reduces points ep0 .. ep1-1 over the
      // 32 rows of warp wq (TMEM lanes 32wq ..) ----
      if (!tc::mbar_wait(acc_full, nitem & 1, err, 12)) break;
      tc::fence_after_sync();
      // 16-byte loads of phi_lhs when every row segment starts 16-byte aligned
      const bool vec2 = (B.stride_grid % 2 == 0) && (p.blk % 2 == 0) &&
                        (reinterpret_cast<uintptr_t>(B.ao_lhs) % 16 == 0);
      const uint32_t trow = tmem + (uint32_t(32 * wq) << 16);
      const size_t slot =
          size_t(B.partial_off) + ((size_t(bg) * p.max_ut + ut) * B.nset + s) * EPI_PARTS + wq;
#pragma unroll 1
      for (int cc = ep0; cc < ep1; cc += 8) {
        double a[8];  // phi_lhs of this row at 8 points, then its products
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
          const int gl = cc + j;
          if (ev && gl + 1 < gw && vec2) {
            const double2 q = *reinterpret_cast<const double2*>(lrow + gl);
            a[j] = q.x;
            a[j + 1] = q.y;
          } else {
            a[j] = (ev && gl < gw) ? lrow[gl] : 0.0;
            a[j + 1] = (ev && gl + 1 < gw) ? lrow[gl + 1] : 0.0;
          }
        }
        uint32_t v[NSL][8];
#pragma unroll
        for (int L = 0; L < NSL; ++L) tc::tmem_ld_32x32b_x8(trow + uint32_t(L * TG + cc), v[L]);
        tc::tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int gl = cc + j;
          const int sg = __shfl_sync(0xffffffffu, sg_lane, gl - ep0);
          if (ev && gl < gw) {
            // X = sum_L S_L 2^-8L: levels 0-2 and 3-6 combined exactly in 64-bit
            // integers (below 2^48 and 2^56), then one FMA
            const long long hi = (static_cast<long long>(int(v[0][j])) << 16) +
                                 (static_cast<long long>(int(v[1][j])) << 8) + int(v[2][j]);
            const long long lo = (static_cast<long long>(int(v[3][j])) << 24) +
                                 (static_cast<long long>(int(v[4][j])) << 16) +
                                 (static_cast<long long>(int(v[5][j])) << 8) + int(v[6][j]);
            const double x = fma(double(lo), 0x1p-48, double(hi) * 0x1p-16);
            const int e = -(tu + sg);
            a[j] = (tu == kBadExp || sg == kBadExp) ? __longlong_as_double(0x7ff8000000000000LL)
                   : (e >= -1022 && e <= 1023)      ? x * pow2(e) * a[j]
                                                    : ldexp(x, e) * a[j];
          }
        }
        // reduce-scatter over the 32 rows: 9 shuffles leave the lanes 4m .. 4m+3
        // with the sum of point m (fixed order: deterministic)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const bool up = (lane & 16) != 0;
          const double keep = up ? a[j + 4] : a[j];
          a[j] = keep + __shfl_xor_sync(0xffffffffu, up ? a[j] : a[j + 4], 16);
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const bool up = (lane & 8) != 0;
          const double keep = up ? a[j + 2] : a[j];
          a[j] = keep + __shfl_xor_sync(0xffffffffu, up ? a[j] : a[j + 2], 8);
        }
        {
          const bool up = (lane & 4) != 0;
          const double keep = up ? a[1] : a[0];
          a[0] = keep + __shfl_xor_sync(0xffffffffu, up ? a[0] : a[1], 4);
        }
        a[0] += __shfl_xor_sync(0xffffffffu, a[0], 2);
        a[0] += __shfl_xor_sync(0xffffffffu, a[0], 1);
        const int m = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
        if ((lane & 3) == 0) p.partial[slot * TG + cc + m] = sym ? 2.0 * a[0] : a[0];
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(acc_empty);  // the MMA warp may overwrite the accumulators
    }
  } else if (warp == GATHER_WARPS) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_i8(TU, TG);
      uint32_t seq = 0, nitem = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++nitem) {
        const int4 it = item_at(p, t, per_set);
        const int nb = batch_of(p, it.w).counts[it.x / p.gsub];
        const int kc = (nb + TK - 1) / TK;
        const int kc0 = sym ? it.y * (TU / TK) : 0;
        if (nitem > 0 && !tc::mbar_wait(acc_empty, (nitem - 1) & 1, err, 13)) break;
        tc::fence_after_sync();
        for (int c = kc0; c < kc; ++c, ++seq) {
          const int stg = int(seq % STAGES);
          const uint32_t par = (seq / STAGES) & 1;
          if (!tc::mbar_wait(&full_a[stg], par, err, 14) ||
              !tc::mbar_wait(&full_b[stg], par, err, 15)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          const uint32_t a0 = tc::smem_u32(smem + stg * STAGE);
          const uint32_t b0 = a0 + A_STAGE;
          // D digit i meets phi digits 0 .. NSL-1-i (levels i .. NSL-1) in
          // consecutive MMAs, so its plane is read from shared memory once and
          // held in the collector buffer for the rest; level L still receives
          // its products in the order i = 0, 1, ..., L.
#pragma unroll
          for (int i = 0; i < NSL; ++i) {
            const uint64_t ad = tc::smem_desc_k32(a0 + i * A_SLICE);
            const bool acc = c > kc0 || i > 0;
#pragma unroll
            for (int L = i; L < NSL; ++L) {
              const uint32_t d = tmem + uint32_t(L * TG);
              const uint64_t bd = tc::smem_desc_k32(b0 + (L - i) * B_SLICE);
              if (i == NSL - 1)
                tc::mma_i8(d, ad, bd, idesc, acc);
              else if (L == i)
                tc::mma_i8_collect<tc::ACollector::kFill>(d, ad, bd, idesc, acc);
              else if (L == NSL - 1)
                tc::mma_i8_collect<tc::ACollector::kLastUse>(d, ad, bd, idesc, acc);
              else
                tc::mma_i8_collect<tc::ACollector::kUse>(d, ad, bd, idesc, acc);
            }
          }
          tc::mma_commit(&empty[stg]);
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
      uint32_t seq = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
        const int4 it = item_at(p, t, per_set);
        const SplitBatch& B = batch_of(p, it.w);
        const int nb = B.counts[it.x / p.gsub];
        const int kc = (nb + TK - 1) / TK;
        const int kc0 = sym ? it.y * (TU / TK) : 0;
        const uint8_t* src = p.phisl + size_t(B.cbase[it.x]) * B_STAGE;
        for (int c = kc0; c < kc; ++c, ++seq) {
          const int stg = int(seq % STAGES);
          const uint32_t use = seq / STAGES;
          if (use > 0 && !tc::mbar_wait(&empty[stg], (use - 1) & 1, err, 17)) {
            ok = false;
            break;
          }
          tc::mbar_arrive_expect_tx(&full_b[stg], B_STAGE);
          tc::bulk_load(smem + stg * STAGE + A_STAGE, src + size_t(c) * B_STAGE, B_STAGE,
                        &full_b[stg]);
        }
      }
      // copies still in flight complete before the CTA exits
      for (int s = 0; s < STAGES; ++s) {
        const uint32_t uses = (seq + STAGES - 1 - s) / STAGES;  // chunks n < seq with n % STAGES == s
        if (uses > 0) tc::mbar_wait(&full_b[s], (uses - 1) & 1, err, 18, true);
      }
    }
  }

  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == GATHER_WARPS) tc::tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------------------
// deterministic reduction of the (row tile, row quarter) partials into rho
// ---------------------------------------------------------------------------
__global__ void split_reduce(SplitArgs p, const int2* __restrict__ pairs, int npairs) {
  const int pi = blockIdx.x;
  if (pi >= npairs) return;
  const int2 pr = pairs ? pairs[pi] : make_int2(0, pi);  // (batch, 64-point tile)
  const SplitBatch& B = batch_of(p, pr.x);
  const int bg = pr.y;
  const int b = bg / p.gsub, gt = bg % p.gsub;
  const int nt = (B.counts[b] + TU - 1) / TU;
  if (nt == 0) return;  // fully masked block: rho untouched
  const int g0 = b * p.blk + gt * TG;
  const int gend = min(min((b + 1) * p.blk, B.ngrid), g0 + TG);
  for (int t = threadIdx.x; t < B.nset * TG; t += blockDim.x) {
    const int s = t / TG, j = t % TG;
    if (g0 + j >= gend) continue;
    double v = 0.0;
    for (int u = 0; u < nt; ++u) {
      const double* q = p.partial + (size_t(B.partial_off) +
                                     ((size_t(bg) * p.max_ut + u) * B.nset + s) * EPI_PARTS) * TG + j;
      for (int w = 0; w < EPI_PARTS; ++w) v += q[w * TG];
    }
    double* r = B.rhos + size_t(s) * B.stride_grid + g0 + j;
    *r = v + *r;
  }
}

template <int STAGES>
cudaError_t launch_main_t(int nsm, const SplitArgs& a, cudaStream_t stream, bool attrs_only) {
  constexpr size_t smem = size_t(STAGES) * STAGE + 1024 + 256;
  cudaError_t err = cudaFuncSetAttribute(split_main<STAGES>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (err != cudaSuccess || attrs_only) return err;
  split_main<STAGES><<<nsm, THREADS, smem, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_main(int stages, int nsm, const SplitArgs& a, cudaStream_t stream,
                        bool attrs_only) {
  static_assert(kMinStages == 3, "instantiated depths: 3, 4, 5");
  switch (stages < kMinStages ? kMinStages : stages) {
    case 3: return launch_main_t<3>(nsm, a, stream, attrs_only);
    case 5: return launch_main_t<5>(nsm, a, stream, attrs_only);
    default: return launch_main_t<4>(nsm, a, stream, attrs_only);
  }
}

int split_stages() {
  static const int v = [] {
    const char* e = std::getenv("CFGMM_SPLIT_STAGES");
    const int s = e ? std::atoi(e) : kDefaultStages;
    return (s >= kMinStages && s <= 5) ? s : kDefaultStages;
  }();
  return v;
}

size_t a256(size_t v) { return (v + 255) / 256 * 256; }

struct Layout {
  size_t lists, counts, cbase, items, total, dsl, tau, sigma, pmax, phisl, partial, bytes;
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
  L.pmax = L.sigma + a256(ngrid * sizeof(int));
  L.phisl = L.pmax + a256(ngrid * sizeof(unsigned long long));
  L.partial = L.phisl + a256(nbg * max_kc * B_STAGE);
  L.bytes = L.partial + nbg * max_ut * nset * EPI_PARTS * TG * sizeof(double);
  return L;
}

}  // namespace

// Which form a call runs: the row form of this file (one block tile, 128
// compacted rows per item) unless CFGMM_SPLIT_FORM=pair selects the pair form
// (two alike block tiles per item, aodmao2rho_split_pair.cu).  Read on every
// call; the workspace covers both.
bool split_pair_form(size_t nao, size_t points) {
  const char* e = std::getenv("CFGMM_SPLIT_FORM");
  if (e && e[0] == 'p') return true;
  if (e && e[0] == 'r') return false;
  // the pair form's pairing and tile building pay off on large problems
  return nao >= kPairMinAos && points >= kPairMinPoints;
}

size_t aodmao2rho_split_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk) {
  size_t w = layout(nao, ngrid, nset, blk).bytes;
  for (int nsl = 6; nsl <= 7; ++nsl) {
    const size_t wp = aodmao2rho_split_pair_workspace(nao, ngrid, nset, blk, nsl);
    w = wp > w ? wp : w;
  }
  return w;
}

cudaError_t aodmao2rho_split(double* rhos, const double* dms, const double* ao_lhs,
                             const double* ao_rhs, size_t stride_ao, size_t stride_grid, int nao,
                             int ngrid, int nset, const uint8_t* tab, size_t ldtab, int blk,
                             void* workspace, cudaStream_t stream) {
  if (nao <= 0 || ngrid <= 0 || nset <= 0) return cudaSuccess;
  if (split_pair_form(size_t(nao), size_t(ngrid)))
    return aodmao2rho_split_pair(rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, nao, ngrid,
                                 nset, tab, ldtab, blk, split_pair_digits(), workspace, stream);
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
  unsigned long long* pmax = reinterpret_cast<unsigned long long*>(ws + L.pmax);
  uint8_t* phisl = reinterpret_cast<uint8_t*>(ws + L.phisl);
  double* partial = reinterpret_cast<double*>(ws + L.partial);

  // The D chain (symmetry check, D slices) runs on a side stream beside the phi
  // chain (block lists, items, phi slices); the side stream joins back before
  // the main kernel.
  SideScope side(side_stream(), stream);
  cudaError_t err = side.fork();
  if (err != cudaSuccess) return err;
  const cudaStream_t sd = side.stream();
  // total[2]: asymmetry flag; the half contraction needs D = D^T and phi_lhs = phi_rhs
  int* asym = aodm_sym_enabled() && ao_lhs == ao_rhs ? total + 2 : nullptr;
  if (asym) {
    if ((err = cudaMemsetAsync(asym, 0, sizeof(int), sd)) != cudaSuccess) return err;
    if ((err = aodm_launch_sym_check(dms, stride_ao, nao, nset, asym, sd)) != cudaSuccess)
      return err;
  }
  if ((err = split_prepare_d(dms, stride_ao, nao, nset, dsl, tau, sd, asym)) != cudaSuccess)
    return err;
  if ((err = aodm_block_lists_launch(tab, ldtab, nao, nblk, lists, counts, stream)) != cudaSuccess)
    return err;
  split_build<<<1, 1024, 0, stream>>>(counts, nbg, gsub, nset, max_ut, cbase, items, total);
  if ((err = split_prepare_phi(ao_rhs, stride_grid, lists, counts, cbase, nao, ngrid, blk, pmax,
                               sigma, phisl, stream)) != cudaSuccess)
    return err;
  if ((err = side.join()) != cudaSuccess) return err;

  SplitArgs a{};
  a.dsl = dsl;
  a.tau = tau;
  a.phisl = phisl;
  a.batches = nullptr;
  a.one = SplitBatch{ao_lhs, rhos, lists, counts, cbase, sigma, stride_grid, ngrid, nset, 0};
  a.items = items;
  a.total = total;
  a.partial = partial;
  a.nao = nao;
  a.blk = blk;
  a.gsub = gsub;
  a.max_ut = max_ut;
  a.asym = asym;
  if ((err = split_launch_main(a, stream)) != cudaSuccess) return err;
  return split_launch_reduce(a, nullptr, nbg, stream);
}

cudaError_t split_prepare_d(const double* dms, size_t stride_ao, int nao, int nset, uint2* dsl,
                            int* tau, cudaStream_t stream, const int* asym) {
  split_d_slices<<<(nset * nao + 7) / 8, 256, 0, stream>>>(dms, stride_ao, stride_ao * stride_ao,
                                                           nao, nset * nao, dsl, tau, asym);
  return cudaGetLastError();
}

cudaError_t split_prepare_phi(const double* ao_rhs, size_t stride_grid, const int* lists,
                              const int* counts, const int* cbase, int nao, int ngrid, int blk,
                              unsigned long long* pmax, int* sigma, uint8_t* phisl,
                              cudaStream_t stream) {
  const int nbg = ((ngrid + blk - 1) / blk) * ((blk + TG - 1) / TG);
  const int gsub = (blk + TG - 1) / TG;
  cudaError_t err = cudaMemsetAsync(pmax, 0, size_t(ngrid) * sizeof(unsigned long long), stream);
  if (err != cudaSuccess) return err;
  split_phi_max<<<dim3(nbg, (nao + 63) / 64), 256, 0, stream>>>(ao_rhs, stride_grid, lists, counts,
                                                                nao, ngrid, blk, gsub, pmax);
  split_phi_digits<<<dim3(nbg, (nao + TK - 1) / TK), 256, 0, stream>>>(
      ao_rhs, stride_grid, lists, counts, cbase, pmax, nao, ngrid, blk, gsub, sigma, phisl);
  return cudaGetLastError();
}

cudaError_t split_launch_main(const SplitArgs& a, cudaStream_t stream, int stages,
                              bool attrs_only) {
  int dev = 0, nsm = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (err != cudaSuccess) return err;
  return launch_main(stages > 0 ? stages : split_stages(), nsm, a, stream, attrs_only);
}

cudaError_t split_launch_reduce(const SplitArgs& a, const int2* pairs, int npairs,
                                cudaStream_t stream) {
  if (npairs <= 0) return cudaSuccess;
  split_reduce<<<npairs, 128, 0, stream>>>(a, pairs, npairs);
  return cudaGetLastError();
}

int split_min_stages() { return kMinStages; }
int split_row_tile() { return TU; }
int split_point_tile() { return TG; }
int split_chunk() { return TK; }
size_t split_chunk_bytes() { return B_STAGE; }
int split_epi_parts() { return EPI_PARTS; }

cudaError_t aodmao2rho_split_reset_error(cudaStream_t stream) {
  static const int zero = 0;
  cudaError_t err = cudaMemcpyToSymbolAsync(g_split_error, &zero, sizeof(int), 0,
                                            cudaMemcpyHostToDevice, stream);
  return err != cudaSuccess ? err : aodmao2rho_split_pair_reset_error(stream);
}

// Either form's first timed-out wait (0: none).
cudaError_t aodmao2rho_split_read_error(int* code) {
  cudaError_t err = cudaMemcpyFromSymbol(code, g_split_error, sizeof(int));
  if (err != cudaSuccess || *code != 0) return err;
  return aodmao2rho_split_pair_read_error(code);
}

}  // namespace cfgmm
