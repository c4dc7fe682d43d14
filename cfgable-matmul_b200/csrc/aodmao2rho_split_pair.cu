// aodmao2rho_split_pair.cu -- the masked AO-DM-AO contraction in split
// precision with two grid block tiles per work item.
//
// Arithmetic: the slice form of the Ozaki scheme (Ozaki, Ogita, Oishi and Rump
// 2012), restated.  Every row u of D_s is scaled by 2^tau_u and every grid
// point g of phi by 2^sigma_g so that the scaled values are below 2^6; each is
// written as NSL signed base-256 digits x' = sum_{j<NSL} x_j 2^(-8j) read off
// the bytes of round(x' 2^(8(NSL-1))) (digits_of below).  The digit products
// whose levels add up to L = i + j <= NSL-1 are summed EXACTLY in one INT32
// TMEM accumulator per level (INT8 tcgen05.mma, NSL(NSL+1)/2 MMAs per chunk):
//   S_L[g][u] = sum_{i+j=L} sum_v phi_j(v,g) d_i(u,v),
// and X[u][g] = 2^-(tau_u + sigma_g) sum_L 2^(-8L) S_L[g][u] in FP64.  With
// NSL = 7 the dropped levels weigh about 2^-51 of sum_v |D_uv| |phi_vg|, with
// NSL = 6 about 2^-43.  |S_L| <= NSL 2^14 nao keeps the INT32 sums exact for
// nao <= 16384.
//
// Work items.  The contraction follows aodmao2rho_loop_parallel
// (src/impl_aodmao2rho.rs:171-244): per grid block b the active AO list I(b)
// (the reference's compaction, impl_matmul_non0tab.rs:118-129) and
// rho[s][g] += sum_{u,v in I(b)} phi[u][g] D_s[u][v] phi[v][g].  Here one item
// covers TWO 64-point block tiles whose active lists are alike (atom-centred
// grids put many blocks around one centre): the MMA's M = 128 rows are the
// points of both tiles, K runs over the union U of the two lists, N = TN rows
// of D (TN = 80 for NSL = 6, 64 for NSL = 7: NSL x TN <= 512 TMEM columns).
// Where an AO of U is inactive in a point's block the point's phi digits are
// zero there (in the tiles below) and the AO takes no part in the point's
// epilogue, so each point's sum runs over exactly its own block's list: the
// integer sums are unchanged by the zero digits.  Every D element gathered
// from L2 then serves 128 points instead of 64.  The pairing is a matching on
// the mask, on the device: tiles sorted by a min-hash signature of their
// lists, each tile scored against its kWin neighbours on either side by the
// MMA work that pairing saves (|I_a|^2 + |I_b|^2 - |I_a u I_b|^2), mutual best
// candidates paired; tiles without a profitable partner run alone (the other
// half of the lanes idle).
//
// Kernels (one call):
//   pair_sig      per block tile: bit set of I(b) and a 64-bit min-hash key
//   pair_sort     one CTA: tiles in key order (bitonic sort in shared memory)
//   pair_scores   per tile: the profitable neighbours, best first
//   pair_match    one CTA: mutual-best rounds -> pairs and singles
//   pair_union    per pair: the union list U and per-AO membership flags
//   pair_build    one CTA: chunk offsets and the work list (pair, row tile,
//                 DM), heaviest items first
//   pair_phi_max, pair_phi_tiles  point scales and the phi digit tiles of
//                 every (pair, chunk of 32 union AOs): NSL planes of 128 rows
//                 (points) x 32 bytes in the UMMA 32-byte-swizzled K-major
//                 layout, so one bulk copy moves a chunk
//   pair_d_digits D digits (8 bytes per element) and row scales
//   pair_main     persistent, 14 warps: 12 warps gather the D digits of TN
//                 rows x 32 union columns in three groups that take turns by
//                 chunk and run the epilogue; 1 warp issues the MMAs; 1 warp
//                 draws work items (dynamic, through a ring in shared memory)
//                 and bulk-loads the phi tiles.  A group copies the item's
//                 phi_lhs values to shared memory as the item starts, loads
//                 its first chunk of the next item before the accumulator
//                 wait and stores it right after reading TMEM, so the MMAs
//                 resume at once.  The epilogue reads each point's TMEM row
//                 (lane = point), rebuilds X in FP64, weights it with phi_lhs
//                 and sums over the row's AOs -- no cross-lane reduction; X
//                 never leaves the SM.
//   pair_reduce   adds the partial sums of each point (per row tile and
//                 gather group) in a fixed order (deterministic).
// Every mbarrier wait is bounded (tcgen05.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdlib>

#include "aodmao2rho_fp64.cuh"
#include "aodmao2rho_split.cuh"
#include "common.cuh"
#include "side_stream.cuh"
#include "tcgen05.cuh"

namespace cfgmm {
namespace {

constexpr int PT = 128;   // points per item: MMA M, TMEM lanes
constexpr int HT = 64;    // points per block tile (half an item)
constexpr int TK = 32;    // union AOs per chunk: one INT8 MMA K step
constexpr int NG = 3;     // gather groups of four warps
constexpr int GW = 4 * NG;
constexpr int THREADS = 32 * (GW + 2);
constexpr int kStages = 3;        // pipeline depth (at least NG: see the row form)
constexpr int kBadExp = INT_MAX;  // scale of a row / point holding Inf or NaN
constexpr int kWin = 32;          // pairing candidates on each side in key order
constexpr int kSortMax = 4096;    // tiles sorted in shared memory (more: caller's order)
constexpr int kRounds = 8;        // mutual-best matching rounds
constexpr int kMatchCandMax = 600;  // tiles whose candidate lists the matching stages in shared memory
constexpr int kRing = 4;          // work items in flight between the kernel's roles
constexpr int kAhead = 2;         // items drawn ahead of the one being loaded (< kRing)
static_assert(kStages >= NG, "a group's parity wait needs at least NG stages");

template <int NSL>
struct Cfg {
  static constexpr int TN = NSL == 6 ? 80 : 64;  // D rows per item (MMA N)
  static constexpr uint32_t A_SLICE = PT * TK;   // one phi digit plane: 4096 B
  static constexpr uint32_t B_SLICE = TN * TK;   // one D digit plane
  static constexpr uint32_t A_STAGE = NSL * A_SLICE;
  static constexpr uint32_t B_STAGE = NSL * B_SLICE;
  static constexpr uint32_t STAGE = A_STAGE + B_STAGE;
  static constexpr int WROWS = TN / 4;     // D rows per gather warp
  static constexpr int STEPS = WROWS / 4;  // four rows per step
  static constexpr int OCTETS = TN / 8;    // TMEM column octets of one level
  static constexpr int MAXQ = 2 * ((OCTETS + NG - 1) / NG);  // epilogue quartets per group
  // shared memory of a launch: stages, barriers, the item ring and the
  // epilogue's phi_lhs values ([warp][column][lane])
  template <int STAGES>
  static constexpr size_t smem_bytes() {
    return size_t(STAGES) * STAGE + 1024 + 256 + kRing * (16 + 4) +
           size_t(GW) * 4 * MAXQ * 32 * 8;
  }
  static_assert(NSL * TN <= 512, "level accumulators exceed the TMEM columns");
  static_assert(STAGE % 256 == 0 && A_STAGE % 256 == 0, "32-byte swizzle atoms");
  static_assert(WROWS % 4 == 0 && (OCTETS + NG - 1) / NG * 8 <= 32, "epilogue columns per group");
};

__device__ int g_pair_error;

__device__ __forceinline__ int exp_for(double amax) {  // 2^6 > amax * 2^exp
  if (!(amax <= 1.7976931348623157e308)) return kBadExp;
  if (amax == 0.0) return 0;
  int E;
  frexp(amax, &E);
  return 6 - E;
}

__device__ __forceinline__ double pow2(int k) {  // k in [-1022, 1023]
  return __longlong_as_double(static_cast<long long>(k + 1023) << 52);
}

// The NSL digits of x * 2^e (|x * 2^e| < 2^6), digit j (j = 0 leading) in
// byte j of the returned 8 bytes, the rest zero.  X = round(x 2^(e + 8(NSL-1)))
// plus the bias 128 * sum_{j < NSL-1} 256^j makes every low byte the unsigned
// form of a balanced digit in [-128, 127] (flipping bit 7 turns it into the
// signed byte), and leaves the leading digit, in [-64, 64], above them:
//   x 2^e = sum_j d_j 2^(-8j) + r 2^(-8(NSL-1)),  |r| <= 1/2.
// The scaling is done in two exact halves.
template <int NSL>
__device__ __forceinline__ uint2 digits_of(double x, int e) {
  static_assert(NSL == 6 || NSL == 7, "6 or 7 digits");
  constexpr int SH = 8 * (NSL - 1);
  constexpr long long BIAS = NSL == 7 ? 0x808080808080LL : 0x8080808080LL;
  const int k = e + SH;
  const int k1 = k / 2;
  const long long X = __double2ll_rn(x * pow2(k1) * pow2(k - k1));
  const unsigned long long Z = static_cast<unsigned long long>(X + BIAS) ^
                               static_cast<unsigned long long>(BIAS);
  const uint32_t lo = static_cast<uint32_t>(Z), hi = static_cast<uint32_t>(Z >> 32);
  if constexpr (NSL == 7) {
    // hi = d2 d1 d0 -, lo = d6 d5 d4 d3 (byte 0 first)
    return make_uint2(__byte_perm(hi, lo, 0x7012), __byte_perm(lo, 0u, 0x4012));
  } else {
    // hi = d1 d0 - -, lo = d5 d4 d3 d2
    return make_uint2(__byte_perm(hi, lo, 0x6701), __byte_perm(lo, 0u, 0x4401));
  }
}

// 4x4 byte transpose: out_i holds byte i of w0..w3 (w_t in byte t).
__device__ __forceinline__ void transpose4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3,
                                           uint32_t& o0, uint32_t& o1, uint32_t& o2,
                                           uint32_t& o3) {
  const uint32_t a = __byte_perm(w0, w1, 0x5140);
  const uint32_t b = __byte_perm(w0, w1, 0x7362);
  const uint32_t c = __byte_perm(w2, w3, 0x5140);
  const uint32_t d = __byte_perm(w2, w3, 0x7362);
  o0 = __byte_perm(a, c, 0x5410);
  o1 = __byte_perm(a, c, 0x7632);
  o2 = __byte_perm(b, d, 0x5410);
  o3 = __byte_perm(b, d, 0x7632);
}

// X' = sum_L 2^(-8L) S_L, combined exactly in 64-bit integers, then one FMA.
template <int NSL>
__device__ __forceinline__ double combine_levels(const uint32_t (&v)[NSL]) {
  const long long hi = (static_cast<long long>(int(v[0])) << 16) +
                       (static_cast<long long>(int(v[1])) << 8) + int(v[2]);
  if constexpr (NSL == 7) {
    const long long lo = (static_cast<long long>(int(v[3])) << 24) +
                         (static_cast<long long>(int(v[4])) << 16) +
                         (static_cast<long long>(int(v[5])) << 8) + int(v[6]);
    return fma(double(lo), 0x1p-48, double(hi) * 0x1p-16);
  } else {
    const long long lo = (static_cast<long long>(int(v[3])) << 16) +
                         (static_cast<long long>(int(v[4])) << 8) + int(v[5]);
    return fma(double(lo), 0x1p-40, double(hi) * 0x1p-16);
  }
}

// Point range of block tile bg (local to its batch): [*g0, *gend).
__device__ __forceinline__ void tile_points(int bg, int blk, int gsub, int ngrid, int* g0,
                                            int* gend) {
  const int b = bg / gsub, gt = bg % gsub;
  *g0 = b * blk + gt * HT;
  *gend = min(min((b + 1) * blk, ngrid), *g0 + HT);
}

__device__ __forceinline__ const PairBatch& batch_of(const PairArgs& p, int w) {
  return p.batches ? p.batches[w] : p.one;
}

// ---------------------------------------------------------------------------
// pairing
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mix32(uint32_t x, uint32_t seed) {
  x ^= seed;
  x *= 0x9E3779B1u;
  x ^= x >> 15;
  x *= 0x85EBCA77u;
  x ^= x >> 13;
  return x;
}

// Per block tile: bits[bg][w] (bit u%32 of word u/32: AO u active in the
// tile's block), count, and the min-hash key (two hashes; empty -> ~0).
__global__ void __launch_bounds__(256)
pair_sig(const uint8_t* __restrict__ tab, size_t ldtab, int nao, int nbg, int gsub, int nwords,
         uint32_t* __restrict__ bits, int* __restrict__ cnt, unsigned long long* __restrict__ key) {
  const int bg = blockIdx.x;
  if (bg >= nbg) return;
  const int b = bg / gsub;
  const int tid = threadIdx.x, lane = tid & 31;
  uint32_t h1 = 0xffffffffu, h2 = 0xffffffffu;
  int n = 0;
  for (int u0 = 0; u0 < nao; u0 += 256) {
    const int u = u0 + tid;
    const bool on = u < nao && tab[size_t(u) * ldtab + b] != 0;
    const uint32_t bal = __ballot_sync(0xffffffffu, on);
    const int wbase = u0 + (tid & ~31);
    if (lane == 0 && wbase < nao) bits[size_t(bg) * nwords + wbase / 32] = bal;
    n += on;
    if (on) {
      h1 = min(h1, mix32(uint32_t(u), 0x2545F491u));
      h2 = min(h2, mix32(uint32_t(u), 0x6C8E9CF5u));
    }
  }
  __shared__ uint32_t s1[8], s2[8];
  __shared__ int sn[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    h1 = min(h1, __shfl_xor_sync(0xffffffffu, h1, o));
    h2 = min(h2, __shfl_xor_sync(0xffffffffu, h2, o));
    n += __shfl_xor_sync(0xffffffffu, n, o);
  }
  if (lane == 0) {
    s1[tid >> 5] = h1;
    s2[tid >> 5] = h2;
    sn[tid >> 5] = n;
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t a = s1[0], c = s2[0];
    int t = sn[0];
    for (int w = 1; w < 8; ++w) {
      a = min(a, s1[w]);
      c = min(c, s2[w]);
      t += sn[w];
    }
    cnt[bg] = t;
    key[bg] = t == 0 ? ~0ull : (static_cast<unsigned long long>(a) << 32) | c;
  }
}

// The block lists (as aodm_block_lists: ascending active AOs of block b,
// counts[b]) and the signatures of the block's tiles (as pair_sig) from one
// read of the mask column; CTA per block.
__global__ void __launch_bounds__(256)
pair_lists_sig(const uint8_t* __restrict__ tab, size_t ldtab, int nao, int nblk, int gsub,
               int nwords, int* __restrict__ lists, int* __restrict__ counts,
               uint32_t* __restrict__ bits, int* __restrict__ cnt,
               unsigned long long* __restrict__ key) {
  const int b = blockIdx.x;
  if (b >= nblk) return;
  __shared__ int warp_tot[8];
  __shared__ int base_s;
  __shared__ uint32_t s1[8], s2[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) base_s = 0;
  __syncthreads();
  int* out = lists + size_t(b) * nao;
  uint32_t h1 = 0xffffffffu, h2 = 0xffffffffu;
  for (int u0 = 0; u0 < nao; u0 += 256) {
    const int u = u0 + tid;
    const bool on = u < nao && tab[size_t(u) * ldtab + b] != 0;
    const uint32_t bal = __ballot_sync(0xffffffffu, on);
    const int wbase = u0 + (tid & ~31);
    if (lane == 0 && wbase < nao)
      for (int t = 0; t < gsub; ++t) bits[size_t(b * gsub + t) * nwords + wbase / 32] = bal;
    if (on) {
      h1 = min(h1, mix32(uint32_t(u), 0x2545F491u));
      h2 = min(h2, mix32(uint32_t(u), 0x6C8E9CF5u));
    }
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    int before = base_s;
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    if (on) out[before + __popc(bal & ((1u << lane) - 1u))] = u;
    __syncthreads();
    if (tid == 0) {
      int t = 0;
      for (int w = 0; w < 8; ++w) t += warp_tot[w];
      base_s += t;
    }
    __syncthreads();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    h1 = min(h1, __shfl_xor_sync(0xffffffffu, h1, o));
    h2 = min(h2, __shfl_xor_sync(0xffffffffu, h2, o));
  }
  if (lane == 0) {
    s1[warp] = h1;
    s2[warp] = h2;
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t a = s1[0], c = s2[0];
    for (int w = 1; w < 8; ++w) {
      a = min(a, s1[w]);
      c = min(c, s2[w]);
    }
    const int n = base_s;
    counts[b] = n;
    for (int t = 0; t < gsub; ++t) {
      cnt[b * gsub + t] = n;
      key[b * gsub + t] = n == 0 ? ~0ull : (static_cast<unsigned long long>(a) << 32) | c;
    }
  }
}

// order[q] = tile at sorted position q (keys ascending, ties by index); above
// kSortMax tiles the caller's order.
__global__ void __launch_bounds__(1024)
pair_sort(const unsigned long long* __restrict__ key, int nbg, int* __restrict__ order) {
  extern __shared__ unsigned long long sk[];  // kSortMax keys, then kSortMax indices
  int* id = reinterpret_cast<int*>(sk + kSortMax);
  const int tid = threadIdx.x;
  if (nbg > kSortMax) {
    for (int i = tid; i < nbg; i += 1024) order[i] = i;
    return;
  }
  int n2 = 1;
  while (n2 < nbg) n2 <<= 1;
  for (int i = tid; i < n2; i += 1024) {
    sk[i] = i < nbg ? key[i] : ~0ull;
    id[i] = i < nbg ? i : INT_MAX;
  }
  __syncthreads();
  for (int size = 2; size <= n2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < n2; i += 1024) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const bool gt = sk[i] > sk[j] || (sk[i] == sk[j] && id[i] > id[j]);
          if (gt == up) {
            const unsigned long long tk = sk[i];
            sk[i] = sk[j];
            sk[j] = tk;
            const int ti = id[i];
            id[i] = id[j];
            id[j] = ti;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < nbg; i += 1024) order[i] = id[i];
}

// Per sorted position q: the neighbours within kWin positions whose pairing
// with tile order[q] saves MMA work (|I_a|^2 + |I_b|^2 > |I_a u I_b|^2), best
// first: cand[q][0 .. ncand[q]).  CTA per position, thread per candidate.
__global__ void __launch_bounds__(2 * kWin)
pair_scores(const uint32_t* __restrict__ bits, const int* __restrict__ cnt,
            const int* __restrict__ order, int nbg, int nwords, int* __restrict__ cand,
            int* __restrict__ ncand) {
  const int q = blockIdx.x;
  if (q >= nbg) return;
  const int tid = threadIdx.x;
  __shared__ long long sc[2 * kWin];
  __shared__ int who[2 * kWin];
  const int a = order[q];
  const int na = cnt[a];
  const int off = tid < kWin ? tid - kWin : tid - kWin + 1;  // -kWin..-1, 1..kWin
  const int qb = q + off;
  long long score = LLONG_MIN;
  int b = -1;
  if (na > 0 && qb >= 0 && qb < nbg) {
    b = order[qb];
    const int nb = cnt[b];
    if (nb > 0) {
      int inter = 0;
      const uint32_t* x = bits + size_t(a) * nwords;
      const uint32_t* y = bits + size_t(b) * nwords;
      for (int w = 0; w < nwords; ++w) inter += __popc(x[w] & y[w]);
      const long long un = na + nb - inter;
      score = static_cast<long long>(na) * na + static_cast<long long>(nb) * nb - un * un;
    }
  }
  sc[tid] = score;
  who[tid] = b;
  __syncthreads();
  // the profitable candidates (score > 0), best first, ties by tile index: each
  // thread's rank is the number of candidates ordered before its own
  if (score > 0) {
    int rank = 0;
    for (int i = 0; i < 2 * kWin; ++i)
      rank += sc[i] > score || (sc[i] == score && who[i] < b);
    cand[size_t(q) * 2 * kWin + rank] = b;
  }
  const unsigned pos_w = __ballot_sync(0xffffffffu, score > 0);
  __shared__ int npos[2];
  if ((tid & 31) == 0) npos[tid >> 5] = __popc(pos_w);
  __syncthreads();
  if (tid == 0) ncand[q] = npos[0] + npos[1];
}

// Mutual-best matching over the candidate lists (kRounds rounds), then the
// pair list in key order: pairs[i] = (lo tile, hi tile or -1, batch, 0) for
// every non-empty tile in exactly one entry; npairs[0] = their number.
// The per-tile state lives in shared memory when it fits (kSortMax tiles),
// else in the global scratch arrays.
__global__ void __launch_bounds__(1024)
pair_match(const int* __restrict__ order, const int* __restrict__ cand,
           const int* __restrict__ ncand, const int* __restrict__ cnt, int nbg, int batch,
           int* __restrict__ partner_g, int* __restrict__ pos_g, int* __restrict__ choice_g,
           int4* __restrict__ pairs, int* __restrict__ npairs) {
  // 3 * kSortMax ints when nbg <= kSortMax, then the candidate lists when
  // nbg <= kMatchCandMax
  extern __shared__ int match_s[];
  const bool in_smem = nbg <= kSortMax;
  int* partner = in_smem ? match_s : partner_g;
  int* pos = in_smem ? match_s + kSortMax : pos_g;
  int* choice = in_smem ? match_s + 2 * kSortMax : choice_g;
  const int tid = threadIdx.x;
  const int* cl = cand;  // candidate lists, staged in shared memory when they fit
  if (nbg <= kMatchCandMax) {
    int* cs = match_s + 3 * kSortMax;
    for (int i = tid; i < nbg * 2 * kWin; i += 1024) cs[i] = cand[i];
    cl = cs;
  }
  __shared__ int changed;
  __shared__ int warp_tot[32];
  __shared__ int base_s;
  // partner[t]: -2 free, -1 single, -3 empty (never emitted), >= 0 paired
  for (int q = tid; q < nbg; q += 1024) {
    const int t = order[q];
    pos[t] = q;
    partner[t] = cnt[t] > 0 ? -2 : -3;
  }
  __syncthreads();
  for (int r = 0; r < kRounds; ++r) {
    if (tid == 0) changed = 0;
    // every free tile picks its best free candidate
    for (int q = tid; q < nbg; q += 1024) {
      const int t = order[q];
      int pick = -1;
      if (partner[t] == -2) {
        const int n = ncand[q];
        for (int i = 0; i < n; ++i) {
          const int c = cl[size_t(q) * 2 * kWin + i];
          if (partner[c] == -2) {
            pick = c;
            break;
          }
        }
      }
      choice[t] = pick;
    }
    __syncthreads();
    // mutual choices become pairs (written by the member with the lower index)
    for (int q = tid; q < nbg; q += 1024) {
      const int t = order[q];
      const int c = choice[t];
      if (c >= 0 && t < c && choice[c] == t) {
        partner[t] = c;
        partner[c] = t;
        changed = 1;
      }
    }
    __syncthreads();
    const int ch = changed;
    __syncthreads();
    if (!ch) break;
  }
  for (int q = tid; q < nbg; q += 1024) {
    const int t = order[q];
    if (partner[t] == -2) partner[t] = -1;
  }
  if (tid == 0) base_s = 0;
  __syncthreads();
  // one entry per leader (a single, or the member at the lower position)
  const int lane = tid & 31, warp = tid >> 5;
  for (int q0 = 0; q0 < nbg; q0 += 1024) {
    const int q = q0 + tid;
    int t = -1, c = -3;
    bool lead = false;
    if (q < nbg) {
      t = order[q];
      c = partner[t];
      lead = c == -1 || (c >= 0 && pos[c] > q);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, lead);
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    int before = base_s;
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    if (lead)
      pairs[before + __popc(bal & ((1u << lane) - 1u))] = make_int4(t, c >= 0 ? c : -1, batch, 0);
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < 32; ++w) base_s += warp_tot[w];
    __syncthreads();
  }
  if (tid == 0) npairs[0] = base_s;
}

// Per pair: U = ascending union of the two tiles' active lists, flags bit 0 /
// bit 1 = active in the lo / hi tile's block; ucount.
__global__ void __launch_bounds__(256)
pair_union(const uint8_t* __restrict__ tab, size_t ldtab, int nao, int gsub,
           const int4* __restrict__ pairs, const int* __restrict__ npairs, int pair0,
           int* __restrict__ ulist, uint8_t* __restrict__ uflag, int* __restrict__ ucount) {
  const int pl = blockIdx.x;
  if (pl >= npairs[0]) return;
  const int pi = pair0 + pl;
  const int4 pr = pairs[pi];
  const int b0 = pr.x / gsub, b1 = pr.y >= 0 ? pr.y / gsub : -1;
  __shared__ int warp_tot[8];
  __shared__ int base_s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) base_s = 0;
  __syncthreads();
  int* U = ulist + size_t(pi) * nao;
  uint8_t* F = uflag + size_t(pi) * nao;
  for (int u0 = 0; u0 < nao; u0 += 256) {
    const int u = u0 + tid;
    uint32_t f = 0;
    if (u < nao) {
      f = tab[size_t(u) * ldtab + b0] != 0 ? 1u : 0u;
      if (b1 >= 0 && tab[size_t(u) * ldtab + b1] != 0) f |= 2u;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, f != 0);
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    int before = base_s;
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    if (f) {
      const int at = before + __popc(bal & ((1u << lane) - 1u));
      U[at] = u;
      F[at] = uint8_t(f);
    }
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < 8; ++w) base_s += warp_tot[w];
    __syncthreads();
  }
  if (tid == 0) ucount[pi] = base_s;
}

// cbase[pi] (first phi chunk of each pair, from chunk0), and the items
// (pair, row tile, DM, batch) of pairs pair0 .. pair0+npairs-1 appended at
// items + *total: pair-major (all of a pair's items together, so that the
// CTAs running at one time share a few pairs' phi tiles and D rows in L2),
// heaviest pairs first (a counting sort on the pair's chunk count);
// *total grows by their number, *chunks_end is the chunk after the batch's last.
__global__ void __launch_bounds__(1024)
pair_build(const int* __restrict__ ucount, const int* __restrict__ npairs_d, int pair0, int nset,
           int batch, int tn, int max_kc, int chunk0, int* __restrict__ cbase,
           int* __restrict__ cpair, int4* __restrict__ items, int* __restrict__ total,
           int* __restrict__ chunks_end) {
  extern __shared__ int hist[];  // max_kc + 2 counters
  __shared__ int warp_c[32];
  __shared__ int base_c;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int np = npairs_d[0];
  for (int i = tid; i <= max_kc + 1; i += 1024) hist[i] = 0;
  if (tid == 0) base_c = chunk0;
  __syncthreads();
  // chunk offsets
  for (int p0 = 0; p0 < np; p0 += 1024) {
    const int pl = p0 + tid;
    const int kc = pl < np ? (ucount[pair0 + pl] + TK - 1) / TK : 0;
    int ic = kc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, ic, o);
      if (lane >= o) ic += t;
    }
    if (lane == 31) warp_c[warp] = ic;
    __syncthreads();
    int bc = base_c;
    for (int w = 0; w < warp; ++w) bc += warp_c[w];
    if (pl < np) {
      cbase[pair0 + pl] = bc + ic - kc;
      for (int c = 0; c < kc; ++c) cpair[bc + ic - kc - chunk0 + c] = pair0 + pl;
    }
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < 32; ++w) base_c += warp_c[w];
    __syncthreads();
  }
  // items per chunk-count class of the pairs
  for (int pl = tid; pl < np; pl += 1024) {
    const int nu = ucount[pair0 + pl];
    const int kc = (nu + TK - 1) / TK, nt = (nu + tn - 1) / tn;
    atomicAdd(&hist[kc], nt * nset);
  }
  __syncthreads();
  if (tid == 0) {  // heaviest first: cursor[w] = items of pairs with more chunks than w
    int run = 0;
    for (int w = max_kc; w >= 0; --w) {
      const int c = hist[w];
      hist[w] = run;
      run += c;
    }
    hist[max_kc + 1] = run;
  }
  __syncthreads();
  const int start = total[0];
  for (int pl = tid; pl < np; pl += 1024) {
    const int nu = ucount[pair0 + pl];
    const int kc = (nu + TK - 1) / TK, nt = (nu + tn - 1) / tn;
    int at = start + atomicAdd(&hist[kc], nt * nset);
    for (int t = 0; t < nt; ++t)
      for (int s = 0; s < nset; ++s) items[at++] = make_int4(pair0 + pl, t, s, batch);
  }
  __syncthreads();
  if (tid == 0) {
    total[0] = start + hist[max_kc + 1];
    chunks_end[0] = base_c;
  }
}

// pmax[g] = max |phi[u][g]| over the active AOs of g's block (+Inf for Inf or
// NaN); CTA (block tile, slab of 64 active AOs); pmax starts at 0.
__global__ void __launch_bounds__(256)
pair_phi_max(const double* __restrict__ ao, size_t stride_grid, const int* __restrict__ lists,
             const int* __restrict__ counts, int nao, int ngrid, int blk, int gsub,
             unsigned long long* __restrict__ pmax) {
  const int bg = blockIdx.x, slab = blockIdx.y;
  const int b = bg / gsub;
  const int nb = counts[b];
  const int i0 = slab * 64;
  if (i0 >= nb) return;
  int g0, gend;
  tile_points(bg, blk, gsub, ngrid, &g0, &gend);
  const int* I = lists + size_t(b) * nao;
  const int gr = threadIdx.x & (HT - 1), rg = threadIdx.x >> 6;
  const int g = g0 + gr;
  __shared__ double red[4][HT];
  double mx = 0.0;
  if (g < gend) {
    bool bad = false;
    const int iend = min(nb, i0 + 64);
    for (int i = i0 + rg; i < iend; i += 4) {
      const double a = fabs(ao[size_t(__ldg(I + i)) * stride_grid + g]);
      bad |= !(a <= 1.7976931348623157e308);
      mx = fmax(mx, a);
    }
    if (bad) mx = __longlong_as_double(0x7ff0000000000000LL);
  }
  red[rg][gr] = mx;
  __syncthreads();
  if (threadIdx.x < HT && g < gend) {
    const double m = fmax(fmax(red[0][gr], red[1][gr]), fmax(red[2][gr], red[3][gr]));
    atomicMax(pmax + g, static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

// The phi digit tiles of every chunk of the batch (pair pi, chunk c): NSL
// planes of 128 rows (points: rows 0-63 the lo tile, 64-127 the hi tile) x
// 32 bytes (union AOs 32c .. 32c+31), 32-byte swizzled, at phisl + (cbase[pi]
// + c) * A_STAGE; sigma[g] from pmax.  Persistent CTAs take contiguous runs
// of the batch's chunks [chunk0, chunks_end) through the chunk -> pair map.
template <int NSL>
__global__ void __launch_bounds__(256)
pair_phi_tiles(const double* __restrict__ ao, size_t stride_grid,
               const unsigned long long* __restrict__ pmax, const int4* __restrict__ pairs,
               const int* __restrict__ cpair, int chunk0, const int* __restrict__ chunks_end,
               const int* __restrict__ ulist, const uint8_t* __restrict__ uflag,
               const int* __restrict__ ucount, const int* __restrict__ cbase, int nao, int ngrid,
               int blk, int gsub, int* __restrict__ sigma, uint8_t* __restrict__ phisl) {
  using C = Cfg<NSL>;
  // staged digit words [plane][quad of 4 AOs][point], rows padded to 132 words
  __shared__ uint32_t stage[NSL][8][PT + 4];
  const int nch = chunks_end[0] - chunk0;
  // a contiguous run of chunks per CTA: mostly one pair's, whose union list,
  // flags and offsets stay in L1 from one chunk to the next
  const int per = (nch + int(gridDim.x) - 1) / int(gridDim.x);
  const int ci0 = int(blockIdx.x) * per, ci1 = min(nch, ci0 + per);
  for (int ci = ci0; ci < ci1; ++ci) {
    const int pi = cpair[ci];
    const int c = chunk0 + ci - cbase[pi];
    const int nu = ucount[pi];
    const int4 pr = pairs[pi];
    const int* U = ulist + size_t(pi) * nao;
    const uint8_t* F = uflag + size_t(pi) * nao;
    {
      const int r = threadIdx.x & (PT - 1), hq = threadIdx.x >> 7;  // point row, half of the quads
      const int h = r >> 6;
      const int tile = h ? pr.y : pr.x;
      int g = -1;
      if (tile >= 0) {
        int g0, gend;
        tile_points(tile, blk, gsub, ngrid, &g0, &gend);
        if (g0 + (r & (HT - 1)) < gend) g = g0 + (r & (HT - 1));
      }
      const int e = g >= 0 ? exp_for(__longlong_as_double(static_cast<long long>(pmax[g]))) : 0;
      if (c == 0 && hq == 0 && g >= 0) sigma[g] = e;
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        const int q = hq * 4 + qq;
        uint2 w[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int k = c * TK + q * 4 + t;
          const bool on = g >= 0 && k < nu && e != kBadExp && ((__ldg(F + k) >> h) & 1u);
          w[t] = on ? digits_of<NSL>(ao[size_t(__ldg(U + k)) * stride_grid + g], e)
                    : make_uint2(0u, 0u);
        }
        uint32_t o[8];
        transpose4(w[0].x, w[1].x, w[2].x, w[3].x, o[0], o[1], o[2], o[3]);
        transpose4(w[0].y, w[1].y, w[2].y, w[3].y, o[4], o[5], o[6], o[7]);
#pragma unroll
        for (int pl2 = 0; pl2 < NSL; ++pl2) stage[pl2][q][r] = o[pl2];
      }
    }
    __syncthreads();
    uint8_t* tile0 = phisl + (size_t(cbase[pi]) + c) * C::A_STAGE;
    for (int v = threadIdx.x; v < NSL * PT * 2; v += 256) {
      const int hh = v & 1, r = (v >> 1) & (PT - 1), j = v >> 8;
      const uint4 wv = make_uint4(stage[j][4 * hh][r], stage[j][4 * hh + 1][r],
                                  stage[j][4 * hh + 2][r], stage[j][4 * hh + 3][r]);
      *reinterpret_cast<uint4*>(tile0 + j * C::A_SLICE +
                                tc::sw32_offset(uint32_t(r), uint32_t(hh))) = wv;
    }
    __syncthreads();
  }
}

// D digits and the symmetry check in one launch.  CTAs 0 .. nset*nao-1: row
// (s, u) -- tau[s][u], the digits dsl[s][u][v] of the whole row (its max
// first, then the digits, the second read from L1) and dhalf[s][u], the
// digits of D_uu / 2 that the symmetric mode uses for the diagonal.  The
// CTAs after them (when asym is non-null): one 32 x 32 tile pair (i, j),
// j <= i, of a D each, compared with its transpose bitwise; a difference sets
// *asym (zeroed by the caller).
template <int NSL>
__global__ void __launch_bounds__(256)
pair_d_prep(const double* __restrict__ dms, size_t stride_ao, size_t dm_stride, int nao,
            int nset, uint2* __restrict__ dsl, int* __restrict__ tau,
            uint2* __restrict__ dhalf, int* __restrict__ asym) {
  const int nrows = nset * nao;
  if (int(blockIdx.x) >= nrows) {
    // ---- symmetry check: tile pair k of D s (triangular index) ----
    const int nt = (nao + 31) / 32;
    const int ntri = nt * (nt + 1) / 2;
    const int t = int(blockIdx.x) - nrows;
    const int s = t / ntri, k = t % ntri;
    int bx = int((sqrtf(8.f * float(k) + 1.f) - 1.f) * 0.5f);
    while (bx * (bx + 1) / 2 > k) --bx;
    while ((bx + 1) * (bx + 2) / 2 <= k) ++bx;
    const int by = k - bx * (bx + 1) / 2;  // by <= bx
    __shared__ double tile[32][33];
    const double* d = dms + size_t(s) * dm_stride;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double mine[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = ty + 8 * q;
      const int r = by * 32 + i, c = bx * 32 + tx;
      tile[i][tx] = (r < nao && c < nao) ? d[size_t(r) * stride_ao + c] : 0.0;
      const int r2 = bx * 32 + i, c2 = by * 32 + tx;
      mine[q] = (r2 < nao && c2 < nao) ? d[size_t(r2) * stride_ao + c2] : 0.0;
    }
    __syncthreads();
    bool bad = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = ty + 8 * q;
      const int r2 = bx * 32 + i, c2 = by * 32 + tx;
      if (r2 < nao && c2 < nao) bad |= !(mine[q] == tile[tx][i]);
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(asym, 1);
    return;
  }
  // ---- digits of row (s, u) ----
  const int row = blockIdx.x;
  const int s = row / nao, u = row % nao;
  const double* d = dms + size_t(s) * dm_stride + size_t(u) * stride_ao;
  __shared__ double wmax[8];
  __shared__ int wbad[8];
  double mx = 0.0;
  bool bad = false;
#pragma unroll 4
  for (int v = threadIdx.x; v < nao; v += 256) {
    const double a = fabs(d[v]);
    bad |= !(a <= 1.7976931348623157e308);
    mx = fmax(mx, a);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    bad |= __shfl_xor_sync(0xffffffffu, int(bad), o) != 0;
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    wmax[w] = mx;
    wbad[w] = bad;
  }
  __syncthreads();
  mx = wmax[0];
  bad = wbad[0] != 0;
#pragma unroll
  for (int i = 1; i < 8; ++i) {
    mx = fmax(mx, wmax[i]);
    bad |= wbad[i] != 0;
  }
  const int e = bad ? kBadExp : exp_for(mx);
  if (threadIdx.x == 0) {
    tau[row] = e;
    dhalf[row] = e != kBadExp ? digits_of<NSL>(0.5 * d[u], e) : make_uint2(0u, 0u);
  }
  uint2* out = dsl + size_t(row) * nao;
#pragma unroll 4
  for (int v = threadIdx.x; v < nao; v += 256)
    out[v] = e != kBadExp ? digits_of<NSL>(d[v], e) : make_uint2(0u, 0u);
}

// Byte selector assembling, from `keep` (bytes 0..3) and `recv` (4..7) of the
// gather's second shuffle round, the digit word of 4 consecutive columns:
// column qd from keep.b0, qd^2 from keep.b2, qd^1 from recv.b0, qd^3 from
// recv.b2 (the lane's second digit plane: +1 on every nibble).
__device__ __forceinline__ uint32_t gather_selector(int qd) {
  uint32_t sel = 0;
#pragma unroll
  for (int col = 0; col < 4; ++col) {
    const uint32_t src = col == qd ? 0u : col == (qd ^ 2) ? 2u : col == (qd ^ 1) ? 4u : 6u;
    sel |= src << (4 * col);
  }
  return sel;
}

// ---------------------------------------------------------------------------
// main kernel
// ---------------------------------------------------------------------------
template <int NSL, int STAGES>
__global__ void __launch_bounds__(THREADS, 1) pair_main(PairArgs p) {
  using C = Cfg<NSL>;
  constexpr int TN = C::TN;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * C::STAGE);
  uint64_t* full_phi = bars;            // phi tile landed (bulk copy)
  uint64_t* full_d = bars + STAGES;     // D digits stored (4 gather warps)
  uint64_t* empty = bars + 2 * STAGES;  // the stage's MMAs completed
  uint64_t* acc_full = bars + 3 * STAGES;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 5);
  // the work-item ring: the loader thread draws items from the global counter
  // (dynamic scheduling: the list is pair-major, heaviest pairs first) and
  // every role reads them from here in the same order
  uint64_t* ifull = reinterpret_cast<uint64_t*>(smem + STAGES * C::STAGE + 256);  // [kRing]
  uint64_t* iempty = ifull + kRing;                                   // [kRing]
  int* ring = reinterpret_cast<int*>(iempty + kRing);                 // [kRing]
  double* phl_all = reinterpret_cast<double*>(ring + kRing);          // [GW][4 MAXQ][32]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* err = &g_pair_error;
  const uint64_t lim = p.wait_ns ? p.wait_ns : tc::kWaitLimitNs;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full_phi[s], 1);
      tc::mbar_init(&full_d[s], 4);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(acc_full, 1);
    tc::mbar_init(acc_empty, GW);
    tc::mbar_init(drain, 1);
    for (int r = 0; r < kRing; ++r) {
      tc::mbar_init(&ifull[r], 1);
      tc::mbar_init(&iempty[r], GW + 2);  // every warp reads every item
    }
    tc::mbar_fence_init();
  }
  if (warp == GW) {
    tc::tmem_alloc(tmem_slot, 512);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const int total = p.total[0];
  const bool sym = p.asym != nullptr && *p.asym == 0;
  // item n of this CTA (total when there are no more), read from the ring by
  // lane 0 of the calling warp and broadcast; every warp calls it for n = 0, 1, ...
  auto item_of = [&](uint32_t n, bool whole_warp) -> int {
    int t = total;
    if (!whole_warp || lane == 0) {
      if (tc::mbar_wait(&ifull[n % kRing], (n / kRing) & 1, err, 40, false, lim))
        t = *reinterpret_cast<volatile int*>(&ring[n % kRing]);
      tc::mbar_arrive(&iempty[n % kRing]);
    }
    if (whole_warp) t = __shfl_sync(0xffffffffu, t, 0);
    return t;
  };

  if (warp < GW) {
    // ---------------- gather D digits, then the epilogue ----------------
    // Group grp takes the chunks c = kc0 + grp, + NG, ... of every item; warp
    // wq of the group fills D rows WROWS*wq .. of the tile, four rows per step.
    // Lane (qd, ri, hh) = lane bits (4:3, 2:1, 0) loads, for row 4*step+ri,
    // the union columns 16hh + 4k + qd (k = 0..3) and ends up holding digit
    // planes 2qd and 2qd+1 of the 16-byte half hh of that row.
    const int grp = warp >> 2, wq = warp & 3;
    const int qd = lane >> 3, ri = (lane >> 1) & 3, hh = lane & 1;
    const bool b1 = (qd & 2) != 0, b0 = (qd & 1) != 0;
    const uint32_t sel_a = gather_selector(qd), sel_b = sel_a + 0x1111u;
    // this warp's phi_lhs values for the epilogue: [group column][lane]
    double* phl = phl_all + size_t(warp) * (4 * C::MAXQ * 32);
    struct Item {
      int t, pi, ut, s, w, nu, kc, kc0;
      int iu[C::STEPS];  // AO of the D row this lane loads at each step (-1: none)
    };
    auto setup = [&](int t, Item& g) {
      g.t = t;
      if (t >= total) return;
      const int4 it = p.items[t];
      g.pi = it.x;
      g.ut = it.y;
      g.s = it.z;
      g.w = it.w;
      g.nu = p.ucount[g.pi];
      g.kc = (g.nu + TK - 1) / TK;
      g.kc0 = sym ? (g.ut * TN) / TK : 0;
      const int* U = p.ulist + size_t(g.pi) * p.nao;
#pragma unroll
      for (int st = 0; st < C::STEPS; ++st) {
        const int prow = g.ut * TN + C::WROWS * wq + 4 * st + ri;
        g.iu[st] = prow < g.nu ? __ldg(U + prow) : -1;
      }
    };
    // the union columns this lane loads in chunk c (-1: past the list)
    auto columns = [&](const Item& g, int c, int (&iv)[4]) {
      const int* U = p.ulist + size_t(g.pi) * p.nao;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int pc = c * TK + 16 * hh + 4 * k + qd;
        iv[k] = pc < g.nu ? __ldg(U + pc) : -1;
      }
    };
    // The MMAs of every chunk up to `done` (stage sequence number) are known
    // to have completed.  A parity wait names a phase only while the phase
    // before it has completed, so stage_free steps through the completions
    // in order: waiting for chunk y is safe once chunk y - STAGES is done.
    long long done = -1;
    auto stage_free = [&](uint32_t seq) -> bool {
      const long long need = static_cast<long long>(seq) - STAGES;
      while (done < need) {
        const long long y = done + STAGES < need ? done + STAGES : need;
        if (!tc::mbar_wait(&empty[y % STAGES], uint32_t((y / STAGES) & 1), err, 31, false, lim))
          return false;
        done = y;
      }
      return true;
    };
    // D digits of chunk c of item g at this lane's positions (no waits)
    auto load_chunk = [&](const Item& g, int c, const int (&iv)[4], uint2 (&w)[C::STEPS][4]) {
      const uint2* dset = p.dsl + size_t(g.s) * p.nao * p.nao;
      const uint2* dh = p.dhalf + size_t(g.s) * p.nao;
      // symmetric D: only columns from the row's own position on, the
      // diagonal with the digits of D_uu / 2
#pragma unroll
      for (int st = 0; st < C::STEPS; ++st) {
        const int prow = g.ut * TN + C::WROWS * wq + 4 * st + ri;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int pc = c * TK + 16 * hh + 4 * k + qd;
          w[st][k] = (g.iu[st] >= 0 && iv[k] >= 0 && (!sym || pc >= prow))
                         ? __ldg(sym && pc == prow ? dh + g.iu[st]
                                                   : dset + size_t(g.iu[st]) * p.nao + iv[k])
                         : make_uint2(0u, 0u);
        }
      }
    };
    // the loaded digits into stage seq % STAGES as digit planes (false: a wait ran out)
    auto store_chunk = [&](uint32_t seq, const uint2 (&w)[C::STEPS][4]) -> bool {
      if (!stage_free(seq)) return false;
      const int stg = int(seq % STAGES);
      uint8_t* Bs = smem + stg * C::STAGE + C::A_STAGE;
#pragma unroll
      for (int st = 0; st < C::STEPS; ++st) {
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
        const uint32_t off =
            tc::sw32_offset(uint32_t(C::WROWS * wq + 4 * st + ri), uint32_t(hh));
        if (2 * qd < NSL)
          *reinterpret_cast<uint4*>(Bs + (2 * qd) * C::B_SLICE + off) =
              make_uint4(wa[0], wa[1], wa[2], wa[3]);
        if (2 * qd + 1 < NSL)
          *reinterpret_cast<uint4*>(Bs + (2 * qd + 1) * C::B_SLICE + off) =
              make_uint4(wb[0], wb[1], wb[2], wb[3]);
      }
      tc::fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&full_d[stg]);
      return true;
    };

    const int h = wq >> 1;           // the warp's block tile: lo (0) or hi (1)
    const int r = 32 * wq + lane;    // TMEM lane = point row
    const uint32_t trow = tmem + (uint32_t(32 * wq) << 16);
    uint32_t seq0 = 0;  // stage sequence number of the current item's first chunk
    bool ok = true, ahead = false;
    Item cur, nxt;
    setup(item_of(0, true), cur);
    for (uint32_t nitem = 0; ok && cur.t < total; ++nitem) {
      // ---- what the epilogue needs, requested first: lane l holds column l
      // of the group's columns (octets grp, grp+NG, ...): its AO, membership
      // flags and row scale; phi_lhs of every group column at this lane's
      // point, for AOs active in its block (zero-filled elsewhere), is copied
      // to shared memory while the item's chunks run; bit 4qi+j of `on`
      // marks column j of quartet qi ----
      const PairBatch& B = batch_of(p, cur.w);
      int gpt, sg, nq, eg;
      // 2^(-tau - eg) of this lane's column, eg the largest -tau of the
      // group's columns (so every factor is at most 1 and the group's sum
      // is scaled by 2^eg once); 0 for a row holding Inf or NaN
      double s_l;
      uint32_t badbits;  // lanes whose column's D row holds Inf or NaN
      bool gval;
      uint32_t on = 0;
      {
        const int4 pr = p.pairs[cur.pi];
        const int tile = h ? pr.y : pr.x;
        int g0 = 0, gend = 0;
        if (tile >= 0) tile_points(tile, p.blk, p.gsub, B.ngrid, &g0, &gend);
        gpt = g0 + (r & (HT - 1));
        gval = tile >= 0 && gpt < gend;
        // the group's columns of this tile, in quartets (warp-uniform):
        // octets grp, grp+NG, ... below OCTETS whose first column lies inside U
        int nocts = 0;
        while (grp + NG * nocts < C::OCTETS && cur.ut * TN + (grp + NG * nocts) * 8 < cur.nu)
          ++nocts;
        nq = 2 * nocts;
        const int col_l = (grp + NG * (lane >> 3)) * 8 + (lane & 7);
        const int kpos_l = cur.ut * TN + col_l;
        const bool cval_l = col_l < TN && kpos_l < cur.nu;
        const int u_l = cval_l ? __ldg(p.ulist + size_t(cur.pi) * p.nao + kpos_l) : 0;
        const int f_l = cval_l ? int(p.uflag[size_t(cur.pi) * p.nao + kpos_l]) : 0;
        const int tu_l = cval_l ? p.tau[size_t(cur.s) * p.nao + u_l] : kBadExp;
        const bool bad_l = cval_l && tu_l == kBadExp;
        eg = __reduce_max_sync(0xffffffffu, tu_l != kBadExp ? -tu_l : INT_MIN);
        if (eg == INT_MIN) eg = 0;
        s_l = tu_l != kBadExp ? ldexp(1.0, -tu_l - eg) : 0.0;
        badbits = __ballot_sync(0xffffffffu, bad_l);
        sg = gval ? B.sigma[gpt] : 0;
#pragma unroll
        for (int qi = 0; qi < C::MAXQ; ++qi) {
          if (qi < nq) {
            const int col0 = (grp + NG * (qi >> 1)) * 8 + 4 * (qi & 1);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int src = qi * 4 + j;  // lane holding the column
              const int uj = __shfl_sync(0xffffffffu, u_l, src);
              const int fj = __shfl_sync(0xffffffffu, f_l, src);
              const bool o = gval && cur.ut * TN + col0 + j < cur.nu && ((fj >> h) & 1);
              on |= uint32_t(o) << src;
              cp_async_8(phl + src * 32 + lane,
                         B.ao_lhs + (o ? size_t(uj) * B.stride_grid + gpt : 0), o);
            }
          }
        }
        cp_async_commit();
      }
      // ---- the group's chunks of the item (the first one already in its
      // stage when `ahead`), the union columns of the next one loaded a
      // chunk ahead ----
      int c = cur.kc0 + grp + (ahead ? NG : 0);
      int ivn[4];
      columns(cur, c, ivn);
      for (; c < cur.kc; c += NG) {
        int iv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) iv[k] = ivn[k];
        columns(cur, c + NG, ivn);
        uint2 w[C::STEPS][4];
        load_chunk(cur, c, iv, w);
        if (!store_chunk(seq0 + uint32_t(c - cur.kc0), w)) {
          ok = false;
          break;
        }
      }
      if (!ok) break;
      const uint32_t seq1 = seq0 + uint32_t(cur.kc - cur.kc0);
      // ---- the next item's first chunk of this group: loaded now, stored
      // as soon as the accumulators are read, so the MMAs go on at once.
      // Its stage was last used by chunk seq1 + grp - STAGES < seq1
      // (NG <= STAGES): a chunk of this item or before, done once the
      // accumulators are full ----
      setup(item_of(nitem + 1, true), nxt);
      ahead = nxt.t < total && nxt.kc0 + grp < nxt.kc;
      uint2 wn[C::STEPS][4];
      if (ahead) {
        int iv[4];
        columns(nxt, nxt.kc0 + grp, iv);
        load_chunk(nxt, nxt.kc0 + grp, iv, wn);
      }
      // ---- epilogue: this warp's 32 points (TMEM lanes 32wq ..) over the
      // group's column octets ----
      const bool acc_ok = tc::mbar_wait(acc_full, nitem & 1, err, 32, false, lim);
      cp_async_wait<0>();
      if (!acc_ok) break;
      tc::fence_after_sync();
      if (done < static_cast<long long>(seq1) - 1) done = static_cast<long long>(seq1) - 1;
      double acc = 0.0;
      // an active column whose D row holds Inf or NaN makes the point's value NaN
      const bool badrow = (on & badbits) != 0;
#pragma unroll
      for (int qi = 0; qi < C::MAXQ; ++qi) {
        if (qi < nq) {
          const int col0 = (grp + NG * (qi >> 1)) * 8 + 4 * (qi & 1);
          uint32_t v[NSL][4];
#pragma unroll
          for (int L = 0; L < NSL; ++L)
            tc::tmem_ld_32x32b_x4(trow + uint32_t(L * TN + col0), v[L]);
          tc::tmem_ld_wait();
          if (qi + 1 == nq) {  // the accumulators are read: the MMA warp may go on
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(acc_empty);
          }
          // phi_lhs is zero where the AO is inactive in this point's block
          // and s is zero for a row holding Inf or NaN (flagged above), so
          // every column goes through the same branch-free update
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int src = qi * 4 + j;
            const double sj = __shfl_sync(0xffffffffu, s_l, src);
            uint32_t lv[NSL];
#pragma unroll
            for (int L = 0; L < NSL; ++L) lv[L] = v[L][j];
            acc = fma(phl[src * 32 + lane], combine_levels<NSL>(lv) * sj, acc);
          }
        }
      }
      if (nq == 0) {
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(acc_empty);
      }
      if (ahead && !store_chunk(seq1 + uint32_t(grp), wn)) break;
      double res = 0.0;
      if (gval) {
        const int e = eg - sg;
        res = (sg == kBadExp || badrow) ? __longlong_as_double(0x7ff8000000000000LL)
              : (e >= -1022 && e <= 1023) ? acc * pow2(e)
                                          : ldexp(acc, e);
        if (sym) res *= 2.0;
      }
      // each group's own partial sum (the reduction adds the groups and the
      // row tiles in a fixed order), so no group waits for another here
      const size_t pbase = p.poff ? size_t(p.poff[cur.pi]) : size_t(cur.pi) * p.max_t;
      p.partial[(((pbase + cur.ut) * p.nset_max + cur.s) * NG + grp) * PT + r] = res;
      seq0 = seq1;
      cur = nxt;
    }
  } else if (warp == GW) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_i8(PT, TN);
      uint32_t seq = 0, nitem = 0;
      bool ok = true;
      for (;; ++nitem) {
        const int t = item_of(nitem, false);
        if (t >= total || !ok) break;
        const int4 it = p.items[t];
        const int nu = p.ucount[it.x];
        const int kc = (nu + TK - 1) / TK;
        const int kc0 = sym ? (it.y * TN) / TK : 0;
        if (nitem > 0 && !tc::mbar_wait(acc_empty, (nitem - 1) & 1, err, 33, false, lim)) break;
        tc::fence_after_sync();
        for (int c = kc0; c < kc; ++c, ++seq) {
          const int stg = int(seq % STAGES);
          const uint32_t par = (seq / STAGES) & 1;
          if (!tc::mbar_wait(&full_phi[stg], par, err, 34, false, lim) ||
              !tc::mbar_wait(&full_d[stg], par, err, 35, false, lim)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          const uint32_t a0 = tc::smem_u32(smem + stg * C::STAGE);
          const uint32_t b0 = a0 + C::A_STAGE;
          // phi digit j (the A operand) meets D digits 0 .. NSL-1-j (levels
          // j .. NSL-1) in consecutive MMAs: its plane is read from shared
          // memory once and held in the collector buffer for the rest
#pragma unroll
          for (int j = 0; j < NSL; ++j) {
            const uint64_t ad = tc::smem_desc_k32(a0 + j * C::A_SLICE);
            const bool acc = c > kc0 || j > 0;
#pragma unroll
            for (int i = 0; i + j < NSL; ++i) {
              const uint32_t d = tmem + uint32_t((i + j) * TN);
              const uint64_t bd = tc::smem_desc_k32(b0 + i * C::B_SLICE);
              if (j == NSL - 1)
                tc::mma_i8(d, ad, bd, idesc, acc);
              else if (i == 0)
                tc::mma_i8_collect<tc::ACollector::kFill>(d, ad, bd, idesc, acc);
              else if (i + j == NSL - 1)
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
      tc::mbar_wait(drain, 0, err, 36, true, lim);
    }
  } else {
    // ---------------- phi digit tiles: bulk loads ----------------
    if (lane == 0) {
      uint32_t seq = 0;
      uint32_t issued[STAGES];
#pragma unroll
      for (int s = 0; s < STAGES; ++s) issued[s] = 0;
      bool ok = true;
      // Items are drawn kAhead ahead of the one whose tiles are loaded, so a
      // gather group finds the next item in the ring when it reaches it.  A
      // draw waits until every warp has read the slot's previous item; after
      // a failed wait the terminal item goes in, so every role stops.
      int tq[kRing];  // the drawn items by ring slot
      uint32_t ndrawn = 0;
      bool ended = false;
      auto draw = [&]() {
        const uint32_t n = ndrawn++;
        const int slot = int(n % kRing);
        int t = total;
        if (ok && (n < kRing || tc::mbar_wait(&iempty[slot], ((n / kRing) - 1) & 1, err, 41,
                                              false, lim))) {
          t = atomicAdd(p.counter, 1);
          if (t > total) t = total;
        }
        ring[slot] = t;
        tq[slot] = t;
        tc::mbar_arrive(&ifull[slot]);   // release: the slot's value is visible to the waiters
        tc::mbar_arrive(&iempty[slot]);  // this warp's own read
        ended = t >= total;
      };
      for (uint32_t n = 0;; ++n) {
        while (!ended && ndrawn <= n + kAhead) draw();
        const int t = tq[n % kRing];
        if (t >= total) break;
        const int4 it = p.items[t];
        const int nu = p.ucount[it.x];
        const int kc = (nu + TK - 1) / TK;
        const int kc0 = sym ? (it.y * TN) / TK : 0;
        const uint8_t* src = p.phisl + size_t(p.cbase[it.x]) * C::A_STAGE;
        for (int c = kc0; c < kc; ++c, ++seq) {
          const int stg = int(seq % STAGES);
          const uint32_t use = seq / STAGES;
          if (use > 0 && !tc::mbar_wait(&empty[stg], (use - 1) & 1, err, 37, false, lim)) {
            ok = false;
            break;
          }
          // test hook: the first stage is never published, so the MMA warp's
          // bounded wait runs out and the call reports a timeout
          if (p.inject && seq == 0) continue;
          tc::mbar_arrive_expect_tx(&full_phi[stg], C::A_STAGE);
          tc::bulk_load(smem + stg * C::STAGE, src + size_t(c) * C::A_STAGE, C::A_STAGE,
                        &full_phi[stg]);
#pragma unroll
          for (int s = 0; s < STAGES; ++s) issued[s] += s == stg;
        }
        if (!ok) {
          while (!ended) draw();
          break;
        }
      }
      // copies still in flight complete before the CTA exits
#pragma unroll
      for (int s = 0; s < STAGES; ++s)
        if (issued[s] > 0) tc::mbar_wait(&full_phi[s], (issued[s] - 1) & 1, err, 38, true, lim);
    }
  }

  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == GW) tc::tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------------------
// deterministic reduction: rho[s][g] += sum over the row tiles, in order
// ---------------------------------------------------------------------------
template <int TN>
__global__ void __launch_bounds__(256)
pair_reduce(PairArgs p, const int* __restrict__ npairs, int pair0) {
  const int pl = blockIdx.x;
  if (pl >= npairs[0]) return;
  const int pi = pair0 + pl;
  const int4 pr = p.pairs[pi];
  const PairBatch& B = batch_of(p, pr.z);
  const int nt = (p.ucount[pi] + TN - 1) / TN;
  if (nt == 0) return;
  const size_t pbase = p.poff ? size_t(p.poff[pi]) : size_t(pi) * p.max_t;
  for (int v = threadIdx.x; v < B.nset * PT; v += 256) {
    const int s = v / PT, r = v % PT;
    const int h = r >> 6;
    const int tile = h ? pr.y : pr.x;
    if (tile < 0) continue;
    int g0, gend;
    tile_points(tile, p.blk, p.gsub, B.ngrid, &g0, &gend);
    const int g = g0 + (r & (HT - 1));
    if (g >= gend) continue;
    double acc = 0.0;
    for (int t = 0; t < nt; ++t)
#pragma unroll
      for (int gq = 0; gq < NG; ++gq)
        acc += p.partial[(((pbase + t) * p.nset_max + s) * NG + gq) * PT + r];
    double* out = B.rhos + size_t(s) * B.stride_grid + g;
    *out = acc + *out;
  }
}

template <int NSL, int STAGES>
cudaError_t launch_pair_main_t(int nsm, const PairArgs& a, cudaStream_t stream, bool attrs_only) {
  constexpr size_t smem = Cfg<NSL>::template smem_bytes<STAGES>();
  static_assert(smem <= 232448, "shared memory per CTA");
  cudaError_t err = cudaFuncSetAttribute(pair_main<NSL, STAGES>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (err != cudaSuccess || attrs_only) return err;
  pair_main<NSL, STAGES><<<nsm, THREADS, smem, stream>>>(a);
  return cudaGetLastError();
}

size_t a256(size_t v) { return (v + 255) / 256 * 256; }

struct Layout {
  size_t lists, counts, bits, cnt, key, order, cand, ncand, partner, pos, choice, pairs, npairs,
      ulist, uflag, ucount, cbase, cpair, items, total, dsl, tau, dhalf, sigma, pmax, phisl,
      partial, bytes;
};

Layout layout(size_t nao, size_t ngrid, size_t nset, size_t blk, int nsl) {
  const size_t nblk = (ngrid + blk - 1) / blk;
  const size_t gsub = (blk + HT - 1) / HT;
  const size_t nbg = nblk * gsub;
  const size_t tn = nsl == 6 ? Cfg<6>::TN : Cfg<7>::TN;
  const size_t max_t = (nao + tn - 1) / tn;
  const size_t max_kc = (nao + TK - 1) / TK;
  const size_t nwords = (nao + 31) / 32;
  const size_t a_stage = size_t(nsl) * PT * TK;
  Layout L;
  L.lists = 0;
  L.counts = L.lists + a256(nblk * nao * sizeof(int));
  L.bits = L.counts + a256(nblk * sizeof(int));
  L.cnt = L.bits + a256(nbg * nwords * sizeof(uint32_t));
  L.key = L.cnt + a256(nbg * sizeof(int));
  L.order = L.key + a256(nbg * sizeof(unsigned long long));
  L.cand = L.order + a256(nbg * sizeof(int));
  L.ncand = L.cand + a256(nbg * 2 * kWin * sizeof(int));
  L.partner = L.ncand + a256(nbg * sizeof(int));
  L.pos = L.partner + a256(nbg * sizeof(int));
  L.choice = L.pos + a256(nbg * sizeof(int));
  L.pairs = L.choice + a256(nbg * sizeof(int));
  L.npairs = L.pairs + a256(nbg * sizeof(int4));
  L.ulist = L.npairs + 256;
  L.uflag = L.ulist + a256(nbg * nao * sizeof(int));
  L.ucount = L.uflag + a256(nbg * nao);
  L.cbase = L.ucount + a256(nbg * sizeof(int));
  L.cpair = L.cbase + a256((nbg + 1) * sizeof(int));
  L.items = L.cpair + a256(nbg * max_kc * sizeof(int));
  L.total = L.items + a256(nbg * max_t * nset * sizeof(int4));
  L.dsl = L.total + 256;
  L.tau = L.dsl + a256(nset * nao * nao * 8);
  L.dhalf = L.tau + a256(nset * nao * sizeof(int));
  L.sigma = L.dhalf + a256(nset * nao * 8);
  L.pmax = L.sigma + a256(ngrid * sizeof(int));
  L.phisl = L.pmax + a256(ngrid * sizeof(unsigned long long));
  L.partial = L.phisl + a256(nbg * max_kc * a_stage);
  L.bytes = L.partial + nbg * max_t * nset * NG * PT * sizeof(double);
  return L;
}

}  // namespace

int split_pair_row_tile(int nsl) { return nsl == 6 ? Cfg<6>::TN : Cfg<7>::TN; }

int split_pair_digits() {  // read on every call: the workspace covers both counts
  const char* e = std::getenv("CFGMM_SPLIT_DIGITS");
  const int d = e ? std::atoi(e) : 7;
  return (d == 6 || d == 7) ? d : 7;
}

size_t aodmao2rho_split_pair_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk,
                                       int nsl) {
  return layout(nao, ngrid, nset, blk, nsl).bytes;
}

int split_pair_stages() {  // fixed: with the epilogue's phi_lhs values three stages fit
  return kStages;
}

int split_pair_partial_points() { return NG * PT; }

cudaError_t split_pair_launch_main(const PairArgs& a, int nsl, cudaStream_t stream,
                                   bool attrs_only, int /*stages*/) {
  int dev = 0, nsm = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (err != cudaSuccess) return err;
  if (nsl == 6) return launch_pair_main_t<6, kStages>(nsm, a, stream, attrs_only);
  return launch_pair_main_t<7, kStages>(nsm, a, stream, attrs_only);
}

cudaError_t split_pair_launch_reduce(const PairArgs& a, int nsl, const int* npairs, int pair0,
                                     int max_pairs, cudaStream_t stream) {
  if (max_pairs <= 0) return cudaSuccess;
  if (nsl == 6)
    pair_reduce<Cfg<6>::TN><<<max_pairs, 256, 0, stream>>>(a, npairs, pair0);
  else
    pair_reduce<Cfg<7>::TN><<<max_pairs, 256, 0, stream>>>(a, npairs, pair0);
  return cudaGetLastError();
}

cudaError_t split_pair_prepare_d(const double* dms, size_t stride_ao, int nao, int nset, int nsl,
                                 uint2* dsl, int* tau, uint2* dhalf, int* asym,
                                 cudaStream_t stream) {
  const int nt = (nao + 31) / 32;
  const long long tiles = asym ? (long long)nset * (nt * (nt + 1) / 2) : 0;
  const long long grid = (long long)nset * nao + tiles;
  if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  if (nsl == 6)
    pair_d_prep<6><<<unsigned(grid), 256, 0, stream>>>(dms, stride_ao, stride_ao * stride_ao, nao,
                                                         nset, dsl, tau, dhalf, asym);
  else
    pair_d_prep<7><<<unsigned(grid), 256, 0, stream>>>(dms, stride_ao, stride_ao * stride_ao, nao,
                                                         nset, dsl, tau, dhalf, asym);
  return cudaGetLastError();
}

namespace {

struct BatchDims {
  int nbg, gsub, nwords, tn, max_kc;
};

BatchDims batch_dims(const PairPrep& q) {
  BatchDims d;
  d.gsub = (q.blk + HT - 1) / HT;
  d.nbg = ((q.ngrid + q.blk - 1) / q.blk) * d.gsub;
  d.nwords = (q.nao + 31) / 32;
  d.tn = q.nsl == 6 ? Cfg<6>::TN : Cfg<7>::TN;
  d.max_kc = (q.nao + TK - 1) / TK;
  return d;
}

}  // namespace

cudaError_t split_pair_lists_and_signatures(const PairPrep& q, int* lists, int* counts,
                                            cudaStream_t stream) {
  const BatchDims d = batch_dims(q);
  if (d.nbg <= 0) return cudaSuccess;
  const int nblk = d.nbg / d.gsub;
  pair_lists_sig<<<nblk, 256, 0, stream>>>(q.tab, q.ldtab, q.nao, nblk, d.gsub, d.nwords, lists,
                                           counts, q.bits, q.cnt, q.key);
  return cudaGetLastError();
}

cudaError_t split_pair_prepare_pairs(const PairPrep& q, cudaStream_t stream, bool signatures) {
  const BatchDims d = batch_dims(q);
  if (d.nbg <= 0) return cudaSuccess;
  constexpr size_t sort_smem = size_t(kSortMax) * (sizeof(unsigned long long) + sizeof(int));
  static const cudaError_t sort_attr = cudaFuncSetAttribute(
      pair_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sort_smem));
  if (sort_attr != cudaSuccess) return sort_attr;
  if (signatures)
    pair_sig<<<d.nbg, 256, 0, stream>>>(q.tab, q.ldtab, q.nao, d.nbg, d.gsub, d.nwords, q.bits,
                                        q.cnt, q.key);
  pair_sort<<<1, 1024, sort_smem, stream>>>(q.key, d.nbg, q.order);
  pair_scores<<<d.nbg, 2 * kWin, 0, stream>>>(q.bits, q.cnt, q.order, d.nbg, d.nwords, q.cand,
                                              q.ncand);
  constexpr size_t match_base = size_t(3) * kSortMax * sizeof(int);
  constexpr size_t match_cands = size_t(kMatchCandMax) * 2 * kWin * sizeof(int);
  static const cudaError_t match_attr = cudaFuncSetAttribute(
      pair_match, cudaFuncAttributeMaxDynamicSharedMemorySize, int(match_base + match_cands));
  if (match_attr != cudaSuccess) return match_attr;
  const size_t match_smem =
      match_base + (d.nbg <= kMatchCandMax ? size_t(d.nbg) * 2 * kWin * sizeof(int) : 0);
  pair_match<<<1, 1024, match_smem, stream>>>(q.order, q.cand, q.ncand, q.cnt, d.nbg, q.batch,
                                              q.partner, q.pos, q.choice, q.pairs + q.pair0,
                                              q.npairs);
  pair_union<<<d.nbg, 256, 0, stream>>>(q.tab, q.ldtab, q.nao, d.gsub, q.pairs, q.npairs, q.pair0,
                                        q.ulist, q.uflag, q.ucount);
  const size_t hist = size_t(d.max_kc + 2) * sizeof(int);
  pair_build<<<1, 1024, hist, stream>>>(q.ucount, q.npairs, q.pair0, q.nset, q.batch, d.tn,
                                        d.max_kc, q.chunk0, q.cbase, q.cpair, q.items, q.total,
                                        q.chunks_end);
  return cudaGetLastError();
}

cudaError_t split_pair_prepare_scales(const PairPrep& q, cudaStream_t stream) {
  const BatchDims d = batch_dims(q);
  if (d.nbg <= 0) return cudaSuccess;
  cudaError_t err = cudaMemsetAsync(q.pmax, 0, size_t(q.ngrid) * sizeof(unsigned long long),
                                    stream);
  if (err != cudaSuccess) return err;
  pair_phi_max<<<dim3(d.nbg, (q.nao + 63) / 64), 256, 0, stream>>>(
      q.ao_rhs, q.stride_grid, q.lists, q.counts, q.nao, q.ngrid, q.blk, d.gsub, q.pmax);
  return cudaGetLastError();
}

cudaError_t split_pair_prepare_tiles(const PairPrep& q, cudaStream_t stream) {
  const BatchDims d = batch_dims(q);
  if (d.nbg <= 0) return cudaSuccess;
  int dev = 0, nsm = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (err != cudaSuccess) return err;
  // persistent: as many CTAs as fit beside one another (30 KB of shared memory each)
  const unsigned grid = unsigned(std::min<long long>((long long)nsm * 6,
                                                     (long long)d.nbg * d.max_kc));
  if (q.nsl == 6)
    pair_phi_tiles<6><<<grid, 256, 0, stream>>>(q.ao_rhs, q.stride_grid, q.pmax, q.pairs, q.cpair,
                                                q.chunk0, q.chunks_end, q.ulist, q.uflag,
                                                q.ucount, q.cbase, q.nao, q.ngrid, q.blk, d.gsub,
                                                q.sigma, q.phisl);
  else
    pair_phi_tiles<7><<<grid, 256, 0, stream>>>(q.ao_rhs, q.stride_grid, q.pmax, q.pairs, q.cpair,
                                                q.chunk0, q.chunks_end, q.ulist, q.uflag,
                                                q.ucount, q.cbase, q.nao, q.ngrid, q.blk, d.gsub,
                                                q.sigma, q.phisl);
  return cudaGetLastError();
}

namespace {

// poff[pi] = sum over the pairs before pi of their row tiles (ceil(ucount/tn)),
// poff[npairs] the total: the partial sums' offsets.  One CTA.
__global__ void __launch_bounds__(1024)
pair_partial_offsets(const int* __restrict__ ucount, const int* __restrict__ npairs_d, int tn,
                     int* __restrict__ poff) {
  __shared__ int warp_c[32];
  __shared__ int base_s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int np = npairs_d[0];
  if (tid == 0) base_s = 0;
  __syncthreads();
  for (int p0 = 0; p0 < np; p0 += 1024) {
    const int pl = p0 + tid;
    const int nt = pl < np ? (ucount[pl] + tn - 1) / tn : 0;
    int ic = nt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, ic, o);
      if (lane >= o) ic += t;
    }
    if (lane == 31) warp_c[warp] = ic;
    __syncthreads();
    int bc = base_s;
    for (int w = 0; w < warp; ++w) bc += warp_c[w];
    if (pl < np) poff[pl] = bc + ic - nt;
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < 32; ++w) base_s += warp_c[w];
    __syncthreads();
  }
  if (tid == 0) poff[np] = base_s;
}

}  // namespace

cudaError_t split_pair_partial_offsets(const int* ucount, const int* npairs, int tn, int* poff,
                                       cudaStream_t stream) {
  pair_partial_offsets<<<1, 1024, 0, stream>>>(ucount, npairs, tn, poff);
  return cudaGetLastError();
}

cudaError_t split_pair_prepare_batch(const PairPrep& q, cudaStream_t stream) {
  cudaError_t err = split_pair_prepare_scales(q, stream);
  if (err == cudaSuccess) err = split_pair_prepare_pairs(q, stream);
  if (err == cudaSuccess) err = split_pair_prepare_tiles(q, stream);
  return err;
}

cudaError_t aodmao2rho_split_pair(double* rhos, const double* dms, const double* ao_lhs,
                                  const double* ao_rhs, size_t stride_ao, size_t stride_grid,
                                  int nao, int ngrid, int nset, const uint8_t* tab, size_t ldtab,
                                  int blk, int nsl, void* workspace, cudaStream_t stream,
                                  int inject, unsigned long long wait_ns) {
  if (nao <= 0 || ngrid <= 0 || nset <= 0) return cudaSuccess;
  if (nsl != 6 && nsl != 7) return cudaErrorInvalidValue;
  const int nblk = (ngrid + blk - 1) / blk;
  const int gsub = (blk + HT - 1) / HT;
  const int nbg = nblk * gsub;
  const int tn = nsl == 6 ? Cfg<6>::TN : Cfg<7>::TN;
  const Layout L = layout(nao, ngrid, nset, blk, nsl);
  char* ws = static_cast<char*>(workspace);
  auto at = [&](size_t off) { return static_cast<void*>(ws + off); };
  int* lists = static_cast<int*>(at(L.lists));
  int* counts = static_cast<int*>(at(L.counts));
  PairPrep q{};
  q.tab = tab;
  q.ldtab = ldtab;
  q.ao_rhs = ao_rhs;
  q.stride_grid = stride_grid;
  q.nao = nao;
  q.ngrid = ngrid;
  q.blk = blk;
  q.nset = nset;
  q.nsl = nsl;
  q.batch = 0;
  q.pair0 = 0;
  q.chunk0 = 0;
  q.lists = lists;
  q.counts = counts;
  q.bits = static_cast<uint32_t*>(at(L.bits));
  q.cnt = static_cast<int*>(at(L.cnt));
  q.key = static_cast<unsigned long long*>(at(L.key));
  q.order = static_cast<int*>(at(L.order));
  q.cand = static_cast<int*>(at(L.cand));
  q.ncand = static_cast<int*>(at(L.ncand));
  q.partner = static_cast<int*>(at(L.partner));
  q.pos = static_cast<int*>(at(L.pos));
  q.choice = static_cast<int*>(at(L.choice));
  q.pairs = static_cast<int4*>(at(L.pairs));
  q.npairs = static_cast<int*>(at(L.npairs));
  q.ulist = static_cast<int*>(at(L.ulist));
  q.uflag = static_cast<uint8_t*>(at(L.uflag));
  q.ucount = static_cast<int*>(at(L.ucount));
  q.cbase = static_cast<int*>(at(L.cbase));
  q.cpair = static_cast<int*>(at(L.cpair));
  q.items = static_cast<int4*>(at(L.items));
  q.total = static_cast<int*>(at(L.total));
  q.chunks_end = q.total + 2;
  q.sigma = static_cast<int*>(at(L.sigma));
  q.pmax = static_cast<unsigned long long*>(at(L.pmax));
  q.phisl = static_cast<uint8_t*>(at(L.phisl));
  uint2* dsl = static_cast<uint2*>(at(L.dsl));
  int* tau = static_cast<int*>(at(L.tau));
  uint2* dhalf = static_cast<uint2*>(at(L.dhalf));

  // total[0]: items, total[1]: asymmetry flag, total[2]: chunks, total[3]: item counter
  int* asym = aodm_sym_enabled() && ao_lhs == ao_rhs ? q.total + 1 : nullptr;
  cudaError_t err = cudaMemsetAsync(q.total, 0, 4 * sizeof(int), stream);
  if (err != cudaSuccess) return err;
  // Two chains.  On a high-priority side stream the pairing chain (block lists
  // with the tile signatures, sort, scores, matching, unions, work list,
  // then the phi tiles); on the caller's stream the D preparation (digits and
  // symmetry check) and then the point scales (after the block lists).  The
  // phi tiles wait for the scales; the side stream joins back before the
  // main kernel.  (The D preparation after the pairing kernels, or after the
  // scales, measured slower: the preparation as a whole is bound by memory
  // traffic and latency, about 0.22 ms at taxol size.)
  SideScope side(side_stream(true), stream);
  if ((err = side.fork()) != cudaSuccess) return err;
  const cudaStream_t sp = side.stream();
  const SideStream* ss = side_stream(true);
  const bool split_streams = sp != stream && ss;
  if ((err = split_pair_prepare_d(dms, stride_ao, nao, nset, nsl, dsl, tau, dhalf, asym,
                                  stream)) != cudaSuccess)
    return err;
  if ((err = split_pair_lists_and_signatures(q, lists, counts, sp)) != cudaSuccess) return err;
  if (split_streams && (err = side_join(ss, stream)) != cudaSuccess) return err;  // lists -> scales
  if ((err = split_pair_prepare_scales(q, stream)) != cudaSuccess) return err;
  if ((err = split_pair_prepare_pairs(q, sp, false)) != cudaSuccess) return err;
  if (split_streams && (err = side_fork(ss, stream)) != cudaSuccess) return err;  // scales -> tiles
  if ((err = split_pair_prepare_tiles(q, sp)) != cudaSuccess) return err;
  if ((err = side.join()) != cudaSuccess) return err;

  PairArgs a{};
  a.dsl = dsl;
  a.tau = tau;
  a.dhalf = dhalf;
  a.phisl = q.phisl;
  a.items = q.items;
  a.total = q.total;
  a.pairs = q.pairs;
  a.ucount = q.ucount;
  a.ulist = q.ulist;
  a.uflag = q.uflag;
  a.cbase = q.cbase;
  a.batches = nullptr;
  a.one = PairBatch{ao_lhs, rhos, q.sigma, stride_grid, ngrid, nset};
  a.partial = static_cast<double*>(at(L.partial));
  a.poff = nullptr;
  a.nao = nao;
  a.blk = blk;
  a.gsub = gsub;
  a.max_t = (nao + tn - 1) / tn;
  a.nset_max = nset;
  a.asym = asym;
  a.counter = q.total + 3;
  unsigned long long armed_ns = 0;
  if (take_wait_injection(1, &armed_ns)) {  // cfgmm_test_arm_wait_timeout
    inject = 1;
    wait_ns = armed_ns;
  }
  a.wait_ns = wait_ns;
  a.inject = inject;
  if ((err = split_pair_launch_main(a, nsl, stream, false)) != cudaSuccess) return err;
  return split_pair_launch_reduce(a, nsl, q.npairs, 0, nbg, stream);
}

cudaError_t aodmao2rho_split_pair_reset_error(cudaStream_t stream) {
  static const int zero = 0;
  return cudaMemcpyToSymbolAsync(g_pair_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice,
                                 stream);
}

cudaError_t aodmao2rho_split_pair_read_error(int* code) {
  return cudaMemcpyFromSymbol(code, g_pair_error, sizeof(int));
}

}  // namespace cfgmm
