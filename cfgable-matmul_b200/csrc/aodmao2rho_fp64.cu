// aodmao2rho_fp64.cu -- masked AO-DM-AO contraction in FP64 on the FP64 tensor cores.
//
//   rho[s][g] += sum_{u in I(b)} ao_lhs[u][g] * sum_{v in I(b)} D_s[u][v] * ao_rhs[v][g],
//   b = g / BLK,  I(b) = { u < nao : tab[u*ldtab + b] != 0 } in ascending order.
//
// Semantics follow MatmulLoops::aodmao2rho_loop_parallel
// (src/impl_aodmao2rho.rs:171-244): the per-block active lists are exactly the
// reference's compaction (get_indices_from_non0tab, impl_matmul_non0tab.rs:
// 118-129, applied per block in impl_aodmao2rho.rs:126-133), a block with an
// empty list is skipped, masked (AO, block) entries never contribute whatever
// ao_lhs / ao_rhs hold there, and rho is accumulated into.
//
// Design:
//   1. aodm_block_lists: one CTA per grid block builds I(b) on the device
//      (ballot + popc prefix sums); no host round trip.
//   2. aodm_build_items: one CTA turns the per-block counts into a compact
//      work list (block b, 64-point grid tile, 64-row tile of I(b)) and resets
//      the work counters.
//   3. aodm_fp64_kernel: a persistent kernel, one CTA per SM and group of up
//      to 3 density matrices, that draws work items from the list.  It forms
//      X = D_s[I,I] * ao_rhs[I, tile] on the FP64 tensor cores (DMMA
//      m16n8k4) with the gather done by 8-byte cp.async straight from the
//      compacted index list -- no packed copy of D ever reaches HBM -- and
//      then reduces phi_lhs (.) X over the 64 rows in registers, warp
//      shuffles and shared memory, so X never leaves the SM.  The ao_rhs
//      tile is shared by all density matrices of the group.
//      The active list of the current block is staged in shared memory, so
//      the gather addresses never wait on global loads.
//   3b. aodm_fp64_pipe_kernel: the same items with producer warps (D by
//      cp.async; ao_rhs rows by TMA gather4 where the rows are 16-byte
//      aligned and BLKSIZE is even, by cp.async otherwise) and consumer warps
//      (DMMA m16n8k8) meeting on mbarriers; with a symmetric-D mode.  The
//      form used; form 3 remains for CFGMM_AODM_PIPE=0.
//   4. aodm_reduce: adds the per-row-tile partial sums of each grid tile in a
//      fixed order, so results are deterministic run to run (unlike the
//      reference, whose lock order varies).
#include <cstdlib>
#include <mutex>

#include <cudaTypedefs.h>

#include "common.cuh"
#include "aodmao2rho_fp64.cuh"
#include "tcgen05.cuh"

namespace cfgmm {

// Error word of the pipelined kernel's bounded waits (0 = none).
__device__ int g_aodm_error;

namespace {

constexpr int TU = 64;   // compacted rows (u) per work item
constexpr int TG = 64;   // grid points per work item
constexpr int STAGES = 3;
constexpr int THREADS = 256;
constexpr int LIST_CAP = 8192;  // active-list entries staged in shared memory

// ---------------------------------------------------------------------------
// 1. active lists: lists[b*nao + i] = i-th active AO of block b, counts[b]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
aodm_block_lists(const uint8_t* __restrict__ tab, size_t ldtab, int nao, int nblk,
                 int* __restrict__ lists, int* __restrict__ counts) {
  const int b = blockIdx.x;
  if (b >= nblk) return;
  __shared__ int warp_tot[8];
  __shared__ int base_s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) base_s = 0;
  __syncthreads();
  int* out = lists + size_t(b) * nao;
  for (int u0 = 0; u0 < nao; u0 += 256) {
    const int u = u0 + tid;
    const bool on = (u < nao) && tab[size_t(u) * ldtab + b] != 0;
    const unsigned bal = __ballot_sync(0xffffffffu, on);
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
  if (tid == 0) counts[b] = base_s;
}

// ---------------------------------------------------------------------------
// 2. work list: items[i] = (0, b * gsub + gt, utile) for every row tile of every
//    non-empty (block, grid tile), in block order; counters[g] = 0.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
aodm_build_items(const int* __restrict__ counts, int nblk, int gsub, int4* __restrict__ items,
                 int* __restrict__ counters, int ncounters) {
  __shared__ int warp_tot[32];
  __shared__ int base_s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    base_s = 0;
    g_aodm_error = 0;
  }
  // [ncounters] = total, [ncounters + 1] = asymmetry flag
  for (int i = tid; i <= ncounters + 1; i += 1024) counters[i] = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nblk; b0 += 1024) {
    const int b = b0 + tid;
    const int nt = (b < nblk) ? (counts[b] + TU - 1) / TU : 0;
    const int mine = nt * gsub;
    // block-wide exclusive scan of `mine`
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    int before = base_s;
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    before += incl - mine;
    for (int j = 0; j < mine; ++j) items[before + j] = make_int4(0, b * gsub + j / nt, j % nt, 0);
    __syncthreads();
    if (tid == 0) {
      int t = 0;
      for (int w = 0; w < 32; ++w) t += warp_tot[w];
      base_s += t;
    }
    __syncthreads();
  }
  if (tid == 0) counters[ncounters] = base_s;
}

// ---------------------------------------------------------------------------
// 3. main kernel
// ---------------------------------------------------------------------------
template <int NS, int TKT>
__global__ void __launch_bounds__(THREADS, 1) aodm_fp64_kernel(AodmArgs p) {
  extern __shared__ __align__(128) double smem[];
  constexpr int D_TILE = TU * TKT;  // one D tile per set
  constexpr int P_TILE = TG * TKT;  // ao_rhs tile, stored [g][k]
  constexpr int STAGE = NS * D_TILE + P_TILE;
  constexpr int DC = TKT;           // D gather: threads per row (= columns of a chunk)
  constexpr int DR = THREADS / DC;  // D gather: rows per pass
  constexpr int PR = THREADS / TG;  // ao_rhs gather: k rows per pass
  int* list_s = reinterpret_cast<int*>(smem + STAGES * STAGE);  // LIST_CAP entries
  __shared__ int item_s;
  __shared__ long long key_s;

  const int set0 = blockIdx.y * NS;
  const int total = p.counters[p.ngroups];
  int* counter = p.counters + blockIdx.y;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps; warp tile 32 (u) x 16 (g)
  const int g = lane >> 2, q = lane & 3;
  const int c_d = tid % DC, r_d0 = tid / DC;  // D gather: column c_d, rows r_d0 + DR*i
  const int j_p = tid % TG, c_p0 = tid / TG;  // ao_rhs gather: point j_p, k rows c_p0 + PR*i

  if (tid == 0) key_s = -1;
  for (;;) {
    if (tid == 0) item_s = atomicAdd(counter, 1);
    __syncthreads();  // also orders this item's smem use after the previous one's
    const int it = item_s;
    if (it >= total) break;
    const int4 w = p.items[it];
    const AodmBatch& B = p.batches ? p.batches[w.x] : p.one;
    const int ns = min(NS, B.nset - set0);
    if (ns <= 0) continue;  // this batch has fewer density matrices
    const int bg = w.y, utile = w.z;
    const int b = bg / p.gsub, gt = bg % p.gsub;
    const int nb = B.counts[b];
    const int* Ig = B.lists + size_t(b) * p.nao;
    const bool staged = nb <= LIST_CAP;
    const long long key = (long long)w.x << 32 | b;  // (batch, block) whose list is staged
    if (staged && key_s != key) {
      for (int i = tid; i < nb; i += THREADS) list_s[i] = Ig[i];
      __syncthreads();
      if (tid == 0) key_s = key;
    }
    const int* I = staged ? list_s : Ig;
    const int u0 = utile * TU;
    const int g0 = b * p.blk + gt * TG;
    const int gw = min(min((b + 1) * p.blk, B.ngrid), g0 + TG) - g0;
    const int mu = min(TU, nb - u0);
    const bool jok = j_p < gw;

    int urow[TU / DR];
#pragma unroll
    for (int i = 0; i < TU / DR; ++i) {
      const int r = r_d0 + DR * i;
      urow[i] = (r < mu) ? I[u0 + r] : -1;
    }

    const int kchunks = (nb + TKT - 1) / TKT;
    auto issue = [&](int kc) {
      double* st = smem + (kc % STAGES) * STAGE;
      const int k0 = kc * TKT;
      const int kw = min(TKT, nb - k0);
      const bool cok = c_d < kw;
      const int vcol = cok ? I[k0 + c_d] : 0;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        double* Ds = st + s * D_TILE;
        const bool sok = s < ns;
        const double* dm = p.dms + size_t(set0 + (sok ? s : 0)) * p.dm_stride;
#pragma unroll
        for (int i = 0; i < TU / DR; ++i) {
          const int r = r_d0 + DR * i;
          const bool ok = sok && cok && urow[i] >= 0;
          const double* src = ok ? dm + size_t(urow[i]) * p.stride_ao + vcol : p.dms;
          cp_async_8(Ds + swz<TKT>(r, c_d), src, ok);
        }
      }
      double* Ps = st + NS * D_TILE;
#pragma unroll
      for (int i = 0; i < TKT / PR; ++i) {
        const int c = c_p0 + PR * i;
        const bool ok = jok && c < kw;
        const double* src =
            ok ? B.ao_rhs + size_t(I[k0 + c]) * B.stride_grid + (g0 + j_p) : B.ao_rhs;
        cp_async_8(Ps + swz<TKT>(j_p, c), src, ok);
      }
    };

    double acc[NS][2][2][4];
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[s][i][j][e] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < kchunks) issue(s);
      cp_async_commit();
    }
    for (int kc = 0; kc < kchunks; ++kc) {
      cp_async_wait<STAGES - 2>();
      __syncthreads();
      if (kc + STAGES - 1 < kchunks) issue(kc + STAGES - 1);
      cp_async_commit();

      const double* st = smem + (kc % STAGES) * STAGE;
      const double* Ps = st + NS * D_TILE;
#pragma unroll
      for (int kk = 0; kk < TKT; kk += 8) {
        double2 bv[2];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
          bv[nt] = *reinterpret_cast<const double2*>(Ps + swz<TKT>(wn * 16 + nt * 8 + g, kk + 2 * q));
        double2 av[NS][2][2];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const double* Ds = st + s * D_TILE;
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            const int r = wm * 32 + mt * 16 + g;
            av[s][mt][0] = *reinterpret_cast<const double2*>(Ds + swz<TKT>(r, kk + 2 * q));
            av[s][mt][1] = *reinterpret_cast<const double2*>(Ds + swz<TKT>(r + 8, kk + 2 * q));
          }
        }
        // k-slot .x of every tile of every set, then .y: dependent DMMAs on one
        // accumulator are 4*NS instructions apart.
#pragma unroll
        for (int s = 0; s < NS; ++s)
#pragma unroll
          for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
              dmma_16x8x4(acc[s][mt][nt], av[s][mt][0].x, av[s][mt][1].x, bv[nt].x);
#pragma unroll
        for (int s = 0; s < NS; ++s)
#pragma unroll
          for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
              dmma_16x8x4(acc[s][mt][nt], av[s][mt][0].y, av[s][mt][1].y, bv[nt].y);
      }
    }
    cp_async_wait<0>();
    __syncthreads();  // stage buffers are reused below

    // Epilogue: rho_part[s][j] = sum_r ao_lhs[I[u0+r]][g0+j] * X[s][r][j].
    // Thread rows: r = wm*32 + mt*16 + g + 8h; columns j = wn*16 + nt*8 + 2q + e.
    double lhs[2][2][2][2];  // [mt][h][nt][e]
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = wm * 32 + mt * 16 + g + 8 * h;
        const bool rok = r < mu;
        const double* row = rok ? B.ao_lhs + size_t(I[u0 + r]) * B.stride_grid : nullptr;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int j = wn * 16 + nt * 8 + 2 * q + e;
            lhs[mt][h][nt][e] = (rok && j < gw) ? row[g0 + j] : 0.0;
          }
      }
    double* red = smem;  // [NS][2 (wm)][TG]
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          double v = 0.0;
#pragma unroll
          for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) v = fma(acc[s][mt][nt][2 * h + e], lhs[mt][h][nt][e], v);
          v += __shfl_xor_sync(0xffffffffu, v, 4);
          v += __shfl_xor_sync(0xffffffffu, v, 8);
          v += __shfl_xor_sync(0xffffffffu, v, 16);
          if (g == 0) red[(s * 2 + wm) * TG + wn * 16 + nt * 8 + 2 * q + e] = v;
        }
    __syncthreads();
    const size_t slot = B.partial_off + size_t(bg) * p.max_utiles + utile;
    for (int t = tid; t < ns * TG; t += THREADS) {
      const int s = t / TG, j = t % TG;
      p.partial[(slot * p.nset_max + set0 + s) * TG + j] =
          red[(s * 2 + 0) * TG + j] + red[(s * 2 + 1) * TG + j];
    }
    // the __syncthreads at the top of the loop protects `red` and the stages
  }
}

// ---------------------------------------------------------------------------
// 3b. pipelined main kernel: the same work items and partial sums as (3), with
//     the roles split.  Four producer warps gather D_s[I_rows, I(k0..k0+15)]
//     with 8-byte cp.async (lanes along consecutive compacted columns, so a
//     warp's reads coalesce over the runs of active AOs) and one producer lane
//     fetches the ao_rhs rows I(k0..k0+15) x 64 points with TMA gather4 (four
//     arbitrary rows per instruction).  Both complete on the stage's mbarrier;
//     eight consumer warps run DMMA m16n8k8 from the stages and release them
//     through a second mbarrier, so the gather of later stages -- and of the
//     next work item -- overlaps the tensor-core work.  The roles meet only on
//     mbarriers, and every wait is bounded (tc::mbar_wait): on a timeout the
//     kernel records a code in g_aodm_error and every warp leaves (exit
//     decisions are made warp-uniform, so no warp-level sync meets an exited
//     lane).
// ---------------------------------------------------------------------------
namespace pipe {
constexpr int TK = 16;         // compacted AOs per stage
constexpr int PSTAGES = 5;     // 6 leaves too little L1 beside shared memory (measured)
constexpr int NPROD = 128;     // producer threads (4 warps)
constexpr int NCONS = 256;     // consumer threads (8 warps, 2 x 4 over rows x points)
constexpr int PTHREADS = NPROD + NCONS;
constexpr int RING = 4;        // work items in flight between the roles
constexpr int D_BYTES = TU * TK * 8;      // one density matrix's tile per stage
constexpr int PHI_BYTES = TK * TG * 8;    // ao_rhs rows, 64 points each, no swizzle
constexpr int RSTEP = NPROD / TK;              // rows apart of one thread's gathers
constexpr int ROWS_PER_THREAD = TU / RSTEP;     // 16

template <int NS>
constexpr int stage_bytes() { return NS * D_BYTES + PHI_BYTES; }

// consumer warp grid: CWM warps along the item's rows x CWN along its points;
// each warp holds MT x NT m16n8 tiles per density matrix.  Four row warps of
// 16 rows share their phi (B) fragments over 32 points: per k step of 8 a warp
// loads 2 A fragment pairs per matrix and 4 B fragment pairs.
constexpr int CWM = 4, CWN = 2;
constexpr int MT = TU / CWM / 16, NT = TG / CWN / 8;

template <int NS>
constexpr int red_doubles() { return 2 * NS * CWM * TG; }  // double-buffered [2][NS][CWM][TG]

template <int NS>
constexpr size_t smem_bytes() {
  return 1024 + size_t(PSTAGES) * stage_bytes<NS>() + size_t(red_doubles<NS>()) * 8 +
         (2 * PSTAGES + 2 * RING + 2) * 8 + RING * 4;
}

// Offset (doubles) of D element (row r, stage column k) in a TU x TK tile.  The
// 16-byte slot c = 4*(k/8) + k%4 holds columns k and k+4 of an 8-column group,
// i.e. the (a0, a2) or (a1, a3) pair of one m16n8k8 A fragment, and the slots
// of each 128-byte row are XOR-swizzled by swz_key(r): a fragment load's
// phases of 8 lanes (rows 2p, 2p+1, slots c0..c0+3) meet 8 distinct slots.
__device__ __forceinline__ int d_off(int r, int k) {
  const int slot = ((k >> 3) << 2) | (k & 3);
  return r * TK + ((slot ^ swz_key(r)) << 1) + ((k >> 2) & 1);
}

__device__ __forceinline__ void tma_gather4(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                            int r0, int r1, int r2, int r3) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(tc::smem_u32(bar)), "r"(x), "r"(r0), "r"(r1),
      "r"(r2), "r"(r3)
      : "memory");
}

// The mbarrier tracks the completion of all cp.async this thread issued before.
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(tc::smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// wait-site codes recorded in g_aodm_error
enum : int { kErrItemEmpty = 0x4101, kErrItemFull, kErrStageEmpty, kErrStageFull, kErrEpilogue,
             kErrTeardown };

// Decoded work item (both roles decode the same one).
struct Item {
  const AodmBatch* B;
  int ns, bg, utile, nb, u0, mu, g0, gw;
  const int* I;
};

template <int NS>
__device__ __forceinline__ Item decode(const AodmArgs& p, int4 w, int set0) {
  Item t;
  t.B = p.batches ? &p.batches[w.x] : &p.one;
  t.ns = min(NS, t.B->nset - set0);
  t.bg = w.y;
  t.utile = w.z;
  const int b = t.bg / p.gsub, gt = t.bg % p.gsub;
  t.nb = t.B->counts[b];
  t.I = t.B->lists + size_t(b) * p.nao;
  t.u0 = t.utile * TU;
  t.mu = min(TU, t.nb - t.u0);
  t.g0 = b * p.blk + gt * TG;
  t.gw = min(min((b + 1) * p.blk, t.B->ngrid), t.g0 + TG) - t.g0;
  return t;
}

// Weight of D[u0 + r][u0 + c] in the diagonal tile of the symmetric mode.
__device__ __forceinline__ double sym_factor(int r, int c) {
  return c < r ? 0.0 : (c == r ? 0.5 : 1.0);
}

// Bounded wait whose outcome is the same for every lane of the warp.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity, int* err, int code,
                                          uint64_t lim) {
  const bool ok = tc::mbar_wait(bar, parity, err, code, false, lim);
  return __all_sync(0xffffffffu, ok);
}
}  // namespace pipe

template <int NS>
__global__ void __launch_bounds__(pipe::PTHREADS, 1)
aodm_fp64_pipe_kernel(const __grid_constant__ AodmArgs p,
                      const __grid_constant__ CUtensorMap rhs_map) {
  using namespace pipe;
  constexpr int SB = stage_bytes<NS>();
  extern __shared__ uint8_t pipe_smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(pipe_smem_raw) + 1023) &
                                           ~uintptr_t(1023));
  double* red = reinterpret_cast<double*>(sm + PSTAGES * SB);  // [2][NS][2][TG]
  uint64_t* full = reinterpret_cast<uint64_t*>(red + red_doubles<NS>());
  uint64_t* empty = full + PSTAGES;
  uint64_t* ifull = empty + PSTAGES;
  uint64_t* iempty = ifull + RING;
  uint64_t* epi = iempty + RING;  // [2]
  int* ring = reinterpret_cast<int*>(epi + 2);
  int* err = &g_aodm_error;
  const uint64_t lim = p.wait_ns ? p.wait_ns : tc::kWaitLimitNs;

  const int tid = threadIdx.x, lane = tid & 31;
  const int set0 = blockIdx.y * NS;
  const int total = p.counters[p.ngroups];
  int* counter = p.counters + blockIdx.y;
  const bool sym = p.asym != nullptr && *p.asym == 0;

  if (tid == 0) {
    for (int s = 0; s < PSTAGES; ++s) {
      tc::mbar_init(&full[s], NPROD + 1);     // NPROD cp.async arrivals + the TMA's expect_tx
      tc::mbar_init(&empty[s], NCONS / 32);   // one per consumer warp
    }
    for (int r = 0; r < RING; ++r) {
      tc::mbar_init(&ifull[r], 1);
      tc::mbar_init(&iempty[r], PTHREADS / 32);  // every warp reads every item
    }
    for (int e = 0; e < 2; ++e) tc::mbar_init(&epi[e], NCONS);
    tc::mbar_fence_init();
  }
  __syncthreads();

  if (tid < NPROD) {
    // ------------------------------- producers -------------------------------
    const int kcol = tid & (TK - 1);  // stage column gathered by this thread
    const int r0 = tid / TK;          // rows r0 + RSTEP i
    uint32_t fill = 0;                // stage fills issued so far
    for (int n = 0;; ++n) {
      const int slot = n % RING;
      if (tid == 0) {  // fetch the next item for every warp of the CTA
        int it = total;
        if (*reinterpret_cast<volatile int*>(err) == 0 &&
            (n < RING ||
             tc::mbar_wait(&iempty[slot], ((n / RING) - 1) & 1, err, kErrItemEmpty, false, lim)))
          it = min(atomicAdd(counter, 1), total);
        ring[slot] = it;
        tc::mbar_arrive(&ifull[slot]);
      }
      int it = total;
      if (warp_wait(&ifull[slot], (n / RING) & 1, err, kErrItemFull, lim)) it = ring[slot];
      it = __shfl_sync(0xffffffffu, it, 0);
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&iempty[slot]);
      if (it >= total) break;
      const int4 w = p.items[it];
      const Item t = decode<NS>(p, w, set0);
      const CUtensorMap* map = p.batches ? &p.rhs_maps[w.x] : &rhs_map;
      int prow[ROWS_PER_THREAD];  // AO of each gathered row, -1 past the item's rows
#pragma unroll
      for (int i = 0; i < ROWS_PER_THREAD; ++i) {
        const int r = r0 + RSTEP * i;
        prow[i] = r < t.mu ? t.I[t.u0 + r] : -1;
      }
      const int kchunks = (t.nb + TK - 1) / TK;
      const int kc0 = sym ? t.u0 / TK : 0;  // symmetric D: from the tile's own columns on
      // the compacted column index of the next stage is loaded one stage ahead,
      // so the gather addresses never wait for it
      int vnext = t.I[min(kc0 * TK + kcol, t.nb - 1)];
      for (int kc = kc0; kc < kchunks; ++kc, ++fill) {
        const int k = kc * TK + kcol;
        const bool kv = k < t.nb;
        const int v = vnext;  // t.I[min(k, nb - 1)]: the last active AO stands in past the end
        vnext = t.I[min(k + TK, t.nb - 1)];
        const int stage = fill % PSTAGES;
        if (fill >= PSTAGES &&
            !warp_wait(&empty[stage], ((fill / PSTAGES) - 1) & 1, err, kErrStageEmpty, lim)) {
          // nothing is issued for this fill: no asynchronous arrival may be
          // left pending on a barrier that no one waits for when the CTA exits
          break;
        }
        uint8_t* st = sm + stage * SB;
        const double* dm0 = p.dms + size_t(set0) * p.dm_stride + v;
#pragma unroll
        for (int i = 0; i < ROWS_PER_THREAD; ++i) {
          const bool valid = kv && prow[i] >= 0;
          const double* src = valid ? dm0 + size_t(prow[i]) * p.stride_ao : p.dms;
          double* dst = reinterpret_cast<double*>(st) + d_off(r0 + RSTEP * i, kcol);
#pragma unroll 1
          for (int s = 0; s < t.ns; ++s)
            cp_async_8(dst + s * (D_BYTES / 8), valid ? src + s * p.dm_stride : src, valid);
        }
        uint8_t* phi = st + NS * D_BYTES;
        if (!t.B->rhs_tma) {
          // ao_rhs rows [TK][TG] by cp.async: lanes along points; the row of
          // stage column j comes from lane j of this warp (kcol = lane & 15)
          const int pt = tid & (TG - 1);
          const bool pv = t.g0 + pt < t.B->ngrid;
#pragma unroll
          for (int i = 0; i < TK / (NPROD / TG); ++i) {
            const int j = (tid / TG) + (NPROD / TG) * i;
            const int row = __shfl_sync(0xffffffffu, v, j);
            cp_async_8(reinterpret_cast<double*>(phi) + j * TG + pt,
                       pv ? t.B->ao_rhs + size_t(row) * t.B->stride_grid + t.g0 + pt
                          : t.B->ao_rhs,
                       pv);
          }
        }
        cp_async_arrive_noinc(&full[stage]);
        // test hook: the first stage's last arrival (the TMA's expect_tx, or
        // its stand-in) is never made, so the consumers' bounded wait runs out
        const bool withhold = p.inject && fill == 0;
        if (t.B->rhs_tma) {
          if (tid < 32 && !withhold) {
            // ao_rhs rows of the stage columns, from the lanes that gather them
            // (lane j of warp 0 holds column j; D is zero past the list's end)
            int rows[TK];
#pragma unroll
            for (int j = 0; j < TK; ++j) rows[j] = __shfl_sync(0xffffffffu, v, j);
            if (tid == 0) {
              tc::mbar_arrive_expect_tx(&full[stage], PHI_BYTES);
#pragma unroll
              for (int j = 0; j < TK / 4; ++j)
                tma_gather4(phi + j * 4 * TG * 8, map, &full[stage], t.g0, rows[4 * j],
                            rows[4 * j + 1], rows[4 * j + 2], rows[4 * j + 3]);
            }
          }
        } else if (tid == 0 && !withhold) {
          tc::mbar_arrive(&full[stage]);  // the arrival the TMA's expect_tx makes otherwise
        }
      }
    }
    cp_async_wait_all();
    if (tid == 0) {
      // let every TMA this thread issued land before the CTA exits
      for (uint32_t f = fill > PSTAGES ? fill - PSTAGES : 0; f < fill; ++f)
        tc::mbar_wait(&full[f % PSTAGES], (f / PSTAGES) & 1, err, kErrTeardown, true, lim);
    }
  } else {
    // ------------------------------- consumers -------------------------------
    const int ct = tid - NPROD;
    const int warp = ct >> 5;
    const int wm = warp / CWN, wn = warp % CWN;  // warp tile: rows wm*16*MT.., points wn*8*NT..
    const int g = lane >> 2, q = lane & 3;
    uint32_t use = 0;
    for (int n = 0;; ++n) {
      const int slot = n % RING;
      int it = total;
      if (warp_wait(&ifull[slot], (n / RING) & 1, err, kErrItemFull, lim)) it = ring[slot];
      it = __shfl_sync(0xffffffffu, it, 0);
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&iempty[slot]);
      if (it >= total) break;
      const Item t = decode<NS>(p, p.items[it], set0);

      // the phi_lhs rows of this thread's epilogue (rows wm*16*MT + mt*16 + g + 8h,
      // points wn*8*NT + nt*8 + 2q + e) are brought into L2 now, so that the
      // epilogue's loads hit while the tensor pipe waits for them
      int urow[MT][2];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wm * 16 * MT + mt * 16 + g + 8 * h;
          urow[mt][h] = r < t.mu ? t.I[t.u0 + r] : -1;
          if (urow[mt][h] >= 0)
#pragma unroll
            for (int nt = 0; nt < NT; nt += 2)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(
                  t.B->ao_lhs + size_t(urow[mt][h]) * t.B->stride_grid + t.g0 + wn * 8 * NT +
                  nt * 8));
        }

      double acc[NS][MT][NT][4];
#pragma unroll
      for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[s][i][j][e] = 0.0;

      const int kchunks = (t.nb + TK - 1) / TK;
      const int kc0 = sym ? t.u0 / TK : 0;
      bool ok = true;
      for (int kc = kc0; kc < kchunks; ++kc, ++use) {
        const int stage = use % PSTAGES;
        if (!warp_wait(&full[stage], (use / PSTAGES) & 1, err, kErrStageFull, lim)) {
          ok = false;
          break;
        }
        const uint8_t* st = sm + stage * SB;
        const double* phi = reinterpret_cast<const double*>(st + NS * D_BYTES);
        // symmetric D, diagonal tile: D' = strict upper triangle + half diagonal
        const bool diag = sym && kc < kc0 + TU / TK;
#pragma unroll
        for (int kk = 0; kk < TK; kk += 8) {
          double b0[NT], b1[NT];
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            const int col = wn * 8 * NT + nt * 8 + g;
            b0[nt] = phi[(kk + q) * TG + col];
            b1[nt] = phi[(kk + q + 4) * TG + col];
          }
          const int slot8 = ((kk >> 3) << 2) | q;
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            const double* Ds = reinterpret_cast<const double*>(st + s * D_BYTES);
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
              const int r = wm * 16 * MT + mt * 16 + g;
              double2 lo =
                  *reinterpret_cast<const double2*>(Ds + r * TK + ((slot8 ^ swz_key(r)) << 1));
              double2 hi = *reinterpret_cast<const double2*>(
                  Ds + (r + 8) * TK + ((slot8 ^ swz_key(r + 8)) << 1));
              if (diag) {
                const int c = (kc - kc0) * TK + kk + q;  // column within the diagonal tile
                lo.x *= sym_factor(r, c);
                lo.y *= sym_factor(r, c + 4);
                hi.x *= sym_factor(r + 8, c);
                hi.y *= sym_factor(r + 8, c + 4);
              }
#pragma unroll
              for (int nt = 0; nt < NT; ++nt)
                dmma_16x8x8(acc[s][mt][nt], lo.x, hi.x, lo.y, hi.y, b0[nt], b1[nt]);
            }
          }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[stage]);
      }
      if (!ok) break;

      // rho_part[s][j] = sum_r phi_lhs[I[u0+r]][g0+j] * X[s][r][j]: rows reduced
      // in registers and shuffles, the CWM row groups (wm) through `red`
      double lhs[MT][2][NT][2];  // [mt][h][nt][e]
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double* row =
              urow[mt][h] >= 0 ? t.B->ao_lhs + size_t(urow[mt][h]) * t.B->stride_grid : nullptr;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int j = wn * 8 * NT + nt * 8 + 2 * q + e;
              lhs[mt][h][nt][e] = (row && j < t.gw) ? row[t.g0 + j] : 0.0;
            }
        }
      double* rb = red + (n & 1) * (NS * CWM * TG);
#pragma unroll
      for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            double v = 0.0;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
              for (int h = 0; h < 2; ++h)
                v = fma(acc[s][mt][nt][2 * h + e], lhs[mt][h][nt][e], v);
            v += __shfl_xor_sync(0xffffffffu, v, 4);
            v += __shfl_xor_sync(0xffffffffu, v, 8);
            v += __shfl_xor_sync(0xffffffffu, v, 16);
            if (g == 0) rb[(s * CWM + wm) * TG + wn * 8 * NT + nt * 8 + 2 * q + e] = v;
          }
      tc::mbar_arrive(&epi[n & 1]);
      // The buffer is written again two items later, after every consumer has
      // passed the next item's epilogue barrier, i.e. finished reading this one.
      if (!warp_wait(&epi[n & 1], (n >> 1) & 1, err, kErrEpilogue, lim)) break;
      const size_t pslot = t.B->partial_off + size_t(t.bg) * p.max_utiles + t.utile;
      for (int i = ct; i < t.ns * TG; i += NCONS) {
        const int s = i / TG, j = i % TG;
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < CWM; ++w) v += rb[(s * CWM + w) * TG + j];
        p.partial[(pslot * p.nset_max + set0 + s) * TG + j] = sym ? 2.0 * v : v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// 4. deterministic reduction of the row-tile partials into rho
//    one CTA per (batch, block tile): rpairs[i] = (batch, bg), or bg = i
// ---------------------------------------------------------------------------
__global__ void aodm_reduce(AodmArgs p, const int2* __restrict__ rpairs, int npairs) {
  const int i = blockIdx.x;
  if (i >= npairs) return;
  const int2 pr = rpairs ? rpairs[i] : make_int2(0, i);
  const AodmBatch& B = p.batches ? p.batches[pr.x] : p.one;
  const int bg = pr.y;
  const int b = bg / p.gsub, gt = bg % p.gsub;
  const int nt = (B.counts[b] + TU - 1) / TU;
  if (nt == 0) return;  // fully masked block: rho untouched, as in the reference
  const int g0 = b * p.blk + gt * TG;
  const int gend = min(min((b + 1) * p.blk, B.ngrid), g0 + TG);
  for (int t = threadIdx.x; t < B.nset * TG; t += blockDim.x) {
    const int s = t / TG, j = t % TG;
    if (g0 + j >= gend) continue;
    double v = 0.0;
    for (int u = 0; u < nt; ++u)
      v += p.partial[((B.partial_off + size_t(bg) * p.max_utiles + u) * p.nset_max + s) * TG + j];
    double* r = B.rhos + size_t(s) * B.stride_grid + g0 + j;
    *r = v + *r;
  }
}

__global__ void aodm_reset_counters(int* counters, int ngroups) {
  if (threadIdx.x < ngroups) counters[threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    counters[ngroups + 1] = 0;  // asymmetry flag (counters[ngroups] holds the item total)
    g_aodm_error = 0;
  }
}

// *asym = 1 if some D_s differs from its transpose.  Block (bx, by, s) with
// by <= bx compares the 32 x 32 tile (by, bx) with the transpose of (bx, by).
__global__ void __launch_bounds__(256)
aodm_sym_check(const double* __restrict__ dms, size_t stride_ao, size_t dm_stride, int nao,
               int* asym) {
  const int bx = blockIdx.x, by = blockIdx.y;
  if (by > bx) return;
  __shared__ double tile[32][33];
  const double* d = dms + size_t(blockIdx.z) * dm_stride;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  // both tiles are requested before the barrier: tile (by, bx) into shared
  // memory, this thread's elements of tile (bx, by) into registers
  double mine[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int i = ty + 8 * k;
    const int r = by * 32 + i, c = bx * 32 + tx;
    tile[i][tx] = (r < nao && c < nao) ? d[size_t(r) * stride_ao + c] : 0.0;
    const int r2 = bx * 32 + i, c2 = by * 32 + tx;
    mine[k] = (r2 < nao && c2 < nao) ? d[size_t(r2) * stride_ao + c2] : 0.0;
  }
  __syncthreads();
  bool bad = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int i = ty + 8 * k;
    const int r2 = bx * 32 + i, c2 = by * 32 + tx;
    if (r2 < nao && c2 < nao) bad |= !(mine[k] == tile[tx][i]);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(asym, 1);
}

template <int NS, int TKT>
cudaError_t launch_main_t(const AodmArgs& a, cudaStream_t stream, bool attrs_only) {
  constexpr size_t smem = size_t(STAGES) * (NS * TU * TKT + TG * TKT) * sizeof(double) +
                          size_t(LIST_CAP) * sizeof(int);
  static_assert(NS * 2 * TG <= STAGES * (NS * TU * TKT + TG * TKT), "reduction buffer fits");
  static_assert(smem <= 227 * 1024, "shared memory budget");
  cudaError_t err = cudaFuncSetAttribute(aodm_fp64_kernel<NS, TKT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (err != cudaSuccess || attrs_only) return err;
  int dev = 0, nsm = 0;
  if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
  if ((err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return err;
  aodm_fp64_kernel<NS, TKT><<<dim3(nsm, a.ngroups), THREADS, smem, stream>>>(a);
  return cudaGetLastError();
}

template <int NS>
cudaError_t launch_pipe_t(const AodmArgs& a, const CUtensorMap& map, cudaStream_t stream,
                          bool attrs_only) {
  constexpr size_t smem = pipe::smem_bytes<NS>();
  static_assert(smem <= 227 * 1024, "shared memory budget");
  cudaError_t err = cudaFuncSetAttribute(aodm_fp64_pipe_kernel<NS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (err != cudaSuccess || attrs_only) return err;
  int dev = 0, nsm = 0;
  if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
  if ((err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return err;
  aodm_fp64_pipe_kernel<NS><<<dim3(nsm, a.ngroups), pipe::PTHREADS, smem, stream>>>(a, map);
  return cudaGetLastError();
}

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
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

// The pipelined form is used unless CFGMM_AODM_PIPE=0.
bool pipe_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("CFGMM_AODM_PIPE");
    return !(e && e[0] == '0');
  }();
  return on;
}

}  // namespace

bool aodm_pipe_enabled() { return pipe_enabled(); }

bool aodm_rhs_map(CUtensorMap* map, const double* ao_rhs, size_t stride_grid, int nao, int ngrid,
                  int blk) {
  // TMA: 16-byte aligned base and row pitch; the x coordinate of every load
  // (a 64-point tile start b*blk + 64*gt) must be even, so blk must be even.
  if (nao <= 0 || ngrid <= 0 || blk % 2 != 0 ||
      reinterpret_cast<uintptr_t>(ao_rhs) % 16 != 0 || (stride_grid * sizeof(double)) % 16 != 0)
    return false;
  auto enc = encode_tiled();
  if (!enc) return false;
  cuuint64_t dims[2] = {cuuint64_t(ngrid), cuuint64_t(nao)};
  cuuint64_t strides[1] = {cuuint64_t(stride_grid) * sizeof(double)};
  cuuint32_t box[2] = {cuuint32_t(TG), 1};  // gather4: one row per box, four rows per load
  cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(ao_rhs), dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t aodm_launch_pipe(const AodmArgs& a, int ns, const CUtensorMap& map,
                             cudaStream_t stream, bool attrs_only) {
  if (ns == 1) return launch_pipe_t<1>(a, map, stream, attrs_only);
  if (ns == 2) return launch_pipe_t<2>(a, map, stream, attrs_only);
  if (ns == 3) return launch_pipe_t<3>(a, map, stream, attrs_only);
  return cudaErrorInvalidValue;
}

bool aodm_sym_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("CFGMM_AODM_SYM");
    return !(e && e[0] == '0');
  }();
  return on;
}

cudaError_t aodm_launch_sym_check(const double* dms, size_t stride_ao, int nao, int nset,
                                  int* asym, cudaStream_t stream) {
  if (nao <= 0 || nset <= 0) return cudaSuccess;
  const unsigned nt = unsigned((nao + 31) / 32);
  aodm_sym_check<<<dim3(nt, nt, unsigned(nset)), 256, 0, stream>>>(dms, stride_ao,
                                                                  stride_ao * stride_ao, nao, asym);
  return cudaGetLastError();
}

cudaError_t aodm_read_error(int* code) {
  return cudaMemcpyFromSymbol(code, g_aodm_error, sizeof(int));
}

cudaError_t aodm_reset_error(cudaStream_t stream) {
  static const int zero = 0;
  return cudaMemcpyToSymbolAsync(g_aodm_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice,
                                 stream);
}

namespace {
struct WaitInjection {
  bool armed[2] = {false, false};
  unsigned long long ns = 0;
};
thread_local WaitInjection g_wait_injection;
}  // namespace

void arm_wait_injection(int kind, unsigned long long wait_ns) {
  if (kind < 0 || kind > 1) return;
  g_wait_injection.armed[kind] = true;
  g_wait_injection.ns = wait_ns;
}

bool take_wait_injection(int kind, unsigned long long* wait_ns) {
  if (kind < 0 || kind > 1 || !g_wait_injection.armed[kind]) return false;
  g_wait_injection.armed[kind] = false;
  *wait_ns = g_wait_injection.ns;
  return true;
}

int aodm_groups(const AodmConfig& cfg, int nset_max) {
  return (nset_max + cfg.ns - 1) / cfg.ns;
}

AodmConfig aodm_default_config(int nset) {
  return AodmConfig{nset >= 3 ? 3 : nset, 32};
}

cudaError_t aodm_launch_main(const AodmArgs& a, const AodmConfig& cfg, cudaStream_t stream,
                             bool attrs_only) {
  if (cfg.tk == 0) {  // pipelined form over the batches' maps
    if (!a.batches || !a.rhs_maps) return cudaErrorInvalidValue;
    return aodm_launch_pipe(a, cfg.ns, CUtensorMap{}, stream, attrs_only);
  }
  if (cfg.tk == 32) {
    if (cfg.ns == 1) return launch_main_t<1, 32>(a, stream, attrs_only);
    if (cfg.ns == 2) return launch_main_t<2, 32>(a, stream, attrs_only);
    if (cfg.ns == 3) return launch_main_t<3, 32>(a, stream, attrs_only);
  } else if (cfg.tk == 16) {
    if (cfg.ns == 1) return launch_main_t<1, 16>(a, stream, attrs_only);
    if (cfg.ns == 2) return launch_main_t<2, 16>(a, stream, attrs_only);
    if (cfg.ns == 3) return launch_main_t<3, 16>(a, stream, attrs_only);
  }
  return cudaErrorInvalidValue;
}

cudaError_t aodm_launch_reduce(const AodmArgs& a, const int2* rpairs, int npairs,
                               cudaStream_t stream) {
  if (npairs <= 0) return cudaSuccess;
  aodm_reduce<<<npairs, 128, 0, stream>>>(a, rpairs, npairs);
  return cudaGetLastError();
}

cudaError_t aodm_launch_reset(int* counters, int ngroups, cudaStream_t stream) {
  aodm_reset_counters<<<1, 32, 0, stream>>>(counters, ngroups);
  return cudaGetLastError();
}

namespace {
struct Layout {
  size_t lists, counts, items, counters, partial, total;
};

Layout layout(size_t nao, size_t ngrid, size_t nset, size_t blk) {
  const size_t nblk = (ngrid + blk - 1) / blk;
  const size_t gsub = (blk + TG - 1) / TG;
  const size_t max_utiles = (nao + TU - 1) / TU;
  const size_t ngroups = nset;  // upper bound for any set grouping
  auto a256 = [](size_t v) { return (v + 255) / 256 * 256; };
  Layout L;
  L.lists = 0;
  L.counts = L.lists + a256(nblk * nao * sizeof(int));
  L.items = L.counts + a256(nblk * sizeof(int));
  L.counters = L.items + a256(nblk * gsub * max_utiles * sizeof(int4));
  L.partial = L.counters + a256((ngroups + 2) * sizeof(int));  // + item total, asymmetry flag
  L.total = L.partial + nblk * gsub * max_utiles * nset * TG * sizeof(double);
  return L;
}
}  // namespace

cudaError_t aodm_build_items_launch(const int* counts, int nblk, int gsub, int4* items,
                                    int* counters, int ncounters, cudaStream_t stream) {
  aodm_build_items<<<1, 1024, 0, stream>>>(counts, nblk, gsub, items, counters, ncounters);
  return cudaGetLastError();
}

cudaError_t aodm_block_lists_launch(const uint8_t* tab, size_t ldtab, int nao, int nblk,
                                    int* lists, int* counts, cudaStream_t stream) {
  aodm_block_lists<<<nblk, 256, 0, stream>>>(tab, ldtab, nao, nblk, lists, counts);
  return cudaGetLastError();
}

int aodm_row_tile() { return TU; }
int aodm_point_tile() { return TG; }

size_t aodmao2rho_fp64_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk) {
  return layout(nao, ngrid, nset, blk).total;
}

cudaError_t aodmao2rho_fp64(double* rhos, const double* dms, const double* ao_lhs,
                            const double* ao_rhs, size_t stride_ao, size_t stride_grid, int nao,
                            int ngrid, int nset, const uint8_t* tab, size_t ldtab, int blk,
                            void* workspace, cudaStream_t stream) {
  if (nao <= 0 || ngrid <= 0 || nset <= 0) return cudaSuccess;
  const int nblk = (ngrid + blk - 1) / blk;
  const int gsub = (blk + TG - 1) / TG;
  const int max_utiles = (nao + TU - 1) / TU;
  const AodmConfig cfg = aodm_default_config(nset);
  const int ngroups = aodm_groups(cfg, nset);
  const Layout L = layout(nao, ngrid, nset, blk);
  char* ws = static_cast<char*>(workspace);
  int* lists = reinterpret_cast<int*>(ws + L.lists);
  int* counts = reinterpret_cast<int*>(ws + L.counts);
  int4* items = reinterpret_cast<int4*>(ws + L.items);
  int* counters = reinterpret_cast<int*>(ws + L.counters);
  double* partial = reinterpret_cast<double*>(ws + L.partial);

  aodm_block_lists<<<nblk, 256, 0, stream>>>(tab, ldtab, nao, nblk, lists, counts);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  aodm_build_items<<<1, 1024, 0, stream>>>(counts, nblk, gsub, items, counters, ngroups);
  if ((err = cudaGetLastError()) != cudaSuccess) return err;

  AodmArgs a{};
  a.dms = dms;
  a.stride_ao = stride_ao;
  a.dm_stride = stride_ao * stride_ao;
  a.nao = nao;
  a.blk = blk;
  a.gsub = gsub;
  a.max_utiles = max_utiles;
  a.nset_max = nset;
  a.batches = nullptr;
  a.one = AodmBatch{ao_lhs, ao_rhs, rhos, lists, counts, stride_grid, ngrid, nset, 0};
  a.items = items;
  a.counters = counters;
  a.ngroups = ngroups;
  a.partial = partial;
  CUtensorMap map{};
  if (pipe_enabled()) {
    a.one.rhs_tma = aodm_rhs_map(&map, ao_rhs, stride_grid, nao, ngrid, blk) ? 1 : 0;
    // the half contraction needs D = D^T and phi_lhs = phi_rhs (one array)
    if (aodm_sym_enabled() && ao_lhs == ao_rhs) {
      a.asym = counters + ngroups + 1;
      if ((err = aodm_launch_sym_check(dms, stride_ao, nao, nset, counters + ngroups + 1,
                                       stream)) != cudaSuccess)
        return err;
    }
    unsigned long long ns = 0;
    if (take_wait_injection(0, &ns)) {  // cfgmm_test_arm_wait_timeout
      a.inject = 1;
      a.wait_ns = ns;
    }
    err = aodm_launch_pipe(a, cfg.ns, map, stream);
  }
  else
    err = aodm_launch_main(a, cfg, stream);
  if (err != cudaSuccess) return err;
  return aodm_launch_reduce(a, nullptr, nblk * gsub, stream);
}

}  // namespace cfgmm
