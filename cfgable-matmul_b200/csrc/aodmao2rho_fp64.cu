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
//   4. aodm_reduce: adds the per-row-tile partial sums of each grid tile in a
//      fixed order, so results are deterministic run to run (unlike the
//      reference, whose lock order varies).
#include "common.cuh"
#include "aodmao2rho_fp64.cuh"

namespace cfgmm {
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
  if (tid == 0) base_s = 0;
  for (int i = tid; i <= ncounters; i += 1024) counters[i] = 0;  // [ncounters] = total
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

}  // namespace

int aodm_groups(const AodmConfig& cfg, int nset_max) {
  return (nset_max + cfg.ns - 1) / cfg.ns;
}

AodmConfig aodm_default_config(int nset) {
  return AodmConfig{nset >= 3 ? 3 : nset, 32};
}

cudaError_t aodm_launch_main(const AodmArgs& a, const AodmConfig& cfg, cudaStream_t stream,
                             bool attrs_only) {
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
  L.partial = L.counters + a256((ngroups + 1) * sizeof(int));
  L.total = L.partial + nblk * gsub * max_utiles * nset * TG * sizeof(double);
  return L;
}
}  // namespace

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
  if ((err = aodm_launch_main(a, cfg, stream)) != cudaSuccess) return err;
  return aodm_launch_reduce(a, nullptr, nblk * gsub, stream);
}

}  // namespace cfgmm
