// fock.cu -- the Fock-build contraction on the per-block compacted AO lists:
//
//   V_s[u][v] += sum_{g in b} phi_lhs[u][g] w_s[g] phi_rhs[v][g],  u, v in I(b),
//
// the transpose of the AO-DM-AO contraction (aodmao2rho_fp64.cu) on its layouts
// and mask: where that one gathers D[I(b), I(b)] as an input, this one scatters
// V[I(b), I(b)] as an output.  Work item = (block, 64-point tile, 64 rows of the
// active list I(b)) for one weight vector w_s, the same items as the AO-DM-AO
// kernels.  The CTA stages A = phi_lhs[I rows, tile] diag(w_s) once, walks the
// compacted columns in chunks of 64 (phi_rhs rows by 8-byte cp.async into a
// double buffer), forms the 64 x 64 product over the 64 points on DMMA
// m16n8k8 and adds it into V[I rows][I chunk] with FP64 atomics (red.add): the
// same (u, v) receives one addition per block in which both are active.  Only
// the masked products are formed (a dense product over all AO pairs runs ~10x
// their number on the taxol-size mask).  When phi_lhs and phi_rhs are the same
// array the block's contribution is symmetric in (u, v): row tile a then walks
// the chunks from its own (chunk a) on and adds each product of a later chunk
// to V[u][v] and V[v][u], half the products.  Sums over blocks arrive in
// completion order, so the last bits of V vary from run to run.
#include "common.cuh"
#include "aodmao2rho_fp64.cuh"
#include "fock.cuh"

namespace cfgmm {
namespace {

constexpr int FT = 64;         // rows per item = columns per chunk = points per tile
constexpr int THREADS = 256;   // 8 warps: 4 along rows (16 each) x 2 along columns (32 each)
constexpr int TILE = FT * FT;  // doubles per staged tile

// Offset (doubles) of element (row, point k) of a 64 x 64 tile: the 16-byte slot
// k/2 of a row holds points k and k+1, contiguous in phi, so one 16-byte copy
// fills it; the slots of a row are XOR-swizzled by swz_key(row), so a fragment
// load's phases of 8 lanes meet 8 distinct slots.  A k step of 8 points gives
// the m16n8k8 index j (0..3) the points 2j and 2j+1 as its k = j and k = j + 4,
// on both operands alike: the products summed are the same, and a fragment
// pair (a0, a2) of A (rows = u) or (b0, b1) of B (rows = v) is one 16-byte load.
__device__ __forceinline__ int f_off(int r, int k) {
  return r * FT + (((k >> 1) ^ swz_key(r)) << 1) + (k & 1);
}

// 16-byte asynchronous copy of which the first `bytes` (0, 8 or 16) are read
// from `src`; the rest of the destination is zero-filled.
__device__ __forceinline__ void cp_async_16_n(void* smem_dst, const void* gmem_src, int bytes) {
  const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(gmem_src),
               "r"(bytes)
               : "memory");
}

struct FockArgs {
  double* v;
  size_t stride_ao, v_stride;  // v_stride = stride_ao^2
  const double* w;
  const double* ao_lhs;
  const double* ao_rhs;
  size_t stride_grid;
  const int* lists;  // [nblk][nao]
  const int* counts;
  int nao, ngrid, blk, gsub;
  int sym;  // ao_lhs == ao_rhs: chunks from the row tile's own on, mirrored
  int vec;  // phi rows and w 16-byte aligned at every tile: pairs of points per copy
  const int4* items;
  int* counters;  // [nset] work counters, [nset] = item total
};

__global__ void __launch_bounds__(THREADS, 2)
fock_compact_kernel(const __grid_constant__ FockArgs p) {
  __shared__ __align__(16) double As[TILE];
  extern __shared__ __align__(16) double Bs[];  // [2][TILE]
  __shared__ int item_s;
  const int set = blockIdx.y;
  const int total = p.counters[gridDim.y];
  int* counter = p.counters + set;
  const double* w = p.w + size_t(set) * p.stride_grid;
  double* V = p.v + size_t(set) * p.v_stride;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, q = lane & 3;

  for (;;) {
    if (tid == 0) item_s = atomicAdd(counter, 1);
    __syncthreads();  // also: the previous item's last reads of As / Bs are done
    const int it = item_s;
    if (it >= total) break;
    const int4 wi = p.items[it];
    const int bg = wi.y, a = wi.z;
    const int b = bg / p.gsub, gt = bg % p.gsub;
    const int nb = p.counts[b];
    const int* I = p.lists + size_t(b) * p.nao;
    const int u0 = a * FT;
    const int mu = min(FT, nb - u0);
    const int g0 = b * p.blk + gt * FT;
    const int gw = min(min((b + 1) * p.blk, p.ngrid), g0 + FT) - g0;

    auto issue = [&](int ch) {
      double* B = Bs + (ch & 1) * TILE;
      const int c0 = ch * FT;
      if (p.vec) {
        // one 16-byte copy per pair of points; a pair past ngrid is zero-filled
        // (one of its points, or both)
#pragma unroll
        for (int e = tid; e < TILE / 2; e += THREADS) {
          const int c = e >> 5, k = 2 * (e & 31);
          const int left = p.ngrid - (g0 + k);
          const int bytes = c0 + c < nb ? (left >= 2 ? 16 : (left == 1 ? 8 : 0)) : 0;
          const double* src =
              bytes ? p.ao_rhs + size_t(I[c0 + c]) * p.stride_grid + g0 + k : p.ao_rhs;
          cp_async_16_n(B + f_off(c, k), src, bytes);
        }
      } else {
#pragma unroll 4
        for (int e = tid; e < TILE; e += THREADS) {
          const int c = e >> 6, k = e & 63;
          const bool valid = c0 + c < nb && g0 + k < p.ngrid;
          const double* src =
              valid ? p.ao_rhs + size_t(I[c0 + c]) * p.stride_grid + g0 + k : p.ao_rhs;
          cp_async_8(B + f_off(c, k), src, valid);
        }
      }
      cp_async_commit();
    };
    const int nch = (nb + FT - 1) / FT;
    const int ch0 = p.sym ? a : 0;
    issue(ch0);  // the first chunk's copies fly while A is staged
    // A = phi_lhs[I[u0 + r]][g0 + k] * w[g0 + k], zero past the rows and points
    if (p.vec) {
      // pairs of points (k even): the partner of the tile's last point lies
      // inside the row (stride_grid is even, so ngrid < stride_grid when odd)
#pragma unroll
      for (int e = tid; e < TILE / 2; e += THREADS) {
        const int r = e >> 5, k = 2 * (e & 31);
        double2 x = make_double2(0.0, 0.0);
        if (r < mu && k < gw) {
          const double2 f = *reinterpret_cast<const double2*>(
              p.ao_lhs + size_t(I[u0 + r]) * p.stride_grid + g0 + k);
          const double2 ww = *reinterpret_cast<const double2*>(w + g0 + k);
          x.x = f.x * ww.x;
          if (k + 1 < gw) x.y = f.y * ww.y;
        }
        *reinterpret_cast<double2*>(As + f_off(r, k)) = x;
      }
    } else {
#pragma unroll 4
      for (int e = tid; e < TILE; e += THREADS) {
        const int r = e >> 6, k = e & 63;
        double x = 0.0;
        if (r < mu && k < gw)
          x = p.ao_lhs[size_t(I[u0 + r]) * p.stride_grid + g0 + k] * w[g0 + k];
        As[f_off(r, k)] = x;
      }
    }
    const int r_lo = wm * 16 + g, r_hi = r_lo + 8;
    const int u_lo = r_lo < mu ? I[u0 + r_lo] : -1;
    const int u_hi = r_hi < mu ? I[u0 + r_hi] : -1;
    for (int ch = ch0; ch < nch; ++ch) {
      if (ch + 1 < nch) {
        issue(ch + 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();  // chunk ch (and A) visible to every warp
      const double* B = Bs + (ch & 1) * TILE;
      double acc[4][4];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[nt][e] = 0.0;
#pragma unroll
      for (int kk = 0; kk < FT; kk += 8) {
        const int slot = ((kk >> 3) << 2) | q;
        const double2 lo =
            *reinterpret_cast<const double2*>(As + r_lo * FT + ((slot ^ swz_key(r_lo)) << 1));
        const double2 hi =
            *reinterpret_cast<const double2*>(As + r_hi * FT + ((slot ^ swz_key(r_hi)) << 1));
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int c = wn * 32 + nt * 8 + g;
          const double2 bv =
              *reinterpret_cast<const double2*>(B + c * FT + ((slot ^ swz_key(c)) << 1));
          dmma_16x8x8(acc[nt], lo.x, hi.x, lo.y, hi.y, bv.x, bv.y);
        }
      }
      // V[u][v] += the chunk's products (and V[v][u] past the diagonal tile)
      const int c0 = ch * FT;
      const bool mirror = p.sym && ch != a;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = c0 + wn * 32 + nt * 8 + 2 * q + e;
          if (c >= nb) continue;
          const size_t vcol = size_t(I[c]);
          if (u_lo >= 0) atomicAdd(V + size_t(u_lo) * p.stride_ao + vcol, acc[nt][e]);
          if (u_hi >= 0) atomicAdd(V + size_t(u_hi) * p.stride_ao + vcol, acc[nt][2 + e]);
          if (mirror) {
            if (u_lo >= 0) atomicAdd(V + vcol * p.stride_ao + u_lo, acc[nt][e]);
            if (u_hi >= 0) atomicAdd(V + vcol * p.stride_ao + u_hi, acc[nt][2 + e]);
          }
        }
      __syncthreads();  // chunk ch's buffer is refilled by chunk ch + 2
    }
  }
}

struct FockLayout {
  size_t lists, counts, items, counters, total;
};

FockLayout fock_layout(size_t nao, size_t ngrid, size_t nset, size_t blk) {
  const size_t nblk = (ngrid + blk - 1) / blk;
  const size_t gsub = (blk + FT - 1) / FT;
  const size_t max_ut = (nao + FT - 1) / FT;
  auto a256 = [](size_t x) { return (x + 255) / 256 * 256; };
  FockLayout L;
  L.lists = 0;
  L.counts = L.lists + a256(nblk * nao * sizeof(int));
  L.items = L.counts + a256(nblk * sizeof(int));
  L.counters = L.items + a256(nblk * gsub * max_ut * sizeof(int4));
  L.total = L.counters + a256((nset + 2) * sizeof(int));
  return L;
}

}  // namespace

size_t fock_compact_workspace(size_t nao, size_t ngrid, size_t nset, size_t blk) {
  return fock_layout(nao, ngrid, nset, blk).total;
}

cudaError_t fock_compact_fp64(double* vs, const double* ws, const double* ao_lhs,
                              const double* ao_rhs, size_t stride_ao, size_t stride_grid,
                              int nao, int ngrid, int nset, const uint8_t* tab, size_t ldtab,
                              int blk, void* workspace, cudaStream_t stream) {
  if (nao <= 0 || ngrid <= 0 || nset <= 0) return cudaSuccess;
  // the work items are the AO-DM-AO kernels' 64-row, 64-point tiles
  if (aodm_row_tile() != FT || aodm_point_tile() != FT) return cudaErrorInvalidValue;
  const int nblk = (ngrid + blk - 1) / blk;
  const int gsub = (blk + FT - 1) / FT;
  const FockLayout L = fock_layout(nao, ngrid, nset, blk);
  char* wsp = static_cast<char*>(workspace);
  int* lists = reinterpret_cast<int*>(wsp + L.lists);
  int* counts = reinterpret_cast<int*>(wsp + L.counts);
  int4* items = reinterpret_cast<int4*>(wsp + L.items);
  int* counters = reinterpret_cast<int*>(wsp + L.counters);
  cudaError_t err = aodm_block_lists_launch(tab, ldtab, nao, nblk, lists, counts, stream);
  if (err != cudaSuccess) return err;
  if ((err = aodm_build_items_launch(counts, nblk, gsub, items, counters, nset, stream)) !=
      cudaSuccess)
    return err;
  FockArgs a{};
  a.v = vs;
  a.stride_ao = stride_ao;
  a.v_stride = stride_ao * stride_ao;
  a.w = ws;
  a.ao_lhs = ao_lhs;
  a.ao_rhs = ao_rhs;
  a.stride_grid = stride_grid;
  a.lists = lists;
  a.counts = counts;
  a.nao = nao;
  a.ngrid = ngrid;
  a.blk = blk;
  a.gsub = gsub;
  a.sym = ao_lhs == ao_rhs;
  // 16-byte copies need every tile's first point (b * blk + 64 t) 16-byte
  // aligned in phi and w: an even BLKSIZE and row stride, aligned bases
  auto al16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
  a.vec = blk % 2 == 0 && stride_grid % 2 == 0 && al16(ao_lhs) && al16(ao_rhs) && al16(ws);
  a.items = items;
  a.counters = counters;
  const size_t dyn = 2 * TILE * sizeof(double);
  if ((err = cudaFuncSetAttribute(fock_compact_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn))) !=
      cudaSuccess)
    return err;
  int dev = 0, nsm = 0;
  if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
  if ((err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return err;
  fock_compact_kernel<<<dim3(2 * nsm, nset), THREADS, dyn, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace cfgmm
