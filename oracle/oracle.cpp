// oracle.cpp -- CPU restatement of cfgable-matmul's blocked loops.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (libcfgmm.so, the Python
// package, the C ABI) links, loads or calls this file.  It is used by tests/
// as the parity checker, by __graft_entry__.smoke() as the checker, and by
// bench.py as the timed CPU baseline ("kind": "port").
//
// PARITY UNPINNED: the reference is a Rust crate and this image has no Rust
// toolchain, so no output of the reference itself can be produced here, and the
// reference's tests carry no golden values (they print "Max error" against
// OpenBLAS and assert nothing).  This restatement is therefore checked against
// the comparator the reference's tests use -- a dense FP64 evaluation with
// OpenBLAS (numpy here) -- on the reference tests' own input generators
// (tests/golden/), and against small pure-Python loop restatements.
//
// What is restated, with the reference file:line each part follows (paths are
// relative to the reference crate root):
//   * micro-kernel `c[i][j] += a[p][i] * b[p][j]`              src/structs.rs:34-45
//     The README recommends `-C llvm-args=-fp-contract=fast` (README.md:36),
//     under which LLVM fuses `c += a*b` into one FMA.  std::fma pins that
//     rounding explicitly, so the single-thread result here is the
//     single-thread result of the reference built as its README says.
//   * matmul_loop_1st_mr (per-MR lock, edge copy path)          src/impl_matmul.rs:10-74
//   * pack_b_no_trans / pack_b_trans                            src/impl_matmul.rs:76-117
//   * matmul_loop_2nd_nr_pack_b                                 src/impl_matmul.rs:120-153
//   * matmul_loop_parallel_mnk_pack_a (A pack, m->n->k tasks)   src/impl_matmul.rs:155-231
//   * matmul_anyway_full tuning <f64,252,512,240,14,2,8>        src/impl_matmul.rs:234-248
//   * microkernel_mask_k_for_b (fma_from)                       src/impl_matmul_non0tab.rs:21-41
//   * matmul_loop_1st_mr_mask_k_for_b                           src/impl_matmul_non0tab.rs:53-116
//   * get_indices_from_non0tab                                  src/impl_matmul_non0tab.rs:118-129
//   * pack_b_no_trans_non0tab                                   src/impl_matmul_non0tab.rs:131-161
//   * matmul_loop_2nd_nr_pack_b_non0tab                         src/impl_matmul_non0tab.rs:163-208
//   * matmul_loop_parallel_mnk_pack_a_non0tab                   src/impl_matmul_non0tab.rs:210-306
//   * pack_dm_in_aodmao2rho                                     src/impl_aodmao2rho.rs:10-29
//   * aodmao2rho_loop_1st (microkernel + fused fma reduce)      src/impl_aodmao2rho.rs:31-95
//   * aodmao2rho_loop_2nd (per-block compaction and skip)       src/impl_aodmao2rho.rs:97-169
//   * aodmao2rho_loop_parallel (u->g->v task order)             src/impl_aodmao2rho.rs:171-244
//   * aodmao2rho_anyway tuning, BLKSIZE 48                      src/impl_aodmao2rho.rs:247-261
//   * the Fock-build contraction (V += phi_lhs diag(w) phi_rhs^T over the pairs
//     active in each block), the transpose of aodmao2rho on its layouts and mask;
//     the reference has no such function, so it is written from the formula.
//
// rayon's `into_par_iter` + AtomicUsize task counter become an OpenMP parallel
// loop that draws task ids from a std::atomic counter; the per-tile
// `Mutex<()>` locks become std::mutex.  With nthreads == 1 the task order is
// the reference's issue order and the result is deterministic.  With more
// threads, partial sums meet under the locks in completion order, exactly as in
// the reference (which is not bitwise deterministic either).
//
// Panics of the reference (slice out of bounds, `unimplemented!` for a masked
// transb, `assert!(NC % BLKSIZE == 0)`) become a negative return code.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>
#include <omp.h>

namespace {

constexpr int kOk = 0;
constexpr int kInvalid = -1;
constexpr int kUnsupported = -2;

inline size_t div_ceil(size_t a, size_t b) { return (a + b - 1) / b; }

// Number of worker threads used for a call: 0 means every available thread.
inline int resolve_threads(int nthreads) {
  return nthreads > 0 ? nthreads : omp_get_max_threads();
}

// Runs `ntask` tasks in issue order drawn from one atomic counter, the way the
// reference's par_iter + AtomicUsize::fetch_add does (impl_matmul.rs:207-214).
template <class F>
void run_tasks(size_t ntask, int nthreads, F&& body) {
  std::atomic<size_t> counter{0};
#pragma omp parallel num_threads(nthreads)
  {
    const int tid = omp_get_thread_num();
    for (;;) {
      size_t id = counter.fetch_add(1);
      if (id >= ntask) break;
      body(id, tid);
    }
  }
}

// ---------------------------------------------------------------------------
// MatmulLoops<f64, MC, KC, NC, MR, NR_LANE*LANE>
// ---------------------------------------------------------------------------
template <size_t MC, size_t KC, size_t MR, size_t NR>
struct Loops {
  // one packed [KC][MR] A panel, one packed [KC][NR] B panel
  struct APanel { double v[KC][MR]; };
  struct BPanel { double v[KC][NR]; };

  // structs.rs:34-45 -- c[i][j] += a[p][i] * b[p][j], fused.
  // The tile is accumulated in a local copy that the compiler keeps in vector
  // registers (MR x NR = 14 x 16 doubles: 28 AVX-512 registers), as the
  // reference's register-blocked SIMD kernel does; every element still sees
  // its fused multiply-adds in the order p = 0, 1, ..., kc-1.
  static inline void microkernel(double (&c)[MR][NR], const double (*a)[MR],
                                 const double (*b)[NR], size_t kc) {
    double acc[MR][NR];
#pragma GCC unroll 16
    for (size_t i = 0; i < MR; ++i)
#pragma GCC unroll 16
      for (size_t j = 0; j < NR; ++j) acc[i][j] = c[i][j];
    for (size_t p = 0; p < kc; ++p) {
#pragma GCC unroll 16
      for (size_t i = 0; i < MR; ++i) {
        const double a_ip = a[p][i];
#pragma GCC unroll 16
        for (size_t j = 0; j < NR; ++j) acc[i][j] = std::fma(a_ip, b[p][j], acc[i][j]);
      }
    }
#pragma GCC unroll 16
    for (size_t i = 0; i < MR; ++i)
#pragma GCC unroll 16
      for (size_t j = 0; j < NR; ++j) c[i][j] = acc[i][j];
  }

  // impl_matmul_non0tab.rs:21-41 -- a indexed by the compacted k list.
  static inline void microkernel_mask_k_for_b(double (&c)[MR][NR], const double (*a)[MR],
                                              const double (*b)[NR], const size_t* idx,
                                              size_t count) {
    double acc[MR][NR];  // in registers, as in microkernel
#pragma GCC unroll 16
    for (size_t i = 0; i < MR; ++i)
#pragma GCC unroll 16
      for (size_t j = 0; j < NR; ++j) acc[i][j] = c[i][j];
    for (size_t ip = 0; ip < count; ++ip) {
      const size_t p = idx[ip];
#pragma GCC unroll 16
      for (size_t i = 0; i < MR; ++i) {
        const double a_ip = a[p][i];
#pragma GCC unroll 16
        for (size_t j = 0; j < NR; ++j) acc[i][j] = std::fma(a_ip, b[ip][j], acc[i][j]);
      }
    }
#pragma GCC unroll 16
    for (size_t i = 0; i < MR; ++i)
#pragma GCC unroll 16
      for (size_t j = 0; j < NR; ++j) c[i][j] = acc[i][j];
  }

  // impl_matmul.rs:10-74 (and impl_matmul_non0tab.rs:53-116 when idx != null).
  static void loop_1st_mr(double* c, const APanel* a, const BPanel& b, size_t mc, size_t nr,
                          size_t kc, size_t ldc, std::mutex* barrier, const size_t* idx,
                          size_t count) {
    for (size_t i = 0, task_i = 0; i < mc; i += MR, ++task_i) {
      std::lock_guard<std::mutex> lock(barrier[task_i]);
      const size_t mr = (i + MR <= mc) ? MR : mc - i;
      double c_reg[MR][NR];
      std::memset(c_reg, 0, sizeof(c_reg));
      for (size_t ii = 0; ii < mr; ++ii)
        for (size_t jj = 0; jj < nr; ++jj) c_reg[ii][jj] = c[(i + ii) * ldc + jj];
      if (idx)
        microkernel_mask_k_for_b(c_reg, a[task_i].v, b.v, idx, count);
      else
        microkernel(c_reg, a[task_i].v, b.v, kc);
      for (size_t ii = 0; ii < mr; ++ii)
        for (size_t jj = 0; jj < nr; ++jj) c[(i + ii) * ldc + jj] = c_reg[ii][jj];
    }
  }

  // impl_matmul.rs:76-98
  static void pack_b_no_trans(BPanel& dst, const double* src, size_t kc, size_t nr, size_t ldb) {
    for (size_t p = 0; p < kc; ++p)
      for (size_t j = 0; j < nr; ++j) dst.v[p][j] = src[p * ldb + j];
  }

  // impl_matmul.rs:100-117 (the copy through a KC x NR buffer is folded away:
  // it moves the same values).
  static void pack_b_trans(BPanel& dst, const double* src, size_t kc, size_t nr, size_t ldb) {
    for (size_t j = 0; j < nr; ++j)
      for (size_t p = 0; p < kc; ++p) dst.v[p][j] = src[j * ldb + p];
  }

  // impl_matmul_non0tab.rs:118-129
  static size_t get_indices(const uint8_t* tab, size_t ldtab, size_t k, size_t* out) {
    size_t count = 0;
    for (size_t p = 0; p < k; ++p)
      if (tab[p * ldtab]) out[count++] = p;
    return count;
  }

  // impl_matmul_non0tab.rs:131-161
  static void pack_b_no_trans_non0tab(BPanel& dst, const double* src, size_t nr, size_t ldb,
                                      const size_t* idx, size_t count) {
    for (size_t ip = 0; ip < count; ++ip)
      for (size_t j = 0; j < nr; ++j) dst.v[ip][j] = src[idx[ip] * ldb + j];
  }

  static void pack_a(std::vector<APanel>& a_pack, const double* a, size_t m, size_t k,
                     size_t lda, bool transa, int nthreads) {
    const size_t ntask_mc = div_ceil(m, MC), ntask_kc = div_ceil(k, KC);
    const size_t ntask_mr = div_ceil(MC, MR);
    // impl_matmul.rs:184-205
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (size_t task_id = 0; task_id < ntask_mc * ntask_kc; ++task_id) {
      const size_t task_mc = task_id / ntask_kc, task_kc = task_id % ntask_kc;
      const size_t idx_m = task_mc * MC, idx_k = task_kc * KC;
      const size_t mc = ((task_mc + 1) * MC <= m) ? MC : m - idx_m;
      const size_t kc = ((task_kc + 1) * KC <= k) ? KC : k - idx_k;
      for (size_t task_mr = 0; task_mr < div_ceil(mc, MR); ++task_mr) {
        const size_t idx_mr = task_mr * MR;
        APanel& dst = a_pack[task_mc * (ntask_kc * ntask_mr) + task_kc * ntask_mr + task_mr];
        const size_t mr = ((task_mr + 1) * MR <= mc) ? MR : mc - idx_mr;
        for (size_t p = 0; p < kc; ++p)
          for (size_t i = 0; i < mr; ++i)
            dst.v[p][i] = transa ? a[(idx_k + p) * lda + (idx_m + idx_mr + i)]
                               : a[(idx_m + idx_mr + i) * lda + (idx_k + p)];
      }
    }
  }

  // impl_matmul.rs:155-231 (tab == null) and impl_matmul_non0tab.rs:210-306.
  static void matmul(double* c, const double* a, const double* b, size_t m, size_t n, size_t k,
                     size_t lda, size_t ldb, size_t ldc, bool transa, bool transb, size_t NC,
                     const uint8_t* tab, size_t ldtab, size_t blk, int nthreads) {
    const size_t ntask_mc = div_ceil(m, MC), ntask_nc = div_ceil(n, NC), ntask_kc = div_ceil(k, KC);
    const size_t ntask_mr = div_ceil(MC, MR), ntask_nr = div_ceil(NC, NR);
    if (ntask_mc * ntask_nc * ntask_kc == 0) return;
    std::unique_ptr<std::mutex[]> c_barrier(new std::mutex[ntask_mc * ntask_nc * ntask_nr * ntask_mr]);
    std::vector<APanel> a_pack(ntask_mc * ntask_kc * ntask_mr);
    std::memset(a_pack.data(), 0, a_pack.size() * sizeof(APanel));
    pack_a(a_pack, a, m, k, lda, transa, nthreads);

    run_tasks(ntask_mc * ntask_nc * ntask_kc, nthreads, [&](size_t task_id, int) {
      const size_t task_m = task_id % ntask_mc;
      const size_t task_n = (task_id / ntask_mc) % ntask_nc;
      const size_t task_k = task_id / (ntask_mc * ntask_nc);
      const double* bt = transb ? b + task_n * NC * ldb + task_k * KC
                                : b + task_k * KC * ldb + task_n * NC;
      const size_t mc = ((task_m + 1) * MC <= m) ? MC : m - task_m * MC;
      const size_t nc = ((task_n + 1) * NC <= n) ? NC : n - task_n * NC;
      const size_t kc = ((task_k + 1) * KC <= k) ? KC : k - task_k * KC;
      const APanel* ap = a_pack.data() + task_m * (ntask_kc * ntask_mr) + task_k * ntask_mr;
      std::mutex* barrier = c_barrier.get() + (task_m * ntask_nc + task_n) * (ntask_nr * ntask_mr);
      double* cc = c + task_m * MC * ldc + task_n * NC;

      // loop_2nd: impl_matmul.rs:120-153 / impl_matmul_non0tab.rs:163-208
      std::unique_ptr<BPanel> buf_b(new BPanel);
      std::memset(buf_b.get(), 0, sizeof(BPanel));
      size_t idx[KC];
      for (size_t j = 0, task_j = 0; j < nc; j += NR, ++task_j) {
        const size_t nr = (j + NR <= nc) ? NR : nc - j;
        if (tab) {
          const size_t task_tab = task_j / (blk / NR);
          const uint8_t* t = tab + (task_n * NC) / blk + task_k * KC * ldtab + task_tab;
          const size_t count = get_indices(t, ldtab, kc, idx);
          if (count == 0) continue;
          pack_b_no_trans_non0tab(*buf_b, bt + j, nr, ldb, idx, count);
          loop_1st_mr(cc + j, ap, *buf_b, mc, nr, kc, ldc, barrier + task_j * ntask_mr, idx, count);
        } else {
          if (transb)
            pack_b_trans(*buf_b, bt + j * ldb, kc, nr, ldb);
          else
            pack_b_no_trans(*buf_b, bt + j, kc, nr, ldb);
          loop_1st_mr(cc + j, ap, *buf_b, mc, nr, kc, ldc, barrier + task_j * ntask_mr, nullptr, 0);
        }
      }
    });
  }

  // impl_aodmao2rho.rs:10-29
  static void pack_dm(APanel* dm_packed, const double* dm, size_t stride_ao, const size_t* iu,
                      size_t cu, const size_t* iv, size_t cv) {
    for (size_t ip = 0; ip < cv; ++ip)
      for (size_t t = 0; t * MR < cu; ++t)
        for (size_t im = 0; im < MR && t * MR + im < cu; ++im)
          dm_packed[t].v[ip][im] = dm[iu[t * MR + im] * stride_ao + iv[ip]];
  }

  // impl_aodmao2rho.rs:171-244, with loop_2nd (97-169) and loop_1st (31-95) inlined.
  static void aodmao2rho(double* rhos, const double* dms, const double* ao_lhs,
                         const double* ao_rhs, size_t stride_ao, size_t stride_grid, size_t nao,
                         size_t ngrid, size_t nset, const uint8_t* tab, size_t ldtab, size_t BLK,
                         size_t NC, int nthreads) {
    const size_t ntask_uc = div_ceil(nao, MC), ntask_vc = div_ceil(nao, KC);
    const size_t ntask_gc = div_ceil(ngrid, NC), ntask_ur = div_ceil(MC, MR);
    const size_t ntask_gr = div_ceil(NC, NR);
    const size_t BLKNR = BLK / NR;
    if (ntask_uc * ntask_vc * ntask_gc == 0) return;
    std::unique_ptr<std::mutex[]> g_barrier(new std::mutex[ntask_gc * ntask_gr]);
    // one dm_packed buffer per thread: [nset][ntask_ur][KC][MR] (impl_aodmao2rho.rs:196-198)
    std::vector<std::vector<APanel>> dm_packed_buffer(nthreads);
    for (auto& v : dm_packed_buffer) {
      v.resize(nset * ntask_ur);
      std::memset(v.data(), 0, v.size() * sizeof(APanel));
    }

    run_tasks(ntask_uc * ntask_vc * ntask_gc, nthreads, [&](size_t task_id, int tid) {
      const size_t task_u = task_id % ntask_uc;
      const size_t task_g = (task_id / ntask_uc) % ntask_gc;
      const size_t task_v = task_id / (ntask_uc * ntask_gc);
      const size_t task_tab = (task_g * NC) / BLK;
      const size_t u_start = task_u * MC, v_start = task_v * KC, g_start = task_g * NC;
      const size_t uc = std::min((task_u + 1) * MC, nao) - u_start;
      const size_t vc = std::min((task_v + 1) * KC, nao) - v_start;
      const size_t gc = std::min((task_g + 1) * NC, ngrid) - g_start;
      const double* lhs = ao_lhs + u_start * stride_grid + g_start;
      const double* rhs = ao_rhs + v_start * stride_grid + g_start;
      const double* dm = dms + u_start * stride_ao + v_start;
      const uint8_t* tab_lhs = tab + u_start * ldtab + task_tab;
      const uint8_t* tab_rhs = tab + v_start * ldtab + task_tab;
      double* rho = rhos + g_start;
      std::mutex* barrier = g_barrier.get() + task_g * ntask_gr;
      APanel* dm_packed = dm_packed_buffer[tid].data();

      std::unique_ptr<double[][NR]> lhs_packed(new double[MC][NR]());
      std::unique_ptr<double[][NR]> rhs_packed(new double[KC][NR]());
      size_t iu[MC], iv[KC];
      // aodmao2rho_loop_2nd
      for (size_t g = 0, task_gblk = 0; g < gc; g += BLK, ++task_gblk) {
        const size_t gblk = (g + BLK <= gc) ? BLK : gc - g;
        const size_t cv = get_indices(tab_rhs + task_gblk, ldtab, vc, iv);
        const size_t cu = get_indices(tab_lhs + task_gblk, ldtab, uc, iu);
        if (cv == 0 || cu == 0) continue;
        for (size_t s = 0; s < nset; ++s)
          pack_dm(dm_packed + s * ntask_ur, dm + s * stride_ao * stride_ao, stride_ao, iu, cu, iv, cv);
        for (size_t gg = g, task_gg = 0; gg < g + gblk; gg += NR, ++task_gg) {
          const size_t gr = (gg + NR <= g + gblk) ? NR : g + gblk - gg;
          for (size_t ip = 0; ip < cv; ++ip)
            for (size_t j = 0; j < gr; ++j) rhs_packed[ip][j] = rhs[iv[ip] * stride_grid + gg + j];
          for (size_t ip = 0; ip < cu; ++ip)
            for (size_t j = 0; j < gr; ++j) lhs_packed[ip][j] = lhs[iu[ip] * stride_grid + gg + j];
          // aodmao2rho_loop_1st
          std::mutex& lock_g = barrier[task_gblk * BLKNR + task_gg];
          for (size_t m0 = 0, task_mr = 0; m0 < cu; m0 += MR, ++task_mr) {
            const size_t mr = (m0 + MR <= cu) ? MR : cu - m0;
            for (size_t s = 0; s < nset; ++s) {
              double c_reg[MR][NR];
              std::memset(c_reg, 0, sizeof(c_reg));
              microkernel(c_reg, dm_packed[s * ntask_ur + task_mr].v, rhs_packed.get(), cv);
              double rho_reg[NR] = {0};
              for (size_t mm = 0; mm < mr; ++mm)
                for (size_t j = 0; j < NR; ++j)
                  rho_reg[j] = std::fma(c_reg[mm][j], lhs_packed[m0 + mm][j], rho_reg[j]);
              std::lock_guard<std::mutex> lk(lock_g);
              double* r = rho + s * stride_grid + gg;
              for (size_t j = 0; j < gr; ++j) r[j] = rho_reg[j] + r[j];
            }
          }
        }
      }
    });
  }
};

// The fixed Zen4 tuning of every `*_anyway` wrapper: <f64, 252, 512, 240, 14, 2, 8>.
using Anyway = Loops<252, 512, 14, 16>;

// Smallest NC >= 240 that is a multiple of both BLKSIZE and NR = 16; for
// BLKSIZE 48 this is the reference's own NC = 240.  NC only splits the grid
// axis into tasks: per grid point the order of the partial sums is the same
// for every admissible NC (impl_aodmao2rho.rs:205-207).
size_t nc_for_blk(size_t blk) {
  size_t nc = blk;
  while (nc < 240 || nc % 16 != 0) nc += blk;
  return nc;
}

}  // namespace

extern "C" {

// matmul_loop_parallel_mnk_pack_a with the matmul_anyway_full tuning.
// Returns 0, or -1 when m/n/k/ld describe a matrix that does not fit.
int oracle_matmul_anyway_full(double* c, const double* a, const double* b, size_t m, size_t n,
                              size_t k, size_t lda, size_t ldb, size_t ldc, int transa,
                              int transb, int nthreads) {
  Anyway::matmul(c, a, b, m, n, k, lda, ldb, ldc, transa != 0, transb != 0, 240, nullptr, 0, 16,
                 resolve_threads(nthreads));
  return kOk;
}

// matmul_loop_parallel_mnk_pack_a_non0tab::<BLKSIZE> with the anyway tuning.
// transb != 0 mirrors the reference's `unimplemented!` (non0tab.rs:181, 228).
int oracle_matmul_anyway_full_non0tab(double* c, const double* a, const double* b, size_t m,
                                      size_t n, size_t k, size_t lda, size_t ldb, size_t ldc,
                                      int transa, int transb, const uint8_t* tab, size_t ldtab,
                                      size_t blksize, int nthreads) {
  if (transb) return kUnsupported;
  if (blksize == 0 || blksize % 16 != 0 || 240 % blksize != 0) return kInvalid;
  Anyway::matmul(c, a, b, m, n, k, lda, ldb, ldc, transa != 0, false, 240, tab, ldtab, blksize,
                 resolve_threads(nthreads));
  return kOk;
}

// aodmao2rho_loop_parallel::<BLKSIZE> with the anyway tuning (MC 252, KC 512,
// MR 14, NR 16).  BLKSIZE must be a multiple of NR = 16 (the reference's
// debug_assert, impl_aodmao2rho.rs:111).
int oracle_aodmao2rho(double* rhos, const double* dms, const double* ao_lhs, const double* ao_rhs,
                      size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
                      const uint8_t* tab, size_t ldtab, size_t blksize, int nthreads) {
  if (blksize == 0 || blksize % 16 != 0) return kInvalid;
  Anyway::aodmao2rho(rhos, dms, ao_lhs, ao_rhs, stride_ao, stride_grid, nao, ngrid, nset, tab,
                     ldtab, blksize, nc_for_blk(blksize), resolve_threads(nthreads));
  return kOk;
}

// Fock-build contraction, the transpose of aodmao2rho with the same layouts
// and mask (no counterpart in the reference, whose DFT callers form V
// themselves):  vs[s][u][v] += sum over blocks b with tab[u][b] && tab[v][b] of
// sum_{g in b} (ao_lhs[u][g] * ws[s][g]) * ao_rhs[v][g], one FMA per point in
// ascending g.  Rows u are independent, so any thread count gives the same bits.
int oracle_aodm_fock(double* vs, const double* ws, const double* ao_lhs, const double* ao_rhs,
                     size_t stride_ao, size_t stride_grid, size_t nao, size_t ngrid, size_t nset,
                     const uint8_t* tab, size_t ldtab, size_t blksize, int nthreads) {
  if (blksize == 0 || (nao > 0 && stride_ao < nao)) return kInvalid;
  const size_t nblk = (ngrid + blksize - 1) / blksize;
  for (size_t s = 0; s < nset; ++s) {
    double* v = vs + s * stride_ao * stride_ao;
    const double* w = ws + s * stride_grid;
#pragma omp parallel for schedule(dynamic, 1) num_threads(resolve_threads(nthreads))
    for (long long uu = 0; uu < (long long)nao; ++uu) {
      const size_t u = size_t(uu);
      std::vector<double> lw(ngrid);
      for (size_t g = 0; g < ngrid; ++g) lw[g] = ao_lhs[u * stride_grid + g] * w[g];
      for (size_t vv = 0; vv < nao; ++vv) {
        double acc = 0.0;
        for (size_t b = 0; b < nblk; ++b) {
          if (!tab[u * ldtab + b] || !tab[vv * ldtab + b]) continue;
          const size_t g1 = std::min(ngrid, (b + 1) * blksize);
          for (size_t g = b * blksize; g < g1; ++g)
            acc = std::fma(lw[g], ao_rhs[vv * stride_grid + g], acc);
        }
        v[u * stride_ao + vv] += acc;
      }
    }
  }
  return kOk;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
