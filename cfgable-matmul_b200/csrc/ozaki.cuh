// ozaki.cuh -- internal interface of the Ozaki-scheme split-precision paths.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "gemm_i8.cuh"

namespace cfgmm {

// Exact INT32 accumulation needs k * 128 * 128 < 2^31; the epilogue's
// float-quotient reduction is exact (after two corrections) for |acc| < 2^30.
constexpr int kOzakiMaxK = 65536;
// Default operand precision (bits kept relative to each row / column max).
constexpr int kOzakiMinBits = 46;
// Upper bound of the operand precision (exactness of the residue arithmetic).
constexpr int kOzakiMaxBits = 52;

struct OzakiPlan {
  int nmod;             // number of moduli N
  int alpha, beta;      // bits of the scaled integer operands A', B'
  int mod[kMaxModuli];  // moduli, 256 first
  float inv_f[kMaxModuli];
  double inv_d[kMaxModuli];
  // CRT weights w_l (sum_l r_l w_l = C' mod M), split at 2^T:
  double w_hi[kMaxModuli];    // w_l >> T (exact)
  double w_lo[kMaxModuli];    // w_l mod 2^T (rounded)
  double M_hi, M_lo, two_T;   // M >> T, M mod 2^T, 2^T
  double t_x, t_y;            // 2^T / M, 1 / M: the quotient from the hi / lo sums
};

// Plan for contraction length k with `nmod` moduli (<= 0: the fewest moduli
// that keep min_bits bits of both operands).
OzakiPlan ozaki_plan(int k, int nmod, int min_bits);

// Moduli used for contraction length k (environment CFGMM_OZAKI_MODULI
// overrides, 2..16).
int ozaki_default_moduli(int k);
// Moduli that give operands of at least `bits` bits at this k (26 for f32 data).
int ozaki_moduli_for_bits(int k, int bits);

size_t ozaki_dgemm_workspace(int m, int n, int k, int nmod);

// C[i*ldc+j] += sum_p opA(i,p) opB(p,j) by INT8 tensor-core emulation; device
// pointers; workspace of ozaki_dgemm_workspace bytes (256-byte aligned).
// `events` (optional, 4 entries) are recorded before the residue preparation
// and after the preparation, the INT8 GEMM and the reconstruction.  With `tab`
// this is the masked GEMM (B not transposed): element (p, j) of B takes part
// only when tab[p * ldtab + j / blk] != 0.  C is first read by the
// reconstruction: when `c_ready` is given the stream waits for it just before,
// so that C may still be arriving while the residues and the INT8 GEMM run.
// Blocks of one product: every call lays the workspace out for `m_layout`
// rows and `n_layout` columns (>= m, n; 0: m, n), so that a call with
// `reuse_a` (`reuse_b`) takes the residues and exponents of A (B) that an
// earlier call on the same stream, workspace, A (B), k and nmod left there
// instead of forming them again.
cudaError_t ozaki_dgemm(double* c, const double* a, const double* b, int m, int n, int k,
                        size_t lda, size_t ldb, size_t ldc, bool transa, bool transb, int nmod,
                        void* workspace, cudaStream_t stream,
                        const cudaEvent_t* events = nullptr, const uint8_t* tab = nullptr,
                        size_t ldtab = 0, int blk = 1, cudaEvent_t c_ready = nullptr,
                        int m_layout = 0, int n_layout = 0, bool reuse_a = false,
                        bool reuse_b = false);

}  // namespace cfgmm
