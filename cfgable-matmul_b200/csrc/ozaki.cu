// ozaki.cu -- FP64 GEMM emulated on the INT8 tensor cores by the Ozaki
// scheme in its Chinese-remainder form ("Ozaki scheme II": Ozaki, Uchino and
// Imamura, 2024/2025), restated here from the mathematics:
//
//   1. scaling: row i of op(A) is multiplied by 2^e_i and column j of op(B)
//      by 2^f_j and rounded to integers A', B' with |A'| <= 2^alpha,
//      |B'| <= 2^beta, where k 2^(alpha+beta) <= M/8 and M = prod m_l;
//   2. residues: A'_l = A' mods m_l, B'_l = B' mods m_l (int8) for N pairwise
//      coprime moduli m_l <= 256;
//   3. N exact INT8 GEMMs C_l = A'_l B'_l (INT32 in TMEM, gemm_i8.cu), each
//      reduced to r_l = C_l mods m_l in its epilogue;
//   4. reconstruction: C' = A'B' is the unique integer with |C'| < M/2 and
//      C' = r_l (mod m_l): C' = sum_l r_l w_l - q M with the CRT weights w_l and
//      q = round(sum_l r_l w_l / M).  Evaluated in FP64 with each w_l and M
//      split at 2^T into a high part (exact products and sums, < 2^53) and a
//      low part, so C' comes out with one rounding; C = C' 2^-(e_i + f_j).
//
// The only error is the rounding of A and B to alpha / beta bits relative to
// their row / column maxima; the number of moduli sets alpha and beta.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "gemm_i8.cuh"
#include "ozaki.cuh"
#include "side_stream.cuh"

namespace cfgmm {

// Pairwise coprime moduli, largest first (256 = 2^8, 255 = 3*5*17,
// 253 = 11*23, 247 = 13*19, 217 = 7*31, the rest prime).
static const int kModuli[kMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233,
                                        229, 227, 223, 217, 211, 199, 197, 193};

namespace {

using u128 = unsigned __int128;

int bit_length(u128 v) {
  int n = 0;
  while (v) {
    ++n;
    v >>= 1;
  }
  return n;
}

long long mod_inverse(long long a, long long m) {  // a^-1 mod m, gcd(a, m) = 1
  long long t = 0, nt = 1, r = m, nr = a % m;
  while (nr) {
    const long long qq = r / nr;
    long long tmp = t - qq * nt;
    t = nt;
    nt = tmp;
    tmp = r - qq * nr;
    r = nr;
    nr = tmp;
  }
  return t < 0 ? t + m : t;
}

int ceil_log2(long long v) {
  int n = 0;
  while ((1LL << n) < v) ++n;
  return n;
}

}  // namespace

OzakiPlan ozaki_plan(int k, int nmod, int min_bits) {
  OzakiPlan p{};
  if (nmod <= 0) {
    // smallest N whose operand precision reaches min_bits
    for (nmod = 2; nmod < kMaxModuli; ++nmod) {
      OzakiPlan t = ozaki_plan(k, nmod, min_bits);
      if (t.alpha >= min_bits && t.beta >= min_bits) break;
    }
  }
  if (nmod > kMaxModuli) nmod = kMaxModuli;
  p.nmod = nmod;
  u128 M = 1;
  for (int l = 0; l < nmod; ++l) M *= u128(kModuli[l]);
  const int logM = bit_length(M) - 1;  // floor(log2 M)
  const int P = logM - 3 - ceil_log2(k > 1 ? k : 2);
  // at most 52 bits each: the FP32 residue computation is exact up to 2^52
  // op(B) takes the smaller half when P is odd: in a host call it is split once
  // for every row block of A, and at 47 bits or fewer its residues take the
  // three-digit form (the headline shape has the larger B)
  p.beta = std::min(P / 2, kOzakiMaxBits);
  p.alpha = std::min(P - P / 2, kOzakiMaxBits);
  // split point T: sum_l |r_l| hi_l + |q| H < 2^53 with |r_l| <= 128, |q| <= 128 N
  const int T = std::max(0, logM + 1 + 7 + ceil_log2(nmod + 1) + 1 - 52);
  p.two_T = std::ldexp(1.0, T);
  const u128 lo_mask = (T >= 128) ? ~u128(0) : ((u128(1) << T) - 1);
  const double Md = double(M);
  for (int l = 0; l < nmod; ++l) {
    const long long m = kModuli[l];
    const u128 Ml = M / u128(m);
    const long long inv = mod_inverse(static_cast<long long>(Ml % u128(m)), m);
    const u128 w = Ml * u128(inv);  // < M
    p.mod[l] = int(m);
    p.inv_f[l] = 1.0f / float(m);
    p.inv_d[l] = 1.0 / double(m);
    p.w_hi[l] = double(w >> T);
    p.w_lo[l] = double(w & lo_mask);
  }
  p.M_hi = double(M >> T);
  p.M_lo = double(M & lo_mask);
  p.t_x = std::ldexp(1.0, T) / Md;
  p.t_y = 1.0 / Md;
  return p;
}

namespace {

constexpr int kNonFinite = INT_MAX;  // exponent sentinel of a row holding Inf/NaN

// ---------------------------------------------------------------------------
// exponents: e[r] = bits - E_r with max_p |x(r,p)| < 2^E_r  (0 for a zero row)
// Computed in two steps: Emax[r] = max over chunks of the binary exponent of
// the chunk maximum (INT_MAX for Inf/NaN, INT_MIN for all-zero), then e[r].
// ---------------------------------------------------------------------------
__device__ __forceinline__ int exponent_of(double amax) {
  if (!(amax <= 1.7976931348623157e308)) return INT_MAX;  // Inf or NaN
  if (amax == 0.0) return INT_MIN;
  int E;
  frexp(amax, &E);  // amax = f 2^E, f in [0.5, 1): amax < 2^E
  return E;
}

__global__ void fill_int(int* __restrict__ v, int n, int value) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i < n) v[i] = value;
}

// element (r, p) at x[r*ld + p]: one CTA per row
__global__ void __launch_bounds__(256)
emax_rows(const double* __restrict__ x, size_t ld, int rows, int k, int* __restrict__ emax) {
  const int r = blockIdx.x;
  if (r >= rows) return;
  const double* row = x + size_t(r) * ld;
  int E = INT_MIN;
  for (int p = threadIdx.x; p < k; p += 256) E = max(E, exponent_of(fabs(row[p])));
  for (int o = 16; o > 0; o >>= 1) E = max(E, __shfl_xor_sync(0xffffffffu, E, o));
  __shared__ int red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = E;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) E = max(E, red[w]);
    emax[r] = max(E, red[0]);
  }
}

// Optional mask of the masked GEMM: element (r, p) of op(B)^T takes part only
// when tab[p * ldtab + r / blk] != 0 (impl_matmul_non0tab.rs:196-207).
struct Mask {
  const uint8_t* tab;  // null: no mask
  size_t ldtab;
  int blk;
  __device__ __forceinline__ bool on(int r, int p) const {
    return !tab || tab[size_t(p) * ldtab + r / blk] != 0;
  }
};

// element (r, p) at x[p*ld + r]: thread per r (coalesced), CTA rows of p chunks
constexpr int kColChunk = 128;
__global__ void __launch_bounds__(256)
emax_cols(const double* __restrict__ x, size_t ld, int rows, int k, int* __restrict__ emax,
          Mask mask) {
  const int r = blockIdx.x * 256 + threadIdx.x;
  const int p0 = blockIdx.y * kColChunk;
  if (r >= rows) return;
  const int p1 = min(k, p0 + kColChunk);
  double mx = 0.0;
  bool bad = false;
  for (int p = p0; p < p1; ++p) {
    const double v = mask.on(r, p) ? fabs(x[size_t(p) * ld + r]) : 0.0;
    bad |= !(v <= 1.7976931348623157e308);
    mx = fmax(mx, v);
  }
  atomicMax(&emax[r], bad ? INT_MAX : exponent_of(mx));
}

__global__ void finalize_exps(const int* __restrict__ emax, int rows, int bits, int* __restrict__ e) {
  const int r = blockIdx.x * 256 + threadIdx.x;
  if (r >= rows) return;
  const int E = emax[r];
  e[r] = (E == INT_MAX) ? kNonFinite : (E == INT_MIN ? 0 : bits - E);
}

// ---------------------------------------------------------------------------
// residues: Y[l][r][p] = rint(x(r,p) 2^e[r]) mods m_l  (int8), p < k
// The integer v (|v| <= 2^52) is written in balanced 14-bit digits:
// w = v + 2^13 (1 + 2^14 + 2^28) gives u_t = (w >> 14t) & 0x3fff (t < 3) and
// d_3 = w >> 42 with v = sum_{t<3} (u_t - 2^13) 2^14t + d_3 2^42.  With the
// symmetric c_t = 2^(14t) mods m (|c_t| <= 127) and the balanced digits
// b_t = u_t - 2^13 (formed once per element, before the modulus loop)
//   s = b_0 + b_1 c_14 + b_2 c_28 + d_3 c_42,   |s| < 2.3e6 < 2^22,
// (three FMAs per modulus, every partial sum below 2^22) is exact in FP32 and
// congruent to v.  Then q = rint(s / m) comes out exact
// from one FMA against MAGIC = 1.5 2^23 (|s| < 2^22 keeps the error of s*inv
// below 1/(2m), the least distance of s/m from a half-integer for odd m), the
// residue r = s - m q is exact, and r + MAGIC holds r in the low byte of its
// bits.  Two elements go through each packed FP32x2 instruction (sm_100).
// Modulus 256 is the low byte of v's two's complement.
// ---------------------------------------------------------------------------
using f32x2 = unsigned long long;  // two FP32 lanes in a 64-bit register

// Per modulus l (index 0 is 256, taken from the low byte): c_14, c_28, c_42,
// 1/m and -m, each in both lanes of an FP32x2 word.
struct ResidueArgs {
  int nmod;
  f32x2 c14[kMaxModuli], c28[kMaxModuli], c42[kMaxModuli], inv[kMaxModuli], nm[kMaxModuli];
  f32x2 c16[kMaxModuli], c32[kMaxModuli];  // the 16-bit digit form's 2^16, 2^32 mods m
};

__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack2(f32x2 v, uint32_t& lo, uint32_t& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// rint(x 2^e) for a row exponent e (0 for a row holding Inf/NaN).  The power
// of two is applied as one or two exact multiplications (ldexp outside the
// normal range of the factor).
__device__ __forceinline__ double scaled_int(double x, int e) {
  if (e == kNonFinite) return 0.0;
  if (e >= -1022 && e <= 1023)
    return rint(x * __longlong_as_double(static_cast<long long>(e + 1023) << 52));
  return rint(ldexp(x, e));
}

constexpr long long kDigitBias = 8192LL * (1 + (1LL << 14) + (1LL << 28));
// 1.5 2^52 + kDigitBias: for an integer v with |v| <= 2^50, v + kRoundBias lies in
// [2^52, 2^53), where the spacing of doubles is 1, so its mantissa field holds
// w + 2^51 (w = v + kDigitBias) and the rounding that forms it is rint(v).
constexpr double kRoundBias = 6755399441055744.0 + double(kDigitBias);
// The 16-bit digit form, for |v| <= 2^47: w = v + kDigitBias16 in [0, 2^49),
// v = sum_{t<3} (u_t - 2^15) 2^16t with u_t = (w >> 16t) & 0xffff (t < 2) and
// u_2 = w >> 32, every balanced digit within [-2^15, 2^15]; then
//   s = b_0 + b_1 c_16 + b_2 c_32,  |s| <= 2^15 (1 + 2 * 127) < 2^23,
// two FMAs per modulus, exact, and |s| < 2^23 is what the quotient needs
// (|s| 2^-24 / m, the error of s * fl(1/m), stays below 1/(2m)).
constexpr long long kDigitBias16 = 32768LL * (1 + (1LL << 16) + (1LL << 32));
constexpr double kRoundBias16 = 6755399441055744.0 + double(kDigitBias16);

// Digit forms of write_residues8: plain (integers up to 2^52, four 14-bit
// digits), biased (up to 2^50, four 14-bit digits read off the double's bits)
// and biased16 (up to 2^47, three 16-bit digits).
enum : int { kPlain = 0, kBiased14 = 1, kBiased16 = 2 };

// The operand element x(r, p) 2^e as the input of write_residues8: rint(x 2^e)
// (the plain form), or that integer plus the form's round bias, rounded once by
// the FMA (the biased forms).  e = kNonFinite gives 0.
template <int kForm>
__device__ __forceinline__ double scaled(double x, int e) {
  if constexpr (kForm != kPlain) {
    constexpr double bias = kForm == kBiased16 ? kRoundBias16 : kRoundBias;
    if (e == kNonFinite) return bias;
    if (e >= -1022 && e <= 1023)
      return fma(x, __longlong_as_double(static_cast<long long>(e + 1023) << 52), bias);
    return rint(ldexp(x, e)) + bias;
  } else {
    return scaled_int(x, e);
  }
}
template <int kForm>
__device__ __forceinline__ double scaled_zero() {
  return kForm == kBiased16 ? kRoundBias16 : (kForm == kBiased14 ? kRoundBias : 0.0);
}

// The residues of 8 consecutive elements for every modulus, 8 bytes per modulus
// plane at Y + l * plane + off (8-byte aligned).  v[] holds integers |v| <= 2^52
// (plain form) or |v| <= 2^50 (2^47) plus the form's round bias (biased forms:
// the digits are bit fields of the double, with no conversion to a 64-bit
// integer).  The low byte of w is v's (both digit biases are multiples of 256).
template <int kForm>
__device__ __forceinline__ void write_residues8(const ResidueArgs& a, int8_t* Y, size_t plane,
                                                size_t off, const double (&v)[8]) {
  constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
  f32x2 P0[4], P1[4], P2[4], P3[4];
  uint32_t lowb[2] = {0u, 0u};
#pragma unroll
  for (int j = 0; j < 8; j += 2) {
    float u[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if constexpr (kForm == kBiased16) {
        // mantissa field = w + 2^51: bits 0..31 are w's, bits 32..51 are (w >> 32) + 2^19
        const uint32_t lo = __double2loint(v[j + h]), hi = __double2hiint(v[j + h]);
        lowb[(j + h) >> 2] |= (lo & 0xffu) << (8 * ((j + h) & 3));  // modulus 256
        u[h][0] = float(int(lo & 0xffffu) - 32768);
        u[h][1] = float(int(lo >> 16) - 32768);
        u[h][2] = float(int(hi & 0xfffffu) - (1 << 19) - 32768);
        u[h][3] = 0.0f;
      } else if constexpr (kForm == kBiased14) {
        // mantissa field = w + 2^51: bits 0..41 are w's, bits 42..51 are (w >> 42) + 2^9
        const uint32_t lo = __double2loint(v[j + h]), hi = __double2hiint(v[j + h]);
        lowb[(j + h) >> 2] |= (lo & 0xffu) << (8 * ((j + h) & 3));  // modulus 256
        u[h][0] = float(int(lo & 0x3fffu) - 8192);
        u[h][1] = float(int((lo >> 14) & 0x3fffu) - 8192);
        u[h][2] = float(int(__funnelshift_r(lo, hi, 28) & 0x3fffu) - 8192);
        u[h][3] = float(int((hi >> 10) & 0x3ffu) - 512);
      } else {
        const long long iv = static_cast<long long>(v[j + h]);
        lowb[(j + h) >> 2] |= uint32_t(iv & 0xff) << (8 * ((j + h) & 3));  // modulus 256
        const long long w = iv + kDigitBias;
        u[h][0] = float(int(w & 0x3fff) - 8192);
        u[h][1] = float(int((w >> 14) & 0x3fff) - 8192);
        u[h][2] = float(int((w >> 28) & 0x3fff) - 8192);
        u[h][3] = float(int(w >> 42));
      }
    }
    P0[j >> 1] = pack2(u[0][0], u[1][0]);
    P1[j >> 1] = pack2(u[0][1], u[1][1]);
    P2[j >> 1] = pack2(u[0][2], u[1][2]);
    P3[j >> 1] = pack2(u[0][3], u[1][3]);
  }
  *reinterpret_cast<uint2*>(Y + off) = make_uint2(lowb[0], lowb[1]);
  const f32x2 MAG = pack2(kMagic, kMagic), NMAG = pack2(-kMagic, -kMagic);
  // unrolled: every constant is read at a fixed offset of the parameter bank
#pragma unroll
  for (int l = 1; l < kMaxModuli; ++l) {
    if (l >= a.nmod) break;
    const f32x2 INV = a.inv[l], NM = a.nm[l];
    uint32_t bits[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      f32x2 S;
      if constexpr (kForm == kBiased16) {
        S = fma2(P1[q], a.c16[l], P0[q]);
        S = fma2(P2[q], a.c32[l], S);                 // s, exact
      } else {
        S = fma2(P1[q], a.c14[l], P0[q]);
        S = fma2(P2[q], a.c28[l], S);
        S = fma2(P3[q], a.c42[l], S);                 // s, exact
      }
      const f32x2 Q = add2(fma2(S, INV, MAG), NMAG);  // rint(s / m), exact
      const f32x2 R = add2(fma2(NM, Q, S), MAG);      // (s - m q) + MAGIC
      unpack2(R, bits[2 * q], bits[2 * q + 1]);
    }
    const uint32_t w0 = __byte_perm(__byte_perm(bits[0], bits[1], 0x0040),
                                    __byte_perm(bits[2], bits[3], 0x0040), 0x5410);
    const uint32_t w1 = __byte_perm(__byte_perm(bits[4], bits[5], 0x0040),
                                    __byte_perm(bits[6], bits[7], 0x0040), 0x5410);
    *reinterpret_cast<uint2*>(Y + size_t(l) * plane + off) = make_uint2(w0, w1);
  }
}

// element (r, p) at x[r*ld + p]: CTA per row, thread per 8 consecutive p
template <int kForm>
__global__ void __launch_bounds__(256, 5)
residues_rows(const double* __restrict__ x, size_t ld, int rows, int k, size_t kpad,
              const int* __restrict__ e, int8_t* __restrict__ Y, ResidueArgs a) {
  const int r = blockIdx.x;
  if (r >= rows) return;
  const int er = e[r];
  const double* row = x + size_t(r) * ld;
  const size_t plane = size_t(rows) * kpad;
  for (int p = 8 * threadIdx.x; p < k; p += 8 * 256) {
    double v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
      v[j] = (p + j < k) ? scaled<kForm>(row[p + j], er) : scaled_zero<kForm>();
    write_residues8<kForm>(a, Y, plane, size_t(r) * kpad + p, v);
  }
}

// element (r, p) at x[p*ld + r]: 32 (r) x 64 (p) tiles transposed through shared
// memory.  Element (p, r) sits in column r ^ 2 (p / 8) of row p: a row is written
// by one warp (a permutation of its 32 columns), and each half-warp of the
// read side (two r, eight groups of p) meets 16 distinct 8-byte bank pairs.
__device__ __forceinline__ int tile_col(int p, int r) { return r ^ ((p >> 2) & 14); }

template <int kForm>
__global__ void __launch_bounds__(256, 5)
residues_cols(const double* __restrict__ x, size_t ld, int rows, int k, size_t kpad,
              const int* __restrict__ e, int8_t* __restrict__ Y, ResidueArgs a, Mask mask) {
  __shared__ double tile[64][32];
  const int r0 = blockIdx.x * 32, p0 = blockIdx.y * 64;
  const int tr = threadIdx.x & 31, tp = threadIdx.x >> 5;  // 8 rows of p per pass
#pragma unroll
  for (int pp = tp; pp < 64; pp += 8) {
    const int p = p0 + pp, r = r0 + tr;
    tile[pp][tile_col(pp, tr)] =
        (p < k && r < rows && mask.on(r, p)) ? x[size_t(p) * ld + r] : 0.0;
  }
  __syncthreads();
  const size_t plane = size_t(rows) * kpad;
  // 32 rows x 8 groups of 8 p: one unit per thread
  const int rr = threadIdx.x >> 3, pg = (threadIdx.x & 7) * 8;
  const int r = r0 + rr, p = p0 + pg;
  if (r >= rows || p >= k) return;
  const int er = e[r];
  double v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j)
    v[j] = (p + j < k) ? scaled<kForm>(tile[pg + j][tile_col(pg + j, rr)], er)
                       : scaled_zero<kForm>();
  write_residues8<kForm>(a, Y, plane, size_t(r) * kpad + p, v);
}

// ---------------------------------------------------------------------------
// reconstruction: C[i][j] += 2^-(e_i + f_j) * CRT(r_0..r_{N-1})
// ---------------------------------------------------------------------------
struct ReconArgs {
  int nmod;
  double w_hi[kMaxModuli], w_lo[kMaxModuli];
  double M_hi, M_lo, two_T;
  double t_x, t_y;  // 2^T / M and 1 / M (the quotient estimate)
};

// A thread rebuilds 4 consecutive C[i][j]: its residue loads (4 bytes per
// modulus plane) are all issued before the arithmetic.  A residue byte becomes
// an exact double without a conversion instruction: with its sign bit flipped
// it is r + 128 in [0, 255], placed in the low word of 2^52 and the 2^52 + 128
// subtracted again.  X = sum_l r_l w_hi[l] is exact (every partial sum is
// below 2^53) and Y = sum_l r_l w_lo[l] rounded, so t = X 2^T / M + Y / M, two
// operations, is within ~1e-12 of sum_l r_l w_l / M (|X 2^T / M| <= 128 N);
// |C'| <= M/8 keeps that exact value within 1/8 of the integer q, so
// q = rint(t) is the one of exact arithmetic.
__global__ void __launch_bounds__(256)
reconstruct(double* __restrict__ c, size_t ldc, int m, int n, const int8_t* __restrict__ R,
            size_t ldr, const int* __restrict__ ea, const int* __restrict__ eb, ReconArgs a) {
  const int bpr = (n + 1023) / 1024;  // CTAs per row of C
  const int i = blockIdx.x / bpr;
  const int j0 = ((blockIdx.x % bpr) * 256 + threadIdx.x) * 4;
  if (j0 >= n || i >= m) return;
  const size_t plane = size_t(m) * ldr;
  // ldr is a multiple of 16 and j0 of 4: the 4 bytes at j0 lie inside row i
  const int8_t* Ri = R + size_t(i) * ldr + j0;
  uint32_t rv[kMaxModuli];
#pragma unroll
  for (int l = 0; l < kMaxModuli; ++l)
    if (l < a.nmod) rv[l] = __ldg(reinterpret_cast<const uint32_t*>(Ri + size_t(l) * plane));
  // C and the column scales are requested with the residues (one round trip)
  double* ci = c + size_t(i) * ldc;
  double c_old[4];
  int fj[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const bool in = j0 + u < n;
    c_old[u] = in ? ci[j0 + u] : 0.0;
    fj[u] = in ? __ldg(eb + j0 + u) : 0;
  }
  constexpr double kBias = 4503599627370624.0;  // 2^52 + 128
  double X[4], Y[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) X[u] = Y[u] = 0.0;
#pragma unroll
  for (int l = 0; l < kMaxModuli; ++l) {
    if (l >= a.nmod) break;
    const uint32_t wb = rv[l] ^ 0x80808080u;  // r + 128 in every byte
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double r = __hiloint2double(0x43300000, int(__byte_perm(wb, 0u, 0x4440u + u))) - kBias;
      X[u] = fma(r, a.w_hi[l], X[u]);  // exact
      Y[u] = fma(r, a.w_lo[l], Y[u]);
    }
  }
  const int ei = ea[i];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int j = j0 + u;
    if (j >= n) break;
    const double q = rint(fma(X[u], a.t_x, Y[u] * a.t_y));
    const double hi = fma(-q, a.M_hi, X[u]);  // exact
    const double lo = fma(-q, a.M_lo, Y[u]);
    const double cp = fma(hi, a.two_T, lo);   // C' with one rounding
    const int sc = -(ei + fj[u]);
    double val;
    if (ei == kNonFinite || fj[u] == kNonFinite)
      val = __longlong_as_double(0x7ff8000000000000LL);
    else if (sc >= -1022 && sc <= 1023)  // exact scaling by a normal power of two
      val = cp * __longlong_as_double(static_cast<long long>(sc + 1023) << 52);
    else
      val = ldexp(cp, sc);
    ci[j] = c_old[u] + val;
  }
}

// ---------------------------------------------------------------------------
// tensor maps
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

bool make_plane_map(CUtensorMap* map, void* base, int k, int rows, int nplanes, size_t kpad,
                    int box_rows) {
  auto enc = encode_fn();
  if (!enc) return false;
  cuuint64_t dims[3] = {cuuint64_t(k), cuuint64_t(rows), cuuint64_t(nplanes)};
  cuuint64_t strides[2] = {cuuint64_t(kpad), cuuint64_t(rows) * kpad};
  cuuint32_t box[3] = {128, cuuint32_t(box_rows), 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

size_t a256(size_t v) { return (v + 255) / 256 * 256; }

struct DgemmLayout {
  size_t kpad, ldr, a_res, b_res, r, ea, eb, emax_a, emax_b, total;
};

DgemmLayout dgemm_layout(int m, int n, int k, int nmod) {
  DgemmLayout L;
  L.kpad = (size_t(k) + 127) / 128 * 128;
  L.ldr = (size_t(n) + 15) / 16 * 16;
  L.a_res = 0;
  L.b_res = L.a_res + a256(size_t(nmod) * m * L.kpad);
  L.r = L.b_res + a256(size_t(nmod) * n * L.kpad);
  L.ea = L.r + a256(size_t(nmod) * m * L.ldr);
  L.eb = L.ea + a256(size_t(m) * sizeof(int));
  L.emax_a = L.eb + a256(size_t(n) * sizeof(int));
  L.emax_b = L.emax_a + a256(size_t(m) * sizeof(int));
  L.total = L.emax_b + a256(size_t(n) * sizeof(int));
  return L;
}

int mods_host(long long v, int m) {  // symmetric residue
  long long r = v % m;
  if (r < 0) r += m;
  if (r > (m - 1) / 2) r -= m;
  return int(r);
}

// both FP32 lanes of a packed word set to v
f32x2 splat2(float v) {
  uint32_t b;
  std::memcpy(&b, &v, sizeof b);
  return (f32x2(b) << 32) | b;
}

ResidueArgs residue_args(const OzakiPlan& p) {
  ResidueArgs a{};
  a.nmod = p.nmod;
  for (int l = 0; l < p.nmod; ++l) {
    a.inv[l] = splat2(p.inv_f[l]);
    a.nm[l] = splat2(-float(p.mod[l]));
    a.c14[l] = splat2(float(mods_host(1LL << 14, p.mod[l])));
    a.c28[l] = splat2(float(mods_host(1LL << 28, p.mod[l])));
    a.c42[l] = splat2(float(mods_host(1LL << 42, p.mod[l])));
    a.c16[l] = splat2(float(mods_host(1LL << 16, p.mod[l])));
    a.c32[l] = splat2(float(mods_host(1LL << 32, p.mod[l])));
  }
  return a;
}

// Scales, rounds and splits op(X) into residue planes Y[nmod][rows][kpad];
// `emax` is scratch for rows ints.
cudaError_t prepare(const double* x, size_t ld, bool rows_contig, int rows, int k, size_t kpad,
                    int bits, int* emax, int* e, int8_t* Y, const ResidueArgs& ra,
                    cudaStream_t s, Mask mask = Mask{nullptr, 0, 1}) {
  const int rb = (rows + 255) / 256;
  if (rows_contig) {
    emax_rows<<<rows, 256, 0, s>>>(x, ld, rows, k, emax);
  } else {
    fill_int<<<rb, 256, 0, s>>>(emax, rows, INT_MIN);
    emax_cols<<<dim3(rb, (k + kColChunk - 1) / kColChunk), 256, 0, s>>>(x, ld, rows, k, emax,
                                                                         mask);
  }
  finalize_exps<<<rb, 256, 0, s>>>(emax, rows, bits, e);
  // scaled elements up to 2^47 take three 16-bit digits, up to 2^50 the
  // biased form of four 14-bit digits, the rest the plain form
  const int form = bits <= 47 ? kBiased16 : (bits <= 50 ? kBiased14 : kPlain);
  if (rows_contig) {
    auto kern = form == kBiased16 ? residues_rows<kBiased16>
                                  : (form == kBiased14 ? residues_rows<kBiased14>
                                                       : residues_rows<kPlain>);
    kern<<<rows, 256, 0, s>>>(x, ld, rows, k, kpad, e, Y, ra);
  } else {
    dim3 grid((rows + 31) / 32, (k + 63) / 64);
    auto kern = form == kBiased16 ? residues_cols<kBiased16>
                                  : (form == kBiased14 ? residues_cols<kBiased14>
                                                       : residues_cols<kPlain>);
    kern<<<grid, 256, 0, s>>>(x, ld, rows, k, kpad, e, Y, ra, mask);
  }
  return cudaGetLastError();
}

}  // namespace

const SideStream* side_stream(bool high_priority) {
  constexpr int kMaxDevices = 64;
  thread_local SideStream streams[kMaxDevices][2];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  SideStream& st = streams[dev][high_priority ? 1 : 0];
  if (!st.join) {
    // made in place; a partial set (one creation failed) is kept, released at
    // thread exit, and completed by a later call
    int lo = 0, hi = 0;
    if (high_priority && cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) return nullptr;
    if (!st.s && cudaStreamCreateWithPriority(&st.s, cudaStreamNonBlocking, high_priority ? hi : 0) !=
                     cudaSuccess) {
      st.s = nullptr;
      return nullptr;
    }
    if (!st.fork && cudaEventCreateWithFlags(&st.fork, cudaEventDisableTiming) != cudaSuccess) {
      st.fork = nullptr;
      return nullptr;
    }
    if (cudaEventCreateWithFlags(&st.join, cudaEventDisableTiming) != cudaSuccess) {
      st.join = nullptr;
      return nullptr;
    }
  }
  return &st;
}


int ozaki_default_moduli(int k) {
  const char* env = std::getenv("CFGMM_OZAKI_MODULI");
  if (env) {
    const int v = std::atoi(env);
    if (v >= 2 && v <= kMaxModuli) return v;
  }
  return ozaki_plan(k, 0, kOzakiMinBits).nmod;
}

int ozaki_moduli_for_bits(int k, int bits) { return ozaki_plan(k, 0, bits).nmod; }

size_t ozaki_dgemm_workspace(int m, int n, int k, int nmod) {
  return dgemm_layout(m, n, k, nmod).total;
}

cudaError_t ozaki_dgemm(double* c, const double* a, const double* b, int m, int n, int k,
                        size_t lda, size_t ldb, size_t ldc, bool transa, bool transb, int nmod,
                        void* workspace, cudaStream_t stream, const cudaEvent_t* events,
                        const uint8_t* tab, size_t ldtab, int blk, cudaEvent_t c_ready,
                        int m_layout, int n_layout, bool reuse_a, bool reuse_b) {
  if (tab && transb) return cudaErrorInvalidValue;  // the masked GEMM has no transb
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  auto mark = [&](int i) { if (events) cudaEventRecord(events[i], stream); };
  if (k > kOzakiMaxK) return cudaErrorInvalidValue;
  const OzakiPlan plan = ozaki_plan(k, nmod, 0);
  if (m_layout < m) m_layout = m;
  if (n_layout < n) n_layout = n;
  const DgemmLayout L = dgemm_layout(m_layout, n_layout, k, plan.nmod);
  char* ws = static_cast<char*>(workspace);
  int8_t* a_res = reinterpret_cast<int8_t*>(ws + L.a_res);
  int8_t* b_res = reinterpret_cast<int8_t*>(ws + L.b_res);
  int8_t* r = reinterpret_cast<int8_t*>(ws + L.r);
  int* ea = reinterpret_cast<int*>(ws + L.ea);
  int* eb = reinterpret_cast<int*>(ws + L.eb);
  const ResidueArgs ra = residue_args(plan);
  mark(0);
  // op(A) rows are i (k contiguous unless transa); op(B) "rows" are j
  // (k contiguous only when transb).
  int* emax_a = reinterpret_cast<int*>(ws + L.emax_a);
  int* emax_b = reinterpret_cast<int*>(ws + L.emax_b);
  cudaError_t err = cudaSuccess;
  // With both operands to prepare, A's kernels run on a side stream beside B's:
  // the residue kernels are bound by instruction issue and the exponent scans
  // by DRAM, so the two chains overlap.  The side stream joins back before the
  // GEMM (the fork and join are events, so a stream capture follows them).
  SideScope side((!reuse_a && !reuse_b) ? side_stream() : nullptr, stream);
  if ((err = side.fork()) != cudaSuccess) return err;
  const cudaStream_t sa = side.stream();
  if (!reuse_a) {
    err = prepare(a, lda, !transa, m, k, L.kpad, plan.alpha, emax_a, ea, a_res, ra, sa);
    if (err != cudaSuccess) return err;
  }
  if (!reuse_b) {
    err = prepare(b, ldb, transb, n, k, L.kpad, plan.beta, emax_b, eb, b_res, ra, stream,
                  Mask{tab, ldtab, blk > 0 ? blk : 1});
    if (err != cudaSuccess) return err;
  }
  if ((err = side.join()) != cudaSuccess) return err;

  mark(1);
  CUtensorMap tmA, tmB;
  if (!make_plane_map(&tmA, a_res, k, m, plan.nmod, L.kpad, gemm_i8_tile_rows_a()) ||
      !make_plane_map(&tmB, b_res, k, n, plan.nmod, L.kpad, gemm_i8_tile_rows_b()))
    return cudaErrorInvalidValue;
  GemmI8Args g{};
  g.rows_a = m;
  g.rows_b = n;
  g.k = k;
  g.nmod = plan.nmod;
  g.out = r;
  g.ldr = L.ldr;
  for (int l = 0; l < plan.nmod; ++l) {
    g.mod[l] = plan.mod[l];
    g.inv[l] = plan.inv_f[l];
  }
  if ((err = gemm_i8_mod(tmA, tmB, g, stream)) != cudaSuccess) return err;
  mark(2);

  ReconArgs rc{};
  rc.nmod = plan.nmod;
  for (int l = 0; l < plan.nmod; ++l) {
    rc.w_hi[l] = plan.w_hi[l];
    rc.w_lo[l] = plan.w_lo[l];
  }
  rc.M_hi = plan.M_hi;
  rc.M_lo = plan.M_lo;
  rc.two_T = plan.two_T;
  rc.t_x = plan.t_x;
  rc.t_y = plan.t_y;
  const long long rgrid = (long long)((n + 1023) / 1024) * m;
  if (rgrid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  if (c_ready && (err = cudaStreamWaitEvent(stream, c_ready, 0)) != cudaSuccess) return err;
  reconstruct<<<unsigned(rgrid), 256, 0, stream>>>(c, ldc, m, n, r, L.ldr, ea, eb, rc);
  mark(3);
  return cudaGetLastError();
}

}  // namespace cfgmm
