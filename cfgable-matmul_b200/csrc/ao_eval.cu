// ao_eval.cu -- the step before the contraction: Gaussian atomic orbitals on
// the grid, evaluated on the device so phi never crosses PCIe.
//
//   phi[row0(sh) + f][g] = N_sh exp(-alpha_sh r^2) Y_f(x, y, z),
//   (x, y, z) = point g - centre of shell sh, r^2 = x^2 + y^2 + z^2,
// with Y_f the 2l+1 real solid harmonics (unnormalised polynomials) of the
// shell's angular momentum l <= 3, in the order
//   l=0: 1;  l=1: x, y, z;  l=2: xy, yz, 3z^2-r^2, xz, x^2-y^2;
//   l=3: y(3x^2-y^2), xyz, y(5z^2-r^2), z(5z^2-3r^2), x(5z^2-r^2), z(x^2-y^2), x(x^2-3y^2).
// The kernel also records max_g |phi| per (shell, block of `blksize`
// points); a second kernel turns a threshold on those maxima into the
// per-(AO, block) mask of the contraction (rows of one shell share a mask, as
// in a non0tab) and zeroes phi outside it.
#include <cuda_runtime.h>

#include <cstdint>

#include "ao_eval.cuh"

namespace cfgmm {
namespace {

__device__ __forceinline__ int harmonics(int l, double x, double y, double z, double* out) {
  if (l == 0) {
    out[0] = 1.0;
    return 1;
  }
  if (l == 1) {
    out[0] = x;
    out[1] = y;
    out[2] = z;
    return 3;
  }
  const double r2 = x * x + y * y + z * z;
  if (l == 2) {
    out[0] = x * y;
    out[1] = y * z;
    out[2] = 3.0 * z * z - r2;
    out[3] = x * z;
    out[4] = x * x - y * y;
    return 5;
  }
  out[0] = y * (3.0 * x * x - y * y);
  out[1] = x * y * z;
  out[2] = y * (5.0 * z * z - r2);
  out[3] = z * (5.0 * z * z - 3.0 * r2);
  out[4] = x * (5.0 * z * z - r2);
  out[5] = z * (x * x - y * y);
  out[6] = x * (x * x - 3.0 * y * y);
  return 7;
}

// one CTA per (block of `blksize` points, up to 256 points) x 8 shells; a
// thread per point, looping over its shells
__global__ void __launch_bounds__(256)
eval_ao(double* __restrict__ ao, size_t stride_grid, const double* __restrict__ pts, int ngrid,
        const double* __restrict__ sxyz, const int* __restrict__ sl, const double* __restrict__ salpha,
        const double* __restrict__ snorm, const int* __restrict__ srow, int nshell,
        double* __restrict__ bmax, int blksize, int nblk) {
  const int g = blockIdx.x * 256 + threadIdx.x;
  const int sh0 = blockIdx.y * 8;
  const bool ok = g < ngrid;
  double px = 0, py = 0, pz = 0;
  if (ok) {
    px = pts[3 * size_t(g)];
    py = pts[3 * size_t(g) + 1];
    pz = pts[3 * size_t(g) + 2];
  }
  for (int sh = sh0; sh < min(nshell, sh0 + 8); ++sh) {
    const double x = px - sxyz[3 * sh], y = py - sxyz[3 * sh + 1], z = pz - sxyz[3 * sh + 2];
    double Y[7];
    const int nf = harmonics(sl[sh], x, y, z, Y);
    const double rad = snorm[sh] * exp(-salpha[sh] * (x * x + y * y + z * z));
    double m = 0.0;
    for (int f = 0; f < nf; ++f) {
      const double v = rad * Y[f];
      if (ok) ao[size_t(srow[sh] + f) * stride_grid + g] = v;
      m = fmax(m, fabs(v));
    }
    if (bmax) {  // max over the points of each block: warp reduce, then atomic max
      const int b = ok ? g / blksize : -1;
      // points of one warp may straddle blocks: reduce per block id
      for (int o = 16; o > 0; o >>= 1) {
        const double mo = __shfl_down_sync(0xffffffffu, m, o);
        const int bo = __shfl_down_sync(0xffffffffu, b, o);
        if ((threadIdx.x & 31) + o < 32 && bo == b) m = fmax(m, mo);
      }
      const int bprev = __shfl_up_sync(0xffffffffu, b, 1);
      const bool leader = ok && ((threadIdx.x & 31) == 0 || bprev != b);
      if (leader && b < nblk) {
        // non-negative doubles order like their bit patterns
        atomicMax(reinterpret_cast<unsigned long long*>(bmax + size_t(sh) * nblk + b),
                  static_cast<unsigned long long>(__double_as_longlong(m)));
      }
    }
  }
}

// tab[row][b] = bmax[sh][b] > thr for every row of shell sh; phi zeroed where 0
__global__ void __launch_bounds__(256)
mask_ao(double* __restrict__ ao, size_t stride_grid, int ngrid, const int* __restrict__ sl,
        const int* __restrict__ srow, int nshell, const double* __restrict__ bmax, double thr,
        uint8_t* __restrict__ tab, size_t ldtab, int blksize, int nblk) {
  const int sh = blockIdx.y;
  const int nf = 2 * sl[sh] + 1;
  for (int g = blockIdx.x * 256 + threadIdx.x; g < ngrid; g += gridDim.x * 256) {
    const int b = g / blksize;
    const bool on = bmax[size_t(sh) * nblk + b] > thr;
    if (!on)
      for (int f = 0; f < nf; ++f) ao[size_t(srow[sh] + f) * stride_grid + g] = 0.0;
    if (g % blksize == 0)
      for (int f = 0; f < nf; ++f) tab[size_t(srow[sh] + f) * ldtab + b] = on ? 1 : 0;
  }
}

}  // namespace

cudaError_t eval_ao(double* ao, size_t stride_grid, const double* pts, int ngrid, const double* sxyz,
                    const int* sl, const double* salpha, const double* snorm, const int* srow,
                    int nshell, double* bmax, int blksize, cudaStream_t stream) {
  if (ngrid <= 0 || nshell <= 0) return cudaSuccess;
  const int nblk = (ngrid + blksize - 1) / blksize;
  if (bmax) {
    cudaError_t err = cudaMemsetAsync(bmax, 0, size_t(nshell) * nblk * sizeof(double), stream);
    if (err != cudaSuccess) return err;
  }
  dim3 grid((ngrid + 255) / 256, (nshell + 7) / 8);
  eval_ao<<<grid, 256, 0, stream>>>(ao, stride_grid, pts, ngrid, sxyz, sl, salpha, snorm, srow,
                                    nshell, bmax, blksize, nblk);
  return cudaGetLastError();
}

cudaError_t mask_ao(double* ao, size_t stride_grid, int ngrid, const int* sl, const int* srow,
                    int nshell, const double* bmax, double thr, uint8_t* tab, size_t ldtab,
                    int blksize, cudaStream_t stream) {
  if (ngrid <= 0 || nshell <= 0) return cudaSuccess;
  const int nblk = (ngrid + blksize - 1) / blksize;
  dim3 grid(min((ngrid + 255) / 256, 1024), nshell);
  mask_ao<<<grid, 256, 0, stream>>>(ao, stride_grid, ngrid, sl, srow, nshell, bmax, thr, tab,
                                    ldtab, blksize, nblk);
  return cudaGetLastError();
}

}  // namespace cfgmm
