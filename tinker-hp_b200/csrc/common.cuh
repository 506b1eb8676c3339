// common.cuh -- shared device/host helpers of the B200 polarization library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "../../include/thp.h"

#define THP_WARP 32

namespace thp {

constexpr double kPi = 3.141592653589793238;
constexpr double kSqrtPi = 1.772453850905516027;
constexpr double kElectric = 332.063714;        // MOD_units.f:81
constexpr double kTinyPol = (double)1e-5f;      // MOD_polar.f:36 (single-precision literal)

// Orthogonal periodic box, the reference's replicated cell (lattice.f:35-45).
struct Box {
  double l[3];      // xcell, ycell, zcell
  double half[3];   // xcell2 ...
  double recip[3];  // recip(d,d) of lattice.f:111-120 (diagonal for orthogonal boxes)
};

// image.f:122-138, orthogonal branch, with explicitly unfused arithmetic so
// the result is bit-identical to the reference's scalar Fortran.
__device__ __forceinline__ double image1(double r, double cell, double cell2) {
  if (fabs(r) > cell2) {
    double cel = copysign(cell, r);
    double f = floor(__ddiv_rn(fabs(r), cell));
    r = __dadd_rn(r, -__dmul_rn(cel, f));
    if (fabs(r) > cell2) r = __dadd_rn(r, -copysign(cell, r));
  }
  return r;
}

// r^2 = x*x + y*y + z*z evaluated left to right without contraction
// (nblist.f:214-222, newinduce_pme.f:1163).
__device__ __forceinline__ double r2_exact(double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

__device__ __forceinline__ void image3(const Box& b, double& x, double& y, double& z) {
  x = image1(x, b.l[0], b.half[0]);
  y = image1(y, b.l[1], b.half[1]);
  z = image1(z, b.l[2], b.half[2]);
}

// Deterministic block reduction of NV doubles (blockDim.x multiple of 32,
// at most 1024 threads).  Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV]) {
  __shared__ double sred[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) sred[q][wid] = v[q];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double t = lane < nw ? sred[q][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      v[q] = t;
    }
  }
  __syncthreads();
}

}  // namespace thp
