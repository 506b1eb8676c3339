// realspace_dev.cuh -- device side of the real-space dipole-dipole matvec.
//
// tmatxb_pme (newinduce_pme.f:1392-1668) restated for a full per-atom list
// with the per-pair mutual coefficients precomputed once per solve:
//   dmp3 = B1 - (1 - u*l3)/r^3,  dmp5 = B2 - 3(1 - u*l5)/r^5
// (dampewald order 7 + dampthole order 5).  One thread owns atom i and sums
//   efi_i = -sum_k (dmp5 r (r.mu_k) - dmp3 mu_k)
// over its interacting partners, so no atomics are needed and the result is
// bitwise reproducible.
#pragma once

#include "common.cuh"

namespace thp {

struct PairRows {
  int n, npad;
  const int* npr;   // partners per atom
  const int* pk;    // partner index, slot-major [s*npad + i]
  const void* pc3;  // coefficient dmp3 (double or float), slot-major
  const void* pc5;  // coefficient dmp5
};

// FP64 row: positions double4, mu [n][6] double
__device__ __forceinline__ void tmatxb_row64(const PairRows& pr, const Box& box, int i,
                                             const double4* __restrict__ pos, const double* __restrict__ mu,
                                             double (&acc)[6]) {
  const double4 pi = pos[i];
  const int m = pr.npr[i];
  const int* __restrict__ pk = pr.pk;
  const double* __restrict__ c3p = (const double*)pr.pc3;
  const double* __restrict__ c5p = (const double*)pr.pc5;
#pragma unroll 1
  for (int s = 0; s < m; ++s) {
    const size_t q = (size_t)s * pr.npad + i;
    const int k = __ldg(pk + q);
    const double c3 = __ldg(c3p + q), c5 = __ldg(c5p + q);
    const double4 pk4 = pos[k];
    double xr = pk4.x - pi.x, yr = pk4.y - pi.y, zr = pk4.z - pi.z;
    image3(box, xr, yr, zr);
    const double2* m2 = reinterpret_cast<const double2*>(mu + (size_t)k * 6);
    const double2 u0 = m2[0], u1 = m2[1], u2 = m2[2];
    const double dd = xr * u0.x + yr * u0.y + zr * u1.x;
    const double dp = xr * u1.y + yr * u2.x + zr * u2.y;
    const double sd = c5 * dd, sp = c5 * dp;
    acc[0] += c3 * u0.x - sd * xr;
    acc[1] += c3 * u0.y - sd * yr;
    acc[2] += c3 * u1.x - sd * zr;
    acc[3] += c3 * u1.y - sp * xr;
    acc[4] += c3 * u2.x - sp * yr;
    acc[5] += c3 * u2.y - sp * zr;
  }
}

// FP32 row (mixed form): positions float4 wrapped into the box, mu [n][6] float
__device__ __forceinline__ void tmatxb_row32(const PairRows& pr, float bx, float by, float bz, int i,
                                             const float4* __restrict__ pos, const float* __restrict__ mu,
                                             float (&acc)[6]) {
  const float4 pi = pos[i];
  const int m = pr.npr[i];
  const int* __restrict__ pk = pr.pk;
  const float* __restrict__ c3p = (const float*)pr.pc3;
  const float* __restrict__ c5p = (const float*)pr.pc5;
  const float hx = 0.5f * bx, hy = 0.5f * by, hz = 0.5f * bz;
#pragma unroll 2
  for (int s = 0; s < m; ++s) {
    const size_t q = (size_t)s * pr.npad + i;
    const int k = __ldg(pk + q);
    const float c3 = __ldg(c3p + q), c5 = __ldg(c5p + q);
    const float4 pk4 = pos[k];
    float xr = pk4.x - pi.x, yr = pk4.y - pi.y, zr = pk4.z - pi.z;
    xr = fabsf(xr) > hx ? xr - copysignf(bx, xr) : xr;
    yr = fabsf(yr) > hy ? yr - copysignf(by, yr) : yr;
    zr = fabsf(zr) > hz ? zr - copysignf(bz, zr) : zr;
    const float2* m2 = reinterpret_cast<const float2*>(mu + (size_t)k * 6);
    const float2 u0 = m2[0], u1 = m2[1], u2 = m2[2];
    const float dd = xr * u0.x + yr * u0.y + zr * u1.x;
    const float dp = xr * u1.y + yr * u2.x + zr * u2.y;
    const float sd = c5 * dd, sp = c5 * dp;
    acc[0] += c3 * u0.x - sd * xr;
    acc[1] += c3 * u0.y - sd * yr;
    acc[2] += c3 * u1.x - sd * zr;
    acc[3] += c3 * u1.y - sp * xr;
    acc[4] += c3 * u2.x - sp * yr;
    acc[5] += c3 * u2.y - sp * zr;
  }
}

}  // namespace thp
