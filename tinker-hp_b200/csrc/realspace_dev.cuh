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

// pairs loaded ahead per thread in the matvec rows (FP64 / FP32 forms)
#ifndef THP_MATVEC_G64
#define THP_MATVEC_G64 2
#endif
#ifndef THP_MATVEC_G32
#define THP_MATVEC_G32 4
#endif

namespace thp {

struct PairRows {
  int n, npad;
  const int* npr;   // partners per atom
  const int* pk;    // partner index, slot-major [s*npad + i]
  const void* pc3;  // coefficient dmp3 (double or float), slot-major
  const void* pc5;  // coefficient dmp5
};

// G partner pairs of one FP64 row, the partner indices and coefficients
// already loaded: every gather of the group is issued before the arithmetic,
// so each thread keeps several in flight.  The pairs are summed in order.
template <int G>
__device__ __forceinline__ void pairs64(const int (&k)[G], const double (&c3)[G], const double (&c5)[G],
                                        const double4& pi, const Box& box, const double4* __restrict__ pos,
                                        const double* __restrict__ mu, double (&acc)[6]) {
  double4 pk4[G];
  double2 u0[G], u1[G], u2[G];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    pk4[g] = pos[k[g]];
    const double2* m2 = reinterpret_cast<const double2*>(mu + (size_t)k[g] * 6);
    u0[g] = m2[0];
    u1[g] = m2[1];
    u2[g] = m2[2];
  }
#pragma unroll
  for (int g = 0; g < G; ++g) {
    double xr = pk4[g].x - pi.x, yr = pk4[g].y - pi.y, zr = pk4[g].z - pi.z;
    image3(box, xr, yr, zr);
    const double dd = xr * u0[g].x + yr * u0[g].y + zr * u1[g].x;
    const double dp = xr * u1[g].y + yr * u2[g].x + zr * u2[g].y;
    const double sd = c5[g] * dd, sp = c5[g] * dp;
    acc[0] += c3[g] * u0[g].x - sd * xr;
    acc[1] += c3[g] * u0[g].y - sd * yr;
    acc[2] += c3[g] * u1[g].x - sd * zr;
    acc[3] += c3[g] * u1[g].y - sp * xr;
    acc[4] += c3[g] * u2[g].x - sp * yr;
    acc[5] += c3[g] * u2[g].y - sp * zr;
  }
}

// the same for the FP32 row (positions wrapped into the box, half edges h)
template <int G>
__device__ __forceinline__ void pairs32(const int (&k)[G], const float (&c3)[G], const float (&c5)[G],
                                        const float4& pi, float bx, float by, float bz,
                                        const float4* __restrict__ pos, const float* __restrict__ mu,
                                        float (&acc)[6]) {
  const float hx = 0.5f * bx, hy = 0.5f * by, hz = 0.5f * bz;
  float4 pk4[G];
  float2 u0[G], u1[G], u2[G];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    pk4[g] = pos[k[g]];
    const float2* m2 = reinterpret_cast<const float2*>(mu + (size_t)k[g] * 6);
    u0[g] = m2[0];
    u1[g] = m2[1];
    u2[g] = m2[2];
  }
#pragma unroll
  for (int g = 0; g < G; ++g) {
    float xr = pk4[g].x - pi.x, yr = pk4[g].y - pi.y, zr = pk4[g].z - pi.z;
    xr = fabsf(xr) > hx ? xr - copysignf(bx, xr) : xr;
    yr = fabsf(yr) > hy ? yr - copysignf(by, yr) : yr;
    zr = fabsf(zr) > hz ? zr - copysignf(bz, zr) : zr;
    const float dd = xr * u0[g].x + yr * u0[g].y + zr * u1[g].x;
    const float dp = xr * u1[g].y + yr * u2[g].x + zr * u2[g].y;
    const float sd = c5[g] * dd, sp = c5[g] * dp;
    acc[0] += c3[g] * u0[g].x - sd * xr;
    acc[1] += c3[g] * u0[g].y - sd * yr;
    acc[2] += c3[g] * u1[g].x - sd * zr;
    acc[3] += c3[g] * u1[g].y - sp * xr;
    acc[4] += c3[g] * u2[g].x - sp * yr;
    acc[5] += c3[g] * u2[g].y - sp * zr;
  }
}

// FP64 row: positions double4, mu [n][6] double; the partner indices and
// coefficients are read straight from the slot-major stream, THP_MATVEC_G64
// pairs per group.  A short last group repeats slot s with zero coefficients.
__device__ __forceinline__ void tmatxb_row64(const PairRows& pr, const Box& box, int i,
                                             const double4* __restrict__ pos, const double* __restrict__ mu,
                                             double (&acc)[6]) {
  const double4 pi = pos[i];
  const int m = pr.npr[i];
  const int* __restrict__ pk = pr.pk;
  const double* __restrict__ c3p = (const double*)pr.pc3;
  const double* __restrict__ c5p = (const double*)pr.pc5;
  constexpr int G = THP_MATVEC_G64;
  for (int s = 0; s < m; s += G) {
    int k[G];
    double c3[G], c5[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const bool ok = s + g < m;
      const size_t q = (size_t)(ok ? s + g : s) * pr.npad + i;
      k[g] = __ldg(pk + q);
      c3[g] = ok ? __ldg(c3p + q) : 0.0;
      c5[g] = ok ? __ldg(c5p + q) : 0.0;
    }
    pairs64<G>(k, c3, c5, pi, box, pos, mu, acc);
  }
}

// FP32 row (mixed form): positions float4 wrapped into the box, mu [n][6]
// float; THP_MATVEC_G32 pairs per group.
__device__ __forceinline__ void tmatxb_row32(const PairRows& pr, float bx, float by, float bz, int i,
                                             const float4* __restrict__ pos, const float* __restrict__ mu,
                                             float (&acc)[6]) {
  const float4 pi = pos[i];
  const int m = pr.npr[i];
  const int* __restrict__ pk = pr.pk;
  const float* __restrict__ c3p = (const float*)pr.pc3;
  const float* __restrict__ c5p = (const float*)pr.pc5;
  constexpr int G = THP_MATVEC_G32;
  for (int s = 0; s < m; s += G) {
    int k[G];
    float c3[G], c5[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const bool ok = s + g < m;
      const size_t q = (size_t)(ok ? s + g : s) * pr.npad + i;
      k[g] = __ldg(pk + q);
      c3[g] = ok ? __ldg(c3p + q) : 0.f;
      c5[g] = ok ? __ldg(c5p + q) : 0.f;
    }
    pairs32<G>(k, c3, c5, pi, bx, by, bz, pos, mu, acc);
  }
}

// Stream loads of the CG rows, read once per matvec.  NOL1: not kept in L1,
// so the partner records gathered beside them stay resident (used when the
// stream streams from DRAM; an L2-resident stream does better cached).
template <bool NOL1>
__device__ __forceinline__ int ld_stream(const int* p) {
  if constexpr (NOL1) {
    int v;
    asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
  } else {
    return __ldg(p);
  }
}
template <bool NOL1>
__device__ __forceinline__ float ld_stream(const float* p) {
  if constexpr (NOL1) {
    float v;
    asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
  } else {
    return __ldg(p);
  }
}

// 256-bit read-only load of one 32-byte aligned record
__device__ __forceinline__ void ld_rec8(const float* p, float (&v)[8]) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
      : "l"(p));
}

// FP32 row over the atom records (rec[k] = {x, y, z, d dipole, p dipole x, y},
// mpz[k] = p dipole z): two gathers per partner instead of four (position,
// then the six dipole components in three pieces).  The partner gathers of
// this kernel are scattered, and each one costs the L1 data pipe about one
// wavefront per distinct cache line touched, so halving them halves the
// pipe's work.  The arithmetic and the order of the sums are those of
// pairs32.
template <bool NOL1>
__device__ __forceinline__ void tmatxb_row32_rec(const PairRows& pr, float bx, float by, float bz, int i,
                                                 const float* __restrict__ rec, const float* __restrict__ mpz,
                                                 float (&acc)[6]) {
  const float4 pi = *reinterpret_cast<const float4*>(rec + (size_t)i * 8);
  const int m = pr.npr[i];
  const int* __restrict__ pk = pr.pk;
  const float* __restrict__ c3p = (const float*)pr.pc3;
  const float* __restrict__ c5p = (const float*)pr.pc5;
  const float hx = 0.5f * bx, hy = 0.5f * by, hz = 0.5f * bz;
  constexpr int G = THP_MATVEC_G32;
  for (int s = 0; s < m; s += G) {
    int k[G];
    float c3[G], c5[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const bool ok = s + g < m;
      const size_t q = (size_t)(ok ? s + g : s) * pr.npad + i;
      k[g] = ld_stream<NOL1>(pk + q);
      c3[g] = ok ? ld_stream<NOL1>(c3p + q) : 0.f;
      c5[g] = ok ? ld_stream<NOL1>(c5p + q) : 0.f;
    }
    float v[G][8], w[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      ld_rec8(rec + (size_t)k[g] * 8, v[g]);
      w[g] = __ldg(mpz + k[g]);
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      float xr = v[g][0] - pi.x, yr = v[g][1] - pi.y, zr = v[g][2] - pi.z;
      xr = fabsf(xr) > hx ? xr - copysignf(bx, xr) : xr;
      yr = fabsf(yr) > hy ? yr - copysignf(by, yr) : yr;
      zr = fabsf(zr) > hz ? zr - copysignf(bz, zr) : zr;
      const float dd = xr * v[g][3] + yr * v[g][4] + zr * v[g][5];
      const float dp = xr * v[g][6] + yr * v[g][7] + zr * w[g];
      const float sd = c5[g] * dd, sp = c5[g] * dp;
      acc[0] += c3[g] * v[g][3] - sd * xr;
      acc[1] += c3[g] * v[g][4] - sd * yr;
      acc[2] += c3[g] * v[g][5] - sd * zr;
      acc[3] += c3[g] * v[g][6] - sp * xr;
      acc[4] += c3[g] * v[g][7] - sp * yr;
      acc[5] += c3[g] * w[g] - sp * zr;
    }
  }
}

}  // namespace thp
