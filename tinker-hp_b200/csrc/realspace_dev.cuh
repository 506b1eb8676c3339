// realspace_dev.cuh -- device side of the real-space dipole-dipole matvec.
//
// tmatxb_pme (newinduce_pme.f:1392-1668) restated for a full per-atom list
// with the per-pair mutual coefficients precomputed once per solve:
//   dmp3 = B1 - (1 - u*l3)/r^3,  dmp5 = B2 - 3(1 - u*l5)/r^5
// (dampewald order 7 + dampthole order 5), summed as
//   efi_i = -sum_k (dmp5 r (r.mu_k) - dmp3 mu_k).
//
// Work split: atoms (in cell-sorted order) form groups of four consecutive
// atoms, and one warp sums one group's rows: eight lanes per atom, lane j
// taking the atom's partners j, j+8, j+16, ...  An atom's partners are in
// ascending index within each cell row, so eight consecutive partners lie
// in a few consecutive partner records, and the four atoms of a group, close
// in space, share most of them: a warp's 32 partner gathers touch about 16
// cache lines, where one atom per lane touched about 29.  The eight partial
// sums of an atom are combined with warp shuffles in a fixed tree, so the
// result is reproducible bit for bit.
//
// The pair stream is laid out for this split (pair_slot): a group's slots
// come in blocks of 32 entries, 8 consecutive slots of each of its four
// atoms side by side, so one warp step reads 32 consecutive entries: the
// partner index (pk) and the two coefficients side by side (pcc).
#pragma once

#include "common.cuh"

namespace thp {

struct PairRows {
  int n;
  int cap8;         // slot blocks of 8 per atom (capacity maxpr = 8 cap8)
  const int* npr;   // partners per atom
  const int* pk;    // partner index, at pair_slot(cap8, i, s)
  const void* pcc;  // (dmp3, dmp5) as double2 or float2, at the same entries
};

// Entry of slot s of atom i in the pair stream.
__host__ __device__ __forceinline__ size_t pair_slot(int cap8, int i, int s) {
  return ((size_t)(i >> 2) * (size_t)cap8 + (size_t)(s >> 3)) * 32 + (size_t)((i & 3) << 3) + (size_t)(s & 7);
}

constexpr unsigned kFullMask = 0xffffffffu;

// Stream loads of the rows, read once per matvec.  NOL1: not kept in L1, so
// the partner records gathered beside them stay resident (used when the
// stream comes from DRAM; an L2-resident stream does better cached).
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
__device__ __forceinline__ float2 ld_stream(const float2* p) {
  if constexpr (NOL1) {
    float2 v;
    asm("ld.global.nc.L1::no_allocate.v2.f32 {%0,%1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
  } else {
    return __ldg(p);
  }
}
template <bool NOL1>
__device__ __forceinline__ double2 ld_stream(const double2* p) {
  if constexpr (NOL1) {
    double2 v;
    asm("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
  } else {
    return __ldg(p);
  }
}

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

// 256-bit read-only load of one 32-byte aligned record
__device__ __forceinline__ void ld_rec8(const float* p, float (&v)[8]) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
      : "l"(p));
}

// Partner data of the three row forms: position (in the form's own frame)
// and the six dipole components (d xyz, p xyz) of atom k.
struct Partner64 {  // FP64: double4 positions as given, mu [n][6] double
  const double4* __restrict__ pos;
  const double* __restrict__ mu;
  __device__ __forceinline__ void load(int k, double (&p)[3], double (&u)[6]) const {
    const double4 q = pos[k];
    const double2* m2 = reinterpret_cast<const double2*>(mu + (size_t)k * 6);
    const double2 a = m2[0], b = m2[1], c = m2[2];
    p[0] = q.x; p[1] = q.y; p[2] = q.z;
    u[0] = a.x; u[1] = a.y; u[2] = b.x; u[3] = b.y; u[4] = c.x; u[5] = c.y;
  }
};
struct Partner32 {  // FP32: float4 positions wrapped into the box, mu [n][6] float
  const float4* __restrict__ pos;
  const float* __restrict__ mu;
  __device__ __forceinline__ void load(int k, float (&p)[3], float (&u)[6]) const {
    const float4 q = pos[k];
    const float2* m2 = reinterpret_cast<const float2*>(mu + (size_t)k * 6);
    const float2 a = m2[0], b = m2[1], c = m2[2];
    p[0] = q.x; p[1] = q.y; p[2] = q.z;
    u[0] = a.x; u[1] = a.y; u[2] = b.x; u[3] = b.y; u[4] = c.x; u[5] = c.y;
  }
};
// FP32 atom records (rec[k] = {x, y, z, d dipole, p dipole x, y} with the
// position wrapped into the box, mpz[k] = p dipole z): two gathers per
// partner, one of them a 256-bit load.
struct PartnerRec {
  const float* __restrict__ rec;
  const float* __restrict__ mpz;
  __device__ __forceinline__ void load(int k, float (&p)[3], float (&u)[6]) const {
    float v[8];
    ld_rec8(rec + (size_t)k * 8, v);
    p[0] = v[0]; p[1] = v[1]; p[2] = v[2];
    u[0] = v[3]; u[1] = v[4]; u[2] = v[5]; u[3] = v[6]; u[4] = v[7];
    u[5] = __ldg(mpz + k);
  }
};

// Displacement imaged into the box: FP64 by image.f's rule, FP32 by one wrap
// of coordinates that already lie in the box.
struct Image64 {
  Box box;
  __device__ __forceinline__ void apply(double& x, double& y, double& z) const { image3(box, x, y, z); }
};
struct Image32 {
  float bx, by, bz;
  __device__ __forceinline__ void apply(float& x, float& y, float& z) const {
    x = fabsf(x) > 0.5f * bx ? x - copysignf(bx, x) : x;
    y = fabsf(y) > 0.5f * by ? y - copysignf(by, y) : y;
    z = fabsf(z) > 0.5f * bz ? z - copysignf(bz, z) : z;
  }
};

// 1: the stream entries of a round's U blocks are loaded one round ahead of
// their partner gathers, so the stream's DRAM latency overlaps the gathers
// and arithmetic of the round before
#ifndef THP_GROW_PF
#define THP_GROW_PF 1
#endif

// Stream entries (partner, dmp3, dmp5) of the U blocks of one round for this
// lane; a slot past the atom's count (8 b < mj fails) gives the lane's own
// atom with zero coefficients.  Blocks past the group's last (the same for
// the whole warp) are not read at all.
template <typename T, int U, bool NOL1>
__device__ __forceinline__ void stream_round(const int* pk, const typename Vec2<T>::type* pc, int b, int mj,
                                             int nblk, int i_safe, int (&k)[U], T (&c3)[U], T (&c5)[U]) {
  using T2 = typename Vec2<T>::type;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    k[u] = i_safe;
    c3[u] = T(0);
    c5[u] = T(0);
    if (b + u < nblk) {
      const int kr = ld_stream<NOL1>(pk + 32 * u);
      const T2 cr = ld_stream<NOL1>(pc + 32 * u);
      const bool ok = 8 * (b + u) < mj;
      k[u] = ok ? kr : i_safe;
      c3[u] = ok ? cr.x : T(0);
      c5[u] = ok ? cr.y : T(0);
    }
  }
}

// One lane's share of the row of atom i (slots j, j+8, j+16, ... of its m
// partners), U blocks of slots per round.  base = this lane's entry in the
// group's first block.  Every lane of the warp loads every block of a round
// up to the group's last; a slot past m counts as the lane's own atom with
// zero coefficients.  WRAP = false skips the periodic wrap: the caller has
// checked that the group's atoms lie farther than the cutoff from every face
// of the box, so no pair crosses one.
template <typename T, int U, bool NOL1, bool WRAP, typename Ld, typename Im>
__device__ __forceinline__ void group_row_part(const PairRows& pr, const Ld& ld, const Im& im, const T (&pi)[3],
                                               int i_safe, int j, int m, int nblk, size_t base, T (&acc)[6]) {
  using T2 = typename Vec2<T>::type;
  const int* __restrict__ pk = pr.pk + base;
  const T2* __restrict__ pc = (const T2*)pr.pcc + base;
  const int mj = m - j;  // slot 8 b + j is a partner while 8 b < mj
  int k[U];
  T c3[U], c5[U];
  if (THP_GROW_PF) stream_round<T, U, NOL1>(pk, pc, 0, mj, nblk, i_safe, k, c3, c5);
#pragma unroll 1
  for (int b = 0; b < nblk; b += U) {
    if (!THP_GROW_PF) stream_round<T, U, NOL1>(pk + 32 * b, pc + 32 * b, b, mj, nblk, i_safe, k, c3, c5);
    T p[U][3], w[U][6];
#pragma unroll
    for (int u = 0; u < U; ++u) ld.load(k[u], p[u], w[u]);
    int kn[U];
    T c3n[U], c5n[U];
    if (THP_GROW_PF)
      stream_round<T, U, NOL1>(pk + 32 * (b + U), pc + 32 * (b + U), b + U, mj, nblk, i_safe, kn, c3n, c5n);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      T xr = p[u][0] - pi[0], yr = p[u][1] - pi[1], zr = p[u][2] - pi[2];
      if (WRAP) im.apply(xr, yr, zr);
      const T dd = xr * w[u][0] + yr * w[u][1] + zr * w[u][2];
      const T dp = xr * w[u][3] + yr * w[u][4] + zr * w[u][5];
      const T sd = c5[u] * dd, sp = c5[u] * dp;
      acc[0] += c3[u] * w[u][0] - sd * xr;
      acc[1] += c3[u] * w[u][1] - sd * yr;
      acc[2] += c3[u] * w[u][2] - sd * zr;
      acc[3] += c3[u] * w[u][3] - sp * xr;
      acc[4] += c3[u] * w[u][4] - sp * yr;
      acc[5] += c3[u] * w[u][5] - sp * zr;
    }
    if (THP_GROW_PF) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        k[u] = kn[u];
        c3[u] = c3n[u];
        c5[u] = c5n[u];
      }
    }
  }
}

// The whole row of the lane's atom i = 4 g + (lane >> 3), summed over its
// eight lanes; every lane of the atom returns the total.  Lanes of atoms
// past n (the last group) return zeros.  All 32 lanes of the warp must call.
// interior: a group whose atoms all have |coordinate| <= interior (in the
// frame the partner data holds) skips the periodic wrap; pass a negative
// bound where that frame is not the wrapped box.
template <typename T, int U, bool NOL1, typename Ld, typename Im>
__device__ __forceinline__ void group_row(const PairRows& pr, const Ld& ld, const Im& im, int g, int lane,
                                          T (&acc)[6], T interior) {
  const int a = lane >> 3, j = lane & 7;
  const int i = 4 * g + a;
  const bool live = i < pr.n;
  const int m = live ? __ldg(pr.npr + i) : 0;
  int mb = max(m, __shfl_xor_sync(kFullMask, m, 8));
  mb = max(mb, __shfl_xor_sync(kFullMask, mb, 16));
  const int nblk = (mb + 7) >> 3;
  const int i_safe = live ? i : 4 * g;
  T pi[3], wi[6];
  ld.load(i_safe, pi, wi);
#pragma unroll
  for (int q = 0; q < 6; ++q) acc[q] = T(0);
  const bool inside = fabs(pi[0]) <= interior && fabs(pi[1]) <= interior && fabs(pi[2]) <= interior;
  const size_t base = (size_t)g * pr.cap8 * 32 + lane;
  if (__all_sync(kFullMask, inside))
    group_row_part<T, U, NOL1, false>(pr, ld, im, pi, i_safe, j, m, nblk, base, acc);
  else
    group_row_part<T, U, NOL1, true>(pr, ld, im, pi, i_safe, j, m, nblk, base, acc);
#pragma unroll
  for (int o = 4; o > 0; o >>= 1)
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] += __shfl_xor_sync(kFullMask, acc[q], o);
}

// Component j (0..5) of a six-vector held in registers, without local memory.
template <typename T>
__device__ __forceinline__ T pick6(const T (&v)[6], int j) {
  T r = v[0];
  r = j == 1 ? v[1] : r;
  r = j == 2 ? v[2] : r;
  r = j == 3 ? v[3] : r;
  r = j == 4 ? v[4] : r;
  r = j == 5 ? v[5] : r;
  return r;
}

// An atom's eight lanes' partial sums combined (fixed tree); every lane of
// the atom gets the total.
template <int NV>
__device__ __forceinline__ void lane8_sum(double (&v)[NV]) {
#pragma unroll
  for (int o = 4; o > 0; o >>= 1)
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] += __shfl_xor_sync(kFullMask, v[q], o);
}

}  // namespace thp
