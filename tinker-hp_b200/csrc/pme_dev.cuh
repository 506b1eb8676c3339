// pme_dev.cuh -- device helpers of the smooth-PME dipole/multipole passes.
#pragma once

#include <cufft.h>

#include <type_traits>

#include "common.cuh"

namespace thp {

constexpr int kBs = 5;  // B-spline order (kewald.f:78 bsporder)

// bsplgen (pmestuff.f:64-157) for order 5: th[m][lev] = thetai(lev+1, m+1).
// LEVEL = number of derivative levels kept (value, 1st, 2nd, 3rd).
template <int LEVEL, typename T>
__device__ __forceinline__ void bsplgen5(T w, T (&th)[kBs][LEVEL]) {
  T t[6][6];  // 1-based rows/cols as in the reference
  const T one = T(1), half = T(0.5);
  t[2][2] = w;
  t[2][1] = one - w;
  t[3][3] = half * w * t[2][2];
  t[3][2] = half * ((one + w) * t[2][1] + (T(2) - w) * t[2][2]);
  t[3][1] = half * (one - w) * t[2][1];
#pragma unroll
  for (int i = 4; i <= kBs; ++i) {
    const int k = i - 1;
    const T denom = one / T(k);
    t[i][i] = denom * w * t[k][k];
#pragma unroll
    for (int j = 1; j <= i - 2; ++j)
      t[i][i - j] = denom * ((w + T(j)) * t[k][i - j - 1] + (T(i - j) - w) * t[k][i - j]);
    t[i][1] = denom * (one - w) * t[k][1];
  }
  // first derivative
  {
    const int k = kBs - 1;
    t[k][kBs] = t[k][kBs - 1];
#pragma unroll
    for (int i = kBs - 1; i >= 2; --i) t[k][i] = t[k][i - 1] - t[k][i];
    t[k][1] = -t[k][1];
  }
  if (LEVEL >= 3) {
    const int k = kBs - 2;
    t[k][kBs - 1] = t[k][kBs - 2];
#pragma unroll
    for (int i = kBs - 2; i >= 2; --i) t[k][i] = t[k][i - 1] - t[k][i];
    t[k][1] = -t[k][1];
    t[k][kBs] = t[k][kBs - 1];
#pragma unroll
    for (int i = kBs - 1; i >= 2; --i) t[k][i] = t[k][i - 1] - t[k][i];
    t[k][1] = -t[k][1];
  }
  if (LEVEL >= 4) {
    const int k = kBs - 3;
    t[k][kBs - 2] = t[k][kBs - 3];
#pragma unroll
    for (int i = kBs - 3; i >= 2; --i) t[k][i] = t[k][i - 1] - t[k][i];
    t[k][1] = -t[k][1];
    t[k][kBs - 1] = t[k][kBs - 2];
#pragma unroll
    for (int i = kBs - 2; i >= 2; --i) t[k][i] = t[k][i - 1] - t[k][i];
    t[k][1] = -t[k][1];
    t[k][kBs] = t[k][kBs - 1];
#pragma unroll
    for (int i = kBs - 1; i >= 2; --i) t[k][i] = t[k][i - 1] - t[k][i];
    t[k][1] = -t[k][1];
  }
#pragma unroll
  for (int m = 1; m <= kBs; ++m)
#pragma unroll
    for (int lev = 1; lev <= LEVEL; ++lev) th[m - 1][lev - 1] = t[kBs - lev + 1][m];
}

// bspline_fill_site (pmestuff.f:13-51), one axis: returns the 0-based grid
// index of the first stencil point (may be negative, >= -4) and the weights.
template <int LEVEL, typename T>
__device__ __forceinline__ int bspline_axis(double coord, double recip, int nfft, T (&th)[kBs][LEVEL]) {
  double w = coord * recip;
  double fr = (double)nfft * (w - round(w) + 0.5);
  int ifr = (int)(fr - 1.0e-8);
  ifr = ifr < 0 ? 0 : (ifr >= nfft ? nfft - 1 : ifr);  // keeps every stencil index inside the grid
  T wf = (T)(fr - (double)ifr);
  bsplgen5<LEVEL, T>(wf, th);
  return ifr - 4;  // reference igrid = ifr - bsorder; first point igrid + 1
}

__device__ __forceinline__ int wrapk(int v, int n) { return v < 0 ? v + n : v; }

struct PmeGeom {
  int n1, n2, n3;
  double recip[3];
  double a[3];  // nfft_d * recip(d,d)
};

template <typename T>
struct Cplx;
template <>
struct Cplx<double> {
  using type = cufftDoubleComplex;
};
template <>
struct Cplx<float> {
  using type = cufftComplex;
};


// Fire-and-forget reductions (PTX red): the spread never reads the old value,
// so no thread waits on the atomic's return.
__device__ __forceinline__ void red_add(double* a, double v) {
  asm volatile("red.global.add.f64 [%0], %1;" ::"l"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void red_add(float* a, float v) {
  asm volatile("red.global.add.f32 [%0], %1;" ::"l"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void red_add2(float* a, float x, float y) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(a), "f"(x), "f"(y) : "memory");
}
__device__ __forceinline__ void grid_add(cufftDoubleComplex* g, size_t idx, double re, double im) {
  red_add(&g[idx].x, re);
  red_add(&g[idx].y, im);
}
__device__ __forceinline__ void grid_add(cufftComplex* g, size_t idx, float re, float im) {
  red_add2(&g[idx].x, re, im);
}
// 1: neighbouring grid points of a stencil row share one reduction where
// alignment allows (FP32 grid)
#ifndef THP_SPREAD_PAIRS
#define THP_SPREAD_PAIRS 1
#endif

// two neighbouring complex points of the FP32 grid in one reduction; the
// caller guarantees idx is even (a 16-byte boundary) and idx + 1 is the
// next point of the same row
__device__ __forceinline__ void grid_add_pair(cufftComplex* g, size_t idx, float re0, float im0, float re1,
                                              float im1) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(&g[idx].x), "f"(re0), "f"(im0), "f"(re1),
               "f"(im1)
               : "memory");
}
__device__ __forceinline__ void grid_add_pair(cufftDoubleComplex* g, size_t idx, double re0, double im0, double re1,
                                              double im1) {
  grid_add(g, idx, re0, im0);
  grid_add(g, idx + 1, re1, im1);
}

// grid_uind_site (pmestuff.f:280-405) for one site: d dipole components
// v[0..2] into Re, p dipole v[3..5] into Im of the 125 stencil points.
template <typename T>
__device__ __forceinline__ void spread_dip_site(const PmeGeom& g, double4 p, const double (&v)[6],
                                                typename Cplx<T>::type* __restrict__ grid) {
  T tx[kBs][2], ty[kBs][2], tz[kBs][2];
  int gx = bspline_axis<2, T>(p.x, g.recip[0], g.n1, tx);
  int gy = bspline_axis<2, T>(p.y, g.recip[1], g.n2, ty);
  int gz = bspline_axis<2, T>(p.z, g.recip[2], g.n3, tz);
  T fd[3] = {(T)(g.a[0] * v[0]), (T)(g.a[1] * v[1]), (T)(g.a[2] * v[2])};
  T fp[3] = {(T)(g.a[0] * v[3]), (T)(g.a[1] * v[4]), (T)(g.a[2] * v[5])};
#pragma unroll
  for (int c = 0; c < kBs; ++c) {
    size_t kk = (size_t)wrapk(gz + c, g.n3);
    T v0 = tz[c][0], v1 = tz[c][1];
#pragma unroll
    for (int b = 0; b < kBs; ++b) {
      size_t jj = (size_t)wrapk(gy + b, g.n2);
      T u0 = ty[b][0], u1 = ty[b][1];
      T term01 = fd[1] * u1 * v0 + fd[2] * u0 * v1;
      T term11 = fd[0] * u0 * v0;
      T term02 = fp[1] * u1 * v0 + fp[2] * u0 * v1;
      T term12 = fp[0] * u0 * v0;
      size_t row = (kk * g.n2 + jj) * g.n1;
      if (THP_SPREAD_PAIRS && std::is_same<T, float>::value) {
        T re[kBs], im[kBs];
#pragma unroll
        for (int a = 0; a < kBs; ++a) {
          re[a] = term01 * tx[a][0] + term11 * tx[a][1];
          im[a] = term02 * tx[a][0] + term12 * tx[a][1];
        }
        // neighbouring points of the row go in pairs where the pair starts
        // on an even (16-byte aligned) point and does not cross the wrap
        bool done = false;
#pragma unroll
        for (int a = 0; a < kBs; ++a) {
          if (done) {
            done = false;
            continue;
          }
          const size_t gi = row + wrapk(gx + a, g.n1);
          if (a + 1 < kBs && gx + a != -1 && (gi & 1) == 0) {
            grid_add_pair(grid, gi, re[a], im[a], re[a + 1], im[a + 1]);
            done = true;
          } else {
            grid_add(grid, gi, re[a], im[a]);
          }
        }
      } else {
#pragma unroll
        for (int a = 0; a < kBs; ++a) {
          int ii = wrapk(gx + a, g.n1);
          grid_add(grid, row + ii, term01 * tx[a][0] + term11 * tx[a][1], term02 * tx[a][0] + term12 * tx[a][1]);
        }
      }
    }
  }
}

// fphi_uind_site field part (pmestuff.f:746-1045, fdip_phi(2:4)) and the
// fractional -> Cartesian conversion of tmatxbrecip (:2094-2121).
template <typename T>
__device__ __forceinline__ void gather_dip(const PmeGeom& g, double4 p, const typename Cplx<T>::type* __restrict__ grid,
                                           double (&out)[6]) {
  T tx[kBs][2], ty[kBs][2], tz[kBs][2];
  int gx = bspline_axis<2, T>(p.x, g.recip[0], g.n1, tx);
  int gy = bspline_axis<2, T>(p.y, g.recip[1], g.n2, ty);
  int gz = bspline_axis<2, T>(p.z, g.recip[2], g.n3, tz);
  T a100 = 0, a010 = 0, a001 = 0, b100 = 0, b010 = 0, b001 = 0;
#pragma unroll
  for (int c = 0; c < kBs; ++c) {
    size_t kk = (size_t)wrapk(gz + c, g.n3);
    T v0 = tz[c][0], v1 = tz[c][1];
    T a00 = 0, a10 = 0, a01 = 0, b00 = 0, b10 = 0, b01 = 0;
#pragma unroll
    for (int b = 0; b < kBs; ++b) {
      size_t jj = (size_t)wrapk(gy + b, g.n2);
      T u0 = ty[b][0], u1 = ty[b][1];
      T t0a = 0, t1a = 0, t0b = 0, t1b = 0;
      size_t row = (kk * g.n2 + jj) * g.n1;
#pragma unroll
      for (int a = 0; a < kBs; ++a) {
        auto q = grid[row + wrapk(gx + a, g.n1)];
        t0a += q.x * tx[a][0];
        t1a += q.x * tx[a][1];
        t0b += q.y * tx[a][0];
        t1b += q.y * tx[a][1];
      }
      a00 += t0a * u0;
      a10 += t1a * u0;
      a01 += t0a * u1;
      b00 += t0b * u0;
      b10 += t1b * u0;
      b01 += t0b * u1;
    }
    a100 += a10 * v0;
    a010 += a01 * v0;
    a001 += a00 * v1;
    b100 += b10 * v0;
    b010 += b01 * v0;
    b001 += b00 * v1;
  }
  out[0] = g.a[0] * (double)a100;
  out[1] = g.a[1] * (double)a010;
  out[2] = g.a[2] * (double)a001;
  out[3] = g.a[0] * (double)b100;
  out[4] = g.a[1] * (double)b010;
  out[5] = g.a[2] * (double)b001;
}


}  // namespace thp
