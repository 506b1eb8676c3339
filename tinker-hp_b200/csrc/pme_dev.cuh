// pme_dev.cuh -- device helpers of the smooth-PME dipole/multipole passes.
#pragma once

#include <cufft.h>

#include <atomic>
#include <climits>
#include <cstdint>
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
// The 125 stencil points of one site from its weights (tx, ty, tz: value and
// first derivative per axis), first grid indices and scaled dipoles.
template <typename T>
__device__ __forceinline__ void spread_dip_stencil(const PmeGeom& g, int gx, int gy, int gz, const T (&tx)[kBs][2],
                                                   const T (&ty)[kBs][2], const T (&tz)[kBs][2], const T (&fd)[3],
                                                   const T (&fp)[3], typename Cplx<T>::type* __restrict__ grid) {
  // paired reductions need the grid on a 16-byte boundary
  const bool aligned = (reinterpret_cast<uintptr_t>(grid) & 15) == 0;
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
      if (THP_SPREAD_PAIRS && std::is_same<T, float>::value && aligned) {
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

template <typename T>
__device__ __forceinline__ void spread_dip_site(const PmeGeom& g, double4 p, const double (&v)[6],
                                                typename Cplx<T>::type* __restrict__ grid) {
  T tx[kBs][2], ty[kBs][2], tz[kBs][2];
  const int gx = bspline_axis<2, T>(p.x, g.recip[0], g.n1, tx);
  const int gy = bspline_axis<2, T>(p.y, g.recip[1], g.n2, ty);
  const int gz = bspline_axis<2, T>(p.z, g.recip[2], g.n3, tz);
  const T fd[3] = {(T)(g.a[0] * v[0]), (T)(g.a[1] * v[1]), (T)(g.a[2] * v[2])};
  const T fp[3] = {(T)(g.a[0] * v[3]), (T)(g.a[1] * v[4]), (T)(g.a[2] * v[5])};
  spread_dip_stencil<T>(g, gx, gy, gz, tx, ty, tz, fd, fp, grid);
}

// Warp-aggregated spread.  The sites of a warp are consecutive in the cell
// order, so their stencils overlap heavily: 16 sites of the 288k water box
// touch about 900 distinct grid points instead of 2,000.  The warp sums the
// contributions of 16 sites at a time in a shared-memory tile (the bounding
// box of their stencils) and adds the tile to the grid once, one reduction
// per nonzero point, instead of one reduction per site and stencil point.
//
// Tile layout: point (z, y, x) at z*SZ + y*SY + x with SY odd and
// SZ = 5*SY (mod 16).  Lane l < 25 owns stencil line (dy, dz) = (l%5, l/5)
// of the site being added: the 25 lanes write 25 distinct lines (no shared
// atomics), and the strides put the lanes of each half-warp (8-byte points)
// or quarter-warp (16-byte points) on distinct bank slots.
#ifndef THP_SPREAD_TILE_PTS
#define THP_SPREAD_TILE_PTS 1280  // FP32 grid: 10 KB of tile per warp
#endif
#ifndef THP_SPREAD_TILE_PTS_F64
#define THP_SPREAD_TILE_PTS_F64 1024  // FP64 grid: 16 KB of tile per warp
#endif
// Raises a kernel's dynamic shared-memory limit on the current device, once
// per device: the attribute belongs to each device's copy of the kernel, so
// a process with contexts on several devices sets it on each.
template <typename K>
inline void smem_limit_once(K* kernel, size_t bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  const unsigned long long bit = 1ull << dev;
  if (done.load(std::memory_order_acquire) & bit) return;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  done.fetch_or(bit, std::memory_order_acq_rel);
}

constexpr int kSpreadRec = 36;      // staged weights per site: tx, ty, tz (10 each), fd, fp
constexpr int kSpreadThreads = 64;  // block of the tiled spread kernels: two warps

template <typename T>
struct SpreadWarp {
  static constexpr int kPts = std::is_same<T, float>::value ? THP_SPREAD_TILE_PTS : THP_SPREAD_TILE_PTS_F64;
  static_assert(kPts >= kBs * kBs * kBs, "a tile holds at least one site's stencil");
  T w[32][kSpreadRec];
  int4 off[32];  // the site's stencil origin in the tile
  typename Cplx<T>::type tile[kPts];
};

template <typename T>
struct Pair;
template <>
struct Pair<float> {
  using type = float2;
};
template <>
struct Pair<double> {
  using type = double2;
};

// One axis of a tile: the stencil origins of the sites in `mine` as the tile
// indexes them and their minimum (lo).  A cell-sorted run of sites that
// crosses from the end of one cell row to the start of the next is compact
// only through the periodic boundary, so when the plain span is wide the
// upper half of the grid is taken one period down instead, whichever span is
// shorter.  Tile indexes stay in [-n, n) for wrapk.
__device__ __forceinline__ int tile_axis(bool mine, int v, int n, int& lo) {
  lo = __reduce_min_sync(~0u, mine ? v : INT_MAX);
  const int hi = __reduce_max_sync(~0u, mine ? v : INT_MIN);
  if (hi - lo + kBs <= 16) return v;
  const int vs = v >= (n >> 1) ? v - n : v;
  const int lo2 = __reduce_min_sync(~0u, mine ? vs : INT_MAX);
  const int hi2 = __reduce_max_sync(~0u, mine ? vs : INT_MIN);
  if (hi2 - lo2 >= hi - lo) return v;
  lo = lo2;
  return vs;
}

// Weights of stencil points k and k+1 along x (value, derivative each).
__device__ __forceinline__ void tx_pairs(const float* r, float (&t)[2 * kBs]) {
  const float4 a = *reinterpret_cast<const float4*>(r), b = *reinterpret_cast<const float4*>(r + 4);
  const float2 c = *reinterpret_cast<const float2*>(r + 8);
  t[0] = a.x; t[1] = a.y; t[2] = a.z; t[3] = a.w; t[4] = b.x; t[5] = b.y; t[6] = b.z; t[7] = b.w;
  t[8] = c.x; t[9] = c.y;
}
__device__ __forceinline__ void tx_pairs(const double* r, double (&t)[2 * kBs]) {
#pragma unroll
  for (int k = 0; k < kBs; ++k) {
    const double2 a = *reinterpret_cast<const double2*>(r + 2 * k);
    t[2 * k] = a.x;
    t[2 * k + 1] = a.y;
  }
}

// Adds the nonzero points of a tile line segment to the grid and zeroes
// them.  Pairs of neighbouring points go in one 16-byte reduction (FP32 grid
// with an even row length, the pair starting on an even grid point); the
// other points one by one.
__device__ __forceinline__ void flush_point(cufftComplex* grid, size_t gi, cufftComplex* q) {
  const cufftComplex e = *q;
  if (e.x != 0.f || e.y != 0.f) {
    *q = cufftComplex{0.f, 0.f};
    grid_add(grid, gi, e.x, e.y);
  }
}
__device__ __forceinline__ void flush_point(cufftDoubleComplex* grid, size_t gi, cufftDoubleComplex* q) {
  const cufftDoubleComplex e = *q;
  if (e.x != 0.0 || e.y != 0.0) {
    *q = cufftDoubleComplex{0.0, 0.0};
    grid_add(grid, gi, e.x, e.y);
  }
}

// One tile over the sites in mk (their weights staged in s.w): sums their
// stencils in the tile and adds the tile's nonzero points to the grid.
// Returns false, having done nothing, when the stencils do not fit a tile
// (x span above 32 points or a box past kPts points); a single site always
// fits.  Warp-collective.
template <typename T>
__device__ __forceinline__ bool spread_tile_pass(const PmeGeom& g, unsigned mk, int lane, int gx, int gy, int gz,
                                                 typename Cplx<T>::type* __restrict__ grid, SpreadWarp<T>& s) {
  using C = typename Cplx<T>::type;
  using T2 = typename Pair<T>::type;
  const bool mine = (mk >> lane) & 1u;
  int x0, y0, z0;
  const int lx = tile_axis(mine, gx, g.n1, x0), ly = tile_axis(mine, gy, g.n2, y0), lz = tile_axis(mine, gz, g.n3, z0);
  const int X = __reduce_max_sync(~0u, mine ? lx : INT_MIN) - x0 + kBs;
  const int Y = __reduce_max_sync(~0u, mine ? ly : INT_MIN) - y0 + kBs;
  const int Z = __reduce_max_sync(~0u, mine ? lz : INT_MIN) - z0 + kBs;
  const int SY = X | 1;
  const int SZ = Y * SY + ((5 * SY - Y * SY) & 15);
  if (X > 32 || Z > SpreadWarp<T>::kPts || Z * SZ > SpreadWarp<T>::kPts) return false;
  if (mine) s.off[lane] = make_int4(lx - x0, ly - y0, lz - z0, 0);
  __syncwarp();
  const int dy = lane % 5, dz = lane / 5;
  const int lane_off = dz * SZ + dy * SY;
  unsigned mm = mk;
  while (mm) {
    const int a = __ffs(mm) - 1;
    mm &= mm - 1;
    if (lane < 25) {
      const T* r = s.w[a];
      const int4 o = s.off[a];
      const T2 u = *reinterpret_cast<const T2*>(r + 10 + 2 * dy);
      const T2 vz = *reinterpret_cast<const T2*>(r + 20 + 2 * dz);
      const T2 f0 = *reinterpret_cast<const T2*>(r + 30);  // fd0 fd1
      const T2 f1 = *reinterpret_cast<const T2*>(r + 32);  // fd2 fp0
      const T2 f2 = *reinterpret_cast<const T2*>(r + 34);  // fp1 fp2
      T t[2 * kBs];
      tx_pairs(r, t);
      const T u0v0 = u.x * vz.x, u1v0 = u.y * vz.x, u0v1 = u.x * vz.y;
      C* q = s.tile + lane_off + o.z * SZ + o.y * SY + o.x;
      if constexpr (std::is_same<T, float>::value) {
        // (Re, Im) as one packed pair: terms (t01, t02) and (t11, t12)
        const float2 a = __ffma2_rn(make_float2(f0.y, f2.x), make_float2(u1v0, u1v0),
                                    __fmul2_rn(make_float2(f1.x, f2.y), make_float2(u0v1, u0v1)));
        const float2 b = __fmul2_rn(make_float2(f0.x, f1.y), make_float2(u0v0, u0v0));
#pragma unroll
        for (int k = 0; k < kBs; ++k) {
          float2* qk = reinterpret_cast<float2*>(q + k);
          float2 e = *qk;
          e = __ffma2_rn(a, make_float2(t[2 * k], t[2 * k]), e);
          e = __ffma2_rn(b, make_float2(t[2 * k + 1], t[2 * k + 1]), e);
          *qk = e;
        }
      } else {
        const T term01 = f0.y * u1v0 + f1.x * u0v1;
        const T term11 = f0.x * u0v0;
        const T term02 = f2.x * u1v0 + f2.y * u0v1;
        const T term12 = f1.y * u0v0;
#pragma unroll
        for (int k = 0; k < kBs; ++k) {
          C e = q[k];
          e.x += term01 * t[2 * k] + term11 * t[2 * k + 1];
          e.y += term02 * t[2 * k] + term12 * t[2 * k + 1];
          q[k] = e;
        }
      }
    }
    __syncwarp();
  }
  // flush, lines in (z, y) order; the flushed points are zeroed for the next
  // tile.  FP32 grid with an even row length: each lane takes a pair of
  // points starting on an even grid point (the tile's column -1 or X, outside
  // the tile, reads as zero); otherwise one point per lane.
  constexpr bool kPairs = std::is_same<T, float>::value;
  const bool pairs = kPairs && (g.n1 & 1) == 0 && (reinterpret_cast<uintptr_t>(grid) & 15) == 0;
  const int shift = pairs ? ((x0 & 1) ? -1 : 0) : 0;     // tile column of the lane's first point
  const int cols = pairs ? (X - shift + 1) >> 1 : X;     // pairs or points per line
  const int xw = cols <= 8 ? 8 : (cols <= 16 ? 16 : 32);  // lanes per line
  const int per = 32 / xw, c = lane & (xw - 1);
  const bool cin = c < cols;
  const int xa = pairs ? shift + 2 * c : c;  // tile column of the lane's (first) point
  const size_t xi = (size_t)wrapk(x0 + (cin ? xa : 0), g.n1);
  int z = 0, y = lane / xw;
  int wz = wrapk(z0, g.n3), wy = wrapk(y0 + y, g.n2);  // grid plane and row of (z, y)
  const int ymod = Y % g.n2;
  for (int L = lane / xw; L < Y * Z; L += per) {
    if (cin) {
      C* q = s.tile + z * SZ + y * SY + xa;
      const size_t gi = ((size_t)wz * g.n2 + wy) * g.n1 + xi;
      if (pairs) {
        if constexpr (kPairs) {
          const bool l0 = xa >= 0, l1 = xa + 1 < X;
          const C e0 = l0 ? q[0] : C{0.f, 0.f};
          const C e1 = l1 ? q[1] : C{0.f, 0.f};
          if (e0.x != 0.f || e0.y != 0.f || e1.x != 0.f || e1.y != 0.f) {
            if (l0) q[0] = C{0.f, 0.f};
            if (l1) q[1] = C{0.f, 0.f};
            grid_add_pair(grid, gi, e0.x, e0.y, e1.x, e1.y);
          }
        }
      } else {
        flush_point(grid, gi, q);
      }
    }
    y += per;
    wy += per;
    if (wy >= g.n2) wy -= g.n2;
    if (y >= Y) {
      y -= Y;
      wy -= ymod;
      if (wy < 0) wy += g.n2;
      ++z;
      if (++wz == g.n3) wz = 0;
    }
  }
  __syncwarp();
  return true;
}

// Every lane of the warp calls this with its site (live false for none).
// The sites of each half-warp form one tile; a half whose stencils do not
// fit is split into two tiles of 8 sites, and an 8-site group that still
// does not fit into tiles of one site.  The tile must be zero on entry and is
// zero again on return.
template <typename T>
__device__ __forceinline__ void spread_dip_warp(const PmeGeom& g, double4 p, const double (&v)[6], bool live,
                                                typename Cplx<T>::type* __restrict__ grid, SpreadWarp<T>& s) {
  const int lane = threadIdx.x & 31;
  int gx = 0, gy = 0, gz = 0;
  if (live) {
    T w[kSpreadRec];
    T tx[kBs][2], ty[kBs][2], tz[kBs][2];
    gx = bspline_axis<2, T>(p.x, g.recip[0], g.n1, tx);
    gy = bspline_axis<2, T>(p.y, g.recip[1], g.n2, ty);
    gz = bspline_axis<2, T>(p.z, g.recip[2], g.n3, tz);
#pragma unroll
    for (int k = 0; k < kBs; ++k) {
      w[2 * k] = tx[k][0];
      w[2 * k + 1] = tx[k][1];
      w[10 + 2 * k] = ty[k][0];
      w[11 + 2 * k] = ty[k][1];
      w[20 + 2 * k] = tz[k][0];
      w[21 + 2 * k] = tz[k][1];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      w[30 + d] = (T)(g.a[d] * v[d]);
      w[33 + d] = (T)(g.a[d] * v[3 + d]);
    }
    using T2 = typename Pair<T>::type;
    T2* dst = reinterpret_cast<T2*>(s.w[lane]);
#pragma unroll
    for (int k = 0; k < kSpreadRec / 2; ++k) dst[k] = T2{w[2 * k], w[2 * k + 1]};
  }
  // groups of 16, then 8, then 1 site; level moves down when a group does
  // not fit and back up when the group above it is done
  unsigned pending = __ballot_sync(~0u, live);
  int level = 0;
#pragma unroll 1
  while (pending) {
    const int first = __ffs(pending) - 1;
    const unsigned gm = level == 0 ? (0xffffu << (first & 16)) : (level == 1 ? (0xffu << (first & 24)) : (1u << first));
    const unsigned mk = pending & gm;
    if (spread_tile_pass<T>(g, mk, lane, gx, gy, gz, grid, s)) {
      pending &= ~mk;
      if (!(pending & (0xffffu << (first & 16))))
        level = 0;
      else if (!(pending & (0xffu << (first & 24))))
        level = 1;
    } else {
      ++level;  // a single site always fits, so level stays <= 2
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
