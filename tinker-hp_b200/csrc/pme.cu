// pme.cu -- smooth PME for the permanent field and the dipole matvec.
//
// efld0_recip (newinduce_pme.f:1671-1917) and tmatxbrecip (:1919-2128):
// B-splines recomputed per pass from positions (bsplgen, pmestuff.f:64),
// spread with global atomics into one complex grid (d dipoles in Re, p in Im,
// as qgrid2in_2d), cuFFT forward / influence function qfac / cuFFT backward
// (unnormalised, fft_mpi.f90:65,115), and a gather of the potential
// derivatives (fphi_mpole_site :453, fphi_uind_site :746).  Orthogonal boxes:
// the fractional <-> Cartesian matrices reduce to a_d = nfft_d * recip(d,d).
#include <vector>

#include <map>
#include <mutex>
#include <type_traits>

#include "kernels.h"
#include "pme_dev.cuh"

namespace thp {

namespace {

constexpr int kBlock = 128;

__device__ __forceinline__ void grid_add_re(cufftDoubleComplex* g, size_t idx, double re) { red_add(&g[idx].x, re); }
__device__ __forceinline__ void grid_add_re(cufftComplex* g, size_t idx, float re) { red_add(&g[idx].x, re); }

// grid_mpole_site (pmestuff.f:163-278) for every site; rpole10 sorted
template <typename T>
__global__ void k_spread_mpole(int n, PmeGeom g, const double4* __restrict__ pos, const double* __restrict__ rp,
                               typename Cplx<T>::type* __restrict__ grid) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p = pos[i];
  T tx[kBs][3], ty[kBs][3], tz[kBs][3];
  int gx = bspline_axis<3, T>(p.x, g.recip[0], g.n1, tx);
  int gy = bspline_axis<3, T>(p.y, g.recip[1], g.n2, ty);
  int gz = bspline_axis<3, T>(p.z, g.recip[2], g.n3, tz);
  const double* r = rp + (size_t)i * 10;
  // cmp (newinduce_pme.f:1750-1759) -> fmp via cart_to_frac (pmestuff.f:1131)
  T f[10];
  f[0] = (T)r[0];
  f[1] = (T)(g.a[0] * r[1]);
  f[2] = (T)(g.a[1] * r[2]);
  f[3] = (T)(g.a[2] * r[3]);
  f[4] = (T)(g.a[0] * g.a[0] * r[4]);
  f[5] = (T)(g.a[1] * g.a[1] * r[7]);
  f[6] = (T)(g.a[2] * g.a[2] * r[9]);
  f[7] = (T)(g.a[0] * g.a[1] * (2.0 * r[5]));
  f[8] = (T)(g.a[0] * g.a[2] * (2.0 * r[6]));
  f[9] = (T)(g.a[1] * g.a[2] * (2.0 * r[8]));
#pragma unroll
  for (int c = 0; c < kBs; ++c) {
    size_t kk = (size_t)wrapk(gz + c, g.n3);
    T v0 = tz[c][0], v1 = tz[c][1], v2 = tz[c][2];
#pragma unroll
    for (int b = 0; b < kBs; ++b) {
      size_t jj = (size_t)wrapk(gy + b, g.n2);
      T u0 = ty[b][0], u1 = ty[b][1], u2 = ty[b][2];
      T term0 = f[0] * u0 * v0 + f[2] * u1 * v0 + f[3] * u0 * v1 + f[5] * u2 * v0 + f[6] * u0 * v2 + f[9] * u1 * v1;
      T term1 = f[1] * u0 * v0 + f[7] * u1 * v0 + f[8] * u0 * v1;
      T term2 = f[4] * u0 * v0;
      size_t row = (kk * g.n2 + jj) * g.n1;
#pragma unroll
      for (int a = 0; a < kBs; ++a) {
        int ii = wrapk(gx + a, g.n1);
        grid_add_re(grid, row + ii, term0 * tx[a][0] + term1 * tx[a][1] + term2 * tx[a][2]);
      }
    }
  }
}

// grid_mpole_site for the two multipole sets of eprecip1's virial
// (epolar1.f:932-1040): the permanent moments with uinp added to the dipole
// into the real part, with uind added into the imaginary part, of one
// complex grid.  mu sorted [n][6] (uind xyz, uinp xyz).
template <typename T>
__global__ void k_spread_mpole2(int n, PmeGeom g, const double4* __restrict__ pos, const double* __restrict__ rp,
                                const double* __restrict__ mu, typename Cplx<T>::type* __restrict__ grid) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p = pos[i];
  T tx[kBs][3], ty[kBs][3], tz[kBs][3];
  int gx = bspline_axis<3, T>(p.x, g.recip[0], g.n1, tx);
  int gy = bspline_axis<3, T>(p.y, g.recip[1], g.n2, ty);
  int gz = bspline_axis<3, T>(p.z, g.recip[2], g.n3, tz);
  const double* r = rp + (size_t)i * 10;
  const double* m = mu + (size_t)i * 6;
  T f[10], fb[3];
  f[0] = (T)r[0];
  f[1] = (T)(g.a[0] * (r[1] + m[3]));
  f[2] = (T)(g.a[1] * (r[2] + m[4]));
  f[3] = (T)(g.a[2] * (r[3] + m[5]));
  fb[0] = (T)(g.a[0] * (r[1] + m[0]));
  fb[1] = (T)(g.a[1] * (r[2] + m[1]));
  fb[2] = (T)(g.a[2] * (r[3] + m[2]));
  f[4] = (T)(g.a[0] * g.a[0] * r[4]);
  f[5] = (T)(g.a[1] * g.a[1] * r[7]);
  f[6] = (T)(g.a[2] * g.a[2] * r[9]);
  f[7] = (T)(g.a[0] * g.a[1] * (2.0 * r[5]));
  f[8] = (T)(g.a[0] * g.a[2] * (2.0 * r[6]));
  f[9] = (T)(g.a[1] * g.a[2] * (2.0 * r[8]));
#pragma unroll
  for (int c = 0; c < kBs; ++c) {
    size_t kk = (size_t)wrapk(gz + c, g.n3);
    T v0 = tz[c][0], v1 = tz[c][1], v2 = tz[c][2];
#pragma unroll
    for (int b = 0; b < kBs; ++b) {
      size_t jj = (size_t)wrapk(gy + b, g.n2);
      T u0 = ty[b][0], u1 = ty[b][1], u2 = ty[b][2];
      // the terms without a dipole are shared by the two sets
      T q0 = f[0] * u0 * v0 + f[5] * u2 * v0 + f[6] * u0 * v2 + f[9] * u1 * v1;
      T term0a = q0 + f[2] * u1 * v0 + f[3] * u0 * v1, term0b = q0 + fb[1] * u1 * v0 + fb[2] * u0 * v1;
      T q1 = f[7] * u1 * v0 + f[8] * u0 * v1;
      T term1a = q1 + f[1] * u0 * v0, term1b = q1 + fb[0] * u0 * v0;
      T term2 = f[4] * u0 * v0;
      size_t row = (kk * g.n2 + jj) * g.n1;
#pragma unroll
      for (int a = 0; a < kBs; ++a) {
        int ii = wrapk(gx + a, g.n1);
        grid_add(grid, row + ii, term0a * tx[a][0] + term1a * tx[a][1] + term2 * tx[a][2],
                 term0b * tx[a][0] + term1b * tx[a][1] + term2 * tx[a][2]);
      }
    }
  }
}

// Sum over the reciprocal lattice (all k but 0 with qfac > 0) of the PME
// virial terms h h vterm - eterm (eterm = 0.5 f qfac struc2, vterm =
// (2/h^2)(1 + pterm h^2) eterm; emrecip1 / eprecip1, epolar1.f:1041-1091)
// of the forward-transformed grid, times sign.  mode 0: struc2 = |G(k)|^2
// (one real grid); mode 1: struc2 = Re(A(k) conj B(k)) of the two real grids
// A (real part) and B (imaginary part) packed in G, separated by
// A = (G(k) + conj G(-k)) / 2, B = (G(k) - conj G(-k)) / 2i.  Each block
// writes its 6 sums (xx, xy, xz, yy, yz, zz) to part[block].
template <typename C, typename Q>
__global__ void __launch_bounds__(256) k_kspace_virial(int n1, int n2, int n3, const C* __restrict__ grid,
                                                       const Q* __restrict__ qfac, double r1, double r2, double r3,
                                                       double pterm, double f, int mode, double sign,
                                                       double* __restrict__ part) {
  double v[6] = {0, 0, 0, 0, 0, 0};
  const long ng = (long)n1 * n2 * n3;
  const int nf1 = (n1 + 1) / 2, nf2 = (n2 + 1) / 2, nf3 = (n3 + 1) / 2;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < ng; idx += (long)gridDim.x * blockDim.x) {
    const double qf = (double)qfac[idx];
    if (qf == 0.0) continue;
    const int k1 = (int)(idx % n1), k2 = (int)((idx / n1) % n2), k3 = (int)(idx / ((long)n1 * n2));
    const int m1 = k1 + 1 > nf1 ? k1 - n1 : k1, m2 = k2 + 1 > nf2 ? k2 - n2 : k2, m3 = k3 + 1 > nf3 ? k3 - n3 : k3;
    const C gk = grid[idx];
    double struc2;
    if (mode == 0) {
      struc2 = (double)gk.x * gk.x + (double)gk.y * gk.y;
    } else {
      const long mi = ((long)((n3 - k3) % n3) * n2 + (n2 - k2) % n2) * n1 + (n1 - k1) % n1;
      const C gm = grid[mi];  // conj G(-k) = (gm.x, -gm.y)
      const double ax = 0.5 * ((double)gk.x + gm.x), ay = 0.5 * ((double)gk.y - gm.y);
      const double bx = 0.5 * ((double)gk.y + gm.y), by = -0.5 * ((double)gk.x - gm.x);
      struc2 = ax * bx + ay * by;
    }
    const double h1 = r1 * m1, h2 = r2 * m2, h3 = r3 * m3;
    const double hsq = h1 * h1 + h2 * h2 + h3 * h3;
    const double eterm = 0.5 * f * qf * struc2;
    const double vterm = (2.0 / hsq) * (1.0 + pterm * hsq) * eterm;
    v[0] += h1 * h1 * vterm - eterm;
    v[1] += h1 * h2 * vterm;
    v[2] += h1 * h3 * vterm;
    v[3] += h2 * h2 * vterm - eterm;
    v[4] += h2 * h3 * vterm;
    v[5] += h3 * h3 * vterm - eterm;
  }
  block_reduce<6>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 6; ++q) part[(size_t)blockIdx.x * 6 + q] = sign * v[q];
}

// The vector a site spreads: vec[i] (mode 1: zr + beta vec, written back),
// with the FP32 copy in vecf when given.
template <typename V>
__device__ __forceinline__ void spread_load(int i, V* __restrict__ vec, const double* __restrict__ zr,
                                            float* __restrict__ vecf, const CgScalars* __restrict__ cg, int mode,
                                            double (&v)[6]) {
  if constexpr (std::is_same<V, float>::value) {
    const float2* v2 = reinterpret_cast<const float2*>(vec + (size_t)i * 6);
    const float2 a0 = v2[0], a1 = v2[1], a2 = v2[2];
    v[0] = a0.x; v[1] = a0.y; v[2] = a1.x; v[3] = a1.y; v[4] = a2.x; v[5] = a2.y;
  } else {
    const double2* v2 = reinterpret_cast<const double2*>(vec + (size_t)i * 6);
    double2 a0 = v2[0], a1 = v2[1], a2 = v2[2];
    v[0] = a0.x; v[1] = a0.y; v[2] = a1.x; v[3] = a1.y; v[4] = a2.x; v[5] = a2.y;
  }
  if constexpr (std::is_same<V, double>::value) {
    if (mode == 1) {
      const double2* z2 = reinterpret_cast<const double2*>(zr + (size_t)i * 6);
      double2 b0 = z2[0], b1 = z2[1], b2 = z2[2];
      double bd = cg->beta[0], bp = cg->beta[1];
      v[0] = b0.x + bd * v[0];
      v[1] = b0.y + bd * v[1];
      v[2] = b1.x + bd * v[2];
      v[3] = b1.y + bp * v[3];
      v[4] = b2.x + bp * v[4];
      v[5] = b2.y + bp * v[5];
      double2* w2 = reinterpret_cast<double2*>(vec + (size_t)i * 6);
      w2[0] = make_double2(v[0], v[1]);
      w2[1] = make_double2(v[2], v[3]);
      w2[2] = make_double2(v[4], v[5]);
    }
  }
  if (vecf) {
    float2* o = reinterpret_cast<float2*>(vecf + (size_t)i * 6);
    o[0] = make_float2((float)v[0], (float)v[1]);
    o[1] = make_float2((float)v[2], (float)v[3]);
    o[2] = make_float2((float)v[4], (float)v[5]);
  }
}

// grid_uind_site (pmestuff.f:280-405); d dipoles in Re, p dipoles in Im.
// One thread per site.  TA = 0: each site adds its 125 stencil points to the
// grid itself (a warp-per-site variant that made them contiguous measured
// 1.6x slower); TA = 16: the warp sums the stencils of 16 neighbouring sites
// at a time in a shared-memory tile first (spread_dip_warp), blocks of
// kSpreadThreads threads with one SpreadWarp<T> per warp in dynamic shared
// memory.  mode 1 first forms pp = zr + beta*pp (inducepcg_pme2.f:553-559) and
// writes it back.
// V: the stored type of vec (FP32 for the mixed form's overlapped CG, which
// spreads in mode 2 only)
template <typename T, typename V = double, int TA = 0>
__global__ void __launch_bounds__(128) k_spread_dip(int n, PmeGeom g, const double4* __restrict__ pos,
                                                   V* __restrict__ vec, const double* __restrict__ zr,
                                                   float* __restrict__ vecf, const CgScalars* __restrict__ cg,
                                                   int mode, typename Cplx<T>::type* __restrict__ grid) {
  if (mode >= 1 && cg->stop) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  SpreadWarp<T>* sw = nullptr;
  if constexpr (TA > 0) {
    extern __shared__ __align__(16) unsigned char spread_smem[];
    sw = reinterpret_cast<SpreadWarp<T>*>(spread_smem) + (threadIdx.x >> 5);
    for (int q = threadIdx.x & 31; q < SpreadWarp<T>::kPts; q += 32) sw->tile[q] = {T(0), T(0)};
  } else if (i >= n) {
    return;
  }
  const bool live = i < n;
  double v[6] = {0, 0, 0, 0, 0, 0};
  double4 pi = make_double4(0, 0, 0, 0);
  if (live) {
    spread_load(i, vec, zr, vecf, cg, mode, v);
    pi = pos[i];
  }
  if constexpr (TA > 0)
    spread_dip_warp<T>(g, pi, v, live, grid, *sw);
  else
    spread_dip_site<T>(g, pi, v, grid);
}

template <typename C, typename T>
__global__ void k_qfac(size_t ng, const T* __restrict__ qfac, C* __restrict__ grid, const CgScalars* __restrict__ cg,
                       int check_stop) {
  if (check_stop && cg->stop) return;
  size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; q < ng; q += stride) {
    T f = qfac[q];
    C v = grid[q];
    v.x *= f;
    v.y *= f;
    grid[q] = v;
  }
}

// fphi_mpole_site (pmestuff.f:453-600) restricted to the 10 components of
// cphi, then fphi_to_cphi_site (:1190) and the E0 assembly of
// newinduce_pme2.f:133-148: ef -= cphi(2:4); ef += term * d_perm.
template <typename T>
__global__ void k_gather_mpole(int n, PmeGeom g, const double4* __restrict__ pos,
                               const typename Cplx<T>::type* __restrict__ grid, const double* __restrict__ rp,
                               double term, double* __restrict__ cphi4, double* __restrict__ cphi10,
                               double* __restrict__ ef) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p = pos[i];
  T tx[kBs][3], ty[kBs][3], tz[kBs][3];
  int gx = bspline_axis<3, T>(p.x, g.recip[0], g.n1, tx);
  int gy = bspline_axis<3, T>(p.y, g.recip[1], g.n2, ty);
  int gz = bspline_axis<3, T>(p.z, g.recip[2], g.n3, tz);
  T tuv000 = 0, tuv100 = 0, tuv010 = 0, tuv001 = 0, tuv200 = 0, tuv020 = 0, tuv002 = 0, tuv110 = 0, tuv101 = 0,
    tuv011 = 0;
#pragma unroll
  for (int c = 0; c < kBs; ++c) {
    size_t kk = (size_t)wrapk(gz + c, g.n3);
    T v0 = tz[c][0], v1 = tz[c][1], v2 = tz[c][2];
    T tu00 = 0, tu10 = 0, tu01 = 0, tu20 = 0, tu11 = 0, tu02 = 0;
#pragma unroll
    for (int b = 0; b < kBs; ++b) {
      size_t jj = (size_t)wrapk(gy + b, g.n2);
      T u0 = ty[b][0], u1 = ty[b][1], u2 = ty[b][2];
      T t0 = 0, t1 = 0, t2 = 0;
      size_t row = (kk * g.n2 + jj) * g.n1;
#pragma unroll
      for (int a = 0; a < kBs; ++a) {
        T tq = grid[row + wrapk(gx + a, g.n1)].x;
        t0 += tq * tx[a][0];
        t1 += tq * tx[a][1];
        t2 += tq * tx[a][2];
      }
      tu00 += t0 * u0;
      tu10 += t1 * u0;
      tu01 += t0 * u1;
      tu20 += t2 * u0;
      tu11 += t1 * u1;
      tu02 += t0 * u2;
    }
    tuv000 += tu00 * v0;
    tuv100 += tu10 * v0;
    tuv010 += tu01 * v0;
    tuv001 += tu00 * v1;
    tuv200 += tu20 * v0;
    tuv020 += tu02 * v0;
    tuv002 += tu00 * v2;
    tuv110 += tu11 * v0;
    tuv101 += tu10 * v1;
    tuv011 += tu01 * v1;
  }
  double c1 = g.a[0] * (double)tuv100, c2 = g.a[1] * (double)tuv010, c3 = g.a[2] * (double)tuv001;
  double* cp = cphi4 + (size_t)i * 4;
  cp[0] = (double)tuv000;
  cp[1] = c1;
  cp[2] = c2;
  cp[3] = c3;
  if (cphi10) {
    double* q = cphi10 + (size_t)i * 10;
    q[0] = (double)tuv000;
    q[1] = c1;
    q[2] = c2;
    q[3] = c3;
    q[4] = g.a[0] * g.a[0] * (double)tuv200;
    q[5] = g.a[1] * g.a[1] * (double)tuv020;
    q[6] = g.a[2] * g.a[2] * (double)tuv002;
    q[7] = g.a[0] * g.a[1] * (double)tuv110;
    q[8] = g.a[0] * g.a[2] * (double)tuv101;
    q[9] = g.a[1] * g.a[2] * (double)tuv011;
  }
  if (ef) {
    const double* r = rp + (size_t)i * 10;
    double* e = ef + (size_t)i * 6;
    double cc[3] = {c1, c2, c3};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      e[j] = (e[j] - cc[j]) + term * r[1 + j];
      e[3 + j] = (e[3 + j] - cc[j]) + term * r[1 + j];
    }
  }
}

}  // namespace

namespace {

// fphi_uind_site (pmestuff.f:746-1045) field part, one thread per site,
// output dipfield [n][6] (tmatxbrecip, newinduce_pme.f:2094-2121).
template <typename T>
__global__ void __launch_bounds__(128) k_gather_dip(int n, PmeGeom g, const double4* __restrict__ pos,
                                                    const typename Cplx<T>::type* __restrict__ grid,
                                                    double* __restrict__ out, const CgScalars* __restrict__ cg,
                                                    int check_stop) {
  if (check_stop && cg->stop) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double o[6];
  gather_dip<T>(g, pos[i], grid, o);
  double2* d = reinterpret_cast<double2*>(out + (size_t)i * 6);
  d[0] = make_double2(o[0], o[1]);
  d[1] = make_double2(o[2], o[3]);
  d[2] = make_double2(o[4], o[5]);
}

// kewald.f:693-717 (bspline) and :747-812 (dftmod)
std::vector<double> dftmod_host(int nfft, int order) {
  std::vector<double> arr(order + 2, 0.0), bsarray(nfft + 2, 0.0), bsmod(nfft + 1, 0.0);
  double x = 0.0;
  arr[1] = 1.0 - x;
  arr[2] = x;
  for (int k = 3; k <= order; ++k) {
    double denom = 1.0 / (double)(k - 1);
    arr[k] = x * arr[k - 1] * denom;
    for (int i = 1; i <= k - 2; ++i) arr[k - i] = ((x + i) * arr[k - i - 1] + ((k - i) - x) * arr[k - i]) * denom;
    arr[1] = (1.0 - x) * arr[1] * denom;
  }
  for (int i = 2; i <= order + 1 && i <= nfft; ++i) bsarray[i] = arr[i - 1];
  double factor = 2.0 * kPi / (double)nfft;
  for (int i = 1; i <= nfft; ++i) {
    double s1 = 0.0, s2 = 0.0;
    for (int j = 1; j <= nfft; ++j) {
      double arg = factor * (double)((i - 1) * (j - 1));
      s1 += bsarray[j] * cos(arg);
      s2 += bsarray[j] * sin(arg);
    }
    bsmod[i] = s1 * s1 + s2 * s2;
  }
  double eps = 1.0e-7;
  if (bsmod[1] < eps) bsmod[1] = 0.5 * bsmod[2];
  for (int i = 2; i <= nfft - 1; ++i)
    if (bsmod[i] < eps) bsmod[i] = 0.5 * (bsmod[i - 1] + bsmod[i + 1]);
  if (bsmod[nfft] < eps) bsmod[nfft] = 0.5 * bsmod[nfft - 1];
  for (int i = 1; i <= nfft; ++i) {
    int k = i - 1;
    if (i > nfft / 2) k -= nfft;
    double zeta = 1.0;
    if (k != 0) {
      double s1 = 1.0, s2 = 1.0, fac = kPi * (double)k / (double)nfft;
      for (int j = 1; j <= 50; ++j) {
        double arg = fac / (fac + kPi * j);
        s1 += pow(arg, order);
        s2 += pow(arg, 2 * order);
      }
      for (int j = 1; j <= 50; ++j) {
        double arg = fac / (fac - kPi * j);
        s1 += pow(arg, order);
        s2 += pow(arg, 2 * order);
      }
      zeta = s2 / s1;
    }
    bsmod[i] = bsmod[i] * zeta * zeta;
  }
  return bsmod;
}

PmeGeom geom_of(const Ctx& c) {
  PmeGeom g;
  g.n1 = c.nfft[0];
  g.n2 = c.nfft[1];
  g.n3 = c.nfft[2];
  for (int d = 0; d < 3; ++d) {
    g.recip[d] = c.box.recip[d];
    g.a[d] = c.a_frac[d];
  }
  return g;
}

int fft(Ctx& c, int dir) {
  cufftResult r;
  if (c.mixed)
    r = cufftExecC2C(c.plan, (cufftComplex*)c.d_grid, (cufftComplex*)c.d_grid, dir);
  else
    r = cufftExecZ2Z(c.plan, (cufftDoubleComplex*)c.d_grid, (cufftDoubleComplex*)c.d_grid, dir);
  if (r != CUFFT_SUCCESS) {
    c.last_msg = "cuFFT exec failed";
    return THP_E_CUDA;
  }
  return THP_OK;
}

int convolve(Ctx& c, int check_stop) {
  int st = fft(c, CUFFT_FORWARD);
  if (st) return st;
  int blocks = 148 * 8;
  if (c.mixed)
    k_qfac<cufftComplex, float><<<blocks, 256, 0, c.stream>>>(c.ngrid, (const float*)c.d_qfac,
                                                             (cufftComplex*)c.d_grid, c.d_cg, check_stop);
  else
    k_qfac<cufftDoubleComplex, double><<<blocks, 256, 0, c.stream>>>(
        c.ngrid, (const double*)c.d_qfac, (cufftDoubleComplex*)c.d_grid, c.d_cg, check_stop);
  st = cuda_status(cudaGetLastError(), &c, "qfac");
  if (st) return st;
  return fft(c, CUFFT_INVERSE);
}

// Process-wide cache of cuFFT plans by device, dimensions and type: a
// context that is destroyed or re-targeted to another grid gives its plan
// back, and the next context of that shape takes it instead of planning
// again (planning allocates a work area and can take milliseconds).
struct PlanKey {
  int device, n1, n2, n3, mixed;
  bool operator==(const PlanKey& o) const {
    return device == o.device && n1 == o.n1 && n2 == o.n2 && n3 == o.n3 && mixed == o.mixed;
  }
};
std::mutex g_plan_mu;
std::vector<std::pair<PlanKey, cufftHandle>> g_plans;
constexpr size_t kMaxCachedPlans = 64;

bool take_plan(const PlanKey& k, cufftHandle* out) {
  std::lock_guard<std::mutex> g(g_plan_mu);
  for (size_t q = 0; q < g_plans.size(); ++q)
    if (g_plans[q].first == k) {
      *out = g_plans[q].second;
      g_plans.erase(g_plans.begin() + q);
      return true;
    }
  return false;
}

void give_plan(const PlanKey& k, cufftHandle plan) {
  std::lock_guard<std::mutex> g(g_plan_mu);
  if (g_plans.size() >= kMaxCachedPlans) {
    cufftDestroy(g_plans.front().second);
    g_plans.erase(g_plans.begin());
  }
  g_plans.emplace_back(k, plan);
}

PlanKey plan_key(const Ctx& c) { return PlanKey{c.device, c.plan_dims[0], c.plan_dims[1], c.plan_dims[2], c.mixed}; }

bool plan_cached(const PlanKey& k) {
  std::lock_guard<std::mutex> g(g_plan_mu);
  for (const auto& p : g_plans)
    if (p.first == k) return true;
  return false;
}

// qfac(k) = exp(-pi^2 h^2 / a^2) / (pi V h^2 bsmod1 bsmod2 bsmod3), zero at
// h = 0 and where the exponent is below -50 (newinduce_pme.f:1802-1854)
template <typename T>
__global__ void k_qfac_init(int n1, int n2, int n3, const double* __restrict__ bsm, double r1, double r2, double r3,
                            double pterm, double volterm, T* __restrict__ q) {
  const size_t ng = (size_t)n1 * n2 * n3;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < ng; t += (size_t)gridDim.x * blockDim.x) {
    const int k1 = (int)(t % n1), k2 = (int)((t / n1) % n2), k3 = (int)(t / ((size_t)n1 * n2));
    const int m1 = k1 < (n1 + 1) / 2 ? k1 : k1 - n1;
    const int m2 = k2 < (n2 + 1) / 2 ? k2 : k2 - n2;
    const int m3 = k3 < (n3 + 1) / 2 ? k3 : k3 - n3;
    double v = 0.0;
    if (m1 != 0 || m2 != 0 || m3 != 0) {
      const double h1 = r1 * m1, h2 = r2 * m2, h3 = r3 * m3;
      const double hsq = h1 * h1 + h2 * h2 + h3 * h3;
      const double term = -pterm * hsq;
      if (term > -50.0) v = exp(term) / (volterm * hsq * bsm[k1] * bsm[n1 + k2] * bsm[n1 + n2 + k3]);
    }
    q[t] = (T)v;
  }
}

}  // namespace

// B-spline moduli by grid length, computed once per process (an O(K^2)
// trigonometric sum per axis; servers re-target contexts to new grids often)
static const std::vector<double>& dftmod_cached(int nfft) {
  static std::mutex mu;
  static std::map<int, std::vector<double>> cache;
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(nfft);
  if (it == cache.end()) it = cache.emplace(nfft, dftmod_host(nfft, kBs)).first;
  return it->second;  // map nodes are stable: the reference outlives the lock
}

int pme_init(Ctx& c) {
  for (int d = 0; d < 3; ++d) c.nfft[d] = c.cfg.nfft[d];
  c.ngrid = (size_t)c.nfft[0] * c.nfft[1] * c.nfft[2];
  for (int d = 0; d < 3; ++d) c.a_frac[d] = (double)c.nfft[d] * c.box.recip[d];
  // influence function (newinduce_pme.f:1802-1854)
  const std::vector<double>& m1 = dftmod_cached(c.nfft[0]);
  const std::vector<double>& m2 = dftmod_cached(c.nfft[1]);
  const std::vector<double>& m3 = dftmod_cached(c.nfft[2]);
  size_t esz = c.mixed ? sizeof(float) : sizeof(double);
  size_t csz = c.mixed ? sizeof(cufftComplex) : sizeof(cufftDoubleComplex);
  // grid buffers are kept while they are large enough (a re-targeted
  // context reuses them)
  if (c.ngrid > c.cap_ngrid) {
    cudaFree(c.d_qfac);
    cudaFree(c.d_grid);
    c.d_qfac = c.d_grid = nullptr;
    c.cap_ngrid = 0;
    if (cuda_status(cudaMalloc(&c.d_qfac, esz * c.ngrid), &c, "alloc qfac")) return THP_E_CUDA;
    if (cuda_status(cudaMalloc(&c.d_grid, csz * c.ngrid), &c, "alloc grid")) return THP_E_CUDA;
    c.cap_ngrid = c.ngrid;
  }
  // influence function on the device (newinduce_pme.f:1802-1854): the
  // B-spline moduli go through the front of the grid buffer
  std::vector<double> bsm(m1.begin() + 1, m1.begin() + 1 + c.nfft[0]);
  bsm.insert(bsm.end(), m2.begin() + 1, m2.begin() + 1 + c.nfft[1]);
  bsm.insert(bsm.end(), m3.begin() + 1, m3.begin() + 1 + c.nfft[2]);
  double* d_bsm = reinterpret_cast<double*>(c.d_grid);  // ngrid complex >= n1+n2+n3 doubles
  cudaMemcpyAsync(d_bsm, bsm.data(), sizeof(double) * bsm.size(), cudaMemcpyHostToDevice, c.stream);
  const double a = c.cfg.aewald;
  const double pterm = (kPi / a) * (kPi / a);
  const double volterm = kPi * (c.cfg.box[0] * c.cfg.box[1] * c.cfg.box[2]);
  const int blocks = (int)std::min<size_t>((c.ngrid + 255) / 256, 148 * 16);
  if (c.mixed)
    k_qfac_init<float><<<blocks, 256, 0, c.stream>>>(c.nfft[0], c.nfft[1], c.nfft[2], d_bsm, c.box.recip[0],
                                                     c.box.recip[1], c.box.recip[2], pterm, volterm,
                                                     (float*)c.d_qfac);
  else
    k_qfac_init<double><<<blocks, 256, 0, c.stream>>>(c.nfft[0], c.nfft[1], c.nfft[2], d_bsm, c.box.recip[0],
                                                      c.box.recip[1], c.box.recip[2], pterm, volterm,
                                                      (double*)c.d_qfac);
  // no host wait: the influence function is ready, stream-ordered, for the
  // context's next solve (bsm is copied out before the call returns)
  if (cuda_status(cudaGetLastError(), &c, "qfac")) return THP_E_CUDA;
  // cuFFT dims: slowest first; data [n3][n2][n1]; the plan is kept when the
  // grid dimensions are unchanged
  const bool same = c.have_plan && c.plan_dims[0] == c.nfft[0] && c.plan_dims[1] == c.nfft[1] &&
                    c.plan_dims[2] == c.nfft[2];
  if (!same) {
    if (c.have_plan) give_plan(plan_key(c), c.plan);
    c.have_plan = false;
    for (int d = 0; d < 3; ++d) c.plan_dims[d] = c.nfft[d];
    if (!take_plan(plan_key(c), &c.plan)) {
      cufftResult r = cufftPlan3d(&c.plan, c.nfft[2], c.nfft[1], c.nfft[0], c.mixed ? CUFFT_C2C : CUFFT_Z2Z);
      if (r != CUFFT_SUCCESS) {
        c.last_msg = "cufftPlan3d failed";
        return THP_E_CUDA;
      }
    }
    c.have_plan = true;
  }
  cufftSetStream(c.plan, c.stream);
  return cuda_status(cudaGetLastError(), &c, "pme init");
}

// Plans one grid shape ahead of use (a server does this when a system is
// registered, so the first request of a new shape does not wait for it).
int plan_prefetch(int device, const int nfft[3], int mixed) {
  const PlanKey k{device, nfft[0], nfft[1], nfft[2], mixed};
  if (plan_cached(k)) return THP_OK;
  if (cudaSetDevice(device) != cudaSuccess) return THP_E_CUDA;
  cufftHandle plan;
  if (cufftPlan3d(&plan, nfft[2], nfft[1], nfft[0], mixed ? CUFFT_C2C : CUFFT_Z2Z) != CUFFT_SUCCESS)
    return THP_E_CUDA;
  give_plan(k, plan);
  return THP_OK;
}

void pme_free(Ctx& c) {
  if (c.have_plan) give_plan(plan_key(c), c.plan);
  c.have_plan = false;
  cudaFree(c.d_qfac);
  cudaFree(c.d_grid);
  c.d_qfac = c.d_grid = nullptr;
  c.cap_ngrid = 0;
}

int zero_grid(Ctx& c) {
  size_t csz = c.mixed ? sizeof(cufftComplex) : sizeof(cufftDoubleComplex);
  return cuda_status(cudaMemsetAsync(c.d_grid, 0, csz * c.ngrid, c.stream), &c, "zero grid");
}

// Permanent-multipole PME: d_cphi (and cphi10 when non-null) and, when
// with_e0, completes d_ef = E_direct - cphi(2:4) + (4/3) a^3/sqrt(pi) d.
int launch_mpole_grid(Ctx& c) {
  PmeGeom g = geom_of(c);
  int nb = (c.n + kBlock - 1) / kBlock;
  int st = zero_grid(c);
  if (st) return st;
  if (c.mixed)
    k_spread_mpole<float><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, c.d_rpole, (cufftComplex*)c.d_grid);
  else
    k_spread_mpole<double><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, c.d_rpole, (cufftDoubleComplex*)c.d_grid);
  if ((st = cuda_status(cudaGetLastError(), &c, "spread mpole"))) return st;
  return convolve(c, 0);
}

// blocks of the k-space virial sums (each writes 6 partial sums)
int kspace_virial_blocks() { return 148 * 2; }

static int kspace_virial(Ctx& c, int mode, double sign, double* d_part) {
  const double pterm = (kPi / c.cfg.aewald) * (kPi / c.cfg.aewald);
  const PmeGeom g = geom_of(c);
  if (c.mixed)
    k_kspace_virial<cufftComplex, float><<<kspace_virial_blocks(), 256, 0, c.stream>>>(
        g.n1, g.n2, g.n3, (const cufftComplex*)c.d_grid, (const float*)c.d_qfac, g.recip[0], g.recip[1], g.recip[2],
        pterm, kElectric, mode, sign, d_part);
  else
    k_kspace_virial<cufftDoubleComplex, double><<<kspace_virial_blocks(), 256, 0, c.stream>>>(
        g.n1, g.n2, g.n3, (const cufftDoubleComplex*)c.d_grid, (const double*)c.d_qfac, g.recip[0], g.recip[1],
        g.recip[2], pterm, kElectric, mode, sign, d_part);
  return cuda_status(cudaGetLastError(), &c, "k-space virial");
}

// launch_mpole_grid with, between the forward transform and qfac, the
// permanent-only scalar-sum virial (emrecip1), subtracted as eprecip1 does
// (epolar1.f:534-541): kspace_virial_blocks() rows of 6 into d_part.
int launch_mpole_grid_virial(Ctx& c, double* d_part, double sign) {
  PmeGeom g = geom_of(c);
  int nb = (c.n + kBlock - 1) / kBlock;
  int st = zero_grid(c);
  if (st) return st;
  if (c.mixed)
    k_spread_mpole<float><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, c.d_rpole, (cufftComplex*)c.d_grid);
  else
    k_spread_mpole<double><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, c.d_rpole, (cufftDoubleComplex*)c.d_grid);
  if ((st = cuda_status(cudaGetLastError(), &c, "spread mpole"))) return st;
  if ((st = fft(c, CUFFT_FORWARD))) return st;
  if ((st = kspace_virial(c, 0, sign, d_part))) return st;
  int blocks = 148 * 8;
  if (c.mixed)
    k_qfac<cufftComplex, float><<<blocks, 256, 0, c.stream>>>(c.ngrid, (const float*)c.d_qfac,
                                                             (cufftComplex*)c.d_grid, c.d_cg, 0);
  else
    k_qfac<cufftDoubleComplex, double><<<blocks, 256, 0, c.stream>>>(
        c.ngrid, (const double*)c.d_qfac, (cufftDoubleComplex*)c.d_grid, c.d_cg, 0);
  if ((st = cuda_status(cudaGetLastError(), &c, "qfac"))) return st;
  return fft(c, CUFFT_INVERSE);
}

// The (rpole + uinp) x (rpole + uind) scalar-sum virial of eprecip1
// (epolar1.f:932-1091) into kspace_virial_blocks() rows of d_part; uses
// (and leaves transformed) the context's grid.
int launch_pair_grid_virial(Ctx& c, double* d_part) {
  PmeGeom g = geom_of(c);
  int nb = (c.n + kBlock - 1) / kBlock;
  int st = zero_grid(c);
  if (st) return st;
  if (c.mixed)
    k_spread_mpole2<float><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, c.d_rpole, c.d_mu, (cufftComplex*)c.d_grid);
  else
    k_spread_mpole2<double><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, c.d_rpole, c.d_mu,
                                                         (cufftDoubleComplex*)c.d_grid);
  if ((st = cuda_status(cudaGetLastError(), &c, "spread mpole pair"))) return st;
  if ((st = fft(c, CUFFT_FORWARD))) return st;
  return kspace_virial(c, 1, 1.0, d_part);
}

int launch_efld0_recip_ex(Ctx& c, double* cphi10, bool with_e0) {
  int st = launch_mpole_grid(c);
  if (st) return st;
  return launch_gather_mpole(c, cphi10, with_e0);
}

int launch_gather_mpole(Ctx& c, double* cphi10, bool with_e0) {
  PmeGeom g = geom_of(c);
  int nb = (c.n + kBlock - 1) / kBlock;
  double a = c.cfg.aewald;
  double term = (4.0 / 3.0) * a * a * a / kSqrtPi;
  if (c.mixed)
    k_gather_mpole<float><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftComplex*)c.d_grid, c.d_rpole,
                                                       term, c.d_cphi, cphi10, with_e0 ? c.d_ef : nullptr);
  else
    k_gather_mpole<double><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftDoubleComplex*)c.d_grid,
                                                        c.d_rpole, term, c.d_cphi, cphi10,
                                                        with_e0 ? c.d_ef : nullptr);
  return cuda_status(cudaGetLastError(), &c, "gather mpole");
}

int launch_efld0_recip(Ctx& c) { return launch_efld0_recip_ex(c, nullptr, true); }

// Dipole PME pass.  mode 0: spread d_vec as is (the mixed form also writes
// its FP32 copy); mode 1: pp update first (CG loop, honours the stop flag);
// mode 2: spread as is, no FP32 copy, honours the stop flag.  d_out (if non-null) receives the gathered
// field gradient [n][6] (tmatxbrecip's dipfield); the CG loop passes null and
// gathers inside its fused matvec kernel.
// 1: the dipole spread of systems of at least THP_SPREAD_TILE_ATOMS (FP32
// grid) / THP_SPREAD_TILE_ATOMS_F64 atoms sums the stencils of 16
// neighbouring sites in a shared-memory tile per warp before adding them to
// the grid (at 288k atoms 105 -> 85 us per FP32 spread, 340 -> 200 us FP64);
// smaller systems, and 0, let every site add its own stencil (measured
// faster below those sizes: mixed solves of 4.5k-32k atoms against the tile's
// gain from 96k; FP64 solves of 4.5k-12k atoms against its gain from 32k).
#ifndef THP_SPREAD_TILE
#define THP_SPREAD_TILE 1
#endif
#ifndef THP_SPREAD_TILE_ATOMS
#define THP_SPREAD_TILE_ATOMS 50000
#endif
#ifndef THP_SPREAD_TILE_ATOMS_F64
#define THP_SPREAD_TILE_ATOMS_F64 20000
#endif

template <typename T, typename V, int TA>
static void spread_tiled(Ctx& c, const PmeGeom& g, V* vec, float* vf, int mode, typename Cplx<T>::type* grid) {
  constexpr size_t smem = sizeof(SpreadWarp<T>) * (kSpreadThreads / 32);
  static std::atomic<unsigned long long> limit_set{0};
  smem_limit_once(k_spread_dip<T, V, TA>, smem, limit_set);
  const int nb = (c.n + kSpreadThreads - 1) / kSpreadThreads;
  k_spread_dip<T, V, TA><<<nb, kSpreadThreads, smem, c.stream>>>(c.n, g, c.d_pos, vec, c.d_zr, vf, c.d_cg, mode,
                                                                  grid);
}

template <typename T, typename V>
static void spread_dipoles(Ctx& c, const PmeGeom& g, V* vec, float* vf, int mode, typename Cplx<T>::type* grid) {
  constexpr int kMin = std::is_same<T, float>::value ? THP_SPREAD_TILE_ATOMS : THP_SPREAD_TILE_ATOMS_F64;
  if (THP_SPREAD_TILE && c.n >= kMin)
    spread_tiled<T, V, 16>(c, g, vec, vf, mode, grid);
  else
    k_spread_dip<T, V, 0><<<(c.n + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, vec, c.d_zr, vf,
                                                                             c.d_cg, mode, grid);
}

int launch_pme_dipole(Ctx& c, const double* d_vec, double* d_out, int mode) {
  PmeGeom g = geom_of(c);
  int st = zero_grid(c);
  if (st) return st;
  float* vf = (c.mixed && mode != 2) ? c.d_vecf : nullptr;
  if (c.mixed)
    spread_dipoles<float, double>(c, g, const_cast<double*>(d_vec), vf, mode, (cufftComplex*)c.d_grid);
  else
    spread_dipoles<double, double>(c, g, const_cast<double*>(d_vec), vf, mode, (cufftDoubleComplex*)c.d_grid);
  if ((st = cuda_status(cudaGetLastError(), &c, "spread dip"))) return st;
  if ((st = convolve(c, mode >= 1))) return st;
  if (d_out) st = launch_gather_dip(c, d_out, false);
  return st;
}

// The overlapped mixed CG's spread of its FP32 search direction (mode 2:
// stop flag honoured, no update, no FP32 copy), then the convolution.
int launch_pme_dipole_f32(Ctx& c, const float* d_vec) {
  PmeGeom g = geom_of(c);
  int st = zero_grid(c);
  if (st) return st;
  spread_dipoles<float, float>(c, g, const_cast<float*>(d_vec), nullptr, 2, (cufftComplex*)c.d_grid);
  if ((st = cuda_status(cudaGetLastError(), &c, "spread dip"))) return st;
  return convolve(c, true);
}

int launch_gather_dip(Ctx& c, double* d_out, bool check_stop) {
  PmeGeom g = geom_of(c);
  const int nb = (c.n + kBlock - 1) / kBlock;
  if (c.mixed)
    k_gather_dip<float><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftComplex*)c.d_grid, d_out, c.d_cg,
                                                  check_stop ? 1 : 0);
  else
    k_gather_dip<double><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftDoubleComplex*)c.d_grid, d_out,
                                                   c.d_cg, check_stop ? 1 : 0);
  return cuda_status(cudaGetLastError(), &c, "gather dip");
}

PmeGeom pme_geom(const Ctx& c) { return geom_of(c); }

}  // namespace thp
