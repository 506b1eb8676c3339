// forces.cu -- polarization energy gradient on the device (epolar1c).
//
// Restates epolar1c (epolar1.f:57-372) for a converged solve:
//   * eprecip1 (epolar1.f:397-1213): the dipole grid of uind (Re) / uinp (Im)
//     gathered to all 20 potential derivatives (fphi_uind_site), combined with
//     the permanent-multipole potential fphirec kept from the field pass;
//   * epreal1c (epolar1.f:1215-2540, Thole branch): per pair the gradient of
//     the d- and p-scaled permanent field on uinp / uind and of the mutual
//     tensor (uscale) on uind x uinp, plus the induced field and its gradient
//     at every site for the torques;
//   * self torque (epolar1.f:190-206), and torque (torque.f:6-390) for the
//     Z-then-X and Bisector frames.
// One thread owns atom i over the full neighbor list (each pair is evaluated
// from both ends, the i-side terms only).  The three torques of a site are
// summed before one torque distribution.  Gradients are accumulated in 64-bit
// fixed point with 2^-34 kcal/mol/A resolution, so the order in which threads
// add their contributions does not change the sums.
#include <type_traits>

#include "grad_dev.cuh"
#include "kernels.h"
#include "pme_dev.cuh"
#include "realspace_dev.cuh"

namespace thp {

namespace {

constexpr int kBlock = 128;
// fphi_uind_site (pmestuff.f:746-1045) in full and the force / torque of
// eprecip1 (epolar1.f:636-720).  fphirec: [n][20] permanent potential
// (unscaled), written by the field pass.
// VIR: each block also writes the sum of its sites' induced-dipole virial
// terms (epolar1.f:846-908) to vpart[block][6].
template <typename T, bool VIR>
__global__ void __launch_bounds__(kBlock) k_force_recip(int n, PmeGeom g, const double4* __restrict__ pos,
                                                        const typename Cplx<T>::type* __restrict__ grid,
                                                        const double* __restrict__ fphirec,
                                                        const double* __restrict__ mu, const double* __restrict__ rp,
                                                        double* __restrict__ trq_out,
                                                        unsigned long long* __restrict__ dep,
                                                        double* __restrict__ vpart) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double vs[6] = {0, 0, 0, 0, 0, 0};
  if (i < n) {
  const double4 p = pos[i];
  T tx[kBs][4], ty[kBs][4], tz[kBs][4];
  const int gx = bspline_axis<4, T>(p.x, g.recip[0], g.n1, tx);
  const int gy = bspline_axis<4, T>(p.y, g.recip[1], g.n2, ty);
  const int gz = bspline_axis<4, T>(p.z, g.recip[2], g.n3, tz);
  // T1/T2: 100,010,001,200,020,002,110,101,011 of the d / p grids; S: 20 of their sum
  T T1[9] = {0}, T2[9] = {0}, S[20] = {0};
#pragma unroll
  for (int c = 0; c < kBs; ++c) {
    const size_t kk = (size_t)wrapk(gz + c, g.n3);
    const T v0 = tz[c][0], v1 = tz[c][1], v2 = tz[c][2], v3 = tz[c][3];
    T a1[6] = {0}, a2[6] = {0}, s[10] = {0};
#pragma unroll
    for (int b = 0; b < kBs; ++b) {
      const size_t jj = (size_t)wrapk(gy + b, g.n2);
      const T u0 = ty[b][0], u1 = ty[b][1], u2 = ty[b][2], u3 = ty[b][3];
      T ta[3] = {0, 0, 0}, tb[3] = {0, 0, 0}, t3 = 0;
      const size_t row = (kk * g.n2 + jj) * g.n1;
#pragma unroll
      for (int a = 0; a < kBs; ++a) {
        const auto q = grid[row + wrapk(gx + a, g.n1)];
        ta[0] += q.x * tx[a][0];
        ta[1] += q.x * tx[a][1];
        ta[2] += q.x * tx[a][2];
        tb[0] += q.y * tx[a][0];
        tb[1] += q.y * tx[a][1];
        tb[2] += q.y * tx[a][2];
        t3 += (q.x + q.y) * tx[a][3];
      }
      a1[0] += ta[0] * u0; a1[1] += ta[1] * u0; a1[2] += ta[0] * u1;
      a1[3] += ta[2] * u0; a1[4] += ta[1] * u1; a1[5] += ta[0] * u2;
      a2[0] += tb[0] * u0; a2[1] += tb[1] * u0; a2[2] += tb[0] * u1;
      a2[3] += tb[2] * u0; a2[4] += tb[1] * u1; a2[5] += tb[0] * u2;
      const T t0 = ta[0] + tb[0], t1 = ta[1] + tb[1], t2 = ta[2] + tb[2];
      s[0] += t0 * u0; s[1] += t1 * u0; s[2] += t0 * u1; s[3] += t2 * u0; s[4] += t1 * u1;
      s[5] += t0 * u2; s[6] += t3 * u0; s[7] += t2 * u1; s[8] += t1 * u2; s[9] += t0 * u3;
    }
    T1[0] += a1[1] * v0; T1[1] += a1[2] * v0; T1[2] += a1[0] * v1; T1[3] += a1[3] * v0; T1[4] += a1[5] * v0;
    T1[5] += a1[0] * v2; T1[6] += a1[4] * v0; T1[7] += a1[1] * v1; T1[8] += a1[2] * v1;
    T2[0] += a2[1] * v0; T2[1] += a2[2] * v0; T2[2] += a2[0] * v1; T2[3] += a2[3] * v0; T2[4] += a2[5] * v0;
    T2[5] += a2[0] * v2; T2[6] += a2[4] * v0; T2[7] += a2[1] * v1; T2[8] += a2[2] * v1;
    S[0] += s[0] * v0; S[1] += s[1] * v0; S[2] += s[2] * v0; S[3] += s[0] * v1; S[4] += s[3] * v0;
    S[5] += s[5] * v0; S[6] += s[0] * v2; S[7] += s[4] * v0; S[8] += s[1] * v1; S[9] += s[2] * v1;
    S[10] += s[6] * v0; S[11] += s[9] * v0; S[12] += s[0] * v3; S[13] += s[7] * v0; S[14] += s[3] * v1;
    S[15] += s[8] * v0; S[16] += s[5] * v1; S[17] += s[1] * v2; S[18] += s[2] * v2; S[19] += s[4] * v1;
  }
  // 1-based views as in the reference (scaled by electric)
  const double f = kElectric;
  double FD[11], FP[11], FS[21], FR[21];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    FD[q + 2] = f * (double)T1[q];
    FP[q + 2] = f * (double)T2[q];
  }
#pragma unroll
  for (int q = 0; q < 20; ++q) {
    FS[q + 1] = f * (double)S[q];
    FR[q + 1] = f * fphirec[(size_t)i * 20 + q];
  }
  const double* m = mu + (size_t)i * 6;
  const double fd[3] = {g.a[0] * m[0], g.a[1] * m[1], g.a[2] * m[2]};
  const double fp[3] = {g.a[0] * m[3], g.a[1] * m[4], g.a[2] * m[5]};
  const int d1[10] = {2, 5, 8, 9, 11, 16, 18, 14, 15, 20};
  const int d2[10] = {3, 8, 6, 10, 14, 12, 19, 16, 20, 17};
  const int d3[10] = {4, 9, 10, 7, 15, 17, 13, 20, 18, 19};
  double f1 = 0.0, f2 = 0.0, f3 = 0.0;
#pragma unroll
  for (int k = 1; k <= 3; ++k) {
    const double sdp = fd[k - 1] + fp[k - 1];
    f1 += sdp * FR[d1[k]] + fd[k - 1] * FP[d1[k]] + fp[k - 1] * FD[d1[k]];
    f2 += sdp * FR[d2[k]] + fd[k - 1] * FP[d2[k]] + fp[k - 1] * FD[d2[k]];
    f3 += sdp * FR[d3[k]] + fd[k - 1] * FP[d3[k]] + fp[k - 1] * FD[d3[k]];
  }
  // fmp of the permanent moments (cart_to_frac, orthogonal box)
  const double* r = rp + (size_t)i * 10;
  const double cm[10] = {r[0], r[1], r[2], r[3], r[4], r[7], r[9], 2.0 * r[5], 2.0 * r[6], 2.0 * r[8]};
  const double fm[10] = {cm[0], g.a[0] * cm[1], g.a[1] * cm[2], g.a[2] * cm[3], g.a[0] * g.a[0] * cm[4],
                         g.a[1] * g.a[1] * cm[5], g.a[2] * g.a[2] * cm[6], g.a[0] * g.a[1] * cm[7],
                         g.a[0] * g.a[2] * cm[8], g.a[1] * g.a[2] * cm[9]};
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    f1 += fm[k] * FS[d1[k]];
    f2 += fm[k] * FS[d2[k]];
    f3 += fm[k] * FS[d3[k]];
  }
  f1 = 0.5 * (double)g.n1 * f1;
  f2 = 0.5 * (double)g.n2 * f2;
  f3 = 0.5 * (double)g.n3 * f3;
  fix_add(dep + 3 * i + 0, g.recip[0] * f1);
  fix_add(dep + 3 * i + 1, g.recip[1] * f2);
  fix_add(dep + 3 * i + 2, g.recip[2] * f3);
  // cphidprec = fphi_to_cphi(fphidprec/2), torque on the permanent moments
  double cp[10];
  cp[0] = 0.5 * FS[1];
  cp[1] = g.a[0] * 0.5 * FS[2];
  cp[2] = g.a[1] * 0.5 * FS[3];
  cp[3] = g.a[2] * 0.5 * FS[4];
  cp[4] = g.a[0] * g.a[0] * 0.5 * FS[5];
  cp[5] = g.a[1] * g.a[1] * 0.5 * FS[6];
  cp[6] = g.a[2] * g.a[2] * 0.5 * FS[7];
  cp[7] = g.a[0] * g.a[1] * 0.5 * FS[8];
  cp[8] = g.a[0] * g.a[2] * 0.5 * FS[9];
  cp[9] = g.a[1] * g.a[2] * 0.5 * FS[10];
  double* t = trq_out + (size_t)i * 3;
  t[0] = cm[3] * cp[2] - cm[2] * cp[3] + 2.0 * (cm[6] - cm[5]) * cp[9] + cm[8] * cp[7] + cm[9] * cp[5] -
         cm[7] * cp[8] - cm[9] * cp[6];
  t[1] = cm[1] * cp[3] - cm[3] * cp[1] + 2.0 * (cm[4] - cm[6]) * cp[8] + cm[7] * cp[9] + cm[8] * cp[6] -
         cm[8] * cp[4] - cm[9] * cp[7];
  t[2] = cm[2] * cp[1] - cm[1] * cp[2] + 2.0 * (cm[5] - cm[4]) * cp[7] + cm[7] * cp[4] + cm[9] * cp[8] -
         cm[7] * cp[5] - cm[8] * cp[9];
  if (VIR) {
    // induced dipole contribution to the internal virial (epolar1.f:846-908):
    // cphim, cphid, cphip = Cartesian gradients of the permanent, d and p
    // potentials; 1-based cphidprec(1:10) = cp, cmp(1:10) = cm
    const double cmx[4] = {0, g.a[0] * FR[2], g.a[1] * FR[3], g.a[2] * FR[4]};
    const double cdx[4] = {0, g.a[0] * FD[2], g.a[1] * FD[3], g.a[2] * FD[4]};
    const double cpx[4] = {0, g.a[0] * FP[2], g.a[1] * FP[3], g.a[2] * FP[4]};
    const double ui[3] = {m[0], m[1], m[2]}, up[3] = {m[3], m[4], m[5]};
    vs[0] = -cp[1] * cm[1] - 0.5 * (cmx[1] * (ui[0] + up[0]) + cdx[1] * up[0] + cpx[1] * ui[0]);
    vs[1] = -0.5 * (cp[1] * cm[2] + cp[2] * cm[1]) -
            0.25 * (cmx[1] * (ui[1] + up[1]) + cmx[2] * (ui[0] + up[0]) + cdx[1] * up[1] + cpx[1] * ui[1] +
                    cdx[2] * up[0] + cpx[2] * ui[0]);
    vs[2] = -0.5 * (cp[1] * cm[3] + cp[3] * cm[1]) -
            0.25 * (cmx[1] * (ui[2] + up[2]) + cmx[3] * (ui[0] + up[0]) + cdx[1] * up[2] + cpx[1] * ui[2] +
                    cdx[3] * up[0] + cpx[3] * ui[0]);
    vs[3] = -cp[2] * cm[2] - 0.5 * (cmx[2] * (ui[1] + up[1]) + cdx[2] * up[1] + cpx[2] * ui[1]);
    vs[4] = -0.5 * (cp[2] * cm[3] + cp[3] * cm[2]) -
            0.25 * (cmx[2] * (ui[2] + up[2]) + cmx[3] * (ui[1] + up[1]) + cdx[2] * up[2] + cpx[2] * ui[2] +
                    cdx[3] * up[1] + cpx[3] * ui[1]);
    vs[5] = -cp[3] * cm[3] - 0.5 * (cmx[3] * (ui[2] + up[2]) + cdx[3] * up[2] + cpx[3] * ui[2]);
    vs[0] += -2.0 * cm[4] * cp[4] - cm[7] * cp[7] - cm[8] * cp[8];
    vs[1] += -(cm[4] + cm[5]) * cp[7] - 0.5 * (cm[7] * (cp[5] + cp[4]) + cm[8] * cp[9] + cm[9] * cp[8]);
    vs[2] += -(cm[4] + cm[6]) * cp[8] - 0.5 * (cm[8] * (cp[4] + cp[6]) + cm[7] * cp[9] + cm[9] * cp[7]);
    vs[3] += -2.0 * cm[5] * cp[5] - cm[7] * cp[7] - cm[9] * cp[9];
    vs[4] += -(cm[5] + cm[6]) * cp[9] - 0.5 * (cm[9] * (cp[5] + cp[6]) + cm[7] * cp[8] + cm[8] * cp[7]);
    vs[5] += -2.0 * cm[6] * cp[6] - cm[8] * cp[8] - cm[9] * cp[9];
  }
  }  // i < n
  if (VIR) {
    block_reduce<6>(vs);
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < 6; ++q) vpart[(size_t)blockIdx.x * 6 + q] = vs[q];
  }
}

// fphi_mpole_site (pmestuff.f:453-600): the 20 fractional potential
// derivatives of the permanent-multipole grid, unscaled.
template <typename T>
__global__ void __launch_bounds__(kBlock) k_fphi_mpole20(int n, PmeGeom g, const double4* __restrict__ pos,
                                                         const typename Cplx<T>::type* __restrict__ grid,
                                                         double* __restrict__ fphi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pos[i];
  T tx[kBs][4], ty[kBs][4], tz[kBs][4];
  const int gx = bspline_axis<4, T>(p.x, g.recip[0], g.n1, tx);
  const int gy = bspline_axis<4, T>(p.y, g.recip[1], g.n2, ty);
  const int gz = bspline_axis<4, T>(p.z, g.recip[2], g.n3, tz);
  T S[20] = {0};
#pragma unroll
  for (int c = 0; c < kBs; ++c) {
    const size_t kk = (size_t)wrapk(gz + c, g.n3);
    const T v0 = tz[c][0], v1 = tz[c][1], v2 = tz[c][2], v3 = tz[c][3];
    T s[10] = {0};  // 00,10,01,20,11,02,30,21,12,03
#pragma unroll
    for (int b = 0; b < kBs; ++b) {
      const size_t jj = (size_t)wrapk(gy + b, g.n2);
      const T u0 = ty[b][0], u1 = ty[b][1], u2 = ty[b][2], u3 = ty[b][3];
      T t0 = 0, t1 = 0, t2 = 0, t3 = 0;
      const size_t row = (kk * g.n2 + jj) * g.n1;
#pragma unroll
      for (int a = 0; a < kBs; ++a) {
        const T q = grid[row + wrapk(gx + a, g.n1)].x;
        t0 += q * tx[a][0];
        t1 += q * tx[a][1];
        t2 += q * tx[a][2];
        t3 += q * tx[a][3];
      }
      s[0] += t0 * u0; s[1] += t1 * u0; s[2] += t0 * u1; s[3] += t2 * u0; s[4] += t1 * u1;
      s[5] += t0 * u2; s[6] += t3 * u0; s[7] += t2 * u1; s[8] += t1 * u2; s[9] += t0 * u3;
    }
    S[0] += s[0] * v0; S[1] += s[1] * v0; S[2] += s[2] * v0; S[3] += s[0] * v1; S[4] += s[3] * v0;
    S[5] += s[5] * v0; S[6] += s[0] * v2; S[7] += s[4] * v0; S[8] += s[1] * v1; S[9] += s[2] * v1;
    S[10] += s[6] * v0; S[11] += s[9] * v0; S[12] += s[0] * v3; S[13] += s[7] * v0; S[14] += s[3] * v1;
    S[15] += s[8] * v0; S[16] += s[5] * v1; S[17] += s[1] * v2; S[18] += s[2] * v2; S[19] += s[4] * v1;
  }
  double* f = fphi + (size_t)i * 20;
#pragma unroll
  for (int q = 0; q < 20; ++q) f[q] = (double)S[q];
}

// sorted dipoles [n][6] FP64 -> [n][8] FP32 (d xyz, p xyz, 2 pad): one
// 256-bit load per partner in the mixed pair pass
__global__ void k_mu_f32(int n, const double* __restrict__ mu, float* __restrict__ muf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4* o = reinterpret_cast<float4*>(muf + (size_t)i * 8);
  const double* m = mu + (size_t)i * 6;
  o[0] = make_float4((float)m[0], (float)m[1], (float)m[2], (float)m[3]);
  o[1] = make_float4((float)m[4], (float)m[5], 0.f, 0.f);
}

struct EwC {
  double a, f1, f2, f3, f4;  // 2 a^2 powers / (sqrt(pi) a) of dampewald order 9
};

// epreal1c pair terms seen from atom i over its full list, the self torque,
// and the torque distribution of the summed torque of site i.
// resident blocks of the mixed gradient pass the register budget is cut for
#ifndef THP_FORCE_MINB
#define THP_FORCE_MINB 4
#endif

// lanes per site of the real-space gradient pass (1 or 8)
#ifndef THP_FORCE_LPA
#define THP_FORCE_LPA 8
#endif

// VIR: each block also writes to vpart[block][12] the sum of its sites' pair
// virials (epolar1.f:2326-2342, half from each end of a pair) and the
// frame-atom virial of their real-space torques (:2460-2486) in 0..5, and
// the frame-atom virial of their reciprocal and self torques, which the
// reference does not add, in 6..11.
// LPA: lanes per atom.  1: one thread per site over its whole list; 8: a
// warp takes four consecutive (cell-sorted) sites, eight lanes each, lane j
// taking list entries j, j+8, ...; the lanes' sums are combined in a fixed
// shuffle tree and the first lane of the site finishes it.
template <bool MIXED, bool VIR, int LPA>
__global__ void __launch_bounds__(kBlock, MIXED ? THP_FORCE_MINB : 1) k_force_real(
    int n, int npad, Box box, double off2, EwC ew, const double4* __restrict__ pos,
    const typename std::conditional<MIXED, float, double>::type* __restrict__ mrec, const double* __restrict__ mu,
    const float* __restrict__ erec, const float* __restrict__ muf, const int* __restrict__ perm,
    const int* __restrict__ sp_off, const int* __restrict__ sp_ks, const double* __restrict__ sp_s,
    const int* __restrict__ nnb, const int* __restrict__ nb, int maxnb, const int* __restrict__ frs,
    const double* __restrict__ trq_recip, unsigned long long* __restrict__ dep, double* __restrict__ vpart) {
  using T = typename std::conditional<MIXED, float, double>::type;
  static_assert(LPA == 1 || LPA == 8, "one or eight lanes per site");
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = LPA == 1 ? t : t >> 3, jl = LPA == 1 ? 0 : t & 7;
  const bool live = i0 < n;
  if (LPA == 1 && !live && !VIR) return;
  const int i = live ? i0 : n - 1;  // a valid site for the loads of idle lanes
  double vout[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  {
  const double4 pi4 = pos[i];
  // mixed form: partners from the 64-B FP32 site record (wrapped position,
  // 1/pdamp, thole, multipoles) and the FP32 dipole record, imaged in FP32
  float xi = 0.f, yi = 0.f, zi = 0.f;
  if constexpr (MIXED) {
    xi = erec[(size_t)i * 16 + 0];
    yi = erec[(size_t)i * 16 + 1];
    zi = erec[(size_t)i * 16 + 2];
  }
  const float bxf = (float)box.l[0], byf = (float)box.l[1], bzf = (float)box.l[2];
  const float hxf = 0.5f * bxf, hyf = 0.5f * byf, hzf = 0.5f * bzf;
  const float off2f = (float)off2;
  const T* ri = mrec + (size_t)i * 12;
  const T pti = (T)ri[0], ci = (T)ri[1], dix = (T)ri[2], diy = (T)ri[3], diz = (T)ri[4];
  const T qixx = (T)ri[5], qixy = (T)ri[6], qixz = (T)ri[7], qiyy = (T)ri[8], qiyz = (T)ri[9], qizz = (T)ri[10];
  const double* mi = mu + (size_t)i * 6;
  const T uix = (T)mi[0], uiy = (T)mi[1], uiz = (T)mi[2], uixp = (T)mi[3], uiyp = (T)mi[4], uizp = (T)mi[5];
  const T pdi = (T)pi4.w;
  const int io = perm[i];
  const int s0 = sp_off[io], s1 = sp_off[io + 1];
  const T f = (T)(0.5 * kElectric);
  double gx = 0.0, gy = 0.0, gz = 0.0;
  T uf[3] = {0, 0, 0}, duf[6] = {0, 0, 0, 0, 0, 0};
  T vp[6] = {0, 0, 0, 0, 0, 0};  // pair virial, half of each pair's
  const int nn = live ? min(nnb[i], maxnb) : 0;
#pragma unroll 1
  for (int s = jl; s < nn; s += LPA) {
    const int k = __ldg(nb + (size_t)s * npad + i);
    T xr, yr, zr, r2, pdk;
    T ptk, ck, dkx, dky, dkz, qkxx, qkxy, qkxz, qkyy, qkyz, qkzz;
    T ukx, uky, ukz, ukxp, ukyp, ukzp;
    if constexpr (MIXED) {
      float v[16];
      ld_rec8(erec + (size_t)k * 16, *reinterpret_cast<float(*)[8]>(&v[0]));
      float x = v[0] - xi, y = v[1] - yi, z = v[2] - zi;
      x = fabsf(x) > hxf ? x - copysignf(bxf, x) : x;
      y = fabsf(y) > hyf ? y - copysignf(byf, y) : y;
      z = fabsf(z) > hzf ? z - copysignf(bzf, z) : z;
      const float rf2 = x * x + y * y + z * z;
      if (rf2 > off2f) continue;
      ld_rec8(erec + (size_t)k * 16 + 8, *reinterpret_cast<float(*)[8]>(&v[8]));
      float u[8];
      ld_rec8(muf + (size_t)k * 8, u);
      xr = x;
      yr = y;
      zr = z;
      r2 = rf2;
      pdk = v[3] != 0.f ? 1.f / v[3] : 0.f;
      ptk = v[4];
      ck = v[5];
      dkx = v[6];
      dky = v[7];
      dkz = v[8];
      qkxx = v[9];
      qkxy = v[10];
      qkxz = v[11];
      qkyy = v[12];
      qkyz = v[13];
      qkzz = v[14];
      ukx = u[0];
      uky = u[1];
      ukz = u[2];
      ukxp = u[3];
      ukyp = u[4];
      ukzp = u[5];
    } else {
      const double4 pk4 = pos[k];
      double xrd = pk4.x - pi4.x, yrd = pk4.y - pi4.y, zrd = pk4.z - pi4.z;
      image3(box, xrd, yrd, zrd);
      const double r2d = r2_exact(xrd, yrd, zrd);
      if (r2d > off2) continue;
      xr = (T)xrd;
      yr = (T)yrd;
      zr = (T)zrd;
      r2 = (T)r2d;
      pdk = (T)pk4.w;
      const T* rk = mrec + (size_t)k * 12;
      ptk = (T)rk[0];
      ck = (T)rk[1];
      dkx = (T)rk[2];
      dky = (T)rk[3];
      dkz = (T)rk[4];
      qkxx = (T)rk[5];
      qkxy = (T)rk[6];
      qkxz = (T)rk[7];
      qkyy = (T)rk[8];
      qkyz = (T)rk[9];
      qkzz = (T)rk[10];
      const double* mk = mu + (size_t)k * 6;
      ukx = (T)mk[0];
      uky = (T)mk[1];
      ukz = (T)mk[2];
      ukxp = (T)mk[3];
      ukyp = (T)mk[4];
      ukzp = (T)mk[5];
    }
    T ds = 1, ps = 1, us = 1;
    for (int q = s0; q < s1; ++q)
      if (__ldg(sp_ks + q) == k) {
        ds = (T)sp_s[3 * q];
        ps = (T)sp_s[3 * q + 1];
        us = (T)sp_s[3 * q + 2];
        break;
      }
    // the mixed form: one rsqrt, then products in place of the divisions
    T r, rinv, r2inv;
    if constexpr (MIXED) {
      rinv = rsqrtf(r2);
      r = r2 * rinv;
      r2inv = rinv * rinv;
    } else {
      r = sqrt(r2);
      rinv = T(1) / r;
      r2inv = T(1) / r2;
    }
    const T dir = dix * xr + diy * yr + diz * zr;
    const T qix = qixx * xr + qixy * yr + qixz * zr, qiy = qixy * xr + qiyy * yr + qiyz * zr,
            qiz = qixz * xr + qiyz * yr + qizz * zr;
    const T qir = qix * xr + qiy * yr + qiz * zr;
    const T dkr = dkx * xr + dky * yr + dkz * zr;
    const T qkx = qkxx * xr + qkxy * yr + qkxz * zr, qky = qkxy * xr + qkyy * yr + qkyz * zr,
            qkz = qkxz * xr + qkyz * yr + qkzz * zr;
    const T qkr = qkx * xr + qky * yr + qkz * zr;
    const T uir = uix * xr + uiy * yr + uiz * zr, uirp = uixp * xr + uiyp * yr + uizp * zr;
    const T ukr = ukx * xr + uky * yr + ukz * zr, ukrp = ukxp * xr + ukyp * yr + ukzp * zr;
    T rr1, rr3, rr5, rr7, rr9, b0, b1, b2, b3, b4;
    // dampewald(9, r, r2, f) (damping.f:17-55)
    const T ra = (T)ew.a * r;
    const T ex = exp(-ra * ra);
    if constexpr (MIXED) {
      rr1 = f * rinv;
      rr3 = rr1 * r2inv;
      rr5 = T(3) * rr3 * r2inv;
      rr7 = T(5) * rr5 * r2inv;
      rr9 = T(7) * rr7 * r2inv;
      b0 = erfc(ra) * rinv;
      b1 = (b0 + (T)ew.f1 * ex) * r2inv;
      b2 = (T(3) * b1 + (T)ew.f2 * ex) * r2inv;
      b3 = (T(5) * b2 + (T)ew.f3 * ex) * r2inv;
      b4 = (T(7) * b3 + (T)ew.f4 * ex) * r2inv;
    } else {
      rr1 = f / r;
      rr3 = rr1 / r2;
      rr5 = T(3) * rr3 / r2;
      rr7 = T(5) * rr5 / r2;
      rr9 = T(7) * rr7 / r2;
      b0 = erfc(ra) / r;
      b1 = (b0 + (T)ew.f1 * ex) / r2;
      b2 = (T(3) * b1 + (T)ew.f2 * ex) / r2;
      b3 = (T(5) * b2 + (T)ew.f3 * ex) / r2;
      b4 = (T(7) * b3 + (T)ew.f4 * ex) / r2;
    }
    const T e3 = f * b1, e5 = f * b2, e7 = f * b3, e9 = f * b4;
    // Thole factors and their r-derivatives (epolar1.f:1620-1660)
    T sc3 = 1, sc5 = 1, sc7 = 1, rc3[3] = {0, 0, 0}, rc5[3] = {0, 0, 0}, rc7[3] = {0, 0, 0};
    T l3d = 1, l5d = 1, l7d = 1;  // damptholed order 7 for the energy-field (same values)
    T damp = pdi * pdk;
    T pg = min(pti, ptk);
    if (pg == T(0)) pg = max(pti, ptk);
    if (damp != T(0) && pg != T(0)) {
      const T t = MIXED ? r * (T(1) / damp) : r / damp;
      damp = pg * (t * t * t);
      if (damp < T(50)) {
        const T ed = exp(-damp);
        sc3 = T(1) - ed;
        sc5 = T(1) - (T(1) + damp) * ed;
        sc7 = T(1) - (T(1) + damp + T(0.6) * damp * damp) * ed;
        const T temp3 = MIXED ? T(3) * damp * ed * r2inv : T(3) * damp * ed / r2, temp5 = damp,
                temp7 = T(-0.2) + T(0.6) * damp;
        rc3[0] = xr * temp3;
        rc3[1] = yr * temp3;
        rc3[2] = zr * temp3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          rc5[j] = rc3[j] * temp5;
          rc7[j] = rc5[j] * temp7;
        }
        l3d = sc3;
        l5d = sc5;
        l7d = sc7;
      }
    }
    (void)l3d;
    (void)l5d;
    (void)l7d;
    const T psc3 = T(1) - sc3 * ps, psc5 = T(1) - sc5 * ps, psc7 = T(1) - sc7 * ps;
    const T dsc3 = T(1) - sc3 * ds, dsc5 = T(1) - sc5 * ds, dsc7 = T(1) - sc7 * ds;
    const T usc3 = T(1) - sc3 * us, usc5 = T(1) - sc5 * us;
    const T psr3 = e3 - psc3 * rr3, psr5 = e5 - psc5 * rr5, psr7 = e7 - psc7 * rr7;
    const T dsr3 = e3 - dsc3 * rr3, dsr5 = e5 - dsc5 * rr5, dsr7 = e7 - dsc7 * rr7;
    const T usr5 = e5 - usc5 * rr5;
    // induced field and gradient at i (ufld, dufld)
    {
      const T tix3 = psr3 * ukx + dsr3 * ukxp, tiy3 = psr3 * uky + dsr3 * ukyp, tiz3 = psr3 * ukz + dsr3 * ukzp;
      const T tuir3 = -psr5 * ukr - dsr5 * ukrp;
      uf[0] += tix3 + xr * tuir3;
      uf[1] += tiy3 + yr * tuir3;
      uf[2] += tiz3 + zr * tuir3;
      const T tix5 = T(2) * (psr5 * ukx + dsr5 * ukxp), tiy5 = T(2) * (psr5 * uky + dsr5 * ukyp),
              tiz5 = T(2) * (psr5 * ukz + dsr5 * ukzp);
      const T tuir = -psr7 * ukr - dsr7 * ukrp;
      duf[0] += xr * tix5 + xr * xr * tuir;
      duf[1] += xr * tiy5 + yr * tix5 + T(2) * xr * yr * tuir;
      duf[2] += yr * tiy5 + yr * yr * tuir;
      duf[3] += xr * tiz5 + zr * tix5 + T(2) * xr * zr * tuir;
      duf[4] += yr * tiz5 + zr * tiy5 + T(2) * yr * zr * tuir;
      duf[5] += zr * tiz5 + zr * zr * tuir;
    }
    // permanent-field gradient parts (d with uinp, p with uind)
    T frc[3] = {0, 0, 0};
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      const T s3 = part ? psc3 : dsc3, s5 = part ? psc5 : dsc5, s7 = part ? psc7 : dsc7;
      const T sr3 = part ? psr3 : dsr3, sr5 = part ? psr5 : dsr5, sr7 = part ? psr7 : dsr7;
      const T sc = part ? ps : ds;
      const T vkx = part ? ukx : ukxp, vky = part ? uky : ukyp, vkz = part ? ukz : ukzp;
      const T vix = part ? uix : uixp, viy = part ? uiy : uiyp, viz = part ? uiz : uizp;
      const T term1 = e5 - s3 * rr5, term2 = e7 - s5 * rr7, e9s = e9 - s7 * rr9;
      const T x3[3] = {rc3[0] * sc, rc3[1] * sc, rc3[2] * sc};
      const T x5[3] = {rc5[0] * sc, rc5[1] * sc, rc5[2] * sc};
      const T x7[3] = {rc7[0] * sc, rc7[1] * sc, rc7[2] * sc};
      T term3 = -sr3 + term1 * xr * xr - rr3 * xr * x3[0];
      T term4 = rr3 * x3[0] - term1 * xr - sr5 * xr;
      T term5 = term2 * xr * xr - sr5 - rr5 * xr * x5[0];
      T term6 = e9s * xr * xr - e7 - rr7 * xr * x7[0];
      T term7 = rr5 * x5[0] - T(2) * e7 * xr + (s5 + T(1.5) * s7) * rr7 * xr;
      const T tixx = ci * term3 + dix * term4 + dir * term5 + T(2) * sr5 * qixx + (qiy * yr + qiz * zr) * s7 * rr7 +
                     T(2) * qix * term7 + qir * term6;
      const T tkxx = ck * term3 - dkx * term4 - dkr * term5 + T(2) * sr5 * qkxx + (qky * yr + qkz * zr) * s7 * rr7 +
                     T(2) * qkx * term7 + qkr * term6;
      term3 = -sr3 + term1 * yr * yr - rr3 * yr * x3[1];
      term4 = rr3 * x3[1] - term1 * yr - sr5 * yr;
      term5 = term2 * yr * yr - sr5 - rr5 * yr * x5[1];
      term6 = e9s * yr * yr - e7 - rr7 * yr * x7[1];
      term7 = rr5 * x5[1] - T(2) * e7 * yr + (s5 + T(1.5) * s7) * rr7 * yr;
      const T tiyy = ci * term3 + diy * term4 + dir * term5 + T(2) * sr5 * qiyy + (qix * xr + qiz * zr) * s7 * rr7 +
                     T(2) * qiy * term7 + qir * term6;
      const T tkyy = ck * term3 - dky * term4 - dkr * term5 + T(2) * sr5 * qkyy + (qkx * xr + qkz * zr) * s7 * rr7 +
                     T(2) * qky * term7 + qkr * term6;
      term3 = -sr3 + term1 * zr * zr - rr3 * zr * x3[2];
      term4 = rr3 * x3[2] - term1 * zr - sr5 * zr;
      term5 = term2 * zr * zr - sr5 - rr5 * zr * x5[2];
      term6 = e9s * zr * zr - e7 - rr7 * zr * x7[2];
      term7 = rr5 * x5[2] - T(2) * e7 * zr + (s5 + T(1.5) * s7) * rr7 * zr;
      const T tizz = ci * term3 + diz * term4 + dir * term5 + T(2) * sr5 * qizz + (qix * xr + qiy * yr) * s7 * rr7 +
                     T(2) * qiz * term7 + qir * term6;
      const T tkzz = ck * term3 - dkz * term4 - dkr * term5 + T(2) * sr5 * qkzz + (qkx * xr + qky * yr) * s7 * rr7 +
                     T(2) * qkz * term7 + qkr * term6;
      term3 = term1 * xr * yr - rr3 * yr * x3[0];
      term4 = rr3 * x3[0] - term1 * xr;
      term5 = term2 * xr * yr - rr5 * yr * x5[0];
      term6 = e9s * xr * yr - rr7 * yr * x7[0];
      term7 = rr5 * x5[0] - term2 * xr;
      const T tixy = ci * term3 - sr5 * dix * yr + diy * term4 + dir * term5 + T(2) * sr5 * qixy -
                     T(2) * sr7 * yr * qix + T(2) * qiy * term7 + qir * term6;
      const T tkxy = ck * term3 + sr5 * dkx * yr - dky * term4 - dkr * term5 + T(2) * sr5 * qkxy -
                     T(2) * sr7 * yr * qkx + T(2) * qky * term7 + qkr * term6;
      term3 = term1 * xr * zr - rr3 * zr * x3[0];
      term5 = term2 * xr * zr - rr5 * zr * x5[0];
      term6 = e9s * xr * zr - rr7 * zr * x7[0];
      const T tixz = ci * term3 - sr5 * dix * zr + diz * term4 + dir * term5 + T(2) * sr5 * qixz -
                     T(2) * sr7 * zr * qix + T(2) * qiz * term7 + qir * term6;
      const T tkxz = ck * term3 + sr5 * dkx * zr - dkz * term4 - dkr * term5 + T(2) * sr5 * qkxz -
                     T(2) * sr7 * zr * qkx + T(2) * qkz * term7 + qkr * term6;
      term3 = term1 * yr * zr - rr3 * zr * x3[1];
      term4 = rr3 * x3[1] - term1 * yr;
      term5 = term2 * yr * zr - rr5 * zr * x5[1];
      term6 = e9s * yr * zr - rr7 * zr * x7[1];
      term7 = rr5 * x5[1] - term2 * yr;
      const T tiyz = ci * term3 - sr5 * diy * zr + diz * term4 + dir * term5 + T(2) * sr5 * qiyz -
                     T(2) * sr7 * zr * qiy + T(2) * qiz * term7 + qir * term6;
      const T tkyz = ck * term3 + sr5 * dky * zr - dkz * term4 - dkr * term5 + T(2) * sr5 * qkyz -
                     T(2) * sr7 * zr * qky + T(2) * qkz * term7 + qkr * term6;
      frc[0] += tixx * vkx + tixy * vky + tixz * vkz - tkxx * vix - tkxy * viy - tkxz * viz;
      frc[1] += tixy * vkx + tiyy * vky + tiyz * vkz - tkxy * vix - tkyy * viy - tkyz * viz;
      frc[2] += tixz * vkx + tiyz * vky + tizz * vkz - tkxz * vix - tkyz * viy - tkzz * viz;
    }
    // mutual part (uscale)
    {
      const T term1 = e5 - usc3 * rr5, term2 = e7 - usc5 * rr7, term3 = usr5 + term1;
      T term4 = rr3 * us;
      T term5 = -xr * term3 + rc3[0] * term4;
      T term6 = -usr5 + xr * xr * term2 - rr5 * xr * rc5[0] * us;
      const T tixx = uix * term5 + uir * term6, tkxx = ukx * term5 + ukr * term6;
      term5 = -yr * term3 + rc3[1] * term4;
      term6 = -usr5 + yr * yr * term2 - rr5 * yr * rc5[1] * us;
      const T tiyy = uiy * term5 + uir * term6, tkyy = uky * term5 + ukr * term6;
      term5 = -zr * term3 + rc3[2] * term4;
      term6 = -usr5 + zr * zr * term2 - rr5 * zr * rc5[2] * us;
      const T tizz = uiz * term5 + uir * term6, tkzz = ukz * term5 + ukr * term6;
      term4 = -usr5 * yr;
      term5 = -xr * term1 + rr3 * rc3[0] * us;
      term6 = xr * yr * term2 - rr5 * yr * rc5[0] * us;
      const T tixy = uix * term4 + uiy * term5 + uir * term6, tkxy = ukx * term4 + uky * term5 + ukr * term6;
      term4 = -usr5 * zr;
      term6 = xr * zr * term2 - rr5 * zr * rc5[0] * us;
      const T tixz = uix * term4 + uiz * term5 + uir * term6, tkxz = ukx * term4 + ukz * term5 + ukr * term6;
      term5 = -yr * term1 + rr3 * rc3[1] * us;
      term6 = yr * zr * term2 - rr5 * zr * rc5[1] * us;
      const T tiyz = uiy * term4 + uiz * term5 + uir * term6, tkyz = uky * term4 + ukz * term5 + ukr * term6;
      frc[0] += tixx * ukxp + tixy * ukyp + tixz * ukzp + tkxx * uixp + tkxy * uiyp + tkxz * uizp;
      frc[1] += tixy * ukxp + tiyy * ukyp + tiyz * ukzp + tkxy * uixp + tkyy * uiyp + tkyz * uizp;
      frc[2] += tixz * ukxp + tiyz * ukyp + tizz * ukzp + tkxz * uixp + tkyz * uiyp + tkzz * uizp;
    }
    gx -= (double)frc[0];
    gy -= (double)frc[1];
    gz -= (double)frc[2];
    if (VIR) {
      const T h = T(0.5);
      vp[0] += h * (xr * frc[0]);
      vp[1] += h * (T(0.5) * (yr * frc[0] + xr * frc[1]));
      vp[2] += h * (T(0.5) * (zr * frc[0] + xr * frc[2]));
      vp[3] += h * (yr * frc[1]);
      vp[4] += h * (T(0.5) * (zr * frc[1] + yr * frc[2]));
      vp[5] += h * (zr * frc[2]);
    }
  }
  if (LPA == 8) {
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      gx += __shfl_xor_sync(0xffffffffu, gx, o);
      gy += __shfl_xor_sync(0xffffffffu, gy, o);
      gz += __shfl_xor_sync(0xffffffffu, gz, o);
#pragma unroll
      for (int q = 0; q < 3; ++q) uf[q] += __shfl_xor_sync(0xffffffffu, uf[q], o);
#pragma unroll
      for (int q = 0; q < 6; ++q) duf[q] += __shfl_xor_sync(0xffffffffu, duf[q], o);
      if (VIR)
#pragma unroll
        for (int q = 0; q < 6; ++q) vp[q] += __shfl_xor_sync(0xffffffffu, vp[q], o);
    }
  }
  if (live && jl == 0) {
  fix_add(dep + 3 * i + 0, gx);
  fix_add(dep + 3 * i + 1, gy);
  fix_add(dep + 3 * i + 2, gz);
  // torques: real-space induced field (epolar1.f:2427-2470) + reciprocal + self
  const double* u6 = mu + (size_t)i * 6;
  const double sterm = (4.0 / 3.0) * kElectric * ew.a * ew.a * ew.a / kSqrtPi;
  const double hx = 0.5 * (u6[0] + u6[3]), hy = 0.5 * (u6[1] + u6[4]), hz = 0.5 * (u6[2] + u6[5]);
  const double rdx = (double)ri[2], rdy = (double)ri[3], rdz = (double)ri[4];
  double tep[3];
  tep[0] = (double)(diz * uf[1] - diy * uf[2] + qixz * duf[1] - qixy * duf[3] + T(2) * qiyz * (duf[2] - duf[5]) +
                    (qizz - qiyy) * duf[4]);
  tep[1] = (double)(dix * uf[2] - diz * uf[0] - qiyz * duf[1] + qixy * duf[4] + T(2) * qixz * (duf[5] - duf[0]) +
                    (qixx - qizz) * duf[3]);
  tep[2] = (double)(diy * uf[0] - dix * uf[1] + qiyz * duf[3] - qixz * duf[4] + T(2) * qixy * (duf[0] - duf[2]) +
                    (qiyy - qixx) * duf[1]);
  const int iz = frs[3 * i], ix = frs[3 * i + 1], axt = frs[3 * i + 2];
  if (VIR) {
#pragma unroll
    for (int q = 0; q < 6; ++q) vout[q] = (double)vp[q];
    if (axt == 1 || axt == 2) {
      // the real-space torque (in the reference's virial) and the reciprocal +
      // self torque (not in it), converted apart; the gradient takes both
      const double tx[3] = {trq_recip[(size_t)i * 3 + 0] + sterm * (rdy * hz - rdz * hy),
                            trq_recip[(size_t)i * 3 + 1] + sterm * (rdz * hx - rdx * hz),
                            trq_recip[(size_t)i * 3 + 2] + sterm * (rdx * hy - rdy * hx)};
      double du[3], dv[3], dux[3], dvx[3];
      torque_frame(pos, i, iz, ix, axt, tep, du, dv);
      torque_frame(pos, i, iz, ix, axt, tx, dux, dvx);
      double vr[6] = {0, 0, 0, 0, 0, 0}, vx[6] = {0, 0, 0, 0, 0, 0};
      frame_virial(pos, i, iz, ix, du, dv, vr);
      frame_virial(pos, i, iz, ix, dux, dvx, vx);
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        vout[q] += vr[q];
        vout[6 + q] = vx[q];
      }
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        fix_add(dep + 3 * iz + j, du[j] + dux[j]);
        fix_add(dep + 3 * ix + j, dv[j] + dvx[j]);
        fix_add(dep + 3 * i + j, -(du[j] + dux[j]) - (dv[j] + dvx[j]));
      }
    }
  } else {
    tep[0] += trq_recip[(size_t)i * 3 + 0] + sterm * (rdy * hz - rdz * hy);
    tep[1] += trq_recip[(size_t)i * 3 + 1] + sterm * (rdz * hx - rdx * hz);
    tep[2] += trq_recip[(size_t)i * 3 + 2] + sterm * (rdx * hy - rdy * hx);
    if (axt == 1 || axt == 2) torque_dist(pos, i, iz, ix, axt, tep, dep);
  }
  }  // the site's first lane
  }
  if (VIR) {
    block_reduce<12>(vout);
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < 12; ++q) vpart[(size_t)blockIdx.x * 12 + q] = vout[q];
  }
}

// The virial of one gradient call from the partial sums, in a fixed order:
// nk rows of 6 (k-space sums), nr rows of 6 (reciprocal sites), ne rows of
// 12 (real space: the reference's terms, then the reciprocal and self
// torques' frame-atom terms).  out: 6 + 6 (xx xy xz yy yz zz twice).
__global__ void __launch_bounds__(256) k_virial_sum(int nk, const double* __restrict__ kpart, int nr,
                                                     const double* __restrict__ rpart, int ne,
                                                     const double* __restrict__ epart, double* __restrict__ out) {
  double v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nk; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] += kpart[(size_t)b * 6 + q];
  for (int b = threadIdx.x; b < nr; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] += rpart[(size_t)b * 6 + q];
  for (int b = threadIdx.x; b < ne; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < 12; ++q) v[q] += epart[(size_t)b * 12 + q];
  block_reduce<12>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 12; ++q) out[q] = v[q];
}

}  // namespace

template <typename P>
static int alloc_once(Ctx& c, P** p, size_t count, const char* what) {
  if (*p) return THP_OK;
  return cuda_status(cudaMalloc((void**)p, sizeof(P) * count), &c, what);
}

// fphirec [n][20] (unscaled) of the convolved permanent-multipole grid
int launch_fphi_mpole20(Ctx& c) {
  int st = alloc_once(c, &c.d_fphirec, 20 * (size_t)c.n, "alloc fphirec");
  if (st) return st;
  const int nb = (c.n + kBlock - 1) / kBlock;
  PmeGeom g = pme_geom(c);
  if (c.mixed)
    k_fphi_mpole20<float><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftComplex*)c.d_grid, c.d_fphirec);
  else
    k_fphi_mpole20<double><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftDoubleComplex*)c.d_grid,
                                                        c.d_fphirec);
  return cuda_status(cudaGetLastError(), &c, "fphi mpole");
}

// sorted frame atoms of every site into d_frs
int launch_frames_sorted(Ctx& c) {
  int st = alloc_once(c, &c.d_frs, 3 * (size_t)c.n, "alloc frames");
  if (st) return st;
  const int nb = (c.n + kBlock - 1) / kBlock;
  k_frames_sorted<<<nb, kBlock, 0, c.stream>>>(c.n, c.d_perm, c.d_iperm, c.d_frames, c.d_frs);
  return cuda_status(cudaGetLastError(), &c, "frames");
}

// fixed-point gradient (sorted) -> dE/dx [n][3] in original order
int launch_gradient_out(Ctx& c, const unsigned long long* dep, double* d_out) {
  const int nb = (c.n + kBlock - 1) / kBlock;
  k_dep_out<<<nb, kBlock, 0, c.stream>>>(c.n, c.d_perm, dep, d_out);
  return cuda_status(cudaGetLastError(), &c, "gradient out");
}

// Partial-sum rows of one gradient call's virial: 2 kspace_virial_blocks()
// rows of 6 (k-space sums), nb rows of 6 and nb rows of 12 (per-block site
// and pair terms), then 12 totals; grown on demand.
int virial_scratch(Ctx& c, int nr, int ne, double** kpart, double** rpart, double** epart) {
  const int nk = 2 * kspace_virial_blocks();
  const size_t rows = (size_t)nk * 6 + (size_t)nr * 6 + (size_t)ne * 12 + 12;
  if (c.virp_cap < rows) {
    cudaFree(c.d_virp);
    c.d_virp = nullptr;
    c.virp_cap = 0;
    int st = cuda_status(cudaMalloc((void**)&c.d_virp, sizeof(double) * rows), &c, "alloc virial");
    if (st) return st;
    c.virp_cap = rows;
  }
  *kpart = c.d_virp;
  *rpart = *kpart + (size_t)nk * 6;
  *epart = *rpart + (size_t)nr * 6;
  return THP_OK;
}

// The 12 totals of the partial sums (in a fixed order; nk k-space rows)
// copied to h_out when the stream reaches them.
int virial_total(Ctx& c, int nk, int nr, int ne, const double* kpart, const double* rpart, const double* epart,
                 double* h_out) {
  double* tot = const_cast<double*>(epart) + (size_t)ne * 12;
  k_virial_sum<<<1, 256, 0, c.stream>>>(nk, kpart, nr, rpart, ne, epart, tot);
  const int st = cuda_status(cudaGetLastError(), &c, "virial sum");
  if (!st) cudaMemcpyAsync(h_out, tot, sizeof(double) * 12, cudaMemcpyDeviceToHost, c.stream);
  return st;
}

// Gradient of the polarization energy for the converged dipoles in d_mu
// (sorted); writes dE/dx [n][3] in ORIGINAL atom order into d_out.
int launch_forces(Ctx& c, double* d_out) {
  int st;
  const int nb = (c.n + kBlock - 1) / kBlock;
  if (!c.have_axes) return THP_E_STATE;
  const size_t n = c.n;
  if ((st = alloc_once(c, &c.d_fphirec, 20 * n, "alloc fphirec"))) return st;
  if ((st = alloc_once(c, &c.d_depfix, 3 * n, "alloc gradient"))) return st;
  if ((st = alloc_once(c, &c.d_trq, 3 * n, "alloc torque"))) return st;
  if ((st = alloc_once(c, &c.d_frs, 3 * n, "alloc frames"))) return st;
  const bool vir = c.want_virial;
  const int nk = 2 * kspace_virial_blocks();
  double *kpart = nullptr, *rpart = nullptr, *epart = nullptr;
  // the real-space pass: eight lanes per site (blocks of 16 sites)
  const int nbr = THP_FORCE_LPA == 8 ? (c.n + 15) / 16 : nb;
  if (vir && (st = virial_scratch(c, nb, nbr, &kpart, &rpart, &epart))) return st;
  unsigned long long* dep = c.d_depfix;
  if ((st = cuda_status(cudaMemsetAsync(dep, 0, sizeof(unsigned long long) * 3 * n, c.stream), &c, "zero gradient")))
    return st;
  k_frames_sorted<<<nb, kBlock, 0, c.stream>>>(c.n, c.d_perm, c.d_iperm, c.d_frames, c.d_frs);
  PmeGeom g = pme_geom(c);
  // permanent-multipole potential, 20 derivatives per site (and the
  // permanent-only k-space virial, subtracted)
  if ((st = vir ? launch_mpole_grid_virial(c, kpart, -1.0) : launch_mpole_grid(c))) return st;
  if ((st = launch_fphi_mpole20(c))) return st;
  // dipole grid of uind (Re) / uinp (Im), convolved
  if ((st = launch_pme_dipole(c, c.d_mu, nullptr, 0))) return st;
#define THP_RECIP_ARGS c.n, g, c.d_pos, c.d_grid, c.d_fphirec, c.d_mu, c.d_rpole, c.d_trq, dep, rpart
  if (c.mixed && vir)
    k_force_recip<float, true><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftComplex*)c.d_grid,
                                                            c.d_fphirec, c.d_mu, c.d_rpole, c.d_trq, dep, rpart);
  else if (c.mixed)
    k_force_recip<float, false><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftComplex*)c.d_grid,
                                                             c.d_fphirec, c.d_mu, c.d_rpole, c.d_trq, dep, rpart);
  else if (vir)
    k_force_recip<double, true><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftDoubleComplex*)c.d_grid,
                                                             c.d_fphirec, c.d_mu, c.d_rpole, c.d_trq, dep, rpart);
  else
    k_force_recip<double, false><<<nb, kBlock, 0, c.stream>>>(c.n, g, c.d_pos, (const cufftDoubleComplex*)c.d_grid,
                                                              c.d_fphirec, c.d_mu, c.d_rpole, c.d_trq, dep, rpart);
#undef THP_RECIP_ARGS
  if ((st = cuda_status(cudaGetLastError(), &c, "force recip"))) return st;
  // (rpole + uinp) x (rpole + uind) k-space virial: the grid is free again
  if (vir && (st = launch_pair_grid_virial(c, kpart + (size_t)kspace_virial_blocks() * 6))) return st;
  EwC ew;
  const double a = c.cfg.aewald;
  double aesq2 = 2.0 * a * a, afac = 1.0 / (kSqrtPi * a);
  ew.a = a;
  afac *= aesq2;
  ew.f1 = afac;
  afac *= aesq2;
  ew.f2 = afac;
  afac *= aesq2;
  ew.f3 = afac;
  afac *= aesq2;
  ew.f4 = afac;
  const double off2 = c.cfg.ewaldcut * c.cfg.ewaldcut;
  if (c.mixed) {
    if ((st = alloc_once(c, &c.d_muf, 8 * n, "alloc dipoles f32"))) return st;
    k_mu_f32<<<nb, kBlock, 0, c.stream>>>(c.n, c.d_mu, c.d_muf);
    if ((st = cuda_status(cudaGetLastError(), &c, "dipoles f32"))) return st;
  }
#define THP_FORCE_ARGS                                                                                      \
  c.n, c.npad, c.box, off2, ew, c.d_pos, MREC, c.d_mu, c.d_erec, c.d_muf, c.d_perm, c.d_sp_off, c.d_sp_ks, \
      c.d_sp_s, c.d_nnb, c.d_nb, c.maxnb, c.d_frs, c.d_trq, dep, epart
  constexpr int LPA = THP_FORCE_LPA;
  if (c.mixed) {
#define MREC c.d_mrecf
    if (vir)
      k_force_real<true, true, LPA><<<nbr, kBlock, 0, c.stream>>>(THP_FORCE_ARGS);
    else
      k_force_real<true, false, LPA><<<nbr, kBlock, 0, c.stream>>>(THP_FORCE_ARGS);
#undef MREC
  } else {
#define MREC c.d_mrec
    if (vir)
      k_force_real<false, true, LPA><<<nbr, kBlock, 0, c.stream>>>(THP_FORCE_ARGS);
    else
      k_force_real<false, false, LPA><<<nbr, kBlock, 0, c.stream>>>(THP_FORCE_ARGS);
#undef MREC
  }
#undef THP_FORCE_ARGS
  if ((st = cuda_status(cudaGetLastError(), &c, "force real"))) return st;
  if (vir && (st = virial_total(c, nk, nb, nbr, kpart, rpart, epart, c.h_vir))) return st;
  k_dep_out<<<nb, kBlock, 0, c.stream>>>(c.n, c.d_perm, dep, d_out);
  return cuda_status(cudaGetLastError(), &c, "force out");
}

}  // namespace thp
