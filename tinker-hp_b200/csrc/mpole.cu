// mpole.cu -- permanent-multipole energy and gradient on the device (empole1c).
//
// Restates empole1c (empole1.f:42-340) for the TINFOIL boundary, without
// charge penetration, charge flux or lambda dynamics (the AMOEBA terms):
//   * emrecip1 (empole1.f:349-861): the convolved permanent-multipole grid --
//     the one the polarization solve builds for its direct field -- gathered
//     to the 20 fractional potential derivatives of every site; energy
//     1/2 sum fmp.fphi, gradient from the derivative indices deriv1..3 and the
//     torque from cphi (fphi_to_cphi);
//   * emreal1c (empole1.f:873-1555, standard branch): Ewald-damped
//     multipole-multipole pair terms to order 11 with the 1-2..1-5 mscale
//     factors;
//   * the Ewald self energy (empole1.f:134-160);
//   * torque (torque.f:6-390) of each site's summed torque.
// One thread owns site i over the full neighbor list: each pair is evaluated
// from both ends, and each end keeps its own force, torque and half of the
// pair energy (the reference's Newton's-third-law half-list loop gives the
// same sums).  Gradients are accumulated in 64-bit fixed point, the energy
// by per-block partials summed in block order, so both are deterministic.
#include <type_traits>

#include "grad_dev.cuh"
#include "kernels.h"
#include "pme_dev.cuh"
#include "realspace_dev.cuh"

namespace thp {

namespace {

constexpr int kBlock = 128;

// resident blocks of the mixed pair kernel the register budget is cut for
#ifndef THP_EMPOLE_MINB
#define THP_EMPOLE_MINB 6
#endif

struct EwM {
  double a;
  double f[5];  // (2 a^2)^j / (sqrt(pi) a), j = 1..5 (dampewald order 11)
};

struct MScale {
  double v[5];  // m2scale..m5scale, then 1 for pairs outside the 1-2..1-5 lists
};

// emreal1c pair terms (standard branch) seen from site i: adds half the pair
// energy, the force on i and the torque on i.  m = (q, d, Qxx, Qxy, Qxz,
// Qyy, Qyz, Qzz) of each site; scalek = 1 - mscale.
// v6 (optional): adds half the pair's virial (empole1.f:1428-1442; the
// other half comes from the k end) as xx xy xz yy yz zz.
template <typename U>
__device__ __forceinline__ void mpole_pair(U xr, U yr, U zr, U r2, U scalek, const U* mi, const U* mk, const EwM& ew,
                                           double& e_acc, double g[3], double t[3], double* v6 = nullptr) {
  const U ci = mi[0], dix = mi[1], diy = mi[2], diz = mi[3];
  const U qixx = mi[4], qixy = mi[5], qixz = mi[6], qiyy = mi[7], qiyz = mi[8], qizz = mi[9];
  const U ck = mk[0], dkx = mk[1], dky = mk[2], dkz = mk[3];
  const U qkxx = mk[4], qkxy = mk[5], qkxz = mk[6], qkyy = mk[7], qkyz = mk[8], qkzz = mk[9];
  const U f = (U)kElectric;
  // one reciprocal square root, then products (FP32: the approximate rsqrt)
  U rinv;
  if constexpr (std::is_same<U, float>::value)
    rinv = rsqrtf(r2);
  else
    rinv = U(1) / sqrt(r2);
  const U r = r2 * rinv;
  const U r2inv = rinv * rinv;
  // intermediates involving moments and separation distance
  const U dir = dix * xr + diy * yr + diz * zr;
  const U qix = qixx * xr + qixy * yr + qixz * zr, qiy = qixy * xr + qiyy * yr + qiyz * zr,
          qiz = qixz * xr + qiyz * yr + qizz * zr;
  const U qir = qix * xr + qiy * yr + qiz * zr;
  const U dkr = dkx * xr + dky * yr + dkz * zr;
  const U qkx = qkxx * xr + qkxy * yr + qkxz * zr, qky = qkxy * xr + qkyy * yr + qkyz * zr,
          qkz = qkxz * xr + qkyz * yr + qkzz * zr;
  const U qkr = qkx * xr + qky * yr + qkz * zr;
  const U dik = dix * dkx + diy * dky + diz * dkz;
  const U qik = qix * qkx + qiy * qky + qiz * qkz;
  const U diqk = dix * qkx + diy * qky + diz * qkz;
  const U dkqi = dkx * qix + dky * qiy + dkz * qiz;
  const U qiqk = U(2) * (qixy * qkxy + qixz * qkxz + qiyz * qkyz) + qixx * qkxx + qiyy * qkyy + qizz * qkzz;
  // reciprocal distance terms with the Ewald damping to order 11
  // (damping.f:17-55); the bare terms only for scaled pairs
  const U ra = (U)ew.a * r;
  const U ex = exp(-ra * ra);
  const U b0 = erfc(ra) * rinv;
  const U b1 = (b0 + (U)ew.f[0] * ex) * r2inv;
  const U b2 = (U(3) * b1 + (U)ew.f[1] * ex) * r2inv;
  const U b3 = (U(5) * b2 + (U)ew.f[2] * ex) * r2inv;
  const U b4 = (U(7) * b3 + (U)ew.f[3] * ex) * r2inv;
  const U b5 = (U(9) * b4 + (U)ew.f[4] * ex) * r2inv;
  U rr1 = f * b0, rr3 = f * b1, rr5 = f * b2, rr7 = f * b3, rr9 = f * b4, rr11 = f * b5;
  if (scalek != U(0)) {
    const U s1 = f * rinv;
    const U s3 = s1 * r2inv;
    const U s5 = U(3) * s3 * r2inv;
    const U s7 = U(5) * s5 * r2inv;
    const U s9 = U(7) * s7 * r2inv;
    const U s11 = U(9) * s9 * r2inv;
    rr1 -= scalek * s1;
    rr3 -= scalek * s3;
    rr5 -= scalek * s5;
    rr7 -= scalek * s7;
    rr9 -= scalek * s9;
    rr11 -= scalek * s11;
  }
  const U term1 = ci * ck;
  const U term2 = ck * dir - ci * dkr + dik;
  const U term3 = ci * qkr + ck * qir - dir * dkr + U(2) * (dkqi - diqk + qiqk);
  const U term4 = dir * qkr - dkr * qir - U(4) * qik;
  const U term5 = qir * qkr;
  const U e = term1 * rr1 + term2 * rr3 + term3 * rr5 + term4 * rr7 + term5 * rr9;
  const U de = term1 * rr3 + term2 * rr5 + term3 * rr7 + term4 * rr9 + term5 * rr11;
  const U t1 = -ck * rr3 + dkr * rr5 - qkr * rr7;
  const U t2 = ci * rr3 + dir * rr5 + qir * rr7;
  const U t3 = U(2) * rr5;
  const U t4 = U(-2) * (ck * rr5 - dkr * rr7 + qkr * rr9);
  const U t5 = U(-2) * (ci * rr5 + dir * rr7 + qir * rr9);
  const U t6 = U(4) * rr7;
  // force on site i (emreal1c's frc; the k end computes its own)
  const U qixk = qixx * qkx + qixy * qky + qixz * qkz;
  const U qiyk = qixy * qkx + qiyy * qky + qiyz * qkz;
  const U qizk = qixz * qkx + qiyz * qky + qizz * qkz;
  const U qkxi = qkxx * qix + qkxy * qiy + qkxz * qiz;
  const U qkyi = qkxy * qix + qkyy * qiy + qkyz * qiz;
  const U qkzi = qkxz * qix + qkyz * qiy + qkzz * qiz;
  const U diqkx = dix * qkxx + diy * qkxy + diz * qkxz;
  const U diqky = dix * qkxy + diy * qkyy + diz * qkyz;
  const U diqkz = dix * qkxz + diy * qkyz + diz * qkzz;
  const U dkqix = dkx * qixx + dky * qixy + dkz * qixz;
  const U dkqiy = dkx * qixy + dky * qiyy + dkz * qiyz;
  const U dkqiz = dkx * qixz + dky * qiyz + dkz * qizz;
  const double fx = (double)(de * xr + t1 * dix + t2 * dkx + t3 * (diqkx - dkqix) + t4 * qix + t5 * qkx +
                             t6 * (qixk + qkxi));
  const double fy = (double)(de * yr + t1 * diy + t2 * dky + t3 * (diqky - dkqiy) + t4 * qiy + t5 * qky +
                             t6 * (qiyk + qkyi));
  const double fz = (double)(de * zr + t1 * diz + t2 * dkz + t3 * (diqkz - dkqiz) + t4 * qiz + t5 * qkz +
                             t6 * (qizk + qkzi));
  g[0] += fx;
  g[1] += fy;
  g[2] += fz;
  if (v6) {
    const double x = xr, y = yr, z = zr;
    v6[0] -= 0.5 * x * fx;
    v6[1] -= 0.25 * (y * fx + x * fy);
    v6[2] -= 0.25 * (z * fx + x * fz);
    v6[3] -= 0.5 * y * fy;
    v6[4] -= 0.25 * (z * fy + y * fz);
    v6[5] -= 0.5 * z * fz;
  }
  // torque on site i (emreal1c's ttmi)
  const U dirx = diy * zr - diz * yr, diry = diz * xr - dix * zr, dirz = dix * yr - diy * xr;
  const U dikx = diy * dkz - diz * dky, diky = diz * dkx - dix * dkz, dikz = dix * dky - diy * dkx;
  const U qirx = qiz * yr - qiy * zr, qiry = qix * zr - qiz * xr, qirz = qiy * xr - qix * yr;
  const U qikx = qky * qiz - qkz * qiy, qiky = qkz * qix - qkx * qiz, qikz = qkx * qiy - qky * qix;
  const U qikrx = qizk * yr - qiyk * zr, qikry = qixk * zr - qizk * xr, qikrz = qiyk * xr - qixk * yr;
  const U dkqirx = dkqiz * yr - dkqiy * zr, dkqiry = dkqix * zr - dkqiz * xr, dkqirz = dkqiy * xr - dkqix * yr;
  const U dqikx = diy * qkz - diz * qky + dky * qiz - dkz * qiy -
                  U(2) * (qixy * qkxz + qiyy * qkyz + qiyz * qkzz - qixz * qkxy - qiyz * qkyy - qizz * qkyz);
  const U dqiky = diz * qkx - dix * qkz + dkz * qix - dkx * qiz -
                  U(2) * (qixz * qkxx + qiyz * qkxy + qizz * qkxz - qixx * qkxz - qixy * qkyz - qixz * qkzz);
  const U dqikz = dix * qky - diy * qkx + dkx * qiy - dky * qix -
                  U(2) * (qixx * qkxy + qixy * qkyy + qixz * qkyz - qixy * qkxx - qiyy * qkxy - qiyz * qkxz);
  t[0] += (double)(-rr3 * dikx + t1 * dirx + t3 * (dqikx + dkqirx) - t4 * qirx - t6 * (qikrx + qikx));
  t[1] += (double)(-rr3 * diky + t1 * diry + t3 * (dqiky + dkqiry) - t4 * qiry - t6 * (qikry + qiky));
  t[2] += (double)(-rr3 * dikz + t1 * dirz + t3 * (dqikz + dkqirz) - t4 * qirz - t6 * (qikrz + qikz));
  e_acc += 0.5 * (double)e;
}

// Pairs outside the 1-2..1-5 lists, in the form's precision over the list:
// force and torque of site i, half of each pair energy (partials per block).
// The FP64 form reads the sorted positions and the FP64 multipole records
// and tests the cutoff in FP64; the mixed form reads one 64-B record per
// partner (wrapped position and multipoles, FP32) and images and tests in
// FP32, as its direct-field pass does.
// VIR: each block also writes the sum of its sites' pair virial halves and
// the frame-atom virial of their pair torques (6 values) to vpart.
template <bool MIXED, bool VIR>
__global__ void __launch_bounds__(kBlock, MIXED ? THP_EMPOLE_MINB : 4) k_empole_pairs(
    int n, int npad, Box box, double off2, EwM ew, const double4* __restrict__ pos, const double* __restrict__ mrec,
    const float* __restrict__ erec, const int* __restrict__ perm, const int* __restrict__ sp_off,
    const int* __restrict__ sp_ks, const int* __restrict__ sp_c, const int* __restrict__ nnb,
    const int* __restrict__ nb, int maxnb, const int* __restrict__ frs, unsigned long long* __restrict__ dem,
    double* __restrict__ epart, double* __restrict__ vpart) {
  using T = typename std::conditional<MIXED, float, double>::type;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double eacc = 0.0;
  double v6[6] = {0, 0, 0, 0, 0, 0};
  if (i < n) {
    T mi[10];
    double4 pi4 = make_double4(0.0, 0.0, 0.0, 0.0);
    float xi = 0.f, yi = 0.f, zi = 0.f;
    if constexpr (MIXED) {
      float v[16];
      ld_rec8(erec + (size_t)i * 16, *reinterpret_cast<float(*)[8]>(&v[0]));
      ld_rec8(erec + (size_t)i * 16 + 8, *reinterpret_cast<float(*)[8]>(&v[8]));
      xi = v[0];
      yi = v[1];
      zi = v[2];
#pragma unroll
      for (int q = 0; q < 10; ++q) mi[q] = v[5 + q];
    } else {
      pi4 = pos[i];
#pragma unroll
      for (int q = 0; q < 10; ++q) mi[q] = mrec[(size_t)i * 12 + 1 + q];
    }
    const float bx = (float)box.l[0], by = (float)box.l[1], bz = (float)box.l[2];
    const float hx = 0.5f * bx, hy = 0.5f * by, hz = 0.5f * bz;
    const float off2f = (float)off2;
    const int io = perm[i];
    const int s0 = sp_off[io], s1 = sp_off[io + 1];
    double g3[3] = {0.0, 0.0, 0.0}, t3[3] = {0.0, 0.0, 0.0};
    const int nn = min(nnb[i], maxnb);
    int knext = nn > 0 ? __ldg(nb + i) : 0;  // list entries fetched one pair ahead
#pragma unroll 1
    for (int s = 0; s < nn; ++s) {
      const int k = knext;
      if (s + 1 < nn) knext = __ldg(nb + (size_t)(s + 1) * npad + i);
      T xr, yr, zr, r2;
      T mk[10];
      if constexpr (MIXED) {
        float v[16];
        ld_rec8(erec + (size_t)k * 16, *reinterpret_cast<float(*)[8]>(&v[0]));
        ld_rec8(erec + (size_t)k * 16 + 8, *reinterpret_cast<float(*)[8]>(&v[8]));
        float x = v[0] - xi, y = v[1] - yi, z = v[2] - zi;
        x = fabsf(x) > hx ? x - copysignf(bx, x) : x;
        y = fabsf(y) > hy ? y - copysignf(by, y) : y;
        z = fabsf(z) > hz ? z - copysignf(bz, z) : z;
        r2 = x * x + y * y + z * z;
        if (r2 > off2f) continue;
        xr = x;
        yr = y;
        zr = z;
#pragma unroll
        for (int q = 0; q < 10; ++q) mk[q] = v[5 + q];
      } else {
        const double4 pk4 = pos[k];
        double xrd = pk4.x - pi4.x, yrd = pk4.y - pi4.y, zrd = pk4.z - pi4.z;
        image3(box, xrd, yrd, zrd);
        const double r2d = r2_exact(xrd, yrd, zrd);
        if (r2d > off2) continue;
        xr = xrd;
        yr = yrd;
        zr = zrd;
        r2 = r2d;
#pragma unroll
        for (int q = 0; q < 10; ++q) mk[q] = mrec[(size_t)k * 12 + 1 + q];
      }
      bool scaled = false;
      for (int q = s0; q < s1; ++q)
        if (__ldg(sp_ks + q) == k) {
          scaled = __ldg(sp_c + q) < 4;
          break;
        }
      if (scaled) continue;
      mpole_pair<T>(xr, yr, zr, r2, T(0), mi, mk, ew, eacc, g3, t3, VIR ? v6 : nullptr);
    }
    fix_add(dem + 3 * i + 0, g3[0]);
    fix_add(dem + 3 * i + 1, g3[1]);
    fix_add(dem + 3 * i + 2, g3[2]);
    const int iz = frs[3 * i], ix = frs[3 * i + 1], axt = frs[3 * i + 2];
    if (axt == 1 || axt == 2) {
      if (VIR) {
        double du[3], dv[3];
        torque_frame(pos, i, iz, ix, axt, t3, du, dv);
        frame_virial(pos, i, iz, ix, du, dv, v6);  // empole1.f:1466-1497
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          fix_add(dem + 3 * iz + j, du[j]);
          fix_add(dem + 3 * ix + j, dv[j]);
          fix_add(dem + 3 * i + j, -du[j] - dv[j]);
        }
      } else {
        torque_dist(pos, i, iz, ix, axt, t3, dem);
      }
    }
  }
  block_partial<kBlock>(eacc, epart);
  if (VIR) {
    block_reduce<6>(v6);
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < 6; ++q) vpart[(size_t)blockIdx.x * 6 + q] = v6[q];
  }
}

// Per site, in FP64: the 1-2..1-5 pairs within the cutoff (all are in the
// list when it is valid; the damped and bare terms cancel there to a small
// difference), the emrecip1 terms from fphirec and the self energy.
// VIR: each block also writes 12 virial sums to vpart: the reference's terms
// (scaled pair halves, the frame-atom virial of their torques and emrecip1's
// site terms, empole1.f:741-761) and the frame-atom virial of the reciprocal
// torques, which the reference leaves out.
template <bool VIR>
__global__ void __launch_bounds__(kBlock) k_empole_site(
    int n, Box box, double off2, EwM ew, MScale ms, PmeGeom g, const double4* __restrict__ pos,
    const double* __restrict__ rp, const int* __restrict__ perm, const int* __restrict__ sp_off,
    const int* __restrict__ sp_ks, const int* __restrict__ sp_c, const double* __restrict__ fphirec,
    const int* __restrict__ frs, unsigned long long* __restrict__ dem, double* __restrict__ epart,
    double* __restrict__ vpart) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double eacc = 0.0;
  double v12[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (i < n) {
    const double4 pi4 = pos[i];
    const int io = perm[i];
    const int s0 = sp_off[io], s1 = sp_off[io + 1];
    double g3[3] = {0.0, 0.0, 0.0}, t3[3] = {0.0, 0.0, 0.0};
    double mid[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) mid[q] = rp[(size_t)i * 10 + q];
#pragma unroll 1
    for (int q = s0; q < s1; ++q) {
      const int cls = __ldg(sp_c + q);
      if (cls >= 4) continue;
      const int k = __ldg(sp_ks + q);
      const double4 pk4 = pos[k];
      double xrd = pk4.x - pi4.x, yrd = pk4.y - pi4.y, zrd = pk4.z - pi4.z;
      image3(box, xrd, yrd, zrd);
      const double r2d = r2_exact(xrd, yrd, zrd);
      if (r2d > off2) continue;
      double mkd[10];
#pragma unroll
      for (int w = 0; w < 10; ++w) mkd[w] = rp[(size_t)k * 10 + w];
      mpole_pair<double>(xrd, yrd, zrd, r2d, 1.0 - ms.v[cls], mid, mkd, ew, eacc, g3, t3, VIR ? v12 : nullptr);
    }
    double gx = g3[0], gy = g3[1], gz = g3[2];
    const double tx = t3[0], ty = t3[1], tz = t3[2];
    // emrecip1 terms of site i from fphirec (FP64 multipoles)
    const double fe = kElectric;
    const double* r = rp + (size_t)i * 10;
    const double cm[10] = {r[0], r[1], r[2], r[3], r[4], r[7], r[9], 2.0 * r[5], 2.0 * r[6], 2.0 * r[8]};
    const double fm[10] = {cm[0], g.a[0] * cm[1], g.a[1] * cm[2], g.a[2] * cm[3], g.a[0] * g.a[0] * cm[4],
                           g.a[1] * g.a[1] * cm[5], g.a[2] * g.a[2] * cm[6], g.a[0] * g.a[1] * cm[7],
                           g.a[0] * g.a[2] * cm[8], g.a[1] * g.a[2] * cm[9]};
    double FR[21];
#pragma unroll
    for (int q = 0; q < 20; ++q) FR[q + 1] = fe * fphirec[(size_t)i * 20 + q];
    const int d1[10] = {2, 5, 8, 9, 11, 16, 18, 14, 15, 20};
    const int d2[10] = {3, 8, 6, 10, 14, 12, 19, 16, 20, 17};
    const int d3[10] = {4, 9, 10, 7, 15, 17, 13, 20, 18, 19};
    double erec = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      erec += fm[k] * FR[k + 1];
      f1 += fm[k] * FR[d1[k]];
      f2 += fm[k] * FR[d2[k]];
      f3 += fm[k] * FR[d3[k]];
    }
    gx += g.recip[0] * ((double)g.n1 * f1);
    gy += g.recip[1] * ((double)g.n2 * f2);
    gz += g.recip[2] * ((double)g.n3 * f3);
    const double cp[10] = {FR[1],
                           g.a[0] * FR[2],
                           g.a[1] * FR[3],
                           g.a[2] * FR[4],
                           g.a[0] * g.a[0] * FR[5],
                           g.a[1] * g.a[1] * FR[6],
                           g.a[2] * g.a[2] * FR[7],
                           g.a[0] * g.a[1] * FR[8],
                           g.a[0] * g.a[2] * FR[9],
                           g.a[1] * g.a[2] * FR[10]};
    double trq[3];
    trq[0] = cm[3] * cp[2] - cm[2] * cp[3] + 2.0 * (cm[6] - cm[5]) * cp[9] + cm[8] * cp[7] + cm[9] * cp[5] -
             cm[7] * cp[8] - cm[9] * cp[6];
    trq[1] = cm[1] * cp[3] - cm[3] * cp[1] + 2.0 * (cm[4] - cm[6]) * cp[8] + cm[7] * cp[9] + cm[8] * cp[6] -
             cm[8] * cp[4] - cm[9] * cp[7];
    trq[2] = cm[2] * cp[1] - cm[1] * cp[2] + 2.0 * (cm[5] - cm[4]) * cp[7] + cm[7] * cp[4] + cm[9] * cp[8] -
             cm[7] * cp[5] - cm[8] * cp[9];
    if (VIR) {
      // emrecip1's permanent-multipole site terms (empole1.f:741-761)
      v12[0] -= cm[1] * cp[1] + 2.0 * cm[4] * cp[4] + cm[7] * cp[7] + cm[8] * cp[8];
      v12[1] -= 0.5 * (cm[2] * cp[1] + cm[1] * cp[2]) + (cm[4] + cm[5]) * cp[7] + 0.5 * cm[7] * (cp[4] + cp[5]) +
                0.5 * (cm[8] * cp[9] + cm[9] * cp[8]);
      v12[2] -= 0.5 * (cm[3] * cp[1] + cm[1] * cp[3]) + (cm[4] + cm[6]) * cp[8] + 0.5 * cm[8] * (cp[4] + cp[6]) +
                0.5 * (cm[7] * cp[9] + cm[9] * cp[7]);
      v12[3] -= cm[2] * cp[2] + 2.0 * cm[5] * cp[5] + cm[7] * cp[7] + cm[9] * cp[9];
      v12[4] -= 0.5 * (cm[3] * cp[2] + cm[2] * cp[3]) + (cm[5] + cm[6]) * cp[9] + 0.5 * cm[9] * (cp[5] + cp[6]) +
                0.5 * (cm[7] * cp[8] + cm[8] * cp[7]);
      v12[5] -= cm[3] * cp[3] + 2.0 * cm[6] * cp[6] + cm[8] * cp[8] + cm[9] * cp[9];
    }
    // Ewald self energy (empole1.f:134-160)
    const double term = 2.0 * ew.a * ew.a;
    const double fterm = -fe * ew.a / kSqrtPi;
    const double dii = cm[1] * cm[1] + cm[2] * cm[2] + cm[3] * cm[3];
    const double qii = 2.0 * (r[5] * r[5] + r[6] * r[6] + r[8] * r[8]) + r[4] * r[4] + r[7] * r[7] + r[9] * r[9];
    const double eself = fterm * (cm[0] * cm[0] + term * (dii / 3.0 + 2.0 * term * qii / 5.0));
    eacc += 0.5 * erec + eself;
    fix_add(dem + 3 * i + 0, gx);
    fix_add(dem + 3 * i + 1, gy);
    fix_add(dem + 3 * i + 2, gz);
    const int iz = frs[3 * i], ix = frs[3 * i + 1], axt = frs[3 * i + 2];
    if ((axt == 1 || axt == 2) && VIR) {
      // the scaled pairs' torque (real space) and the reciprocal torque apart
      double tr[3] = {tx, ty, tz}, du[3], dv[3], dux[3], dvx[3];
      torque_frame(pos, i, iz, ix, axt, tr, du, dv);
      torque_frame(pos, i, iz, ix, axt, trq, dux, dvx);
      frame_virial(pos, i, iz, ix, du, dv, *reinterpret_cast<double(*)[6]>(&v12[0]));
      frame_virial(pos, i, iz, ix, dux, dvx, *reinterpret_cast<double(*)[6]>(&v12[6]));
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        fix_add(dem + 3 * iz + j, du[j] + dux[j]);
        fix_add(dem + 3 * ix + j, dv[j] + dvx[j]);
        fix_add(dem + 3 * i + j, -(du[j] + dux[j]) - (dv[j] + dvx[j]));
      }
    } else if (axt == 1 || axt == 2) {
      const double tt[3] = {tx + trq[0], ty + trq[1], tz + trq[2]};
      torque_dist(pos, i, iz, ix, axt, tt, dem);
    }
  }
  block_partial<kBlock>(eacc, epart);
  if (VIR) {
    block_reduce<12>(v12);
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < 12; ++q) vpart[(size_t)blockIdx.x * 12 + q] = v12[q];
  }
}

// buffers made on first use, sized by n (freed when a re-targeted context
// grows)
template <typename P>
int alloc_once(Ctx& c, P** p, size_t count, const char* what) {
  if (*p) return THP_OK;
  return cuda_status(cudaMalloc((void**)p, sizeof(P) * count), &c, what);
}

}  // namespace

// Permanent-multipole energy (into d_em) and gradient (into d_out, original
// order) for the sorted positions, multipoles and list of the context.
int launch_empole(Ctx& c, double* d_out) {
  int st;
  if (!c.have_axes) return THP_E_STATE;
  const size_t n = c.n;
  const int nb = (c.n + kBlock - 1) / kBlock;
  if ((st = alloc_once(c, &c.d_depfix, 3 * n, "alloc gradient"))) return st;
  if ((st = alloc_once(c, &c.d_empart, 2 * (size_t)nb + 1, "alloc mpole partials"))) return st;
  c.d_em = c.d_empart + 2 * nb;
  unsigned long long* dem = c.d_depfix;
  if ((st = cuda_status(cudaMemsetAsync(dem, 0, sizeof(unsigned long long) * 3 * n, c.stream), &c, "zero dem")))
    return st;
  if ((st = launch_frames_sorted(c))) return st;
  const bool vir = c.want_virial;
  double *kpart = nullptr, *rpart = nullptr, *spart = nullptr;
  if (vir && (st = virial_scratch(c, nb, nb, &kpart, &rpart, &spart))) return st;
  // the convolved multipole grid (and emrecip1's scalar sum over the
  // reciprocal lattice, empole1.f:560-598)
  if ((st = vir ? launch_mpole_grid_virial(c, kpart, 1.0) : launch_mpole_grid(c))) return st;
  if ((st = launch_fphi_mpole20(c))) return st;
  EwM ew;
  const double a = c.cfg.aewald;
  ew.a = a;
  const double aesq2 = 2.0 * a * a;
  double afac = 1.0 / (kSqrtPi * a);
  for (int j = 0; j < 5; ++j) {
    afac *= aesq2;
    ew.f[j] = afac;
  }
  MScale ms;
  for (int j = 0; j < 4; ++j) ms.v[j] = c.mscale[j];
  ms.v[4] = 1.0;
  const double off2 = c.cfg.ewaldcut * c.cfg.ewaldcut;
  const PmeGeom g = pme_geom(c);
#define THP_EMPOLE_ARGS                                                                                          \
  c.n, c.npad, c.box, off2, ew, c.d_pos, c.d_mrec, c.d_erec, c.d_perm, c.d_sp_off, c.d_sp_ks, c.d_sp_c, c.d_nnb, c.d_nb, \
      c.maxnb, c.d_frs, dem, c.d_empart, rpart
  if (c.mixed && vir)
    k_empole_pairs<true, true><<<nb, kBlock, 0, c.stream>>>(THP_EMPOLE_ARGS);
  else if (c.mixed)
    k_empole_pairs<true, false><<<nb, kBlock, 0, c.stream>>>(THP_EMPOLE_ARGS);
  else if (vir)
    k_empole_pairs<false, true><<<nb, kBlock, 0, c.stream>>>(THP_EMPOLE_ARGS);
  else
    k_empole_pairs<false, false><<<nb, kBlock, 0, c.stream>>>(THP_EMPOLE_ARGS);
#undef THP_EMPOLE_ARGS
  if ((st = cuda_status(cudaGetLastError(), &c, "empole pairs"))) return st;
#define THP_SITE_ARGS                                                                                              \
  c.n, c.box, off2, ew, ms, g, c.d_pos, c.d_rpole, c.d_perm, c.d_sp_off, c.d_sp_ks, c.d_sp_c, c.d_fphirec, c.d_frs, \
      dem, c.d_empart + nb, spart
  if (vir)
    k_empole_site<true><<<nb, kBlock, 0, c.stream>>>(THP_SITE_ARGS);
  else
    k_empole_site<false><<<nb, kBlock, 0, c.stream>>>(THP_SITE_ARGS);
#undef THP_SITE_ARGS
  if ((st = cuda_status(cudaGetLastError(), &c, "empole"))) return st;
  k_sum_partials<<<1, 256, 0, c.stream>>>(2 * nb, c.d_empart, c.d_em);
  if ((st = cuda_status(cudaGetLastError(), &c, "empole energy"))) return st;
  if (vir && (st = virial_total(c, kspace_virial_blocks(), nb, nb, kpart, rpart, spart, c.h_mvir))) return st;
  return launch_gradient_out(c, dem, d_out);
}

}  // namespace thp
