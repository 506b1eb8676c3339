// realspace.cu -- direct permanent field and mutual-field coefficients.
//
// One pass over the full neighbor list per solve computes, for every pair
// with r^2 <= ewaldcut^2 (same unfused r^2 and image as newinduce_pme.f:1160):
//   * the direct permanent field of efld0_direct (newinduce_pme.f:948-1389),
//     d field with dscale and p field with pscale, Thole branch, dampewald
//     order 7 and damptholed order 7 (damping.f:17-55, 142-216);
//   * the mutual coefficients dmp3/dmp5 of tmatxb_pme (:1524-1560) with
//     uscale, stored slot-major for the matvec of every CG iteration.
// Scaled (special) pairs come from the connectivity lists, applied with the
// reference's assignment order (host side); the kernel looks the scale up in
// the owner's short special-pair list.
#include <type_traits>

#include "kernels.h"
#include "realspace_dev.cuh"

namespace thp {

namespace {

constexpr int kBlock = 128;
// threads per block of the field / coefficient pass
#ifndef THP_EFLD0_BLOCK
#define THP_EFLD0_BLOCK 128
#endif
constexpr int kFieldBlock = THP_EFLD0_BLOCK;

// list entries whose loads are issued together in the field / coefficient pass
#ifndef THP_EFLD0_G32
#define THP_EFLD0_G32 2
#endif
#ifndef THP_EFLD0_G64
#define THP_EFLD0_G64 1
#endif

struct EwaldConst {
  double a, afac1, afac2, afac3;  // 2a/sqrt(pi), 4a^3/sqrt(pi), 8a^5/sqrt(pi)
};

template <bool MIXED>
struct Rec;
template <>
struct Rec<false> {  // FP64 record: thole, q, d(3), Q(6)
  double th, q, dx, dy, dz, qxx, qxy, qxz, qyy, qyz, qzz;
  __device__ __forceinline__ void load(const double* m, const float*, int k) {
    const double2* p = reinterpret_cast<const double2*>(m + (size_t)k * 12);
    double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3), e = __ldg(p + 4), f = __ldg(p + 5);
    th = a.x; q = a.y; dx = b.x; dy = b.y; dz = c.x; qxx = c.y; qxy = d.x; qxz = d.y; qyy = e.x; qyz = e.y;
    qzz = f.x;
  }
};
template <>
struct Rec<true> {  // FP32 record of the mixed form
  float th, q, dx, dy, dz, qxx, qxy, qxz, qyy, qyz, qzz;
  __device__ __forceinline__ void load(const double*, const float* m, int k) {
    const float4* p = reinterpret_cast<const float4*>(m + (size_t)k * 12);
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    th = a.x; q = a.y; dx = a.z; dy = a.w; dz = b.x; qxx = b.y; qxy = b.z; qxz = b.w; qyy = c.x; qyz = c.y;
    qzz = c.z;
  }
};

// 1: the mixed form's pass runs k_efld0_coef32 (FP32 pair terms); 0: the
// FP64-geometry pass shared with the FP64 form
#ifndef THP_EFLD0_F32
#define THP_EFLD0_F32 1
#endif

// minimum resident blocks per SM asked of the compiler (0: its own choice)
#ifndef THP_EFLD0_MINB
#define THP_EFLD0_MINB 0
#endif

template <bool MIXED, bool FIELD>
__global__ void __launch_bounds__(kFieldBlock, THP_EFLD0_MINB) k_efld0_coef(
    int n, int npad, Box box, double cut2, EwaldConst ew, const double4* __restrict__ pos,
    const double* __restrict__ mrec, const float* __restrict__ mrecf, const int* __restrict__ perm,
    const int* __restrict__ sp_off, const int* __restrict__ sp_ks, const double* __restrict__ sp_s,
    const int* __restrict__ nnb, const int* __restrict__ nb, int maxnb, int* __restrict__ npr,
    int* __restrict__ pk_out, void* __restrict__ pc3v, void* __restrict__ pc5v, int maxpr, double* __restrict__ ef, int* __restrict__ flags) {
  using T = typename std::conditional<MIXED, float, double>::type;
  constexpr int G = MIXED ? THP_EFLD0_G32 : THP_EFLD0_G64;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T* pc3 = (T*)pc3v;
  T* pc5 = (T*)pc5v;
  const double4 pi = pos[i];
  const double thi = mrec[(size_t)i * 12];
  const int io = perm[i];
  const int s0 = sp_off[io], s1 = sp_off[io + 1];
  double e[6] = {0, 0, 0, 0, 0, 0};
  const int nn = min(nnb[i], maxnb);
  int cnt = 0;
  // list entries one group ahead of their gathers (the list streams from DRAM)
  int nxt[G];
#pragma unroll
  for (int g = 0; g < G; ++g) nxt[g] = g < nn ? __ldg(nb + (size_t)g * npad + i) : i;
#pragma unroll 1
  for (int sb = 0; sb < nn; sb += G) {
    // every load of the group is issued before the arithmetic of any pair
    int kk[G];
    double4 pk[G];
    Rec<MIXED> rk[G];
#pragma unroll
    for (int g = 0; g < G; ++g) kk[g] = nxt[g];
#pragma unroll
    for (int g = 0; g < G; ++g) nxt[g] = sb + G + g < nn ? __ldg(nb + (size_t)(sb + G + g) * npad + i) : i;
#pragma unroll
    for (int g = 0; g < G; ++g) pk[g] = pos[kk[g]];
#pragma unroll
    for (int g = 0; g < G; ++g) rk[g].load(mrec, mrecf, kk[g]);
#pragma unroll
    for (int g = 0; g < G; ++g) {
      if (sb + g >= nn) break;
      const int k = kk[g];
      const double4 pk4 = pk[g];
      double xr = pk4.x - pi.x, yr = pk4.y - pi.y, zr = pk4.z - pi.z;
      image3(box, xr, yr, zr);
      const double r2d = r2_exact(xr, yr, zr);
      if (r2d > cut2) continue;
      // scale factors of this pair (1 unless listed), partners in sorted numbering
      double ds = 1.0, ps = 1.0, us = 1.0;
      for (int q = s0; q < s1; ++q)
        if (__ldg(sp_ks + q) == k) {
          ds = sp_s[3 * q];
          ps = sp_s[3 * q + 1];
          us = sp_s[3 * q + 2];
          break;
        }
      const Rec<MIXED>& r_k = rk[g];
      const T x = (T)xr, y = (T)yr, z = (T)zr, r2 = (T)r2d;
      const T r = sqrt(r2);
      const T rr1 = T(1) / r;
      const T rr2 = rr1 * rr1;
      const T rr3 = rr2 * rr1;
      const T rr5 = T(3) * rr2 * rr3;
      const T rr7 = T(5) * rr2 * rr5;
      // dampewald (order 7)
      const T ra = (T)ew.a * r;
      const T bn0 = erfc(ra) * rr1;
      const T expterm = exp(-ra * ra);
      const T bn1 = (bn0 + (T)ew.afac1 * expterm) * rr2;
      const T bn2 = (T(3) * bn1 + (T)ew.afac2 * expterm) * rr2;
      const T bn3 = (T(5) * bn2 + (T)ew.afac3 * expterm) * rr2;
      // dampthole / damptholed (AMOEBA branch)
      T l3 = 1, l5 = 1, l7 = 1;
      const double pdd = pi.w * pk4.w;
      double pg = fmin(thi, (double)r_k.th);
      if (pg == 0.0) pg = fmax(thi, (double)r_k.th);
      if (pdd != 0.0 && pg != 0.0) {
        const T t = r / (T)pdd;
        const T damp = (T)pg * (t * t * t);
        if (damp < T(50)) {
          const T ex = exp(-damp);
          l3 = T(1) - ex;
          l5 = T(1) - ex * (T(1) + damp);
          l7 = T(1) - ex * (T(1) + damp + T(0.6) * damp * damp);
        }
      }
      if (FIELD) {
        const T ck = r_k.q, dkx = r_k.dx, dky = r_k.dy, dkz = r_k.dz;
        const T dkr = dkx * x + dky * y + dkz * z;
        const T qkx = r_k.qxx * x + r_k.qxy * y + r_k.qxz * z;
        const T qky = r_k.qxy * x + r_k.qyy * y + r_k.qyz * z;
        const T qkz = r_k.qxz * x + r_k.qyz * y + r_k.qzz * z;
        const T qkr = qkx * x + qky * y + qkz * z;
        T sc = (T)ds;
        T dmp3 = bn1 - (T(1) - sc * l3) * rr3;
        T dmp5 = bn2 - (T(1) - sc * l5) * rr5;
        T dmp7 = bn3 - (T(1) - sc * l7) * rr7;
        T rad = dmp3 * ck - dmp5 * dkr + dmp7 * qkr;
        e[0] += (double)(-x * rad - dmp3 * dkx + T(2) * dmp5 * qkx);
        e[1] += (double)(-y * rad - dmp3 * dky + T(2) * dmp5 * qky);
        e[2] += (double)(-z * rad - dmp3 * dkz + T(2) * dmp5 * qkz);
        sc = (T)ps;
        dmp3 = bn1 - (T(1) - sc * l3) * rr3;
        dmp5 = bn2 - (T(1) - sc * l5) * rr5;
        dmp7 = bn3 - (T(1) - sc * l7) * rr7;
        rad = dmp3 * ck - dmp5 * dkr + dmp7 * qkr;
        e[3] += (double)(-x * rad - dmp3 * dkx + T(2) * dmp5 * qkx);
        e[4] += (double)(-y * rad - dmp3 * dky + T(2) * dmp5 * qky);
        e[5] += (double)(-z * rad - dmp3 * dkz + T(2) * dmp5 * qkz);
      }
      const T su = (T)us;
      if (cnt < maxpr) {
        const size_t q = (size_t)cnt * npad + i;
        pk_out[q] = k;
        pc3[q] = bn1 - (T(1) - su * l3) * rr3;
        pc5[q] = bn2 - (T(1) - su * l5) * rr5;
      }
      ++cnt;
    }
  }
  npr[i] = min(cnt, maxpr);
  if (cnt > maxpr) atomicOr(flags, DEV_PAIR_OVERFLOW);
  if (FIELD) {
    double* o = ef + (size_t)i * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q] = e[q];
  }
}

// Mixed form of the same pass, restated for FP32 throughout the pair terms:
//   * partner data from one 64-byte record (two 256-bit loads): the wrapped
//     FP32 position and 1/pdamp, thole, charge, dipole and quadrupole;
//   * the displacement and the 7.0 A test in FP32 (only list pairs within
//     ulps of the cutoff can change side; their terms are ~1e-10 of the
//     field there);
//   * the Thole argument as r * (1/pdamp_i) * (1/pdamp_k);
//   * the special partners of the atom held in registers (the first
//     kSpCache of them; a longer list is searched past those);
//   * d and p fields computed once when the pair's two scales agree (every
//     pair but the few special pairs with dscale != pscale);
//   * FP32 field sums over runs of kFlush list entries, added into FP64.
// The FP32 coefficients written for the CG rows follow the same formulas.
constexpr int kSpCache = 4;
constexpr int kFlush = 8;

template <bool FIELD>
__global__ void __launch_bounds__(kFieldBlock, THP_EFLD0_MINB) k_efld0_coef32(
    int n, int npad, float bx, float by, float bz, float cut2, EwaldConst ew, const float* __restrict__ erec,
    const int* __restrict__ perm, const int* __restrict__ sp_off, const int* __restrict__ sp_ks,
    const double* __restrict__ sp_s, const int* __restrict__ nnb, const int* __restrict__ nb, int maxnb,
    int* __restrict__ npr, int* __restrict__ pk_out, float* __restrict__ pc3, float* __restrict__ pc5, int maxpr,
    double* __restrict__ ef, int* __restrict__ flags) {
  constexpr int G = THP_EFLD0_G32;
  static_assert(kFlush % G == 0, "flush runs are whole groups");
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 pi = *reinterpret_cast<const float4*>(erec + (size_t)i * 16);
  const float thi = erec[(size_t)i * 16 + 4];
  const int io = perm[i];
  const int s0 = sp_off[io], s1 = sp_off[io + 1];
  int spk[kSpCache];
#pragma unroll
  for (int v = 0; v < kSpCache; ++v) spk[v] = s0 + v < s1 ? __ldg(sp_ks + s0 + v) : -1;
  const bool sp_more = s1 - s0 > kSpCache;
  const float hx = 0.5f * bx, hy = 0.5f * by, hz = 0.5f * bz;
  const float ea = (float)ew.a, af1 = (float)ew.afac1, af2 = (float)ew.afac2, af3 = (float)ew.afac3;
  double e[6] = {0, 0, 0, 0, 0, 0};
  const int nn = min(nnb[i], maxnb);
  int cnt = 0;
  // list entries one group ahead: the list streams from DRAM, and its load
  // would otherwise sit in front of every group's record gathers
  int nxt[G];
#pragma unroll
  for (int g = 0; g < G; ++g) nxt[g] = g < nn ? __ldg(nb + (size_t)g * npad + i) : i;
#pragma unroll 1
  for (int sf = 0; sf < nn; sf += kFlush) {
    float f[6] = {0, 0, 0, 0, 0, 0};
    const int se = min(sf + kFlush, nn);
#pragma unroll 1
    for (int sb = sf; sb < se; sb += G) {
      int kk[G];
      float v[G][16];
#pragma unroll
      for (int g = 0; g < G; ++g) kk[g] = nxt[g];
#pragma unroll
      for (int g = 0; g < G; ++g) nxt[g] = sb + G + g < nn ? __ldg(nb + (size_t)(sb + G + g) * npad + i) : i;
#pragma unroll
      for (int g = 0; g < G; ++g) {
        ld_rec8(erec + (size_t)kk[g] * 16, *reinterpret_cast<float(*)[8]>(&v[g][0]));
        ld_rec8(erec + (size_t)kk[g] * 16 + 8, *reinterpret_cast<float(*)[8]>(&v[g][8]));
      }
#pragma unroll
      for (int g = 0; g < G; ++g) {
        if (sb + g >= se) break;
        const int k = kk[g];
        float x = v[g][0] - pi.x, y = v[g][1] - pi.y, z = v[g][2] - pi.z;
        x = fabsf(x) > hx ? x - copysignf(bx, x) : x;
        y = fabsf(y) > hy ? y - copysignf(by, y) : y;
        z = fabsf(z) > hz ? z - copysignf(bz, z) : z;
        const float r2 = x * x + y * y + z * z;
        if (r2 > cut2) continue;
        int q = -1;
#pragma unroll
        for (int w = 0; w < kSpCache; ++w)
          if (spk[w] == k) q = s0 + w;
        if (q < 0 && sp_more)
          for (int w = s0 + kSpCache; w < s1; ++w)
            if (__ldg(sp_ks + w) == k) {
              q = w;
              break;
            }
        float ds = 1.f, ps = 1.f, us = 1.f;
        if (q >= 0) {
          ds = (float)sp_s[3 * q];
          ps = (float)sp_s[3 * q + 1];
          us = (float)sp_s[3 * q + 2];
        }
        const float r = sqrtf(r2);
        const float rr1 = 1.f / r;
        const float rr2 = rr1 * rr1;
        const float rr3 = rr2 * rr1;
        const float rr5 = 3.f * rr2 * rr3;
        const float rr7 = 5.f * rr2 * rr5;
        // dampewald (order 7)
        const float ra = ea * r;
        const float bn0 = erfcf(ra) * rr1;
        const float expterm = expf(-ra * ra);
        const float bn1 = (bn0 + af1 * expterm) * rr2;
        const float bn2 = (3.f * bn1 + af2 * expterm) * rr2;
        const float bn3 = (5.f * bn2 + af3 * expterm) * rr2;
        // dampthole / damptholed (AMOEBA branch)
        float l3 = 1.f, l5 = 1.f, l7 = 1.f;
        const float ipd = pi.w * v[g][3];
        float pg = fminf(thi, v[g][4]);
        if (pg == 0.f) pg = fmaxf(thi, v[g][4]);
        if (ipd != 0.f && pg != 0.f) {
          const float t = r * ipd;
          const float damp = pg * (t * t * t);
          if (damp < 50.f) {
            const float ex = expf(-damp);
            l3 = 1.f - ex;
            l5 = 1.f - ex * (1.f + damp);
            l7 = 1.f - ex * (1.f + damp + 0.6f * damp * damp);
          }
        }
        if (FIELD) {
          const float ck = v[g][5], dkx = v[g][6], dky = v[g][7], dkz = v[g][8];
          const float qxx = v[g][9], qxy = v[g][10], qxz = v[g][11], qyy = v[g][12], qyz = v[g][13],
                      qzz = v[g][14];
          const float dkr = dkx * x + dky * y + dkz * z;
          const float qkx = qxx * x + qxy * y + qxz * z;
          const float qky = qxy * x + qyy * y + qyz * z;
          const float qkz = qxz * x + qyz * y + qzz * z;
          const float qkr = qkx * x + qky * y + qkz * z;
          float dmp3 = bn1 - (1.f - ds * l3) * rr3;
          float dmp5 = bn2 - (1.f - ds * l5) * rr5;
          float dmp7 = bn3 - (1.f - ds * l7) * rr7;
          float rad = dmp3 * ck - dmp5 * dkr + dmp7 * qkr;
          const float fx = -x * rad - dmp3 * dkx + 2.f * dmp5 * qkx;
          const float fy = -y * rad - dmp3 * dky + 2.f * dmp5 * qky;
          const float fz = -z * rad - dmp3 * dkz + 2.f * dmp5 * qkz;
          f[0] += fx;
          f[1] += fy;
          f[2] += fz;
          if (ps == ds) {
            f[3] += fx;
            f[4] += fy;
            f[5] += fz;
          } else {
            dmp3 = bn1 - (1.f - ps * l3) * rr3;
            dmp5 = bn2 - (1.f - ps * l5) * rr5;
            dmp7 = bn3 - (1.f - ps * l7) * rr7;
            rad = dmp3 * ck - dmp5 * dkr + dmp7 * qkr;
            f[3] += -x * rad - dmp3 * dkx + 2.f * dmp5 * qkx;
            f[4] += -y * rad - dmp3 * dky + 2.f * dmp5 * qky;
            f[5] += -z * rad - dmp3 * dkz + 2.f * dmp5 * qkz;
          }
        }
        if (cnt < maxpr) {
          const size_t o = (size_t)cnt * npad + i;
          pk_out[o] = k;
          pc3[o] = bn1 - (1.f - us * l3) * rr3;
          pc5[o] = bn2 - (1.f - us * l5) * rr5;
        }
        ++cnt;
      }
    }
    if (FIELD)
#pragma unroll
      for (int u = 0; u < 6; ++u) e[u] += (double)f[u];
  }
  npr[i] = min(cnt, maxpr);
  if (cnt > maxpr) atomicOr(flags, DEV_PAIR_OVERFLOW);
  if (FIELD) {
    double* o = ef + (size_t)i * 6;
#pragma unroll
    for (int u = 0; u < 6; ++u) o[u] = e[u];
  }
}

__global__ void __launch_bounds__(kBlock) k_tmatxb64(PairRows pr, Box box, const double4* __restrict__ pos,
                                                     const double* __restrict__ mu, const double* __restrict__ pol,
                                                     int dodiag, double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pr.n) return;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  tmatxb_row64(pr, box, i, pos, mu, acc);
  double* o = out + (size_t)i * 6;
  if (dodiag) {
    double p = pol[i];
    double ip = (p == 0.0) ? 1.0 / kTinyPol : 1.0 / p;
    const double* m = mu + (size_t)i * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] += m[q] * ip;
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) o[q] = acc[q];
}

__global__ void __launch_bounds__(kBlock) k_tmatxb32(PairRows pr, float bx, float by, float bz,
                                                     const float4* __restrict__ pos, const float* __restrict__ muf,
                                                     const double* __restrict__ mu, const double* __restrict__ pol,
                                                     int dodiag, double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pr.n) return;
  float acc[6] = {0, 0, 0, 0, 0, 0};
  tmatxb_row32(pr, bx, by, bz, i, pos, muf, acc);
  double* o = out + (size_t)i * 6;
  double a[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) a[q] = (double)acc[q];
  if (dodiag) {
    double p = pol[i];
    double ip = (p == 0.0) ? 1.0 / kTinyPol : 1.0 / p;
    const double* m = mu + (size_t)i * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) a[q] += m[q] * ip;
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) o[q] = a[q];
}

__global__ void k_to_float(int m, const double* __restrict__ in, float* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[i] = (float)in[i];
}

EwaldConst ewald_const(double a) {
  // dampewald recursion (damping.f:41-50): afac_i = (2 a^2)^i / (sqrt(pi) a)
  EwaldConst e;
  e.a = a;
  double aesq2 = 2.0 * a * a;
  double afac = 1.0 / (kSqrtPi * a);
  afac = aesq2 * afac;
  e.afac1 = afac;
  afac = aesq2 * afac;
  e.afac2 = afac;
  afac = aesq2 * afac;
  e.afac3 = afac;
  return e;
}

}  // namespace

PairRows pair_rows(const Ctx& c) {
  PairRows pr;
  pr.n = c.n;
  pr.npad = c.npad;
  pr.npr = c.d_npr;
  pr.pk = c.d_pk;
  pr.pc3 = c.d_pc3;
  pr.pc5 = c.d_pc5;
  return pr;
}

int launch_efld0_coef(Ctx& c, bool with_field) { return launch_efld0_coef_on(c, with_field, c.stream); }

int launch_efld0_coef_on(Ctx& c, bool with_field, cudaStream_t s) {
  const int nb = (c.n + kFieldBlock - 1) / kFieldBlock;
  const double cut2 = c.cfg.ewaldcut * c.cfg.ewaldcut;
  EwaldConst ew = ewald_const(c.cfg.aewald);
#define THP_EFLD0_ARGS                                                                                          \
  c.n, c.npad, c.box, cut2, ew, c.d_pos, c.d_mrec, c.d_mrecf, c.d_perm, c.d_sp_off, c.d_sp_ks, c.d_sp_s, c.d_nnb, \
      c.d_nb, c.maxnb, c.d_npr, c.d_pk, c.d_pc3, c.d_pc5, c.maxpr, c.d_ef, c.d_flags
  if (c.mixed) {
#if THP_EFLD0_F32
    const float bx = (float)c.box.l[0], by = (float)c.box.l[1], bz = (float)c.box.l[2];
#define THP_EFLD0_ARGS32                                                                                        \
  c.n, c.npad, bx, by, bz, (float)cut2, ew, c.d_erec, c.d_perm, c.d_sp_off, c.d_sp_ks, c.d_sp_s, c.d_nnb, c.d_nb, \
      c.maxnb, c.d_npr, c.d_pk, (float*)c.d_pc3, (float*)c.d_pc5, c.maxpr, c.d_ef, c.d_flags
    if (with_field)
      k_efld0_coef32<true><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS32);
    else
      k_efld0_coef32<false><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS32);
#undef THP_EFLD0_ARGS32
#else
    if (with_field)
      k_efld0_coef<true, true><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS);
    else
      k_efld0_coef<true, false><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS);
#endif
  } else {
    if (with_field)
      k_efld0_coef<false, true><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS);
    else
      k_efld0_coef<false, false><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS);
  }
#undef THP_EFLD0_ARGS
  c.have_coef = true;
  return cuda_status(cudaGetLastError(), &c, "efld0/coef");
}

int launch_tmatxb(Ctx& c, const double* d_in, double* d_out, bool dodiag) {
  const int nb = (c.n + kBlock - 1) / kBlock;
  PairRows pr = pair_rows(c);
  if (c.mixed) {
    int m = c.n * 6;
    k_to_float<<<(m + 255) / 256, 256, 0, c.stream>>>(m, d_in, c.d_vecf);
    k_tmatxb32<<<nb, kBlock, 0, c.stream>>>(pr, (float)c.box.l[0], (float)c.box.l[1], (float)c.box.l[2], c.d_posf,
                                            c.d_vecf, d_in, c.d_pol, dodiag ? 1 : 0, d_out);
  } else {
    k_tmatxb64<<<nb, kBlock, 0, c.stream>>>(pr, c.box, c.d_pos, d_in, c.d_pol, dodiag ? 1 : 0, d_out);
  }
  return cuda_status(cudaGetLastError(), &c, "tmatxb");
}

}  // namespace thp
