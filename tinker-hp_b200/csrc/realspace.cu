// realspace.cu -- direct permanent field and mutual-field coefficients.
//
// One pass over the full neighbor list per solve computes, for every pair
// with r^2 <= ewaldcut^2 (same unfused r^2 and image as newinduce_pme.f:1160):
//   * the direct permanent field of efld0_direct (newinduce_pme.f:948-1389),
//     d field with dscale and p field with pscale, Thole branch, dampewald
//     order 7 and damptholed order 7 (damping.f:17-55, 142-216);
//   * the mutual coefficients dmp3/dmp5 of tmatxb_pme (:1524-1560) with
//     uscale, stored in the grouped pair stream (realspace_dev.cuh) for the
//     matvec of every CG iteration.
// Scaled (special) pairs come from the connectivity lists, applied with the
// reference's assignment order (host side); the kernel looks the scale up in
// the owner's short special-pair list.
#include <algorithm>

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

struct EwaldConst {
  double a, afac1, afac2, afac3;  // 2a/sqrt(pi), 4a^3/sqrt(pi), 8a^5/sqrt(pi)
};

struct Rec64 {  // FP64 record: thole, q, d(3), Q(6)
  double th, q, dx, dy, dz, qxx, qxy, qxz, qyy, qyz, qzz;
  __device__ __forceinline__ void load(const double* m, int k) {
    const double2* p = reinterpret_cast<const double2*>(m + (size_t)k * 12);
    double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3), e = __ldg(p + 4), f = __ldg(p + 5);
    th = a.x; q = a.y; dx = b.x; dy = b.y; dz = c.x; qxx = c.y; qxy = d.x; qxz = d.y; qyy = e.x; qyz = e.y;
    qzz = f.x;
  }
};

// minimum resident blocks per SM asked of the compiler (0: its own choice)
#ifndef THP_EFLD0_MINB
#define THP_EFLD0_MINB 0
#endif

// The two field passes share the group frame of the matvec rows: a warp
// takes a group of four consecutive atoms, lane (a, j) walks the list
// entries j, j+8, j+16, ... of atom a.  The pairs within ewaldcut an atom's
// eight lanes accept at one step go to consecutive slots of its pair stream
// (ranked by lane), so each warp step writes into the group's current block:
// a handful of sectors, not one partial sector per atom.  An atom's field is
// the sum of its lanes' partial sums, combined in a fixed tree.
struct GroupLane {
  int a, j, i, is;  // atom of the group, lane of the atom, atom index, a valid index for short last groups
  bool live;
  __device__ __forceinline__ GroupLane(int g, int lane, int n) {
    a = lane >> 3;
    j = lane & 7;
    i = 4 * g + a;
    live = i < n;
    is = live ? i : 4 * g;
  }
};

// After one step: the accepted pair of this lane (take) goes to slot
// cnt + (accepted lanes of the atom before it); cnt advances by the atom's
// accepted count.  Returns the slot (or -1).
__device__ __forceinline__ int step_slot(bool take, int a, int j, int& cnt) {
  const unsigned ball = __ballot_sync(kFullMask, take);
  const unsigned mine = (ball >> (8 * a)) & 0xffu;
  const int slot = take ? cnt + __popc(mine & ((1u << j) - 1u)) : -1;
  cnt += __popc(mine);
  return slot;
}

// FP64 pass (the FP64 form): exact r^2 test and FP64 pair terms.
template <bool FIELD>
__global__ void __launch_bounds__(kFieldBlock, THP_EFLD0_MINB) k_efld0_coef(
    int n, int npad, Box box, double cut2, EwaldConst ew, const double4* __restrict__ pos,
    const double* __restrict__ mrec, const int* __restrict__ perm, const int* __restrict__ sp_off,
    const int* __restrict__ sp_ks, const double* __restrict__ sp_s, const int* __restrict__ nnb,
    const int* __restrict__ nb, int maxnb, int* __restrict__ npr, int* __restrict__ pk_out,
    double2* __restrict__ pcc, int cap8, double* __restrict__ ef, int* __restrict__ flags) {
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (4 * g >= n) return;
  const GroupLane L(g, threadIdx.x & 31, n);
  const int maxpr = 8 * cap8;
  const double4 pi = pos[L.is];
  const double thi = mrec[(size_t)L.is * 12];
  const int io = perm[L.is];
  const int s0 = sp_off[io], s1 = sp_off[io + 1];
  const int nn = L.live ? min(nnb[L.is], maxnb) : 0;
  int mb = max(nn, __shfl_xor_sync(kFullMask, nn, 8));
  mb = max(mb, __shfl_xor_sync(kFullMask, mb, 16));
  double e[6] = {0, 0, 0, 0, 0, 0};
  int cnt = 0;
  // list entries one step ahead of their gathers (the list streams from DRAM)
  int knext = L.j < nn ? __ldg(nb + (size_t)L.j * npad + L.is) : L.is;
#pragma unroll 1
  for (int s = L.j; s - L.j < mb; s += 8) {
    const int k = knext;
    knext = s + 8 < nn ? __ldg(nb + (size_t)(s + 8) * npad + L.is) : L.is;
    const double4 pk4 = pos[k];
    Rec64 r_k;
    r_k.load(mrec, k);
    double xr = pk4.x - pi.x, yr = pk4.y - pi.y, zr = pk4.z - pi.z;
    image3(box, xr, yr, zr);
    const double r2 = r2_exact(xr, yr, zr);
    const bool take = s < nn && r2 <= cut2;
    double c3 = 0.0, c5 = 0.0;
    if (take) {
      // scale factors of this pair (1 unless listed), partners in sorted numbering
      double ds = 1.0, ps = 1.0, us = 1.0;
      for (int q = s0; q < s1; ++q)
        if (__ldg(sp_ks + q) == k) {
          ds = sp_s[3 * q];
          ps = sp_s[3 * q + 1];
          us = sp_s[3 * q + 2];
          break;
        }
      const double x = xr, y = yr, z = zr;
      const double r = sqrt(r2);
      const double rr1 = 1.0 / r;
      const double rr2 = rr1 * rr1;
      const double rr3 = rr2 * rr1;
      const double rr5 = 3.0 * rr2 * rr3;
      const double rr7 = 5.0 * rr2 * rr5;
      // dampewald (order 7)
      const double ra = ew.a * r;
      const double bn0 = erfc(ra) * rr1;
      const double expterm = exp(-ra * ra);
      const double bn1 = (bn0 + ew.afac1 * expterm) * rr2;
      const double bn2 = (3.0 * bn1 + ew.afac2 * expterm) * rr2;
      const double bn3 = (5.0 * bn2 + ew.afac3 * expterm) * rr2;
      // dampthole / damptholed (AMOEBA branch)
      double l3 = 1, l5 = 1, l7 = 1;
      const double pdd = pi.w * pk4.w;
      double pg = fmin(thi, r_k.th);
      if (pg == 0.0) pg = fmax(thi, r_k.th);
      if (pdd != 0.0 && pg != 0.0) {
        const double t = r / pdd;
        const double damp = pg * (t * t * t);
        if (damp < 50.0) {
          const double ex = exp(-damp);
          l3 = 1.0 - ex;
          l5 = 1.0 - ex * (1.0 + damp);
          l7 = 1.0 - ex * (1.0 + damp + 0.6 * damp * damp);
        }
      }
      if (FIELD) {
        const double ck = r_k.q, dkx = r_k.dx, dky = r_k.dy, dkz = r_k.dz;
        const double dkr = dkx * x + dky * y + dkz * z;
        const double qkx = r_k.qxx * x + r_k.qxy * y + r_k.qxz * z;
        const double qky = r_k.qxy * x + r_k.qyy * y + r_k.qyz * z;
        const double qkz = r_k.qxz * x + r_k.qyz * y + r_k.qzz * z;
        const double qkr = qkx * x + qky * y + qkz * z;
        double sc = ds;
        double dmp3 = bn1 - (1.0 - sc * l3) * rr3;
        double dmp5 = bn2 - (1.0 - sc * l5) * rr5;
        double dmp7 = bn3 - (1.0 - sc * l7) * rr7;
        double rad = dmp3 * ck - dmp5 * dkr + dmp7 * qkr;
        e[0] += -x * rad - dmp3 * dkx + 2.0 * dmp5 * qkx;
        e[1] += -y * rad - dmp3 * dky + 2.0 * dmp5 * qky;
        e[2] += -z * rad - dmp3 * dkz + 2.0 * dmp5 * qkz;
        sc = ps;
        dmp3 = bn1 - (1.0 - sc * l3) * rr3;
        dmp5 = bn2 - (1.0 - sc * l5) * rr5;
        dmp7 = bn3 - (1.0 - sc * l7) * rr7;
        rad = dmp3 * ck - dmp5 * dkr + dmp7 * qkr;
        e[3] += -x * rad - dmp3 * dkx + 2.0 * dmp5 * qkx;
        e[4] += -y * rad - dmp3 * dky + 2.0 * dmp5 * qky;
        e[5] += -z * rad - dmp3 * dkz + 2.0 * dmp5 * qkz;
      }
      c3 = bn1 - (1.0 - us * l3) * rr3;
      c5 = bn2 - (1.0 - us * l5) * rr5;
    }
    const int slot = step_slot(take, L.a, L.j, cnt);
    if (slot >= 0 && slot < maxpr) {
      const size_t q = pair_slot(cap8, L.i, slot);
      pk_out[q] = k;
      pcc[q] = make_double2(c3, c5);
    }
  }
  if (FIELD) lane8_sum<6>(e);
  if (!L.live) return;
  if (L.j == 0) {
    npr[L.i] = min(cnt, maxpr);
    if (cnt > maxpr) atomicOr(flags, DEV_PAIR_OVERFLOW);
  }
  if (FIELD && L.j < 6) ef[(size_t)L.i * 6 + L.j] = pick6(e, L.j);
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
//   * each pair's FP32 field added into the lane's FP64 sums.
// The FP32 coefficients written for the CG rows follow the same formulas.
constexpr int kSpCache = 4;

template <bool FIELD>
__global__ void __launch_bounds__(kFieldBlock, THP_EFLD0_MINB) k_efld0_coef32(
    int n, int npad, float bx, float by, float bz, float cut2, EwaldConst ew, const float* __restrict__ erec,
    const int* __restrict__ perm, const int* __restrict__ sp_off, const int* __restrict__ sp_ks,
    const double* __restrict__ sp_s, const int* __restrict__ nnb, const int* __restrict__ nb, int maxnb,
    int* __restrict__ npr, int* __restrict__ pk_out, float2* __restrict__ pcc, int cap8,
    double* __restrict__ ef, int* __restrict__ flags) {
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (4 * g >= n) return;
  const GroupLane L(g, threadIdx.x & 31, n);
  const int maxpr = 8 * cap8;
  const float4 pi = *reinterpret_cast<const float4*>(erec + (size_t)L.is * 16);
  const float thi = erec[(size_t)L.is * 16 + 4];
  const int io = perm[L.is];
  const int s0 = sp_off[io], s1 = sp_off[io + 1];
  int spk[kSpCache];
#pragma unroll
  for (int v = 0; v < kSpCache; ++v) spk[v] = s0 + v < s1 ? __ldg(sp_ks + s0 + v) : -1;
  const bool sp_more = s1 - s0 > kSpCache;
  const float hx = 0.5f * bx, hy = 0.5f * by, hz = 0.5f * bz;
  const float ea = (float)ew.a, af1 = (float)ew.afac1, af2 = (float)ew.afac2, af3 = (float)ew.afac3;
  const int nn = L.live ? min(nnb[L.is], maxnb) : 0;
  int mb = max(nn, __shfl_xor_sync(kFullMask, nn, 8));
  mb = max(mb, __shfl_xor_sync(kFullMask, mb, 16));
  double e[6] = {0, 0, 0, 0, 0, 0};
  int cnt = 0;
  // list entries one step ahead: the list streams from DRAM, and its load
  // would otherwise sit in front of every step's record gathers
  int knext = L.j < nn ? __ldg(nb + (size_t)L.j * npad + L.is) : L.is;
#pragma unroll 1
  for (int s = L.j; s - L.j < mb; s += 8) {
    const int k = knext;
    knext = s + 8 < nn ? __ldg(nb + (size_t)(s + 8) * npad + L.is) : L.is;
    float v[16];
    ld_rec8(erec + (size_t)k * 16, *reinterpret_cast<float(*)[8]>(&v[0]));
    ld_rec8(erec + (size_t)k * 16 + 8, *reinterpret_cast<float(*)[8]>(&v[8]));
    float x = v[0] - pi.x, y = v[1] - pi.y, z = v[2] - pi.z;
    x = fabsf(x) > hx ? x - copysignf(bx, x) : x;
    y = fabsf(y) > hy ? y - copysignf(by, y) : y;
    z = fabsf(z) > hz ? z - copysignf(bz, z) : z;
    const float r2 = x * x + y * y + z * z;
    const bool take = s < nn && r2 <= cut2;
    float c3 = 0.f, c5 = 0.f;
    if (take) {
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
      const float ipd = pi.w * v[3];
      float pg = fminf(thi, v[4]);
      if (pg == 0.f) pg = fmaxf(thi, v[4]);
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
        const float ck = v[5], dkx = v[6], dky = v[7], dkz = v[8];
        const float qxx = v[9], qxy = v[10], qxz = v[11], qyy = v[12], qyz = v[13], qzz = v[14];
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
        e[0] += (double)fx;
        e[1] += (double)fy;
        e[2] += (double)fz;
        if (ps == ds) {
          e[3] += (double)fx;
          e[4] += (double)fy;
          e[5] += (double)fz;
        } else {
          dmp3 = bn1 - (1.f - ps * l3) * rr3;
          dmp5 = bn2 - (1.f - ps * l5) * rr5;
          dmp7 = bn3 - (1.f - ps * l7) * rr7;
          rad = dmp3 * ck - dmp5 * dkr + dmp7 * qkr;
          e[3] += (double)(-x * rad - dmp3 * dkx + 2.f * dmp5 * qkx);
          e[4] += (double)(-y * rad - dmp3 * dky + 2.f * dmp5 * qky);
          e[5] += (double)(-z * rad - dmp3 * dkz + 2.f * dmp5 * qkz);
        }
      }
      c3 = bn1 - (1.f - us * l3) * rr3;
      c5 = bn2 - (1.f - us * l5) * rr5;
    }
    const int slot = step_slot(take, L.a, L.j, cnt);
    if (slot >= 0 && slot < maxpr) {
      const size_t o = pair_slot(cap8, L.i, slot);
      pk_out[o] = k;
      pcc[o] = make_float2(c3, c5);
    }
  }
  if (FIELD) lane8_sum<6>(e);
  if (!L.live) return;
  if (L.j == 0) {
    npr[L.i] = min(cnt, maxpr);
    if (cnt > maxpr) atomicOr(flags, DEV_PAIR_OVERFLOW);
  }
  if (FIELD && L.j < 6) ef[(size_t)L.i * 6 + L.j] = pick6(e, L.j);
}

// tmatxb_pme for one call (the API's single matvec): one warp per group of
// four atoms; lane j < 6 of an atom writes component j, plus mu/alpha when
// dodiag.
#ifndef THP_GROW_U64
#define THP_GROW_U64 2
#endif
#ifndef THP_GROW_U32
#define THP_GROW_U32 4
#endif

__global__ void __launch_bounds__(kBlock) k_tmatxb64(PairRows pr, Box box, const double4* __restrict__ pos,
                                                     const double* __restrict__ mu, const double* __restrict__ pol,
                                                     int dodiag, double* __restrict__ out) {
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (4 * g >= pr.n) return;
  const int lane = threadIdx.x & 31;
  double acc[6];
  group_row<double, THP_GROW_U64, false>(pr, Partner64{pos, mu}, Image64{box}, g, lane, acc, -1.0);
  const int i = 4 * g + (lane >> 3), j = lane & 7;
  if (j >= 6 || i >= pr.n) return;
  double v = pick6(acc, j);
  if (dodiag) {
    const double p = pol[i];
    v += mu[(size_t)i * 6 + j] * ((p == 0.0) ? 1.0 / kTinyPol : 1.0 / p);
  }
  out[(size_t)i * 6 + j] = v;
}

__global__ void __launch_bounds__(kBlock) k_tmatxb32(PairRows pr, float bx, float by, float bz,
                                                     const float4* __restrict__ pos, const float* __restrict__ muf,
                                                     const double* __restrict__ mu, const double* __restrict__ pol,
                                                     int dodiag, float interior, double* __restrict__ out) {
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (4 * g >= pr.n) return;
  const int lane = threadIdx.x & 31;
  float acc[6];
  group_row<float, THP_GROW_U32, false>(pr, Partner32{pos, muf}, Image32{bx, by, bz}, g, lane, acc, interior);
  const int i = 4 * g + (lane >> 3), j = lane & 7;
  if (j >= 6 || i >= pr.n) return;
  double v = (double)pick6(acc, j);
  if (dodiag) {
    const double p = pol[i];
    v += mu[(size_t)i * 6 + j] * ((p == 0.0) ? 1.0 / kTinyPol : 1.0 / p);
  }
  out[(size_t)i * 6 + j] = v;
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

// Bound on the wrapped FP32 coordinates of a group whose pairs (all within
// ewaldcut) cannot cross a face of the box, with 0.05 A to spare for the
// rounding of the wrap; negative for boxes too small to have an interior.
float row_interior(const Ctx& c) {
  const double h = std::min(c.box.half[0], std::min(c.box.half[1], c.box.half[2]));
  return (float)(h - c.cfg.ewaldcut - 0.05);
}

PairRows pair_rows(const Ctx& c) {
  PairRows pr;
  pr.n = c.n;
  pr.cap8 = c.maxpr / 8;
  pr.npr = c.d_npr;
  pr.pk = c.d_pk;
  pr.pcc = c.d_pcc;
  return pr;
}

// blocks of kBlock threads for one warp per group of four atoms
int group_blocks(int n, int block) { return (((n + 3) / 4) * 32 + block - 1) / block; }

int launch_efld0_coef(Ctx& c, bool with_field) { return launch_efld0_coef_on(c, with_field, c.stream); }

int launch_efld0_coef_on(Ctx& c, bool with_field, cudaStream_t s) {
  const int nb = group_blocks(c.n, kFieldBlock);
  const double cut2 = c.cfg.ewaldcut * c.cfg.ewaldcut;
  EwaldConst ew = ewald_const(c.cfg.aewald);
  const int cap8 = c.maxpr / 8;
  if (c.mixed) {
    const float bx = (float)c.box.l[0], by = (float)c.box.l[1], bz = (float)c.box.l[2];
#define THP_EFLD0_ARGS32                                                                                        \
  c.n, c.npad, bx, by, bz, (float)cut2, ew, c.d_erec, c.d_perm, c.d_sp_off, c.d_sp_ks, c.d_sp_s, c.d_nnb, c.d_nb, \
      c.maxnb, c.d_npr, c.d_pk, (float2*)c.d_pcc, cap8, c.d_ef, c.d_flags
    if (with_field)
      k_efld0_coef32<true><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS32);
    else
      k_efld0_coef32<false><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS32);
#undef THP_EFLD0_ARGS32
  } else {
#define THP_EFLD0_ARGS                                                                                          \
  c.n, c.npad, c.box, cut2, ew, c.d_pos, c.d_mrec, c.d_perm, c.d_sp_off, c.d_sp_ks, c.d_sp_s, c.d_nnb, c.d_nb,   \
      c.maxnb, c.d_npr, c.d_pk, (double2*)c.d_pcc, cap8, c.d_ef, c.d_flags
    if (with_field)
      k_efld0_coef<true><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS);
    else
      k_efld0_coef<false><<<nb, kFieldBlock, 0, s>>>(THP_EFLD0_ARGS);
#undef THP_EFLD0_ARGS
  }
  c.have_coef = true;
  return cuda_status(cudaGetLastError(), &c, "efld0/coef");
}

int launch_tmatxb(Ctx& c, const double* d_in, double* d_out, bool dodiag) {
  const int nb = group_blocks(c.n, kBlock);
  PairRows pr = pair_rows(c);
  if (c.mixed) {
    int m = c.n * 6;
    k_to_float<<<(m + 255) / 256, 256, 0, c.stream>>>(m, d_in, c.d_vecf);
    k_tmatxb32<<<nb, kBlock, 0, c.stream>>>(pr, (float)c.box.l[0], (float)c.box.l[1], (float)c.box.l[2], c.d_posf,
                                            c.d_vecf, d_in, c.d_pol, dodiag ? 1 : 0, row_interior(c), d_out);
  } else {
    k_tmatxb64<<<nb, kBlock, 0, c.stream>>>(pr, c.box, c.d_pos, d_in, c.d_pol, dodiag ? 1 : 0, d_out);
  }
  return cuda_status(cudaGetLastError(), &c, "tmatxb");
}

}  // namespace thp
