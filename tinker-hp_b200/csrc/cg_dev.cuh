// cg_dev.cuh -- block-level bodies of the CG kernels (inducepcg_pme2,
// newinduce_pme2.f:285-636), shared by the single-system kernels (one launch
// per system, block b = blockIdx.x) and the batched persistent kernels (one
// launch for many systems, block b = the work item's block of its system).
// A block covers kBlock consecutive (cell-sorted) atoms.  The per-system
// reductions write one partial per block and the last block to arrive sums
// them in block order, so the scalars do not depend on scheduling.
#pragma once

#include "context.h"
#include "pme_dev.cuh"
#include "realspace_dev.cuh"

// pairs loaded ahead per lane in the group rows (FP64 / FP32 forms)
#ifndef THP_GROW_U64
#define THP_GROW_U64 2
#endif
#ifndef THP_GROW_U32
#define THP_GROW_U32 4
#endif

namespace thp {
namespace cg {

constexpr int kBlock = 128;

// Deterministic grid reduction; returns true in the last block (all threads),
// with the totals valid in thread 0.
// blk / nblk: this block's slot among the nblk blocks (or persistent-kernel
// work items) that share the counter.
template <int NV>
__device__ bool grid_reduce_of(double (&v)[NV], double* __restrict__ partials, unsigned* counter, int blk,
                               int nblk, double (&tot)[NV]) {
  block_reduce<NV>(v);
  __shared__ bool amlast;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[(size_t)blk * NV + q] = v[q];
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    amlast = (t == (unsigned)nblk - 1);
  }
  __syncthreads();
  if (!amlast) return false;
  __threadfence();
  double s[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) s[q] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < NV; ++q) s[q] += __ldcg(partials + (size_t)b * NV + q);
  block_reduce<NV>(s);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) tot[q] = s[q];
    *counter = 0;
  }
  return true;
}

__device__ __forceinline__ void load6(const double* p, double (&v)[6]) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = q[0], b = q[1], c = q[2];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
}
__device__ __forceinline__ void store6(double* p, const double (&v)[6]) {
  double2* q = reinterpret_cast<double2*>(p);
  q[0] = make_double2(v[0], v[1]);
  q[1] = make_double2(v[2], v[3]);
  q[2] = make_double2(v[4], v[5]);
}

// FP32-stored vectors of the mixed form's overlapped CG, computed in FP64
__device__ __forceinline__ void load6(const float* p, double (&v)[6]) {
  const float2* q = reinterpret_cast<const float2*>(p);
  const float2 a = q[0], b = q[1], c = q[2];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
}
__device__ __forceinline__ void store6(float* p, const double (&v)[6]) {
  float2* q = reinterpret_cast<float2*>(p);
  q[0] = make_float2((float)v[0], (float)v[1]);
  q[1] = make_float2((float)v[2], (float)v[3]);
  q[2] = make_float2((float)v[4], (float)v[5]);
}

__device__ __forceinline__ double diag_of(double p) { return p == 0.0 ? kTinyPol : p; }
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double* __restrict__ partials, unsigned* counter,
                                            double (&tot)[NV]) {
  return grid_reduce_of<NV>(v, partials, counter, (int)blockIdx.x, (int)gridDim.x, tot);
}


// h = T_real x + x/alpha + dipfield(x) - term x  (newinduce_pme2.f:398-405, 469-475)
// init: also res = ef - h, zr = diag res, pp = zr, ggold = sum res.zr
// iter: gg = sum pp.h, alpha = ggold / gg
// A block covers kBlock consecutive atoms: each warp sums the rows of eight
// groups of four atoms (group_row) into shared memory, then every thread
// finishes its own atom.
// REC (mixed form): partners from the 32-byte records rec / mpz (the
// position and the dipoles of x, PartnerRec) instead of posf and xf.
// GPW: groups of four atoms per warp; a block of kBlock threads covers
// 16 GPW atoms (GPW = 8: one atom per thread in the combine step; smaller
// blocks for small systems, whose few blocks would otherwise each run a long
// chain of group rows).
template <bool MIXED, int GATHER, bool REC = false, int GPW = 8>
__device__ __forceinline__ void cg_matvec_block(int blk, int nblk, const PairRows& pr, const Box& box,
                                                const double4* __restrict__ pos, const float4* __restrict__ posf,
                                                const double* __restrict__ dipf, const PmeGeom& pg,
                                                const void* __restrict__ grid, const double* __restrict__ x,
                                                const float* __restrict__ xf, const float* __restrict__ rec,
                                                const float* __restrict__ mpz, const double* __restrict__ pol,
                                                const double* __restrict__ ef, double term, int init,
                                                double* __restrict__ h, double* __restrict__ res,
                                                double* __restrict__ zr, double* __restrict__ pp, CgScalars* cg,
                                                double* __restrict__ partials, float interior) {
  static_assert(kBlock == 128 && GPW >= 1 && GPW <= 8, "four warps, up to eight groups each");
  constexpr int AB = 16 * GPW;  // atoms per block
  __shared__ double srow[AB * 6];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blk * 4 * GPW + warp * GPW;  // first group of this warp
  for (int gg = 0; gg < GPW; ++gg) {
    const int g = gw + gg;
    if (4 * g >= pr.n) break;  // the same for every lane of the warp
    const int t = warp * 4 * GPW + gg * 4 + (lane >> 3), j = lane & 7;
    if (MIXED) {
      float a32[6];
      const Image32 im{(float)box.l[0], (float)box.l[1], (float)box.l[2]};
      if constexpr (REC)
        group_row<float, THP_GROW_U32, false>(pr, PartnerRec{rec, mpz}, im, g, lane, a32, interior);
      else
        group_row<float, THP_GROW_U32, false>(pr, Partner32{posf, xf}, im, g, lane, a32, interior);
      if (j < 6) srow[t * 6 + j] = (double)pick6(a32, j);
    } else {
      double a64[6];
      group_row<double, THP_GROW_U64, false>(pr, Partner64{pos, x}, Image64{box}, g, lane, a64, -1.0);
      if (j < 6) srow[t * 6 + j] = pick6(a64, j);
    }
  }
  __syncthreads();
  const int i = blk * AB + threadIdx.x;
  double red[2] = {0.0, 0.0};
  if (threadIdx.x < AB && i < pr.n) {
    double acc[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] = srow[threadIdx.x * 6 + q];
    double dip[6], xi[6];
    if constexpr (GATHER == 1)
      gather_dip<float>(pg, pos[i], reinterpret_cast<const cufftComplex*>(grid), dip);
    else if constexpr (GATHER == 2)
      gather_dip<double>(pg, pos[i], reinterpret_cast<const cufftDoubleComplex*>(grid), dip);
    else
      load6(dipf + (size_t)i * 6, dip);
    load6(x + (size_t)i * 6, xi);
    const double p = pol[i];
    const double ip = (p == 0.0) ? 1.0 / kTinyPol : 1.0 / p;
    double hv[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) hv[q] = ((acc[q] + xi[q] * ip) + dip[q]) - term * xi[q];
    store6(h + (size_t)i * 6, hv);
    if (init) {
      double e6[6], r6[6], z6[6];
      load6(ef + (size_t)i * 6, e6);
      const double dg = diag_of(p);
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        r6[q] = e6[q] - hv[q];
        z6[q] = dg * r6[q];
      }
      store6(res + (size_t)i * 6, r6);
      store6(zr + (size_t)i * 6, z6);
      store6(pp + (size_t)i * 6, z6);
      red[0] = r6[0] * z6[0] + r6[1] * z6[1] + r6[2] * z6[2];
      red[1] = r6[3] * z6[3] + r6[4] * z6[4] + r6[5] * z6[5];
    } else {
      red[0] = xi[0] * hv[0] + xi[1] * hv[1] + xi[2] * hv[2];
      red[1] = xi[3] * hv[3] + xi[4] * hv[4] + xi[5] * hv[5];
    }
  }
  __syncthreads();  // srow is reused by the block's next item
  double tot[2];
  if (grid_reduce_of<2>(red, partials, &cg->counter[0], blk, nblk, tot) && threadIdx.x == 0) {
    if (init) {
      cg->ggold[0] = tot[0];
      cg->ggold[1] = tot[1];
      cg->beta[0] = 0.0;
      cg->beta[1] = 0.0;
    } else {
      cg->gg[0] = tot[0];
      cg->gg[1] = tot[1];
      if (tot[0] == 0.0 || tot[1] == 0.0) {
        cg->stop = 1;  // newinduce_pme2.f:505 returns on gg == 0
      } else {
        cg->alpha[0] = cg->ggold[0] / tot[0];
        cg->alpha[1] = cg->ggold[1] / tot[1];
      }
    }
  }
}


// h = hreal + x/alpha + dipfield(x) - term x, then the reductions of
// k_cg_matvec (init: residual, zr, pp and ggold; iter: gg and alpha).
// GATHER 0 reads dipfield from dipf; 1 / 2 gather it here from the
// convolved FP32 / FP64 grid (the work of k_gather_dip, without the round
// trip of dipfield through memory).
template <int GATHER, typename XV, typename V>
__device__ __forceinline__ void cg_combine_block(int blk, int nblk, int n, const double* __restrict__ dipf,
                                                 const PmeGeom& g, const double4* __restrict__ pos,
                                                 const void* __restrict__ grid, const XV* __restrict__ x,
                                                 const double* __restrict__ pol, const double* __restrict__ ef,
                                                 double term, int init, V* __restrict__ h, V* __restrict__ res,
                                                 V* __restrict__ zr, V* __restrict__ pp, CgScalars* cg,
                                                 double* __restrict__ partials) {
  const int i = blk * kBlock + threadIdx.x;
  double red[2] = {0.0, 0.0};
  if (i < n) {
    double acc[6], dip[6], xi[6];
    if constexpr (GATHER == 1)
      gather_dip<float>(g, pos[i], reinterpret_cast<const cufftComplex*>(grid), dip);
    else if constexpr (GATHER == 2)
      gather_dip<double>(g, pos[i], reinterpret_cast<const cufftDoubleComplex*>(grid), dip);
    else
      load6(dipf + (size_t)i * 6, dip);
    load6(h + (size_t)i * 6, acc);
    load6(x + (size_t)i * 6, xi);
    const double p = pol[i];
    const double ip = (p == 0.0) ? 1.0 / kTinyPol : 1.0 / p;
    double hv[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) hv[q] = ((acc[q] + xi[q] * ip) + dip[q]) - term * xi[q];
    store6(h + (size_t)i * 6, hv);
    if (init) {
      double e6[6], r6[6], z6[6];
      load6(ef + (size_t)i * 6, e6);
      const double dg = diag_of(p);
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        r6[q] = e6[q] - hv[q];
        z6[q] = dg * r6[q];
      }
      store6(res + (size_t)i * 6, r6);
      store6(zr + (size_t)i * 6, z6);
      store6(pp + (size_t)i * 6, z6);
      red[0] = r6[0] * z6[0] + r6[1] * z6[1] + r6[2] * z6[2];
      red[1] = r6[3] * z6[3] + r6[4] * z6[4] + r6[5] * z6[5];
    } else {
      red[0] = xi[0] * hv[0] + xi[1] * hv[1] + xi[2] * hv[2];
      red[1] = xi[3] * hv[3] + xi[4] * hv[4] + xi[5] * hv[5];
    }
  }
  double tot[2];
  if (grid_reduce_of<2>(red, partials, &cg->counter[0], blk, nblk, tot) && threadIdx.x == 0) {
    if (init) {
      cg->ggold[0] = tot[0];
      cg->ggold[1] = tot[1];
      cg->beta[0] = 0.0;
      cg->beta[1] = 0.0;
    } else {
      cg->gg[0] = tot[0];
      cg->gg[1] = tot[1];
      if (tot[0] == 0.0 || tot[1] == 0.0) {
        cg->stop = 1;  // newinduce_pme2.f:505 returns on gg == 0
      } else {
        cg->alpha[0] = cg->ggold[0] / tot[0];
        cg->alpha[1] = cg->ggold[1] / tot[1];
      }
    }
  }
}

// The real-space rows T_real x of the atoms of block blk (16 GPW atoms:
// four warps of GPW groups of four), hreal[i][6] in FP64; lane j < 6 of an
// atom writes component j.  Partners as in cg_matvec_block.
template <bool MIXED, bool REC, int GPW>
__device__ __forceinline__ void row_block(int blk, const PairRows& pr, const Box& box,
                                          const double4* __restrict__ pos, const float4* __restrict__ posf,
                                          const double* __restrict__ x, const float* __restrict__ xf,
                                          const float* __restrict__ rec, const float* __restrict__ mpz,
                                          float interior, double* __restrict__ hreal) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blk * 4 * GPW + warp * GPW;  // first group of this warp
  for (int gg = 0; gg < GPW; ++gg) {
    const int g = gw + gg;
    if (4 * g >= pr.n) break;  // the same for every lane of the warp
    const int i = 4 * g + (lane >> 3), j = lane & 7;
    if (MIXED) {
      float a32[6];
      const Image32 im{(float)box.l[0], (float)box.l[1], (float)box.l[2]};
      if constexpr (REC)
        group_row<float, THP_GROW_U32, false>(pr, PartnerRec{rec, mpz}, im, g, lane, a32, interior);
      else
        group_row<float, THP_GROW_U32, false>(pr, Partner32{posf, xf}, im, g, lane, a32, interior);
      if (j < 6 && i < pr.n) hreal[(size_t)i * 6 + j] = (double)pick6(a32, j);
    } else {
      double a64[6];
      group_row<double, THP_GROW_U64, false>(pr, Partner64{pos, x}, Image64{box}, g, lane, a64, -1.0);
      if (j < 6 && i < pr.n) hreal[(size_t)i * 6 + j] = pick6(a64, j);
    }
  }
}

// newinduce_pme2.f:512-572.  The reference's per-iteration energy ene (a
// diagnostic printed at each step) is formed once, after the loop, from the
// final mu and residual (k_epol / kb_finish): the same value the last
// iteration would give, without reading E0 on every iteration.
template <typename V>
__device__ __forceinline__ void cg_update_block(int blk, int nblk, int n, const double* __restrict__ pol,
                                                const V* __restrict__ h, const V* __restrict__ pp,
                                                double* __restrict__ mu, V* __restrict__ res, V* __restrict__ zr,
                                                CgScalars* cg, double* __restrict__ partials, double poleps,
                                                int politer) {
  const int i = blk * kBlock + threadIdx.x;
  double red[2] = {0, 0};
  if (i < n) {
    const double ad = cg->alpha[0], ap = cg->alpha[1];
    double m6[6], r6[6], p6[6], h6[6], z6[6];
    load6(mu + (size_t)i * 6, m6);
    load6(res + (size_t)i * 6, r6);
    load6(pp + (size_t)i * 6, p6);
    load6(h + (size_t)i * 6, h6);
    const double dg = diag_of(pol[i]);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const double a = q < 3 ? ad : ap;
      m6[q] = m6[q] + a * p6[q];
      r6[q] = r6[q] - a * h6[q];
      z6[q] = dg * r6[q];
    }
    store6(mu + (size_t)i * 6, m6);
    store6(res + (size_t)i * 6, r6);
    store6(zr + (size_t)i * 6, z6);
#pragma unroll
    for (int q = 0; q < 6; ++q) red[q < 3 ? 0 : 1] += r6[q] * z6[q];
  }
  double tot[2];
  if (grid_reduce_of<2>(red, partials, &cg->counter[1], blk, nblk, tot) && threadIdx.x == 0) {
    const double nrm = (double)(3 * n);
    double resnrm = 0.0;
    bool bad = false;
    for (int k = 0; k < 2; ++k) {
      cg->ggnew[k] = tot[k];
      const double gn = sqrt(tot[k] / nrm);
      resnrm = fmax(resnrm, gn);
      bad |= !isfinite(tot[k]);
      cg->beta[k] = tot[k] / cg->ggold[k];
      cg->ggold[k] = tot[k];
    }
    cg->resnrm = resnrm;
    cg->niter += 1;
    if (bad) {
      cg->status = THP_E_NAN;
      cg->stop = 1;
    } else if (resnrm < poleps) {
      cg->converged = 1;
      cg->stop = 1;
    } else if (cg->niter >= politer) {
      cg->stop = 1;
    }
  }
}


}  // namespace cg
}  // namespace thp
