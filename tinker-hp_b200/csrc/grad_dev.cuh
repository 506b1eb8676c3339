// grad_dev.cuh -- device helpers shared by the gradient kernels: 64-bit
// fixed-point accumulation and the torque-to-force conversion of torque.f.
#pragma once

#include "common.cuh"

namespace thp {
namespace {

constexpr double kFix = 17179869184.0;  // 2^34

__device__ __forceinline__ void fix_add(unsigned long long* a, double v) {
  atomicAdd(a, (unsigned long long)(long long)llrint(v * kFix));
}

// torque.f:6-390, Z-then-X (axt 1) and Bisector (axt 2); site ib, z atom ia,
// x atom ic: the derivatives du (z atom) and dv (x atom) of the energy of
// the torque trq; the site itself takes -(du + dv).
__device__ __forceinline__ void torque_frame(const double4* __restrict__ pos, int ib, int ia, int ic, int axt,
                                             const double trq[3], double du[3], double dv[3]) {
  const double4 pb = pos[ib], pa = pos[ia], pc = pos[ic];
  double u[3] = {pa.x - pb.x, pa.y - pb.y, pa.z - pb.z};
  double v[3] = {pc.x - pb.x, pc.y - pb.y, pc.z - pb.z};
  const double usiz = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  const double vsiz = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double w[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
  const double wsiz = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    u[j] /= usiz;
    v[j] /= vsiz;
    w[j] /= wsiz;
  }
  double uv[3] = {v[1] * u[2] - v[2] * u[1], v[2] * u[0] - v[0] * u[2], v[0] * u[1] - v[1] * u[0]};
  double uw[3] = {w[1] * u[2] - w[2] * u[1], w[2] * u[0] - w[0] * u[2], w[0] * u[1] - w[1] * u[0]};
  double vw[3] = {w[1] * v[2] - w[2] * v[1], w[2] * v[0] - w[0] * v[2], w[0] * v[1] - w[1] * v[0]};
  const double uvsiz = sqrt(uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2]);
  const double uwsiz = sqrt(uw[0] * uw[0] + uw[1] * uw[1] + uw[2] * uw[2]);
  const double vwsiz = sqrt(vw[0] * vw[0] + vw[1] * vw[1] + vw[2] * vw[2]);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    uv[j] /= uvsiz;
    uw[j] /= uwsiz;
    vw[j] /= vwsiz;
  }
  const double uvcos = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
  const double uvsin = sqrt(1.0 - uvcos * uvcos);
  const double dphidu = -trq[0] * u[0] - trq[1] * u[1] - trq[2] * u[2];
  const double dphidv = -trq[0] * v[0] - trq[1] * v[1] - trq[2] * v[2];
  const double dphidw = -trq[0] * w[0] - trq[1] * w[1] - trq[2] * w[2];
  const double hw = axt == 2 ? 0.5 : 1.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    du[j] = uv[j] * dphidv / (usiz * uvsin) + hw * uw[j] * dphidw / usiz;
    dv[j] = -uv[j] * dphidu / (vsiz * uvsin);
    if (axt == 2) dv[j] += 0.5 * vw[j] * dphidw / vsiz;
  }
}

// adds d(energy)/d(coordinates) of the torque trq on site ib
__device__ void torque_dist(const double4* __restrict__ pos, int ib, int ia, int ic, int axt, const double trq[3],
                            unsigned long long* __restrict__ dep) {
  double du[3], dv[3];
  torque_frame(pos, ib, ia, ic, axt, trq, du, dv);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    fix_add(dep + 3 * ia + j, du[j]);
    fix_add(dep + 3 * ic + j, dv[j]);
    fix_add(dep + 3 * ib + j, -du[j] - dv[j]);
  }
}

// the virial of a torque's frame-atom derivatives (epolar1.f:2460-2486):
// du on the z atom ia, dv on the x atom ic of site ib; adds xx xy xz yy yz zz
__device__ __forceinline__ void frame_virial(const double4* __restrict__ pos, int ib, int ia, int ic,
                                             const double du[3], const double dv[3], double (&v)[6]) {
  const double4 pb = pos[ib], pa = pos[ia], pc = pos[ic];
  const double xiz = pa.x - pb.x, yiz = pa.y - pb.y, ziz = pa.z - pb.z;
  const double xix = pc.x - pb.x, yix = pc.y - pb.y, zix = pc.z - pb.z;
  v[0] += xix * dv[0] + xiz * du[0];
  v[1] += 0.5 * (yix * dv[0] + yiz * du[0] + xix * dv[1] + xiz * du[1]);
  v[2] += 0.5 * (zix * dv[0] + ziz * du[0] + xix * dv[2] + xiz * du[2]);
  v[3] += yix * dv[1] + yiz * du[1];
  v[4] += 0.5 * (zix * dv[1] + ziz * du[1] + yix * dv[2] + yiz * du[2]);
  v[5] += zix * dv[2] + ziz * du[2];
}

// sorted frame atoms: frs[s] = (iperm[zaxis], iperm[xaxis], axt) of perm[s]
__global__ void k_frames_sorted(int n, const int* __restrict__ perm, const int* __restrict__ iperm,
                                const int* __restrict__ frames, int* __restrict__ frs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = perm[s];
  frs[3 * s] = iperm[frames[3 * o]];
  frs[3 * s + 1] = iperm[frames[3 * o + 1]];
  frs[3 * s + 2] = frames[3 * o + 2];
}

__global__ void k_dep_out(int n, const int* __restrict__ perm, const unsigned long long* __restrict__ dep,
                          double* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = perm[s];
#pragma unroll
  for (int j = 0; j < 3; ++j) out[3 * (size_t)o + j] = (double)(long long)dep[3 * (size_t)s + j] / kFix;
}

// per-block energy partial (warp shuffles, then the warps in order)
template <int B>
__device__ __forceinline__ void block_partial(double eacc, double* __restrict__ epart) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) eacc += __shfl_down_sync(0xffffffffu, eacc, o);
  __shared__ double ws[B / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = eacc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < B / 32; ++w) t += ws[w];
    epart[blockIdx.x] = t;
  }
}

// one block: the partials in block order, strided per thread, then a tree
__global__ void __launch_bounds__(256) k_sum_partials(int m, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double s[256];
  double t = 0.0;
  for (int q = threadIdx.x; q < m; q += 256) t += part[q];
  s[threadIdx.x] = t;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

}  // namespace
}  // namespace thp
