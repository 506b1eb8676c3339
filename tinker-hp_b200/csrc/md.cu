// md.cu -- velocity-Verlet kernels (verlet.f:17-200) for dynamics driven by
// the polarization gradient.  Positions live in the context's original-order
// planar array d_xyz_orig [3][n]; velocities and masses are [n][3] / [n].
#include "kernels.h"

namespace thp {

namespace {

constexpr int kBlock = 256;
constexpr double kConvert = 418.4;  // kcal/mol -> g A^2/ps^2 (units.f:76)

// v += a dt/2 with a = -convert * dE/dx / m (verlet.f:57-61, 163-167)
__global__ void k_kick(int n, double half_dt, const double* __restrict__ mass, const double* __restrict__ grad,
                       double* __restrict__ vel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = -kConvert * half_dt / mass[i];
#pragma unroll
  for (int j = 0; j < 3; ++j) vel[3 * (size_t)i + j] += s * grad[3 * (size_t)i + j];
}

// x += v dt (verlet.f:65-67)
__global__ void k_drift(int n, double dt, const double* __restrict__ vel, double* __restrict__ xyz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int j = 0; j < 3; ++j) xyz[(size_t)j * n + i] += vel[3 * (size_t)i + j] * dt;
}

// per-block partial sums of m v^2 (fixed block order, summed by one block)
__global__ void k_ekin_partial(int n, const double* __restrict__ mass, const double* __restrict__ vel,
                               double* __restrict__ partial) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (i < n) {
    const double* u = vel + 3 * (size_t)i;
    v[0] = mass[i] * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  }
  block_reduce<1>(v);
  if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

__global__ void k_ekin_final(int nblk, const double* __restrict__ partial, double* __restrict__ out) {
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) v[0] += partial[b];
  block_reduce<1>(v);
  if (threadIdx.x == 0) *out = 0.5 * v[0] / kConvert;  // kcal/mol (mdstat eksum)
}

}  // namespace

int launch_kick(Ctx& c, double half_dt, const double* d_mass, const double* d_grad, double* d_vel) {
  k_kick<<<(c.n + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(c.n, half_dt, d_mass, d_grad, d_vel);
  return cuda_status(cudaGetLastError(), &c, "kick");
}

int launch_drift(Ctx& c, double dt, const double* d_vel) {
  k_drift<<<(c.n + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(c.n, dt, d_vel, c.d_xyz_orig);
  return cuda_status(cudaGetLastError(), &c, "drift");
}

// d_scratch holds at least ceil(n/256)+1 doubles; the kinetic energy lands in
// d_scratch[0] after the per-block partials (stored from index 1).
int launch_ekin(Ctx& c, const double* d_mass, const double* d_vel, double* d_scratch) {
  const int nblk = (c.n + kBlock - 1) / kBlock;
  k_ekin_partial<<<nblk, kBlock, 0, c.stream>>>(c.n, d_mass, d_vel, d_scratch + 1);
  k_ekin_final<<<1, kBlock, 0, c.stream>>>(nblk, d_scratch + 1, d_scratch);
  return cuda_status(cudaGetLastError(), &c, "kinetic energy");
}

}  // namespace thp
