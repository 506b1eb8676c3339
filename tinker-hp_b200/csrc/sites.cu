// sites.cu -- batched forms of the reference's per-site PME dipole routines
// grid_uind_site (pmestuff.f:280-405) and fphi_uind_site (pmestuff.f:746-1045)
// on a caller-owned FP64 grid qgrid2in_2d(2,n1,n2,n3), one rank (every
// stencil point is local).  Sites are atoms in original order; their
// B-splines come from the context's current positions, as bspline_fill_site
// does from x, y, z.
#include "kernels.h"
#include "pme_dev.cuh"

namespace thp {

namespace {

constexpr int kBlock = 128;

// one thread per listed site: 5x5x5 stencil of the fractional dipoles,
// Re = fuind, Im = fuinp, added with FP64 reductions
__global__ void __launch_bounds__(kBlock) k_grid_uind_sites(int nsites, const int* __restrict__ site, int n,
                                                            const double* __restrict__ xyz, PmeGeom g,
                                                            const double* __restrict__ fuind,
                                                            const double* __restrict__ fuinp,
                                                            cufftDoubleComplex* __restrict__ grid) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsites) return;
  const int i = site[q];
  double tx[kBs][2], ty[kBs][2], tz[kBs][2];
  const int gx = bspline_axis<2, double>(xyz[i], g.recip[0], g.n1, tx);
  const int gy = bspline_axis<2, double>(xyz[(size_t)n + i], g.recip[1], g.n2, ty);
  const int gz = bspline_axis<2, double>(xyz[2 * (size_t)n + i], g.recip[2], g.n3, tz);
  const double* fd = fuind + 3 * (size_t)q;
  const double* fp = fuinp + 3 * (size_t)q;
#pragma unroll 1
  for (int c = 0; c < kBs; ++c) {
    const size_t kk = (size_t)wrapk(gz + c, g.n3);
    const double v0 = tz[c][0], v1 = tz[c][1];
#pragma unroll 1
    for (int b = 0; b < kBs; ++b) {
      const size_t jj = (size_t)wrapk(gy + b, g.n2);
      const double u0 = ty[b][0], u1 = ty[b][1];
      const double term01 = fd[1] * u1 * v0 + fd[2] * u0 * v1, term11 = fd[0] * u0 * v0;
      const double term02 = fp[1] * u1 * v0 + fp[2] * u0 * v1, term12 = fp[0] * u0 * v0;
      const size_t row = (kk * g.n2 + jj) * g.n1;
#pragma unroll
      for (int a = 0; a < kBs; ++a) {
        cufftDoubleComplex* p = grid + row + wrapk(gx + a, g.n1);
        atomicAdd(&p->x, term01 * tx[a][0] + term11 * tx[a][1]);
        atomicAdd(&p->y, term02 * tx[a][0] + term12 * tx[a][1]);
      }
    }
  }
}

// one thread per listed site: fdip_phi1/2(2:10) of the Re / Im grid and the
// 20 derivatives fdip_sum_phi of Re + Im (slot 1 of fdip_phi1/2 is zero)
__global__ void __launch_bounds__(kBlock) k_fphi_uind_sites(int nsites, const int* __restrict__ site, int n,
                                                            const double* __restrict__ xyz, PmeGeom g,
                                                            const cufftDoubleComplex* __restrict__ grid,
                                                            double* __restrict__ phi1, double* __restrict__ phi2,
                                                            double* __restrict__ sum) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsites) return;
  const int i = site[q];
  double tx[kBs][4], ty[kBs][4], tz[kBs][4];
  const int gx = bspline_axis<4, double>(xyz[i], g.recip[0], g.n1, tx);
  const int gy = bspline_axis<4, double>(xyz[(size_t)n + i], g.recip[1], g.n2, ty);
  const int gz = bspline_axis<4, double>(xyz[2 * (size_t)n + i], g.recip[2], g.n3, tz);
  double T1[10] = {0}, T2[10] = {0}, S[20] = {0};
#pragma unroll
  for (int c = 0; c < kBs; ++c) {
    const size_t kk = (size_t)wrapk(gz + c, g.n3);
    const double v0 = tz[c][0], v1 = tz[c][1], v2 = tz[c][2], v3 = tz[c][3];
    double a1[6] = {0}, a2[6] = {0}, s[10] = {0};
#pragma unroll
    for (int b = 0; b < kBs; ++b) {
      const size_t jj = (size_t)wrapk(gy + b, g.n2);
      const double u0 = ty[b][0], u1 = ty[b][1], u2 = ty[b][2], u3 = ty[b][3];
      double ta[3] = {0, 0, 0}, tb[3] = {0, 0, 0}, t3 = 0;
      const size_t row = (kk * g.n2 + jj) * g.n1;
#pragma unroll
      for (int a = 0; a < kBs; ++a) {
        const cufftDoubleComplex v = grid[row + wrapk(gx + a, g.n1)];
        ta[0] += v.x * tx[a][0];
        ta[1] += v.x * tx[a][1];
        ta[2] += v.x * tx[a][2];
        tb[0] += v.y * tx[a][0];
        tb[1] += v.y * tx[a][1];
        tb[2] += v.y * tx[a][2];
        t3 += (v.x + v.y) * tx[a][3];
      }
      a1[0] += ta[0] * u0; a1[1] += ta[1] * u0; a1[2] += ta[0] * u1;
      a1[3] += ta[2] * u0; a1[4] += ta[1] * u1; a1[5] += ta[0] * u2;
      a2[0] += tb[0] * u0; a2[1] += tb[1] * u0; a2[2] += tb[0] * u1;
      a2[3] += tb[2] * u0; a2[4] += tb[1] * u1; a2[5] += tb[0] * u2;
      const double t0 = ta[0] + tb[0], t1 = ta[1] + tb[1], t2 = ta[2] + tb[2];
      s[0] += t0 * u0; s[1] += t1 * u0; s[2] += t0 * u1; s[3] += t2 * u0; s[4] += t1 * u1;
      s[5] += t0 * u2; s[6] += t3 * u0; s[7] += t2 * u1; s[8] += t1 * u2; s[9] += t0 * u3;
    }
    T1[1] += a1[1] * v0; T1[2] += a1[2] * v0; T1[3] += a1[0] * v1; T1[4] += a1[3] * v0; T1[5] += a1[5] * v0;
    T1[6] += a1[0] * v2; T1[7] += a1[4] * v0; T1[8] += a1[1] * v1; T1[9] += a1[2] * v1;
    T2[1] += a2[1] * v0; T2[2] += a2[2] * v0; T2[3] += a2[0] * v1; T2[4] += a2[3] * v0; T2[5] += a2[5] * v0;
    T2[6] += a2[0] * v2; T2[7] += a2[4] * v0; T2[8] += a2[1] * v1; T2[9] += a2[2] * v1;
    S[0] += s[0] * v0; S[1] += s[1] * v0; S[2] += s[2] * v0; S[3] += s[0] * v1; S[4] += s[3] * v0;
    S[5] += s[5] * v0; S[6] += s[0] * v2; S[7] += s[4] * v0; S[8] += s[1] * v1; S[9] += s[2] * v1;
    S[10] += s[6] * v0; S[11] += s[9] * v0; S[12] += s[0] * v3; S[13] += s[7] * v0; S[14] += s[3] * v1;
    S[15] += s[8] * v0; S[16] += s[5] * v1; S[17] += s[1] * v2; S[18] += s[2] * v2; S[19] += s[4] * v1;
  }
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    phi1[10 * (size_t)q + k] = T1[k];
    phi2[10 * (size_t)q + k] = T2[k];
  }
#pragma unroll
  for (int k = 0; k < 20; ++k) sum[20 * (size_t)q + k] = S[k];
}

}  // namespace

// The FP64 site grid (d_sgrid, ngrid complex) is allocated on first use and
// kept; sites are 0-based original atom numbers already on the device.
int launch_grid_uind_sites(Ctx& c, int nsites, const int* d_site, const double* d_fuind, const double* d_fuinp,
                           cufftDoubleComplex* d_sgrid) {
  if (nsites <= 0) return THP_OK;
  PmeGeom g = pme_geom(c);
  k_grid_uind_sites<<<(nsites + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(nsites, d_site, c.n, c.d_xyz_orig, g,
                                                                             d_fuind, d_fuinp, d_sgrid);
  return cuda_status(cudaGetLastError(), &c, "grid_uind_sites");
}

int launch_fphi_uind_sites(Ctx& c, int nsites, const int* d_site, const cufftDoubleComplex* d_sgrid, double* d_phi1,
                           double* d_phi2, double* d_sum) {
  if (nsites <= 0) return THP_OK;
  PmeGeom g = pme_geom(c);
  k_fphi_uind_sites<<<(nsites + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(nsites, d_site, c.n, c.d_xyz_orig, g,
                                                                             d_sgrid, d_phi1, d_phi2, d_sum);
  return cuda_status(cudaGetLastError(), &c, "fphi_uind_sites");
}

}  // namespace thp
