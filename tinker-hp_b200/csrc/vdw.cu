// vdw.cu -- buffered 14-7 van der Waals energy and gradient on the device
// (ehal1c).
//
// Restates ehal1c (ehal1.f:69-482, standard branch: no soft core, groups or
// short/long split) for the pairs of vlistcell (nblist.f:1148-1305):
//   * reduced sites: each atom's vdW site moves towards its reduction parent,
//     x_red = kred (x - x_parent) + x_parent (ehal1.f:193-205);
//   * e = eps tau^7 Rmin^7 ((1+g) Rmin^7 / (r^7 + g Rmin^7) - 2) with
//     tau = (1+d) / (r + d Rmin), the 1-2..1-5 vscale factors and the 1-4
//     Rmin / eps, the 5th-degree taper between vdwtaper and vdwcut
//     (switch.f:80-117);
//   * the force on a reduced site split between the atom (kred) and its
//     parent (1 - kred).
// The pairs come from a vdW list in the context's sorted numbering (the
// reference's vlistcell): every site within vdwcut + lbuffer of the reduced
// site, found by scanning the cells of the cell sort within reach (vdwcut,
// lbuffer for the atoms' drift since the sort, and the largest allowed
// reduction shift on both sides).  The list is rebuilt after a re-sort or
// once an atom has moved lbuffer/2 since the positions it was built from, as
// the reference's list update does.  One thread per site evaluates each pair
// from its own end (no atomics for the pair terms): its list is dense in
// interacting pairs, so the lanes of a warp stay together through the pair
// arithmetic.  The site's summed force goes to the atom and its parent in
// 64-bit fixed point, the energy through per-block partials summed in order.
#include <algorithm>
#include <type_traits>

#include "grad_dev.cuh"
#include "kernels.h"

namespace thp {

namespace {

constexpr int kBlock = 128;
// largest reduction shift |x_red - x| the cell reach allows (A); a larger one
// is reported instead of silently missing pairs
constexpr double kShiftMax = 0.3;
// per-site capacity of the vdW list without a max_neighbors setting (a 9.5 A
// sphere of liquid water holds about 370 sites)
constexpr int kDefaultMaxVnb = 640;

struct VdwConst {
  double off2, cut2, off, cut;
  double c0, c1, c2, c3, c4, c5;  // taper coefficients (switch.f:80-117)
  double ghal, dhal;
  double vscale[5];               // v2..v5scale, then 1
  int nclass;
};

// sorted reduced sites: (x, y, z, kred) and (class, parent in sorted order)
__global__ void k_vdw_sites(int n, const int* __restrict__ perm, const int* __restrict__ iperm,
                            const double4* __restrict__ pos, const int* __restrict__ cls,
                            const int* __restrict__ ired, const double* __restrict__ kred, Box box,
                            double shift2max, double4* __restrict__ vred, float4* __restrict__ vredf,
                            int2* __restrict__ vinfo, int* __restrict__ flags) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = perm[s];
  const int ps = iperm[ired[o]];
  const double4 p = pos[s], q = pos[ps];
  const double r = kred[o];
  const double dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
  const double x = r * dx + q.x, y = r * dy + q.y, z = r * dz + q.z;
  const double sx = x - p.x, sy = y - p.y, sz = z - p.z;
  if (sx * sx + sy * sy + sz * sz > shift2max) atomicOr(flags, DEV_VDW_REACH);
  vred[s] = make_double4(x, y, z, r);
  double wx = x, wy = y, wz = z;  // wrapped into the box for the FP32 screen of the list build
  image3(box, wx, wy, wz);
  vredf[s] = make_float4((float)wx, (float)wy, (float)wz, 0.f);
  vinfo[s] = make_int2(cls[o], ps);
}

// cells of one axis within +-w of cell c (all of them when 2w+1 >= nc)
__device__ __forceinline__ int axis_count(int nc, int w) { return 2 * w + 1 >= nc ? nc : 2 * w + 1; }
__device__ __forceinline__ int axis_cell(int c, int nc, int w, int q) {
  return 2 * w + 1 >= nc ? q : ((c + q - w) % nc + nc) % nc;
}

// vlistcell (nblist.f:1148-1305) over the cell sort: every other site whose
// reduced minimum-image distance is within vbuf (both directions)
__global__ void __launch_bounds__(kBlock) k_vdw_list(int n, int npad, Box box, double vbuf2, int prefilter, float lo,
                                                     float hi, int wx, int wy, int wz, const double4* __restrict__ vred,
                                                     const float4* __restrict__ vredf, const int2* __restrict__ vinfo,
                                                     const double* __restrict__ vtab, int nclass,
                                                     const int* __restrict__ scell,
                                                     const int* __restrict__ cell_start,
                                                     const int* __restrict__ cell_count, int ncx, int ncy, int ncz,
                                                     int maxvnb, int* __restrict__ vnnb, int* __restrict__ vnb,
                                                     int* __restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // sites of a class without a vdW radius take no part (kvdw.f:592-598:
  // they are not vdW sites; vlistcell skips them as partners)
  if (__ldg(vtab + (size_t)vinfo[i].x * (nclass + 1)) == 0.0) {
    vnnb[i] = 0;
    return;
  }
  const double4 ri = vred[i];
  const float4 fi = vredf[i];
  const float bx = (float)box.l[0], by = (float)box.l[1], bz = (float)box.l[2];
  const float hx = 0.5f * bx, hy = 0.5f * by, hz = 0.5f * bz;
  const int c = scell[i];
  const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
  // x ranges of the window: [a0, a1] and the wrapped [b0, b1]
  int a0, a1, b0 = 1, b1 = 0;
  if (2 * wx + 1 >= ncx) {
    a0 = 0;
    a1 = ncx - 1;
  } else {
    const int lo = cx - wx, hi = cx + wx;
    if (lo < 0) {
      a0 = 0;
      a1 = hi;
      b0 = lo + ncx;
      b1 = ncx - 1;
    } else if (hi >= ncx) {
      a0 = lo;
      a1 = ncx - 1;
      b0 = 0;
      b1 = hi - ncx;
    } else {
      a0 = lo;
      a1 = hi;
    }
  }
  const int my = axis_count(ncy, wy), mz = axis_count(ncz, wz);
  int cnt = 0;
  for (int qz = 0; qz < mz; ++qz) {
    const int z = axis_cell(cz, ncz, wz, qz);
    for (int qy = 0; qy < my; ++qy) {
      const int y = axis_cell(cy, ncy, wy, qy);
      const int rowbase = (z * ncy + y) * ncx;
      for (int part = 0; part < 2; ++part) {
        const int x0 = part ? b0 : a0, x1 = part ? b1 : a1;
        if (x0 > x1) continue;
        const int k0 = cell_start[rowbase + x0];
        const int k1 = cell_start[rowbase + x1] + cell_count[rowbase + x1];
#pragma unroll 4
        for (int k = k0; k < k1; ++k) {
          if (k == i) continue;
          // FP32 screen: accept below lo, reject above hi, exact FP64 test
          // between (lo/hi bracket vbuf2 by twice the FP32 error bound)
          bool take = false, exact = true;
          if (prefilter) {
            const float4 fk = vredf[k];
            float xf = fi.x - fk.x, yf = fi.y - fk.y, zf = fi.z - fk.z;
            xf = fabsf(xf) > hx ? xf - copysignf(bx, xf) : xf;
            yf = fabsf(yf) > hy ? yf - copysignf(by, yf) : yf;
            zf = fabsf(zf) > hz ? zf - copysignf(bz, zf) : zf;
            const float r2f = xf * xf + yf * yf + zf * zf;
            if (r2f > hi) continue;
            take = r2f < lo;
            exact = !take;
          }
          if (exact) {
            const double4 rk = vred[k];
            double xr = ri.x - rk.x, yr = ri.y - rk.y, zr = ri.z - rk.z;
            image3(box, xr, yr, zr);
            take = r2_exact(xr, yr, zr) <= vbuf2;
          }
          if (take && __ldg(vtab + (size_t)__ldg(&vinfo[k].x) * (nclass + 1)) == 0.0) take = false;
          if (take) {
            if (cnt < maxvnb) vnb[(size_t)cnt * npad + i] = k;
            ++cnt;
          }
        }
      }
    }
  }
  vnnb[i] = min(cnt, maxvnb);
  if (cnt > maxvnb) atomicOr(flags, DEV_LIST_OVERFLOW);
}

// buffered 14-7 pair terms of one pair at distance r (r2 = r^2): adds
// e/2 to eacc and returns de/r.  FP64: the reference's arithmetic with the
// taper in powers of r (switch.f:103-111); FP32: the same polynomial in the
// smoothstep form 1 - t^3 (10 - 15 t + 6 t^2), t = (r - cut)/(off - cut),
// since the expanded coefficients (up to 1e5 for a 0.9 A window) cancel far
// beyond FP32 precision.
template <typename U>
__device__ __forceinline__ U hal_pair(U r2, U rv, U eps, const VdwConst& vc, double& eacc) {
  const U rik = sqrt(r2);
  const U ghal = (U)vc.ghal, dhal = (U)vc.dhal;
  const U rv2 = rv * rv, rv7 = rv2 * rv2 * rv2 * rv;
  const U rik6 = r2 * r2 * r2;
  const U rik7 = rik6 * rik;
  const U rho = rik7 + ghal * rv7;
  const U tau = (dhal + U(1)) / (rik + dhal * rv);
  const U tau2 = tau * tau, tau7 = tau2 * tau2 * tau2 * tau;
  const U dtau = tau / (dhal + U(1));
  const U q7 = rv7 / rho;
  const U gtau = eps * tau7 * rik6 * (ghal + U(1)) * q7 * q7;
  U e = eps * tau7 * rv7 * ((ghal + U(1)) * q7 - U(2));
  U de = U(-7) * (dtau * e + gtau);
  if (r2 > (U)vc.cut2) {
    U taper, dtaper;
    if constexpr (std::is_same<U, double>::value) {
      const double rik3 = r2 * rik, rik4 = r2 * r2, rik5 = r2 * rik3;
      taper = vc.c5 * rik5 + vc.c4 * rik4 + vc.c3 * rik3 + vc.c2 * r2 + vc.c1 * rik + vc.c0;
      dtaper = 5.0 * vc.c5 * rik4 + 4.0 * vc.c4 * rik3 + 3.0 * vc.c3 * r2 + 2.0 * vc.c2 * rik + vc.c1;
    } else {
      const U w = (U)(1.0 / (vc.off - vc.cut));
      const U t = (rik - (U)vc.cut) * w;
      const U t2 = t * t;
      taper = U(1) - t2 * t * (U(10) - U(15) * t + U(6) * t2);
      dtaper = U(-30) * t2 * (U(1) - t) * (U(1) - t) * w;
    }
    de = e * dtaper + de * taper;
    e = e * taper;
  }
  eacc += 0.5 * (double)e;
  return de / rik;
}

// VIR: each block also writes the sum of its sites' pair virials (half of
// each pair from each end, ehal1.f:431-446) to vpart[block][6].
template <bool MIXED, bool VIR>
__global__ void __launch_bounds__(kBlock) k_ehal(int n, int npad, Box box, VdwConst vc,
                                                 const double4* __restrict__ vred, const float4* __restrict__ vredf,
                                                 const int2* __restrict__ vinfo, const double* __restrict__ vtab,
                                                 const int* __restrict__ perm, const int* __restrict__ sp_off,
                                                 const int* __restrict__ sp_ks, const int* __restrict__ sp_c,
                                                 const int* __restrict__ vnnb, const int* __restrict__ vnb,
                                                 unsigned long long* __restrict__ dev, double* __restrict__ epart,
                                                 double* __restrict__ vpart) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double eacc = 0.0;
  double v6[6] = {0, 0, 0, 0, 0, 0};
  if (i < n) {
    const double4 ri = vred[i];
    const float4 fi = vredf[i];
    const float bx = (float)box.l[0], by = (float)box.l[1], bz = (float)box.l[2];
    const float hx = 0.5f * bx, hy = 0.5f * by, hz = 0.5f * bz;
    const float off2f = (float)vc.off2;
    const int2 inf = vinfo[i];
    const int it = inf.x;
    const int io = perm[i];
    const int s0 = sp_off[io], s1 = sp_off[io + 1];
    const int nc2 = vc.nclass * vc.nclass;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    const int nn = vnnb[i];
    int knext = nn > 0 ? __ldg(vnb + i) : 0;  // list entries fetched one pair ahead
#pragma unroll 1
    for (int s = 0; s < nn; ++s) {
      const int k = knext;
      if (s + 1 < nn) knext = __ldg(vnb + (size_t)(s + 1) * npad + i);
      double xr, yr, zr;
      float xf = 0.f, yf = 0.f, zf = 0.f, r2f = 0.f;
      double rik2 = 0.0;
      if constexpr (MIXED) {
        const float4 fk = vredf[k];
        xf = fi.x - fk.x;
        yf = fi.y - fk.y;
        zf = fi.z - fk.z;
        xf = fabsf(xf) > hx ? xf - copysignf(bx, xf) : xf;
        yf = fabsf(yf) > hy ? yf - copysignf(by, yf) : yf;
        zf = fabsf(zf) > hz ? zf - copysignf(bz, zf) : zf;
        r2f = xf * xf + yf * yf + zf * zf;
        if (r2f > off2f) continue;
      } else {
        const double4 rk = vred[k];
        xr = ri.x - rk.x;
        yr = ri.y - rk.y;
        zr = ri.z - rk.z;
        image3(box, xr, yr, zr);
        rik2 = r2_exact(xr, yr, zr);
        if (rik2 > vc.off2) continue;
      }
      const int kt = __ldg(&vinfo[k].x);
      double vs = 1.0;
      bool is14 = false;
      for (int q = s0; q < s1; ++q)
        if (__ldg(sp_ks + q) == k) {
          const int cls = __ldg(sp_c + q);
          vs = cls == 0 ? vc.vscale[0] : cls == 1 ? vc.vscale[1] : cls == 2 ? vc.vscale[2]
                                                            : cls == 3 ? vc.vscale[3] : 1.0;
          is14 = cls == 2;
          break;
        }
      const int t = kt * vc.nclass + it;
      const double rv = __ldg(vtab + (is14 ? 2 * nc2 : 0) + t);
      const double eps = __ldg(vtab + (is14 ? 3 * nc2 : nc2) + t) * vs;
      double dx, dy, dz, px, py, pz;  // dE/dx of the pair and its separation
      if constexpr (MIXED) {
        const float de = hal_pair<float>(r2f, (float)rv, (float)eps, vc, eacc);
        dx = (double)(de * xf);
        dy = (double)(de * yf);
        dz = (double)(de * zf);
        px = xf;
        py = yf;
        pz = zf;
      } else {
        const double de = hal_pair<double>(rik2, rv, eps, vc, eacc);
        dx = de * xr;
        dy = de * yr;
        dz = de * zr;
        px = xr;
        py = yr;
        pz = zr;
      }
      gx += dx;
      gy += dy;
      gz += dz;
      if (VIR) {
        v6[0] += 0.5 * px * dx;
        v6[1] += 0.5 * py * dx;
        v6[2] += 0.5 * pz * dx;
        v6[3] += 0.5 * py * dy;
        v6[4] += 0.5 * pz * dy;
        v6[5] += 0.5 * pz * dz;
      }
    }
    // the site's force: to the atom (kred) and its parent (1 - kred)
    const int iv = inf.y;
    if (iv == i) {
      fix_add(dev + 3 * i + 0, gx);
      fix_add(dev + 3 * i + 1, gy);
      fix_add(dev + 3 * i + 2, gz);
    } else {
      const double redi = ri.w, rediv = 1.0 - redi;
      fix_add(dev + 3 * i + 0, gx * redi);
      fix_add(dev + 3 * i + 1, gy * redi);
      fix_add(dev + 3 * i + 2, gz * redi);
      fix_add(dev + 3 * iv + 0, gx * rediv);
      fix_add(dev + 3 * iv + 1, gy * rediv);
      fix_add(dev + 3 * iv + 2, gz * rediv);
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

template <typename P>
int alloc_once(Ctx& c, P** p, size_t count, const char* what) {
  if (*p) return THP_OK;
  return cuda_status(cudaMalloc((void**)p, sizeof(P) * count), &c, what);
}

}  // namespace

// Reduced sites for the current positions, and the vdW list when it is stale.
int launch_vdw_list(Ctx& c) {
  int st;
  if (!c.have_vdw) return THP_E_STATE;
  const size_t n = c.n;
  const int nb = (c.n + kBlock - 1) / kBlock;
  if ((st = alloc_once(c, &c.d_vred, n, "alloc vdw sites"))) return st;
  if ((st = alloc_once(c, &c.d_vinfo, n, "alloc vdw sites"))) return st;
  if ((st = alloc_once(c, &c.d_vredf, n, "alloc vdw sites"))) return st;
  k_vdw_sites<<<nb, kBlock, 0, c.stream>>>(c.n, c.d_perm, c.d_iperm, c.d_pos, c.d_vcls, c.d_vired, c.d_vkred, c.box,
                                           kShiftMax * kShiftMax, c.d_vred, c.d_vredf, c.d_vinfo, c.d_flags);
  if ((st = cuda_status(cudaGetLastError(), &c, "vdw sites"))) return st;
  // the vdW list: built after a re-sort, or once an atom has moved
  // lbuffer/2 since the positions it was built from (nblist.f:88-109)
  bool build = !c.have_vlist || c.vlist_epoch != c.sort_epoch;
  if (!build) {
    double disp = 0.0;
    if ((st = launch_max_displacement_from(c, c.d_vpos_built, &disp))) return st;
    build = disp >= 0.5 * c.cfg.lbuffer;
  }
  if (!build) return THP_OK;
  if (!c.d_vnb) {
    c.maxvnb = c.cfg.max_neighbors > 0 ? 2 * c.cfg.max_neighbors : kDefaultMaxVnb;
    if ((st = cuda_status(cudaMalloc((void**)&c.d_vnb, sizeof(int) * (size_t)c.maxvnb * c.npad), &c,
                          "alloc vdw list")))
      return st;
  }
  if ((st = alloc_once(c, &c.d_vnnb, n, "alloc vdw list"))) return st;
  if ((st = alloc_once(c, &c.d_vpos_built, n, "alloc vdw list"))) return st;
  // cells within reach: vdwcut + lbuffer, the atoms' drift since the sort
  // (below lbuffer/2 each) and the reduction shift on each side
  const double reach = c.vdw_cut + 2.0 * c.cfg.lbuffer + 2.0 * kShiftMax;
  int w[3];
  for (int d = 0; d < 3; ++d) w[d] = (int)ceil(reach / (c.cfg.box[d] / c.nc[d]) - 1e-12);
  const double vbuf = c.vdw_cut + c.cfg.lbuffer;
  const double vbuf2 = vbuf * vbuf;
  // the FP32 screen, bracketed as the polarization list build's: each
  // coordinate of a wrapped FP32 difference is off by at most 4 * 2^-24 *
  // Lmax, r^2 then by 2 vbuf dr + dr^2; pairs must sit well inside half a box
  const double hmin = std::min(c.box.half[0], std::min(c.box.half[1], c.box.half[2]));
  const int prefilter = hmin > vbuf + 1.0 ? 1 : 0;
  const double lmax = std::max(c.box.l[0], std::max(c.box.l[1], c.box.l[2]));
  const double dr = 1.7320508075688772 * 4.0 * lmax * 5.9604644775390625e-08;
  const double band = std::max(1e-5, 2.0 * (2.0 * vbuf * dr + dr * dr) / vbuf2);
  const float lo = (float)(vbuf2 * (1.0 - band)), hi = (float)(vbuf2 * (1.0 + band));
  k_vdw_list<<<nb, kBlock, 0, c.stream>>>(c.n, c.npad, c.box, vbuf2, prefilter, lo, hi, w[0], w[1], w[2], c.d_vred,
                                          c.d_vredf, c.d_vinfo, c.d_vtab, c.vdw_nclass, c.d_scell,
                                          c.d_cell_start, c.d_cell_count, c.nc[0], c.nc[1], c.nc[2], c.maxvnb, c.d_vnnb,
                                          c.d_vnb, c.d_flags);
  if ((st = cuda_status(cudaGetLastError(), &c, "vdw list"))) return st;
  cudaMemcpyAsync(c.d_vpos_built, c.d_pos, sizeof(double4) * n, cudaMemcpyDeviceToDevice, c.stream);
  c.have_vlist = true;
  c.vlist_epoch = c.sort_epoch;
  return THP_OK;
}

// van der Waals energy (into d_ev) and gradient (into d_out, original order)
// for the sorted positions and the cell sort of the context.
int launch_ehal(Ctx& c, double* d_out) {
  int st;
  if (!c.have_vdw) return THP_E_STATE;
  const size_t n = c.n;
  const int nb = (c.n + kBlock - 1) / kBlock;
  if ((st = alloc_once(c, &c.d_depfix, 3 * n, "alloc gradient"))) return st;
  if ((st = alloc_once(c, &c.d_evpart, (size_t)nb + 1, "alloc vdw partials"))) return st;
  c.d_ev = c.d_evpart + nb;
  unsigned long long* dev = c.d_depfix;
  if ((st = cuda_status(cudaMemsetAsync(dev, 0, sizeof(unsigned long long) * 3 * n, c.stream), &c, "zero dev")))
    return st;
  if ((st = launch_vdw_list(c))) return st;
  VdwConst vc;
  const double off = c.vdw_cut, cut = c.vdw_taper;
  vc.off = off;
  vc.cut = cut;
  vc.off2 = off * off;
  vc.cut2 = cut * cut;
  vc.c0 = vc.c1 = vc.c2 = vc.c3 = vc.c4 = vc.c5 = 0.0;
  if (cut < off) {  // switch.f:103-111
    const double off2 = off * off, cut2 = cut * cut;
    const double denom = pow(off - cut, 5.0);
    vc.c0 = off * off2 * (off2 - 5.0 * off * cut + 10.0 * cut2) / denom;
    vc.c1 = -30.0 * off2 * cut2 / denom;
    vc.c2 = 30.0 * (off2 * cut + off * cut2) / denom;
    vc.c3 = -10.0 * (off2 + 4.0 * off * cut + cut2) / denom;
    vc.c4 = 15.0 * (off + cut) / denom;
    vc.c5 = -6.0 / denom;
  }
  vc.ghal = c.vdw_ghal;
  vc.dhal = c.vdw_dhal;
  for (int j = 0; j < 4; ++j) vc.vscale[j] = c.vdw_scale[j];
  vc.vscale[4] = 1.0;
  vc.nclass = c.vdw_nclass;
  const bool vir = c.want_virial;
  double *kpart = nullptr, *vpart = nullptr, *epart = nullptr;
  if (vir && (st = virial_scratch(c, nb, 0, &kpart, &vpart, &epart))) return st;
#define THP_EHAL_ARGS                                                                                             \
  c.n, c.npad, c.box, vc, c.d_vred, c.d_vredf, c.d_vinfo, c.d_vtab, c.d_perm, c.d_sp_off, c.d_sp_ks, c.d_sp_c, \
      c.d_vnnb, c.d_vnb, dev, c.d_evpart, vpart
  if (c.mixed && vir)
    k_ehal<true, true><<<nb, kBlock, 0, c.stream>>>(THP_EHAL_ARGS);
  else if (c.mixed)
    k_ehal<true, false><<<nb, kBlock, 0, c.stream>>>(THP_EHAL_ARGS);
  else if (vir)
    k_ehal<false, true><<<nb, kBlock, 0, c.stream>>>(THP_EHAL_ARGS);
  else
    k_ehal<false, false><<<nb, kBlock, 0, c.stream>>>(THP_EHAL_ARGS);
#undef THP_EHAL_ARGS
  if ((st = cuda_status(cudaGetLastError(), &c, "ehal"))) return st;
  k_sum_partials<<<1, 256, 0, c.stream>>>(nb, c.d_evpart, c.d_ev);
  if ((st = cuda_status(cudaGetLastError(), &c, "ehal energy"))) return st;
  if (vir && (st = virial_total(c, 0, nb, 0, kpart, vpart, epart, c.h_vvir))) return st;
  return launch_gradient_out(c, dev, d_out);
}

}  // namespace thp
