// nblist.cu -- cell sort and polarization neighbor list on the device.
//
// Restates the pair set of mlistcell/build_cell_list (nblist.f:117-247,
// 607-866): every pair with minimum-image r^2 <= (ewaldcut+lbuffer)^2, r^2
// evaluated as (xi-xk) imaged by image.f:122-138 and summed unfused, so the
// set is bit-identical to the reference's.  The device layout differs: atoms
// are counting-sorted into cells of edge >= (ewaldcut+lbuffer)/2 and the list
// is a FULL list (both directions), slot-major nb[s*npad + i] so that a warp
// of consecutive atoms reads one coalesced row per slot.
#include <algorithm>

#include "kernels.h"

namespace thp {

namespace {

constexpr int kBlock = 256;

__global__ void k_cell_count(int n, Box box, int ncx, int ncy, int ncz, const double* __restrict__ xyz,
                             int* __restrict__ atom_cell, int* __restrict__ cell_count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = xyz[i], y = xyz[n + i], z = xyz[2 * n + i];
  image3(box, x, y, z);  // build_cell_list images the absolute coordinates
  int nc[3] = {ncx, ncy, ncz};
  double v[3] = {x, y, z};
  int c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double f = (v[d] + box.half[d]) / box.l[d];
    int q = (int)floor(f * nc[d]);
    c[d] = q < 0 ? 0 : (q >= nc[d] ? nc[d] - 1 : q);
  }
  int cell = (c[2] * ncy + c[1]) * ncx + c[0];
  atom_cell[i] = cell;
  atomicAdd(&cell_count[cell], 1);
}

// exclusive scan of m ints by one block of 1024 threads
__global__ void k_scan_single(int m, const int* __restrict__ in, int* __restrict__ out) {
  __shared__ int s[1024];
  int t = threadIdx.x;
  int chunk = (m + 1023) / 1024;
  int b = t * chunk, e = min(m, b + chunk);
  int sum = 0;
  for (int q = b; q < e; ++q) sum += in[q];
  s[t] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int v = t >= o ? s[t - o] : 0;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  int run = s[t] - sum;
  for (int q = b; q < e; ++q) {
    out[q] = run;
    run += in[q];
  }
}

// The same scan over many blocks: each block scans 1024 cells (k_scan_tiles,
// writing its total), one block scans the totals (k_scan_totals), and every
// block adds its offset (k_scan_offsets).  Used up to 1024 x 1024 cells.
__device__ __forceinline__ int block_excl_scan_1024(int v, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = s_warp[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    s_warp[lane] = t;  // inclusive totals of the warps
  }
  __syncthreads();
  const int before = w > 0 ? s_warp[w - 1] : 0;
  *total = s_warp[31];
  return before + x - v;
}

__global__ void __launch_bounds__(1024) k_scan_tiles(int m, const int* __restrict__ in, int* __restrict__ out,
                                                      int* __restrict__ tile_sum) {
  __shared__ int s_warp[32];
  const int i = blockIdx.x * 1024 + threadIdx.x;
  const int v = i < m ? in[i] : 0;
  int total;
  const int e = block_excl_scan_1024(v, s_warp, &total);
  if (i < m) out[i] = e;
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_totals(int nt, int* __restrict__ tile_sum) {
  __shared__ int s_warp[32];
  const int v = threadIdx.x < nt ? tile_sum[threadIdx.x] : 0;
  int total;
  const int e = block_excl_scan_1024(v, s_warp, &total);
  if (threadIdx.x < nt) tile_sum[threadIdx.x] = e;
}

__global__ void k_scan_offsets(int m, int* __restrict__ out, const int* __restrict__ tile_sum) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[i] += tile_sum[i >> 10];
}

__global__ void k_cell_fill(int n, const int* __restrict__ atom_cell, const int* __restrict__ cell_start,
                            int* __restrict__ cell_fill, int* __restrict__ perm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = atom_cell[i];
  int p = cell_start[c] + atomicAdd(&cell_fill[c], 1);
  perm[p] = i;
}

// deterministic order inside a cell: ascending original index
__global__ void k_cell_sort(int ncell, const int* __restrict__ cell_start, const int* __restrict__ cell_count,
                            int* __restrict__ perm, int* __restrict__ iperm, int* __restrict__ scell) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int b = cell_start[c], m = cell_count[c];
  for (int a = 1; a < m; ++a) {
    int v = perm[b + a];
    int q = a - 1;
    while (q >= 0 && perm[b + q] > v) {
      perm[b + q + 1] = perm[b + q];
      --q;
    }
    perm[b + q + 1] = v;
  }
  for (int a = 0; a < m; ++a) {
    iperm[perm[b + a]] = b + a;
    scell[b + a] = c;
  }
}

__global__ void k_gather_sorted(int n, Box box, const int* __restrict__ perm, const double* __restrict__ xyz,
                                const double* __restrict__ pdamp, const double* __restrict__ thole,
                                const double* __restrict__ pol, const double* __restrict__ rpole13,
                                int have_rpole, double4* __restrict__ pos, float4* __restrict__ posf,
                                double* __restrict__ sthole, double* __restrict__ spol,
                                double* __restrict__ srpole, double* __restrict__ mrec, float* __restrict__ mrecf,
                                float* __restrict__ erec, int* __restrict__ flags) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int o = perm[s];
  double x = xyz[o], y = xyz[n + o], z = xyz[2 * n + o];
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) atomicOr(flags, DEV_BAD_INPUT);
  pos[s] = make_double4(x, y, z, pdamp[o]);
  if (posf) {
    double wx = x, wy = y, wz = z;
    image3(box, wx, wy, wz);
    posf[s] = make_float4((float)wx, (float)wy, (float)wz, (float)pdamp[o]);
  }
  sthole[s] = thole[o];
  spol[s] = pol[o];
  // pair-pass record: thole always, multipoles once they are known
  double rec[12] = {thole[o], 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (have_rpole) {
    const double* r = rpole13 + (size_t)o * 13;
    double* q = srpole + (size_t)s * 10;
    q[0] = r[0];
    q[1] = r[1];
    q[2] = r[2];
    q[3] = r[3];
    q[4] = r[4];
    q[5] = r[5];
    q[6] = r[6];
    q[7] = r[8];
    q[8] = r[9];
    q[9] = r[12];
    const double m[10] = {r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[8], r[9], r[12]};
#pragma unroll
    for (int k = 0; k < 10; ++k) rec[1 + k] = m[k];
  }
  double2* m2 = reinterpret_cast<double2*>(mrec + (size_t)s * 12);
#pragma unroll
  for (int k = 0; k < 6; ++k) m2[k] = make_double2(rec[2 * k], rec[2 * k + 1]);
  if (mrecf) {
    float4* f4 = reinterpret_cast<float4*>(mrecf + (size_t)s * 12);
#pragma unroll
    for (int k = 0; k < 3; ++k)
      f4[k] = make_float4((float)rec[4 * k], (float)rec[4 * k + 1], (float)rec[4 * k + 2], (float)rec[4 * k + 3]);
  }
  if (erec) {
    // mixed direct-field record: wrapped position, 1/pdamp (0 for no
    // damping), thole, charge, dipole, quadrupole
    double wx = x, wy = y, wz = z;
    image3(box, wx, wy, wz);
    const double pd = pdamp[o];
    float4* f4 = reinterpret_cast<float4*>(erec + (size_t)s * 16);
    f4[0] = make_float4((float)wx, (float)wy, (float)wz, pd != 0.0 ? (float)(1.0 / pd) : 0.f);
    f4[1] = make_float4((float)rec[0], (float)rec[1], (float)rec[2], (float)rec[3]);
    f4[2] = make_float4((float)rec[4], (float)rec[5], (float)rec[6], (float)rec[7]);
    f4[3] = make_float4((float)rec[8], (float)rec[9], (float)rec[10], 0.f);
  }
}

__global__ void k_sp_to_sorted(int m, const int* __restrict__ iperm, const int* __restrict__ sp_k,
                               int* __restrict__ sp_ks) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < m) sp_ks[q] = iperm[sp_k[q]];
}

// Candidate search over the +-2 cell neighbourhood.  For every (dz, dy) row
// the cells cx-2..cx+2 are consecutive in the cell order, so their atoms form
// one contiguous range of sorted indices (two at a periodic wrap); a thread
// scans 25 such ranges instead of 125 cells.  Grids narrower than 5 cells in
// a dimension visit each cell of that dimension once.
__device__ __forceinline__ void row_ranges(int c, int nc, int& a0, int& a1, int& b0, int& b1) {
  // cell x-intervals [a0, a1] and [b0, b1] (b empty when b0 > b1)
  if (nc <= 5) {
    a0 = 0;
    a1 = nc - 1;
    b0 = 1;
    b1 = 0;
    return;
  }
  int lo = c - 2, hi = c + 2;
  if (lo < 0) {
    a0 = 0;
    a1 = hi;
    b0 = lo + nc;
    b1 = nc - 1;
  } else if (hi >= nc) {
    a0 = lo;
    a1 = nc - 1;
    b0 = 0;
    b1 = hi - nc;
  } else {
    a0 = lo;
    a1 = hi;
    b0 = 1;
    b1 = 0;
  }
}

__device__ __forceinline__ int axis_cells(int c, int nc, int q) {
  // q-th distinct cell of the +-2 window along y or z (q < min(nc, 5))
  return nc <= 5 ? q : ((c + q - 2) % nc + nc) % nc;
}

// minimum resident blocks per SM asked of the compiler (0: its own choice)
#ifndef THP_LIST_MINB
#define THP_LIST_MINB 0
#endif

// systems below this many atoms build their list with one warp per atom
#ifndef THP_LIST_WARP_ATOMS
#define THP_LIST_WARP_ATOMS 20000
#endif

// candidates loaded together by the per-row-shift list build
#ifndef THP_LIST_BATCH
#define THP_LIST_BATCH 8
#endif

// 1: larger systems with at least 7 cells per axis screen their candidates
// with one periodic shift per candidate row (list_row_shifted)
#ifndef THP_LIST_SHIFTED
#define THP_LIST_SHIFTED 1
#endif

// The list decision for candidate k of atom i: the FP32 screen accepts below
// lo and rejects above hi; between them (and for every candidate when the
// screen is off) the exact FP64 r^2 of the reference decides.
struct ListTest {
  Box box;
  double mbuf2;
  int prefilter;
  float lo, hi, bx, by, bz, hx, hy, hz;
  // the FP32 screen alone: 1 accept, 0 reject, 2 undecided
  __device__ __forceinline__ int screen(const float4& fi, const float4& fk) const {
    float xr = fi.x - fk.x, yr = fi.y - fk.y, zr = fi.z - fk.z;
    xr = fabsf(xr) > hx ? xr - copysignf(bx, xr) : xr;
    yr = fabsf(yr) > hy ? yr - copysignf(by, yr) : yr;
    zr = fabsf(zr) > hz ? zr - copysignf(bz, zr) : zr;
    const float r2f = xr * xr + yr * yr + zr * zr;
    return r2f > hi ? 0 : (r2f < lo ? 1 : 2);
  }
  __device__ __forceinline__ bool exact(const double4& pi, int k, const double4* __restrict__ pos) const {
    const double4 pk = pos[k];
    // midpointimage (domdecstuff.f:1773): pos = xi - xk, imaged
    double xr = __dadd_rn(pi.x, -pk.x), yr = __dadd_rn(pi.y, -pk.y), zr = __dadd_rn(pi.z, -pk.z);
    image3(box, xr, yr, zr);
    return r2_exact(xr, yr, zr) <= mbuf2;
  }
  __device__ __forceinline__ bool take(const double4& pi, const float4& fi, int k, const double4* __restrict__ pos,
                                       const float4* __restrict__ posf) const {
    if (prefilter) {
      const int d = screen(fi, posf[k]);
      if (d != 2) return d == 1;
    }
    return exact(pi, k, pos);
  }
};

// The list row of atom i, its candidates read from global memory.
__device__ __forceinline__ void list_row_global(int i, int npad, const ListTest& lt, int ncx, int ncy, int ncz,
                                                const double4* __restrict__ pos, const float4* __restrict__ posf,
                                                const int* __restrict__ scell, const int* __restrict__ cell_start,
                                                const int* __restrict__ cell_count, int maxnb,
                                                int* __restrict__ nnb, int* __restrict__ nb,
                                                int* __restrict__ flags) {
  const double4 pi = pos[i];
  const float4 fi = posf[i];
  const int c = scell[i];
  const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
  int a0, a1, b0, b1;
  row_ranges(cx, ncx, a0, a1, b0, b1);
  const int my = min(ncy, 5), mz = min(ncz, 5);
  int cnt = 0;
  for (int qz = 0; qz < mz; ++qz) {
    const int z = axis_cells(cz, ncz, qz);
    for (int qy = 0; qy < my; ++qy) {
      const int y = axis_cells(cy, ncy, qy);
      const int rowbase = (z * ncy + y) * ncx;
#pragma unroll
      for (int part = 0; part < 2; ++part) {
        const int x0 = part ? b0 : a0, x1 = part ? b1 : a1;
        if (x0 > x1) continue;
        const int k0 = cell_start[rowbase + x0];
        const int k1 = cell_start[rowbase + x1] + cell_count[rowbase + x1];
#pragma unroll 4
        for (int k = k0; k < k1; ++k) {
          if (k == i) continue;
          if (lt.take(pi, fi, k, pos, posf)) {
            if (cnt < maxnb) nb[(size_t)cnt * npad + i] = k;
            ++cnt;
          }
        }
      }
    }
  }
  nnb[i] = cnt;
  if (cnt > maxnb) atomicOr(flags, DEV_LIST_OVERFLOW);
}

// The same row with one periodic shift per candidate row instead of a wrap
// per candidate: with at least 7 cells along every axis, every candidate of
// the +-2 window lies within 3 cells (< half a box) of the atom once the
// rows past a face are shifted by one box length, so the FP32 screen is
// fi - shift - fk with no per-candidate image.  The screen's error bound is
// the same (two roundings per coordinate); the exact FP64 test still images
// each undecided pair itself.
__device__ __forceinline__ void list_row_shifted(int i, int npad, const ListTest& lt, int ncx, int ncy, int ncz,
                                                 const double4* __restrict__ pos, const float4* __restrict__ posf,
                                                 const int* __restrict__ scell, const int* __restrict__ cell_start,
                                                 const int* __restrict__ cell_count, int maxnb,
                                                 int* __restrict__ nnb, int* __restrict__ nb,
                                                 int* __restrict__ flags) {
  const double4 pi = pos[i];
  const float4 fi = posf[i];
  const int c = scell[i];
  const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
  int a0, a1, b0, b1;
  row_ranges(cx, ncx, a0, a1, b0, b1);
  // part b lies past the lower face (cx - 2 < 0) or the upper one
  const float fxb = cx < 2 ? fi.x + lt.bx : fi.x - lt.bx;
  int cnt = 0;
  for (int qz = 0; qz < 5; ++qz) {
    const int zr = cz + qz - 2;
    const int z = zr < 0 ? zr + ncz : (zr >= ncz ? zr - ncz : zr);
    const float fz = zr < 0 ? fi.z + lt.bz : (zr >= ncz ? fi.z - lt.bz : fi.z);
    for (int qy = 0; qy < 5; ++qy) {
      const int yr = cy + qy - 2;
      const int y = yr < 0 ? yr + ncy : (yr >= ncy ? yr - ncy : yr);
      const float fy = yr < 0 ? fi.y + lt.by : (yr >= ncy ? fi.y - lt.by : fi.y);
      const int rowbase = (z * ncy + y) * ncx;
#pragma unroll
      for (int part = 0; part < 2; ++part) {
        const int x0 = part ? b0 : a0, x1 = part ? b1 : a1;
        if (x0 > x1) continue;
        const float fx = part ? fxb : fi.x;
        const int k0 = cell_start[rowbase + x0];
        const int k1 = cell_start[rowbase + x1] + cell_count[rowbase + x1];
        // candidates in batches of THP_LIST_BATCH, all loads of a batch
        // issued before its tests (a slot past the range reads as far away)
        for (int kb = k0; kb < k1; kb += THP_LIST_BATCH) {
          float4 fk[THP_LIST_BATCH];
#pragma unroll
          for (int u = 0; u < THP_LIST_BATCH; ++u)
            fk[u] = kb + u < k1 ? __ldg(posf + kb + u) : make_float4(3.0e18f, 3.0e18f, 3.0e18f, 0.f);
#pragma unroll
          for (int u = 0; u < THP_LIST_BATCH; ++u) {
            const int k = kb + u;
            const float dx = fx - fk[u].x, dy = fy - fk[u].y, dz = fz - fk[u].z;
            const float r2f = dx * dx + dy * dy + dz * dz;
            if (r2f > lt.hi || k == i) continue;
            if (r2f >= lt.lo && !lt.exact(pi, k, pos)) continue;
            if (cnt < maxnb) nb[(size_t)cnt * npad + i] = k;
            ++cnt;
          }
        }
      }
    }
  }
  nnb[i] = cnt;
  if (cnt > maxnb) atomicOr(flags, DEV_LIST_OVERFLOW);
}

__global__ void __launch_bounds__(128, THP_LIST_MINB) k_build_list_shifted(int n, int npad, ListTest lt, int ncx,
                                                    int ncy, int ncz, const double4* __restrict__ pos,
                                                    const float4* __restrict__ posf, const int* __restrict__ scell,
                                                    const int* __restrict__ cell_start,
                                                    const int* __restrict__ cell_count, int maxnb,
                                                    int* __restrict__ nnb, int* __restrict__ nb,
                                                    int* __restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  list_row_shifted(i, npad, lt, ncx, ncy, ncz, pos, posf, scell, cell_start, cell_count, maxnb, nnb, nb, flags);
}

__global__ void __launch_bounds__(128, THP_LIST_MINB) k_build_list(int n, int npad, ListTest lt, int ncx,
                                                    int ncy, int ncz, const double4* __restrict__ pos,
                                                    const float4* __restrict__ posf, const int* __restrict__ scell,
                                                    const int* __restrict__ cell_start,
                                                    const int* __restrict__ cell_count, int maxnb,
                                                    int* __restrict__ nnb, int* __restrict__ nb,
                                                    int* __restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  list_row_global(i, npad, lt, ncx, ncy, ncz, pos, posf, scell, cell_start, cell_count, maxnb, nnb, nb, flags);
}

// The same list with one warp per atom: the lanes test 32 consecutive
// candidates of a cell-row range at a time and the accepted ones are written
// in candidate order (ballot prefix), so the list is the thread-per-atom
// kernel's entry for entry.  The ranges of all 25 rows are loaded at once
// (row q by lane q, passed around by shuffles), and each chunk's positions
// one chunk ahead of its tests, so a warp waits on far fewer dependent
// loads.  Small systems, where the +-2 cell window spans most of the box and
// few atoms leave most of the GPU idle, use it.
__global__ void __launch_bounds__(128) k_build_list_warp(int n, int npad, ListTest lt, int ncx, int ncy, int ncz,
                                                        const double4* __restrict__ pos,
                                                        const float4* __restrict__ posf,
                                                        const int* __restrict__ scell,
                                                        const int* __restrict__ cell_start,
                                                        const int* __restrict__ cell_count, int maxnb,
                                                        int* __restrict__ nnb, int* __restrict__ nb,
                                                        int* __restrict__ flags) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;  // the same for the whole warp
  const int lane = threadIdx.x & 31;
  const double4 pi = pos[i];
  const float4 fi = posf[i];
  const int c = scell[i];
  const int cx = c % ncx, cy = (c / ncx) % ncy, cz = c / (ncx * ncy);
  int a0, a1, b0, b1;
  row_ranges(cx, ncx, a0, a1, b0, b1);
  const int my = min(ncy, 5), mz = min(ncz, 5), nrow = my * mz;
  // the candidate ranges of all rows at once, row q on lane q: parts a and b
  int ra0 = 0, ra1 = 0, rb0 = 0, rb1 = 0;
  if (lane < nrow) {
    const int qz = lane / my, qy = lane - qz * my;
    const int rowbase = (axis_cells(cz, ncz, qz) * ncy + axis_cells(cy, ncy, qy)) * ncx;
    ra0 = cell_start[rowbase + a0];
    ra1 = cell_start[rowbase + a1] + cell_count[rowbase + a1];
    if (b0 <= b1) {
      rb0 = cell_start[rowbase + b0];
      rb1 = cell_start[rowbase + b1] + cell_count[rowbase + b1];
    }
  }
  // chunks of 32 candidates in the order row, part, position; each chunk's
  // positions are loaded one chunk ahead of its tests
  int q = 0, part = 0, kb = __shfl_sync(0xffffffffu, ra0, 0), ke = __shfl_sync(0xffffffffu, ra1, 0);
  auto advance = [&]() {  // to the next non-empty chunk; q == nrow past the last
    kb += 32;
    while (kb >= ke && q < nrow) {
      if (part == 0 && b0 <= b1) {
        part = 1;
        kb = __shfl_sync(0xffffffffu, rb0, q);
        ke = __shfl_sync(0xffffffffu, rb1, q);
      } else if (++q < nrow) {
        part = 0;
        kb = __shfl_sync(0xffffffffu, ra0, q);
        ke = __shfl_sync(0xffffffffu, ra1, q);
      }
    }
  };
  if (kb >= ke) {
    kb -= 32;
    advance();
  }
  auto load = [&](int k0, int k1) {
    const int k = k0 + lane;
    return (lt.prefilter && k < k1) ? __ldg(posf + k) : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  float4 fcur = q < nrow ? load(kb, ke) : make_float4(0.f, 0.f, 0.f, 0.f);
  int cnt = 0;
  while (q < nrow) {
    const int ck = kb, ce = ke;
    advance();
    const float4 fnext = q < nrow ? load(kb, ke) : make_float4(0.f, 0.f, 0.f, 0.f);
    const int k = ck + lane;
    bool t = false;
    if (k < ce && k != i) {
      if (lt.prefilter) {
        const int d = lt.screen(fi, fcur);
        t = d == 2 ? lt.exact(pi, k, pos) : d == 1;
      } else {
        t = lt.exact(pi, k, pos);
      }
    }
    fcur = fnext;
    const unsigned ball = __ballot_sync(0xffffffffu, t);
    if (t) {
      const int slot = cnt + __popc(ball & ((1u << lane) - 1u));
      if (slot < maxnb) nb[(size_t)slot * npad + i] = k;
    }
    cnt += __popc(ball);
  }
  if (lane == 0) {
    nnb[i] = cnt;
    if (cnt > maxnb) atomicOr(flags, DEV_LIST_OVERFLOW);
  }
}

// reference-format half list: row perm[i], partners with larger original index
__global__ void k_export(int n, int npad, int maxnb, const int* __restrict__ perm, const int* __restrict__ nnb,
                         const int* __restrict__ nb, int maxelst, int* __restrict__ nelst, int* __restrict__ elst,
                         int* __restrict__ flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int io = perm[i];
  int m = min(nnb[i], maxnb), c = 0;
  for (int s = 0; s < m; ++s) {
    int ko = perm[nb[(size_t)s * npad + i]];
    if (ko > io) {
      if (c < maxelst) elst[(size_t)io * maxelst + c] = ko;
      ++c;
    }
  }
  nelst[io] = min(c, maxelst);
  if (c >= maxelst) atomicOr(flags, DEV_LIST_OVERFLOW);
}

// rotpole.f:58-200 (Z-then-X = 1, Bisector = 2) and rotsite (rotpole.f:300-339)
__global__ void k_rotpole(int n, const double* __restrict__ xyz, const double* __restrict__ pole,
                          const int* __restrict__ frames, double* __restrict__ rpole) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* X = xyz;
  const double* Y = xyz + n;
  const double* Z = xyz + 2 * n;
  int iz = frames[3 * i], ix = frames[3 * i + 1], axt = frames[3 * i + 2];
  double a[3][3] = {{1, 0, 0}, {0, 0, 0}, {0, 0, 1}};
  double xi = X[i], yi = Y[i], zi = Z[i];
  if (axt == 1) {
    double dx = X[iz] - xi, dy = Y[iz] - yi, dz = Z[iz] - zi;
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    a[0][2] = dx / r; a[1][2] = dy / r; a[2][2] = dz / r;
    dx = X[ix] - xi; dy = Y[ix] - yi; dz = Z[ix] - zi;
    double dot = dx * a[0][2] + dy * a[1][2] + dz * a[2][2];
    dx -= dot * a[0][2]; dy -= dot * a[1][2]; dz -= dot * a[2][2];
    r = sqrt(dx * dx + dy * dy + dz * dz);
    a[0][0] = dx / r; a[1][0] = dy / r; a[2][0] = dz / r;
  } else if (axt == 2) {
    double dx = X[iz] - xi, dy = Y[iz] - yi, dz = Z[iz] - zi;
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    double dx1 = dx / r, dy1 = dy / r, dz1 = dz / r;
    dx = X[ix] - xi; dy = Y[ix] - yi; dz = Z[ix] - zi;
    r = sqrt(dx * dx + dy * dy + dz * dz);
    double dx2 = dx / r, dy2 = dy / r, dz2 = dz / r;
    dx = dx1 + dx2; dy = dy1 + dy2; dz = dz1 + dz2;
    r = sqrt(dx * dx + dy * dy + dz * dz);
    a[0][2] = dx / r; a[1][2] = dy / r; a[2][2] = dz / r;
    double dot = dx2 * a[0][2] + dy2 * a[1][2] + dz2 * a[2][2];
    dx = dx2 - dot * a[0][2]; dy = dy2 - dot * a[1][2]; dz = dz2 - dot * a[2][2];
    r = sqrt(dx * dx + dy * dy + dz * dz);
    a[0][0] = dx / r; a[1][0] = dy / r; a[2][0] = dz / r;
  }
  a[0][1] = a[2][0] * a[1][2] - a[1][0] * a[2][2];
  a[1][1] = a[0][0] * a[2][2] - a[2][0] * a[0][2];
  a[2][1] = a[1][0] * a[0][2] - a[0][0] * a[1][2];
  const double* p = pole + (size_t)i * 13;
  double* rp = rpole + (size_t)i * 13;
  rp[0] = p[0];
  for (int q = 0; q < 3; ++q) rp[1 + q] = p[1] * a[q][0] + p[2] * a[q][1] + p[3] * a[q][2];
  double r2[3][3];
  for (int q = 0; q < 3; ++q)
    for (int j = 0; j < 3; ++j) {
      if (j < q) {
        r2[q][j] = r2[j][q];
      } else {
        double s = 0.0;
        for (int k = 0; k < 3; ++k)
          for (int m = 0; m < 3; ++m) s += a[q][k] * a[j][m] * p[4 + 3 * k + m];
        r2[q][j] = s;
      }
    }
  for (int q = 0; q < 3; ++q)
    for (int j = 0; j < 3; ++j) rp[4 + 3 * q + j] = r2[q][j];
}

__global__ void k_max_disp(int n, const double4* __restrict__ pos, const double4* __restrict__ ref, Box box,
                           unsigned long long* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0.0;
  if (i < n) {
    double4 a = pos[i], b = ref[i];
    double x = a.x - b.x, y = a.y - b.y, z = a.z - b.z;
    d2 = x * x + y * y + z * z;
  }
  for (int o = 16; o > 0; o >>= 1) d2 = fmax(d2, __shfl_down_sync(0xffffffffu, d2, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(d2));
}

}  // namespace

int launch_sort_atoms(Ctx& c) {
  const int n = c.n;
  ++c.sort_epoch;  // sorted numbering changes: lists in it are stale
  const int nb = (n + kBlock - 1) / kBlock;
  cudaStream_t s = c.stream;
  // the last dipoles (warm start) follow their atoms into the new order; the
  // CG residual buffer is free between solves and holds them meanwhile
  const bool keep_mu = c.have_perm && c.have_dipoles;
  const bool keep_ef = c.have_perm && c.have_ef_prev;  // so does the last E0 (d_zr is free too)
  if (keep_mu) {
    int st = launch_to_orig6(c, c.d_mu, c.d_res, 2);
    if (st) return st;
  }
  if (keep_ef) {
    int st = launch_to_orig6(c, c.d_ef_prev, c.d_zr, 2);
    if (st) return st;
  }
  if (!c.have_perm) c.have_ef_prev = false;
  cudaMemsetAsync(c.d_cell_count, 0, sizeof(int) * c.ncell, s);
  cudaMemsetAsync(c.d_cell_fill, 0, sizeof(int) * c.ncell, s);
  k_cell_count<<<nb, kBlock, 0, s>>>(n, c.box, c.nc[0], c.nc[1], c.nc[2], c.d_xyz_orig, c.d_atom_cell,
                                     c.d_cell_count);
  const int ntile = (c.ncell + 1023) / 1024;
  // the tile totals live in the reduction partials (free outside the CG),
  // which hold 8 ints per 128 atoms plus 64
  if (ntile <= 1024 && (size_t)ntile <= 8 * ((size_t)c.nblk_reduce + 8)) {
    int* tile_sum = reinterpret_cast<int*>(c.d_partials);
    k_scan_tiles<<<ntile, 1024, 0, s>>>(c.ncell, c.d_cell_count, c.d_cell_start, tile_sum);
    k_scan_totals<<<1, 1024, 0, s>>>(ntile, tile_sum);
    k_scan_offsets<<<(c.ncell + 255) / 256, 256, 0, s>>>(c.ncell, c.d_cell_start, tile_sum);
  } else {
    k_scan_single<<<1, 1024, 0, s>>>(c.ncell, c.d_cell_count, c.d_cell_start);
  }
  k_cell_fill<<<nb, kBlock, 0, s>>>(n, c.d_atom_cell, c.d_cell_start, c.d_cell_fill, c.d_perm);
  k_cell_sort<<<(c.ncell + kBlock - 1) / kBlock, kBlock, 0, s>>>(c.ncell, c.d_cell_start, c.d_cell_count,
                                                                 c.d_perm, c.d_iperm, c.d_scell);
  c.have_perm = true;
  const int m = (int)c.sp_k.size();
  if (m > 0) k_sp_to_sorted<<<(m + 255) / 256, 256, 0, s>>>(m, c.d_iperm, c.d_sp_k, c.d_sp_ks);
  int st = cuda_status(cudaGetLastError(), &c, "sort atoms");
  if (!st && keep_mu) st = launch_to_sorted6(c, c.d_res, c.d_mu, 2);
  if (!st && keep_ef) st = launch_to_sorted6(c, c.d_zr, c.d_ef_prev, 2);
  return st;
}

int launch_gather_sorted(Ctx& c) {
  const int n = c.n;
  const int nb = (n + kBlock - 1) / kBlock;
  // d_par_orig holds pdamp, thole, polarity planes in original order
  k_gather_sorted<<<nb, kBlock, 0, c.stream>>>(n, c.box, c.d_perm, c.d_xyz_orig, c.d_par_orig,
                                               c.d_par_orig + n, c.d_par_orig + 2 * n, c.d_rpole_orig,
                                               c.have_rpole ? 1 : 0, c.d_pos, c.d_posf,
                                               c.d_thole, c.d_pol, c.d_rpole, c.d_mrec,
                                               c.mixed ? c.d_mrecf : nullptr, c.mixed ? c.d_erec : nullptr,
                                               c.d_flags);
  return cuda_status(cudaGetLastError(), &c, "gather sorted");
}

int launch_build_list(Ctx& c) { return launch_build_list_on(c, c.stream); }

int launch_build_list_on(Ctx& c, cudaStream_t s) {
  const int n = c.n;
  const double rl = c.cfg.ewaldcut + c.cfg.lbuffer;
  const double mbuf2 = rl * rl;
  // the FP32 screen needs every list pair far from the half-box wrap point
  const double hmin = std::min(c.box.half[0], std::min(c.box.half[1], c.box.half[2]));
  const int prefilter = hmin > rl + 1.0 ? 1 : 0;
  // |x| <= L/2 in FP32: each coordinate of a difference is off by at most
  // 4 * 2^-24 * Lmax (two roundings, the wrap by L); r^2 then by 2 rl dr + dr^2
  const double lmax = std::max(c.box.l[0], std::max(c.box.l[1], c.box.l[2]));
  const double dr = 1.7320508075688772 * 4.0 * lmax * 5.9604644775390625e-08;
  const double band = std::max(1e-5, 2.0 * (2.0 * rl * dr + dr * dr) / mbuf2);
  ListTest lt;
  lt.box = c.box;
  lt.mbuf2 = mbuf2;
  lt.prefilter = prefilter;
  lt.lo = (float)(mbuf2 * (1.0 - band));
  lt.hi = (float)(mbuf2 * (1.0 + band));
  lt.bx = (float)c.box.l[0];
  lt.by = (float)c.box.l[1];
  lt.bz = (float)c.box.l[2];
  lt.hx = 0.5f * lt.bx;
  lt.hy = 0.5f * lt.by;
  lt.hz = 0.5f * lt.bz;
  if (n < THP_LIST_WARP_ATOMS)
    k_build_list_warp<<<(n + 3) / 4, 128, 0, s>>>(n, c.npad, lt, c.nc[0], c.nc[1], c.nc[2], c.d_pos, c.d_posf,
                                                  c.d_scell, c.d_cell_start, c.d_cell_count, c.maxnb, c.d_nnb,
                                                  c.d_nb, c.d_flags);
  else if (THP_LIST_SHIFTED && prefilter && c.nc[0] >= 7 && c.nc[1] >= 7 && c.nc[2] >= 7)
    k_build_list_shifted<<<(n + 127) / 128, 128, 0, s>>>(n, c.npad, lt, c.nc[0], c.nc[1], c.nc[2], c.d_pos,
                                                         c.d_posf, c.d_scell, c.d_cell_start, c.d_cell_count,
                                                         c.maxnb, c.d_nnb, c.d_nb, c.d_flags);
  else
    k_build_list<<<(n + 127) / 128, 128, 0, s>>>(n, c.npad, lt, c.nc[0], c.nc[1], c.nc[2], c.d_pos, c.d_posf,
                                                 c.d_scell, c.d_cell_start, c.d_cell_count, c.maxnb, c.d_nnb,
                                                 c.d_nb, c.d_flags);
  cudaMemcpyAsync(c.d_pos_built, c.d_pos, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s);
  return cuda_status(cudaGetLastError(), &c, "build list");
}

int launch_export_list(Ctx& c, int maxelst, int* d_nelst, int* d_elst) {
  return launch_export_pairs(c, c.d_nnb, c.d_nb, c.maxnb, maxelst, d_nelst, d_elst);
}

int launch_export_pairs(Ctx& c, const int* nnb, const int* nb, int maxnb, int maxelst, int* d_nelst, int* d_elst) {
  const int n = c.n;
  k_export<<<(n + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(n, c.npad, maxnb, c.d_perm, nnb, nb, maxelst, d_nelst,
                                                               d_elst, c.d_flags);
  return cuda_status(cudaGetLastError(), &c, "export list");
}

int launch_rotpole(Ctx& c) {
  const int n = c.n;
  k_rotpole<<<(n + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(n, c.d_xyz_orig, c.d_pole_local, c.d_frames,
                                                                c.d_rpole_orig);
  return cuda_status(cudaGetLastError(), &c, "rotpole");
}

int launch_max_displacement(Ctx& c, double* h_out) { return launch_max_displacement_from(c, c.d_pos_built, h_out); }

int launch_max_displacement_from(Ctx& c, const double4* ref, double* h_out) {
  unsigned long long* d = reinterpret_cast<unsigned long long*>(c.d_partials);
  cudaMemsetAsync(d, 0, sizeof(unsigned long long), c.stream);
  k_max_disp<<<(c.n + kBlock - 1) / kBlock, kBlock, 0, c.stream>>>(c.n, c.d_pos, ref, c.box, d);
  unsigned long long v = 0;
  cudaMemcpyAsync(&v, d, sizeof(v), cudaMemcpyDeviceToHost, c.stream);
  int st = cuda_status(cudaStreamSynchronize(c.stream), &c, "max displacement");
  double d2;
  memcpy(&d2, &v, sizeof(d2));
  *h_out = sqrt(d2);
  return st;
}

}  // namespace thp
