// solver.cu -- device-resident preconditioned conjugate gradient.
//
// inducepcg_pme2 (newinduce_pme2.f:285-636) with every vector and scalar on
// the device.  Per iteration (systems of THP_OVERLAP_MIN_ATOMS atoms and
// more; smaller ones run one fused matvec kernel after the PME branch):
//   1. pp = zr + beta*pp (the mixed form also writes the 32-byte partner
//      records of its FP32 real-space row);
//   2. fork: the real-space row T_real pp runs on the side stream while the
//      main stream spreads pp on the PME grid, runs cuFFT forward, qfac and
//      cuFFT backward;
//   3. join, then the combine kernel gathers the dipole field from the grid
//      and forms h = T_real pp + pp/alpha + dipfield - self term; partial
//      pp.h; the last block forms gg and alpha;
//   4. update kernel: mu += alpha pp, res -= alpha h, zr = diag res; partial
//      ggnew and ene; the last block forms beta, the residual norm and the
//      convergence / stop flags.
// Reductions write per-block partials summed in a fixed order by the last
// block, so the CG scalars do not depend on thread scheduling.  Once the
// stop flag is set every later kernel returns at entry, so the host can
// enqueue iterations ahead and read the flag only once per chunk.
#include <cstring>

#include "cg_dev.cuh"
#include "kernels.h"

// Systems of at least THP_OVERLAP_MIN_ATOMS atoms run the real-space row of
// each CG matvec on a side stream, concurrent with the PME branch.  Smaller
// systems are launch-bound (and overlap with each other when batched), so
// they use one fused matvec kernel after the PME branch.
// 1: the CG loop runs on the device as one graph with a conditional WHILE
// node; 0: graph-replayed chunks of kCgChunk iterations with a host check
#ifndef THP_DEVICE_LOOP
#define THP_DEVICE_LOOP 1
#endif

// minimum resident blocks per SM asked of the compiler for the real-space row
#ifndef THP_ROW_MINB
#define THP_ROW_MINB 0
#endif

// systems of at least this many atoms read the mixed row's pair stream
// (~1.7 kB per atom, far beyond L2 from here on) without allocating in L1
#ifndef THP_STREAM_NO_L1_ATOMS
#define THP_STREAM_NO_L1_ATOMS 80000
#endif

#ifndef THP_OVERLAP_MIN_ATOMS
#define THP_OVERLAP_MIN_ATOMS 20000
#endif

// systems below this many atoms run the fused matvec in blocks of 32 atoms
#ifndef THP_MATVEC_SMALL_ATOMS
#define THP_MATVEC_SMALL_ATOMS 8000
#endif

namespace thp {

PairRows pair_rows(const Ctx& c);
float row_interior(const Ctx& c);
int group_blocks(int n, int block);

namespace {

using namespace cg;




// h = T_real x + x/alpha + dipfield(x) - term x and the reductions of one
// CG step (cg_matvec_block); dipfield comes from k_gather_dip.
template <bool MIXED, int GPW>
__global__ void __launch_bounds__(kBlock) k_cg_matvec(PairRows pr, Box box, const double4* __restrict__ pos,
                                                      const float4* __restrict__ posf, const double* __restrict__ dipf,
                                                      const double* __restrict__ x, const float* __restrict__ xf,
                                                      const double* __restrict__ pol, const double* __restrict__ ef,
                                                      double term, int init, double* __restrict__ h,
                                                      double* __restrict__ res, double* __restrict__ zr,
                                                      double* __restrict__ pp, CgScalars* cg,
                                                      double* __restrict__ partials, float interior) {
  if (cg->stop) return;
  cg_matvec_block<MIXED, 0, false, GPW>((int)blockIdx.x, (int)gridDim.x, pr, box, pos, posf, dipf, PmeGeom{},
                                        nullptr, x, xf, nullptr, nullptr, pol, ef, term, init, h, res, zr, pp, cg,
                                        partials, interior);
}

// pp = zr + beta pp (newinduce_pme2.f:553-559) of the overlapped FP64 rows.
__global__ void __launch_bounds__(256) k_pp_update(int n, const double* __restrict__ zr, double* __restrict__ x,
                                                  const CgScalars* __restrict__ cg) {
  if (cg->stop) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6 * n) return;
  x[t] = zr[t] + cg->beta[(t % 6) < 3 ? 0 : 1] * x[t];
}

// The same update for the overlapped rows of the mixed form, which read the
// FP32 dipoles from the per-atom records (rec, mpz) with the wrapped FP32
// position beside them; one thread per atom.  update 0 only writes the
// records of x.
template <typename V>
__global__ void __launch_bounds__(256) k_pp_rec(int n, int update, const V* __restrict__ zr,
                                               V* __restrict__ x, const float4* __restrict__ posf,
                                               float* __restrict__ rec, float* __restrict__ mpz,
                                               const CgScalars* __restrict__ cg) {
  if (update && cg->stop) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v[6];
  load6(x + (size_t)i * 6, v);
  if (update) {
    double z[6];
    load6(zr + (size_t)i * 6, z);
    const double bd = cg->beta[0], bp = cg->beta[1];
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] = z[q] + (q < 3 ? bd : bp) * v[q];
    store6(x + (size_t)i * 6, v);
  }
  const float4 p = posf[i];
  float4* r = reinterpret_cast<float4*>(rec + (size_t)i * 8);
  r[0] = make_float4(p.x, p.y, p.z, (float)v[0]);
  r[1] = make_float4((float)v[1], (float)v[2], (float)v[3], (float)v[4]);
  mpz[i] = (float)v[5];
}

// real-space part of h only: hreal = T_real x (tmatxb_pme without the
// diagonal), one warp per group of four atoms; lane j < 6 of an atom writes
// component j
template <bool MIXED, bool NOL1, typename HV>
__global__ void __launch_bounds__(kBlock, THP_ROW_MINB) k_real_row(PairRows pr, Box box, const double4* __restrict__ pos,
                                                     const float* __restrict__ rec, const double* __restrict__ x,
                                                     const float* __restrict__ mpz, const CgScalars* __restrict__ cg,
                                                     int check_stop, float interior, HV* __restrict__ hreal) {
  if (check_stop && cg->stop) return;
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (4 * g >= pr.n) return;
  const int lane = threadIdx.x & 31;
  const int i = 4 * g + (lane >> 3), j = lane & 7;
  if (MIXED) {
    float a32[6];
    group_row<float, THP_GROW_U32, NOL1>(pr, PartnerRec{rec, mpz},
                                         Image32{(float)box.l[0], (float)box.l[1], (float)box.l[2]}, g, lane, a32,
                                         interior);
    if (j < 6 && i < pr.n) hreal[(size_t)i * 6 + j] = (HV)pick6(a32, j);
  } else {
    double a64[6];
    group_row<double, THP_GROW_U64, NOL1>(pr, Partner64{pos, x}, Image64{box}, g, lane, a64, -1.0);
    if (j < 6 && i < pr.n) hreal[(size_t)i * 6 + j] = (HV)pick6(a64, j);
  }
}

// h = hreal + x/alpha + dipfield(x) - term x and the reductions of one CG
// step (cg_combine_block); hreal comes from k_real_row.
template <int GATHER, typename XV, typename V>
__global__ void __launch_bounds__(kBlock) k_cg_combine(int n, const double* __restrict__ dipf, PmeGeom g,
                                                       const double4* __restrict__ pos, const void* __restrict__ grid,
                                                       const XV* __restrict__ x, const double* __restrict__ pol,
                                                       const double* __restrict__ ef, double term, int init,
                                                       V* __restrict__ h, V* __restrict__ res, V* __restrict__ zr,
                                                       V* __restrict__ pp, CgScalars* cg,
                                                       double* __restrict__ partials) {
  if (cg->stop) return;
  cg_combine_block<GATHER, XV, V>((int)blockIdx.x, (int)gridDim.x, n, dipf, g, pos, grid, x, pol, ef, term, init, h,
                                  res, zr, pp, cg, partials);
}

// mu, residual and preconditioned residual of one CG step (cg_update_block)
template <typename V>
__global__ void __launch_bounds__(kBlock) k_cg_update(int n, const double* __restrict__ pol,
                                                      const V* __restrict__ h, const V* __restrict__ pp,
                                                      double* __restrict__ mu, V* __restrict__ res,
                                                      V* __restrict__ zr, CgScalars* cg, double* __restrict__ partials,
                                                      double poleps, int politer) {
  if (cg->stop) return;
  cg_update_block<V>((int)blockIdx.x, (int)gridDim.x, n, pol, h, pp, mu, res, zr, cg, partials, poleps, politer);
}

// Last node of the device-side loop body: keep looping while the CG has not
// stopped, and never more than max_loops bodies (a hard bound on the loop,
// whatever the kernels before it did).
__global__ void k_loop_cond(CgScalars* cg, cudaGraphConditionalHandle handle, int max_loops) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int l = ++cg->loops;
  unsigned keep = (cg->stop == 0 && l < max_loops) ? 1u : 0u;
  if (!keep) cg->stop = 1;
  cudaGraphSetConditional(handle, keep);
}

__global__ void k_guess_direct(int n, const double* __restrict__ pol, const double* __restrict__ ef,
                               double* __restrict__ mu) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * 6) return;
  mu[t] = pol[t / 6] * ef[t];
}

// Warm start corrected to first order for the change of the direct field
// since the last solve: mu += alpha (E0 - E0_prev).  Then E0_prev = E0.
__global__ void k_guess_delta(int n, const double* __restrict__ pol, const double* __restrict__ ef,
                              double* __restrict__ ef_prev, double* __restrict__ mu) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * 6) return;
  const double e = ef[t];
  mu[t] += pol[t / 6] * (e - ef_prev[t]);
  ef_prev[t] = e;
}

// epolar0c via the identity Epol = -1/2 electric sum uind . E_p(perm)
// (epreal0c + eprecip + self of epolar.f:47-520 sum to exactly this form)
// Epol = -1/2 electric sum uind . E_p, and the CG's ene (newinduce_pme2.f:
// 560-566: -1/2 sum mu . (res + ef) for the d and p sets, in units of
// electric) from the final mu and residual; res is stored as V.
template <typename V>
__global__ void __launch_bounds__(kBlock) k_epol(int n, const double* __restrict__ mu, const double* __restrict__ ef,
                                                 const V* __restrict__ res, CgScalars* cg,
                                                 double* __restrict__ partials) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double red[3] = {0.0, 0.0, 0.0};
  if (i < n) {
    double m[6], e[6], r[6];
    load6(mu + (size_t)i * 6, m);
    load6(ef + (size_t)i * 6, e);
    load6(res + (size_t)i * 6, r);
    red[0] = m[0] * e[3] + m[1] * e[4] + m[2] * e[5];
#pragma unroll
    for (int q = 0; q < 6; ++q) red[q < 3 ? 1 : 2] -= 0.5 * (m[q] * (r[q] + e[q]));
  }
  double tot[3];
  if (grid_reduce<3>(red, partials, &cg->counter[2], tot) && threadIdx.x == 0) {
    cg->epol = -0.5 * kElectric * tot[0];
    cg->ene[0] = tot[1];
    cg->ene[1] = tot[2];
  }
}

// original [n][nrhs][3] <-> sorted [n][6]
__global__ void k_to_sorted6(int n, int nrhs, const int* __restrict__ iperm, const double* __restrict__ in,
                             double* __restrict__ out) {
  int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  int s = iperm[o];
  for (int q = 0; q < 6; ++q) out[(size_t)s * 6 + q] = (q < 3 * nrhs) ? in[(size_t)o * 3 * nrhs + q] : 0.0;
}
__global__ void k_to_orig6(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ in,
                           double* __restrict__ out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int o = perm[s];
  for (int q = 0; q < 3 * nrhs; ++q) out[(size_t)o * 3 * nrhs + q] = in[(size_t)s * 6 + q];
}

// sorted [n][6] -> original-order d dipoles [n][3] followed by p dipoles [n][3]
__global__ void k_split_dipoles(int n, const int* __restrict__ perm, const double* __restrict__ in,
                                double* __restrict__ out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const size_t o = (size_t)perm[s] * 3;
  const double* v = in + (size_t)s * 6;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    out[o + q] = v[q];
    out[(size_t)3 * n + o + q] = v[3 + q];
  }
}

}  // namespace

int launch_split_dipoles(Ctx& c, const double* d_sorted, double* d_out) {
  k_split_dipoles<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.d_perm, d_sorted, d_out);
  return cuda_status(cudaGetLastError(), &c, "split dipoles");
}

int launch_to_sorted6(Ctx& c, const double* d_orig, double* d_sorted, int nrhs) {
  k_to_sorted6<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, nrhs, c.d_iperm, d_orig, d_sorted);
  return cuda_status(cudaGetLastError(), &c, "to sorted");
}
int launch_to_orig6(Ctx& c, const double* d_sorted, double* d_orig, int nrhs) {
  k_to_orig6<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, nrhs, c.d_perm, d_sorted, d_orig);
  return cuda_status(cudaGetLastError(), &c, "to orig");
}

static void prof_mark(Ctx& c, cudaStream_t s) {
  if (!c.profiling) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, s);
  c.prof_events.push_back(e);
}

bool overlap_rows(const Ctx& c) { return c.n >= THP_OVERLAP_MIN_ATOMS; }
static bool overlapped(const Ctx& c) { return overlap_rows(c); }

// One application of the CG matrix with the real-space row on the side
// stream and the PME branch (spread, FFTs) on the main stream; x and, for
// the mixed form, its partner records (k_pp_rec) are final when this is
// enqueued.
template <typename XV>
static int matvec_overlapped(Ctx& c, const XV* x, int init) {
  const int nb = (c.n + kBlock - 1) / kBlock;
  int st;
  cudaEventRecord(c.ev_fork, c.stream);
  cudaStreamWaitEvent(c.stream2, c.ev_fork, 0);
  PairRows pr = pair_rows(c);
  const int nbr = group_blocks(c.n, kBlock);  // one warp per group of four atoms
  const float interior = row_interior(c);
  prof_mark(c, c.stream2);
  if (c.mixed && c.n >= THP_STREAM_NO_L1_ATOMS)
    k_real_row<true, true, float><<<nbr, kBlock, 0, c.stream2>>>(pr, c.box, c.d_pos, c.d_rec, nullptr, c.d_mpz, c.d_cg,
                                                                 !init, interior, c.d_hf);
  else if (c.mixed)
    k_real_row<true, false, float><<<nbr, kBlock, 0, c.stream2>>>(pr, c.box, c.d_pos, c.d_rec, nullptr, c.d_mpz,
                                                                  c.d_cg, !init, interior, c.d_hf);
  else if constexpr (std::is_same<XV, double>::value)
    k_real_row<false, false, double><<<nbr, kBlock, 0, c.stream2>>>(pr, c.box, c.d_pos, nullptr, x, nullptr, c.d_cg,
                                                                    !init, -1.f, c.d_h);
  prof_mark(c, c.stream2);
  if ((st = cuda_status(cudaGetLastError(), &c, "real row"))) return st;
  cudaEventRecord(c.ev_join, c.stream2);
  if constexpr (std::is_same<XV, float>::value)
    st = launch_pme_dipole_f32(c, x);
  else
    st = launch_pme_dipole(c, x, nullptr, 2);
  if (st) return st;
  const double a = c.cfg.aewald;
  const double term = (4.0 / 3.0) * a * a * a / kSqrtPi;
  const PmeGeom g = pme_geom(c);
  cudaStreamWaitEvent(c.stream, c.ev_join, 0);
  if (c.mixed)
    k_cg_combine<1, XV, float><<<nb, kBlock, 0, c.stream>>>(c.n, nullptr, g, c.d_pos, c.d_grid, x, c.d_pol, c.d_ef,
                                                            term, init, c.d_hf, c.d_resf, c.d_zrf, c.d_ppf, c.d_cg,
                                                            c.d_partials);
  else if constexpr (std::is_same<XV, double>::value)
    k_cg_combine<2, double, double><<<nb, kBlock, 0, c.stream>>>(c.n, nullptr, g, c.d_pos, c.d_grid, x, c.d_pol,
                                                                 c.d_ef, term, init, c.d_h, c.d_res, c.d_zr, c.d_pp,
                                                                 c.d_cg, c.d_partials);
  return cuda_status(cudaGetLastError(), &c, "cg combine");
}

static int launch_matvec(Ctx& c, const double* x, int init) {
  int st = launch_gather_dip(c, c.d_dip, init == 0);
  if (st) return st;
  prof_mark(c, c.stream);
  PairRows pr = pair_rows(c);
  const double a = c.cfg.aewald;
  const double term = (4.0 / 3.0) * a * a * a / kSqrtPi;
  const float interior = c.mixed ? row_interior(c) : -1.f;
#define THP_MATVEC_ARGS                                                                                          \
  pr, c.box, c.d_pos, c.d_posf, c.d_dip, x, c.d_vecf, c.d_pol, c.d_ef, term, init, c.d_h, c.d_res, c.d_zr, c.d_pp, \
      c.d_cg, c.d_partials, interior
  // small systems: two groups per warp (blocks of 32 atoms), so their few
  // atoms spread over many blocks instead of long per-warp chains
  if (c.n < THP_MATVEC_SMALL_ATOMS) {
    const int nb = (c.n + 31) / 32;
    if (c.mixed)
      k_cg_matvec<true, 2><<<nb, kBlock, 0, c.stream>>>(THP_MATVEC_ARGS);
    else
      k_cg_matvec<false, 2><<<nb, kBlock, 0, c.stream>>>(THP_MATVEC_ARGS);
  } else {
    const int nb = (c.n + kBlock - 1) / kBlock;
    if (c.mixed)
      k_cg_matvec<true, 8><<<nb, kBlock, 0, c.stream>>>(THP_MATVEC_ARGS);
    else
      k_cg_matvec<false, 8><<<nb, kBlock, 0, c.stream>>>(THP_MATVEC_ARGS);
  }
#undef THP_MATVEC_ARGS
  prof_mark(c, c.stream);
  return cuda_status(cudaGetLastError(), &c, "cg matvec");
}

static int enqueue_iteration(Ctx& c) {
  int st;
  const int nb = (c.n + kBlock - 1) / kBlock;
  if (overlapped(c) && c.mixed) {
    k_pp_rec<float><<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, 1, c.d_zrf, c.d_ppf, c.d_posf, c.d_rec, c.d_mpz,
                                                             c.d_cg);
    if ((st = cuda_status(cudaGetLastError(), &c, "pp update"))) return st;
    if ((st = matvec_overlapped<float>(c, c.d_ppf, 0))) return st;
    k_cg_update<float><<<nb, kBlock, 0, c.stream>>>(c.n, c.d_pol, c.d_hf, c.d_ppf, c.d_mu, c.d_resf,
                                                    c.d_zrf, c.d_cg, c.d_partials, c.cfg.poleps, c.cfg.politer);
    return cuda_status(cudaGetLastError(), &c, "cg update");
  }
  if (overlapped(c)) {
    k_pp_update<<<(6 * c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.d_zr, c.d_pp, c.d_cg);
    if ((st = cuda_status(cudaGetLastError(), &c, "pp update"))) return st;
    if ((st = matvec_overlapped<double>(c, c.d_pp, 0))) return st;
  } else {
    if ((st = launch_pme_dipole(c, c.d_pp, nullptr, 1))) return st;
    if ((st = launch_matvec(c, c.d_pp, 0))) return st;
  }
  k_cg_update<double><<<nb, kBlock, 0, c.stream>>>(c.n, c.d_pol, c.d_h, c.d_pp, c.d_mu, c.d_res, c.d_zr,
                                                   c.d_cg, c.d_partials, c.cfg.poleps, c.cfg.politer);
  return cuda_status(cudaGetLastError(), &c, "cg update");
}

// Initial residual on the guess (newinduce_pme2.f:161-200, 398-417), async.
int pcg_begin(Ctx& c, int guess) {
  int st;
  cudaMemsetAsync(c.d_cg, 0, sizeof(CgScalars), c.stream);
  if (guess == THP_GUESS_DIRECT) {
    k_guess_direct<<<(c.n * 6 + 255) / 256, 256, 0, c.stream>>>(c.n, c.d_pol, c.d_ef, c.d_mu);
  }
  // the last dipoles plus alpha times the change of E0 since their solve
  // (about one CG iteration fewer for a small displacement of the atoms);
  // every start records this solve's E0 for the next one
  if (guess == THP_GUESS_PREVIOUS && c.have_ef_prev)
    k_guess_delta<<<(c.n * 6 + 255) / 256, 256, 0, c.stream>>>(c.n, c.d_pol, c.d_ef, c.d_ef_prev, c.d_mu);
  else
    cudaMemcpyAsync(c.d_ef_prev, c.d_ef, sizeof(double) * 6 * c.n, cudaMemcpyDeviceToDevice, c.stream);
  c.have_ef_prev = true;
  if ((st = cuda_status(cudaGetLastError(), &c, "cg start"))) return st;
  if (overlapped(c)) {
    if (c.mixed) {
      k_pp_rec<double><<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, 0, nullptr, c.d_mu, c.d_posf, c.d_rec, c.d_mpz,
                                                                c.d_cg);
      if ((st = cuda_status(cudaGetLastError(), &c, "mu copy"))) return st;
    }
    return matvec_overlapped<double>(c, c.d_mu, 1);
  }
  if ((st = launch_pme_dipole(c, c.d_mu, nullptr, 0))) return st;
  return launch_matvec(c, c.d_mu, 1);
}

static int enqueue_chunk(Ctx& c) {
  int st;
  for (int q = 0; q < kCgChunk; ++q)
    if ((st = enqueue_iteration(c))) return st;
  return cuda_status(cudaMemcpyAsync(c.h_cg, c.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost, c.stream), &c,
                     "cg scalars");
}

// kCgChunk iterations plus the copy of the CG scalars to pinned host memory,
// replayed from a CUDA graph captured on first use (all buffers and the cuFFT
// plan are fixed for the life of the context).  Returns without waiting.
int pcg_chunk_async(Ctx& c) {
  // no capture while profiling, nor on the legacy default stream
  if (c.profiling || c.stream == nullptr) return enqueue_chunk(c);
  if (!c.chunk_exec) {
    cudaGraph_t g = nullptr;
    int st = cuda_status(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal), &c, "capture");
    if (st) return st;
    int st_enq = enqueue_chunk(c);
    st = cuda_status(cudaStreamEndCapture(c.stream, &g), &c, "end capture");
    if (st_enq || st) {
      if (g) cudaGraphDestroy(g);
      return st_enq ? st_enq : st;
    }
    st = cuda_status(cudaGraphInstantiate(&c.chunk_exec, g, 0), &c, "instantiate");
    cudaGraphDestroy(g);
    if (st) {
      c.chunk_exec = nullptr;
      return st;
    }
  }
  return cuda_status(cudaGraphLaunch(c.chunk_exec, c.stream), &c, "graph launch");
}

// Builds the CG loop graph: a conditional WHILE node whose body is one
// iteration plus k_loop_cond.  Returns false (and leaves the chunked graph
// in charge) when the runtime refuses any step.
static bool build_loop_graph(Ctx& c) {
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
  bool ok = false;
  cudaGraphConditionalHandle handle;
  cudaGraphNodeParams p = {};
  cudaGraphNode_t node;
  if (cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault) == cudaSuccess) {
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    if (cudaGraphAddNode(&node, g, nullptr, 0, &p) == cudaSuccess) {
      cudaGraph_t body = p.conditional.phGraph_out[0];
      if (cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
          cudaSuccess) {
        int st = enqueue_iteration(c);
        if (!st) k_loop_cond<<<1, 32, 0, c.stream>>>(c.d_cg, handle, c.cfg.politer + 2);
        cudaGraph_t out = nullptr;
        const cudaError_t e = cudaStreamEndCapture(c.stream, &out);
        ok = !st && e == cudaSuccess && cudaGetLastError() == cudaSuccess;
      }
    }
  }
  if (ok) ok = cudaGraphInstantiate(&c.loop_exec, g, 0) == cudaSuccess;
  if (!ok) {
    c.loop_exec = nullptr;
    cudaGetLastError();  // clear a refused step so later status checks see only their own errors
  }
  cudaGraphDestroy(g);
  return ok;
}

// Runs the rest of the CG after pcg_begin on the device: one launch of the
// loop graph and the copy of the CG scalars to pinned host memory; returns
// without waiting.  -1 when the loop graph is not available.
int pcg_loop_async(Ctx& c) {
  if (!THP_DEVICE_LOOP || c.profiling || c.stream == nullptr) return -1;
  if (c.loop_state == 0) c.loop_state = build_loop_graph(c) ? 1 : -1;
  if (c.loop_state < 0) return -1;
  int st = cuda_status(cudaGraphLaunch(c.loop_exec, c.stream), &c, "loop graph launch");
  if (st) return st;
  return cuda_status(cudaMemcpyAsync(c.h_cg, c.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost, c.stream), &c,
                     "cg scalars");
}

int pcg_status(Ctx& c) {
  c.have_dipoles = true;
  if (c.h_cg->status) return c.h_cg->status;
  return c.h_cg->converged ? THP_OK : THP_E_NOT_CONVERGED;
}

// Runs the CG from the current d_ef; guess selects the start (see thp.h).
// The host reads the stop flag once per chunk of kCgChunk iterations; kernels
// after the stop return at entry.
// Like run_pcg, but with the device loop available it only enqueues the CG
// and the copy of its scalars (*pending = true); the caller synchronises and
// then reads pcg_status.
int run_pcg_async(Ctx& c, int guess, bool* pending) {
  *pending = false;
  int st = pcg_begin(c, guess);
  if (st) return st;
  st = pcg_loop_async(c);
  if (st >= 0) {
    *pending = st == THP_OK;
    return st;
  }
  int done = 0;
  while (true) {
    if ((st = pcg_chunk_async(c))) return st;
    done += kCgChunk;
    if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "cg sync"))) return st;
    if (c.h_cg->stop) break;
    if (done > c.cfg.politer + kCgChunk) break;  // defensive bound; stop is raised at politer
  }
  return THP_OK;
}

int run_pcg(Ctx& c, int guess) {
  int st = pcg_begin(c, guess);
  if (st) return st;
  st = pcg_loop_async(c);
  if (st >= 0) {
    if (st) return st;
    if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "cg sync"))) return st;
    return pcg_status(c);
  }
  int done = 0;
  while (true) {
    if ((st = pcg_chunk_async(c))) return st;
    done += kCgChunk;
    if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "cg sync"))) return st;
    if (c.h_cg->stop) break;
    if (done > c.cfg.politer + kCgChunk) break;  // defensive bound; stop is raised at politer
  }
  return pcg_status(c);
}

int launch_epol(Ctx& c) {
  const int nb = (c.n + kBlock - 1) / kBlock;
  if (overlapped(c) && c.mixed)
    k_epol<float><<<nb, kBlock, 0, c.stream>>>(c.n, c.d_mu, c.d_ef, c.d_resf, c.d_cg, c.d_partials);
  else
    k_epol<double><<<nb, kBlock, 0, c.stream>>>(c.n, c.d_mu, c.d_ef, c.d_res, c.d_cg, c.d_partials);
  return cuda_status(cudaGetLastError(), &c, "epol");
}

}  // namespace thp
