// batch.cu -- the CG iterations of many small systems as batched persistent
// kernels.
//
// inducepcg_pme2 (newinduce_pme2.f:285-636) for a batch of independent
// systems of uneven size.  The per-system form launches about nine kernels per
// CG iteration per system, each too small to fill the GPU; here one launch of
// each kernel serves every system.  A kernel walks its work list of
// (system, tile) items (the per-system queues laid end to end), each resident
// block taking items round-robin, and runs the same block-level code as the
// single-system kernels (cg_dev.cuh) on the item's system.  Per iteration:
//   1. kb_spread: pp = zr + beta pp (FP32 copy for the mixed rows) and the
//      dipole spread into grid A (grid_uind_site, pmestuff.f:280-405);
//   2. kb_dft x5: the convolution as DFTs along x, y, z of the small grids,
//      each line in two stages of short DFTs (the forward z pass, the
//      influence function and the inverse z pass fused), A -> B; the first
//      pass zeroes A behind it for the next spread;
//   3. kb_matvec: real-space rows, the dipole field gathered from B
//      (fphi_uind_site), h, pp.h and alpha;
//   4. kb_update: mu, residual, preconditioned residual, beta and the stop
//      test;
//   5. kb_cond: keeps the conditional WHILE node looping while a system runs.
// A system that has converged skips its items.  The whole loop is one CUDA
// graph.  The item tiles and the resident blocks per SM come from an online
// autotuner: the first solves of a plan each run one candidate, timed with
// events per CG iteration, and the fastest is kept (and remembered for plans
// of the same size class).
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "cg_dev.cuh"
#include "kernels.h"

namespace thp {

namespace {

using namespace cg;

// One system of the batch: its sizes and the device buffers its context owns
// (grid2, the DFT's output grid, belongs to the plan).
struct BatchSys {
  int n, nblk;  // atoms; blocks of kBlock atoms
  int nfft[3];
  int ngrid;
  int politer;
  double poleps, term;
  float interior;
  PairRows pr;
  Box box;
  PmeGeom g;
  const double4* pos;
  const float4* posf;
  const double* pol;
  const double* ef;
  double *mu, *res, *h, *zr, *pp;
  float *rec, *mpz;  // mixed form: 32-byte partner records of pp (PartnerRec)
  void* grid;   // A: the spread's target, the context's PME grid
  void* grid2;  // B: the convolved grid the matvec gathers from
  const void* qfac;
  CgScalars* cg;
  double* partials;
  const int* flags;  // the context's device error bits
};

// One system's results as the batch's last kernel leaves them in mapped host
// memory: the CG scalars (with Epol) and the device error bits.
struct BatchOut {
  CgScalars cg;
  int flags;
};

constexpr int kDftThreads = 256;
constexpr int kDftMaxN = 64;       // grid lengths the batched DFT takes
constexpr int kMaxLines = 32;      // lines per DFT tile
constexpr int kDftMaxOut = kMaxLines * kDftMaxN / kDftThreads;  // outputs per thread

// pp = zr + beta pp and the spread of the new pp (the work of k_spread_dip,
// mode 1); the mixed form also writes the 32-byte partner records its
// real-space rows read (wrapped FP32 position and the FP32 dipoles of pp).
template <bool MIXED>
__global__ void __launch_bounds__(kBlock) kb_spread(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                    int nitems) {
  using T = typename std::conditional<MIXED, float, double>::type;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;
    const int i = w.y * kBlock + threadIdx.x;
    if (i >= s.n) continue;
    double v[6], z[6];
    load6(s.pp + (size_t)i * 6, v);
    load6(s.zr + (size_t)i * 6, z);
    const double bd = s.cg->beta[0], bp = s.cg->beta[1];
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] = z[q] + (q < 3 ? bd : bp) * v[q];
    store6(s.pp + (size_t)i * 6, v);
    if (MIXED) {
      const float4 pf = s.posf[i];
      float4* r = reinterpret_cast<float4*>(s.rec + (size_t)i * 8);
      r[0] = make_float4(pf.x, pf.y, pf.z, (float)v[0]);
      r[1] = make_float4((float)v[1], (float)v[2], (float)v[3], (float)v[4]);
      s.mpz[i] = (float)v[5];
    }
    spread_dip_site<T>(s.g, s.pos[i], v, reinterpret_cast<typename Cplx<T>::type*>(s.grid));
  }
}

// Lines of one DFT pass: dimension d of the [n3][n2][n1] grid, line l of
// the lines_of(d) lines starts at line_base and steps by line_stride.
__device__ __forceinline__ int lines_of(const BatchSys& s, int d) { return s.ngrid / s.nfft[d]; }
__device__ __forceinline__ int line_stride(const BatchSys& s, int d) {
  return d == 0 ? 1 : (d == 1 ? s.nfft[0] : s.nfft[0] * s.nfft[1]);
}
__device__ __forceinline__ int line_base(const BatchSys& s, int d, int l) {
  if (d == 0) return l * s.nfft[0];
  if (d == 1) return (l / s.nfft[0]) * s.nfft[0] * s.nfft[1] + l % s.nfft[0];
  return l;
}

// Transforms of one line as two stages of short DFTs (Cooley-Tukey with
// N = N1 N2, n = N2 n1 + n2, k = k1 + N1 k2):
//   Y[k1 N2 + n2] = W^(n2 k1) sum_n1 x[N2 n1 + n2] W^(N2 n1 k1)
//   X[k1 + N1 k2] = sum_n2 Y[k1 N2 + n2] W^(N1 n2 k2)
// with W = exp(-2 pi i / N) forward (cuFFT's sign) and its conjugate
// inverse; N (N1 + N2) products per line instead of N^2.
template <typename T, typename C>
__device__ __forceinline__ C cmul(C a, C w, bool forward) {
  C r;
  if (forward) {
    r.x = a.x * w.x + a.y * w.y;
    r.y = a.y * w.x - a.x * w.y;
  } else {
    r.x = a.x * w.x - a.y * w.y;
    r.y = a.y * w.x + a.x * w.y;
  }
  return r;
}
template <typename T, typename C>
__device__ __forceinline__ C dft_stage1(const C* x, const C* tw, int N, int N1, int N2, int o, bool forward) {
  const int k1 = o / N2, n2 = o - k1 * N2;
  const int step = (N2 * k1) % N;
  T re = T(0), im = T(0);
  int m = 0;
  for (int n1 = 0; n1 < N1; ++n1) {
    const C v = cmul<T>(x[N2 * n1 + n2], tw[m], forward);
    re += v.x;
    im += v.y;
    m += step;
    if (m >= N) m -= N;
  }
  C r;
  r.x = re;
  r.y = im;
  return cmul<T>(r, tw[(n2 * k1) % N], forward);
}
template <typename T, typename C>
__device__ __forceinline__ C dft_stage2(const C* y, const C* tw, int N, int N1, int N2, int k, bool forward) {
  const int k2 = k / N1, k1 = k - k2 * N1;
  const int step = (N1 * k2) % N;
  const C* yk = y + k1 * N2;
  T re = T(0), im = T(0);
  int m = 0;
  for (int n2 = 0; n2 < N2; ++n2) {
    const C v = cmul<T>(yk[n2], tw[m], forward);
    re += v.x;
    im += v.y;
    m += step;
    if (m >= N) m -= N;
  }
  C r;
  r.x = re;
  r.y = im;
  return r;
}

// the larger factor pair N1 <= N2 of N with N1 as close to sqrt(N) as it gets
__device__ __forceinline__ int dft_split(int N) {
  int best = 1;
  for (int f = 2; f * f <= N; ++f)
    if (N % f == 0) best = f;
  return best;
}

// Position of element e of a tile of lt lines: x lines walk each line, y and
// z lines walk across lines first (neighbouring lines are neighbouring
// points of the grid).
__device__ __forceinline__ void tile_pos(int d, int e, int lt, int N, int& l, int& j) {
  if (d == 0) {
    l = e / N;
    j = e - l * N;
  } else {
    j = e / lt;
    l = e - j * lt;
  }
}

// One transform of every line of the tile held in buf (row pitch N + 1): the
// results end in the threads' out[] (element e = threadIdx.x + q blockDim.x).
template <typename T, typename C>
__device__ __forceinline__ void tile_dft(C* buf, const C* tw, int d, int lt, int N, int N1, int N2, bool forward,
                                         C (&out)[kDftMaxOut]) {
  const int ne = lt * N;
#pragma unroll
  for (int q = 0; q < kDftMaxOut; ++q) {
    const int e = threadIdx.x + q * kDftThreads;
    if (e < ne) {
      int l, o;
      tile_pos(d, e, lt, N, l, o);
      out[q] = dft_stage1<T>(buf + l * (N + 1), tw, N, N1, N2, o, forward);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kDftMaxOut; ++q) {
    const int e = threadIdx.x + q * kDftThreads;
    if (e < ne) {
      int l, o;
      tile_pos(d, e, lt, N, l, o);
      buf[l * (N + 1) + o] = out[q];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kDftMaxOut; ++q) {
    const int e = threadIdx.x + q * kDftThreads;
    if (e < ne) {
      int l, k;
      tile_pos(d, e, lt, N, l, k);
      out[q] = dft_stage2<T>(buf + l * (N + 1), tw, N, N1, N2, k, forward);
    }
  }
}

// One pass of the convolution over tiles of L lines (pass 0: x forward, A ->
// B with A zeroed; 1: y forward; 2: z forward, times qfac, z inverse; 3: y
// inverse; 4: x inverse; passes 1-4 on B).  Unnormalised transforms, as the
// single-system path's cuFFT C2C / Z2Z (fft_mpi.f90:65,115).
template <typename T>
__global__ void __launch_bounds__(kDftThreads) kb_dft(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                      int nitems, int pass, int L) {
  using C = typename Cplx<T>::type;
  extern __shared__ __align__(16) unsigned char dft_smem[];
  C* tw = reinterpret_cast<C*>(dft_smem);
  C* buf = tw + kDftMaxN;
  const int d = pass == 0 || pass == 4 ? 0 : (pass == 1 || pass == 3 ? 1 : 2);
  const bool forward = pass <= 2;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;  // the same for the whole block
    const int N = s.nfft[d], nl = lines_of(s, d), stride = line_stride(s, d);
    const int N1 = dft_split(N), N2 = N / N1;
    const int l0 = w.y * L;
    const int lt = min(L, nl - l0);
    const int ne = lt * N;
    C* src = reinterpret_cast<C*>(pass == 0 ? s.grid : s.grid2);
    C* dst = reinterpret_cast<C*>(s.grid2);
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
      double sn, cs;
      sincospi(2.0 * m / N, &sn, &cs);
      tw[m].x = (T)cs;
      tw[m].y = (T)sn;
    }
    for (int e = threadIdx.x; e < ne; e += blockDim.x) {
      int l, j;
      tile_pos(d, e, lt, N, l, j);
      const size_t gi = (size_t)line_base(s, d, l0 + l) + (size_t)j * stride;
      buf[l * (N + 1) + j] = src[gi];
      if (pass == 0) {
        C zero;
        zero.x = zero.y = T(0);
        src[gi] = zero;
      }
    }
    __syncthreads();
    C out[kDftMaxOut];
    tile_dft<T>(buf, tw, d, lt, N, N1, N2, forward, out);
    if (pass == 2) {
      // influence function on the transformed line, then the inverse z pass
      const T* qf = reinterpret_cast<const T*>(s.qfac);
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kDftMaxOut; ++q) {
        const int e = threadIdx.x + q * kDftThreads;
        if (e < ne) {
          int l, k;
          tile_pos(d, e, lt, N, l, k);
          const T f = qf[(size_t)line_base(s, d, l0 + l) + (size_t)k * stride];
          C v = out[q];
          v.x *= f;
          v.y *= f;
          buf[l * (N + 1) + k] = v;
        }
      }
      __syncthreads();
      tile_dft<T>(buf, tw, d, lt, N, N1, N2, false, out);
    }
#pragma unroll
    for (int q = 0; q < kDftMaxOut; ++q) {
      const int e = threadIdx.x + q * kDftThreads;
      if (e < ne) {
        int l, k;
        tile_pos(d, e, lt, N, l, k);
        dst[(size_t)line_base(s, d, l0 + l) + (size_t)k * stride] = out[q];
      }
    }
    __syncthreads();  // buf and tw are reused by the block's next item
  }
}

// real-space rows + dipole field gathered from B + h, pp.h, alpha
template <bool MIXED>
__global__ void __launch_bounds__(kBlock) kb_matvec(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                    int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;
    cg_matvec_block<MIXED, MIXED ? 1 : 2, MIXED>(w.y, s.nblk, s.pr, s.box, s.pos, s.posf, nullptr, s.g, s.grid2,
                                                 s.pp, nullptr, s.rec, s.mpz, s.pol, s.ef, s.term, 0, s.h, s.res,
                                                 s.zr, s.pp, s.cg, s.partials, s.interior);
  }
}

__global__ void __launch_bounds__(kBlock) kb_update(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                    int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;
    cg_update_block<double>(w.y, s.nblk, s.n, s.pol, s.ef, s.h, s.pp, s.mu, s.res, s.zr, s.cg, s.partials, s.poleps,
                            s.politer);
  }
}

// Epol of every system (the identity of k_epol: -1/2 electric sum
// uind . E_p) and each system's CG scalars and error bits written to mapped
// host memory by the system's last block, so one host synchronisation after
// the batch's graph sees every result.
__global__ void __launch_bounds__(kBlock) kb_finish(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                    int nitems, BatchOut* __restrict__ out) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    const int i = w.y * kBlock + threadIdx.x;
    double red[1] = {0.0};
    if (i < s.n) {
      const double* m = s.mu + (size_t)i * 6;
      const double* e = s.ef + (size_t)i * 6;
      red[0] = m[0] * e[3] + m[1] * e[4] + m[2] * e[5];
    }
    double tot[1];
    if (grid_reduce_of<1>(red, s.partials, &s.cg->counter[2], w.y, s.nblk, tot) && threadIdx.x == 0) {
      s.cg->epol = -0.5 * kElectric * tot[0];
      __threadfence();
      out[w.x].cg = *s.cg;
      out[w.x].flags = *s.flags;
    }
  }
}

// Last node of the loop body: loop while any system runs, and never more
// than max_loops bodies; on the way out every system is marked stopped.
__global__ void kb_cond(const BatchSys* __restrict__ sys, int count, unsigned* loops, int max_loops,
                        cudaGraphConditionalHandle handle) {
  const int lane = threadIdx.x;
  bool run = false;
  for (int q = lane; q < count; q += 32) run |= sys[q].cg->stop == 0;
  run = __any_sync(kFullMask, run);
  unsigned l = 0;
  if (lane == 0) l = ++*loops;
  l = __shfl_sync(kFullMask, l, 0);
  const bool keep = run && (int)l < max_loops;
  if (!keep)
    for (int q = lane; q < count; q += 32) sys[q].cg->stop = 1;
  if (lane == 0) cudaGraphSetConditional(handle, keep ? 1u : 0u);
}

// number of systems still running (the eager loop's host check)
__global__ void kb_running(const BatchSys* __restrict__ sys, int count, int* out) {
  int r = 0;
  for (int q = threadIdx.x; q < count; q += 32) r += sys[q].cg->stop == 0;
  for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(kFullMask, r, o);
  if (threadIdx.x == 0) *out = r;
}

// A grids of every system to zero (before the first spread of a solve)
template <typename T>
__global__ void kb_zero(const BatchSys* __restrict__ sys, int count, unsigned* loops) {
  using C = typename Cplx<T>::type;
  if (blockIdx.x == 0 && threadIdx.x == 0) *loops = 0;
  for (int q = 0; q < count; ++q) {
    C* g = reinterpret_cast<C*>(sys[q].grid);
    C zero;
    zero.x = zero.y = T(0);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < sys[q].ngrid; e += gridDim.x * blockDim.x) g[e] = zero;
  }
}

int sm_count(int device) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  return v > 0 ? v : 1;
}

}  // namespace

// Autotuner candidates: resident blocks per SM of the atom kernels (spread,
// matvec, update) and of the DFT passes, and lines per DFT tile.
struct BatchTune {
  int atom_blocks, dft_blocks, lines;
};
static const BatchTune kCandidates[] = {{4, 4, 32}, {8, 8, 32}, {16, 8, 32}, {8, 8, 16}, {16, 16, 16}, {4, 8, 16}};
constexpr int kNumCandidates = (int)(sizeof(kCandidates) / sizeof(kCandidates[0]));

// size class of a plan: precision, log2 of its atoms and of its systems
using TuneKey = std::tuple<int, int, int, int>;
static std::mutex g_tune_mu;
static std::map<TuneKey, int> g_tuned;

struct BatchPlan {
  int device = 0, mixed = 0, count = 0, sms = 1;
  int politer_max = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_loop = nullptr, ev_done = nullptr;
  BatchSys* d_sys = nullptr;
  int2* d_atom_items = nullptr;
  int n_atom_items = 0;
  int2* d_dft_items[2][3] = {};  // [lines 32 / 16][dimension]
  int n_dft_items[2][3] = {};
  void* d_grid2 = nullptr;
  unsigned* d_loops = nullptr;
  std::vector<int> sys_atoms;
  // the buffers each system's descriptor points at, checked before every
  // solve (a context re-targeted since the plan was made invalidates it)
  std::vector<std::tuple<int, const void*, const void*, const void*, const void*>> sig;
  cudaGraphExec_t exec[kNumCandidates] = {};
  float best_ms_per_it[kNumCandidates];
  int tried = 0;          // candidates measured so far (online tuning)
  int chosen = -1;        // the kept candidate
  int running = -1;       // candidate of the solve in flight
  TuneKey key;
  std::string msg;
  // profiling: the loop runs eagerly, one host-checked iteration at a time,
  // with events around each kernel (spread, five DFT passes, matvec, update)
  bool profiling = false;
  static constexpr int kKernels = 8;
  cudaEvent_t prof_ev[kKernels + 1] = {};
  double prof_ms[kKernels] = {};
  int prof_iterations = 0;
  int* h_running = nullptr;  // pinned
  int* d_running = nullptr;
  // whole-solve graphs (fronts, loop, results) per (guess, dipole carry,
  // candidate), and the mapped host records their last kernel writes
  std::map<std::tuple<int, int, int>, cudaGraphExec_t> solve_exec;
  BatchOut* h_out = nullptr;
  BatchOut* d_out = nullptr;
};

static int lines_index(int lines) { return lines == 32 ? 0 : 1; }

// One batched CG iteration; with events (profiling) each kernel is bracketed
// and no condition node is written.
static int enqueue_body(BatchPlan& p, const BatchTune& t, cudaGraphConditionalHandle handle, bool events = false) {
  const int ab = std::max(1, std::min(p.n_atom_items, t.atom_blocks * p.sms));
  int ke = 0;
  auto mark = [&]() {
    if (events) cudaEventRecord(p.prof_ev[ke++], p.stream);
  };
  mark();
  if (p.mixed)
    kb_spread<true><<<ab, kBlock, 0, p.stream>>>(p.d_sys, p.d_atom_items, p.n_atom_items);
  else
    kb_spread<false><<<ab, kBlock, 0, p.stream>>>(p.d_sys, p.d_atom_items, p.n_atom_items);
  const int li = lines_index(t.lines);
  const size_t csz = p.mixed ? sizeof(cufftComplex) : sizeof(cufftDoubleComplex);
  const size_t smem = csz * (kDftMaxN + (size_t)t.lines * (kDftMaxN + 1));
  for (int pass = 0; pass < 5; ++pass) {
    const int d = pass == 0 || pass == 4 ? 0 : (pass == 1 || pass == 3 ? 1 : 2);
    const int ni = p.n_dft_items[li][d];
    const int db = std::max(1, std::min(ni, t.dft_blocks * p.sms));
    mark();
    if (p.mixed)
      kb_dft<float><<<db, kDftThreads, smem, p.stream>>>(p.d_sys, p.d_dft_items[li][d], ni, pass, t.lines);
    else
      kb_dft<double><<<db, kDftThreads, smem, p.stream>>>(p.d_sys, p.d_dft_items[li][d], ni, pass, t.lines);
  }
  mark();
  if (p.mixed)
    kb_matvec<true><<<ab, kBlock, 0, p.stream>>>(p.d_sys, p.d_atom_items, p.n_atom_items);
  else
    kb_matvec<false><<<ab, kBlock, 0, p.stream>>>(p.d_sys, p.d_atom_items, p.n_atom_items);
  mark();
  kb_update<<<ab, kBlock, 0, p.stream>>>(p.d_sys, p.d_atom_items, p.n_atom_items);
  mark();
  if (!events) kb_cond<<<1, 32, 0, p.stream>>>(p.d_sys, p.count, p.d_loops, p.politer_max + 2, handle);
  return cudaGetLastError() == cudaSuccess ? THP_OK : THP_E_CUDA;
}

// Adds the loop of one candidate to g: a conditional WHILE node (after deps)
// whose body is one batched iteration.
static int add_loop_node(BatchPlan& p, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndeps, int cand,
                         cudaGraphNode_t* node) {
  cudaGraphConditionalHandle handle;
  if (cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) return THP_E_CUDA;
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = handle;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  if (cudaGraphAddNode(node, g, deps, ndeps, &np) != cudaSuccess) return THP_E_CUDA;
  cudaGraph_t body = np.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(p.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
      cudaSuccess)
    return THP_E_CUDA;
  const int se = enqueue_body(p, kCandidates[cand], handle);
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(p.stream, &out);
  return (!se && e == cudaSuccess) ? THP_OK : THP_E_CUDA;
}

// The loop graph of one candidate (the loop alone; the fronts run per system).
static int build_graph(BatchPlan& p, int cand) {
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return THP_E_CUDA;
  cudaGraphNode_t node;
  int st = add_loop_node(p, g, nullptr, 0, cand, &node);
  if (!st && cudaGraphInstantiate(&p.exec[cand], g, 0) != cudaSuccess) st = THP_E_CUDA;
  if (st) {
    p.exec[cand] = nullptr;
    p.msg = "batch: the loop graph could not be built";
    cudaGetLastError();
  }
  cudaGraphDestroy(g);
  return st;
}

void batch_plan_destroy(BatchPlan* p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  for (auto& e : p->exec)
    if (e) cudaGraphExecDestroy(e);
  for (auto& kv : p->solve_exec)
    if (kv.second) cudaGraphExecDestroy(kv.second);
  if (p->h_out) cudaFreeHost(p->h_out);
  cudaFree(p->d_sys);
  cudaFree(p->d_atom_items);
  for (auto& a : p->d_dft_items)
    for (auto& q : a) cudaFree(q);
  cudaFree(p->d_grid2);
  cudaFree(p->d_loops);
  for (auto& e : p->prof_ev)
    if (e) cudaEventDestroy(e);
  if (p->h_running) cudaFreeHost(p->h_running);
  cudaFree(p->d_running);
  if (p->ev_start) cudaEventDestroy(p->ev_start);
  if (p->ev_loop) cudaEventDestroy(p->ev_loop);
  if (p->ev_done) cudaEventDestroy(p->ev_done);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

static int log2i(long v) {
  int r = 0;
  while (v > 1) {
    v >>= 1;
    ++r;
  }
  return r;
}

int batch_plan_create(Ctx* const* cs, int count, BatchPlan** out, std::string* msg) {
  *out = nullptr;
  auto fail = [&](int st, const char* why) {
    if (msg) *msg = why;
    return st;
  };
  if (count <= 0) return fail(THP_E_INVALID, "batch: no systems");
  const Ctx& c0 = *cs[0];
  for (int q = 0; q < count; ++q) {
    const Ctx& c = *cs[q];
    if (c.device != c0.device || c.mixed != c0.mixed)
      return fail(THP_E_INVALID, "batch: systems on different devices or in different precisions");
    if (overlap_rows(c)) return fail(THP_E_INVALID, "batch: a system too large for the batched kernels");
    for (int d = 0; d < 3; ++d)
      if (c.cfg.nfft[d] > kDftMaxN) return fail(THP_E_INVALID, "batch: a PME grid longer than 64 points");
    if (!c.d_grid || !c.d_qfac || !c.d_pp) return fail(THP_E_STATE, "batch: a context without buffers");
  }
  BatchPlan* p = new BatchPlan();
  p->device = c0.device;
  p->mixed = c0.mixed;
  p->count = count;
  p->sms = sm_count(p->device);
  cudaSetDevice(p->device);
  int st = THP_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && !st) st = THP_E_CUDA;
    return e == cudaSuccess;
  };
  ok(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  ok(cudaEventCreate(&p->ev_start));
  ok(cudaEventCreate(&p->ev_loop));
  ok(cudaEventCreate(&p->ev_done));
  const size_t csz = p->mixed ? sizeof(cufftComplex) : sizeof(cufftDoubleComplex);
  size_t grid_total = 0;
  long atoms = 0;
  for (int q = 0; q < count; ++q) {
    grid_total += cs[q]->ngrid;
    atoms += cs[q]->n;
  }
  ok(cudaMalloc(&p->d_grid2, grid_total * csz));
  ok(cudaMalloc(&p->d_loops, sizeof(unsigned)));
  if (ok(cudaHostAlloc((void**)&p->h_out, sizeof(BatchOut) * count, cudaHostAllocMapped)))
    ok(cudaHostGetDevicePointer((void**)&p->d_out, p->h_out, 0));
  std::vector<BatchSys> hs(count);
  std::vector<int2> atom_items;
  std::vector<int2> dft_items[2][3];
  size_t goff = 0;
  // large systems first, so the round-robin ends on small items
  std::vector<int> order(count);
  for (int q = 0; q < count; ++q) order[q] = q;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cs[a]->n > cs[b]->n; });
  for (int q = 0; q < count; ++q) {
    Ctx& c = *cs[q];
    BatchSys& s = hs[q];
    s.n = c.n;
    s.nblk = (c.n + kBlock - 1) / kBlock;
    for (int d = 0; d < 3; ++d) s.nfft[d] = c.cfg.nfft[d];
    s.ngrid = (int)c.ngrid;
    s.politer = c.cfg.politer;
    s.poleps = c.cfg.poleps;
    const double a = c.cfg.aewald;
    s.term = (4.0 / 3.0) * a * a * a / kSqrtPi;
    s.interior = row_interior(c);
    s.pr = pair_rows(c);
    s.box = c.box;
    s.g = pme_geom(c);
    s.pos = c.d_pos;
    s.posf = c.d_posf;
    s.pol = c.d_pol;
    s.ef = c.d_ef;
    s.mu = c.d_mu;
    s.res = c.d_res;
    s.h = c.d_h;
    s.zr = c.d_zr;
    s.pp = c.d_pp;
    s.rec = c.d_rec;
    s.mpz = c.d_mpz;
    s.grid = c.d_grid;
    s.grid2 = static_cast<char*>(p->d_grid2) + goff * csz;
    goff += c.ngrid;
    s.qfac = c.d_qfac;
    s.cg = c.d_cg;
    s.partials = c.d_partials;
    s.flags = c.d_flags;
    p->politer_max = std::max(p->politer_max, c.cfg.politer);
    p->sys_atoms.push_back(c.n);
    p->sig.emplace_back(c.n, c.d_pp, c.d_grid, c.d_pk, c.d_cg);
  }
  for (int q : order) {
    for (int b = 0; b < hs[q].nblk; ++b) atom_items.push_back(make_int2(q, b));
    for (int li = 0; li < 2; ++li)
      for (int d = 0; d < 3; ++d) {
        const int L = li == 0 ? 32 : 16;
        const int nl = hs[q].ngrid / hs[q].nfft[d];
        for (int t = 0; t * L < nl; ++t) dft_items[li][d].push_back(make_int2(q, t));
      }
  }
  ok(cudaMalloc(&p->d_sys, sizeof(BatchSys) * count));
  ok(cudaMemcpy(p->d_sys, hs.data(), sizeof(BatchSys) * count, cudaMemcpyHostToDevice));
  p->n_atom_items = (int)atom_items.size();
  ok(cudaMalloc(&p->d_atom_items, sizeof(int2) * atom_items.size()));
  ok(cudaMemcpy(p->d_atom_items, atom_items.data(), sizeof(int2) * atom_items.size(), cudaMemcpyHostToDevice));
  for (int li = 0; li < 2; ++li)
    for (int d = 0; d < 3; ++d) {
      const auto& v = dft_items[li][d];
      p->n_dft_items[li][d] = (int)v.size();
      ok(cudaMalloc(&p->d_dft_items[li][d], sizeof(int2) * std::max<size_t>(1, v.size())));
      ok(cudaMemcpy(p->d_dft_items[li][d], v.data(), sizeof(int2) * v.size(), cudaMemcpyHostToDevice));
    }
  p->key = TuneKey(p->mixed, log2i(atoms), log2i(count), 0);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto f = g_tuned.find(p->key);
    if (f != g_tuned.end()) p->chosen = f->second;
  }
  for (auto& m : p->best_ms_per_it) m = 1e30f;
  if (st) {
    if (msg) *msg = "batch: device allocation or copy failed";
    batch_plan_destroy(p);
    return st;
  }
  *out = p;
  return THP_OK;
}

// Enqueues the batched CG loop on the plan's stream after every system's
// front (the callers' streams wait for ev_done).  Returns without waiting.
int batch_plan_check(const BatchPlan& p, Ctx* const* cs) {
  for (int q = 0; q < p.count; ++q) {
    const Ctx& c = *cs[q];
    if (p.sig[q] != std::make_tuple(c.n, (const void*)c.d_pp, (const void*)c.d_grid, (const void*)c.d_pk,
                                    (const void*)c.d_cg))
      return THP_E_STATE;
  }
  return THP_OK;
}

int batch_plan_loop(BatchPlan& p, Ctx* const* cs) {
  cudaSetDevice(p.device);
  const int cand = p.chosen >= 0 ? p.chosen : p.tried;
  if (!p.exec[cand] && !p.profiling) {
    int st = build_graph(p, cand);
    if (st) return st;
  }
  for (int q = 0; q < p.count; ++q) {
    cudaEventRecord(cs[q]->ev_fork, cs[q]->stream);
    cudaStreamWaitEvent(p.stream, cs[q]->ev_fork, 0);
  }
  if (p.mixed)
    kb_zero<float><<<2 * p.sms, 256, 0, p.stream>>>(p.d_sys, p.count, p.d_loops);
  else
    kb_zero<double><<<2 * p.sms, 256, 0, p.stream>>>(p.d_sys, p.count, p.d_loops);
  cudaEventRecord(p.ev_start, p.stream);
  if (p.profiling) {
    // eager iterations with a host check of the running systems after each
    const BatchTune& t = kCandidates[cand];
    for (int it = 0; it < p.politer_max + 2; ++it) {
      if (enqueue_body(p, t, cudaGraphConditionalHandle{}, true)) return THP_E_CUDA;
      kb_running<<<1, 32, 0, p.stream>>>(p.d_sys, p.count, p.d_running);
      cudaMemcpyAsync(p.h_running, p.d_running, sizeof(int), cudaMemcpyDeviceToHost, p.stream);
      if (cudaStreamSynchronize(p.stream) != cudaSuccess) return THP_E_CUDA;
      for (int k = 0; k < BatchPlan::kKernels; ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.prof_ev[k], p.prof_ev[k + 1]);
        p.prof_ms[k] += ms;
      }
      ++p.prof_iterations;
      if (*p.h_running == 0) break;
    }
  } else {
    cudaGraphLaunch(p.exec[cand], p.stream);
  }
  cudaEventRecord(p.ev_loop, p.stream);
  cudaEventRecord(p.ev_done, p.stream);
  p.running = cand;
  for (int q = 0; q < p.count; ++q) cudaStreamWaitEvent(cs[q]->stream, p.ev_done, 0);
  return cudaGetLastError() == cudaSuccess ? THP_OK : THP_E_CUDA;
}

// After the systems' streams have synchronised: the loop's time per CG
// iteration (the loop runs as long as the slowest system) feeds the tuner.
void batch_plan_finish(BatchPlan& p, int max_iterations) {
  if (p.chosen >= 0 || p.running < 0 || p.profiling) return;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, p.ev_start, p.ev_loop) != cudaSuccess) return;
  const float per_it = ms / (float)std::max(1, max_iterations);
  float& best = p.best_ms_per_it[p.running];
  best = std::min(best, per_it);
  p.running = -1;
  if (++p.tried < kNumCandidates) return;
  int arg = 0;
  for (int q = 1; q < kNumCandidates; ++q)
    if (p.best_ms_per_it[q] < p.best_ms_per_it[arg]) arg = q;
  p.chosen = arg;
  for (int q = 0; q < kNumCandidates; ++q)
    if (q != arg && p.exec[q]) {
      cudaGraphExecDestroy(p.exec[q]);
      p.exec[q] = nullptr;
    }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[p.key] = arg;
}

int batch_plan_tuning(const BatchPlan& p, int* atom_blocks, int* dft_blocks, int* lines, float* ms_per_iteration) {
  const int c = p.chosen;
  if (c < 0) return THP_E_STATE;
  *atom_blocks = kCandidates[c].atom_blocks;
  *dft_blocks = kCandidates[c].dft_blocks;
  *lines = kCandidates[c].lines;
  *ms_per_iteration = p.best_ms_per_it[c] < 1e29f ? p.best_ms_per_it[c] : -1.f;
  return THP_OK;
}

int batch_plan_candidates() { return kNumCandidates; }

int batch_plan_candidate(const BatchPlan& p) { return p.chosen >= 0 ? p.chosen : p.tried; }

bool batch_plan_profiling(const BatchPlan& p) { return p.profiling; }

cudaGraphExec_t batch_plan_solve_exec(const BatchPlan& p, int guess, int carry, int cand) {
  auto f = p.solve_exec.find(std::make_tuple(guess, carry, cand));
  return f == p.solve_exec.end() ? nullptr : f->second;
}

// The whole batched solve as one graph: every system's front (child graphs,
// in parallel), the zeroing of the A grids, the loop of candidate cand, and
// kb_finish.  fronts[q] are the captured fronts (copied into the graph).
int batch_plan_make_solve_exec(BatchPlan& p, const std::vector<cudaGraph_t>& fronts, int guess, int carry, int cand) {
  cudaSetDevice(p.device);
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return THP_E_CUDA;
  int st = THP_OK;
  std::vector<cudaGraphNode_t> fn(fronts.size());
  for (size_t q = 0; q < fronts.size() && !st; ++q)
    if (cudaGraphAddChildGraphNode(&fn[q], g, nullptr, 0, fronts[q]) != cudaSuccess) st = THP_E_CUDA;
  cudaGraphNode_t zero = nullptr, loop = nullptr, fin = nullptr;
  if (!st) {
    cudaKernelNodeParams kp = {};
    void* args[] = {&p.d_sys, &p.count, &p.d_loops};
    kp.func = p.mixed ? (void*)kb_zero<float> : (void*)kb_zero<double>;
    kp.gridDim = dim3(2 * p.sms);
    kp.blockDim = dim3(256);
    kp.kernelParams = args;
    if (cudaGraphAddKernelNode(&zero, g, fn.data(), fn.size(), &kp) != cudaSuccess) st = THP_E_CUDA;
  }
  if (!st) st = add_loop_node(p, g, &zero, 1, cand, &loop);
  if (!st) {
    cudaKernelNodeParams kp = {};
    void* args[] = {&p.d_sys, &p.d_atom_items, &p.n_atom_items, &p.d_out};
    kp.func = (void*)kb_finish;
    kp.gridDim = dim3(std::max(1, std::min(p.n_atom_items, 8 * p.sms)));
    kp.blockDim = dim3(kBlock);
    kp.kernelParams = args;
    if (cudaGraphAddKernelNode(&fin, g, &loop, 1, &kp) != cudaSuccess) st = THP_E_CUDA;
  }
  cudaGraphExec_t ex = nullptr;
  if (!st && cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) st = THP_E_CUDA;
  cudaGraphDestroy(g);
  if (st) {
    cudaGetLastError();
    return st;
  }
  p.solve_exec[std::make_tuple(guess, carry, cand)] = ex;
  return THP_OK;
}

// Launches a whole-solve graph and waits for it; the records of every system
// are then in out (mapped host memory, count entries).
int batch_plan_run_solve(BatchPlan& p, cudaGraphExec_t ex, const CgScalars** cg_out, const int** flags_out,
                         float* ms) {
  cudaSetDevice(p.device);
  const int cand = batch_plan_candidate(p);
  cudaEventRecord(p.ev_start, p.stream);
  if (cudaGraphLaunch(ex, p.stream) != cudaSuccess) return THP_E_CUDA;
  cudaEventRecord(p.ev_loop, p.stream);
  if (cudaStreamSynchronize(p.stream) != cudaSuccess) return THP_E_CUDA;
  p.running = cand;
  cudaEventElapsedTime(ms, p.ev_start, p.ev_loop);
  for (int q = 0; q < p.count; ++q) {
    cg_out[q] = &p.h_out[q].cg;
    flags_out[q] = &p.h_out[q].flags;
  }
  return THP_OK;
}

int batch_plan_profile(BatchPlan& p, int enable, double* ms, int* iterations) {
  cudaSetDevice(p.device);
  if (ms)
    for (int k = 0; k < BatchPlan::kKernels; ++k) ms[k] = p.prof_ms[k];
  if (iterations) *iterations = p.prof_iterations;
  if (enable < 0) return THP_OK;  // read only
  if (enable && !p.prof_ev[0]) {
    for (auto& e : p.prof_ev)
      if (cudaEventCreate(&e) != cudaSuccess) return THP_E_CUDA;
    if (cudaMallocHost(&p.h_running, sizeof(int)) != cudaSuccess) return THP_E_CUDA;
    if (cudaMalloc(&p.d_running, sizeof(int)) != cudaSuccess) return THP_E_CUDA;
  }
  p.profiling = enable != 0;
  for (auto& m : p.prof_ms) m = 0.0;
  p.prof_iterations = 0;
  return THP_OK;
}

}  // namespace thp
