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
//   1. kb_spread: pp = zr + beta pp (the 32-byte partner records of the mixed
//      rows beside it) and the dipole spread (grid_uind_site,
//      pmestuff.f:280-405) into the plan's grids, zeroed just before;
//   2. the convolution: one batched cuFFT transform per grid-size class (the
//      classes' grids lie end to end, and the classes run as parallel
//      branches), kb_qfac over every grid, the batched inverse transforms;
//   3. kb_row: real-space rows (tmatxb_pme); kb_combine: the dipole field
//      gathered from the grid (fphi_uind_site), h, pp.h and alpha;
//   4. kb_update: mu, residual, preconditioned residual, beta and the stop
//      test;
//   5. kb_cond: keeps the conditional WHILE node looping while a system runs.
// A system that has converged skips its items.  The whole loop is one CUDA
// graph, and the whole solve (every system's front as a child graph, the
// loop, Epol and the results written to mapped host memory) another.  The
// resident blocks per SM and the matvec's tile come from an online
// autotuner: the first solves of a plan each run one candidate, timed with
// events, and the fastest is kept (and remembered for plans of the same size
// class).
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
// (grid, its PME grid in the batched transforms' layout, belongs to the plan).
struct BatchSys {
  int n, nblk;       // atoms; blocks of kBlock atoms
  int nblk_mv[2];    // blocks of 16 and 32 atoms (the rows' items)
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
  void* grid;  // the system's grid in the plan's class-ordered grid array
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

// pp = zr + beta pp and the spread of the new pp (the work of k_spread_dip,
// mode 1); the mixed form also writes the 32-byte partner records its
// real-space rows read (wrapped FP32 position and the FP32 dipoles of pp).
// TILE: each warp sums the stencils of its sites in a shared-memory tile
// before adding them to the grid (spread_dip_warp; one SpreadWarp<T> per warp
// in dynamic shared memory); otherwise every site adds its own stencil.  The
// FP64 form uses the tile (64 boxes of 300-6,000 atoms: 157 -> 118 us per
// batched spread); the mixed form does not (59 -> 68 us: in boxes this small
// fewer warps' stencils fit one tile, and the tile's shared memory costs
// occupancy).
#ifndef THP_BATCH_SPREAD_TILE_F64
#define THP_BATCH_SPREAD_TILE_F64 1
#endif
#ifndef THP_BATCH_SPREAD_TILE_F32
#define THP_BATCH_SPREAD_TILE_F32 0
#endif
template <bool MIXED, bool TILE>
__global__ void __launch_bounds__(kBlock) kb_spread(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                    int nitems) {
  using T = typename std::conditional<MIXED, float, double>::type;
  SpreadWarp<T>* sw = nullptr;
  if constexpr (TILE) {
    extern __shared__ __align__(16) unsigned char spread_smem[];
    sw = reinterpret_cast<SpreadWarp<T>*>(spread_smem) + (threadIdx.x >> 5);
    for (int q = threadIdx.x & 31; q < SpreadWarp<T>::kPts; q += 32) sw->tile[q] = {T(0), T(0)};
  }
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;
    const int i = w.y * kBlock + threadIdx.x;
    const bool live = i < s.n;
    if (!TILE && !live) continue;
    double v[6] = {0, 0, 0, 0, 0, 0};
    double4 pi = make_double4(0, 0, 0, 0);
    if (live) {
      double z[6];
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
      pi = s.pos[i];
    }
    auto* grid = reinterpret_cast<typename Cplx<T>::type*>(s.grid);
    if constexpr (TILE)
      spread_dip_warp<T>(s.g, pi, v, live, grid, *sw);
    else
      spread_dip_site<T>(s.g, pi, v, grid);
  }
}

template <bool MIXED>
static void launch_kb_spread(cudaStream_t st, const BatchSys* sys, const int2* items, int nitems, int blocks) {
  if (MIXED ? THP_BATCH_SPREAD_TILE_F32 : THP_BATCH_SPREAD_TILE_F64) {
    using T = typename std::conditional<MIXED, float, double>::type;
    constexpr size_t smem = sizeof(SpreadWarp<T>) * (kBlock / 32);
    static std::atomic<unsigned long long> limit_set{0};
    smem_limit_once(kb_spread<MIXED, true>, smem, limit_set);
    kb_spread<MIXED, true><<<blocks, kBlock, smem, st>>>(sys, items, nitems);
  } else {
    kb_spread<MIXED, false><<<blocks, kBlock, 0, st>>>(sys, items, nitems);
  }
}

// The influence function on every running system's transformed grid; items
// (system, chunk of kQfacChunk points).
constexpr int kQfacChunk = 2048;
template <typename T>
__global__ void __launch_bounds__(256) kb_qfac(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                               int nitems) {
  using C = typename Cplx<T>::type;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;
    C* g = reinterpret_cast<C*>(s.grid);
    const T* f = reinterpret_cast<const T*>(s.qfac);
    const int e1 = min(s.ngrid, (w.y + 1) * kQfacChunk);
    for (int e = w.y * kQfacChunk + threadIdx.x; e < e1; e += blockDim.x) {
      C v = g[e];
      const T q = f[e];
      v.x *= q;
      v.y *= q;
      g[e] = v;
    }
  }
}

// real-space rows T_real pp into h (FP64); items of 16 GPW atoms
template <bool MIXED, int GPW>
__global__ void __launch_bounds__(kBlock) kb_row(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                 int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;
    row_block<MIXED, MIXED, GPW>(w.y, s.pr, s.box, s.pos, s.posf, s.pp, nullptr, s.rec, s.mpz, s.interior, s.h);
  }
}

// h = T_real pp + pp/alpha + dipfield(pp) - self term, the dipole field
// gathered from the convolved grid (fphi_uind_site), pp.h and alpha
template <bool MIXED>
__global__ void __launch_bounds__(kBlock) kb_combine(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                     int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;
    cg_combine_block<MIXED ? 1 : 2, double, double>(w.y, s.nblk, s.n, nullptr, s.g, s.pos, s.grid, s.pp, s.pol,
                                                    s.ef, s.term, 0, s.h, s.res, s.zr, s.pp, s.cg, s.partials);
  }
}

__global__ void __launch_bounds__(kBlock) kb_update(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                    int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    if (s.cg->stop) continue;
    cg_update_block<double>(w.y, s.nblk, s.n, s.pol, s.h, s.pp, s.mu, s.res, s.zr, s.cg, s.partials, s.poleps,
                            s.politer);
  }
}

// Epol of every system (the identity of k_epol: -1/2 electric sum
// uind . E_p), its CG energy ene, and each system's CG scalars and error bits written to mapped
// host memory by the system's last block, so one host synchronisation after
// the batch's graph sees every result.
__global__ void __launch_bounds__(kBlock) kb_finish(const BatchSys* __restrict__ sys, const int2* __restrict__ items,
                                                    int nitems, BatchOut* __restrict__ out) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const BatchSys& s = sys[w.x];
    const int i = w.y * kBlock + threadIdx.x;
    double red[3] = {0.0, 0.0, 0.0};
    if (i < s.n) {
      double m[6], e[6], r[6];
      load6(s.mu + (size_t)i * 6, m);
      load6(s.ef + (size_t)i * 6, e);
      load6(s.res + (size_t)i * 6, r);
      red[0] = m[0] * e[3] + m[1] * e[4] + m[2] * e[5];
#pragma unroll
      for (int q = 0; q < 6; ++q) red[q < 3 ? 1 : 2] -= 0.5 * (m[q] * (r[q] + e[q]));
    }
    double tot[3];
    if (grid_reduce_of<3>(red, s.partials, &s.cg->counter[2], w.y, s.nblk, tot) && threadIdx.x == 0) {
      s.cg->epol = -0.5 * kElectric * tot[0];
      s.cg->ene[0] = tot[1];
      s.cg->ene[1] = tot[2];
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

// the loop counter of kb_cond, before each solve's loop
__global__ void kb_reset(unsigned* loops) { *loops = 0; }

int sm_count(int device) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  return v > 0 ? v : 1;
}

}  // namespace

// Autotuner candidates: resident blocks per SM of the batched kernels and
// groups of four atoms per warp in the real-space rows (tiles of 16 GPW
// atoms).
struct BatchTune {
  int blocks, gpw;
};
static const BatchTune kCandidates[] = {{4, 2}, {8, 2}, {16, 2}, {4, 1}, {8, 1}, {16, 1}};
constexpr int kNumCandidates = (int)(sizeof(kCandidates) / sizeof(kCandidates[0]));

// size class of a plan: precision, log2 of its atoms and of its systems
using TuneKey = std::tuple<int, int, int>;
static std::mutex g_tune_mu;
static std::map<TuneKey, int> g_tuned;

// The systems of one grid shape: their grids lie end to end in the plan's
// grid array and one batched cuFFT plan transforms them all, on a stream of
// its own (a parallel branch of the graph).
struct FftClass {
  int n[3] = {0, 0, 0};
  int count = 0;
  size_t offset = 0;  // first grid point of the class in the plan's array
  cufftHandle plan = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

struct BatchPlan {
  int device = 0, mixed = 0, count = 0, sms = 1;
  int politer_max = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_loop = nullptr, ev_done = nullptr, ev_fork = nullptr;
  BatchSys* d_sys = nullptr;
  int2* d_atom_items = nullptr;  // (system, block of kBlock atoms)
  int n_atom_items = 0;
  int2* d_mv_items[2] = {};      // (system, block of 16 / 32 atoms): the rows' items
  int n_mv_items[2] = {};
  int2* d_qfac_items = nullptr;  // (system, chunk of grid points)
  int n_qfac_items = 0;
  void* d_grid = nullptr;        // every system's grid, class by class
  size_t grid_bytes = 0;
  std::vector<FftClass> classes;
  unsigned* d_loops = nullptr;
  // the buffers each system's descriptor points at, checked before every
  // solve (a context re-targeted since the plan was made invalidates it)
  std::vector<std::tuple<int, const void*, const void*, const void*>> sig;
  cudaGraphExec_t exec[kNumCandidates] = {};
  float best_ms[kNumCandidates];
  int tried = 0;    // candidates measured so far (online tuning)
  int chosen = -1;  // the kept candidate
  int running = -1; // candidate of the solve in flight
  TuneKey key;
  // profiling: the loop runs eagerly, one host-checked iteration at a time,
  // with events around each step (spread, forward FFTs, qfac, inverse FFTs,
  // matvec, update)
  bool profiling = false;
  static constexpr int kKernels = 6;
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

// Every class's batched transform in one direction, as parallel branches.
static int enqueue_ffts(BatchPlan& p, int dir) {
  cudaEventRecord(p.ev_fork, p.stream);
  for (FftClass& k : p.classes) {
    cudaStreamWaitEvent(k.stream, p.ev_fork, 0);
    cufftResult r;
    if (p.mixed) {
      cufftComplex* g = static_cast<cufftComplex*>(p.d_grid) + k.offset;
      r = cufftExecC2C(k.plan, g, g, dir);
    } else {
      cufftDoubleComplex* g = static_cast<cufftDoubleComplex*>(p.d_grid) + k.offset;
      r = cufftExecZ2Z(k.plan, g, g, dir);
    }
    if (r != CUFFT_SUCCESS) return THP_E_CUDA;
    cudaEventRecord(k.done, k.stream);
    cudaStreamWaitEvent(p.stream, k.done, 0);
  }
  return THP_OK;
}

// One batched CG iteration; with events (profiling) each step is bracketed
// and no condition node is written.
static int enqueue_body(BatchPlan& p, const BatchTune& t, cudaGraphConditionalHandle handle, bool events = false) {
  const int ab = std::max(1, std::min(p.n_atom_items, t.blocks * p.sms));
  int ke = 0;
  auto mark = [&]() {
    if (events) cudaEventRecord(p.prof_ev[ke++], p.stream);
  };
  mark();
  cudaMemsetAsync(p.d_grid, 0, p.grid_bytes, p.stream);
  if (p.mixed)
    launch_kb_spread<true>(p.stream, p.d_sys, p.d_atom_items, p.n_atom_items, ab);
  else
    launch_kb_spread<false>(p.stream, p.d_sys, p.d_atom_items, p.n_atom_items, ab);
  mark();
  if (enqueue_ffts(p, CUFFT_FORWARD)) return THP_E_CUDA;
  mark();
  const int qb = std::max(1, std::min(p.n_qfac_items, 8 * p.sms));
  if (p.mixed)
    kb_qfac<float><<<qb, 256, 0, p.stream>>>(p.d_sys, p.d_qfac_items, p.n_qfac_items);
  else
    kb_qfac<double><<<qb, 256, 0, p.stream>>>(p.d_sys, p.d_qfac_items, p.n_qfac_items);
  mark();
  if (enqueue_ffts(p, CUFFT_INVERSE)) return THP_E_CUDA;
  mark();
  const int g = t.gpw - 1;
  const int mb = std::max(1, std::min(p.n_mv_items[g], 2 * t.blocks * p.sms));
  if (p.mixed) {
    if (t.gpw == 1)
      kb_row<true, 1><<<mb, kBlock, 0, p.stream>>>(p.d_sys, p.d_mv_items[g], p.n_mv_items[g]);
    else
      kb_row<true, 2><<<mb, kBlock, 0, p.stream>>>(p.d_sys, p.d_mv_items[g], p.n_mv_items[g]);
    kb_combine<true><<<ab, kBlock, 0, p.stream>>>(p.d_sys, p.d_atom_items, p.n_atom_items);
  } else {
    if (t.gpw == 1)
      kb_row<false, 1><<<mb, kBlock, 0, p.stream>>>(p.d_sys, p.d_mv_items[g], p.n_mv_items[g]);
    else
      kb_row<false, 2><<<mb, kBlock, 0, p.stream>>>(p.d_sys, p.d_mv_items[g], p.n_mv_items[g]);
    kb_combine<false><<<ab, kBlock, 0, p.stream>>>(p.d_sys, p.d_atom_items, p.n_atom_items);
  }
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
  for (FftClass& k : p->classes) {
    if (k.plan) cufftDestroy(k.plan);
    if (k.stream) cudaStreamDestroy(k.stream);
    if (k.done) cudaEventDestroy(k.done);
  }
  if (p->h_out) cudaFreeHost(p->h_out);
  cudaFree(p->d_sys);
  cudaFree(p->d_atom_items);
  for (auto& m : p->d_mv_items) cudaFree(m);
  cudaFree(p->d_qfac_items);
  cudaFree(p->d_grid);
  cudaFree(p->d_loops);
  for (auto& e : p->prof_ev)
    if (e) cudaEventDestroy(e);
  if (p->h_running) cudaFreeHost(p->h_running);
  cudaFree(p->d_running);
  for (cudaEvent_t e : {p->ev_start, p->ev_loop, p->ev_done, p->ev_fork})
    if (e) cudaEventDestroy(e);
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
  for (cudaEvent_t* e : {&p->ev_start, &p->ev_loop, &p->ev_done}) ok(cudaEventCreate(e));
  ok(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
  const size_t csz = p->mixed ? sizeof(cufftComplex) : sizeof(cufftDoubleComplex);
  long atoms = 0;
  for (int q = 0; q < count; ++q) atoms += cs[q]->n;
  // grid-shape classes, in order of first appearance; each system's grid
  // goes to its class's run of the grid array
  std::vector<int> cls(count);
  for (int q = 0; q < count; ++q) {
    const int* n = cs[q]->cfg.nfft;
    int k = 0;
    while (k < (int)p->classes.size() &&
           !(p->classes[k].n[0] == n[0] && p->classes[k].n[1] == n[1] && p->classes[k].n[2] == n[2]))
      ++k;
    if (k == (int)p->classes.size()) {
      p->classes.emplace_back();
      for (int d = 0; d < 3; ++d) p->classes[k].n[d] = n[d];
    }
    cls[q] = k;
    ++p->classes[k].count;
  }
  // each system's grid starts on an even point (16-byte boundary of the FP32
  // grid, which the paired reductions and vector gathers need)
  auto slot = [](const FftClass& k) {
    const size_t pts = (size_t)k.n[0] * k.n[1] * k.n[2];
    return pts + (pts & 1);
  };
  size_t off = 0;
  for (FftClass& k : p->classes) {
    k.offset = off;
    off += (size_t)k.count * slot(k);
  }
  p->grid_bytes = off * csz;
  ok(cudaMalloc(&p->d_grid, p->grid_bytes));
  for (FftClass& k : p->classes) {
    const int dims[3] = {k.n[2], k.n[1], k.n[0]};
    const int dist = (int)slot(k);
    // the storage dimensions given, so that cuFFT honours the padded distance
    if (cufftPlanMany(&k.plan, 3, const_cast<int*>(dims), const_cast<int*>(dims), 1, dist,
                      const_cast<int*>(dims), 1, dist,
                      p->mixed ? CUFFT_C2C : CUFFT_Z2Z, k.count) != CUFFT_SUCCESS && !st)
      st = THP_E_CUDA;
    ok(cudaStreamCreateWithFlags(&k.stream, cudaStreamNonBlocking));
    ok(cudaEventCreateWithFlags(&k.done, cudaEventDisableTiming));
    if (k.plan) cufftSetStream(k.plan, k.stream);
  }
  ok(cudaMalloc(&p->d_loops, sizeof(unsigned)));
  if (ok(cudaHostAlloc((void**)&p->h_out, sizeof(BatchOut) * count, cudaHostAllocMapped)))
    ok(cudaHostGetDevicePointer((void**)&p->d_out, p->h_out, 0));
  std::vector<BatchSys> hs(count);
  std::vector<size_t> next(p->classes.size());
  for (size_t k = 0; k < p->classes.size(); ++k) next[k] = p->classes[k].offset;
  for (int q = 0; q < count; ++q) {
    Ctx& c = *cs[q];
    BatchSys& s = hs[q];
    s.n = c.n;
    s.nblk = (c.n + kBlock - 1) / kBlock;
    s.nblk_mv[0] = (c.n + 15) / 16;
    s.nblk_mv[1] = (c.n + 31) / 32;
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
    s.grid = static_cast<char*>(p->d_grid) + next[cls[q]] * csz;
    next[cls[q]] += slot(p->classes[cls[q]]);
    s.qfac = c.d_qfac;
    s.cg = c.d_cg;
    s.partials = c.d_partials;
    s.flags = c.d_flags;
    p->politer_max = std::max(p->politer_max, c.cfg.politer);
    p->sig.emplace_back(c.n, c.d_pp, c.d_pk, c.d_cg);
  }
  // work lists, large systems first so the round-robin ends on small items
  std::vector<int> order(count);
  for (int q = 0; q < count; ++q) order[q] = q;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cs[a]->n > cs[b]->n; });
  std::vector<int2> atom_items, mv_items[2], qfac_items;
  for (int q : order) {
    for (int b = 0; b * kQfacChunk < hs[q].ngrid; ++b) qfac_items.push_back(make_int2(q, b));
    for (int b = 0; b < hs[q].nblk; ++b) atom_items.push_back(make_int2(q, b));
    for (int g = 0; g < 2; ++g)
      for (int b = 0; b < hs[q].nblk_mv[g]; ++b) mv_items[g].push_back(make_int2(q, b));
  }
  ok(cudaMalloc(&p->d_sys, sizeof(BatchSys) * count));
  ok(cudaMemcpy(p->d_sys, hs.data(), sizeof(BatchSys) * count, cudaMemcpyHostToDevice));
  p->n_atom_items = (int)atom_items.size();
  ok(cudaMalloc(&p->d_atom_items, sizeof(int2) * atom_items.size()));
  ok(cudaMemcpy(p->d_atom_items, atom_items.data(), sizeof(int2) * atom_items.size(), cudaMemcpyHostToDevice));
  p->n_qfac_items = (int)qfac_items.size();
  ok(cudaMalloc(&p->d_qfac_items, sizeof(int2) * qfac_items.size()));
  ok(cudaMemcpy(p->d_qfac_items, qfac_items.data(), sizeof(int2) * qfac_items.size(), cudaMemcpyHostToDevice));
  for (int g = 0; g < 2; ++g) {
    p->n_mv_items[g] = (int)mv_items[g].size();
    ok(cudaMalloc(&p->d_mv_items[g], sizeof(int2) * mv_items[g].size()));
    ok(cudaMemcpy(p->d_mv_items[g], mv_items[g].data(), sizeof(int2) * mv_items[g].size(), cudaMemcpyHostToDevice));
  }
  p->key = TuneKey(p->mixed, log2i(atoms), log2i(count));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto f = g_tuned.find(p->key);
    if (f != g_tuned.end()) p->chosen = f->second;
  }
  for (auto& m : p->best_ms) m = 1e30f;
  if (st) {
    if (msg) *msg = "batch: device allocation, copy or FFT plan failed";
    batch_plan_destroy(p);
    return st;
  }
  *out = p;
  return THP_OK;
}

int batch_plan_check(const BatchPlan& p, Ctx* const* cs) {
  for (int q = 0; q < p.count; ++q) {
    const Ctx& c = *cs[q];
    if (p.sig[q] != std::make_tuple(c.n, (const void*)c.d_pp, (const void*)c.d_pk, (const void*)c.d_cg))
      return THP_E_STATE;
  }
  return THP_OK;
}

int batch_plan_candidate(const BatchPlan& p) { return p.chosen >= 0 ? p.chosen : p.tried; }

bool batch_plan_profiling(const BatchPlan& p) { return p.profiling; }

// Enqueues the batched CG loop on the plan's stream after every system's
// front (the callers' streams wait for ev_done).  Returns without waiting.
int batch_plan_loop(BatchPlan& p, Ctx* const* cs) {
  cudaSetDevice(p.device);
  const int cand = batch_plan_candidate(p);
  if (!p.exec[cand] && !p.profiling) {
    int st = build_graph(p, cand);
    if (st) return st;
  }
  for (int q = 0; q < p.count; ++q) {
    cudaEventRecord(cs[q]->ev_fork, cs[q]->stream);
    cudaStreamWaitEvent(p.stream, cs[q]->ev_fork, 0);
  }
  kb_reset<<<1, 1, 0, p.stream>>>(p.d_loops);
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

// After the solve: its device time (fronts and loop) feeds the tuner, one
// candidate per solve until all are measured.
void batch_plan_finish(BatchPlan& p) {
  if (p.chosen >= 0 || p.running < 0 || p.profiling) return;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, p.ev_start, p.ev_loop) != cudaSuccess) return;
  float& best = p.best_ms[p.running];
  best = std::min(best, ms);
  p.running = -1;
  if (++p.tried < kNumCandidates) return;
  int arg = 0;
  for (int q = 1; q < kNumCandidates; ++q)
    if (p.best_ms[q] < p.best_ms[arg]) arg = q;
  p.chosen = arg;
  for (int q = 0; q < kNumCandidates; ++q)
    if (q != arg && p.exec[q]) {
      cudaGraphExecDestroy(p.exec[q]);
      p.exec[q] = nullptr;
    }
  for (auto it = p.solve_exec.begin(); it != p.solve_exec.end();) {
    if (std::get<2>(it->first) != arg) {
      cudaGraphExecDestroy(it->second);
      it = p.solve_exec.erase(it);
    } else {
      ++it;
    }
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[p.key] = arg;
}

int batch_plan_tuning(const BatchPlan& p, int* blocks_per_sm, int* matvec_atoms, float* ms) {
  const int c = p.chosen;
  if (c < 0) return THP_E_STATE;
  *blocks_per_sm = kCandidates[c].blocks;
  *matvec_atoms = 16 * kCandidates[c].gpw;
  *ms = p.best_ms[c] < 1e29f ? p.best_ms[c] : -1.f;
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

cudaGraphExec_t batch_plan_solve_exec(const BatchPlan& p, int guess, int carry, int cand) {
  auto f = p.solve_exec.find(std::make_tuple(guess, carry, cand));
  return f == p.solve_exec.end() ? nullptr : f->second;
}

// The whole batched solve as one graph: every system's front (child graphs,
// in parallel), the reset of the loop counter, the loop of candidate cand,
// and kb_finish.  fronts[q] are the captured fronts (copied into the graph).
int batch_plan_make_solve_exec(BatchPlan& p, const std::vector<cudaGraph_t>& fronts, int guess, int carry, int cand) {
  cudaSetDevice(p.device);
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return THP_E_CUDA;
  int st = THP_OK;
  std::vector<cudaGraphNode_t> fn(fronts.size());
  for (size_t q = 0; q < fronts.size() && !st; ++q)
    if (cudaGraphAddChildGraphNode(&fn[q], g, nullptr, 0, fronts[q]) != cudaSuccess) st = THP_E_CUDA;
  cudaGraphNode_t reset = nullptr, loop = nullptr, fin = nullptr;
  if (!st) {
    cudaKernelNodeParams kp = {};
    void* args[] = {&p.d_loops};
    kp.func = (void*)kb_reset;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    if (cudaGraphAddKernelNode(&reset, g, fn.data(), fn.size(), &kp) != cudaSuccess) st = THP_E_CUDA;
  }
  if (!st) st = add_loop_node(p, g, &reset, 1, cand, &loop);
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
// are then in mapped host memory.
int batch_plan_run_solve(BatchPlan& p, cudaGraphExec_t ex, const CgScalars** cg_out, const int** flags_out,
                         float* ms) {
  cudaSetDevice(p.device);
  cudaEventRecord(p.ev_start, p.stream);
  if (cudaGraphLaunch(ex, p.stream) != cudaSuccess) return THP_E_CUDA;
  cudaEventRecord(p.ev_loop, p.stream);
  if (cudaStreamSynchronize(p.stream) != cudaSuccess) return THP_E_CUDA;
  p.running = batch_plan_candidate(p);
  cudaEventElapsedTime(ms, p.ev_start, p.ev_loop);
  for (int q = 0; q < p.count; ++q) {
    cg_out[q] = &p.h_out[q].cg;
    flags_out[q] = &p.h_out[q].flags;
  }
  return THP_OK;
}

}  // namespace thp
