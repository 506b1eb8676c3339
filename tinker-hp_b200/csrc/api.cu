// api.cu -- C-ABI of the library: contexts, uploads, solve driver and the
// Fortran-named drop-ins of the reference's polarization subroutines.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <vector>

#include "kernels.h"

using namespace thp;

struct thp_ctx {
  Ctx c;
  bool pos_dirty = true;      // positions uploaded but not yet in sorted order
  bool rpole_dirty = true;    // multipoles uploaded / frames need rotation
  bool field_valid = false;   // d_ef holds E0 for the current positions
  bool guess_uploaded = false;
  bool solved_once = false;
  bool rpole_current = false;  // rotpole has run for the current positions and frames
};

namespace thp {
int cuda_status(cudaError_t e, Ctx* c, const char* what) {
  if (e == cudaSuccess) return THP_OK;
  if (c) {
    c->last_msg = std::string(what) + ": " + cudaGetErrorString(e);
  }
  return THP_E_CUDA;
}
}  // namespace thp

namespace {

thread_local int g_last_error = THP_OK;
thp_ctx* g_current = nullptr;

constexpr int kDefaultMaxNb = 320;

template <class T>
int dmalloc(Ctx& c, T** p, size_t count, const char* what) {
  if (count == 0) count = 1;
  return cuda_status(cudaMalloc((void**)p, sizeof(T) * count), &c, what);
}

// Special pairs with their (d, p, u) scales, in the assignment order of
// efld0_direct (newinduce_pme.f:1062-1136, dpequal false) and tmatxb_pme
// (:1495-1518): pscale from i12..i15 (p*iscale when the partner is in ip11),
// dscale and uscale from ip11..ip14.  Each entry also carries the 1-2..1-5
// class that selects m2scale..m5scale in emreal1c (empole1.f:1040-1051; a
// later list overrides an earlier one, as there).  Pairs whose three scales
// are all 1 and that are in no 1-2..1-5 list are dropped.
static void special_pairs(int n, const int* const* off, const int* const* idx, const double* sc,
                          std::vector<int>& sp_off, std::vector<int>& sp_k, std::vector<double>& sp_s,
                          std::vector<int>& sp_c) {
  sp_off.assign(n + 1, 0);
  sp_k.clear();
  sp_s.clear();
  sp_c.clear();
  auto row = [&](int slot, int i, std::vector<int>& out) {
    out.clear();
    if (!off || !off[slot] || !idx[slot]) return;
    for (int q = off[slot][i]; q < off[slot][i + 1]; ++q) out.push_back(idx[slot][q]);
  };
  std::vector<int> lst, ip11;
  // this atom's partners with their (d, p, u) scales, 1 until a rule sets
  // one, and their bond class; a short list searched linearly and reused
  // across atoms (no per-atom allocation: servers build this for every new
  // system)
  struct Ent {
    int k;
    std::array<double, 3> s;
    int mc;
  };
  std::vector<Ent> m;
  m.reserve(64);
  for (int i = 0; i < n; ++i) {
    m.clear();
    auto get = [&](int k) -> Ent& {
      for (Ent& e : m)
        if (e.k == k) return e;
      m.push_back(Ent{k, {1.0, 1.0, 1.0}, 4});
      return m.back();
    };
    row(THP_IP11, i, ip11);
    for (int b = 0; b < 4; ++b) {
      row(THP_I12 + b, i, lst);
      for (int k : lst) {
        double p = sc[b];
        if (std::find(ip11.begin(), ip11.end(), k) != ip11.end()) p = sc[4 + b];
        Ent& e = get(k);
        e.s[1] = p;
        e.mc = b;
      }
    }
    for (int b = 0; b < 4; ++b) {
      row(THP_IP11 + b, i, lst);
      for (int k : lst) get(k).s[0] = sc[8 + b];
    }
    for (int b = 0; b < 4; ++b) {
      row(THP_IP11 + b, i, lst);
      for (int k : lst) get(k).s[2] = sc[12 + b];
    }
    std::sort(m.begin(), m.end(), [](const Ent& a, const Ent& b) { return a.k < b.k; });  // ascending partners
    for (const Ent& e : m) {
      if (e.k == i) continue;
      const auto& s = e.s;
      if (s[0] == 1.0 && s[1] == 1.0 && s[2] == 1.0 && e.mc == 4) continue;
      sp_k.push_back(e.k);
      sp_s.push_back(s[0]);
      sp_s.push_back(s[1]);
      sp_s.push_back(s[2]);
      sp_c.push_back(e.mc);
    }
    sp_off[i + 1] = (int)sp_k.size();
  }
}

void build_special_pairs(Ctx& c, const int* const* off, const int* const* idx, const double* sc) {
  special_pairs(c.n, off, idx, sc, c.sp_off, c.sp_k, c.sp_s, c.sp_c);
}

// Device buffers for the special pairs of the context's system (kept while
// large enough).
static int reserve_special_pairs(Ctx& c) {
  int st;
  // buffers are kept while large enough, so re-targeting a context does not
  // free device memory (cudaFree waits for the whole device)
  if ((size_t)c.n + 1 > c.cap_sp_off) {
    cudaFree(c.d_sp_off);
    c.d_sp_off = nullptr;
    c.cap_sp_off = 0;
    if ((st = dmalloc(c, &c.d_sp_off, c.n + 1, "alloc sp_off"))) return st;
    c.cap_sp_off = c.n + 1;
  }
  const size_t m = std::max<size_t>(1, c.sp_k.size());
  if (m > c.cap_sp) {
    cudaFree(c.d_sp_k);
    cudaFree(c.d_sp_ks);
    cudaFree(c.d_sp_s);
    cudaFree(c.d_sp_c);
    c.d_sp_k = c.d_sp_ks = c.d_sp_c = nullptr;
    c.d_sp_s = nullptr;
    c.cap_sp = 0;
    if ((st = dmalloc(c, &c.d_sp_k, m, "alloc sp_k"))) return st;
    if ((st = dmalloc(c, &c.d_sp_ks, m, "alloc sp_ks"))) return st;
    if ((st = dmalloc(c, &c.d_sp_s, 3 * m, "alloc sp_s"))) return st;
    if ((st = dmalloc(c, &c.d_sp_c, m, "alloc sp_c"))) return st;
    c.cap_sp = m;
  }
  return THP_OK;
}

int upload_special_pairs(Ctx& c) {
  c.have_list = false;  // sorted partner numbers are made at the next sort
  int st = reserve_special_pairs(c);
  if (st) return st;
  cudaMemcpyAsync(c.d_sp_off, c.sp_off.data(), sizeof(int) * (c.n + 1), cudaMemcpyHostToDevice, c.stream);
  if (!c.sp_k.empty()) {
    cudaMemcpyAsync(c.d_sp_k, c.sp_k.data(), sizeof(int) * c.sp_k.size(), cudaMemcpyHostToDevice, c.stream);
    cudaMemcpyAsync(c.d_sp_s, c.sp_s.data(), sizeof(double) * c.sp_s.size(), cudaMemcpyHostToDevice, c.stream);
    cudaMemcpyAsync(c.d_sp_c, c.sp_c.data(), sizeof(int) * c.sp_c.size(), cudaMemcpyHostToDevice, c.stream);
  }
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "upload special pairs");
}

void cell_grid(const thp_config& cfg, int nc[3]) {
  const double half_cut = 0.5 * (cfg.ewaldcut + cfg.lbuffer) + 1e-6;
  for (int d = 0; d < 3; ++d) nc[d] = std::max(1, (int)std::floor(cfg.box[d] / half_cut));
}

// Maps the device error bits copied into h_flags to a status (and clears
// them on the device).
static int flags_status(Ctx& c) {
  int f = *c.h_flags;
  if (f) {
    cudaMemsetAsync(c.d_flags, 0, sizeof(int), c.stream);
    if (f & DEV_BAD_INPUT) {
      c.last_msg = "non-finite coordinates";
      return THP_E_INVALID;
    }
    if (f & DEV_VDW_REACH) {
      c.last_msg = "a vdW reduction shift exceeds the 0.3 A the pair search allows";
      return THP_E_INVALID;
    }
    if (f & (DEV_LIST_OVERFLOW | DEV_PAIR_OVERFLOW)) {
      c.last_msg = "neighbor capacity exceeded";
      return THP_E_LIST_OVERFLOW;
    }
    return THP_E_NAN;
  }
  return THP_OK;
}

int check_flags(thp_ctx* h) {
  Ctx& c = h->c;
  cudaMemcpyAsync(c.h_flags, c.d_flags, sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  int st = cuda_status(cudaStreamSynchronize(c.stream), &c, "sync");
  if (st) return st;
  return flags_status(c);
}

int set_current_device(Ctx& c) { return cuda_status(cudaSetDevice(c.device), &c, "set device"); }

// Brings the sorted arrays up to date with the uploaded positions and
// decides whether the list must be rebuilt: on the first call or when an atom
// moved by more than lbuffer/2 since the last build (the reference rebuilds
// every ineigup steps; the displacement test keeps the same interacting set).
// On *rebuild the atoms are re-sorted, and the caller launches the build.
static int prepare_list(thp_ctx* h, bool force_rebuild, bool* rebuild_out) {
  Ctx& c = h->c;
  int st;
  if (!c.have_pos) return THP_E_STATE;
  bool rebuild = force_rebuild || !c.have_list;
  if (!rebuild && h->pos_dirty) {
    if ((st = launch_gather_sorted(c))) return st;
    double disp = 0.0;
    if ((st = launch_max_displacement(c, &disp))) return st;
    if (disp >= 0.5 * c.cfg.lbuffer) rebuild = true;
    h->pos_dirty = false;
    h->rpole_dirty = false;
    c.have_coef = false;
    h->field_valid = false;
  }
  if (rebuild) {
    if ((st = launch_sort_atoms(c))) return st;
    if ((st = launch_gather_sorted(c))) return st;
    c.have_list = false;
    c.have_coef = false;
    h->field_valid = false;
  } else if (h->pos_dirty || h->rpole_dirty) {
    if ((st = launch_gather_sorted(c))) return st;
    h->field_valid = false;
  }
  h->pos_dirty = false;
  h->rpole_dirty = false;
  *rebuild_out = rebuild;
  return THP_OK;
}

// E0 = direct + reciprocal + self (newinduce_pme2.f:110-148) and the matvec
// coefficients, after the list build when `build` is set.  A system whose CG
// rows run on the side stream runs the list build and the direct pass there
// too, concurrent with the spread and FFTs of the permanent multipoles on the
// main stream; the gather that completes E0 follows the join.  Returns with
// the main stream joined, on error as well.
#ifndef THP_FRONT_OVERLAP
#define THP_FRONT_OVERLAP 1
#endif

static int launch_fields(Ctx& c, bool build) {
  int st;
  if (!THP_FRONT_OVERLAP || !overlap_rows(c)) {
    if (build && (st = launch_build_list(c))) return st;
    if ((st = launch_efld0_coef(c, true))) return st;
    return launch_efld0_recip(c);
  }
  cudaEventRecord(c.ev_fork, c.stream);
  cudaStreamWaitEvent(c.stream2, c.ev_fork, 0);
  st = build ? launch_build_list_on(c, c.stream2) : THP_OK;
  if (!st) st = launch_efld0_coef_on(c, true, c.stream2);
  cudaEventRecord(c.ev_join, c.stream2);
  int st2 = launch_mpole_grid(c);
  cudaStreamWaitEvent(c.stream, c.ev_join, 0);
  if (st || st2) return st ? st : st2;
  return launch_gather_mpole(c, nullptr, true);
}

// Ensures the sorted arrays match the uploaded positions and the list is
// valid (see prepare_list).
int ensure_list(thp_ctx* h, bool force_rebuild) {
  Ctx& c = h->c;
  int st;
  if (!c.have_pos) return THP_E_STATE;
  bool rebuild = force_rebuild || !c.have_list;
  if (!rebuild && h->pos_dirty) {
    if ((st = launch_gather_sorted(c))) return st;
    double disp = 0.0;
    if ((st = launch_max_displacement(c, &disp))) return st;
    if (disp >= 0.5 * c.cfg.lbuffer) rebuild = true;
    h->pos_dirty = false;
    h->rpole_dirty = false;
    c.have_coef = false;
    h->field_valid = false;
  }
  if (rebuild) {
    if ((st = launch_sort_atoms(c))) return st;
    if ((st = launch_gather_sorted(c))) return st;
    if ((st = launch_build_list(c))) return st;
    if ((st = check_flags(h))) return st;
    c.have_list = true;
    c.have_coef = false;
    h->field_valid = false;
    h->pos_dirty = false;
    h->rpole_dirty = false;
  } else if (h->pos_dirty || h->rpole_dirty) {
    if ((st = launch_gather_sorted(c))) return st;
    h->pos_dirty = false;
    h->rpole_dirty = false;
    h->field_valid = false;
  }
  return THP_OK;
}

int ensure_rpole(thp_ctx* h) {
  Ctx& c = h->c;
  if (c.have_frames && !h->rpole_current) {  // the same positions rotate to the same multipoles
    int st = launch_rotpole(c);
    if (st) return st;
    c.have_rpole = true;
    h->rpole_dirty = true;
    h->rpole_current = true;
  }
  return c.have_rpole ? THP_OK : THP_E_STATE;
}

// E0 = direct + reciprocal + self (newinduce_pme2.f:110-148) and the matvec
// coefficients, for the current positions and multipoles.  check: read the
// device error bits now (a host sync); otherwise the caller reads them with
// its own later sync.
int compute_field(thp_ctx* h, bool check = true) {
  Ctx& c = h->c;
  int st;
  if ((st = ensure_rpole(h))) return st;
  bool rebuild = false;
  if ((st = prepare_list(h, false, &rebuild))) return st;
  if ((st = launch_fields(c, rebuild))) return st;
  c.have_list = true;
  if (check) {
    if ((st = check_flags(h))) return st;
    h->field_valid = true;
  }
  return THP_OK;
}

int ensure_coef(thp_ctx* h) {
  Ctx& c = h->c;
  int st;
  if ((st = ensure_list(h, false))) return st;
  if (!c.have_coef) {
    if ((st = launch_efld0_coef(c, false))) return st;
    if ((st = check_flags(h))) return st;
  }
  return THP_OK;
}

// Pinned blocks for the per-context CG scalars and flags are recycled
// process-wide: cudaMallocHost is slow and serialises with other threads.
namespace {
std::mutex g_pinned_mu;
std::vector<void*> g_pinned_free;
constexpr size_t kPinnedBlock = 4096;
}  // namespace

static int pinned_take(Ctx& c) {
  {
    std::lock_guard<std::mutex> g(g_pinned_mu);
    if (!g_pinned_free.empty()) {
      c.h_pinned = g_pinned_free.back();
      g_pinned_free.pop_back();
    }
  }
  if (!c.h_pinned) {
    int st = cuda_status(cudaMallocHost(&c.h_pinned, kPinnedBlock), &c, "pinned");
    if (st) return st;
  }
  c.h_cg = static_cast<CgScalars*>(c.h_pinned);
  c.h_flags = reinterpret_cast<int*>(static_cast<char*>(c.h_pinned) + 2048);
  return THP_OK;
}

static void pinned_give(Ctx& c) {
  if (!c.h_pinned) return;
  std::lock_guard<std::mutex> g(g_pinned_mu);
  g_pinned_free.push_back(c.h_pinned);
  c.h_pinned = nullptr;
  c.h_cg = nullptr;
  c.h_flags = nullptr;
}

void free_ctx(Ctx& c) {
  void* ptrs[] = {c.slab_cells, c.slab_atoms, c.slab_pairs, c.d_sp_off, c.d_sp_k, c.d_sp_ks, c.d_sp_s, c.d_sp_c,
                  c.d_cg, c.d_flags, c.d_fphirec, c.d_depfix, c.d_trq, c.d_frs, c.d_grad, c.d_sgrid, c.d_sscratch,
                  c.d_alt, c.d_empart, c.d_vcls, c.d_vired, c.d_vkred, c.d_vtab, c.d_vred, c.d_vinfo,
                  c.d_evpart, c.d_vnb, c.d_vnnb, c.d_vpos_built, c.d_vredf, c.d_muf, c.d_virp};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  pme_free(c);
  if (c.chunk_exec) cudaGraphExecDestroy(c.chunk_exec);
  if (c.loop_exec) cudaGraphExecDestroy(c.loop_exec);
  for (auto& row : c.front_exec)
    for (auto& ex : row)
      if (ex) cudaGraphExecDestroy(ex);
  pinned_give(c);
  if (c.ev_fork) cudaEventDestroy(c.ev_fork);
  if (c.ev_join) cudaEventDestroy(c.ev_join);
  if (c.stream2) cudaStreamDestroy(c.stream2);
  if (c.ev0) cudaEventDestroy(c.ev0);
  if (c.ev1) cudaEventDestroy(c.ev1);
  if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
}

// graphs that hold a system's structure (rotpole on/off, special pairs,
// sizes) are dropped when it changes
static void drop_front_graphs(Ctx& c) {
  for (auto& row : c.front_exec)
    for (auto& ex : row)
      if (ex) {
        cudaGraphExecDestroy(ex);
        ex = nullptr;
      }
  c.front_failed = false;
}

size_t footprint_bytes(const thp_config& cfg, int* ncell_out) {
  const size_t n = cfg.n, npad = (n + 31) / 32 * 32;
  const size_t maxnb = ((cfg.max_neighbors > 0 ? cfg.max_neighbors : kDefaultMaxNb) + 7) / 8 * 8;
  int nc[3];
  cell_grid(cfg, nc);
  const size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
  if (ncell_out) *ncell_out = (int)ncell;
  const bool mixed = cfg.precision == THP_MIXED;
  const size_t ngrid = (size_t)cfg.nfft[0] * cfg.nfft[1] * cfg.nfft[2];
  size_t b = 0;
  b += 3 * ncell * 4 + 2 * n * 4 + 2 * n * 4;          // cells, perm
  b += (3 + 3 + 13 + 13) * n * 8 + 3 * n * 4;            // staging
  b += n * 32 + n * 16 + 2 * n * 8 + 10 * n * 8 + n * 32 + n * 64;  // sorted data
  b += n * 4 + maxnb * npad * 4;                         // list
  b += n * 4 + maxnb * npad * (4 + 2 * (mixed ? 4 : 8));  // pairs
  b += ngrid * (mixed ? 12 : 24);                        // grid + qfac
  b += 10 * n * 6 * 8 + 4 * n * 8 + n * 6 * 4 + n * 9 * 4 + 4 * n * 6 * 4;  // vectors, FP32 row input and CG vectors
  b += (n / 128 + 2) * 4 * 8 + 4096;
  b += 64 << 20;  // cuFFT work area and runtime slack
  return b;
}

}  // namespace

// ===========================================================================
extern "C" {

const char* thp_status_string(int s) {
  switch (s) {
    case THP_OK: return "ok";
    case THP_E_INVALID: return "invalid argument";
    case THP_E_LIST_OVERFLOW: return "neighbor list overflow";
    case THP_E_NOT_CONVERGED: return "CG not converged";
    case THP_E_NAN: return "non-finite value";
    case THP_E_CUDA: return "CUDA error";
    case THP_E_TIMEOUT: return "device wait timed out";
    case THP_E_OOM_ADMISSION: return "device memory budget exceeded";
    case THP_E_BOX_TOO_SMALL: return "cutoff exceeds half box";
    case THP_E_NO_DEVICE: return "no CUDA device";
    case THP_E_STATE: return "inputs not set";
    default: return "unknown";
  }
}

size_t thp_footprint(const thp_config* cfg) { return cfg ? footprint_bytes(*cfg, nullptr) : 0; }

static int check_config(const thp_config& k) {
  if (k.n <= 0 || k.box[0] <= 0 || k.box[1] <= 0 || k.box[2] <= 0 || k.aewald <= 0 || k.ewaldcut <= 0 ||
      k.lbuffer < 0 || k.bsorder != 5 || k.nfft[0] < 5 || k.nfft[1] < 5 || k.nfft[2] < 5 || k.politer <= 0 ||
      (k.precision != THP_FP64 && k.precision != THP_MIXED))
    return THP_E_INVALID;
  const double rl = k.ewaldcut + k.lbuffer;
  const double half = 0.5 * std::min(k.box[0], std::min(k.box[1], k.box[2]));
  if (rl * rl > half * half) return THP_E_BOX_TOO_SMALL;  // nblist.f:147-156
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return THP_E_NO_DEVICE;
  if (k.device < 0 || k.device >= ndev) return THP_E_INVALID;
  return THP_OK;
}

// System geometry and sizes from a configuration (no device work).
static void apply_config(Ctx& c, const thp_config& k) {
  c.cfg = k;
  c.n = k.n;
  c.npad = (k.n + 31) / 32 * 32;
  c.mixed = k.precision == THP_MIXED;
  c.device = k.device;
  c.maxnb = k.max_neighbors > 0 ? k.max_neighbors : kDefaultMaxNb;
  c.maxpr = (c.maxnb + 7) / 8 * 8;  // the pair stream holds an atom's slots in blocks of 8
  for (int d = 0; d < 3; ++d) {
    c.box.l[d] = k.box[d];
    c.box.half[d] = 0.5 * k.box[d];
  }
  // lattice.f:111-120 for an orthogonal box: recip(d,d) = (product of the
  // other two edges) / volbox
  const double vol = k.box[0] * k.box[1] * k.box[2];
  c.box.recip[0] = (k.box[1] * 1.0 * (k.box[2] * 1.0) - (k.box[2] * 0.0) * 0.0) / vol;
  c.box.recip[1] = ((k.box[2] * 1.0) * k.box[0] - 0.0 * (k.box[2] * 0.0)) / vol;
  c.box.recip[2] = (k.box[0] * (k.box[1] * 1.0) - (k.box[1] * 0.0) * 0.0) / vol;
  cell_grid(k, c.nc);
  c.ncell = c.nc[0] * c.nc[1] * c.nc[2];
  c.nblk_reduce = (c.n + 31) / 32;  // partial sums of up to one block per 32 atoms
}

extern "C++" {
template <class... P>
static void free_all(P**... p) {
  ((cudaFree(*p), *p = nullptr), ...);
}
}

// Grows each buffer group that is smaller than the current sizes need; a
// group that is large enough is kept as it is.
struct SlabItem {
  void** ptr;
  size_t bytes;
};

// One cudaMalloc for a group of arrays, each starting on a 256-byte boundary.
static int alloc_slab(Ctx& c, void** base, std::initializer_list<SlabItem> items, const char* what) {
  auto up = [](size_t b) { return (std::max<size_t>(b, 1) + 255) / 256 * 256; };
  size_t total = 0;
  for (const SlabItem& it : items) total += up(it.bytes);
  void* b = nullptr;
  int st = cuda_status(cudaMalloc(&b, total), &c, what);
  if (st) return st;
  size_t off = 0;
  for (const SlabItem& it : items) {
    *it.ptr = static_cast<char*>(b) + off;
    off += up(it.bytes);
  }
  *base = b;
  return THP_OK;
}

extern "C++" {
template <class T>
static SlabItem item(T** p, size_t count) {
  return SlabItem{reinterpret_cast<void**>(p), count * sizeof(T)};
}
}

// Grows each buffer group that is smaller than the current sizes need; a
// group that is large enough is kept as it is.
static int size_buffers(Ctx& c) {
  int st = THP_OK;
  const size_t n = c.n, npad = c.npad;
  const size_t esz = c.mixed ? 4 : 8;
  if ((size_t)c.ncell > c.cap_ncell) {
    cudaFree(c.slab_cells);
    c.slab_cells = nullptr;
    c.cap_ncell = 0;
    const size_t m = c.ncell;
    st = alloc_slab(c, &c.slab_cells, {item(&c.d_cell_count, m), item(&c.d_cell_start, m), item(&c.d_cell_fill, m)},
                    "cells");
    if (!st) c.cap_ncell = c.ncell;
  }
  if (!st && n > c.cap_n) {
    cudaFree(c.slab_atoms);
    c.slab_atoms = nullptr;
    // buffers made on first use are sized by n as well
    free_all(&c.d_fphirec, &c.d_depfix, &c.d_trq, &c.d_frs, &c.d_grad, &c.d_empart, &c.d_vcls, &c.d_vired,
             &c.d_vkred, &c.d_vred, &c.d_vredf, &c.d_vinfo, &c.d_evpart, &c.d_vnb, &c.d_vnnb, &c.d_vpos_built,
             &c.d_muf);
    c.have_vlist = false;
    c.d_em = c.d_ev = nullptr;
    c.have_vdw = false;
    c.cap_n = 0;
    st = alloc_slab(c, &c.slab_atoms,
                    {item(&c.d_atom_cell, n), item(&c.d_scell, n), item(&c.d_perm, n), item(&c.d_iperm, n),
                     item(&c.d_xyz_orig, 3 * n), item(&c.d_par_orig, 3 * n), item(&c.d_rpole_orig, 13 * n),
                     item(&c.d_pole_local, 13 * n), item(&c.d_frames, 3 * n), item(&c.d_pos, n),
                     item(&c.d_posf, n), item(&c.d_thole, n), item(&c.d_pol, n), item(&c.d_rpole, 10 * n),
                     item(&c.d_mrec, 12 * n), item(&c.d_mrecf, 12 * n), item(&c.d_erec, 16 * n), item(&c.d_pos_built, n),
                     item(&c.d_nnb, n), item(&c.d_npr, n), item(&c.d_ef, 6 * n), item(&c.d_mu, 6 * n),
                     item(&c.d_res, 6 * n), item(&c.d_h, 6 * n), item(&c.d_pp, 6 * n), item(&c.d_zr, 6 * n),
                     item(&c.d_dip, 6 * n), item(&c.d_tmp6, 6 * n), item(&c.d_tmp6b, 6 * n), item(&c.d_cphi, 4 * n),
                     item(&c.d_vecf, 6 * n), item(&c.d_rec, 8 * n), item(&c.d_mpz, n), item(&c.d_ef_prev, 6 * n),
                     item(&c.d_ppf, 6 * n), item(&c.d_hf, 6 * n), item(&c.d_resf, 6 * n), item(&c.d_zrf, 6 * n),
                     item(&c.d_partials, (size_t)(c.nblk_reduce + 8) * 4)},
                    "per-atom buffers");
    if (!st) c.cap_n = n;
  }
  const size_t pairs = (size_t)c.maxpr * npad;  // list (maxnb <= maxpr slots) and pair stream
  if (!st && pairs > c.cap_pairs) {
    cudaFree(c.slab_pairs);
    c.slab_pairs = nullptr;
    c.cap_pairs = 0;
    st = alloc_slab(c, &c.slab_pairs,
                    {item(&c.d_nb, pairs), item(&c.d_pk, pairs), SlabItem{&c.d_pcc, 2 * esz * pairs}},
                    "pair buffers");
    if (!st) c.cap_pairs = pairs;
  }
  if (!st && !c.d_cg) st = dmalloc(c, &c.d_cg, 1, "cg");
  if (!st && !c.d_flags) st = dmalloc(c, &c.d_flags, 1, "flags");
  if (!st && !c.h_pinned) st = pinned_take(c);
  return st;
}

// Clears everything that belongs to the system a context serves, after
// apply_config/size_buffers/pme_init: no parameters, positions,
// multipoles, list or dipoles; no special pairs.
static int clear_system_state(thp_ctx* h) {
  Ctx& c = h->c;
  c.have_params = c.have_pos = c.have_rpole = c.have_conn = c.have_frames = c.have_axes = false;
  c.have_perm = c.have_list = c.have_coef = c.have_dipoles = c.have_ef_prev = false;
  c.pred_mode = c.nualt = c.alt_head = 0;
  h->pos_dirty = h->rpole_dirty = true;
  h->rpole_current = false;
  h->field_valid = h->guess_uploaded = h->solved_once = false;
  c.bx = c.by = c.bz = c.brpole = c.buind = c.buinp = c.bep = c.bdep = c.bqgrid = nullptr;
  c.bem = c.bdem = c.bev = c.bdev = nullptr;
  c.bnvlst = c.bvlst = nullptr;
  c.bmaxvlst = 0;
  c.have_vdw = false;
  c.mscale[0] = c.mscale[1] = 0.0;  // initprm.f:413-416
  c.mscale[2] = c.mscale[3] = 1.0;
  c.bnelst = c.belst = nullptr;
  c.bmaxelst = 0;
  cudaMemsetAsync(c.d_flags, 0, sizeof(int), c.stream);
  cudaMemsetAsync(c.d_cg, 0, sizeof(CgScalars), c.stream);
  cudaMemsetAsync(c.d_mu, 0, sizeof(double) * 6 * c.n, c.stream);
  c.sp_off.assign(c.n + 1, 0);
  c.sp_k.clear();
  c.sp_s.clear();
  c.sp_c.clear();
  return upload_special_pairs(c);  // synchronises the stream
}

int thp_ctx_create(const thp_config* cfg, thp_ctx** out) {
  if (!cfg || !out) return THP_E_INVALID;
  *out = nullptr;
  int st = check_config(*cfg);
  if (st) return st;
  thp_ctx* h = new thp_ctx();
  Ctx& c = h->c;
  apply_config(c, *cfg);
  st = set_current_device(c);
  if (!st) st = cuda_status(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), &c, "stream");
  c.own_stream = true;
  if (!st) st = cuda_status(cudaStreamCreateWithFlags(&c.stream2, cudaStreamNonBlocking), &c, "stream");
  if (!st) st = cuda_status(cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming), &c, "event");
  if (!st) st = cuda_status(cudaEventCreateWithFlags(&c.ev_join, cudaEventDisableTiming), &c, "event");
  if (!st) st = cuda_status(cudaEventCreate(&c.ev0), &c, "event");
  if (!st) st = cuda_status(cudaEventCreate(&c.ev1), &c, "event");
  if (!st) st = size_buffers(c);
  if (!st) st = pme_init(c);
  if (!st) st = clear_system_state(h);
  if (st) {
    fprintf(stderr, "thp_ctx_create: %s\n", c.last_msg.c_str());
    free_ctx(c);
    delete h;
    return st;
  }
  *out = h;
  return THP_OK;
}

int thp_ctx_reset(thp_ctx* h, const thp_config* cfg) {
  if (!h || !cfg) return THP_E_INVALID;
  Ctx& c = h->c;
  int st = check_config(*cfg);
  if (st) return st;
  if ((cfg->precision == THP_MIXED) != (c.mixed != 0) || cfg->device != c.device) return THP_E_INVALID;
  if (set_current_device(c)) return THP_E_CUDA;
  if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "reset"))) return st;
  // graphs hold this system's sizes and launch shapes
  if (c.chunk_exec) cudaGraphExecDestroy(c.chunk_exec);
  if (c.loop_exec) cudaGraphExecDestroy(c.loop_exec);
  c.chunk_exec = c.loop_exec = nullptr;
  c.loop_state = 0;
  drop_front_graphs(c);
  for (cudaEvent_t e : c.prof_events) cudaEventDestroy(e);
  c.prof_events.clear();
  c.profiling = false;
  const size_t old_ngrid = c.ngrid;
  apply_config(c, *cfg);
  if ((st = size_buffers(c))) return st;
  if ((st = pme_init(c))) return st;
  if (c.ngrid > old_ngrid && c.d_sgrid) {
    cudaFree(c.d_sgrid);
    c.d_sgrid = nullptr;
  }
  if (g_current == h) g_current = nullptr;
  return clear_system_state(h);
}

size_t thp_ctx_footprint(thp_ctx* h) {
  if (!h) return 0;
  thp_config k = h->c.cfg;
  k.n = (int)std::max<size_t>(h->c.cap_n, (size_t)k.n);
  const size_t ng = std::max<size_t>(h->c.cap_ngrid, 1);
  // the grid term of the footprint depends only on the product of the dims
  k.nfft[0] = (int)ng;
  k.nfft[1] = k.nfft[2] = 1;
  return footprint_bytes(k, nullptr);
}

int thp_ctx_destroy(thp_ctx* h) {
  if (!h) return THP_E_INVALID;
  cudaSetDevice(h->c.device);
  cudaStreamSynchronize(h->c.stream);
  if (g_current == h) g_current = nullptr;
  free_ctx(h->c);
  delete h;
  return THP_OK;
}

int thp_set_stream(thp_ctx* h, void* stream) {
  if (!h) return THP_E_INVALID;
  Ctx& c = h->c;
  cudaStreamSynchronize(c.stream);
  if (c.own_stream) cudaStreamDestroy(c.stream);
  c.stream = (cudaStream_t)stream;
  c.own_stream = false;
  if (c.have_plan) cufftSetStream(c.plan, c.stream);
  return THP_OK;
}

int thp_set_params(thp_ctx* h, const double* polarity, const double* thole, const double* pdamp) {
  if (!h || !polarity || !thole || !pdamp) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  const size_t n = c.n;
  c.h_polarity.assign(polarity, polarity + n);
  c.h_thole.assign(thole, thole + n);
  c.h_pdamp.assign(pdamp, pdamp + n);
  cudaMemcpyAsync(c.d_par_orig, pdamp, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_par_orig + n, thole, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_par_orig + 2 * n, polarity, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
  c.have_params = true;
  h->pos_dirty = true;
  h->rpole_current = false;
  c.have_coef = false;
  h->field_valid = false;
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "set params");
}

int thp_set_connectivity(thp_ctx* h, const int* const* off, const int* const* idx, const double* scales) {
  if (!h || !scales) return THP_E_INVALID;
  Ctx& c = h->c;
  drop_front_graphs(c);
  if (set_current_device(c)) return THP_E_CUDA;
  std::memcpy(c.scales, scales, sizeof(c.scales));
  build_special_pairs(c, off, idx, scales);
  c.have_conn = true;
  c.have_coef = false;
  h->field_valid = false;
  return upload_special_pairs(c);
}

// Uploads the coordinates; host_check rejects non-finite values before the
// copy, otherwise the sorted gather flags them on the device and the next
// flag check returns THP_E_INVALID.  (Also used by the request loop.)
}  // extern "C"
namespace thp {

// A system's inputs prepared once on the host for the request loop: checked,
// special pairs built, frames packed, all in pinned memory when the driver
// gives it.  Loading the image onto a context is then a few asynchronous
// copies on the context's stream with no host wait, where thp_set_params,
// thp_set_connectivity and thp_set_frames each build, stage and synchronise.
struct SystemImage {
  int n = 0, m = 0;
  double scales[16] = {};
  bool pinned = false;
  double* par = nullptr;   // [3n] pdamp, thole, polarity (the d_par_orig planes)
  double* pole = nullptr;  // [13n] local-frame multipoles
  int* frames = nullptr;   // [3n] z-axis, x-axis, frame type
  int* sp_off = nullptr;   // [n+1]
  int* sp_k = nullptr;     // [m]
  int* sp_c = nullptr;     // [m]
  double* sp_s = nullptr;  // [3m]
  void* block = nullptr;
};

void image_free(SystemImage* img) {
  if (!img) return;
  if (img->pinned)
    cudaFreeHost(img->block);
  else
    std::free(img->block);
  delete img;
}

int image_create(const thp_config& cfg, const double* polarity, const double* thole, const double* pdamp,
                 const int* const* off, const int* const* idx, const double* scales, const double* pole,
                 const int* zaxis, const int* xaxis, const int* axt, SystemImage** out) {
  *out = nullptr;
  const int n = cfg.n;
  if (n <= 0 || !polarity || !thole || !pdamp || !scales || !pole || !zaxis || !xaxis || !axt)
    return THP_E_INVALID;
  for (int i = 0; i < n; ++i)
    if (zaxis[i] < 0 || zaxis[i] >= n || xaxis[i] < 0 || xaxis[i] >= n || (axt[i] != 1 && axt[i] != 2))
      return THP_E_INVALID;
  std::vector<int> so, sk, sc;
  std::vector<double> ss;
  special_pairs(n, off, idx, scales, so, sk, ss, sc);
  auto* img = new SystemImage();
  img->n = n;
  img->m = (int)sk.size();
  std::memcpy(img->scales, scales, sizeof(img->scales));
  const size_t nd = 3 * (size_t)n + 13 * (size_t)n + 3 * (size_t)img->m;
  const size_t ni = 3 * (size_t)n + (size_t)n + 1 + 2 * (size_t)img->m;
  const size_t bytes = nd * sizeof(double) + ni * sizeof(int);
  if (cudaHostAlloc(&img->block, bytes, cudaHostAllocDefault) == cudaSuccess) {
    img->pinned = true;
  } else {
    cudaGetLastError();  // no device here: the requests will report it
    img->block = std::malloc(bytes);
    if (!img->block) {
      delete img;
      return THP_E_INVALID;
    }
  }
  double* d = static_cast<double*>(img->block);
  img->par = d;
  img->pole = d + 3 * (size_t)n;
  img->sp_s = img->pole + 13 * (size_t)n;
  int* q = reinterpret_cast<int*>(img->sp_s + 3 * (size_t)img->m);
  img->frames = q;
  img->sp_off = q + 3 * (size_t)n;
  img->sp_k = img->sp_off + n + 1;
  img->sp_c = img->sp_k + img->m;
  std::memcpy(img->par, pdamp, sizeof(double) * n);
  std::memcpy(img->par + n, thole, sizeof(double) * n);
  std::memcpy(img->par + 2 * (size_t)n, polarity, sizeof(double) * n);
  std::memcpy(img->pole, pole, sizeof(double) * 13 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    img->frames[3 * i] = zaxis[i];
    img->frames[3 * i + 1] = xaxis[i];
    img->frames[3 * i + 2] = axt[i];
  }
  std::memcpy(img->sp_off, so.data(), sizeof(int) * (n + 1));
  if (img->m) {
    std::memcpy(img->sp_k, sk.data(), sizeof(int) * img->m);
    std::memcpy(img->sp_s, ss.data(), sizeof(double) * 3 * (size_t)img->m);
    std::memcpy(img->sp_c, sc.data(), sizeof(int) * img->m);
  }
  *out = img;
  return THP_OK;
}

// Parameters, connectivity and frames of the image onto a context sized for
// it (the state thp_set_params, thp_set_connectivity and thp_set_frames
// leave), stream-ordered before the context's next solve.
int image_load(thp_ctx* h, const SystemImage* img) {
  if (!h || !img) return THP_E_INVALID;
  Ctx& c = h->c;
  if (img->n != c.n) return THP_E_INVALID;
  drop_front_graphs(c);
  if (set_current_device(c)) return THP_E_CUDA;
  const size_t n = c.n;
  c.h_pdamp.assign(img->par, img->par + n);
  c.h_thole.assign(img->par + n, img->par + 2 * n);
  c.h_polarity.assign(img->par + 2 * n, img->par + 3 * n);
  cudaMemcpyAsync(c.d_par_orig, img->par, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c.stream);
  c.have_params = true;
  std::memcpy(c.scales, img->scales, sizeof(c.scales));
  c.sp_off.assign(img->sp_off, img->sp_off + n + 1);
  c.sp_k.assign(img->sp_k, img->sp_k + img->m);
  c.sp_s.assign(img->sp_s, img->sp_s + 3 * (size_t)img->m);
  c.sp_c.assign(img->sp_c, img->sp_c + img->m);
  c.have_conn = true;
  int st = reserve_special_pairs(c);
  if (st) return st;
  cudaMemcpyAsync(c.d_sp_off, img->sp_off, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c.stream);
  if (img->m) {
    cudaMemcpyAsync(c.d_sp_k, img->sp_k, sizeof(int) * img->m, cudaMemcpyHostToDevice, c.stream);
    cudaMemcpyAsync(c.d_sp_s, img->sp_s, sizeof(double) * 3 * img->m, cudaMemcpyHostToDevice, c.stream);
    cudaMemcpyAsync(c.d_sp_c, img->sp_c, sizeof(int) * img->m, cudaMemcpyHostToDevice, c.stream);
  }
  cudaMemcpyAsync(c.d_pole_local, img->pole, sizeof(double) * 13 * n, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_frames, img->frames, sizeof(int) * 3 * n, cudaMemcpyHostToDevice, c.stream);
  c.have_frames = true;
  h->rpole_current = false;
  c.have_axes = true;
  c.have_list = false;
  c.have_coef = false;
  h->pos_dirty = true;
  h->rpole_current = false;
  h->rpole_dirty = true;
  h->field_valid = false;
  return cuda_status(cudaGetLastError(), &c, "load system");
}

int upload_positions(thp_ctx* h, const double* x, const double* y, const double* z, bool host_check) {
  if (!h || !x || !y || !z) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  const size_t n = c.n;
  if (host_check)
    for (size_t i = 0; i < n; ++i)
      if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(z[i])) return THP_E_INVALID;
  cudaMemcpyAsync(c.d_xyz_orig, x, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_xyz_orig + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_xyz_orig + 2 * n, z, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
  c.have_pos = true;
  h->pos_dirty = true;
  h->rpole_current = false;
  h->field_valid = false;
  c.have_coef = false;
  if (c.have_frames) h->rpole_dirty = true;
  return cuda_status(cudaGetLastError(), &c, "set positions");
}
}  // namespace thp
extern "C" {

int thp_set_positions(thp_ctx* h, const double* x, const double* y, const double* z) {
  return thp::upload_positions(h, x, y, z, true);
}

int thp_set_rpole(thp_ctx* h, const double* rpole) {
  if (!h || !rpole) return THP_E_INVALID;
  Ctx& c = h->c;
  drop_front_graphs(c);
  if (set_current_device(c)) return THP_E_CUDA;
  cudaMemcpyAsync(c.d_rpole_orig, rpole, sizeof(double) * 13 * c.n, cudaMemcpyHostToDevice, c.stream);
  c.have_rpole = true;
  c.have_frames = false;
  h->rpole_dirty = true;
  h->field_valid = false;
  return cuda_status(cudaGetLastError(), &c, "set rpole");
}

int thp_set_frames(thp_ctx* h, const double* pole, const int* zaxis, const int* xaxis, const int* axt) {
  if (!h || !pole || !zaxis || !xaxis || !axt) return THP_E_INVALID;
  Ctx& c = h->c;
  drop_front_graphs(c);
  if (set_current_device(c)) return THP_E_CUDA;
  const int n = c.n;
  std::vector<int> fr(3 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    if (zaxis[i] < 0 || zaxis[i] >= n || xaxis[i] < 0 || xaxis[i] >= n || (axt[i] != 1 && axt[i] != 2))
      return THP_E_INVALID;
    fr[3 * i] = zaxis[i];
    fr[3 * i + 1] = xaxis[i];
    fr[3 * i + 2] = axt[i];
  }
  cudaMemcpy(c.d_pole_local, pole, sizeof(double) * 13 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(c.d_frames, fr.data(), sizeof(int) * 3 * n, cudaMemcpyHostToDevice);
  c.have_frames = true;
  h->rpole_current = false;
  c.have_axes = true;
  h->rpole_dirty = true;
  h->field_valid = false;
  return cuda_status(cudaGetLastError(), &c, "set frames");
}

int thp_set_guess(thp_ctx* h, const double* mu) {
  if (!h || !mu) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  int st = ensure_list(h, false);
  if (st) return st;
  cudaMemcpyAsync(c.d_tmp6, mu, sizeof(double) * 6 * c.n, cudaMemcpyHostToDevice, c.stream);
  if ((st = launch_to_sorted6(c, c.d_tmp6, c.d_mu, 2))) return st;
  h->guess_uploaded = true;
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "set guess");
}

int thp_nblist(thp_ctx* h) {
  if (!h) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  if (!c.have_params) return THP_E_STATE;
  int st = ensure_list(h, false);
  if (st) return st;
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "nblist");
}

int thp_invalidate_list(thp_ctx* h) {
  if (!h) return THP_E_INVALID;
  h->c.have_list = false;
  h->c.have_coef = false;
  h->field_valid = false;
  return THP_OK;
}

int thp_profile(thp_ctx* h, int enable, double* ms_total, int* launches) {
  if (!h) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  if (ms_total || launches) {
    int st = cuda_status(cudaStreamSynchronize(c.stream), &c, "profile");
    if (st) return st;
    double tot = 0.0;
    for (size_t q = 0; q + 1 < c.prof_events.size(); q += 2) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, c.prof_events[q], c.prof_events[q + 1]);
      tot += ms;
    }
    if (ms_total) *ms_total = tot;
    if (launches) *launches = (int)(c.prof_events.size() / 2);
  }
  for (cudaEvent_t e : c.prof_events) cudaEventDestroy(e);
  c.prof_events.clear();
  c.profiling = enable != 0;
  return THP_OK;
}

int thp_set_mpole_scales(thp_ctx* h, const double* m) {
  if (!h || !m) return THP_E_INVALID;
  for (int j = 0; j < 4; ++j)
    if (!std::isfinite(m[j])) return THP_E_INVALID;
  for (int j = 0; j < 4; ++j) h->c.mscale[j] = m[j];
  return THP_OK;
}

int thp_empole1(thp_ctx* h, double* em, double* dem) {
  if (!h || (!em && !dem)) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_axes || !c.have_conn) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  int st;
  if ((st = ensure_rpole(h))) return st;
  if ((st = ensure_list(h, false))) return st;
  if (!c.d_grad && (st = cuda_status(cudaMalloc((void**)&c.d_grad, sizeof(double) * 3 * c.n), &c, "alloc gradient")))
    return st;
  c.have_mvirial = false;
  if ((st = launch_empole(c, c.d_grad))) return st;
  c.have_mvirial = c.want_virial;  // totals land in h_mvir with the copies below
  double e = 0.0;
  cudaMemcpyAsync(&e, c.d_em, sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (dem) cudaMemcpyAsync(dem, c.d_grad, sizeof(double) * 3 * c.n, cudaMemcpyDeviceToHost, c.stream);
  if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "empole"))) return st;
  if (!std::isfinite(e)) return THP_E_NAN;
  if (em) *em = e;
  return THP_OK;
}

int thp_set_vdw(thp_ctx* h, const int* cls, int nclass, const double* tables, const int* ired,
                const double* kred, const double* vscale, double vdwcut, double vdwtaper, double ghal, double dhal) {
  if (!h || !cls || !tables || !ired || !kred || !vscale || nclass <= 0 || nclass > 4096) return THP_E_INVALID;
  Ctx& c = h->c;
  const int n = c.n;
  if (!(vdwcut > 0.0) || !(vdwtaper > 0.0) || !std::isfinite(ghal) || !std::isfinite(dhal)) return THP_E_INVALID;
  for (int i = 0; i < n; ++i)
    if (cls[i] < 0 || cls[i] >= nclass || ired[i] < 0 || ired[i] >= n || !std::isfinite(kred[i]))
      return THP_E_INVALID;
  const size_t nt = 4 * (size_t)nclass * nclass;
  for (size_t q = 0; q < nt; ++q)
    if (!std::isfinite(tables[q])) return THP_E_INVALID;
  for (int j = 0; j < 4; ++j)
    if (!std::isfinite(vscale[j])) return THP_E_INVALID;
  if (2.0 * (vdwcut + c.cfg.lbuffer) > std::min(c.cfg.box[0], std::min(c.cfg.box[1], c.cfg.box[2]))) {
    c.last_msg = "vdW cutoff + list buffer exceeds half the box";
    return THP_E_BOX_TOO_SMALL;
  }
  if (set_current_device(c)) return THP_E_CUDA;
  int st;
  auto once = [&](auto** p, size_t count, const char* what) {
    return *p ? THP_OK : cuda_status(cudaMalloc((void**)p, sizeof(**p) * count), &c, what);
  };
  if ((st = once(&c.d_vcls, (size_t)n, "alloc vdw"))) return st;
  if ((st = once(&c.d_vired, (size_t)n, "alloc vdw"))) return st;
  if ((st = once(&c.d_vkred, (size_t)n, "alloc vdw"))) return st;
  if (nt > c.cap_vtab) {
    cudaFree(c.d_vtab);
    c.d_vtab = nullptr;
    c.cap_vtab = 0;
    if ((st = once(&c.d_vtab, nt, "alloc vdw tables"))) return st;
    c.cap_vtab = nt;
  }
  cudaMemcpyAsync(c.d_vcls, cls, sizeof(int) * n, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_vired, ired, sizeof(int) * n, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_vkred, kred, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
  cudaMemcpyAsync(c.d_vtab, tables, sizeof(double) * nt, cudaMemcpyHostToDevice, c.stream);
  if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "upload vdw"))) return st;
  c.have_vlist = false;  // parents, classes or cutoff may have changed
  c.vdw_nclass = nclass;
  c.vdw_cut = vdwcut;
  c.vdw_taper = vdwtaper;
  c.vdw_ghal = ghal;
  c.vdw_dhal = dhal;
  for (int j = 0; j < 4; ++j) c.vdw_scale[j] = vscale[j];
  c.have_vdw = true;
  return THP_OK;
}

int thp_ehal1(thp_ctx* h, double* ev, double* dev) {
  if (!h || (!ev && !dev)) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_vdw || !c.have_conn) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  int st;
  if ((st = ensure_list(h, false))) return st;
  if (!c.d_grad && (st = cuda_status(cudaMalloc((void**)&c.d_grad, sizeof(double) * 3 * c.n), &c, "alloc gradient")))
    return st;
  c.have_vvirial = false;
  if ((st = launch_ehal(c, c.d_grad))) return st;
  c.have_vvirial = c.want_virial;  // totals land in h_vvir with the copies below
  double e = 0.0;
  cudaMemcpyAsync(&e, c.d_ev, sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (dev) cudaMemcpyAsync(dev, c.d_grad, sizeof(double) * 3 * c.n, cudaMemcpyDeviceToHost, c.stream);
  if ((st = check_flags(h))) {  // synchronises the stream
    c.have_vlist = false;       // a list that overflowed is not kept
    return st;
  }
  if (!std::isfinite(e)) return THP_E_NAN;
  if (ev) *ev = e;
  return THP_OK;
}

int thp_set_predictor(thp_ctx* h, int mode) {
  if (!h || mode < THP_PRED_NONE || mode > THP_PRED_LSQR) return THP_E_INVALID;
  h->c.pred_mode = mode;
  h->c.nualt = 0;
  h->c.alt_head = 0;
  return THP_OK;
}

// THP_GUESS_PREDICT after the field (and any re-sort): the predicted dipoles
// when the history is full, else the direct guess (newinduce_pme2.f:165-190).
static int resolve_predict(Ctx& c, int* guess) {
  if (*guess != THP_GUESS_PREDICT) return THP_OK;
  const int r = predictor_guess(c);
  if (r > 0) return r;
  *guess = r == 0 ? THP_GUESS_HOST : THP_GUESS_DIRECT;  // HOST: start from d_mu as written
  return THP_OK;
}

// After a solve that failed on its inputs or in the CG (non-finite
// coordinates, parameters or field, list overflow): the dipoles, the last E0,
// the predictor history and the list may hold values of the failed inputs,
// so the next solve starts cold and rebuilds the list.
static void forget_solution(thp_ctx* h) {
  Ctx& c = h->c;
  c.have_dipoles = false;
  c.have_ef_prev = false;
  c.have_list = false;
  c.nualt = 0;
  c.alt_head = 0;
  h->field_valid = false;
}

static int solve_one(thp_ctx* h, int guess, thp_solve_info* info);

int thp_solve(thp_ctx* h, int guess, thp_solve_info* info) {
  if (!h) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  if (!c.have_params || !c.have_pos || (!c.have_rpole && !c.have_frames)) return THP_E_STATE;
  if (guess < THP_GUESS_DIRECT || guess > THP_GUESS_PREDICT) return THP_E_INVALID;
  if (guess == THP_GUESS_PREVIOUS && !c.have_dipoles) guess = THP_GUESS_DIRECT;
  if (guess == THP_GUESS_HOST && !h->guess_uploaded) return THP_E_STATE;
  const int st = solve_one(h, guess, info);
  if (st != THP_OK && st != THP_E_NOT_CONVERGED) forget_solution(h);
  return st;
}

static int solve_one(thp_ctx* h, int guess, thp_solve_info* info) {
  Ctx& c = h->c;
  cudaEventRecord(c.ev0, c.stream);
  // one host sync per solve: the list/pair overflow bits and the CG scalars
  // are read together after Epol (the predictor's least-squares fit and the
  // host-checked CG chunks, where used, sync on their own)
  int st = compute_field(h, false);
  if (st) return st;
  if ((st = resolve_predict(c, &guess))) return st;
  bool pending = false;
  if ((st = run_pcg_async(c, guess, &pending))) return st;
  h->guess_uploaded = false;
  if ((st = predictor_push(c))) return st;
  if ((st = launch_epol(c))) return st;
  cudaEventRecord(c.ev1, c.stream);
  cudaMemcpyAsync(c.h_cg, c.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(c.h_flags, c.d_flags, sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "solve"))) return st;
  if ((st = flags_status(c))) return st;
  h->field_valid = true;
  st = pcg_status(c);
  if (st && st != THP_E_NOT_CONVERGED) return st;
  h->solved_once = true;
  if (info) {
    info->niter = c.h_cg->niter;
    info->converged = c.h_cg->converged;
    info->resnrm = c.h_cg->resnrm;
    info->epol = c.h_cg->epol;
    info->ene[0] = c.h_cg->ene[0] * kElectric;
    info->ene[1] = c.h_cg->ene[1] * kElectric;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.ev0, c.ev1);
    info->ms_total = ms;
  }
  return st;
}

// E0 and the CG start of one system, fully asynchronous (forced list
// rebuild, no host read-back); the overflow flags are checked after the solve.
static int solve_front_eager(thp_ctx* h, int guess) {
  Ctx& c = h->c;
  int st;
  if (c.have_frames) {
    if ((st = launch_rotpole(c))) return st;
    c.have_rpole = true;
    h->rpole_current = true;
  }
  if ((st = launch_sort_atoms(c))) return st;
  if ((st = launch_gather_sorted(c))) return st;
  h->pos_dirty = false;
  h->rpole_dirty = false;
  if ((st = launch_fields(c, true))) return st;
  c.have_list = true;
  h->field_valid = true;
  if ((st = resolve_predict(c, &guess))) return st;
  return pcg_begin(c, guess);
}

#ifndef THP_FRONT_GRAPH
#define THP_FRONT_GRAPH 1
#endif

// The front of a batched solve (rotpole, sort, list, fields, CG start) as one
// CUDA graph per guess mode and per whether the last dipoles follow a
// re-sort, captured on first use: a batch of many small systems would
// otherwise spend its time in the host's launch calls.  The predictor's
// guess (host-side coefficients) and profiling take the eager path.
static void front_replayed(thp_ctx* h);

static int solve_front_async(thp_ctx* h, int guess) {
  Ctx& c = h->c;
  const int keep_mu = (c.have_perm && c.have_dipoles) ? 1 : 0;
  if (!THP_FRONT_GRAPH || guess < THP_GUESS_DIRECT || guess > THP_GUESS_HOST || c.profiling || !c.stream ||
      c.front_failed)
    return solve_front_eager(h, guess);
  cudaGraphExec_t& ex = c.front_exec[guess][keep_mu];
  if (!ex) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      c.front_failed = true;
      cudaGetLastError();
      return solve_front_eager(h, guess);
    }
    const int st = solve_front_eager(h, guess);
    const cudaError_t e = cudaStreamEndCapture(c.stream, &g);
    if (st || e != cudaSuccess || cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
      ex = nullptr;
      c.front_failed = true;
      cudaGetLastError();
      if (g) cudaGraphDestroy(g);
      if (st) return st;
      return solve_front_eager(h, guess);  // the refused capture did not run: run it now
    }
    cudaGraphDestroy(g);
  }
  front_replayed(h);
  return cuda_status(cudaGraphLaunch(ex, c.stream), &c, "front graph launch");
}

// The host-side state a replayed front leaves behind (what solve_front_eager
// records as it enqueues): rotated multipoles, a fresh sort and list, E0, and
// this solve's E0 kept for the next warm start.
static void front_replayed(thp_ctx* h) {
  Ctx& c = h->c;
  if (c.have_frames) c.have_rpole = h->rpole_current = true;
  c.have_perm = c.have_list = true;
  ++c.sort_epoch;  // the replay re-sorted the atoms: lists in the old numbering are stale
  c.have_ef_prev = true;
  h->pos_dirty = h->rpole_dirty = false;
  h->field_valid = true;
}



// The fronts of a batch: every valid system's E0 and CG start enqueued on
// its own stream (replayed from its front graph); active[i] marks those that
// started.
static void batch_fronts(thp_ctx** hs, int count, int guess, std::vector<int>& st, std::vector<char>& active) {
  for (int i = 0; i < count; ++i) {
    thp_ctx* h = hs[i];
    if (!h) {
      st[i] = THP_E_INVALID;
      continue;
    }
    Ctx& c = h->c;
    if (set_current_device(c)) {
      st[i] = THP_E_CUDA;
      continue;
    }
    if (!c.have_params || !c.have_pos || (!c.have_rpole && !c.have_frames)) {
      st[i] = THP_E_STATE;
      continue;
    }
    int g = guess;
    if (g < THP_GUESS_DIRECT || g > THP_GUESS_PREDICT) {
      st[i] = THP_E_INVALID;
      continue;
    }
    if (g == THP_GUESS_PREVIOUS && !c.have_dipoles) g = THP_GUESS_DIRECT;
    if (g == THP_GUESS_HOST && !h->guess_uploaded) {
      st[i] = THP_E_STATE;
      continue;
    }
    cudaEventRecord(c.ev0, c.stream);
    st[i] = solve_front_async(h, g);
    h->guess_uploaded = false;
    active[i] = st[i] == THP_OK;
  }
}

// The end of a batch once every CG has stopped and its scalars are in h_cg:
// status, predictor, Epol, flags and the per-system results.
static int batch_finish(thp_ctx** hs, int count, std::vector<int>& st, thp_solve_info* infos) {
  for (int i = 0; i < count; ++i) {
    if (st[i]) continue;
    Ctx& c = hs[i]->c;
    set_current_device(c);
    st[i] = pcg_status(c);
    if (st[i] && st[i] != THP_E_NOT_CONVERGED) continue;
    if (int sp = predictor_push(c)) {
      st[i] = sp;
      continue;
    }
    int s2 = launch_epol(c);
    if (s2) {
      st[i] = s2;
      continue;
    }
    cudaEventRecord(c.ev1, c.stream);
    cudaMemcpyAsync(c.h_cg, c.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost, c.stream);
  }
  int worst = THP_OK;
  for (int i = 0; i < count; ++i) {
    if (!st[i] || st[i] == THP_E_NOT_CONVERGED) {
      thp_ctx* h = hs[i];
      Ctx& c = h->c;
      set_current_device(c);
      int f = check_flags(h);  // synchronises the stream
      if (f) st[i] = f;
      h->solved_once = true;
      if (infos) {
        infos[i].niter = c.h_cg->niter;
        infos[i].converged = c.h_cg->converged;
        infos[i].resnrm = c.h_cg->resnrm;
        infos[i].epol = c.h_cg->epol;
        infos[i].ene[0] = c.h_cg->ene[0] * kElectric;
        infos[i].ene[1] = c.h_cg->ene[1] * kElectric;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c.ev0, c.ev1);
        infos[i].ms_total = ms;
      }
    } else if (infos) {
      infos[i] = thp_solve_info{};
    }
    if (st[i] && st[i] != THP_E_NOT_CONVERGED) forget_solution(hs[i]);
    if (st[i] && (worst == THP_OK || worst == THP_E_NOT_CONVERGED)) worst = st[i];
  }
  return worst;
}

int thp_solve_batch(thp_ctx** hs, int count, int guess, thp_solve_info* infos) {
  if (!hs || count <= 0) return THP_E_INVALID;
  std::vector<int> st(count, THP_OK), rounds(count, 0);
  std::vector<char> active(count, 0);
  batch_fronts(hs, count, guess, st, active);
  // the whole CG loop of each system as one graph launch where available;
  // the others take chunk rounds with a host check of the stop flags
  std::vector<char> looped(count, 0);
  for (int i = 0; i < count; ++i) {
    if (!active[i]) continue;
    Ctx& c = hs[i]->c;
    set_current_device(c);
    const int r = pcg_loop_async(c);
    if (r >= 0) {
      active[i] = 0;
      looped[i] = r == 0;
      if (r > 0) st[i] = r;
    }
  }
  for (int i = 0; i < count; ++i) {
    if (!looped[i]) continue;
    Ctx& c = hs[i]->c;
    set_current_device(c);
    st[i] = cuda_status(cudaStreamSynchronize(c.stream), &c, "batch sync");
  }
  for (bool any = true; any;) {
    any = false;
    for (int i = 0; i < count; ++i) {
      if (!active[i]) continue;
      Ctx& c = hs[i]->c;
      set_current_device(c);
      if ((st[i] = pcg_chunk_async(c))) active[i] = 0;
    }
    for (int i = 0; i < count; ++i) {
      if (!active[i]) continue;
      Ctx& c = hs[i]->c;
      set_current_device(c);
      if ((st[i] = cuda_status(cudaStreamSynchronize(c.stream), &c, "batch sync"))) {
        active[i] = 0;
        continue;
      }
      rounds[i] += kCgChunk;
      if (c.h_cg->stop || rounds[i] > c.cfg.politer + kCgChunk) active[i] = 0;
      any |= active[i] != 0;
    }
  }
  return batch_finish(hs, count, st, infos);
}

// ---- batch plans: the CG iterations of many systems as batched kernels ----

struct thp_batch {
  std::vector<thp_ctx*> hs;
  std::vector<Ctx*> cs;
  BatchPlan* plan = nullptr;
  bool no_graph = false;  // the whole-solve graph could not be built: per-system fronts
};

int thp_batch_create(thp_ctx** hs, int count, thp_batch** out) {
  if (!hs || !out || count <= 0) return THP_E_INVALID;
  *out = nullptr;
  thp_batch* b = new thp_batch();
  for (int i = 0; i < count; ++i) {
    if (!hs[i]) {
      delete b;
      return THP_E_INVALID;
    }
    b->hs.push_back(hs[i]);
    b->cs.push_back(&hs[i]->c);
  }
  if (set_current_device(*b->cs[0])) {
    delete b;
    return THP_E_CUDA;
  }
  std::string msg;
  const int st = batch_plan_create(b->cs.data(), count, &b->plan, &msg);
  if (st) {
    b->cs[0]->last_msg = msg;
    delete b;
    return st;
  }
  *out = b;
  return THP_OK;
}

// The whole batched solve as one graph launch (every system's front, the
// batched loop, Epol and the results in mapped host memory), when every
// system takes the same graphable start: guess DIRECT / PREVIOUS / HOST
// after resolution, the same dipole carry, no profiling.  Returns -1 when the
// solve does not qualify (the caller runs the per-system fronts).
static int batch_solve_graph(thp_batch* b, int guess, thp_solve_info* infos) {
  BatchPlan& p = *b->plan;
  const int count = (int)b->hs.size();
  if (b->no_graph || batch_plan_profiling(p) || guess == THP_GUESS_PREDICT || guess < THP_GUESS_DIRECT ||
      guess > THP_GUESS_HOST)
    return -1;
  int g0 = -1, carry0 = -1;
  for (int i = 0; i < count; ++i) {
    thp_ctx* h = b->hs[i];
    Ctx& c = h->c;
    if (!THP_FRONT_GRAPH || c.profiling || !c.stream || c.front_failed || c.pred_mode) return -1;
    if (!c.have_params || !c.have_pos || (!c.have_rpole && !c.have_frames)) return THP_E_STATE;
    int g = guess;
    if (g == THP_GUESS_PREVIOUS && !c.have_dipoles) g = THP_GUESS_DIRECT;
    if (g == THP_GUESS_HOST && !h->guess_uploaded) return THP_E_STATE;
    const int carry = (c.have_perm && c.have_dipoles) ? 1 : 0;
    if ((g0 >= 0 && g != g0) || (carry0 >= 0 && carry != carry0)) return -1;
    g0 = g;
    carry0 = carry;
  }
  const int cand = batch_plan_candidate(p);
  cudaGraphExec_t ex = batch_plan_solve_exec(p, g0, carry0, cand);
  if (!ex) {
    // capture every front (the host state moves as it is enqueued) and build
    std::vector<cudaGraph_t> fronts;
    int st = THP_OK;
    for (int i = 0; i < count && !st; ++i) {
      Ctx& c = b->hs[i]->c;
      set_current_device(c);
      if (cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        st = -1;
        break;
      }
      const int se = solve_front_eager(b->hs[i], g0);
      cudaGraph_t gr = nullptr;
      const cudaError_t e = cudaStreamEndCapture(c.stream, &gr);
      if (se || e != cudaSuccess) {
        cudaGetLastError();
        if (gr) cudaGraphDestroy(gr);
        st = se ? se : -1;
        break;
      }
      fronts.push_back(gr);
    }
    if (!st) st = batch_plan_make_solve_exec(p, fronts, g0, carry0, cand) ? -1 : THP_OK;
    for (cudaGraph_t gr : fronts) cudaGraphDestroy(gr);
    if (st) {
      // nothing of the captured fronts ran: run them eagerly on the usual path
      // (cold: a capture may have moved a context's host state)
      for (int i = 0; i < count; ++i) forget_solution(b->hs[i]);
      b->no_graph = true;
      return -1;
    }
    ex = batch_plan_solve_exec(p, g0, carry0, cand);
  } else {
    for (int i = 0; i < count; ++i) front_replayed(b->hs[i]);
  }
  for (int i = 0; i < count; ++i) b->hs[i]->guess_uploaded = false;
  std::vector<const CgScalars*> cgs(count);
  std::vector<const int*> fls(count);
  float ms = 0.f;
  const int sr = batch_plan_run_solve(p, ex, cgs.data(), fls.data(), &ms);
  int worst = THP_OK;
  for (int i = 0; i < count; ++i) {
    thp_ctx* h = b->hs[i];
    Ctx& c = h->c;
    int st = sr;
    if (!st) {
      *c.h_cg = *cgs[i];
      *c.h_flags = *fls[i];
      st = flags_status(c);
      if (!st) st = pcg_status(c);
    }
    if (!st || st == THP_E_NOT_CONVERGED) {
      h->solved_once = true;
      if (infos) {
        infos[i].niter = c.h_cg->niter;
        infos[i].converged = c.h_cg->converged;
        infos[i].resnrm = c.h_cg->resnrm;
        infos[i].epol = c.h_cg->epol;
        infos[i].ene[0] = c.h_cg->ene[0] * kElectric;
        infos[i].ene[1] = c.h_cg->ene[1] * kElectric;
        infos[i].ms_total = ms;
      }
    } else {
      if (infos) infos[i] = thp_solve_info{};
      forget_solution(h);
    }
    if (st && (worst == THP_OK || worst == THP_E_NOT_CONVERGED)) worst = st;
  }
  if (!sr) batch_plan_finish(p);
  return worst;
}

int thp_batch_solve(thp_batch* b, int guess, thp_solve_info* infos) {
  if (!b) return THP_E_INVALID;
  const int count = (int)b->hs.size();
  thp_ctx** hs = b->hs.data();
  if (int s = batch_plan_check(*b->plan, b->cs.data())) return s;
  if (set_current_device(*b->cs[0])) return THP_E_CUDA;
  const int gs = batch_solve_graph(b, guess, infos);
  if (gs >= 0) return gs;
  std::vector<int> st(count, THP_OK);
  std::vector<char> active(count, 0);
  batch_fronts(hs, count, guess, st, active);
  for (int i = 0; i < count; ++i) {
    Ctx& c = *b->cs[i];
    if (active[i]) continue;
    // a system whose front did not start takes no part in the loop
    set_current_device(c);
    cudaMemsetAsync(c.d_cg, 0, sizeof(CgScalars), c.stream);
    cudaMemsetAsync(&c.d_cg->stop, 1, sizeof(int), c.stream);
  }
  const int sl = batch_plan_loop(*b->plan, b->cs.data());
  for (int i = 0; i < count; ++i) {
    Ctx& c = *b->cs[i];
    set_current_device(c);
    if (sl && !st[i]) st[i] = sl;
    cudaMemcpyAsync(c.h_cg, c.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost, c.stream);
    const int ss = cuda_status(cudaStreamSynchronize(c.stream), &c, "batch sync");
    if (ss && !st[i]) st[i] = ss;
  }
  if (!sl) batch_plan_finish(*b->plan);
  return batch_finish(hs, count, st, infos);
}

int thp_batch_tuning(thp_batch* b, int* blocks_per_sm, int* matvec_atoms, double* ms_per_solve) {
  if (!b || !blocks_per_sm || !matvec_atoms) return THP_E_INVALID;
  float ms = 0.f;
  const int st = batch_plan_tuning(*b->plan, blocks_per_sm, matvec_atoms, &ms);
  if (ms_per_solve) *ms_per_solve = ms;
  return st;
}

int thp_batch_profile(thp_batch* b, int enable, double* ms, int* iterations) {
  if (!b) return THP_E_INVALID;
  return batch_plan_profile(*b->plan, enable, ms, iterations);
}

int thp_batch_destroy(thp_batch* b) {
  if (!b) return THP_E_INVALID;
  batch_plan_destroy(b->plan);
  delete b;
  return THP_OK;
}

int thp_get_dipoles(thp_ctx* h, double* uind, double* uinp) {
  if (!h) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_dipoles) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  // laid out on the device as the caller's two [n][3] arrays, then copied
  // straight into them (a DMA when the caller's buffers are pinned)
  int st = launch_split_dipoles(c, c.d_mu, c.d_tmp6);
  if (st) return st;
  const size_t b = sizeof(double) * 3 * c.n;
  if (uind) cudaMemcpyAsync(uind, c.d_tmp6, b, cudaMemcpyDeviceToHost, c.stream);
  if (uinp) cudaMemcpyAsync(uinp, c.d_tmp6 + 3 * (size_t)c.n, b, cudaMemcpyDeviceToHost, c.stream);
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "get dipoles");
}

int thp_get_gradient_device(thp_ctx* h, double* d_dep) {
  if (!h || !d_dep) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_axes || !c.have_dipoles || !h->field_valid || !h->solved_once) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  c.have_virial = false;
  const int st = launch_forces(c, d_dep);
  c.have_virial = st == THP_OK && c.want_virial;  // totals land in h_vir when the stream reaches them
  return st;
}

int thp_get_empole_virial(thp_ctx* h, int form, double* vir) {
  if (!h || !vir || form < 0 || form > 1) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_mvirial) return THP_E_STATE;
  double v[6];
  for (int q = 0; q < 6; ++q) v[q] = c.h_mvir[q] + (form == 1 ? c.h_mvir[6 + q] : 0.0);
  const double t[9] = {v[0], v[1], v[2], v[1], v[3], v[4], v[2], v[4], v[5]};
  std::memcpy(vir, t, sizeof(t));
  return THP_OK;
}

int thp_get_ehal_virial(thp_ctx* h, double* vir) {
  if (!h || !vir) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_vvirial) return THP_E_STATE;
  const double* v = c.h_vvir;
  const double t[9] = {v[0], v[1], v[2], v[1], v[3], v[4], v[2], v[4], v[5]};
  std::memcpy(vir, t, sizeof(t));
  return THP_OK;
}

int thp_set_virial(thp_ctx* h, int on) {
  if (!h) return THP_E_INVALID;
  h->c.want_virial = on != 0;
  return THP_OK;
}

int thp_get_virial(thp_ctx* h, int form, double* vir) {
  if (!h || !vir || form < 0 || form > 1) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_virial) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  int st = cuda_status(cudaStreamSynchronize(c.stream), &c, "virial");
  if (st) return st;
  double v[6];
  for (int q = 0; q < 6; ++q) v[q] = c.h_vir[q] + (form == 1 ? c.h_vir[6 + q] : 0.0);
  const double t[9] = {v[0], v[1], v[2], v[1], v[3], v[4], v[2], v[4], v[5]};
  std::memcpy(vir, t, sizeof(t));
  return THP_OK;
}

int thp_get_gradient(thp_ctx* h, double* dep, double* ep) {
  if (!h || !dep) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  if (!c.d_grad) {
    int st = cuda_status(cudaMalloc((void**)&c.d_grad, sizeof(double) * 3 * c.n), &c, "alloc gradient");
    if (st) return st;
  }
  int st = thp_get_gradient_device(h, c.d_grad);
  if (st) return st;
  cudaMemcpyAsync(dep, c.d_grad, sizeof(double) * 3 * c.n, cudaMemcpyDeviceToHost, c.stream);
  if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "gradient"))) return st;
  if (ep) *ep = c.h_cg->epol;
  return THP_OK;
}

int thp_get_positions(thp_ctx* h, double* x, double* y, double* z) {
  if (!h || !x || !y || !z) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_pos) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  const size_t n = c.n;
  cudaMemcpyAsync(x, c.d_xyz_orig, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(y, c.d_xyz_orig + n, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream);
  cudaMemcpyAsync(z, c.d_xyz_orig + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream);
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "get positions");
}

int thp_md_verlet(thp_ctx* h, int nsteps, double dt, const double* mass, double* vel, double* energies,
                  int* niters) {
  if (!h || !mass || !vel || nsteps < 0 || !(dt > 0.0)) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_axes || !c.have_params || !c.have_pos) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  const size_t n = c.n;
  for (size_t i = 0; i < n; ++i)
    if (!(mass[i] > 0.0)) return THP_E_INVALID;
  double *d_mass = nullptr, *d_vel = nullptr, *d_grad = nullptr, *d_scr = nullptr;
  const size_t nscr = (n + 255) / 256 + 2;
  int st = cuda_status(cudaMalloc((void**)&d_mass, sizeof(double) * n), &c, "md alloc");
  if (!st) st = cuda_status(cudaMalloc((void**)&d_vel, sizeof(double) * 3 * n), &c, "md alloc");
  if (!st) st = cuda_status(cudaMalloc((void**)&d_grad, sizeof(double) * 3 * n), &c, "md alloc");
  if (!st) st = cuda_status(cudaMalloc((void**)&d_scr, sizeof(double) * nscr), &c, "md alloc");
  if (!st) {
    cudaMemcpyAsync(d_mass, mass, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream);
    cudaMemcpyAsync(d_vel, vel, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c.stream);
    st = cuda_status(cudaGetLastError(), &c, "md upload");
  }
  const int guess = c.pred_mode ? THP_GUESS_PREDICT : THP_GUESS_PREVIOUS;
  thp_solve_info info;
  // gradient at the starting positions (mdinit's first gradient call)
  if (!st) {
    st = thp_solve(h, guess, &info);
    if (st == THP_E_NOT_CONVERGED) st = THP_OK;
  }
  if (!st) st = launch_forces(c, d_grad);
  for (int step = 0; step < nsteps && !st; ++step) {
    if ((st = launch_kick(c, 0.5 * dt, d_mass, d_grad, d_vel))) break;
    if ((st = launch_drift(c, dt, d_vel))) break;
    h->pos_dirty = true;
    h->rpole_current = false;
    h->field_valid = false;
    c.have_coef = false;
    if (c.have_frames) h->rpole_dirty = true;
    st = thp_solve(h, guess, &info);
    if (st && st != THP_E_NOT_CONVERGED) break;
    st = THP_OK;
    if ((st = launch_forces(c, d_grad))) break;
    if ((st = launch_kick(c, 0.5 * dt, d_mass, d_grad, d_vel))) break;
    if ((st = launch_ekin(c, d_mass, d_vel, d_scr))) break;
    double ek = 0.0;
    cudaMemcpyAsync(&ek, d_scr, sizeof(double), cudaMemcpyDeviceToHost, c.stream);
    if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "md step"))) break;
    if (energies) {
      energies[3 * (size_t)step] = info.epol;
      energies[3 * (size_t)step + 1] = ek;
      energies[3 * (size_t)step + 2] = info.epol + ek;
    }
    if (niters) niters[step] = info.niter;
  }
  if (!st) {
    cudaMemcpyAsync(vel, d_vel, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c.stream);
    st = cuda_status(cudaStreamSynchronize(c.stream), &c, "md download");
  }
  cudaStreamSynchronize(c.stream);
  cudaFree(d_mass);
  cudaFree(d_vel);
  cudaFree(d_grad);
  cudaFree(d_scr);
  return st;
}

int thp_get_field(thp_ctx* h, double* ef) {
  if (!h || !ef) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!h->field_valid) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  int st = launch_to_orig6(c, c.d_ef, c.d_tmp6, 2);
  if (st) return st;
  cudaMemcpyAsync(ef, c.d_tmp6, sizeof(double) * 6 * c.n, cudaMemcpyDeviceToHost, c.stream);
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "get field");
}

int thp_get_rpole(thp_ctx* h, double* rpole) {
  if (!h || !rpole) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  int st = ensure_rpole(h);
  if (st) return st;
  cudaMemcpyAsync(rpole, c.d_rpole_orig, sizeof(double) * 13 * c.n, cudaMemcpyDeviceToHost, c.stream);
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "get rpole");
}

int thp_get_nblist(thp_ctx* h, int maxelst, int* nelst, int* elst) {
  if (!h || !nelst || !elst || maxelst <= 0) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  int st = ensure_list(h, false);
  if (st) return st;
  int *dn = nullptr, *de = nullptr;
  if ((st = dmalloc(c, &dn, c.n, "export"))) return st;
  if ((st = dmalloc(c, &de, (size_t)c.n * maxelst, "export"))) {
    cudaFree(dn);
    return st;
  }
  st = launch_export_list(c, maxelst, dn, de);
  if (!st) {
    cudaMemcpyAsync(nelst, dn, sizeof(int) * c.n, cudaMemcpyDeviceToHost, c.stream);
    cudaMemcpyAsync(elst, de, sizeof(int) * (size_t)c.n * maxelst, cudaMemcpyDeviceToHost, c.stream);
    st = check_flags(h);
  }
  cudaFree(dn);
  cudaFree(de);
  return st;
}

int thp_get_vlist(thp_ctx* h, int maxvlst, int* nvlst, int* vlst) {
  if (!h || !nvlst || !vlst || maxvlst <= 0) return THP_E_INVALID;
  Ctx& c = h->c;
  if (!c.have_vdw) return THP_E_STATE;
  if (set_current_device(c)) return THP_E_CUDA;
  int st = ensure_list(h, false);
  if (!st) st = launch_vdw_list(c);
  if (st) return st;
  int *dn = nullptr, *de = nullptr;
  if ((st = dmalloc(c, &dn, c.n, "export"))) return st;
  if ((st = dmalloc(c, &de, (size_t)c.n * maxvlst, "export"))) {
    cudaFree(dn);
    return st;
  }
  st = launch_export_pairs(c, c.d_vnnb, c.d_vnb, c.maxvnb, maxvlst, dn, de);
  if (!st) {
    cudaMemcpyAsync(nvlst, dn, sizeof(int) * c.n, cudaMemcpyDeviceToHost, c.stream);
    cudaMemcpyAsync(vlst, de, sizeof(int) * (size_t)c.n * maxvlst, cudaMemcpyDeviceToHost, c.stream);
    st = check_flags(h);
    if (st) c.have_vlist = false;  // the device list may have overflowed too
  }
  cudaFree(dn);
  cudaFree(de);
  return st;
}

int thp_bind_vlist(thp_ctx* h, int* nvlst, int* vlst, int maxvlst) {
  if (!h || maxvlst < 0) return THP_E_INVALID;
  h->c.bnvlst = nvlst;
  h->c.bvlst = vlst;
  h->c.bmaxvlst = maxvlst;
  return THP_OK;
}

int thp_tmatxb(thp_ctx* h, int nrhs, int dodiag, const double* mu, double* efi) {
  if (!h || !mu || !efi || nrhs < 1 || nrhs > 2) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  int st = ensure_coef(h);
  if (st) return st;
  const size_t n = c.n;
  cudaMemcpyAsync(c.d_tmp6b, mu, sizeof(double) * 3 * nrhs * n, cudaMemcpyHostToDevice, c.stream);
  if ((st = launch_to_sorted6(c, c.d_tmp6b, c.d_tmp6, nrhs))) return st;
  if ((st = launch_tmatxb(c, c.d_tmp6, c.d_dip, dodiag != 0))) return st;
  if ((st = launch_to_orig6(c, c.d_dip, c.d_tmp6b, nrhs))) return st;
  cudaMemcpyAsync(efi, c.d_tmp6b, sizeof(double) * 3 * nrhs * n, cudaMemcpyDeviceToHost, c.stream);
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "tmatxb");
}

int thp_efld0_direct(thp_ctx* h, int nrhs, double* ef) {
  if (!h || !ef || nrhs < 1 || nrhs > 2) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  int st;
  if ((st = ensure_rpole(h))) return st;
  if ((st = ensure_list(h, false))) return st;
  if ((st = launch_efld0_coef(c, true))) return st;
  h->field_valid = false;  // d_ef holds only the direct part now
  if ((st = check_flags(h))) return st;
  if ((st = launch_to_orig6(c, c.d_ef, c.d_tmp6, 2))) return st;
  std::vector<double> buf((size_t)6 * c.n);
  cudaMemcpyAsync(buf.data(), c.d_tmp6, sizeof(double) * 6 * c.n, cudaMemcpyDeviceToHost, c.stream);
  if ((st = cuda_status(cudaStreamSynchronize(c.stream), &c, "efld0 direct"))) return st;
  for (int i = 0; i < c.n; ++i)
    for (int r = 0; r < nrhs; ++r)
      for (int j = 0; j < 3; ++j) ef[((size_t)i * nrhs + r) * 3 + j] += buf[6 * (size_t)i + 3 * r + j];
  return THP_OK;
}

int thp_efld0_recip(thp_ctx* h, double* cphi) {
  if (!h || !cphi) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  int st;
  if ((st = ensure_rpole(h))) return st;
  if ((st = ensure_list(h, false))) return st;
  double* d10 = nullptr;
  if ((st = dmalloc(c, &d10, (size_t)10 * c.n, "cphi10"))) return st;
  st = launch_efld0_recip_ex(c, d10, false);
  std::vector<double> buf((size_t)10 * c.n);
  std::vector<int> perm(c.n);
  if (!st) {
    cudaMemcpyAsync(buf.data(), d10, sizeof(double) * 10 * c.n, cudaMemcpyDeviceToHost, c.stream);
    cudaMemcpyAsync(perm.data(), c.d_perm, sizeof(int) * c.n, cudaMemcpyDeviceToHost, c.stream);
    st = cuda_status(cudaStreamSynchronize(c.stream), &c, "efld0 recip");
  }
  cudaFree(d10);
  if (st) return st;
  for (int s = 0; s < c.n; ++s) std::memcpy(cphi + (size_t)perm[s] * 10, &buf[(size_t)s * 10], sizeof(double) * 10);
  return THP_OK;
}

int thp_tmatxbrecip(thp_ctx* h, int nrhs, const double* mu, double* dipfield) {
  if (!h || !mu || !dipfield || nrhs < 1 || nrhs > 2) return THP_E_INVALID;
  Ctx& c = h->c;
  if (set_current_device(c)) return THP_E_CUDA;
  int st = ensure_list(h, false);
  if (st) return st;
  const size_t n = c.n;
  cudaMemcpyAsync(c.d_tmp6b, mu, sizeof(double) * 3 * nrhs * n, cudaMemcpyHostToDevice, c.stream);
  if ((st = launch_to_sorted6(c, c.d_tmp6b, c.d_tmp6, nrhs))) return st;
  if ((st = launch_pme_dipole(c, c.d_tmp6, c.d_dip, 0))) return st;
  if ((st = launch_to_orig6(c, c.d_dip, c.d_tmp6b, nrhs))) return st;
  cudaMemcpyAsync(dipfield, c.d_tmp6b, sizeof(double) * 3 * nrhs * n, cudaMemcpyDeviceToHost, c.stream);
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "tmatxbrecip");
}

int thp_solve_host(thp_ctx* h, const double* x, const double* y, const double* z, const double* rpole,
                   double* uind, double* uinp, thp_solve_info* info) {
  int st = thp::upload_positions(h, x, y, z, false);
  if (st) return st;
  if (rpole && (st = thp_set_rpole(h, rpole))) return st;
  st = thp_solve(h, THP_GUESS_DIRECT, info);
  if (st && st != THP_E_NOT_CONVERGED) return st;
  int st2 = thp_get_dipoles(h, uind, uinp);
  return st2 ? st2 : st;
}

// ---- Fortran drop-ins ------------------------------------------------------

int thp_bind_state(thp_ctx* h, double* x, double* y, double* z, double* rpole, double* uind, double* uinp,
                   int* nelst, int* elst, int maxelst, double* ep) {
  if (!h) return THP_E_INVALID;
  Ctx& c = h->c;
  c.bx = x;
  c.by = y;
  c.bz = z;
  c.brpole = rpole;
  c.buind = uind;
  c.buinp = uinp;
  c.bnelst = nelst;
  c.belst = elst;
  c.bmaxelst = maxelst;
  c.bep = ep;
  g_current = h;
  return THP_OK;
}

int thp_last_error(void) { return g_last_error; }

int thp_bind_grid(thp_ctx* h, double* qgrid) {
  if (!h) return THP_E_INVALID;
  h->c.bqgrid = qgrid;
  return THP_OK;
}

int thp_bind_virial(thp_ctx* h, double* vir) {
  if (!h) return THP_E_INVALID;
  h->c.bvir = vir;
  return THP_OK;
}

int thp_bind_gradient(thp_ctx* h, double* dep) {
  if (!h) return THP_E_INVALID;
  h->c.bdep = dep;
  return THP_OK;
}

int thp_bind_vdw(thp_ctx* h, double* ev, double* dev) {
  if (!h) return THP_E_INVALID;
  h->c.bev = ev;
  h->c.bdev = dev;
  return THP_OK;
}

int thp_bind_mpole(thp_ctx* h, double* em, double* dem) {
  if (!h) return THP_E_INVALID;
  h->c.bem = em;
  h->c.bdem = dem;
  return THP_OK;
}

static int sync_bound_inputs(thp_ctx* h) {
  Ctx& c = h->c;
  if (!c.bx || !c.by || !c.bz) return THP_E_STATE;
  int st = thp_set_positions(h, c.bx, c.by, c.bz);
  if (st) return st;
  if (c.brpole) st = thp_set_rpole(h, c.brpole);
  return st;
}

void mlistcell_(void) {
  thp_ctx* h = g_current;
  if (!h) {
    g_last_error = THP_E_STATE;
    return;
  }
  int st = sync_bound_inputs(h);
  if (!st) st = ensure_list(h, true);
  if (!st && h->c.bnelst && h->c.belst) {
    st = thp_get_nblist(h, h->c.bmaxelst, h->c.bnelst, h->c.belst);
    if (!st) {  // Fortran pole indices are 1-based
      const size_t n = h->c.n, m = h->c.bmaxelst;
      for (size_t i = 0; i < n; ++i)
        for (int j = 0; j < h->c.bnelst[i]; ++j) h->c.belst[i * m + j] += 1;
    }
  }
  g_last_error = st;
}

// nblist.f:1148 -- with a vdW description and a bound vdW list, the vdW list
// of vlistcell (reduced sites, vdwcut + lbuffer); otherwise the polarization
// list under this name
void vlistcell_(void) {
  thp_ctx* h = g_current;
  if (!h || !h->c.have_vdw || !h->c.bnvlst || !h->c.bvlst) {
    mlistcell_();
    return;
  }
  int st = sync_bound_inputs(h);
  if (!st) st = thp_get_vlist(h, h->c.bmaxvlst, h->c.bnvlst, h->c.bvlst);
  if (!st) {  // Fortran atom numbers are 1-based
    const size_t n = h->c.n, m = h->c.bmaxvlst;
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < h->c.bnvlst[i]; ++j) h->c.bvlst[i * m + j] += 1;
  }
  g_last_error = st;
}

void newinduce_pme2_(void) {
  thp_ctx* h = g_current;
  if (!h) {
    g_last_error = THP_E_STATE;
    return;
  }
  int st = sync_bound_inputs(h);
  thp_solve_info info;
  if (!st) st = thp_solve(h, THP_GUESS_DIRECT, &info);
  if ((!st || st == THP_E_NOT_CONVERGED) && h->c.buind) {
    int st2 = thp_get_dipoles(h, h->c.buind, h->c.buinp);
    if (st2) st = st2;
  }
  g_last_error = st;
}

void epolar_(void) {
  thp_ctx* h = g_current;
  if (!h) {
    g_last_error = THP_E_STATE;
    return;
  }
  int st = sync_bound_inputs(h);
  thp_solve_info info;
  if (!st) st = thp_solve(h, THP_GUESS_DIRECT, &info);
  if (!st || st == THP_E_NOT_CONVERGED) {
    if (h->c.bep) *h->c.bep = info.epol;
    if (h->c.buind) thp_get_dipoles(h, h->c.buind, h->c.buinp);
  }
  g_last_error = st;
}

void epolar1_(void) {
  thp_ctx* h = g_current;
  if (!h) {
    g_last_error = THP_E_STATE;
    return;
  }
  int st = sync_bound_inputs(h);
  thp_solve_info info;
  if (!st) st = thp_solve(h, THP_GUESS_DIRECT, &info);
  if (!st || st == THP_E_NOT_CONVERGED) {
    int st2 = THP_OK;
    if (h->c.bdep) {
      h->c.want_virial = h->c.bvir != nullptr;
      st2 = thp_get_gradient(h, h->c.bdep, nullptr);
      if (!st2 && h->c.bvir) {  // epolar1c adds into vir (epolar1.f:2334-2342)
        double v[9];
        st2 = thp_get_virial(h, 0, v);
        for (int q = 0; !st2 && q < 9; ++q) h->c.bvir[q] += v[q];
      }
    }
    if (!st2 && h->c.bep) *h->c.bep = info.epol;
    if (!st2 && h->c.buind) st2 = thp_get_dipoles(h, h->c.buind, h->c.buinp);
    if (st2) st = st2;
  }
  g_last_error = st;
}

void empole1_(void) {
  thp_ctx* h = g_current;
  if (!h) {
    g_last_error = THP_E_STATE;
    return;
  }
  int st = sync_bound_inputs(h);
  double em = 0.0;
  h->c.want_virial = h->c.bvir != nullptr;
  if (!st) st = thp_empole1(h, &em, h->c.bdem);
  if (!st && h->c.bem) *h->c.bem = em;
  if (!st && h->c.bvir) {  // empole1c adds into vir (empole1.f:820-828, 1435-1443)
    double v[9];
    st = thp_get_empole_virial(h, 0, v);
    for (int q = 0; !st && q < 9; ++q) h->c.bvir[q] += v[q];
  }
  g_last_error = st;
}

void ehal1_(void) {
  thp_ctx* h = g_current;
  if (!h) {
    g_last_error = THP_E_STATE;
    return;
  }
  int st = sync_bound_inputs(h);
  double ev = 0.0;
  h->c.want_virial = h->c.bvir != nullptr;
  if (!st) st = thp_ehal1(h, &ev, h->c.bdev);
  if (!st && h->c.bev) *h->c.bev = ev;
  if (!st && h->c.bvir) {  // ehal1c adds into vir (ehal1.f:438-446)
    double v[9];
    st = thp_get_ehal_virial(h, v);
    for (int q = 0; !st && q < 9; ++q) h->c.bvir[q] += v[q];
  }
  g_last_error = st;
}

// Staging for the per-site PME routines: the FP64 grid, the 0-based site
// numbers (validated) and `doubles` values per site, on the device.
static int site_staging(thp_ctx* h, int nsites, const int* isite, int doubles, int** d_site, double** d_vals) {
  Ctx& c = h->c;
  if (nsites < 0 || (nsites > 0 && !isite)) return THP_E_INVALID;
  if (!c.have_pos) return THP_E_STATE;
  std::vector<int> s0(std::max(nsites, 1));
  for (int q = 0; q < nsites; ++q) {
    if (isite[q] < 1 || isite[q] > c.n) return THP_E_INVALID;
    s0[q] = isite[q] - 1;  // Fortran atom numbers are 1-based
  }
  if (!c.d_sgrid) {
    int st = cuda_status(cudaMalloc((void**)&c.d_sgrid, sizeof(cufftDoubleComplex) * c.ngrid), &c, "site grid");
    if (st) return st;
  }
  const size_t need = ((size_t)nsites * 4 + 255) / 256 * 256 + sizeof(double) * doubles * (size_t)std::max(nsites, 1);
  if (c.sscratch_bytes < need) {
    cudaFree(c.d_sscratch);
    c.d_sscratch = nullptr;
    c.sscratch_bytes = 0;
    int st = cuda_status(cudaMalloc(&c.d_sscratch, need), &c, "site scratch");
    if (st) return st;
    c.sscratch_bytes = need;
  }
  *d_site = static_cast<int*>(c.d_sscratch);
  *d_vals = reinterpret_cast<double*>(static_cast<char*>(c.d_sscratch) + ((size_t)nsites * 4 + 255) / 256 * 256);
  cudaMemcpyAsync(*d_site, s0.data(), sizeof(int) * nsites, cudaMemcpyHostToDevice, c.stream);
  return cuda_status(cudaStreamSynchronize(c.stream), &c, "site upload");
}

void grid_uind_sites_(const int* nsites, const int* isite, const double* fuind, const double* fuinp, double* qgrid) {
  thp_ctx* h = g_current;
  if (!h || !nsites || !qgrid || (*nsites > 0 && (!fuind || !fuinp))) {
    g_last_error = h ? THP_E_INVALID : THP_E_STATE;
    return;
  }
  Ctx& c = h->c;
  const int ns = *nsites;
  int st = c.bx ? thp_set_positions(h, c.bx, c.by, c.bz) : THP_OK;
  int* d_site = nullptr;
  double* d_fu = nullptr;
  if (!st) st = site_staging(h, ns, isite, 6, &d_site, &d_fu);
  if (!st) {
    cudaMemcpyAsync(d_fu, fuind, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, c.stream);
    cudaMemcpyAsync(d_fu + 3 * (size_t)ns, fuinp, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, c.stream);
    cudaMemsetAsync(c.d_sgrid, 0, sizeof(cufftDoubleComplex) * c.ngrid, c.stream);
    st = launch_grid_uind_sites(c, ns, d_site, d_fu, d_fu + 3 * (size_t)ns, c.d_sgrid);
  }
  if (!st) {
    c.h_sgrid.resize(2 * c.ngrid);
    cudaMemcpyAsync(c.h_sgrid.data(), c.d_sgrid, sizeof(cufftDoubleComplex) * c.ngrid, cudaMemcpyDeviceToHost,
                    c.stream);
    st = cuda_status(cudaStreamSynchronize(c.stream), &c, "grid_uind_sites");
  }
  if (!st)  // grid_uind_site adds into qgrid2loc
    for (size_t q = 0; q < 2 * c.ngrid; ++q) qgrid[q] += c.h_sgrid[q];
  g_last_error = st;
}

void fphi_uind_sites_(const int* nsites, const int* isite, const double* qgrid, double* fdip_phi1, double* fdip_phi2,
                      double* fdip_sum_phi) {
  thp_ctx* h = g_current;
  if (!h || !nsites || !qgrid || (*nsites > 0 && (!fdip_phi1 || !fdip_phi2 || !fdip_sum_phi))) {
    g_last_error = h ? THP_E_INVALID : THP_E_STATE;
    return;
  }
  Ctx& c = h->c;
  const int ns = *nsites;
  int st = c.bx ? thp_set_positions(h, c.bx, c.by, c.bz) : THP_OK;
  int* d_site = nullptr;
  double* d_out = nullptr;
  if (!st) st = site_staging(h, ns, isite, 40, &d_site, &d_out);
  if (!st) {
    cudaMemcpyAsync(c.d_sgrid, qgrid, sizeof(cufftDoubleComplex) * c.ngrid, cudaMemcpyHostToDevice, c.stream);
    st = launch_fphi_uind_sites(c, ns, d_site, c.d_sgrid, d_out, d_out + 10 * (size_t)ns, d_out + 20 * (size_t)ns);
  }
  if (!st) {
    cudaMemcpyAsync(fdip_phi1, d_out, sizeof(double) * 10 * ns, cudaMemcpyDeviceToHost, c.stream);
    cudaMemcpyAsync(fdip_phi2, d_out + 10 * (size_t)ns, sizeof(double) * 10 * ns, cudaMemcpyDeviceToHost, c.stream);
    cudaMemcpyAsync(fdip_sum_phi, d_out + 20 * (size_t)ns, sizeof(double) * 20 * ns, cudaMemcpyDeviceToHost,
                    c.stream);
    st = cuda_status(cudaStreamSynchronize(c.stream), &c, "fphi_uind_sites");
  }
  g_last_error = st;
}

void grid_uind_site_(const int* isite, const int* impi, const double* fuind, const double* fuinp,
                     double* qgrid2loc) {
  (void)impi;
  const int one = 1;
  grid_uind_sites_(&one, isite, fuind, fuinp, qgrid2loc);
}

void fphi_uind_site_(const int* isite, const int* impi, double* fdip_phi1, double* fdip_phi2,
                     double* fdip_sum_phi) {
  (void)impi;
  const int one = 1;
  if (!g_current || !g_current->c.bqgrid) {
    g_last_error = THP_E_STATE;
    return;
  }
  fphi_uind_sites_(&one, isite, g_current->c.bqgrid, fdip_phi1, fdip_phi2, fdip_sum_phi);
}

void tmatxb_pme_(const int* nrhs, const int* dodiag, const double* mu, double* efi) {
  if (!g_current) {
    g_last_error = THP_E_STATE;
    return;
  }
  g_last_error = thp_tmatxb(g_current, *nrhs, *dodiag, mu, efi);
}

void efld0_direct_(const int* nrhs, double* ef) {
  if (!g_current) {
    g_last_error = THP_E_STATE;
    return;
  }
  g_last_error = thp_efld0_direct(g_current, *nrhs, ef);
}

void efld0_recip_(double* cphi) {
  if (!g_current) {
    g_last_error = THP_E_STATE;
    return;
  }
  g_last_error = thp_efld0_recip(g_current, cphi);
}

void tmatxbrecip_(const double* mu, const double* murec, const int* nrhs, double* dipfield, double* dipfieldbis) {
  (void)murec;
  (void)dipfieldbis;
  if (!g_current) {
    g_last_error = THP_E_STATE;
    return;
  }
  g_last_error = thp_tmatxbrecip(g_current, *nrhs, mu, dipfield);
}

void inducepcg_pme2_(void (*matvec)(const int*, const int*, const double*, double*), const int* nrhs,
                     const int* precnd, const double* ef, double* mu, double* murec) {
  (void)murec;
  thp_ctx* h = g_current;
  if (!h || !matvec || !nrhs || !ef || !mu) {
    g_last_error = THP_E_STATE;
    return;
  }
  Ctx& c = h->c;
  const int nr = *nrhs;
  const size_t n = c.n, nv = n * 3 * nr;
  int st = ensure_coef(h);
  if (st) {
    g_last_error = st;
    return;
  }
  if ((matvec == tmatxb_pme_ || matvec == thp_f_tmatxb_pme) && nr == 2 && *precnd) {
    // device loop on the caller's E0 and guess
    cudaMemcpyAsync(c.d_tmp6, ef, sizeof(double) * nv, cudaMemcpyHostToDevice, c.stream);
    st = launch_to_sorted6(c, c.d_tmp6, c.d_ef, 2);
    cudaMemcpyAsync(c.d_tmp6b, mu, sizeof(double) * nv, cudaMemcpyHostToDevice, c.stream);
    if (!st) st = launch_to_sorted6(c, c.d_tmp6b, c.d_mu, 2);
    if (!st) st = run_pcg(c, THP_GUESS_HOST);
    if (!st || st == THP_E_NOT_CONVERGED) {
      int st2 = launch_to_orig6(c, c.d_mu, c.d_tmp6, 2);
      cudaMemcpyAsync(mu, c.d_tmp6, sizeof(double) * nv, cudaMemcpyDeviceToHost, c.stream);
      cudaStreamSynchronize(c.stream);
      if (st2) st = st2;
    }
    h->field_valid = false;
    g_last_error = st;
    return;
  }
  // host loop with the caller's matvec (newinduce_pme2.f:285-636, same recurrences)
  std::vector<double> res(nv), hh(nv), pp(nv), zr(nv), dip(nv), diag(n);
  for (size_t i = 0; i < n; ++i) {
    double p = c.h_polarity.empty() ? 1.0 : c.h_polarity[i];
    diag[i] = *precnd ? (p == 0.0 ? kTinyPol : p) : 1.0;
  }
  const double a = c.cfg.aewald, term = (4.0 / 3.0) * a * a * a / kSqrtPi;
  const int t = 1;
  auto recip = [&](const double* v) { return thp_tmatxbrecip(h, nr, v, dip.data()); };
  if ((st = recip(mu))) {
    g_last_error = st;
    return;
  }
  matvec(&nr, &t, mu, hh.data());
  double ggold[2] = {0, 0}, gg[2], ggnew[2];
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < nr; ++k)
      for (int j = 0; j < 3; ++j) {
        size_t q = (i * nr + k) * 3 + j;
        hh[q] = hh[q] + dip[q] - term * mu[q];
        res[q] = ef[q] - hh[q];
        zr[q] = diag[i] * res[q];
        pp[q] = zr[q];
        ggold[k] += res[q] * zr[q];
      }
  st = THP_E_NOT_CONVERGED;
  for (int it = 1; it <= c.cfg.politer; ++it) {
    if (recip(pp.data())) break;
    matvec(&nr, &t, pp.data(), hh.data());
    gg[0] = gg[1] = 0.0;
    for (size_t i = 0; i < n; ++i)
      for (int k = 0; k < nr; ++k)
        for (int j = 0; j < 3; ++j) {
          size_t q = (i * nr + k) * 3 + j;
          hh[q] = hh[q] + dip[q] - term * pp[q];
          gg[k] += pp[q] * hh[q];
        }
    bool zero = false;
    for (int k = 0; k < nr; ++k) zero |= (gg[k] == 0.0);
    if (zero) {
      st = THP_OK;
      break;
    }
    double al[2] = {ggold[0] / gg[0], nr > 1 ? ggold[1] / gg[1] : 0.0};
    ggnew[0] = ggnew[1] = 0.0;
    for (size_t i = 0; i < n; ++i)
      for (int k = 0; k < nr; ++k)
        for (int j = 0; j < 3; ++j) {
          size_t q = (i * nr + k) * 3 + j;
          mu[q] += al[k] * pp[q];
          res[q] -= al[k] * hh[q];
          zr[q] = diag[i] * res[q];
          ggnew[k] += res[q] * zr[q];
        }
    double resnrm = 0.0;
    for (int k = 0; k < nr; ++k) resnrm = std::max(resnrm, std::sqrt(ggnew[k] / (double)(3 * n)));
    for (size_t i = 0; i < n; ++i)
      for (int k = 0; k < nr; ++k)
        for (int j = 0; j < 3; ++j) {
          size_t q = (i * nr + k) * 3 + j;
          pp[q] = zr[q] + ggnew[k] / ggold[k] * pp[q];
        }
    ggold[0] = ggnew[0];
    ggold[1] = ggnew[1];
    if (resnrm < c.cfg.poleps) {
      st = THP_OK;
      break;
    }
  }
  g_last_error = st;
}

// Fortran-callable aliases of the drop-ins under names no Tinker-HP object
// defines, for a build that keeps the reference sources and calls the
// library through the ISO_C_BINDING shim.
void thp_f_newinduce_pme2(void) { newinduce_pme2_(); }
void thp_f_inducepcg_pme2(void (*matvec)(const int*, const int*, const double*, double*), const int* nrhs,
                          const int* precnd, const double* ef, double* mu, double* murec) {
  inducepcg_pme2_(matvec, nrhs, precnd, ef, mu, murec);
}
void thp_f_tmatxb_pme(const int* nrhs, const int* dodiag, const double* mu, double* efi) {
  tmatxb_pme_(nrhs, dodiag, mu, efi);
}
void thp_f_efld0_direct(const int* nrhs, double* ef) { efld0_direct_(nrhs, ef); }
void thp_f_efld0_recip(double* cphi) { efld0_recip_(cphi); }
void thp_f_tmatxbrecip(const double* mu, const double* murec, const int* nrhs, double* dipfield,
                       double* dipfieldbis) {
  tmatxbrecip_(mu, murec, nrhs, dipfield, dipfieldbis);
}
void thp_f_grid_uind_sites(const int* nsites, const int* isite, const double* fuind, const double* fuinp,
                           double* qgrid) {
  grid_uind_sites_(nsites, isite, fuind, fuinp, qgrid);
}
void thp_f_fphi_uind_sites(const int* nsites, const int* isite, const double* qgrid, double* fdip_phi1,
                           double* fdip_phi2, double* fdip_sum_phi) {
  fphi_uind_sites_(nsites, isite, qgrid, fdip_phi1, fdip_phi2, fdip_sum_phi);
}
void thp_f_mlistcell(void) { mlistcell_(); }
void thp_f_vlistcell(void) { vlistcell_(); }
void thp_f_epolar(void) { epolar_(); }
void thp_f_epolar1(void) { epolar1_(); }
void thp_f_empole1(void) { empole1_(); }
void thp_f_ehal1(void) { ehal1_(); }

}  // extern "C"
