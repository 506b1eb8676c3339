// context.h -- per-system device state of the polarization library (internal).
#pragma once

#include <cufft.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace thp {

// Scalars of the device-resident CG (newinduce_pme2.f:308-312), one per RHS.
struct CgScalars {
  double ggold[2];
  double gg[2];
  double ggnew[2];
  double ene[2];
  double alpha[2];
  double beta[2];
  double resnrm;
  double epol;
  double epart;  // spare accumulator
  int converged;
  int stop;      // 1: converged or failed, later kernels return at once
  int niter;
  int status;    // THP_* code raised on the device
  unsigned counter[4];  // last-block counters of the grid reductions
  int loops;            // bodies run by the device-side CG loop
};

// CG iterations per host check of the stop flag
constexpr int kCgChunk = 4;

// device error flags (bit set)
enum : int { DEV_LIST_OVERFLOW = 1, DEV_PAIR_OVERFLOW = 2, DEV_NAN = 4, DEV_BAD_INPUT = 8, DEV_VDW_REACH = 16 };

// dipole solutions kept for the predictor (MOD_uprior.f: maxualt)
constexpr int kMaxAlt = 7;

struct Ctx {
  thp_config cfg{};
  int n = 0, npad = 0;
  // allocated capacities (a context re-targeted to a new system keeps every
  // buffer that is large enough)
  size_t cap_n = 0, cap_ncell = 0, cap_pairs = 0, cap_sp = 0, cap_sp_off = 0;
  // one allocation per buffer group (cells, per-atom arrays, pair arrays);
  // the d_* pointers of a group point into its slab
  void* slab_cells = nullptr;
  void* slab_atoms = nullptr;
  void* slab_pairs = nullptr;
  void* h_pinned = nullptr;  // pinned block holding h_cg and h_flags
  int mixed = 0;
  Box box{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // side stream of the CG iteration: the real-space row runs there while the
  // PME branch runs on `stream` (fork / join events, captured in the graph)
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

  // host copies (original atom order)
  std::vector<double> h_polarity, h_thole, h_pdamp;
  bool have_params = false, have_pos = false, have_rpole = false, have_conn = false;
  bool have_frames = false;    // rpole comes from rotpole of d_pole_local
  bool have_axes = false;      // d_frames holds the frame atoms (torques need them)
  std::vector<int> sp_off;     // special (scaled) pairs, original indices, CSR
  std::vector<int> sp_k;
  std::vector<double> sp_s;    // (d, p, u) per entry
  std::vector<int> sp_c;       // 1-2..1-5 class of the entry (0..3; 4: none) for the mpole scales
  double scales[16] = {0};
  double mscale[4] = {0.0, 0.0, 1.0, 1.0};  // m2scale..m5scale (initprm.f:413-416)

  // cell grid of the list build
  int nc[3] = {1, 1, 1};
  unsigned sort_epoch = 0;  // counts re-sorts of the atoms
  int ncell = 1;
  int* d_cell_count = nullptr;
  int* d_cell_start = nullptr;
  int* d_cell_fill = nullptr;
  int* d_atom_cell = nullptr;   // original order
  int* d_scell = nullptr;       // cell of sorted atom

  // permutation
  int* d_perm = nullptr;   // sorted -> original
  int* d_iperm = nullptr;  // original -> sorted
  bool have_perm = false;

  // staging in original order
  double* d_xyz_orig = nullptr;   // [3][n]
  double* d_par_orig = nullptr;   // [3][n] pdamp, thole, polarity
  double* d_rpole_orig = nullptr; // [n][13]
  double* d_pole_local = nullptr; // [n][13]
  int* d_frames = nullptr;        // [n][3] zaxis, xaxis, axt (original indices)

  // sorted per-atom data
  double4* d_pos = nullptr;       // x, y, z, pdamp
  float4* d_posf = nullptr;       // mixed form positions (x,y,z wrapped, pdamp)
  double* d_thole = nullptr;
  double* d_pol = nullptr;
  double* d_rpole = nullptr;      // [n][10]: q, d(3), Qxx,Qxy,Qxz,Qyy,Qyz,Qzz
  double* d_mrec = nullptr;       // [n][12]: thole, q, d(3), Q(6), 0 -- pair-pass record (96 B)
  float* d_mrecf = nullptr;       // [n][12] FP32 copy for the mixed form (48 B)
  float* d_erec = nullptr;        // [n][16] mixed direct-field record (64 B, see k_gather_sorted)
  int* d_sp_ks = nullptr;         // special partners renumbered to sorted indices
  int* d_sp_off = nullptr;        // special pairs, ORIGINAL indices, CSR [n+1]
  int* d_sp_k = nullptr;
  double* d_sp_s = nullptr;       // (d, p, u) scale per entry
  int* d_sp_c = nullptr;          // 1-2..1-5 class per entry (4: none)
  // van der Waals (thp_set_vdw): classes, reduction parents and factors in
  // original order; pair tables [4][nclass][nclass] (Rmin, eps, 1-4 Rmin,
  // 1-4 eps); sorted reduced sites and energy partials made on first use
  bool have_vdw = false;
  int vdw_nclass = 0;
  double vdw_cut = 9.0, vdw_taper = 8.1, vdw_ghal = 0.12, vdw_dhal = 0.07;
  double vdw_scale[4] = {0.0, 0.0, 1.0, 1.0};
  size_t cap_vtab = 0;
  int* d_vcls = nullptr;
  int* d_vired = nullptr;
  double* d_vkred = nullptr;
  double* d_vtab = nullptr;
  double4* d_vred = nullptr;
  float4* d_vredf = nullptr;      // the same sites wrapped into the box, FP32 (list screen)
  float* d_muf = nullptr;         // [n][8] FP32 sorted dipoles for the mixed gradient pass
  int2* d_vinfo = nullptr;
  // vdW pair list (vlistcell): full list within vdwcut + lbuffer of the
  // reduced sites, slot-major [s*npad + i], rebuilt after a re-sort or when an
  // atom has moved lbuffer/2 since the positions it was built from
  int maxvnb = 0;
  int* d_vnb = nullptr;
  int* d_vnnb = nullptr;
  double4* d_vpos_built = nullptr;
  bool have_vlist = false;
  unsigned vlist_epoch = 0;
  double* d_evpart = nullptr;
  double* d_ev = nullptr;
  double* d_empart = nullptr;     // per-block partial sums of the permanent-multipole energy, then
  double* d_em = nullptr;         // their total (d_empart + blocks), made on first use
  double4* d_pos_built = nullptr; // positions at the last list build

  // full neighbor list within ewaldcut+lbuffer (slot-major: nb[s*npad+i])
  int maxnb = 0;
  int* d_nnb = nullptr;
  int* d_nb = nullptr;
  bool have_list = false;

  // interacting pairs within ewaldcut with mutual-field coefficients
  int maxpr = 0;
  int* d_npr = nullptr;
  int* d_pk = nullptr;
  void* d_pcc = nullptr;   // (dmp3, dmp5) per pair-stream entry: double2 or float2
  bool have_coef = false;

  // PME
  int nfft[3] = {0, 0, 0};
  size_t ngrid = 0;
  cufftHandle plan = 0;
  bool have_plan = false;
  int plan_dims[3] = {0, 0, 0};
  size_t cap_ngrid = 0;
  void* d_grid = nullptr;  // cufftDoubleComplex or cufftComplex
  void* d_qfac = nullptr;  // double or float
  double a_frac[3] = {0, 0, 0};  // nfft_d * recip(d,d)

  // CG vectors, sorted order, [n][6] = (d xyz, p xyz)
  double* d_ef = nullptr;
  double* d_mu = nullptr;
  double* d_res = nullptr;
  double* d_h = nullptr;
  double* d_pp = nullptr;
  double* d_zr = nullptr;
  double* d_dip = nullptr;
  double* d_cphi = nullptr;   // [n][4] permanent potential and gradient (Cartesian)
  float* d_vecf = nullptr;    // mixed form matvec input [n][6]
  // mixed form matvec input of the overlapped CG rows: per atom one 32-byte
  // record {x, y, z (wrapped), d dipole, p dipole x, y} and the p dipole z
  float* d_rec = nullptr;     // [n][8]
  // E0 of the last CG start (sorted order), for the corrected warm start
  double* d_ef_prev = nullptr;  // [n][6]
  bool have_ef_prev = false;
  float* d_mpz = nullptr;     // [n]
  // the mixed form's overlapped CG keeps its search direction, h, residual
  // and preconditioned residual in FP32 (dot products and scalars in FP64)
  float *d_ppf = nullptr, *d_hf = nullptr, *d_resf = nullptr, *d_zrf = nullptr;  // [n][6]
  double* d_tmp6 = nullptr;   // [n][6] original-order staging for host I/O
  double* d_tmp6b = nullptr;
  bool have_dipoles = false;

  // reductions
  double* d_partials = nullptr;  // [blocks][8]
  int nblk_reduce = 0;
  CgScalars* d_cg = nullptr;
  CgScalars* h_cg = nullptr;     // pinned mirror
  int* d_flags = nullptr;        // device error bits
  int* h_flags = nullptr;        // pinned

  // predictor history: kMaxAlt solutions [slot][n][6] in ORIGINAL order
  int pred_mode = 0;
  int nualt = 0, alt_head = 0;
  double* d_alt = nullptr;
  size_t alt_cap = 0;

  // polarization gradient (allocated on first use)
  double* d_fphirec = nullptr;    // [n][20] permanent-multipole potential, fractional
  unsigned long long* d_depfix = nullptr;  // [n][3] 64-bit fixed-point gradient, sorted
  double* d_trq = nullptr;        // [n][3] reciprocal-space torque
  // virial of the polarization gradient (thp_set_virial): partial sums on
  // the device, and the last gradient call's totals: the reference's terms
  // (xx xy xz yy yz zz), then the reciprocal and self torques' frame terms
  bool want_virial = false, have_virial = false;
  double* d_virp = nullptr;
  size_t virp_cap = 0;
  double h_vir[12] = {};
  // the same for the last empole1 call (thp_get_empole_virial) and the
  // last ehal1 call (thp_get_ehal_virial; 6 values used)
  bool have_mvirial = false, have_vvirial = false;
  double h_mvir[12] = {};
  double h_vvir[12] = {};
  int* d_frs = nullptr;           // [n][3] frame atoms (sorted indices), axis type
  double* d_grad = nullptr;       // [n][3] gradient, original order

  // batched per-site PME routines on a caller grid (allocated on first use)
  cufftDoubleComplex* d_sgrid = nullptr;  // FP64 copy of qgrid2in_2d
  void* d_sscratch = nullptr;             // site numbers and per-site values
  size_t sscratch_bytes = 0;
  std::vector<double> h_sgrid;            // host staging of the grid

  // Fortran binding
  double *bx = nullptr, *by = nullptr, *bz = nullptr, *brpole = nullptr;
  double *buind = nullptr, *buinp = nullptr, *bep = nullptr;
  int *bnelst = nullptr, *belst = nullptr;
  int bmaxelst = 0;
  double* bdep = nullptr;
  double* bvir = nullptr;  // virial::vir(3,3), added to by epolar1_
  double *bem = nullptr, *bdem = nullptr;  // energi::em, deriv::dem(3,n), written by empole1_
  double *bev = nullptr, *bdev = nullptr;  // energi::ev, deriv::dev(3,n), written by ehal1_
  int *bnvlst = nullptr, *bvlst = nullptr;  // neigh::nvlst(n), vlst(maxvlst,n), filled by vlistcell_
  int bmaxvlst = 0;
  double* bqgrid = nullptr;  // pme::qgrid2in_2d(2,n1,n2,n3), read by fphi_uind_site_

  // CUDA graph of one CG chunk (captured on first use)
  cudaGraphExec_t chunk_exec = nullptr;
  // the whole CG loop as one graph (conditional WHILE node); loop_state:
  // 0 not built yet, 1 built, -1 not available (the chunked graph is used)
  cudaGraphExec_t loop_exec = nullptr;
  int loop_state = 0;
  // front of a batched solve per guess mode and dipole carry (api.cu)
  cudaGraphExec_t front_exec[3][2] = {};
  bool front_failed = false;

  // optional event pairs around the fused CG matvec launches
  bool profiling = false;
  std::vector<cudaEvent_t> prof_events;

  std::string last_msg;
};

}  // namespace thp
