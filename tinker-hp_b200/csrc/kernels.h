// kernels.h -- host launchers of the device kernels (internal).
#pragma once

#include "context.h"

namespace thp {

// nblist.cu
int launch_sort_atoms(Ctx& c);          // cell sort, permutation, sorted copies
int launch_gather_sorted(Ctx& c);       // positions/params/rpole into sorted order
int launch_build_list(Ctx& c);
int launch_build_list_on(Ctx& c, cudaStream_t s);          // full list within ewaldcut + lbuffer
int launch_export_list(Ctx& c, int maxelst, int* d_nelst, int* d_elst);
int launch_rotpole(Ctx& c);             // local-frame multipoles -> d_rpole_orig
int launch_max_displacement(Ctx& c, double* h_out);
int launch_max_displacement_from(Ctx& c, const double4* ref, double* h_out);  // largest move since ref (sorted)

// realspace.cu
int launch_efld0_coef(Ctx& c, bool with_field);
int launch_efld0_coef_on(Ctx& c, bool with_field, cudaStream_t s);  // direct field into d_ef, coefficients
int launch_tmatxb(Ctx& c, const double* d_in, double* d_out, bool dodiag);  // sorted [n][6]

// pme.cu
int pme_init(Ctx& c);
int plan_prefetch(int device, const int nfft[3], int mixed);  // puts a plan of that shape in the cache
void pme_free(Ctx& c);
int launch_efld0_recip(Ctx& c);         // d_cphi and E0 completion
int launch_efld0_recip_ex(Ctx& c, double* cphi10, bool with_e0);
int launch_mpole_grid(Ctx& c);          // permanent-multipole grid, convolved (grid holds the potential)
// the same, with the permanent-only k-space virial (times sign) into d_part
int launch_mpole_grid_virial(Ctx& c, double* d_part, double sign);
int launch_pair_grid_virial(Ctx& c, double* d_part);   // (rpole+uinp) x (rpole+uind) k-space virial
int kspace_virial_blocks();
int launch_gather_mpole(Ctx& c, double* cphi10, bool with_e0);  // cphi from the convolved grid, E0 completion
int launch_pme_dipole_f32(Ctx& c, const float* d_vec);  // mode-2 spread of an FP32 vector + convolution
bool overlap_rows(const Ctx& c);  // the system runs real-space passes on the side stream
int zero_grid(Ctx& c);
struct PmeGeom;
PmeGeom pme_geom(const Ctx& c);
int launch_pme_dipole(Ctx& c, const double* d_vec, double* d_out, int mode);
int launch_gather_dip(Ctx& c, double* d_out, bool check_stop);

// forces.cu
int launch_forces(Ctx& c, double* d_out);  // dE/dx [n][3], original order, for the dipoles in d_mu
// virial partial sums of a gradient call (k-space, per-block rows of 6 and
// 12) and their 12 totals copied to h_out
int virial_scratch(Ctx& c, int nr, int ne, double** kpart, double** rpart, double** epart);
int virial_total(Ctx& c, int nk, int nr, int ne, const double* kpart, const double* rpart, const double* epart,
                 double* h_out);
int launch_fphi_mpole20(Ctx& c);          // fphirec [n][20] of the convolved multipole grid
int launch_frames_sorted(Ctx& c);         // frame atoms in sorted numbering (d_frs)
int launch_gradient_out(Ctx& c, const unsigned long long* dep, double* d_out);  // fixed point -> original order
// permanent-multipole energy into d_em and dE/dx [n][3] (original order) into
// d_out, for the current sorted positions, multipoles and list
int launch_empole(Ctx& c, double* d_out);
// buffered 14-7 van der Waals energy into d_ev and dE/dx [n][3] (original
// order) into d_out, for the current sorted positions and cell sort
int launch_ehal(Ctx& c, double* d_out);
int launch_vdw_list(Ctx& c);  // reduced sites, and the vdW list when it is stale
// reference-format half list (k > i, original numbering) of a slot-major list
int launch_export_pairs(Ctx& c, const int* nnb, const int* nb, int maxnb, int maxelst, int* d_nelst, int* d_elst);

// sites.cu
int launch_grid_uind_sites(Ctx& c, int nsites, const int* d_site, const double* d_fuind, const double* d_fuinp,
                           cufftDoubleComplex* d_sgrid);
int launch_fphi_uind_sites(Ctx& c, int nsites, const int* d_site, const cufftDoubleComplex* d_sgrid, double* d_phi1,
                           double* d_phi2, double* d_sum);

// predict.cu
int predictor_push(Ctx& c);   // d_mu becomes the newest stored solution
int predictor_guess(Ctx& c);  // predicted d_mu; -1 when fewer than kMaxAlt are stored

// md.cu
int launch_kick(Ctx& c, double half_dt, const double* d_mass, const double* d_grad, double* d_vel);
int launch_drift(Ctx& c, double dt, const double* d_vel);          // advances d_xyz_orig
int launch_ekin(Ctx& c, const double* d_mass, const double* d_vel, double* d_scratch);

// solver.cu
int run_pcg(Ctx& c, int guess);
int run_pcg_async(Ctx& c, int guess, bool* pending);  // see solver.cu
int pcg_status(Ctx& c);
int pcg_begin(Ctx& c, int guess);
int pcg_chunk_async(Ctx& c);
int pcg_loop_async(Ctx& c);  // whole CG loop in one graph launch; -1 when unavailable
int pcg_status(Ctx& c);
int launch_epol(Ctx& c);

// reorder helpers (solver.cu)
int launch_to_sorted6(Ctx& c, const double* d_orig, double* d_sorted, int nrhs);
int launch_to_orig6(Ctx& c, const double* d_sorted, double* d_orig, int nrhs);
int launch_split_dipoles(Ctx& c, const double* d_sorted, double* d_out);  // uind [n][3] then uinp [n][3], original order

int cuda_status(cudaError_t e, Ctx* c, const char* what);

// realspace.cu
struct PairRows;
PairRows pair_rows(const Ctx& c);   // the context's pair stream
float row_interior(const Ctx& c);   // bound of the groups that skip the periodic wrap

// batch.cu: the CG iterations of many small systems as batched persistent
// kernels in one graph (a plan per set of contexts)
struct BatchPlan;
int batch_plan_create(Ctx* const* cs, int count, BatchPlan** out, std::string* msg);
void batch_plan_destroy(BatchPlan* p);
int batch_plan_check(const BatchPlan& p, Ctx* const* cs);  // THP_E_STATE if a context was re-targeted
int batch_plan_loop(BatchPlan& p, Ctx* const* cs);   // after the fronts; the contexts' streams wait for it
void batch_plan_finish(BatchPlan& p);  // after the solve synchronised: tuner bookkeeping
int batch_plan_tuning(const BatchPlan& p, int* blocks_per_sm, int* matvec_atoms, float* ms);
// enable 1: later solves run the loop eagerly with per-kernel events (0: back
// to the graph; -1: read only); ms[6] receives the accumulated device time of
// spread, forward FFTs, qfac, inverse FFTs, matvec and update
int batch_plan_profile(BatchPlan& p, int enable, double* ms, int* iterations);
int batch_plan_candidate(const BatchPlan& p);  // the launch shape the next solve uses
bool batch_plan_profiling(const BatchPlan& p);
// whole-solve graphs: every system's front, the batched loop and the results
cudaGraphExec_t batch_plan_solve_exec(const BatchPlan& p, int guess, int carry, int cand);
int batch_plan_make_solve_exec(BatchPlan& p, const std::vector<cudaGraph_t>& fronts, int guess, int carry, int cand);
int batch_plan_run_solve(BatchPlan& p, cudaGraphExec_t ex, const CgScalars** cg_out, const int** flags_out,
                         float* ms);

}  // namespace thp
