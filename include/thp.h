/*
 * thp.h -- C-ABI of the B200-native AMOEBA induced-dipole polarization path.
 *
 * Two layers:
 *   1. Native API (thp_*): an opaque per-system context owning device state.
 *      Plain pointers and sizes, host arrays in the reference's layouts:
 *        - per-atom vectors (3,nrhs,n) Fortran order == C [n][nrhs][3];
 *        - multipoles rpole(13,n) == C [n][13] (q, dx,dy,dz, Qxx,Qxy,Qxz,
 *          Qyx,Qyy,Qyz,Qzx,Qzy,Qzz in e, e*A, e*A^2, traceless, /3 as stored
 *          by kmpole.f:534-537);
 *        - neighbor lists nelst(n), elst(maxelst,n) == C [n][maxelst].
 *      Every entry point returns a THP_* status and never exits.
 *   2. Fortran drop-ins with the reference's subroutine names (gfortran
 *      mangling name_, arguments by reference).  They act on the context made
 *      current by thp_bind_state() and record failures in thp_last_error().
 *
 * Threading: thread-safe across contexts, not within one context.  All device
 * work of a context is ordered on its stream.
 */
#ifndef THP_H
#define THP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define THP_OK 0
#define THP_E_INVALID 1        /* bad argument or unsupported option */
#define THP_E_LIST_OVERFLOW 2  /* neighbor capacity exceeded (nblist.f:232 fatal) */
#define THP_E_NOT_CONVERGED 3  /* CG reached politer without meeting poleps */
#define THP_E_NAN 4            /* non-finite value in the CG recurrences */
#define THP_E_CUDA 5           /* CUDA runtime or cuFFT failure */
#define THP_E_TIMEOUT 6        /* a bounded device wait gave up */
#define THP_E_OOM_ADMISSION 7  /* request does not fit the device-memory budget */
#define THP_E_BOX_TOO_SMALL 8  /* list cutoff exceeds half a box edge (nblist.f:148) */
#define THP_E_NO_DEVICE 9      /* no usable CUDA device */
#define THP_E_STATE 10         /* call made before its inputs were set */

/* ---- precision forms ---------------------------------------------------- */
#define THP_FP64 0  /* everything in FP64 */
#define THP_MIXED 1 /* FP32 pair fields, PME and CG vectors, FP64 CG scalars, mu and energy */

/* ---- connectivity slots (modules couple and polgrp) -------------------- */
#define THP_I12 0
#define THP_I13 1
#define THP_I14 2
#define THP_I15 3
#define THP_IP11 4
#define THP_IP12 5
#define THP_IP13 6
#define THP_IP14 7
#define THP_NCONN 8

/* ---- initial guess of the dipoles (newinduce_pme2.f:161-200) ----------- */
#define THP_GUESS_DIRECT 0   /* mu = alpha * E0 (polgsf = 0) */
#define THP_GUESS_PREVIOUS 1 /* mu = last converged dipoles kept on the device, plus the
                                polarizability times the change of the direct field E0 since
                                their solve (a first-order correction for moved atoms) */
#define THP_GUESS_HOST 2     /* mu = caller-provided array (thp_set_guess) */
#define THP_GUESS_PREDICT 3  /* predictor over the stored solutions (thp_set_predictor); the direct
                                guess until seven are stored (newinduce_pme2.f:165-190) */

/* predictors of the dipoles in dynamics (ulspred, newinduce_pme2.f:910;
 * coefficients kpolar.f:405-425) */
#define THP_PRED_NONE 0
#define THP_PRED_ASPC 1
#define THP_PRED_GEAR 2
#define THP_PRED_LSQR 3

typedef struct thp_config {
  int n;            /* polarizable sites (npole == npolar == n) */
  double box[3];    /* orthogonal box edges xbox, ybox, zbox (A) */
  double aewald;    /* Ewald coefficient (1/A), kewald.f:apewald */
  double ewaldcut;  /* real-space cutoff (A), cutoffs.f:ewaldcut */
  double lbuffer;   /* neighbor-list buffer (A), cutoffs.f:lbuffer */
  int nfft[3];      /* PME grid nfft1..3 */
  int bsorder;      /* B-spline order; 5 is supported */
  int politer;      /* max CG iterations (initprm.f:441) */
  double poleps;    /* CG stop: max_k sqrt(sum res.zr / 3n) < poleps */
  int precision;    /* THP_FP64 or THP_MIXED */
  int max_neighbors;/* per-atom capacity of the full list (0: 320) */
  int device;       /* CUDA device ordinal */
} thp_config;

typedef struct thp_solve_info {
  int niter;        /* CG iterations taken */
  int converged;    /* 1 when resnrm < poleps */
  double resnrm;    /* final residual norm (reference units) */
  double epol;      /* polarization energy, kcal/mol (epolar.f:epolar0c) */
  double ene[2];    /* CG energies -1/2 sum mu.(res+ef) * electric (inducepcg) */
  double ms_total;  /* device time of the solve, ms */
} thp_solve_info;

typedef struct thp_ctx thp_ctx;

/* ---- native API ---------------------------------------------------------- */
int thp_ctx_create(const thp_config* cfg, thp_ctx** out);
int thp_ctx_destroy(thp_ctx* ctx);
/* Re-target a context to another system (same precision and device): every
 * device buffer that is large enough and the cuFFT plan of an unchanged grid
 * are kept, so no device memory is freed or allocated unless the new system
 * is larger.  All system state is cleared (parameters, connectivity,
 * positions, multipoles, list, dipoles, bindings), as after thp_ctx_create. */
int thp_ctx_reset(thp_ctx* ctx, const thp_config* cfg);
/* device bytes the context holds at its current capacity */
size_t thp_ctx_footprint(thp_ctx* ctx);
/* use an external CUDA stream (cudaStream_t passed as void*) */
int thp_set_stream(thp_ctx* ctx, void* stream);
/* polarity(n) A^3, thole(n), pdamp(n) = polarity^(1/6) (kpolar.f:225-300) */
int thp_set_params(thp_ctx* ctx, const double* polarity, const double* thole, const double* pdamp);
/* CSR connectivity, slot order THP_I12..THP_IP14: off[slot][n+1], idx[slot][];
 * scales[16] = p2..p5scale, p2i..p5iscale, d1..d4scale, u1..u4scale. */
int thp_set_connectivity(thp_ctx* ctx, const int* const* off, const int* const* idx,
                         const double* scales);
int thp_set_positions(thp_ctx* ctx, const double* x, const double* y, const double* z);
int thp_set_rpole(thp_ctx* ctx, const double* rpole);
/* local-frame multipoles and frames; rotpole runs on the device.
 * axt: 1 = Z-then-X, 2 = Bisector (rotpole.f:58-200); axes 0-based. */
int thp_set_frames(thp_ctx* ctx, const double* pole, const int* zaxis, const int* xaxis,
                   const int* axt);
int thp_set_guess(thp_ctx* ctx, const double* mu /*[n][2][3]*/);
/* Chooses the predictor (THP_PRED_*) and clears the stored solutions.  With a
 * predictor set, every solve stores its dipoles (the last seven are kept, in
 * original atom order, so list rebuilds do not disturb them) and
 * THP_GUESS_PREDICT extrapolates from them. */
int thp_set_predictor(thp_ctx* ctx, int mode);
/* list build (mlistcell), incremental when displacements allow */
int thp_nblist(thp_ctx* ctx);
/* full rebuild (cell sort + list) on the next list use, as nblist(0) does */
int thp_invalidate_list(thp_ctx* ctx);
/* device time of the real-space CG matvec kernels since the last reset:
 * enable != 0 starts recording events around each launch (and resets). */
int thp_profile(thp_ctx* ctx, int enable, double* ms_total, int* launches);
/* E0 + PCG + Epol on the device (newinduce_pme2 + epolar0c) */
int thp_solve(thp_ctx* ctx, int guess, thp_solve_info* info);
int thp_get_dipoles(thp_ctx* ctx, double* uind, double* uinp);
int thp_get_field(thp_ctx* ctx, double* ef /*[n][2][3]*/);
int thp_get_rpole(thp_ctx* ctx, double* rpole /*[n][13]*/);
/* reference-format half list (k > i, 0-based) copied to the host */
int thp_get_nblist(thp_ctx* ctx, int maxelst, int* nelst, int* elst);
/* single operators on host arrays, reference semantics */
int thp_tmatxb(thp_ctx* ctx, int nrhs, int dodiag, const double* mu, double* efi);
int thp_efld0_direct(thp_ctx* ctx, int nrhs, double* ef);
int thp_efld0_recip(thp_ctx* ctx, double* cphi /*[n][10]*/);
int thp_tmatxbrecip(thp_ctx* ctx, int nrhs, const double* mu, double* dipfield);
/* Solve several resident systems together (batched form): each context runs
 * on its own stream; the fields of all systems are enqueued first, then CG
 * chunks (replayed CUDA graphs) for every unconverged system per round, with
 * one host check of all stop flags per round.  The list is rebuilt for every
 * system (single-point solves).  infos[i] receives system i's result;
 * returns the first non-OK status (THP_E_NOT_CONVERGED only if nothing
 * worse happened). */
int thp_solve_batch(thp_ctx** ctxs, int count, int guess, thp_solve_info* infos);
/* Batch plans (the reference has no batched form; the loop each plan runs is
 * inducepcg_pme2, newinduce_pme2.f:285-636).  A plan binds a fixed set of
 * contexts on one device in one precision, each below 20,000 atoms, and runs
 * the CG iterations of all of them as batched persistent kernels: one launch
 * per kernel per iteration walks a device work list of (system, tile) items,
 * the convolution runs as one batched cuFFT transform per grid shape, and the
 * loop is a conditional WHILE node that runs until every system has stopped.
 * A solve whose systems all take the same start (guess DIRECT, PREVIOUS or
 * HOST after resolution, and the same dipole carry) runs as one graph launch:
 * every system's front (E0, list, CG start) as a parallel branch, the loop,
 * and the energies and CG scalars written to mapped host memory; other solves
 * run the fronts per system as thp_solve_batch does.  An autotuner times the
 * first solves of a plan, one candidate launch shape each, and keeps the
 * fastest (remembered for later plans of the same size class).
 * thp_batch_create returns THP_E_INVALID for systems outside those limits;
 * thp_batch_solve returns THP_E_STATE if a context was re-targeted
 * (thp_ctx_reset) since the plan was made; results as thp_solve_batch, with
 * ms_total the device time of the whole batch. */
typedef struct thp_batch thp_batch;
int thp_batch_create(thp_ctx** ctxs, int count, thp_batch** out);
int thp_batch_solve(thp_batch* b, int guess, thp_solve_info* infos);
/* the kept launch shape: resident blocks per SM of the batched kernels, atoms
 * per matvec tile, and the device time of the solve it was measured on (ms);
 * THP_E_STATE while the plan is still tuning */
int thp_batch_tuning(thp_batch* b, int* blocks_per_sm, int* matvec_atoms, double* ms_per_solve);
/* Per-kernel device time of the batched loop.  enable = 1: later solves run
 * the loop eagerly, one host-checked iteration at a time, with events around
 * each step (the accumulators restart); 0: back to the graph; -1: only read.
 * ms[6] receives the accumulated ms of the spread, the forward FFTs, the
 * influence function, the inverse FFTs, the matvec and the update;
 * iterations the batched iterations timed. */
int thp_batch_profile(thp_batch* b, int enable, double* ms, int* iterations);
int thp_batch_destroy(thp_batch* b);
/* Gradient of the polarization energy, epolar1c (epolar1.f:57-372): eprecip1
 * (:397), epreal1c (:1215, Thole branch), the self torque (:190-206) and the
 * torque-to-force conversion of torque.f:6, for the dipoles of the last solve
 * at the current positions.  dep [n][3] (kcal/mol/A, x fastest as dep(3,n))
 * on the host, original atom order; ep (may be NULL) receives that solve's
 * energy.  The torques need the frame atoms given to thp_set_frames (kept
 * when thp_set_rpole later replaces the multipoles).  THP_E_STATE without
 * frames or without a solve since the last position / multipole change.
 * Gradients accumulate in 64-bit fixed point (2^-34 kcal/mol/A) in both
 * precisions, so the order of the per-atom additions does not matter. */
int thp_get_gradient(thp_ctx* ctx, double* dep, double* ep);
/* same gradient into device memory d_dep [n][3], enqueued on the context's
 * stream without a host synchronisation */
int thp_get_gradient_device(thp_ctx* ctx, double* d_dep);
/* on != 0: every later gradient call also computes the internal virial of
 * the polarization energy (TINFOIL boundary): eprecip1's induced-dipole
 * site terms (epolar1.f:846-908) and scalar sums over the reciprocal
 * lattice ((rpole+uinp) x (rpole+uind) minus the permanent-only sum,
 * :534-541, :932-1091), epreal1c's pair terms (:2326-2342) and the frame-atom
 * terms of its torques (:2460-2486).  It costs one more grid spread and
 * forward transform and two passes over the grid per call. */
int thp_set_virial(thp_ctx* ctx, int on);
/* vir [3][3] (kcal/mol, symmetric) of the last gradient call made with the
 * virial on (THP_E_STATE otherwise).  form 0: as the reference accumulates
 * it; form 1: plus the frame-atom virial of the reciprocal and self torques,
 * which the reference does not add (torque_rec / torque carry no virial):
 * the derivative of the energy with respect to a homogeneous strain of the
 * box and the coordinates. */
int thp_get_virial(thp_ctx* ctx, int form, double* vir);
/* The virial of the last thp_empole1 call made with thp_set_virial on
 * (empole1c: emrecip1's site terms and scalar sum, empole1.f:560-598,
 * 741-761; emreal1c's pair and torque frame terms, :1428-1443, 1466-1497),
 * form as thp_get_virial (1 adds the frame-atom virial of the reciprocal
 * torques, which the reference leaves out); THP_E_STATE before such a call.
 * empole1_ adds form 0 into the bound vir when one is bound. */
int thp_get_empole_virial(thp_ctx* ctx, int form, double* vir);
/* The virial [3][3] of the last thp_ehal1 call made with thp_set_virial on
 * (ehal1c's pair terms over the reduced sites, ehal1.f:431-446);
 * THP_E_STATE before such a call.  ehal1_ adds it into the bound vir when
 * one is bound. */
int thp_get_ehal_virial(thp_ctx* ctx, double* vir);
/* m2scale..m5scale [4] of the permanent-multipole pair terms (mplpot module;
 * defaults initprm.f:413-416: 0, 0, 1, 1; AMOEBA water03.prm:34-37: 0, 0,
 * 0.4, 0.8).  The 1-2..1-5 lists come from thp_set_connectivity. */
int thp_set_mpole_scales(thp_ctx* ctx, const double* m);
/* Permanent-multipole energy and gradient, empole1c (empole1.f:42-340):
 * emrecip1 (:349), emreal1c (:873, standard branch, mscale), the Ewald self
 * energy (:134-160) and torque (torque.f:6), TINFOIL boundary, at the current
 * positions and multipoles (rotpole on the device when frames are set, once per
 * change of the positions or frames, so a call between a solve and its
 * gradient leaves the solve valid).  No virial.
 * em (kcal/mol) and dem [n][3] (kcal/mol/A, original order; either may be
 * NULL).  Needs frames (thp_set_frames) and connectivity; THP_E_STATE
 * otherwise.  The list is built or reused as for a solve.  The mixed form
 * evaluates the unscaled pairs and the grid in FP32 and the 1-2..1-5 pairs,
 * the reciprocal-space sums and the self term in FP64; gradients accumulate
 * in 64-bit fixed point as thp_get_gradient's. */
int thp_empole1(thp_ctx* ctx, double* em, double* dem);
/* van der Waals description (kvdw.f): cls [n] vdW class of each atom
 * (0-based, < nclass); tables [4][nclass][nclass] = pair Rmin (A), pair
 * epsilon (kcal/mol), and their 1-4 forms, already combined by the force
 * field's rules (kvdw.f:318-480); ired [n] reduction parent (0-based, the
 * atom itself when unreduced) and kred [n] reduction factor (kvdw.f:490-503);
 * vscale [4] v2scale..v5scale; vdwcut and vdwtaper in A (the taper start as
 * a distance, cutoffs.f:241); ghal, dhal the buffered 14-7 constants
 * (0.12, 0.07).  THP_E_BOX_TOO_SMALL when vdwcut + lbuffer exceeds half the
 * box (nblist.f:1183-1193). */
int thp_set_vdw(thp_ctx* ctx, const int* cls, int nclass, const double* tables, const int* ired,
                const double* kred, const double* vscale, double vdwcut, double vdwtaper, double ghal,
                double dhal);
/* Buffered 14-7 van der Waals energy and gradient, ehal1c (ehal1.f:69-482,
 * standard branch; no long-range correction) over the pairs vlistcell
 * (nblist.f:1148) would list: ev (kcal/mol) and dev [n][3] (kcal/mol/A,
 * original order; either may be NULL).  FP64 pair terms in the FP64 form;
 * the mixed form evaluates them in FP32 from FP32 sites (the taper in its
 * smoothstep form) and accumulates in FP64.  The pair list is kept in the
 * context and rebuilt after a re-sort or a move of lbuffer/2;
 * THP_E_INVALID when a reduction moves a site by more than 0.3 A. */
int thp_ehal1(thp_ctx* ctx, double* ev, double* dev);
/* reference-format vdW half list (vlistcell, nblist.f:1148-1305: reduced
 * sites within vdwcut + lbuffer, partners k > i, 0-based) copied to the host;
 * THP_E_LIST_OVERFLOW when a row exceeds maxvlst */
int thp_get_vlist(thp_ctx* ctx, int maxvlst, int* nvlst, int* vlst);
/* Velocity-Verlet NVE dynamics driven by the polarization gradient alone
 * (verlet.f:17-200 with gradient = epolar1): per step a half kick, a drift of
 * the positions on the device, a solve warm-started from the predictor when
 * one is set (thp_set_predictor), else from the previous step's dipoles
 * (list rebuilt when an atom moved more than lbuffer/2), the gradient,
 * and the second half kick.  Starts with a solve and gradient at the current
 * positions.  mass [n] g/mol; vel [n][3] A/ps, updated in place; dt in ps.
 * energies [nsteps][3] (may be NULL): epol, kinetic, total (kcal/mol) after
 * each step; niters [nsteps] (may be NULL): CG iterations of each solve.
 * thp_get_positions reads the advanced positions back. */
int thp_md_verlet(thp_ctx* ctx, int nsteps, double dt, const double* mass, double* vel,
                  double* energies, int* niters);
int thp_get_positions(thp_ctx* ctx, double* x, double* y, double* z);
/* one-call solve on host buffers (positions in, dipoles and energy out).
 * The buffers are copied as they are: pinned buffers are DMA'd.  Non-finite
 * coordinates are detected on the device and return THP_E_INVALID, as
 * thp_set_positions does on the host. */
int thp_solve_host(thp_ctx* ctx, const double* x, const double* y, const double* z,
                   const double* rpole, double* uind, double* uinp, thp_solve_info* info);
/* bytes of device memory a context of this configuration needs */
size_t thp_footprint(const thp_config* cfg);
const char* thp_status_string(int status);

/* ---- serving: a request loop over resident systems ---------------------- */
/* A system's topology and parameters (arrays are copied at registration).
 * cfg gives n, box, aewald, cutoffs, nfft, bsorder and max_neighbors; the
 * server's precision, poleps, politer and device replace cfg's. */
typedef struct thp_system {
  thp_config cfg;
  const double* polarity;      /* [n] */
  const double* thole;         /* [n] */
  const double* pdamp;         /* [n] */
  const int* const* conn_off;  /* as thp_set_connectivity */
  const int* const* conn_idx;
  const double* scales;        /* [16] */
  const double* pole;          /* [n][13] local frame, as thp_set_frames */
  const int* zaxis;
  const int* xaxis;
  const int* axt;
} thp_system;

typedef struct thp_server_config {
  int precision;        /* THP_FP64 or THP_MIXED */
  double poleps;
  int politer;
  int device;
  size_t budget_bytes;  /* device memory all resident and pooled contexts may hold */
  int workers;          /* host threads driving the GPU; each system has its own stream */
  int max_resident;     /* systems kept on the device beyond the one being served (0: the
                           budget alone decides); past it the least recently used idle
                           system's context is re-targeted rather than a new one created */
} thp_server_config;

typedef struct thp_result {
  int status;
  int niter;
  int warm;             /* 1: started from the system's previous dipoles */
  double epol;
  double queue_ms;      /* submit -> a worker took the request */
  double latency_ms;    /* submit -> dipoles in the caller's buffers */
  double wait_ms;       /* taken -> the system's context was free and in budget */
  double setup_ms;      /* context created or re-targeted and the system loaded (0 when resident) */
  double solve_ms;      /* positions, solve and dipoles */
} thp_result;

typedef struct thp_server_stats {
  long completed, failed;
  double p50_ms, p99_ms;   /* latency over the completed requests */
  int resident, pooled;    /* contexts holding a system / idle for reuse */
  long created, reused, evicted;
  size_t bytes;            /* device bytes held by resident and pooled contexts */
} thp_server_stats;

typedef struct thp_server thp_server;

/* Starts the worker threads; touches no device until the first request. */
int thp_server_create(const thp_server_config* cfg, thp_server** out);
/* Registers (or replaces) the system under key; copies every array and
 * plans the system's FFT shape ahead of its first request. */
int thp_server_register(thp_server* s, unsigned long long key, const thp_system* sys);
/* Queues one single-point solve of system key at positions x, y, z.  They
 * are read when the request starts (pinned buffers are DMA'd); like
 * uind/uinp [n][3] (may be NULL), which receive the dipoles, they must stay
 * valid until thp_server_wait returns for the ticket.  Non-finite
 * coordinates fail the request with THP_E_INVALID.  Admission: a system whose
 * footprint exceeds the budget fails at once with THP_E_OOM_ADMISSION; others
 * wait until enough idle systems are evicted.  An evicted system's context
 * goes to a pool and is re-targeted (thp_ctx_reset) for the next system
 * instead of being freed.  A repeat of a resident system starts from its
 * previous dipoles. */
int thp_server_submit(thp_server* s, unsigned long long key, const double* x, const double* y,
                      const double* z, double* uind, double* uinp, unsigned long long* ticket);
/* Start-up: creates up to count idle contexts sized for the largest
 * registered system (within the budget) and pools them, so the first
 * requests of new systems re-target a context instead of creating one. */
int thp_server_warm(thp_server* s, int count);
/* Blocks until the request finishes; res receives its outcome. */
int thp_server_wait(thp_server* s, unsigned long long ticket, thp_result* res);
/* As thp_server_wait, but gives up after timeout_ms milliseconds of host
 * time with THP_E_TIMEOUT; the request is not cancelled and its ticket stays
 * valid for a later wait (its buffers stay the caller's responsibility until
 * then).  A caller that must not block on a stalled device polls with it. */
int thp_server_wait_for(thp_server* s, unsigned long long ticket, double timeout_ms, thp_result* res);
/* paused != 0: the workers take no new request from the queue (requests
 * already on the GPU finish); submissions still queue.  0 resumes.  For
 * draining a server for maintenance without refusing requests.  Destroying a
 * paused server still serves its queue first. */
int thp_server_pause(thp_server* s, int paused);
int thp_server_query(thp_server* s, thp_server_stats* out);
/* Waits for queued work, then frees every context. */
int thp_server_destroy(thp_server* s);

/* ---- allocation-free energy (no counterpart in the reference) ------------ */
/* For callers that cannot allocate device memory at the point of use: a host
 * code whose device memory is pooled up front by another runtime (OpenACC /
 * CUDA-Fortran data regions), work enqueued during a CUDA stream capture, or
 * a latency-critical loop that must not synchronise on cudaMalloc/cudaFree.
 * Computes Epol = -1/2 * electric * sum_i uind_i . E_p,i (kcal/mol) from
 * device arrays d_uind [n][3] and d_ef [n][2][3] (E0 with the p field second,
 * as ef(3,2,n)) into the device scalar d_epol, on the caller's current device
 * and stream (cudaStream_t as void*, NULL = legacy default stream).
 * Allocates nothing: its scratch (per-block partial sums and a counter,
 * 128 KiB) is a fixed array in the library's device image, held on every GPU
 * that loads the library until the process exits.  n must be at most
 * THP_NOALLOC_MAX_ATOMS, otherwise THP_E_INVALID.  The first call on a device
 * looks up the scratch's device address and should come before any stream
 * capture.  All calls share the scratch: calls that overlap on the GPU race,
 * so order them on one stream.  The looked-up address is kept for the life
 * of the process: calls after a cudaDeviceReset of that device are not
 * supported. */
#define THP_NOALLOC_MAX_ATOMS 4194304
int thp_epolar_noalloc(int n, const double* d_uind, const double* d_ef, double* d_epol, void* stream);

/* ---- Fortran drop-ins ---------------------------------------------------- */
/* Make ctx current and bind the module arrays the reference reads/writes:
 * atoms::x,y,z(n), mpole::rpole(13,n), polar::uind,uinp(3,n),
 * neigh::nelst(n), elst(maxelst,n) (may be NULL), energi::ep (may be NULL). */
int thp_bind_state(thp_ctx* ctx, double* x, double* y, double* z, double* rpole, double* uind,
                   double* uinp, int* nelst, int* elst, int maxelst, double* ep);
int thp_last_error(void);
/* bind deriv::dep(3,n), written by epolar1_ */
int thp_bind_gradient(thp_ctx* ctx, double* dep);
/* bind virial::vir(3,3) (may be NULL): epolar1_ adds the polarization virial
 * into it (form 0 of thp_get_virial), as epolar1c adds into vir */
int thp_bind_virial(thp_ctx* ctx, double* vir);
/* bind neigh::nvlst(n) and vlst(maxvlst,n), filled by vlistcell_ */
int thp_bind_vlist(thp_ctx* ctx, int* nvlst, int* vlst, int maxvlst);
/* bind energi::ev and deriv::dev(3,n), written by ehal1_ (may be NULL) */
int thp_bind_vdw(thp_ctx* ctx, double* ev, double* dev);
/* bind energi::em and deriv::dem(3,n), written by empole1_ (may be NULL) */
int thp_bind_mpole(thp_ctx* ctx, double* em, double* dem);
/* bind pme::qgrid2in_2d(2,n1,n2,n3), read by fphi_uind_site_ */
int thp_bind_grid(thp_ctx* ctx, double* qgrid);

/* newinduce_pme2.f:16 -- fields, guess, PCG, writeback of uind/uinp */
void newinduce_pme2_(void);
/* newinduce_pme2.f:285 -- PCG on caller arrays ef,mu(3,nrhs,n); murec unused
 * on one device.  matvec == tmatxb_pme_ runs the device loop; any other
 * matvec is called back from a host loop. */
void inducepcg_pme2_(void (*matvec)(const int* nrhs, const int* dodiag, const double* mu,
                                    double* efi),
                     const int* nrhs, const int* precnd, const double* ef, double* mu,
                     double* murec);
/* newinduce_pme.f:1392 -- efi = -T_real mu (+ mu/alpha when dodiag), overwrites efi */
void tmatxb_pme_(const int* nrhs, const int* dodiag, const double* mu, double* efi);
/* newinduce_pme.f:948 -- adds the direct permanent field to ef(3,nrhs,n) */
void efld0_direct_(const int* nrhs, double* ef);
/* newinduce_pme.f:1671 -- reciprocal permanent potential cphi(10,n) */
void efld0_recip_(double* cphi);
/* newinduce_pme.f:1919 -- reciprocal dipole field; murec/dipfieldbis unused */
void tmatxbrecip_(const double* mu, const double* murec, const int* nrhs, double* dipfield,
                  double* dipfieldbis);
/* pmestuff.f:280 grid_uind_site, batched: adds the fractional dipoles
 * fuind/fuinp(3,nsites) of atoms isite(nsites) (1-based) into the caller's
 * grid qgrid(2,n1,n2,n3) (one rank: the whole grid is local).  B-splines come
 * from the bound positions.  Spread on the device (FP64); the grid crosses
 * the bus once per call. */
void grid_uind_sites_(const int* nsites, const int* isite, const double* fuind, const double* fuinp,
                      double* qgrid);
/* pmestuff.f:746 fphi_uind_site, batched: fdip_phi1/2(10,nsites) and
 * fdip_sum_phi(20,nsites) of the caller's grid at atoms isite (1-based);
 * slot 1 of fdip_phi1/2 is zero as the reference leaves it unset. */
void fphi_uind_sites_(const int* nsites, const int* isite, const double* qgrid, double* fdip_phi1,
                      double* fdip_phi2, double* fdip_sum_phi);
/* the reference's per-site signatures (impi unused: B-splines are recomputed
 * from the positions).  Each call moves the whole grid across the bus, so
 * they exist for completeness; the batched forms above are the fast path.
 * fphi_uind_site_ reads the grid bound by thp_bind_grid. */
void grid_uind_site_(const int* isite, const int* impi, const double* fuind, const double* fuinp,
                     double* qgrid2loc);
void fphi_uind_site_(const int* isite, const int* impi, double* fdip_phi1, double* fdip_phi2,
                     double* fdip_sum_phi);
/* nblist.f:117 -- rebuild the polarization list; fills the bound elst/nelst */
void mlistcell_(void);
/* nblist.f:1148 -- the vdW list into the bound nvlst/vlst (1-based) when the
 * context has a vdW description (thp_set_vdw) and a bound vdW list
 * (thp_bind_vlist); otherwise the polarization list, as mlistcell_ */
void vlistcell_(void);
/* ehal1.f:17 -- van der Waals energy into the bound ev and its gradient
 * into the bound dev (overwritten, as ehal1c zeroes it) */
void ehal1_(void);
/* empole1.f:10 -- permanent-multipole energy into the bound em and its
 * gradient into the bound dem (overwritten, as empole1c zeroes it) */
void empole1_(void);
/* epolar.f:17 -- polarization energy into the bound ep (solves first) */
void epolar_(void);
/* epolar1.f:17 -- solve, then energy into the bound ep and the gradient into
 * the bound dep (overwritten, as epolar1c zeroes it first) */
void epolar1_(void);

/* The same entry points under names no Tinker-HP object defines, for a
 * build that keeps the reference's own sources and reaches the library
 * through the ISO_C_BINDING shim (tinker-hp_b200/fortran/thp_shim.f90): the
 * reference-named symbols above would collide there with the reference's
 * newinduce_pme2.f, newinduce_pme.f, pmestuff.f, nblist.f, epolar.f,
 * epolar1.f, empole1.f and ehal1.f objects.  inducepcg_pme2 runs its device
 * loop for either tmatxb_pme_ or thp_f_tmatxb_pme as the matvec. */
void thp_f_newinduce_pme2(void);
void thp_f_inducepcg_pme2(void (*matvec)(const int* nrhs, const int* dodiag, const double* mu,
                                         double* efi),
                          const int* nrhs, const int* precnd, const double* ef, double* mu,
                          double* murec);
void thp_f_tmatxb_pme(const int* nrhs, const int* dodiag, const double* mu, double* efi);
void thp_f_efld0_direct(const int* nrhs, double* ef);
void thp_f_efld0_recip(double* cphi);
void thp_f_tmatxbrecip(const double* mu, const double* murec, const int* nrhs, double* dipfield,
                       double* dipfieldbis);
void thp_f_grid_uind_sites(const int* nsites, const int* isite, const double* fuind, const double* fuinp,
                           double* qgrid);
void thp_f_fphi_uind_sites(const int* nsites, const int* isite, const double* qgrid, double* fdip_phi1,
                           double* fdip_phi2, double* fdip_sum_phi);
void thp_f_mlistcell(void);
void thp_f_vlistcell(void);
void thp_f_epolar(void);
void thp_f_epolar1(void);
void thp_f_empole1(void);
void thp_f_ehal1(void);

#ifdef __cplusplus
}
#endif
#endif /* THP_H */
