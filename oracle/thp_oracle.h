/*
 * thp_oracle.h -- TEST INFRASTRUCTURE, NOT THE PRODUCT.
 *
 * CPU FP64 restatement of the Tinker-HP v1.2 AMOEBA induced-dipole path
 * (v1.2/source/newinduce_pme2.f, newinduce_pme.f, pmestuff.f, damping.f,
 * erf.f, image.f, nblist.f, kewald.f, epolar.f).  It is the checker for the
 * CUDA library: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs may load it.
 *
 * Parity status: UNPINNED by the reference.  The reference is Fortran+MPI
 * (no Fortran compiler or MPI in this image) and ships no golden vectors for
 * this path, so this restatement is pinned by self-consistency tests instead
 * (CG residual, Ewald-alpha invariance, classical-Ewald cross-check,
 * numpy FFT cross-check, translation invariance).
 *
 * Conventions: 0-based atom indices; per-atom vectors interleaved as in the
 * reference's (3,nrhs,n) Fortran arrays, i.e. v[(i*nrhs + r)*3 + c].
 * Orthogonal periodic boxes only.
 */
#ifndef THP_ORACLE_H
#define THP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* connectivity list slots, same meaning as the reference's couple/polgrp
 * modules (n12/i12 ... n15/i15, np11/ip11 ... np14/ip14) */
enum { OR_I12 = 0, OR_I13, OR_I14, OR_I15, OR_IP11, OR_IP12, OR_IP13, OR_IP14, OR_NCONN };

typedef struct OrSystem {
  int n;
  double xbox, ybox, zbox;
  const double* x;
  const double* y;
  const double* z;
  const double* rpole;    /* [n][13] global-frame multipoles (e, e*A, e*A^2) */
  const double* polarity; /* [n] A^3 */
  const double* thole;    /* [n] */
  const double* pdamp;    /* [n] polarity^(1/6) */
  const int* conn_off[OR_NCONN]; /* CSR offsets [n+1] (may be NULL = empty) */
  const int* conn_idx[OR_NCONN]; /* CSR indices, 0-based */
  double p_scale[4];  /* p2scale..p5scale */
  double pi_scale[4]; /* p2iscale..p5iscale */
  double d_scale[4];  /* d1scale..d4scale */
  double u_scale[4];  /* u1scale..u4scale */
  double aewald;
  double ewaldcut;    /* real-space cutoff (A) */
  double lbuffer;     /* neighbor-list buffer (A) */
  double vdwcut;      /* only sizes the cells of build_cell_list */
  int nfft1, nfft2, nfft3;
  int bsorder;
  int politer;
  double poleps;
  int nthreads;       /* OpenMP threads for the CPU baseline; 1 = scalar */
  double m_scale[4];  /* m2scale..m5scale (initprm.f:413-416, water03.prm:34-37) */
} OrSystem;

typedef struct OrSolveInfo {
  int niter;
  int converged;
  double resnrm;
  double ene[2];
} OrSolveInfo;

typedef struct OrCtx OrCtx;

/* status codes (same numbering as the CUDA library's THP_* codes) */
#define OR_OK 0
#define OR_E_LIST_OVERFLOW 2
#define OR_E_BOX_TOO_SMALL 8

OrCtx* or_create(const OrSystem* sys);
void or_destroy(OrCtx* c);

/* Half neighbor list in the reference's layout: nelst[i], elst[i*maxelst+j]
 * holding k>i (0-based) in the reference's cell-traversal order. */
int or_mlistcell(OrCtx* c, int maxelst, int* nelst, int* elst);

void or_efld0_direct(OrCtx* c, double* ef /*[n][2][3]*/);
void or_tmatxb_pme(OrCtx* c, int nrhs, int dodiag, const double* mu, double* efi);
void or_efld0_recip(OrCtx* c, double* cphi /*[n][10]*/);
void or_tmatxbrecip(OrCtx* c, int nrhs, const double* mu, double* dipfield);

/* Full driver: fields, guess (mu_guess==NULL -> alpha*E0), PCG, writeback.
 * ef_out (optional) receives E0 [n][2][3]. */
int or_newinduce_pme2(OrCtx* c, const double* mu_guess, double* uind, double* uinp,
                      double* ef_out, OrSolveInfo* info);

/* epolar0c: polarization energy (kcal/mol) from uind and the permanent field
 * of the last or_efld0_recip call. Returns also the three parts. */
double or_epolar(OrCtx* c, const double* uind, double* ereal, double* erecip, double* eself);

/* epolar1c (epolar1.f:57-372): polarization energy and its gradient dep
 * [n][3] (kcal/mol/A) from converged uind/uinp; frames (zaxis, xaxis, axt
 * as in or_rotpole) distribute the torques (torque.f:6).  vir (may be NULL):
 * the internal virial vir(3,3) (kcal/mol, symmetric, row-major) of the
 * TINFOIL boundary as the reference accumulates it; vir_frame (may be NULL):
 * the frame-atom virial of the reciprocal and self torques, which the
 * reference leaves out (vir + vir_frame is the strain derivative). */
int or_epolar1(OrCtx* c, const double* uind, const double* uinp, const int* zaxis, const int* xaxis,
               const int* axt, double* dep, double* ep, double* vir, double* vir_frame);

/* empole1c (empole1.f:42-340): permanent-multipole energy and gradient dem
 * [n][3] (kcal/mol/A) at the current positions, TINFOIL boundary; needs the
 * list (or_mlistcell).  parts (may be NULL) [4]: total, real, recip, self.
 * vir (may be NULL): the internal virial vir(3,3) as the reference
 * accumulates it (emrecip1's site terms and scalar sum, emreal1c's pair and
 * torque frame terms); vir_frame (may be NULL): the frame-atom virial of the
 * reciprocal torques, which the reference leaves out. */
int or_empole1(OrCtx* c, const int* zaxis, const int* xaxis, const int* axt, double* dem, double* parts,
               double* vir, double* vir_frame);

/* van der Waals parameters of ehal1c (kvdw.f): per-atom class (0-based),
 * pair tables [nclass][nclass] of Rmin and epsilon (combined by the
 * caller's rules) and their 1-4 forms, reduction parent (0-based) and factor,
 * the 1-2..1-5 scales, cutoff and taper start (absolute, A), buffer
 * constants. */
typedef struct OrVdw {
  int nclass;
  const int* cls;
  const double* radmin;
  const double* eps;
  const double* radmin4;
  const double* eps4;
  const int* ired;
  const double* kred;
  double v_scale[4];
  double vdwcut, vdwtaper;
  double ghal, dhal;
} OrVdw;

/* ehal1c (ehal1.f:69-482, standard branch): buffered 14-7 energy and
 * gradient dev [n][3] over the pairs of the vdW list (vlistcell,
 * nblist.f:1148-1305: reduced coordinates, half list within vdwcut +
 * lbuffer), with the 5th-degree taper (switch.f:80-117).  vir (may be
 * NULL): the internal virial vir(3,3) of the pairs (ehal1.f:431-446). */
int or_ehal1(OrCtx* c, const OrVdw* v, double* dev, double* ev, double* vir);

/* grid_uind_site (pmestuff.f:280-405) for nsites sites (0-based atom
 * numbers): adds the fractional dipoles fuind/fuinp (3 per site) into the
 * interleaved complex grid [n3][n2][n1] (qgrid2in_2d(2,n1,n2,n3)). */
int or_grid_uind_sites(OrCtx* c, int nsites, const int* isite, const double* fuind, const double* fuinp,
                       double* grid);
/* fphi_uind_site (pmestuff.f:746-1045) for nsites sites on a caller grid:
 * phi1/phi2 [nsites][10] (fdip_phi1/2, slot 0 unused), sum [nsites][20]. */
int or_fphi_uind_sites(OrCtx* c, int nsites, const int* isite, const double* grid, double* phi1, double* phi2,
                       double* sum);

/* rotpole for the water frames used here (Bisector and Z-then-X),
 * pole [n][13] local frame -> rpole [n][13] global frame.
 * axt: 1 = Z-then-X, 2 = Bisector. zaxis/xaxis 0-based. */
void or_rotpole(int n, const double* x, const double* y, const double* z, const double* pole,
                const int* zaxis, const int* xaxis, const int* axt, double* rpole);

/* ewaldcof: Ewald coefficient for a cutoff at 1e-8 tolerance (kewald.f:575). */
double or_ewaldcof(double cutoff);

/* Cody rational erfc (erf.f:44) exposed for tests. */
double or_erfc(double x);

/* 3-D complex FFT used by the oracle (tests cross-check it with numpy).
 * data: interleaved complex [n3][n2][n1]; sign -1 forward, +1 backward. */
void or_fft3d(double* data, int n1, int n2, int n3, int sign);

#ifdef __cplusplus
}
#endif
#endif
