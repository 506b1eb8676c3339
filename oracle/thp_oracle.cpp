// thp_oracle.cpp -- TEST INFRASTRUCTURE, NOT THE PRODUCT.
//
// CPU FP64 restatement of the Tinker-HP v1.2 induced-dipole polarization path.
// Each routine cites the reference routine it restates (paths are relative to
// the Tinker-HP repository).  Only tests/, __graft_entry__.smoke() and the CPU
// baseline legs of bench.py load this code; the CUDA library never does.
//
// Parity status: unpinned by the reference (no Fortran toolchain here, no
// golden vectors for this path); pinned by self-consistency tests.
//
// Build: oracle/Makefile (-O2 -ffp-contract=off so that r^2 tests round like
// the reference's unfused Fortran arithmetic).

#include "thp_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.141592653589793238;
constexpr double kSqrtPi = 1.772453850905516027;
constexpr double kElectric = 332.063714;  // MOD_units.f:81 (coulomb)
constexpr double kTinyPol = (double)1e-5f; // MOD_polar.f:36 (single-precision literal)

int nthreads_of(const OrSystem* s) { return s->nthreads > 0 ? s->nthreads : 1; }

// ---------------------------------------------------------------------------
// image.f:113-138, orthogonal branch
struct Cell {
  double xcell, ycell, zcell, xcell2, ycell2, zcell2;
};

inline void image1(double& r, double cell, double cell2) {
  if (std::fabs(r) > cell2) {
    double cel = std::copysign(cell, r);
    r = r - cel * std::floor(std::fabs(r) / cell);
    if (std::fabs(r) > cell2) r = r - std::copysign(cell, r);
  }
}
inline void image(const Cell& c, double& xr, double& yr, double& zr) {
  image1(xr, c.xcell, c.xcell2);
  image1(yr, c.ycell, c.ycell2);
  image1(zr, c.zcell, c.zcell2);
}

// ---------------------------------------------------------------------------
// erf.f:44-200 (erfcore, mode 1): W. J. Cody, "Rational Chebyshev
// Approximations for the Error Function", Math. Comp. 23, 631-638 (1969).
double erfc_cody(double arg) {
  static const double a[5] = {3.16112374387056560e0, 1.13864154151050156e2, 3.77485237685302021e2,
                              3.20937758913846947e3, 1.85777706184603153e-1};
  static const double b[4] = {2.36012909523441209e1, 2.44024637934444173e2, 1.28261652607737228e3,
                              2.84423683343917062e3};
  static const double c[9] = {5.64188496988670089e-1, 8.88314979438837594e0, 6.61191906371416295e1,
                              2.98635138197400131e2,  8.81952221241769090e2, 1.71204761263407058e3,
                              2.05107837782607147e3,  1.23033935479799725e3, 2.15311535474403846e-8};
  static const double d[8] = {1.57449261107098347e1, 1.17693950891312499e2, 5.37181101862009858e2,
                              1.62138957456669019e3, 3.29079923573345963e3, 4.36261909014324716e3,
                              3.43936767414372164e3, 1.23033935480374942e3};
  static const double p[6] = {3.05326634961232344e-1, 3.60344899949804439e-1, 1.25781726111229246e-1,
                              1.60837851487422766e-2, 6.58749161529837803e-4, 1.63153871373020978e-2};
  static const double q[5] = {2.56852019228982242e0, 1.87295284992346047e0, 5.27905102951428412e-1,
                              6.05183413124413191e-2, 2.33520497626869185e-3};
  const double sqrpi = 5.6418958354775628695e-1;
  const double xtiny = 1.11e-16, xbig = 26.543;
  double x = arg, y = std::fabs(x), result;
  if (y <= 0.46875) {
    double ysq = 0.0;
    if (y > xtiny) ysq = y * y;
    double xnum = a[4] * ysq, xden = ysq;
    for (int i = 0; i < 3; ++i) {
      xnum = (xnum + a[i]) * ysq;
      xden = (xden + b[i]) * ysq;
    }
    result = x * (xnum + a[3]) / (xden + b[3]);
    result = 1.0 - result;
  } else if (y <= 4.0) {
    double xnum = c[8] * y, xden = y;
    for (int i = 0; i < 7; ++i) {
      xnum = (xnum + c[i]) * y;
      xden = (xden + d[i]) * y;
    }
    result = (xnum + c[7]) / (xden + d[7]);
    double ysq = std::trunc(16.0 * y) / 16.0;
    double del = (y - ysq) * (y + ysq);
    result = std::exp(-ysq * ysq - del) * result;
    if (x < 0.0) result = 2.0 - result;
  } else {
    result = 0.0;
    if (y < xbig) {
      double ysq = 1.0 / (y * y);
      double xnum = p[5] * ysq, xden = ysq;
      for (int i = 0; i < 4; ++i) {
        xnum = (xnum + p[i]) * ysq;
        xden = (xden + q[i]) * ysq;
      }
      result = ysq * (xnum + p[4]) / (xden + q[4]);
      result = (sqrpi - result) / y;
      ysq = std::trunc(16.0 * y) / 16.0;
      double del = (y - ysq) * (y + ysq);
      result = std::exp(-ysq * ysq - del) * result;
    }
    if (x < 0.0) result = 2.0 - result;
  }
  return result;
}

// damping.f:17-55 (dampewald)
inline void dampewald(int rorder, double r, double r2, double scale, double aewald, double* dmpe) {
  for (int i = 1; i <= rorder; ++i) dmpe[i] = scale;
  double ra = aewald * r;
  double bn[6];
  bn[0] = erfc_cody(ra) / r;
  dmpe[1] = scale * bn[0];
  double expterm = std::exp(-ra * ra);
  double aesq2 = 2.0 * aewald * aewald;
  double afac = 0.0;
  if (aewald > 0.0) afac = 1.0 / (kSqrtPi * aewald);
  int niter = (rorder - 1) / 2;
  for (int i = 1; i <= niter; ++i) {
    double bfac = (double)(2 * i - 1);
    afac = aesq2 * afac;
    bn[i] = (bfac * bn[i - 1] + afac * expterm) / r2;
    dmpe[2 * i + 1] = scale * bn[i];
  }
}

// damping.f:74-124 (dampthole) == damping.f:142-216 (damptholed, AMOEBA branch)
inline void dampthole(double pdi, double pdk, double thi, double thk, int rorder, double r,
                      double* dmpik) {
  for (int j = 1; j <= rorder; ++j) dmpik[j] = 1.0;
  double damp = pdi * pdk;
  // kpolar.f:281-290 pair rule: min, or max when the min is zero
  double pgamma = std::min(thi, thk);
  if (pgamma == 0.0) pgamma = std::max(thi, thk);
  if (damp != 0.0 && pgamma != 0.0) {
    double t = r / damp;
    damp = pgamma * (t * t * t);
    if (damp < 50.0) {
      double expdamp = std::exp(-damp);
      dmpik[3] = 1.0 - expdamp;
      dmpik[5] = 1.0 - expdamp * (1.0 + damp);
      if (rorder >= 7) {
        double damp2 = damp * damp;
        dmpik[7] = 1.0 - expdamp * (1.0 + damp + 0.6 * damp2);
        if (rorder >= 9) {
          double damp3 = damp * damp2;
          dmpik[9] = 1.0 - expdamp * (1.0 + damp + (18.0 / 35.0) * damp2 + (9.0 / 35.0) * damp3);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Mixed-radix complex FFT (factors 2, 3, 5 and any other prime by direct DFT),
// unnormalised, used in place of 2DECOMP's generic engine (fft_mpi.f90:65,115).
using cd = std::complex<double>;

void factorize(int n, std::vector<int>& f) {
  f.clear();
  for (int p : {4, 2, 3, 5}) {
    while (n % p == 0) {
      f.push_back(p);
      n /= p;
    }
  }
  for (int p = 7; n > 1; p += 2)
    while (n % p == 0) {
      f.push_back(p);
      n /= p;
    }
}

void fft_rec(const cd* in, cd* out, int n, int stride, int sign, const int* fac, const cd* tw,
             int twn, cd* scratch) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = fac[0], m = n / p;
  for (int q = 0; q < p; ++q) fft_rec(in + q * stride, out + q * m, m, stride * p, sign, fac + 1, tw, twn, scratch);
  // butterfly: X[k + m*s] = sum_q W_n^{q(k+m s)} Y_q[k]
  int step = twn / n;
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) scratch[q] = out[q * m + k];
    for (int s = 0; s < p; ++s) {
      cd acc = 0.0;
      int idx = k + m * s;
      for (int q = 0; q < p; ++q) {
        long e = ((long)q * idx) % n;
        cd w = tw[e * step];
        if (sign > 0) w = std::conj(w);
        acc += w * scratch[q];
      }
      out[idx] = acc;
    }
  }
}

struct Fft1d {
  int n = 0;
  std::vector<int> fac;
  std::vector<cd> tw;  // exp(-2 pi i k / n)
  void init(int n_) {
    n = n_;
    factorize(n, fac);
    fac.push_back(1);
    tw.resize(n);
    for (int k = 0; k < n; ++k) tw[k] = cd(std::cos(2.0 * kPi * k / n), -std::sin(2.0 * kPi * k / n));
  }
  void run(cd* line, int sign, cd* tmp, cd* scratch) const {
    std::memcpy(tmp, line, sizeof(cd) * n);
    fft_rec(tmp, line, n, 1, sign, fac.data(), tw.data(), n, scratch);
  }
};

void fft3d_impl(cd* g, int n1, int n2, int n3, int sign, int nthr) {
  Fft1d f1, f2, f3;
  f1.init(n1);
  f2.init(n2);
  f3.init(n3);
  int nmax = std::max(n1, std::max(n2, n3));
  // axis 1 (contiguous)
#pragma omp parallel num_threads(nthr)
  {
    std::vector<cd> line(nmax), tmp(nmax), scr(nmax);
#pragma omp for schedule(static)
    for (int l = 0; l < n2 * n3; ++l) f1.run(g + (size_t)l * n1, sign, tmp.data(), scr.data());
#pragma omp for schedule(static)
    for (int l = 0; l < n1 * n3; ++l) {
      int i = l % n1, k = l / n1;
      for (int j = 0; j < n2; ++j) line[j] = g[((size_t)k * n2 + j) * n1 + i];
      f2.run(line.data(), sign, tmp.data(), scr.data());
      for (int j = 0; j < n2; ++j) g[((size_t)k * n2 + j) * n1 + i] = line[j];
    }
#pragma omp for schedule(static)
    for (int l = 0; l < n1 * n2; ++l) {
      for (int k = 0; k < n3; ++k) line[k] = g[(size_t)k * n1 * n2 + l];
      f3.run(line.data(), sign, tmp.data(), scr.data());
      for (int k = 0; k < n3; ++k) g[(size_t)k * n1 * n2 + l] = line[k];
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
struct OrCtx {
  OrSystem s;
  Cell cell;
  double recip[3][3];  // recip[i][j] == reference recip(i+1,j+1)
  double volbox;
  // neighbor list (half, k>i)
  int maxelst = 0;
  std::vector<int> nelst, elst;
  bool have_list = false;
  // PME state
  int bsorder = 5, grdoff = 0, nlpts = 0, nrpts = 0;
  std::vector<double> bsmod1, bsmod2, bsmod3;
  std::vector<double> qfac;          // [n3][n2][n1]
  std::vector<double> theta1, theta2, theta3;  // [n][5][4]: (level j, point m) -> [(i*bs + m)*4 + j]
  std::vector<int> igrid;            // [n][3]
  std::vector<double> fphirec;       // [n][20]
  std::vector<cd> grid;              // [n3][n2][n1]
  bool have_bspline = false;
};

namespace {

// lattice.f:20-126 for orthogonal boxes
void setup_box(OrCtx* c) {
  const OrSystem& s = c->s;
  c->cell.xcell = s.xbox;
  c->cell.ycell = s.ybox;
  c->cell.zcell = s.zbox;
  c->cell.xcell2 = 0.5 * s.xbox;
  c->cell.ycell2 = 0.5 * s.ybox;
  c->cell.zcell2 = 0.5 * s.zbox;
  double ar1 = s.xbox, ar2 = 0.0, ar3 = 0.0;
  double br1 = s.ybox * 0.0, br2 = s.ybox * 1.0, br3 = 0.0;
  double cr1 = s.zbox * 0.0, cr2 = s.zbox * 0.0, cr3 = s.zbox * 1.0;
  c->volbox = s.xbox * s.ybox * s.zbox;
  double v = c->volbox;
  c->recip[0][0] = (br2 * cr3 - cr2 * br3) / v;
  c->recip[1][0] = (br3 * cr1 - cr3 * br1) / v;
  c->recip[2][0] = (br1 * cr2 - cr1 * br2) / v;
  c->recip[0][1] = (cr2 * ar3 - ar2 * cr3) / v;
  c->recip[1][1] = (cr3 * ar1 - ar3 * cr1) / v;
  c->recip[2][1] = (cr1 * ar2 - ar1 * cr2) / v;
  c->recip[0][2] = (ar2 * br3 - br2 * ar3) / v;
  c->recip[1][2] = (ar3 * br1 - br3 * ar1) / v;
  c->recip[2][2] = (ar1 * br2 - br1 * ar2) / v;
}

// kewald.f:693-717 (bspline)
void bspline_coef(double x, int n, double* cc /*1-based*/) {
  cc[1] = 1.0 - x;
  cc[2] = x;
  for (int k = 3; k <= n; ++k) {
    double denom = 1.0 / (double)(k - 1);
    cc[k] = x * cc[k - 1] * denom;
    for (int i = 1; i <= k - 2; ++i) cc[k - i] = ((x + (double)i) * cc[k - i - 1] + ((double)(k - i) - x) * cc[k - i]) * denom;
    cc[1] = (1.0 - x) * cc[1] * denom;
  }
}

// kewald.f:747-812 (dftmod)
void dftmod(std::vector<double>& bsmod, const std::vector<double>& bsarray, int nfft, int order) {
  bsmod.assign(nfft + 1, 0.0);  // 1-based
  double factor = 2.0 * kPi / (double)nfft;
  for (int i = 1; i <= nfft; ++i) {
    double sum1 = 0.0, sum2 = 0.0;
    for (int j = 1; j <= nfft; ++j) {
      double arg = factor * (double)((i - 1) * (j - 1));
      sum1 = sum1 + bsarray[j] * std::cos(arg);
      sum2 = sum2 + bsarray[j] * std::sin(arg);
    }
    bsmod[i] = sum1 * sum1 + sum2 * sum2;
  }
  double eps = 1.0e-7;
  if (bsmod[1] < eps) bsmod[1] = 0.5 * bsmod[2];
  for (int i = 2; i <= nfft - 1; ++i)
    if (bsmod[i] < eps) bsmod[i] = 0.5 * (bsmod[i - 1] + bsmod[i + 1]);
  if (bsmod[nfft] < eps) bsmod[nfft] = 0.5 * bsmod[nfft - 1];
  int jcut = 50;
  int order2 = 2 * order;
  for (int i = 1; i <= nfft; ++i) {
    int k = i - 1;
    if (i > nfft / 2) k = k - nfft;
    double zeta;
    if (k == 0) {
      zeta = 1.0;
    } else {
      double sum1 = 1.0, sum2 = 1.0;
      double fac = kPi * (double)k / (double)nfft;
      for (int j = 1; j <= jcut; ++j) {
        double arg = fac / (fac + kPi * (double)j);
        sum1 = sum1 + std::pow(arg, order);
        sum2 = sum2 + std::pow(arg, order2);
      }
      for (int j = 1; j <= jcut; ++j) {
        double arg = fac / (fac - kPi * (double)j);
        sum1 = sum1 + std::pow(arg, order);
        sum2 = sum2 + std::pow(arg, order2);
      }
      zeta = sum2 / sum1;
    }
    bsmod[i] = bsmod[i] * zeta * zeta;
  }
}

// kewald.f:672-690 (moduli) and newinduce_pme.f:1802-1854 (qfac)
void setup_pme(OrCtx* c) {
  const OrSystem& s = c->s;
  c->bsorder = s.bsorder;
  c->nlpts = (c->bsorder - 1) / 2;
  c->nrpts = c->bsorder - c->nlpts - 1;
  c->grdoff = (c->bsorder + 1) / 2 + 1;
  int maxfft = std::max(s.nfft1, std::max(s.nfft2, s.nfft3));
  std::vector<double> arr(c->bsorder + 2, 0.0), bsarray(maxfft + 2, 0.0);
  bspline_coef(0.0, c->bsorder, arr.data());
  for (int i = 2; i <= c->bsorder + 1; ++i) bsarray[i] = arr[i - 1];
  dftmod(c->bsmod1, bsarray, s.nfft1, c->bsorder);
  dftmod(c->bsmod2, bsarray, s.nfft2, c->bsorder);
  dftmod(c->bsmod3, bsarray, s.nfft3, c->bsorder);
  size_t ng = (size_t)s.nfft1 * s.nfft2 * s.nfft3;
  c->qfac.assign(ng, 0.0);
  c->grid.assign(ng, cd(0.0, 0.0));
  double pterm = (kPi / s.aewald) * (kPi / s.aewald);
  double volterm = kPi * c->volbox;
  int nf1 = (s.nfft1 + 1) / 2, nf2 = (s.nfft2 + 1) / 2, nf3 = (s.nfft3 + 1) / 2;
  for (int k3 = 1; k3 <= s.nfft3; ++k3)
    for (int k2 = 1; k2 <= s.nfft2; ++k2)
      for (int k1 = 1; k1 <= s.nfft1; ++k1) {
        int m1 = k1 - 1, m2 = k2 - 1, m3 = k3 - 1;
        if (k1 > nf1) m1 -= s.nfft1;
        if (k2 > nf2) m2 -= s.nfft2;
        if (k3 > nf3) m3 -= s.nfft3;
        size_t idx = ((size_t)(k3 - 1) * s.nfft2 + (k2 - 1)) * s.nfft1 + (k1 - 1);
        if (m1 == 0 && m2 == 0 && m3 == 0) continue;
        double r1 = m1, r2 = m2, r3 = m3;
        double h1 = c->recip[0][0] * r1 + c->recip[0][1] * r2 + c->recip[0][2] * r3;
        double h2 = c->recip[1][0] * r1 + c->recip[1][1] * r2 + c->recip[1][2] * r3;
        double h3 = c->recip[2][0] * r1 + c->recip[2][1] * r2 + c->recip[2][2] * r3;
        double hsq = h1 * h1 + h2 * h2 + h3 * h3;
        double term = -pterm * hsq;
        if (term > -50.0) {
          double denom = volterm * hsq * c->bsmod1[k1] * c->bsmod2[k2] * c->bsmod3[k3];
          c->qfac[idx] = std::exp(term) / denom;
        }
      }
}

// pmestuff.f:64-157 (bsplgen), level 4 (use_polar)
void bsplgen(double w, int bsorder, double* thetai /*[bsorder][4]*/) {
  const int level = 4;
  double temp[12][12];  // 1-based (maxorder <= 10)
  temp[2][2] = w;
  temp[2][1] = 1.0 - w;
  temp[3][3] = 0.5 * w * temp[2][2];
  temp[3][2] = 0.5 * ((1.0 + w) * temp[2][1] + (2.0 - w) * temp[2][2]);
  temp[3][1] = 0.5 * (1.0 - w) * temp[2][1];
  for (int i = 4; i <= bsorder; ++i) {
    int k = i - 1;
    double denom = 1.0 / (double)k;
    temp[i][i] = denom * w * temp[k][k];
    for (int j = 1; j <= i - 2; ++j)
      temp[i][i - j] = denom * ((w + (double)j) * temp[k][i - j - 1] + ((double)(i - j) - w) * temp[k][i - j]);
    temp[i][1] = denom * (1.0 - w) * temp[k][1];
  }
  int k = bsorder - 1;
  temp[k][bsorder] = temp[k][bsorder - 1];
  for (int i = bsorder - 1; i >= 2; --i) temp[k][i] = temp[k][i - 1] - temp[k][i];
  temp[k][1] = -temp[k][1];
  // second derivative
  k = bsorder - 2;
  temp[k][bsorder - 1] = temp[k][bsorder - 2];
  for (int i = bsorder - 2; i >= 2; --i) temp[k][i] = temp[k][i - 1] - temp[k][i];
  temp[k][1] = -temp[k][1];
  temp[k][bsorder] = temp[k][bsorder - 1];
  for (int i = bsorder - 1; i >= 2; --i) temp[k][i] = temp[k][i - 1] - temp[k][i];
  temp[k][1] = -temp[k][1];
  // third derivative
  k = bsorder - 3;
  temp[k][bsorder - 2] = temp[k][bsorder - 3];
  for (int i = bsorder - 3; i >= 2; --i) temp[k][i] = temp[k][i - 1] - temp[k][i];
  temp[k][1] = -temp[k][1];
  temp[k][bsorder - 1] = temp[k][bsorder - 2];
  for (int i = bsorder - 2; i >= 2; --i) temp[k][i] = temp[k][i - 1] - temp[k][i];
  temp[k][1] = -temp[k][1];
  temp[k][bsorder] = temp[k][bsorder - 1];
  for (int i = bsorder - 1; i >= 2; --i) temp[k][i] = temp[k][i - 1] - temp[k][i];
  temp[k][1] = -temp[k][1];
  for (int i = 1; i <= bsorder; ++i)
    for (int j = 1; j <= level; ++j) thetai[(i - 1) * 4 + (j - 1)] = temp[bsorder - j + 1][i];
}

// pmestuff.f:13-51 (bspline_fill_site) for every site
void bspline_fill(OrCtx* c) {
  const OrSystem& s = c->s;
  int n = s.n, bs = c->bsorder;
  c->theta1.resize((size_t)n * bs * 4);
  c->theta2.resize((size_t)n * bs * 4);
  c->theta3.resize((size_t)n * bs * 4);
  c->igrid.resize((size_t)n * 3);
  const double eps = 1.0e-8;
  int nf[3] = {s.nfft1, s.nfft2, s.nfft3};
  double* th[3] = {c->theta1.data(), c->theta2.data(), c->theta3.data()};
  for (int i = 0; i < n; ++i) {
    double xi = s.x[i], yi = s.y[i], zi = s.z[i];
    for (int d = 0; d < 3; ++d) {
      double w = xi * c->recip[0][d] + yi * c->recip[1][d] + zi * c->recip[2][d];
      double fr = (double)nf[d] * (w - std::round(w) + 0.5);
      int ifr = (int)(fr - eps);
      w = fr - (double)ifr;
      c->igrid[i * 3 + d] = ifr - bs;
      bsplgen(w, bs, th[d] + (size_t)i * bs * 4);
    }
  }
  c->have_bspline = true;
}

inline int wrap0(int v, int n) { return v < 0 ? v + n : v; }

// 0-based grid index of stencil point t (0..bsorder-1) along one axis
// (grid_*_site with adjust: kk = igrid+grdoff-nlpts+t, 1-based, wrapped once)
inline int stencil_index(const OrCtx* c, int ig, int t, int nfft) {
  int kk = ig + c->grdoff - c->nlpts + t;  // 1-based
  if (kk < 1) kk += nfft;
  return kk - 1;
}

// cart_to_frac (pmestuff.f:1131-1185)
void cart_to_frac(const OrCtx* c, double ctf[10][10]) {
  const OrSystem& s = c->s;
  double a[3][3];
  int nf[3] = {s.nfft1, s.nfft2, s.nfft3};
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) a[d][i] = (double)nf[d] * c->recip[i][d];
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j) ctf[j][i] = 0.0;
  ctf[0][0] = 1.0;
  for (int i = 1; i < 4; ++i)
    for (int j = 1; j < 4; ++j) ctf[i][j] = a[i - 1][j - 1];
  const int qi1[6] = {0, 1, 2, 0, 0, 1}, qi2[6] = {0, 1, 2, 1, 2, 2};
  for (int i1 = 0; i1 < 3; ++i1) {
    int k = qi1[i1];
    for (int i2 = 0; i2 < 6; ++i2) {
      int i = qi1[i2], j = qi2[i2];
      ctf[i1 + 4][i2 + 4] = a[k][i] * a[k][j];
    }
  }
  for (int i1 = 3; i1 < 6; ++i1) {
    int k = qi1[i1], m = qi2[i1];
    for (int i2 = 0; i2 < 6; ++i2) {
      int i = qi1[i2], j = qi2[i2];
      ctf[i1 + 4][i2 + 4] = a[k][i] * a[m][j] + a[k][j] * a[m][i];
    }
  }
}

// frac_to_cart (pmestuff.f:1237-1290)
void frac_to_cart(const OrCtx* c, double ftc[10][10]) {
  const OrSystem& s = c->s;
  double a[3][3];
  int nf[3] = {s.nfft1, s.nfft2, s.nfft3};
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) a[i][d] = (double)nf[d] * c->recip[i][d];
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j) ftc[j][i] = 0.0;
  ftc[0][0] = 1.0;
  for (int i = 1; i < 4; ++i)
    for (int j = 1; j < 4; ++j) ftc[i][j] = a[i - 1][j - 1];
  const int qi1[6] = {0, 1, 2, 0, 0, 1}, qi2[6] = {0, 1, 2, 1, 2, 2};
  for (int i1 = 0; i1 < 3; ++i1) {
    int k = qi1[i1];
    for (int i2 = 0; i2 < 3; ++i2) {
      int i = qi1[i2];
      ftc[i1 + 4][i2 + 4] = a[k][i] * a[k][i];
    }
    for (int i2 = 3; i2 < 6; ++i2) {
      int i = qi1[i2], j = qi2[i2];
      ftc[i1 + 4][i2 + 4] = 2.0 * a[k][i] * a[k][j];
    }
  }
  for (int i1 = 3; i1 < 6; ++i1) {
    int k = qi1[i1], m = qi2[i1];
    for (int i2 = 0; i2 < 3; ++i2) {
      int i = qi1[i2];
      ftc[i1 + 4][i2 + 4] = a[k][i] * a[m][i];
    }
    for (int i2 = 3; i2 < 6; ++i2) {
      int i = qi1[i2], j = qi2[i2];
      ftc[i1 + 4][i2 + 4] = a[k][i] * a[m][j] + a[m][i] * a[k][j];
    }
  }
}

// Grid spread, parallel over z-plane slabs so that every grid point is
// written by one thread (the same sums as the reference's serial loop,
// accumulated per point in atom order).
template <class F>
void spread_sites(OrCtx* c, F&& site_terms) {
  const OrSystem& s = c->s;
  int n = s.n, bs = c->bsorder;
  int n1 = s.nfft1, n2 = s.nfft2, n3 = s.nfft3;
  std::fill(c->grid.begin(), c->grid.end(), cd(0.0, 0.0));
  int nthr = nthreads_of(&s);
#pragma omp parallel num_threads(nthr)
  {
    int tid = 0, nt = 1;
#ifdef _OPENMP
    tid = omp_get_thread_num();
    nt = omp_get_num_threads();
#endif
    int z0 = (int)((long)n3 * tid / nt), z1 = (int)((long)n3 * (tid + 1) / nt);
    for (int i = 0; i < n; ++i) {
      const double* t1 = &c->theta1[(size_t)i * bs * 4];
      const double* t2 = &c->theta2[(size_t)i * bs * 4];
      const double* t3 = &c->theta3[(size_t)i * bs * 4];
      const int* ig = &c->igrid[i * 3];
      for (int it3 = 0; it3 < bs; ++it3) {
        int k = stencil_index(c, ig[2], it3, n3);
        if (k < z0 || k >= z1) continue;
        for (int it2 = 0; it2 < bs; ++it2) {
          int j = stencil_index(c, ig[1], it2, n2);
          for (int it1 = 0; it1 < bs; ++it1) {
            int ii = stencil_index(c, ig[0], it1, n1);
            cd add = site_terms(i, t1 + it1 * 4, t2 + it2 * 4, t3 + it3 * 4);
            c->grid[((size_t)k * n2 + j) * n1 + ii] += add;
          }
        }
      }
    }
  }
}

// fphi_uind_site (pmestuff.f:746-1045) for site i on grid g: phi1/phi2 hold
// fdip_phi1/2(1:10) (index 0 unused, 1..9 = 100,010,001,200,020,002,110,101,
// 011 of the Re / Im grid), sum holds fdip_sum_phi(1:20) of Re + Im.
void fphi_dip_site(const OrCtx* c, int i, const cd* g, double phi1[10], double phi2[10], double sum[20]);

void convolve(OrCtx* c) {
  const OrSystem& s = c->s;
  int nthr = nthreads_of(&s);
  fft3d_impl(c->grid.data(), s.nfft1, s.nfft2, s.nfft3, -1, nthr);
  size_t ng = c->grid.size();
#pragma omp parallel for num_threads(nthr) schedule(static)
  for (long q = 0; q < (long)ng; ++q) c->grid[q] *= c->qfac[q];
  fft3d_impl(c->grid.data(), s.nfft1, s.nfft2, s.nfft3, +1, nthr);
}

// grid value at stencil point, 0-based index per fphi_*_site:
// i0 = igrid + it (it=1..bs), i = i0 mod nfft
inline int gather_index(int ig, int it1based, int nfft) {
  int i0 = ig + it1based;
  return i0 >= 0 ? i0 : i0 + nfft;
}

// fphi_mpole_site (pmestuff.f:453-600): 20 potential derivatives per site
void fphi_mpole(OrCtx* c) {
  const OrSystem& s = c->s;
  int n = s.n, bs = c->bsorder;
  c->fphirec.assign((size_t)n * 20, 0.0);
  int nthr = nthreads_of(&s);
#pragma omp parallel for num_threads(nthr) schedule(static)
  for (int i = 0; i < n; ++i) {
    const double* th1 = &c->theta1[(size_t)i * bs * 4];
    const double* th2 = &c->theta2[(size_t)i * bs * 4];
    const double* th3 = &c->theta3[(size_t)i * bs * 4];
    const int* ig = &c->igrid[i * 3];
    double tuv000 = 0, tuv100 = 0, tuv010 = 0, tuv001 = 0, tuv200 = 0, tuv020 = 0, tuv002 = 0, tuv110 = 0,
           tuv101 = 0, tuv011 = 0, tuv300 = 0, tuv030 = 0, tuv003 = 0, tuv210 = 0, tuv201 = 0, tuv120 = 0,
           tuv021 = 0, tuv102 = 0, tuv012 = 0, tuv111 = 0;
    for (int it3 = 1; it3 <= bs; ++it3) {
      int k = gather_index(ig[2], it3, s.nfft3);
      double v0 = th3[(it3 - 1) * 4 + 0], v1 = th3[(it3 - 1) * 4 + 1], v2 = th3[(it3 - 1) * 4 + 2],
             v3 = th3[(it3 - 1) * 4 + 3];
      double tu00 = 0, tu10 = 0, tu01 = 0, tu20 = 0, tu11 = 0, tu02 = 0, tu30 = 0, tu21 = 0, tu12 = 0, tu03 = 0;
      for (int it2 = 1; it2 <= bs; ++it2) {
        int j = gather_index(ig[1], it2, s.nfft2);
        double u0 = th2[(it2 - 1) * 4 + 0], u1 = th2[(it2 - 1) * 4 + 1], u2 = th2[(it2 - 1) * 4 + 2],
               u3 = th2[(it2 - 1) * 4 + 3];
        double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
        for (int it1 = 1; it1 <= bs; ++it1) {
          int ii = gather_index(ig[0], it1, s.nfft1);
          double tq = c->grid[((size_t)k * s.nfft2 + j) * s.nfft1 + ii].real();
          t0 = t0 + tq * th1[(it1 - 1) * 4 + 0];
          t1 = t1 + tq * th1[(it1 - 1) * 4 + 1];
          t2 = t2 + tq * th1[(it1 - 1) * 4 + 2];
          t3 = t3 + tq * th1[(it1 - 1) * 4 + 3];
        }
        tu00 = tu00 + t0 * u0;
        tu10 = tu10 + t1 * u0;
        tu01 = tu01 + t0 * u1;
        tu20 = tu20 + t2 * u0;
        tu11 = tu11 + t1 * u1;
        tu02 = tu02 + t0 * u2;
        tu30 = tu30 + t3 * u0;
        tu21 = tu21 + t2 * u1;
        tu12 = tu12 + t1 * u2;
        tu03 = tu03 + t0 * u3;
      }
      tuv000 = tuv000 + tu00 * v0;
      tuv100 = tuv100 + tu10 * v0;
      tuv010 = tuv010 + tu01 * v0;
      tuv001 = tuv001 + tu00 * v1;
      tuv200 = tuv200 + tu20 * v0;
      tuv020 = tuv020 + tu02 * v0;
      tuv002 = tuv002 + tu00 * v2;
      tuv110 = tuv110 + tu11 * v0;
      tuv101 = tuv101 + tu10 * v1;
      tuv011 = tuv011 + tu01 * v1;
      tuv300 = tuv300 + tu30 * v0;
      tuv030 = tuv030 + tu03 * v0;
      tuv003 = tuv003 + tu00 * v3;
      tuv210 = tuv210 + tu21 * v0;
      tuv201 = tuv201 + tu20 * v1;
      tuv120 = tuv120 + tu12 * v0;
      tuv021 = tuv021 + tu02 * v1;
      tuv102 = tuv102 + tu10 * v2;
      tuv012 = tuv012 + tu01 * v2;
      tuv111 = tuv111 + tu11 * v1;
    }
    double* f = &c->fphirec[(size_t)i * 20];
    f[0] = tuv000; f[1] = tuv100; f[2] = tuv010; f[3] = tuv001; f[4] = tuv200;
    f[5] = tuv020; f[6] = tuv002; f[7] = tuv110; f[8] = tuv101; f[9] = tuv011;
    f[10] = tuv300; f[11] = tuv030; f[12] = tuv003; f[13] = tuv210; f[14] = tuv201;
    f[15] = tuv120; f[16] = tuv021; f[17] = tuv102; f[18] = tuv012; f[19] = tuv111;
  }
}

// scale-factor workspace, reset after each i exactly as the reference does
struct ScaleWs {
  std::vector<double> d, p, u;
  void init(int n) {
    d.assign(n, 1.0);
    p.assign(n, 1.0);
    u.assign(n, 1.0);
  }
};

inline bool in_list(const OrSystem& s, int slot, int i, int k) {
  if (!s.conn_off[slot]) return false;
  for (int q = s.conn_off[slot][i]; q < s.conn_off[slot][i + 1]; ++q)
    if (s.conn_idx[slot][q] == k) return true;
  return false;
}

template <class F>
inline void for_conn(const OrSystem& s, int slot, int i, F&& f) {
  if (!s.conn_off[slot]) return;
  for (int q = s.conn_off[slot][i]; q < s.conn_off[slot][i + 1]; ++q) f(s.conn_idx[slot][q]);
}

// newinduce_pme.f:1062-1136 (dpequal false branch)
void set_dp_scales(const OrSystem& s, int i, ScaleWs& w) {
  const int islot[4] = {OR_I12, OR_I13, OR_I14, OR_I15};
  for (int b = 0; b < 4; ++b)
    for_conn(s, islot[b], i, [&](int k) {
      w.p[k] = s.p_scale[b];
      if (in_list(s, OR_IP11, i, k)) w.p[k] = s.pi_scale[b];
    });
  const int pslot[4] = {OR_IP11, OR_IP12, OR_IP13, OR_IP14};
  for (int b = 0; b < 4; ++b) for_conn(s, pslot[b], i, [&](int k) { w.d[k] = s.d_scale[b]; });
}
void reset_dp_scales(const OrSystem& s, int i, ScaleWs& w) {
  const int islot[4] = {OR_I12, OR_I13, OR_I14, OR_I15};
  for (int b = 0; b < 4; ++b) for_conn(s, islot[b], i, [&](int k) { w.p[k] = 1.0; });
  const int pslot[4] = {OR_IP11, OR_IP12, OR_IP13, OR_IP14};
  for (int b = 0; b < 4; ++b) for_conn(s, pslot[b], i, [&](int k) { w.d[k] = 1.0; });
}
// newinduce_pme.f:1495-1518 (uscale part)
void set_u_scales(const OrSystem& s, int i, ScaleWs& w, bool reset) {
  const int pslot[4] = {OR_IP11, OR_IP12, OR_IP13, OR_IP14};
  for (int b = 0; b < 4; ++b) for_conn(s, pslot[b], i, [&](int k) { w.u[k] = reset ? 1.0 : s.u_scale[b]; });
}
// epolar.f:300-330 (pscale only)
void set_p_scales(const OrSystem& s, int i, ScaleWs& w, bool reset) {
  const int islot[4] = {OR_I12, OR_I13, OR_I14, OR_I15};
  for (int b = 0; b < 4; ++b)
    for_conn(s, islot[b], i, [&](int k) {
      if (reset) {
        w.p[k] = 1.0;
      } else {
        w.p[k] = s.p_scale[b];
        if (in_list(s, OR_IP11, i, k)) w.p[k] = s.pi_scale[b];
      }
    });
}

// Per-thread accumulation for Newton's-3rd-law pair loops over the half list.
template <class F>
void pair_loop(OrCtx* c, int ncomp, double* out, F&& body) {
  const OrSystem& s = c->s;
  int n = s.n, nthr = nthreads_of(&s);
  std::vector<std::vector<double>> acc(nthr);
#pragma omp parallel num_threads(nthr)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    acc[tid].assign((size_t)n * ncomp, 0.0);
    ScaleWs w;
    w.init(n);
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) body(i, w, acc[tid].data());
  }
  for (int t = 0; t < nthr; ++t)
    for (size_t q = 0; q < (size_t)n * ncomp; ++q) out[q] += acc[t][q];
}

}  // namespace

// ===========================================================================
extern "C" {

double or_erfc(double x) { return erfc_cody(x); }

// kewald.f:575-620 (ewaldcof)
double or_ewaldcof(double cutoff) {
  double eps = 1.0e-8;
  double ratio = eps + 1.0, x = 0.5;
  int i = 0;
  while (ratio >= eps) {
    i++;
    x = 2.0 * x;
    ratio = erfc_cody(x * cutoff) / cutoff;
  }
  int k = i + 60;
  double xlo = 0.0, xhi = x;
  for (int it = 1; it <= k; ++it) {
    x = (xlo + xhi) / 2.0;
    ratio = erfc_cody(x * cutoff) / cutoff;
    if (ratio >= eps)
      xlo = x;
    else
      xhi = x;
  }
  return x;
}

void or_fft3d(double* data, int n1, int n2, int n3, int sign) {
  fft3d_impl(reinterpret_cast<cd*>(data), n1, n2, n3, sign, 1);
}

OrCtx* or_create(const OrSystem* sys) {
  OrCtx* c = new OrCtx();
  c->s = *sys;
  setup_box(c);
  setup_pme(c);
  return c;
}

void or_destroy(OrCtx* c) { delete c; }

// nblist.f:117-247 (mlistcell) with build_cell_list (nblist.f:607-866) at nproc=1
int or_mlistcell(OrCtx* c, int maxelst, int* nelst, int* elst) {
  const OrSystem& s = c->s;
  int n = s.n;
  double mbuf2 = (s.ewaldcut + s.lbuffer) * (s.ewaldcut + s.lbuffer);
  double vbuf2 = (s.vdwcut + s.lbuffer) * (s.vdwcut + s.lbuffer);
  double boxedge2 = std::min(c->cell.xcell2, std::min(c->cell.ycell2, c->cell.zcell2));
  if (mbuf2 > boxedge2 * boxedge2) return OR_E_BOX_TOO_SMALL;
  // build_cell_list
  double eps1 = 1.0e-10, eps2 = 1.0e-8;
  double mbuf = std::sqrt(mbuf2);
  double vbuf = std::sqrt(vbuf2) + 2.0;
  double bigbuf = ((mbuf + s.lbuffer) > vbuf) ? (mbuf + s.lbuffer) / 3 : vbuf / 3;
  double xmin = -c->cell.xcell2, xmax = c->cell.xcell2;
  double ymin = -c->cell.ycell2, ymax = c->cell.ycell2;
  double zmin = -c->cell.zcell2, zmax = c->cell.zcell2;
  double lenx = std::fabs(xmax - xmin), leny = std::fabs(ymax - ymin), lenz = std::fabs(zmax - zmin);
  int nx = std::max(1, (int)(lenx / bigbuf)), ny = std::max(1, (int)(leny / bigbuf)),
      nz = std::max(1, (int)(lenz / bigbuf));
  double lxc = lenx / nx, lyc = leny / ny, lzc = lenz / nz;
  std::vector<double> xb(nx), xe(nx), yb(ny), ye(ny), zb(nz), ze(nz);
  for (int i = 0; i < nx; ++i) { xb[i] = xmin + i * lxc; xe[i] = xmin + (i + 1) * lxc; }
  for (int i = 0; i < ny; ++i) { yb[i] = ymin + i * lyc; ye[i] = ymin + (i + 1) * lyc; }
  for (int i = 0; i < nz; ++i) { zb[i] = zmin + i * lzc; ze[i] = zmin + (i + 1) * lzc; }
  int ncell = nx * ny * nz;
  // neighbor cells: p (x) outer, q (y), r (z) inner, first occurrence kept
  std::vector<std::vector<int>> neig(ncell);
  std::vector<int> filled(ncell);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int icell = (k * ny + j) * nx + i;
        std::fill(filled.begin(), filled.end(), 0);
        filled[icell] = 1;
        for (int p = -3; p <= 3; ++p)
          for (int q = -3; q <= 3; ++q)
            for (int r = -3; r <= 3; ++r) {
              if (p == 0 && q == 0 && r == 0) continue;
              int tx = ((i + p) % nx + nx) % nx, ty = ((j + q) % ny + ny) % ny, tz = ((k + r) % nz + nz) % nz;
              int t = (tz * ny + ty) * nx + tx;
              if (filled[t]) continue;
              filled[t] = 1;
              neig[icell].push_back(t);
            }
      }
  auto find_cell = [](double v, const std::vector<double>& b, const std::vector<double>& e) {
    int nc = (int)b.size();
    for (int q = 0; q < nc; ++q)
      if (v >= b[q] && v < e[q]) return q;
    return -1;
  };
  std::vector<int> repart(n), cell_len(ncell, 0);
  std::vector<std::vector<int>> cell_atoms(ncell);
  for (int i = 0; i < n; ++i) {
    double xr = s.x[i], yr = s.y[i], zr = s.z[i];
    image(c->cell, xr, yr, zr);
    if (std::fabs(xr - xmax) < eps1) xr = xr - eps2;
    if (std::fabs(yr - ymax) < eps1) yr = yr - eps2;
    if (std::fabs(zr - zmax) < eps1) zr = zr - eps2;
    int ci = find_cell(xr, xb, xe), cj = find_cell(yr, yb, ye), ck = find_cell(zr, zb, ze);
    if (ci < 0 || cj < 0 || ck < 0) return OR_E_BOX_TOO_SMALL;  // not reachable for imaged inputs
    int icell = (ck * ny + cj) * nx + ci;
    repart[i] = icell;
    cell_atoms[icell].push_back(i);
  }
  // mlistcell
  int status = OR_OK;
  for (int i = 0; i < n; ++i) {
    int icell = repart[i];
    double xi = s.x[i], yi = s.y[i], zi = s.z[i];
    int j = 0;
    auto visit = [&](int k) {
      if (k <= i) return;
      double px = xi - s.x[k], py = yi - s.y[k], pz = zi - s.z[k];
      image(c->cell, px, py, pz);  // midpointimage (domdecstuff.f:1773) always accepts at nproc=1
      double r2 = px * px + py * py + pz * pz;
      if (r2 <= mbuf2) {
        if (j < maxelst) elst[(size_t)i * maxelst + j] = k;
        j++;
      }
    };
    for (int k : cell_atoms[icell]) visit(k);
    for (int kc : neig[icell])
      for (int k : cell_atoms[kc]) visit(k);
    nelst[i] = std::min(j, maxelst);
    if (j >= maxelst) status = OR_E_LIST_OVERFLOW;
  }
  c->maxelst = maxelst;
  c->nelst.assign(nelst, nelst + n);
  c->elst.assign(elst, elst + (size_t)n * maxelst);
  c->have_list = (status == OR_OK);
  return status;
}

// newinduce_pme.f:948-1389 (efld0_direct), Thole branch
void or_efld0_direct(OrCtx* c, double* ef) {
  const OrSystem& s = c->s;
  const double cutoff2 = s.ewaldcut * s.ewaldcut;
  const int maxelst = c->maxelst;
  pair_loop(c, 6, ef, [&](int i, ScaleWs& w, double* acc) {
    const double* ri = &s.rpole[(size_t)i * 13];
    double ci = ri[0], dix = ri[1], diy = ri[2], diz = ri[3];
    double qixx = ri[4], qixy = ri[5], qixz = ri[6], qiyy = ri[8], qiyz = ri[9], qizz = ri[12];
    set_dp_scales(s, i, w);
    for (int kkk = 0; kkk < c->nelst[i]; ++kkk) {
      int k = c->elst[(size_t)i * maxelst + kkk];
      double xr = s.x[k] - s.x[i], yr = s.y[k] - s.y[i], zr = s.z[k] - s.z[i];
      image(c->cell, xr, yr, zr);
      double r2 = xr * xr + yr * yr + zr * zr;
      if (r2 > cutoff2) continue;
      double r = std::sqrt(r2);
      double rr1 = 1.0 / r, rr2 = rr1 * rr1, rr3 = rr2 * rr1;
      double rr5 = 3.0 * rr2 * rr3, rr7 = 5.0 * rr2 * rr5;
      const double* rk = &s.rpole[(size_t)k * 13];
      double ck = rk[0], dkx = rk[1], dky = rk[2], dkz = rk[3];
      double qkxx = rk[4], qkxy = rk[5], qkxz = rk[6], qkyy = rk[8], qkyz = rk[9], qkzz = rk[12];
      double dir = dix * xr + diy * yr + diz * zr;
      double qix = qixx * xr + qixy * yr + qixz * zr;
      double qiy = qixy * xr + qiyy * yr + qiyz * zr;
      double qiz = qixz * xr + qiyz * yr + qizz * zr;
      double qir = qix * xr + qiy * yr + qiz * zr;
      double dkr = dkx * xr + dky * yr + dkz * zr;
      double qkx = qkxx * xr + qkxy * yr + qkxz * zr;
      double qky = qkxy * xr + qkyy * yr + qkyz * zr;
      double qkz = qkxz * xr + qkyz * yr + qkzz * zr;
      double qkr = qkx * xr + qky * yr + qkz * zr;
      double dmpe[8], dmpik[8];
      dampewald(7, r, r2, 1.0, s.aewald, dmpe);
      dampthole(s.pdamp[i], s.pdamp[k], s.thole[i], s.thole[k], 7, r, dmpik);
      double fid[3], fkd[3], fip[3], fkp[3];
      double scalek = w.d[k];
      double dmp3 = dmpe[3] - (1.0 - scalek * dmpik[3]) * rr3;
      double dmp5 = dmpe[5] - (1.0 - scalek * dmpik[5]) * rr5;
      double dmp7 = dmpe[7] - (1.0 - scalek * dmpik[7]) * rr7;
      fid[0] = -xr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dkx + 2.0 * dmp5 * qkx;
      fid[1] = -yr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dky + 2.0 * dmp5 * qky;
      fid[2] = -zr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dkz + 2.0 * dmp5 * qkz;
      fkd[0] = xr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * dix - 2.0 * dmp5 * qix;
      fkd[1] = yr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * diy - 2.0 * dmp5 * qiy;
      fkd[2] = zr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * diz - 2.0 * dmp5 * qiz;
      scalek = w.p[k];
      dmp3 = dmpe[3] - (1.0 - scalek * dmpik[3]) * rr3;
      dmp5 = dmpe[5] - (1.0 - scalek * dmpik[5]) * rr5;
      dmp7 = dmpe[7] - (1.0 - scalek * dmpik[7]) * rr7;
      fip[0] = -xr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dkx + 2.0 * dmp5 * qkx;
      fip[1] = -yr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dky + 2.0 * dmp5 * qky;
      fip[2] = -zr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dkz + 2.0 * dmp5 * qkz;
      fkp[0] = xr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * dix - 2.0 * dmp5 * qix;
      fkp[1] = yr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * diy - 2.0 * dmp5 * qiy;
      fkp[2] = zr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * diz - 2.0 * dmp5 * qiz;
      for (int j = 0; j < 3; ++j) {
        acc[(size_t)i * 6 + j] += fid[j];
        acc[(size_t)k * 6 + j] += fkd[j];
        acc[(size_t)i * 6 + 3 + j] += fip[j];
        acc[(size_t)k * 6 + 3 + j] += fkp[j];
      }
    }
    reset_dp_scales(s, i, w);
  });
}

// newinduce_pme.f:1392-1668 (tmatxb_pme), Thole branch
void or_tmatxb_pme(OrCtx* c, int nrhs, int dodiag, const double* mu, double* efi) {
  const OrSystem& s = c->s;
  const int n = s.n, maxelst = c->maxelst;
  const double off2 = s.ewaldcut * s.ewaldcut;
  std::fill(efi, efi + (size_t)n * 3 * nrhs, 0.0);
  pair_loop(c, 3 * nrhs, efi, [&](int i, ScaleWs& w, double* acc) {
    set_u_scales(s, i, w, false);
    for (int kkk = 0; kkk < c->nelst[i]; ++kkk) {
      int k = c->elst[(size_t)i * maxelst + kkk];
      double xr = s.x[k] - s.x[i], yr = s.y[k] - s.y[i], zr = s.z[k] - s.z[i];
      image(c->cell, xr, yr, zr);
      double r2 = xr * xr + yr * yr + zr * zr;
      if (r2 > off2) continue;
      double r = std::sqrt(r2);
      double rr1 = 1.0 / r, rr2 = rr1 * rr1, rr3 = rr2 * rr1, rr5 = 3.0 * rr2 * rr3;
      double dmpe[8], dmpik[8];
      dampewald(7, r, r2, 1.0, s.aewald, dmpe);
      dampthole(s.pdamp[i], s.pdamp[k], s.thole[i], s.thole[k], 5, r, dmpik);
      double scalek = w.u[k];
      double dmp3 = dmpe[3] - (1.0 - scalek * dmpik[3]) * rr3;
      double dmp5 = dmpe[5] - (1.0 - scalek * dmpik[5]) * rr5;
      double d1 = -dmp3 + dmp5 * xr * xr, d2 = dmp5 * xr * yr, d3 = dmp5 * xr * zr;
      double d4 = -dmp3 + dmp5 * yr * yr, d5 = dmp5 * yr * zr, d6 = -dmp3 + dmp5 * zr * zr;
      for (int rh = 0; rh < nrhs; ++rh) {
        const double* uk = &mu[((size_t)k * nrhs + rh) * 3];
        const double* ui = &mu[((size_t)i * nrhs + rh) * 3];
        double fi0 = d1 * uk[0] + d2 * uk[1] + d3 * uk[2];
        double fi1 = d2 * uk[0] + d4 * uk[1] + d5 * uk[2];
        double fi2 = d3 * uk[0] + d5 * uk[1] + d6 * uk[2];
        double fk0 = d1 * ui[0] + d2 * ui[1] + d3 * ui[2];
        double fk1 = d2 * ui[0] + d4 * ui[1] + d5 * ui[2];
        double fk2 = d3 * ui[0] + d5 * ui[1] + d6 * ui[2];
        double* ai = &acc[((size_t)i * nrhs + rh) * 3];
        double* ak = &acc[((size_t)k * nrhs + rh) * 3];
        ai[0] -= fi0; ai[1] -= fi1; ai[2] -= fi2;
        ak[0] -= fk0; ak[1] -= fk1; ak[2] -= fk2;
      }
    }
    set_u_scales(s, i, w, true);
  });
  if (dodiag) {
    for (int i = 0; i < n; ++i) {
      double pol = (s.polarity[i] == 0.0) ? 1.0 / kTinyPol : 1.0 / s.polarity[i];
      for (int rh = 0; rh < nrhs; ++rh)
        for (int j = 0; j < 3; ++j) efi[((size_t)i * nrhs + rh) * 3 + j] += mu[((size_t)i * nrhs + rh) * 3 + j] * pol;
    }
  }
}

// newinduce_pme.f:1671-1917 (efld0_recip)
void or_efld0_recip(OrCtx* c, double* cphi) {
  const OrSystem& s = c->s;
  int n = s.n;
  bspline_fill(c);
  double ctf[10][10], ftc[10][10];
  cart_to_frac(c, ctf);
  frac_to_cart(c, ftc);
  std::vector<double> fmp((size_t)n * 10);
  for (int i = 0; i < n; ++i) {
    const double* rp = &s.rpole[(size_t)i * 13];
    double cmp[10] = {rp[0], rp[1], rp[2], rp[3], rp[4], rp[8], rp[12], 2.0 * rp[5], 2.0 * rp[6], 2.0 * rp[9]};
    double* f = &fmp[(size_t)i * 10];
    f[0] = ctf[0][0] * cmp[0];
    for (int j = 1; j < 4; ++j) {
      f[j] = 0.0;
      for (int k = 1; k < 4; ++k) f[j] = f[j] + ctf[j][k] * cmp[k];
    }
    for (int j = 4; j < 10; ++j) {
      f[j] = 0.0;
      for (int k = 4; k < 10; ++k) f[j] = f[j] + ctf[j][k] * cmp[k];
    }
  }
  // grid_mpole_site (pmestuff.f:163-278)
  spread_sites(c, [&](int i, const double* t, const double* u, const double* v) {
    const double* f = &fmp[(size_t)i * 10];
    double term0 = f[0] * u[0] * v[0] + f[2] * u[1] * v[0] + f[3] * u[0] * v[1] + f[5] * u[2] * v[0] +
                   f[6] * u[0] * v[2] + f[9] * u[1] * v[1];
    double term1 = f[1] * u[0] * v[0] + f[7] * u[1] * v[0] + f[8] * u[0] * v[1];
    double term2 = f[4] * u[0] * v[0];
    return cd(term0 * t[0] + term1 * t[1] + term2 * t[2], 0.0);
  });
  convolve(c);
  fphi_mpole(c);
  for (int i = 0; i < n; ++i) {
    const double* fp = &c->fphirec[(size_t)i * 20];
    double* cp = &cphi[(size_t)i * 10];
    cp[0] = ftc[0][0] * fp[0];
    for (int j = 1; j < 4; ++j) {
      cp[j] = 0.0;
      for (int k = 1; k < 4; ++k) cp[j] = cp[j] + ftc[j][k] * fp[k];
    }
    for (int j = 4; j < 10; ++j) {
      cp[j] = 0.0;
      for (int k = 4; k < 10; ++k) cp[j] = cp[j] + ftc[j][k] * fp[k];
    }
  }
}

// newinduce_pme.f:1919-2128 (tmatxbrecip) with grid_uind_site (pmestuff.f:280)
// and fphi_uind_site (pmestuff.f:746)
void or_tmatxbrecip(OrCtx* c, int nrhs, const double* mu, double* dipfield) {
  const OrSystem& s = c->s;
  int n = s.n, bs = c->bsorder;
  if (!c->have_bspline) bspline_fill(c);
  double a[3][3];
  int nf[3] = {s.nfft1, s.nfft2, s.nfft3};
  for (int j = 0; j < 3; ++j)
    for (int d = 0; d < 3; ++d) a[d][j] = (double)nf[d] * c->recip[j][d];
  std::vector<double> fu((size_t)n * 6);
  for (int i = 0; i < n; ++i) {
    const double* ud = &mu[((size_t)i * nrhs + 0) * 3];
    const double* up = &mu[((size_t)i * nrhs + (nrhs > 1 ? 1 : 0)) * 3];
    for (int k = 0; k < 3; ++k) {
      fu[i * 6 + k] = a[k][0] * ud[0] + a[k][1] * ud[1] + a[k][2] * ud[2];
      fu[i * 6 + 3 + k] = a[k][0] * up[0] + a[k][1] * up[1] + a[k][2] * up[2];
    }
  }
  spread_sites(c, [&](int i, const double* t, const double* u, const double* v) {
    const double* fd = &fu[i * 6];
    const double* fp = &fu[i * 6 + 3];
    double term01 = fd[1] * u[1] * v[0] + fd[2] * u[0] * v[1];
    double term11 = fd[0] * u[0] * v[0];
    double term02 = fp[1] * u[1] * v[0] + fp[2] * u[0] * v[1];
    double term12 = fp[0] * u[0] * v[0];
    return cd(term01 * t[0] + term11 * t[1], term02 * t[0] + term12 * t[1]);
  });
  convolve(c);
  int nthr = nthreads_of(&s);
#pragma omp parallel for num_threads(nthr) schedule(static)
  for (int i = 0; i < n; ++i) {
    const double* th1 = &c->theta1[(size_t)i * bs * 4];
    const double* th2 = &c->theta2[(size_t)i * bs * 4];
    const double* th3 = &c->theta3[(size_t)i * bs * 4];
    const int* ig = &c->igrid[i * 3];
    double tuv100_1 = 0, tuv010_1 = 0, tuv001_1 = 0, tuv100_2 = 0, tuv010_2 = 0, tuv001_2 = 0;
    for (int it3 = 1; it3 <= bs; ++it3) {
      int k = gather_index(ig[2], it3, s.nfft3);
      double v0 = th3[(it3 - 1) * 4 + 0], v1 = th3[(it3 - 1) * 4 + 1];
      double tu00_1 = 0, tu01_1 = 0, tu10_1 = 0, tu00_2 = 0, tu01_2 = 0, tu10_2 = 0;
      for (int it2 = 1; it2 <= bs; ++it2) {
        int j = gather_index(ig[1], it2, s.nfft2);
        double u0 = th2[(it2 - 1) * 4 + 0], u1 = th2[(it2 - 1) * 4 + 1];
        double t0_1 = 0, t1_1 = 0, t0_2 = 0, t1_2 = 0;
        for (int it1 = 1; it1 <= bs; ++it1) {
          int ii = gather_index(ig[0], it1, s.nfft1);
          cd g = c->grid[((size_t)k * s.nfft2 + j) * s.nfft1 + ii];
          double tq_1 = g.real(), tq_2 = g.imag();
          t0_1 = t0_1 + tq_1 * th1[(it1 - 1) * 4 + 0];
          t1_1 = t1_1 + tq_1 * th1[(it1 - 1) * 4 + 1];
          t0_2 = t0_2 + tq_2 * th1[(it1 - 1) * 4 + 0];
          t1_2 = t1_2 + tq_2 * th1[(it1 - 1) * 4 + 1];
        }
        tu00_1 = tu00_1 + t0_1 * u0;
        tu10_1 = tu10_1 + t1_1 * u0;
        tu01_1 = tu01_1 + t0_1 * u1;
        tu00_2 = tu00_2 + t0_2 * u0;
        tu10_2 = tu10_2 + t1_2 * u0;
        tu01_2 = tu01_2 + t0_2 * u1;
      }
      tuv100_1 = tuv100_1 + tu10_1 * v0;
      tuv010_1 = tuv010_1 + tu01_1 * v0;
      tuv001_1 = tuv001_1 + tu00_1 * v1;
      tuv100_2 = tuv100_2 + tu10_2 * v0;
      tuv010_2 = tuv010_2 + tu01_2 * v0;
      tuv001_2 = tuv001_2 + tu00_2 * v1;
    }
    double p1[3] = {tuv100_1, tuv010_1, tuv001_1}, p2[3] = {tuv100_2, tuv010_2, tuv001_2};
    for (int k = 0; k < 3; ++k) {
      dipfield[((size_t)i * nrhs + 0) * 3 + k] = a[k][0] * p1[0] + a[k][1] * p1[1] + a[k][2] * p1[2];
      if (nrhs > 1) dipfield[((size_t)i * nrhs + 1) * 3 + k] = a[k][0] * p2[0] + a[k][1] * p2[1] + a[k][2] * p2[2];
    }
  }
}

// newinduce_pme2.f:16-283 (newinduce_pme2) + :285-636 (inducepcg_pme2)
int or_newinduce_pme2(OrCtx* c, const double* mu_guess, double* uind, double* uinp, double* ef_out,
                      OrSolveInfo* info) {
  const OrSystem& s = c->s;
  const int n = s.n, nrhs = 2;
  const size_t nv = (size_t)n * nrhs * 3;
  if (!c->have_list) return OR_E_LIST_OVERFLOW;
  std::vector<double> ef(nv, 0.0), mu(nv, 0.0), cphi((size_t)n * 10, 0.0);
  or_efld0_recip(c, cphi.data());
  or_efld0_direct(c, ef.data());
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < 3; ++j) {
      ef[(i * 2 + 0) * 3 + j] = ef[(i * 2 + 0) * 3 + j] - cphi[i * 10 + j + 1];
      ef[(i * 2 + 1) * 3 + j] = ef[(i * 2 + 1) * 3 + j] - cphi[i * 10 + j + 1];
    }
  double term = (4.0 / 3.0) * s.aewald * s.aewald * s.aewald / kSqrtPi;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < 3; ++j) {
      ef[(i * 2 + 0) * 3 + j] = ef[(i * 2 + 0) * 3 + j] + term * s.rpole[(size_t)i * 13 + j + 1];
      ef[(i * 2 + 1) * 3 + j] = ef[(i * 2 + 1) * 3 + j] + term * s.rpole[(size_t)i * 13 + j + 1];
    }
  if (ef_out) std::copy(ef.begin(), ef.end(), ef_out);
  if (mu_guess) {
    std::copy(mu_guess, mu_guess + nv, mu.begin());
  } else {
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < nrhs; ++k)
        for (int j = 0; j < 3; ++j) mu[(i * 2 + k) * 3 + j] = s.polarity[i] * ef[(i * 2 + k) * 3 + j];
  }
  // inducepcg_pme2
  std::vector<double> res(nv, 0.0), h(nv, 0.0), pp(nv, 0.0), zr(nv, 0.0), dipfield(nv, 0.0), diag(n);
  for (int i = 0; i < n; ++i) diag[i] = (s.polarity[i] == 0.0) ? kTinyPol : s.polarity[i];
  double ggold[2] = {0, 0}, ggnew[2], gg[2], alphacg[2], ene[2] = {0, 0}, gnorm[2] = {0, 0};
  or_tmatxbrecip(c, nrhs, mu.data(), dipfield.data());
  or_tmatxb_pme(c, nrhs, 1, mu.data(), h.data());
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < nrhs; ++k)
      for (int j = 0; j < 3; ++j) {
        size_t q = (i * 2 + k) * 3 + j;
        h[q] = h[q] + dipfield[q] - term * mu[q];
        res[q] = ef[q] - h[q];
        zr[q] = diag[i] * res[q];
      }
  pp = zr;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < nrhs; ++k)
      for (int j = 0; j < 3; ++j) ggold[k] = ggold[k] + res[(i * 2 + k) * 3 + j] * zr[(i * 2 + k) * 3 + j];
  int it, converged = 0;
  double resnrm = 0.0;
  for (it = 1; it <= s.politer; ++it) {
    or_tmatxbrecip(c, nrhs, pp.data(), dipfield.data());
    or_tmatxb_pme(c, nrhs, 1, pp.data(), h.data());
    for (size_t q = 0; q < nv; ++q) h[q] = h[q] + dipfield[q] - term * pp[q];
    gg[0] = gg[1] = 0.0;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < nrhs; ++k)
        for (int j = 0; j < 3; ++j) gg[k] = gg[k] + pp[(i * 2 + k) * 3 + j] * h[(i * 2 + k) * 3 + j];
    bool zero = false;
    for (int k = 0; k < nrhs; ++k) {
      if (gg[k] == 0.0) zero = true;
    }
    if (zero) break;  // reference returns (newinduce_pme2.f:505)
    for (int k = 0; k < nrhs; ++k) alphacg[k] = ggold[k] / gg[k];
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < nrhs; ++k)
        for (int j = 0; j < 3; ++j) {
          size_t q = (i * 2 + k) * 3 + j;
          mu[q] = mu[q] + alphacg[k] * pp[q];
          res[q] = res[q] - alphacg[k] * h[q];
        }
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < nrhs; ++k)
        for (int j = 0; j < 3; ++j) zr[(i * 2 + k) * 3 + j] = diag[i] * res[(i * 2 + k) * 3 + j];
    ggnew[0] = ggnew[1] = 0.0;
    ene[0] = ene[1] = 0.0;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < nrhs; ++k)
        for (int j = 0; j < 3; ++j) {
          size_t q = (i * 2 + k) * 3 + j;
          ggnew[k] = ggnew[k] + res[q] * zr[q];
          ene[k] = ene[k] - 0.5 * (mu[q] * (res[q] + ef[q]));
        }
    resnrm = 0.0;
    for (int k = 0; k < nrhs; ++k) {
      gnorm[k] = std::sqrt(ggnew[k] / (double)(3 * n));
      resnrm = std::max(resnrm, gnorm[k]);
    }
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < nrhs; ++k)
        for (int j = 0; j < 3; ++j) {
          size_t q = (i * 2 + k) * 3 + j;
          pp[q] = zr[q] + ggnew[k] / ggold[k] * pp[q];
        }
    ggold[0] = ggnew[0];
    ggold[1] = ggnew[1];
    if (resnrm < s.poleps) {
      converged = 1;
      break;
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < 3; ++j) {
      uind[i * 3 + j] = mu[(i * 2 + 0) * 3 + j];
      uinp[i * 3 + j] = mu[(i * 2 + 1) * 3 + j];
    }
  if (info) {
    info->niter = std::min(it, s.politer);
    info->converged = converged;
    info->resnrm = resnrm;
    info->ene[0] = ene[0] * kElectric;
    info->ene[1] = ene[1] * kElectric;
  }
  return OR_OK;
}

// epolar.f:47-520: epolar0c = eprecip + epreal0c + self (TINFOIL boundary)
double or_epolar(OrCtx* c, const double* uind, double* ereal_out, double* erecip_out, double* eself_out) {
  const OrSystem& s = c->s;
  const int n = s.n, maxelst = c->maxelst;
  const double off2 = s.ewaldcut * s.ewaldcut;
  // eprecip (epolar.f:524-712), needs fphirec from the permanent-field PME pass
  if (c->fphirec.size() != (size_t)n * 20) {
    std::vector<double> cphi((size_t)n * 10);
    or_efld0_recip(c, cphi.data());
  }
  double a[3][3];
  int nf[3] = {s.nfft1, s.nfft2, s.nfft3};
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) a[d][i] = (double)nf[d] * c->recip[i][d];
  double erec = 0.0;
  for (int i = 0; i < n; ++i) {
    double fuind[3];
    for (int j = 0; j < 3; ++j) fuind[j] = a[j][0] * uind[i * 3 + 0] + a[j][1] * uind[i * 3 + 1] + a[j][2] * uind[i * 3 + 2];
    for (int k = 0; k < 3; ++k) erec = erec + fuind[k] * c->fphirec[(size_t)i * 20 + k + 1];
  }
  erec = 0.5 * kElectric * erec;
  // epreal0c (epolar.f:207-520), mode MPOLE -> off = mpolecut = ewaldcut
  const double f = 0.5 * kElectric;
  double ereal_acc = 0.0;
  {
    std::vector<double> e1(1, 0.0);
    int nthr = nthreads_of(&s);
    std::vector<double> part(nthr, 0.0);
#pragma omp parallel num_threads(nthr)
    {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
      ScaleWs w;
      w.init(n);
      double ep = 0.0;
#pragma omp for schedule(dynamic, 64)
      for (int i = 0; i < n; ++i) {
        const double* ri = &s.rpole[(size_t)i * 13];
        double ci = ri[0], dix = ri[1], diy = ri[2], diz = ri[3];
        double qixx = ri[4], qixy = ri[5], qixz = ri[6], qiyy = ri[8], qiyz = ri[9], qizz = ri[12];
        double uix = uind[i * 3], uiy = uind[i * 3 + 1], uiz = uind[i * 3 + 2];
        set_p_scales(s, i, w, false);
        for (int kkk = 0; kkk < c->nelst[i]; ++kkk) {
          int k = c->elst[(size_t)i * maxelst + kkk];
          double xr = s.x[k] - s.x[i], yr = s.y[k] - s.y[i], zr = s.z[k] - s.z[i];
          image(c->cell, xr, yr, zr);
          double r2 = xr * xr + yr * yr + zr * zr;
          if (r2 > off2) continue;
          double r = std::sqrt(r2);
          const double* rk = &s.rpole[(size_t)k * 13];
          double ck = rk[0], dkx = rk[1], dky = rk[2], dkz = rk[3];
          double qkxx = rk[4], qkxy = rk[5], qkxz = rk[6], qkyy = rk[8], qkyz = rk[9], qkzz = rk[12];
          double ukx = uind[k * 3], uky = uind[k * 3 + 1], ukz = uind[k * 3 + 2];
          double dir = dix * xr + diy * yr + diz * zr;
          double qix = qixx * xr + qixy * yr + qixz * zr;
          double qiy = qixy * xr + qiyy * yr + qiyz * zr;
          double qiz = qixz * xr + qiyz * yr + qizz * zr;
          double qir = qix * xr + qiy * yr + qiz * zr;
          double dkr = dkx * xr + dky * yr + dkz * zr;
          double qkx = qkxx * xr + qkxy * yr + qkxz * zr;
          double qky = qkxy * xr + qkyy * yr + qkyz * zr;
          double qkz = qkxz * xr + qkyz * yr + qkzz * zr;
          double qkr = qkx * xr + qky * yr + qkz * zr;
          double diu = dix * ukx + diy * uky + diz * ukz;
          double qiu = qix * ukx + qiy * uky + qiz * ukz;
          double uir = uix * xr + uiy * yr + uiz * zr;
          double dku = dkx * uix + dky * uiy + dkz * uiz;
          double qku = qkx * uix + qky * uiy + qkz * uiz;
          double ukr = ukx * xr + uky * yr + ukz * zr;
          double dmpe[8], dmpik[8];
          dampewald(7, r, r2, f, s.aewald, dmpe);
          dampthole(s.pdamp[i], s.pdamp[k], s.thole[i], s.thole[k], 7, r, dmpik);
          double scalek = w.p[k];
          double rr3 = f / (r * r2);
          double rr5 = 3.0 * rr3 / r2;
          double rr7 = 5.0 * rr5 / r2;
          double sr3 = scalek * dmpik[3] * rr3;
          double sr5 = scalek * dmpik[5] * rr5;
          double sr7 = scalek * dmpik[7] * rr7;
          sr3 = dmpe[3] - rr3 + sr3;
          sr5 = dmpe[5] - rr5 + sr5;
          sr7 = dmpe[7] - rr7 + sr7;
          double term1 = ck * uir - ci * ukr + diu + dku;
          double term2 = 2.0 * (qiu - qku) - uir * dkr - dir * ukr;
          double term3 = uir * qkr - ukr * qir;
          ep += term1 * sr3 + term2 * sr5 + term3 * sr7;
        }
        set_p_scales(s, i, w, true);
      }
      part[tid] = ep;
    }
    for (int t = 0; t < nthr; ++t) ereal_acc += part[t];
  }
  // self term (epolar.f:131-146)
  double term = 2.0 * s.aewald * s.aewald;
  double fterm = -kElectric * s.aewald / kSqrtPi;
  double eself = 0.0;
  for (int i = 0; i < n; ++i) {
    const double* rp = &s.rpole[(size_t)i * 13];
    double uii = rp[1] * uind[i * 3] + rp[2] * uind[i * 3 + 1] + rp[3] * uind[i * 3 + 2];
    eself = eself + fterm * term * uii / 3.0;
  }
  if (ereal_out) *ereal_out = ereal_acc;
  if (erecip_out) *erecip_out = erec;
  if (eself_out) *eself_out = eself;
  return erec + ereal_acc + eself;
}

// rotpole.f:17-339 (rotmat for Z-then-X and Bisector, rotsite)
void or_rotpole(int n, const double* x, const double* y, const double* z, const double* pole, const int* zaxis,
                const int* xaxis, const int* axt, double* rpole) {
  for (int i = 0; i < n; ++i) {
    double a[3][3] = {{1, 0, 0}, {0, 0, 0}, {0, 0, 1}};
    // a[row][col] == reference a(row+1,col+1)
    a[0][0] = 1.0; a[1][0] = 0.0; a[2][0] = 0.0;
    a[0][2] = 0.0; a[1][2] = 0.0; a[2][2] = 1.0;
    double xi = x[i], yi = y[i], zi = z[i];
    int iz = zaxis[i], ix = xaxis[i];
    if (axt[i] == 1) {  // Z-then-X
      double dx = x[iz] - xi, dy = y[iz] - yi, dz = z[iz] - zi;
      double r = std::sqrt(dx * dx + dy * dy + dz * dz);
      a[0][2] = dx / r; a[1][2] = dy / r; a[2][2] = dz / r;
      dx = x[ix] - xi; dy = y[ix] - yi; dz = z[ix] - zi;
      double dot = dx * a[0][2] + dy * a[1][2] + dz * a[2][2];
      dx = dx - dot * a[0][2]; dy = dy - dot * a[1][2]; dz = dz - dot * a[2][2];
      r = std::sqrt(dx * dx + dy * dy + dz * dz);
      a[0][0] = dx / r; a[1][0] = dy / r; a[2][0] = dz / r;
    } else if (axt[i] == 2) {  // Bisector
      double dx = x[iz] - xi, dy = y[iz] - yi, dz = z[iz] - zi;
      double r = std::sqrt(dx * dx + dy * dy + dz * dz);
      double dx1 = dx / r, dy1 = dy / r, dz1 = dz / r;
      dx = x[ix] - xi; dy = y[ix] - yi; dz = z[ix] - zi;
      r = std::sqrt(dx * dx + dy * dy + dz * dz);
      double dx2 = dx / r, dy2 = dy / r, dz2 = dz / r;
      dx = dx1 + dx2; dy = dy1 + dy2; dz = dz1 + dz2;
      r = std::sqrt(dx * dx + dy * dy + dz * dz);
      a[0][2] = dx / r; a[1][2] = dy / r; a[2][2] = dz / r;
      double dot = dx2 * a[0][2] + dy2 * a[1][2] + dz2 * a[2][2];
      dx = dx2 - dot * a[0][2]; dy = dy2 - dot * a[1][2]; dz = dz2 - dot * a[2][2];
      r = std::sqrt(dx * dx + dy * dy + dz * dz);
      a[0][0] = dx / r; a[1][0] = dy / r; a[2][0] = dz / r;
    }
    a[0][1] = a[2][0] * a[1][2] - a[1][0] * a[2][2];
    a[1][1] = a[0][0] * a[2][2] - a[2][0] * a[0][2];
    a[2][1] = a[1][0] * a[0][2] - a[0][0] * a[1][2];
    const double* p = &pole[(size_t)i * 13];
    double* rp = &rpole[(size_t)i * 13];
    rp[0] = p[0];
    for (int ii = 0; ii < 3; ++ii) {
      rp[1 + ii] = 0.0;
      for (int j = 0; j < 3; ++j) rp[1 + ii] = rp[1 + ii] + p[1 + j] * a[ii][j];
    }
    double m2[3][3], r2[3][3];
    int k = 4;
    for (int ii = 0; ii < 3; ++ii)
      for (int j = 0; j < 3; ++j) {
        m2[ii][j] = p[k];
        r2[ii][j] = 0.0;
        k++;
      }
    for (int ii = 0; ii < 3; ++ii)
      for (int j = 0; j < 3; ++j) {
        if (j < ii) {
          r2[ii][j] = r2[j][ii];
        } else {
          for (int kk = 0; kk < 3; ++kk)
            for (int m = 0; m < 3; ++m) r2[ii][j] = r2[ii][j] + a[ii][kk] * a[j][m] * m2[kk][m];
        }
      }
    k = 4;
    for (int ii = 0; ii < 3; ++ii)
      for (int j = 0; j < 3; ++j) rp[k++] = r2[ii][j];
  }
}

}  // extern "C"

// ===========================================================================
// Polarization forces: epolar1c (epolar1.f:57-372) = eprecip1 (:397-1213)
// + epreal1c (:1215-2540, Thole branch, dpequal false) + self energy and
// self torque (:181-206), torques distributed by torque (torque.f:6-390).
// With vir_out, also the internal virial (TINFOIL boundary, no charge flux):
// eprecip1's per-site induced terms (:846-908) and scalar sums over the
// reciprocal lattice ((rpole+uinp) x (rpole+uind) minus the permanent-only
// sum, :534-541, :932-1091), epreal1c's pairwise terms (:2326-2342) and the
// torque's frame-atom terms (:2460-2486).  The reference adds no virial for
// the frame-atom forces of the reciprocal torque (distributed by torque_rec)
// nor of the self torque; vir_frame (may be NULL) receives those separately:
// vir + vir_frame is the strain derivative of the energy.
namespace {

// torque.f:6-390 for Z-then-X and Bisector frames (the water frames);
// frame atoms 0-based; adds the forces of a torque on site i into de[n][3]
void torque_site(const double* x, const double* y, const double* z, int ib, int ia, int ic, int axt,
                 const double trq[3], double* de, double* fz = nullptr, double* fx = nullptr) {
  double u[3] = {x[ia] - x[ib], y[ia] - y[ib], z[ia] - z[ib]};
  double usiz = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  double v[3] = {x[ic] - x[ib], y[ic] - y[ib], z[ic] - z[ib]};
  double vsiz = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double w[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
  double wsiz = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  for (int j = 0; j < 3; ++j) {
    u[j] /= usiz;
    v[j] /= vsiz;
    w[j] /= wsiz;
  }
  double uv[3] = {v[1] * u[2] - v[2] * u[1], v[2] * u[0] - v[0] * u[2], v[0] * u[1] - v[1] * u[0]};
  double uw[3] = {w[1] * u[2] - w[2] * u[1], w[2] * u[0] - w[0] * u[2], w[0] * u[1] - w[1] * u[0]};
  double vw[3] = {w[1] * v[2] - w[2] * v[1], w[2] * v[0] - w[0] * v[2], w[0] * v[1] - w[1] * v[0]};
  double uvsiz = std::sqrt(uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2]);
  double uwsiz = std::sqrt(uw[0] * uw[0] + uw[1] * uw[1] + uw[2] * uw[2]);
  double vwsiz = std::sqrt(vw[0] * vw[0] + vw[1] * vw[1] + vw[2] * vw[2]);
  for (int j = 0; j < 3; ++j) {
    uv[j] /= uvsiz;
    uw[j] /= uwsiz;
    vw[j] /= vwsiz;
  }
  double uvcos = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
  double uvsin = std::sqrt(1.0 - uvcos * uvcos);
  double dphidu = -trq[0] * u[0] - trq[1] * u[1] - trq[2] * u[2];
  double dphidv = -trq[0] * v[0] - trq[1] * v[1] - trq[2] * v[2];
  double dphidw = -trq[0] * w[0] - trq[1] * w[1] - trq[2] * w[2];
  for (int j = 0; j < 3; ++j) {
    double du, dv;
    if (axt == 1) {  // Z-then-X
      du = uv[j] * dphidv / (usiz * uvsin) + uw[j] * dphidw / usiz;
      dv = -uv[j] * dphidu / (vsiz * uvsin);
    } else {  // Bisector
      du = uv[j] * dphidv / (usiz * uvsin) + 0.5 * uw[j] * dphidw / usiz;
      dv = -uv[j] * dphidu / (vsiz * uvsin) + 0.5 * vw[j] * dphidw / vsiz;
    }
    de[ia * 3 + j] += du;
    de[ic * 3 + j] += dv;
    de[ib * 3 + j] -= du + dv;
    if (fz) fz[j] = du;  // frcz of torque.f: on the z-axis atom
    if (fx) fx[j] = dv;  // frcx: on the x-axis atom
  }
}

// the virial tensor, symmetric, in the accumulation order of the reference
struct Vir {
  double xx = 0, xy = 0, xz = 0, yy = 0, yz = 0, zz = 0;
  void add(double a, double b, double c, double d, double e, double f) {
    xx += a; xy += b; xz += c; yy += d; yz += e; zz += f;
  }
  // the k-space scalar-sum terms: h h vterm - eterm (emrecip1 / eprecip1)
  void add_k(double h1, double h2, double h3, double vterm, double eterm, double sign) {
    add(sign * (h1 * h1 * vterm - eterm), sign * h1 * h2 * vterm, sign * h1 * h3 * vterm,
        sign * (h2 * h2 * vterm - eterm), sign * h2 * h3 * vterm, sign * (h3 * h3 * vterm - eterm));
  }
  void out(double* v) const {
    v[0] = xx; v[1] = xy; v[2] = xz; v[3] = xy; v[4] = yy; v[5] = yz; v[6] = xz; v[7] = yz; v[8] = zz;
  }
};

// Sum over the reciprocal lattice (all k but 0, where qfac > 0) of the PME
// virial terms of a structure factor product struc2(k): eterm =
// 0.5 f qfac struc2, vterm = (2/h^2)(1 + pterm h^2) eterm (eprecip1,
// epolar1.f:1041-1091; emrecip1 for the permanent-only sum).
template <class S2>
void kspace_virial(const OrCtx* c, double f, double sign, S2&& struc2, Vir& v) {
  const OrSystem& s = c->s;
  const double pterm = (kPi / s.aewald) * (kPi / s.aewald);
  const int nf1 = (s.nfft1 + 1) / 2, nf2 = (s.nfft2 + 1) / 2, nf3 = (s.nfft3 + 1) / 2;
  for (int k3 = 0; k3 < s.nfft3; ++k3)
    for (int k2 = 0; k2 < s.nfft2; ++k2)
      for (int k1 = 0; k1 < s.nfft1; ++k1) {
        const size_t idx = ((size_t)k3 * s.nfft2 + k2) * s.nfft1 + k1;
        const double qf = c->qfac[idx];
        if (qf == 0.0) continue;
        int m1 = k1, m2 = k2, m3 = k3;
        if (k1 + 1 > nf1) m1 -= s.nfft1;
        if (k2 + 1 > nf2) m2 -= s.nfft2;
        if (k3 + 1 > nf3) m3 -= s.nfft3;
        const double h1 = c->recip[0][0] * m1 + c->recip[0][1] * m2 + c->recip[0][2] * m3;
        const double h2 = c->recip[1][0] * m1 + c->recip[1][1] * m2 + c->recip[1][2] * m3;
        const double h3 = c->recip[2][0] * m1 + c->recip[2][1] * m2 + c->recip[2][2] * m3;
        const double hsq = h1 * h1 + h2 * h2 + h3 * h3;
        const double eterm = 0.5 * f * qf * struc2(k1, k2, k3, idx);
        const double vterm = (2.0 / hsq) * (1.0 + pterm * hsq) * eterm;
        v.add_k(h1, h2, h3, vterm, eterm, sign);
      }
}

// The virial of a torque's frame-atom forces (epolar1.f:2460-2486): fz on
// the z-axis atom, fx on the x-axis atom (water frames have no y-axis atom).
void frame_virial(const double* x, const double* y, const double* z, int i, int iz, int ix, const double fz[3],
                  const double fx[3], Vir& v) {
  const double xiz = x[iz] - x[i], yiz = y[iz] - y[i], ziz = z[iz] - z[i];
  const double xix = x[ix] - x[i], yix = y[ix] - y[i], zix = z[ix] - z[i];
  v.add(xix * fx[0] + xiz * fz[0], 0.5 * (yix * fx[0] + yiz * fz[0] + xix * fx[1] + xiz * fz[1]),
        0.5 * (zix * fx[0] + ziz * fz[0] + xix * fx[2] + xiz * fz[2]), yix * fx[1] + yiz * fz[1],
        0.5 * (zix * fx[1] + ziz * fz[1] + yix * fx[2] + yiz * fz[2]), zix * fx[2] + ziz * fz[2]);
}

// fmp (fractional multipoles) of cmp with the dipole replaced by dip + add3
void frac_moments(const double ctf[10][10], const double cm[10], const double* add3, double fm[10]) {
  double c2[10];
  for (int q = 0; q < 10; ++q) c2[q] = cm[q];
  if (add3)
    for (int q = 0; q < 3; ++q) c2[1 + q] += add3[q];
  fm[0] = ctf[0][0] * c2[0];
  for (int j = 1; j < 4; ++j) {
    fm[j] = 0.0;
    for (int k = 1; k < 4; ++k) fm[j] += ctf[j][k] * c2[k];
  }
  for (int j = 4; j < 10; ++j) {
    fm[j] = 0.0;
    for (int k = 4; k < 10; ++k) fm[j] += ctf[j][k] * c2[k];
  }
}

// grid_mpole_site (pmestuff.f:163-278) terms of one site's fmp
inline double mpole_stencil(const double* f, const double* t, const double* u, const double* v) {
  double term0 = f[0] * u[0] * v[0] + f[2] * u[1] * v[0] + f[3] * u[0] * v[1] + f[5] * u[2] * v[0] +
                 f[6] * u[0] * v[2] + f[9] * u[1] * v[1];
  double term1 = f[1] * u[0] * v[0] + f[7] * u[1] * v[0] + f[8] * u[0] * v[1];
  double term2 = f[4] * u[0] * v[0];
  return term0 * t[0] + term1 * t[1] + term2 * t[2];
}

}  // namespace

namespace {

void fphi_dip_site(const OrCtx* c, int i, const cd* g, double phi1[10], double phi2[10], double sum[20]) {
  const OrSystem& s = c->s;
  const int bs = c->bsorder;
  const double* th1 = &c->theta1[(size_t)i * bs * 4];
  const double* th2 = &c->theta2[(size_t)i * bs * 4];
  const double* th3 = &c->theta3[(size_t)i * bs * 4];
  const int* ig = &c->igrid[i * 3];
  double* T1 = phi1;
  double* T2 = phi2;
  double* S = sum;
  for (int q = 0; q < 10; ++q) T1[q] = T2[q] = 0.0;
  for (int q = 0; q < 20; ++q) S[q] = 0.0;
  for (int it3 = 1; it3 <= bs; ++it3) {
    int k = gather_index(ig[2], it3, s.nfft3);
    double v0 = th3[(it3 - 1) * 4], v1 = th3[(it3 - 1) * 4 + 1], v2 = th3[(it3 - 1) * 4 + 2],
           v3 = th3[(it3 - 1) * 4 + 3];
    double tu1[6] = {0}, tu2[6] = {0}, tu[10] = {0};  // 00,10,01,20,11,02 ; sum: +30,21,12,03
    for (int it2 = 1; it2 <= bs; ++it2) {
      int j = gather_index(ig[1], it2, s.nfft2);
      double u0 = th2[(it2 - 1) * 4], u1 = th2[(it2 - 1) * 4 + 1], u2 = th2[(it2 - 1) * 4 + 2],
             u3 = th2[(it2 - 1) * 4 + 3];
      double t1a[3] = {0}, t1b[3] = {0}, t3 = 0.0;
      for (int it1 = 1; it1 <= bs; ++it1) {
        int ii = gather_index(ig[0], it1, s.nfft1);
        cd q = g[((size_t)k * s.nfft2 + j) * s.nfft1 + ii];
        const double* w = &th1[(it1 - 1) * 4];
        t1a[0] += q.real() * w[0];
        t1a[1] += q.real() * w[1];
        t1a[2] += q.real() * w[2];
        t1b[0] += q.imag() * w[0];
        t1b[1] += q.imag() * w[1];
        t1b[2] += q.imag() * w[2];
        t3 += (q.real() + q.imag()) * w[3];
      }
      tu1[0] += t1a[0] * u0; tu1[1] += t1a[1] * u0; tu1[2] += t1a[0] * u1;
      tu1[3] += t1a[2] * u0; tu1[4] += t1a[1] * u1; tu1[5] += t1a[0] * u2;
      tu2[0] += t1b[0] * u0; tu2[1] += t1b[1] * u0; tu2[2] += t1b[0] * u1;
      tu2[3] += t1b[2] * u0; tu2[4] += t1b[1] * u1; tu2[5] += t1b[0] * u2;
      double t0 = t1a[0] + t1b[0], t1 = t1a[1] + t1b[1], t2 = t1a[2] + t1b[2];
      tu[0] += t0 * u0; tu[1] += t1 * u0; tu[2] += t0 * u1; tu[3] += t2 * u0; tu[4] += t1 * u1;
      tu[5] += t0 * u2; tu[6] += t3 * u0; tu[7] += t2 * u1; tu[8] += t1 * u2; tu[9] += t0 * u3;
    }
    // (_1): 100,010,001,200,020,002,110,101,011
    T1[1] += tu1[1] * v0; T1[2] += tu1[2] * v0; T1[3] += tu1[0] * v1; T1[4] += tu1[3] * v0;
    T1[5] += tu1[5] * v0; T1[6] += tu1[0] * v2; T1[7] += tu1[4] * v0; T1[8] += tu1[1] * v1;
    T1[9] += tu1[2] * v1;
    T2[1] += tu2[1] * v0; T2[2] += tu2[2] * v0; T2[3] += tu2[0] * v1; T2[4] += tu2[3] * v0;
    T2[5] += tu2[5] * v0; T2[6] += tu2[0] * v2; T2[7] += tu2[4] * v0; T2[8] += tu2[1] * v1;
    T2[9] += tu2[2] * v1;
    // sum: 000,100,010,001,200,020,002,110,101,011,300,030,003,210,201,120,021,102,012,111
    S[0] += tu[0] * v0; S[1] += tu[1] * v0; S[2] += tu[2] * v0; S[3] += tu[0] * v1;
    S[4] += tu[3] * v0; S[5] += tu[5] * v0; S[6] += tu[0] * v2; S[7] += tu[4] * v0;
    S[8] += tu[1] * v1; S[9] += tu[2] * v1; S[10] += tu[6] * v0; S[11] += tu[9] * v0;
    S[12] += tu[0] * v3; S[13] += tu[7] * v0; S[14] += tu[3] * v1; S[15] += tu[8] * v0;
    S[16] += tu[5] * v1; S[17] += tu[1] * v2; S[18] += tu[2] * v2; S[19] += tu[4] * v1;
  }
}

}  // namespace

extern "C" {

int or_grid_uind_sites(OrCtx* c, int nsites, const int* isite, const double* fuind, const double* fuinp,
                       double* grid) {
  const OrSystem& s = c->s;
  const int bs = c->bsorder;
  if (!c->have_bspline) bspline_fill(c);
  cd* g = reinterpret_cast<cd*>(grid);
  // grid_uind_site (pmestuff.f:280-405), one rank: every stencil point is local
  for (int q = 0; q < nsites; ++q) {
    const int i = isite[q];
    if (i < 0 || i >= s.n) return 1;
    const double* fd = fuind + 3 * (size_t)q;
    const double* fp = fuinp + 3 * (size_t)q;
    const double* t1 = &c->theta1[(size_t)i * bs * 4];
    const double* t2 = &c->theta2[(size_t)i * bs * 4];
    const double* t3 = &c->theta3[(size_t)i * bs * 4];
    const int* ig = &c->igrid[i * 3];
    for (int it3 = 0; it3 < bs; ++it3) {
      int k = stencil_index(c, ig[2], it3, s.nfft3);
      double v0 = t3[it3 * 4], v1 = t3[it3 * 4 + 1];
      for (int it2 = 0; it2 < bs; ++it2) {
        int j = stencil_index(c, ig[1], it2, s.nfft2);
        double u0 = t2[it2 * 4], u1 = t2[it2 * 4 + 1];
        double term01 = fd[1] * u1 * v0 + fd[2] * u0 * v1;
        double term11 = fd[0] * u0 * v0;
        double term02 = fp[1] * u1 * v0 + fp[2] * u0 * v1;
        double term12 = fp[0] * u0 * v0;
        for (int it1 = 0; it1 < bs; ++it1) {
          int ii = stencil_index(c, ig[0], it1, s.nfft1);
          double tt0 = t1[it1 * 4], tt1 = t1[it1 * 4 + 1];
          g[((size_t)k * s.nfft2 + j) * s.nfft1 + ii] += cd(term01 * tt0 + term11 * tt1, term02 * tt0 + term12 * tt1);
        }
      }
    }
  }
  return 0;
}

int or_fphi_uind_sites(OrCtx* c, int nsites, const int* isite, const double* grid, double* phi1, double* phi2,
                       double* sum) {
  if (!c->have_bspline) bspline_fill(c);
  const cd* g = reinterpret_cast<const cd*>(grid);
  for (int q = 0; q < nsites; ++q) {
    if (isite[q] < 0 || isite[q] >= c->s.n) return 1;
    fphi_dip_site(c, isite[q], g, phi1 + 10 * (size_t)q, phi2 + 10 * (size_t)q, sum + 20 * (size_t)q);
  }
  return 0;
}

int or_epolar1(OrCtx* c, const double* uind, const double* uinp, const int* zaxis, const int* xaxis,
               const int* axt, double* dep, double* ep_out, double* vir_out, double* vir_frame) {
  const OrSystem& s = c->s;
  const int n = s.n, bs = c->bsorder, maxelst = c->maxelst;
  if (!c->have_list) return OR_E_LIST_OVERFLOW;
  std::fill(dep, dep + (size_t)n * 3, 0.0);
  double ep = 0.0;
  Vir vir, vframe;  // the reference's virial; the frame-atom virial of the reciprocal and self torques
  // permanent-multipole potential fphirec (20 per site) from efld0_recip
  {
    std::vector<double> cphi((size_t)n * 10);
    or_efld0_recip(c, cphi.data());
  }
  std::vector<double> fphirec = c->fphirec;
  // ---- eprecip1 ---------------------------------------------------------
  {
    static const int deriv1[10] = {2, 5, 8, 9, 11, 16, 18, 14, 15, 20};
    static const int deriv2[10] = {3, 8, 6, 10, 14, 12, 19, 16, 20, 17};
    static const int deriv3[10] = {4, 9, 10, 7, 15, 17, 13, 20, 18, 19};
    const double f = kElectric;
    double a[3][3];
    int nf[3] = {s.nfft1, s.nfft2, s.nfft3};
    for (int i = 0; i < 3; ++i)
      for (int d = 0; d < 3; ++d) a[d][i] = (double)nf[d] * c->recip[i][d];
    double ctf[10][10], ftc[10][10];
    cart_to_frac(c, ctf);
    frac_to_cart(c, ftc);
    std::vector<double> cmp((size_t)n * 10), fmp((size_t)n * 10), fu((size_t)n * 6);
    for (int i = 0; i < n; ++i) {
      const double* rp = &s.rpole[(size_t)i * 13];
      double* cm = &cmp[(size_t)i * 10];
      cm[0] = rp[0]; cm[1] = rp[1]; cm[2] = rp[2]; cm[3] = rp[3]; cm[4] = rp[4]; cm[5] = rp[8];
      cm[6] = rp[12]; cm[7] = 2.0 * rp[5]; cm[8] = 2.0 * rp[6]; cm[9] = 2.0 * rp[9];
      double* fm = &fmp[(size_t)i * 10];
      fm[0] = ctf[0][0] * cm[0];
      for (int j = 1; j < 4; ++j) {
        fm[j] = 0.0;
        for (int k = 1; k < 4; ++k) fm[j] += ctf[j][k] * cm[k];
      }
      for (int j = 4; j < 10; ++j) {
        fm[j] = 0.0;
        for (int k = 4; k < 10; ++k) fm[j] += ctf[j][k] * cm[k];
      }
      for (int j = 0; j < 3; ++j) {
        fu[i * 6 + j] = a[j][0] * uind[i * 3] + a[j][1] * uind[i * 3 + 1] + a[j][2] * uind[i * 3 + 2];
        fu[i * 6 + 3 + j] = a[j][0] * uinp[i * 3] + a[j][1] * uinp[i * 3 + 1] + a[j][2] * uinp[i * 3 + 2];
      }
    }
    if (!c->have_bspline) bspline_fill(c);
    spread_sites(c, [&](int i, const double* t, const double* u, const double* v) {
      const double* fd = &fu[i * 6];
      const double* fp = &fu[i * 6 + 3];
      double term01 = fd[1] * u[1] * v[0] + fd[2] * u[0] * v[1];
      double term11 = fd[0] * u[0] * v[0];
      double term02 = fp[1] * u[1] * v[0] + fp[2] * u[0] * v[1];
      double term12 = fp[0] * u[0] * v[0];
      return cd(term01 * t[0] + term11 * t[1], term02 * t[0] + term12 * t[1]);
    });
    convolve(c);
    double erec = 0.0;
    std::vector<double> fphid(10), fphip(10), fsum(20), fper(20);
    for (int i = 0; i < n; ++i) {
      double T1[10], T2[10], S[20];
      fphi_dip_site(c, i, c->grid.data(), T1, T2, S);
      // 1-based arrays as in the reference: fphid(2:10), fphidprec(1:20), fphirec(1:20)
      double FD[11], FP[11], FS[21], FR[21];
      for (int q = 1; q <= 9; ++q) {
        FD[q + 1] = f * T1[q];
        FP[q + 1] = f * T2[q];
      }
      for (int q = 0; q < 20; ++q) {
        FS[q + 1] = f * S[q];
        FR[q + 1] = f * fphirec[(size_t)i * 20 + q];
      }
      const double* fd = &fu[i * 6];
      const double* fp = &fu[i * 6 + 3];
      double f1 = 0.0, f2 = 0.0, f3 = 0.0;
      for (int k = 1; k <= 3; ++k) {
        int j1 = deriv1[k], j2 = deriv2[k], j3 = deriv3[k];
        erec += fd[k - 1] * FR[k + 1];
        f1 += (fd[k - 1] + fp[k - 1]) * FR[j1] + fd[k - 1] * FP[j1] + fp[k - 1] * FD[j1];
        f2 += (fd[k - 1] + fp[k - 1]) * FR[j2] + fd[k - 1] * FP[j2] + fp[k - 1] * FD[j2];
        f3 += (fd[k - 1] + fp[k - 1]) * FR[j3] + fd[k - 1] * FP[j3] + fp[k - 1] * FD[j3];
      }
      const double* fm = &fmp[(size_t)i * 10];
      for (int k = 1; k <= 10; ++k) {
        f1 += fm[k - 1] * FS[deriv1[k - 1]];
        f2 += fm[k - 1] * FS[deriv2[k - 1]];
        f3 += fm[k - 1] * FS[deriv3[k - 1]];
      }
      f1 = 0.5 * (double)s.nfft1 * f1;
      f2 = 0.5 * (double)s.nfft2 * f2;
      f3 = 0.5 * (double)s.nfft3 * f3;
      dep[i * 3 + 0] += c->recip[0][0] * f1 + c->recip[0][1] * f2 + c->recip[0][2] * f3;
      dep[i * 3 + 1] += c->recip[1][0] * f1 + c->recip[1][1] * f2 + c->recip[1][2] * f3;
      dep[i * 3 + 2] += c->recip[2][0] * f1 + c->recip[2][1] * f2 + c->recip[2][2] * f3;
      // torque from the dipole-grid potential on the permanent moments
      double fh[10];
      for (int q = 0; q < 10; ++q) fh[q] = 0.5 * FS[q + 1];
      double cp[10];
      cp[0] = ftc[0][0] * fh[0];
      for (int j = 1; j < 4; ++j) {
        cp[j] = 0.0;
        for (int k = 1; k < 4; ++k) cp[j] += ftc[j][k] * fh[k];
      }
      for (int j = 4; j < 10; ++j) {
        cp[j] = 0.0;
        for (int k = 4; k < 10; ++k) cp[j] += ftc[j][k] * fh[k];
      }
      const double* cm = &cmp[(size_t)i * 10];
      double trq[3];
      // 1-based: cmp(1..10) = cm[0..9], cphidprec(1..10) = cp[0..9]
      trq[0] = cm[3] * cp[2] - cm[2] * cp[3] + 2.0 * (cm[6] - cm[5]) * cp[9] + cm[8] * cp[7] + cm[9] * cp[5] -
               cm[7] * cp[8] - cm[9] * cp[6];
      trq[1] = cm[1] * cp[3] - cm[3] * cp[1] + 2.0 * (cm[4] - cm[6]) * cp[8] + cm[7] * cp[9] + cm[8] * cp[6] -
               cm[8] * cp[4] - cm[9] * cp[7];
      trq[2] = cm[2] * cp[1] - cm[1] * cp[2] + 2.0 * (cm[5] - cm[4]) * cp[7] + cm[7] * cp[4] + cm[9] * cp[8] -
               cm[7] * cp[5] - cm[8] * cp[9];
      {
        double fz[3], fx[3];
        torque_site(s.x, s.y, s.z, i, zaxis[i], xaxis[i], axt[i], trq, dep, fz, fx);
        frame_virial(s.x, s.y, s.z, i, zaxis[i], xaxis[i], fz, fx, vframe);
      }
      if (vir_out) {
        // induced dipole contribution to the internal virial (epolar1.f:846-908);
        // 1-based names: cphim/cphid/cphip(2:4), cphidprec(1:10) = cp, cmp(1:10) = cm
        double cm_[4] = {0, 0, 0, 0}, cd_[4] = {0, 0, 0, 0}, cq_[4] = {0, 0, 0, 0};
        for (int j = 1; j <= 3; ++j)
          for (int k = 1; k <= 3; ++k) {
            cm_[j] += ftc[j][k] * FR[k + 1];
            cd_[j] += ftc[j][k] * FD[k + 1];
            cq_[j] += ftc[j][k] * FP[k + 1];
          }
        const double* ui = &uind[i * 3];
        const double* up = &uinp[i * 3];
        double vxx = -cp[1] * cm[1] - 0.5 * (cm_[1] * (ui[0] + up[0]) + cd_[1] * up[0] + cq_[1] * ui[0]);
        double vxy = -0.5 * (cp[1] * cm[2] + cp[2] * cm[1]) -
                     0.25 * (cm_[1] * (ui[1] + up[1]) + cm_[2] * (ui[0] + up[0]) + cd_[1] * up[1] + cq_[1] * ui[1] +
                             cd_[2] * up[0] + cq_[2] * ui[0]);
        double vxz = -0.5 * (cp[1] * cm[3] + cp[3] * cm[1]) -
                     0.25 * (cm_[1] * (ui[2] + up[2]) + cm_[3] * (ui[0] + up[0]) + cd_[1] * up[2] + cq_[1] * ui[2] +
                             cd_[3] * up[0] + cq_[3] * ui[0]);
        double vyy = -cp[2] * cm[2] - 0.5 * (cm_[2] * (ui[1] + up[1]) + cd_[2] * up[1] + cq_[2] * ui[1]);
        double vyz = -0.5 * (cp[2] * cm[3] + cp[3] * cm[2]) -
                     0.25 * (cm_[2] * (ui[2] + up[2]) + cm_[3] * (ui[1] + up[1]) + cd_[2] * up[2] + cq_[2] * ui[2] +
                             cd_[3] * up[1] + cq_[3] * ui[1]);
        double vzz = -cp[3] * cm[3] - 0.5 * (cm_[3] * (ui[2] + up[2]) + cd_[3] * up[2] + cq_[3] * ui[2]);
        vxx += -2.0 * cm[4] * cp[4] - cm[7] * cp[7] - cm[8] * cp[8];
        vxy += -(cm[4] + cm[5]) * cp[7] - 0.5 * (cm[7] * (cp[5] + cp[4]) + cm[8] * cp[9] + cm[9] * cp[8]);
        vxz += -(cm[4] + cm[6]) * cp[8] - 0.5 * (cm[8] * (cp[4] + cp[6]) + cm[7] * cp[9] + cm[9] * cp[7]);
        vyy += -2.0 * cm[5] * cp[5] - cm[7] * cp[7] - cm[9] * cp[9];
        vyz += -(cm[5] + cm[6]) * cp[9] - 0.5 * (cm[9] * (cp[5] + cp[6]) + cm[7] * cp[8] + cm[8] * cp[7]);
        vzz += -2.0 * cm[6] * cp[6] - cm[8] * cp[8] - cm[9] * cp[9];
        vir.add(vxx, vxy, vxz, vyy, vyz, vzz);
      }
    }
    ep += 0.5 * erec;
    if (vir_out) {
      const int nthr = nthreads_of(&s);
      const int n1 = s.nfft1, n2 = s.nfft2, n3 = s.nfft3;
      // minus the permanent-only scalar sum (the multipole term's own virial,
      // removed as eprecip1 does with -vmxx..., epolar1.f:534-541)
      spread_sites(c, [&](int i, const double* t, const double* u, const double* v) {
        return cd(mpole_stencil(&fmp[(size_t)i * 10], t, u, v), 0.0);
      });
      fft3d_impl(c->grid.data(), n1, n2, n3, -1, nthr);
      kspace_virial(c, f, -1.0, [&](int, int, int, size_t idx) { return std::norm(c->grid[idx]); }, vir);
      // (rpole + uinp) x (rpole + uind) scalar sum (epolar1.f:932-1091): the two
      // real grids in the real and imaginary parts of one transform
      std::vector<double> fa((size_t)n * 10), fb((size_t)n * 10);
      for (int i = 0; i < n; ++i) {
        frac_moments(ctf, &cmp[(size_t)i * 10], &uinp[i * 3], &fa[(size_t)i * 10]);
        frac_moments(ctf, &cmp[(size_t)i * 10], &uind[i * 3], &fb[(size_t)i * 10]);
      }
      spread_sites(c, [&](int i, const double* t, const double* u, const double* v) {
        return cd(mpole_stencil(&fa[(size_t)i * 10], t, u, v), mpole_stencil(&fb[(size_t)i * 10], t, u, v));
      });
      fft3d_impl(c->grid.data(), n1, n2, n3, -1, nthr);
      kspace_virial(c, f, 1.0, [&](int k1, int k2, int k3, size_t idx) {
        const size_t mi = ((size_t)((n3 - k3) % n3) * n2 + (n2 - k2) % n2) * n1 + (n1 - k1) % n1;
        const cd g = c->grid[idx], gm = std::conj(c->grid[mi]);
        const cd fa_k = 0.5 * (g + gm), fb_k = cd(0.0, -0.5) * (g - gm);
        return fa_k.real() * fb_k.real() + fa_k.imag() * fb_k.imag();
      }, vir);
    }
  }
  // ---- epreal1c (Thole branch) -------------------------------------------
  {
    const double f = 0.5 * kElectric;
    const double off2 = s.ewaldcut * s.ewaldcut;
    std::vector<double> ufld((size_t)n * 3, 0.0), dufld((size_t)n * 6, 0.0);
    ScaleWs w;
    w.init(n);
    for (int i = 0; i < n; ++i) {
      const double* ri = &s.rpole[(size_t)i * 13];
      double ci = ri[0], dix = ri[1], diy = ri[2], diz = ri[3];
      double qixx = ri[4], qixy = ri[5], qixz = ri[6], qiyy = ri[8], qiyz = ri[9], qizz = ri[12];
      double uix = uind[i * 3], uiy = uind[i * 3 + 1], uiz = uind[i * 3 + 2];
      double uixp = uinp[i * 3], uiyp = uinp[i * 3 + 1], uizp = uinp[i * 3 + 2];
      double pdi = s.pdamp[i], pti = s.thole[i];
      set_dp_scales(s, i, w);
      set_u_scales(s, i, w, false);
      for (int kkk = 0; kkk < c->nelst[i]; ++kkk) {
        int k = c->elst[(size_t)i * maxelst + kkk];
        double xr = s.x[k] - s.x[i], yr = s.y[k] - s.y[i], zr = s.z[k] - s.z[i];
        image(c->cell, xr, yr, zr);
        double r2 = xr * xr + yr * yr + zr * zr;
        if (r2 > off2) continue;
        double r = std::sqrt(r2);
        const double* rk = &s.rpole[(size_t)k * 13];
        double ck = rk[0], dkx = rk[1], dky = rk[2], dkz = rk[3];
        double qkxx = rk[4], qkxy = rk[5], qkxz = rk[6], qkyy = rk[8], qkyz = rk[9], qkzz = rk[12];
        double ukx = uind[k * 3], uky = uind[k * 3 + 1], ukz = uind[k * 3 + 2];
        double ukxp = uinp[k * 3], ukyp = uinp[k * 3 + 1], ukzp = uinp[k * 3 + 2];
        double dir = dix * xr + diy * yr + diz * zr;
        double qix = qixx * xr + qixy * yr + qixz * zr;
        double qiy = qixy * xr + qiyy * yr + qiyz * zr;
        double qiz = qixz * xr + qiyz * yr + qizz * zr;
        double qir = qix * xr + qiy * yr + qiz * zr;
        double dkr = dkx * xr + dky * yr + dkz * zr;
        double qkx = qkxx * xr + qkxy * yr + qkxz * zr;
        double qky = qkxy * xr + qkyy * yr + qkyz * zr;
        double qkz = qkxz * xr + qkyz * yr + qkzz * zr;
        double qkr = qkx * xr + qky * yr + qkz * zr;
        double uir = uix * xr + uiy * yr + uiz * zr;
        double uirp = uixp * xr + uiyp * yr + uizp * zr;
        double ukr = ukx * xr + uky * yr + ukz * zr;
        double ukrp = ukxp * xr + ukyp * yr + ukzp * zr;
        double rr1 = f / r;
        double rr3 = rr1 / r2;
        double rr5 = 3.0 * rr3 / r2;
        double rr7 = 5.0 * rr5 / r2;
        double rr9 = 7.0 * rr7 / r2;
        double dmpe[10];
        dampewald(9, r, r2, f, s.aewald, dmpe);
        double sc3 = 1.0, sc5 = 1.0, sc7 = 1.0;
        double rc3[3] = {0, 0, 0}, rc5[3] = {0, 0, 0}, rc7[3] = {0, 0, 0};
        double damp = pdi * s.pdamp[k];
        double pgamma = std::min(pti, s.thole[k]);
        if (pgamma == 0.0) pgamma = std::max(pti, s.thole[k]);
        if (damp != 0.0 && pgamma != 0.0) {
          double t = r / damp;
          damp = pgamma * (t * t * t);
          if (damp < 50.0) {
            double expdamp = std::exp(-damp);
            sc3 = 1.0 - expdamp;
            sc5 = 1.0 - (1.0 + damp) * expdamp;
            sc7 = 1.0 - (1.0 + damp + 0.6 * damp * damp) * expdamp;
            double temp3 = 3.0 * damp * expdamp / r2;
            double temp5 = damp;
            double temp7 = -0.2 + 0.6 * damp;
            rc3[0] = xr * temp3; rc3[1] = yr * temp3; rc3[2] = zr * temp3;
            for (int j = 0; j < 3; ++j) {
              rc5[j] = rc3[j] * temp5;
              rc7[j] = rc5[j] * temp7;
            }
          }
        }
        double ps = w.p[k], ds = w.d[k], us = w.u[k];
        double psc3 = 1.0 - sc3 * ps, psc5 = 1.0 - sc5 * ps, psc7 = 1.0 - sc7 * ps;
        double dsc3 = 1.0 - sc3 * ds, dsc5 = 1.0 - sc5 * ds, dsc7 = 1.0 - sc7 * ds;
        double usc3 = 1.0 - sc3 * us, usc5 = 1.0 - sc5 * us;
        double psr3 = dmpe[3] - psc3 * rr3, psr5 = dmpe[5] - psc5 * rr5, psr7 = dmpe[7] - psc7 * rr7;
        double dsr3 = dmpe[3] - dsc3 * rr3, dsr5 = dmpe[5] - dsc5 * rr5, dsr7 = dmpe[7] - dsc7 * rr7;
        double usr5 = dmpe[5] - usc5 * rr5;
        double prc3[3], prc5[3], prc7[3], drc3[3], drc5[3], drc7[3], urc3[3], urc5[3];
        for (int j = 0; j < 3; ++j) {
          prc3[j] = rc3[j] * ps; prc5[j] = rc5[j] * ps; prc7[j] = rc7[j] * ps;
          drc3[j] = rc3[j] * ds; drc5[j] = rc5[j] * ds; drc7[j] = rc7[j] * ds;
          urc3[j] = rc3[j] * us; urc5[j] = rc5[j] * us;
        }
        (void)usc3;
        // induced field at i and k for the torques
        double tix3 = psr3 * ukx + dsr3 * ukxp, tiy3 = psr3 * uky + dsr3 * ukyp, tiz3 = psr3 * ukz + dsr3 * ukzp;
        double tkx3 = psr3 * uix + dsr3 * uixp, tky3 = psr3 * uiy + dsr3 * uiyp, tkz3 = psr3 * uiz + dsr3 * uizp;
        double tuir = -psr5 * ukr - dsr5 * ukrp;
        double tukr = -psr5 * uir - dsr5 * uirp;
        ufld[i * 3 + 0] += tix3 + xr * tuir;
        ufld[i * 3 + 1] += tiy3 + yr * tuir;
        ufld[i * 3 + 2] += tiz3 + zr * tuir;
        ufld[k * 3 + 0] += tkx3 + xr * tukr;
        ufld[k * 3 + 1] += tky3 + yr * tukr;
        ufld[k * 3 + 2] += tkz3 + zr * tukr;
        // energy with the p-scaled permanent field (damptholed order 7)
        {
          double dmpik[8];
          dampthole(pdi, s.pdamp[k], pti, s.thole[k], 7, r, dmpik);
          double scalek = ps;
          double dmp3 = dmpe[3] - (1.0 - scalek * dmpik[3]) * rr3;
          double dmp5 = dmpe[5] - (1.0 - scalek * dmpik[5]) * rr5;
          double dmp7 = dmpe[7] - (1.0 - scalek * dmpik[7]) * rr7;
          double fip[3], fkp[3];
          fip[0] = -xr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dkx + 2.0 * dmp5 * qkx;
          fip[1] = -yr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dky + 2.0 * dmp5 * qky;
          fip[2] = -zr * (dmp3 * ck - dmp5 * dkr + dmp7 * qkr) - dmp3 * dkz + 2.0 * dmp5 * qkz;
          fkp[0] = xr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * dix - 2.0 * dmp5 * qix;
          fkp[1] = yr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * diy - 2.0 * dmp5 * qiy;
          fkp[2] = zr * (dmp3 * ci + dmp5 * dir + dmp7 * qir) - dmp3 * diz - 2.0 * dmp5 * qiz;
          double e = 0.0;
          for (int j = 0; j < 3; ++j) e = e - uind[i * 3 + j] * fip[j] - uind[k * 3 + j] * fkp[j];
          ep += e;
        }
        double tix5 = 2.0 * (psr5 * ukx + dsr5 * ukxp), tiy5 = 2.0 * (psr5 * uky + dsr5 * ukyp),
               tiz5 = 2.0 * (psr5 * ukz + dsr5 * ukzp);
        double tkx5 = 2.0 * (psr5 * uix + dsr5 * uixp), tky5 = 2.0 * (psr5 * uiy + dsr5 * uiyp),
               tkz5 = 2.0 * (psr5 * uiz + dsr5 * uizp);
        tuir = -psr7 * ukr - dsr7 * ukrp;
        tukr = -psr7 * uir - dsr7 * uirp;
        double* dfi = &dufld[i * 6];
        double* dfk = &dufld[k * 6];
        dfi[0] += xr * tix5 + xr * xr * tuir;
        dfi[1] += xr * tiy5 + yr * tix5 + 2.0 * xr * yr * tuir;
        dfi[2] += yr * tiy5 + yr * yr * tuir;
        dfi[3] += xr * tiz5 + zr * tix5 + 2.0 * xr * zr * tuir;
        dfi[4] += yr * tiz5 + zr * tiy5 + 2.0 * yr * zr * tuir;
        dfi[5] += zr * tiz5 + zr * zr * tuir;
        dfk[0] -= xr * tkx5 + xr * xr * tukr;
        dfk[1] -= xr * tky5 + yr * tkx5 + 2.0 * xr * yr * tukr;
        dfk[2] -= yr * tky5 + yr * yr * tukr;
        dfk[3] -= xr * tkz5 + zr * tkx5 + 2.0 * xr * zr * tukr;
        dfk[4] -= yr * tkz5 + zr * tky5 + 2.0 * yr * zr * tukr;
        dfk[5] -= zr * tkz5 + zr * zr * tukr;
        // gradient of the permanent field times the dipoles: d part (uinp) and p part (uind)
        auto perm_part = [&](double sc3_, double sc5_, double sc7_, double sr3, double sr5, double sr7,
                             const double* xc3, const double* xc5, const double* xc7, double vkx, double vky,
                             double vkz, double vix, double viy, double viz, double out[3]) {
          double term1 = dmpe[5] - sc3_ * rr5;
          double term2 = dmpe[7] - sc5_ * rr7;
          double term3 = -sr3 + term1 * xr * xr - rr3 * xr * xc3[0];
          double term4 = rr3 * xc3[0] - term1 * xr - sr5 * xr;
          double term5 = term2 * xr * xr - sr5 - rr5 * xr * xc5[0];
          double term6 = (dmpe[9] - sc7_ * rr9) * xr * xr - dmpe[7] - rr7 * xr * xc7[0];
          double term7 = rr5 * xc5[0] - 2.0 * dmpe[7] * xr + (sc5_ + 1.5 * sc7_) * rr7 * xr;
          double tixx = ci * term3 + dix * term4 + dir * term5 + 2.0 * sr5 * qixx + (qiy * yr + qiz * zr) * sc7_ * rr7 +
                        2.0 * qix * term7 + qir * term6;
          double tkxx = ck * term3 - dkx * term4 - dkr * term5 + 2.0 * sr5 * qkxx + (qky * yr + qkz * zr) * sc7_ * rr7 +
                        2.0 * qkx * term7 + qkr * term6;
          term3 = -sr3 + term1 * yr * yr - rr3 * yr * xc3[1];
          term4 = rr3 * xc3[1] - term1 * yr - sr5 * yr;
          term5 = term2 * yr * yr - sr5 - rr5 * yr * xc5[1];
          term6 = (dmpe[9] - sc7_ * rr9) * yr * yr - dmpe[7] - rr7 * yr * xc7[1];
          term7 = rr5 * xc5[1] - 2.0 * dmpe[7] * yr + (sc5_ + 1.5 * sc7_) * rr7 * yr;
          double tiyy = ci * term3 + diy * term4 + dir * term5 + 2.0 * sr5 * qiyy + (qix * xr + qiz * zr) * sc7_ * rr7 +
                        2.0 * qiy * term7 + qir * term6;
          double tkyy = ck * term3 - dky * term4 - dkr * term5 + 2.0 * sr5 * qkyy + (qkx * xr + qkz * zr) * sc7_ * rr7 +
                        2.0 * qky * term7 + qkr * term6;
          term3 = -sr3 + term1 * zr * zr - rr3 * zr * xc3[2];
          term4 = rr3 * xc3[2] - term1 * zr - sr5 * zr;
          term5 = term2 * zr * zr - sr5 - rr5 * zr * xc5[2];
          term6 = (dmpe[9] - sc7_ * rr9) * zr * zr - dmpe[7] - rr7 * zr * xc7[2];
          term7 = rr5 * xc5[2] - 2.0 * dmpe[7] * zr + (sc5_ + 1.5 * sc7_) * rr7 * zr;
          double tizz = ci * term3 + diz * term4 + dir * term5 + 2.0 * sr5 * qizz + (qix * xr + qiy * yr) * sc7_ * rr7 +
                        2.0 * qiz * term7 + qir * term6;
          double tkzz = ck * term3 - dkz * term4 - dkr * term5 + 2.0 * sr5 * qkzz + (qkx * xr + qky * yr) * sc7_ * rr7 +
                        2.0 * qkz * term7 + qkr * term6;
          term3 = term1 * xr * yr - rr3 * yr * xc3[0];
          term4 = rr3 * xc3[0] - term1 * xr;
          term5 = term2 * xr * yr - rr5 * yr * xc5[0];
          term6 = (dmpe[9] - sc7_ * rr9) * xr * yr - rr7 * yr * xc7[0];
          term7 = rr5 * xc5[0] - term2 * xr;
          double tixy = ci * term3 - sr5 * dix * yr + diy * term4 + dir * term5 + 2.0 * sr5 * qixy -
                        2.0 * sr7 * yr * qix + 2.0 * qiy * term7 + qir * term6;
          double tkxy = ck * term3 + sr5 * dkx * yr - dky * term4 - dkr * term5 + 2.0 * sr5 * qkxy -
                        2.0 * sr7 * yr * qkx + 2.0 * qky * term7 + qkr * term6;
          term3 = term1 * xr * zr - rr3 * zr * xc3[0];
          term5 = term2 * xr * zr - rr5 * zr * xc5[0];
          term6 = (dmpe[9] - sc7_ * rr9) * xr * zr - rr7 * zr * xc7[0];
          double tixz = ci * term3 - sr5 * dix * zr + diz * term4 + dir * term5 + 2.0 * sr5 * qixz -
                        2.0 * sr7 * zr * qix + 2.0 * qiz * term7 + qir * term6;
          double tkxz = ck * term3 + sr5 * dkx * zr - dkz * term4 - dkr * term5 + 2.0 * sr5 * qkxz -
                        2.0 * sr7 * zr * qkx + 2.0 * qkz * term7 + qkr * term6;
          term3 = term1 * yr * zr - rr3 * zr * xc3[1];
          term4 = rr3 * xc3[1] - term1 * yr;
          term5 = term2 * yr * zr - rr5 * zr * xc5[1];
          term6 = (dmpe[9] - sc7_ * rr9) * yr * zr - rr7 * zr * xc7[1];
          term7 = rr5 * xc5[1] - term2 * yr;
          double tiyz = ci * term3 - sr5 * diy * zr + diz * term4 + dir * term5 + 2.0 * sr5 * qiyz -
                        2.0 * sr7 * zr * qiy + 2.0 * qiz * term7 + qir * term6;
          double tkyz = ck * term3 + sr5 * dky * zr - dkz * term4 - dkr * term5 + 2.0 * sr5 * qkyz -
                        2.0 * sr7 * zr * qky + 2.0 * qkz * term7 + qkr * term6;
          out[0] = tixx * vkx + tixy * vky + tixz * vkz - tkxx * vix - tkxy * viy - tkxz * viz;
          out[1] = tixy * vkx + tiyy * vky + tiyz * vkz - tkxy * vix - tkyy * viy - tkyz * viz;
          out[2] = tixz * vkx + tiyz * vky + tizz * vkz - tkxz * vix - tkyz * viy - tkzz * viz;
        };
        double frc[3], dp[3];
        perm_part(dsc3, dsc5, dsc7, dsr3, dsr5, dsr7, drc3, drc5, drc7, ukxp, ukyp, ukzp, uixp, uiyp, uizp, frc);
        perm_part(psc3, psc5, psc7, psr3, psr5, psr7, prc3, prc5, prc7, ukx, uky, ukz, uix, uiy, uiz, dp);
        for (int j = 0; j < 3; ++j) frc[j] += dp[j];
        // mutual part: uind . grad T . uinp with uscale
        {
          double term1 = dmpe[5] - usc3 * rr5;
          double term2 = dmpe[7] - usc5 * rr7;
          double term3 = usr5 + term1;
          double term4 = rr3 * us;
          double term5 = -xr * term3 + rc3[0] * term4;
          double term6 = -usr5 + xr * xr * term2 - rr5 * xr * urc5[0];
          double tixx = uix * term5 + uir * term6;
          double tkxx = ukx * term5 + ukr * term6;
          term5 = -yr * term3 + rc3[1] * term4;
          term6 = -usr5 + yr * yr * term2 - rr5 * yr * urc5[1];
          double tiyy = uiy * term5 + uir * term6;
          double tkyy = uky * term5 + ukr * term6;
          term5 = -zr * term3 + rc3[2] * term4;
          term6 = -usr5 + zr * zr * term2 - rr5 * zr * urc5[2];
          double tizz = uiz * term5 + uir * term6;
          double tkzz = ukz * term5 + ukr * term6;
          term4 = -usr5 * yr;
          term5 = -xr * term1 + rr3 * urc3[0];
          term6 = xr * yr * term2 - rr5 * yr * urc5[0];
          double tixy = uix * term4 + uiy * term5 + uir * term6;
          double tkxy = ukx * term4 + uky * term5 + ukr * term6;
          term4 = -usr5 * zr;
          term6 = xr * zr * term2 - rr5 * zr * urc5[0];
          double tixz = uix * term4 + uiz * term5 + uir * term6;
          double tkxz = ukx * term4 + ukz * term5 + ukr * term6;
          term5 = -yr * term1 + rr3 * urc3[1];
          term6 = yr * zr * term2 - rr5 * zr * urc5[1];
          double tiyz = uiy * term4 + uiz * term5 + uir * term6;
          double tkyz = uky * term4 + ukz * term5 + ukr * term6;
          frc[0] += tixx * ukxp + tixy * ukyp + tixz * ukzp + tkxx * uixp + tkxy * uiyp + tkxz * uizp;
          frc[1] += tixy * ukxp + tiyy * ukyp + tiyz * ukzp + tkxy * uixp + tkyy * uiyp + tkyz * uizp;
          frc[2] += tixz * ukxp + tiyz * ukyp + tizz * ukzp + tkxz * uixp + tkyz * uiyp + tkzz * uizp;
        }
        for (int j = 0; j < 3; ++j) {
          dep[i * 3 + j] -= frc[j];
          dep[k * 3 + j] += frc[j];
        }
        // the virial of the pairwise Cartesian forces (epolar1.f:2326-2342)
        vir.add(xr * frc[0], 0.5 * (yr * frc[0] + xr * frc[1]), 0.5 * (zr * frc[0] + xr * frc[2]), yr * frc[1],
                0.5 * (zr * frc[1] + yr * frc[2]), zr * frc[2]);
      }
      reset_dp_scales(s, i, w);
      set_u_scales(s, i, w, true);
    }
    // torque of the induced field and gradient on the permanent moments
    for (int i = 0; i < n; ++i) {
      const double* ri = &s.rpole[(size_t)i * 13];
      double dix = ri[1], diy = ri[2], diz = ri[3];
      double qixx = ri[4], qixy = ri[5], qixz = ri[6], qiyy = ri[8], qiyz = ri[9], qizz = ri[12];
      const double* uf = &ufld[i * 3];
      const double* du = &dufld[i * 6];
      double tep[3];
      tep[0] = diz * uf[1] - diy * uf[2] + qixz * du[1] - qixy * du[3] + 2.0 * qiyz * (du[2] - du[5]) +
               (qizz - qiyy) * du[4];
      tep[1] = dix * uf[2] - diz * uf[0] - qiyz * du[1] + qixy * du[4] + 2.0 * qixz * (du[5] - du[0]) +
               (qixx - qizz) * du[3];
      tep[2] = diy * uf[0] - dix * uf[1] + qiyz * du[3] - qixz * du[4] + 2.0 * qixy * (du[0] - du[2]) +
               (qiyy - qixx) * du[1];
      double fz[3], fx[3];
      torque_site(s.x, s.y, s.z, i, zaxis[i], xaxis[i], axt[i], tep, dep, fz, fx);
      // the virial of the torque's frame-atom forces (epolar1.f:2460-2486)
      frame_virial(s.x, s.y, s.z, i, zaxis[i], xaxis[i], fz, fx, vir);
    }
  }
  // ---- self energy and self torque (epolar1.f:181-206) --------------------
  {
    const double f = kElectric;
    double term = 2.0 * s.aewald * s.aewald;
    double fterm = -f * s.aewald / kSqrtPi;
    for (int i = 0; i < n; ++i) {
      const double* rp = &s.rpole[(size_t)i * 13];
      double uii = rp[1] * uind[i * 3] + rp[2] * uind[i * 3 + 1] + rp[3] * uind[i * 3 + 2];
      ep += fterm * term * uii / 3.0;
    }
    term = (4.0 / 3.0) * f * s.aewald * s.aewald * s.aewald / kSqrtPi;
    for (int i = 0; i < n; ++i) {
      const double* rp = &s.rpole[(size_t)i * 13];
      double dix = rp[1], diy = rp[2], diz = rp[3];
      double uix = 0.5 * (uind[i * 3] + uinp[i * 3]);
      double uiy = 0.5 * (uind[i * 3 + 1] + uinp[i * 3 + 1]);
      double uiz = 0.5 * (uind[i * 3 + 2] + uinp[i * 3 + 2]);
      double trq[3] = {term * (diy * uiz - diz * uiy), term * (diz * uix - dix * uiz), term * (dix * uiy - diy * uix)};
      double fz[3], fx[3];
      torque_site(s.x, s.y, s.z, i, zaxis[i], xaxis[i], axt[i], trq, dep, fz, fx);
      frame_virial(s.x, s.y, s.z, i, zaxis[i], xaxis[i], fz, fx, vframe);
    }
  }
  if (ep_out) *ep_out = ep;
  if (vir_out) vir.out(vir_out);
  if (vir_frame) vframe.out(vir_frame);
  return OR_OK;
}

// ===========================================================================
// Permanent-multipole energy and gradient: empole1c (empole1.f:42-340) for the
// TINFOIL boundary, without charge penetration, charge flux or lambda terms:
// emrecip1 (:349-861), emreal1c (:873-1555, standard branch) over the half
// list, the Ewald self energy (:134-160), torques distributed by torque
// (torque.f:6-390).  Virial terms are not restated.
int or_empole1(OrCtx* c, const int* zaxis, const int* xaxis, const int* axt, double* dem, double* parts,
               double* vir_out, double* vir_frame) {
  const OrSystem& s = c->s;
  const int n = s.n, maxelst = c->maxelst;
  if (!c->have_list) return OR_E_LIST_OVERFLOW;
  std::fill(dem, dem + (size_t)n * 3, 0.0);
  const double f = kElectric;  // electric / dielec, dielec = 1
  double erecip = 0.0, ereal = 0.0, eself = 0.0;
  Vir vir, vframe;
  // ---- emrecip1 ----------------------------------------------------------
  {
    // the multipole grid, convolved, and fphirec(20) (unscaled)
    std::vector<double> cphi0((size_t)n * 10);
    or_efld0_recip(c, cphi0.data());
    static const int deriv1[10] = {2, 5, 8, 9, 11, 16, 18, 14, 15, 20};
    static const int deriv2[10] = {3, 8, 6, 10, 14, 12, 19, 16, 20, 17};
    static const int deriv3[10] = {4, 9, 10, 7, 15, 17, 13, 20, 18, 19};
    double ctf[10][10], ftc[10][10];
    cart_to_frac(c, ctf);
    frac_to_cart(c, ftc);
    const int nf[3] = {s.nfft1, s.nfft2, s.nfft3};
    std::vector<double> demrec((size_t)n * 3, 0.0), fmp(vir_out ? (size_t)n * 10 : 0);
    for (int i = 0; i < n; ++i) {
      const double* rp = &s.rpole[(size_t)i * 13];
      const double cm[10] = {rp[0], rp[1], rp[2], rp[3], rp[4], rp[8], rp[12], 2.0 * rp[5], 2.0 * rp[6], 2.0 * rp[9]};
      double fm[10];
      fm[0] = ctf[0][0] * cm[0];
      for (int j = 1; j < 4; ++j) {
        fm[j] = 0.0;
        for (int k = 1; k < 4; ++k) fm[j] += ctf[j][k] * cm[k];
      }
      for (int j = 4; j < 10; ++j) {
        fm[j] = 0.0;
        for (int k = 4; k < 10; ++k) fm[j] += ctf[j][k] * cm[k];
      }
      // fphirec = electric * fphirec; 1-based view FR[1..20]
      double FR[21];
      for (int q = 0; q < 20; ++q) FR[q + 1] = f * c->fphirec[(size_t)i * 20 + q];
      double cp[10];  // fphi_to_cphi_site
      cp[0] = ftc[0][0] * FR[1];
      for (int j = 1; j < 4; ++j) {
        cp[j] = 0.0;
        for (int k = 1; k < 4; ++k) cp[j] += ftc[j][k] * FR[k + 1];
      }
      for (int j = 4; j < 10; ++j) {
        cp[j] = 0.0;
        for (int k = 4; k < 10; ++k) cp[j] += ftc[j][k] * FR[k + 1];
      }
      double f1 = 0.0, f2 = 0.0, f3 = 0.0;
      for (int k = 0; k < 10; ++k) {
        erecip += fm[k] * FR[k + 1];
        f1 += fm[k] * FR[deriv1[k]];
        f2 += fm[k] * FR[deriv2[k]];
        f3 += fm[k] * FR[deriv3[k]];
      }
      f1 = (double)nf[0] * f1;
      f2 = (double)nf[1] * f2;
      f3 = (double)nf[2] * f3;
      demrec[i * 3 + 0] += c->recip[0][0] * f1 + c->recip[0][1] * f2 + c->recip[0][2] * f3;
      demrec[i * 3 + 1] += c->recip[1][0] * f1 + c->recip[1][1] * f2 + c->recip[1][2] * f3;
      demrec[i * 3 + 2] += c->recip[2][0] * f1 + c->recip[2][1] * f2 + c->recip[2][2] * f3;
      double trq[3];
      trq[0] = cm[3] * cp[2] - cm[2] * cp[3] + 2.0 * (cm[6] - cm[5]) * cp[9] + cm[8] * cp[7] + cm[9] * cp[5] -
               cm[7] * cp[8] - cm[9] * cp[6];
      trq[1] = cm[1] * cp[3] - cm[3] * cp[1] + 2.0 * (cm[4] - cm[6]) * cp[8] + cm[7] * cp[9] + cm[8] * cp[6] -
               cm[8] * cp[4] - cm[9] * cp[7];
      trq[2] = cm[2] * cp[1] - cm[1] * cp[2] + 2.0 * (cm[5] - cm[4]) * cp[7] + cm[7] * cp[4] + cm[9] * cp[8] -
               cm[7] * cp[5] - cm[8] * cp[9];
      double fz[3], fx[3];
      torque_site(s.x, s.y, s.z, i, zaxis[i], xaxis[i], axt[i], trq, demrec.data(), fz, fx);  // torque_rec
      if (vir_out) {
        // the frame-atom virial of the reciprocal torque, which the reference
        // does not add (torque_rec carries no virial)
        frame_virial(s.x, s.y, s.z, i, zaxis[i], xaxis[i], fz, fx, vframe);
        for (int q = 0; q < 10; ++q) fmp[(size_t)i * 10 + q] = fm[q];
        // permanent multipole contribution to the internal virial (empole1.f:741-761)
        vir.add(-cm[1] * cp[1] - 2.0 * cm[4] * cp[4] - cm[7] * cp[7] - cm[8] * cp[8],
                -0.5 * (cm[2] * cp[1] + cm[1] * cp[2]) - (cm[4] + cm[5]) * cp[7] - 0.5 * cm[7] * (cp[4] + cp[5]) -
                    0.5 * (cm[8] * cp[9] + cm[9] * cp[8]),
                -0.5 * (cm[3] * cp[1] + cm[1] * cp[3]) - (cm[4] + cm[6]) * cp[8] - 0.5 * cm[8] * (cp[4] + cp[6]) -
                    0.5 * (cm[7] * cp[9] + cm[9] * cp[7]),
                -cm[2] * cp[2] - 2.0 * cm[5] * cp[5] - cm[7] * cp[7] - cm[9] * cp[9],
                -0.5 * (cm[3] * cp[2] + cm[2] * cp[3]) - (cm[5] + cm[6]) * cp[9] - 0.5 * cm[9] * (cp[5] + cp[6]) -
                    0.5 * (cm[7] * cp[8] + cm[8] * cp[7]),
                -cm[3] * cp[3] - 2.0 * cm[6] * cp[6] - cm[8] * cp[8] - cm[9] * cp[9]);
      }
    }
    erecip = 0.5 * erecip;
    for (size_t q = 0; q < (size_t)n * 3; ++q) dem[q] += demrec[q];
    if (vir_out) {
      // the scalar sum over the reciprocal lattice (empole1.f:560-598)
      spread_sites(c, [&](int i, const double* t, const double* u, const double* v) {
        return cd(mpole_stencil(&fmp[(size_t)i * 10], t, u, v), 0.0);
      });
      fft3d_impl(c->grid.data(), s.nfft1, s.nfft2, s.nfft3, -1, nthreads_of(&s));
      kspace_virial(c, f, 1.0, [&](int, int, int, size_t idx) { return std::norm(c->grid[idx]); }, vir);
    }
  }
  // ---- emreal1c (standard branch) ----------------------------------------
  {
    const double off2 = s.ewaldcut * s.ewaldcut;
    std::vector<double> mscale(n, 1.0), tem((size_t)n * 3, 0.0);
    const int mslot[4] = {OR_I12, OR_I13, OR_I14, OR_I15};
    for (int i = 0; i < n; ++i) {
      const double* ri = &s.rpole[(size_t)i * 13];
      const double ci = ri[0], dix = ri[1], diy = ri[2], diz = ri[3];
      const double qixx = ri[4], qixy = ri[5], qixz = ri[6], qiyy = ri[8], qiyz = ri[9], qizz = ri[12];
      for (int b = 0; b < 4; ++b) for_conn(s, mslot[b], i, [&](int k) { mscale[k] = s.m_scale[b]; });
      for (int kkk = 0; kkk < c->nelst[i]; ++kkk) {
        const int k = c->elst[(size_t)i * maxelst + kkk];
        double xr = s.x[k] - s.x[i], yr = s.y[k] - s.y[i], zr = s.z[k] - s.z[i];
        image(c->cell, xr, yr, zr);
        const double r2 = xr * xr + yr * yr + zr * zr;
        if (!(r2 <= off2)) continue;
        const double r = std::sqrt(r2);
        const double* rk = &s.rpole[(size_t)k * 13];
        const double ck = rk[0], dkx = rk[1], dky = rk[2], dkz = rk[3];
        const double qkxx = rk[4], qkxy = rk[5], qkxz = rk[6], qkyy = rk[8], qkyz = rk[9], qkzz = rk[12];
        // intermediates involving moments and separation distance
        const double dir = dix * xr + diy * yr + diz * zr;
        const double qix = qixx * xr + qixy * yr + qixz * zr;
        const double qiy = qixy * xr + qiyy * yr + qiyz * zr;
        const double qiz = qixz * xr + qiyz * yr + qizz * zr;
        const double qir = qix * xr + qiy * yr + qiz * zr;
        const double dkr = dkx * xr + dky * yr + dkz * zr;
        const double qkx = qkxx * xr + qkxy * yr + qkxz * zr;
        const double qky = qkxy * xr + qkyy * yr + qkyz * zr;
        const double qkz = qkxz * xr + qkyz * yr + qkzz * zr;
        const double qkr = qkx * xr + qky * yr + qkz * zr;
        const double dik = dix * dkx + diy * dky + diz * dkz;
        const double qik = qix * qkx + qiy * qky + qiz * qkz;
        const double diqk = dix * qkx + diy * qky + diz * qkz;
        const double dkqi = dkx * qix + dky * qiy + dkz * qiz;
        const double qiqk = 2.0 * (qixy * qkxy + qixz * qkxz + qiyz * qkyz) + qixx * qkxx + qiyy * qkyy + qizz * qkzz;
        // additional intermediates involving moments and distance
        const double dirx = diy * zr - diz * yr, diry = diz * xr - dix * zr, dirz = dix * yr - diy * xr;
        const double dkrx = dky * zr - dkz * yr, dkry = dkz * xr - dkx * zr, dkrz = dkx * yr - dky * xr;
        const double dikx = diy * dkz - diz * dky, diky = diz * dkx - dix * dkz, dikz = dix * dky - diy * dkx;
        const double qirx = qiz * yr - qiy * zr, qiry = qix * zr - qiz * xr, qirz = qiy * xr - qix * yr;
        const double qkrx = qkz * yr - qky * zr, qkry = qkx * zr - qkz * xr, qkrz = qky * xr - qkx * yr;
        const double qikx = qky * qiz - qkz * qiy, qiky = qkz * qix - qkx * qiz, qikz = qkx * qiy - qky * qix;
        const double qixk = qixx * qkx + qixy * qky + qixz * qkz;
        const double qiyk = qixy * qkx + qiyy * qky + qiyz * qkz;
        const double qizk = qixz * qkx + qiyz * qky + qizz * qkz;
        const double qkxi = qkxx * qix + qkxy * qiy + qkxz * qiz;
        const double qkyi = qkxy * qix + qkyy * qiy + qkyz * qiz;
        const double qkzi = qkxz * qix + qkyz * qiy + qkzz * qiz;
        const double qikrx = qizk * yr - qiyk * zr, qikry = qixk * zr - qizk * xr, qikrz = qiyk * xr - qixk * yr;
        const double qkirx = qkzi * yr - qkyi * zr, qkiry = qkxi * zr - qkzi * xr, qkirz = qkyi * xr - qkxi * yr;
        const double diqkx = dix * qkxx + diy * qkxy + diz * qkxz;
        const double diqky = dix * qkxy + diy * qkyy + diz * qkyz;
        const double diqkz = dix * qkxz + diy * qkyz + diz * qkzz;
        const double dkqix = dkx * qixx + dky * qixy + dkz * qixz;
        const double dkqiy = dkx * qixy + dky * qiyy + dkz * qiyz;
        const double dkqiz = dkx * qixz + dky * qiyz + dkz * qizz;
        const double diqkrx = diqkz * yr - diqky * zr, diqkry = diqkx * zr - diqkz * xr,
                     diqkrz = diqky * xr - diqkx * yr;
        const double dkqirx = dkqiz * yr - dkqiy * zr, dkqiry = dkqix * zr - dkqiz * xr,
                     dkqirz = dkqiy * xr - dkqix * yr;
        const double dqikx = diy * qkz - diz * qky + dky * qiz - dkz * qiy -
                             2.0 * (qixy * qkxz + qiyy * qkyz + qiyz * qkzz - qixz * qkxy - qiyz * qkyy - qizz * qkyz);
        const double dqiky = diz * qkx - dix * qkz + dkz * qix - dkx * qiz -
                             2.0 * (qixz * qkxx + qiyz * qkxy + qizz * qkxz - qixx * qkxz - qixy * qkyz - qixz * qkzz);
        const double dqikz = dix * qky - diy * qkx + dkx * qiy - dky * qix -
                             2.0 * (qixx * qkxy + qixy * qkyy + qixz * qkyz - qixy * qkxx - qiyy * qkxy - qiyz * qkxz);
        // reciprocal distance terms and the Ewald damping (dampewald order 11)
        double rr1 = f / r;
        double rr3 = rr1 / r2;
        double rr5 = 3.0 * rr3 / r2;
        double rr7 = 5.0 * rr5 / r2;
        double rr9 = 7.0 * rr7 / r2;
        double rr11 = 9.0 * rr9 / r2;
        double dmpe[12];
        dampewald(11, r, r2, f, s.aewald, dmpe);
        const double term1 = ci * ck;
        const double term2 = ck * dir - ci * dkr + dik;
        const double term3 = ci * qkr + ck * qir - dir * dkr + 2.0 * (dkqi - diqk + qiqk);
        const double term4 = dir * qkr - dkr * qir - 4.0 * qik;
        const double term5 = qir * qkr;
        const double scalek = 1.0 - mscale[k];
        rr1 = dmpe[1] - scalek * rr1;
        rr3 = dmpe[3] - scalek * rr3;
        rr5 = dmpe[5] - scalek * rr5;
        rr7 = dmpe[7] - scalek * rr7;
        rr9 = dmpe[9] - scalek * rr9;
        rr11 = dmpe[11] - scalek * rr11;
        const double e = term1 * rr1 + term2 * rr3 + term3 * rr5 + term4 * rr7 + term5 * rr9;
        const double de = term1 * rr3 + term2 * rr5 + term3 * rr7 + term4 * rr9 + term5 * rr11;
        const double t1 = -ck * rr3 + dkr * rr5 - qkr * rr7;
        const double t2 = ci * rr3 + dir * rr5 + qir * rr7;
        const double t3 = 2.0 * rr5;
        const double t4 = -2.0 * (ck * rr5 - dkr * rr7 + qkr * rr9);
        const double t5 = -2.0 * (ci * rr5 + dir * rr7 + qir * rr9);
        const double t6 = 4.0 * rr7;
        ereal += e;
        const double frcx = de * xr + t1 * dix + t2 * dkx + t3 * (diqkx - dkqix) + t4 * qix + t5 * qkx +
                            t6 * (qixk + qkxi);
        const double frcy = de * yr + t1 * diy + t2 * dky + t3 * (diqky - dkqiy) + t4 * qiy + t5 * qky +
                            t6 * (qiyk + qkyi);
        const double frcz = de * zr + t1 * diz + t2 * dkz + t3 * (diqkz - dkqiz) + t4 * qiz + t5 * qkz +
                            t6 * (qizk + qkzi);
        tem[i * 3 + 0] += -rr3 * dikx + t1 * dirx + t3 * (dqikx + dkqirx) - t4 * qirx - t6 * (qikrx + qikx);
        tem[i * 3 + 1] += -rr3 * diky + t1 * diry + t3 * (dqiky + dkqiry) - t4 * qiry - t6 * (qikry + qiky);
        tem[i * 3 + 2] += -rr3 * dikz + t1 * dirz + t3 * (dqikz + dkqirz) - t4 * qirz - t6 * (qikrz + qikz);
        tem[k * 3 + 0] += rr3 * dikx + t2 * dkrx - t3 * (dqikx + diqkrx) - t5 * qkrx - t6 * (qkirx - qikx);
        tem[k * 3 + 1] += rr3 * diky + t2 * dkry - t3 * (dqiky + diqkry) - t5 * qkry - t6 * (qkiry - qiky);
        tem[k * 3 + 2] += rr3 * dikz + t2 * dkrz - t3 * (dqikz + diqkrz) - t5 * qkrz - t6 * (qkirz - qikz);
        dem[i * 3 + 0] += frcx;
        dem[i * 3 + 1] += frcy;
        dem[i * 3 + 2] += frcz;
        dem[k * 3 + 0] -= frcx;
        dem[k * 3 + 1] -= frcy;
        dem[k * 3 + 2] -= frcz;
        // the virial of the pairwise Cartesian forces (empole1.f:1428-1442)
        vir.add(-xr * frcx, -0.5 * (yr * frcx + xr * frcy), -0.5 * (zr * frcx + xr * frcz), -yr * frcy,
                -0.5 * (zr * frcy + yr * frcz), -zr * frcz);
      }
      for (int b = 0; b < 4; ++b) for_conn(s, mslot[b], i, [&](int k) { mscale[k] = 1.0; });
    }
    for (int i = 0; i < n; ++i) {
      double fz[3], fx[3];
      torque_site(s.x, s.y, s.z, i, zaxis[i], xaxis[i], axt[i], &tem[(size_t)i * 3], dem, fz, fx);
      // the virial of the torque's frame-atom forces (empole1.f:1466-1497)
      frame_virial(s.x, s.y, s.z, i, zaxis[i], xaxis[i], fz, fx, vir);
    }
  }
  // ---- self energy (empole1.f:134-160) -------------------------------------
  {
    const double term = 2.0 * s.aewald * s.aewald;
    const double fterm = -f * s.aewald / kSqrtPi;
    for (int i = 0; i < n; ++i) {
      const double* rp = &s.rpole[(size_t)i * 13];
      const double ci = rp[0], dix = rp[1], diy = rp[2], diz = rp[3];
      const double qixx = rp[4], qixy = rp[5], qixz = rp[6], qiyy = rp[8], qiyz = rp[9], qizz = rp[12];
      const double cii = ci * ci;
      const double dii = dix * dix + diy * diy + diz * diz;
      const double qii = 2.0 * (qixy * qixy + qixz * qixz + qiyz * qiyz) + qixx * qixx + qiyy * qiyy + qizz * qizz;
      eself += fterm * (cii + term * (dii / 3.0 + 2.0 * term * qii / 5.0));
    }
  }
  if (parts) {
    parts[0] = ereal + erecip + eself;
    parts[1] = ereal;
    parts[2] = erecip;
    parts[3] = eself;
  }
  if (vir_out) vir.out(vir_out);
  if (vir_frame) vframe.out(vir_frame);
  return OR_OK;
}

// ===========================================================================
// van der Waals: ehal1c (ehal1.f:69-482, standard branch) over the list of
// vlistcell (nblist.f:1148-1305).  The list is restated as every pair k > i
// whose reduced minimum-image distance is within vdwcut + lbuffer (the
// reference finds the same pairs through its cells); the energy loop then
// applies r <= vdwcut and the taper above vdwtaper.
int or_ehal1(OrCtx* c, const OrVdw* v, double* dev, double* ev_out, double* vir_out) {
  const OrSystem& s = c->s;
  const int n = s.n;
  std::fill(dev, dev + (size_t)n * 3, 0.0);
  Vir vir;
  const double vbuf = v->vdwcut + s.lbuffer;
  if (vbuf > 0.5 * std::min(s.xbox, std::min(s.ybox, s.zbox))) return OR_E_BOX_TOO_SMALL;
  // reduced coordinates (ehal1.f:193-205)
  std::vector<double> xr((size_t)n), yr((size_t)n), zr((size_t)n);
  for (int i = 0; i < n; ++i) {
    const int iv = v->ired[i];
    const double rdn = v->kred[i];
    xr[i] = rdn * (s.x[i] - s.x[iv]) + s.x[iv];
    yr[i] = rdn * (s.y[i] - s.y[iv]) + s.y[iv];
    zr[i] = rdn * (s.z[i] - s.z[iv]) + s.z[iv];
  }
  // switch.f:80-117 (mode VDW): off = vdwcut, cut = vdwtaper
  const double off = v->vdwcut, cut = v->vdwtaper;
  const double off2 = off * off, cut2 = cut * cut;
  double c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0;
  if (cut < off) {
    const double denom = std::pow(off - cut, 5);
    c0 = off * off2 * (off2 - 5.0 * off * cut + 10.0 * cut2) / denom;
    c1 = -30.0 * off2 * cut2 / denom;
    c2 = 30.0 * (off2 * cut + off * cut2) / denom;
    c3 = -10.0 * (off2 + 4.0 * off * cut + cut2) / denom;
    c4 = 15.0 * (off + cut) / denom;
    c5 = -6.0 / denom;
  }
  const double ghal = v->ghal, dhal = v->dhal;
  const int nc = v->nclass;
  std::vector<double> vscale((size_t)n, 1.0);
  std::vector<int> iv14((size_t)n, -1);
  const int slot[4] = {OR_I12, OR_I13, OR_I14, OR_I15};
  double ev = 0.0;
  auto vdw_site = [&](int a) { return v->radmin[v->cls[a] * nc + v->cls[a]] != 0.0; };  // kvdw.f:592-598
  for (int i = 0; i < n; ++i) {
    const int iv = v->ired[i];
    const double redi = v->kred[i], rediv = 1.0 - redi;
    const int it = v->cls[i];
    if (!vdw_site(i)) continue;
    for (int b = 0; b < 4; ++b)
      for_conn(s, slot[b], i, [&](int k) {
        vscale[k] = v->v_scale[b];
        if (b == 2) iv14[k] = i;
      });
    for (int k = i + 1; k < n; ++k) {
      if (!vdw_site(k)) continue;  // vlistcell skips partners without a radius
      double xd = xr[i] - xr[k], yd = yr[i] - yr[k], zd = zr[i] - zr[k];
      image(c->cell, xd, yd, zd);
      const double rik2 = xd * xd + yd * yd + zd * zd;
      if (rik2 > vbuf * vbuf) continue;  // not in the list
      if (!(rik2 <= off2)) continue;
      const int kv = v->ired[k];
      const double redk = v->kred[k], redkv = 1.0 - redk;
      const int kt = v->cls[k];
      const double rik = std::sqrt(rik2);
      double rv = v->radmin[kt * nc + it];
      double eps = v->eps[kt * nc + it];
      if (iv14[k] == i) {
        rv = v->radmin4[kt * nc + it];
        eps = v->eps4[kt * nc + it];
      }
      eps = eps * vscale[k];
      const double rv7 = std::pow(rv, 7);
      const double rik6 = rik2 * rik2 * rik2;
      const double rik7 = rik6 * rik;
      const double rho = rik7 + ghal * rv7;
      const double tau = (dhal + 1.0) / (rik + dhal * rv);
      const double tau7 = std::pow(tau, 7);
      const double dtau = tau / (dhal + 1.0);
      const double gtau = eps * tau7 * rik6 * (ghal + 1.0) * (rv7 / rho) * (rv7 / rho);
      double e = eps * tau7 * rv7 * ((ghal + 1.0) * rv7 / rho - 2.0);
      double de = -7.0 * (dtau * e + gtau);
      if (rik2 > cut2) {
        const double rik3 = rik2 * rik, rik4 = rik2 * rik2, rik5 = rik2 * rik3;
        const double taper = c5 * rik5 + c4 * rik4 + c3 * rik3 + c2 * rik2 + c1 * rik + c0;
        const double dtaper = 5.0 * c5 * rik4 + 4.0 * c4 * rik3 + 3.0 * c3 * rik2 + 2.0 * c2 * rik + c1;
        de = e * dtaper + de * taper;
        e = e * taper;
      }
      ev += e;
      de = de / rik;
      const double dedx = de * xd, dedy = de * yd, dedz = de * zd;
      // the virial of the pair (ehal1.f:431-446), reduced-site separation
      vir.add(xd * dedx, yd * dedx, zd * dedx, yd * dedy, zd * dedy, zd * dedz);
      if (i == iv) {
        dev[i * 3 + 0] += dedx;
        dev[i * 3 + 1] += dedy;
        dev[i * 3 + 2] += dedz;
      } else {
        dev[i * 3 + 0] += dedx * redi;
        dev[i * 3 + 1] += dedy * redi;
        dev[i * 3 + 2] += dedz * redi;
        dev[iv * 3 + 0] += dedx * rediv;
        dev[iv * 3 + 1] += dedy * rediv;
        dev[iv * 3 + 2] += dedz * rediv;
      }
      if (k == kv) {
        dev[k * 3 + 0] -= dedx;
        dev[k * 3 + 1] -= dedy;
        dev[k * 3 + 2] -= dedz;
      } else {
        dev[k * 3 + 0] -= dedx * redk;
        dev[k * 3 + 1] -= dedy * redk;
        dev[k * 3 + 2] -= dedz * redk;
        dev[kv * 3 + 0] -= dedx * redkv;
        dev[kv * 3 + 1] -= dedy * redkv;
        dev[kv * 3 + 2] -= dedz * redkv;
      }
    }
    for (int b = 0; b < 4; ++b) for_conn(s, slot[b], i, [&](int k) { vscale[k] = 1.0; });
  }
  if (vir_out) vir.out(vir_out);
  if (ev_out) *ev_out = ev;
  return OR_OK;
}

}  // extern "C"
