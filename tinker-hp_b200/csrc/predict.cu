// predict.cu -- induced-dipole predictor for dynamics (ulspred,
// newinduce_pme2.f:160-180, 250-265, 910-1010).
//
// The last seven solutions (uind, uinp) are kept in ORIGINAL atom order, so a
// re-sort of the atoms never touches them.  Once seven are stored the guess
// is mu = sum_k b_k alt_k over the six most recent, with the ASPC or Gear
// constants or least-squares coefficients fitted on the stored history.
#include <cmath>
#include <vector>

#include "kernels.h"

namespace thp {

namespace {

constexpr int kBlock = 256;

struct PredCoef {
  double bd[kMaxAlt], bp[kMaxAlt];  // coefficients of the d and p dipoles, newest first
  int slot[kMaxAlt];                 // ring slot of the k-th newest solution
  int m;                             // number of terms
};

// mu (sorted) = sum_k b_k alt_k (original order)
__global__ void k_predict(int n, PredCoef pc, const double* __restrict__ alt, const int* __restrict__ iperm,
                          double* __restrict__ mu) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int k = 0; k < pc.m; ++k) {
    const double* a = alt + ((size_t)pc.slot[k] * n + o) * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] += (q < 3 ? pc.bd[k] : pc.bp[k]) * a[q];
  }
  double* out = mu + (size_t)iperm[o] * 6;
#pragma unroll
  for (int q = 0; q < 6; ++q) out[q] = v[q];
}

// partial dot products <alt_k, alt_l> (k <= l) of the d and p dipoles, one
// row of 2 * kPairs values per block, summed on the host in block order
constexpr int kPairs = kMaxAlt * (kMaxAlt + 1) / 2;

__global__ void __launch_bounds__(kBlock) k_alt_dots(int n, PredCoef pc, const double* __restrict__ alt,
                                                     double* __restrict__ partial) {
  double v[2 * kPairs];
#pragma unroll
  for (int q = 0; q < 2 * kPairs; ++q) v[q] = 0.0;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < n) {
    double a[kMaxAlt][6];
#pragma unroll
    for (int k = 0; k < kMaxAlt; ++k)
#pragma unroll
      for (int q = 0; q < 6; ++q) a[k][q] = alt[((size_t)pc.slot[k] * n + o) * 6 + q];
    int t = 0;
#pragma unroll
    for (int k = 0; k < kMaxAlt; ++k)
#pragma unroll
      for (int l = k; l < kMaxAlt; ++l, ++t) {
        v[t] = a[k][0] * a[l][0] + a[k][1] * a[l][1] + a[k][2] * a[l][2];
        v[kPairs + t] = a[k][3] * a[l][3] + a[k][4] * a[l][4] + a[k][5] * a[l][5];
      }
  }
  block_reduce<2 * kPairs>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 2 * kPairs; ++q) partial[(size_t)blockIdx.x * 2 * kPairs + q] = v[q];
}

// Solves the symmetric positive definite system a x = b (dimension k, a
// dense k x k) by Cholesky factorisation; leaves b unchanged when a is not
// positive definite.
void spd_solve(int k, double a[kMaxAlt][kMaxAlt], double b[kMaxAlt]) {
  double l[kMaxAlt][kMaxAlt] = {};
  for (int i = 0; i < k; ++i) {
    for (int j = 0; j <= i; ++j) {
      double s = a[i][j];
      for (int q = 0; q < j; ++q) s -= l[i][q] * l[j][q];
      if (i == j) {
        if (!(s > 0.0)) return;
        l[i][i] = sqrt(s);
      } else {
        l[i][j] = s / l[j][j];
      }
    }
  }
  double y[kMaxAlt];
  for (int i = 0; i < k; ++i) {
    double s = b[i];
    for (int q = 0; q < i; ++q) s -= l[i][q] * y[q];
    y[i] = s / l[i][i];
  }
  for (int i = k - 1; i >= 0; --i) {
    double s = y[i];
    for (int q = i + 1; q < k; ++q) s -= l[q][i] * b[q];
    b[i] = s / l[i][i];
  }
}

// kpolar.f:405-425
constexpr double kGear[kMaxAlt] = {6.0, -15.0, 20.0, -15.0, 6.0, -1.0, 0.0};
constexpr double kAspc[kMaxAlt] = {22.0 / 7.0, -55.0 / 14.0, 55.0 / 21.0, -22.0 / 21.0, 5.0 / 21.0, -1.0 / 42.0, 0.0};

}  // namespace

int predictor_alloc(Ctx& c) {
  if (c.d_alt && c.alt_cap >= (size_t)c.n) return THP_OK;
  cudaFree(c.d_alt);
  c.d_alt = nullptr;
  c.alt_cap = 0;
  int st = cuda_status(cudaMalloc((void**)&c.d_alt, sizeof(double) * kMaxAlt * 6 * (size_t)c.n), &c, "alloc alt");
  if (!st) c.alt_cap = c.n;
  return st;
}

// The sorted dipoles in d_mu become the newest stored solution
// (newinduce_pme2.f:252-265).
int predictor_push(Ctx& c) {
  if (!c.pred_mode) return THP_OK;
  int st = predictor_alloc(c);
  if (st) return st;
  c.alt_head = (c.alt_head + 1) % kMaxAlt;
  c.nualt = c.nualt < kMaxAlt ? c.nualt + 1 : kMaxAlt;
  return launch_to_orig6(c, c.d_mu, c.d_alt + (size_t)c.alt_head * 6 * c.n, 2);
}

// Writes the predicted dipoles into d_mu (sorted) when seven solutions are
// stored; returns -1 (nothing written) otherwise.
int predictor_guess(Ctx& c) {
  if (!c.pred_mode || c.nualt < kMaxAlt || !c.d_alt) return -1;
  PredCoef pc{};
  pc.m = kMaxAlt - 1;
  for (int k = 0; k < kMaxAlt; ++k) pc.slot[k] = ((c.alt_head - k) % kMaxAlt + kMaxAlt) % kMaxAlt;
  const int nb = (c.n + kBlock - 1) / kBlock;
  if (c.pred_mode == THP_PRED_ASPC || c.pred_mode == THP_PRED_GEAR) {
    const double* b = c.pred_mode == THP_PRED_ASPC ? kAspc : kGear;
    for (int k = 0; k < kMaxAlt; ++k) pc.bd[k] = pc.bp[k] = b[k];
  } else {
    // least-squares fit (ulspred, newinduce_pme2.f:950-1008): the newest
    // solution from the six before it; the same weights then extrapolate
    const int m = kMaxAlt;
    const size_t rows = 2 * kPairs;
    std::vector<double> part((size_t)nb * rows);
    double* d_part = nullptr;
    int st = cuda_status(cudaMalloc((void**)&d_part, sizeof(double) * part.size()), &c, "alt dots");
    if (st) return st;
    k_alt_dots<<<nb, kBlock, 0, c.stream>>>(c.n, pc, c.d_alt, d_part);
    cudaMemcpyAsync(part.data(), d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, c.stream);
    st = cuda_status(cudaStreamSynchronize(c.stream), &c, "alt dots");
    cudaFree(d_part);
    if (st) return st;
    double cd[kMaxAlt][kMaxAlt] = {}, cp[kMaxAlt][kMaxAlt] = {};
    for (int blk = 0; blk < nb; ++blk) {
      int t = 0;
      for (int k = 0; k < m; ++k)
        for (int l = k; l < m; ++l, ++t) {
          cd[k][l] += part[(size_t)blk * rows + t];
          cp[k][l] += part[(size_t)blk * rows + kPairs + t];
        }
    }
    double ad[kMaxAlt][kMaxAlt] = {}, ap[kMaxAlt][kMaxAlt] = {}, bd[kMaxAlt] = {}, bp[kMaxAlt] = {};
    const int k1 = m - 1;
    for (int k = 1; k < m; ++k) {
      bd[k - 1] = cd[0][k];
      bp[k - 1] = cp[0][k];
      for (int l = k; l < m; ++l) {
        ad[k - 1][l - 1] = ad[l - 1][k - 1] = cd[k][l];
        ap[k - 1][l - 1] = ap[l - 1][k - 1] = cp[k][l];
      }
    }
    spd_solve(k1, ad, bd);
    spd_solve(k1, ap, bp);
    for (int k = 0; k < k1; ++k) {
      pc.bd[k] = bd[k];
      pc.bp[k] = bp[k];
    }
  }
  k_predict<<<nb, kBlock, 0, c.stream>>>(c.n, pc, c.d_alt, c.d_iperm, c.d_mu);
  return cuda_status(cudaGetLastError(), &c, "predict");
}

}  // namespace thp
