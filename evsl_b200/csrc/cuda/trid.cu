// Eigenvalues of a symmetric tridiagonal matrix on the GPU, for the
// convergence tests of the filtered Lanczos solvers (the trace test of
// ChebLanNr, SRC/cheblanNr.c:241-262, needs every eigenvalue of T_k every
// 20 steps; the reference calls LAPACK dstev there).
//
// Multisection on Sturm counts: one warp per eigenvalue index i; each round
// the warp evaluates the count of eigenvalues below 128 equally spaced
// shifts of its bracket (4 per lane, their recurrences interleaved) and keeps
// the sub-interval where the count passes i, shrinking the bracket 129-fold.
// The bracket [lo, hi] always satisfies count(lo) <= i < count(hi), whatever
// the rounding of the counts, so the result lies within the final bracket
// of the computed spectrum.  Rounds stop at a relative width of 2 eps or
// after kRounds (bounded).  The count uses the LDL^T recurrence
// q_j = (d_j - x) - e_{j-1}^2 / q_{j-1} with tiny pivots replaced by -pivmin.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace evslcu {
namespace {

constexpr int kPts = 4;                   // shifts per lane
constexpr int kShifts = 32 * kPts;        // shifts per round
constexpr int kSections = kShifts + 1;    // sub-intervals per round
constexpr int kRounds = 12;               // 129^12 > 2e25
constexpr int kTridThreads = 256;

__global__ void __launch_bounds__(kTridThreads)
    k_trid_bisect(int k, int i0, const double *__restrict__ d, const double *__restrict__ e2, double glo,
                  double ghi, double pivmin, double *__restrict__ w) {
  const int lane = threadIdx.x & 31;
  const int i = i0 + (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (i >= k) return;  // uniform over the warp
  double lo = glo, hi = ghi;
  for (int round = 0; round < kRounds; ++round) {
    const double width = hi - lo;
    if (width <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin) break;
    double x[kPts], q[kPts];
    int c[kPts];
#pragma unroll
    for (int p = 0; p < kPts; ++p) {
      x[p] = lo + width * (double)(lane * kPts + p + 1) / (double)kSections;
      q[p] = __ldg(d) - x[p];
      if (fabs(q[p]) < pivmin) q[p] = -pivmin;
      c[p] = q[p] < 0.0;
    }
    for (int j = 1; j < k; ++j) {
      const double dj = __ldg(d + j), ej = __ldg(e2 + j - 1);
#pragma unroll
      for (int p = 0; p < kPts; ++p) {
        q[p] = (dj - x[p]) - ej / q[p];
        if (fabs(q[p]) < pivmin) q[p] = -pivmin;
        c[p] += q[p] < 0.0;
      }
    }
    // first shift whose count exceeds i
    int first = kShifts;
#pragma unroll
    for (int p = kPts - 1; p >= 0; --p)
      if (c[p] > i) first = lane * kPts + p;
    first = __reduce_min_sync(0xffffffffu, first);
    const double nlo = (first == 0) ? lo : lo + width * (double)first / (double)kSections;
    const double nhi = (first == kShifts) ? hi : lo + width * (double)(first + 1) / (double)kSections;
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) w[i] = 0.5 * (lo + hi);
}

double *g_trid_buf = nullptr;
int g_trid_cap = 0;

}  // namespace
}  // namespace evslcu

using namespace evslcu;

extern "C" {

void evslcu_trid_release(void) {
  evslcu_free(g_trid_buf);
  g_trid_buf = nullptr;
  g_trid_cap = 0;
}

int evslcu_trid_eigvals_above(int k, const double *d, const double *e, double xmin, double *w) {
  if (k <= 0) return 0;
  if (!d || !w || (k > 1 && !e)) return fail(EVSLCU_ERR_ARG, "evslcu_trid_eigvals: bad arguments");
  if (k > g_trid_cap) {
    evslcu_free(g_trid_buf);
    g_trid_cap = std::max(k, 1024);
    g_trid_buf = (double *)evslcu_malloc(sizeof(double) * 3 * (size_t)g_trid_cap);
    if (!g_trid_buf) {
      g_trid_cap = 0;
      return fail(EVSLCU_ERR_NOMEM, "tridiagonal eigenvalues: out of device memory");
    }
  }
  // squared off-diagonals, Gershgorin interval and the pivot floor
  std::vector<double> e2((size_t)std::max(k - 1, 1), 0.0);
  double emax = 0.0, glo = d[0], ghi = d[0];
  for (int j = 0; j < k; ++j) {
    const double ej = (j + 1 < k) ? fabs(e[j]) : 0.0;
    const double ejm = (j > 0) ? fabs(e[j - 1]) : 0.0;
    glo = std::min(glo, d[j] - ej - ejm);
    ghi = std::max(ghi, d[j] + ej + ejm);
    if (j + 1 < k) {
      e2[j] = e[j] * e[j];
      emax = std::max(emax, e2[j]);
    }
  }
  const double pivmin = DBL_MIN * std::max(1.0, emax);
  const double fudge = 2.0 * DBL_EPSILON * std::max(fabs(glo), fabs(ghi)) * k + 2.0 * pivmin;
  glo -= fudge;
  ghi += fudge;
  // Indices below i0 are skipped: their eigenvalues lie below xc, far
  // enough under xmin (1e-8 of the spectral scale, four orders above the
  // counts' rounding) that none of them can reach xmin.  One index of slack
  // on top.  The others are bisected from the same bracket as in the full
  // computation, so they come out bit for bit the same.
  int i0 = 0;
  if (xmin > glo) {
    const double xc = xmin - 1e-8 * std::max(1.0, std::max(fabs(glo), fabs(ghi)));
    double q = d[0] - xc;
    if (fabs(q) < pivmin) q = -pivmin;
    int cnt = q < 0.0;
    for (int j = 1; j < k; ++j) {
      q = (d[j] - xc) - e2[j - 1] / q;
      if (fabs(q) < pivmin) q = -pivmin;
      cnt += q < 0.0;
    }
    i0 = std::max(0, cnt - 1);
  }
  double *dd = g_trid_buf, *de2 = g_trid_buf + g_trid_cap, *dw = g_trid_buf + 2 * (size_t)g_trid_cap;
  int rc = evslcu_h2d_async(dd, d, sizeof(double) * (size_t)k);
  if (!rc && k > 1) rc = evslcu_h2d_async(de2, e2.data(), sizeof(double) * (size_t)(k - 1));
  if (rc) return rc;
  if (i0 < k) {
    const long long threads = 32LL * (k - i0);
    const int grid = (int)((threads + kTridThreads - 1) / kTridThreads);
    k_trid_bisect<<<grid, kTridThreads, 0, stream()>>>(k, i0, dd, de2, glo, ghi, pivmin, dw);
    count_launch();
    if ((rc = check_launch("k_trid_bisect"))) return rc;
    if ((rc = evslcu_d2h(w + i0, dw + i0, sizeof(double) * (size_t)(k - i0)))) return rc;
  }
  for (int i = 0; i < i0; ++i) w[i] = glo;  // below every computed eigenvalue and below xmin
  std::sort(w, w + k);
  return 0;
}

int evslcu_trid_eigvals(int k, const double *d, const double *e, double *w) {
  return evslcu_trid_eigvals_above(k, d, e, -HUGE_VAL, w);
}

}  // extern "C"
