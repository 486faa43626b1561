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
#include <cstring>
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

// Side-stream form for the convergence tests: inputs staged in pinned host
// memory, the bisection on its own stream, the result copied back
// asynchronously; the solver reads it when it needs it.
cudaStream_t g_side = nullptr;
cudaEvent_t g_main_mark = nullptr, g_side_done = nullptr;
double *g_pin = nullptr;  // pinned: d | e2 | w, g_pin_cap each
int g_pin_cap = 0;
struct {
  bool pending;
  int k, i0;
  double glo;
} g_async = {false, 0, 0, 0.0};

// Gershgorin interval (widened), pivot floor, squared off-diagonals (into
// e2[0..k-1)) and the first index that may reach xmin (see below).
struct TridPrep {
  double glo, ghi, pivmin;
  int i0;
};

TridPrep trid_prep(int k, const double *d, const double *e, double xmin, double *e2) {
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
  return {glo, ghi, pivmin, i0};
}

int trid_device_buffers(int k) {
  if (k <= g_trid_cap) return 0;
  evslcu_free(g_trid_buf);
  g_trid_cap = std::max(k, 1024);
  g_trid_buf = (double *)evslcu_malloc(sizeof(double) * 3 * (size_t)g_trid_cap);
  if (!g_trid_buf) {
    g_trid_cap = 0;
    return fail(EVSLCU_ERR_NOMEM, "tridiagonal eigenvalues: out of device memory");
  }
  return 0;
}

int trid_launch(int k, const TridPrep &p, cudaStream_t st) {
  if (p.i0 >= k) return 0;
  double *dd = g_trid_buf, *de2 = g_trid_buf + g_trid_cap, *dw = g_trid_buf + 2 * (size_t)g_trid_cap;
  const long long threads = 32LL * (k - p.i0);
  const int grid = (int)((threads + kTridThreads - 1) / kTridThreads);
  k_trid_bisect<<<grid, kTridThreads, 0, st>>>(k, p.i0, dd, de2, p.glo, p.ghi, p.pivmin, dw);
  count_launch();
  return check_launch("k_trid_bisect");
}

}  // namespace
}  // namespace evslcu

using namespace evslcu;

extern "C" {

void evslcu_trid_release(void) {
  if (g_async.pending) {
    cudaEventSynchronize(g_side_done);
    g_async.pending = false;
  }
  evslcu_free(g_trid_buf);
  g_trid_buf = nullptr;
  g_trid_cap = 0;
  if (g_pin) cudaFreeHost(g_pin);
  g_pin = nullptr;
  g_pin_cap = 0;
  if (g_side) {
    cudaStreamDestroy(g_side);
    cudaEventDestroy(g_main_mark);
    cudaEventDestroy(g_side_done);
    g_side = nullptr;
    g_main_mark = g_side_done = nullptr;
  }
}

int evslcu_trid_eigvals_above(int k, const double *d, const double *e, double xmin, double *w) {
  if (k <= 0) return 0;
  if (!d || !w || (k > 1 && !e)) return fail(EVSLCU_ERR_ARG, "evslcu_trid_eigvals: bad arguments");
  // a side-stream test still reading the device buffers goes first
  if (g_async.pending) EVSLCU_CUDA(cudaStreamWaitEvent(stream(), g_side_done, 0));
  int rc = trid_device_buffers(k);
  if (rc) return rc;
  std::vector<double> e2((size_t)std::max(k - 1, 1), 0.0);
  const TridPrep p = trid_prep(k, d, e, xmin, e2.data());
  double *dd = g_trid_buf, *de2 = g_trid_buf + g_trid_cap, *dw = g_trid_buf + 2 * (size_t)g_trid_cap;
  rc = evslcu_h2d_async(dd, d, sizeof(double) * (size_t)k);
  if (!rc && k > 1) rc = evslcu_h2d_async(de2, e2.data(), sizeof(double) * (size_t)(k - 1));
  if (!rc) rc = trid_launch(k, p, stream());
  if (!rc && p.i0 < k) rc = evslcu_d2h(w + p.i0, dw + p.i0, sizeof(double) * (size_t)(k - p.i0));
  if (rc) return rc;
  for (int i = 0; i < p.i0; ++i) w[i] = p.glo;  // below every computed eigenvalue and below xmin
  std::sort(w, w + k);
  return 0;
}

int evslcu_trid_eigvals_async(int k, const double *d, const double *e, double xmin) {
  if (k <= 0 || !d || (k > 1 && !e)) return fail(EVSLCU_ERR_ARG, "evslcu_trid_eigvals_async: bad arguments");
  if (g_async.pending) return fail(EVSLCU_ERR_ARG, "evslcu_trid_eigvals_async: a test is still in flight");
  if (!g_side) {
    EVSLCU_CUDA(cudaStreamCreateWithFlags(&g_side, cudaStreamNonBlocking));
    EVSLCU_CUDA(cudaEventCreateWithFlags(&g_main_mark, cudaEventDisableTiming));
    EVSLCU_CUDA(cudaEventCreateWithFlags(&g_side_done, cudaEventDisableTiming));
  }
  if (k > g_pin_cap) {
    if (g_pin) cudaFreeHost(g_pin);
    g_pin = nullptr;
    const int cap = std::max(k, 2 * g_pin_cap);
    EVSLCU_CUDA(cudaMallocHost(&g_pin, sizeof(double) * 3 * (size_t)cap));
    g_pin_cap = cap;
  }
  int rc = trid_device_buffers(k);
  if (rc) return rc;
  double *pd = g_pin, *pe2 = g_pin + g_pin_cap, *pw = g_pin + 2 * (size_t)g_pin_cap;
  memcpy(pd, d, sizeof(double) * (size_t)k);
  const TridPrep p = trid_prep(k, d, e, xmin, pe2);
  double *dd = g_trid_buf, *de2 = g_trid_buf + g_trid_cap, *dw = g_trid_buf + 2 * (size_t)g_trid_cap;
  // the device buffers come from the library stream's pool: order the side
  // stream after it
  EVSLCU_CUDA(cudaEventRecord(g_main_mark, stream()));
  EVSLCU_CUDA(cudaStreamWaitEvent(g_side, g_main_mark, 0));
  EVSLCU_CUDA(cudaMemcpyAsync(dd, pd, sizeof(double) * (size_t)k, cudaMemcpyHostToDevice, g_side));
  if (k > 1) EVSLCU_CUDA(cudaMemcpyAsync(de2, pe2, sizeof(double) * (size_t)(k - 1), cudaMemcpyHostToDevice, g_side));
  if ((rc = trid_launch(k, p, g_side))) return rc;
  if (p.i0 < k)
    EVSLCU_CUDA(cudaMemcpyAsync(pw + p.i0, dw + p.i0, sizeof(double) * (size_t)(k - p.i0), cudaMemcpyDeviceToHost,
                                g_side));
  EVSLCU_CUDA(cudaEventRecord(g_side_done, g_side));
  g_async = {true, k, p.i0, p.glo};
  return 0;
}

int evslcu_trid_eigvals_async_ready(void) {
  if (!g_async.pending) return 1;
  const cudaError_t e = cudaEventQuery(g_side_done);
  if (e == cudaErrorNotReady) return 0;
  return 1;  // finished, or failed: the wait reports the error
}

int evslcu_trid_eigvals_async_wait(double *w) {
  if (!g_async.pending) return fail(EVSLCU_ERR_ARG, "evslcu_trid_eigvals_async_wait: no test in flight");
  g_async.pending = false;
  EVSLCU_CUDA(cudaEventSynchronize(g_side_done));
  const int k = g_async.k, i0 = g_async.i0;
  const double *pw = g_pin + 2 * (size_t)g_pin_cap;
  if (i0 < k) memcpy(w + i0, pw + i0, sizeof(double) * (size_t)(k - i0));
  for (int i = 0; i < i0; ++i) w[i] = g_async.glo;
  std::sort(w, w + k);
  return 0;
}

int evslcu_trid_eigvals(int k, const double *d, const double *e, double *w) {
  return evslcu_trid_eigvals_above(k, d, e, -HUGE_VAL, w);
}

}  // extern "C"
