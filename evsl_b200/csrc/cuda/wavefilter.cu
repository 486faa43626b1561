// Pipelined ("wavefront") Chebyshev filter: all degrees of one filter
// application in one launch, without a grid-wide barrier between degrees.
//
// Rows are cut into tiles of kWaveRows rows.  Work items (step s, tile t),
// s = 1..deg, are handed out in the order s*T + t by an atomic counter.
// Step s at tile t needs the vector of step s-1 at the rows its stored
// entries reach: the tiles within delta = ceil(bandwidth / kWaveRows) of t.
// It waits until those tiles have published step s-1 (done[t'] >= s-1),
// computes its rows exactly as k_cheb does (same rounded operations, same
// order, so results are bitwise those of the per-degree path) and publishes
// done[t] = s.  Two rotating vectors suffice: step s overwrites the vector of
// step s-2, whose other readers (step s-1 at the neighbouring tiles) it has
// just waited for.
//
// Progress: an item only waits for items handed out before it, and every
// handed-out item belongs to a running block, so the pipeline cannot
// deadlock whatever the number of resident blocks.  Every wait is bounded;
// a wait that gives up raises an abort flag that stops all blocks, and the
// host reports EVSLCU_ERR_TIMEOUT.  Data written during the launch is read
// through L2 only (ld.global.cg); publication is a release store after a
// fence, observation an acquire load.
#include <algorithm>

#include "common.cuh"
#include "sparse_types.cuh"

namespace evslcu {

namespace {

constexpr int kWaveThreads = 256;
constexpr int kWaveRows = 2048;  // rows per tile (8 per thread)
constexpr unsigned kWaveSpinLimit = 1u << 22;
unsigned g_wave_polls = kWaveSpinLimit;  // polls per dependency wait

struct WaveArgs {
  int n, T, delta, deg;
  const double *mu;  // device copy of mu[0..deg]
  double t1, t2, ncc;
  const double *v;
  double *y;
  double *B0, *B1;
  unsigned long long *next;  // work-item counter
  unsigned *abort_flag;
  int *err;
  unsigned *done;  // done[t] = last step published for tile t
  unsigned polls;  // dependency wait limit
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <class VT, class IT>
__global__ void __launch_bounds__(kWaveThreads) k_filter_wave(SellT<VT, IT> A, WaveArgs P) {
  __shared__ unsigned long long sh_item;
  __shared__ int sh_stop;
  const unsigned long long total = (unsigned long long)P.deg * (unsigned long long)P.T;
  for (;;) {
    if (threadIdx.x == 0) {
      sh_stop = *(volatile unsigned *)P.abort_flag ? 1 : 0;
      sh_item = sh_stop ? total : atomicAdd(P.next, 1ull);
    }
    __syncthreads();
    const unsigned long long item = sh_item;
    if (item >= total) break;
    const int s = (int)(item / P.T) + 1;
    const int t = (int)(item % P.T);
    // wait for step s-1 on the tiles this tile's rows reach
    if (s > 1 && threadIdx.x < 32) {
      const int lo = max(0, t - P.delta), hi = min(P.T - 1, t + P.delta);
      int ok = 1;
      for (int base = lo; base <= hi && ok; base += 32) {
        const int tt = base + (int)threadIdx.x;
        if (tt <= hi) {
          unsigned spins = 0;
          while (ld_acquire(P.done + tt) < (unsigned)(s - 1)) {
            if (++spins > P.polls || *(volatile unsigned *)P.abort_flag) {
              ok = 0;
              break;
            }
            __nanosleep(64);
          }
        }
        ok = __all_sync(0xffffffffu, ok);
      }
      if (threadIdx.x == 0 && !ok) {
        atomicExch(P.err, 1);
        atomicExch(P.abort_flag, 1u);
        sh_stop = 1;
      }
    }
    __syncthreads();
    if (sh_stop) break;
    const double *xp = (s == 1) ? P.v : ((s % 2 == 0) ? P.B1 : P.B0);   // step s-1
    const double *xpp = (s == 2) ? P.v : ((s % 2 == 0) ? P.B0 : P.B1);  // step s-2 (same buffer as the output)
    double *out = (s % 2 == 0) ? P.B0 : P.B1;
    const double tc = (s == 1) ? P.t1 : P.t2;
    const double mus = P.mu[s];
    const double mu0 = P.mu[0];
    const int r0 = t * kWaveRows, r1 = min(P.n, r0 + kWaveRows);
    for (int r = r0 + (int)threadIdx.x; r < r1; r += kWaveThreads) {
      long long p;
      int w;
      row_start(A, r, p, w);
      double acc = 0.0;
#pragma unroll 4
      for (int j = 0; j < w; ++j, p += 32) {
        const double av = (double)__ldg(A.val + p);
        const int col = decode_col(__ldg(A.col + p), r);
        acc = __dadd_rn(acc, __dmul_rn(av, __ldcg(xp + col)));
      }
      const double x = __ldcg(xp + r);
      double wv = __dmul_rn(tc, __dadd_rn(acc, __dmul_rn(P.ncc, x)));
      if (s > 1) wv = __dadd_rn(wv, -__ldcg(xpp + r));
      out[r] = wv;
      const double yo = (s == 1) ? __dmul_rn(mu0, x) : __ldcg(P.y + r);
      P.y[r] = __dadd_rn(yo, __dmul_rn(mus, wv));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release(P.done + t, (unsigned)s);
    }
  }
}

template <class VT, class IT>
int launch_wave(const SellT<VT, IT> &A, const WaveArgs &P) {
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_filter_wave<VT, IT>, kWaveThreads, 0);
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  const long long items = (long long)P.deg * P.T;
  const int grid = (int)std::min<long long>(items, (long long)sm_count() * blocks_per_sm);
  k_filter_wave<VT, IT><<<grid, kWaveThreads, 0, stream()>>>(A, P);
  count_launch();
  return check_launch("k_filter_wave");
}

}  // namespace

void set_wave_wait_limit(unsigned long long polls) {
  g_wave_polls = (polls == 0 || polls > kWaveSpinLimit) ? kWaveSpinLimit : (unsigned)polls;
}

// Filter application through the pipelined kernel (the matrix must use the
// SELL-32 storage with rows in their original order: a tile's dependencies
// are computed from row numbers).  work: 2n doubles.
int chebav_wave(evslcu_mat *A, const double *mu, int deg, double cc, double dd, const double *v, double *y,
                double *work) {
  if (A->perm) return fail(EVSLCU_ERR_ARG, "the pipelined filter needs the unsorted SELL-32 row order");
  const int n = A->n;
  const int T = (n + kWaveRows - 1) / kWaveRows;
  const size_t need = 8 + (size_t)T;  // 2 words of counter, abort flag, padding, then done[]
  if (!A->wave_ctl || A->wave_ctl_words < need) {
    evslcu_free(A->wave_ctl);
    A->wave_ctl = (unsigned *)evslcu_malloc(sizeof(unsigned) * need);
    A->wave_ctl_words = A->wave_ctl ? need : 0;
    if (!A->wave_ctl) return fail(EVSLCU_ERR_NOMEM, "wave filter: out of device memory");
  }
  if (!A->wave_mu || A->wave_mu_cap < deg + 1) {
    evslcu_free(A->wave_mu);
    A->wave_mu_cap = std::max(deg + 1, 4096);
    A->wave_mu = (double *)evslcu_malloc(sizeof(double) * A->wave_mu_cap);
    if (!A->wave_mu) {
      A->wave_mu_cap = 0;
      return fail(EVSLCU_ERR_NOMEM, "wave filter: out of device memory");
    }
  }
  int rc = evslcu_h2d_async(A->wave_mu, mu, sizeof(double) * (deg + 1));
  if (!rc) rc = evslcu_memset(A->wave_ctl, 0, sizeof(unsigned) * need);
  if (!rc) rc = evslcu_memset(counters() + 10, 0, sizeof(int));
  if (rc) return rc;
  WaveArgs P;
  P.n = n;
  P.T = T;
  P.delta = (int)std::min<long long>((A->bandwidth + kWaveRows - 1) / kWaveRows, T);
  P.deg = deg;
  P.mu = A->wave_mu;
  P.t1 = 1.0 / dd;
  P.t2 = 2.0 / dd;
  P.ncc = -cc;
  P.v = v;
  P.y = y;
  P.B0 = work;
  P.B1 = work + n;
  P.next = (unsigned long long *)A->wave_ctl;
  P.abort_flag = A->wave_ctl + 2;
  P.err = (int *)(counters() + 10);
  P.done = A->wave_ctl + 8;
  P.polls = g_wave_polls;
  if (A->vfmt == 0 && A->ifmt == 0)
    return launch_wave(sell_view<double, int>(A), P);
  if (A->vfmt == 0 && A->ifmt == 1)
    return launch_wave(sell_view<double, short>(A), P);
  if (A->vfmt == 1 && A->ifmt == 0)
    return launch_wave(sell_view<float, int>(A), P);
  return launch_wave(sell_view<float, short>(A), P);
}

}  // namespace evslcu
