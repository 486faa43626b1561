// Chebyshev filter application y = p((A - cc)/dd) v (reference ChebAv,
// SRC/chebpoly.c:519-598) and its dispatch.
//
// Default path: one fused kernel per degree (sparse.cu), launched with
// programmatic dependent launch.  Optional path (evslx_set_filter_persistent):
// one cooperative launch for all degrees.  Every warp owns a fixed
// set of SELL-32 chunks for the whole filter; each lane keeps, for each of
// its rows, y and v_{k-1} in shared memory, so a degree step only streams A,
// writes the new vector once and gathers the previous one (mostly from L2).
// Degrees are separated by a grid-wide barrier whose wait is bounded: if a
// barrier does not complete within ~2 s the kernel records an error, every
// block returns, and the host reports EVSLCU_ERR_TIMEOUT.  The arithmetic per
// row is the same as the per-degree kernels (rounded multiply/add, same
// order), so both paths give identical results.
//
// Fallbacks: the per-degree kernels (one launch per degree) when the rows do
// not fit the shared memory of one resident grid, and a user matvec path
// (SetAMatvec) using the reference's three-vector rotation.
#include <algorithm>
#include <vector>

#include "sparse_types.cuh"

using namespace evslcu;

namespace {

constexpr unsigned long long kBarrierSpinLimit = 1ull << 26;
// Polls a block of the single-launch filter makes at a grid barrier before
// it gives up (evslcu_set_wait_limit; 0 restores kBarrierSpinLimit).
unsigned long long g_barrier_polls = kBarrierSpinLimit;

// ---------------------------------------------------------------------------
// profiling of filter applications
// ---------------------------------------------------------------------------
struct FilterProf {
  bool on = false;
  struct Rec {
    cudaEvent_t a, b;
    double bytes;
    int launches;
  };
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;
  double seconds = 0.0, bytes = 0.0;
  uint64_t launches = 0, calls = 0;
};
FilterProf g_prof;

cudaEvent_t prof_event() {
  if (!g_prof.pool.empty()) {
    cudaEvent_t e = g_prof.pool.back();
    g_prof.pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void prof_resolve() {
  for (auto &r : g_prof.pending) {
    float ms = 0.f;
    cudaEventSynchronize(r.b);
    cudaEventElapsedTime(&ms, r.a, r.b);
    g_prof.seconds += 1e-3 * ms;
    g_prof.bytes += r.bytes;
    g_prof.launches += (uint64_t)r.launches;
    g_prof.calls += 1;
    g_prof.pool.push_back(r.a);
    g_prof.pool.push_back(r.b);
  }
  g_prof.pending.clear();
}

// Algorithmic bytes of a degree-`deg` filter application (formula of the
// spectrum-slicing roofline): A once per degree (8-byte value and 4-byte
// column per nonzero, 4-byte row pointer per row) plus the 8-byte vectors the
// three-term step touches: k = 1 reads v and writes w and y; k > 1 reads vk,
// vkm1, y and writes w, y; the Lanczos epilogue reads zold and v.
double filter_bytes(const evslcu_mat *A, int deg, const evslcu_cheb_epi *epi) {
  const double n = (double)A->n;
  const double abytes = 12.0 * (double)A->nnz + 4.0 * (n + 1.0);
  double b = 0.0;
  for (int k = 1; k <= deg; ++k) b += abytes + 8.0 * n * ((k == 1) ? 3.0 : 5.0);
  if (epi) b += 8.0 * n * ((epi->zold ? 1.0 : 0.0) + (epi->dotv ? 1.0 : 0.0));
  return b;
}

// ---------------------------------------------------------------------------
// bounded grid barrier (all blocks are co-resident: cooperative launch)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_volatile(const unsigned *p) { return *(const volatile unsigned *)p; }

// Two-level barrier: blocks arrive on their group's counter (groups of
// kBarGroup blocks, each counter on its own 128-byte line); the last block
// of a group arrives on the top-level counter; the last group bumps the
// generation word that every block polls.  Polling is tight for the first
// spins and then backs off; after `limit` polls (kBarrierSpinLimit unless
// set lower) the block records an error and the whole grid leaves the kernel.
constexpr int kBarGroup = 16;

__device__ __forceinline__ bool grid_barrier(unsigned *area, int *err, unsigned long long limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned *gen = area;
    unsigned *top = area + 32;
    const unsigned ngroups = (gridDim.x + kBarGroup - 1) / kBarGroup;
    const unsigned g = blockIdx.x / kBarGroup;
    const unsigned gsize = min((unsigned)kBarGroup, gridDim.x - g * kBarGroup);
    unsigned *grp = area + 64 + 32 * g;
    int ok = 1;
    const unsigned my = ld_volatile(gen);
    __threadfence();
    bool release = false;
    if (atomicAdd(grp, 1u) == gsize - 1) {
      atomicExch(grp, 0u);
      if (atomicAdd(top, 1u) == ngroups - 1) {
        atomicExch(top, 0u);
        __threadfence();
        atomicAdd(gen, 1u);
        release = true;
      }
    }
    if (!release) {
      unsigned long long spins = 0;
      while (ld_volatile(gen) == my) {
        ++spins;
        if (spins > limit) {
          atomicExch(err, 1);
          ok = 0;
          break;
        }
        if (spins > 4096) __nanosleep(64);
      }
    }
    __threadfence();
    if (ok && *(volatile int *)err) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

struct PersistArgs {
  int nchunks;
  int deg;
  const double *mu;  // device, deg+1
  double t1, t2, ncc;
  const double *v;
  double *y;
  double *W0, *W1;
  const double *zold;
  double nbeta;
  const double *dotv;
  double *part;
  unsigned *ctr_dot;
  double *dot_out;
  unsigned *bar;
  int *err;
  unsigned long long polls;  // barrier wait limit
};

// Per-row state lives in dynamic shared memory: for slot i of thread t,
// y at st[i*NT + t] and v_{k-1} at st[(S + i)*NT + t].
template <class VIEW, int NT>
__global__ void __launch_bounds__(NT) k_filter_persistent(VIEW A, PersistArgs P, int S) {
  extern __shared__ double st[];
  __shared__ double sh[NT / 32];
  double *ys = st, *vs = st + (size_t)S * NT;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int gwarp = blockIdx.x * (NT / 32) + (tid >> 5);
  const int nwarps = gridDim.x * (NT / 32);
  const double mu0 = P.mu[0];
  for (int k = 1; k <= P.deg; ++k) {
    const double t = (k == 1) ? P.t1 : P.t2;
    const double s = P.mu[k];
    const double *x = (k == 1) ? P.v : ((k & 1) ? P.W1 : P.W0);
    double *out = ((k - 1) & 1) ? P.W1 : P.W0;
    for (int i = 0; i < S; ++i) {
      const int c = gwarp + i * nwarps;
      const int sl = c * 32 + lane;
      if (c < P.nchunks && sl < A.n) {
        const int r = row_of(A, sl);
        double acc, xv;
        if (k == 1) {
          acc = row_dot<false>(A, sl, x);
          xv = __ldg(x + r);
        } else {
          acc = row_dot<true>(A, sl, x);
          xv = __ldcg(x + r);
        }
        double w = __dmul_rn(t, __dadd_rn(acc, __dmul_rn(P.ncc, xv)));
        if (k > 1) w = __dadd_rn(w, -vs[i * NT + tid]);
        __stcg(out + r, w);
        const double yo = (k == 1) ? __dmul_rn(mu0, xv) : ys[i * NT + tid];
        ys[i * NT + tid] = __dadd_rn(yo, __dmul_rn(s, w));
        vs[i * NT + tid] = xv;
      }
    }
    if (k < P.deg && !grid_barrier(P.bar, P.err, P.polls)) return;
  }
  double dsum = 0.0;
  for (int i = 0; i < S; ++i) {
    const int c = gwarp + i * nwarps;
    const int sl = c * 32 + lane;
    if (c < P.nchunks && sl < A.n) {
      const int r = row_of(A, sl);
      double yy = ys[i * NT + tid];
      if (P.zold) yy = __dadd_rn(yy, __dmul_rn(P.nbeta, P.zold[r]));
      P.y[r] = yy;
      if (P.dotv) dsum += P.dotv[r] * yy;
    }
  }
  if (P.dot_out) {
    const double b = block_sum(dsum, sh);
    if (threadIdx.x == 0) P.part[blockIdx.x] = b;
    if (last_block(P.ctr_dot)) {
      const double tot = reduce_partials(P.part, gridDim.x, P.ctr_dot, sh);
      if (threadIdx.x == 0) *P.dot_out = tot;
    }
  }
}

// Launch with the most resident blocks per SM whose shared-memory state
// still covers every chunk; returns with *launched = false if none does.
template <class VIEW, int NT>
int launch_persistent_nt(const VIEW &view, int nchunks, PersistArgs &P, bool *launched) {
  static int smem_max = -1;
  const void *fn = (const void *)k_filter_persistent<VIEW, NT>;
  if (smem_max < 0) {
    int dev = 0, coop = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    smem_max = coop ? optin - 1024 : 0;
    if (smem_max > 0 && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max) !=
                            cudaSuccess) {
      cudaGetLastError();
      smem_max = 0;
    }
  }
  if (smem_max <= 0) return 0;
  const int sms = sm_count();
  for (int b = 2048 / NT; b >= 1; --b) {
    const long long warps = (long long)b * sms * (NT / 32);
    const int S = (int)((nchunks + warps - 1) / warps);
    const size_t smem = (size_t)S * NT * 2 * sizeof(double);
    if ((long long)smem > smem_max) continue;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NT, smem) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (per_sm < b) continue;
    const int grid = b * sms;
    if (grid > kMaxPartials) continue;
    int Sarg = S;
    void *args[] = {(void *)&view, (void *)&P, (void *)&Sarg};
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(NT), args, smem, stream());
    count_launch();
    if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "cooperative filter launch failed: %s", cudaGetErrorString(e));
    *launched = true;
    return 0;
  }
  return 0;
}

int g_filter_block = 1024;  // threads per block of the single-launch filter

template <class VIEW>
int launch_persistent(const VIEW &view, int nchunks, PersistArgs &P, bool *launched) {
  int rc = 0;
  if (g_filter_block >= 1024) {
    if ((rc = launch_persistent_nt<VIEW, 1024>(view, nchunks, P, launched)) || *launched) return rc;
  }
  if (g_filter_block >= 512) {
    if ((rc = launch_persistent_nt<VIEW, 512>(view, nchunks, P, launched)) || *launched) return rc;
  }
  return launch_persistent_nt<VIEW, 256>(view, nchunks, P, launched);
}

// device copy of the coefficients
double *g_mu_dev = nullptr;
int g_mu_cap = 0;

}  // namespace

extern "C" {

int evslcu_filter_error(void) {
  int h = 0;
  int *err = (int *)(counters() + 10);
  if (evslcu_d2h(&h, err, sizeof(int))) return EVSLCU_ERR_CUDA;
  if (h) {
    // blocks that gave up left before the final reduction: clear every
    // counter (all are zero between kernels) along with the flag
    evslcu_memset(counters(), 0, sizeof(unsigned) * kNumCounters);
    return fail(EVSLCU_ERR_TIMEOUT, "a wait of the filter kernel did not complete within its bound");
  }
  return 0;
}

int evslcu_set_wait_limit(unsigned long long polls) {
  g_barrier_polls = polls ? polls : kBarrierSpinLimit;
  set_wave_wait_limit(polls);
  set_batch_wait_limit(polls);
  return 0;
}

int evslcu_chebav(const evslcu_op *op, const double *mu, int deg, double cc, double dd, const double *v, double *y,
                  double *work, const evslcu_cheb_epi *epi) {
  if (!op || !mu || deg < 0 || !v || !y || !work) return fail(EVSLCU_ERR_ARG, "evslcu_chebav: bad arguments");
  const int n = op->n;
  const double t1 = 1.0 / dd, t2 = 2.0 / dd, ncc = -cc;
  if (deg == 0) {
    int rc = launch_scale_copy(n, mu[0], v, y);
    if (!rc && epi) rc = launch_lan_epi(n, epi, y);
    return rc;
  }
  if (!op->A) return chebav_user_matvec(op, mu, deg, cc, dd, v, y, work, epi);
  const evslcu_mat *A = op->A;
  cudaEvent_t ev_a = nullptr;
  if (g_prof.on) {
    ev_a = prof_event();
    cudaEventRecord(ev_a, stream());
  }
  bool launched = false;
  int rc = 0;
  if (A->wave && A->kernel == 0 && !A->perm && deg >= 2) {
    rc = chebav_wave((evslcu_mat *)A, mu, deg, cc, dd, v, y, work);
    if (!rc) rc = evslcu_filter_error();
    if (!rc && epi) rc = launch_lan_epi(n, epi, y);
    if (rc) return rc;
    launched = true;
  }
  const bool allow = !launched && A->persistent && A->kernel == 0 && deg >= 2;
  if (allow) {
    if (deg + 1 > g_mu_cap) {
      if (g_mu_dev) evslcu_free(g_mu_dev);
      g_mu_cap = std::max(deg + 1, 4096);
      g_mu_dev = (double *)evslcu_malloc(sizeof(double) * g_mu_cap);
      if (!g_mu_dev) return EVSLCU_ERR_NOMEM;
    }
    if ((rc = evslcu_h2d_async(g_mu_dev, mu, sizeof(double) * (deg + 1)))) return rc;
    if ((rc = evslcu_memset(barrier_area(), 0, sizeof(unsigned) * kBarrierWords)) ||
        (rc = evslcu_memset(counters() + 10, 0, sizeof(int))))
      return rc;
    PersistArgs P;
    P.nchunks = A->nchunks;
    P.deg = deg;
    P.mu = g_mu_dev;
    P.t1 = t1;
    P.t2 = t2;
    P.ncc = ncc;
    P.v = v;
    P.y = y;
    P.W0 = work;
    P.W1 = work + n;
    P.zold = epi ? epi->zold : nullptr;
    P.nbeta = epi ? epi->nbeta : 0.0;
    P.dotv = epi ? epi->dotv : nullptr;
    P.part = partials();
    P.ctr_dot = counters() + CTR_CHEB;
    P.dot_out = epi ? epi->dot_out : nullptr;
    P.bar = barrier_area();
    P.err = (int *)(counters() + 10);
    P.polls = g_barrier_polls;
    if (evslcu_mat_uses_patterns(A))
      rc = A->pat_f32 ? launch_persistent(pat_pview(A), A->nchunks, P, &launched)
                      : launch_persistent(pat_view(A), A->nchunks, P, &launched);
    else
      rc = with_view(A, [&](auto view) { return launch_persistent(view, A->nchunks, P, &launched); });
    if (rc) return rc;
  }
  if (!launched) rc = chebav_per_degree(A, mu, deg, cc, dd, v, y, work, epi);
  else if (allow && !rc) rc = evslcu_filter_error();
  if (rc) return rc;
  if (g_prof.on) {
    cudaEvent_t ev_b = prof_event();
    cudaEventRecord(ev_b, stream());
    g_prof.pending.push_back({ev_a, ev_b, filter_bytes(A, deg, epi), deg});
  }
  return 0;
}

int evslcu_filter_profile(int enable) {
  prof_resolve();
  g_prof.on = enable != 0;
  g_prof.seconds = g_prof.bytes = 0.0;
  g_prof.launches = g_prof.calls = 0;
  return 0;
}

int evslcu_filter_stats(double *seconds, double *bytes, uint64_t *launches, uint64_t *calls) {
  prof_resolve();
  if (seconds) *seconds = g_prof.seconds;
  if (bytes) *bytes = g_prof.bytes;
  if (launches) *launches = g_prof.launches;
  if (calls) *calls = g_prof.calls;
  return 0;
}

void *evslcu_stream_handle(void) { return (void *)stream(); }

int evslcu_set_filter_block(int threads) {
  if (threads != 256 && threads != 512 && threads != 1024)
    return fail(EVSLCU_ERR_ARG, "filter block size must be 256, 512 or 1024");
  g_filter_block = threads;
  return 0;
}

int evslcu_mat_set_persistent(evslcu_mat *A, int on) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  A->persistent = on ? 1 : 0;
  return 0;
}

int evslcu_mat_set_wave(evslcu_mat *A, int on) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  A->wave = on ? 1 : 0;
  return 0;
}

}  // extern "C"
