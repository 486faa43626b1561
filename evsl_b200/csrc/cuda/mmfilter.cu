// Filters of many slices on many matrices in one launch per degree: the
// batched form of ChebAv (SRC/chebpoly.c:519-598) for the request engine.
//
// A batch is a list of columns, each with its own matrix (a registered
// matrix, read through its SELL-C-sigma copy), polynomial (degree,
// coefficients on the device, cc,
// dd), input and output vectors and a 2n recurrence workspace.  Degree k is
// one launch for every column whose degree is at least k: the columns are
// sorted by degree, largest first, so those are a prefix of the list, and the
// launch's blocks are that prefix's row blocks (a block-to-column table maps
// each block to its column).  Independent instances of uneven size (the
// batched-instances configuration, small serving requests) then cost one
// launch per degree of the batch instead of one per degree per instance.
//
// Each row is read through the matrix's SELL-C-sigma copy and summed left to
// right with rounded multiply and add, and the three-term update is the
// single-vector kernel's: every column's output equals ChebAv of that column
// bit for bit, whatever else is in the batch.
#include <algorithm>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "sparse_types.cuh"

namespace evslcu {
namespace {

// One column of the batch.  The matrix is read through its SELL-C-sigma copy
// (coalesced chunks, compressed values / column offsets where lossless);
// fmt = 2 * (values stored as float) + (columns stored as int16 offsets).
struct MMItem {
  const long long *cptr;
  const int *cw;
  const void *scol, *sval;
  const int *perm;
  // row-pattern dictionary (fmt 4: double2 entries, 5: packed entries)
  const unsigned short *pid;
  const int2 *phdr;
  const void *pent;
  const double *mu;  // device, deg + 1
  const double *x;
  double *y;
  double *w;  // 2n
  double t1, t2, ncc;
  int n, deg, block0, fmt, ellw, pmax;  // pmax: longest row pattern (fmt 4, 5)
};

template <class VT, class IT>
__device__ __forceinline__ double mm_row(const MMItem &I, int s, const double *x) {
  const SellT<VT, IT> A{I.n, I.cptr, I.cw, (const IT *)I.scol, (const VT *)I.sval, I.ellw, I.perm};
  return row_dot<false>(A, s, x);
}
__device__ __forceinline__ int mm_row_of(const MMItem &I, int s) { return I.perm ? __ldg(I.perm + s) : s; }

// A row of a matrix read through its row-pattern dictionary (slot = row).
// Patterns of at most 8 entries (stencils) take the unrolled row product:
// every load of the row in flight before the first add, same rounded
// operations in the same order.
__device__ __forceinline__ double mm_row_pat(const MMItem &I, int r, const double *x) {
  if (I.fmt == 4) {
    const PatView v{I.n, I.pid, I.phdr, (const double2 *)I.pent};
    return I.pmax <= 8 ? row_dot_w<8, false>(v, r, x) : row_dot<false>(v, r, x);
  }
  const PatPView v{I.n, I.pid, I.phdr, (const unsigned long long *)I.pent};
  return I.pmax <= 8 ? row_dot_w<8, false>(v, r, x) : row_dot<false>(v, r, x);
}

constexpr int kMMThreads = 256;

template <bool FIRST>
__global__ void __launch_bounds__(kMMThreads) k_mm_cheb(const MMItem *__restrict__ items,
                                                        const int *__restrict__ blk_item, int k) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const MMItem &I = items[__ldg(blk_item + blockIdx.x)];
  const int n = I.n;
  const int sl = (blockIdx.x - I.block0) * kMMThreads + threadIdx.x;  // SELL slot
  if (k > I.deg || sl >= n) return;
  const int r = mm_row_of(I, sl);
  double *W0 = I.w, *W1 = I.w + n;
  const double *vk = FIRST ? I.x : (((k - 2) & 1) ? W1 : W0);
  const double *vkm1 = FIRST ? nullptr : ((k == 2) ? I.x : (((k - 1) & 1) ? W1 : W0));
  double *out = ((k - 1) & 1) ? W1 : W0;
  const double t = FIRST ? I.t1 : I.t2;
  const double s = I.mu[k];
  const double xm1 = FIRST ? 0.0 : vkm1[r];
  double *y = I.y;
  const double yo = FIRST ? 0.0 : y[r];
  double acc;
  switch (I.fmt) {
    case 0: acc = mm_row<double, int>(I, sl, vk); break;
    case 1: acc = mm_row<double, short>(I, sl, vk); break;
    case 2: acc = mm_row<float, int>(I, sl, vk); break;
    case 3: acc = mm_row<float, short>(I, sl, vk); break;
    default: acc = mm_row_pat(I, r, vk); break;
  }
  const double x = vk[r];
  double w = __dmul_rn(t, __dadd_rn(acc, __dmul_rn(I.ncc, x)));
  if (!FIRST) w = __dadd_rn(w, -xm1);
  out[r] = w;
  double yv = FIRST ? __dmul_rn(I.mu[0], x) : yo;
  yv = __dadd_rn(yv, __dmul_rn(s, w));
  y[r] = yv;
}

// degree 0: y = mu0 x
__global__ void k_mm_deg0(const MMItem *__restrict__ items, const int *__restrict__ blk_item) {
  const MMItem &I = items[__ldg(blk_item + blockIdx.x)];
  const int r = (blockIdx.x - I.block0) * kMMThreads + threadIdx.x;
  if (I.deg != 0 || r >= I.n) return;
  I.y[r] = __dmul_rn(I.mu[0], I.x[r]);
}

// ---- persistent form: every degree of every column in one launch ---------
//
// Work items are (degree k, block b of the active columns' blocks), numbered
// degree by degree: doff[k-1] .. doff[k]-1 are degree k's blocks, in the
// block-to-column table's order.  A thread block takes the next item from a
// ticket counter; before degree k of a column it waits (bounded) until its
// column's done counter shows every block of degree k-1 finished, which also
// means nothing still reads the buffer degree k overwrites (degree k-2's).
// Items are handed out in order and every item depends only on items handed
// out before it, so the launch always makes progress, whatever number of
// thread blocks is resident.  Vectors the launch writes are read through L2
// (ld.global.cg); a block publishes with a fence and an atomic add, and
// observes with an acquire load.  A wait that runs out of polls sets err and
// every block leaves at its next item.
struct MMPersist {
  const MMItem *items;
  const int *blk_item;
  const long long *doff;  // maxdeg + 1 item offsets
  unsigned *done;         // per column: blocks finished over all degrees
  unsigned long long *ticket;
  unsigned *err;
  int maxdeg;
  unsigned polls;
};

__device__ __forceinline__ unsigned mm_ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <class VT, class IT>
__device__ __forceinline__ double mm_row_cg(const MMItem &I, int s, const double *x) {
  const SellT<VT, IT> A{I.n, I.cptr, I.cw, (const IT *)I.scol, (const VT *)I.sval, I.ellw, I.perm};
  return row_dot<true>(A, s, x);
}

__global__ void __launch_bounds__(kMMThreads) k_mm_persistent(MMPersist P) {
  __shared__ long long sh_t;
  __shared__ int sh_stop;
  const long long total = P.doff[P.maxdeg];
  for (;;) {
    if (threadIdx.x == 0) {
      sh_stop = *(volatile unsigned *)P.err ? 1 : 0;
      sh_t = sh_stop ? total : (long long)atomicAdd(P.ticket, 1ull);
    }
    __syncthreads();
    const long long t = sh_t;
    if (t >= total) break;
    // degree k of item t: doff[k-1] <= t < doff[k]
    int lo = 1, hi = P.maxdeg;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(P.doff + mid) <= t)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int k = lo;
    const int bb = (int)(t - __ldg(P.doff + k - 1));
    const int ci = __ldg(P.blk_item + bb);
    const MMItem &I = P.items[ci];
    const int n = I.n;
    const unsigned nblk = (unsigned)((n + kMMThreads - 1) / kMMThreads);
    if (k > 1 && threadIdx.x == 0) {
      const unsigned need = (unsigned)(k - 1) * nblk;
      unsigned spins = 0;
      while (mm_ld_acquire(P.done + ci) < need) {
        if (++spins > P.polls || *(volatile unsigned *)P.err) {
          atomicExch(P.err, 1u);
          sh_stop = 1;
          break;
        }
        __nanosleep(64);
      }
    }
    __syncthreads();
    if (sh_stop) break;
    const int sl = (bb - I.block0) * kMMThreads + threadIdx.x;  // SELL slot
    if (sl < n) {
      const bool first = (k == 1);
      const int r = mm_row_of(I, sl);
      double *W0 = I.w, *W1 = I.w + n;
      const double *vk = first ? I.x : (((k - 2) & 1) ? W1 : W0);
      const double *vkm1 = first ? nullptr : ((k == 2) ? I.x : (((k - 1) & 1) ? W1 : W0));
      double *out = ((k - 1) & 1) ? W1 : W0;
      const double tt = first ? I.t1 : I.t2;
      const double sk = I.mu[k];
      const double xm1 = first ? 0.0 : __ldcg(vkm1 + r);
      double *y = I.y;
      const double yo = first ? 0.0 : __ldcg(y + r);
      double acc;
      switch (I.fmt) {
        case 0: acc = mm_row_cg<double, int>(I, sl, vk); break;
        case 1: acc = mm_row_cg<double, short>(I, sl, vk); break;
        case 2: acc = mm_row_cg<float, int>(I, sl, vk); break;
        default: acc = mm_row_cg<float, short>(I, sl, vk); break;
      }
      const double x = __ldcg(vk + r);
      double w = __dmul_rn(tt, __dadd_rn(acc, __dmul_rn(I.ncc, x)));
      if (!first) w = __dadd_rn(w, -xm1);
      out[r] = w;
      double yv = first ? __dmul_rn(I.mu[0], x) : yo;
      yv = __dadd_rn(yv, __dmul_rn(sk, w));
      y[r] = yv;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(P.done + ci, 1u);
    }
  }
}

unsigned g_mm_polls = 1u << 22;  // polls per dependency wait of the persistent form
int g_mm_patterns = 1;           // 1: matrices with a row-pattern dictionary are read through it
int g_mm_persistent = 0;         // 1: the persistent form

template <class F>
int launch_mm(F fn, int grid, const MMItem *items, const int *blk, int k) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kMMThreads);
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, fn, items, blk, k);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "batched filter launch failed: %s", cudaGetErrorString(e));
  count_launch();
  return check_launch("k_mm_cheb");
}

}  // namespace
}  // namespace evslcu

using namespace evslcu;

extern "C" {

// Most degrees the persistent form handles (its item offsets live in the table).
constexpr int kMMMaxDeg = 1 << 14;

size_t evslcu_filter_batch_table_bytes(int ncols, long long total_rows) {
  const long long blocks = total_rows / kMMThreads + ncols;
  return (sizeof(MMItem) * (size_t)std::max(ncols, 1) + 255) / 256 * 256 + sizeof(int) * (size_t)blocks + 256 +
         sizeof(long long) * (kMMMaxDeg + 1) + sizeof(unsigned) * (size_t)std::max(ncols, 1) + 256;
}

int evslcu_set_batch_persistent(int on) {
  g_mm_persistent = on ? 1 : 0;
  return 0;
}

int evslcu_filter_batch(int ncols, const evslcu_batch_col *cols, void *table, size_t table_bytes) {
  if (ncols <= 0) return 0;
  if (!cols || !table) return fail(EVSLCU_ERR_ARG, "filter_batch: bad arguments");
  std::vector<int> order(ncols);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return cols[p].deg > cols[q].deg; });
  std::vector<MMItem> items(ncols);
  std::vector<int> prefix(ncols + 1, 0);  // blocks of the first i columns in degree order
  long long rows = 0;
  for (int i = 0; i < ncols; ++i) {
    const evslcu_batch_col &c = cols[order[i]];
    if (!c.A || !c.mu || !c.x || !c.y || !c.w || c.deg < 0 || c.dd == 0.0)
      return fail(EVSLCU_ERR_ARG, "filter_batch: bad column %d", order[i]);
    const int n = c.A->n;
    MMItem &I = items[i];
    I.cptr = c.A->cptr;
    I.cw = c.A->cw;
    I.scol = c.A->scol;
    I.sval = c.A->sval;
    I.perm = c.A->perm;
    I.fmt = 2 * (c.A->vfmt ? 1 : 0) + (c.A->ifmt ? 1 : 0);
    I.pid = nullptr;
    I.phdr = nullptr;
    I.pent = nullptr;
    if (g_mm_patterns && !g_mm_persistent && evslcu_mat_uses_patterns(c.A) && !c.A->perm) {
      // the dictionary in global memory (PatView / PatPView): the same
      // rounded row products as the SELL copy
      if (c.A->pat_f32) {
        const PatPView v = pat_pview(c.A);
        I.pid = v.pid;
        I.phdr = v.hdr;
        I.pent = v.pk;
        I.fmt = 5;
      } else {
        const PatView v = pat_view(c.A);
        I.pid = v.pid;
        I.phdr = v.hdr;
        I.pent = v.ent;
        I.fmt = 4;
      }
    }
    I.ellw = c.A->ellw;
    I.mu = c.mu;
    I.x = c.x;
    I.y = c.y;
    I.w = c.w;
    I.t1 = 1.0 / c.dd;
    I.t2 = 2.0 / c.dd;
    I.ncc = -c.cc;
    I.n = n;
    I.deg = c.deg;
    I.block0 = prefix[i];
    I.pmax = c.A->pat_maxlen;
    prefix[i + 1] = prefix[i] + (n + kMMThreads - 1) / kMMThreads;
    rows += n;
  }
  const size_t ibytes = (sizeof(MMItem) * (size_t)ncols + 255) / 256 * 256;
  const int nblocks = prefix[ncols];
  const int maxdeg = items[0].deg;
  const bool persist = g_mm_persistent && maxdeg >= 1 && maxdeg <= kMMMaxDeg;
  // persistent form: item offsets per degree, then the zeroed counters
  const size_t boff = ibytes + sizeof(int) * (size_t)nblocks;
  const size_t doff_at = (boff + 15) / 16 * 16;
  const size_t done_at = doff_at + sizeof(long long) * (size_t)(maxdeg + 1);
  const size_t tick_at = (done_at + sizeof(unsigned) * (size_t)ncols + 15) / 16 * 16;
  const size_t host_bytes = persist ? tick_at + 16 : boff;
  if (host_bytes > table_bytes)
    return fail(EVSLCU_ERR_ARG, "filter_batch: table too small (%zu bytes for %d blocks)", table_bytes, nblocks);
  std::vector<unsigned char> host(host_bytes, 0);
  memcpy(host.data(), items.data(), sizeof(MMItem) * (size_t)ncols);
  int *blk = reinterpret_cast<int *>(host.data() + ibytes);
  for (int i = 0; i < ncols; ++i)
    for (int b = prefix[i]; b < prefix[i + 1]; ++b) blk[b] = i;
  if (persist) {
    long long *doff = reinterpret_cast<long long *>(host.data() + doff_at);
    int act = ncols;
    doff[0] = 0;
    for (int k = 1; k <= maxdeg; ++k) {
      while (act > 0 && items[act - 1].deg < k) --act;
      doff[k] = doff[k - 1] + prefix[act];
    }
  }
  int rc = evslcu_h2d(table, host.data(), host.size());
  if (rc) return rc;
  unsigned char *tb = static_cast<unsigned char *>(table);
  const MMItem *ditems = reinterpret_cast<const MMItem *>(table);
  const int *dblk = reinterpret_cast<const int *>(tb + ibytes);
  if (items[ncols - 1].deg == 0) {
    k_mm_deg0<<<nblocks, kMMThreads, 0, stream()>>>(ditems, dblk);
    count_launch();
    if ((rc = check_launch("k_mm_deg0"))) return rc;
  }
  if (persist) {
    MMPersist P;
    P.items = ditems;
    P.blk_item = dblk;
    P.doff = reinterpret_cast<const long long *>(tb + doff_at);
    P.done = reinterpret_cast<unsigned *>(tb + done_at);
    P.ticket = reinterpret_cast<unsigned long long *>(tb + tick_at);
    P.err = reinterpret_cast<unsigned *>(tb + tick_at + 8);
    P.maxdeg = maxdeg;
    P.polls = g_mm_polls;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mm_persistent, kMMThreads, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    const long long total = (long long)prefix[ncols] * 1;  // at least the first degree's blocks
    const int grid = (int)std::max(1LL, std::min<long long>((long long)sm_count() * per_sm, std::max(total, 1LL)));
    k_mm_persistent<<<grid, kMMThreads, 0, stream()>>>(P);
    count_launch();
    if ((rc = check_launch("k_mm_persistent"))) return rc;
    unsigned herr = 0;
    if ((rc = evslcu_d2h(&herr, P.err, sizeof(unsigned)))) return rc;
    if (herr) return fail(EVSLCU_ERR_TIMEOUT, "batched filter: a dependency wait ran out of polls");
    return 0;
  }
  // degree k runs the columns with deg >= k: the first `active` in degree order
  int active = ncols;
  for (int k = 1; k <= items[0].deg && !rc; ++k) {
    while (active > 0 && items[active - 1].deg < k) --active;
    rc = (k == 1) ? launch_mm(k_mm_cheb<true>, prefix[active], ditems, dblk, k)
                  : launch_mm(k_mm_cheb<false>, prefix[active], ditems, dblk, k);
  }
  (void)rows;
  return rc;
}

}  // extern "C"

namespace evslcu {
void set_batch_wait_limit(unsigned long long polls) {
  g_mm_polls = (polls == 0 || polls > (1ull << 22)) ? (1u << 22) : (unsigned)polls;
}
}  // namespace evslcu
