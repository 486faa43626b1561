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
  const double *mu;  // device, deg + 1
  const double *x;
  double *y;
  double *w;  // 2n
  double t1, t2, ncc;
  int n, deg, block0, fmt, ellw, pad;
};

template <class VT, class IT>
__device__ __forceinline__ double mm_row(const MMItem &I, int s, const double *x) {
  const SellT<VT, IT> A{I.n, I.cptr, I.cw, (const IT *)I.scol, (const VT *)I.sval, I.ellw, I.perm};
  return row_dot<false>(A, s, x);
}
__device__ __forceinline__ int mm_row_of(const MMItem &I, int s) { return I.perm ? __ldg(I.perm + s) : s; }

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
    default: acc = mm_row<float, short>(I, sl, vk); break;
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

size_t evslcu_filter_batch_table_bytes(int ncols, long long total_rows) {
  const long long blocks = total_rows / kMMThreads + ncols;
  return (sizeof(MMItem) * (size_t)std::max(ncols, 1) + 255) / 256 * 256 + sizeof(int) * (size_t)blocks + 256;
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
    I.pad = 0;
    prefix[i + 1] = prefix[i] + (n + kMMThreads - 1) / kMMThreads;
    rows += n;
  }
  const size_t ibytes = (sizeof(MMItem) * (size_t)ncols + 255) / 256 * 256;
  const int nblocks = prefix[ncols];
  if (ibytes + sizeof(int) * (size_t)nblocks > table_bytes)
    return fail(EVSLCU_ERR_ARG, "filter_batch: table too small (%zu bytes for %d blocks)", table_bytes, nblocks);
  std::vector<unsigned char> host(ibytes + sizeof(int) * (size_t)nblocks);
  memcpy(host.data(), items.data(), sizeof(MMItem) * (size_t)ncols);
  int *blk = reinterpret_cast<int *>(host.data() + ibytes);
  for (int i = 0; i < ncols; ++i)
    for (int b = prefix[i]; b < prefix[i + 1]; ++b) blk[b] = i;
  int rc = evslcu_h2d(table, host.data(), host.size());
  if (rc) return rc;
  const MMItem *ditems = reinterpret_cast<const MMItem *>(table);
  const int *dblk = reinterpret_cast<const int *>(static_cast<unsigned char *>(table) + ibytes);
  if (items[ncols - 1].deg == 0) {
    k_mm_deg0<<<nblocks, kMMThreads, 0, stream()>>>(ditems, dblk);
    count_launch();
    if ((rc = check_launch("k_mm_deg0"))) return rc;
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
