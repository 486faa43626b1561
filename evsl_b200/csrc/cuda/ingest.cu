// Building the device matrix formats on the GPU: COO -> CSR and CSR -> SELL-32.
//
// COO -> CSR gives the arrays of the reference's cooMat_to_csrMat
// (SRC/spmat.c:160-190) followed by sortrow (SRC/spmat.c:67-85): rows in
// order, and inside each row the entries sorted by column with ties kept in
// input order (the double transposition of sortrow is a stable sort by
// column).  Here every entry gets the key (column << 32 | input position);
// the keys are unique, so a merge sort of each row's keys is deterministic
// and equals that stable order.
//
//   1. check every index (nothing is written before the check passes);
//   2. count entries per row (integer atomics), exclusive scan -> ia;
//   3. scatter keys to their rows (slot order inside a row is arbitrary);
//   4. merge passes of widths 1, 2, 4, ... below the longest row: an element
//      of run A lands at (its index in A) + (#keys of run B below it), and
//      the same with A and B swapped -- a pure gather/scatter with no ties;
//   5. gather ja and a through the sorted keys.
//
// CSR -> SELL-32 (the filter's layout): chunk widths, a scan of the chunk
// sizes, and one fill pass writing every padded slot, with the lossless
// compression checks (values exactly floats, column offsets within int16)
// computed on the device as well.
#include <string.h>

#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "common.cuh"
#include "sparse_types.cuh"

namespace evslcu {

namespace {

inline int launched(const char *what) {
  count_launch();
  return check_launch(what);
}

constexpr int kScanItems = 8;
constexpr int kScanTile = kThreads * kScanItems;

// Exclusive scan of one tile of kScanTile inputs; writes the tile's
// prefixes to out and its total to tsum[blockIdx.x].
template <class IT, class OT>
__global__ void __launch_bounds__(kThreads) k_scan_tile(const IT *in, long long m, OT *out, long long *tsum) {
  __shared__ long long wsum[kThreads / 32];
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  long long v[kScanItems];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const long long i = base + k;
    v[k] = (i < m) ? (long long)in[i] : 0;
    s += v[k];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  long long x = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    long long t = (lane < kThreads / 32) ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < kThreads / 32) wsum[lane] = t;
  }
  __syncthreads();
  long long run = x - s + (w > 0 ? wsum[w - 1] : 0);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const long long i = base + k;
    if (i < m) out[i] = (OT)run;
    run += v[k];
  }
  if (threadIdx.x == kThreads - 1) tsum[blockIdx.x] = run;
}

// In-place exclusive scan of the T tile totals by one block; the grand total
// goes to *total.
__global__ void __launch_bounds__(kThreads) k_scan_totals(long long *tsum, long long T, long long *total) {
  __shared__ long long wsum[kThreads / 32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (long long b = 0; b < T; b += kThreads) {
    const long long i = b + threadIdx.x;
    const long long s = (i < T) ? tsum[i] : 0;
    long long x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      long long t = (lane < kThreads / 32) ? wsum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      if (lane < kThreads / 32) wsum[lane] = t;
    }
    __syncthreads();
    const long long ex = x - s + (w > 0 ? wsum[w - 1] : 0);
    if (i < T) tsum[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == kThreads - 1) carry += ex + s;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

template <class OT>
__global__ void k_scan_add(OT *out, long long m, const long long *tsum, const long long *total) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    out[i] = (OT)((long long)out[i] + tsum[i / kScanTile]);
  if (blockIdx.x == 0 && threadIdx.x == 0) out[m] = (OT)*total;
}

// out[0..m] = exclusive prefix sums of in[0..m) with out[m] = the total.
template <class IT, class OT>
int scan_exclusive(const IT *in, long long m, OT *out) {
  const long long T = std::max(1LL, (m + kScanTile - 1) / kScanTile);
  long long *tsum = (long long *)evslcu_malloc(sizeof(long long) * (size_t)(T + 1));
  if (!tsum) return EVSLCU_ERR_NOMEM;
  k_scan_tile<IT, OT><<<(unsigned)T, kThreads, 0, stream()>>>(in, m, out, tsum);
  int rc = launched("k_scan_tile");
  if (!rc) {
    k_scan_totals<<<1, kThreads, 0, stream()>>>(tsum, T, tsum + T);
    rc = launched("k_scan_totals");
  }
  if (!rc) {
    k_scan_add<OT><<<grid_for(std::max(m, 1LL)), kThreads, 0, stream()>>>(out, m, tsum, tsum + T);
    rc = launched("k_scan_add");
  }
  evslcu_free(tsum);
  return rc;
}

__device__ __forceinline__ long long lower_bound_u64(const unsigned long long *a, long long len,
                                                     unsigned long long key) {
  long long lo = 0, hi = len;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (a[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// ---- COO -> CSR ---------------------------------------------------------------

__global__ void k_coo_check(long long nnz, const int *ir, const int *jc, int n, int base,
                            unsigned long long *first_bad) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
    const int r = ir[e] - base, c = jc[e] - base;
    if (r < 0 || r >= n || c < 0 || c >= n) atomicMin(first_bad, (unsigned long long)e);
  }
}

__global__ void k_coo_count(long long nnz, const int *ir, int base, int *cnt) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x)
    atomicAdd(&cnt[ir[e] - base], 1);
}

__global__ void k_max_len(int n, const int *ia, int *mx) {
  int m = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) m = max(m, ia[r + 1] - ia[r]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mx, m);
}

__global__ void k_coo_scatter(long long nnz, const int *ir, const int *jc, int base, const int *ia, int *fill,
                              unsigned long long *keys, int *rowid) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
    const int r = ir[e] - base;
    const int slot = atomicAdd(&fill[r], 1);
    const long long p = (long long)ia[r] + slot;
    keys[p] = ((unsigned long long)(unsigned)(jc[e] - base) << 32) | (unsigned long long)(unsigned)e;
    rowid[p] = r;
  }
}

// One merge pass of width w inside every row.
__global__ void k_row_merge(long long nnz, const int *ia, const int *rowid, const unsigned long long *in,
                            unsigned long long *out, long long w) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
    const int r = rowid[e];
    const long long b0 = ia[r], L = (long long)ia[r + 1] - b0, p = e - b0;
    const long long k = p / w, pb = (k & ~1LL) * w;
    const unsigned long long key = in[e];
    long long dst;
    if ((k & 1) == 0) {
      const long long bs = pb + w, be = min(pb + 2 * w, L);
      const long long below = (bs < be) ? lower_bound_u64(in + b0 + bs, be - bs, key) : 0;
      dst = b0 + p + below;
    } else {
      const long long below = lower_bound_u64(in + b0 + pb, w, key);
      dst = b0 + pb + (p - pb - w) + below;
    }
    out[dst] = key;
  }
}

__global__ void k_coo_gather(long long nnz, const unsigned long long *keys, const double *vv, int *ja, double *a) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
    const unsigned long long key = keys[e];
    ja[e] = (int)(key >> 32);
    a[e] = vv[key & 0xffffffffull];
  }
}

// ---- CSR checks and SELL-32 -----------------------------------------------------

// flags[0]: first row whose pointer decreases (INT_MAX if none).
__global__ void k_csr_check_ptr(int n, const int *ia, int *flags) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    if (ia[r + 1] < ia[r]) atomicMin(&flags[0], r);
}

// flags[1]: first entry position with a column outside [0, n) (INT_MAX if
// none); flags[2]: some value is not exactly a finite float; flags[3]: some
// |col - row| does not fit int16; flags[4]: the largest |col - row|.
__global__ void k_csr_check_entries(int n, const int *ia, const int *ja, const double *a, int *flags) {
  int not_float = 0, not_16 = 0, bw = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    for (int j = ia[r]; j < ia[r + 1]; ++j) {
      const int c = ja[j];
      if (c < 0 || c >= n) atomicMin(&flags[1], j);
      if (c - r > 32767 || c - r < -32768) not_16 = 1;
      bw = max(bw, abs(c - r));
      const double v = a[j];
      if (!(isfinite(v) && (double)(float)v == v)) not_float = 1;
    }
  }
  if (__any_sync(0xffffffffu, not_float) && (threadIdx.x & 31) == 0) atomicOr(&flags[2], 1);
  if (__any_sync(0xffffffffu, not_16) && (threadIdx.x & 31) == 0) atomicOr(&flags[3], 1);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bw = max(bw, __shfl_down_sync(0xffffffffu, bw, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&flags[4], bw);
}

// Row lengths of the sort and chunk-width kernels: a CSR row's, or an
// explicit per-row count (the rows' entries in one column range).
struct LenCsr {
  const int *ia;
  __device__ __forceinline__ int operator()(int r) const { return ia[r + 1] - ia[r]; }
};
struct LenArr {
  const int *len;
  __device__ __forceinline__ int operator()(int r) const { return len[r]; }
};

// Width of each chunk: its longest row (slot s holds row perm[s], or row s
// when perm is null).
template <class L>
__global__ void k_chunk_width(int n, int nch, L len, const int *perm, int *cw, long long *csize) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nch; c += gridDim.x * blockDim.x) {
    int w = 0;
    const int s1 = min(n, 32 * c + 32);
    for (int s = 32 * c; s < s1; ++s) {
      const int r = perm ? perm[s] : s;
      w = max(w, len(r));
    }
    cw[c] = w;
    csize[c] = 32LL * w;
  }
}

// SELL-C-sigma row order: one block per window of W consecutive rows (W a
// power of two, at most 4096) sorts the window's rows by length, longest
// first, ties in row order, with a bitonic network on 64-bit keys
// (0x7fffffff - length, position in the window) in shared memory; slot
// w0 + i then holds row perm[w0 + i].  Positions past the last row carry the
// largest key and sort to the end.
template <int W, class L>
__global__ void __launch_bounds__(1024) k_sigma_sort(int n, L len, int *perm) {
  __shared__ unsigned long long key[W];
  const int w0 = blockIdx.x * W;
  for (int i = threadIdx.x; i < W; i += blockDim.x) {
    const int r = w0 + i;
    key[i] = (r < n) ? ((unsigned long long)(0x7fffffff - len(r)) << 32) | (unsigned)i : ~0ULL;
  }
  __syncthreads();
  for (int k = 2; k <= W; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < W; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long x = key[i], y = key[ixj];
          if ((x > y) == ((i & k) == 0)) {
            key[i] = y;
            key[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < W; i += blockDim.x)
    if (w0 + i < n) perm[w0 + i] = w0 + (int)(key[i] & 0xffffffffu);
}

// Thread per (chunk, lane) slot; entry j of lane l at cptr[c] + 32 j + l.
// Padding: value 0 in the row's own column (adds 0 * x[r]).  Slot s holds
// row perm[s] (row s when perm is null); slots past the last row are all
// padding and point at row 0.
template <class VT, class IT>
__global__ void k_sell_fill(int n, int nch, const int *ia, const int *ja, const double *a, const int *perm,
                            const long long *cptr, const int *cw, IT *scol, VT *sval) {
  const long long slots = 32LL * nch;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(s >> 5), l = (int)(s & 31);
    const bool live = s < n;
    const int r = live ? (perm ? perm[s] : (int)s) : 0;
    const int len = live ? ia[r + 1] - ia[r] : 0;
    const int rr = r;
    const int beg = live ? ia[r] : 0;
    for (int j = 0; j < cw[c]; ++j) {
      const long long p = cptr[c] + 32LL * j + l;
      const int col = (j < len) ? ja[beg + j] : rr;
      const double v = (j < len) ? a[beg + j] : 0.0;
      if (sizeof(IT) == 2)
        scol[p] = (IT)(col - rr);
      else
        scol[p] = (IT)col;
      sval[p] = (VT)v;
    }
  }
}

// ---- column-split copy (multi-column filter on large general matrices) -----
//
// Range p of the columns is [p * width, (p + 1) * width).  For each row the
// entries of every range form one run of its CSR entries, because the row's
// columns increase; beg/len (P x n, range-major) hold each run.

// Walks each row once, recording where every range's run starts and how long
// it is, and flags rows whose columns do not increase.
__global__ void k_xs_bounds(int n, const int *ia, const int *ja, int P, int width, int *beg, int *len, int *bad) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int hi = ia[r + 1];
    int j = ia[r], prev = -1;
    bool ok = true;
    for (int p = 0; p < P; ++p) {
      const long long lim = (long long)(p + 1) * width;
      const int b = j;
      while (j < hi) {
        const int c = ja[j];
        if (c <= prev) ok = false;
        if (c >= lim) break;
        prev = c;
        ++j;
      }
      beg[(size_t)p * n + r] = b;
      len[(size_t)p * n + r] = j - b;
    }
    if (!ok) atomicExch(bad, 1);
  }
}

// Thread per (chunk, lane) slot of one range; entry j of lane l at
// cptr[c] + 32 j + l.  Padding slots get column -1 (the filter skips them).
__global__ void k_xs_fill(int n, int nch, const int *beg, const int *len, const int *ja, const double *a,
                          const int *perm, const long long *cptr, const int *cw, int *col, double *val) {
  const long long slots = 32LL * nch;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(s >> 5), l = (int)(s & 31);
    const bool live = s < n;
    const int r = live ? perm[s] : 0;
    const int ln = live ? len[r] : 0;
    const int b = live ? beg[r] : 0;
    for (int j = 0; j < cw[c]; ++j) {
      const long long p = cptr[c] + 32LL * j + l;
      col[p] = (j < ln) ? ja[b + j] : -1;
      val[p] = (j < ln) ? a[b + j] : 0.0;
    }
  }
}

// ---- row-pattern dictionary --------------------------------------------------
//
// A row's pattern is its sequence of (value bits, column - row) pairs in CSR
// order.  Pass 1 hashes every row into an open-addressing table of 64-bit
// keys (insert-or-find by compare-and-swap; the smallest row with a key is its
// representative); pass 2 compares every row with its representative entry
// by entry, so a hash collision can only cancel the dictionary, never change
// a result.  The build gives up as soon as more than kPatMax distinct keys
// appear.

constexpr int kPatSlots = 4096;  // hash slots (power of two)
constexpr int kPatMax = 1024;    // most distinct patterns kept
constexpr int kPatMaxEntries = 1 << 16;

// 64-bit finaliser of MurmurHash3 (fmix64).
__device__ __forceinline__ unsigned long long pat_mix(unsigned long long z) {
  z ^= z >> 33;
  z *= 0xff51afd7ed558ccdULL;
  z ^= z >> 33;
  z *= 0xc4ceb9fe1a85ec53ULL;
  z ^= z >> 33;
  return z;
}

// ctl[0]: distinct keys inserted; ctl[1]: gave up (too many patterns);
// ctl[2]: a row differs from its representative (hash collision).
__global__ void k_pat_insert(int n, const int *ia, const int *ja, const double *a, unsigned long long *keys,
                             int *rep, int *slot_of, int *ctl) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    if (*(volatile int *)(ctl + 1)) return;
    const int b = ia[r], e = ia[r + 1];
    unsigned long long h = pat_mix(0x9e3779b97f4a7c15ULL + (unsigned long long)(e - b));
    for (int j = b; j < e; ++j) {
      h = pat_mix(h ^ (unsigned long long)(unsigned)(ja[j] - r));
      h = pat_mix(h ^ (unsigned long long)__double_as_longlong(a[j]));
    }
    h |= 1ULL;  // 0 marks an empty slot
    int s = (int)(h & (kPatSlots - 1)), found = -1;
    for (int i = 0; i < kPatSlots; ++i) {
      if (*(volatile int *)(ctl + 1)) return;
      const unsigned long long prev = atomicCAS(keys + s, 0ULL, h);
      if (prev == 0ULL) {
        if (atomicAdd(ctl, 1) >= kPatMax) atomicExch(ctl + 1, 1);
        found = s;
        break;
      }
      if (prev == h) {
        found = s;
        break;
      }
      s = (s + 1) & (kPatSlots - 1);
    }
    if (found < 0) {
      atomicExch(ctl + 1, 1);
      return;
    }
    atomicMin(rep + found, r);
    slot_of[r] = found;
  }
}

__global__ void k_pat_verify(int n, const int *ia, const int *ja, const double *a, const int *rep,
                             const int *slot_of, int *ctl) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int q = rep[slot_of[r]];
    if (q == r) continue;
    const int b = ia[r], len = ia[r + 1] - b;
    const int bq = ia[q];
    bool same = (ia[q + 1] - bq) == len;
    for (int j = 0; same && j < len; ++j)
      same = (ja[b + j] - r == ja[bq + j] - q) &&
             (__double_as_longlong(a[b + j]) == __double_as_longlong(a[bq + j]));
    if (!same) atomicExch(ctl + 2, 1);
  }
}

__global__ void k_pat_len(int npat, const int *reps, const int *ia, int *lens) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npat; p += gridDim.x * blockDim.x)
    lens[p] = ia[reps[p] + 1] - ia[reps[p]];
}

__global__ void k_pat_fill(int npat, const int *reps, const int *ia, const int *ja, const double *a,
                           const int2 *hdr, double2 *ent) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npat; p += gridDim.x * blockDim.x) {
    const int q = reps[p], b = ia[q];
    for (int j = 0; j < hdr[p].y; ++j)
      ent[hdr[p].x + j] = make_double2(a[b + j], __longlong_as_double((long long)(ja[b + j] - q)));
  }
}

__global__ void k_pat_assign(int n, const int *slot_of, const int *slot2id, unsigned short *pid) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    pid[r] = (unsigned short)slot2id[slot_of[r]];
}

}  // namespace

int build_patterns_device(evslcu_mat *M) {
  const int n = M->n;
  if (n <= 0) return 0;
  // scratch: keys, rep, ctl, slot_of
  const size_t kb = sizeof(unsigned long long) * kPatSlots, rb = sizeof(int) * kPatSlots, cb = 256;
  char *scr = (char *)evslcu_malloc(kb + rb + cb + sizeof(int) * (size_t)n);
  if (!scr) return 0;  // the dictionary is optional
  unsigned long long *keys = (unsigned long long *)scr;
  int *rep = (int *)(scr + kb);
  int *ctl = (int *)(scr + kb + rb);
  int *slot_of = (int *)(scr + kb + rb + cb);
  std::vector<int> hrep(kPatSlots, 0x7fffffff);
  int rc = evslcu_memset(keys, 0, kb);
  if (!rc) rc = evslcu_memset(ctl, 0, cb);
  if (!rc) rc = evslcu_h2d_async(rep, hrep.data(), rb);
  if (!rc) {
    k_pat_insert<<<grid_for(n), kThreads, 0, stream()>>>(n, M->ia, M->ja, M->a, keys, rep, slot_of, ctl);
    rc = launched("k_pat_insert");
  }
  int hctl[3] = {0, 0, 0};
  if (!rc) rc = evslcu_d2h(hctl, ctl, sizeof(hctl));
  if (!rc && !hctl[1]) {
    k_pat_verify<<<grid_for(n), kThreads, 0, stream()>>>(n, M->ia, M->ja, M->a, rep, slot_of, ctl);
    rc = launched("k_pat_verify");
    if (!rc) rc = evslcu_d2h(hctl, ctl, sizeof(hctl));
  }
  if (rc || hctl[1] || hctl[2] || hctl[0] <= 0) {
    evslcu_free(scr);
    return rc;
  }
  std::vector<unsigned long long> hkeys(kPatSlots);
  rc = evslcu_d2h(hkeys.data(), keys, kb);
  if (!rc) rc = evslcu_d2h(hrep.data(), rep, rb);
  if (rc) {
    evslcu_free(scr);
    return rc;
  }
  // patterns numbered in the order of their first row
  std::vector<std::pair<int, int>> used;  // (representative row, slot)
  for (int s = 0; s < kPatSlots; ++s)
    if (hkeys[s]) used.push_back({hrep[s], s});
  std::sort(used.begin(), used.end());
  const int npat = (int)used.size();
  std::vector<int> slot2id(kPatSlots, 0), reps(npat), lens(npat);
  for (int p = 0; p < npat; ++p) {
    slot2id[used[p].second] = p;
    reps[p] = used[p].first;
  }
  // device: slot2id [kPatSlots], reps [npat], lens [npat] (reuses the key area)
  int *d_slot2id = (int *)keys, *d_reps = d_slot2id + kPatSlots, *d_lens = d_reps + kPatMax;
  rc = evslcu_h2d_async(d_slot2id, slot2id.data(), sizeof(int) * kPatSlots);
  if (!rc) rc = evslcu_h2d_async(d_reps, reps.data(), sizeof(int) * npat);
  if (!rc) {
    k_pat_len<<<grid_for(npat), kThreads, 0, stream()>>>(npat, d_reps, M->ia, d_lens);
    rc = launched("k_pat_len");
  }
  if (!rc) rc = evslcu_d2h(lens.data(), d_lens, sizeof(int) * npat);
  std::vector<int2> hdr(npat);
  long long total = 0;
  int maxlen = 0;
  for (int p = 0; p < npat; ++p) {
    hdr[p] = make_int2((int)total, lens[p]);
    total += lens[p];
    maxlen = std::max(maxlen, lens[p]);
  }
  if (rc || total > kPatMaxEntries) {
    evslcu_free(scr);
    return rc;
  }
  const size_t hbytes = pat_hdr_bytes(npat);
  void *table = evslcu_malloc(hbytes + (sizeof(double2) + sizeof(unsigned long long)) * (size_t)std::max(total, 1LL));
  unsigned short *pid = (unsigned short *)evslcu_malloc(sizeof(unsigned short) * (size_t)n);
  if (!table || !pid) {
    evslcu_free(table);
    evslcu_free(pid);
    evslcu_free(scr);
    return 0;
  }
  int2 *d_hdr = (int2 *)table;
  double2 *d_ent = (double2 *)((char *)table + hbytes);
  rc = evslcu_h2d_async(d_hdr, hdr.data(), sizeof(int2) * npat);
  if (!rc) {
    k_pat_fill<<<grid_for(npat), kThreads, 0, stream()>>>(npat, d_reps, M->ia, M->ja, M->a, d_hdr, d_ent);
    rc = launched("k_pat_fill");
  }
  if (!rc) {
    k_pat_assign<<<grid_for(n), kThreads, 0, stream()>>>(n, slot_of, d_slot2id, pid);
    rc = launched("k_pat_assign");
  }
  if (!rc) rc = evslcu_sync();  // the host vectors above are read by queued copies
  evslcu_free(scr);
  // packed entries when every value is exactly a float
  int f32 = 0;
  if (!rc) {
    std::vector<double2> ent((size_t)total);
    std::vector<unsigned long long> pk((size_t)total);
    rc = evslcu_d2h(ent.data(), d_ent, sizeof(double2) * (size_t)total);
    f32 = 1;
    for (long long j = 0; j < total && !rc && f32; ++j) {
      const double v = ent[j].x;
      if (!(std::isfinite(v) && (double)(float)v == v)) {
        f32 = 0;
        break;
      }
      const float fv = (float)v;
      unsigned fb;
      long long ob;
      memcpy(&fb, &fv, sizeof(fb));
      memcpy(&ob, &ent[j].y, sizeof(ob));
      pk[j] = ((unsigned long long)fb << 32) | (unsigned long long)(unsigned)(int)ob;
    }
    if (!rc && f32) rc = evslcu_h2d(d_ent + total, pk.data(), sizeof(unsigned long long) * (size_t)total);
  }
  if (rc) {
    evslcu_free(table);
    evslcu_free(pid);
    return rc;
  }
  M->pat_f32 = f32;
  M->pat_id = pid;
  M->pat_table = table;
  M->npat = npat;
  M->pat_entries = (int)total;
  M->pat_maxlen = maxlen;
  return 0;
}

// Window of the SELL-C-sigma length sort: -1 automatic (g_sigma_auto rows
// when the plain layout pads more than kSigmaTrigger times the entries),
// 0 never, otherwise that window (a power of two from 32 to 4096) always.
int g_sell_sigma = -1;
int g_sigma_auto = 256;
constexpr double kSigmaTrigger = 1.10;

template <class L>
int launch_sigma_sort(int n, int sigma, L len, int *perm) {
  const int nwin = (int)(((long long)n + sigma - 1) / sigma);
  switch (sigma) {
    case 32: k_sigma_sort<32><<<nwin, 32, 0, stream()>>>(n, len, perm); break;
    case 64: k_sigma_sort<64><<<nwin, 64, 0, stream()>>>(n, len, perm); break;
    case 128: k_sigma_sort<128><<<nwin, 128, 0, stream()>>>(n, len, perm); break;
    case 256: k_sigma_sort<256><<<nwin, 256, 0, stream()>>>(n, len, perm); break;
    case 512: k_sigma_sort<512><<<nwin, 512, 0, stream()>>>(n, len, perm); break;
    case 1024: k_sigma_sort<1024><<<nwin, 1024, 0, stream()>>>(n, len, perm); break;
    case 2048: k_sigma_sort<2048><<<nwin, 1024, 0, stream()>>>(n, len, perm); break;
    case 4096: k_sigma_sort<4096><<<nwin, 1024, 0, stream()>>>(n, len, perm); break;
    default: return fail(EVSLCU_ERR_ARG, "SELL sort window must be a power of two from 32 to 4096 (got %d)", sigma);
  }
  return launched("k_sigma_sort");
}

// Builds the SELL-C-sigma copy of M's device CSR (M->n, M->nnz, M->ia/ja/a
// set) after validating it.  allow_compress: use the compressed formats when
// the values and columns allow it.
int build_sell_device(evslcu_mat *M, int allow_compress) {
  const int n = M->n;
  int *flags = (int *)evslcu_malloc(sizeof(int) * 5);
  if (!flags) return EVSLCU_ERR_NOMEM;
  const int init[5] = {0x7fffffff, 0x7fffffff, 0, 0, 0};
  int hf[5];
  int rc = evslcu_h2d(flags, init, sizeof(init));
  if (!rc) {
    k_csr_check_ptr<<<grid_for(n), kThreads, 0, stream()>>>(n, M->ia, flags);
    rc = launched("k_csr_check_ptr");
  }
  if (!rc) rc = evslcu_d2h(hf, flags, sizeof(hf));
  if (!rc && hf[0] != 0x7fffffff) rc = fail(EVSLCU_ERR_ARG, "CSR row pointer decreases at row %d", hf[0]);
  if (!rc) {
    k_csr_check_entries<<<grid_for(n), kThreads, 0, stream()>>>(n, M->ia, M->ja, M->a, flags);
    rc = launched("k_csr_check_entries");
  }
  if (!rc) rc = evslcu_d2h(hf, flags, sizeof(hf));
  evslcu_free(flags);
  if (rc) return rc;
  if (hf[1] != 0x7fffffff) {
    int bad = 0;
    evslcu_d2h(&bad, M->ja + hf[1], sizeof(int));
    return fail(EVSLCU_ERR_ARG, "CSR column index %d at position %d is outside [0, %d)", bad, hf[1], n);
  }
  M->bandwidth = hf[4];
  M->vfmt = (allow_compress && !hf[2]) ? 1 : 0;
  M->ifmt = (allow_compress && !hf[3]) ? 1 : 0;
  const int nch = (n + 31) / 32;
  M->nchunks = nch;
  M->cptr = (long long *)evslcu_malloc(sizeof(long long) * (nch + 1));
  M->cw = (int *)evslcu_malloc(sizeof(int) * nch);
  long long *csize = (long long *)evslcu_malloc(sizeof(long long) * nch);
  if (!M->cptr || !M->cw || !csize) {
    evslcu_free(csize);
    return fail(EVSLCU_ERR_NOMEM, "SELL build: out of device memory");
  }
  k_chunk_width<<<grid_for(nch), kThreads, 0, stream()>>>(n, nch, LenCsr{M->ia}, nullptr, M->cw, csize);
  rc = launched("k_chunk_width");
  if (!rc) rc = scan_exclusive<long long, long long>(csize, nch, M->cptr);
  long long padded = 0;
  if (!rc) rc = evslcu_d2h(&padded, M->cptr + nch, sizeof(long long));
  M->padded_plain = padded;
  // SELL-C-sigma: sort the rows of each window by length when the chunks of
  // the plain layout carry much padding, and keep the order when it cuts
  // the stored slots by at least 5%.
  const int sigma = g_sell_sigma < 0 ? g_sigma_auto : g_sell_sigma;
  const bool try_sort = sigma > 0 && (g_sell_sigma > 0 || (double)padded > kSigmaTrigger * (double)std::max(M->nnz, 1LL));
  if (!rc && try_sort) {
    int *perm = (int *)evslcu_malloc(sizeof(int) * 32 * (size_t)nch);
    if (!perm) rc = fail(EVSLCU_ERR_NOMEM, "SELL build: out of device memory (row order)");
    if (!rc) rc = evslcu_memset(perm, 0, sizeof(int) * 32 * (size_t)nch);
    if (!rc) rc = launch_sigma_sort(n, sigma, LenCsr{M->ia}, perm);
    long long *cptr2 = nullptr;
    int *cw2 = nullptr;
    if (!rc) {
      cptr2 = (long long *)evslcu_malloc(sizeof(long long) * (nch + 1));
      cw2 = (int *)evslcu_malloc(sizeof(int) * nch);
      if (!cptr2 || !cw2) rc = fail(EVSLCU_ERR_NOMEM, "SELL build: out of device memory");
    }
    if (!rc) {
      k_chunk_width<<<grid_for(nch), kThreads, 0, stream()>>>(n, nch, LenCsr{M->ia}, perm, cw2, csize);
      rc = launched("k_chunk_width");
    }
    if (!rc) rc = scan_exclusive<long long, long long>(csize, nch, cptr2);
    long long padded2 = 0;
    if (!rc) rc = evslcu_d2h(&padded2, cptr2 + nch, sizeof(long long));
    if (!rc && (g_sell_sigma > 0 || (double)padded2 < 0.95 * (double)padded)) {
      std::swap(M->cptr, cptr2);
      std::swap(M->cw, cw2);
      M->perm = perm;
      perm = nullptr;
      M->sigma = sigma;
      padded = padded2;
    }
    evslcu_free(perm);
    evslcu_free(cptr2);
    evslcu_free(cw2);
  }
  evslcu_free(csize);
  if (rc) return rc;
  // uniform chunk width: the filter kernels compute row offsets instead of
  // loading them (one dependent load less per row)
  {
    int *hcw = (int *)malloc(sizeof(int) * (size_t)nch);
    M->ellw = 0;
    if (hcw && !evslcu_d2h(hcw, M->cw, sizeof(int) * (size_t)nch)) {
      int u = hcw[0], mx = 0;
      for (int c = 0; c < nch; ++c) {
        if (hcw[c] != u) u = 0;
        mx = std::max(mx, hcw[c]);
      }
      M->ellw = u > 0 ? u : 0;
      M->maxw = mx;
    }
    free(hcw);
  }
  M->padded = padded;
  const size_t cap = (size_t)std::max(padded, 1LL);
  const size_t colb = M->ifmt ? sizeof(short) : sizeof(int);
  const size_t valb = M->vfmt ? sizeof(float) : sizeof(double);
  // scol and sval in one allocation so that one L2 access-policy window
  // covers the stored matrix
  const size_t colbytes = (colb * cap + 255) / 256 * 256;
  M->sell_bytes = colbytes + valb * cap;
  M->sell_block = evslcu_malloc(M->sell_bytes);
  if (!M->sell_block) return fail(EVSLCU_ERR_NOMEM, "SELL build: out of device memory (%lld slots)", padded);
  M->scol = M->sell_block;
  M->sval = (char *)M->sell_block + colbytes;
  const int g = grid_for(32LL * nch);
  if (M->vfmt && M->ifmt)
    k_sell_fill<float, short><<<g, kThreads, 0, stream()>>>(n, nch, M->ia, M->ja, M->a, M->perm, M->cptr, M->cw,
                                                            (short *)M->scol, (float *)M->sval);
  else if (M->vfmt)
    k_sell_fill<float, int><<<g, kThreads, 0, stream()>>>(n, nch, M->ia, M->ja, M->a, M->perm, M->cptr, M->cw,
                                                          (int *)M->scol, (float *)M->sval);
  else if (M->ifmt)
    k_sell_fill<double, short><<<g, kThreads, 0, stream()>>>(n, nch, M->ia, M->ja, M->a, M->perm, M->cptr, M->cw,
                                                             (short *)M->scol, (double *)M->sval);
  else
    k_sell_fill<double, int><<<g, kThreads, 0, stream()>>>(n, nch, M->ia, M->ja, M->a, M->perm, M->cptr, M->cw,
                                                           (int *)M->scol, (double *)M->sval);
  return launched("k_sell_fill");
}

// Column-split copy: P ranges of `width` columns, each a SELL-C-sigma with a
// 256-row sort window over the rows' lengths in that range.
int build_xsplit_device(evslcu_mat *M, int P, int width, evslcu_xsplit *X) {
  const int n = M->n, nch = (n + 31) / 32;
  if (P < 1 || P > evslcu_xsplit::kMaxRanges || width < 1 || (long long)P * width < n)
    return fail(EVSLCU_ERR_ARG, "column-split copy: bad range count %d or width %d", P, width);
  int *beg = (int *)evslcu_malloc(sizeof(int) * (size_t)P * n);
  int *len = (int *)evslcu_malloc(sizeof(int) * (size_t)P * n);
  int *bad = (int *)evslcu_malloc(sizeof(int));
  long long *csize = (long long *)evslcu_malloc(sizeof(long long) * (size_t)nch);
  int rc = (beg && len && bad && csize) ? 0 : fail(EVSLCU_ERR_NOMEM, "column-split copy: out of device memory");
  if (!rc) rc = evslcu_memset(bad, 0, sizeof(int));
  if (!rc) {
    k_xs_bounds<<<grid_for(n), kThreads, 0, stream()>>>(n, M->ia, M->ja, P, width, beg, len, bad);
    rc = launched("k_xs_bounds");
  }
  int hbad = 0;
  if (!rc) rc = evslcu_d2h(&hbad, bad, sizeof(int));
  if (!rc && hbad) {
    M->xs_bad = 1;
    rc = fail(EVSLCU_ERR_ARG, "column-split copy needs strictly increasing column indices in every row");
  }
  X->P = P;
  X->width = width;
  X->nch = nch;
  X->slots = 0;
  for (int p = 0; !rc && p < P; ++p) {
    const LenArr lp{len + (size_t)p * n};
    X->perm[p] = (int *)evslcu_malloc(sizeof(int) * 32 * (size_t)nch);
    X->cw[p] = (int *)evslcu_malloc(sizeof(int) * (size_t)nch);
    X->cptr[p] = (long long *)evslcu_malloc(sizeof(long long) * ((size_t)nch + 1));
    if (!X->perm[p] || !X->cw[p] || !X->cptr[p]) rc = fail(EVSLCU_ERR_NOMEM, "column-split copy: out of device memory");
    if (!rc) rc = evslcu_memset(X->perm[p], 0, sizeof(int) * 32 * (size_t)nch);
    if (!rc) rc = launch_sigma_sort(n, 256, lp, X->perm[p]);
    if (!rc) {
      k_chunk_width<<<grid_for(nch), kThreads, 0, stream()>>>(n, nch, lp, X->perm[p], X->cw[p], csize);
      rc = launched("k_chunk_width");
    }
    if (!rc) rc = scan_exclusive<long long, long long>(csize, nch, X->cptr[p]);
    long long sp = 0;
    if (!rc) rc = evslcu_d2h(&sp, X->cptr[p] + nch, sizeof(long long));
    if (!rc) {
      const size_t cap = (size_t)std::max(sp, 1LL);
      X->col[p] = (int *)evslcu_malloc(sizeof(int) * cap);
      X->val[p] = (double *)evslcu_malloc(sizeof(double) * cap);
      if (!X->col[p] || !X->val[p]) rc = fail(EVSLCU_ERR_NOMEM, "column-split copy: out of device memory");
    }
    if (!rc) {
      k_xs_fill<<<grid_for(32LL * nch), kThreads, 0, stream()>>>(n, nch, beg + (size_t)p * n, len + (size_t)p * n,
                                                                M->ja, M->a, X->perm[p], X->cptr[p], X->cw[p],
                                                                X->col[p], X->val[p]);
      rc = launched("k_xs_fill");
    }
    X->slots += sp;
  }
  evslcu_free(beg);
  evslcu_free(len);
  evslcu_free(bad);
  evslcu_free(csize);
  return rc;
}

void xsplit_free(evslcu_mat *M) {
  for (evslcu_xsplit *&X : M->xs) {
    if (!X) continue;
    for (int p = 0; p < evslcu_xsplit::kMaxRanges; ++p) {
      evslcu_free(X->cptr[p]);
      evslcu_free(X->cw[p]);
      evslcu_free(X->perm[p]);
      evslcu_free(X->col[p]);
      evslcu_free(X->val[p]);
      evslcu_free(X->val32[p]);
    }
    delete X;
    X = nullptr;
  }
  evslcu_free(M->xs_acc);
  M->xs_acc = nullptr;
}

}  // namespace evslcu

using namespace evslcu;

extern "C" {

int evslcu_set_sell_sigma(int sigma) {
  if (sigma < -1 || (sigma > 0 && (sigma < 32 || sigma > 4096 || (sigma & (sigma - 1)))))
    return fail(EVSLCU_ERR_ARG, "SELL sort window must be -1 (automatic), 0 (off) or a power of two from 32 to 4096");
  g_sell_sigma = sigma;
  return 0;
}

int evslcu_mat_sell_layout(const evslcu_mat *A, int *sigma, long long *padded, long long *padded_plain) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  if (sigma) *sigma = A->perm ? A->sigma : 0;
  if (padded) *padded = A->padded;
  if (padded_plain) *padded_plain = A->padded_plain;
  return 0;
}

int evslcu_coo_to_csr(int n, long long nnz, const int *ir, const int *jc, const double *vv, int base, int **ia_out,
                      int **ja_out, double **a_out) {
  if (n <= 0 || nnz < 0 || nnz > 0x7fffffffLL || (nnz > 0 && (!ir || !jc || !vv)) || !ia_out || !ja_out || !a_out)
    return fail(EVSLCU_ERR_ARG, "coo_to_csr: bad arguments (n=%d nnz=%lld)", n, nnz);
  *ia_out = nullptr;
  *ja_out = nullptr;
  *a_out = nullptr;
  int *ia = (int *)evslcu_malloc(sizeof(int) * ((size_t)n + 1));
  int *ja = (int *)evslcu_malloc(sizeof(int) * (size_t)std::max(nnz, 1LL));
  double *a = (double *)evslcu_malloc(sizeof(double) * (size_t)std::max(nnz, 1LL));
  int *cnt = (int *)evslcu_malloc(sizeof(int) * (size_t)n + 2 * sizeof(int));
  unsigned long long *keys = (unsigned long long *)evslcu_malloc(sizeof(unsigned long long) * 2 * (size_t)std::max(nnz, 1LL));
  int *rowid = (int *)evslcu_malloc(sizeof(int) * (size_t)std::max(nnz, 1LL));
  unsigned long long *bad = (unsigned long long *)evslcu_malloc(sizeof(unsigned long long));
  int rc = 0;
  if (!ia || !ja || !a || !cnt || !keys || !rowid || !bad) rc = fail(EVSLCU_ERR_NOMEM, "coo_to_csr: out of device memory");
  const unsigned long long none = ~0ull;
  unsigned long long hb = none;
  int *maxlen = cnt + n;
  const int gz = grid_for(std::max(nnz, 1LL));
  if (!rc) rc = evslcu_h2d(bad, &none, sizeof(none));
  if (!rc && nnz > 0) {
    k_coo_check<<<gz, kThreads, 0, stream()>>>(nnz, ir, jc, n, base, bad);
    rc = launched("k_coo_check");
    if (!rc) rc = evslcu_d2h(&hb, bad, sizeof(hb));
    if (!rc && hb != none) {
      int r = 0, c = 0;
      evslcu_d2h(&r, ir + hb, sizeof(int));
      evslcu_d2h(&c, jc + hb, sizeof(int));
      rc = fail(EVSLCU_ERR_ARG, "COO entry %llu has index (%d, %d) outside the %d x %d matrix (base %d)", hb, r, c, n,
                n, base);
    }
  }
  if (!rc) rc = evslcu_memset(cnt, 0, sizeof(int) * (size_t)n + 2 * sizeof(int));
  if (!rc && nnz > 0) {
    k_coo_count<<<gz, kThreads, 0, stream()>>>(nnz, ir, base, cnt);
    rc = launched("k_coo_count");
  }
  if (!rc) rc = scan_exclusive<int, int>(cnt, n, ia);
  int hmax = 0;
  if (!rc && nnz > 0) {
    k_max_len<<<grid_for(n), kThreads, 0, stream()>>>(n, ia, maxlen);
    rc = launched("k_max_len");
    if (!rc) rc = evslcu_d2h(&hmax, maxlen, sizeof(int));
    if (!rc) rc = evslcu_memset(cnt, 0, sizeof(int) * (size_t)n);
    if (!rc) {
      k_coo_scatter<<<gz, kThreads, 0, stream()>>>(nnz, ir, jc, base, ia, cnt, keys, rowid);
      rc = launched("k_coo_scatter");
    }
    unsigned long long *cur = keys, *nxt = keys + nnz;
    for (long long w = 1; !rc && w < hmax; w *= 2) {
      k_row_merge<<<gz, kThreads, 0, stream()>>>(nnz, ia, rowid, cur, nxt, w);
      rc = launched("k_row_merge");
      std::swap(cur, nxt);
    }
    if (!rc) {
      k_coo_gather<<<gz, kThreads, 0, stream()>>>(nnz, cur, vv, ja, a);
      rc = launched("k_coo_gather");
    }
  }
  if (!rc) rc = evslcu_sync();
  evslcu_free(cnt);
  evslcu_free(keys);
  evslcu_free(rowid);
  evslcu_free(bad);
  if (rc) {
    evslcu_free(ia);
    evslcu_free(ja);
    evslcu_free(a);
    return rc;
  }
  *ia_out = ia;
  *ja_out = ja;
  *a_out = a;
  return 0;
}

}  // extern "C"
