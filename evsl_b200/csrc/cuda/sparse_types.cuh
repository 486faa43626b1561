// Device representation of the registered sparse matrix and the row kernels
// shared by the SpMV, filter and KPM kernels.
#pragma once

#include "common.cuh"

// Prepared matrix.  The filter uses SELL-C-sigma with C = 32: rows in chunks
// of 32 slots, entries of a chunk stored column-major (entry j of slot l at
// cptr[c] + 32 j + l), chunks padded to their longest row with zero values
// pointing at the row itself.  When the row lengths vary (general sparse
// matrices), the rows of each window of sigma consecutive rows are sorted by
// length (longest first) before they are cut into chunks, so that the rows
// of a chunk have nearly equal lengths and padding is small; perm[s] is then
// the row stored in slot s (a permutation inside each window).  Vectors stay
// in the original row order: a kernel reads and writes row perm[s] for slot
// s.  Each row's entries keep their CSR order, so row sums are unchanged.
// Storage is compressed losslessly when the matrix allows it:
//   vfmt 1: values stored as float because every value is exactly a float;
//   ifmt 1: columns stored as int16 offsets from the row (|col-row| < 32768).
// Every variant multiplies in FP64 in the same order, so results are
// identical bit for bit across variants.
struct evslcu_panels;  // column-panel layout (panel.cu)

// Column-split SELL-C-sigma copy for the multi-column filter on large
// general matrices (built by build_xsplit_device, ingest.cu).  The columns
// are cut into P >= 1 ranges of `width` consecutive columns; range p holds, for
// every row, the row's entries whose column lies in the range, in CSR order,
// stored as its own SELL-C-sigma (chunks of 32 slots, rows of each 256-row
// window sorted by their length in this range, slot -> row map perm).
// Padding slots carry column -1 and are skipped.  A degree step of a
// B-column block then runs range by range: the rows of x a range gathers
// from (width x B values) stay in L2 while the range is processed, and each
// row's running sum is carried from range to range in a partial-sum block.
// Ranges are visited in column order and the entries of a range in CSR
// order, so each row is still summed left to right in its CSR order.
struct evslcu_xsplit {
  static constexpr int kMaxRanges = 32;
  int P = 0;
  int width = 0;  // columns per range (the last one may be shorter)
  int nch = 0;    // chunks per range
  long long slots = 0;  // stored slots over all ranges
  long long *cptr[kMaxRanges] = {};  // nch + 1 chunk offsets of each range
  int *cw[kMaxRanges] = {};          // chunk widths
  int *perm[kMaxRanges] = {};        // slot -> row (32 nch entries)
  int *col[kMaxRanges] = {};         // column of each stored slot (-1: padding)
  double *val[kMaxRanges] = {};      // value of each stored slot
  float *val32[kMaxRanges] = {};     // FP32 copy, made on first FP32 use
};

struct evslcu_mat {
  int n = 0;
  long long nnz = 0;
  const int *ia = nullptr;  // CSR on the device
  const int *ja = nullptr;
  const double *a = nullptr;
  bool own_csr = false;
  int nchunks = 0;
  long long padded = 0;
  long long *cptr = nullptr;
  int *cw = nullptr;
  int vfmt = 0;
  int ifmt = 0;
  void *scol = nullptr;
  void *sval = nullptr;
  void *sell_block = nullptr;  // one allocation holding scol and sval (L2 window)
  size_t sell_bytes = 0;
  void *sval32 = nullptr;  // FP32 copy of sval for the FP32 filter (when vfmt == 0)
  signed char mf_variant[2][5] = {{-1, -1, -1, -1, -1}, {-1, -1, -1, -1, -1}};  // tuned kernel per (fp32, log2 B)
  float mf_cost_us[2][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};  // its measured time per degree step
  long long bandwidth = 0;  // max |col - row| over the stored entries
  int ellw = 0;             // > 0: every SELL-32 chunk has this width
  int maxw = 0;             // widest SELL-32 chunk
  int *perm = nullptr;      // slot -> row when the rows are sigma-sorted (null: slot s holds row s)
  int sigma = 0;            // window of the length sort (0: rows in their original order)
  long long padded_plain = 0;  // stored slots the unsorted SELL-32 layout would need
  int wave = 0;             // 1: pipelined single-launch filter (wavefilter.cu)
  unsigned *wave_ctl = nullptr;
  size_t wave_ctl_words = 0;
  double *wave_mu = nullptr;
  int wave_mu_cap = 0;
  int kernel = 0;      // 0 SELL-32, 1 CSR (thread per row)
  int persistent = 0;  // 1: single cooperative launch per filter application
  // Row-pattern dictionary, built when the rows take few distinct forms
  // (structured-grid operators): row r holds the entries of pattern
  // pat_id[r], each a (value, column - r) pair, in the CSR order of the row.
  unsigned short *pat_id = nullptr;
  void *pat_table = nullptr;  // int2 {first entry, count} per pattern, then double2 entries
  int npat = 0;
  int pat_entries = 0;
  int pat_maxlen = 0;  // longest pattern
  int pat_f32 = 0;     // 1: every table value is exactly a float (packed entries exist)
  int pat_cent = -1;   // first entry of the table's copy in the constant pool (-1: not there)
  int pat_chdr = -1;   // first header there
  unsigned *pat_desc = nullptr;  // per row: (first pool entry << 8) | count, when in the pool
  int use_pat = 0;     // 1: the FP64 single-vector filter and SpMV read the dictionary
  evslcu_panels *pn64 = nullptr;  // column-panel layout for the FP64 kernels (large general matrices)
  evslcu_panels *pn32 = nullptr;  // the same for the FP32 kernels
  evslcu_xsplit *xs[6] = {};      // column-split copies with 1, 2, 4, 8, 16, 32 ranges (null: not built)
  void *xs_acc = nullptr;         // partial-sum block of the column-split filter (n x 16 doubles)
  int xs_bad = 0;                 // 1: no column-split copy (a row's columns are not increasing)
  int cheb_variant = -1;      // single-vector filter kernel chosen by timing (-1: not yet)
  float cheb_us[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // measured time per degree step of each variant
  int cheb_grid = 0;                      // tuned block limit per degree step (0: one row per thread)
  float cheb_best_us = 0.0f;              // time per degree step of the chosen variant and grid
};

namespace evslcu {

// Validates M's device CSR and builds its SELL-32 copy on the device
// (ingest.cu).
int build_sell_device(evslcu_mat *M, int allow_compress);
// Builds M's row-pattern dictionary when its rows take at most 1024
// distinct forms; leaves M->pat_id null otherwise (ingest.cu).
int build_patterns_device(evslcu_mat *M);
// Builds M's column-split copy with P column ranges of `width` columns into X
// (ingest.cu).  Fails with EVSLCU_ERR_ARG, and sets M->xs_bad, when a row's
// column indices are not strictly increasing.
int build_xsplit_device(evslcu_mat *M, int P, int width, evslcu_xsplit *X);
void xsplit_free(evslcu_mat *M);
// The column-split copy for blocks of row_bytes bytes per row, built on first
// use (multifilter.cu); null when the matrix has none (or is smaller than
// the size worth a copy, unless any_size).
const evslcu_xsplit *xsplit_for(evslcu_mat *M, size_t row_bytes, bool any_size = false);

// One column range of a column-split copy, as the kernels read it.
template <class VT>
struct XsRange {
  int n;
  const long long *__restrict__ cptr;
  const int *__restrict__ cw;
  const int *__restrict__ col;
  const VT *__restrict__ val;
  const int *__restrict__ perm;
};

template <class VT, class IT>
struct SellT {
  int n;
  const long long *__restrict__ cptr;
  const int *__restrict__ cw;
  const IT *__restrict__ col;
  const VT *__restrict__ val;
  int ellw;  // > 0: every chunk has this width (offsets computed, not loaded)
  const int *__restrict__ perm;  // slot -> row (null: identity)
};

// The row stored in slot s (the views without a slot order map s to s).
template <class VT, class IT>
__device__ __forceinline__ int row_of(const SellT<VT, IT> &A, int s) {
  return A.perm ? __ldg(A.perm + s) : s;
}
template <class V>
__device__ __forceinline__ int row_of(const V &, int s) {
  return s;
}

// Start of slot s's entries and the width of its chunk.
template <class VT, class IT>
__device__ __forceinline__ void row_start(const SellT<VT, IT> &A, int s, long long &p, int &w) {
  const int c = s >> 5;
  if (A.ellw > 0) {
    w = A.ellw;
    p = (long long)c * 32 * A.ellw + (s & 31);
  } else {
    p = A.cptr[c] + (s & 31);
    w = A.cw[c];
  }
}

struct CsrView {
  int n;
  const int *__restrict__ ia;
  const int *__restrict__ ja;
  const double *__restrict__ a;
};

__device__ __forceinline__ int decode_col(int c, int) { return c; }
__device__ __forceinline__ int decode_col(short c, int r) { return r + (int)c; }

// Load from a vector that this kernel may have written (bypass L1).
template <bool COHERENT>
__device__ __forceinline__ double ldx(const double *p) {
  if (COHERENT) return __ldcg(p);
  return __ldg(p);
}

// The row in slot s of A times x, summed left to right with rounded multiply
// and add.  Entries are taken 4 at a time with their gathers in flight
// together, and the next 4 stored entries are loaded while those gathers are
// outstanding; the sum is still formed entry by entry in row order.
template <bool COHERENT, class VT, class IT>
__device__ __forceinline__ double row_dot(const SellT<VT, IT> &A, int s, const double *x) {
  constexpr int U = 4;
  long long p;
  int w;
  row_start(A, s, p, w);
  const int r = row_of(A, s);
  VT v[U];
  int col[U];
#pragma unroll
  for (int u = 0; u < U; ++u)
    if (u < w) {
      v[u] = __ldg(A.val + p + 32 * u);
      col[u] = decode_col(__ldg(A.col + p + 32 * u), r);
    }
  double acc = 0.0;
  for (int j = 0; j < w; j += U, p += 32 * U) {
    double g[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (j + u < w) g[u] = ldx<COHERENT>(x + col[u]);
    VT vn[U];
    int cn[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (j + U + u < w) {
        vn[u] = __ldg(A.val + p + 32 * (U + u));
        cn[u] = decode_col(__ldg(A.col + p + 32 * (U + u)), r);
      }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (j + u < w) acc = __dadd_rn(acc, __dmul_rn((double)v[u], g[u]));
#pragma unroll
    for (int u = 0; u < U; ++u) {
      v[u] = vn[u];
      col[u] = cn[u];
    }
  }
  return acc;
}

// Slots s0 and s0 + 32 (same lane of chunks c and c+1) with their loads
// interleaved: two independent dependency chains per thread.  Each row is
// still summed left to right, so results equal row_dot's.  A slot past the
// last row (has0 / has1 false) reads nothing and gives 0.
template <bool COHERENT, class VT, class IT>
__device__ __forceinline__ void row_dot2(const SellT<VT, IT> &A, int s0, bool has0, bool has1, const double *x,
                                         double &acc0, double &acc1) {
  long long p0 = 0, p1 = 0;
  int w0 = 0, w1 = 0;
  if (has0) row_start(A, s0, p0, w0);
  if (has1) row_start(A, s0 + 32, p1, w1);
  const int r0 = has0 ? row_of(A, s0) : 0;
  const int r1 = has1 ? row_of(A, s0 + 32) : 0;
  acc0 = 0.0;
  acc1 = 0.0;
  const int wm = w0 > w1 ? w0 : w1;
#pragma unroll 4
  for (int j = 0; j < wm; ++j, p0 += 32, p1 += 32) {
    if (j < w0) {
      const double v = (double)__ldg(A.val + p0);
      const int col = decode_col(__ldg(A.col + p0), r0);
      acc0 = __dadd_rn(acc0, __dmul_rn(v, ldx<COHERENT>(x + col)));
    }
    if (j < w1) {
      const double v = (double)__ldg(A.val + p1);
      const int col = decode_col(__ldg(A.col + p1), r1);
      acc1 = __dadd_rn(acc1, __dmul_rn(v, ldx<COHERENT>(x + col)));
    }
  }
}

// Calls f(value, column) for the entries of the row in slot s, left to right.
template <class VT, class IT, class F>
__device__ __forceinline__ void row_for_each(const SellT<VT, IT> &A, int s, F &&f) {
  long long p;
  int w;
  row_start(A, s, p, w);
  const int r = row_of(A, s);
  for (int j = 0; j < w; ++j, p += 32) f((double)__ldg(A.val + p), decode_col(__ldg(A.col + p), r));
}

template <class F>
__device__ __forceinline__ void row_for_each(const struct CsrView &A, int r, F &&f);

template <bool COHERENT>
__device__ __forceinline__ double row_dot(const CsrView &A, int r, const double *x) {
  const int b = A.ia[r], e = A.ia[r + 1];
  double acc = 0.0;
#pragma unroll 4
  for (int j = b; j < e; ++j) acc = __dadd_rn(acc, __dmul_rn(__ldg(A.a + j), ldx<COHERENT>(x + __ldg(A.ja + j))));
  return acc;
}

template <class F>
__device__ __forceinline__ void row_for_each(const CsrView &A, int r, F &&f) {
  const int b = A.ia[r], e = A.ia[r + 1];
  for (int j = b; j < e; ++j) f(__ldg(A.a + j), __ldg(A.ja + j));
}

// Row-pattern dictionary view.  The table is a few KB and is read through the
// L1 cache; per row only the 2-byte pattern id comes from memory.
struct PatView {
  int n;
  const unsigned short *__restrict__ pid;
  const int2 *__restrict__ hdr;     // {first entry, count} per pattern
  const double2 *__restrict__ ent;  // {value, column offset as 64-bit integer bits}
};

// Same products in the same order as the CSR row (no padding entries).
template <bool COHERENT>
__device__ __forceinline__ double row_dot(const PatView &A, int r, const double *x) {
  const int2 h = __ldg(A.hdr + __ldg(A.pid + r));
  const double *xr = x + r;
  double acc = 0.0;
#pragma unroll 4
  for (int j = 0; j < h.y; ++j) {
    const double2 e = __ldg(A.ent + h.x + j);
    const int off = (int)__double_as_longlong(e.y);
    acc = __dadd_rn(acc, __dmul_rn(e.x, ldx<COHERENT>(xr + off)));
  }
  return acc;
}

// Row products with every load of the row issued before the first add:
// widths up to WMAX are unrolled and predicated, so the row's gathers are in
// flight together instead of one per loop trip.  Same order of rounded
// operations as row_dot.
template <int WMAX, bool COHERENT>
__device__ __forceinline__ double row_dot_w(const PatView &A, int r, const double *x) {
  const int2 h = __ldg(A.hdr + __ldg(A.pid + r));
  const double *xr = x + r;
  double g[WMAX];
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < h.y) g[j] = ldx<COHERENT>(xr + (int)__double_as_longlong(__ldg(&A.ent[h.x + j].y)));
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < h.y) acc = __dadd_rn(acc, __dmul_rn(__ldg(&A.ent[h.x + j].x), g[j]));
  return acc;
}

template <int WMAX, bool COHERENT, class VT, class IT>
__device__ __forceinline__ double row_dot_w(const SellT<VT, IT> &A, int s, const double *x) {
  long long p;
  int w;
  row_start(A, s, p, w);
  const int r = row_of(A, s);
  VT v[WMAX];
  double g[WMAX];
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < w) {
      v[j] = __ldg(A.val + p + 32 * j);
      g[j] = ldx<COHERENT>(x + decode_col(__ldg(A.col + p + 32 * j), r));
    }
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < w) acc = __dadd_rn(acc, __dmul_rn((double)v[j], g[j]));
  return acc;
}

template <int WMAX, bool COHERENT>
__device__ __forceinline__ double row_dot_w(const CsrView &A, int r, const double *x) {
  return row_dot<COHERENT>(A, r, x);
}

// WMAX 0: the loop form (any width).
template <int WMAX, bool COHERENT, class M>
__device__ __forceinline__ double row_dot_any(const M &A, int r, const double *x) {
  if constexpr (WMAX == 0)
    return row_dot<COHERENT>(A, r, x);
  else
    return row_dot_w<WMAX, COHERENT>(A, r, x);
}

// Packed table (every value exactly a float): one 64-bit entry per stored
// value, float bits in the high word, column offset in the low word; the
// float widens to the same double, so products are unchanged.  One table
// load per entry instead of two.
struct PatPView {
  int n;
  const unsigned short *__restrict__ pid;
  const int2 *__restrict__ hdr;
  const unsigned long long *__restrict__ pk;
};

__device__ __forceinline__ double pat_val(unsigned long long e) { return (double)__uint_as_float((unsigned)(e >> 32)); }
__device__ __forceinline__ int pat_off(unsigned long long e) { return (int)(unsigned)(e & 0xffffffffULL); }

template <bool COHERENT>
__device__ __forceinline__ double row_dot(const PatPView &A, int r, const double *x) {
  const int2 h = __ldg(A.hdr + __ldg(A.pid + r));
  const double *xr = x + r;
  double acc = 0.0;
#pragma unroll 4
  for (int j = 0; j < h.y; ++j) {
    const unsigned long long e = __ldg(A.pk + h.x + j);
    acc = __dadd_rn(acc, __dmul_rn(pat_val(e), ldx<COHERENT>(xr + pat_off(e))));
  }
  return acc;
}

template <int WMAX, bool COHERENT>
__device__ __forceinline__ double row_dot_w(const PatPView &A, int r, const double *x) {
  const int2 h = __ldg(A.hdr + __ldg(A.pid + r));
  const double *xr = x + r;
  unsigned long long e[WMAX];
  double g[WMAX];
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < h.y) {
      e[j] = __ldg(A.pk + h.x + j);
      g[j] = ldx<COHERENT>(xr + pat_off(e[j]));
    }
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < h.y) acc = __dadd_rn(acc, __dmul_rn(pat_val(e[j]), g[j]));
  return acc;
}

// Bytes of the global table: headers (padded to 16), double2 entries, then
// the packed entries.
inline size_t pat_hdr_bytes(int npat) { return ((size_t)npat * sizeof(int2) + 15) / 16 * 16; }

inline PatPView pat_pview(const evslcu_mat *A) {
  const size_t hbytes = pat_hdr_bytes(A->npat);
  return PatPView{A->n, A->pat_id, (const int2 *)A->pat_table,
                  (const unsigned long long *)((const char *)A->pat_table + hbytes + 16 * (size_t)A->pat_entries)};
}

inline PatView pat_view(const evslcu_mat *A) {
  const size_t hbytes = ((size_t)A->npat * sizeof(int2) + 15) / 16 * 16;
  return PatView{A->n, A->pat_id, (const int2 *)A->pat_table,
                 (const double2 *)((const char *)A->pat_table + hbytes)};
}

template <class VT, class IT>
inline SellT<VT, IT> sell_view(const evslcu_mat *A) {
  return SellT<VT, IT>{A->n, A->cptr, A->cw, (const IT *)A->scol, (const VT *)A->sval, A->ellw, A->perm};
}

// The same storage with the values read from another array (the FP32 copy).
template <class VT, class IT>
inline SellT<VT, IT> sell_view_vals(const evslcu_mat *A, const void *vals) {
  return SellT<VT, IT>{A->n, A->cptr, A->cw, (const IT *)A->scol, (const VT *)vals, A->ellw, A->perm};
}

inline CsrView csr_view(const evslcu_mat *A) { return CsrView{A->n, A->ia, A->ja, A->a}; }

// Calls f(view) with the matrix's storage variant (SELL-32 or CSR).
template <class F>
inline int with_view(const evslcu_mat *A, F &&f) {
  if (A->kernel == 1) return f(csr_view(A));
  if (A->vfmt == 0 && A->ifmt == 0) return f(sell_view<double, int>(A));
  if (A->vfmt == 0 && A->ifmt == 1) return f(sell_view<double, short>(A));
  if (A->vfmt == 1 && A->ifmt == 0) return f(sell_view<float, int>(A));
  return f(sell_view<float, short>(A));
}

// Column-panel layout (panel.cu): x staged through shared memory panel by
// panel, for large matrices whose gathers miss every cache line.
bool panel_candidate(const evslcu_mat *M);
int panel_build(evslcu_mat *M, int fp32);
void panel_free(evslcu_mat *M);
int panel_cheb_step(const evslcu_mat *M, bool first, bool epi, const double *vk, const double *vkm1, double *out,
                    double *y, double t, double ncc, double s, double mu0, const double *zold, double nbeta,
                    const double *dotv, double *dout);
template <class VT>
int panel_mf_step(const evslcu_mat *M, int k, const VT *vk, const VT *vkm1, VT *out, VT *y, const VT *coef);

// Wait limit of the pipelined filter's dependency waits (0: default).
void set_wave_wait_limit(unsigned long long polls);
void set_batch_wait_limit(unsigned long long polls);
// Pipelined single-launch filter (wavefilter.cu); work: 2n doubles.
int chebav_wave(evslcu_mat *A, const double *mu, int deg, double cc, double dd, const double *v, double *y,
                double *work);
// Per-degree filter path (sparse.cu): one fused kernel per degree.
int chebav_per_degree(const evslcu_mat *A, const double *mu, int deg, double cc, double dd, const double *v,
                      double *y, double *work, const evslcu_cheb_epi *epi);
// Filter through a user matvec callback (sparse.cu).
int chebav_user_matvec(const evslcu_op *op, const double *mu, int deg, double cc, double dd, const double *v,
                       double *y, double *work, const evslcu_cheb_epi *epi);
int launch_scale_copy(int n, double a, const double *x, double *y);
int launch_lan_epi(int n, const evslcu_cheb_epi *epi, double *y);

}  // namespace evslcu
