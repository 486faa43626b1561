// Device representation of the registered sparse matrix and the row kernels
// shared by the SpMV, filter and KPM kernels.
#pragma once

#include "common.cuh"

// Prepared matrix.  The filter uses SELL-32: rows in chunks of 32, entries of
// a chunk stored column-major (entry j of lane l at cptr[c] + 32 j + l),
// chunks padded to their longest row with zero values pointing at the row
// itself.  Storage is compressed losslessly when the matrix allows it:
//   vfmt 1: values stored as float because every value is exactly a float;
//   ifmt 1: columns stored as int16 offsets from the row (|col-row| < 32768).
// Every variant multiplies in FP64 in the same order, so results are
// identical bit for bit across variants.
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
  int wave = 0;             // 1: pipelined single-launch filter (wavefilter.cu)
  unsigned *wave_ctl = nullptr;
  size_t wave_ctl_words = 0;
  double *wave_mu = nullptr;
  int wave_mu_cap = 0;
  int kernel = 0;      // 0 SELL-32, 1 CSR (thread per row)
  int persistent = 0;  // 1: single cooperative launch per filter application
};

namespace evslcu {

// Validates M's device CSR and builds its SELL-32 copy on the device
// (ingest.cu).
int build_sell_device(evslcu_mat *M, int allow_compress);

template <class VT, class IT>
struct SellT {
  int n;
  const long long *__restrict__ cptr;
  const int *__restrict__ cw;
  const IT *__restrict__ col;
  const VT *__restrict__ val;
  int ellw;  // > 0: every chunk has this width (offsets computed, not loaded)
};

// Start of row r's entries and the width of its chunk.
template <class VT, class IT>
__device__ __forceinline__ void row_start(const SellT<VT, IT> &A, int r, long long &p, int &w) {
  const int c = r >> 5;
  if (A.ellw > 0) {
    w = A.ellw;
    p = (long long)c * 32 * A.ellw + (r & 31);
  } else {
    p = A.cptr[c] + (r & 31);
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

// Row r of A times x, summed left to right with rounded multiply and add.
template <bool COHERENT, class VT, class IT>
__device__ __forceinline__ double row_dot(const SellT<VT, IT> &A, int r, const double *x) {
  long long p;
  int w;
  row_start(A, r, p, w);
  double acc = 0.0;
#pragma unroll 4
  for (int j = 0; j < w; ++j, p += 32) {
    const double v = (double)__ldg(A.val + p);
    const int col = decode_col(__ldg(A.col + p), r);
    acc = __dadd_rn(acc, __dmul_rn(v, ldx<COHERENT>(x + col)));
  }
  return acc;
}

// Rows r0 and r1 = r0 + 32 (same lane of chunks c and c+1) with their loads
// interleaved: two independent dependency chains per thread.  Each row is
// still summed left to right, so results equal row_dot's.
template <bool COHERENT, class VT, class IT>
__device__ __forceinline__ void row_dot2(const SellT<VT, IT> &A, int r0, bool has1, const double *x, double &acc0,
                                         double &acc1) {
  long long p0, p1 = 0;
  int w0, w1 = 0;
  row_start(A, r0, p0, w0);
  if (has1) row_start(A, r0 + 32, p1, w1);
  const int r1 = r0 + 32;
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

// Calls f(value, column) for the entries of row r, left to right.
template <class VT, class IT, class F>
__device__ __forceinline__ void row_for_each(const SellT<VT, IT> &A, int r, F &&f) {
  long long p;
  int w;
  row_start(A, r, p, w);
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

template <class VT, class IT>
inline SellT<VT, IT> sell_view(const evslcu_mat *A) {
  return SellT<VT, IT>{A->n, A->cptr, A->cw, (const IT *)A->scol, (const VT *)A->sval, A->ellw};
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
