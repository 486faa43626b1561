// Chebyshev filter applied to many columns at once, each with its own
// polynomial (mu, degree, cc, dd): the block form of ChebAv
// (SRC/chebpoly.c:519-598) used by the batched slice solver.
//
// Columns are interleaved in HBM as [n][B] (the B values of a row are
// contiguous), so each stored entry of A is read once per degree for all B
// columns and the gather x[col] is one contiguous B-value load.  One thread
// per SELL-32 row, B accumulators in registers.
//
//   FP64 mode: rounded multiply and add in the reference's order, so every
//   column equals ChebAv of that column bit for bit, whatever B and the
//   other columns are.
//   FP32 mode: A's values and the recurrence in float with float
//   accumulation (fused multiply-add); deterministic per column as well.
//
// A column whose degree is below the current degree is masked: its y is
// final and is not written again.
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "sparse_types.cuh"

namespace evslcu {

namespace {

constexpr int kMaxB = 16;

// Contiguous B-value loads/stores of a row of an interleaved block, as
// 16-byte (or 8-byte) vector accesses unpacked into registers.
template <bool CG, class VT, int B>
__device__ __forceinline__ void load_row_impl(const VT *p, VT (&x)[B]) {
  if constexpr (std::is_same<VT, float>::value && B % 4 == 0) {
#pragma unroll
    for (int i = 0; i < B / 4; ++i) {
      const float4 f = CG ? __ldcg(reinterpret_cast<const float4 *>(p) + i) : __ldg(reinterpret_cast<const float4 *>(p) + i);
      x[4 * i] = f.x;
      x[4 * i + 1] = f.y;
      x[4 * i + 2] = f.z;
      x[4 * i + 3] = f.w;
    }
  } else if constexpr (std::is_same<VT, float>::value && B == 2) {
    const float2 f = CG ? __ldcg(reinterpret_cast<const float2 *>(p)) : __ldg(reinterpret_cast<const float2 *>(p));
    x[0] = f.x;
    x[1] = f.y;
  } else if constexpr (std::is_same<VT, double>::value && B % 2 == 0) {
#pragma unroll
    for (int i = 0; i < B / 2; ++i) {
      const double2 f =
          CG ? __ldcg(reinterpret_cast<const double2 *>(p) + i) : __ldg(reinterpret_cast<const double2 *>(p) + i);
      x[2 * i] = f.x;
      x[2 * i + 1] = f.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < B; ++c) x[c] = CG ? __ldcg(p + c) : __ldg(p + c);
  }
}

template <class VT, int B>
__device__ __forceinline__ void load_row(const VT *p, VT (&x)[B]) {
  load_row_impl<false, VT, B>(p, x);
}

// Same for data this launch sequence writes (L2 only, no read-only path).
template <class VT, int B>
__device__ __forceinline__ void load_row_cg(const VT *p, VT (&x)[B]) {
  load_row_impl<true, VT, B>(p, x);
}

template <class VT, int B>
__device__ __forceinline__ void store_row(VT *p, const VT (&x)[B]) {
  if constexpr (std::is_same<VT, float>::value && B % 4 == 0) {
#pragma unroll
    for (int i = 0; i < B / 4; ++i)
      reinterpret_cast<float4 *>(p)[i] = make_float4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
  } else if constexpr (std::is_same<VT, float>::value && B == 2) {
    *reinterpret_cast<float2 *>(p) = make_float2(x[0], x[1]);
  } else if constexpr (std::is_same<VT, double>::value && B % 2 == 0) {
#pragma unroll
    for (int i = 0; i < B / 2; ++i) reinterpret_cast<double2 *>(p)[i] = make_double2(x[2 * i], x[2 * i + 1]);
  } else {
#pragma unroll
    for (int c = 0; c < B; ++c) p[c] = x[c];
  }
}

__device__ __forceinline__ double fmadd(double a, double b, double acc) { return __dadd_rn(acc, __dmul_rn(a, b)); }
__device__ __forceinline__ float fmadd(float a, float b, float acc) { return fmaf(a, b, acc); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }

// Coefficients of one launch sequence live in a device table, 4 values per
// (degree, column): t (1/dd at k = 1, 2/dd after), -cc, mu_k, and 1 while
// k <= deg_c (0 after: the column's y is final).  Degree 0 row: mu_0.
constexpr int kCoef = 4;

// P = pack(x_c) (converted to VT); Y = mu0_c * P.  The column pointers come
// from a device table so that a captured launch sequence can be replayed on
// other vectors.
template <class VT, int B>
__global__ void k_mf_pack(int n, int ncols, const double *const *xtab, const VT *coef0, VT *P, VT *Y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)n * B;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / B), c = (int)(i % B);
    const VT v = (c < ncols) ? (VT)xtab[c][r] : (VT)0;
    P[i] = v;
    Y[i] = mul(__ldg(coef0 + kCoef * c + 2), v);
  }
}

template <class VT, int B>
__global__ void k_mf_unpack(int n, int ncols, const VT *Y, double *const *ytab) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)n * B;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / B), c = (int)(i % B);
    if (c < ncols) ytab[c][r] = (double)Y[i];
  }
}

// Columns per thread: two doubles or four floats (one 16-byte access); a row
// is shared by B / CPT threads.
template <class VT, int B>
struct Split {
  static constexpr int CPT = (B < (int)(16 / sizeof(VT))) ? B : (int)(16 / sizeof(VT));
  static constexpr int TPR = B / CPT;
};

// One degree of the recurrence for all columns: thread (row r, part q)
// handles columns q*CPT .. q*CPT+CPT-1 of row r.
template <class VT, int B, class AV, class IT, bool FIRST>
__global__ void __launch_bounds__(kThreads)
    k_mf_step(SellT<AV, IT> A, const VT *__restrict__ vk, const VT *vkm1, VT *out, VT *__restrict__ y,
              const VT *__restrict__ coef) {
  constexpr int CPT = Split<VT, B>::CPT, TPR = Split<VT, B>::TPR;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const long long total = (long long)A.n * TPR;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
    const int r = (int)(g / TPR), q = (int)(g % TPR);
    const int cb = q * CPT;
    // this row's own values first: independent of the gathers below, so
    // their latency overlaps with them
    const long long base = (long long)r * B + cb;
    VT xr[CPT], wv[CPT], yv[CPT], vm[CPT];
    load_row<VT, CPT>(vk + base, xr);
    load_row_cg<VT, CPT>(y + base, yv);
    if (!FIRST) load_row_cg<VT, CPT>(vkm1 + base, vm);
    VT acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = (VT)0;
    const int ch = r >> 5;
    long long p = A.cptr[ch] + (r & 31);
    const int w = A.cw[ch];
    // U stored entries at a time: their gathers are in flight together,
    // then accumulated in order j = 0, 1, ...  Slots past the row's width
    // act as 0 * x[r].
    constexpr int U = 4;
    for (int j = 0; j < w; j += U, p += 32 * U) {
      VT v[U];
      int col[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (j + u < w) {
          v[u] = (VT)__ldg(A.val + p + 32 * u);
          col[u] = decode_col(__ldg(A.col + p + 32 * u), r);
        } else {
          v[u] = (VT)0;
          col[u] = r;
        }
      }
      VT x[U][CPT];
#pragma unroll
      for (int u = 0; u < U; ++u) load_row<VT, CPT>(vk + (long long)col[u] * B + cb, x[u]);
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = fmadd(v[u], x[u][c], acc[c]);
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const VT *cf = coef + kCoef * (cb + c);
      VT t = mul(__ldg(cf), add(acc[c], mul(__ldg(cf + 1), xr[c])));
      if (!FIRST) t = add(t, -vm[c]);
      wv[c] = t;
      if (__ldg(cf + 3) != (VT)0) yv[c] = add(yv[c], mul(__ldg(cf + 2), t));
    }
    store_row<VT, CPT>(out + base, wv);
    store_row<VT, CPT>(y + base, yv);
  }
}

template <class VT, int B, class AV, class IT>
int mf_step(const SellT<AV, IT> &A, int k, const VT *vk, const VT *vkm1, VT *out, VT *y, const VT *coef) {
  constexpr int TPR = Split<VT, B>::TPR;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid_for((long long)A.n * TPR, kThreads, 1 << 20));
  cfg.blockDim = dim3(kThreads);
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = (k == 1) ? cudaLaunchKernelEx(&cfg, k_mf_step<VT, B, AV, IT, true>, A, vk, vkm1, out, y, coef)
                           : cudaLaunchKernelEx(&cfg, k_mf_step<VT, B, AV, IT, false>, A, vk, vkm1, out, y, coef);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "multi-column filter launch failed: %s", cudaGetErrorString(e));
  return check_launch("k_mf_step");
}

// Number of VT values of the coefficient table of one group.
inline size_t coef_count(int B, int maxdeg) { return (size_t)(maxdeg + 1) * B * kCoef; }

// Fills the host coefficient table of one group (B columns, ncols used).
template <class VT>
void fill_coef(VT *h, int B, int ncols, const evslcu_filter_col *cols, int maxdeg) {
  memset(h, 0, sizeof(VT) * coef_count(B, maxdeg));
  for (int c = 0; c < ncols; ++c) h[kCoef * c + 2] = (VT)cols[c].mu[0];
  for (int k = 1; k <= maxdeg; ++k) {
    VT *row = h + (size_t)k * B * kCoef;
    for (int c = 0; c < B; ++c) {
      VT *e = row + kCoef * c;
      if (c < ncols) {
        const evslcu_filter_col &q = cols[c];
        e[0] = (VT)((k == 1) ? 1.0 / q.dd : 2.0 / q.dd);
        e[1] = (VT)(-q.cc);
        if (k <= q.deg) {
          e[2] = (VT)q.mu[k];
          e[3] = (VT)1;
        }
      } else {
        e[0] = (VT)1;
      }
    }
  }
}

// The launch sequence for one group of <= 16 columns: pack, one step per
// degree, unpack.  coef: the group's device coefficient table.
template <class VT, int B, class AV, class IT>
int mf_group(const SellT<AV, IT> &A, int ncols, int maxdeg, const VT *coef, const double *const *xtab,
             double *const *ytab, VT *P, VT *W0, VT *W1, VT *Y, int *nlaunch) {
  const int n = A.n;
  const int g = grid_for((long long)n * B);
  k_mf_pack<VT, B><<<g, kThreads, 0, stream()>>>(n, ncols, xtab, coef, P, Y);
  int rc = check_launch("k_mf_pack");
  VT *W[2] = {W0, W1};
  for (int k = 1; !rc && k <= maxdeg; ++k) {
    const VT *vk = (k == 1) ? P : W[(k - 2) % 2];
    const VT *vkm1 = (k == 1) ? nullptr : ((k == 2) ? P : W[(k - 1) % 2]);
    rc = mf_step<VT, B>(A, k, vk, vkm1, W[(k - 1) % 2], Y, coef + (size_t)k * B * kCoef);
  }
  if (!rc) {
    k_mf_unpack<VT, B><<<g, kThreads, 0, stream()>>>(n, ncols, Y, ytab);
    rc = check_launch("k_mf_unpack");
  }
  *nlaunch += maxdeg + 2;
  return rc;
}

template <class VT, class AV, class IT>
int mf_dispatch(const SellT<AV, IT> &A, int B, int ncols, int maxdeg, const VT *coef, const double *const *xtab,
                double *const *ytab, VT *P, VT *W0, VT *W1, VT *Y, int *nl) {
  switch (B) {
    case 1: return mf_group<VT, 1>(A, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
    case 2: return mf_group<VT, 2>(A, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
    case 4: return mf_group<VT, 4>(A, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
    case 8: return mf_group<VT, 8>(A, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
    default: return mf_group<VT, 16>(A, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
  }
}

__global__ void k_to_float(long long m, const double *src, float *dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

int group_width(int ncols) {
  int b = 1;
  while (b < ncols && b < kMaxB) b *= 2;
  return b;
}

}  // namespace

}  // namespace evslcu

using namespace evslcu;

extern "C" {

size_t evslcu_filter_columns_work(int n, int fp32, int ncols) {
  const int B = group_width(std::min(std::max(ncols, 1), kMaxB));
  const size_t blk = ((size_t)n * B * (fp32 ? sizeof(float) : sizeof(double)) + 255) / 256 * 256;
  const size_t tab = (2 * sizeof(double *) * (size_t)std::max(ncols, 1) + 255) / 256 * 256;
  return 4 * blk + tab;
}

int evslcu_mat_prepare_fp32(evslcu_mat *A) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  if (A->vfmt == 1 || A->sval32) return 0;
  A->sval32 = evslcu_malloc(sizeof(float) * (size_t)std::max(A->padded, 1LL));
  if (!A->sval32) return fail(EVSLCU_ERR_NOMEM, "FP32 copy of the matrix values: out of device memory");
  k_to_float<<<grid_for(A->padded), kThreads, 0, stream()>>>(A->padded, (const double *)A->sval, (float *)A->sval32);
  count_launch();
  return check_launch("k_to_float");
}

}  // extern "C"

namespace evslcu {
namespace {

inline int group_maxdeg(int gc, const evslcu_filter_col *cols) {
  int m = 0;
  for (int c = 0; c < gc; ++c) m = std::max(m, cols[c].deg);
  return m;
}

// Device coefficient tables of every group of the sequence, back to back.
void *coef_build(int fp32, int ncols, const evslcu_filter_col *cols, int *err) {
  size_t total = 0;
  for (int c0 = 0; c0 < ncols; c0 += kMaxB) {
    const int gc = std::min(kMaxB, ncols - c0);
    total += coef_count(group_width(gc), group_maxdeg(gc, cols + c0));
  }
  const size_t vb = fp32 ? sizeof(float) : sizeof(double);
  char *h = (char *)malloc(total * vb);
  void *d = evslcu_malloc(total * vb);
  if (!h || !d) {
    free(h);
    evslcu_free(d);
    *err = fail(EVSLCU_ERR_NOMEM, "filter coefficients: out of memory");
    return nullptr;
  }
  size_t off = 0;
  for (int c0 = 0; c0 < ncols; c0 += kMaxB) {
    const int gc = std::min(kMaxB, ncols - c0), B = group_width(gc), md = group_maxdeg(gc, cols + c0);
    if (fp32)
      fill_coef<float>((float *)(h + off * vb), B, gc, cols + c0, md);
    else
      fill_coef<double>((double *)(h + off * vb), B, gc, cols + c0, md);
    off += coef_count(B, md);
  }
  *err = evslcu_h2d(d, h, total * vb);
  free(h);
  if (*err) {
    evslcu_free(d);
    return nullptr;
  }
  return d;
}

// The whole launch sequence for ncols columns; x and y pointers are read
// from the device table tab (x[0..ncols), then y[0..ncols)); coef from
// coef_build.
int mf_sequence(const evslcu_mat *A, int fp32, int ncols, const evslcu_filter_col *cols, const void *coef,
                void *work, size_t work_bytes, const double *const *tab, int *nlaunch) {
  const int n = A->n;
  int rc = 0;
  size_t off = 0;
  for (int c0 = 0; !rc && c0 < ncols; c0 += kMaxB) {
    const int gc = std::min(kMaxB, ncols - c0);
    const int B = group_width(gc);
    const int md = group_maxdeg(gc, cols + c0);
    const size_t vb = fp32 ? sizeof(float) : sizeof(double);
    const size_t blk = ((size_t)n * B * vb + 255) / 256 * 256;
    if (4 * blk > work_bytes) return fail(EVSLCU_ERR_ARG, "filter_columns: work too small");
    char *w = (char *)work;
    const double *const *xt = tab + c0;
    double *const *yt = (double *const *)(tab + ncols + c0);
    if (fp32) {
      float *P = (float *)w, *W0 = (float *)(w + blk), *W1 = (float *)(w + 2 * blk), *Y = (float *)(w + 3 * blk);
      const float *cf = (const float *)coef + off;
      const void *vals = (A->vfmt == 1) ? A->sval : A->sval32;
      if (A->ifmt)
        rc = mf_dispatch<float>(SellT<float, short>{n, A->cptr, A->cw, (const short *)A->scol, (const float *)vals},
                                B, gc, md, cf, xt, yt, P, W0, W1, Y, nlaunch);
      else
        rc = mf_dispatch<float>(SellT<float, int>{n, A->cptr, A->cw, (const int *)A->scol, (const float *)vals}, B,
                                gc, md, cf, xt, yt, P, W0, W1, Y, nlaunch);
    } else {
      double *P = (double *)w, *W0 = (double *)(w + blk), *W1 = (double *)(w + 2 * blk), *Y = (double *)(w + 3 * blk);
      const double *cf = (const double *)coef + off;
      rc = with_view(A, [&](auto view) -> int {
        if constexpr (std::is_same<decltype(view), CsrView>::value) {
          return fail(EVSLCU_ERR_ARG, "filter_columns needs the SELL-32 storage");
        } else {
          return mf_dispatch<double>(view, B, gc, md, cf, xt, yt, P, W0, W1, Y, nlaunch);
        }
      });
    }
    off += coef_count(B, md);
  }
  return rc;
}

int check_cols(const evslcu_mat *A, int fp32, int ncols, const evslcu_filter_col *cols, int need_ptrs) {
  if (!A || ncols < 1 || !cols) return fail(EVSLCU_ERR_ARG, "filter_columns: bad arguments");
  if (A->kernel != 0) return fail(EVSLCU_ERR_ARG, "filter_columns needs the SELL-32 storage");
  if (fp32 && A->vfmt == 0 && !A->sval32) return fail(EVSLCU_ERR_STATE, "FP32 values not prepared");
  for (int c = 0; c < ncols; ++c)
    if ((need_ptrs && (!cols[c].x || !cols[c].y)) || !cols[c].mu || cols[c].deg < 0 || cols[c].dd == 0.0)
      return fail(EVSLCU_ERR_ARG, "filter_columns: bad column %d", c);
  return 0;
}

}  // namespace
}  // namespace evslcu

struct evslcu_filter_plan {
  const evslcu_mat *A;
  int fp32, ncols, nodes;
  void *coef;
  void *work;
  size_t work_bytes;
  const double **tab_dev;
  const double **tab_host;
  cudaGraphExec_t exec;
};

extern "C" {

int evslcu_filter_columns(const evslcu_mat *A, int fp32, int ncols, const evslcu_filter_col *cols, void *work,
                          size_t work_bytes) {
  if (ncols == 0) return 0;
  int rc = check_cols(A, fp32, ncols, cols, 1);
  if (rc) return rc;
  if (!work || work_bytes < evslcu_filter_columns_work(A->n, fp32, ncols))
    return fail(EVSLCU_ERR_ARG, "filter_columns: work too small");
  const size_t tabb = 2 * sizeof(double *) * (size_t)ncols;
  const size_t tab_off = work_bytes - (tabb + 255) / 256 * 256;
  const double **tab = (const double **)((char *)work + tab_off);
  const double **htab = (const double **)malloc(tabb);
  if (!htab) return fail(EVSLCU_ERR_NOMEM, "filter_columns: out of host memory");
  for (int c = 0; c < ncols; ++c) {
    htab[c] = cols[c].x;
    htab[ncols + c] = cols[c].y;
  }
  rc = evslcu_h2d(tab, htab, tabb);
  free(htab);
  void *coef = rc ? nullptr : coef_build(fp32, ncols, cols, &rc);
  int nl = 0;
  if (!rc) rc = mf_sequence(A, fp32, ncols, cols, coef, work, tab_off, tab, &nl);
  count_launch(nl);
  evslcu_free(coef);
  return rc;
}

evslcu_filter_plan *evslcu_filter_plan_create(const evslcu_mat *A, int fp32, int ncols,
                                              const evslcu_filter_col *cols) {
  if (check_cols(A, fp32, ncols, cols, 0)) return nullptr;
  evslcu_filter_plan *P = new evslcu_filter_plan();
  P->A = A;
  P->fp32 = fp32;
  P->ncols = ncols;
  P->work_bytes = evslcu_filter_columns_work(A->n, fp32, ncols);
  P->work = evslcu_malloc(P->work_bytes);
  P->tab_host = (const double **)calloc(2 * (size_t)ncols, sizeof(double *));
  const size_t tabb = 2 * sizeof(double *) * (size_t)ncols;
  const size_t tab_off = P->work_bytes - (tabb + 255) / 256 * 256;
  P->tab_dev = (const double **)((char *)P->work + tab_off);
  if (!P->work || !P->tab_host) {
    fail(EVSLCU_ERR_NOMEM, "filter plan: out of memory");
    evslcu_filter_plan_destroy(P);
    return nullptr;
  }
  int err = 0;
  P->coef = coef_build(fp32, ncols, cols, &err);
  if (!P->coef) {
    evslcu_filter_plan_destroy(P);
    return nullptr;
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    fail(EVSLCU_ERR_CUDA, "filter plan: capture failed: %s", cudaGetErrorString(e));
    evslcu_filter_plan_destroy(P);
    return nullptr;
  }
  int nl = 0;
  int rc = mf_sequence(A, fp32, ncols, cols, P->coef, P->work, tab_off, P->tab_dev, &nl);
  e = cudaStreamEndCapture(stream(), &graph);
  if (!rc && e != cudaSuccess) rc = fail(EVSLCU_ERR_CUDA, "filter plan: capture failed: %s", cudaGetErrorString(e));
  if (!rc) {
    e = cudaGraphInstantiate(&P->exec, graph, 0);
    if (e != cudaSuccess) rc = fail(EVSLCU_ERR_CUDA, "filter plan: instantiate failed: %s", cudaGetErrorString(e));
  }
  if (graph) cudaGraphDestroy(graph);
  if (rc) {
    cudaGetLastError();
    evslcu_filter_plan_destroy(P);
    return nullptr;
  }
  P->nodes = nl;
  return P;
}

int evslcu_filter_plan_run(evslcu_filter_plan *P, const double *const *x, double *const *y) {
  if (!P || !x || !y) return fail(EVSLCU_ERR_ARG, "filter plan: bad arguments");
  for (int c = 0; c < P->ncols; ++c) {
    P->tab_host[c] = x[c];
    P->tab_host[P->ncols + c] = y[c];
  }
  int rc = evslcu_h2d_async((void *)P->tab_dev, P->tab_host, 2 * sizeof(double *) * (size_t)P->ncols);
  if (rc) return rc;
  cudaError_t e = cudaGraphLaunch(P->exec, stream());
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "filter plan: launch failed: %s", cudaGetErrorString(e));
  count_launch((uint64_t)P->nodes);
  return 0;
}

int evslcu_filter_plan_columns(const evslcu_filter_plan *P) { return P ? P->ncols : 0; }

void evslcu_filter_plan_destroy(evslcu_filter_plan *P) {
  if (!P) return;
  if (P->exec) cudaGraphExecDestroy(P->exec);
  evslcu_free(P->work);
  evslcu_free(P->coef);
  free(P->tab_host);
  delete P;
}

}  // extern "C"
