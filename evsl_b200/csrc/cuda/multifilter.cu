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

// Loads by cache policy: 0 read-only path, 1 L2 only (data this launch
// sequence writes), 2 streaming (evict first: read once, keeps L2 for the
// gathered vector).
template <int MODE, class T>
__device__ __forceinline__ T ldm(const T *p) {
  if constexpr (MODE == 0) return __ldg(p);
  else if constexpr (MODE == 1) return __ldcg(p);
  else return __ldcs(p);
}

// Contiguous B-value loads/stores of a row of an interleaved block, as
// 16-byte (or 8-byte) vector accesses unpacked into registers.
template <int MODE, class VT, int B>
__device__ __forceinline__ void load_row_impl(const VT *p, VT (&x)[B]) {
  if constexpr (std::is_same<VT, float>::value && B % 4 == 0) {
#pragma unroll
    for (int i = 0; i < B / 4; ++i) {
      const float4 f = ldm<MODE>(reinterpret_cast<const float4 *>(p) + i);
      x[4 * i] = f.x;
      x[4 * i + 1] = f.y;
      x[4 * i + 2] = f.z;
      x[4 * i + 3] = f.w;
    }
  } else if constexpr (std::is_same<VT, float>::value && B == 2) {
    const float2 f = ldm<MODE>(reinterpret_cast<const float2 *>(p));
    x[0] = f.x;
    x[1] = f.y;
  } else if constexpr (std::is_same<VT, double>::value && B % 2 == 0) {
#pragma unroll
    for (int i = 0; i < B / 2; ++i) {
      const double2 f = ldm<MODE>(reinterpret_cast<const double2 *>(p) + i);
      x[2 * i] = f.x;
      x[2 * i + 1] = f.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < B; ++c) x[c] = ldm<MODE>(p + c);
  }
}

template <class VT, int B>
__device__ __forceinline__ void load_row(const VT *p, VT (&x)[B]) {
  load_row_impl<0, VT, B>(p, x);
}

// Same for data this launch sequence writes (L2 only, no read-only path).
template <class VT, int B>
__device__ __forceinline__ void load_row_cg(const VT *p, VT (&x)[B]) {
  load_row_impl<1, VT, B>(p, x);
}

// Same, streaming (evict first).
template <class VT, int B>
__device__ __forceinline__ void load_row_cs(const VT *p, VT (&x)[B]) {
  load_row_impl<2, VT, B>(p, x);
}

// Stores by cache policy: CS = streaming (evict first).
template <bool CS, class T>
__device__ __forceinline__ void stm(T *p, T v) {
  if constexpr (CS) __stcs(p, v);
  else *p = v;
}

template <class VT, int B, bool CS = false>
__device__ __forceinline__ void store_row(VT *p, const VT (&x)[B]) {
  if constexpr (std::is_same<VT, float>::value && B % 4 == 0) {
#pragma unroll
    for (int i = 0; i < B / 4; ++i)
      stm<CS>(reinterpret_cast<float4 *>(p) + i, make_float4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]));
  } else if constexpr (std::is_same<VT, float>::value && B == 2) {
    stm<CS>(reinterpret_cast<float2 *>(p), make_float2(x[0], x[1]));
  } else if constexpr (std::is_same<VT, double>::value && B % 2 == 0) {
#pragma unroll
    for (int i = 0; i < B / 2; ++i) stm<CS>(reinterpret_cast<double2 *>(p) + i, make_double2(x[2 * i], x[2 * i + 1]));
  } else {
#pragma unroll
    for (int c = 0; c < B; ++c) stm<CS>(p + c, x[c]);
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

// Columns per thread: CPTB bytes of a row (16: two doubles or four floats;
// 32: four doubles or eight floats); a row is shared by B / CPT threads.
template <class VT, int B, int CPTB>
struct Split {
  static constexpr int CPT = (B < (int)(CPTB / sizeof(VT))) ? B : (int)(CPTB / sizeof(VT));
  static constexpr int TPR = B / CPT;
};

// Kernel variants: the column part per thread (16 or 32 bytes) and whether
// the TPR threads of a row load its stored entries cooperatively (each a
// share, broadcast by warp shuffles) instead of each loading all of them
// (0..3, SELL-32), or the row-pattern dictionary with 16- or 32-byte parts
// (4, 5).  -1: each matrix uses the variant the autotuner measured fastest
// for it (per precision and block width); 0..5: that variant everywhere.
// Variant 6: one column on the column-panel layout (panel.cu), x staged
// through shared memory; built for large general matrices.  Variant 7: 2-16
// columns on the column-split copy (ranges of columns whose rows of the
// block fit in L2), for large general matrices whose block does not.
static int g_mf_variant = -1;
constexpr int kMfVariants = 8;

// One degree of the recurrence for all columns: thread (row r, part q)
// handles columns q*CPT .. q*CPT+CPT-1 of row r.  Rows run over the padded
// SELL-32 range so that every warp is full (rows past n only skip stores).
template <class VT, int B, int CPTB, bool SHARE, class AV, class IT, bool FIRST>
__global__ void __launch_bounds__(kThreads)
    k_mf_step(SellT<AV, IT> A, const VT *__restrict__ vk, const VT *vkm1, VT *out, VT *__restrict__ y,
              const VT *__restrict__ coef) {
  constexpr int CPT = Split<VT, B, CPTB>::CPT, TPR = Split<VT, B, CPTB>::TPR;
  constexpr bool COOP = SHARE && TPR > 1;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int npad = (A.n + 31) & ~31;
  const long long total = (long long)npad * TPR;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
    const int sl = (int)(g / TPR), q = (int)(g % TPR);
    const bool live = sl < A.n;
    const int r = live ? row_of(A, sl) : 0;  // the row stored in slot sl
    const int cb = q * CPT;
    // this row's own values first: independent of the gathers below, so
    // their latency overlaps with them
    const long long base = (long long)r * B + cb;
    VT xr[CPT], wv[CPT], yv[CPT], vm[CPT];
    if (live) {
      load_row<VT, CPT>(vk + base, xr);
      load_row_cg<VT, CPT>(y + base, yv);
      if (!FIRST) load_row_cg<VT, CPT>(vkm1 + base, vm);
    }
    VT acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = (VT)0;
    long long p;
    int w;
    row_start(A, sl, p, w);
    if constexpr (COOP) {
      // TPR entries per batch: thread q loads entry j0 + q of its row, the
      // row's threads exchange them, then gather and accumulate in order
      const int seg = (threadIdx.x & 31) & ~(TPR - 1);
      for (int j0 = 0; j0 < w; j0 += TPR) {
        VT vmine = (VT)0;
        int cmine = live ? r : 0;
        if (live && j0 + q < w) {
          vmine = (VT)__ldg(A.val + p + 32LL * (j0 + q));
          cmine = decode_col(__ldg(A.col + p + 32LL * (j0 + q)), r);
        }
        VT v[TPR];
        int col[TPR];
#pragma unroll
        for (int u = 0; u < TPR; ++u) {
          v[u] = __shfl_sync(0xffffffffu, vmine, seg + u);
          col[u] = __shfl_sync(0xffffffffu, cmine, seg + u);
        }
        VT x[TPR][CPT];
#pragma unroll
        for (int u = 0; u < TPR; ++u) load_row<VT, CPT>(vk + (long long)col[u] * B + cb, x[u]);
#pragma unroll
        for (int u = 0; u < TPR; ++u)
#pragma unroll
          for (int c = 0; c < CPT; ++c) acc[c] = fmadd(v[u], x[u][c], acc[c]);
      }
    } else {
      // U stored entries at a time: their gathers are in flight together,
      // then accumulated in order j = 0, 1, ...; the next U entries of the
      // stored matrix are loaded while the gathers are outstanding, so the
      // streamed matrix loads do not wait behind the gathers.  Slots past
      // the row's width act as 0 * x[r].  One column with 32-byte parts
      // (variant 1; the same split as variant 0 at B = 1) takes 8 entries
      // per batch instead of 4.
      constexpr int U = (B == 1 && CPTB == 32) ? 8 : 4;
      VT v[U];
      int col[U];
      auto fetch = [&](int j0, long long pp, VT(&vv)[U], int(&cc)[U]) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (live && j0 + u < w) {
            vv[u] = (VT)__ldg(A.val + pp + 32 * u);
            cc[u] = decode_col(__ldg(A.col + pp + 32 * u), r);
          } else {
            vv[u] = (VT)0;
            cc[u] = live ? r : 0; /* rows past n gather row 0, unused */
          }
        }
      };
      fetch(0, p, v, col);
      for (int j = 0; j < w; j += U, p += 32 * U) {
        VT x[U][CPT];
#pragma unroll
        for (int u = 0; u < U; ++u) load_row<VT, CPT>(vk + (long long)col[u] * B + cb, x[u]);
        VT vn[U];
        int cn[U];
        fetch(j + U, p + 32 * U, vn, cn);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
          for (int c = 0; c < CPT; ++c) acc[c] = fmadd(v[u], x[u][c], acc[c]);
#pragma unroll
        for (int u = 0; u < U; ++u) {
          v[u] = vn[u];
          col[u] = cn[u];
        }
      }
    }
    if (!live) continue;
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

template <class VT, int B, int CPTB, bool SHARE, class AV, class IT>
int mf_step_v(const SellT<AV, IT> &A, int k, const VT *vk, const VT *vkm1, VT *out, VT *y, const VT *coef) {
  constexpr int TPR = Split<VT, B, CPTB>::TPR;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid_for((long long)((A.n + 31) & ~31) * TPR, kThreads, 1 << 20));
  cfg.blockDim = dim3(kThreads);
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e =
      (k == 1) ? cudaLaunchKernelEx(&cfg, k_mf_step<VT, B, CPTB, SHARE, AV, IT, true>, A, vk, vkm1, out, y, coef)
               : cudaLaunchKernelEx(&cfg, k_mf_step<VT, B, CPTB, SHARE, AV, IT, false>, A, vk, vkm1, out, y, coef);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "multi-column filter launch failed: %s", cudaGetErrorString(e));
  return check_launch("k_mf_step");
}

// ---- column-split filter (variant 7) -------------------------------------
//
// On a large general matrix the gathers x[col] of a degree step land on
// random rows of the whole block; once the block (n x B values) is larger
// than L2 most of them miss L2 and each stored entry costs a DRAM line.  The
// column-split copy (evslcu_xsplit) cuts the columns into ranges whose rows
// of x fit in L2, and a degree step runs one launch per range: the range's
// rows of x stay in L2 while every row adds the products of its entries in
// that range to its running sum, which is carried from range to range in a
// partial-sum block (read and written with streaming hints, like the stored
// matrix, so that L2 keeps the gathered rows).  The last range applies the
// three-term update of k_mf_step.  Ranges follow the columns and each range
// keeps the CSR order, so every row is summed in its CSR order: FP64 columns
// equal ChebAv bit for bit; padding slots (column -1) are skipped.
size_t g_xs_range_bytes = (size_t)40 << 20;  // gathered rows of x per range

template <class VT, int B, bool PFIRST, bool PLAST, bool FIRST>
__global__ void __launch_bounds__(kThreads)
    k_xs_step(XsRange<VT> A, const VT *__restrict__ vk, const VT *vkm1, VT *out, VT *__restrict__ y, VT *part,
              const VT *__restrict__ coef) {
  // 16-byte column parts: the TPR threads of a row gather its B values with
  // one warp instruction (one L1 wavefront per gathered row, the bound on
  // random columns)
  constexpr int CPT = Split<VT, B, 16>::CPT, TPR = Split<VT, B, 16>::TPR;
  constexpr int U = 4;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int npad = (A.n + 31) & ~31;
  const long long total = (long long)npad * TPR;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
    const int sl = (int)(g / TPR), q = (int)(g % TPR);
    const bool live = sl < A.n;
    const int r = live ? __ldg(A.perm + sl) : 0;
    const int cb = q * CPT;
    const long long base = (long long)r * B + cb;
    VT acc[CPT], xr[CPT], yv[CPT], vm[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = (VT)0;
    if (!PFIRST && live) load_row_cs<VT, CPT>(part + base, acc);
    if (PLAST && live) {
      load_row<VT, CPT>(vk + base, xr);
      load_row_cs<VT, CPT>(y + base, yv);
      if (!FIRST) load_row_cs<VT, CPT>(vkm1 + base, vm);
    }
    const int ch = sl >> 5;
    long long p = __ldg(A.cptr + ch) + (sl & 31);
    const int w = __ldg(A.cw + ch);
    VT v[U];
    int col[U];
    auto fetch = [&](int j0, long long pp, VT(&vv)[U], int(&cc)[U]) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (live && j0 + u < w) {
          vv[u] = __ldcs(A.val + pp + 32 * u);
          cc[u] = __ldcs(A.col + pp + 32 * u);
        } else {
          vv[u] = (VT)0;
          cc[u] = -1;
        }
      }
    };
    fetch(0, p, v, col);
    for (int j = 0; j < w; j += U, p += 32 * U) {
      VT x[U][CPT];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (col[u] >= 0) {
          load_row<VT, CPT>(vk + (long long)col[u] * B + cb, x[u]);
        } else {
#pragma unroll
          for (int c = 0; c < CPT; ++c) x[u][c] = (VT)0;
        }
      }
      VT vn[U];
      int cn[U];
      fetch(j + U, p + 32 * U, vn, cn);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (col[u] >= 0) {
#pragma unroll
          for (int c = 0; c < CPT; ++c) acc[c] = fmadd(v[u], x[u][c], acc[c]);
        }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        v[u] = vn[u];
        col[u] = cn[u];
      }
    }
    if (!live) continue;
    if constexpr (!PLAST) {
      store_row<VT, CPT, true>(part + base, acc);
    } else {
      VT wv[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const VT *cf = coef + kCoef * (cb + c);
        VT t = mul(__ldg(cf), add(acc[c], mul(__ldg(cf + 1), xr[c])));
        if (!FIRST) t = add(t, -vm[c]);
        wv[c] = t;
        if (__ldg(cf + 3) != (VT)0) yv[c] = add(yv[c], mul(__ldg(cf + 2), t));
      }
      store_row<VT, CPT>(out + base, wv);
      store_row<VT, CPT, true>(y + base, yv);
    }
  }
}

// Ranges of the column-split copy for a B-column block: the fewest (a power
// of two up to 32) whose rows of x fit g_xs_range_bytes -- one when the
// whole block fits (the kernel then only adds streaming cache hints and
// skips padding); 0 when 32 ranges are not enough.
inline int xs_ranges_rows(const evslcu_mat *M, size_t row) {
  for (int P = 1; P <= evslcu_xsplit::kMaxRanges; P *= 2)
    if ((((size_t)M->n + P - 1) / P) * row <= g_xs_range_bytes) return P;
  return 0;
}
inline int xs_ranges(const evslcu_mat *M, int fp32, int B) {
  return xs_ranges_rows(M, (size_t)B * (fp32 ? sizeof(float) : sizeof(double)));
}
inline int xs_slot(int P) { return P <= 1 ? 0 : P <= 2 ? 1 : P <= 4 ? 2 : P <= 8 ? 3 : P <= 16 ? 4 : 5; }

// The column-split copy a (precision, width) uses, or null when it has none
// (not applicable or not built).
inline const evslcu_xsplit *xs_of(const evslcu_mat *M, int fp32, int B) {
  const int P = xs_ranges(M, fp32, B);
  if (!P) return nullptr;
  const evslcu_xsplit *X = M->xs[xs_slot(P)];
  if (X && (!fp32 || X->val32[0])) return X;
  // the range budget changed since this width was tuned: every copy holds the
  // whole matrix, so any built one serves (its ranges are just sized for
  // another budget)
  for (const evslcu_xsplit *Y : M->xs)
    if (Y && (!fp32 || Y->val32[0])) return Y;
  return nullptr;
}

template <class VT, int B, bool PF, bool PL>
cudaError_t xs_launch(cudaLaunchConfig_t &cfg, bool first, const XsRange<VT> &R, const VT *vk, const VT *vkm1, VT *out,
                      VT *y, VT *part, const VT *coef) {
  return first ? cudaLaunchKernelEx(&cfg, k_xs_step<VT, B, PF, PL, true>, R, vk, vkm1, out, y, part, coef)
               : cudaLaunchKernelEx(&cfg, k_xs_step<VT, B, PF, PL, false>, R, vk, vkm1, out, y, part, coef);
}

template <class VT, int B>
int xs_step(const evslcu_mat *M, int k, const VT *vk, const VT *vkm1, VT *out, VT *y, const VT *coef) {
  constexpr bool F32 = std::is_same<VT, float>::value;
  const evslcu_xsplit *X = xs_of(M, F32 ? 1 : 0, B);
  if constexpr (B == 1) {
    return fail(EVSLCU_ERR_ARG, "filter variant 7 takes 2 to 16 columns");
  } else {
    if (!X || !M->xs_acc) return fail(EVSLCU_ERR_ARG, "filter variant 7 needs a column-split copy for this width");
    constexpr int TPR = Split<VT, B, 16>::TPR;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid_for((long long)((M->n + 31) & ~31) * TPR, kThreads, 1 << 20));
    cfg.blockDim = dim3(kThreads);
    cfg.stream = stream();
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    VT *part = (VT *)M->xs_acc;
    for (int p = 0; p < X->P; ++p) {
      const VT *val;
      if constexpr (F32) val = X->val32[p];
      else val = X->val[p];
      const XsRange<VT> R{M->n, X->cptr[p], X->cw[p], X->col[p], val, X->perm[p]};
      const bool first = (k == 1);
      cudaError_t e;
      if (X->P == 1)
        e = xs_launch<VT, B, true, true>(cfg, first, R, vk, vkm1, out, y, part, coef);
      else if (p == 0)
        e = xs_launch<VT, B, true, false>(cfg, first, R, vk, vkm1, out, y, part, coef);
      else if (p == X->P - 1)
        e = xs_launch<VT, B, false, true>(cfg, first, R, vk, vkm1, out, y, part, coef);
      else
        e = xs_launch<VT, B, false, false>(cfg, first, R, vk, vkm1, out, y, part, coef);
      if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "column-split filter launch failed: %s", cudaGetErrorString(e));
      int rc = check_launch("k_xs_step");
      if (rc) return rc;
    }
    return 0;
  }
}

// One table entry of a row pattern: the value as a double and the column
// offset from the row.
__device__ __forceinline__ void pat_entry(const PatPView &A, int idx, double &v, int &off) {
  const unsigned long long e = __ldg(A.pk + idx);
  v = pat_val(e);
  off = pat_off(e);
}
__device__ __forceinline__ void pat_entry(const PatView &A, int idx, double &v, int &off) {
  const double2 e = __ldg(A.ent + idx);
  v = e.x;
  off = (int)__double_as_longlong(e.y);
}

// The same degree step on the row-pattern dictionary: a row's entries come
// from the pattern table (a few KB, read through L1) instead of the stored
// matrix, in CSR order and without padding entries.  Each table entry is
// read once per row part and applied to all CPT columns of the part.
template <class VT, int B, int CPTB, class PV, bool FIRST>
__global__ void __launch_bounds__(kThreads)
    k_mf_step_pat(PV A, const VT *__restrict__ vk, const VT *vkm1, VT *out, VT *__restrict__ y,
                  const VT *__restrict__ coef) {
  constexpr int CPT = Split<VT, B, CPTB>::CPT, TPR = Split<VT, B, CPTB>::TPR;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const long long total = (long long)A.n * TPR;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
    const int r = (int)(g / TPR), q = (int)(g % TPR);
    const int cb = q * CPT;
    const long long base = (long long)r * B + cb;
    VT xr[CPT], wv[CPT], yv[CPT], vm[CPT];
    load_row<VT, CPT>(vk + base, xr);
    load_row_cg<VT, CPT>(y + base, yv);
    if (!FIRST) load_row_cg<VT, CPT>(vkm1 + base, vm);
    VT acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = (VT)0;
    const int2 h = __ldg(A.hdr + __ldg(A.pid + r));
    constexpr int U = 4;
    for (int j = 0; j < h.y; j += U) {
      VT v[U];
      int col[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        col[u] = r;
        v[u] = (VT)0;
        if (j + u < h.y) {
          double dv;
          int off;
          pat_entry(A, h.x + j + u, dv, off);
          v[u] = (VT)dv;
          col[u] = r + off;
        }
      }
      VT x[U][CPT];
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (j + u < h.y) load_row<VT, CPT>(vk + (long long)col[u] * B + cb, x[u]);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (j + u < h.y)
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

template <class VT, int B, int CPTB, class PV>
int mf_step_pat_v(const PV &A, int k, const VT *vk, const VT *vkm1, VT *out, VT *y, const VT *coef) {
  constexpr int TPR = Split<VT, B, CPTB>::TPR;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid_for((long long)A.n * TPR, kThreads, 1 << 20));
  cfg.blockDim = dim3(kThreads);
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = (k == 1) ? cudaLaunchKernelEx(&cfg, k_mf_step_pat<VT, B, CPTB, PV, true>, A, vk, vkm1, out, y, coef)
                           : cudaLaunchKernelEx(&cfg, k_mf_step_pat<VT, B, CPTB, PV, false>, A, vk, vkm1, out, y, coef);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "multi-column filter launch failed: %s", cudaGetErrorString(e));
  return check_launch("k_mf_step_pat");
}

// Variants 4 and 5 (16- or 32-byte column parts) read the row-pattern
// dictionary; they need one (A->pat_id and in use).
inline bool mf_pattern_ok(const evslcu_mat *M) { return M->pat_id && M->use_pat && M->kernel == 0; }

template <class VT, int B, class AV, class IT>
int mf_step(const evslcu_mat *M, const SellT<AV, IT> &A, int variant, int k, const VT *vk, const VT *vkm1, VT *out,
            VT *y, const VT *coef) {
  switch (variant) {
    case 1: return mf_step_v<VT, B, 32, false>(A, k, vk, vkm1, out, y, coef);
    case 2: return mf_step_v<VT, B, 16, true>(A, k, vk, vkm1, out, y, coef);
    case 3: return mf_step_v<VT, B, 32, true>(A, k, vk, vkm1, out, y, coef);
    case 6:
      if constexpr (B == 1) return panel_mf_step<VT>(M, k, vk, vkm1, out, y, coef);
      return fail(EVSLCU_ERR_ARG, "filter variant 6 takes one column");
    case 7: return xs_step<VT, B>(M, k, vk, vkm1, out, y, coef);
    case 4:
    case 5:
      if (!mf_pattern_ok(M)) return fail(EVSLCU_ERR_ARG, "filter variant %d needs the row-pattern dictionary", variant);
      if (variant == 4)
        return M->pat_f32 ? mf_step_pat_v<VT, B, 16>(pat_pview(M), k, vk, vkm1, out, y, coef)
                          : mf_step_pat_v<VT, B, 16>(pat_view(M), k, vk, vkm1, out, y, coef);
      return M->pat_f32 ? mf_step_pat_v<VT, B, 32>(pat_pview(M), k, vk, vkm1, out, y, coef)
                        : mf_step_pat_v<VT, B, 32>(pat_view(M), k, vk, vkm1, out, y, coef);
    default: return mf_step_v<VT, B, 16, false>(A, k, vk, vkm1, out, y, coef);
  }
}

// Kernel launches of one degree step: one, or one per column range
// (variant 7).
inline int launches_per_step(const evslcu_mat *M, int fp32, int B, int variant) {
  const evslcu_xsplit *X = (variant == 7) ? xs_of(M, fp32, B) : nullptr;
  return X ? X->P : 1;
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
int mf_group(const evslcu_mat *M, const SellT<AV, IT> &A, int variant, int ncols, int maxdeg, const VT *coef, const double *const *xtab,
             double *const *ytab, VT *P, VT *W0, VT *W1, VT *Y, int *nlaunch) {
  const int n = A.n;
  const int g = grid_for((long long)n * B);
  k_mf_pack<VT, B><<<g, kThreads, 0, stream()>>>(n, ncols, xtab, coef, P, Y);
  int rc = check_launch("k_mf_pack");
  VT *W[2] = {W0, W1};
  for (int k = 1; !rc && k <= maxdeg; ++k) {
    const VT *vk = (k == 1) ? P : W[(k - 2) % 2];
    const VT *vkm1 = (k == 1) ? nullptr : ((k == 2) ? P : W[(k - 1) % 2]);
    rc = mf_step<VT, B>(M, A, variant, k, vk, vkm1, W[(k - 1) % 2], Y, coef + (size_t)k * B * kCoef);
  }
  if (!rc) {
    k_mf_unpack<VT, B><<<g, kThreads, 0, stream()>>>(n, ncols, Y, ytab);
    rc = check_launch("k_mf_unpack");
  }
  *nlaunch += maxdeg * launches_per_step(M, std::is_same<VT, float>::value ? 1 : 0, B, variant) + 2;
  return rc;
}

template <class VT, class AV, class IT>
int mf_dispatch(const evslcu_mat *M, const SellT<AV, IT> &A, int variant, int B, int ncols, int maxdeg, const VT *coef,
                const double *const *xtab, double *const *ytab, VT *P, VT *W0, VT *W1, VT *Y, int *nl) {
  switch (B) {
    case 1: return mf_group<VT, 1>(M, A, variant, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
    case 2: return mf_group<VT, 2>(M, A, variant, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
    case 4: return mf_group<VT, 4>(M, A, variant, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
    case 8: return mf_group<VT, 8>(M, A, variant, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
    default: return mf_group<VT, 16>(M, A, variant, ncols, maxdeg, coef, xtab, ytab, P, W0, W1, Y, nl);
  }
}

inline int log2_width(int B) { return B <= 1 ? 0 : B <= 2 ? 1 : B <= 4 ? 2 : B <= 8 ? 3 : 4; }

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

int variant_of(const evslcu_mat *A, int fp32, int B) {
  if (g_mf_variant >= 0) return g_mf_variant;
  const int v = A->mf_variant[fp32 ? 1 : 0][log2_width(B)];
  return v >= 0 ? v : 0;
}

constexpr int kXsMinRows = 1 << 18;

// Builds the column-split copy a (precision, width) would use, with its FP32
// values and the shared partial-sum block, when the matrix is a candidate:
// SELL storage, no row-pattern dictionary in use, rows with increasing
// columns, at least kXsMinRows rows.  0 when the copy is there afterwards
// (or not applicable).
int xs_build(evslcu_mat *A, int P);

int xs_prepare(evslcu_mat *A, int fp32, int B) {
  if (A->kernel != 0 || A->xs_bad || mf_pattern_ok(A) || !A->ia) return 0;
  // the copy costs another stored matrix: only large matrices get one, unless
  // the variant is forced
  if (A->n < kXsMinRows && g_mf_variant != 7) return 0;
  const int P = xs_ranges(A, fp32, B);
  if (!P) return 0;
  int rc = xs_build(A, P);
  if (rc) return rc;
  evslcu_xsplit *X = A->xs[xs_slot(P)];
  if (fp32 && !X->val32[0]) {
    for (int p = 0; p < X->P; ++p) {
      long long sp = 0;
      rc = evslcu_d2h(&sp, X->cptr[p] + X->nch, sizeof(long long));
      if (rc) return rc;
      X->val32[p] = (float *)evslcu_malloc(sizeof(float) * (size_t)std::max(sp, 1LL));
      if (!X->val32[p]) return fail(EVSLCU_ERR_NOMEM, "column-split filter: out of device memory (FP32 values)");
      k_to_float<<<grid_for(std::max(sp, 1LL)), kThreads, 0, stream()>>>(sp, X->val[p], X->val32[p]);
      count_launch();
      if ((rc = check_launch("k_to_float"))) return rc;
    }
  }
  return 0;
}

// Builds (once) the copy with P ranges and the shared partial-sum block.
int xs_build(evslcu_mat *A, int P) {
  evslcu_xsplit *&X = A->xs[xs_slot(P)];
  if (!X) {
    evslcu_xsplit *nx = new evslcu_xsplit();
    const int width = (int)(((long long)A->n + P - 1) / P);
    int rc = build_xsplit_device(A, P, width, nx);
    if (rc) {
      for (int p = 0; p < evslcu_xsplit::kMaxRanges; ++p) {
        evslcu_free(nx->cptr[p]);
        evslcu_free(nx->cw[p]);
        evslcu_free(nx->perm[p]);
        evslcu_free(nx->col[p]);
        evslcu_free(nx->val[p]);
      }
      delete nx;
      return rc;
    }
    X = nx;
  }
  if (!A->xs_acc) {
    A->xs_acc = evslcu_malloc(sizeof(double) * kMaxB * (size_t)A->n);
    if (!A->xs_acc) return fail(EVSLCU_ERR_NOMEM, "column-split filter: out of device memory (partial sums)");
  }
  return 0;
}

// Autotuner: times every kernel variant for this matrix, precision and block
// width on a few degree steps (CUDA events on the library stream, zero
// vectors) and records the fastest in the matrix.  Runs once per
// (matrix, precision, width), outside any stream capture.
int autotune(evslcu_mat *A, int fp32, int B) {
  signed char &slot = A->mf_variant[fp32 ? 1 : 0][log2_width(B)];
  if (slot >= 0) return 0;
  const int n = A->n, steps = 6;
  const size_t vb = fp32 ? sizeof(float) : sizeof(double);
  const size_t blk = ((size_t)n * B * vb + 255) / 256 * 256;
  const size_t cf_n = coef_count(B, 1);
  char *buf = (char *)evslcu_malloc(4 * blk + cf_n * vb);
  if (!buf) return fail(EVSLCU_ERR_NOMEM, "filter autotune: out of device memory");
  int rc = evslcu_memset(buf, 0, 4 * blk + cf_n * vb);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bestv = 0;
  if (B == 1 && panel_candidate(A) && !(fp32 ? A->pn32 : A->pn64) && panel_build(A, fp32))
    cudaGetLastError();  // without the panel layout the SELL kernels serve
  if (B > 1 && xs_prepare(A, fp32, B)) cudaGetLastError();  // without the split copy the SELL kernels serve
  for (int v = 0; !rc && v < kMfVariants; ++v) {
    if (g_mf_variant >= 0 && v != g_mf_variant) continue;  // a forced variant is only timed
    if ((v == 4 || v == 5) && !mf_pattern_ok(A)) continue;
    if (v == 6 && !(B == 1 && (fp32 ? A->pn32 : A->pn64))) continue;
    if (v == 7 && !(B > 1 && xs_of(A, fp32, B))) continue;
    float ms = 0.0f;
    for (int rep = 0; !rc && rep < 2; ++rep) {
      cudaEventRecord(e0, stream());
      for (int k = 2; !rc && k < 2 + steps; ++k) {
        void *P = buf, *W0 = buf + blk, *W1 = buf + 2 * blk, *Y = buf + 3 * blk;
        const void *cf = buf + 4 * blk;
        if (fp32) {
          const void *vals = (A->vfmt == 1) ? A->sval : A->sval32;
          auto go = [&](auto view) -> int {
            switch (B) {
              case 1: return mf_step<float, 1>(A, view, v, k, (const float *)P, (const float *)W0, (float *)W1, (float *)Y, (const float *)cf);
              case 2: return mf_step<float, 2>(A, view, v, k, (const float *)P, (const float *)W0, (float *)W1, (float *)Y, (const float *)cf);
              case 4: return mf_step<float, 4>(A, view, v, k, (const float *)P, (const float *)W0, (float *)W1, (float *)Y, (const float *)cf);
              case 8: return mf_step<float, 8>(A, view, v, k, (const float *)P, (const float *)W0, (float *)W1, (float *)Y, (const float *)cf);
              default: return mf_step<float, 16>(A, view, v, k, (const float *)P, (const float *)W0, (float *)W1, (float *)Y, (const float *)cf);
            }
          };
          rc = A->ifmt ? go(sell_view_vals<float, short>(A, vals)) : go(sell_view_vals<float, int>(A, vals));
        } else {
          rc = with_view(A, [&](auto view) -> int {
            if constexpr (std::is_same<decltype(view), CsrView>::value) {
              return fail(EVSLCU_ERR_ARG, "filter_columns needs the SELL-32 storage");
            } else {
              switch (B) {
                case 1: return mf_step<double, 1>(A, view, v, k, (const double *)P, (const double *)W0, (double *)W1, (double *)Y, (const double *)cf);
                case 2: return mf_step<double, 2>(A, view, v, k, (const double *)P, (const double *)W0, (double *)W1, (double *)Y, (const double *)cf);
                case 4: return mf_step<double, 4>(A, view, v, k, (const double *)P, (const double *)W0, (double *)W1, (double *)Y, (const double *)cf);
                case 8: return mf_step<double, 8>(A, view, v, k, (const double *)P, (const double *)W0, (double *)W1, (double *)Y, (const double *)cf);
                default: return mf_step<double, 16>(A, view, v, k, (const double *)P, (const double *)W0, (double *)W1, (double *)Y, (const double *)cf);
              }
            }
          });
        }
        count_launch(launches_per_step(A, fp32, B, v));
      }
      cudaEventRecord(e1, stream());
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(EVSLCU_ERR_CUDA, "filter autotune: timing failed");
      if (!rc && rep == 1) cudaEventElapsedTime(&ms, e0, e1);
    }
    if (!rc && ms < best) {
      best = ms;
      bestv = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  evslcu_free(buf);
  if (!rc) {
    slot = (signed char)bestv;
    A->mf_cost_us[fp32 ? 1 : 0][log2_width(B)] = 1000.0f * best / steps;
  }
  return rc;
}

int autotune_groups(const evslcu_mat *A, int fp32, int ncols) {
  int rc = 0;
  for (int c0 = 0; !rc && c0 < ncols; c0 += kMaxB) rc = autotune((evslcu_mat *)A, fp32, group_width(std::min(kMaxB, ncols - c0)));
  return rc;
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
        rc = mf_dispatch<float>(A, sell_view_vals<float, short>(A, vals),
                                variant_of(A, 1, B), B, gc, md, cf, xt, yt, P, W0, W1, Y, nlaunch);
      else
        rc = mf_dispatch<float>(A, sell_view_vals<float, int>(A, vals),
                                variant_of(A, 1, B), B, gc, md, cf, xt, yt, P, W0, W1, Y, nlaunch);
    } else {
      double *P = (double *)w, *W0 = (double *)(w + blk), *W1 = (double *)(w + 2 * blk), *Y = (double *)(w + 3 * blk);
      const double *cf = (const double *)coef + off;
      rc = with_view(A, [&](auto view) -> int {
        if constexpr (std::is_same<decltype(view), CsrView>::value) {
          return fail(EVSLCU_ERR_ARG, "filter_columns needs the SELL-32 storage");
        } else {
          return mf_dispatch<double>(A, view, variant_of(A, 0, B), B, gc, md, cf, xt, yt, P, W0, W1, Y, nlaunch);
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

// The column-split copy for blocks of row_bytes bytes per row (built on first
// use, with the shared partial-sum block of n x 16 doubles); null when the
// matrix has none (fewer than kXsMinRows rows unless any_size, no SELL
// storage, a row-pattern dictionary in use, decreasing columns in a row, or
// 32 ranges are not enough).
const evslcu_xsplit *xsplit_for(evslcu_mat *A, size_t row_bytes, bool any_size) {
  if (A->kernel != 0 || A->xs_bad || mf_pattern_ok(A) || !A->ia || (A->n < kXsMinRows && !any_size)) return nullptr;
  const int P = xs_ranges_rows(A, row_bytes);
  if (!P || xs_build(A, P)) {
    cudaGetLastError();
    return nullptr;
  }
  return A->xs[xs_slot(P)];
}

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
  if (!rc) rc = autotune_groups(A, fp32, ncols);
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
  int err = autotune_groups(A, fp32, ncols);
  P->coef = err ? nullptr : coef_build(fp32, ncols, cols, &err);
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

int evslcu_set_filter_variant(int v) {
  if (v < -1 || v >= kMfVariants) return fail(EVSLCU_ERR_ARG, "filter variant must be -1 (tuned) or 0..7");
  g_mf_variant = v;
  return 0;
}

int evslcu_get_filter_variant(void) { return g_mf_variant; }

int evslcu_set_xs_range_bytes(long long bytes) {
  if (bytes < 0) return fail(EVSLCU_ERR_ARG, "split range bytes must be >= 0");
  g_xs_range_bytes = bytes ? (size_t)bytes : ((size_t)40 << 20);
  return 0;
}

int evslcu_mat_filter_variant(const evslcu_mat *A, int fp32, int B) {
  return A ? A->mf_variant[fp32 ? 1 : 0][log2_width(B)] : -1;
}

double evslcu_filter_step_cost(evslcu_mat *A, int fp32, int B) {
  if (!A || A->kernel != 0 || B < 1) return -1.0;
  if (fp32 && A->vfmt == 0 && !A->sval32) return -1.0;
  const int Bp = group_width(std::min(B, kMaxB));
  if (autotune(A, fp32, Bp)) return -1.0;
  return (double)A->mf_cost_us[fp32 ? 1 : 0][log2_width(Bp)];
}

void evslcu_filter_plan_destroy(evslcu_filter_plan *P) {
  if (!P) return;
  if (P->exec) cudaGraphExecDestroy(P->exec);
  evslcu_free(P->work);
  evslcu_free(P->coef);
  free(P->tab_host);
  delete P;
}

}  // extern "C"
