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

template <class VT, int B>
struct Coef {
  VT t[B], ncc[B], s[B];
  unsigned mask;
};

template <int B>
struct ColPtrs {
  const double *p[B];
};

template <int B>
struct ColOut {
  double *p[B];
};

// Contiguous B-value loads/stores of a row of an interleaved block.
template <class VT, int B>
__device__ __forceinline__ void load_row(const VT *p, VT (&x)[B]) {
  if constexpr (sizeof(VT) * B % 16 == 0) {
    constexpr int NV = sizeof(VT) * B / 16;
    const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      const float4 f = __ldg(q + i);
      memcpy(reinterpret_cast<char *>(x) + 16 * i, &f, 16);
    }
  } else {
#pragma unroll
    for (int c = 0; c < B; ++c) x[c] = __ldg(p + c);
  }
}

template <class VT, int B>
__device__ __forceinline__ void load_row_cg(const VT *p, VT (&x)[B]) {
#pragma unroll
  for (int c = 0; c < B; ++c) x[c] = p[c];
}

template <class VT, int B>
__device__ __forceinline__ void store_row(VT *p, const VT (&x)[B]) {
  if constexpr (sizeof(VT) * B % 16 == 0) {
    constexpr int NV = sizeof(VT) * B / 16;
    float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      float4 f;
      memcpy(&f, reinterpret_cast<const char *>(x) + 16 * i, 16);
      q[i] = f;
    }
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

// P = pack(x_c) (converted to VT); Y = mu0_c * P.
template <class VT, int B>
__global__ void k_mf_pack(int n, int ncols, ColPtrs<B> x, Coef<VT, B> mu0, VT *P, VT *Y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)n * B;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / B), c = (int)(i % B);
    const VT v = (c < ncols) ? (VT)x.p[c][r] : (VT)0;
    P[i] = v;
    Y[i] = mul(mu0.s[c], v);
  }
}

template <class VT, int B>
__global__ void k_mf_unpack(int n, int ncols, const VT *Y, ColOut<B> y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)n * B;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / B), c = (int)(i % B);
    if (c < ncols) y.p[c][r] = (double)Y[i];
  }
}

// One degree of the recurrence for all columns (thread per row).
template <class VT, int B, class AV, class IT, bool FIRST>
__global__ void __launch_bounds__(kThreads)
    k_mf_step(SellT<AV, IT> A, const VT *__restrict__ vk, const VT *vkm1, VT *out, VT *__restrict__ y,
              Coef<VT, B> cf) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int nthreads = gridDim.x * blockDim.x;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < A.n; r += nthreads) {
    VT acc[B];
#pragma unroll
    for (int c = 0; c < B; ++c) acc[c] = (VT)0;
    const int ch = r >> 5;
    long long p = A.cptr[ch] + (r & 31);
    const int w = A.cw[ch];
    for (int j = 0; j < w; ++j, p += 32) {
      const VT v = (VT)__ldg(A.val + p);
      const int col = decode_col(__ldg(A.col + p), r);
      VT x[B];
      load_row<VT, B>(vk + (long long)col * B, x);
#pragma unroll
      for (int c = 0; c < B; ++c) acc[c] = fmadd(v, x[c], acc[c]);
    }
    const long long base = (long long)r * B;
    VT xr[B], wv[B], yv[B], vm[B];
    load_row<VT, B>(vk + base, xr);
    load_row_cg<VT, B>(y + base, yv);
    if (!FIRST) load_row_cg<VT, B>(vkm1 + base, vm);
#pragma unroll
    for (int c = 0; c < B; ++c) {
      VT t = mul(cf.t[c], add(acc[c], mul(cf.ncc[c], xr[c])));
      if (!FIRST) t = add(t, -vm[c]);
      wv[c] = t;
      if ((cf.mask >> c) & 1u) yv[c] = add(yv[c], mul(cf.s[c], t));
    }
    store_row<VT, B>(out + base, wv);
    store_row<VT, B>(y + base, yv);
  }
}

template <class VT, int B, class AV, class IT>
int mf_step(const SellT<AV, IT> &A, int k, const VT *vk, const VT *vkm1, VT *out, VT *y, const Coef<VT, B> &cf) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid_for(A.n, kThreads, 1 << 20));
  cfg.blockDim = dim3(kThreads);
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = (k == 1) ? cudaLaunchKernelEx(&cfg, k_mf_step<VT, B, AV, IT, true>, A, vk, vkm1, out, y, cf)
                           : cudaLaunchKernelEx(&cfg, k_mf_step<VT, B, AV, IT, false>, A, vk, vkm1, out, y, cf);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "multi-column filter launch failed: %s", cudaGetErrorString(e));
  count_launch();
  return check_launch("k_mf_step");
}

template <class VT, int B, class AV, class IT>
int mf_group(const SellT<AV, IT> &A, int ncols, const evslcu_filter_col *cols, VT *P, VT *W0, VT *W1, VT *Y) {
  const int n = A.n;
  ColPtrs<B> xin = {};
  ColOut<B> yout = {};
  Coef<VT, B> mu0 = {};
  int maxdeg = 0;
  for (int c = 0; c < ncols; ++c) {
    xin.p[c] = cols[c].x;
    yout.p[c] = cols[c].y;
    mu0.s[c] = (VT)cols[c].mu[0];
    maxdeg = std::max(maxdeg, cols[c].deg);
  }
  const int g = grid_for((long long)n * B);
  k_mf_pack<VT, B><<<g, kThreads, 0, stream()>>>(n, ncols, xin, mu0, P, Y);
  count_launch();
  int rc = check_launch("k_mf_pack");
  VT *W[2] = {W0, W1};
  for (int k = 1; !rc && k <= maxdeg; ++k) {
    Coef<VT, B> cf = {};
    for (int c = 0; c < ncols; ++c) {
      const evslcu_filter_col &q = cols[c];
      cf.t[c] = (VT)((k == 1) ? 1.0 / q.dd : 2.0 / q.dd);
      cf.ncc[c] = (VT)(-q.cc);
      if (k <= q.deg) {
        cf.s[c] = (VT)q.mu[k];
        cf.mask |= 1u << c;
      }
    }
    const VT *vk = (k == 1) ? P : W[(k - 2) % 2];
    const VT *vkm1 = (k == 1) ? nullptr : ((k == 2) ? P : W[(k - 1) % 2]);
    rc = mf_step<VT, B>(A, k, vk, vkm1, W[(k - 1) % 2], Y, cf);
  }
  if (!rc) {
    k_mf_unpack<VT, B><<<g, kThreads, 0, stream()>>>(n, ncols, Y, yout);
    count_launch();
    rc = check_launch("k_mf_unpack");
  }
  return rc;
}

template <class VT, class AV, class IT>
int mf_dispatch(const SellT<AV, IT> &A, int ncols, const evslcu_filter_col *cols, VT *P, VT *W0, VT *W1, VT *Y) {
  if (ncols <= 1) return mf_group<VT, 1>(A, ncols, cols, P, W0, W1, Y);
  if (ncols <= 2) return mf_group<VT, 2>(A, ncols, cols, P, W0, W1, Y);
  if (ncols <= 4) return mf_group<VT, 4>(A, ncols, cols, P, W0, W1, Y);
  if (ncols <= 8) return mf_group<VT, 8>(A, ncols, cols, P, W0, W1, Y);
  return mf_group<VT, 16>(A, ncols, cols, P, W0, W1, Y);
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
  return 4 * blk;
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

int evslcu_filter_columns(const evslcu_mat *A, int fp32, int ncols, const evslcu_filter_col *cols, void *work,
                          size_t work_bytes) {
  if (!A || ncols < 0 || (ncols > 0 && (!cols || !work))) return fail(EVSLCU_ERR_ARG, "filter_columns: bad arguments");
  if (A->kernel != 0) return fail(EVSLCU_ERR_ARG, "filter_columns needs the SELL-32 storage");
  if (fp32 && A->vfmt == 0 && !A->sval32) return fail(EVSLCU_ERR_STATE, "FP32 values not prepared");
  const int n = A->n;
  for (int c = 0; c < ncols; ++c)
    if (!cols[c].x || !cols[c].y || !cols[c].mu || cols[c].deg < 0 || cols[c].dd == 0.0)
      return fail(EVSLCU_ERR_ARG, "filter_columns: bad column %d", c);
  int rc = 0;
  for (int c0 = 0; !rc && c0 < ncols; c0 += kMaxB) {
    const int gc = std::min(kMaxB, ncols - c0);
    const int B = group_width(gc);
    const size_t vb = fp32 ? sizeof(float) : sizeof(double);
    const size_t blk = ((size_t)n * B * vb + 255) / 256 * 256;
    if (4 * blk > work_bytes) return fail(EVSLCU_ERR_ARG, "filter_columns: work too small");
    char *w = (char *)work;
    if (fp32) {
      float *P = (float *)w, *W0 = (float *)(w + blk), *W1 = (float *)(w + 2 * blk), *Y = (float *)(w + 3 * blk);
      const void *vals = (A->vfmt == 1) ? A->sval : A->sval32;
      if (A->ifmt)
        rc = mf_dispatch<float>(SellT<float, short>{n, A->cptr, A->cw, (const short *)A->scol, (const float *)vals},
                                gc, cols + c0, P, W0, W1, Y);
      else
        rc = mf_dispatch<float>(SellT<float, int>{n, A->cptr, A->cw, (const int *)A->scol, (const float *)vals}, gc,
                                cols + c0, P, W0, W1, Y);
    } else {
      double *P = (double *)w, *W0 = (double *)(w + blk), *W1 = (double *)(w + 2 * blk), *Y = (double *)(w + 3 * blk);
      rc = with_view(A, [&](auto view) -> int {
        if constexpr (std::is_same<decltype(view), CsrView>::value) {
          return fail(EVSLCU_ERR_ARG, "filter_columns needs the SELL-32 storage");
        } else {
          return mf_dispatch<double>(view, gc, cols + c0, P, W0, W1, Y);
        }
      });
    }
  }
  return rc;
}

}  // extern "C"
