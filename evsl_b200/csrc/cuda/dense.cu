// Dense FP64 kernels: level-1 operations with device-resident scalars,
// classical Gram-Schmidt with the DGKS test, GEMV/GEMM and the batched Ritz
// pair evaluation.
//
// Reductions are deterministic: every block writes one partial in a fixed
// thread order and the last block to finish sums the partials in index order.
// Element-wise updates use explicitly rounded multiply/add so they match the
// reference CPU build's daxpy/dscal/dgemv('N') arithmetic element for element
// (SRC/blas/daxpy.c, dscal.c, dgemv.c); only dot products and norms are summed
// in a different (tree) order.
#include <algorithm>
#include <vector>

#include "common.cuh"

using namespace evslcu;

namespace {

constexpr double kEta = 0.70710678118654752440;  // 1/sqrt(2), SRC/misc_la.c:226
constexpr int EVSL_NGS_MAX_CU = 2;                 // Gram-Schmidt passes, INC/internal_header.h:24

__global__ void k_dot(int n, const double *x, const double *y, double *part, unsigned int *ctr, double *out,
                      int sqrt_result) {
  __shared__ double sh[kThreads / 32];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += x[i] * y[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
  if (last_block(ctr)) {
    double t = reduce_partials(part, gridDim.x, ctr, sh);
    if (threadIdx.x == 0) *out = sqrt_result ? sqrt(t) : t;
  }
}

__global__ void k_axpy_ds(int n, const double *coef, double sign, const double *x, double *y) {
  const double c = sign * (*coef);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = __dadd_rn(y[i], __dmul_rn(c, x[i]));
}

__global__ void k_axpy(int n, double a, const double *x, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = __dadd_rn(y[i], __dmul_rn(a, x[i]));
}

__global__ void k_scal_inv_ds(int n, const double *s, double *x) {
  const double t = 1.0 / (*s);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = __dmul_rn(t, x[i]);
}

__global__ void k_scal(int n, double a, double *x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = __dmul_rn(a, x[i]);
}

// ---------------------------------------------------------------------------
// Gram-Schmidt building blocks.  State slots: [0] old norm, [1] new norm,
// [2] done flag (1.0 once the DGKS test has passed).
// ---------------------------------------------------------------------------
constexpr int kGemvTRows = 1024;   // rows per chunk of the transposed product
constexpr int kGemvTCols = 32;     // columns per block
constexpr int kGemvNChunk = 2048;  // h values staged in shared memory at once

// part[chunk * k + j] = sum over the chunk's rows of Q[r, j] * v[r]; block
// (bx, by) of the chunk x column-tile grid.  Shared by the single-vector
// kernel and the engine's batched one, so both round alike.
__device__ __forceinline__ void gemvT_partial_body(int n, int k, const double *__restrict__ Q, long long ld,
                                                   const double *__restrict__ v, double *__restrict__ part, int bx,
                                                   int by, double *sv) {
  const int r0 = bx * kGemvTRows;
  const int rows = min(kGemvTRows, n - r0);
  for (int i = threadIdx.x; i < kGemvTRows; i += blockDim.x) sv[i] = (i < rows) ? v[r0 + i] : 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int jj = warp; jj < kGemvTCols; jj += kThreads / 32) {
    const int j = by * kGemvTCols + jj;
    if (j >= k) break;
    const double *q = Q + (long long)j * ld + r0;
    double acc = 0.0;
#pragma unroll 8
    for (int i = lane; i < rows; i += 32) acc += __ldg(q + i) * sv[i];  // 32 loads per lane, unrolled
    acc = warp_sum(acc);
    if (lane == 0) part[(long long)bx * k + j] = acc;
  }
}

__global__ void __launch_bounds__(kThreads)
    k_gemvT_partial(int n, int k, const double *__restrict__ Q, long long ld, const double *__restrict__ v,
                    double *__restrict__ part, const double *state) {
  if (state && state[2] != 0.0) return;
  __shared__ double sv[kGemvTRows];
  gemvT_partial_body(n, k, Q, ld, v, part, blockIdx.x, blockIdx.y, sv);
}

// h[j] = alpha * sum_chunks part[chunk*k + j] (+ beta * h[j] when beta != 0).
// Block of 256 threads = 8 warps per 32 columns: lane = column, warp w sums
// chunks w, w+8, ...; the 8 warp sums are added in warp order (fixed order).
__device__ __forceinline__ void gemvT_reduce_body(int nchunks, int k, const double *part, double alpha, double beta,
                                                  double *h, int bx, double (*sh)[33]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = bx * 32 + lane;
  double s = 0.0;
  if (j < k)
    for (int c = warp; c < nchunks; c += 8) s += part[(long long)c * k + j];
  sh[warp][lane] = s;
  __syncthreads();
  if (warp == 0 && j < k) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) t += sh[w][lane];
    h[j] = (beta == 0.0) ? alpha * t : __dadd_rn(__dmul_rn(beta, h[j]), alpha * t);
  }
}

__global__ void __launch_bounds__(256)
    k_gemvT_reduce(int nchunks, int k, const double *part, double alpha, double beta, double *h,
                   const double *state) {
  if (state && state[2] != 0.0) return;
  __shared__ double sh[8][33];
  gemvT_reduce_body(nchunks, k, part, alpha, beta, h, blockIdx.x, sh);
}

// v[r] <- v[r] + sum_j (alpha*h[j]) * Q[r, j], summed over j in order as the
// reference dgemv('N') does.  With `state`, also computes ||v|| and applies
// the DGKS decision of SRC/misc_la.c:246-250.
// Rows bx*blockDim.x + threadIdx.x + i*gx*blockDim.x of the update; returns
// this thread's sum of the new z^2.
__device__ __forceinline__ double gemvN_body(int n, int k, const double *__restrict__ Q, long long ld,
                                             const double *__restrict__ h, double alpha, double *v, int bx, int gx,
                                             double *sh_h) {
  double nsum = 0.0;
  for (long long base = (long long)bx * blockDim.x; base < n; base += (long long)gx * blockDim.x) {
    const long long r = base + threadIdx.x;
    double z = (r < n) ? v[r] : 0.0;
    for (int j0 = 0; j0 < k; j0 += kGemvNChunk) {
      const int cnt = min(kGemvNChunk, k - j0);
      __syncthreads();
      for (int j = threadIdx.x; j < cnt; j += blockDim.x) sh_h[j] = alpha * h[j0 + j];
      __syncthreads();
      if (r < n) {
        // 16 column loads in flight per thread, then the updates in column
        // order (the summation order is unchanged)
        const double *q = Q + (long long)j0 * ld + r;
        int j = 0;
        for (; j + 16 <= cnt; j += 16) {
          double x[16];
#pragma unroll
          for (int u = 0; u < 16; ++u) x[u] = __ldg(q + (long long)(j + u) * ld);
#pragma unroll
          for (int u = 0; u < 16; ++u) z = __dadd_rn(z, __dmul_rn(sh_h[j + u], x[u]));
        }
        for (; j < cnt; ++j) z = __dadd_rn(z, __dmul_rn(sh_h[j], __ldg(q + (long long)j * ld)));
      }
    }
    if (r < n) {
      v[r] = z;
      nsum += z * z;
    }
  }
  return nsum;
}

// The DGKS decision of SRC/misc_la.c:246-250 from the new norm's square.
__device__ __forceinline__ void dgks_decide(double t, double *state) {
  const double nw = sqrt(t);
  state[1] = nw;
  if (nw > kEta * state[0])
    state[2] = 1.0;
  else
    state[0] = nw;
}

__global__ void __launch_bounds__(kThreads)
    k_gemvN(int n, int k, const double *__restrict__ Q, long long ld, const double *__restrict__ h, double alpha,
            double *v, double *part, unsigned int *ctr, double *state) {
  if (state && state[2] != 0.0) return;
  __shared__ double sh_h[kGemvNChunk];
  __shared__ double sh[kThreads / 32];
  double nsum = gemvN_body(n, k, Q, ld, h, alpha, v, blockIdx.x, gridDim.x, sh_h);
  if (state) {
    nsum = block_sum(nsum, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = nsum;
    if (last_block(ctr)) {
      double t = reduce_partials(part, gridDim.x, ctr, sh);
      if (threadIdx.x == 0) dgks_decide(t, state);
    }
  }
}

__global__ void k_cgs_init(double *state, const double *nrm) {
  state[0] = *nrm;
  state[1] = 0.0;
  state[2] = 0.0;
}

__global__ void k_copy_scalar(const double *src, double *dst) { *dst = *src; }

// ---------------------------------------------------------------------------
// The request engine's Lanczos step for many slots at once.  Every slot's
// work is split into blocks exactly as the single-slot kernels split it (the
// same grids, per slot), and a block finds its slot in a prefix table of
// block counts, so each slot's arithmetic -- including every reduction
// order -- is that of evslcu_axpy / evslcu_dot / evslcu_cgs_dgks on it alone.
// Reductions that the single-slot kernels finish in their last block are
// finished here by one block per slot in a separate launch, with the same
// code and thread count.
// ---------------------------------------------------------------------------
struct LzSlot {
  int n, kc;            // rows; basis columns orthogonalised against (k + 1)
  int g_dot, nchunks;   // grids of the dot / norm and of the transposed GEMV
  int ctiles, g_n;      // column tiles of the transposed GEMV; grid of the GEMV
  double nbeta;         // -beta of the previous step (0 at k = 0: no update)
  const double *V;      // basis, ld = n
  const double *v;      // V(:, k)
  const double *vprev;  // V(:, k-1), or null
  double *z;            // V(:, k+1): the filtered vector, orthogonalised in place
  double *ds;           // ds[0] = alpha, ds[1] = new norm
  double *part;         // transposed GEMV partials (nchunks x kc), then h (kc), state (4)
  double *npart;        // norm / dot partials (g_n >= g_dot entries)
};
enum { LZ_DOT = 0, LZ_T, LZ_TR, LZ_N, LZ_ONE, LZ_NPREF };

__device__ __forceinline__ int lz_slot_of(const int *pre, int ns, int b) {
  int lo = 0, hi = ns;  // pre[0] = 0 <= b < pre[ns]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= b)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}
__device__ __forceinline__ double *lz_h(const LzSlot &S) { return S.part + (size_t)S.nchunks * S.kc; }
__device__ __forceinline__ double *lz_state(const LzSlot &S) { return lz_h(S) + S.kc; }

// z -= beta v_prev (k > 0), then partial sums of z . v (k_axpy + k_dot)
__global__ void __launch_bounds__(kThreads) k_lz_axpy_dot(const LzSlot *__restrict__ SS, const int *__restrict__ pre,
                                                         int ns) {
  __shared__ double sh[kThreads / 32];
  const int si = lz_slot_of(pre, ns, blockIdx.x);
  const LzSlot &S = SS[si];
  const int b = blockIdx.x - pre[si];
  double acc = 0.0;
  for (int i = b * blockDim.x + threadIdx.x; i < S.n; i += S.g_dot * blockDim.x) {
    double zi = S.z[i];
    if (S.vprev) zi = __dadd_rn(zi, __dmul_rn(S.nbeta, S.vprev[i]));
    S.z[i] = zi;
    acc += zi * S.v[i];
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) S.npart[b] = acc;
}

// alpha = the sum of the dot partials (reduce_partials' order)
__global__ void __launch_bounds__(kThreads) k_lz_alpha(const LzSlot *__restrict__ SS) {
  __shared__ double sh[kThreads / 32];
  const LzSlot &S = SS[blockIdx.x];
  double s = 0.0;
  for (int i = threadIdx.x; i < S.g_dot; i += blockDim.x) s += __ldcg(S.npart + i);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) S.ds[0] = s;
}

// z -= alpha v (k_axpy_ds), then partial sums of z . z (the norm of k_dot)
__global__ void __launch_bounds__(kThreads) k_lz_axpy_nrm(const LzSlot *__restrict__ SS, const int *__restrict__ pre,
                                                         int ns) {
  __shared__ double sh[kThreads / 32];
  const int si = lz_slot_of(pre, ns, blockIdx.x);
  const LzSlot &S = SS[si];
  const int b = blockIdx.x - pre[si];
  const double c = -1.0 * __ldcg(S.ds);
  double acc = 0.0;
  for (int i = b * blockDim.x + threadIdx.x; i < S.n; i += S.g_dot * blockDim.x) {
    const double zi = __dadd_rn(S.z[i], __dmul_rn(c, S.v[i]));
    S.z[i] = zi;
    acc += zi * zi;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) S.npart[b] = acc;
}

// the starting norm of the Gram-Schmidt passes (k_cgs_init)
__global__ void __launch_bounds__(kThreads) k_lz_cgs_init(const LzSlot *__restrict__ SS) {
  __shared__ double sh[kThreads / 32];
  const LzSlot &S = SS[blockIdx.x];
  double s = 0.0;
  for (int i = threadIdx.x; i < S.g_dot; i += blockDim.x) s += __ldcg(S.npart + i);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    double *st = lz_state(S);
    st[0] = sqrt(s);
    st[1] = 0.0;
    st[2] = 0.0;
  }
}

__global__ void __launch_bounds__(kThreads) k_lz_gemvT(const LzSlot *__restrict__ SS, const int *__restrict__ pre,
                                                      int ns) {
  __shared__ double sv[kGemvTRows];
  const int si = lz_slot_of(pre, ns, blockIdx.x);
  const LzSlot &S = SS[si];
  if (lz_state(S)[2] != 0.0) return;
  const int b = blockIdx.x - pre[si];
  gemvT_partial_body(S.n, S.kc, S.V, S.n, S.z, S.part, b % S.nchunks, b / S.nchunks, sv);
}

__global__ void __launch_bounds__(256) k_lz_gemvT_reduce(const LzSlot *__restrict__ SS, const int *__restrict__ pre,
                                                         int ns) {
  __shared__ double sh[8][33];
  const int si = lz_slot_of(pre, ns, blockIdx.x);
  const LzSlot &S = SS[si];
  if (lz_state(S)[2] != 0.0) return;
  gemvT_reduce_body(S.nchunks, S.kc, S.part, 1.0, 0.0, lz_h(S), blockIdx.x - pre[si], sh);
}

__global__ void __launch_bounds__(kThreads) k_lz_gemvN(const LzSlot *__restrict__ SS, const int *__restrict__ pre,
                                                      int ns) {
  __shared__ double sh_h[kGemvNChunk];
  __shared__ double sh[kThreads / 32];
  const int si = lz_slot_of(pre, ns, blockIdx.x);
  const LzSlot &S = SS[si];
  if (lz_state(S)[2] != 0.0) return;
  const int b = blockIdx.x - pre[si];
  double nsum = gemvN_body(S.n, S.kc, S.V, S.n, lz_h(S), -1.0, S.z, b, S.g_n, sh_h);
  nsum = block_sum(nsum, sh);
  if (threadIdx.x == 0) S.npart[b] = nsum;
}

// the pass's norm and DGKS decision; the norm goes to ds[1]
__global__ void __launch_bounds__(kThreads) k_lz_dgks(const LzSlot *__restrict__ SS) {
  __shared__ double sh[kThreads / 32];
  const LzSlot &S = SS[blockIdx.x];
  double *st = lz_state(S);
  if (st[2] != 0.0) return;
  double s = 0.0;
  for (int i = threadIdx.x; i < S.g_n; i += blockDim.x) s += __ldcg(S.npart + i);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    dgks_decide(s, st);
    S.ds[1] = st[1];
  }
}

// x_s *= a_s for a list of vectors (k_scal)
struct LzScale {
  int n, g;
  double a;
  double *x;
};
__global__ void __launch_bounds__(kThreads) k_lz_scal(const LzScale *__restrict__ SS, const int *__restrict__ pre,
                                                     int ns) {
  const int si = lz_slot_of(pre, ns, blockIdx.x);
  const LzScale &S = SS[si];
  const int b = blockIdx.x - pre[si];
  for (int i = b * blockDim.x + threadIdx.x; i < S.n; i += S.g * blockDim.x) S.x[i] = __dmul_rn(S.a, S.x[i]);
}

// y = beta*y for the transposed GEMV when alpha == 0 etc. (rarely used)
__global__ void k_scale_vec(int n, double beta, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = (beta == 0.0) ? 0.0 : __dmul_rn(beta, y[i]);
}

// ---------------------------------------------------------------------------
// GEMM: C = alpha op(A) op(B) + beta C, column-major, 64x64 tiles, 4x4 per
// thread, FP64 FMA.
// ---------------------------------------------------------------------------
constexpr int BM = 64, BN = 64, BK = 16;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256)
    k_dgemm(int m, int n, int kbeg, int k, double alpha, const double *__restrict__ A, long long lda,
            const double *__restrict__ B, long long ldb, double beta, double *C, long long ldc, long long cstride,
            int kchunk) {
  // split-K: blockIdx.z selects the inner-dimension range and the output slab
  if (kchunk > 0) {
    kbeg = blockIdx.z * kchunk;
    k = min(k, kbeg + kchunk);
    C += (long long)blockIdx.z * cstride;
  }
  __shared__ double sA[BK][BM + 1];
  __shared__ double sB[BK][BN + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  double acc[4][4] = {};
  for (int k0 = kbeg; k0 < k; k0 += BK) {
    for (int i = threadIdx.x; i < BM * BK; i += 256) {
      const int mm = i % BM, kk = i / BM;
      const int gm = m0 + mm, gk = k0 + kk;
      double val = 0.0;
      if (gm < m && gk < k) val = TA ? A[(long long)gm * lda + gk] : A[(long long)gk * lda + gm];
      sA[kk][mm] = val;
    }
    for (int i = threadIdx.x; i < BN * BK; i += 256) {
      const int kk = i % BK, nn = i / BK;
      const int gk = k0 + kk, gn = n0 + nn;
      double val = 0.0;
      if (gk < k && gn < n) val = TB ? B[(long long)gk * ldb + gn] : B[(long long)gn * ldb + gk];
      sB[kk][nn] = val;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sA[kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sB[kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gm = m0 + tx + 16 * i, gn = n0 + ty + 16 * j;
      if (gm < m && gn < n) {
        double *c = C + (long long)gn * ldc + gm;
        *c = (beta == 0.0) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * (*c);
      }
    }
}

// ---------------------------------------------------------------------------
// GEMM C = alpha A B + beta C (A m x k, B k x n, column-major) for the Ritz
// vectors V(:, 1:K) Y and the other tall products: 128 x 128 tiles, 16-deep
// k slices double-buffered in shared memory by cp.async, 256 threads in 8
// warps of 64 x 32, 8 x 8 accumulators per thread, FP64 FMA.  Each C entry
// is the FMA chain over k = 0, 1, ... from 0, then alpha acc (+ beta C), as
// k_dgemm computes it, so both kernels give the same bits.  Needs A, B and
// their leading dimensions 16-byte aligned (the caller checks).
//
// Thread (lane l of warp w): warp tile rows 64 (w % 2) .. +63, columns
// 32 (w / 2) .. +31; the thread's rows are 2 (l % 8) + 16 q + {0, 1}
// (q = 0..3) and its columns l / 8 + 4 j (j = 0..7), so that a warp's
// shared-memory reads of A (16-byte pairs) and of B (one double per column,
// B tile rows padded to 18 doubles) fall in distinct banks.
// ---------------------------------------------------------------------------
constexpr int GT = 128, GK = 16, GKP = 18;  // tile, k slice, padded B row (doubles)
constexpr size_t kGemmSmem = 2 * (size_t)(GK * GT + GT * GKP) * sizeof(double);

__device__ __forceinline__ void cpa16(void *dst, const void *src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cpa8(void *dst, const void *src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
// A pair of doubles into 16-byte aligned shared memory: one 16-byte copy
// when the source pair is 16-byte aligned (AL), else two 8-byte copies.
// bytes: 16 (both in range), 8 (only the first), 0 (neither; zero fill).
template <bool AL>
__device__ __forceinline__ void cp_pair(double *dst, const double *src, const double *base, int bytes) {
  if (AL) {
    cpa16(dst, bytes ? src : base, bytes);
  } else {
    cpa8(dst, bytes ? src : base, bytes >= 8 ? 8 : 0);
    cpa8(dst + 1, bytes == 16 ? src + 1 : base, bytes == 16 ? 8 : 0);
  }
}

template <bool A16, bool B16>
__global__ void __launch_bounds__(256, 1)
    k_dgemm_nn128(int m, int n, int k, double alpha, const double *__restrict__ A, long long lda,
                  const double *__restrict__ B, long long ldb, double beta, double *C, long long ldc) {
  extern __shared__ __align__(16) double gsm[];
  // stage st: A slice at gsm + st GK GT ([k][m]); B slice at gsm + 2 GK GT + st GT GKP ([n][k])
  double *const sA0 = gsm;
  double *const sB0 = gsm + 2 * GK * GT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.x * GT, n0 = blockIdx.y * GT;
  const int wm = 64 * (warp & 1), wn = 32 * (warp >> 1);
  const int tx = lane & 7, ty = lane >> 3;
  auto load = [&](int st, int k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int c = tid + 256 * i;
      // A: k row kk = c / 64, pair p = c % 64 -> rows m0 + 2p, +1
      const int kk = c >> 6, pa = c & 63;
      const int gr = m0 + 2 * pa, gk = k0 + kk;
      int bytes = 0;
      if (gk < k) bytes = (gr + 1 < m) ? 16 : ((gr < m) ? 8 : 0);
      cp_pair<A16>(sA0 + st * (GK * GT) + kk * GT + 2 * pa, A + (long long)gk * lda + gr, A, bytes);
      // B: column nn = c / 8, pair q = c % 8 -> k0 + 2q, +1
      const int nn = c >> 3, q = c & 7;
      const int gc = n0 + nn, gk2 = k0 + 2 * q;
      int bb = 0;
      if (gc < n) bb = (gk2 + 1 < k) ? 16 : ((gk2 < k) ? 8 : 0);
      cp_pair<B16>(sB0 + st * (GT * GKP) + nn * GKP + 2 * q, B + (long long)gc * ldb + gk2, B, bb);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  const int nk = (k + GK - 1) / GK;
  load(0, 0);
  for (int t = 0; t < nk; ++t) {
    const int st = t & 1;
    if (t + 1 < nk) {
      load(st ^ 1, (t + 1) * GK);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const double *a_s = sA0 + st * (GK * GT) + wm + 2 * tx;
    const double *b_s = sB0 + st * (GT * GKP) + (wn + ty) * GKP;
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      double a[8], b[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double2 v = *reinterpret_cast<const double2 *>(a_s + kk * GT + 16 * q);
        a[2 * q] = v.x;
        a[2 * q + 1] = v.y;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = b_s[4 * j * GKP + kk];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int gn = n0 + wn + ty + 4 * j;
    if (gn >= n) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int gm = m0 + wm + 2 * tx + 16 * (i >> 1) + (i & 1);
      if (gm < m) {
        double *c = C + (long long)gn * ldc + gm;
        *c = (beta == 0.0) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * (*c);
      }
    }
  }
}

// The same tall GEMM on the FP64 tensor instruction mma.sync m8n8k4: the
// staging is k_dgemm_nn128's (A slices padded to GTA doubles per k row so the
// fragment loads of a warp spread over the banks); each warp's 64 x 32 tile
// is 8 x 4 accumulator fragments of 8 x 8, and a 16-deep k slice is four
// steps of (8 A + 4 B fragment loads, 32 mma).  One mma does 256 multiply-adds
// of a warp, so the k loop issues about a fifth of the shared loads and an
// eighth of the arithmetic instructions of the DFMA kernel.  The products are
// summed in the instruction's order, not the FMA chain's: results agree with
// k_dgemm_nn128 to rounding, not bit for bit.
constexpr int GTA = GT + 4;
// B rows padded to 20 doubles: the B fragment loads (row = lane/4, k =
// lane%4) then fall on 4 row + k distinct bank pairs in each half-warp
constexpr int GKM = GK + 4;
constexpr size_t kGemmMmaSmem = 2 * (size_t)(GK * GTA + GT * GKM) * sizeof(double);

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <bool A16, bool B16>
__global__ void __launch_bounds__(256, 1)
    k_dgemm_mma(int m, int n, int k, double alpha, const double *__restrict__ A, long long lda,
                const double *__restrict__ B, long long ldb, double beta, double *C, long long ldc) {
  extern __shared__ __align__(16) double gsm[];
  double *const sA0 = gsm;                 // 2 stages of [GK][GTA]
  double *const sB0 = gsm + 2 * GK * GTA;  // 2 stages of [GT][GKM]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.x * GT, n0 = blockIdx.y * GT;
  const int wm = 64 * (warp & 1), wn = 32 * (warp >> 1);
  const int fr = lane >> 2, fc = lane & 3;  // fragment row / column of this lane
  auto load = [&](int st, int k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int c = tid + 256 * i;
      const int kk = c >> 6, pa = c & 63;
      const int gr = m0 + 2 * pa, gk = k0 + kk;
      int bytes = 0;
      if (gk < k) bytes = (gr + 1 < m) ? 16 : ((gr < m) ? 8 : 0);
      cp_pair<A16>(sA0 + st * (GK * GTA) + kk * GTA + 2 * pa, A + (long long)gk * lda + gr, A, bytes);
      const int nn = c >> 3, q = c & 7;
      const int gc = n0 + nn, gk2 = k0 + 2 * q;
      int bb = 0;
      if (gc < n) bb = (gk2 + 1 < k) ? 16 : ((gk2 < k) ? 8 : 0);
      cp_pair<B16>(sB0 + st * (GT * GKM) + nn * GKM + 2 * q, B + (long long)gc * ldb + gk2, B, bb);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int nk = (k + GK - 1) / GK;
  load(0, 0);
  for (int t = 0; t < nk; ++t) {
    const int st = t & 1;
    if (t + 1 < nk) {
      load(st ^ 1, (t + 1) * GK);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const double *a_s = sA0 + st * (GK * GTA) + fc * GTA + wm + fr;
    const double *b_s = sB0 + st * (GT * GKM) + (wn + fr) * GKM + fc;
#pragma unroll
    for (int k4 = 0; k4 < GK; k4 += 4) {
      double a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = a_s[k4 * GTA + 8 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = b_s[8 * j * GKM + k4];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gn = n0 + wn + 8 * j + 2 * fc + h;
      if (gn >= n) continue;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int gm = m0 + wm + 8 * i + fr;
        if (gm < m) {
          double *c = C + (long long)gn * ldc + gm;
          *c = (beta == 0.0) ? alpha * acc[i][j][h] : alpha * acc[i][j][h] + beta * (*c);
        }
      }
    }
  }
}

// C = sum over slabs of part (slab stride m*n, ld m) scaled: C = S + beta C
__global__ void k_splitk_reduce(int m, int n, int slabs, const double *part, double beta, double *C, long long ldc) {
  const long long total = (long long)m * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int z = 0; z < slabs; ++z) s += part[(long long)z * total + i];
    const int r = (int)(i % m), c = (int)(i / m);
    double *p = C + (long long)c * ldc + r;
    *p = (beta == 0.0) ? s : s + beta * (*p);
  }
}

// ---------------------------------------------------------------------------
// Batched column operations for Ritz pairs.  Grid (gx, m); part[c*gx + b].
// ---------------------------------------------------------------------------
// mode 0: out_c = sqrt(sum U_c^2)
// mode 1: out_c = sum U_c * W_c
// mode 2: out_c = sqrt(sum (W_c - lam_c U_c)^2), with the reference's rounding
__global__ void k_colred(int n, int m, int mode, const double *U, const double *W, const double *lam,
                         double *part, unsigned int *ctr, double *out) {
  __shared__ double sh[kThreads / 32];
  const int c = blockIdx.y;
  const double *u = U + (long long)c * n;
  const double *w = W ? W + (long long)c * n : nullptr;
  const double nl = (mode == 2) ? -lam[c] : 0.0;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (mode == 0)
      s += u[i] * u[i];
    else if (mode == 1)
      s += w[i] * u[i];
    else {
      const double r = __dadd_rn(w[i], __dmul_rn(nl, u[i]));
      s += r * r;
    }
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[(long long)c * gridDim.x + blockIdx.x] = s;
  if (last_block(ctr)) {
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
      double t = 0.0;
      for (int b = 0; b < (int)gridDim.x; ++b) t += __ldcg(part + (long long)q * gridDim.x + b);
      out[q] = (mode == 1) ? t : sqrt(t);
    }
    __syncthreads();
    if (threadIdx.x == 0) *ctr = 0u;
  }
}

// U_c *= 1/norm_c
__global__ void k_colscale_inv(int n, const double *nrm, double *U) {
  const int c = blockIdx.y;
  const double t = 1.0 / nrm[c];
  double *u = U + (long long)c * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) u[i] = __dmul_rn(t, u[i]);
}

int colred(int n, int m, int mode, const double *U, const double *W, const double *lam, double *out) {
  const int gx = std::max(1, std::min(grid_for(n), std::max(1, 2048 / std::max(1, m))));
  double *part = (double *)evslcu_malloc(sizeof(double) * (size_t)gx * m);
  if (!part) return EVSLCU_ERR_NOMEM;
  dim3 g(gx, m);
  k_colred<<<g, kThreads, 0, stream()>>>(n, m, mode, U, W, lam, part, counters() + CTR_COL, out);
  count_launch();
  int rc = check_launch("k_colred");
  int rc2 = evslcu_free(part);
  return rc ? rc : rc2;
}

}  // namespace

extern "C" {

int evslcu_dot(int n, const double *x, const double *y, double *out_dev) {
  k_dot<<<grid_for(n, kThreads, 1024), kThreads, 0, stream()>>>(n, x, y, partials(), counters() + CTR_DOT, out_dev,
                                                                 0);
  EVSLCU_LAUNCH_CHECK("k_dot");
  return 0;
}

int evslcu_nrm2(int n, const double *x, double *out_dev) {
  k_dot<<<grid_for(n, kThreads, 1024), kThreads, 0, stream()>>>(n, x, x, partials(), counters() + CTR_NRM, out_dev,
                                                                 1);
  EVSLCU_LAUNCH_CHECK("k_nrm2");
  return 0;
}

int evslcu_axpy_ds(int n, const double *coef_dev, double sign, const double *x, double *y) {
  k_axpy_ds<<<grid_for(n), kThreads, 0, stream()>>>(n, coef_dev, sign, x, y);
  EVSLCU_LAUNCH_CHECK("k_axpy_ds");
  return 0;
}

int evslcu_axpy(int n, double a, const double *x, double *y) {
  k_axpy<<<grid_for(n), kThreads, 0, stream()>>>(n, a, x, y);
  EVSLCU_LAUNCH_CHECK("k_axpy");
  return 0;
}

int evslcu_scal_inv_ds(int n, const double *s_dev, double *x) {
  k_scal_inv_ds<<<grid_for(n), kThreads, 0, stream()>>>(n, s_dev, x);
  EVSLCU_LAUNCH_CHECK("k_scal_inv_ds");
  return 0;
}

int evslcu_scal(int n, double a, double *x) {
  k_scal<<<grid_for(n), kThreads, 0, stream()>>>(n, a, x);
  EVSLCU_LAUNCH_CHECK("k_scal");
  return 0;
}

int evslcu_copy(int n, const double *x, double *y) { return evslcu_d2d(y, x, sizeof(double) * (size_t)n); }

// Host staging for the batched engine operations: pinned, so the copies of
// the slot tables are asynchronous; one buffer per call site, rewritten only
// once the event recorded after its last copy has completed.
static void *g_lz_stage[2] = {nullptr, nullptr};
static size_t g_lz_stage_cap[2] = {0, 0};
static cudaEvent_t g_lz_evt[2] = {nullptr, nullptr};

static void *lz_stage(int which, size_t bytes) {
  if (g_lz_evt[which]) cudaEventSynchronize(g_lz_evt[which]);
  if (bytes > g_lz_stage_cap[which]) {
    if (g_lz_stage[which]) {
      cudaStreamSynchronize(stream());
      cudaFreeHost(g_lz_stage[which]);
    }
    g_lz_stage[which] = nullptr;
    g_lz_stage_cap[which] = 0;
    if (cudaMallocHost(&g_lz_stage[which], bytes) != cudaSuccess) {
      cudaGetLastError();
      g_lz_stage[which] = nullptr;
      return nullptr;
    }
    g_lz_stage_cap[which] = bytes;
  }
  return g_lz_stage[which];
}

// Marks the end of the copy just issued from staging buffer `which`.
static int lz_staged(int which) {
  if (!g_lz_evt[which] && cudaEventCreateWithFlags(&g_lz_evt[which], cudaEventDisableTiming) != cudaSuccess)
    return fail(EVSLCU_ERR_CUDA, "batched engine operations: event creation failed");
  if (cudaEventRecord(g_lz_evt[which], stream()) != cudaSuccess)
    return fail(EVSLCU_ERR_CUDA, "batched engine operations: event record failed");
  return 0;
}

void evslcu_lz_release(void) {
  for (int i = 0; i < 2; ++i) {
    if (g_lz_evt[i]) {
      cudaEventSynchronize(g_lz_evt[i]);
      cudaEventDestroy(g_lz_evt[i]);
    }
    g_lz_evt[i] = nullptr;
    if (g_lz_stage[i]) cudaFreeHost(g_lz_stage[i]);
    g_lz_stage[i] = nullptr;
    g_lz_stage_cap[i] = 0;
  }
}

size_t evslcu_lz_scratch_doubles(void) { return (size_t)kMaxPartials; }

size_t evslcu_lanczos_batch_table_bytes(int ns) {
  return (sizeof(LzSlot) * (size_t)std::max(ns, 1) + 255) / 256 * 256 + sizeof(int) * LZ_NPREF * ((size_t)ns + 1);
}

int evslcu_lanczos_batch(int ns, const evslcu_lz_col *cols, int imax, void *table, size_t table_bytes) {
  if (ns <= 0) return 0;
  if (!cols || !table || table_bytes < evslcu_lanczos_batch_table_bytes(ns))
    return fail(EVSLCU_ERR_ARG, "lanczos_batch: bad arguments");
  const size_t sbytes = (sizeof(LzSlot) * (size_t)ns + 255) / 256 * 256;
  const size_t bytes = evslcu_lanczos_batch_table_bytes(ns);
  unsigned char *h = (unsigned char *)lz_stage(0, bytes);
  if (!h) return fail(EVSLCU_ERR_NOMEM, "lanczos_batch: out of pinned host memory");
  LzSlot *S = reinterpret_cast<LzSlot *>(h);
  int *pre = reinterpret_cast<int *>(h + sbytes);
  for (int q = 0; q < LZ_NPREF; ++q) pre[q * (ns + 1)] = 0;
  for (int i = 0; i < ns; ++i) {
    const evslcu_lz_col &c = cols[i];
    if (c.n < 1 || c.k < 0 || !c.V || !c.ds || !c.cgsw || !c.npart)
      return fail(EVSLCU_ERR_ARG, "lanczos_batch: bad column %d", i);
    LzSlot &L = S[i];
    L.n = c.n;
    L.kc = c.k + 1;
    L.g_dot = grid_for(c.n, kThreads, 1024);
    L.nchunks = (c.n + kGemvTRows - 1) / kGemvTRows;
    L.ctiles = (L.kc + kGemvTCols - 1) / kGemvTCols;
    L.g_n = grid_for(c.n, kThreads, kMaxPartials);
    L.nbeta = -c.beta;
    L.V = c.V;
    L.v = c.V + (size_t)c.k * c.n;
    L.vprev = c.k > 0 ? c.V + (size_t)(c.k - 1) * c.n : nullptr;
    L.z = c.V + (size_t)(c.k + 1) * c.n;
    L.ds = c.ds;
    L.part = c.cgsw;
    L.npart = c.npart;
    const int cnt[LZ_NPREF] = {L.g_dot, L.nchunks * L.ctiles, (L.kc + 31) / 32, L.g_n, 1};
    for (int q = 0; q < LZ_NPREF; ++q) pre[q * (ns + 1) + i + 1] = pre[q * (ns + 1) + i] + cnt[q];
  }
  int rc = evslcu_h2d_async(table, h, bytes);
  if (!rc) rc = lz_staged(0);
  if (rc) return rc;
  const LzSlot *dS = reinterpret_cast<const LzSlot *>(table);
  const int *dpre = reinterpret_cast<const int *>(static_cast<unsigned char *>(table) + sbytes);
  auto P = [&](int q) { return dpre + q * (ns + 1); };
  auto G = [&](int q) { return pre[q * (ns + 1) + ns]; };
  cudaStream_t st = stream();
  k_lz_axpy_dot<<<G(LZ_DOT), kThreads, 0, st>>>(dS, P(LZ_DOT), ns);
  EVSLCU_LAUNCH_CHECK("k_lz_axpy_dot");
  k_lz_alpha<<<ns, kThreads, 0, st>>>(dS);
  EVSLCU_LAUNCH_CHECK("k_lz_alpha");
  k_lz_axpy_nrm<<<G(LZ_DOT), kThreads, 0, st>>>(dS, P(LZ_DOT), ns);
  EVSLCU_LAUNCH_CHECK("k_lz_axpy_nrm");
  k_lz_cgs_init<<<ns, kThreads, 0, st>>>(dS);
  EVSLCU_LAUNCH_CHECK("k_lz_cgs_init");
  for (int pass = 0; pass < imax; ++pass) {
    k_lz_gemvT<<<G(LZ_T), kThreads, 0, st>>>(dS, P(LZ_T), ns);
    EVSLCU_LAUNCH_CHECK("k_lz_gemvT");
    k_lz_gemvT_reduce<<<G(LZ_TR), 256, 0, st>>>(dS, P(LZ_TR), ns);
    EVSLCU_LAUNCH_CHECK("k_lz_gemvT_reduce");
    k_lz_gemvN<<<G(LZ_N), kThreads, 0, st>>>(dS, P(LZ_N), ns);
    EVSLCU_LAUNCH_CHECK("k_lz_gemvN");
    k_lz_dgks<<<ns, kThreads, 0, st>>>(dS);
    EVSLCU_LAUNCH_CHECK("k_lz_dgks");
  }
  return 0;
}

size_t evslcu_scal_batch_table_bytes(int ns) {
  return (sizeof(LzScale) * (size_t)std::max(ns, 1) + 255) / 256 * 256 + sizeof(int) * ((size_t)ns + 1);
}

int evslcu_scal_batch(int ns, const int *n, double *const *x, const double *a, void *table, size_t table_bytes) {
  if (ns <= 0) return 0;
  if (!n || !x || !a || !table || table_bytes < evslcu_scal_batch_table_bytes(ns))
    return fail(EVSLCU_ERR_ARG, "scal_batch: bad arguments");
  const size_t sbytes = (sizeof(LzScale) * (size_t)ns + 255) / 256 * 256;
  const size_t bytes = evslcu_scal_batch_table_bytes(ns);
  unsigned char *h = (unsigned char *)lz_stage(1, bytes);
  if (!h) return fail(EVSLCU_ERR_NOMEM, "scal_batch: out of pinned host memory");
  LzScale *S = reinterpret_cast<LzScale *>(h);
  int *pre = reinterpret_cast<int *>(h + sbytes);
  pre[0] = 0;
  for (int i = 0; i < ns; ++i) {
    S[i].n = n[i];
    S[i].g = grid_for(n[i]);
    S[i].a = a[i];
    S[i].x = x[i];
    pre[i + 1] = pre[i] + S[i].g;
  }
  int rc = evslcu_h2d_async(table, h, bytes);
  if (!rc) rc = lz_staged(1);
  if (rc) return rc;
  k_lz_scal<<<pre[ns], kThreads, 0, stream()>>>(reinterpret_cast<const LzScale *>(table),
                                                reinterpret_cast<const int *>(static_cast<unsigned char *>(table) +
                                                                              sbytes),
                                                ns);
  EVSLCU_LAUNCH_CHECK("k_lz_scal");
  return 0;
}

size_t evslcu_cgs_work_size(int n, int k) {
  const size_t nchunks = ((size_t)n + kGemvTRows - 1) / kGemvTRows;
  return nchunks * (size_t)std::max(k, 1) + (size_t)std::max(k, 1) + 8;
}

// Block classical Gram-Schmidt, twice (BCGS2), on the m columns of W (ld
// n): each block of b columns is first projected against every earlier
// column by two passes of two GEMMs (H = W_prev^T W_b, W_b -= W_prev H: the
// earlier columns are read once per block, not once per column), then its
// columns are orthonormalised among themselves by classical Gram-Schmidt
// with the DGKS test (SRC/misc_la.c:221-261) and scaled to unit norm.
// H: (m - b) x b doubles of device scratch; norm_dev: one device double;
// cgsw: evslcu_cgs_work_size(n, b) doubles.
int evslcu_block_cgs2(int n, int m, double *W, int b, double *H, double *norm_dev, double *cgsw) {
  if (n < 1 || m < 1 || b < 1 || !W || !H || !norm_dev || !cgsw) return fail(EVSLCU_ERR_ARG, "block_cgs2: bad arguments");
  int rc = 0;
  for (int c0 = 0; !rc && c0 < m; c0 += b) {
    const int nb = std::min(b, m - c0);
    double *Wb = W + (size_t)c0 * n;
    for (int pass = 0; !rc && c0 > 0 && pass < 2; ++pass) {
      rc = evslcu_dgemm('T', 'N', c0, nb, n, 1.0, W, n, Wb, n, 0.0, H, c0);
      if (!rc) rc = evslcu_dgemm('N', 'N', n, nb, c0, -1.0, W, n, H, c0, 1.0, Wb, n);
    }
    for (int j = 0; !rc && j < nb; ++j) {
      double *wj = Wb + (size_t)j * n;
      rc = (j == 0) ? evslcu_nrm2(n, wj, norm_dev) : evslcu_cgs_dgks(n, j, EVSL_NGS_MAX_CU, Wb, n, wj, norm_dev, cgsw);
      if (!rc) rc = evslcu_scal_inv_ds(n, norm_dev, wj);
    }
  }
  return rc;
}

int evslcu_cgs_dgks(int n, int k, int imax, const double *Q, long long ldq, double *v, double *nrm_out_dev,
                    double *work) {
  if (k < 1 || n < 1) return fail(EVSLCU_ERR_ARG, "cgs: bad sizes n=%d k=%d", n, k);
  const int nchunks = (n + kGemvTRows - 1) / kGemvTRows;
  double *part = work;
  double *h = work + (size_t)nchunks * k;
  double *state = h + k;
  double *nrm0 = state + 4;
  cudaStream_t st = stream();
  int rc;
  if ((rc = evslcu_nrm2(n, v, nrm0))) return rc;
  k_cgs_init<<<1, 1, 0, st>>>(state, nrm0);
  EVSLCU_LAUNCH_CHECK("k_cgs_init");
  const dim3 gT(nchunks, (k + kGemvTCols - 1) / kGemvTCols);
  const int gN = grid_for(n, kThreads, kMaxPartials);
  for (int pass = 0; pass < imax; ++pass) {
    k_gemvT_partial<<<gT, kThreads, 0, st>>>(n, k, Q, ldq, v, part, state);
    EVSLCU_LAUNCH_CHECK("k_gemvT_partial");
    k_gemvT_reduce<<<(k + 31) / 32, 256, 0, st>>>(nchunks, k, part, 1.0, 0.0, h, state);
    EVSLCU_LAUNCH_CHECK("k_gemvT_reduce");
    k_gemvN<<<gN, kThreads, 0, st>>>(n, k, Q, ldq, h, -1.0, v, partials(), counters() + CTR_CGS, state);
    EVSLCU_LAUNCH_CHECK("k_gemvN");
  }
  if (nrm_out_dev) {
    k_copy_scalar<<<1, 1, 0, st>>>(state + 1, nrm_out_dev);
    EVSLCU_LAUNCH_CHECK("k_copy_scalar");
  }
  return 0;
}

int evslcu_dgemv(char trans, int m, int n, double alpha, const double *A, long long lda, const double *x,
                 double beta, double *y) {
  cudaStream_t st = stream();
  const bool T = (trans == 'T' || trans == 't');
  if (m <= 0 || n <= 0) return 0;
  if (T) {
    // y (n) = alpha A^T x + beta y; A is m x n
    const int nchunks = (m + kGemvTRows - 1) / kGemvTRows;
    double *part = (double *)evslcu_malloc(sizeof(double) * (size_t)nchunks * n);
    if (!part) return EVSLCU_ERR_NOMEM;
    const dim3 gT(nchunks, (n + kGemvTCols - 1) / kGemvTCols);
    k_gemvT_partial<<<gT, kThreads, 0, st>>>(m, n, A, lda, x, part, nullptr);
    count_launch();
    int rc = check_launch("k_gemvT_partial");
    if (!rc) {
      k_gemvT_reduce<<<(n + 31) / 32, 256, 0, st>>>(nchunks, n, part, alpha, beta, y, nullptr);
      count_launch();
      rc = check_launch("k_gemvT_reduce");
    }
    evslcu_free(part);
    return rc;
  }
  // y (m) = beta y + alpha A x
  if (beta != 1.0) {
    k_scale_vec<<<grid_for(m), kThreads, 0, st>>>(m, beta, y);
    EVSLCU_LAUNCH_CHECK("k_scale_vec");
  }
  k_gemvN<<<grid_for(m, kThreads, kMaxPartials), kThreads, 0, st>>>(m, n, A, lda, x, alpha, y, nullptr, nullptr,
                                                                      nullptr);
  EVSLCU_LAUNCH_CHECK("k_gemvN");
  return 0;
}

// FP64 throughput probe (the roofline's FP64 peak): chains of FMA on each
// thread, and chains of mma.sync m8n8k4 f64 on each warp, registers only;
// every thread writes one value so the work is kept.  out: blocks x 256.
__global__ void __launch_bounds__(256) k_probe_dfma(int iters, double seed, double *out) {
  double a[8];
  const double b = seed * 0.5 + 1.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + i;
  for (int it = 0; it < iters; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = fma(a[i], b, 1e-9);
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_probe_dmma(int iters, double seed, double *out) {
  double c[8][2];
  const double a = seed + threadIdx.x * 1e-3, b = seed - threadIdx.x * 1e-3;
#pragma unroll
  for (int i = 0; i < 8; ++i) c[i][0] = c[i][1] = 0.0;
  for (int it = 0; it < iters; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(c[i][0]), "+d"(c[i][1])
                   : "d"(a), "d"(b));
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += c[i][0] + c[i][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

static int g_dgemm_tiled = 2;

int evslcu_fp64_probe(double *dfma_tflops, double *dmma_tflops) {
  const int blocks = 4 * sm_count(), iters = 1 << 14;
  double *out = (double *)evslcu_malloc(sizeof(double) * (size_t)blocks * 256);
  if (!out) return EVSLCU_ERR_NOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float ms[2] = {0.f, 0.f};
  int rc = 0;
  for (int rep = 0; rep < 2 && !rc; ++rep)
    for (int which = 0; which < 2 && !rc; ++which) {
      cudaEventRecord(e0, stream());
      if (which == 0)
        k_probe_dfma<<<blocks, 256, 0, stream()>>>(iters, 1.0, out);
      else
        k_probe_dmma<<<blocks, 256, 0, stream()>>>(iters, 1.0, out);
      count_launch();
      cudaEventRecord(e1, stream());
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(EVSLCU_ERR_CUDA, "fp64 probe failed");
      if (!rc) rc = check_launch("fp64 probe");
      if (!rc) cudaEventElapsedTime(&ms[which], e0, e1);
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  evslcu_free(out);
  if (rc) return rc;
  const double threads = (double)blocks * 256;
  if (dfma_tflops) *dfma_tflops = 2.0 * 8 * iters * threads / (ms[0] * 1e-3) / 1e12;
  if (dmma_tflops) *dmma_tflops = 2.0 * 256 * 8 * iters * (threads / 32) / (ms[1] * 1e-3) / 1e12;
  return 0;
}

int evslcu_set_dgemm_tiled(int on) {
  const int prev = g_dgemm_tiled;
  g_dgemm_tiled = (on == 2) ? 2 : (on ? 1 : 0);
  return prev;
}

static double *g_splitk = nullptr;  // split-K partial products (cached)
static size_t g_splitk_cap = 0;

int evslcu_dgemm(char ta, char tb, int m, int n, int k, double alpha, const double *A, long long lda,
                 const double *B, long long ldb, double beta, double *C, long long ldc) {
  if (m <= 0 || n <= 0) return 0;
  const bool TA = (ta == 'T' || ta == 't'), TB = (tb == 'T' || tb == 't');
  cudaStream_t st = stream();
  // tall products (Ritz vectors V Y, block updates): the 128 x 128 kernel
  if (!TA && !TB && g_dgemm_tiled && m >= 2 * GT && n >= 32 && k >= GK &&
      ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 7) == 0) {
    const bool a16 = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda & 1) == 0;
    const bool b16 = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb & 1) == 0;
    if (g_dgemm_tiled == 2) {
      auto gom = [&](auto fn) -> int {
        static bool smem_set[4] = {false, false, false, false};
        const int idx = (a16 ? 2 : 0) + (b16 ? 1 : 0);
        if (!smem_set[idx]) {
          cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmMmaSmem);
          if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "dgemm: shared memory limit: %s", cudaGetErrorString(e));
          smem_set[idx] = true;
        }
        dim3 g((m + GT - 1) / GT, (n + GT - 1) / GT);
        fn<<<g, 256, kGemmMmaSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
        count_launch();
        return check_launch("k_dgemm_mma");
      };
      if (a16 && b16) return gom(k_dgemm_mma<true, true>);
      if (a16) return gom(k_dgemm_mma<true, false>);
      if (b16) return gom(k_dgemm_mma<false, true>);
      return gom(k_dgemm_mma<false, false>);
    }
    auto go = [&](auto fn) -> int {
      static bool smem_set[4] = {false, false, false, false};
      const int idx = (a16 ? 2 : 0) + (b16 ? 1 : 0);
      if (!smem_set[idx]) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
        if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "dgemm: shared memory limit: %s", cudaGetErrorString(e));
        smem_set[idx] = true;
      }
      dim3 g((m + GT - 1) / GT, (n + GT - 1) / GT);
      fn<<<g, 256, kGemmSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
      count_launch();
      return check_launch("k_dgemm_nn128");
    };
    if (a16 && b16) return go(k_dgemm_nn128<true, true>);
    if (a16) return go(k_dgemm_nn128<true, false>);
    if (b16) return go(k_dgemm_nn128<false, true>);
    return go(k_dgemm_nn128<false, false>);
  }
  const int gm = (m + BM - 1) / BM, gn = (n + BN - 1) / BN;
  // Long inner dimension with few output tiles (V^T W): split K into slabs
  // (at least 2048 deep) so that the blocks fill the GPU about four times,
  // computed in parallel, then summed in slab order (deterministic).
  int slabs = 1, kchunk = 0;
  const long long tiles = (long long)gm * gn, fill = 4LL * sm_count();
  if ((long long)k >= 8192 && tiles < fill) {
    slabs = (int)std::min<long long>((fill + tiles - 1) / tiles, (k + 2047) / 2048);
    kchunk = (int)(((k + slabs - 1) / slabs + BK - 1) / BK * BK);
    slabs = (k + kchunk - 1) / kchunk;
  }
  double *part = nullptr;
  double *Cout = C;
  long long ldo = ldc, cstride = 0;
  double a = alpha, b = beta;
  if (slabs > 1) {
    // the slabs' partial products live in a cached buffer (grown, never
    // shrunk until finish): no allocation per call
    const size_t need = (size_t)slabs * m * n;
    if (need > g_splitk_cap) {
      if (g_splitk) {
        cudaStreamSynchronize(st);
        evslcu_free(g_splitk);
      }
      g_splitk = (double *)evslcu_malloc(sizeof(double) * need);
      g_splitk_cap = g_splitk ? need : 0;
      if (!g_splitk) return EVSLCU_ERR_NOMEM;
    }
    part = g_splitk;
    Cout = part;
    ldo = m;
    cstride = (long long)m * n;
    b = 0.0;
  }
  dim3 g(gm, gn, slabs);
  const int kc = (slabs > 1) ? kchunk : 0;
  if (!TA && !TB)
    k_dgemm<false, false><<<g, 256, 0, st>>>(m, n, 0, k, a, A, lda, B, ldb, b, Cout, ldo, cstride, kc);
  else if (TA && !TB)
    k_dgemm<true, false><<<g, 256, 0, st>>>(m, n, 0, k, a, A, lda, B, ldb, b, Cout, ldo, cstride, kc);
  else if (!TA && TB)
    k_dgemm<false, true><<<g, 256, 0, st>>>(m, n, 0, k, a, A, lda, B, ldb, b, Cout, ldo, cstride, kc);
  else
    k_dgemm<true, true><<<g, 256, 0, st>>>(m, n, 0, k, a, A, lda, B, ldb, b, Cout, ldo, cstride, kc);
  count_launch();
  int rc = check_launch("k_dgemm");
  if (!rc && slabs > 1) {
    k_splitk_reduce<<<grid_for((long long)m * n), kThreads, 0, st>>>(m, n, slabs, part, beta, C, ldc);
    count_launch();
    rc = check_launch("k_splitk_reduce");
  }
  return rc;
}

void evslcu_gemm_release(void) {
  evslcu_free(g_splitk);
  g_splitk = nullptr;
  g_splitk_cap = 0;
}

int evslcu_ritz_eval(const evslcu_op *op, int n, int m, double *U, double *W, double *norm, double *lam,
                     double *res) {
  if (m <= 0) return 0;
  double *d = (double *)evslcu_malloc(sizeof(double) * 3 * (size_t)m);
  if (!d) return EVSLCU_ERR_NOMEM;
  double *dn = d, *dl = d + m, *dr = d + 2 * m;
  int rc = colred(n, m, 0, U, nullptr, nullptr, dn);
  if (!rc) {
    dim3 g(std::min(grid_for(n), 1024), m);
    k_colscale_inv<<<g, kThreads, 0, stream()>>>(n, dn, U);
    count_launch();
    rc = check_launch("k_colscale_inv");
  }
  if (!rc && op->A) rc = evslcu_spmv_cols(op->A, U, W, m);  // all m products in one launch
  for (int c = 0; !rc && !op->A && c < m; ++c) {
    cudaError_t e = cudaStreamSynchronize(stream());
    if (e != cudaSuccess) rc = fail(EVSLCU_ERR_CUDA, "sync before matvec: %s", cudaGetErrorString(e));
    if (!rc) op->func(U + (size_t)c * n, W + (size_t)c * n, op->data);
  }
  if (!rc) rc = colred(n, m, 1, U, W, nullptr, dl);
  if (!rc) rc = colred(n, m, 2, U, W, dl, dr);
  if (!rc) rc = evslcu_d2h(norm, dn, sizeof(double) * m);
  if (!rc) rc = evslcu_d2h(lam, dl, sizeof(double) * m);
  if (!rc) rc = evslcu_d2h(res, dr, sizeof(double) * m);
  evslcu_free(d);
  return rc;
}

int evslcu_gather_cols(int n, int cnt, const int *idx, const double *src, double *dst) {
  for (int j = 0; j < cnt; ++j) {
    if (idx[j] == j && src == dst) continue;
    int rc = evslcu_d2d(dst + (size_t)j * n, src + (size_t)idx[j] * n, sizeof(double) * (size_t)n);
    if (rc) return rc;
  }
  return 0;
}

int evslcu_colnorms(int n, int m, const double *U, double *norms) {
  if (m <= 0) return 0;
  double *d = (double *)evslcu_malloc(sizeof(double) * (size_t)m);
  if (!d) return EVSLCU_ERR_NOMEM;
  int rc = colred(n, m, 0, U, nullptr, nullptr, d);
  if (!rc) rc = evslcu_d2h(norms, d, sizeof(double) * m);
  evslcu_free(d);
  return rc;
}

}  // extern "C"
