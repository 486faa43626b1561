// Sparse operator, fused Chebyshev filter steps, KPM block moments and the
// device random-vector generator.
//
// Filter kernels (reference ChebAv, SRC/chebpoly.c:519-598, and its CUDA
// update kernel SRC/evsl_cuda.cu:175-191):
//   * one thread per row; the row's products are summed left to right with
//     explicitly rounded multiply and add (no FMA contraction), which is the
//     arithmetic of the reference CPU build's CSR matvec (SRC/spmat.c:257-298);
//   * the Chebyshev update w = t*(A vk - cc vk) - vkm1, y += mu_k w is applied
//     in the reference's operation order (daxpy, dscal, daxpy, daxpy;
//     SRC/chebpoly.c:575-582) in the epilogue, so the filtered vector equals
//     the reference CPU result bit for bit;
//   * matrix storage is SELL-32 (chunks of 32 rows, column-major inside the
//     chunk, padded with zeros) so every warp load is coalesced; the plain
//     CSR thread-per-row kernel is kept as an alternative.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "sparse_types.cuh"

using namespace evslcu;

// ---------------------------------------------------------------------------
// Constant-memory copy of the row-pattern tables.  The rows of a warp mostly
// share one pattern, so the table reads are warp-uniform and the constant
// cache serves them without using the L1 data path that the vector gathers
// need.  Matrices claim regions of this fixed pool when they are created; a
// table that does not fit is read from global memory instead (PatView).
// ---------------------------------------------------------------------------
constexpr int kCPoolEntries = 3072;
constexpr int kCPoolHeaders = 1024;
// c_pat_w: packed entries (float value, offset) for tables whose values are
// all exactly floats, otherwise the double value bits with the offset in
// c_pat_off.
__constant__ unsigned long long c_pat_w[kCPoolEntries];
__constant__ int c_pat_off[kCPoolEntries];
__constant__ int2 c_pat_hdr[kCPoolHeaders];

namespace evslcu {

struct PatCView {
  int n;
  const unsigned short *__restrict__ pid;
  int hbase;  // this matrix's first header in the pool
};

template <bool COHERENT>
__device__ __forceinline__ double row_dot(const PatCView &A, int r, const double *x) {
  const int2 h = c_pat_hdr[A.hbase + __ldg(A.pid + r)];
  const double *xr = x + r;
  double acc = 0.0;
  for (int j = 0; j < h.y; ++j)
    acc = __dadd_rn(acc, __dmul_rn(__longlong_as_double((long long)c_pat_w[h.x + j]),
                                   ldx<COHERENT>(xr + c_pat_off[h.x + j])));
  return acc;
}

template <int WMAX, bool COHERENT>
__device__ __forceinline__ double row_dot_w(const PatCView &A, int r, const double *x) {
  const int2 h = c_pat_hdr[A.hbase + __ldg(A.pid + r)];
  const double *xr = x + r;
  double g[WMAX];
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < h.y) g[j] = ldx<COHERENT>(xr + c_pat_off[h.x + j]);
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < h.y) acc = __dadd_rn(acc, __dmul_rn(__longlong_as_double((long long)c_pat_w[h.x + j]), g[j]));
  return acc;
}

// Packed constant table: one constant load per entry.
struct PatCPView {
  int n;
  const unsigned short *__restrict__ pid;
  int hbase;
};

template <bool COHERENT>
__device__ __forceinline__ double row_dot(const PatCPView &A, int r, const double *x) {
  const int2 h = c_pat_hdr[A.hbase + __ldg(A.pid + r)];
  const double *xr = x + r;
  double acc = 0.0;
  for (int j = 0; j < h.y; ++j) {
    const unsigned long long e = c_pat_w[h.x + j];
    acc = __dadd_rn(acc, __dmul_rn(pat_val(e), ldx<COHERENT>(xr + pat_off(e))));
  }
  return acc;
}

template <int WMAX, bool COHERENT>
__device__ __forceinline__ double row_dot_w(const PatCPView &A, int r, const double *x) {
  const int2 h = c_pat_hdr[A.hbase + __ldg(A.pid + r)];
  const double *xr = x + r;
  unsigned long long e[WMAX];
  double g[WMAX];
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < h.y) {
      e[j] = c_pat_w[h.x + j];
      g[j] = ldx<COHERENT>(xr + pat_off(e[j]));
    }
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < h.y) acc = __dadd_rn(acc, __dmul_rn(pat_val(e[j]), g[j]));
  return acc;
}

// Constant table addressed by a per-row descriptor (first pool entry << 8 |
// count) instead of a pattern id: no header lookup on the row's dependent
// chain, for 2 more bytes per row.  PACKED: entries as in PatCPView, else
// double values with the offsets in c_pat_off.
template <bool PACKED>
struct PatCDView {
  int n;
  const unsigned *__restrict__ desc;
};

template <bool PACKED>
__device__ __forceinline__ void pat_centry(int idx, double &v, int &off) {
  const unsigned long long e = c_pat_w[idx];
  if (PACKED) {
    v = pat_val(e);
    off = pat_off(e);
  } else {
    v = __longlong_as_double((long long)e);
    off = c_pat_off[idx];
  }
}

template <bool COHERENT, bool PACKED>
__device__ __forceinline__ double row_dot(const PatCDView<PACKED> &A, int r, const double *x) {
  const unsigned d = __ldg(A.desc + r);
  const int b = (int)(d >> 8), len = (int)(d & 255u);
  const double *xr = x + r;
  double acc = 0.0;
  for (int j = 0; j < len; ++j) {
    double v;
    int off;
    pat_centry<PACKED>(b + j, v, off);
    acc = __dadd_rn(acc, __dmul_rn(v, ldx<COHERENT>(xr + off)));
  }
  return acc;
}

template <int WMAX, bool COHERENT, bool PACKED>
__device__ __forceinline__ double row_dot_w(const PatCDView<PACKED> &A, int r, const double *x) {
  const unsigned d = __ldg(A.desc + r);
  const int b = (int)(d >> 8), len = (int)(d & 255u);
  const double *xr = x + r;
  double v[WMAX], g[WMAX];
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < len) {
      int off;
      pat_centry<PACKED>(b + j, v[j], off);
      g[j] = ldx<COHERENT>(xr + off);
    }
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < WMAX; ++j)
    if (j < len) acc = __dadd_rn(acc, __dmul_rn(v[j], g[j]));
  return acc;
}

}  // namespace evslcu

namespace {

// desc[r] = (first pool entry of r's pattern) << 8 | its count.
__global__ void k_pat_desc(int n, const unsigned short *pid, const int2 *hdr, int ebase, unsigned *desc) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int2 h = hdr[pid[r]];
    desc[r] = ((unsigned)(h.x + ebase) << 8) | (unsigned)h.y;
  }
}

// First-fit allocator of pool slots (host side; the library runs on one
// stream and one host thread per process).
struct SlotPool {
  int cap;
  std::vector<std::pair<int, int>> used;  // (base, length), sorted by base
  int claim(int len) {
    int at = 0;
    size_t i = 0;
    for (; i < used.size(); ++i) {
      if (used[i].first - at >= len) break;
      at = used[i].first + used[i].second;
    }
    if (len <= 0 || at + len > cap) return -1;
    used.insert(used.begin() + (long)i, {at, len});
    return at;
  }
  void release(int base) {
    for (size_t i = 0; i < used.size(); ++i)
      if (used[i].first == base) {
        used.erase(used.begin() + (long)i);
        return;
      }
  }
};

SlotPool g_cpool_ent{kCPoolEntries, {}};
SlotPool g_cpool_hdr{kCPoolHeaders, {}};
int g_pattern_const = 1;

// Copies M's pattern table into the constant pool when there is room.
int pat_const_claim(evslcu_mat *M) {
  if (!M->pat_id || M->npat <= 0) return 0;
  const int eb = g_cpool_ent.claim(M->pat_entries), hb = g_cpool_hdr.claim(M->npat);
  if (eb < 0 || hb < 0) {
    if (eb >= 0) g_cpool_ent.release(eb);
    if (hb >= 0) g_cpool_hdr.release(hb);
    return 0;
  }
  const size_t hbytes = pat_hdr_bytes(M->npat);
  std::vector<int2> hdr(M->npat);
  std::vector<double2> ent(M->pat_entries);
  std::vector<unsigned long long> w(M->pat_entries);
  int rc = evslcu_d2h(hdr.data(), M->pat_table, sizeof(int2) * M->npat);
  if (!rc) rc = evslcu_d2h(ent.data(), (const char *)M->pat_table + hbytes, sizeof(double2) * M->pat_entries);
  if (!rc && M->pat_f32)
    rc = evslcu_d2h(w.data(), (const char *)M->pat_table + hbytes + sizeof(double2) * M->pat_entries,
                    sizeof(unsigned long long) * M->pat_entries);
  std::vector<int> off(M->pat_entries);
  for (int j = 0; j < M->pat_entries; ++j) {
    long long bits;
    memcpy(&bits, &ent[j].y, sizeof(bits));
    off[j] = (int)bits;
    if (!M->pat_f32) memcpy(&w[j], &ent[j].x, sizeof(double));
  }
  for (auto &h : hdr) h.x += eb;
  cudaError_t e = cudaSuccess;
  if (!rc) {
    e = cudaMemcpyToSymbolAsync(c_pat_w, w.data(), sizeof(unsigned long long) * w.size(),
                                sizeof(unsigned long long) * eb, cudaMemcpyHostToDevice, stream());
    if (e == cudaSuccess)
      e = cudaMemcpyToSymbolAsync(c_pat_off, off.data(), sizeof(int) * off.size(), sizeof(int) * eb,
                                  cudaMemcpyHostToDevice, stream());
    if (e == cudaSuccess)
      e = cudaMemcpyToSymbolAsync(c_pat_hdr, hdr.data(), sizeof(int2) * hdr.size(), sizeof(int2) * hb,
                                  cudaMemcpyHostToDevice, stream());
    if (e == cudaSuccess) rc = evslcu_sync();
  }
  if (rc || e != cudaSuccess) {
    g_cpool_ent.release(eb);
    g_cpool_hdr.release(hb);
    if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "pattern table copy failed: %s", cudaGetErrorString(e));
    return rc;
  }
  M->pat_cent = eb;
  M->pat_chdr = hb;
  // per-row descriptors (optional: counts must fit 8 bits)
  if (M->pat_maxlen <= 255) {
    M->pat_desc = (unsigned *)evslcu_malloc(sizeof(unsigned) * (size_t)M->n);
    if (M->pat_desc) {
      k_pat_desc<<<grid_for(M->n), kThreads, 0, stream()>>>(M->n, M->pat_id, (const int2 *)M->pat_table, eb,
                                                            M->pat_desc);
      count_launch();
      if (check_launch("k_pat_desc")) {
        evslcu_free(M->pat_desc);
        M->pat_desc = nullptr;
      }
    }
  }
  return 0;
}

void pat_const_release(evslcu_mat *M) {
  evslcu_free(M->pat_desc);
  M->pat_desc = nullptr;
  if (M->pat_chdr < 0) return;
  g_cpool_ent.release(M->pat_cent);
  g_cpool_hdr.release(M->pat_chdr);
  M->pat_cent = M->pat_chdr = -1;
}

}  // namespace


namespace {

template <class M>
__global__ void __launch_bounds__(kThreads) k_spmv(M A, const double *__restrict__ x, double *__restrict__ y) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < A.n; s += gridDim.x * blockDim.x)
    y[row_of(A, s)] = row_dot<false>(A, s, x);
}

// Y(:, c) = A X(:, c) for the m columns of column-major X, Y (leading
// dimension ld), column c in blockIdx.y: each row is k_spmv's row product,
// so every column equals evslcu_spmv of that column bit for bit.
template <class M>
__global__ void __launch_bounds__(kThreads)
    k_spmv_cols(M A, const double *__restrict__ X, double *__restrict__ Y, long long ld) {
  const double *x = X + (long long)blockIdx.y * ld;
  double *y = Y + (long long)blockIdx.y * ld;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < A.n; s += gridDim.x * blockDim.x)
    y[row_of(A, s)] = row_dot<false>(A, s, x);
}

// One Chebyshev degree step k (FIRST: k == 1; EPI: k == deg, Lanczos epilogue).
//   out may alias vkm1 (each thread reads vkm1[r] before writing out[r]).
//   WMAX > 0: rows have at most WMAX stored entries (unrolled row products);
//   the epilogue's loads of vkm1[r] and y[r] are issued before the row's
//   gathers so that their latency overlaps.
template <class M, bool FIRST, bool EPI, int WMAX>
__global__ void __launch_bounds__(kThreads)
    k_cheb(M A, const double *__restrict__ vk, const double *vkm1, double *out, double *__restrict__ y, double t,
           double ncc, double s, double mu0, const double *__restrict__ zold, double nbeta,
           const double *__restrict__ dotv, double *part, unsigned int *ctr, double *dot_out) {
  __shared__ double sh[kThreads / 32];
  // Programmatic dependent launch: let the next degree's kernel start its
  // launch now, and wait here until the previous kernel has completed and its
  // writes are visible (no-ops when launched without the attribute).
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  double dsum = 0.0;
  for (int sl = blockIdx.x * blockDim.x + threadIdx.x; sl < A.n; sl += gridDim.x * blockDim.x) {
    const int r = row_of(A, sl);  // slot sl holds row r (sigma-sorted SELL storage), else r == sl
    const double xm1 = FIRST ? 0.0 : vkm1[r];
    const double yo = FIRST ? 0.0 : y[r];
    const double acc = row_dot_any<WMAX, false>(A, sl, vk);
    const double x = vk[r];
    // vkp1 = A vk; vkp1 += (-cc) vk; vkp1 *= t; vkp1 += (-1) vkm1
    double w = __dmul_rn(t, __dadd_rn(acc, __dmul_rn(ncc, x)));
    if (!FIRST) w = __dadd_rn(w, -xm1);
    out[r] = w;
    // k == 1: y = mu0 * v (v == vk); then y += mu_k * w
    double yv = FIRST ? __dmul_rn(mu0, x) : yo;
    yv = __dadd_rn(yv, __dmul_rn(s, w));
    if (EPI) {
      if (zold) yv = __dadd_rn(yv, __dmul_rn(nbeta, zold[r]));
      if (dotv) dsum += dotv[r] * yv;
    }
    y[r] = yv;
  }
  if (EPI && dot_out) {
    double b = block_sum(dsum, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = b;
    if (last_block(ctr)) {
      double tot = reduce_partials(part, gridDim.x, ctr, sh);
      if (threadIdx.x == 0) *dot_out = tot;
    }
  }
}

// Two rows per thread (SELL-32 only): thread (warp w, lane l) handles rows
// 64*w' + l and 64*w' + 32 + l of chunk pair w'.  Same arithmetic per row.
template <class VT, class IT, bool FIRST, bool EPI>
__global__ void __launch_bounds__(kThreads)
    k_cheb2(SellT<VT, IT> A, const double *__restrict__ vk, const double *vkm1, double *out, double *__restrict__ y,
            double t, double ncc, double s, double mu0, const double *__restrict__ zold, double nbeta,
            const double *__restrict__ dotv, double *part, unsigned int *ctr, double *dot_out) {
  __shared__ double sh[kThreads / 32];
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  double dsum = 0.0;
  const int lane = threadIdx.x & 31;
  const int nwt = gridDim.x * (kThreads / 32);
  const int npairs = (A.n + 63) / 64;
  for (int pr = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); pr < npairs; pr += nwt) {
    const int s0 = pr * 64 + lane;
    const bool has0 = s0 < A.n, has1 = s0 + 32 < A.n;
    double acc[2];
    row_dot2<false>(A, s0, has0, has1, vk, acc[0], acc[1]);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 0 ? has0 : has1) {
        const int r = row_of(A, s0 + 32 * h);
        const double x = vk[r];
        double w = __dmul_rn(t, __dadd_rn(acc[h], __dmul_rn(ncc, x)));
        if (!FIRST) w = __dadd_rn(w, -vkm1[r]);
        out[r] = w;
        double yv = FIRST ? __dmul_rn(mu0, x) : y[r];
        yv = __dadd_rn(yv, __dmul_rn(s, w));
        if (EPI) {
          if (zold) yv = __dadd_rn(yv, __dmul_rn(nbeta, zold[r]));
          if (dotv) dsum += dotv[r] * yv;
        }
        y[r] = yv;
      }
    }
  }
  if (EPI && dot_out) {
    double b = block_sum(dsum, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = b;
    if (last_block(ctr)) {
      double tot = reduce_partials(part, gridDim.x, ctr, sh);
      if (threadIdx.x == 0) *dot_out = tot;
    }
  }
}

// Stand-alone update for a user matvec (SRC/evsl_cuda.cu:175-184 semantics,
// CPU-build operation order).
__global__ void k_cheb_update(int n, int k, double t, double s, double ncc, double *vkp1, const double *vk,
                              const double *vkm1, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double w = __dmul_rn(t, __dadd_rn(vkp1[i], __dmul_rn(ncc, vk[i])));
    if (k > 1) w = __dadd_rn(w, -vkm1[i]);
    vkp1[i] = w;
    y[i] = __dadd_rn(y[i], __dmul_rn(s, w));
  }
}

__global__ void k_scale_copy(int n, double a, const double *x, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = __dmul_rn(a, x[i]);
}

// Lanczos epilogue when the last step could not be fused (user matvec).
__global__ void k_lan_epi(int n, const double *zold, double nbeta, const double *dotv, double *y, double *part,
                          unsigned int *ctr, double *dot_out) {
  __shared__ double sh[kThreads / 32];
  double dsum = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double yv = y[r];
    if (zold) yv = __dadd_rn(yv, __dmul_rn(nbeta, zold[r]));
    y[r] = yv;
    if (dotv) dsum += dotv[r] * yv;
  }
  if (dot_out) {
    double b = block_sum(dsum, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = b;
    if (last_block(ctr)) {
      double tot = reduce_partials(part, gridDim.x, ctr, sh);
      if (threadIdx.x == 0) *dot_out = tot;
    }
  }
}


int g_rows_per_thread = 1;

template <class F, class M>
int launch_pdl(F fn, int grid, M view, const double *vk, const double *vkm1, double *out, double *y, double t,
               double ncc, double s, double mu0, const double *zold, double nbeta, const double *dotv, double *dout) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, fn, view, vk, vkm1, out, y, t, ncc, s, mu0, zold, nbeta, dotv, partials(),
                                     counters() + CTR_CHEB, dout);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "filter kernel launch failed: %s", cudaGetErrorString(e));
  EVSLCU_LAUNCH_CHECK("k_cheb");
  return 0;
}

int g_row_unroll = 1;
int g_cheb_max_grid = 0;  // > 0: at most this many blocks per degree step (grid-stride rows)
int g_call_grid = 0;      // the limit of the launches being issued (forced or the matrix's tuned one)

// Unroll width for rows of at most wmax stored entries (0: loop form).
inline int unroll_width(int wmax) {
  if (!g_row_unroll || wmax <= 0) return 0;
  if (wmax <= 8) return 8;
  if (wmax <= 16) return 16;
  return 0;
}

template <class M>
using ChebFn = void (*)(M, const double *, const double *, double *, double *, double, double, double, double,
                        const double *, double, const double *, double *, unsigned int *, double *);

template <class M, int W>
ChebFn<M> cheb_fn(bool first, bool epi) {
  if (first && epi) return k_cheb<M, true, true, W>;
  if (first) return k_cheb<M, true, false, W>;
  if (epi) return k_cheb<M, false, true, W>;
  return k_cheb<M, false, false, W>;
}

// One degree step, one thread per row.
template <class M>
int launch_cheb_rows(const M &view, int n, int wmax, bool first, bool epi, const double *vk, const double *vkm1,
                     double *out, double *y, double t, double ncc, double s, double mu0, const evslcu_cheb_epi *ep) {
  const double *zold = (epi && ep) ? ep->zold : nullptr;
  const double nbeta = (epi && ep) ? ep->nbeta : 0.0;
  const double *dotv = (epi && ep) ? ep->dotv : nullptr;
  double *dout = (epi && ep) ? ep->dot_out : nullptr;
  const int grid = g_call_grid > 0 ? std::min(grid_for(n), g_call_grid) : grid_for(n);
  ChebFn<M> fn;
  switch (unroll_width(wmax)) {
    case 8: fn = cheb_fn<M, 8>(first, epi); break;
    case 16: fn = cheb_fn<M, 16>(first, epi); break;
    default: fn = cheb_fn<M, 0>(first, epi); break;
  }
  return launch_pdl(fn, grid, view, vk, vkm1, out, y, t, ncc, s, mu0, zold, nbeta, dotv, dout);
}

template <class M>
int launch_cheb_step(const M &view, int n, int wmax, bool first, bool epi, const double *vk, const double *vkm1,
                     double *out, double *y, double t, double ncc, double s, double mu0, const evslcu_cheb_epi *ep) {
  return launch_cheb_rows(view, n, wmax, first, epi, vk, vkm1, out, y, t, ncc, s, mu0, ep);
}

template <class VT, class IT>
int launch_cheb_step(const SellT<VT, IT> &view, int n, int wmax, bool first, bool epi, const double *vk,
                     const double *vkm1, double *out, double *y, double t, double ncc, double s, double mu0,
                     const evslcu_cheb_epi *ep) {
  if (g_rows_per_thread != 2)
    return launch_cheb_rows(view, n, wmax, first, epi, vk, vkm1, out, y, t, ncc, s, mu0, ep);
  const double *zold = (epi && ep) ? ep->zold : nullptr;
  const double nbeta = (epi && ep) ? ep->nbeta : 0.0;
  const double *dotv = (epi && ep) ? ep->dotv : nullptr;
  double *dout = (epi && ep) ? ep->dot_out : nullptr;
  const int grid = grid_for(((long long)n + 1) / 2);
  if (first && epi)
    return launch_pdl(k_cheb2<VT, IT, true, true>, grid, view, vk, vkm1, out, y, t, ncc, s, mu0, zold, nbeta, dotv,
                      dout);
  if (first)
    return launch_pdl(k_cheb2<VT, IT, true, false>, grid, view, vk, vkm1, out, y, t, ncc, s, mu0, zold, nbeta, dotv,
                      dout);
  if (epi)
    return launch_pdl(k_cheb2<VT, IT, false, true>, grid, view, vk, vkm1, out, y, t, ncc, s, mu0, zold, nbeta, dotv,
                      dout);
  return launch_pdl(k_cheb2<VT, IT, false, false>, grid, view, vk, vkm1, out, y, t, ncc, s, mu0, zold, nbeta, dotv,
                    dout);
}

// ---------------------------------------------------------------------------
// KPM block moments: warp per row, lane = probe; vectors interleaved [n][B].
// ---------------------------------------------------------------------------
constexpr int kKpmRows = 4;  // rows a warp works on at once (independent chains)

inline int kpm_grid(int n) {
  return (int)std::min<long long>(((long long)n + 8 * kKpmRows - 1) / (8 * kKpmRows), 4096);
}

template <int G, bool FIRST>
__global__ void __launch_bounds__(kThreads)
    k_kpm(CsrView A, int B, const double *__restrict__ vk, const double *vkm1, double *out, double scal, double nctr,
          const double *__restrict__ v0, double *part, unsigned int *ctr, double *dots_row) {
  __shared__ double sh[kThreads / 32][G * 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps_total = gridDim.x * (kThreads / 32);
  double dsum[G];
#pragma unroll
  for (int g = 0; g < G; ++g) dsum[g] = 0.0;
  for (int r0 = (blockIdx.x * (kThreads / 32) + warp) * kKpmRows; r0 < A.n; r0 += nwarps_total * kKpmRows) {
    int b[kKpmRows], len[kKpmRows], maxlen = 0;
#pragma unroll
    for (int i = 0; i < kKpmRows; ++i) {
      const int r = r0 + i;
      b[i] = (r < A.n) ? A.ia[r] : 0;
      len[i] = (r < A.n) ? A.ia[r + 1] - b[i] : 0;
      maxlen = max(maxlen, len[i]);
    }
    double acc[kKpmRows][G];
#pragma unroll
    for (int i = 0; i < kKpmRows; ++i)
#pragma unroll
      for (int g = 0; g < G; ++g) acc[i][g] = 0.0;
    for (int j = 0; j < maxlen; ++j) {
#pragma unroll
      for (int i = 0; i < kKpmRows; ++i) {
        if (j < len[i]) {
          const double aj = __ldg(A.a + b[i] + j);
          const long long cj = (long long)__ldg(A.ja + b[i] + j) * B;
#pragma unroll
          for (int g = 0; g < G; ++g) {
            const int p = lane + 32 * g;
            if (p < B) acc[i][g] = __dadd_rn(acc[i][g], __dmul_rn(aj, __ldg(vk + cj + p)));
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kKpmRows; ++i) {
      const int r = r0 + i;
      if (r >= A.n) continue;
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int p = lane + 32 * g;
        if (p < B) {
          const long long idx = (long long)r * B + p;
          double w = __dmul_rn(scal, __dadd_rn(acc[i][g], __dmul_rn(nctr, vk[idx])));
          if (!FIRST) w = __dadd_rn(w, -vkm1[idx]);
          out[idx] = w;
          dsum[g] += w * v0[idx];
        }
      }
    }
  }
#pragma unroll
  for (int g = 0; g < G; ++g) sh[warp][lane + 32 * g] = dsum[g];
  __syncthreads();
  // block partials stored probe-major (part[p * gridDim.x + block]) so that
  // the last block's reduction reads them coalesced
  for (int p = threadIdx.x; p < B; p += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += sh[w][p];
    part[(long long)p * gridDim.x + blockIdx.x] = s;
  }
  if (last_block(ctr)) {
    // one warp per probe: lanes sum strided blocks, then a shuffle tree;
    // the order depends only on the grid (a function of n), not on B
    for (int p = warp; p < B; p += kThreads / 32) {
      double s = 0.0;
      for (int b2 = lane; b2 < (int)gridDim.x; b2 += 32) s += __ldcg(part + (long long)p * gridDim.x + b2);
      s = warp_sum(s);
      if (lane == 0) dots_row[p] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *ctr = 0u;
  }
}

// KPM degree step that yields two moments per matrix product (Chebyshev
// product identities T_2k = 2 T_k^2 - T_0 and T_2k+1 = 2 T_k+1 T_k - T_1):
// per probe, <w_k+1, w_k+1> and <w_k+1, w_k> (and <w_0, w_0> at the first
// step).  No pass over the probes per degree, and ceil(M/2) products give M
// moments.
//
// One launch handles probes p0 .. p0+nb-1 (nb <= 32) of the interleaved
// [n][B] block.  Each half-warp owns 4 consecutive rows per iteration (a warp
// 8), each lane 2 probes of them; a half-warp loads its rows' entries once
// (2 per lane, rows of at most 8 entries) and passes them round by shuffles,
// so a row's gathers for both probes are in flight together.  VEC: the two
// probes are read as one 16-byte access (B and p0 even).  Block sums go to
// part[(s * B + p) * gridDim.x + block] and k_kpm_reduce adds them up.  The
// rows a lane visits, and the order of every sum, depend on n and the grid
// only -- not on B, nb or VEC -- so probe shards reproduce the full block.
constexpr int kKpmHalfRows = 4;  // rows per half-warp and iteration

// PRE: the rows' own v_k and v_k-1 values are loaded before the gathers (so
// their DRAM latency overlaps the gathers') and the new vector is stored with
// 16-byte stores; same arithmetic, more registers (3 blocks per SM).
template <bool FIRST, bool VEC, bool PRE>
__global__ void __launch_bounds__(kThreads, PRE ? 3 : 4)
    k_kpm_dbl(CsrView A, int B, int p0, int nb, const double *__restrict__ vk, const double *vkm1, double *out,
              double scal, double nctr, double *part) {
  constexpr int NS = FIRST ? 3 : 2;
  __shared__ double sh[NS][kThreads / 32][2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int h = lane >> 4, hl = lane & 15;
  const int q = 2 * hl;  // first of this lane's two probes, relative to p0
  const bool onA = q < nb, onB = q + 1 < nb;
  const int pa = p0 + q;
  const int rows_per_iter = gridDim.x * (kThreads / 32) * 2 * kKpmHalfRows;
  double sum[NS][2];
#pragma unroll
  for (int s = 0; s < NS; ++s) sum[s][0] = sum[s][1] = 0.0;
  for (int base = (blockIdx.x * (kThreads / 32) + warp) * 2 * kKpmHalfRows; base < A.n; base += rows_per_iter) {
    const int r0 = base + h * kKpmHalfRows;  // this half-warp's first row
    int b[kKpmHalfRows], len[kKpmHalfRows], mymax = 0;
#pragma unroll
    for (int i = 0; i < kKpmHalfRows; ++i) {
      const int r = r0 + i;
      b[i] = (r < A.n) ? A.ia[r] : 0;
      len[i] = (r < A.n) ? A.ia[r + 1] - b[i] : 0;
      mymax = max(mymax, len[i]);
    }
    const int maxlen = __reduce_max_sync(0xffffffffu, mymax);
    double px[kKpmHalfRows][2], pm[kKpmHalfRows][2];
    if constexpr (PRE) {
#pragma unroll
      for (int i = 0; i < kKpmHalfRows; ++i) {
        const int r = r0 + i;
        px[i][0] = px[i][1] = pm[i][0] = pm[i][1] = 0.0;
        if (r < A.n) {
          const long long idx = (long long)r * B + pa;
          if (VEC && onB) {
            const double2 t = __ldg(reinterpret_cast<const double2 *>(vk + idx));
            px[i][0] = t.x;
            px[i][1] = t.y;
            if (!FIRST) {
              // v_k-1 is overwritten by this step's output: plain loads
              const double2 u = *reinterpret_cast<const double2 *>(vkm1 + idx);
              pm[i][0] = u.x;
              pm[i][1] = u.y;
            }
          } else {
            if (onA) {
              px[i][0] = vk[idx];
              if (!FIRST) pm[i][0] = vkm1[idx];
            }
            if (onB) {
              px[i][1] = vk[idx + 1];
              if (!FIRST) pm[i][1] = vkm1[idx + 1];
            }
          }
        }
      }
    }
    double acc[kKpmHalfRows][2];
#pragma unroll
    for (int i = 0; i < kKpmHalfRows; ++i) acc[i][0] = acc[i][1] = 0.0;
    if (maxlen <= 8) {
      // entries e = i * 8 + j of the half-warp's 4 rows: e < 16 in slot 0 of
      // half-lane e, e >= 16 in slot 1 of half-lane e - 16
      double ae[2];
      int ce[2];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int e = hl + 16 * t, i = e >> 3, j = e & 7;
        const int lr = (i == 0) ? len[0] : (i == 1) ? len[1] : (i == 2) ? len[2] : len[3];
        const int br = (i == 0) ? b[0] : (i == 1) ? b[1] : (i == 2) ? b[2] : b[3];
        ae[t] = 0.0;
        ce[t] = 0;
        if (j < lr) {
          ae[t] = __ldg(A.a + br + j);
          ce[t] = __ldg(A.ja + br + j);
        }
      }
#pragma unroll
      for (int i = 0; i < kKpmHalfRows; ++i) {
        double xa[8], xb[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int e = i * 8 + j;
          const int cj = __shfl_sync(0xffffffffu, ce[e >> 4], e & 15, 16);
          xa[j] = 0.0;
          xb[j] = 0.0;
          if (j < len[i]) {
            const double *src = vk + (long long)cj * B + pa;
            if (VEC && onB) {
              const double2 v2 = __ldg(reinterpret_cast<const double2 *>(src));
              xa[j] = v2.x;
              xb[j] = v2.y;
            } else {
              if (onA) xa[j] = __ldg(src);
              if (onB) xb[j] = __ldg(src + 1);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int e = i * 8 + j;
          const double av = __shfl_sync(0xffffffffu, ae[e >> 4], e & 15, 16);
          if (j < len[i]) {
            acc[i][0] = __dadd_rn(acc[i][0], __dmul_rn(av, xa[j]));
            acc[i][1] = __dadd_rn(acc[i][1], __dmul_rn(av, xb[j]));
          }
        }
      }
    } else {
      for (int j = 0; j < maxlen; ++j) {
#pragma unroll
        for (int i = 0; i < kKpmHalfRows; ++i) {
          if (j < len[i]) {
            const double aj = __ldg(A.a + b[i] + j);
            const double *src = vk + (long long)__ldg(A.ja + b[i] + j) * B + pa;
            if (onA) acc[i][0] = __dadd_rn(acc[i][0], __dmul_rn(aj, __ldg(src)));
            if (onB) acc[i][1] = __dadd_rn(acc[i][1], __dmul_rn(aj, __ldg(src + 1)));
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kKpmHalfRows; ++i) {
      const int r = r0 + i;
      if (r >= A.n) continue;
      double wv[2] = {0.0, 0.0};
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (!(c == 0 ? onA : onB)) continue;
        const long long idx = (long long)r * B + pa + c;
        const double x = PRE ? px[i][c] : vk[idx];
        double w = __dmul_rn(scal, __dadd_rn(acc[i][c], __dmul_rn(nctr, x)));
        if (!FIRST) w = __dadd_rn(w, -(PRE ? pm[i][c] : vkm1[idx]));
        if (!PRE || !(VEC && onB)) out[idx] = w;
        wv[c] = w;
        sum[0][c] += w * w;
        sum[1][c] += w * x;
        if (FIRST) sum[NS - 1][c] += x * x;
      }
      if (PRE && VEC && onB) *reinterpret_cast<double2 *>(out + (long long)r * B + pa) = make_double2(wv[0], wv[1]);
    }
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    sh[s][warp][h][q] = sum[s][0];
    sh[s][warp][h][q + 1] = sum[s][1];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < NS * 32; t += blockDim.x) {
    const int s = t / 32, l = t % 32;
    if (l >= nb) continue;
    double v = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) v += sh[s][w][0][l] + sh[s][w][1][l];
    part[((long long)s * B + p0 + l) * gridDim.x + blockIdx.x] = v;
  }
}

// The same KPM block step on the column-split copy of a large general
// matrix, for 8 probes p0 .. p0+nb-1 at a time.  With random columns the
// gathers of k_kpm_dbl land on random rows of the whole probe block, most of
// which miss L2; here the columns are cut into ranges whose rows of the
// 8 probes (64 bytes each) fit in L2, one launch per range, each row's
// running sum carried from range to range in xpart ([n][8], streaming
// loads and stores).  The last range forms w_k+1 and the per-probe sums
// <w_k+1, w_k+1>, <w_k+1, w_k> (and <w_0, w_0> first) into part, laid out as
// k_kpm_dbl's so that k_kpm_reduce adds them up.  Four threads per row, two
// probes each (one 16-byte access when VEC); a probe's sums run over the
// rows in an order fixed by n and the grid, not by the other probes.
constexpr int kKpmChunk = 8;

template <bool PFIRST, bool PLAST, bool FIRST, bool VEC>
__global__ void __launch_bounds__(kThreads)
    k_kpm_xs(XsRange<double> A, int B, int p0, int nb, const double *__restrict__ vk, const double *vkm1,
             double *out, double scal, double nctr, double *xpart, double *part) {
  constexpr int TPR = kKpmChunk / 2, U = 4;
  constexpr int NS = FIRST ? 3 : 2;
  __shared__ double sh[NS][kThreads / 32][kKpmChunk];
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int q = lane & (TPR - 1);
  const bool onA = 2 * q < nb, onB = 2 * q + 1 < nb;
  double sum[NS][2];
#pragma unroll
  for (int t = 0; t < NS; ++t) sum[t][0] = sum[t][1] = 0.0;
  const int npad = (A.n + 31) & ~31;
  const long long total = (long long)npad * TPR;
  const long long stride = (long long)gridDim.x * blockDim.x;
  auto ld2 = [&](const double *src, double &a, double &b, bool cs) {
    if (VEC && onB) {
      const double2 v = cs ? __ldcs(reinterpret_cast<const double2 *>(src)) : __ldg(reinterpret_cast<const double2 *>(src));
      a = v.x;
      b = v.y;
    } else {
      a = onA ? (cs ? __ldcs(src) : __ldg(src)) : 0.0;
      b = onB ? (cs ? __ldcs(src + 1) : __ldg(src + 1)) : 0.0;
    }
  };
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
    const int sl = (int)(g / TPR);
    const bool live = sl < A.n;
    const int r = live ? __ldg(A.perm + sl) : 0;
    const long long base = (long long)r * B + p0 + 2 * q;
    double* const xp = xpart + (long long)r * kKpmChunk + 2 * q;
    double acc0 = 0.0, acc1 = 0.0;
    if (!PFIRST && live) {
      const double2 v = __ldcs(reinterpret_cast<const double2 *>(xp));
      acc0 = v.x;
      acc1 = v.y;
    }
    double x0 = 0.0, x1 = 0.0, m0 = 0.0, m1 = 0.0;
    if (PLAST && live) {
      ld2(vk + base, x0, x1, false);
      if (!FIRST) ld2(vkm1 + base, m0, m1, true);
    }
    const int ch = sl >> 5;
    long long p = __ldg(A.cptr + ch) + (sl & 31);
    const int w = __ldg(A.cw + ch);
    double v[U];
    int col[U];
    auto fetch = [&](int j0, long long pp, double(&vv)[U], int(&cc)[U]) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (live && j0 + u < w) {
          vv[u] = __ldcs(A.val + pp + 32 * u);
          cc[u] = __ldcs(A.col + pp + 32 * u);
        } else {
          vv[u] = 0.0;
          cc[u] = -1;
        }
      }
    };
    fetch(0, p, v, col);
    for (int j = 0; j < w; j += U, p += 32 * U) {
      double g0[U], g1[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        g0[u] = g1[u] = 0.0;
        if (col[u] >= 0) ld2(vk + (long long)col[u] * B + p0 + 2 * q, g0[u], g1[u], false);
      }
      double vn[U];
      int cn[U];
      fetch(j + U, p + 32 * U, vn, cn);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (col[u] >= 0) {
          acc0 = __dadd_rn(acc0, __dmul_rn(v[u], g0[u]));
          acc1 = __dadd_rn(acc1, __dmul_rn(v[u], g1[u]));
        }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        v[u] = vn[u];
        col[u] = cn[u];
      }
    }
    if (!live) continue;
    if (!PLAST) {
      __stcs(reinterpret_cast<double2 *>(xp), make_double2(acc0, acc1));
      continue;
    }
    double w0 = __dmul_rn(scal, __dadd_rn(acc0, __dmul_rn(nctr, x0)));
    double w1 = __dmul_rn(scal, __dadd_rn(acc1, __dmul_rn(nctr, x1)));
    if (!FIRST) {
      w0 = __dadd_rn(w0, -m0);
      w1 = __dadd_rn(w1, -m1);
    }
    if (onA) out[base] = w0;
    if (onB) out[base + 1] = w1;
    sum[0][0] += w0 * w0;
    sum[0][1] += w1 * w1;
    sum[1][0] += w0 * x0;
    sum[1][1] += w1 * x1;
    if (FIRST) {
      sum[NS - 1][0] += x0 * x0;
      sum[NS - 1][1] += x1 * x1;
    }
  }
  if constexpr (PLAST) {
    // lanes q, q+4, ..., q+28 hold the same probes: fixed butterfly over them
#pragma unroll
    for (int t = 0; t < NS; ++t)
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int o = TPR; o < 32; o <<= 1) sum[t][c] += __shfl_xor_sync(0xffffffffu, sum[t][c], o);
    if (lane < TPR) {
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        sh[t][warp][2 * q] = sum[t][0];
        sh[t][warp][2 * q + 1] = sum[t][1];
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NS * kKpmChunk; t += blockDim.x) {
      const int s = t / kKpmChunk, l = t % kKpmChunk;
      if (l >= nb) continue;
      double acc = 0.0;
      for (int wi = 0; wi < kThreads / 32; ++wi) acc += sh[s][wi][l];
      part[((long long)s * B + p0 + l) * gridDim.x + blockIdx.x] = acc;
    }
  }
}

// raw[q] = sum over the nb block partials of sum q (block q; fixed order).
__global__ void __launch_bounds__(kThreads) k_kpm_reduce(int nb, const double *__restrict__ part, double *raw) {
  __shared__ double sh[kThreads / 32];
  const double *pq = part + (long long)blockIdx.x * nb;
  double t = 0.0;
  for (int i = threadIdx.x; i < nb; i += kThreads) t += pq[i];
  t = block_sum(t, sh);
  if (threadIdx.x == 0) raw[blockIdx.x] = t;
}

// Column sums of squares of a column-major n x B block: part[blk*B + p].
__global__ void k_colsq_partial(int n, int B, const double *X, double *part, unsigned int *ctr, double *nrm) {
  __shared__ double sh[kThreads / 32];
  const int p = blockIdx.y;
  double s = 0.0;
  const double *x = X + (long long)p * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += x[i] * x[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[(long long)p * gridDim.x + blockIdx.x] = s;
  if (last_block(ctr)) {
    for (int q = threadIdx.x; q < B; q += blockDim.x) {
      double t = 0.0;
      for (int b = 0; b < (int)gridDim.x; ++b) t += __ldcg(part + (long long)q * gridDim.x + b);
      nrm[q] = sqrt(t);
    }
    __syncthreads();
    if (threadIdx.x == 0) *ctr = 0u;
  }
}

// v0[r*B + p] = (1/nrm_p) * probes[p*n + r]   (t = 1/||v||; dscal(t))
__global__ void k_interleave_scaled(int n, int B, const double *probes, const double *nrm, double *v0) {
  const long long total = (long long)n * B;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / B), p = (int)(i % B);
    const double t = 1.0 / nrm[p];
    v0[i] = __dmul_rn(t, probes[(long long)p * n + r]);
  }
}

// ---------------------------------------------------------------------------
// Random vectors
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform_pm1(uint64_t seed, uint64_t draw, uint64_t i) {
  const uint64_t key = seed * 0x9E3779B97F4A7C15ULL + (draw << 32) + i;
  const double u = (double)(mix64(key) >> 11) * (1.0 / 9007199254740992.0);
  return 2.0 * u - 1.0;
}

__global__ void k_rand_pm1(int n, int count, uint64_t seed, uint64_t draw, double *v) {
  const long long total = (long long)n * count;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long d = i / n, r = i % n;
    v[i] = uniform_pm1(seed, draw + (uint64_t)d, (uint64_t)r);
  }
}

__global__ void k_randn(int n, uint64_t seed, uint64_t draw, double *v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double u1 = 0.5 * (uniform_pm1(seed, draw, 2 * (uint64_t)i) + 1.0);
    double u2 = 0.5 * (uniform_pm1(seed, draw, 2 * (uint64_t)i + 1) + 1.0);
    if (u1 < 1e-300) u1 = 1e-300;
    v[i] = sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
  }
}



// Sequential accumulation of the KPM moments and the eigenvalue count from
// the raw dot products, in the same order and with the same rounded
// operations as the host accumulation of kpmdos (probe-major, then degree).
__global__ void k_kpm_accumulate(int Mdeg, int nvec, const double *jac, const double *sdiff, const double *dots,
                                 double bdiff, double t, double nd, double *mu, double *ecnt) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int k = 0; k <= Mdeg; ++k) mu[k] = 0.0;
  double tcnt = 0.0;
  for (int m = 0; m < nvec; ++m) {
    mu[0] = __dadd_rn(mu[0], jac[0]);
    tcnt = __dsub_rn(tcnt, __dmul_rn(jac[0], bdiff));
    for (int k = 0; k < Mdeg; ++k) {
      const int k1 = k + 1;
      const double tk = __dmul_rn(__dmul_rn(2.0, jac[k1]), dots[(size_t)k * nvec + m]);
      mu[k1] = __dadd_rn(mu[k1], tk);
      tcnt = __dsub_rn(tcnt, __ddiv_rn(__dmul_rn(tk, sdiff[k]), (double)k1));
    }
  }
  for (int k = 0; k <= Mdeg; ++k) mu[k] = __dmul_rn(t, mu[k]);
  *ecnt = __dmul_rn(tcnt, __dmul_rn(t, nd));
}

// Scratch of the allocation-free KPM entry point: a fixed 32 MiB array in the
// device image of the library.  Every GPU that loads the library holds it
// until the process exits.  All calls share it.
constexpr size_t kNoAllocDoubles = (size_t)1 << 22;
static __device__ __align__(256) double g_kpm_noalloc_scratch[kNoAllocDoubles];

// Device address of the scratch array on the library's device, looked up
// once (again only if a later EVSLStart picks another device).
double *g_noalloc_ptr = nullptr;
int g_noalloc_dev = -1;

}  // namespace

int evslcu::launch_scale_copy(int n, double a, const double *x, double *y) {
  k_scale_copy<<<grid_for(n), kThreads, 0, stream()>>>(n, a, x, y);
  EVSLCU_LAUNCH_CHECK("k_scale_copy");
  return 0;
}

int evslcu::launch_lan_epi(int n, const evslcu_cheb_epi *epi, double *y) {
  k_lan_epi<<<grid_for(n), kThreads, 0, stream()>>>(n, epi->zold, epi->nbeta, epi->dotv, y, partials(),
                                                    counters() + CTR_CHEB, epi->dot_out);
  EVSLCU_LAUNCH_CHECK("k_lan_epi");
  return 0;
}

// User matvec (SetAMatvec): the reference's three-vector rotation
// (SRC/chebpoly.c:532-589) with the callback computing vkp1 = A vk.  The
// callback must enqueue on the legacy default stream (which orders with the
// library stream) or finish its work before returning.
int evslcu::chebav_user_matvec(const evslcu_op *op, const double *mu, int deg, double cc, double dd,
                               const double *v, double *y, double *work, const evslcu_cheb_epi *epi) {
  if (!op->func) return fail(EVSLCU_ERR_STATE, "no matrix or matvec registered");
  const int n = op->n;
  const double t1 = 1.0 / dd, t2 = 2.0 / dd;
  double *vk = work, *vkp1 = work + n, *vkm1 = work + 2 * (size_t)n;
  if (evslcu_d2d(vk, v, sizeof(double) * n)) return EVSLCU_ERR_CUDA;
  int rc = launch_scale_copy(n, mu[0], v, y);
  if (rc) return rc;
  for (int k = 1; k <= deg; ++k) {
    const double t = (k == 1) ? t1 : t2;
    cudaError_t e = cudaStreamSynchronize(stream());
    if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "sync before matvec: %s", cudaGetErrorString(e));
    op->func(vk, vkp1, op->data);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "user matvec failed: %s", cudaGetErrorString(e));
    k_cheb_update<<<grid_for(n), kThreads, 0, stream()>>>(n, k, t, mu[k], -cc, vkp1, vk, vkm1, y);
    EVSLCU_LAUNCH_CHECK("k_cheb_update");
    double *tmp = vkm1;
    vkm1 = vk;
    vk = vkp1;
    vkp1 = tmp;
  }
  if (epi) return launch_lan_epi(n, epi, y);
  return 0;
}

// ---------------------------------------------------------------------------
// Per-matrix choice of the single-vector filter kernel.  The variants give
// identical results (same rounded operations in the same order) and differ
// only in where the row entries come from and how the row loop is issued:
//   0  SELL-32, loop form            1  SELL-32, unrolled
//   2  pattern table (global), unrolled   3  pattern table (global), loop form
//   4  pattern table (constant), loop form  5  pattern table (constant), unrolled
// Which is fastest depends on the size of the matrix (latency-bound small
// operators favour the unrolled forms, L2-bound large ones the constant
// table), so the first filter call on a matrix times every allowed variant on
// scratch vectors and keeps the fastest.
// ---------------------------------------------------------------------------
namespace {

constexpr int kChebVariants = 8;
int g_cheb_force = -1;

bool cheb_variant_ok(const evslcu_mat *A, int v) {
  if (A->kernel != 0) return false;
  const bool pat = evslcu_mat_uses_patterns(A) != 0;
  const bool pconst = pat && A->pat_chdr >= 0 && g_pattern_const;
  switch (v) {
    case 0: return true;
    case 1: return unroll_width(A->maxw) > 0;
    case 2: return pat && unroll_width(A->pat_maxlen) > 0;
    case 3: return pat;
    case 4: return pconst;
    case 5: return pconst && unroll_width(A->pat_maxlen) > 0;
    case 6: return pconst && A->pat_desc;
    case 7: return A->pn64 != nullptr;
    default: return false;
  }
}

int launch_variant(const evslcu_mat *A, int v, bool first, bool epi, const double *vk, const double *vkm1,
                   double *out, double *y, double t, double ncc, double s, double mu0, const evslcu_cheb_epi *ep,
                   int grid_limit) {
  const int n = A->n;
  g_call_grid = g_cheb_max_grid > 0 ? g_cheb_max_grid : grid_limit;
  switch (v) {
    case 0:
    case 1: {
      const int wmax = (v == 1) ? A->maxw : 0;
      return with_view(A, [&](auto view) {
        return launch_cheb_step(view, n, wmax, first, epi, vk, vkm1, out, y, t, ncc, s, mu0, ep);
      });
    }
    case 2:
    case 3: {
      const int wmax = (v == 2) ? A->pat_maxlen : 0;
      if (A->pat_f32)
        return launch_cheb_step(pat_pview(A), n, wmax, first, epi, vk, vkm1, out, y, t, ncc, s, mu0, ep);
      return launch_cheb_step(pat_view(A), n, wmax, first, epi, vk, vkm1, out, y, t, ncc, s, mu0, ep);
    }
    case 7: {
      const bool e = epi && ep;
      return panel_cheb_step(A, first, e, vk, vkm1, out, y, t, ncc, s, mu0, e ? ep->zold : nullptr,
                             e ? ep->nbeta : 0.0, e ? ep->dotv : nullptr, e ? ep->dot_out : nullptr);
    }
    case 6:
      if (A->pat_f32)
        return launch_cheb_step(PatCDView<true>{n, A->pat_desc}, n, 0, first, epi, vk, vkm1, out, y, t, ncc, s, mu0,
                                ep);
      return launch_cheb_step(PatCDView<false>{n, A->pat_desc}, n, 0, first, epi, vk, vkm1, out, y, t, ncc, s, mu0,
                              ep);
    default: {
      const int wmax = (v == 5) ? A->pat_maxlen : 0;
      if (A->pat_f32)
        return launch_cheb_step(PatCPView{n, A->pat_id, A->pat_chdr}, n, wmax, first, epi, vk, vkm1, out, y, t, ncc,
                                s, mu0, ep);
      return launch_cheb_step(PatCView{n, A->pat_id, A->pat_chdr}, n, wmax, first, epi, vk, vkm1, out, y, t, ncc, s,
                              mu0, ep);
    }
  }
}

// Microseconds per degree step of variant v with grid limit g (12 timed
// steps after 3 untimed ones) on the zero-filled scratch vectors; 0 on error.
float time_variant(const evslcu_mat *A, int v, int g, double *scr, cudaEvent_t e0, cudaEvent_t e1, int *rc) {
  constexpr int kWarm = 3, kTimed = 12;
  const size_t n = (size_t)A->n;
  for (int i = 0; i < kWarm + kTimed && !*rc; ++i) {
    if (i == kWarm) cudaEventRecord(e0, stream());
    *rc = launch_variant(A, v, false, false, scr, scr + n, scr + n, scr + 2 * n, 2.0, 0.0, 1.0, 1.0, nullptr, g);
  }
  cudaEventRecord(e1, stream());
  float ms = 0.0f;
  if (*rc || cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) return 0.0f;
  return 1e3f * ms / kTimed;
}

// Times every allowed variant on zero-filled scratch vectors and keeps the
// fastest in A->cheb_variant, then its best grid limit in A->cheb_grid.
int tune_cheb(evslcu_mat *A) {
  static const int pref[kChebVariants] = {4, 6, 2, 3, 1, 0, 5, 7};
  int fallback = 0;
  for (int v : pref)
    if (cheb_variant_ok(A, v)) {
      fallback = v;
      break;
    }
  for (int v = 0; v < kChebVariants; ++v) A->cheb_us[v] = 0.0f;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream(), &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return fallback;
  const int n = A->n;
  // large general matrices also get the column-panel layout, timed with the rest
  if (panel_candidate(A) && !A->pn64 && panel_build(A, 0)) cudaGetLastError();  // without it the SELL kernels serve
  double *scr = (double *)evslcu_malloc(sizeof(double) * 3 * (size_t)n);
  if (!scr) return fallback;
  int best = fallback;
  float best_us = 0.0f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = evslcu_memset(scr, 0, sizeof(double) * 3 * (size_t)n);
  if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) rc = EVSLCU_ERR_CUDA;
  for (int v = 0; v < kChebVariants && !rc; ++v) {
    if (!cheb_variant_ok(A, v)) continue;
    const float us = time_variant(A, v, 0, scr, e0, e1, &rc);
    if (us > 0.0f) {
      A->cheb_us[v] = us;
      if (best_us == 0.0f || us < best_us) {
        best_us = us;
        best = v;
      }
    }
  }
  // then the grid limit for the chosen variant: one row per thread, or
  // 16 / 8 blocks per SM going round a grid-stride loop
  A->cheb_grid = 0;
  for (int g : {16 * sm_count(), 8 * sm_count()}) {
    if (rc || best_us == 0.0f) break;
    const float us = time_variant(A, best, g, scr, e0, e1, &rc);
    if (us > 0.0f && us < best_us) {
      best_us = us;
      A->cheb_grid = g;
    }
  }
  A->cheb_best_us = best_us;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  evslcu_free(scr);
  if (rc) return rc;  // an error code (<= EVSLCU_ERR_CUDA)
  return best;
}

// The variant for this call: forced, tuned earlier, or tuned now.  -1: the
// CSR kernel is selected; -2: the forced variant is not available; an error
// code (<= EVSLCU_ERR_CUDA) if timing failed.
int cheb_variant(const evslcu_mat *A_) {
  evslcu_mat *A = const_cast<evslcu_mat *>(A_);
  if (A->kernel != 0) return -1;
  if (g_cheb_force == 7 && panel_candidate(A) && !A->pn64) {
    const int prc = panel_build(A, 0);
    if (prc) return prc;
  }
  if (g_cheb_force >= 0) return cheb_variant_ok(A, g_cheb_force) ? g_cheb_force : -2;
  if (A->cheb_variant >= 0 && cheb_variant_ok(A, A->cheb_variant)) return A->cheb_variant;
  const int v = tune_cheb(A);
  if (v < 0) return v;
  A->cheb_variant = v;
  return v;
}

}  // namespace

// Per-degree filter: one fused kernel launch per degree (matrix path).
int evslcu::chebav_per_degree(const evslcu_mat *A, const double *mu, int deg, double cc, double dd, const double *v,
                      double *y, double *work, const evslcu_cheb_epi *epi) {
  const int n = A->n;
  const double t1 = 1.0 / dd, t2 = 2.0 / dd, ncc = -cc;
  double *W[2] = {work, work + n};
  const int var = cheb_variant(A);
  if (var == -2) return fail(EVSLCU_ERR_ARG, "filter kernel variant %d is not available for this matrix", g_cheb_force);
  if (var <= EVSLCU_ERR_CUDA) return var;
  for (int k = 1; k <= deg; ++k) {
    const double t = (k == 1) ? t1 : t2;
    const double *vk = (k == 1) ? v : W[(k - 2) % 2];
    const double *vkm1 = (k == 1) ? nullptr : ((k == 2) ? v : W[(k - 1) % 2]);
    double *out = W[(k - 1) % 2];
    const bool last = (k == deg);
    if (var >= 0) {
      const int rc =
          launch_variant(A, var, k == 1, last && epi, vk, vkm1, out, y, t, ncc, mu[k], mu[0], epi, A->cheb_grid);
      if (rc) return rc;
      continue;
    }
    g_call_grid = g_cheb_max_grid;
    int rc = with_view(A, [&](auto view) {
      return launch_cheb_step(view, n, A->maxw, k == 1, last && epi, vk, vkm1, out, y, t, ncc, mu[k], mu[0], epi);
    });
    if (rc) return rc;
  }
  return 0;
}



extern "C" {

static int g_compress = 1;
static int g_patterns = 1;

int evslcu_set_compression(int on) {
  g_compress = on ? 1 : 0;
  return 0;
}

int evslcu_set_row_patterns(int on) {
  g_patterns = on ? 1 : 0;
  return 0;
}

int evslcu_set_pattern_const(int on) {
  g_pattern_const = on ? 1 : 0;
  return 0;
}

int evslcu_set_cheb_variant(int v) {
  if (v < -1 || v >= kChebVariants) return fail(EVSLCU_ERR_ARG, "filter kernel variant must be -1..%d", kChebVariants - 1);
  g_cheb_force = v;
  return 0;
}

int evslcu_mat_cheb_grid(const evslcu_mat *A) { return A ? A->cheb_grid : 0; }

double evslcu_chebav_step_cost(evslcu_mat *A) {
  if (!A || A->kernel != 0) return -1.0;
  const int v = cheb_variant(A);  // tunes on first use
  if (v < 0) return -1.0;
  return A->cheb_best_us > 0.0f ? (double)A->cheb_best_us : (double)A->cheb_us[v];
}

int evslcu_mat_cheb_variant(const evslcu_mat *A, float *us) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  if (us)
    for (int v = 0; v < kChebVariants; ++v) us[v] = A->cheb_us[v];
  return A->cheb_variant;
}

int evslcu_set_cheb_max_grid(int blocks) {
  if (blocks < 0) return fail(EVSLCU_ERR_ARG, "grid limit must be >= 0");
  g_cheb_max_grid = blocks;
  return 0;
}

int evslcu_set_row_unroll(int on) {
  g_row_unroll = on ? 1 : 0;
  return 0;
}

int evslcu_mat_set_patterns(evslcu_mat *A, int on) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  A->use_pat = (on && A->pat_id) ? 1 : 0;
  return 0;
}

int evslcu_mat_pattern_count(const evslcu_mat *A) { return (A && A->pat_id) ? A->npat : 0; }
int evslcu_mat_uses_patterns(const evslcu_mat *A) { return (A && A->pat_id && A->use_pat && A->kernel == 0) ? 1 : 0; }

int evslcu_mat_storage(const evslcu_mat *A, int *vfmt, int *ifmt) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  if (vfmt) *vfmt = A->vfmt;
  if (ifmt) *ifmt = A->ifmt;
  return 0;
}

evslcu_mat *evslcu_mat_create(int n, int nnz, const int *ia, const int *ja, const double *a, int on_device) {
  if (!evslcu_initialized()) {
    fail(EVSLCU_ERR_STATE, "library not started (EVSLStart)");
    return nullptr;
  }
  if (n <= 0 || nnz < 0 || !ia || (nnz > 0 && (!ja || !a))) {
    fail(EVSLCU_ERR_ARG, "invalid CSR matrix (n=%d nnz=%d)", n, nnz);
    return nullptr;
  }
  // The row pointer's ends are checked here; monotonicity, column range and
  // the compression checks run on the device (build_sell_device).
  int ends[2] = {0, 0};
  if (on_device) {
    if (evslcu_d2h(&ends[0], ia, sizeof(int)) || evslcu_d2h(&ends[1], ia + n, sizeof(int))) return nullptr;
    nnz = ends[1];
  } else {
    ends[0] = ia[0];
    ends[1] = ia[n];
  }
  if (ends[0] != 0 || ends[1] != nnz || nnz < 0) {
    fail(EVSLCU_ERR_ARG, "CSR row pointer must start at 0 and end at nnz (%d vs %d)", ends[1], nnz);
    return nullptr;
  }
  if (nnz > 0 && (!ja || !a)) {
    fail(EVSLCU_ERR_ARG, "invalid CSR matrix (nnz=%d without column/value arrays)", nnz);
    return nullptr;
  }
  evslcu_mat *M = new evslcu_mat;
  M->n = n;
  M->nnz = nnz;
  if (on_device) {
    M->ia = ia;
    M->ja = ja;
    M->a = a;
    M->own_csr = false;
  } else {
    int *dia = (int *)evslcu_malloc(sizeof(int) * (n + 1));
    int *dja = (int *)evslcu_malloc(sizeof(int) * (size_t)std::max(nnz, 1));
    double *da = (double *)evslcu_malloc(sizeof(double) * (size_t)std::max(nnz, 1));
    M->ia = dia;
    M->ja = dja;
    M->a = da;
    M->own_csr = true;
    if (!dia || !dja || !da || evslcu_h2d(dia, ia, sizeof(int) * (n + 1)) ||
        (nnz > 0 && (evslcu_h2d(dja, ja, sizeof(int) * (size_t)nnz) ||
                     evslcu_h2d(da, a, sizeof(double) * (size_t)nnz)))) {
      evslcu_mat_destroy(M);
      return nullptr;
    }
  }
  if (build_sell_device(M, g_compress != 0) || evslcu_sync() || (g_patterns && build_patterns_device(M)) ||
      pat_const_claim(M)) {
    evslcu_mat_destroy(M);
    return nullptr;
  }
  M->kernel = 0;
  M->use_pat = M->pat_id ? 1 : 0;
  return M;
}

void evslcu_mat_destroy(evslcu_mat *M) {
  if (!M) return;
  if (M->own_csr) {
    evslcu_free((void *)M->ia);
    evslcu_free((void *)M->ja);
    evslcu_free((void *)M->a);
  }
  evslcu_free(M->cptr);
  evslcu_free(M->cw);
  evslcu_free(M->perm);
  panel_free(M);
  xsplit_free(M);
  evslcu_mat_l2_persist(M, 0);
  evslcu_free(M->sell_block);
  evslcu_free(M->wave_ctl);
  evslcu_free(M->wave_mu);
  evslcu_free(M->sval32);
  pat_const_release(M);
  evslcu_free(M->pat_id);
  evslcu_free(M->pat_table);
  delete M;
}

int evslcu_mat_n(const evslcu_mat *A) { return A ? A->n : 0; }
long long evslcu_mat_nnz(const evslcu_mat *A) { return A ? A->nnz : 0; }
long long evslcu_mat_padded_nnz(const evslcu_mat *A) { return A ? A->padded : 0; }

int evslcu_mat_set_kernel(evslcu_mat *A, int which) {
  if (!A || which < 0 || which > 1) return fail(EVSLCU_ERR_ARG, "invalid kernel choice %d", which);
  A->kernel = which;
  return 0;
}

int evslcu_mat_get_kernel(const evslcu_mat *A) { return A ? A->kernel : -1; }

int evslcu_spmv(const evslcu_mat *A, const double *x, double *y) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  const int grid = grid_for(A->n);
  if (evslcu_mat_uses_patterns(A)) {
    if (A->pat_chdr >= 0 && g_pattern_const && A->pat_f32)
      k_spmv<PatCPView><<<grid, kThreads, 0, stream()>>>(PatCPView{A->n, A->pat_id, A->pat_chdr}, x, y);
    else if (A->pat_chdr >= 0 && g_pattern_const)
      k_spmv<PatCView><<<grid, kThreads, 0, stream()>>>(PatCView{A->n, A->pat_id, A->pat_chdr}, x, y);
    else if (A->pat_f32)
      k_spmv<PatPView><<<grid, kThreads, 0, stream()>>>(pat_pview(A), x, y);
    else
      k_spmv<PatView><<<grid, kThreads, 0, stream()>>>(pat_view(A), x, y);
    EVSLCU_LAUNCH_CHECK("k_spmv");
    return 0;
  }
  return with_view(A, [&](auto view) {
    k_spmv<decltype(view)><<<grid, kThreads, 0, stream()>>>(view, x, y);
    EVSLCU_LAUNCH_CHECK("k_spmv");
    return 0;
  });
}


int evslcu_spmv_cols(const evslcu_mat *A, const double *X, double *Y, int m) {
  if (!A) return fail(EVSLCU_ERR_ARG, "null matrix");
  if (m <= 0) return 0;
  const long long ld = A->n;
  for (int c0 = 0; c0 < m; c0 += 65535) {  // grid.y limit
    const int mc = std::min(65535, m - c0);
    // enough blocks in all to fill the GPU a few times; the row products do
    // not depend on the grid
    const int gx = std::max(1, std::min(grid_for(A->n), (16 * sm_count() + mc - 1) / mc));
    const dim3 g(gx, mc);
    const double *Xc = X + (size_t)c0 * ld;
    double *Yc = Y + (size_t)c0 * ld;
    if (evslcu_mat_uses_patterns(A)) {
      if (A->pat_chdr >= 0 && g_pattern_const && A->pat_f32)
        k_spmv_cols<PatCPView><<<g, kThreads, 0, stream()>>>(PatCPView{A->n, A->pat_id, A->pat_chdr}, Xc, Yc, ld);
      else if (A->pat_chdr >= 0 && g_pattern_const)
        k_spmv_cols<PatCView><<<g, kThreads, 0, stream()>>>(PatCView{A->n, A->pat_id, A->pat_chdr}, Xc, Yc, ld);
      else if (A->pat_f32)
        k_spmv_cols<PatPView><<<g, kThreads, 0, stream()>>>(pat_pview(A), Xc, Yc, ld);
      else
        k_spmv_cols<PatView><<<g, kThreads, 0, stream()>>>(pat_view(A), Xc, Yc, ld);
      EVSLCU_LAUNCH_CHECK("k_spmv_cols");
      continue;
    }
    int rc = with_view(A, [&](auto view) {
      k_spmv_cols<decltype(view)><<<g, kThreads, 0, stream()>>>(view, Xc, Yc, ld);
      EVSLCU_LAUNCH_CHECK("k_spmv_cols");
      return 0;
    });
    if (rc) return rc;
  }
  return 0;
}

int evslcu_cheb_update(int n, int k, double t, double s, double cc, double *vkp1, const double *vk,
                       const double *vkm1, double *y) {
  k_cheb_update<<<grid_for(n), kThreads, 0, stream()>>>(n, k, t, s, -cc, vkp1, vk, vkm1, y);
  EVSLCU_LAUNCH_CHECK("k_cheb_update");
  return 0;
}

static int g_kpm_doubling = 1;
static int g_kpm_split = -1;  // -1: automatic, 0: never, 1: whenever the matrix has a column-split copy
static int g_kpm_pre = 0;     // 1: the k_kpm_dbl form that loads the rows' own values before the gathers

// The column-split copy the KPM block step runs on, or null for k_kpm_dbl:
// automatically for matrices whose columns reach far from the diagonal (the
// gathers of one step then spread over the whole probe block), whatever the
// probe count, so that probe shards take the same path as the full block.
static const evslcu_xsplit *kpm_split_copy(const evslcu_op *op) {
  if (g_kpm_split == 0 || !op->A) return nullptr;
  evslcu_mat *M = const_cast<evslcu_mat *>(op->A);
  if (g_kpm_split < 0 && M->bandwidth < (1 << 17)) return nullptr;
  return xsplit_for(M, sizeof(double) * kKpmChunk, g_kpm_split == 1);
}

}  // extern "C"

namespace evslcu {

template <bool PF, bool PL, bool FIRST>
static cudaError_t kpm_xs_launch(int grid, bool vec, const XsRange<double> &R, int B, int p0, int nb, const double *vk,
                                 const double *vkm1, double *o, double scal, double nctr, double *xpart, double *part) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return vec ? cudaLaunchKernelEx(&cfg, k_kpm_xs<PF, PL, FIRST, true>, R, B, p0, nb, vk, vkm1, o, scal, nctr, xpart, part)
             : cudaLaunchKernelEx(&cfg, k_kpm_xs<PF, PL, FIRST, false>, R, B, p0, nb, vk, vkm1, o, scal, nctr, xpart, part);
}

// One KPM block step of all probes on the column-split copy X: per chunk of 8
// probes, one launch per column range.
static int kpm_xs_step(const evslcu_mat *M, const evslcu_xsplit *X, int grid, int B, bool first, const double *vk,
                       const double *vkm1, double *o, double scal, double nctr, double *part) {
  const bool vec = (B % 2 == 0);
  double *xpart = (double *)M->xs_acc;
  for (int p0 = 0; p0 < B; p0 += kKpmChunk) {
    const int nb = std::min(kKpmChunk, B - p0);
    for (int p = 0; p < X->P; ++p) {
      const XsRange<double> R{M->n, X->cptr[p], X->cw[p], X->col[p], X->val[p], X->perm[p]};
      const bool pf = (p == 0), pl = (p == X->P - 1);
      cudaError_t e;
      if (pf && pl)
        e = first ? kpm_xs_launch<true, true, true>(grid, vec, R, B, p0, nb, vk, vkm1, o, scal, nctr, xpart, part)
                  : kpm_xs_launch<true, true, false>(grid, vec, R, B, p0, nb, vk, vkm1, o, scal, nctr, xpart, part);
      else if (pf)
        e = kpm_xs_launch<true, false, false>(grid, vec, R, B, p0, nb, vk, vkm1, o, scal, nctr, xpart, part);
      else if (pl)
        e = first ? kpm_xs_launch<false, true, true>(grid, vec, R, B, p0, nb, vk, vkm1, o, scal, nctr, xpart, part)
                  : kpm_xs_launch<false, true, false>(grid, vec, R, B, p0, nb, vk, vkm1, o, scal, nctr, xpart, part);
      else
        e = kpm_xs_launch<false, false, false>(grid, vec, R, B, p0, nb, vk, vkm1, o, scal, nctr, xpart, part);
      if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "KPM launch failed: %s", cudaGetErrorString(e));
      count_launch();
      int rc = check_launch("k_kpm_xs");
      if (rc) return rc;
    }
  }
  return 0;
}

}  // namespace evslcu

extern "C" {

static double *g_kpm_ws = nullptr;  // cached KPM workspace (product-identity path)
static size_t g_kpm_ws_cap = 0;

void evslcu_kpm_release(void) {
  evslcu_free(g_kpm_ws);
  g_kpm_ws = nullptr;
  g_kpm_ws_cap = 0;
}

int evslcu_set_kpm_doubling(int on) {
  g_kpm_doubling = on ? 1 : 0;
  return 0;
}

int evslcu_set_kpm_prefetch(int on) {
  g_kpm_pre = on ? 1 : 0;
  return 0;
}

int evslcu_set_kpm_split(int mode) {
  if (mode < -1 || mode > 1) return fail(EVSLCU_ERR_ARG, "KPM split mode must be -1, 0 or 1");
  g_kpm_split = mode;
  return 0;
}

// KPM dots through the product identities: K = ceil(Mdeg/2) block steps,
// raw sums a_k = <w_k+1, w_k+1>, b_k = <w_k+1, w_k>, c = <w_0, w_0>; then
// mu_2k+1 = 2 b_k - mu_1 (mu_1 = b_0) and mu_2k+2 = 2 a_k - c, per probe.
static int kpm_dots_doubling(const evslcu_op *op, int n, int Mdeg, int nvec, const double *probes, double ctr,
                             double wid, double *dots) {
  const int B = nvec;
  const int K = (Mdeg + 1) / 2;
  const size_t blk = (size_t)n * B;
  const int grid = kpm_grid(n);  // a function of n only: the summation order does not depend on B
  // one cached workspace (grows, never shrinks): repeated DOS estimates do
  // not allocate, and no free synchronises the device between them
  const size_t n_buf = blk * 3, n_raw = (size_t)K * 3 * B, n_nrm = (size_t)B,
               n_part = (size_t)std::max(3 * grid * B, 512 * B);
  const size_t need = n_buf + n_raw + n_nrm + n_part + 4 * 32;
  if (need > g_kpm_ws_cap) {
    evslcu_free(g_kpm_ws);
    g_kpm_ws = (double *)evslcu_malloc(sizeof(double) * need);
    g_kpm_ws_cap = g_kpm_ws ? need : 0;
  }
  double *buf = g_kpm_ws;
  double *raw = buf ? buf + (n_buf + 31) / 32 * 32 : nullptr;
  double *nrm = raw ? raw + (n_raw + 31) / 32 * 32 : nullptr;
  double *part = nrm ? nrm + (n_nrm + 31) / 32 * 32 : nullptr;
  std::vector<double> hraw((size_t)K * 3 * B);
  int rc = 0;
  if (!buf) rc = fail(EVSLCU_ERR_NOMEM, "kpm: out of device memory");
  double *V0 = buf, *W0 = buf + blk, *W1 = buf + 2 * blk;
  if (!rc) {
    dim3 g(std::min(grid_for(n), 512), B);
    k_colsq_partial<<<g, kThreads, 0, stream()>>>(n, B, probes, part, counters() + CTR_COL, nrm);
    count_launch();
    rc = check_launch("k_colsq_partial");
  }
  if (!rc) {
    k_interleave_scaled<<<grid_for(blk), kThreads, 0, stream()>>>(n, B, probes, nrm, V0);
    count_launch();
    rc = check_launch("k_interleave_scaled");
  }
  const CsrView A = csr_view(op->A);
  const double nctr = -ctr;
  double *W[2] = {W0, W1};
  const evslcu_xsplit *X = rc ? nullptr : kpm_split_copy(op);
  for (int k = 0; !rc && k < K; ++k) {
    const double scal = (k == 0 ? 1.0 : 2.0) / wid;
    const double *vk = (k == 0) ? V0 : W[(k - 1) % 2];
    const double *vkm1 = (k == 0) ? nullptr : ((k == 1) ? V0 : W[k % 2]);
    double *o = W[k % 2];
    double *rr = raw + (size_t)k * 3 * B;
    if (X) rc = kpm_xs_step(op->A, X, grid, B, k == 0, vk, vkm1, o, scal, nctr, part);
    for (int p0 = 0; !X && !rc && p0 < B; p0 += 32) {
      const int nb = std::min(32, B - p0);
      const bool vec = (B % 2 == 0);  // two probes per 16-byte access
      if (g_kpm_pre) {
        if (k == 0 && vec)
          k_kpm_dbl<true, true, true><<<grid, kThreads, 0, stream()>>>(A, B, p0, nb, vk, vkm1, o, scal, nctr, part);
        else if (k == 0)
          k_kpm_dbl<true, false, true><<<grid, kThreads, 0, stream()>>>(A, B, p0, nb, vk, vkm1, o, scal, nctr, part);
        else if (vec)
          k_kpm_dbl<false, true, true><<<grid, kThreads, 0, stream()>>>(A, B, p0, nb, vk, vkm1, o, scal, nctr, part);
        else
          k_kpm_dbl<false, false, true><<<grid, kThreads, 0, stream()>>>(A, B, p0, nb, vk, vkm1, o, scal, nctr, part);
      } else if (k == 0 && vec)
        k_kpm_dbl<true, true, false><<<grid, kThreads, 0, stream()>>>(A, B, p0, nb, vk, vkm1, o, scal, nctr, part);
      else if (k == 0)
        k_kpm_dbl<true, false, false><<<grid, kThreads, 0, stream()>>>(A, B, p0, nb, vk, vkm1, o, scal, nctr, part);
      else if (vec)
        k_kpm_dbl<false, true, false><<<grid, kThreads, 0, stream()>>>(A, B, p0, nb, vk, vkm1, o, scal, nctr, part);
      else
        k_kpm_dbl<false, false, false><<<grid, kThreads, 0, stream()>>>(A, B, p0, nb, vk, vkm1, o, scal, nctr, part);
      count_launch();
      rc = check_launch("k_kpm_dbl");
    }
    if (!rc) {
      k_kpm_reduce<<<(k == 0 ? 3 : 2) * B, kThreads, 0, stream()>>>(grid, part, rr);
      count_launch();
      rc = check_launch("k_kpm_reduce");
    }
  }
  if (!rc) rc = evslcu_d2h(hraw.data(), raw, sizeof(double) * hraw.size());
  if (!rc) {
    // dots[(j-1)*B + p] = mu_j, j = 1..Mdeg
    for (int p = 0; p < B; ++p) {
      const double cc0 = hraw[2 * (size_t)B + p];  // <w_0, w_0>
      const double mu1 = hraw[(size_t)B + p];      // <w_1, w_0>
      for (int k = 0; k < K; ++k) {
        const double a = hraw[(size_t)k * 3 * B + p], b = hraw[(size_t)k * 3 * B + B + p];
        const int j1 = 2 * k + 1, j2 = 2 * k + 2;
        dots[(size_t)(j1 - 1) * B + p] = (k == 0) ? mu1 : 2.0 * b - mu1;
        if (j2 <= Mdeg) dots[(size_t)(j2 - 1) * B + p] = 2.0 * a - cc0;
      }
    }
  }
  return rc;
}

int evslcu_kpm_dots(const evslcu_op *op, int n, int Mdeg, int nvec, const double *probes, double ctr, double wid,
                    double *dots) {
  if (!op || !op->A) return fail(EVSLCU_ERR_STATE, "KPM needs a registered CSR matrix");
  if (nvec < 1 || nvec > 128 || Mdeg < 1 || n < 1) return fail(EVSLCU_ERR_ARG, "kpm: bad sizes");
  if (g_kpm_doubling) return kpm_dots_doubling(op, n, Mdeg, nvec, probes, ctr, wid, dots);
  const int B = nvec;
  const size_t blk = (size_t)n * B;
  double *buf = (double *)evslcu_malloc(sizeof(double) * blk * 3);
  double *ddots = (double *)evslcu_malloc(sizeof(double) * (size_t)Mdeg * B);
  double *nrm = (double *)evslcu_malloc(sizeof(double) * B);
  int grid = kpm_grid(n);
  double *part = (double *)evslcu_malloc(sizeof(double) * (size_t)std::max(grid * B, 512 * B));
  if (!buf || !ddots || !nrm || !part) {
    evslcu_free(buf);
    evslcu_free(ddots);
    evslcu_free(nrm);
    evslcu_free(part);
    return EVSLCU_ERR_NOMEM;
  }
  double *V0 = buf, *W0 = buf + blk, *W1 = buf + 2 * blk;
  int rc = 0;
  {
    dim3 g(std::min(grid_for(n), 512), B);
    k_colsq_partial<<<g, kThreads, 0, stream()>>>(n, B, probes, part, counters() + CTR_COL, nrm);
    count_launch();
    if ((rc = check_launch("k_colsq_partial"))) goto done;
    k_interleave_scaled<<<grid_for(blk), kThreads, 0, stream()>>>(n, B, probes, nrm, V0);
    count_launch();
    if ((rc = check_launch("k_interleave_scaled"))) goto done;
  }
  {
    const CsrView A = csr_view(op->A);
    const double nctr = -ctr;
    unsigned int *c = counters() + CTR_KPM;
    double *W[2] = {W0, W1};
    for (int k = 0; k < Mdeg; ++k) {
      const double scal = (k == 0 ? 1.0 : 2.0) / wid;
      const double *vk = (k == 0) ? V0 : W[(k - 1) % 2];
      const double *vkm1 = (k == 0) ? nullptr : ((k == 1) ? V0 : W[k % 2]);
      double *out = W[k % 2];
      double *drow = ddots + (size_t)k * B;
      if (B <= 32) {
        if (k == 0)
          k_kpm<1, true><<<grid, kThreads, 0, stream()>>>(A, B, vk, vkm1, out, scal, nctr, V0, part, c, drow);
        else
          k_kpm<1, false><<<grid, kThreads, 0, stream()>>>(A, B, vk, vkm1, out, scal, nctr, V0, part, c, drow);
      } else if (B <= 64) {
        if (k == 0)
          k_kpm<2, true><<<grid, kThreads, 0, stream()>>>(A, B, vk, vkm1, out, scal, nctr, V0, part, c, drow);
        else
          k_kpm<2, false><<<grid, kThreads, 0, stream()>>>(A, B, vk, vkm1, out, scal, nctr, V0, part, c, drow);
      } else {
        if (k == 0)
          k_kpm<4, true><<<grid, kThreads, 0, stream()>>>(A, B, vk, vkm1, out, scal, nctr, V0, part, c, drow);
        else
          k_kpm<4, false><<<grid, kThreads, 0, stream()>>>(A, B, vk, vkm1, out, scal, nctr, V0, part, c, drow);
      }
      count_launch();
      if ((rc = check_launch("k_kpm"))) goto done;
    }
  }
  rc = evslcu_d2h(dots, ddots, sizeof(double) * (size_t)Mdeg * B);
done:
  evslcu_free(buf);
  evslcu_free(ddots);
  evslcu_free(nrm);
  evslcu_free(part);
  return rc;
}

int evslcu_rand_pm1(int n, int count, uint64_t seed, uint64_t draw, double *v) {
  k_rand_pm1<<<grid_for((long long)n * count), kThreads, 0, stream()>>>(n, count, seed, draw, v);
  EVSLCU_LAUNCH_CHECK("k_rand_pm1");
  return 0;
}

int evslcu_randn(int n, uint64_t seed, uint64_t draw, double *v) {
  k_randn<<<grid_for(n), kThreads, 0, stream()>>>(n, seed, draw, v);
  EVSLCU_LAUNCH_CHECK("k_randn");
  return 0;
}


size_t evslcu_kpm_noalloc_capacity(void) { return kNoAllocDoubles; }

size_t evslcu_kpm_noalloc_need(int n, int Mdeg, int nvec) {
  const int G = kpm_grid(n);
  const int gx = std::min(grid_for(n), 512);
  return 64 + (size_t)nvec /* norms */ + (size_t)(Mdeg + 1) /* jac */ + (size_t)Mdeg /* sdiff */ +
         (size_t)Mdeg * nvec /* dots */ + (size_t)std::max(G, gx) * nvec /* partials */ + (size_t)(Mdeg + 2) /* out */ +
         3 * (size_t)n * nvec /* block vectors */;
}

int evslcu_kpm_noalloc(const evslcu_op *op, int n, int Mdeg, int nvec, const double *probes, double ctr, double wid,
                       const double *jac_h, const double *sdiff_h, double bdiff, double t, double *mu_h,
                       double *ecnt_h) {
  if (!op || !op->A) return fail(EVSLCU_ERR_STATE, "KPM needs a registered CSR matrix");
  if (nvec < 1 || nvec > 128 || Mdeg < 1 || n < 1) return fail(EVSLCU_ERR_ARG, "kpm: bad sizes");
  const size_t need = evslcu_kpm_noalloc_need(n, Mdeg, nvec);
  if (need > kNoAllocDoubles)
    return fail(EVSLCU_ERR_ARG,
                "allocation-free kpmdos needs %zu doubles of scratch (3*n*nvec + Mdeg*nvec + ...) but the fixed "
                "scratch holds %zu (32 MiB); use kpmdos/evslx_kpmdos_probes for this size",
                need, kNoAllocDoubles);
  // The library's stream and the caller's probes live on the device the
  // library was started on; the scratch address is only valid there, so the
  // calling thread must have that device current.
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  if (dev != lib_device())
    return fail(EVSLCU_ERR_STATE,
                "allocation-free kpmdos called with device %d current; the library runs on device %d (make it "
                "current in this thread first)",
                dev, lib_device());
  // set-up, once per device, with that device current
  if (!g_noalloc_ptr || g_noalloc_dev != dev) {
    double *ptr = nullptr;
    e = cudaGetSymbolAddress((void **)&ptr, g_kpm_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(EVSLCU_ERR_CUDA, "cudaGetSymbolAddress of the KPM scratch failed: %s", cudaGetErrorString(e));
    g_noalloc_ptr = ptr;
    g_noalloc_dev = dev;
  }
  double *base = g_noalloc_ptr;
  unsigned int *ctrs = (unsigned int *)base;  // first 64 doubles: counters
  const int B = nvec;
  const int G = kpm_grid(n);
  const int gx = std::min(grid_for(n), 512);
  double *nrm = base + 64;
  double *jac = nrm + B;
  double *sdiff = jac + (Mdeg + 1);
  double *ddots = sdiff + Mdeg;
  double *part = ddots + (size_t)Mdeg * B;
  double *out = part + (size_t)std::max(G, gx) * B;
  double *V0 = out + (Mdeg + 2);
  const size_t blk = (size_t)n * B;
  double *W0 = V0 + blk, *W1 = W0 + blk;
  int rc;
  // the reduction counters must start at zero; the scratch keeps the last call's contents
  if ((rc = evslcu_memset(ctrs, 0, 64 * sizeof(double)))) return rc;
  if ((rc = evslcu_h2d(jac, jac_h, sizeof(double) * (Mdeg + 1))) || (rc = evslcu_h2d(sdiff, sdiff_h, sizeof(double) * Mdeg)))
    return rc;
  cudaStream_t st = stream();
  k_colsq_partial<<<dim3(gx, B), kThreads, 0, st>>>(n, B, probes, part, ctrs + 0, nrm);
  EVSLCU_LAUNCH_CHECK("k_colsq_partial");
  k_interleave_scaled<<<grid_for(blk), kThreads, 0, st>>>(n, B, probes, nrm, V0);
  EVSLCU_LAUNCH_CHECK("k_interleave_scaled");
  const CsrView A = csr_view(op->A);
  const double nctr = -ctr;
  double *W[2] = {W0, W1};
  for (int k = 0; k < Mdeg; ++k) {
    const double scal = (k == 0 ? 1.0 : 2.0) / wid;
    const double *vk = (k == 0) ? V0 : W[(k - 1) % 2];
    const double *vkm1 = (k == 0) ? nullptr : ((k == 1) ? V0 : W[k % 2]);
    double *o = W[k % 2];
    double *drow = ddots + (size_t)k * B;
    if (B <= 32) {
      if (k == 0)
        k_kpm<1, true><<<G, kThreads, 0, st>>>(A, B, vk, vkm1, o, scal, nctr, V0, part, ctrs + 1, drow);
      else
        k_kpm<1, false><<<G, kThreads, 0, st>>>(A, B, vk, vkm1, o, scal, nctr, V0, part, ctrs + 1, drow);
    } else if (B <= 64) {
      if (k == 0)
        k_kpm<2, true><<<G, kThreads, 0, st>>>(A, B, vk, vkm1, o, scal, nctr, V0, part, ctrs + 1, drow);
      else
        k_kpm<2, false><<<G, kThreads, 0, st>>>(A, B, vk, vkm1, o, scal, nctr, V0, part, ctrs + 1, drow);
    } else {
      if (k == 0)
        k_kpm<4, true><<<G, kThreads, 0, st>>>(A, B, vk, vkm1, o, scal, nctr, V0, part, ctrs + 1, drow);
      else
        k_kpm<4, false><<<G, kThreads, 0, st>>>(A, B, vk, vkm1, o, scal, nctr, V0, part, ctrs + 1, drow);
    }
    EVSLCU_LAUNCH_CHECK("k_kpm");
  }
  k_kpm_accumulate<<<1, 1, 0, st>>>(Mdeg, B, jac, sdiff, ddots, bdiff, t, (double)n, out, out + Mdeg + 1);
  EVSLCU_LAUNCH_CHECK("k_kpm_accumulate");
  if ((rc = evslcu_d2h(mu_h, out, sizeof(double) * (Mdeg + 1)))) return rc;
  return evslcu_d2h(ecnt_h, out + Mdeg + 1, sizeof(double));
}

int evslcu_set_rows_per_thread(int r) {
  if (r != 1 && r != 2) return fail(EVSLCU_ERR_ARG, "rows per thread must be 1 or 2");
  g_rows_per_thread = r;
  return 0;
}

int evslcu_chebav_block(const evslcu_op *op, const double *mu, int deg, double cc, double dd, int ncols,
                        const double *V, double *Y, double *work) {
  if (!op || !mu || deg < 0 || ncols < 1 || !V || !Y || !work) return fail(EVSLCU_ERR_ARG, "chebav_block: bad args");
  const int n = op->n;
  if (!op->A || deg == 0 || op->A->kernel != 0) {
    for (int c = 0; c < ncols; ++c) {
      int rc = evslcu_chebav(op, mu, deg, cc, dd, V + (size_t)c * n, Y + (size_t)c * n, work, nullptr);
      if (rc) return rc;
    }
    return 0;
  }
  // the multi-column filter (interleaved blocks of up to 16 columns); each
  // column bitwise equal to evslcu_chebav
  std::vector<evslcu_filter_col> cols((size_t)ncols);
  for (int c = 0; c < ncols; ++c) cols[c] = evslcu_filter_col{mu, deg, cc, dd, V + (size_t)c * n, Y + (size_t)c * n};
  const size_t need = evslcu_filter_columns_work(n, 0, ncols);
  void *w = evslcu_malloc(need);
  if (!w) return fail(EVSLCU_ERR_NOMEM, "chebav_block: out of device memory");
  int rc = evslcu_filter_columns(op->A, 0, ncols, cols.data(), w, need);
  evslcu_free(w);
  return rc;
}

}  // extern "C"
