// Column-panel storage and filter kernels for large general sparse matrices.
//
// On a matrix whose columns are spread at random (no stencil structure, x far
// larger than an SM's L1), every stored entry of the SpMV inside ChebAv
// (SRC/chebpoly.c:519-598; the CSR matvec SRC/spmat.c:257-298) is a gather
// from a different cache line: each costs one L1TEX wavefront and one L2
// sector, and those -- not DRAM -- bound the SELL kernels (one wavefront per
// nonzero).  Here each CTA owns a block of consecutive rows and walks the
// columns in panels of W entries: the panel of x is copied into shared memory
// (cp.async, double buffered with the panel's matrix data), and the gathers of
// the block's entries in that panel read shared memory, where 32 random reads
// cost a few bank wavefronts instead of 32 line requests.
//
// Layout.  Group g = (row block rb, panel p) holds the segments of the rows of
// rb in p: a segment is the contiguous part of a CSR row whose columns fall in
// the panel (columns are sorted, so a row's segments come panel by panel in
// CSR order).  A group's segments are sorted by length, longest first, ties
// in row order, and cut into chunks of 32 (one warp); entry j of lane l of
// chunk c sits at chunk_off[c] + 32 j + l; a lane shorter than its chunk is
// padded with value 0 at column 0.  Per group, 16-byte aligned:
//   meta: chunk_off[nch + 1] (u32) | rowid[32 nch] (u16, 0xffff = no row) |
//         col[E] (u16, column - p W)
//   vals: E values (FP64, and an FP32 copy for the FP32 filter).
// The per-group table holds the meta offset (16-byte units), the value
// offset, the chunk count and E.
//
// Arithmetic.  A lane owns one row's segment per panel and adds its products
// to the row's accumulator (shared memory) one by one, in column order; the
// panels are processed in increasing order with a barrier in between, so
// every row is summed left to right exactly as in the CSR matvec: the FP64
// kernel is bitwise equal to the reference's filter.  The FP32 kernel uses
// fused multiply-add, as the other FP32 kernels do.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "sparse_types.cuh"

struct evslcu_panels {
  int fp32 = 0;  // value type of this layout (its panel width is sized for it)
  int R = 0, W = 0, P = 0, RB = 0;
  size_t mcap = 0;  // largest group meta (bytes)
  int ecap = 0;     // largest group entry count
  int4 *gtab = nullptr;
  unsigned char *meta = nullptr;
  void *vals = nullptr;  // double or float
  size_t smem = 0;       // dynamic shared memory of the kernels
  size_t bytes = 0;      // device bytes held
};

namespace evslcu {

namespace {

constexpr int kPanelThreads = 1024;
constexpr size_t kSmemLimit = 227 * 1024 - 2048;

__host__ __device__ __forceinline__ size_t align16(size_t b) { return (b + 15) / 16 * 16; }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
template <int BYTES>
__device__ __forceinline__ void cp_async_small(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

struct PanelView {
  int n, R, W, P;
  const int4 *gtab;
  const unsigned char *meta;
  size_t mcap;  // bytes of one meta buffer in shared memory
  int ecap;     // entries of one value buffer
};

// Shared memory: acc[R] | x[2][W] | meta[2][mcap] | vals[2][ecap] (16-byte
// aligned parts); stage s of each double buffer is base + s * stride.
template <class VT>
struct PanelSmem {
  VT *acc;
  unsigned char *xb, *mb, *vb;
  size_t xs, ms, vs;  // stage strides (bytes)
  __device__ PanelSmem(unsigned char *base, const PanelView &A) {
    acc = (VT *)base;
    xs = align16(sizeof(VT) * A.W);
    ms = A.mcap;
    vs = align16(sizeof(VT) * A.ecap);
    xb = base + align16(sizeof(VT) * A.R);
    mb = xb + 2 * xs;
    vb = mb + 2 * ms;
  }
  __device__ __forceinline__ VT *x(int s) const { return (VT *)(xb + s * xs); }
  __device__ __forceinline__ unsigned char *m(int s) const { return mb + s * ms; }
  __device__ __forceinline__ VT *v(int s) const { return (VT *)(vb + s * vs); }
};

template <class VT>
size_t panel_smem_bytes(int R, int W, size_t mcap, int ecap) {
  return align16(sizeof(VT) * R) + 2 * align16(sizeof(VT) * W) + 2 * mcap + 2 * align16(sizeof(VT) * ecap);
}

// Issues the copies of panel p (x part, group meta, group values) into stage s.
template <class VT>
__device__ __forceinline__ void panel_load(const PanelView &A, const PanelSmem<VT> &S, int s, int rb, int p,
                                           const VT *__restrict__ x, const VT *__restrict__ vals, bool x16) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int c0 = p * A.W;
  const int nel = min(A.W, A.n - c0);
  const VT *xs = x + c0;
  if (x16) {
    constexpr int PER = 16 / sizeof(VT);
    const int n16 = nel / PER;
    for (int i = tid; i < n16; i += nt) cp_async16(S.x(s) + PER * i, xs + PER * i);
    for (int i = n16 * PER + tid; i < nel; i += nt) cp_async_small<sizeof(VT)>(S.x(s) + i, xs + i);
  } else {
    for (int i = tid; i < nel; i += nt) cp_async_small<sizeof(VT)>(S.x(s) + i, xs + i);
  }
  const int4 g = __ldg(A.gtab + (size_t)rb * A.P + p);
  const int nch = g.z, E = g.w;
  const size_t mbytes = align16(4 * (size_t)(nch + 1)) + align16(64 * (size_t)nch) + align16(2 * (size_t)E);
  const unsigned char *msrc = A.meta + 16 * (size_t)(unsigned)g.x;
  for (size_t i = tid; i < mbytes / 16; i += nt) cp_async16(S.m(s) + 16 * i, msrc + 16 * i);
  const VT *vsrc = vals + (size_t)(unsigned)g.y;
  constexpr int PER = 16 / sizeof(VT);
  for (int i = tid; i < E / PER; i += nt) cp_async16(S.v(s) + PER * i, vsrc + PER * i);
}

__device__ __forceinline__ double pmadd(double a, double v, double x) { return __dadd_rn(a, __dmul_rn(v, x)); }
__device__ __forceinline__ float pmadd(float a, float v, float x) { return fmaf(v, x, a); }

// acc[r - r0] = (row r of A) x for the rows of block rb, panel by panel.
// Ends with a barrier; acc is then complete in shared memory.
template <class VT>
__device__ __forceinline__ void panel_rows(const PanelView &A, const PanelSmem<VT> &S, int rb, int nrows,
                                           const VT *__restrict__ x, const VT *__restrict__ vals) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const bool x16 = ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
  for (int i = tid; i < nrows; i += nt) S.acc[i] = (VT)0;
  panel_load<VT>(A, S, 0, rb, 0, x, vals, x16);
  cp_async_commit();
  if (A.P > 1) panel_load<VT>(A, S, 1, rb, 1, x, vals, x16);
  cp_async_commit();
  for (int p = 0; p < A.P; ++p) {
    const int s = p & 1;
    cp_async_wait1();
    __syncthreads();
    const int4 g = __ldg(A.gtab + (size_t)rb * A.P + p);
    const int nch = g.z;
    const unsigned *coff = reinterpret_cast<const unsigned *>(S.m(s));
    const unsigned short *rid = reinterpret_cast<const unsigned short *>(S.m(s) + align16(4 * (size_t)(nch + 1)));
    const unsigned short *col =
        reinterpret_cast<const unsigned short *>(S.m(s) + align16(4 * (size_t)(nch + 1)) + align16(64 * (size_t)nch));
    const VT *xv = S.x(s);
    const VT *vv = S.v(s);
    for (int c = warp; c < nch; c += nw) {
      const unsigned o = coff[c], w = (coff[c + 1] - o) >> 5;
      const unsigned short r = rid[32 * c + lane];
      if (r != 0xffff) {
        VT a = S.acc[r];
        for (unsigned j = 0; j < w; ++j) {
          const unsigned e = o + 32 * j + lane;
          a = pmadd(a, vv[e], xv[col[e]]);
        }
        S.acc[r] = a;
      }
    }
    __syncthreads();
    if (p + 2 < A.P) panel_load<VT>(A, S, s, rb, p + 2, x, vals, x16);
    cp_async_commit();
  }
}

// FP64 degree step with the k_cheb epilogue (same rounded operations).
template <bool FIRST, bool EPI>
__global__ void __launch_bounds__(kPanelThreads, 1)
    k_cheb_panel(PanelView A, const double *__restrict__ vals, const double *__restrict__ vk, const double *vkm1,
                 double *out, double *__restrict__ y, double t, double ncc, double s, double mu0,
                 const double *__restrict__ zold, double nbeta, const double *__restrict__ dotv, double *part,
                 unsigned int *ctr, double *dot_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sh[kPanelThreads / 32];
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const PanelSmem<double> S(smem_raw, A);
  const int rb = blockIdx.x;
  const int r0 = rb * A.R;
  const int nrows = min(A.R, A.n - r0);
  panel_rows<double>(A, S, rb, nrows, vk, vals);
  double dsum = 0.0;
  for (int i = threadIdx.x; i < nrows; i += blockDim.x) {
    const int r = r0 + i;
    const double xm1 = FIRST ? 0.0 : vkm1[r];
    const double yo = FIRST ? 0.0 : y[r];
    const double x = vk[r];
    double w = __dmul_rn(t, __dadd_rn(S.acc[i], __dmul_rn(ncc, x)));
    if (!FIRST) w = __dadd_rn(w, -xm1);
    out[r] = w;
    double yv = FIRST ? __dmul_rn(mu0, x) : yo;
    yv = __dadd_rn(yv, __dmul_rn(s, w));
    if (EPI) {
      if (zold) yv = __dadd_rn(yv, __dmul_rn(nbeta, zold[r]));
      if (dotv) dsum += dotv[r] * yv;
    }
    y[r] = yv;
  }
  if (EPI && dot_out) {
    const double b = block_sum(dsum, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = b;
    if (last_block(ctr)) {
      const double tot = reduce_partials(part, gridDim.x, ctr, sh);
      if (threadIdx.x == 0) *dot_out = tot;
    }
  }
}

// One column of the multi-column filter (k_mf_step with B = 1), coefficient
// table row of this degree: t, -cc, mu_k, 1 while k <= deg.
template <class VT, bool FIRST>
__global__ void __launch_bounds__(kPanelThreads, 1)
    k_mf_panel(PanelView A, const VT *__restrict__ vals, const VT *__restrict__ vk, const VT *vkm1, VT *out,
               VT *__restrict__ y, const VT *__restrict__ coef) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const PanelSmem<VT> S(smem_raw, A);
  const int rb = blockIdx.x;
  const int r0 = rb * A.R;
  const int nrows = min(A.R, A.n - r0);
  panel_rows<VT>(A, S, rb, nrows, vk, vals);
  const VT c0 = __ldg(coef), c1 = __ldg(coef + 1), c2 = __ldg(coef + 2), c3 = __ldg(coef + 3);
  for (int i = threadIdx.x; i < nrows; i += blockDim.x) {
    const int r = r0 + i;
    const VT xr = vk[r];
    VT w = c0 * (S.acc[i] + c1 * xr);
    if (!FIRST) w = w + (-vkm1[r]);
    out[r] = w;
    if (c3 != (VT)0) y[r] = y[r] + c2 * w;
  }
}

// ---------------------------------------------------------------------------
// Host build
// ---------------------------------------------------------------------------
struct Seg {
  int len, row, start;
};

// Builds the panel layout for row blocks of R rows and panels of W columns
// into host arrays.  Returns false if a group would not fit in shared memory.
bool build_host(int n, const std::vector<int> &ia, const std::vector<int> &ja, const std::vector<double> &a, int R,
                int W, std::vector<int4> &gtab, std::vector<unsigned char> &meta, std::vector<double> &vals,
                size_t &mcap, int &ecap) {
  const int RB = (n + R - 1) / R, P = (n + W - 1) / W;
  gtab.assign((size_t)RB * P, int4{0, 0, 0, 0});
  meta.clear();
  vals.clear();
  mcap = 16;
  ecap = 0;
  std::vector<std::vector<Seg>> lists(P);
  std::vector<int> bucket;
  for (int rb = 0; rb < RB; ++rb) {
    for (auto &l : lists) l.clear();
    const int r0 = rb * R, r1 = std::min(n, r0 + R);
    for (int r = r0; r < r1; ++r) {
      int j = ia[r];
      const int e = ia[r + 1];
      while (j < e) {
        const int p = ja[j] / W;
        int k = j + 1;
        while (k < e && ja[k] / W == p) ++k;
        lists[p].push_back(Seg{k - j, r - r0, j});
        j = k;
      }
    }
    for (int p = 0; p < P; ++p) {
      std::vector<Seg> &L = lists[p];
      std::stable_sort(L.begin(), L.end(), [](const Seg &x, const Seg &y) { return x.len > y.len; });
      const int nseg = (int)L.size();
      const int nch = (nseg + 31) / 32;
      std::vector<unsigned> coff(nch + 1, 0);
      for (int c = 0; c < nch; ++c) coff[c + 1] = coff[c] + 32u * (unsigned)L[32 * c].len;
      const int E = (int)coff[nch];
      const size_t mb = align16(4 * (size_t)(nch + 1)) + align16(64 * (size_t)nch) + align16(2 * (size_t)E);
      while (meta.size() % 16) meta.push_back(0);
      while (vals.size() % 4) vals.push_back(0.0);
      if (meta.size() / 16 > 0x7fffffffULL || vals.size() > 0x7fffffffULL) return false;
      gtab[(size_t)rb * P + p] = int4{(int)(meta.size() / 16), (int)vals.size(), nch, E};
      const size_t mbase = meta.size();
      meta.resize(mbase + mb, 0);
      const size_t vbase = vals.size();
      vals.resize(vbase + (size_t)E, 0.0);
      unsigned char *mp = meta.data() + mbase;
      memcpy(mp, coff.data(), 4 * (size_t)(nch + 1));
      unsigned short *rid = reinterpret_cast<unsigned short *>(mp + align16(4 * (size_t)(nch + 1)));
      unsigned short *col =
          reinterpret_cast<unsigned short *>(mp + align16(4 * (size_t)(nch + 1)) + align16(64 * (size_t)nch));
      for (int i = 0; i < 32 * nch; ++i) rid[i] = 0xffff;
      for (int sg = 0; sg < nseg; ++sg) {
        const int c = sg / 32, l = sg % 32;
        rid[sg] = (unsigned short)L[sg].row;
        for (int j = 0; j < L[sg].len; ++j) {
          const size_t e = coff[c] + 32 * (size_t)j + l;
          col[e] = (unsigned short)(ja[L[sg].start + j] - p * W);
          vals[vbase + e] = a[L[sg].start + j];
        }
      }
      mcap = std::max(mcap, mb);
      ecap = std::max(ecap, E);
    }
  }
  while (vals.size() % 4) vals.push_back(0.0);
  return true;
}

inline PanelView panel_view(const evslcu_mat *M, const evslcu_panels *P) {
  return PanelView{M->n, P->R, P->W, P->P, P->gtab, P->meta, P->mcap, P->ecap};
}

template <class F, class... Args>
int launch_panel(F fn, int grid, size_t smem, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kPanelThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, fn, args...);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "panel filter launch failed: %s", cudaGetErrorString(e));
  count_launch();
  return check_launch("panel filter");
}

template <class F>
int set_smem(F fn, size_t bytes) {
  cudaError_t e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "panel filter: shared memory limit: %s", cudaGetErrorString(e));
  return 0;
}

}  // namespace

// Minimum rows for the panel layout (smaller x stays in L1/L2 well enough).
int g_panel_min_rows = 1 << 18;
int g_panel_enabled = 1;

bool panel_candidate(const evslcu_mat *M) {
  return g_panel_enabled && M->kernel == 0 && M->perm && M->n >= g_panel_min_rows && M->n <= (1 << 30);
}

int panel_build(evslcu_mat *M, int fp32) {
  evslcu_panels *&slot = fp32 ? M->pn32 : M->pn64;
  if (slot) return 0;
  const int n = M->n;
  const long long nnz = M->nnz;
  std::vector<int> ia(n + 1), ja((size_t)std::max(nnz, 1LL));
  std::vector<double> a((size_t)std::max(nnz, 1LL));
  int rc = evslcu_d2h(ia.data(), M->ia, sizeof(int) * (size_t)(n + 1));
  if (!rc && nnz) rc = evslcu_d2h(ja.data(), M->ja, sizeof(int) * (size_t)nnz);
  if (!rc && nnz) rc = evslcu_d2h(a.data(), M->a, sizeof(double) * (size_t)nnz);
  if (rc) return rc;
  const size_t vb = fp32 ? sizeof(float) : sizeof(double);
  // one row block per SM (one wave of one CTA per SM), at most 65504 rows
  const int sms = std::max(1, sm_count());
  int R = (int)std::min<long long>(((long long)n + sms - 1) / sms, 65504);
  R = std::min((R + 31) / 32 * 32, 65504);
  std::vector<int4> gtab;
  std::vector<unsigned char> meta;
  std::vector<double> vals;
  size_t mcap = 0;
  int ecap = 0;
  int W = 0;
  // the widest panel whose kernel fits shared memory with the largest group
  for (int w : {16384, 12288, 8192, 6144, 4096, 3072, 2048, 1024}) {
    if (align16(vb * R) + 2 * align16(vb * w) > kSmemLimit) continue;
    if (!build_host(n, ia, ja, a, R, w, gtab, meta, vals, mcap, ecap)) return 0;
    const size_t need = fp32 ? panel_smem_bytes<float>(R, w, mcap, ecap) : panel_smem_bytes<double>(R, w, mcap, ecap);
    if (need <= kSmemLimit) {
      W = w;
      break;
    }
  }
  if (!W) return 0;  // no layout fits: the SELL kernels stay in use
  evslcu_panels *P = new evslcu_panels();
  P->fp32 = fp32;
  P->R = R;
  P->W = W;
  P->P = (n + W - 1) / W;
  P->RB = (n + R - 1) / R;
  P->mcap = mcap;
  P->ecap = ecap;
  P->smem = fp32 ? panel_smem_bytes<float>(R, W, mcap, ecap) : panel_smem_bytes<double>(R, W, mcap, ecap);
  std::vector<float> vals32;
  if (fp32) vals32.assign(vals.begin(), vals.end());
  const void *vsrc = fp32 ? (const void *)vals32.data() : (const void *)vals.data();
  P->gtab = (int4 *)evslcu_malloc(sizeof(int4) * gtab.size());
  P->meta = (unsigned char *)evslcu_malloc(meta.size());
  P->vals = evslcu_malloc(vb * vals.size());
  P->bytes = sizeof(int4) * gtab.size() + meta.size() + vb * vals.size();
  if (!P->gtab || !P->meta || !P->vals || evslcu_h2d(P->gtab, gtab.data(), sizeof(int4) * gtab.size()) ||
      evslcu_h2d(P->meta, meta.data(), meta.size()) || evslcu_h2d(P->vals, vsrc, vb * vals.size())) {
    evslcu_free(P->gtab);
    evslcu_free(P->meta);
    evslcu_free(P->vals);
    delete P;
    return fail(EVSLCU_ERR_NOMEM, "panel layout: out of device memory");
  }
  slot = P;
  return 0;
}

void panel_free(evslcu_mat *M) {
  for (evslcu_panels **pp : {&M->pn64, &M->pn32}) {
    evslcu_panels *P = *pp;
    if (!P) continue;
    evslcu_free(P->gtab);
    evslcu_free(P->meta);
    evslcu_free(P->vals);
    delete P;
    *pp = nullptr;
  }
}

int panel_cheb_step(const evslcu_mat *M, bool first, bool epi, const double *vk, const double *vkm1, double *out,
                    double *y, double t, double ncc, double s, double mu0, const double *zold, double nbeta,
                    const double *dotv, double *dout) {
  const evslcu_panels *P = M->pn64;
  if (!P) return fail(EVSLCU_ERR_STATE, "panel layout not built");
  const PanelView A = panel_view(M, P);
  static size_t set_bytes[4] = {0, 0, 0, 0};
  auto go = [&](auto fn, int idx) -> int {
    if (set_bytes[idx] < P->smem) {
      int rc = set_smem(fn, P->smem);
      if (rc) return rc;
      set_bytes[idx] = P->smem;
    }
    return launch_panel(fn, P->RB, P->smem, A, (const double *)P->vals, vk, vkm1, out, y, t, ncc, s, mu0, zold,
                        nbeta, dotv, partials(), counters() + CTR_CHEB, dout);
  };
  if (first && epi) return go(k_cheb_panel<true, true>, 0);
  if (first) return go(k_cheb_panel<true, false>, 1);
  if (epi) return go(k_cheb_panel<false, true>, 2);
  return go(k_cheb_panel<false, false>, 3);
}

template <class VT>
int panel_mf_step(const evslcu_mat *M, int k, const VT *vk, const VT *vkm1, VT *out, VT *y, const VT *coef) {
  const bool f32 = sizeof(VT) == 4;
  const evslcu_panels *P = f32 ? M->pn32 : M->pn64;
  if (!P) return fail(EVSLCU_ERR_STATE, "panel layout not built");
  const PanelView A = panel_view(M, P);
  static size_t set_bytes[2] = {0, 0};
  auto go = [&](auto fn, int idx) -> int {
    if (set_bytes[idx] < P->smem) {
      int rc = set_smem(fn, P->smem);
      if (rc) return rc;
      set_bytes[idx] = P->smem;
    }
    return launch_panel(fn, P->RB, P->smem, A, (const VT *)P->vals, vk, vkm1, out, y, coef);
  };
  return (k == 1) ? go(k_mf_panel<VT, true>, 0) : go(k_mf_panel<VT, false>, 1);
}

template int panel_mf_step<float>(const evslcu_mat *, int, const float *, const float *, float *, float *,
                                  const float *);
template int panel_mf_step<double>(const evslcu_mat *, int, const double *, const double *, double *, double *,
                                   const double *);

}  // namespace evslcu

extern "C" {

int evslcu_set_panels(int on, int min_rows) {
  evslcu::g_panel_enabled = on ? 1 : 0;
  if (min_rows > 0) evslcu::g_panel_min_rows = min_rows;
  return 0;
}

int evslcu_mat_panel_layout(const evslcu_mat *A, int fp32, int *rows_per_block, int *panel_width,
                            long long *bytes) {
  if (!A) return evslcu::fail(EVSLCU_ERR_ARG, "null matrix");
  const evslcu_panels *P = fp32 ? A->pn32 : A->pn64;
  if (rows_per_block) *rows_per_block = P ? P->R : 0;
  if (panel_width) *panel_width = P ? P->W : 0;
  if (bytes) *bytes = P ? (long long)P->bytes : 0;
  return 0;
}

}  // extern "C"
