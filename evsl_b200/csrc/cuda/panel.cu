// Column-panel storage and filter kernels for large general sparse matrices.
//
// On a matrix whose columns are spread at random (no stencil structure, x far
// larger than an SM's L1), every stored entry of the SpMV inside ChebAv
// (SRC/chebpoly.c:519-598; the CSR matvec SRC/spmat.c:257-298) is a gather
// from a different cache line: each costs one L1TEX wavefront, and those --
// not DRAM -- bound the SELL kernels (one wavefront per nonzero).  Here each
// CTA owns a block of consecutive rows and walks the columns in panels of W
// entries: the panel of x and the block's matrix entries in that panel are
// copied into shared memory by TMA bulk copies, and the gathers read shared
// memory, where 32 random reads cost a few bank wavefronts instead of 32 line
// requests.
//
// Rows.  The rows are cut into chunks of 32; CTA b owns the chunks c with
// c % RB == b (RB CTAs, one per SM), so that the diagonal entries of its rows
// (and any band around it) spread evenly over all panels instead of crowding
// the few panels next to a contiguous row block.  Local row lr of the CTA is
// row 32 (c / RB) + lr % 32 of its chunk list.
//
// Pipeline.  One producer warp (lane 0) issues the bulk copies of panel p into
// stage p % S of an S-stage ring (full/empty mbarriers) and runs up to S
// panels ahead; NC consumer warps share each panel's chunks as soon as its
// stage is full, meet at a named barrier (the producer warp does not take
// part), and release the stage.  Every mbarrier wait is bounded; a wait that
// runs out records the error flag the host checks after the filter, and the
// kernel finishes without waiting further.
//
// Layout.  Group g = (row block rb, panel p) holds the segments of the rows of
// rb in p: a segment is the contiguous part of a CSR row whose columns fall in
// the panel (columns are sorted, so a row's segments come panel by panel in
// CSR order).  A group's segments are sorted by length, longest first, ties
// in row order, and cut into chunks of 32 lanes; entry j of lane l of chunk c
// sits at coff[c] + 32 j + l; a lane shorter than its chunk is padded with
// value 0 at column 0.  Per group, each part 16-byte aligned:
//   meta: {nch, E} (u32) | coff[nch + 1] (u32) | rowid[32 nch] (u16,
//         0xffff = no row) | col[E] (u16, column - p W)
//   vals: E values (double for the FP64 layout, float for the FP32 one).
//
// Arithmetic.  A lane adds its segment's products to the row's accumulator
// (shared memory) one by one in column order; a row has one segment per
// panel and the panels follow one another behind the consumers' barrier, so
// every row is summed left to right exactly as in the CSR matvec: the FP64
// kernel is bitwise equal to the reference's filter.  The FP32 kernel uses
// fused multiply-add from zero in the same order, as the SELL kernels do.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "sparse_types.cuh"

namespace evslcu {
namespace {
constexpr int kConsumerWarps = 31;
constexpr int kPanelThreads = 32 * (kConsumerWarps + 1);
constexpr int kMaxStages = 8;
}  // namespace
}  // namespace evslcu

struct evslcu_panels {
  int fp32 = 0;  // value type of this layout (its panel width is sized for it)
  int R = 0, W = 0, P = 0, RB = 0, S = 0;
  unsigned mcap = 0, vcap = 0, xcap = 0;  // bytes of one stage's meta, values, x panel
  int4 *gtab = nullptr;
  unsigned char *meta = nullptr;
  void *vals = nullptr;  // double or float
  size_t smem = 0;       // dynamic shared memory of the kernels
  size_t bytes = 0;      // device bytes held
};

namespace evslcu {

namespace {

constexpr size_t kSmemLimit = 227 * 1024 - 4096;
constexpr unsigned long long kPanelWaitPolls = 1ull << 25;  // ~1-2 s with the sleeps

__host__ __device__ __forceinline__ size_t align16(size_t b) { return (b + 15) / 16 * 16; }

// meta of a group: header {nch, E, 0, 0} (u32) | coff[nch + 1] | rowid[32 nch] | col[E]
__host__ __device__ __forceinline__ size_t meta_bytes(int nch, int E) {
  return 16 + align16(4 * (size_t)(nch + 1)) + align16(64 * (size_t)nch) + align16(2 * (size_t)E);
}

struct PanelView {
  int n, R, W, P, S, RB;
  const int4 *gtab;
  const unsigned char *meta;
  unsigned mcap, vcap, xcap;
  int *err;
  unsigned long long polls;
};

// Global row of local row lr of CTA rb (may be >= n in the last chunk).
__device__ __forceinline__ int panel_row(const PanelView &A, int rb, int lr) {
  return 32 * ((lr >> 5) * A.RB + rb) + (lr & 31);
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Non-blocking test of the phase with the given parity (test_wait returns at
// once; try_wait may suspend the thread for a time slice, which put several
// microseconds into every hop of the ring).
__device__ __forceinline__ bool mbar_test_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the completion of the phase with the given parity: polls
// with a short sleep between tests after the first few.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned long long polls) {
  for (unsigned long long i = 0; i < polls; ++i) {
    if (mbar_test_wait(bar, parity)) return true;
    if (i > 8) __nanosleep(32);
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Shared memory: acc[R] | stage 0 .. S-1, each x (xcap) | meta (mcap) | vals (vcap).
template <class VT>
struct PanelSmem {
  VT *acc;
  unsigned char *st;
  unsigned stride, xcap, mcap;
  __device__ PanelSmem(unsigned char *base, const PanelView &A) {
    acc = (VT *)base;
    st = base + align16(sizeof(VT) * A.R);
    xcap = A.xcap;
    mcap = A.mcap;
    stride = A.xcap + A.mcap + A.vcap;
  }
  __device__ __forceinline__ VT *x(int s) const { return (VT *)(st + s * stride); }
  __device__ __forceinline__ unsigned char *m(int s) const { return st + s * stride + xcap; }
  __device__ __forceinline__ VT *v(int s) const { return (VT *)(st + s * stride + xcap + mcap); }
};

template <class VT>
size_t panel_smem_bytes(int R, int S, unsigned xcap, unsigned mcap, unsigned vcap) {
  return align16(sizeof(VT) * R) + (size_t)S * (xcap + mcap + vcap);
}

__device__ __forceinline__ double pmadd(double a, double v, double x) { return __dadd_rn(a, __dmul_rn(v, x)); }
__device__ __forceinline__ float pmadd(float a, float v, float x) { return fmaf(v, x, a); }
// rounded multiply and add of the recurrence's update (as in k_mf_step)
__device__ __forceinline__ double pmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float pmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double padd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float padd(float a, float b) { return __fadd_rn(a, b); }

// Producer (the last warp; lane 0 issues): panel p's x part, the group's meta
// and its values, all completing on full[p % S].  x is copied from its
// address aligned down to 16 bytes (the panel sits at element offset d of the
// stage's x buffer) up to the next 16 bytes past the panel when at least 16
// bytes of x follow the panel; otherwise the copy stops at the panel's last
// whole 16 bytes and lane 0 stores the remaining elements.  The lanes load
// the group table 32 panels at a time, one batch ahead.
template <class VT>
__device__ void panel_produce(const PanelView &A, const PanelSmem<VT> &S, unsigned long long *full,
                              unsigned long long *empty, int rb, const VT *x, const VT *vals, int lane) {
  const uintptr_t xa = reinterpret_cast<uintptr_t>(x);
  const int d = (int)((xa & 15) / sizeof(VT));
  const unsigned char *xbase = reinterpret_cast<const unsigned char *>(xa & ~(uintptr_t)15);
  const int4 *gt = A.gtab + (size_t)rb * A.P;
  int issued = 0;
  int ok = 1;
  int4 gnext = (lane < A.P) ? __ldg(gt + lane) : int4{0, 0, 0, 0};
  for (int p0 = 0; p0 < A.P && ok; p0 += 32) {
    const int4 gcur = gnext;
    if (p0 + 32 + lane < A.P) gnext = __ldg(gt + p0 + 32 + lane);
    const int pend = min(A.P, p0 + 32);
    for (int p = p0; p < pend; ++p) {
      int4 g;
      g.x = __shfl_sync(0xffffffffu, gcur.x, p - p0);
      g.y = __shfl_sync(0xffffffffu, gcur.y, p - p0);
      g.z = __shfl_sync(0xffffffffu, gcur.z, p - p0);
      g.w = __shfl_sync(0xffffffffu, gcur.w, p - p0);
      const int s = p % A.S;
      const int round = p / A.S;
      if (lane == 0 && round > 0 && !mbar_wait(&empty[s], (unsigned)((round - 1) & 1), A.polls)) {
        atomicExch(A.err, 1);
        ok = 0;
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      if (lane == 0) {
        const int c0 = p * A.W;
        const int nel = min(A.W, A.n - c0);
        const bool roomy = (size_t)(c0 + nel) * sizeof(VT) + 16 <= (size_t)A.n * sizeof(VT);
        const size_t span = (size_t)(d + nel) * sizeof(VT);
        const unsigned bulk = (unsigned)(roomy ? align16(span) : (span & ~(size_t)15));
        VT *xs = S.x(s);
        if (!roomy)
          for (int e = max((int)(bulk / sizeof(VT)) - d, 0); e < nel; ++e) xs[d + e] = x[c0 + e];
        const unsigned mb = (unsigned)meta_bytes(g.z, g.w);
        const unsigned vb = (unsigned)(sizeof(VT) * (size_t)g.w);
        if (!roomy) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the stores above
        mbar_arrive_expect_tx(&full[s], bulk + mb + vb);
        if (bulk) {
          // every CTA reads the same panel of x: start each CTA's copy at its
          // own 128-byte line within the panel (two copies, wrapped), so the
          // CTAs do not all stream the same L2 lines at the same moment
          const unsigned lines = bulk / 128;
          const unsigned rot = lines ? 128u * (unsigned)((rb * 37u) % lines) : 0u;
          const unsigned char *src = xbase + (size_t)c0 * sizeof(VT);
          unsigned char *dst = reinterpret_cast<unsigned char *>(xs);
          bulk_g2s(dst + rot, src + rot, bulk - rot, &full[s]);
          if (rot) bulk_g2s(dst, src, rot, &full[s]);
        }
        bulk_g2s(S.m(s), A.meta + 16 * (size_t)(unsigned)g.x, mb, &full[s]);
        if (vb) bulk_g2s(S.v(s), vals + (size_t)(unsigned)g.y, vb, &full[s]);
      }
      issued = p + 1;
    }
  }
  // copies still in flight complete before the block leaves
  if (lane == 0)
    for (int p = max(0, issued - A.S); p < issued; ++p)
      if (!mbar_wait(&full[p % A.S], (unsigned)((p / A.S) & 1), A.polls)) atomicExch(A.err, 1);
}

// Consumer warp w: chunks w, w + NC, ... of every panel, as each stage
// fills, two chunks at a time (their rows differ: a row has one segment per
// panel).  The consumer warps meet at a named barrier after each panel, so
// panel p's updates of a row precede panel p + 1's, and one thread then
// releases the stage.  A wait that runs out sets the error flag and the warp
// skips the remaining work but keeps meeting the barrier, so no warp is left
// waiting.
template <class VT>
__device__ void panel_consume(const PanelView &A, const PanelSmem<VT> &S, unsigned long long *full,
                              unsigned long long *empty, int w, int lane, int d) {
  bool bad = false;
  for (int p = 0; p < A.P; ++p) {
    const int s = p % A.S;
    if (!bad && !mbar_wait(&full[s], (unsigned)((p / A.S) & 1), A.polls)) {
      if (lane == 0) atomicExch(A.err, 1);
      bad = true;
    }
    if (!bad) {
      const unsigned char *m = S.m(s);
      const unsigned nch = reinterpret_cast<const unsigned *>(m)[0];
      const unsigned *coff = reinterpret_cast<const unsigned *>(m + 16);
      const unsigned short *rid = reinterpret_cast<const unsigned short *>(m + 16 + align16(4 * (size_t)(nch + 1)));
      const unsigned short *col = rid + align16(64 * (size_t)nch) / 2;
      const VT *xv = S.x(s) + d;
      const VT *vv = S.v(s);
      for (unsigned c = w; c < nch; c += 2 * kConsumerWarps) {
        const unsigned c2 = c + kConsumerWarps;
        const bool has2 = c2 < nch;
        const unsigned o1 = coff[c], w1 = (coff[c + 1] - o1) >> 5;
        const unsigned o2 = has2 ? coff[c2] : 0, w2 = has2 ? (coff[c2 + 1] - o2) >> 5 : 0;
        const unsigned short r1 = rid[32 * c + lane];
        const unsigned short r2 = has2 ? rid[32 * c2 + lane] : (unsigned short)0xffff;
        VT a1 = (r1 != 0xffff) ? S.acc[r1] : (VT)0;
        VT a2 = (r2 != 0xffff) ? S.acc[r2] : (VT)0;
        const unsigned wm = w1 > w2 ? w1 : w2;
        for (unsigned j = 0; j < wm; ++j) {
          if (j < w1) {
            const unsigned e = o1 + 32 * j + lane;
            a1 = pmadd(a1, vv[e], xv[col[e]]);
          }
          if (j < w2) {
            const unsigned e = o2 + 32 * j + lane;
            a2 = pmadd(a2, vv[e], xv[col[e]]);
          }
        }
        if (r1 != 0xffff) S.acc[r1] = a1;
        if (r2 != 0xffff) S.acc[r2] = a2;
      }
    }
    asm volatile("bar.sync 1, %0;" ::"n"(32 * kConsumerWarps) : "memory");
    if (w == 0 && lane == 0) mbar_arrive(&empty[s]);
  }
}

// acc[lr] = (row of local index lr) x for the rows of CTA rb.  Ends with a
// block barrier; acc is then complete.
template <class VT>
__device__ __forceinline__ void panel_rows(const PanelView &A, const PanelSmem<VT> &S, unsigned long long *full,
                                           unsigned long long *empty, int rb, const VT *x, const VT *vals) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < A.R; i += blockDim.x) S.acc[i] = (VT)0;
  if (tid == 0) {
    for (int s = 0; s < A.S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (warp == kConsumerWarps) {
    panel_produce<VT>(A, S, full, empty, rb, x, vals, lane);
  } else {
    panel_consume<VT>(A, S, full, empty, warp, lane, (int)((reinterpret_cast<uintptr_t>(x) & 15) / sizeof(VT)));
  }
  __syncthreads();
}

// FP64 degree step with the k_cheb epilogue (same rounded operations).
template <bool FIRST, bool EPI>
__global__ void __launch_bounds__(kPanelThreads, 1)
    k_cheb_panel(PanelView A, const double *__restrict__ vals, const double *vk, const double *vkm1, double *out,
                 double *__restrict__ y, double t, double ncc, double s, double mu0, const double *__restrict__ zold,
                 double nbeta, const double *__restrict__ dotv, double *part, unsigned int *ctr, double *dot_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full[kMaxStages], empty[kMaxStages];
  __shared__ double sh[kPanelThreads / 32];
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const PanelSmem<double> S(smem_raw, A);
  const int rb = blockIdx.x;
  panel_rows<double>(A, S, full, empty, rb, vk, vals);
  double dsum = 0.0;
  for (int i = threadIdx.x; i < A.R; i += blockDim.x) {
    const int r = panel_row(A, rb, i);
    if (r >= A.n) continue;
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
    k_mf_panel(PanelView A, const VT *__restrict__ vals, const VT *vk, const VT *vkm1, VT *out, VT *__restrict__ y,
               const VT *__restrict__ coef) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full[kMaxStages], empty[kMaxStages];
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const PanelSmem<VT> S(smem_raw, A);
  const int rb = blockIdx.x;
  panel_rows<VT>(A, S, full, empty, rb, vk, vals);
  const VT c0 = __ldg(coef), c1 = __ldg(coef + 1), c2 = __ldg(coef + 2), c3 = __ldg(coef + 3);
  for (int i = threadIdx.x; i < A.R; i += blockDim.x) {
    const int r = panel_row(A, rb, i);
    if (r >= A.n) continue;
    const VT xr = vk[r];
    VT w = pmul(c0, padd(S.acc[i], pmul(c1, xr)));
    if (!FIRST) w = padd(w, -vkm1[r]);
    out[r] = w;
    if (c3 != (VT)0) y[r] = padd(y[r], pmul(c2, w));
  }
}

// ---------------------------------------------------------------------------
// Host build
// ---------------------------------------------------------------------------
struct Seg {
  int len, row, start;
};

// Builds the panel layout for RB CTAs (interleaved 32-row chunks, R local
// rows each) and panels of W columns into host arrays; mcap / ecap: the
// largest group's meta bytes and entries.
bool build_host(int n, const std::vector<int> &ia, const std::vector<int> &ja, const std::vector<double> &a, int RB,
                int R, int W, std::vector<int4> &gtab, std::vector<unsigned char> &meta, std::vector<double> &vals,
                size_t &mcap, int &ecap) {
  const int P = (n + W - 1) / W;
  gtab.assign((size_t)RB * P, int4{0, 0, 0, 0});
  meta.clear();
  vals.clear();
  mcap = 16;
  ecap = 0;
  std::vector<std::vector<Seg>> lists((size_t)P);
  const int nchunks = (n + 31) / 32;
  for (int rb = 0; rb < RB; ++rb) {
    for (auto &l : lists) l.clear();
    for (int c = rb, cl = 0; c < nchunks; c += RB, ++cl) {
      for (int r = 32 * c; r < std::min(n, 32 * c + 32); ++r) {
        const int lr = 32 * cl + (r & 31);
        int j = ia[r];
        const int e = ia[r + 1];
        while (j < e) {
          const int p = ja[j] / W;
          int k = j + 1;
          while (k < e && ja[k] / W == p) ++k;
          lists[p].push_back(Seg{k - j, lr, j});
          j = k;
        }
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
      const size_t mb = meta_bytes(nch, E);
      while (meta.size() % 16) meta.push_back(0);
      while (vals.size() % 4) vals.push_back(0.0);
      if (meta.size() / 16 > 0x7fffffffULL || vals.size() > 0x7fffffffULL) return false;
      gtab[(size_t)rb * P + p] = int4{(int)(meta.size() / 16), (int)vals.size(), nch, E};
      const size_t mbase = meta.size();
      meta.resize(mbase + mb, 0);
      const size_t vbase = vals.size();
      vals.resize(vbase + (size_t)E, 0.0);
      unsigned char *mp = meta.data() + mbase;
      const unsigned hdr[4] = {(unsigned)nch, (unsigned)E, 0u, 0u};
      memcpy(mp, hdr, 16);
      memcpy(mp + 16, coff.data(), 4 * (size_t)(nch + 1));
      unsigned short *rid = reinterpret_cast<unsigned short *>(mp + 16 + align16(4 * (size_t)(nch + 1)));
      unsigned short *col = rid + align16(64 * (size_t)nch) / 2;
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
  return PanelView{M->n,    P->R,    P->W,    P->P,    P->S,    P->RB, P->gtab, P->meta, P->mcap, P->vcap,
                   P->xcap, (int *)(counters() + 10), kPanelWaitPolls};
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
int g_panel_enabled = 0;  // off by default: measured slower than the SELL kernels (see the header)
int g_panel_max_width = 16384;

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
  // one CTA per SM (one wave), each with at most 65504 local rows
  const int nchunks = (n + 31) / 32;
  int RB = std::max(1, std::min(sm_count(), nchunks));
  while (32LL * ((nchunks + RB - 1) / RB) > 65504) ++RB;
  const int R = 32 * ((nchunks + RB - 1) / RB);
  std::vector<int4> gtab;
  std::vector<unsigned char> meta;
  std::vector<double> vals;
  size_t mcap = 0;
  int ecap = 0;
  int W = 0, S = 0;
  unsigned xcap = 0, vcap = 0;
  // the widest panel whose ring still holds at least 4 stages
  for (int w : {16384, 12288, 8192, 6144, 4096, 3072, 2048, 1536, 1024, 512}) {
    if (w > g_panel_max_width) continue;
    const unsigned xc = (unsigned)align16(vb * (size_t)(w + 16 / vb));
    if (align16(vb * R) + 4 * (size_t)xc > kSmemLimit) continue;
    if (!build_host(n, ia, ja, a, RB, R, w, gtab, meta, vals, mcap, ecap)) return 0;
    const unsigned vc = (unsigned)align16(vb * (size_t)ecap);
    const size_t stage = (size_t)xc + mcap + vc;
    const int s = (int)std::min<size_t>(kMaxStages, (kSmemLimit - align16(vb * R)) / stage);
    if (s >= 4 || (w == 512 && s >= 2)) {
      W = w;
      S = s;
      xcap = xc;
      vcap = vc;
      break;
    }
  }
  if (!W) return 0;  // no layout fits: the SELL kernels stay in use
  evslcu_panels *P = new evslcu_panels();
  P->fp32 = fp32;
  P->R = R;
  P->W = W;
  P->P = (n + W - 1) / W;
  P->RB = RB;
  P->S = S;
  P->mcap = (unsigned)mcap;
  P->vcap = vcap;
  P->xcap = xcap;
  P->smem = fp32 ? panel_smem_bytes<float>(R, S, xcap, P->mcap, vcap)
                 : panel_smem_bytes<double>(R, S, xcap, P->mcap, vcap);
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

int evslcu_set_panels(int on, int min_rows, int max_width) {
  evslcu::g_panel_enabled = on ? 1 : 0;
  if (min_rows > 0) evslcu::g_panel_min_rows = min_rows;
  if (max_width > 0) evslcu::g_panel_max_width = std::max(512, max_width);
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
