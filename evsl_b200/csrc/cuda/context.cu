// Library context: stream, scratch for reductions, memory and error helpers.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <atomic>

#include <algorithm>

#include "common.cuh"
#include "sparse_types.cuh"

namespace evslcu {

namespace {
struct Context {
  bool ready = false;
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  double *partials = nullptr;
  unsigned int *counters = nullptr;
  double *scalars = nullptr;
  unsigned int *barrier = nullptr;
};
Context g_ctx;
char g_err[512] = "";
std::atomic<uint64_t> g_launches{0};
}  // namespace

cudaStream_t stream() { return g_ctx.stream; }
double *partials() { return g_ctx.partials; }
unsigned int *counters() { return g_ctx.counters; }
double *dev_scratch_scalars() { return g_ctx.scalars; }
unsigned int *barrier_area() { return g_ctx.barrier; }
int sm_count() { return g_ctx.sms; }
int lib_device() { return g_ctx.device; }
void count_launch(uint64_t k) { g_launches += k; }

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return 0;
}

}  // namespace evslcu

using namespace evslcu;

extern "C" {

int evslcu_initialized(void) { return g_ctx.ready ? 1 : 0; }

const char *evslcu_errstr(void) { return g_err; }

void evslcu_set_error(int code, const char *msg) { fail(code, "%s", msg ? msg : ""); }

uint64_t evslcu_launch_count(void) { return g_launches.load(); }

int evslcu_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// Device memory of the library comes from a stream-ordered pool on the
// library stream (cudaMallocFromPoolAsync / cudaFreeAsync): a free does not
// wait for the device -- work already queued on the stream that still uses
// the memory runs first -- and freed memory is reused by later allocations
// without a trip to the driver.  Freed memory stays in the pool (up to
// kPoolKeep bytes) for later allocations; EVSLFinish trims it.  The pool outlives EVSLFinish, so that
// buffers handed to the caller (eigenvectors) can be freed afterwards.
static cudaMemPool_t g_pool = nullptr;
static int g_pool_dev = -1;
constexpr unsigned long long kPoolKeep = ~0ull;  // keep freed memory for reuse until EVSLFinish

static void pool_init(int dev) {
  if (g_pool && g_pool_dev == dev) return;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t p = nullptr;
  if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
    cudaGetLastError();  // plain cudaMalloc / cudaFree then
    return;
  }
  unsigned long long keep = kPoolKeep;
  cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
  g_pool = p;
  g_pool_dev = dev;
}

static bool pool_ready() { return g_ctx.ready && g_pool && g_pool_dev == g_ctx.device; }

int evslcu_init(void) {
  if (g_ctx.ready) return 0;
  if (evslcu_device_count() < 1) return fail(EVSLCU_ERR_NODEV, "no CUDA device is visible");
  EVSLCU_CUDA(cudaGetDevice(&g_ctx.device));
  cudaDeviceProp prop;
  EVSLCU_CUDA(cudaGetDeviceProperties(&prop, g_ctx.device));
  if (prop.major < 10)
    return fail(EVSLCU_ERR_NODEV, "device %s is sm_%d%d; this library is built for sm_100a", prop.name,
                prop.major, prop.minor);
  g_ctx.sms = prop.multiProcessorCount;
  // Blocking w.r.t. the legacy default stream, so user matvec callbacks that
  // launch on stream 0 are ordered with the library's work.
  EVSLCU_CUDA(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamDefault));
  EVSLCU_CUDA(cudaMalloc(&g_ctx.partials, sizeof(double) * (size_t)kMaxPartials * 2));
  EVSLCU_CUDA(cudaMalloc(&g_ctx.counters, sizeof(unsigned int) * kNumCounters));
  EVSLCU_CUDA(cudaMemset(g_ctx.counters, 0, sizeof(unsigned int) * kNumCounters));
  EVSLCU_CUDA(cudaMalloc(&g_ctx.scalars, sizeof(double) * 64));
  EVSLCU_CUDA(cudaMalloc(&g_ctx.barrier, sizeof(unsigned int) * kBarrierWords));
  EVSLCU_CUDA(cudaMemset(g_ctx.barrier, 0, sizeof(unsigned int) * kBarrierWords));
  EVSLCU_CUDA(cudaMemset(g_ctx.scalars, 0, sizeof(double) * 64));
  pool_init(g_ctx.device);
  g_ctx.ready = true;
  return 0;
}

// ---------------------------------------------------------------------------
// L2 residency of the stored matrix: an access-policy window on the library
// stream marks the SELL arrays persisting, with the context's persisting L2
// set-aside sized to them (bounded by the device maximum).  The set-aside is
// a limit of this context and is released when the window is cleared.
// ---------------------------------------------------------------------------
static const void *g_l2_owner = nullptr;

extern "C" int evslcu_mat_l2_persist(const evslcu_mat *A, int on) {
  if (!g_ctx.ready || !A) return 0;
  if (!on) {
    if (g_l2_owner != (const void *)A) return 0;
    cudaStreamAttrValue v = {};
    v.accessPolicyWindow.base_ptr = nullptr;
    v.accessPolicyWindow.num_bytes = 0;
    cudaStreamSetAttribute(g_ctx.stream, cudaStreamAttributeAccessPolicyWindow, &v);
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    g_l2_owner = nullptr;
    cudaGetLastError();
    return 0;
  }
  if (!A->sell_block || !A->sell_bytes) return 0;
  int max_persist = 0, max_window = 0;
  cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, g_ctx.device);
  cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, g_ctx.device);
  if (max_persist <= 0 || max_window <= 0) return 0;
  const size_t window = std::min(A->sell_bytes, (size_t)max_window);
  const size_t setaside = std::min(window, (size_t)max_persist);
  EVSLCU_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, setaside));
  cudaStreamAttrValue v = {};
  v.accessPolicyWindow.base_ptr = A->sell_block;
  v.accessPolicyWindow.num_bytes = window;
  v.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)setaside / (double)window);
  v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  EVSLCU_CUDA(cudaStreamSetAttribute(g_ctx.stream, cudaStreamAttributeAccessPolicyWindow, &v));
  g_l2_owner = A;
  return 0;
}

int evslcu_finish(void) {
  if (!g_ctx.ready) return 0;
  cudaStreamSynchronize(g_ctx.stream);
  if (g_l2_owner) {
    cudaStreamAttrValue v = {};
    cudaStreamSetAttribute(g_ctx.stream, cudaStreamAttributeAccessPolicyWindow, &v);
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    g_l2_owner = nullptr;
    cudaGetLastError();
  }
  evslcu_kpm_release();
  evslcu_trid_release();
  evslcu_lz_release();
  evslcu_gemm_release();
  cudaFree(g_ctx.partials);
  cudaFree(g_ctx.counters);
  cudaFree(g_ctx.scalars);
  cudaFree(g_ctx.barrier);
  cudaStreamSynchronize(g_ctx.stream);
  if (g_pool) cudaMemPoolTrimTo(g_pool, 0);
  cudaStreamDestroy(g_ctx.stream);
  g_ctx = Context();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(EVSLCU_ERR_CUDA, "pending CUDA error at finish: %s", cudaGetErrorString(e));
  return 0;
}

int evslcu_sync(void) {
  if (!g_ctx.ready) return fail(EVSLCU_ERR_STATE, "library not started (EVSLStart)");
  EVSLCU_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return 0;
}

int evslcu_device_name(int dev, char *buf, int len, int *sm, size_t *mem) {
  cudaDeviceProp prop;
  EVSLCU_CUDA(cudaGetDeviceProperties(&prop, dev));
  if (buf && len > 0) snprintf(buf, (size_t)len, "%s", prop.name);
  if (sm) *sm = prop.multiProcessorCount;
  if (mem) *mem = prop.totalGlobalMem;
  return 0;
}

int evslcu_last_cuda_error(char *buf, int len) {
  cudaError_t e = cudaGetLastError();
  if (buf && len > 0) snprintf(buf, (size_t)len, "%s", e == cudaSuccess ? "" : cudaGetErrorString(e));
  return e == cudaSuccess ? 0 : EVSLCU_ERR_CUDA;
}

void *evslcu_malloc(size_t nbytes) {
  void *p = nullptr;
  if (nbytes == 0) nbytes = 1;
  cudaError_t e = pool_ready() ? cudaMallocFromPoolAsync(&p, nbytes, g_pool, g_ctx.stream) : cudaMalloc(&p, nbytes);
  if (e == cudaErrorMemoryAllocation && pool_ready()) {
    // the pool keeps freed blocks; blocks of other sizes (an earlier
    // solve's basis) may hold the memory this request needs: return them
    // to the device once the stream has finished with them, then retry
    cudaGetLastError();
    cudaStreamSynchronize(g_ctx.stream);
    cudaMemPoolTrimTo(g_pool, 0);
    e = cudaMallocFromPoolAsync(&p, nbytes, g_pool, g_ctx.stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(EVSLCU_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", nbytes, cudaGetErrorString(e));
    return nullptr;
  }
  return p;
}

int evslcu_free(void *p) {
  if (!p) return 0;
  // Memory may still be in use by work queued on the library stream: a
  // stream-ordered free runs after it; otherwise wait for the stream.
  if (pool_ready()) {
    EVSLCU_CUDA(cudaFreeAsync(p, g_ctx.stream));
    return 0;
  }
  if (g_ctx.ready) cudaStreamSynchronize(g_ctx.stream);
  EVSLCU_CUDA(cudaFree(p));
  return 0;
}

int evslcu_h2d(void *dst, const void *src, size_t nbytes) {
  if (!nbytes) return 0;
  EVSLCU_CUDA(cudaMemcpyAsync(dst, src, nbytes, cudaMemcpyHostToDevice, g_ctx.stream));
  EVSLCU_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return 0;
}

int evslcu_h2d_async(void *dst, const void *src, size_t nbytes) {
  if (!nbytes) return 0;
  EVSLCU_CUDA(cudaMemcpyAsync(dst, src, nbytes, cudaMemcpyHostToDevice, g_ctx.stream));
  return 0;
}

int evslcu_d2h(void *dst, const void *src, size_t nbytes) {
  if (!nbytes) return 0;
  EVSLCU_CUDA(cudaMemcpyAsync(dst, src, nbytes, cudaMemcpyDeviceToHost, g_ctx.stream));
  EVSLCU_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return 0;
}

int evslcu_d2d(void *dst, const void *src, size_t nbytes) {
  if (!nbytes) return 0;
  EVSLCU_CUDA(cudaMemcpyAsync(dst, src, nbytes, cudaMemcpyDeviceToDevice, g_ctx.stream));
  return 0;
}

int evslcu_memset(void *p, int v, size_t nbytes) {
  if (!nbytes) return 0;
  EVSLCU_CUDA(cudaMemsetAsync(p, v, nbytes, g_ctx.stream));
  return 0;
}

int evslcu_get_scalars(const double *dev, double *host, int count) {
  return evslcu_d2h(host, dev, sizeof(double) * (size_t)count);
}

struct evslcu_timer {
  cudaEvent_t a, b;
};

evslcu_timer *evslcu_timer_start(void) {
  evslcu_timer *t = new evslcu_timer;
  cudaEventCreate(&t->a);
  cudaEventCreate(&t->b);
  cudaEventRecord(t->a, g_ctx.stream);
  return t;
}

struct evslcu_marks {
  int count;
  cudaEvent_t *ev;
};

evslcu_marks *evslcu_marks_create(int count) {
  if (count <= 0) return nullptr;
  evslcu_marks *m = new evslcu_marks;
  m->count = count;
  m->ev = new cudaEvent_t[count];
  for (int i = 0; i < count; ++i) cudaEventCreate(&m->ev[i]);
  return m;
}

void evslcu_marks_record(evslcu_marks *m, int i) {
  if (m && i >= 0 && i < m->count) cudaEventRecord(m->ev[i], g_ctx.stream);
}

double evslcu_marks_elapsed(evslcu_marks *m, int i, int j) {
  if (!m || i < 0 || j < 0 || i >= m->count || j >= m->count) return 0.0;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, m->ev[i], m->ev[j]) != cudaSuccess) {
    cudaGetLastError();
    return 0.0;
  }
  return 1e-3 * (double)ms;
}

void evslcu_marks_destroy(evslcu_marks *m) {
  if (!m) return;
  for (int i = 0; i < m->count; ++i) cudaEventDestroy(m->ev[i]);
  delete[] m->ev;
  delete m;
}

double evslcu_timer_stop(evslcu_timer *t) {
  if (!t) return 0.0;
  float ms = 0.f;
  cudaEventRecord(t->b, g_ctx.stream);
  cudaEventSynchronize(t->b);
  cudaEventElapsedTime(&ms, t->a, t->b);
  cudaEventDestroy(t->a);
  cudaEventDestroy(t->b);
  delete t;
  return 1e-3 * (double)ms;
}

}  // extern "C"
