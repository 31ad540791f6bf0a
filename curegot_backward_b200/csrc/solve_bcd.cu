// Single-problem BCD driver and the C-ABI entry points for it.
//
// Follows cuda_sinkhorn_bcd (reference src/sinkhorn_bcd_kernel.cu:429-634)
// with input and output on the device.  The loop runs on the device: the
// host queues chunks of iterations (one row pass + one column pass each)
// and reads the 48-byte state once per chunk; passes after convergence exit
// immediately.  No host synchronisation happens inside an iteration.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "bcd.cuh"
#include "task.cuh"
#include "workspace.cuh"

namespace cg {

namespace {
thread_local std::string g_last_error;
}

namespace {
std::atomic<long long> g_launches{0};
}

void count_launch(long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

namespace {
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};
}  // namespace

int library_pool(int device, cudaMemPool_t* out) {
  if (device < 0 || device >= kMaxPoolDevices) {
    set_last_error("memory pool: device ordinal above 63", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[device]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    CG_TRY_CUDA(cudaMemPoolCreate(&pool, &props));
    // keep freed blocks mapped: serving reuses the same sizes over and over
    unsigned long long keep = ~0ull;
    CG_TRY_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[device] = pool;
  }
  *out = g_pools[device];
  return CG_OK;
}

int pool_alloc_async(void** ptr, size_t bytes, cudaStream_t stream) {
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  cudaMemPool_t pool = nullptr;
  CG_TRY(library_pool(dev, &pool));
  const cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, pool, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return (e == cudaErrorMemoryAllocation) ? CG_ERR_OOM : CG_ERR_CUDA;
  }
  return CG_OK;
}

namespace {
thread_local bool t_wait_yield = false;
}

void host_wait_yield(bool on) { t_wait_yield = on; }

int host_wait(cudaStream_t st) {
  if (!t_wait_yield) {
    CG_TRY_CUDA(cudaStreamSynchronize(st));
    return CG_OK;
  }
  struct Event {
    cudaEvent_t e = nullptr;
    int dev = -1;
    ~Event() {
      if (e) cudaEventDestroy(e);
    }
  };
  thread_local Event ev;
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  if (ev.e && ev.dev != dev) {
    cudaEventDestroy(ev.e);
    ev.e = nullptr;
  }
  if (!ev.e) {
    CG_TRY_CUDA(cudaEventCreateWithFlags(&ev.e, cudaEventDisableTiming));
    ev.dev = dev;
  }
  CG_TRY_CUDA(cudaEventRecord(ev.e, st));
  while (true) {
    const cudaError_t q = cudaEventQuery(ev.e);
    if (q == cudaSuccess) return CG_OK;
    if (q != cudaErrorNotReady) CG_TRY_CUDA(q);
    std::this_thread::yield();
  }
}

int read_device_spans(const ReadSpan* spans, int count, cudaStream_t st) {
  struct Pinned {
    void* p = nullptr;
    ~Pinned() {
      if (p) cudaFreeHost(p);
    }
  };
  thread_local Pinned buf;
  constexpr size_t kBytes = 4096;
  size_t total = 0;
  for (int k = 0; k < count; ++k) total += spans[k].bytes;
  if (total > kBytes) {
    set_last_error("read_device: more than 4096 bytes", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  if (!buf.p) CG_TRY_CUDA(cudaHostAlloc(&buf.p, kBytes, cudaHostAllocDefault));
  char* pin = static_cast<char*>(buf.p);
  size_t off = 0;
  for (int k = 0; k < count; ++k) {
    if (spans[k].bytes)
      CG_TRY_CUDA(cudaMemcpyAsync(pin + off, spans[k].dev, spans[k].bytes, cudaMemcpyDeviceToHost, st));
    off += spans[k].bytes;
  }
  CG_TRY(host_wait(st));
  off = 0;
  for (int k = 0; k < count; ++k) {
    if (spans[k].bytes) std::memcpy(spans[k].host, pin + off, spans[k].bytes);
    off += spans[k].bytes;
  }
  return CG_OK;
}

int read_device_bulk(void* host, const void* dev, size_t bytes, cudaStream_t st) {
  struct Pinned {
    void* p = nullptr;
    size_t cap = 0;
    ~Pinned() {
      if (p) cudaFreeHost(p);
    }
  };
  thread_local Pinned buf;
  if (bytes == 0) return CG_OK;
  if (bytes > buf.cap) {
    if (buf.p) cudaFreeHost(buf.p);
    buf.p = nullptr;
    buf.cap = 0;
    const size_t cap = std::max(bytes, (size_t)1 << 20);
    CG_TRY_CUDA(cudaHostAlloc(&buf.p, cap, cudaHostAllocDefault));
    buf.cap = cap;
  }
  CG_TRY_CUDA(cudaMemcpyAsync(buf.p, dev, bytes, cudaMemcpyDeviceToHost, st));
  CG_TRY(host_wait(st));
  std::memcpy(host, buf.p, bytes);
  return CG_OK;
}

// Pool of (pinned buffer, event) pairs for resumable solves.
namespace {
struct IoSlot {
  void* pinned;
  cudaEvent_t ev;
  int dev;
  void* bulk;
  size_t bulk_cap;
};
std::mutex g_io_mu;
std::vector<IoSlot> g_io_free;
}  // namespace

int TaskIO::init(cudaStream_t s) {
  st = s;
  err = CG_OK;
  posted = false;
  count = 0;
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(g_io_mu);
    for (size_t k = 0; k < g_io_free.size(); ++k)
      if (g_io_free[k].dev == dev) {
        pinned = g_io_free[k].pinned;
        ev = g_io_free[k].ev;
        bulk = g_io_free[k].bulk;
        bulk_cap = g_io_free[k].bulk_cap;
        g_io_free.erase(g_io_free.begin() + k);
        return CG_OK;
      }
  }
  CG_TRY_CUDA(cudaHostAlloc(&pinned, kTaskPinnedBytes, cudaHostAllocDefault));
  const cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cudaFreeHost(pinned);
    pinned = nullptr;
    CG_TRY_CUDA(e);
  }
  return CG_OK;
}

void TaskIO::release() {
  if (!pinned) return;
  int dev = 0;
  cudaGetDevice(&dev);
  if (job_posted) {  // a task destroyed while its job runs: let the job finish
    job.wait();
    job_posted = false;
  }
  std::lock_guard<std::mutex> lk(g_io_mu);
  g_io_free.push_back({pinned, ev, dev, bulk, bulk_cap});
  pinned = nullptr;
  ev = nullptr;
  bulk = nullptr;
  bulk_cap = 0;
}

int TaskIO::wait() {
  if (job_posted) {
    if (!t_wait_yield) {
      job.wait();
    } else {
      while (job.wait_for(std::chrono::seconds(0)) != std::future_status::ready)
        std::this_thread::yield();
    }
    return CG_OK;
  }
  if (!posted) return CG_OK;
  if (!t_wait_yield) {
    CG_TRY_CUDA(cudaEventSynchronize(ev));
    return CG_OK;
  }
  while (true) {
    const cudaError_t q = cudaEventQuery(ev);
    if (q == cudaSuccess) return CG_OK;
    if (q != cudaErrorNotReady) CG_TRY_CUDA(q);
    if (t_wait_yield) std::this_thread::yield();
  }
}

TaskIO::Await TaskIO::read_spans_bulk(const ReadSpan* sp, int cnt) {
  size_t total = 0;
  for (int k = 0; k < cnt; ++k) total += sp[k].bytes;
  if (cnt > kTaskMaxSpans) {
    set_last_error("task read: too many spans", __FILE__, __LINE__);
    err = CG_ERR_INVALID_ARG;
    return Await{this};
  }
  if (total > bulk_cap) {  // no copy into bulk is pending: the task waits on each read
    if (bulk) cudaFreeHost(bulk);
    bulk = nullptr;
    bulk_cap = 0;
    const size_t cap = std::max<size_t>(total + total / 2, size_t(1) << 16);
    const cudaError_t e = cudaHostAlloc(&bulk, cap, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      bulk = nullptr;
      set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
      err = status_from_cuda(e);
      return Await{this};
    }
    bulk_cap = cap;
  }
  use_bulk = true;
  return post_reads(sp, cnt, static_cast<char*>(bulk));
}

TaskIO::Await TaskIO::read_spans(const ReadSpan* sp, int cnt) {
  size_t total = 0;
  for (int k = 0; k < cnt; ++k) total += sp[k].bytes;
  if (cnt > kTaskMaxSpans || total > kTaskPinnedBytes) {
    set_last_error("task read: too many bytes or spans", __FILE__, __LINE__);
    err = CG_ERR_INVALID_ARG;
    return Await{this};
  }
  use_bulk = false;
  return post_reads(sp, cnt, static_cast<char*>(pinned));
}

TaskIO::Await TaskIO::post_reads(const ReadSpan* sp, int cnt, char* pin) {
  count = cnt;
  size_t off = 0;
  for (int k = 0; k < cnt; ++k) {
    spans[k] = sp[k];
    if (sp[k].bytes) {
      const cudaError_t e =
          cudaMemcpyAsync(pin + off, sp[k].dev, sp[k].bytes, cudaMemcpyDeviceToHost, st);
      if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
        err = status_from_cuda(e);
        return Await{this};
      }
    }
    off += sp[k].bytes;
  }
  const cudaError_t e = cudaEventRecord(ev, st);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    err = status_from_cuda(e);
    return Await{this};
  }
  posted = true;
  return Await{this};
}

int read_device(void* host1, const void* dev1, size_t bytes1, cudaStream_t st, void* host2,
                const void* dev2, size_t bytes2) {
  const ReadSpan spans[2] = {{host1, dev1, bytes1}, {host2, dev2, bytes2}};
  return read_device_spans(spans, 2, st);
}

void set_last_error(const char* msg, const char* file, int line) {
  g_last_error = std::string(msg) + " (" + file + ":" + std::to_string(line) + ")";
}

__global__ void bcd_init_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                const double* __restrict__ x0, int n, int m, double s2,
                                double* __restrict__ loga, double* __restrict__ logb,
                                double* __restrict__ alpha0, double* __restrict__ beta0,
                                double* __restrict__ alphas0, double* __restrict__ betas0,
                                unsigned int* counters, int ncounters, BcdState* st,
                                int max_iter, double tol, int fast) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int i = tid; i < n; i += stride) {
    loga[i] = log(a[i]);
    const double v = x0 ? x0[i] : 0.0;
    alpha0[i] = v;
    alphas0[i] = v * s2;
  }
  for (int j = tid; j < m; j += stride) {
    logb[j] = log(b[j]);
    const double v = x0 ? x0[n + j] : 0.0;
    beta0[j] = v;
    betas0[j] = v * s2;
  }
  for (int q = tid; q < ncounters; q += stride) counters[q] = 0u;
  if (tid == 0) {
    st->iter = 0;
    st->phase = 1;
    st->check_pending = 0;
    st->done = (max_iter <= 0) ? 1 : 0;
    st->niter = 0;
    st->max_iter = max_iter;
    st->fast = fast;
    st->stall = 0;
    st->tol = tol;
    st->last_err = 0.0;
    st->best_est = INFINITY;
    st->stat_a[0] = st->stat_a[1] = st->stat_a[2] = 0.0;
    st->fast_iters = 0;
    st->nonfinite = 0;
    st->error = 0;
    st->drift_a = st->drift_b = INFINITY;
    st->acc_a = st->acc_b = 0ull;
    st->split_bad_a = st->split_bad_b = 0;
  }
}

// The returned iterate lives in buffer (niter & 1); resolved on the device.
template <typename TM>
__global__ void plan_from_state_kernel(const TM* __restrict__ M, const BcdState* st,
                                       const BcdProb* p, double* __restrict__ P) {
  const int k = st->niter & 1;
  const double* __restrict__ al = p->alpha[k];
  const double* __restrict__ be = p->beta[k];
  const int n = p->n, m = p->m;
  const double inv_eta = 1.0 / p->eta;
  const size_t total = (size_t)n * m;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / m);
    const int j = (int)(idx - (size_t)i * m);
    P[idx] = exp((al[i] + be[j] - ld1(M + idx)) * inv_eta);
  }
}

__global__ void dual_from_state_kernel(const BcdState* st, const BcdProb* p, double* dual) {
  const int k = st->niter & 1;
  const double* al = p->alpha[k];
  const double* be = p->beta[k];
  const int n = p->n, m = p->m;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x)
    dual[i] = (i < n) ? al[i] : be[i - n];
}

// A stop-test value became NaN or Inf: M, a, b or x0 holds a non-finite
// value (or log(a_i), log(b_j) of a zero marginal met an infinite cost).  The
// reference keeps iterating to max_iter on NaN; here the solve stops at the
// first non-finite test and reports it.
// A bounded wait of a pass kernel's staging ring gave up (the state's error
// flag); the solve stopped there.
static int bcd_timeout() {
  set_last_error("cg_bcd: a staging wait of a pass kernel timed out", __FILE__, __LINE__);
  return CG_ERR_TIMEOUT;
}

static int bcd_nonfinite() {
  set_last_error("cg_bcd: non-finite stopping-test value (non-finite M, a, b or x0)", __FILE__,
                 __LINE__);
  return CG_ERR_NONFINITE;
}

// Whole solve in one cluster-resident launch (problems up to ~3 MB of M).
template <typename TM>
int bcd_solve_cluster(int C, const TM* M, const double* a, const double* b, double* Pout,
                      double reg, int max_iter, double tol, int n, int m, int* niter,
                      const double* x0, double* dual, cudaStream_t stream) {
  Workspace ws(stream);
  const size_t o_st = ws.reserve<BcdState>(1), o_p = ws.reserve<ClusterProb>(1);
  const bool tmp_dual = (!dual && Pout);
  const size_t o_d = ws.reserve<double>(tmp_dual ? (size_t)(n + m) : 1);
  CG_TRY(ws.allocate());
  ClusterProb hp{};
  hp.M = M;
  hp.a = a;
  hp.b = b;
  hp.x0 = x0;
  hp.dual = dual ? dual : (tmp_dual ? ws.at<double>(o_d) : nullptr);
  hp.st = ws.at<BcdState>(o_st);
  hp.n = n;
  hp.m = m;
  hp.max_iter = max_iter;
  hp.eta = reg;
  hp.s2 = kLog2e / reg;
  hp.tol = tol;
  ClusterProb* dp = ws.at<ClusterProb>(o_p);
  CG_TRY_CUDA(cudaMemcpyAsync(dp, &hp, sizeof(ClusterProb), cudaMemcpyHostToDevice, stream));
  CG_TRY(launch_bcd_cluster<TM>(dp, 1, C, stream));
  BcdState hs{};
  CG_TRY(read_device(&hs, hp.st, sizeof(BcdState), stream));
  *niter = hs.niter;
  if (hs.nonfinite) return bcd_nonfinite();
  if (Pout) launch_plan<TM>(M, hp.dual, hp.dual + n, Pout, 1.0 / reg, n, m, stream);
  CG_TRY_CUDA(cudaGetLastError());
  ws.release();
  return CG_OK;
}

template <typename TM>
int bcd_solve(const TM* M, const double* a, const double* b, double* Pout, double reg,
              int max_iter, double tol, int n, int m, int* niter, const double* x0,
              double* dual, cudaStream_t stream) {
  if (!M || !a || !b || !niter || n <= 0 || m <= 0 || !(reg > 0.0) || !std::isfinite(reg)) {
    set_last_error("cg_bcd: invalid argument", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  if (const int C = bcd_cluster_eligible<TM>(n, m))
    return bcd_solve_cluster<TM>(C, M, a, b, Pout, reg, max_iter, tol, n, m, niter, x0, dual,
                                 stream);
  const int sms = sm_count_current();
  BcdProb hp{};
  bcd_geometry(n, m, (int)sizeof(TM), sms, hp);
  const int ncount = 2 + hp.col_strips;

  Workspace ws(stream);
  const size_t o_loga = ws.reserve<double>(n), o_logb = ws.reserve<double>(m);
  size_t o_al[2], o_be[2], o_als[2], o_bes[2];
  for (int k = 0; k < 2; ++k) {
    o_al[k] = ws.reserve<double>(n);
    o_be[k] = ws.reserve<double>(m);
    o_als[k] = ws.reserve<double>(n);
    o_bes[k] = ws.reserve<double>(m);
  }
  const size_t parts = (hp.col_splits > 1) ? (size_t)hp.col_splits * m : 1;
  const size_t o_cm = ws.reserve<double>(parts), o_cs = ws.reserve<double>(parts);
  const size_t o_rp = ws.reserve<double>((size_t)hp.row_ctas * 4);
  const size_t o_cp = ws.reserve<double>((size_t)hp.col_strips * 3);
  const size_t o_cnt = ws.reserve<unsigned int>(ncount);
  const size_t o_st = ws.reserve<BcdState>(1);
  const size_t o_prob = ws.reserve<BcdProb>(1);
  const bool split = sizeof(TM) == 4;  // float-pair duals for the SFU passes
  const size_t o_asp = ws.reserve<float2>(split ? n : 1), o_bsp = ws.reserve<float2>(split ? m : 1);
  CG_TRY(ws.allocate());

  hp.M = M;
  hp.n = n;
  hp.m = m;
  hp.eta = reg;
  hp.s2 = kLog2e / reg;
  hp.a = a;
  hp.loga = ws.at<double>(o_loga);
  hp.logb = ws.at<double>(o_logb);
  for (int k = 0; k < 2; ++k) {
    hp.alpha[k] = ws.at<double>(o_al[k]);
    hp.beta[k] = ws.at<double>(o_be[k]);
    hp.alphas[k] = ws.at<double>(o_als[k]);
    hp.betas[k] = ws.at<double>(o_bes[k]);
  }
  hp.col_m = ws.at<double>(o_cm);
  hp.col_s = ws.at<double>(o_cs);
  hp.row_part = ws.at<double>(o_rp);
  hp.col_part = ws.at<double>(o_cp);
  hp.counters = ws.at<unsigned int>(o_cnt);
  hp.st = ws.at<BcdState>(o_st);
  hp.asplit = split ? ws.at<float2>(o_asp) : nullptr;
  hp.bsplit = split ? ws.at<float2>(o_bsp) : nullptr;
  BcdProb* dprob = ws.at<BcdProb>(o_prob);

  const bool f32 = sizeof(TM) == 4;
  { bcd_init_kernel<<<64, 256, 0, stream>>>(a, b, x0, n, m, hp.s2, const_cast<double*>(hp.loga),
                                          const_cast<double*>(hp.logb), hp.alpha[0], hp.beta[0],
                                          hp.alphas[0], hp.betas[0], hp.counters, ncount, hp.st,
                                          max_iter, tol, f32 ? 1 : 0); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  CG_TRY_CUDA(cudaMemcpyAsync(dprob, &hp, sizeof(BcdProb), cudaMemcpyHostToDevice, stream));

  BcdState hs{};
  int chunk = 4;
  int queued = 0;
  while (true) {
    const int todo = std::min(chunk, std::max(max_iter - queued, 0));
    for (int c = 0; c < todo; ++c) {
      launch_bcd_row(f32, dprob, nullptr, nullptr, hp.row_ctas, stream);
      launch_bcd_col(f32, dprob, nullptr, nullptr, hp.col_strips * hp.col_splits, stream);
    }
    queued += todo;
    CG_TRY_CUDA(cudaGetLastError());
    CG_TRY(read_device(&hs, hp.st, sizeof(BcdState), stream));
    if (hs.done || queued >= max_iter) break;
    chunk = std::min(chunk * 2, 64);
  }
  *niter = hs.niter;
  if (hs.nonfinite) return bcd_nonfinite();
  if (hs.error) return bcd_timeout();

  if (Pout) {
    const size_t total = (size_t)n * m;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((total + 255) / 256, sms * 16));
    { plan_from_state_kernel<TM><<<blocks, 256, 0, stream>>>(M, hp.st, dprob, Pout); cg::count_launch(); }
  }
  { if (dual) dual_from_state_kernel<<<std::max(1, (n + m + 255) / 256), 256, 0, stream>>>(hp.st, dprob, dual); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  ws.release();
  return CG_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free FP64 BCD (cg_bcd_f64_noalloc).
//
// Same kernels, geometry and loop as bcd_solve<double>; the scratch (log
// marginals, the double-buffered duals, column-pass partials, counters, the
// control state and the problem descriptor) lives in one file-scope device
// array instead of a stream-ordered allocation.  Nothing in the array has to
// start at zero: bcd_init_kernel writes the counters, the state and the
// initial duals at the start of every call.  One array per device, so calls
// on the same device must not overlap (the plan/dual kernels of a call still
// read the array after it returns): issue them on one stream, or synchronize
// between them.
constexpr int kNoAllocMaxDim = 16384;
constexpr size_t kNoAllocBytes = size_t(4) << 20;  // 4 MiB; n = m = 16384 needs ~2.5 MiB
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};
}  // namespace

// Device address of this device's scratch array; resolved on the first call
// per device (which may load the module, so it belongs before any capture).
int noalloc_scratch(void** out) {
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_last_error("cg_bcd_f64_noalloc: device ordinal above 63", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_last_error("cg_bcd_f64_noalloc: cudaGetSymbolAddress of the scratch array failed",
                     __FILE__, __LINE__);
      return CG_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return CG_OK;
}

int bcd_solve_noalloc(const double* M, const double* a, const double* b, double* Pout,
                      double reg, int max_iter, double tol, int n, int m, int* niter,
                      const double* x0, double* dual, cudaStream_t stream) {
  if (!M || !a || !b || !niter || n <= 0 || m <= 0 || !(reg > 0.0) || !std::isfinite(reg)) {
    set_last_error("cg_bcd_f64_noalloc: invalid argument", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  if (n > kNoAllocMaxDim || m > kNoAllocMaxDim) {
    set_last_error("cg_bcd_f64_noalloc: n and m must be <= 16384 (fixed scratch array)",
                   __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  const int sms = sm_count_current();
  BcdProb hp{};
  bcd_geometry(n, m, (int)sizeof(double), sms, hp);
  const int ncount = 2 + hp.col_strips;

  // Carve the scratch exactly as bcd_solve sizes its workspace.
  size_t top = 0;
  auto take = [&top](size_t bytes) {
    const size_t off = (top + 255) & ~size_t(255);
    top = off + bytes;
    return off;
  };
  const size_t o_loga = take(n * 8), o_logb = take(m * 8);
  size_t o_al[2], o_be[2], o_als[2], o_bes[2];
  for (int k = 0; k < 2; ++k) {
    o_al[k] = take(n * 8);
    o_be[k] = take(m * 8);
    o_als[k] = take(n * 8);
    o_bes[k] = take(m * 8);
  }
  const size_t parts = (hp.col_splits > 1) ? (size_t)hp.col_splits * m : 1;
  const size_t o_cm = take(parts * 8), o_cs = take(parts * 8);
  const size_t o_rp = take((size_t)hp.row_ctas * 4 * 8);
  const size_t o_cp = take((size_t)hp.col_strips * 3 * 8);
  const size_t o_cnt = take((size_t)ncount * sizeof(unsigned int));
  const size_t o_st = take(sizeof(BcdState));
  const size_t o_prob = take(sizeof(BcdProb));
  if (top > kNoAllocBytes) {
    set_last_error("cg_bcd_f64_noalloc: problem needs more than the 4 MiB scratch array",
                   __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  void* base = nullptr;
  CG_TRY(noalloc_scratch(&base));
  char* s = static_cast<char*>(base);

  hp.M = M;
  hp.n = n;
  hp.m = m;
  hp.eta = reg;
  hp.s2 = kLog2e / reg;
  hp.a = a;
  hp.loga = reinterpret_cast<double*>(s + o_loga);
  hp.logb = reinterpret_cast<double*>(s + o_logb);
  for (int k = 0; k < 2; ++k) {
    hp.alpha[k] = reinterpret_cast<double*>(s + o_al[k]);
    hp.beta[k] = reinterpret_cast<double*>(s + o_be[k]);
    hp.alphas[k] = reinterpret_cast<double*>(s + o_als[k]);
    hp.betas[k] = reinterpret_cast<double*>(s + o_bes[k]);
  }
  hp.col_m = reinterpret_cast<double*>(s + o_cm);
  hp.col_s = reinterpret_cast<double*>(s + o_cs);
  hp.row_part = reinterpret_cast<double*>(s + o_rp);
  hp.col_part = reinterpret_cast<double*>(s + o_cp);
  hp.counters = reinterpret_cast<unsigned int*>(s + o_cnt);
  hp.st = reinterpret_cast<BcdState*>(s + o_st);
  BcdProb* dprob = reinterpret_cast<BcdProb*>(s + o_prob);

  { bcd_init_kernel<<<64, 256, 0, stream>>>(a, b, x0, n, m, hp.s2, const_cast<double*>(hp.loga),
                                          const_cast<double*>(hp.logb), hp.alpha[0], hp.beta[0],
                                          hp.alphas[0], hp.betas[0], hp.counters, ncount, hp.st,
                                          max_iter, tol, 0); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  CG_TRY_CUDA(cudaMemcpyAsync(dprob, &hp, sizeof(BcdProb), cudaMemcpyHostToDevice, stream));

  BcdState hs{};
  int chunk = 4;
  int queued = 0;
  while (true) {
    const int todo = std::min(chunk, std::max(max_iter - queued, 0));
    for (int c = 0; c < todo; ++c) {
      launch_bcd_row(false, dprob, nullptr, nullptr, hp.row_ctas, stream);
      launch_bcd_col(false, dprob, nullptr, nullptr, hp.col_strips * hp.col_splits, stream);
    }
    queued += todo;
    CG_TRY_CUDA(cudaGetLastError());
    CG_TRY(read_device(&hs, hp.st, sizeof(BcdState), stream));
    if (hs.done || queued >= max_iter) break;
    chunk = std::min(chunk * 2, 64);
  }
  *niter = hs.niter;
  if (hs.nonfinite) return bcd_nonfinite();
  if (hs.error) return bcd_timeout();

  if (Pout) {
    const size_t total = (size_t)n * m;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((total + 255) / 256, sms * 16));
    { plan_from_state_kernel<double><<<blocks, 256, 0, stream>>>(M, hp.st, dprob, Pout); cg::count_launch(); }
  }
  if (dual) {
    dual_from_state_kernel<<<std::max(1, (n + m + 255) / 256), 256, 0, stream>>>(hp.st, dprob, dual);
    cg::count_launch();
  }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

__global__ void diag_exp2_kernel(const double* x, double* y, int n, int mode) {
  __shared__ double tab[kExp2TableSize];
  load_exp2_table(tab);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (mode == 0) ? exp2_f64(x[i], tab) : (double)exp2_neg_mixed(x[i]);
}

}  // namespace cg

extern "C" {

const char* cg_last_error(void) { return cg::g_last_error.c_str(); }

const char* cg_version(void) { return "curegot_b200 0.1.0 (sm_100a)"; }

long long cg_launch_count(void) { return cg::g_launches.load(); }

int cg_memory_pool(int device, void** pool) {
  if (!pool) return CG_ERR_INVALID_ARG;
  cudaMemPool_t p = nullptr;
  CG_TRY(cg::library_pool(device, &p));
  *pool = reinterpret_cast<void*>(p);
  return CG_OK;
}

int cg_memory_pool_trim(int device, size_t keep_bytes) {
  cudaMemPool_t p = nullptr;
  CG_TRY(cg::library_pool(device, &p));
  CG_TRY_CUDA(cudaMemPoolTrimTo(p, keep_bytes));
  return CG_OK;
}

void cg_launch_count_reset(void) { cg::g_launches.store(0); }

int cg_bcd_f64(const double* M, const double* a, const double* b, double* P, double reg,
               int max_iter, double tol, int n, int m, int* niter, const double* x0,
               double* dual, cudaStream_t stream) {
  return cg::bcd_solve<double>(M, a, b, P, reg, max_iter, tol, n, m, niter, x0, dual, stream);
}

int cg_bcd_f64_noalloc(const double* M, const double* a, const double* b, double* P, double reg,
                       int max_iter, double tol, int n, int m, int* niter, const double* x0,
                       double* dual, cudaStream_t stream) {
  return cg::bcd_solve_noalloc(M, a, b, P, reg, max_iter, tol, n, m, niter, x0, dual, stream);
}

int cg_bcd_set_staging(int enable) {
  cg::bcd_set_staging(enable != 0);
  return CG_OK;
}

int cg_bcd_set_shifted_lse(int enable) {
  cg::bcd_set_shifted_lse(enable != 0);
  return CG_OK;
}

int cg_bcd_set_l2_prefetch(int chunks) {
  if (chunks < 0 || chunks > 64) return CG_ERR_INVALID_ARG;
  cg::bcd_set_l2_prefetch(chunks);
  return CG_OK;
}

int cg_bcd_mixed(const float* M, const double* a, const double* b, double* P, double reg,
                 int max_iter, double tol, int n, int m, int* niter, const double* x0,
                 double* dual, cudaStream_t stream) {
  return cg::bcd_solve<float>(M, a, b, P, reg, max_iter, tol, n, m, niter, x0, dual, stream);
}

int cg_transport_plan_f64(const double* M, const double* alpha, const double* beta, double* P,
                          double reg, int n, int m, cudaStream_t stream) {
  if (!M || !alpha || !beta || !P || n <= 0 || m <= 0 || !(reg > 0.0)) return CG_ERR_INVALID_ARG;
  cg::launch_plan<double>(M, alpha, beta, P, 1.0 / reg, n, m, stream);
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

int cg_transport_plan_mixed(const float* M, const double* alpha, const double* beta, double* P,
                            double reg, int n, int m, cudaStream_t stream) {
  if (!M || !alpha || !beta || !P || n <= 0 || m <= 0 || !(reg > 0.0)) return CG_ERR_INVALID_ARG;
  cg::launch_plan<float>(M, alpha, beta, P, 1.0 / reg, n, m, stream);
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

int cg_diag_exp2(const double* x, double* y, int n, int mode, cudaStream_t stream) {
  if (!x || !y || n < 0 || mode < 0 || mode > 1) return CG_ERR_INVALID_ARG;
  if (n == 0) return CG_OK;
  { cg::diag_exp2_kernel<<<(n + 255) / 256, 256, 0, stream>>>(x, y, n, mode); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // extern "C"
