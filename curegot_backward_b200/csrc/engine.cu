// Continuous-batching OT serving engine.
//
// No reference counterpart: the reference solves one problem per blocking
// call and batches only by a Python loop (curegot/autograd.py:340-367).
//
//   * Sinkhorn (BCD) requests are packed into shared launches: every admitted
//     problem contributes its CTAs to one row pass and one column pass per
//     tick (bcd.cu kernels map CTAs to problems through cta_prob/cta_start).
//     A chunk of ticks is captured once per batch composition as a CUDA graph
//     (a new composition updates the executable graph's kernel parameters in
//     place) and replayed; finished problems exit their CTAs immediately and are
//     retired at the next chunk boundary, when queued requests are admitted
//     into the freed slots.  Duals and solver state stay on the device.
//   * Two batches run side by side on their own streams: requests with at
//     most 8 MB of M, and the larger ones.  A tick of the small batch takes
//     tens of microseconds, so small requests are not held back by the tick
//     length of the large problems.
//   * SPLR requests run on worker threads, each with its own stream, so their
//     device work overlaps the Sinkhorn batch.  Engine threads wait for their
//     streams by polling and yielding, so 16 workers and the two batch
//     threads share the host cores.
//   * Admission is by HBM footprint: a request enters only while the sum of
//     the footprints of admitted requests stays within the budget.
//   * Each request records submit / admit / finish times (host steady clock)
//     and its iteration count; results are polled by the caller.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bcd.cuh"
#include "splr.cuh"
#include "task.cuh"

namespace cg {
namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// SPLR solves multiplexed by one scheduler thread (2 and 4 per thread were
// measured no better on the serving stream).
#ifndef CG_SPLR_SLOTS
#define CG_SPLR_SLOTS 8
#endif
constexpr int kSplrSlotsPerThread = CG_SPLR_SLOTS;

// Sinkhorn requests with at most this many bytes of M share the small batch.
constexpr size_t kSmallBatchBytes = size_t(8) << 20;

// Batch passes may run as grid-stride launches of at most this many CTAs per
// SM.  0 (the default): one CTA per virtual block.  Short CTAs retire often,
// so the SPLR workers' high-priority kernels find free SM slots sooner; on
// the serving stream this measured faster than caps of 1, 2 or 3 CTAs/SM.
#ifndef CG_ENGINE_CAP
#define CG_ENGINE_CAP 0
#endif
constexpr int kBatchCtasPerSm = CG_ENGINE_CAP;

struct Req {
  cg_request_t r;
  uint64_t id = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  size_t footprint = 0;
  int status = CG_OK;
  int niter = 0;
  int converged = 0;
  int fast_iters = 0;
  double last_err = 0;
  // device state
  void* block = nullptr;
  const void* dM = nullptr;
  const double* da = nullptr;
  const double* db = nullptr;
  double* ddual = nullptr;
  BcdProb prob{};
  int slot = -1;
  int cls = 0;  // Sinkhorn batch: 0 small, 1 large
  std::atomic<bool> cancel{false};  // set by cg_engine_cancel while admitted
};

size_t bcd_footprint(const cg_request_t& r, BcdProb& geo, int sms) {
  const int n = r.n, m = r.m;
  const size_t es = r.m_f32 ? 4 : 8;
  bcd_geometry(n, m, (int)es, sms, geo);
  size_t b = 0;
  if (r.host_inputs) b += align256((size_t)n * m * es) + align256(8 * (size_t)(n + m));
  b += align256(8 * (size_t)(n + m));          // dual out (device)
  b += 2 * align256(8 * (size_t)n) + 2 * align256(8 * (size_t)m);  // loga logb, float-pair duals
  b += 4 * align256(8 * (size_t)n) + 4 * align256(8 * (size_t)m);  // alpha/beta (scaled) x2
  const size_t parts = geo.col_splits > 1 ? (size_t)geo.col_splits * m : 1;
  b += 2 * align256(8 * parts);
  b += align256(8 * (size_t)geo.row_ctas * 4) + align256(8 * (size_t)geo.col_strips * 3);
  b += align256(4 * (size_t)(2 + geo.col_strips)) + align256(sizeof(BcdState));
  return b;
}

size_t splr_footprint(const cg_request_t& r) {
  const size_t n = r.n, m = r.m, H = n + m - 1;
  const double dmax = std::min(10.0 / std::min(n, m), 1.0);
  const size_t kmax = std::max<size_t>((size_t)(dmax * n * (m - 1)), 1);
  const size_t k = std::min(n, m - 1);
  size_t b = (size_t)n * m * (r.m_f32 ? 4 : 8) * (r.host_inputs ? 1 : 0);
  b += kmax * 24 + k * k * 8 + 40 * H * 8 + (size_t)n * m / 64 * 8 + (64u << 20);
  return b;
}

__global__ void engine_init_kernel(const double* a, const double* b, int n, int m, double s2,
                                   double* loga, double* logb, double* al0, double* be0,
                                   double* als0, double* bes0, unsigned int* counters, int nc,
                                   BcdState* st, int max_iter, double tol, int fast) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = tid; i < n; i += stride) {
    loga[i] = log(a[i]);
    al0[i] = 0.0;
    als0[i] = 0.0;
  }
  for (int j = tid; j < m; j += stride) {
    logb[j] = log(b[j]);
    be0[j] = 0.0;
    bes0[j] = 0.0;
  }
  for (int q = tid; q < nc; q += stride) counters[q] = 0u;
  if (tid == 0) {
    st->iter = 0;
    st->phase = 1;
    st->check_pending = 0;
    st->done = (max_iter <= 0);
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

__global__ void gather_states_kernel(const BcdProb* probs, int P, BcdState* out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P; k += gridDim.x * blockDim.x)
    out[k] = *probs[k].st;
}

__global__ void engine_dual_kernel(const BcdProb* p, double* dual) {
  const int k = p->st->niter & 1;
  const int n = p->n, m = p->m;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x)
    dual[i] = (i < n) ? p->alpha[k][i] : p->beta[k][i - n];
}

}  // namespace
}  // namespace cg

struct cg_engine_s {
  int device = 0;
  size_t budget = 0;
  size_t in_use = 0;
  int max_batch = 64;
  int chunk = 8;
  int sms = 148;
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  uint64_t next_id = 1;
  std::deque<cg::Req*> bcd_qs[2], splr_q;  // Sinkhorn batches: small, large
  std::unordered_map<uint64_t, cg::Req*> live;  // submitted, not yet finished (guarded by mu)
  int n_workers = 0;
  std::mutex stat_mu;  // guards the statistics below (two batch threads)
  std::vector<cg::Req*> done;
  std::vector<std::thread> threads;
  std::atomic<long long> active_bcd{0}, active_splr{0};
  // statistics
  std::atomic<long long> n_done{0};
  double bytes_bcd = 0.0;     // algorithmic bytes streamed by Sinkhorn passes
  double gpu_ms_bcd = 0.0;    // device time of the Sinkhorn chunks
  long long chunks = 0, graph_builds = 0;
};

namespace cg {
namespace {

bool try_reserve(cg_engine_s* E, size_t bytes) {
  if (E->in_use + bytes > E->budget) return false;
  E->in_use += bytes;
  return true;
}

void release(cg_engine_s* E, size_t bytes) {
  std::lock_guard<std::mutex> lk(E->mu);
  E->in_use -= std::min(bytes, E->in_use);
}

void finish(cg_engine_s* E, Req* q) {
  q->t_done = now_s();
  std::lock_guard<std::mutex> lk(E->mu);
  E->live.erase(q->id);
  E->done.push_back(q);
  E->n_done++;
  E->cv.notify_all();
}

// Stage a Sinkhorn problem: its device block (stream-ordered on the copy
// stream cst) and, for host inputs, the copies of M, a and b on cst, with
// *ev recorded after them (null for device inputs: nothing to wait for).
// The copies overlap the batch chunks already running on the batch stream.
int bcd_stage(Req* q, cudaStream_t cst, cudaEvent_t ev_free, cudaEvent_t* ev) {
  const cg_request_t& r = q->r;
  *ev = nullptr;
  CG_TRY(pool_alloc_async(&q->block, q->footprint, cst));
  if (r.host_inputs) {
    const int n = r.n, m = r.m;
    const size_t es = r.m_f32 ? 4 : 8;
    char* p = static_cast<char*>(q->block);
    double* dab = reinterpret_cast<double*>(p + align256((size_t)n * m * es));
    CG_TRY_CUDA(cudaMemcpyAsync(p, r.M, (size_t)n * m * es, cudaMemcpyHostToDevice, cst));
    CG_TRY_CUDA(cudaMemcpyAsync(dab, r.a, 8 * (size_t)n, cudaMemcpyHostToDevice, cst));
    CG_TRY_CUDA(cudaMemcpyAsync(dab + n, r.b, 8 * (size_t)m, cudaMemcpyHostToDevice, cst));
    CG_TRY_CUDA(cudaEventRecord(ev_free, cst));
    *ev = ev_free;
  }
  return CG_OK;
}

// Initialise a staged Sinkhorn problem on the batch stream st (its copies,
// if any, have completed or are waited for here).
int bcd_admit(cg_engine_s* E, Req* q, cudaStream_t st, cudaEvent_t ev) {
  const cg_request_t& r = q->r;
  const int n = r.n, m = r.m;
  const size_t es = r.m_f32 ? 4 : 8;
  BcdProb& P = q->prob;
  if (ev) CG_TRY_CUDA(cudaStreamWaitEvent(st, ev, 0));
  char* p = static_cast<char*>(q->block);
  auto take = [&](size_t bytes) {
    char* x = p;
    p += align256(bytes);
    return x;
  };
  if (r.host_inputs) {
    void* dM = take((size_t)n * m * es);
    double* dab = reinterpret_cast<double*>(take(8 * (size_t)(n + m)));
    q->dM = dM;
    q->da = dab;
    q->db = dab + n;
  } else {
    q->dM = r.M;
    q->da = r.a;
    q->db = r.b;
  }
  q->ddual = reinterpret_cast<double*>(take(8 * (size_t)(n + m)));
  double* loga = reinterpret_cast<double*>(take(8 * (size_t)n));
  float2* asplit = reinterpret_cast<float2*>(take(8 * (size_t)n));
  double* logb = reinterpret_cast<double*>(take(8 * (size_t)m));
  float2* bsplit = reinterpret_cast<float2*>(take(8 * (size_t)m));
  for (int k = 0; k < 2; ++k) {
    P.alpha[k] = reinterpret_cast<double*>(take(8 * (size_t)n));
    P.alphas[k] = reinterpret_cast<double*>(take(8 * (size_t)n));
    P.beta[k] = reinterpret_cast<double*>(take(8 * (size_t)m));
    P.betas[k] = reinterpret_cast<double*>(take(8 * (size_t)m));
  }
  const size_t parts = P.col_splits > 1 ? (size_t)P.col_splits * m : 1;
  P.col_m = reinterpret_cast<double*>(take(8 * parts));
  P.col_s = reinterpret_cast<double*>(take(8 * parts));
  P.row_part = reinterpret_cast<double*>(take(8 * (size_t)P.row_ctas * 4));
  P.col_part = reinterpret_cast<double*>(take(8 * (size_t)P.col_strips * 3));
  P.counters = reinterpret_cast<unsigned int*>(take(4 * (size_t)(2 + P.col_strips)));
  P.st = reinterpret_cast<BcdState*>(take(sizeof(BcdState)));
  P.asplit = r.m_f32 ? asplit : nullptr;
  P.bsplit = r.m_f32 ? bsplit : nullptr;
  P.M = q->dM;
  P.n = n;
  P.m = m;
  P.eta = r.eta;
  P.s2 = kLog2e / r.eta;
  P.a = q->da;
  P.loga = loga;
  P.logb = logb;
  { engine_init_kernel<<<std::max(1, std::min((std::max(n, m) + 255) / 256, 64)), 256, 0, st>>>(
      q->da, q->db, n, m, P.s2, loga, logb, P.alpha[0], P.beta[0], P.alphas[0], P.betas[0],
      P.counters, 2 + P.col_strips, P.st, r.max_iter, r.tol, r.m_f32 ? 1 : 0); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

// The Sinkhorn batch scheduler.
void bcd_loop(cg_engine_s* E, int cls) {
  std::deque<Req*>& bq = E->bcd_qs[cls];
  long long my_active = 0;
  cudaSetDevice(E->device);
  host_wait_yield(true);
  cudaStream_t st;
  // lowest priority: the batch passes are throughput work that fills every
  // SM; the latency-bound SPLR kernels of the workers go first
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_lo);
  cudaEvent_t ev0, ev1;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  // host-input copies run on their own streams, overlapping the chunks: one
  // for cost matrices of at least kBigCopy bytes and one for the rest, so a
  // small request's copy is not queued behind a large one (a 8192 x 8192
  // FP32 matrix takes ~5 ms over PCIe); the two share the link
  constexpr size_t kBigCopy = size_t(16) << 20;
  cudaStream_t cst, cst_big;
  cudaStreamCreateWithFlags(&cst, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&cst_big, cudaStreamNonBlocking);
  auto copy_stream_of = [&](const Req* q) {
    const size_t mb = (size_t)q->r.n * q->r.m * (q->r.m_f32 ? 4 : 8);
    return (q->r.host_inputs && mb >= kBigCopy) ? cst_big : cst;
  };
  std::vector<cudaEvent_t> ev_pool;
  auto take_event = [&]() -> cudaEvent_t {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    return e;
  };
  // problems whose block is allocated and whose copies are in flight
  struct Staged {
    Req* q;
    cudaEvent_t ev;
  };
  std::vector<Staged> staging;
  std::vector<Req*> active;  // one precision class per batch (f32 or f64 kernels)
  bool batch_f32 = true;
  // device-side batch description
  BcdProb* d_probs = nullptr;
  int* d_map = nullptr;
  size_t cap_probs = 0, cap_map = 0;
  std::vector<BcdProb> h_probs;
  std::vector<int> h_map;
  BcdState* h_states = nullptr;  // pinned
  BcdState* d_states = nullptr;
  size_t cap_states = 0;
  cudaGraphExec_t gexec = nullptr;
  bool dirty = true;
  int row_total = 0, col_total = 0;
  double batch_bytes_per_tick = 0.0;
  // Ends every admitted problem of this batch with status rc (used when the
  // batch description cannot be allocated): their blocks are released
  // stream-ordered after the work already queued on the batch stream.
  auto fail_batch = [&](int rc) {
    host_wait(st);
    for (Req* q : active) {
      if (q->block) cudaFreeAsync(q->block, st);
      q->block = nullptr;
      q->status = rc;
      release(E, q->footprint);
      finish(E, q);
    }
    active.clear();
    E->active_bcd -= my_active;
    my_active = 0;
    dirty = true;
  };

  while (true) {
    // ---- admission: reserve, allocate and start the copies (staging) -------
    {
      std::unique_lock<std::mutex> lk(E->mu);
      if (active.empty() && staging.empty())
        E->cv.wait(lk, [&] { return E->stop || !bq.empty(); });
      if (E->stop && active.empty() && staging.empty()) break;
      while (!E->stop && !bq.empty() && (int)(active.size() + staging.size()) < E->max_batch) {
        Req* q = bq.front();
        const bool none = active.empty() && staging.empty();
        if (!none && (q->r.m_f32 != 0) != batch_f32) break;
        if (!try_reserve(E, q->footprint)) {
          if (!none || E->in_use > 0) break;
          // larger than the whole budget: reject
          bq.pop_front();
          q->status = CG_ERR_ADMISSION;
          lk.unlock();
          finish(E, q);
          lk.lock();
          continue;
        }
        bq.pop_front();
        lk.unlock();
        q->t_admit = now_s();
        if (none) batch_f32 = q->r.m_f32 != 0;
        cudaEvent_t evq = take_event(), used = nullptr;
        const cudaStream_t qcs = copy_stream_of(q);
        int rc = evq ? bcd_stage(q, qcs, evq, &used) : CG_ERR_CUDA;
        if (evq && !used) ev_pool.push_back(evq);
        lk.lock();
        if (rc != CG_OK) {
          if (q->block) cudaFreeAsync(q->block, qcs);
          q->block = nullptr;
          q->status = rc;
          E->in_use -= q->footprint;
          lk.unlock();
          finish(E, q);
          lk.lock();
          continue;
        }
        staging.push_back({q, used});
      }
    }
    // ---- staged problems whose copies have landed join the batch ------------
    // A copy of at most kJoinWaitBytes lands within ~100 us: it is waited for
    // here, so its problem joins the chunk about to start instead of the one
    // after it (a chunk lasts ~1 ms); larger copies join when they land.
    constexpr size_t kJoinWaitBytes = size_t(4) << 20;
    for (size_t k = 0; k < staging.size();) {
      const Staged sg = staging[k];
      if (sg.ev && cudaEventQuery(sg.ev) == cudaErrorNotReady) {
        const cg_request_t& r = sg.q->r;
        const size_t bytes = (size_t)r.n * r.m * (r.m_f32 ? 4 : 8) + 8 * (size_t)(r.n + r.m);
        if (bytes > kJoinWaitBytes) {
          ++k;
          continue;
        }
        while (cudaEventQuery(sg.ev) == cudaErrorNotReady) std::this_thread::yield();
      }
      staging.erase(staging.begin() + (long)k);
      const int rc = bcd_admit(E, sg.q, st, sg.ev);
      if (sg.ev) ev_pool.push_back(sg.ev);
      if (rc != CG_OK) {
        cudaFreeAsync(sg.q->block, st);
        sg.q->block = nullptr;
        sg.q->status = rc;
        release(E, sg.q->footprint);
        finish(E, sg.q);
        continue;
      }
      active.push_back(sg.q);
      {
        std::lock_guard<std::mutex> lk(E->mu);
        E->active_bcd += (long long)active.size() - my_active;
      }
      my_active = (long long)active.size();
      dirty = true;
    }
    if (active.empty()) {
      if (!staging.empty() && staging.front().ev) {
        // nothing to run until the oldest copy lands
        while (cudaEventQuery(staging.front().ev) == cudaErrorNotReady) std::this_thread::yield();
      }
      continue;
    }
    // ---- (re)build the batch description and its chunk graph ---------------
    if (dirty) {
      h_probs.clear();
      h_map.clear();
      row_total = col_total = 0;
      batch_bytes_per_tick = 0.0;
      for (size_t k = 0; k < active.size(); ++k) {
        Req* q = active[k];
        q->slot = (int)k;
        h_probs.push_back(q->prob);
        row_total += q->prob.row_ctas;
        col_total += q->prob.col_strips * q->prob.col_splits;
        batch_bytes_per_tick += 2.0 * q->r.n * (double)q->r.m * (q->r.m_f32 ? 4 : 8);
      }
      // map layout: [row cta->prob][row start][col cta->prob][col start]
      const int P = (int)active.size();
      h_map.resize((size_t)row_total + P + col_total + P);
      int* rp = h_map.data();
      int* rs = rp + row_total;
      int* cp = rs + P;
      int* cs = cp + col_total;
      int ro = 0, co = 0;
      for (int k = 0; k < P; ++k) {
        rs[k] = ro;
        for (int c = 0; c < active[k]->prob.row_ctas; ++c) rp[ro++] = k;
        cs[k] = co;
        const int nc = active[k]->prob.col_strips * active[k]->prob.col_splits;
        for (int c = 0; c < nc; ++c) cp[co++] = k;
      }
      // Regrow the batch description buffers into temporaries: the old
      // blocks and capacities stay in place unless every allocation
      // succeeded, so an allocation failure never leaves a stale pointer.
      if ((size_t)P > cap_probs || h_map.size() > cap_map || (size_t)P > cap_states) {
        const size_t np_cap = (size_t)P > cap_probs ? std::max<size_t>(P, 2 * cap_probs) : 0;
        const size_t nm_cap = h_map.size() > cap_map ? std::max<size_t>(h_map.size(), 2 * cap_map) : 0;
        const size_t ns_cap = (size_t)P > cap_states ? std::max<size_t>(P, 2 * cap_states) : 0;
        BcdProb* n_probs = nullptr;
        int* n_map = nullptr;
        BcdState* n_dst = nullptr;
        BcdState* n_hst = nullptr;
        bool ok = true;
        if (np_cap) ok = ok && pool_alloc_async(reinterpret_cast<void**>(&n_probs),
                                                np_cap * sizeof(BcdProb), st) == CG_OK;
        if (nm_cap) ok = ok && pool_alloc_async(reinterpret_cast<void**>(&n_map),
                                                nm_cap * sizeof(int), st) == CG_OK;
        if (ns_cap) {
          ok = ok && pool_alloc_async(reinterpret_cast<void**>(&n_dst), ns_cap * sizeof(BcdState),
                                      st) == CG_OK;
          ok = ok && cudaHostAlloc(reinterpret_cast<void**>(&n_hst), ns_cap * sizeof(BcdState),
                                   cudaHostAllocDefault) == cudaSuccess;
        }
        if (!ok) {
          cudaGetLastError();
          if (n_probs) cudaFreeAsync(n_probs, st);
          if (n_map) cudaFreeAsync(n_map, st);
          if (n_dst) cudaFreeAsync(n_dst, st);
          if (n_hst) cudaFreeHost(n_hst);
          set_last_error("engine: batch description allocation failed", __FILE__, __LINE__);
          fail_batch(CG_ERR_OOM);
          continue;
        }
        if (n_probs) {
          if (d_probs) cudaFreeAsync(d_probs, st);
          d_probs = n_probs;
          cap_probs = np_cap;
        }
        if (n_map) {
          if (d_map) cudaFreeAsync(d_map, st);
          d_map = n_map;
          cap_map = nm_cap;
        }
        if (n_dst) {
          host_wait(st);  // the previous pinned block may still be a copy target
          if (d_states) cudaFreeAsync(d_states, st);
          if (h_states) cudaFreeHost(h_states);
          d_states = n_dst;
          h_states = n_hst;
          cap_states = ns_cap;
        }
      }
      cudaMemcpyAsync(d_probs, h_probs.data(), P * sizeof(BcdProb), cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_map, h_map.data(), h_map.size() * sizeof(int), cudaMemcpyHostToDevice,
                      st);
      host_wait(st);  // host vectors are reused below
      cudaGraph_t g;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int* drp = d_map;
        const int* drs = drp + row_total;
        const int* dcp = drs + P;
        const int* dcs = dcp + col_total;
        for (int c = 0; c < E->chunk; ++c) {
          launch_bcd_row(batch_f32, d_probs, drp, drs, row_total, st, kBatchCtasPerSm * E->sms);
          launch_bcd_col(batch_f32, d_probs, dcp, dcs, col_total, st, kBatchCtasPerSm * E->sms);
        }
        count_launch(-2LL * E->chunk);  // captured, not executed
        if (cudaStreamEndCapture(st, &g) == cudaSuccess) {
          // Same topology (2 x chunk kernel nodes) for every composition:
          // update the executable graph's kernel parameters in place when
          // the kernels match, else instantiate a new one.
          cudaGraphExecUpdateResultInfo info;
          if (!gexec || cudaGraphExecUpdate(gexec, g, &info) != cudaSuccess) {
            cudaGetLastError();
            if (gexec) cudaGraphExecDestroy(gexec);
            gexec = nullptr;
            if (cudaGraphInstantiate(&gexec, g, 0) != cudaSuccess) gexec = nullptr;
          }
          cudaGraphDestroy(g);
        } else if (gexec) {
          cudaGraphExecDestroy(gexec);
          gexec = nullptr;
        }
      } else if (gexec) {
        cudaGraphExecDestroy(gexec);
        gexec = nullptr;
      }
      {
        std::lock_guard<std::mutex> sl(E->stat_mu);
        E->graph_builds++;
      }
      dirty = false;
    }
    // ---- run one chunk ------------------------------------------------------
    const int P = (int)active.size();
    cudaEventRecord(ev0, st);
    if (gexec) {
      cudaGraphLaunch(gexec, st);
      count_launch(2LL * E->chunk);
    } else {
      const int* drp = d_map;
      const int* drs = drp + row_total;
      const int* dcp = drs + P;
      const int* dcs = dcp + col_total;
      for (int c = 0; c < E->chunk; ++c) {
        launch_bcd_row(batch_f32, d_probs, drp, drs, row_total, st);
        launch_bcd_col(batch_f32, d_probs, dcp, dcs, col_total, st);
      }
    }
    cudaEventRecord(ev1, st);
    // states of all problems: one gather kernel, one copy
    { gather_states_kernel<<<std::max(1, (P + 127) / 128), 128, 0, st>>>(d_probs, P, d_states); cg::count_launch(); }
    cudaMemcpyAsync(h_states, d_states, P * sizeof(BcdState), cudaMemcpyDeviceToHost, st);
    host_wait(st);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    std::unique_lock<std::mutex> stat_lk(E->stat_mu);
    E->gpu_ms_bcd += ms;
    E->chunks++;
    // algorithmic bytes: problems still running at the chunk start stream
    // 2 n m elements per tick until they finish
    for (int k = 0; k < P; ++k) {
      const Req* q = active[k];
      const int ran = std::min(E->chunk, std::max(0, h_states[k].iter - q->niter));
      E->bytes_bcd += ran * 2.0 * q->r.n * (double)q->r.m * (q->r.m_f32 ? 4 : 8);
      active[k]->niter = h_states[k].iter;
    }
    stat_lk.unlock();
    // ---- retire finished (or cancelled) problems -----------------------------
    std::vector<Req*> keep;
    std::vector<char> retire(P, 0);
    for (int k = 0; k < P; ++k) {
      Req* q = active[k];
      const BcdState& s = h_states[k];
      const bool cancelled = !s.done && q->cancel.load(std::memory_order_relaxed);
      if (!s.done && !cancelled) {
        keep.push_back(q);
        continue;
      }
      retire[k] = 1;
      dirty = true;
      if (cancelled) {
        q->status = CG_ERR_CANCELLED;
        continue;
      }
      q->niter = s.niter;
      if (s.nonfinite) q->status = CG_ERR_NONFINITE;
      if (s.error) q->status = CG_ERR_TIMEOUT;
      q->converged = !s.nonfinite &&
                     ((s.niter < s.max_iter) || (s.phase == 2 && s.last_err < s.tol && !s.fast));
      q->fast_iters = s.fast_iters;
      q->last_err = s.last_err;
      // duals -> output (device or host)
      BcdProb* dp = d_probs + k;
      { engine_dual_kernel<<<std::max(1, std::min((q->r.n + q->r.m + 255) / 256, 64)), 256, 0, st>>>(
          dp, q->ddual); cg::count_launch(); }
      if (q->r.dual_out) {
        cudaMemcpyAsync(q->r.dual_out, q->ddual, 8 * (size_t)(q->r.n + q->r.m),
                        q->r.host_inputs ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st);
      }
    }
    if (dirty) {
      host_wait(st);
      for (int k = 0; k < P; ++k) {
        if (!retire[k]) continue;
        Req* q = active[k];
        cudaFreeAsync(q->block, st);
        q->block = nullptr;
        release(E, q->footprint);
        finish(E, q);
      }
      active.swap(keep);
      E->active_bcd += (long long)active.size() - my_active;
      my_active = (long long)active.size();
    }
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
  cudaStreamSynchronize(cst);
  cudaStreamSynchronize(cst_big);
  cudaStreamDestroy(cst);
  cudaStreamDestroy(cst_big);
  if (d_states) cudaFreeAsync(d_states, st);
  if (h_states) cudaFreeHost(h_states);
  if (d_probs) cudaFreeAsync(d_probs, st);
  if (d_map) cudaFreeAsync(d_map, st);
  host_wait(st);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  cudaStreamDestroy(st);
}

// One SPLR request in flight on a scheduler thread: its stream, its
// resumable solve (splr_task) and the buffers the engine owns for it.
struct SplrJob {
  Req* q = nullptr;
  cudaStream_t st = nullptr;
  TaskIO io;
  SolveTask task;
  void* blk = nullptr;
  double* ddual = nullptr;
  int niter = 0, conv = 0;
  bool finishing = false;  // final copy posted; waiting for its event
};

// SPLR scheduler: up to `slots` solves in flight, each a coroutine on its own
// high-priority stream.  The thread starts admitted requests, then resumes
// whichever solve's posted device read has landed (cudaEventQuery, no
// blocking), so many solves share one host thread and their kernels overlap
// on the device.  Decisions inside every solve are those of cg_splr_mixed /
// cg_splr_f64 (the same coroutine, driven to completion there).
void splr_loop(cg_engine_s* E, int slots) {
  cudaSetDevice(E->device);
  host_wait_yield(true);
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  std::vector<cudaStream_t> streams(slots);
  for (auto& s : streams) cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio_hi);
  std::vector<cudaStream_t> free_streams(streams.rbegin(), streams.rend());
  std::vector<SplrJob*> jobs;

  auto start = [&](SplrJob* j) -> int {
    const cg_request_t& r = j->q->r;
    const int n = r.n, m = r.m;
    const size_t es = r.m_f32 ? 4 : 8;
    const void* dM = r.M;
    const double *da = r.a, *db = r.b;
    const size_t inb = r.host_inputs ? align256((size_t)n * m * es) + align256(8 * (size_t)(n + m)) : 0;
    CG_TRY(pool_alloc_async(&j->blk, inb + align256(8 * (size_t)(n + m)), j->st));
    char* p = static_cast<char*>(j->blk);
    if (r.host_inputs) {
      CG_TRY_CUDA(cudaMemcpyAsync(p, r.M, (size_t)n * m * es, cudaMemcpyHostToDevice, j->st));
      dM = p;
      double* dab = reinterpret_cast<double*>(p + align256((size_t)n * m * es));
      CG_TRY_CUDA(cudaMemcpyAsync(dab, r.a, 8 * (size_t)n, cudaMemcpyHostToDevice, j->st));
      CG_TRY_CUDA(cudaMemcpyAsync(dab + n, r.b, 8 * (size_t)m, cudaMemcpyHostToDevice, j->st));
      da = dab;
      db = dab + n;
    }
    j->ddual = reinterpret_cast<double*>(p + inb);
    CG_TRY(j->io.init(j->st));
    // the engine stops on the full marginal error, so every SPLR result
    // meets tol on rows and on all m columns (the reference's test leaves
    // the gauge column out)
    SplrParams prm{r.eta, r.tol, r.max_iter, std::min(10.0 / std::min(n, m), 1.0), 1e-3, 30, 3,
                   0, 1, 1, &j->q->cancel};
    if (r.m_f32)
      j->task = splr_task<float>(&j->io, static_cast<const float*>(dM), da, db, nullptr, n, m,
                                 prm, nullptr, j->ddual, &j->niter, &j->conv, nullptr, nullptr);
    else
      j->task = splr_task<double>(&j->io, static_cast<const double*>(dM), da, db, nullptr, n, m,
                                  prm, nullptr, j->ddual, &j->niter, &j->conv, nullptr, nullptr);
    j->task.resume();
    return CG_OK;
  };
  // the solve has returned: status, duals out, release its frame and block
  auto conclude = [&](SplrJob* j, int rc) {
    Req* q = j->q;
    const cg_request_t& r = q->r;
    q->niter = j->niter;
    q->converged = j->conv;
    // the SPLR loop ends early without converging only on a non-finite
    // objective or gradient norm (the reference's break, sinkhorn_splr.cu:1128)
    if (rc == CG_OK && !j->conv && j->niter < r.max_iter) {
      set_last_error("engine: SPLR objective or gradient became non-finite", __FILE__, __LINE__);
      rc = CG_ERR_NONFINITE;
    }
    q->status = rc;
    j->task = SolveTask();  // frame released: its workspace is freed stream-ordered
    if (rc == CG_OK && r.dual_out)
      cudaMemcpyAsync(r.dual_out, j->ddual, 8 * (size_t)(r.n + r.m),
                      r.host_inputs ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, j->st);
    if (j->blk) cudaFreeAsync(j->blk, j->st);
    j->blk = nullptr;
    if (j->io.ev) {
      cudaEventRecord(j->io.ev, j->st);
      j->io.posted = true;
    }
    j->finishing = true;
  };
  auto retire = [&](SplrJob* j) {
    j->io.release();
    free_streams.push_back(j->st);
    {
      std::lock_guard<std::mutex> lk(E->mu);
      E->in_use -= std::min(j->q->footprint, E->in_use);
      E->active_splr--;
    }
    E->cv.notify_all();
    finish(E, j->q);
    delete j;
  };

  while (true) {
    std::vector<SplrJob*> admitted;
    {
      std::unique_lock<std::mutex> lk(E->mu);
      auto ready = [&](std::deque<Req*>& dq) {
        if (dq.empty()) return false;
        Req* f = dq.front();
        return f->footprint > E->budget || E->in_use + f->footprint <= E->budget;
      };
      if (jobs.empty()) E->cv.wait(lk, [&] { return E->stop || ready(E->splr_q); });
      if (E->stop && jobs.empty()) break;
      std::deque<Req*>& dq = E->splr_q;
      while (!E->stop && (int)(jobs.size() + admitted.size()) < slots && ready(dq)) {
        Req* q = dq.front();
        dq.pop_front();
        if (q->footprint > E->budget) {
          q->status = CG_ERR_ADMISSION;
          lk.unlock();
          finish(E, q);
          lk.lock();
          continue;
        }
        E->in_use += q->footprint;
        E->active_splr++;
        auto* j = new SplrJob();
        j->q = q;
        j->st = free_streams.back();
        free_streams.pop_back();
        admitted.push_back(j);
      }
    }
    for (SplrJob* j : admitted) {
      j->q->t_admit = now_s();
      const int rc = start(j);
      jobs.push_back(j);
      if (rc != CG_OK) conclude(j, rc);
      else if (j->task.done()) conclude(j, j->task.rc());
    }
    bool progressed = !admitted.empty();
    for (size_t k = 0; k < jobs.size();) {
      SplrJob* j = jobs[k];
      if (j->finishing) {
        if (j->io.ready()) {
          jobs[k] = jobs.back();
          jobs.pop_back();
          retire(j);
          progressed = true;
          continue;
        }
      } else if (j->io.ready()) {
        j->task.resume();
        progressed = true;
        if (j->task.done()) conclude(j, j->task.rc());
      }
      ++k;
    }
    if (!progressed) std::this_thread::yield();
  }
  for (auto& s : streams) cudaStreamDestroy(s);
}

}  // namespace
}  // namespace cg

extern "C" {

int cg_engine_create(size_t budget_bytes, int max_batch, int splr_workers, int chunk,
                     cg_engine** out) {
  if (!out || budget_bytes == 0 || max_batch <= 0 || splr_workers < 0) return CG_ERR_INVALID_ARG;
  auto* E = new cg_engine_s();
  cudaGetDevice(&E->device);
  E->budget = budget_bytes;
  E->max_batch = max_batch;
  E->chunk = chunk > 0 ? chunk : 8;
  E->sms = cg::sm_count_current();
  E->threads.emplace_back(cg::bcd_loop, E, 0);
  E->threads.emplace_back(cg::bcd_loop, E, 1);
  // splr_workers = SPLR solves in flight, spread over scheduler threads of
  // at most kSplrSlotsPerThread solves each
  E->n_workers = splr_workers;
  if (splr_workers > 0) {
    const int nthreads = std::max(1, (splr_workers + cg::kSplrSlotsPerThread - 1) /
                                         cg::kSplrSlotsPerThread);
    for (int w = 0; w < nthreads; ++w) {
      const int slots = splr_workers / nthreads + (w < splr_workers % nthreads ? 1 : 0);
      E->threads.emplace_back(cg::splr_loop, E, slots);
    }
  }
  *out = reinterpret_cast<cg_engine*>(E);
  return CG_OK;
}

int cg_engine_submit(cg_engine* eng, const cg_request_t* req, uint64_t* id) {
  if (!eng || !req || req->n <= 0 || req->m <= 0 || !req->M || !req->a || !req->b ||
      !(req->eta > 0.0) || (req->algo != CG_ALGO_BCD && req->algo != CG_ALGO_SPLR))
    return CG_ERR_INVALID_ARG;
  cg_engine_s* E = reinterpret_cast<cg_engine_s*>(eng);
  auto* q = new cg::Req();
  q->r = *req;
  q->t_submit = cg::now_s();
  if (req->algo == CG_ALGO_BCD) {
    q->footprint = cg::bcd_footprint(q->r, q->prob, E->sms);
    q->cls = ((size_t)req->n * req->m * (req->m_f32 ? 4 : 8) > cg::kSmallBatchBytes) ? 1 : 0;
  } else {
    if (req->m < 2) {
      delete q;
      return CG_ERR_INVALID_ARG;
    }
    q->footprint = cg::splr_footprint(q->r);
  }
  {
    std::lock_guard<std::mutex> lk(E->mu);
    q->id = E->next_id++;
    E->live[q->id] = q;
    if (req->algo == CG_ALGO_BCD) E->bcd_qs[q->cls].push_back(q);
    else E->splr_q.push_back(q);
  }
  E->cv.notify_all();
  if (id) *id = q->id;
  return CG_OK;
}

int cg_engine_poll(cg_engine* eng, cg_result_t* results, int capacity, int wait_ms, int* count) {
  if (!eng || !count || (capacity > 0 && !results)) return CG_ERR_INVALID_ARG;
  cg_engine_s* E = reinterpret_cast<cg_engine_s*>(eng);
  std::unique_lock<std::mutex> lk(E->mu);
  if (E->done.empty() && wait_ms > 0)
    E->cv.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !E->done.empty(); });
  const int k = std::min<int>(capacity, (int)E->done.size());
  for (int i = 0; i < k; ++i) {
    cg::Req* q = E->done[i];
    cg_result_t& o = results[i];
    o.id = q->id;
    o.tag = q->r.tag;
    o.status = q->status;
    o.niter = q->niter;
    o.converged = q->converged;
    o.fast_iters = q->fast_iters;
    o.last_err = q->last_err;
    o.t_submit = q->t_submit;
    o.t_admit = q->t_admit;
    o.t_done = q->t_done;
    delete q;
  }
  E->done.erase(E->done.begin(), E->done.begin() + k);
  *count = k;
  return CG_OK;
}

int cg_engine_cancel(cg_engine* eng, uint64_t id) {
  if (!eng) return CG_ERR_INVALID_ARG;
  cg_engine_s* E = reinterpret_cast<cg_engine_s*>(eng);
  std::unique_lock<std::mutex> lk(E->mu);
  auto it = E->live.find(id);
  if (it == E->live.end()) {
    cg::set_last_error("cg_engine_cancel: unknown or finished request", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  cg::Req* q = it->second;
  for (auto* dq : {&E->bcd_qs[0], &E->bcd_qs[1], &E->splr_q}) {
    auto pos = std::find(dq->begin(), dq->end(), q);
    if (pos == dq->end()) continue;
    // still queued: nothing of it is on the device
    dq->erase(pos);
    q->status = CG_ERR_CANCELLED;
    q->t_done = cg::now_s();
    E->live.erase(it);
    E->done.push_back(q);
    E->n_done++;
    lk.unlock();
    E->cv.notify_all();
    return CG_OK;
  }
  q->cancel.store(true);  // admitted: its scheduler ends it
  return CG_OK;
}

int cg_engine_stats(cg_engine* eng, cg_engine_stats_t* out) {
  if (!eng || !out) return CG_ERR_INVALID_ARG;
  cg_engine_s* E = reinterpret_cast<cg_engine_s*>(eng);
  std::lock_guard<std::mutex> lk(E->mu);
  out->in_use_bytes = E->in_use;
  out->budget_bytes = E->budget;
  out->queued = (long long)(E->bcd_qs[0].size() + E->bcd_qs[1].size() + E->splr_q.size());
  out->active_bcd = E->active_bcd;
  out->active_splr = E->active_splr;
  out->completed = E->n_done;
  out->bcd_bytes = E->bytes_bcd;
  out->bcd_gpu_ms = E->gpu_ms_bcd;
  out->chunks = E->chunks;
  out->graph_builds = E->graph_builds;
  return CG_OK;
}

double cg_engine_clock(void) { return cg::now_s(); }

int cg_engine_destroy(cg_engine* eng) {
  if (!eng) return CG_OK;
  cg_engine_s* E = reinterpret_cast<cg_engine_s*>(eng);
  {
    std::lock_guard<std::mutex> lk(E->mu);
    E->stop = true;
  }
  E->cv.notify_all();
  for (auto& t : E->threads) t.join();
  for (auto* q : E->done) delete q;
  for (auto* q : E->bcd_qs[0]) delete q;
  for (auto* q : E->bcd_qs[1]) delete q;
  for (auto* q : E->splr_q) delete q;
  delete E;
  return CG_OK;
}

}  // extern "C"
