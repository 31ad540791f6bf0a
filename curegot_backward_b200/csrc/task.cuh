// Resumable solves: a solve written as a C++20 coroutine suspends where it
// needs device results on the host, instead of blocking its thread.
//
//   SolveTask t = some_solve(&io, ...);    // created suspended
//   t.resume();                            // runs until the first read is posted
//   while (!t.done()) { wait until io.ready(); t.resume(); }
//   int status = t.rc();
//
// Inside the solve, `CO_TRY(co_await io->read(&host, dev, bytes))` queues the
// device-to-host copy on the solve's stream into pinned memory, records an
// event and suspends; when resumed (after the event completed) the bytes are
// copied to their host destinations.  A blocking caller drives one task with
// polling waits; the serving engine drives many tasks from one thread,
// resuming whichever task's event has completed.
#pragma once

#include <chrono>
#include <coroutine>
#include <cstring>
#include <functional>
#include <future>

#include "common.cuh"

namespace cg {

constexpr size_t kTaskPinnedBytes = 4096;
constexpr int kTaskMaxSpans = 6;

// Pinned buffer + event of one task (taken from a process-wide pool; pinned
// frees and event creation stay off the hot path).
struct TaskIO {
  cudaStream_t st = nullptr;
  void* pinned = nullptr;
  cudaEvent_t ev = nullptr;
  ReadSpan spans[kTaskMaxSpans];
  int count = 0;
  int err = CG_OK;
  bool posted = false;
  // larger reads (sparsity patterns) go through `bulk`, pinned, grown on
  // demand and kept with the pooled buffer
  void* bulk = nullptr;
  size_t bulk_cap = 0;
  bool use_bulk = false;
  // host work run off the driving thread (run_job)
  std::future<int> job;
  bool job_posted = false;

  int init(cudaStream_t s);  // takes a buffer and an event from the pool
  void release();            // returns them (after the stream's work is done)

  // True when nothing is pending or the posted copies / job have finished.
  bool ready() const {
    if (job_posted) return job.wait_for(std::chrono::seconds(0)) == std::future_status::ready;
    if (!posted) return true;
    const cudaError_t q = cudaEventQuery(ev);
    return q != cudaErrorNotReady;
  }
  // Blocking wait for the posted copies (polling, yields when the thread is
  // an engine thread; see host_wait).
  int wait();

  struct Await {
    TaskIO* io;
    bool await_ready() const noexcept { return io->err != CG_OK; }
    void await_suspend(std::coroutine_handle<>) const noexcept {}
    int await_resume() const {
      TaskIO& s = *io;
      s.posted = false;
      if (s.err != CG_OK) return s.err;
      const cudaError_t q = cudaEventQuery(s.ev);
      if (q != cudaSuccess) return status_from_cuda(q == cudaErrorNotReady ? cudaEventSynchronize(s.ev) : q);
      size_t off = 0;
      const char* pin = static_cast<const char*>(s.use_bulk ? s.bulk : s.pinned);
      for (int k = 0; k < s.count; ++k) {
        if (s.spans[k].bytes) std::memcpy(s.spans[k].host, pin + off, s.spans[k].bytes);
        off += s.spans[k].bytes;
      }
      return CG_OK;
    }
  };
  Await read_spans(const ReadSpan* sp, int cnt);
  Await read(void* host, const void* dev, size_t bytes) {
    const ReadSpan one{host, dev, bytes};
    return read_spans(&one, 1);
  }
  // Any number of bytes, through `bulk` (grown on demand, outside the hot loop).
  Await read_spans_bulk(const ReadSpan* sp, int cnt);
  Await post_reads(const ReadSpan* sp, int cnt, char* pin);  // copies + event

  // fn() on a separate thread; the task resumes with its status when it has
  // returned.  fn must not touch the task's stream.
  struct JobAwait {
    TaskIO* io;
    bool await_ready() const noexcept { return !io->job_posted; }
    void await_suspend(std::coroutine_handle<>) const noexcept {}
    int await_resume() const {
      if (!io->job_posted) return io->err != CG_OK ? io->err : CG_ERR_CUDA;
      io->job_posted = false;
      return io->job.get();
    }
  };
  JobAwait run_job(std::function<int()> fn) {
    job = std::async(std::launch::async, std::move(fn));
    job_posted = true;
    return JobAwait{this};
  }
};

struct SolveTask {
  struct promise_type {
    int rc = CG_OK;
    SolveTask get_return_object() {
      return SolveTask{std::coroutine_handle<promise_type>::from_promise(*this)};
    }
    std::suspend_always initial_suspend() noexcept { return {}; }
    std::suspend_always final_suspend() noexcept { return {}; }
    void return_value(int v) { rc = v; }
    void unhandled_exception() { rc = CG_ERR_OOM; }  // host allocation failure in a solve
  };
  std::coroutine_handle<promise_type> h{};

  SolveTask() = default;
  explicit SolveTask(std::coroutine_handle<promise_type> x) : h(x) {}
  SolveTask(SolveTask&& o) noexcept : h(o.h) { o.h = {}; }
  SolveTask& operator=(SolveTask&& o) noexcept {
    if (this != &o) {
      if (h) h.destroy();
      h = o.h;
      o.h = {};
    }
    return *this;
  }
  SolveTask(const SolveTask&) = delete;
  SolveTask& operator=(const SolveTask&) = delete;
  ~SolveTask() {
    if (h) h.destroy();
  }
  bool valid() const { return static_cast<bool>(h); }
  bool done() const { return !h || h.done(); }
  void resume() {
    if (h && !h.done()) h.resume();
  }
  int rc() const { return h ? h.promise().rc : CG_OK; }
};

// Runs a task to completion on the calling thread.
inline int drive_task(SolveTask& t, TaskIO& io) {
  while (true) {
    t.resume();
    if (t.done()) return t.rc();
    const int w = io.wait();
    if (w != CG_OK) {
      io.err = w;  // the task sees the error at its pending read
    }
  }
}

}  // namespace cg

// Early return of a status from inside a coroutine.
#define CO_TRY(expr)                   \
  do {                                 \
    const int cg_co_rc_ = (expr);      \
    if (cg_co_rc_ != CG_OK) co_return cg_co_rc_; \
  } while (0)

#define CO_TRY_CUDA(expr)                                   \
  do {                                                      \
    const cudaError_t cg_co_e_ = (expr);                    \
    if (cg_co_e_ != cudaSuccess) {                          \
      cg::set_last_error(cudaGetErrorString(cg_co_e_), __FILE__, __LINE__); \
      co_return cg::status_from_cuda(cg_co_e_);             \
    }                                                       \
  } while (0)
