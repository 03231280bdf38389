// Serving loop: a kNN-graph server with continuous batching.
//
// Requests (embedding sets of any n, dim and dtype) are queued on submit.
// Worker lanes -- each with its own evoc_gpu_ctx, i.e. its own CUDA stream and
// scratch -- admit the oldest pending request that fits the HBM budget, move
// its rows to the device and build its kNN graph.  Several requests therefore
// run on the device at once, and a request that arrives while others run is
// admitted as soon as a lane and memory free up.  A request's graph stays
// resident in HBM until the caller fetches or releases it.
//
// Admission counts, per request, the bytes it holds while it runs
// (n*dim*size(dtype) rows + n*k*8 for indices and distances) plus the
// workspace a lane's context needs for it (padded f32/BF16/int8 rows,
// candidates, heaps).  A lane's workspace is kept at its high-water mark and
// counted once; the rows are returned to the budget when the graph is built.
// A request that could never fit is refused at submit (EVOC_ERR_OOM).
//
// Per-request device buffers come from the server's own stream-ordered pool
// (cudaMallocFromPoolAsync / cudaFreeAsync); frees go to an idle stream so a
// request finishing on one lane never makes another lane's allocation wait on
// work in flight.
//
// There is no counterpart in evoc-rs, whose fit_predict builds one data set's
// graph at a time (src/clustering.rs:650-716).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/evoc_gpu.h"
#include "ctx_plan.h"
#include "kernels.h"

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

enum JobState { kPending = 0, kRunning = 1, kDone = 2, kFailed = 3, kCancelled = 4 };

struct Job {
  int64_t id = 0;
  int32_t dtype = 0;
  int64_t n = 0, dim = 0;
  int32_t k = 0, keff = 0;
  evoc_gpu_opts opts{};
  int64_t tau[3] = {0, 0, 0};
  bool has_tau = false;
  std::vector<uint8_t> host_copy;  // the caller's rows, copied at submit
  const void* src = nullptr;       // rows to read: host_copy, a borrowed host buffer or device rows
  bool src_on_device = false;
  void* d_rows = nullptr;
  int32_t* d_idx = nullptr;
  float* d_dist = nullptr;
  int64_t row_bytes_total = 0;  // n*dim*size(dtype) when the server copies the rows in
  int64_t out_bytes = 0;        // n*k_eff*8
  evoc::CtxSizes need;          // context buffers the request needs
  int64_t held = 0;             // bytes counted against the budget right now
  int skipped = 0;              // times a later request was admitted first
  int state = kPending;
  bool cancel = false;
  bool reported = false;
  int status = EVOC_OK;
  std::string err;
  int lane = -1;
  int64_t t_submit = 0, t_admit = 0, t_done = 0;
};

int64_t elem_size(int32_t dtype) { return dtype == EVOC_DTYPE_F32 ? 4 : 1; }

// A request passed over this many times by later, smaller ones reserves the
// next admission: first fit without starvation.
constexpr int kMaxSkips = 16;

}  // namespace

struct evoc_gpu_server {
  int device = 0;
  int64_t budget = 0;
  int lanes = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Job>> pending;
  std::deque<int64_t> finished;  // completion order, for wait_any
  std::unordered_map<int64_t, std::shared_ptr<Job>> jobs;
  int64_t next_id = 1;
  int64_t in_use = 0, peak = 0;
  int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, rejected = 0, running = 0;
  std::vector<evoc::CtxSizes> lane_sizes;  // each lane context's buffers (counted in in_use)
  int64_t ws_misses = 0;
  std::vector<evoc_gpu_ctx*> ctxs;
  std::vector<cudaStream_t> streams;
  cudaStream_t free_stream = nullptr;
  std::mutex copy_mu;
  cudaStream_t copy_stream = nullptr;
  cudaMemPool_t pool = nullptr;
  std::vector<std::thread> workers;
  bool stopping = false;
  bool profile = false;
  std::vector<std::string> stage_names;            // first-seen order
  std::unordered_map<std::string, std::pair<double, int64_t>> stage_totals;
  double lane_busy_ms = 0.0;
};

namespace {

// Frees a job's device buffers and returns its bytes to the budget.  Called
// with s->mu held, only when no kernel or copy of the job is in flight.
void free_job_memory_locked(evoc_gpu_server* s, Job* j) {
  if (j->d_rows) cudaFreeAsync(j->d_rows, s->free_stream);
  if (j->d_idx) cudaFreeAsync(j->d_idx, s->free_stream);
  if (j->d_dist) cudaFreeAsync(j->d_dist, s->free_stream);
  j->d_rows = nullptr;
  j->d_idx = nullptr;
  j->d_dist = nullptr;
  s->in_use -= j->held;
  j->held = 0;
  s->cv_work.notify_all();  // memory came back: another request may fit now
}

void finish_locked(evoc_gpu_server* s, Job* j, int state, int status, const std::string& err) {
  j->state = state;
  j->status = status;
  j->err = err;
  j->t_done = now_ns();
  if (state == kDone) s->completed++;
  else if (state == kFailed) s->failed++;
  else s->cancelled++;
  s->finished.push_back(j->id);
  s->cv_done.notify_all();
}

void run_job(evoc_gpu_server* s, int lane, Job* j) {
  evoc_gpu_ctx* ctx = s->ctxs[size_t(lane)];
  cudaStream_t st = s->streams[size_t(lane)];
  nvtxRangePushA("evoc_job");
  int rc = EVOC_OK;
  std::string err;
  const size_t out_elems = size_t(j->n) * size_t(j->keff);
  cudaError_t e = cudaSuccess;
  const void* rows = j->src;
  if (!j->src_on_device) {
    e = cudaMallocFromPoolAsync(&j->d_rows, size_t(j->row_bytes_total), s->pool, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(j->d_rows, j->src, size_t(j->row_bytes_total), cudaMemcpyHostToDevice, st);
    rows = j->d_rows;
  }
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&j->d_idx), out_elems * 4, s->pool, st);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&j->d_dist), out_elems * 4, s->pool, st);
  if (e != cudaSuccess) {
    rc = e == cudaErrorMemoryAllocation ? EVOC_ERR_OOM : EVOC_ERR_CUDA;
    err = std::string("serving: ") + cudaGetErrorString(e);
    cudaGetLastError();
  } else {
    evoc_gpu_opts o = j->opts;
    o.buffers_on_device = 1;
    int32_t kout = 0;
    rc = evoc_gpu_knn_graph(ctx, &o, j->dtype, rows, j->n, j->dim, j->k, j->has_tau ? j->tau : nullptr, j->d_idx,
                            j->d_dist, &kout);
    if (rc != EVOC_OK)
      err = std::string(evoc_gpu_last_error(ctx)) + " [request n=" + std::to_string(j->n) +
            " dim=" + std::to_string(j->dim) + " dtype=" + std::to_string(j->dtype) +
            " form=" + std::to_string(j->opts.form) + " lane=" + std::to_string(lane) + "]";
  }
  // evoc_gpu_knn_graph returns after its stream is idle, so the rows are no
  // longer read; on an error path wait for the copies before freeing.
  if (rc != EVOC_OK) cudaStreamSynchronize(st);
  std::vector<uint8_t>().swap(j->host_copy);
  nvtxRangePop();
  evoc::CtxSizes actual;
  evoc::ctx_buffer_sizes(ctx, &actual);
  std::vector<std::pair<std::string, float>> stages;
  if (s->profile && rc == EVOC_OK) {
    char name[64];
    float ms = 0.0f;
    for (int i = 0, n = evoc_gpu_profile_count(ctx); i < n; i++)
      if (evoc_gpu_profile_stage(ctx, i, name, sizeof(name), &ms) == EVOC_OK) stages.emplace_back(name, ms);
  }
  const int64_t t_end = now_ns();
  std::lock_guard<std::mutex> lock(s->mu);
  s->running--;
  s->lane_busy_ms += double(t_end - j->t_admit) * 1e-6;
  for (const auto& st_ms : stages) {
    auto it = s->stage_totals.find(st_ms.first);
    if (it == s->stage_totals.end()) {
      s->stage_names.push_back(st_ms.first);
      it = s->stage_totals.emplace(st_ms.first, std::make_pair(0.0, int64_t(0))).first;
    }
    it->second.first += st_ms.second;
    it->second.second += 1;
  }
  // The plan should match the context exactly; if it ever falls short, count
  // the real size from now on.
  const int64_t planned = int64_t(s->lane_sizes[size_t(lane)].total());
  if (int64_t(actual.total()) > planned) s->ws_misses++;
  s->in_use += int64_t(actual.total()) - planned;
  s->lane_sizes[size_t(lane)] = actual;
  s->peak = std::max(s->peak, s->in_use);
  if (j->d_rows) {
    cudaFreeAsync(j->d_rows, s->free_stream);
    j->d_rows = nullptr;
  }
  s->in_use -= j->row_bytes_total;
  j->held -= j->row_bytes_total;
  s->cv_work.notify_all();
  if (j->cancel) {
    free_job_memory_locked(s, j);
    finish_locked(s, j, kCancelled, EVOC_ERR_CANCELLED, "cancelled");
  } else if (rc != EVOC_OK) {
    free_job_memory_locked(s, j);
    finish_locked(s, j, kFailed, rc, err);
  } else {
    finish_locked(s, j, kDone, EVOC_OK, "");
  }
}

void worker(evoc_gpu_server* s, int lane) {
  cudaSetDevice(s->device);
  evoc::CtxSizes& mine = s->lane_sizes[size_t(lane)];
  std::unique_lock<std::mutex> lock(s->mu);
  for (;;) {
    std::shared_ptr<Job> pick;
    bool trim = false;
    while (!s->stopping) {
      // First fit over the pending requests, oldest first; a request skipped
      // kMaxSkips times holds the next admission for itself.
      for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
        Job* j = it->get();
        const evoc::CtxSizes grown = evoc::grown_sizes(mine, j->need);
        const int64_t grow = int64_t(grown.total()) - int64_t(mine.total());
        const int64_t need = j->row_bytes_total + j->out_bytes + grow;
        if (s->in_use + need <= s->budget) {
          if (it != s->pending.begin()) s->pending.front()->skipped++;
          pick = *it;
          s->pending.erase(it);
          s->in_use += need;
          j->held = j->row_bytes_total + j->out_bytes;
          mine = grown;
          s->peak = std::max(s->peak, s->in_use);
          break;
        }
        if (it == s->pending.begin() && j->skipped >= kMaxSkips) break;
      }
      if (pick) break;
      // Nothing fits.  An idle lane whose own buffers keep the oldest request
      // out gives them back.
      if (!s->pending.empty() && mine.total() > 0) {
        const Job* head = s->pending.front().get();
        const int64_t alone = int64_t(evoc::grown_sizes(evoc::CtxSizes{}, head->need).total());
        if (s->in_use - int64_t(mine.total()) + head->row_bytes_total + head->out_bytes + alone <= s->budget) {
          trim = true;
          break;
        }
      }
      s->cv_work.wait(lock);
    }
    if (trim) {
      const int64_t held = int64_t(mine.total());
      lock.unlock();
      evoc::ctx_release_buffers(s->ctxs[size_t(lane)]);
      lock.lock();
      s->in_use -= held;
      mine = evoc::CtxSizes{};
      s->cv_work.notify_all();
      continue;
    }
    if (!pick) return;
    pick->state = kRunning;
    pick->lane = lane;
    pick->t_admit = now_ns();
    s->running++;
    lock.unlock();
    run_job(s, lane, pick.get());
    lock.lock();
  }
}

std::shared_ptr<Job> lookup(evoc_gpu_server* s, int64_t id) {
  auto it = s->jobs.find(id);
  return it == s->jobs.end() ? nullptr : it->second;
}

int state_status(const Job& j) {
  switch (j.state) {
    case kDone: return EVOC_OK;
    case kFailed: return j.status;
    case kCancelled: return EVOC_ERR_CANCELLED;
    default: return EVOC_ERR_PENDING;
  }
}

bool finished(const Job& j) { return j.state != kPending && j.state != kRunning; }

void forget_locked(evoc_gpu_server* s, const std::shared_ptr<Job>& j) {
  if (j->state == kPending) {
    for (auto it = s->pending.begin(); it != s->pending.end(); ++it)
      if (it->get() == j.get()) {
        s->pending.erase(it);
        break;
      }
  }
  free_job_memory_locked(s, j.get());
  s->jobs.erase(j->id);
}

}  // namespace

extern "C" {

int64_t evoc_gpu_server_now_ns(void) { return now_ns(); }

void evoc_gpu_server_default_opts(evoc_gpu_server_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->struct_size = sizeof(evoc_gpu_server_opts);
  o->device = 0;
  o->budget_bytes = int64_t(150) * 1000 * 1000 * 1000;
  o->max_inflight = 4;
}

int evoc_gpu_server_create(const evoc_gpu_server_opts* opts, evoc_gpu_server** out) {
  if (!out) return EVOC_ERR_ARG;
  *out = nullptr;
  evoc_gpu_server_opts o;
  evoc_gpu_server_default_opts(&o);
  if (opts) {
    if (opts->struct_size != sizeof(evoc_gpu_server_opts)) return EVOC_ERR_ARG;
    o = *opts;
  }
  if (o.max_inflight < 1 || o.max_inflight > 64 || o.budget_bytes <= 0) return EVOC_ERR_ARG;
  if (cudaSetDevice(o.device) != cudaSuccess) {
    cudaGetLastError();
    return EVOC_ERR_CUDA;
  }
  auto* s = new evoc_gpu_server();
  s->device = o.device;
  s->budget = o.budget_bytes;
  s->lanes = o.max_inflight;
  s->lane_sizes.assign(size_t(s->lanes), evoc::CtxSizes{});
  auto bail = [&](int rc) {
    for (evoc_gpu_ctx* p : s->ctxs) evoc_gpu_ctx_destroy(p);
    if (s->free_stream) cudaStreamDestroy(s->free_stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return rc;
  };
  s->profile = o.profile != 0;
  for (int i = 0; i < s->lanes; i++) {
    evoc_gpu_ctx* c = nullptr;
    const int rc = evoc_gpu_ctx_create(o.device, &c);
    if (rc != EVOC_OK) return bail(rc);
    if (s->profile) evoc_gpu_profile_enable(c, 1);
    s->ctxs.push_back(c);
    s->streams.push_back(static_cast<cudaStream_t>(evoc_gpu_ctx_stream(c)));
  }
  if (cudaStreamCreateWithFlags(&s->free_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(EVOC_ERR_CUDA);
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = o.device;
  if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) return bail(EVOC_ERR_CUDA);
  // Keep freed request memory in the pool between requests.
  uint64_t threshold = uint64_t(o.budget_bytes);
  cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  for (int i = 0; i < s->lanes; i++) s->workers.emplace_back(worker, s, i);
  *out = s;
  return EVOC_OK;
}

void evoc_gpu_server_destroy(evoc_gpu_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stopping = true;
    while (!s->pending.empty()) {
      Job* j = s->pending.front().get();
      s->pending.pop_front();
      finish_locked(s, j, kCancelled, EVOC_ERR_CANCELLED, "server stopped");
    }
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  cudaSetDevice(s->device);
  {
    std::lock_guard<std::mutex> lock(s->mu);
    for (auto& kv : s->jobs) free_job_memory_locked(s, kv.second.get());
    s->jobs.clear();
  }
  cudaStreamSynchronize(s->free_stream);
  for (evoc_gpu_ctx* c : s->ctxs) evoc_gpu_ctx_destroy(c);
  cudaStreamDestroy(s->free_stream);
  cudaStreamDestroy(s->copy_stream);
  cudaMemPoolDestroy(s->pool);
  delete s;
}

int evoc_gpu_server_submit(evoc_gpu_server* s, const evoc_gpu_opts* opts, int32_t dtype, const void* data,
                           int64_t n, int64_t dim, int32_t k, const int64_t* rng_state, int32_t flags,
                           int64_t* job_id) {
  if (!s || !job_id) return EVOC_ERR_ARG;
  *job_id = 0;
  if (k <= 0) return EVOC_ERR_K;
  if (n <= 0) return EVOC_ERR_EMPTY;
  if (!data || dim <= 0 || dtype < EVOC_DTYPE_F32 || dtype > EVOC_DTYPE_U8) return EVOC_ERR_ARG;
  if (flags & ~int32_t(EVOC_SUBMIT_BORROW)) return EVOC_ERR_ARG;
  auto j = std::make_shared<Job>();
  evoc_gpu_default_opts(&j->opts);
  if (opts) {
    if (opts->struct_size != sizeof(evoc_gpu_opts)) return EVOC_ERR_ARG;
    j->opts = *opts;
  }
  if (j->opts.row_begin != 0 || j->opts.row_end != 0) return EVOC_ERR_ARG;
  j->dtype = dtype;
  j->n = n;
  j->dim = dim;
  j->k = k;
  j->keff = int32_t(std::max<int64_t>(1, std::min<int64_t>(k, n - 1)));
  if (rng_state) {
    std::memcpy(j->tau, rng_state, sizeof(j->tau));
    j->has_tau = true;
  }
  const int64_t in_bytes = n * dim * elem_size(dtype);
  j->src_on_device = j->opts.buffers_on_device != 0;
  j->row_bytes_total = j->src_on_device ? 0 : in_bytes;
  j->out_bytes = n * int64_t(j->keff) * 8;
  evoc::knn_buffer_needs(s->ctxs[0], j->opts, dtype, n, dim, k, &j->need);
  const int64_t alone = int64_t(evoc::grown_sizes(evoc::CtxSizes{}, j->need).total());
  if (j->row_bytes_total + j->out_bytes + alone > s->budget) {
    std::lock_guard<std::mutex> lock(s->mu);
    s->rejected++;
    return EVOC_ERR_OOM;
  }
  if (j->src_on_device || (flags & EVOC_SUBMIT_BORROW)) {
    j->src = data;
  } else {
    j->host_copy.assign(static_cast<const uint8_t*>(data), static_cast<const uint8_t*>(data) + in_bytes);
    j->src = j->host_copy.data();
  }
  j->t_submit = now_ns();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stopping) return EVOC_ERR_CANCELLED;
    j->id = s->next_id++;
    s->jobs[j->id] = j;
    s->pending.push_back(j);
    s->submitted++;
    *job_id = j->id;
  }
  s->cv_work.notify_all();
  return EVOC_OK;
}

int evoc_gpu_server_request_bytes(evoc_gpu_server* s, const evoc_gpu_opts* opts, int32_t dtype, int64_t n,
                                  int64_t dim, int32_t k, int64_t* resident, int64_t* workspace) {
  if (!s || n <= 0 || dim <= 0 || k <= 0 || dtype < EVOC_DTYPE_F32 || dtype > EVOC_DTYPE_U8) return EVOC_ERR_ARG;
  evoc_gpu_opts o;
  evoc_gpu_default_opts(&o);
  if (opts) {
    if (opts->struct_size != sizeof(evoc_gpu_opts)) return EVOC_ERR_ARG;
    o = *opts;
  }
  const int64_t keff = std::max<int64_t>(1, std::min<int64_t>(k, n - 1));
  evoc::CtxSizes need;
  evoc::knn_buffer_needs(s->ctxs[0], o, dtype, n, dim, k, &need);
  if (resident) *resident = (o.buffers_on_device ? 0 : n * dim * elem_size(dtype)) + n * keff * 8;
  if (workspace) *workspace = int64_t(evoc::grown_sizes(evoc::CtxSizes{}, need).total());
  return EVOC_OK;
}

int evoc_gpu_server_poll(evoc_gpu_server* s, int64_t job_id) {
  if (!s) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  auto j = lookup(s, job_id);
  return j ? state_status(*j) : EVOC_ERR_ARG;
}

int evoc_gpu_server_wait(evoc_gpu_server* s, int64_t job_id, int64_t timeout_ms) {
  if (!s) return EVOC_ERR_ARG;
  std::unique_lock<std::mutex> lock(s->mu);
  auto j = lookup(s, job_id);
  if (!j) return EVOC_ERR_ARG;
  if (timeout_ms < 0) {
    s->cv_done.wait(lock, [&] { return finished(*j); });
  } else if (!s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return finished(*j); })) {
    return EVOC_ERR_TIMEOUT;
  }
  return state_status(*j);
}

int evoc_gpu_server_wait_any(evoc_gpu_server* s, int64_t timeout_ms, int64_t* job_id) {
  if (!s || !job_id) return EVOC_ERR_ARG;
  *job_id = 0;
  std::unique_lock<std::mutex> lock(s->mu);
  auto ready = [&] {
    while (!s->finished.empty()) {
      auto j = lookup(s, s->finished.front());
      if (j && !j->reported) return true;
      s->finished.pop_front();  // released or fetched before it was reported
    }
    return false;
  };
  if (timeout_ms < 0) s->cv_done.wait(lock, ready);
  else if (!s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready)) return EVOC_ERR_TIMEOUT;
  auto j = lookup(s, s->finished.front());
  s->finished.pop_front();
  j->reported = true;
  *job_id = j->id;
  return state_status(*j);
}

int evoc_gpu_server_result(evoc_gpu_server* s, int64_t job_id, int32_t* out_idx, float* out_dist, int32_t* out_k,
                           int32_t keep_resident) {
  if (!s) return EVOC_ERR_ARG;
  std::shared_ptr<Job> j;
  {
    std::unique_lock<std::mutex> lock(s->mu);
    j = lookup(s, job_id);
    if (!j) return EVOC_ERR_ARG;
    s->cv_done.wait(lock, [&] { return finished(*j); });
    const int rc = state_status(*j);
    if (rc != EVOC_OK) {
      if (!keep_resident) forget_locked(s, j);
      return rc;
    }
    j->reported = true;
  }
  if (out_k) *out_k = j->keff;
  const size_t bytes = size_t(j->n) * size_t(j->keff) * 4;
  cudaError_t e = cudaSuccess;
  {
    // Copies share one stream so they never queue behind a lane's next
    // request.  The buffers stay valid: a finished job's memory is freed only
    // by release or by a result call without keep_resident, and the caller
    // does not make those for this id while this call runs.
    std::lock_guard<std::mutex> copy_lock(s->copy_mu);
    cudaSetDevice(s->device);
    if (out_idx) e = cudaMemcpyAsync(out_idx, j->d_idx, bytes, cudaMemcpyDeviceToHost, s->copy_stream);
    if (e == cudaSuccess && out_dist)
      e = cudaMemcpyAsync(out_dist, j->d_dist, bytes, cudaMemcpyDeviceToHost, s->copy_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->copy_stream);
  }
  std::lock_guard<std::mutex> lock(s->mu);
  if (!keep_resident && lookup(s, job_id)) forget_locked(s, j);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return EVOC_ERR_CUDA;
  }
  return EVOC_OK;
}

int evoc_gpu_server_result_device(evoc_gpu_server* s, int64_t job_id, const int32_t** d_idx, const float** d_dist,
                                  int32_t* out_k) {
  if (!s) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  auto j = lookup(s, job_id);
  if (!j) return EVOC_ERR_ARG;
  const int rc = state_status(*j);
  if (rc != EVOC_OK) return rc;
  if (d_idx) *d_idx = j->d_idx;
  if (d_dist) *d_dist = j->d_dist;
  if (out_k) *out_k = j->keff;
  return EVOC_OK;
}

int evoc_gpu_server_release(evoc_gpu_server* s, int64_t job_id) {
  if (!s) return EVOC_ERR_ARG;
  std::unique_lock<std::mutex> lock(s->mu);
  auto j = lookup(s, job_id);
  if (!j) return EVOC_ERR_ARG;
  if (j->state == kRunning) {
    j->cancel = true;
    s->cv_done.wait(lock, [&] { return finished(*j); });
  }
  if (lookup(s, job_id)) forget_locked(s, j);
  return EVOC_OK;
}

int evoc_gpu_server_cancel(evoc_gpu_server* s, int64_t job_id) {
  if (!s) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  auto j = lookup(s, job_id);
  if (!j) return EVOC_ERR_ARG;
  if (j->state == kPending) {
    for (auto it = s->pending.begin(); it != s->pending.end(); ++it)
      if (it->get() == j.get()) {
        s->pending.erase(it);
        break;
      }
    std::vector<uint8_t>().swap(j->host_copy);
    finish_locked(s, j.get(), kCancelled, EVOC_ERR_CANCELLED, "cancelled");
  } else if (j->state == kRunning) {
    j->cancel = true;  // the graph is discarded when the lane finishes it
  }
  return EVOC_OK;
}

int evoc_gpu_server_job_info(evoc_gpu_server* s, int64_t job_id, evoc_gpu_job_info* info) {
  if (!s || !info) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  auto j = lookup(s, job_id);
  if (!j) return EVOC_ERR_ARG;
  std::memset(info, 0, sizeof(*info));
  info->submit_ns = j->t_submit;
  info->admit_ns = j->t_admit;
  info->done_ns = j->t_done;
  info->n = j->n;
  info->dim = j->dim;
  info->dtype = j->dtype;
  info->k_eff = j->keff;
  info->lane = j->lane;
  info->status = state_status(*j);
  std::strncpy(info->error, j->err.c_str(), sizeof(info->error) - 1);
  return EVOC_OK;
}

int evoc_gpu_server_stats(evoc_gpu_server* s, evoc_gpu_server_counters* out) {
  if (!s || !out) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->failed = s->failed;
  out->cancelled = s->cancelled;
  out->rejected = s->rejected;
  out->pending = int64_t(s->pending.size());
  out->running = s->running;
  out->bytes_in_use = s->in_use;
  out->peak_bytes = s->peak;
  out->budget_bytes = s->budget;
  int64_t ws = 0;
  for (const evoc::CtxSizes& l : s->lane_sizes) ws += int64_t(l.total());
  out->workspace_bytes = ws;
  out->workspace_misses = s->ws_misses;
  out->lanes = s->lanes;
  return EVOC_OK;
}

int evoc_gpu_server_stage_count(evoc_gpu_server* s) {
  if (!s) return 0;
  std::lock_guard<std::mutex> lock(s->mu);
  return int(s->stage_names.size());
}

int evoc_gpu_server_stage(evoc_gpu_server* s, int i, char* name, int32_t name_len, double* total_ms,
                          int64_t* count) {
  if (!s) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  if (i < 0 || i >= int(s->stage_names.size())) return EVOC_ERR_ARG;
  const std::string& nm = s->stage_names[size_t(i)];
  const auto& v = s->stage_totals[nm];
  if (name && name_len > 0) {
    std::strncpy(name, nm.c_str(), size_t(name_len) - 1);
    name[name_len - 1] = '\0';
  }
  if (total_ms) *total_ms = v.first;
  if (count) *count = v.second;
  return EVOC_OK;
}

double evoc_gpu_server_lane_busy_ms(evoc_gpu_server* s) {
  if (!s) return 0.0;
  std::lock_guard<std::mutex> lock(s->mu);
  return s->lane_busy_ms;
}

}  // extern "C"
