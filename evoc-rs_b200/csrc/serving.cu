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
#include "ctx.h"
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
  evoc::CtxSizes need;          // context buffers the request needs alone
  bool batch_ok = false;        // small enough for a multi-request batch
  int32_t form = 0;             // resolved form
  double work = 0.0;            // 2 n^2 dim: the scan's operations
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

// Small requests (f32 BF16+rerank, i8 exact) are admitted together and built
// by one evoc_gpu_knn_graph_batch call: up to kBatchJobs requests of at most
// kBatchRows rows each, and at most kBatchWork scan operations in all, so a
// batch stays a few milliseconds long.
constexpr int64_t kBatchRows = 16384;
constexpr int kBatchJobs = 64;
constexpr double kBatchWork = 4e12;
// A batch forms only under backlog: at least this many compatible small
// requests pending.  With fewer, each runs alone at its lowest latency.
constexpr int kBatchMin = 4;
// Requests below this many rows are latency-sensitive: they run on a lane's
// high-priority stream, and the last lanes (small_lanes of the options; by
// default a quarter of them, with four or more lanes) admit only these, so a
// burst of big requests never leaves the small ones queueing for a lane.
constexpr int64_t kUrgentRows = 65536;
int small_only_lanes(int lanes, int asked) {
  if (asked <= 0) return 0;
  return asked < lanes ? asked : lanes - 1;  // at least one lane takes big requests
}

}  // namespace

struct evoc_gpu_server {
  int device = 0;
  int64_t budget = 0;
  int lanes = 0;
  int small_lanes = 0;  // the last lanes admit only requests under kUrgentRows rows
  bool smallest_first = false;  // admission order: smallest scan first (else oldest first)
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
  std::vector<cudaStream_t> streams;  // each lane context's own stream (normal priority)
  std::vector<cudaStream_t> urgent;   // each lane's high-priority stream, for small requests
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
  int64_t batches = 0, batched = 0;  // multi-request calls and the requests they carried
  int batch_max = kBatchJobs;
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

// Allocates a request's device buffers on the lane's stream and queues the
// copy of its rows; *rows receives the device rows.
cudaError_t stage_job(evoc_gpu_server* s, cudaStream_t st, Job* j, const void** rows) {
  const size_t out_elems = size_t(j->n) * size_t(j->keff);
  cudaError_t e = cudaSuccess;
  *rows = j->src;
  if (!j->src_on_device) {
    e = cudaMallocFromPoolAsync(&j->d_rows, size_t(j->row_bytes_total), s->pool, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(j->d_rows, j->src, size_t(j->row_bytes_total), cudaMemcpyHostToDevice, st);
    *rows = j->d_rows;
  }
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&j->d_idx), out_elems * 4, s->pool, st);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&j->d_dist), out_elems * 4, s->pool, st);
  return e;
}

std::string tag(const Job* j, int lane, size_t batch) {
  return " [request n=" + std::to_string(j->n) + " dim=" + std::to_string(j->dim) +
         " dtype=" + std::to_string(j->dtype) + " form=" + std::to_string(j->opts.form) +
         " lane=" + std::to_string(lane) + (batch > 1 ? " batch of " + std::to_string(batch) : "") + "]";
}

// Builds the graphs of `group` on the lane: one request through
// evoc_gpu_knn_graph, or a batch of small ones through evoc_gpu_knn_graph_batch.
void run_work(evoc_gpu_server* s, int lane, const std::vector<Job*>& group, bool batch) {
  evoc_gpu_ctx* ctx = s->ctxs[size_t(lane)];
  // Small requests (and batches of them) run on the lane's high-priority
  // stream; a big request runs at normal priority with a CTA per query block,
  // so the SMs it holds come free block by block and the small requests'
  // kernels, queued at higher priority, take them first.
  const bool small = batch || group.front()->n < kUrgentRows;
  cudaStream_t st = small ? s->urgent[size_t(lane)] : s->streams[size_t(lane)];
  ctx->stream = st;  // the lane's previous call left its streams idle
  ctx->scan_per_block = !small;
  nvtxRangePushA(batch ? "evoc_batch" : "evoc_job");
  const size_t m = group.size();
  int rc = EVOC_OK;
  std::string err;
  std::vector<const void*> rows(m, nullptr);
  for (size_t i = 0; i < m && rc == EVOC_OK; i++) {
    const cudaError_t e = stage_job(s, st, group[i], &rows[i]);
    if (e != cudaSuccess) {
      rc = e == cudaErrorMemoryAllocation ? EVOC_ERR_OOM : EVOC_ERR_CUDA;
      err = std::string("serving: ") + cudaGetErrorString(e);
      cudaGetLastError();
    }
  }
  if (rc == EVOC_OK) {
    const Job* j0 = group.front();
    evoc_gpu_opts o = j0->opts;
    o.buffers_on_device = 1;
    if (batch) {
      std::vector<int64_t> n(m), dim(m);
      std::vector<int32_t*> idx(m);
      std::vector<float*> dist(m);
      for (size_t i = 0; i < m; i++) {
        n[i] = group[i]->n;
        dim[i] = group[i]->dim;
        idx[i] = group[i]->d_idx;
        dist[i] = group[i]->d_dist;
      }
      rc = evoc_gpu_knn_graph_batch(ctx, &o, j0->dtype, int32_t(m), rows.data(), n.data(), dim.data(), j0->k,
                                    idx.data(), dist.data(), nullptr, nullptr);
    } else {
      int32_t kout = 0;
      rc = evoc_gpu_knn_graph(ctx, &o, j0->dtype, rows[0], j0->n, j0->dim, j0->k, j0->has_tau ? j0->tau : nullptr,
                              j0->d_idx, j0->d_dist, &kout);
    }
    if (rc != EVOC_OK) err = std::string(evoc_gpu_last_error(ctx)) + tag(j0, lane, m);
  }
  // The graph calls return after their stream is idle, so the rows are no
  // longer read; on an error path wait for the copies before freeing.
  if (rc != EVOC_OK) cudaStreamSynchronize(st);
  for (Job* j : group) std::vector<uint8_t>().swap(j->host_copy);
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
  s->running -= int64_t(m);
  s->lane_busy_ms += double(t_end - group.front()->t_admit) * 1e-6;
  if (batch) {
    s->batches++;
    s->batched += int64_t(m);
  }
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
  for (Job* j : group) {
    if (j->d_rows) {
      cudaFreeAsync(j->d_rows, s->free_stream);
      j->d_rows = nullptr;
    }
    s->in_use -= j->row_bytes_total;
    j->held -= j->row_bytes_total;
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
  s->cv_work.notify_all();
}

bool batch_compatible(const Job* a, const Job* b) {
  return b->batch_ok && a->dtype == b->dtype && a->k == b->k && a->form == b->form &&
         a->opts.oversample == b->opts.oversample;
}

// Buffers a batch of `group` needs on a lane (plan of evoc_gpu_knn_graph_batch).
evoc::CtxSizes batch_need(evoc_gpu_server* s, const std::vector<Job*>& group) {
  std::vector<int64_t> n, dim;
  for (const Job* j : group) {
    n.push_back(j->n);
    dim.push_back(j->dim);
  }
  evoc::CtxSizes need;
  evoc::batch_buffer_needs(group.front()->opts, group.front()->dtype, int32_t(group.size()), n.data(), dim.data(),
                           group.front()->k, &need);
  (void)s;
  return need;
}

// Under backlog, admits the small request at `it` with compatible pending
// ones after it as one batch (first fit for each addition).  Returns false,
// admitting nothing, when fewer than kBatchMin would go together.
bool try_admit_batch(evoc_gpu_server* s, std::deque<std::shared_ptr<Job>>::iterator it, evoc::CtxSizes& mine,
                     std::vector<std::shared_ptr<Job>>* group, bool small_only) {
  Job* j = it->get();
  std::vector<Job*> cand{j};
  evoc::CtxSizes grown = evoc::grown_sizes(mine, batch_need(s, cand));
  int64_t held = j->row_bytes_total + j->out_bytes;
  if (s->in_use + held + int64_t(grown.total()) - int64_t(mine.total()) > s->budget) return false;
  double work = j->work;
  for (auto jt = std::next(it); jt != s->pending.end() && int(cand.size()) < s->batch_max; ++jt) {
    Job* o = jt->get();
    if (!batch_compatible(j, o) || work + o->work > kBatchWork) continue;
    cand.push_back(o);
    const evoc::CtxSizes g2 = evoc::grown_sizes(mine, batch_need(s, cand));
    const int64_t h2 = held + o->row_bytes_total + o->out_bytes;
    if (s->in_use + h2 + int64_t(g2.total()) - int64_t(mine.total()) > s->budget) {
      cand.pop_back();
      continue;
    }
    grown = g2;
    held = h2;
    work += o->work;
  }
  if (int(cand.size()) < kBatchMin) return false;
  if (it != s->pending.begin() && !(small_only && s->pending.front()->n >= kUrgentRows))
    s->pending.front()->skipped++;
  s->in_use += held + int64_t(grown.total()) - int64_t(mine.total());
  for (Job* c : cand) {
    for (auto kt = s->pending.begin(); kt != s->pending.end(); ++kt)
      if (kt->get() == c) {
        group->push_back(*kt);
        s->pending.erase(kt);
        break;
      }
    c->held = c->row_bytes_total + c->out_bytes;
  }
  mine = grown;
  s->peak = std::max(s->peak, s->in_use);
  return true;
}

void worker(evoc_gpu_server* s, int lane) {
  cudaSetDevice(s->device);
  evoc::CtxSizes& mine = s->lane_sizes[size_t(lane)];
  const bool small_only = lane >= s->lanes - s->small_lanes;
  std::unique_lock<std::mutex> lock(s->mu);
  for (;;) {
    std::vector<std::shared_ptr<Job>> group;
    bool batch = false;
    bool trim = false;
    while (!s->stopping) {
      // First fit over the pending requests, oldest first (or smallest scan
      // first); a request skipped kMaxSkips times holds the next admission
      // for itself.  A small request takes compatible small ones after it
      // into the same batch.  A small-only lane passes over big requests
      // without counting a skip.
      std::vector<std::deque<std::shared_ptr<Job>>::iterator> order;
      order.reserve(s->pending.size());
      for (auto it = s->pending.begin(); it != s->pending.end(); ++it) order.push_back(it);
      if (s->smallest_first && !s->pending.empty() && s->pending.front()->skipped < kMaxSkips)
        std::stable_sort(order.begin(), order.end(),
                         [](const auto& a, const auto& b) { return (*a)->work < (*b)->work; });
      for (auto it : order) {  // every branch that erases from pending leaves the loop
        Job* j = it->get();
        if (small_only && j->n >= kUrgentRows) continue;
        if (j->batch_ok && s->batch_max > 1 && try_admit_batch(s, it, mine, &group, small_only)) {
          batch = true;
          break;
        }
        const evoc::CtxSizes grown = evoc::grown_sizes(mine, j->need);
        const int64_t grow = int64_t(grown.total()) - int64_t(mine.total());
        const int64_t need = j->row_bytes_total + j->out_bytes + grow;
        if (s->in_use + need <= s->budget) {
          if (it != s->pending.begin() && !(small_only && s->pending.front()->n >= kUrgentRows))
            s->pending.front()->skipped++;
          group.push_back(*it);
          s->pending.erase(it);
          s->in_use += need;
          j->held = j->row_bytes_total + j->out_bytes;
          mine = grown;
          s->peak = std::max(s->peak, s->in_use);
          break;
        }
        if (it == s->pending.begin() && j->skipped >= kMaxSkips) break;
      }
      if (!group.empty()) break;
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
    if (group.empty()) return;
    const int64_t t_admit = now_ns();
    std::vector<Job*> jobs;
    for (auto& g : group) {
      g->state = kRunning;
      g->lane = lane;
      g->t_admit = t_admit;
      jobs.push_back(g.get());
    }
    s->running += int64_t(jobs.size());
    lock.unlock();
    run_work(s, lane, jobs, batch);
    group.clear();
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
  o->batch_max = kBatchJobs;
  o->small_lanes = 0;
  o->admission = 0;
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
  if (o.admission < 0 || o.admission > 1) return EVOC_ERR_ARG;
  if (cudaSetDevice(o.device) != cudaSuccess) {
    cudaGetLastError();
    return EVOC_ERR_CUDA;
  }
  auto* s = new evoc_gpu_server();
  s->device = o.device;
  s->budget = o.budget_bytes;
  s->lanes = o.max_inflight;
  s->small_lanes = small_only_lanes(s->lanes, o.small_lanes);
  s->smallest_first = o.admission == 1;
  s->lane_sizes.assign(size_t(s->lanes), evoc::CtxSizes{});
  auto bail = [&](int rc) {
    for (evoc_gpu_ctx* p : s->ctxs) evoc_gpu_ctx_destroy(p);
    for (cudaStream_t u : s->urgent) cudaStreamDestroy(u);
    if (s->free_stream) cudaStreamDestroy(s->free_stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return rc;
  };
  s->profile = o.profile != 0;
  s->batch_max = std::min(std::max(o.batch_max, 0), kBatchJobs);
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  for (int i = 0; i < s->lanes; i++) {
    evoc_gpu_ctx* c = nullptr;
    const int rc = evoc_gpu_ctx_create(o.device, &c);
    if (rc != EVOC_OK) return bail(rc);
    if (s->profile) evoc_gpu_profile_enable(c, 1);
    s->ctxs.push_back(c);
    s->streams.push_back(static_cast<cudaStream_t>(evoc_gpu_ctx_stream(c)));
    cudaStream_t u = nullptr;
    if (cudaStreamCreateWithPriority(&u, cudaStreamNonBlocking, greatest) != cudaSuccess) return bail(EVOC_ERR_CUDA);
    s->urgent.push_back(u);
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
  for (cudaStream_t u : s->urgent) cudaStreamDestroy(u);
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
  j->form = j->opts.form == EVOC_FORM_AUTO
                ? (dtype == EVOC_DTYPE_F32 ? EVOC_FORM_BF16_RERANK : EVOC_FORM_EXACT_INT)
                : j->opts.form;
  j->work = 2.0 * double(n) * double(n) * double(dim);
  {
    evoc::CtxSizes bneed;
    const int64_t n1 = n, d1 = dim;
    // (the batched forms do not read the tau seed)
    j->batch_ok = n <= kBatchRows && evoc::batch_buffer_needs(j->opts, dtype, 1, &n1, &d1, k, &bneed);
  }
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
  out->batches = s->batches;
  out->batched = s->batched;
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
