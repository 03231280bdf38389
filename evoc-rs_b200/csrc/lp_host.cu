// C ABI of the label-propagation initialisation and the reproducible node
// embedding: argument checks, the caller's NumPy RNG draws (in the
// reference's order), device buffers, the recursion over reduced graphs,
// and dispatch to the kernels in label_prop.cu.
//
// Host logic restated from:
//   label_propagation_init_with_options  src/label_prop.rs:497-674 (recursive
//       or not; PCA, random, spectral or MDS base init below the threshold;
//       partition, jitter or node-embedding upscaling; the defaults are those
//       of label_propagation_init, src/label_prop.rs:464-494)
//   label_prop_loop                      src/label_prop.rs:160-185
//   node_embedding (reproducible)        src/embed.rs:251-369
//   NumpyRandomState randint / normal / shuffle
//                                        src/numpy_rng.rs:35-151, 204-212
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/evoc_gpu.h"
#include "ctx.h"
#include "lp.h"

namespace {

using evoc::cuda_fail;
using evoc::fail;
using evoc::Stage;
namespace lp = evoc::lp;

// ------------------------------------------------------------------ NumPy RandomState (MT19937)

struct Mt {
  evoc_numpy_rng* s;
  uint32_t tempered[624];  // outputs of the current key block, tempered once per block
  bool ready;

  // The 624-word state update, in place: words 0..226 mix with the old words
  // 397 ahead, words 227..622 with the new words 227 behind, word 623 with
  // the new word 396 (split so no index needs a modulo).
  void regen() {
    constexpr uint32_t kUp = 0x80000000u, kLo = 0x7fffffffu, kA = 0x9908b0dfu;
    uint32_t* k = s->key;
    auto mix = [&](int i, uint32_t next, uint32_t far) {
      const uint32_t y = (k[i] & kUp) | (next & kLo);
      k[i] = far ^ (y >> 1) ^ ((0u - (y & 1u)) & kA);
    };
    int i = 0;
    for (; i < 227; i++) mix(i, k[i + 1], k[i + 397]);
    for (; i < 623; i++) mix(i, k[i + 1], k[i - 227]);
    mix(623, k[0], k[396]);
    s->pos = 0;
  }
  void temper_block() {
    for (int i = 0; i < 624; i++) {
      uint32_t y = s->key[i];
      y ^= y >> 11;
      y ^= (y << 7) & 0x9d2c5680u;
      y ^= (y << 15) & 0xefc60000u;
      y ^= y >> 18;
      tempered[i] = y;
    }
    ready = true;
  }
  uint32_t next() {
    if (s->pos >= 624) {
      regen();
      temper_block();
    } else if (!ready) {
      temper_block();
    }
    return tempered[s->pos++];
  }
  // Masked rejection on 32-bit draws (ranges here stay below 2^32).
  uint64_t interval(uint64_t max) {
    if (max == 0) return 0;
    uint64_t mask = max;
    for (int sh = 1; sh < 64; sh <<= 1) mask |= mask >> sh;
    for (;;) {
      const uint64_t v = uint64_t(next()) & mask;
      if (v <= max) return v;
    }
  }
  int64_t randint(int64_t low, int64_t high) {
    const uint64_t range = uint64_t(high - low);
    return range == 0 ? low : low + int64_t(interval(range - 1));
  }
  double next_double() {
    const int32_t a = int32_t(next() >> 5), b = int32_t(next() >> 6);
    return (double(a) * 67108864.0 + double(b)) / 9007199254740992.0;
  }
  double normal() {
    if (s->has_gauss) {
      s->has_gauss = 0;
      const double t = s->gauss;
      s->gauss = 0.0;
      return t;
    }
    for (;;) {
      const double x1 = 2.0 * next_double() - 1.0, x2 = 2.0 * next_double() - 1.0;
      const double r2 = x1 * x1 + x2 * x2;
      if (r2 < 1.0 && r2 != 0.0) {
        const double f = std::sqrt(-2.0 * std::log(r2) / r2);
        s->gauss = f * x1;
        s->has_gauss = 1;
        return f * x2;
      }
    }
  }
  // randint3_for_tau: three draws in [i32::MIN + 1, i32::MAX - 1).
  void tau_seed(int64_t out[3]) {
    for (int j = 0; j < 3; j++) out[j] = randint(-2147483647LL, 2147483646LL);
  }
  // shuffle: for i = n-1 .. 1 swap a[i] with a[randint(0, i + 1)] -- the
  // draws of interval() inlined (n < 2^32 here, so 32-bit masks).
  void shuffle(uint32_t* a, int64_t n) {
    if (!ready && s->pos < 624) temper_block();
    int pos = s->pos;
    for (int64_t i = n - 1; i >= 1; i--) {
      const uint32_t mx = uint32_t(i);
      uint32_t m = mx;
      m |= m >> 1;
      m |= m >> 2;
      m |= m >> 4;
      m |= m >> 8;
      m |= m >> 16;
      uint32_t v;
      do {
        if (pos >= 624) {
          regen();
          temper_block();
          pos = 0;
        }
        v = tempered[pos++] & m;
      } while (v > mx);
      std::swap(a[i], a[v]);
    }
    s->pos = pos;
  }
};

// ------------------------------------------------------------------ stream-ordered device buffers

struct Arena {
  cudaStream_t s;
  cudaMemPool_t pool;
  std::vector<void*> ptrs;
  explicit Arena(evoc_gpu_ctx* ctx) : s(ctx->stream), pool(ctx->lp_pool) {}
  ~Arena() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
  template <class T>
  cudaError_t get(T** out, size_t count) {
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, std::max<size_t>(count, 1) * sizeof(T), pool, s);
    if (e != cudaSuccess) return e;
    ptrs.push_back(p);
    *out = static_cast<T*>(p);
    return cudaSuccess;
  }
};

constexpr int64_t kBaseInitThreshold = 64;  // src/label_prop.rs:489 default
constexpr int64_t kEigenMaxRows = 64;       // the one-block eigen-decompositions (PCA, spectral, MDS)
constexpr int32_t kMaxParts = 65536;        // parts fit the 16-bit fields of the sort keys
// Embedding rows above this many edges get a CTA each.  A block of few nodes
// (every node on its own warp) lasts as long as its longest row, so there the
// threshold is lower; a block of many nodes is bound by throughput instead.
constexpr int64_t kHeavyDegree = 512;
constexpr int64_t kHeavyDegreeSmallBlock = 128;
constexpr int64_t kSmallBlock = 32768;

struct Level {
  int32_t n_iter, n_epochs, ncomp;
  int64_t approx;
  float scaling, noise;
  float random_scale;
  evoc_lp_options opt;
};

int check_status(evoc_gpu_ctx* ctx, int32_t* d_status, const char* what);

// small_graph_init (src/label_prop.rs:425-447) on the level's rows.
int small_graph_init(evoc_gpu_ctx* ctx, Arena& A, int64_t n, const float* x, int64_t d, const Level& L, Mt& rng,
                     float* out) {
  cudaStream_t s = ctx->stream;
  if (L.opt.base_init == EVOC_BASE_INIT_RANDOM) {
    // n x n_components normal(1.0) draws in row order, rows L2-normalised
    std::vector<float> h(static_cast<size_t>(n) * size_t(L.ncomp));
    for (float& v : h) v = float(1.0 * rng.normal());
    Stage st(ctx, "random_init");
    EVOC_TRY(cudaMemcpyAsync(out, h.data(), h.size() * 4, cudaMemcpyHostToDevice, s), "upload draws");
    EVOC_TRY(lp::launch_unit_rows(out, n, L.ncomp, s), "random_init");
    ctx->launches += 1;
    EVOC_TRY(cudaStreamSynchronize(s), "random_init");
    return EVOC_OK;
  }
  if (!x) return fail(ctx, EVOC_ERR_ARG, "base_init 'pca' requires data");
  if (L.opt.base_init != EVOC_BASE_INIT_PCA) {
    Stage st(ctx, L.opt.base_init == EVOC_BASE_INIT_SPECTRAL ? "spectral_init" : "mds_init");
    EVOC_TRY(lp::launch_spectral_mds_init(x, n, d, L.ncomp, L.opt.base_init == EVOC_BASE_INIT_SPECTRAL ? 0 : 1, out,
                                          s),
             "spectral / mds init");
    ctx->launches += 1;
    EVOC_TRY(cudaStreamSynchronize(s), "spectral / mds init");
    return EVOC_OK;
  }
  float* mean_ws;
  double* vws;
  int32_t* status;
  EVOC_TRY(A.get(&mean_ws, size_t(d)), "alloc");
  EVOC_TRY(A.get(&vws, size_t(d)), "alloc");
  EVOC_TRY(A.get(&status, 1), "alloc");
  EVOC_TRY(cudaMemsetAsync(status, 0, 4, s), "memset");
  Stage st(ctx, "pca_init");
  EVOC_TRY(lp::launch_pca_init(x, n, d, L.ncomp, out, mean_ws, vws, status, s), "pca_init");
  ctx->launches += 1;
  st.end();
  return check_status(ctx, status, "pca_init");
}

int check_status(evoc_gpu_ctx* ctx, int32_t* d_status, const char* what) {
  int32_t st = 0;
  EVOC_TRY(cudaMemcpyAsync(&st, d_status, 4, cudaMemcpyDeviceToHost, ctx->stream), "status");
  EVOC_TRY(cudaStreamSynchronize(ctx->stream), what);
  if (st) return fail(ctx, EVOC_ERR_CUDA, std::string(what) + ": kernel check failed (" + std::to_string(st) + ")");
  return EVOC_OK;
}

int64_t read_i64(evoc_gpu_ctx* ctx, const int64_t* d, cudaError_t* err) {
  int64_t v = 0;
  *err = cudaMemcpyAsync(&v, d, 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (*err == cudaSuccess) *err = cudaStreamSynchronize(ctx->stream);
  return v;
}

// Row-overflow tables for the warp-per-row kernels: one table of max_deg
// slots per resident warp, only when some row can outgrow shared memory, and
// (keys below key_bound <= 65537) a direct key -> slot index per warp.
template <class Acc>
int overflow_tables(evoc_gpu_ctx* ctx, Arena& A, int64_t max_deg, int64_t key_bound, int32_t** key, Acc** sum,
                    int32_t** dix) {
  *key = nullptr;
  *sum = nullptr;
  *dix = nullptr;
  if (max_deg <= lp::kVoteSlots) return EVOC_OK;
  const size_t warps = size_t(ctx->sms) * lp::kRowWarps;
  EVOC_TRY(A.get(key, warps * size_t(max_deg)), "alloc overflow tables");
  EVOC_TRY(A.get(sum, warps * size_t(max_deg)), "alloc overflow tables");
  if (key_bound <= 65537) {
    EVOC_TRY(A.get(dix, warps * size_t(key_bound)), "alloc overflow index");
    EVOC_TRY(cudaMemsetAsync(*dix, 0xff, warps * size_t(key_bound) * 4, ctx->stream), "clear overflow index");
  }
  return EVOC_OK;
}

// label_prop_loop on a device graph: labels (int32, n) receive the partition.
int lp_loop_dev(evoc_gpu_ctx* ctx, Arena& A, const lp::Csr& g, Mt& rng, int32_t n_iter, int64_t approx,
                int32_t* labels, int32_t* n_parts_out) {
  cudaStream_t s = ctx->stream;
  int64_t rs[3];
  rng.tau_seed(rs);
  std::vector<int64_t> seeds(size_t(std::max<int64_t>(approx, 0)));
  for (auto& v : seeds) v = rng.randint(0, g.n);
  int64_t *d_rs, *d_seeds, *d_maxdeg;
  int32_t *tmp_lab, *overflow, *n_over, *status, *flags, *map, *d_nparts;
  EVOC_TRY(A.get(&d_rs, 3), "alloc");
  EVOC_TRY(A.get(&d_seeds, seeds.size()), "alloc");
  EVOC_TRY(A.get(&d_maxdeg, 1), "alloc");
  EVOC_TRY(A.get(&tmp_lab, size_t(g.n)), "alloc labels");
  EVOC_TRY(A.get(&overflow, size_t(g.n)), "alloc");
  EVOC_TRY(A.get(&n_over, 1), "alloc");
  EVOC_TRY(A.get(&status, 1), "alloc");
  EVOC_TRY(A.get(&d_nparts, 1), "alloc");
  EVOC_TRY(cudaMemsetAsync(status, 0, 4, s), "memset");
  EVOC_TRY(cudaMemcpyAsync(d_rs, rs, 24, cudaMemcpyHostToDevice, s), "upload tau seed");
  if (!seeds.empty())
    EVOC_TRY(cudaMemcpyAsync(d_seeds, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice, s), "upload seeds");
  EVOC_TRY(lp::launch_max_degree(g.indptr, g.n, d_maxdeg, s), "max degree");
  cudaError_t e;
  const int64_t max_deg = read_i64(ctx, d_maxdeg, &e);
  EVOC_TRY(e, "max degree");
  int32_t *okey, *odix;
  double* osum;
  const int64_t key_bound = std::max<int64_t>(approx, 1) + 1;  // labels -1 .. approx - 1
  if (int rc = overflow_tables(ctx, A, max_deg, key_bound, &okey, &osum, &odix)) return rc;
  {
    Stage st(ctx, "label_prop_iterations");
    EVOC_TRY(cudaMemsetAsync(labels, 0xff, size_t(g.n) * 4, s), "labels");
    EVOC_TRY(lp::launch_seed_labels(labels, d_seeds, int64_t(seeds.size()), s), "seed labels");
    ctx->launches += 1;
    int32_t* cur = labels;
    int32_t* nxt = tmp_lab;
    for (int32_t it = 0; it < n_iter; it++) {
      EVOC_TRY(lp::launch_lp_iteration(g, cur, nxt, overflow, n_over, okey, osum, max_deg, odix, key_bound, ctx->sms,
                                       s),
               "label_prop_iteration");
      ctx->launches += max_deg > lp::kVoteSlots ? 2 : 1;
      std::swap(cur, nxt);
    }
    if (cur != labels) EVOC_TRY(cudaMemcpyAsync(labels, cur, size_t(g.n) * 4, cudaMemcpyDeviceToDevice, s), "copy");
  }
  {
    Stage st(ctx, "label_outliers");
    lp::OutlierScratch ow{};
    const size_t nn = size_t(g.n);
    EVOC_TRY(A.get(&ow.flag, nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.rows, nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.oidx, nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.lab[0], nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.lab[1], nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.nxt[0], nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.nxt[1], nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.big, nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.walk, 2 * nn), "alloc outliers");
    EVOC_TRY(A.get(&ow.stacks, lp::outlier_stack_entries(ctx->sms)), "alloc outlier stacks");
    EVOC_TRY(A.get(&ow.big_stack, size_t(64 * max_deg + 1)), "alloc outlier stack");
    EVOC_TRY(A.get(&ow.count, 1), "alloc");
    EVOC_TRY(A.get(&ow.max_label, 1), "alloc");
    EVOC_TRY(A.get(&ow.n_big, 1), "alloc");
    EVOC_TRY(A.get(&ow.pending, 1), "alloc");
    ow.status = status;
    ow.tmp_bytes = lp::lp_outliers_tmp_bytes(g.n);
    uint8_t* otmp;
    EVOC_TRY(A.get(&otmp, ow.tmp_bytes), "alloc");
    ow.tmp = otmp;
    EVOC_TRY(lp::run_lp_outliers(g, labels, d_rs, ow, max_deg, ctx->sms, s), "label_outliers");
    ctx->launches += 8;
  }
  const int32_t bound = int32_t(std::max<int64_t>(approx, 1));
  EVOC_TRY(A.get(&flags, size_t(bound)), "alloc");
  EVOC_TRY(A.get(&map, size_t(bound)), "alloc");
  const size_t tb = lp::lp_remap_tmp_bytes(bound);
  void* tmp;
  EVOC_TRY(A.get(reinterpret_cast<uint8_t**>(&tmp), tb), "alloc");
  {
    Stage st(ctx, "remap_labels");
    EVOC_TRY(lp::launch_lp_remap(labels, g.n, bound, flags, map, d_nparts, status, tmp, tb, s), "remap_labels");
    ctx->launches += 3;
  }
  if (int rc = check_status(ctx, status, "label propagation")) return rc;
  EVOC_TRY(cudaMemcpyAsync(n_parts_out, d_nparts, 4, cudaMemcpyDeviceToHost, s), "n_parts");
  EVOC_TRY(cudaStreamSynchronize(s), "n_parts");
  return EVOC_OK;
}

// node_embedding(reproducible_flag = true) on a device graph.  emb (n x ncomp)
// holds the initial embedding (have_init) or receives normal(0.25) draws.
int node_embedding_dev(evoc_gpu_ctx* ctx, Arena& A, const lp::Csr& g, const float* weights, int32_t ncomp,
                       int32_t n_epochs, float* emb, bool have_init, float alpha0, float nsr, float noise, Mt& rng) {
  cudaStream_t s = ctx->stream;
  const int64_t n = g.n, m = g.nnz;
  if (!have_init) {
    std::vector<float> init(size_t(n * ncomp));
    for (auto& v : init) v = float(0.25 * rng.normal());
    EVOC_TRY(cudaMemcpyAsync(emb, init.data(), init.size() * 4, cudaMemcpyHostToDevice, s), "upload init");
    EVOC_TRY(cudaStreamSynchronize(s), "upload init");
  }
  float *eps, *epns, *eonn, *eons, *upd, *maxw;
  uint32_t *d_order, *heavy_rows;
  int32_t* heavy_count;
  EVOC_TRY(A.get(&eps, size_t(m)), "alloc schedule");
  EVOC_TRY(A.get(&epns, size_t(m)), "alloc schedule");
  EVOC_TRY(A.get(&eonn, size_t(m)), "alloc schedule");
  EVOC_TRY(A.get(&eons, size_t(m)), "alloc schedule");
  EVOC_TRY(A.get(&maxw, 1), "alloc");
  EVOC_TRY(A.get(&upd, size_t(n * ncomp)), "alloc updates");
  EVOC_TRY(A.get(&d_order, size_t(2 * n)), "alloc node order");
  EVOC_TRY(A.get(&heavy_rows, size_t(std::max<int64_t>(1024, n / 8))), "alloc heavy rows");
  EVOC_TRY(A.get(&heavy_count, 1), "alloc");
  EVOC_TRY(cudaMemsetAsync(upd, 0, size_t(n * ncomp) * 4, s), "memset updates");
  {
    Stage st(ctx, "epochs_per_sample");
    EVOC_TRY(lp::launch_ne_schedule(weights, m, n_epochs, nsr, 1.5f, eps, epns, eonn, eons, maxw, s), "schedule");
    ctx->launches += 2;
  }
  std::vector<uint32_t> seeds(size_t(std::max(n_epochs, 0)));
  for (auto& v : seeds) v = uint32_t(rng.randint(0, 2147483646LL));
  // Node orders: the host shuffles the next epoch's order while the device
  // runs the current one; two pinned slots, each reused once its upload ends.
  uint32_t* h_order = nullptr;
  EVOC_TRY(cudaMallocHost(&h_order, size_t(2 * n) * 4), "pinned order");
  cudaEvent_t up[2] = {nullptr, nullptr};
  auto cleanup = [&]() {
    for (auto& ev : up)
      if (ev) cudaEventDestroy(ev);
    cudaFreeHost(h_order);
  };
  for (auto& ev : up)
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      cleanup();
      return fail(ctx, EVOC_ERR_CUDA, "event create");
    }
  std::vector<uint32_t> order(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; i++) order[size_t(i)] = uint32_t(i);
  const int64_t block = std::max<int64_t>(1024, n / 8);
  float alpha = alpha0, decay = 1.0f;
  int rc = EVOC_OK;
  Stage st(ctx, "node_embedding_epochs");
  for (int32_t ep = 0; ep < n_epochs && rc == EVOC_OK; ep++) {
    const int slot = ep & 1;
    cudaError_t e = cudaEventSynchronize(up[slot]);
    if (e == cudaSuccess) {
      std::memcpy(h_order + size_t(slot) * n, order.data(), size_t(n) * 4);
      e = cudaMemcpyAsync(d_order + size_t(slot) * n, h_order + size_t(slot) * n, size_t(n) * 4,
                          cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) e = cudaEventRecord(up[slot], s);
    const float gamma = n_epochs <= 1 ? 1.0f : 0.5f + (float(ep) / float(n_epochs - 1)) * 1.0f;
    for (int64_t bs = 0; bs < n && e == cudaSuccess; bs += block) {
      const int64_t be = std::min(n, bs + block);
      e = lp::launch_ne_block(g, emb, upd, d_order + size_t(slot) * n, bs, be, eps, epns, eonn, eons,
                              seeds[size_t(ep)], ncomp, alpha, uint8_t(ep), noise, gamma, decay, ep > 0 ? 1 : 0,
                              be - bs < kSmallBlock ? kHeavyDegreeSmallBlock : kHeavyDegree, heavy_rows,
                              heavy_count, ctx->sms, s);
      if (e == cudaSuccess) e = lp::launch_ne_apply(emb, upd, d_order + size_t(slot) * n, bs, be, n, ncomp, s);
      ctx->launches += 3;
    }
    if (e != cudaSuccess) {
      rc = cuda_fail(ctx, e, "node embedding epoch");
      break;
    }
    const double om = 1.0 - double(alpha);
    decay = float(om * om * 0.5);
    rng.shuffle(order.data(), n);
    alpha = alpha0 * (1.0f - (float(ep) / float(n_epochs)));
  }
  st.end();
  cudaError_t e = cudaStreamSynchronize(s);
  cleanup();
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "node embedding");
  return EVOC_OK;
}

// node_embedding(reproducible_flag = false) on a device graph: the epochs of
// node_embedding_epoch (src/embed.rs:57-135) run lock-free on the device;
// same RNG draws as the reference (epoch seeds; no shuffles).
int node_embedding_hogwild_dev(evoc_gpu_ctx* ctx, Arena& A, const lp::Csr& g, int32_t ncomp, int32_t n_epochs,
                               float* emb, bool have_init, float alpha0, float nsr, float noise, Mt& rng) {
  cudaStream_t s = ctx->stream;
  const int64_t n = g.n, m = g.nnz;
  if (!have_init) {
    std::vector<float> init(static_cast<size_t>(n * ncomp));
    for (auto& v : init) v = float(0.25 * rng.normal());
    EVOC_TRY(cudaMemcpyAsync(emb, init.data(), init.size() * 4, cudaMemcpyHostToDevice, s), "upload init");
    EVOC_TRY(cudaStreamSynchronize(s), "upload init");
  }
  float *eps, *epns, *eonn, *eons, *maxw;
  uint32_t* head;
  EVOC_TRY(A.get(&eps, size_t(m)), "alloc schedule");
  EVOC_TRY(A.get(&epns, size_t(m)), "alloc schedule");
  EVOC_TRY(A.get(&eonn, size_t(m)), "alloc schedule");
  EVOC_TRY(A.get(&eons, size_t(m)), "alloc schedule");
  EVOC_TRY(A.get(&maxw, 1), "alloc");
  EVOC_TRY(A.get(&head, size_t(m)), "alloc edge rows");
  {
    Stage st(ctx, "epochs_per_sample");
    EVOC_TRY(lp::launch_ne_schedule(g.data, m, n_epochs, nsr, 1.0f, eps, epns, eonn, eons, maxw, s), "schedule");
    EVOC_TRY(lp::launch_edge_head(g.indptr, n, head, s), "edge rows");
    ctx->launches += 3;
  }
  std::vector<uint32_t> seeds(size_t(std::max(n_epochs, 0)));
  for (auto& v : seeds) v = uint32_t(rng.randint(0, 2147483646LL));
  float alpha = alpha0;
  Stage st(ctx, "node_embedding_epochs");
  for (int32_t ep = 0; ep < n_epochs; ep++) {
    EVOC_TRY(lp::launch_ne_hogwild(g, head, emb, eps, epns, eonn, eons, seeds[size_t(ep)], ncomp, alpha, uint8_t(ep),
                                   noise, ctx->sms, s),
             "node embedding epoch");
    ctx->launches += 1;
    alpha = alpha0 * (1.0f - (float(ep) / float(n_epochs)));
  }
  st.end();
  EVOC_TRY(cudaStreamSynchronize(s), "node embedding");
  return EVOC_OK;
}

// count normal(scale) draws in order, rounded to f32 (normal_scaled(..) as f32), into dev.
int upload_normals(evoc_gpu_ctx* ctx, int64_t count, double scale, Mt& rng, float* dev) {
  std::vector<float> h(static_cast<size_t>(count));
  for (float& v : h) v = float(scale * rng.normal());
  EVOC_TRY(cudaMemcpyAsync(dev, h.data(), h.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "upload draws");
  return EVOC_OK;
}

// One level of label_propagation_init_with_options (recursive on the reduced graph).
int lp_init_level(evoc_gpu_ctx* ctx, const lp::ReduceScratch& W, const lp::Csr& g, const float* x, int64_t d,
                  const Level& L, Mt& rng, float* out) {
  cudaStream_t s = ctx->stream;
  Arena A(ctx);
  if (g.n < L.opt.base_init_threshold) return small_graph_init(ctx, A, g.n, x, d, L, rng, out);
  int32_t* part;
  EVOC_TRY(A.get(&part, size_t(g.n)), "alloc partition");
  int32_t n_parts = 0;
  if (int rc = lp_loop_dev(ctx, A, g, rng, L.n_iter, L.approx, part, &n_parts)) return rc;
  if (n_parts > kMaxParts) return fail(ctx, EVOC_ERR_UNSUPPORTED, "more than 65536 label-propagation parts");
  // reduction maps
  int32_t *count, *members, *keys_tmp, *vals_tmp;
  int64_t* start;
  float *xnorm, *wred;
  EVOC_TRY(A.get(&count, size_t(n_parts)), "alloc");
  EVOC_TRY(A.get(&start, size_t(n_parts)), "alloc");
  EVOC_TRY(A.get(&members, size_t(g.n)), "alloc");
  EVOC_TRY(A.get(&keys_tmp, size_t(g.n)), "alloc");
  EVOC_TRY(A.get(&vals_tmp, size_t(g.n)), "alloc");
  EVOC_TRY(A.get(&xnorm, size_t(n_parts)), "alloc");
  EVOC_TRY(A.get(&wred, size_t(n_parts)), "alloc");
  {
    Stage st(ctx, "partition_maps");
    const size_t tb = lp::part_members_tmp_bytes(g.n, n_parts);
    uint8_t* tmp;
    EVOC_TRY(A.get(&tmp, tb), "alloc");
    EVOC_TRY(lp::launch_part_members(part, g.n, n_parts, count, start, members, xnorm, wred, tmp, tb, keys_tmp,
                                     vals_tmp, s),
             "partition maps");
    ctx->launches += 4;
  }
  float* rdata = nullptr;
  if (x) {
    Stage st(ctx, "reduced_data");
    EVOC_TRY(A.get(&rdata, size_t(n_parts) * size_t(d)), "alloc reduced data");
    EVOC_TRY(lp::launch_reduce_data(x, d, members, start, count, wred, n_parts, rdata, ctx->sms, s), "reduced data");
    ctx->launches += 1;
  }
  int64_t *r_indptr, *r_nnz;
  int32_t* r_indices;
  float* r_data;
  EVOC_TRY(A.get(&r_indptr, size_t(n_parts) + 1), "alloc reduced graph");
  EVOC_TRY(A.get(&r_indices, size_t(g.nnz)), "alloc reduced graph");
  EVOC_TRY(A.get(&r_data, size_t(g.nnz)), "alloc reduced graph");
  EVOC_TRY(A.get(&r_nnz, 1), "alloc");
  {
    Stage st(ctx, "reduced_graph");
    EVOC_TRY(lp::launch_reduce_graph(g, part, xnorm, n_parts, W, r_indptr, r_indices, r_data, r_nnz, s),
             "reduced graph");
    ctx->launches += 12;
  }
  cudaError_t e;
  const int64_t rnnz = read_i64(ctx, r_nnz, &e);
  EVOC_TRY(e, "reduced graph");
  const lp::Csr red{r_indptr, r_indices, r_data, n_parts, rnnz};
  float* rinit;
  EVOC_TRY(A.get(&rinit, size_t(n_parts) * L.ncomp), "alloc reduced init");
  Level sub = L;
  sub.n_epochs = std::min(L.n_epochs, 255);
  sub.approx = L.approx / 4;
  if (L.opt.recursive_init)
    if (int rc = lp_init_level(ctx, W, red, rdata, d, sub, rng, rinit)) return rc;
  // reduced layout: node_embedding of the reduced graph from the recursive
  // init, or from normal(0.25) draws without one
  if (int rc = node_embedding_dev(ctx, A, red, r_data, L.ncomp, L.n_epochs, rinit, L.opt.recursive_init != 0,
                                  0.001f * float(L.n_epochs), 1.0f, L.noise, rng))
    return rc;
  if (L.opt.upscaling == EVOC_UPSCALE_NODE_EMBEDDING) {
    // the part layout plus normal(random_scale) draws, row order
    float *result, *noise;
    double* mean;
    EVOC_TRY(A.get(&result, size_t(g.n) * L.ncomp), "alloc");
    EVOC_TRY(A.get(&noise, size_t(g.n) * L.ncomp), "alloc");
    EVOC_TRY(A.get(&mean, size_t(L.ncomp)), "alloc");
    if (int rc = upload_normals(ctx, g.n * L.ncomp, double(L.random_scale), rng, noise)) return rc;
    Stage st(ctx, "upscale_and_scale");
    EVOC_TRY(lp::launch_upscale(result, part, rinit, noise, g.n, L.ncomp, 0, s), "node-embedding upscaler");
    EVOC_TRY(lp::launch_center_scale(result, g.n, L.ncomp, L.scaling, out, mean, s), "centre and scale");
    ctx->launches += 3;
    st.end();
    EVOC_TRY(cudaStreamSynchronize(s), "label propagation level");
    return EVOC_OK;
  }
  // partition expander (the jitter expander starts from it)
  int64_t *s_indptr, *s_nnz, *d_maxdeg;
  int32_t *s_indices, *overflow, *n_over;
  float *s_data, *result;
  double* mean;
  EVOC_TRY(A.get(&s_indptr, size_t(g.n) + 1), "alloc");
  EVOC_TRY(A.get(&s_indices, size_t(g.nnz)), "alloc");
  EVOC_TRY(A.get(&s_data, size_t(g.nnz)), "alloc");
  EVOC_TRY(A.get(&s_nnz, 1), "alloc");
  EVOC_TRY(A.get(&d_maxdeg, 1), "alloc");
  EVOC_TRY(A.get(&overflow, size_t(g.n)), "alloc");
  EVOC_TRY(A.get(&n_over, 1), "alloc");
  EVOC_TRY(A.get(&result, size_t(g.n) * L.ncomp), "alloc");
  EVOC_TRY(A.get(&mean, size_t(L.ncomp)), "alloc");
  {
    Stage st(ctx, "hadamard_symmetric");
    EVOC_TRY(lp::launch_hadamard_sym(g, W, s_indptr, s_indices, s_data, s_nnz, s), "hadamard_symmetric");
    ctx->launches += 6;
  }
  const int64_t snnz = read_i64(ctx, s_nnz, &e);
  EVOC_TRY(e, "hadamard_symmetric");
  const lp::Csr sym{s_indptr, s_indices, s_data, g.n, snnz};
  EVOC_TRY(lp::launch_max_degree(s_indptr, g.n, d_maxdeg, s), "max degree");
  const int64_t max_deg = read_i64(ctx, d_maxdeg, &e);
  EVOC_TRY(e, "max degree");
  int32_t *okey, *odix;
  float* osum;
  if (int rc = overflow_tables(ctx, A, max_deg, n_parts, &okey, &osum, &odix)) return rc;
  {
    Stage st(ctx, "expand_and_scale");
    EVOC_TRY(lp::launch_expand(sym, part, xnorm, rinit, L.ncomp, result, overflow, n_over, okey, osum, max_deg, odix,
                               n_parts, ctx->sms, s),
             "partition expander");
    ctx->launches += max_deg > lp::kVoteSlots ? 2 : 1;
  }
  if (L.opt.upscaling == EVOC_UPSCALE_JITTER_EXPANDER) {
    // averaged with the part layout plus normal(random_scale / 4) draws
    float* noise;
    EVOC_TRY(A.get(&noise, size_t(g.n) * L.ncomp), "alloc");
    if (int rc = upload_normals(ctx, g.n * L.ncomp, double(L.random_scale / 4.0f), rng, noise)) return rc;
    EVOC_TRY(lp::launch_upscale(result, part, rinit, noise, g.n, L.ncomp, 1, s), "jitter expander");
    ctx->launches += 1;
  }
  {
    Stage st(ctx, "centre_and_scale");
    EVOC_TRY(lp::launch_center_scale(result, g.n, L.ncomp, L.scaling, out, mean, s), "centre and scale");
    ctx->launches += 2;
  }
  EVOC_TRY(cudaStreamSynchronize(s), "label propagation level");
  return EVOC_OK;
}

// Caller's graph on the device: copies host arrays in, or wraps device ones.
int stage_graph(evoc_gpu_ctx* ctx, Arena& A, const int64_t* indptr, const int32_t* indices, const float* data,
                int64_t n, int32_t on_dev, lp::Csr* g) {
  cudaStream_t s = ctx->stream;
  int64_t nnz = 0;
  int32_t* bad;
  EVOC_TRY(A.get(&bad, 1), "alloc");
  if (on_dev) {
    cudaError_t e;
    nnz = read_i64(ctx, indptr + n, &e);
    EVOC_TRY(e, "read nnz");
    if (nnz < 0 || (nnz > 0 && (!indices || !data))) return fail(ctx, EVOC_ERR_ARG, "bad CSR arrays");
    *g = lp::Csr{indptr, indices, data, n, nnz};
    EVOC_TRY(lp::launch_validate_csr(*g, bad, s), "validate graph");
    return check_status(ctx, bad, "graph is not a valid square CSR") ? EVOC_ERR_ARG : EVOC_OK;
  }
  nnz = indptr[n];
  if (nnz < 0 || (nnz > 0 && (!indices || !data))) return fail(ctx, EVOC_ERR_ARG, "bad CSR arrays");
  int64_t* d_ip;
  int32_t* d_ix;
  float* d_dt;
  EVOC_TRY(A.get(&d_ip, size_t(n) + 1), "alloc graph");
  EVOC_TRY(A.get(&d_ix, size_t(nnz)), "alloc graph");
  EVOC_TRY(A.get(&d_dt, size_t(nnz)), "alloc graph");
  EVOC_TRY(cudaMemcpyAsync(d_ip, indptr, size_t(n + 1) * 8, cudaMemcpyHostToDevice, s), "upload indptr");
  if (nnz) {
    EVOC_TRY(cudaMemcpyAsync(d_ix, indices, size_t(nnz) * 4, cudaMemcpyHostToDevice, s), "upload indices");
    EVOC_TRY(cudaMemcpyAsync(d_dt, data, size_t(nnz) * 4, cudaMemcpyHostToDevice, s), "upload data");
  }
  *g = lp::Csr{d_ip, d_ix, d_dt, n, nnz};
  EVOC_TRY(lp::launch_validate_csr(*g, bad, s), "validate graph");
  return check_status(ctx, bad, "graph is not a valid square CSR") ? EVOC_ERR_ARG : EVOC_OK;
}

int begin_call(evoc_gpu_ctx* ctx) {
  ctx->err.clear();
  ctx->n_stages = 0;
  ctx->launches = 0;
  EVOC_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  if (!ctx->lp_pool) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    EVOC_TRY(cudaMemPoolCreate(&ctx->lp_pool, &props), "memory pool");
    uint64_t keep = UINT64_MAX;
    EVOC_TRY(cudaMemPoolSetAttribute(ctx->lp_pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool");
  }
  return EVOC_OK;
}

int label_propagation_init_impl(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices, const float* data,
                                int64_t n, int32_t n_iter, int32_t n_epochs, int64_t approx, int32_t ncomp,
                                float scaling, float random_scale, float noise, evoc_numpy_rng* rs, const float* x,
                                int64_t dim, int32_t on_dev, const evoc_lp_options& opt, float* out) {
  if (int rc = begin_call(ctx)) return rc;
  if (opt.base_init < EVOC_BASE_INIT_PCA || opt.base_init > EVOC_BASE_INIT_MDS)
    return fail(ctx, EVOC_ERR_ARG, "unknown base_init");
  if (opt.upscaling < EVOC_UPSCALE_PARTITION_EXPANDER || opt.upscaling > EVOC_UPSCALE_NODE_EMBEDDING)
    return fail(ctx, EVOC_ERR_ARG, "unknown upscaling");
  if (opt.base_init_threshold < 0) return fail(ctx, EVOC_ERR_ARG, "negative base_init_threshold");
  if (opt.base_init != EVOC_BASE_INIT_RANDOM && opt.base_init_threshold > kEigenMaxRows + 1)
    return fail(ctx, EVOC_ERR_UNSUPPORTED,
                "base_init_threshold above 65 with the pca, spectral or mds base init (one-block "
                "eigen-decompositions of at most 64 rows)");
  if (n <= 0) return fail(ctx, EVOC_ERR_EMPTY, "empty graph");
  if (!indptr || !rs || !out) return fail(ctx, EVOC_ERR_ARG, "null argument");
  if (ncomp < 1 || ncomp > lp::kMaxComponents) return fail(ctx, EVOC_ERR_UNSUPPORTED, "n_components must be 1..32");
  if (x && dim <= 0) return fail(ctx, EVOC_ERR_ARG, "data dimension must be positive");
  if (n_iter < 0 || n_epochs < 0 || approx < 0) return fail(ctx, EVOC_ERR_ARG, "negative count");
  cudaStream_t s = ctx->stream;
  Mt rng{rs, {}, false};
  Stage total(ctx, "total");
  int rc;
  {
    Arena A(ctx);
    lp::Csr g;
    if ((rc = stage_graph(ctx, A, indptr, indices, data, n, on_dev, &g))) return rc;
    if (g.nnz >= (int64_t(1) << 31) - 1) return fail(ctx, EVOC_ERR_UNSUPPORTED, "graphs of 2^31 or more entries");
    const float* d_x = x;
    if (x && !on_dev) {
      float* p;
      EVOC_TRY(A.get(&p, size_t(n) * size_t(dim)), "alloc data");
      EVOC_TRY(cudaMemcpyAsync(p, x, size_t(n) * size_t(dim) * 4, cudaMemcpyHostToDevice, s), "upload data");
      d_x = p;
    }
    float* d_out = out;
    if (!on_dev) EVOC_TRY(A.get(&d_out, size_t(n) * size_t(ncomp)), "alloc output");
    // one sort scratch for every level (the top level is the largest)
    lp::ReduceScratch W{};
    const size_t cap = size_t(std::max<int64_t>(g.nnz, 1));
    W.tmp_bytes = std::max(lp::reduce_sort_tmp_bytes(int64_t(cap)), size_t(1));
    EVOC_TRY(A.get(&W.k0, cap), "alloc sort scratch");
    EVOC_TRY(A.get(&W.k1, cap), "alloc sort scratch");
    EVOC_TRY(A.get(&W.v0, cap), "alloc sort scratch");
    EVOC_TRY(A.get(&W.v1, cap), "alloc sort scratch");
    EVOC_TRY(A.get(&W.v2, cap), "alloc sort scratch");
    EVOC_TRY(A.get(&W.v3, cap), "alloc sort scratch");
    EVOC_TRY(A.get(&W.head, cap + 1), "alloc sort scratch");
    EVOC_TRY(A.get(&W.pos, cap + 1), "alloc sort scratch");
    EVOC_TRY(A.get(&W.rcount, size_t(n) + 2), "alloc sort scratch");
    EVOC_TRY(A.get(&W.counter, 4), "alloc sort scratch");
    EVOC_TRY(A.get(reinterpret_cast<uint8_t**>(&W.tmp), W.tmp_bytes), "alloc sort scratch");
    Level L{n_iter, n_epochs, ncomp, approx, scaling, noise, random_scale, opt};
    if ((rc = lp_init_level(ctx, W, g, d_x, dim, L, rng, d_out))) return rc;
    if (!on_dev)
      EVOC_TRY(cudaMemcpyAsync(out, d_out, size_t(n) * size_t(ncomp) * 4, cudaMemcpyDeviceToHost, s), "download");
  }
  EVOC_TRY(cudaStreamSynchronize(s), "label_propagation_init");
  return EVOC_OK;
}

int node_embedding_impl(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices, const float* data,
                        int64_t n, int32_t ncomp, int32_t n_epochs, const float* initial, float alpha0, float nsr,
                        float noise, evoc_numpy_rng* rs, int32_t reproducible, int32_t on_dev, float* out) {
  if (int rc = begin_call(ctx)) return rc;
  if (n <= 0) return fail(ctx, EVOC_ERR_EMPTY, "empty graph");
  if (!indptr || !rs || !out) return fail(ctx, EVOC_ERR_ARG, "null argument");
  if (ncomp < 1 || ncomp > lp::kMaxComponents) return fail(ctx, EVOC_ERR_UNSUPPORTED, "n_components must be 1..32");
  if (n_epochs < 0) return fail(ctx, EVOC_ERR_ARG, "negative n_epochs");
  if (n > (int64_t(1) << 31) - 1) return fail(ctx, EVOC_ERR_UNSUPPORTED, "2^31 or more vertices");
  cudaStream_t s = ctx->stream;
  Mt rng{rs, {}, false};
  Stage total(ctx, "total");
  {
    Arena A(ctx);
    lp::Csr g;
    if (int rc = stage_graph(ctx, A, indptr, indices, data, n, on_dev, &g)) return rc;
    if (g.nnz > (int64_t(1) << 32) - 1) return fail(ctx, EVOC_ERR_UNSUPPORTED, "2^32 or more edges");
    float* d_out = out;
    if (!on_dev) EVOC_TRY(A.get(&d_out, size_t(n) * size_t(ncomp)), "alloc output");
    if (initial)
      EVOC_TRY(cudaMemcpyAsync(d_out, initial, size_t(n) * size_t(ncomp) * 4,
                               on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s),
               "initial embedding");
    const int rc = reproducible ? node_embedding_dev(ctx, A, g, g.data, ncomp, n_epochs, d_out, initial != nullptr,
                                                     alpha0, nsr, noise, rng)
                                : node_embedding_hogwild_dev(ctx, A, g, ncomp, n_epochs, d_out, initial != nullptr,
                                                             alpha0, nsr, noise, rng);
    if (rc) return rc;
    if (!on_dev)
      EVOC_TRY(cudaMemcpyAsync(out, d_out, size_t(n) * size_t(ncomp) * 4, cudaMemcpyDeviceToHost, s), "download");
  }
  EVOC_TRY(cudaStreamSynchronize(s), "node_embedding");
  return EVOC_OK;
}

int label_prop_loop_impl(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices, const float* data,
                         int64_t n, int32_t n_iter, int64_t approx, evoc_numpy_rng* rs, int32_t on_dev,
                         int64_t* labels, int64_t* n_parts) {
  if (int rc = begin_call(ctx)) return rc;
  if (n <= 0) return fail(ctx, EVOC_ERR_EMPTY, "empty graph");
  if (!indptr || !rs || !labels) return fail(ctx, EVOC_ERR_ARG, "null argument");
  if (n_iter < 0 || approx < 0) return fail(ctx, EVOC_ERR_ARG, "negative count");
  if (approx > (int64_t(1) << 31) - 1) return fail(ctx, EVOC_ERR_UNSUPPORTED, "approx_n_parts above 2^31 - 1");
  cudaStream_t s = ctx->stream;
  Mt rng{rs, {}, false};
  Stage total(ctx, "total");
  {
    Arena A(ctx);
    lp::Csr g;
    if (int rc = stage_graph(ctx, A, indptr, indices, data, n, on_dev, &g)) return rc;
    int32_t* part;
    EVOC_TRY(A.get(&part, size_t(n)), "alloc partition");
    int32_t np = 0;
    if (int rc = lp_loop_dev(ctx, A, g, rng, n_iter, approx, part, &np)) return rc;
    std::vector<int32_t> h(static_cast<size_t>(n));
    EVOC_TRY(cudaMemcpyAsync(h.data(), part, size_t(n) * 4, cudaMemcpyDeviceToHost, s), "download partition");
    EVOC_TRY(cudaStreamSynchronize(s), "label_prop_loop");
    if (on_dev) {
      std::vector<int64_t> h64(h.begin(), h.end());
      EVOC_TRY(cudaMemcpy(labels, h64.data(), size_t(n) * 8, cudaMemcpyHostToDevice), "upload labels");
    } else {
      for (int64_t i = 0; i < n; i++) labels[i] = h[size_t(i)];
    }
    if (n_parts) *n_parts = np;
  }
  EVOC_TRY(cudaStreamSynchronize(s), "label_prop_loop");
  return EVOC_OK;
}

}  // namespace

extern "C" {

int evoc_gpu_label_prop_loop(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices, const float* data,
                             int64_t n, int32_t n_iter, int64_t approx_n_parts, evoc_numpy_rng* rng,
                             int32_t buffers_on_device, int64_t* labels, int64_t* n_parts) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  return label_prop_loop_impl(ctx, indptr, indices, data, n, n_iter, approx_n_parts, rng, buffers_on_device, labels,
                              n_parts);
}

int evoc_gpu_label_propagation_init(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices,
                                    const float* data, int64_t n, int32_t n_label_prop_iter,
                                    int32_t n_embedding_epochs, int64_t approx_n_parts, int32_t n_components,
                                    float scaling, float random_scale, float noise_level, evoc_numpy_rng* rng,
                                    const float* x, int64_t dim, int32_t buffers_on_device, float* out) {
  return evoc_gpu_label_propagation_init_with_options(ctx, indptr, indices, data, n, n_label_prop_iter,
                                                      n_embedding_epochs, approx_n_parts, n_components, scaling,
                                                      random_scale, noise_level, rng, x, dim, buffers_on_device,
                                                      nullptr, out);
}

void evoc_lp_options_default(evoc_lp_options* o) {
  if (!o) return;
  *o = evoc_lp_options{};
  o->recursive_init = 1;
  o->base_init = EVOC_BASE_INIT_PCA;
  o->base_init_threshold = kBaseInitThreshold;
  o->upscaling = EVOC_UPSCALE_PARTITION_EXPANDER;
}

int evoc_gpu_label_propagation_init_with_options(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices,
                                                 const float* data, int64_t n, int32_t n_label_prop_iter,
                                                 int32_t n_embedding_epochs, int64_t approx_n_parts,
                                                 int32_t n_components, float scaling, float random_scale,
                                                 float noise_level, evoc_numpy_rng* rng, const float* x, int64_t dim,
                                                 int32_t buffers_on_device, const evoc_lp_options* options,
                                                 float* out) {
  if (!ctx) return EVOC_ERR_ARG;
  evoc_lp_options opt;
  evoc_lp_options_default(&opt);
  if (options) opt = *options;
  std::lock_guard<std::mutex> lock(ctx->mu);
  return label_propagation_init_impl(ctx, indptr, indices, data, n, n_label_prop_iter, n_embedding_epochs,
                                     approx_n_parts, n_components, scaling, random_scale, noise_level, rng, x, dim,
                                     buffers_on_device, opt, out);
}

int evoc_gpu_node_embedding(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices, const float* data,
                            int64_t n, int32_t n_components, int32_t n_epochs, const float* initial_embedding,
                            float initial_alpha, float negative_sample_rate, float noise_level, evoc_numpy_rng* rng,
                            int32_t reproducible, int32_t buffers_on_device, float* out) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  return node_embedding_impl(ctx, indptr, indices, data, n, n_components, n_epochs, initial_embedding, initial_alpha,
                             negative_sample_rate, noise_level, rng, reproducible, buffers_on_device, out);
}

}  // extern "C"
