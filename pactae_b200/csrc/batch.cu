// batch.cu -- the batch ABI: many instances in one persistent launch,
// captured as a CUDA graph, and the one-launch-per-instance baseline.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>
#include <vector>

#include "batch_kernels.cuh"
#include "common.cuh"
#include "internal.h"

using namespace smpb200;

static_assert(sizeof(smp_instance) == sizeof(BatchInstance), "smp_instance mirrors the device table row");
static_assert(offsetof(smp_instance, n) == offsetof(BatchInstance, n), "layout");
static_assert(offsetof(smp_instance, proposals) == offsetof(BatchInstance, proposals), "layout");

struct smp_batch {
  smp_ctx *ctx = nullptr;
  int count = 0;
  int max_n = 0;
  int block = 512;
  int grid = 0;
  int subs = 8;
  int per_sm = 2;
  int rank_kb = 64;        // shared rank region per CTA (KB)
  int rank_smem_elems = 0;
  bool tuned = false;      // the autotuner chose the shape
  bool use_graph = true;
  size_t slab_elems = 0;
  size_t smem = 0;
  DeviceBuf d_table, d_order, d_queue, d_slabs;
  std::vector<int32_t> order;
  std::vector<smp_instance> inst;   // the table as given (pointers, n)
  smp_instance *h_table = nullptr;  // pinned copy for results
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Instances with n above threshold_n -- the first `routed` of order[] --
  // run the single-instance pipeline on the lanes, contexts with their own
  // streams, forked from the batch's stream while the persistent kernel
  // takes the rest, and joined before the table is read back.
  int threshold_n = -1;  // -1: none routed
  int routed = 0;
  bool thr_tuned = false;
  std::vector<smp_ctx *> lanes;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
};

namespace {

// Total scratch the rank slabs of one batch may take.
constexpr size_t kSlabBudget = 24ull << 30;
// Routed instances are dealt to this many single-instance pipelines.
constexpr int kRouteLanes = 4;
// Instances of at most this n are never routed: their pipeline is all launch
// latency.
constexpr int kRouteMinN = 1024;

int subs_for_window(int window) {
  if (window <= 0) return 8;
  if (window <= 32) return 1;
  if (window <= 64) return 2;
  if (window <= 128) return 4;
  return 8;
}

template <int kSub>
int launch_batch_t(smp_batch &b, cudaStream_t s, int grid, const int32_t *order, int count, int dynamic,
                   BatchInstance *table) {
  k_batch<kSub><<<grid, b.block, b.smem, s>>>(table, order, count, b.d_queue.as<int>(), b.d_slabs.as<uint16_t>(),
                                              b.slab_elems, b.max_n, dynamic, b.rank_smem_elems);
  return b.ctx->c.check_launch("k_batch");
}

// Dynamic shared memory of the chosen kernel (set before any capture).
int set_batch_attribute(smp_batch &b) {
  const Ctx &c = b.ctx->c;
  cudaError_t e;
  switch (b.subs) {
    case 1: e = allow_dynamic_smem(c, k_batch<1>); break;
    case 2: e = allow_dynamic_smem(c, k_batch<2>); break;
    case 4: e = allow_dynamic_smem(c, k_batch<4>); break;
    default: e = allow_dynamic_smem(c, k_batch<8>); break;
  }
  return e == cudaSuccess ? SMP_OK : b.ctx->c.fail_cuda("k_batch smem attribute");
}

int launch_batch(smp_batch &b, cudaStream_t s, int grid, const int32_t *order, int count, int dynamic,
                 BatchInstance *table = nullptr) {
  if (!table) table = b.d_table.as<BatchInstance>();
  switch (b.subs) {
    case 1: return launch_batch_t<1>(b, s, grid, order, count, dynamic, table);
    case 2: return launch_batch_t<2>(b, s, grid, order, count, dynamic, table);
    case 4: return launch_batch_t<4>(b, s, grid, order, count, dynamic, table);
    default: return launch_batch_t<8>(b, s, grid, order, count, dynamic, table);
  }
}

// ---------------------------------------------------------------------------
// Shapes and the autotuner.  A shape is the CTA size, CTAs per SM, the
// look-ahead window and the shared rank region (the size threshold below
// which an instance's rank matrix stays on chip: n*n*2 bytes must fit).  The
// kernel is compiled for at most 64 registers (two 512-thread CTAs per SM),
// so block * ctas_per_sm <= 1024.
// ---------------------------------------------------------------------------
struct Shape {
  int block, per_sm, subs, rank_kb;
};

size_t shape_smem(int max_n, int rank_kb) {
  return batch_smem_bytes(max_n) + static_cast<size_t>(std::max(rank_kb, 0)) * 1024;
}

bool shape_fits(const Ctx &c, int max_n, const Shape &sh) {
  const size_t smem = shape_smem(max_n, sh.rank_kb);
  int per_sm_bytes = 0;
  cudaDeviceGetAttribute(&per_sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c.device);
  return smem <= c.smem_optin && static_cast<size_t>(sh.per_sm) * (smem + 1024) <= static_cast<size_t>(per_sm_bytes) &&
         sh.block * sh.per_sm <= 1024 && sh.block >= 64 && sh.block <= 512;
}

int apply_shape(smp_batch &b, const Shape &sh) {
  const Ctx &c = b.ctx->c;
  b.block = sh.block;
  b.per_sm = sh.per_sm;
  b.subs = sh.subs;
  b.rank_kb = sh.rank_kb;
  b.rank_smem_elems = sh.rank_kb > 0 ? sh.rank_kb * 512 : 0;
  b.smem = shape_smem(b.max_n, sh.rank_kb);
  const size_t slab_bytes = b.slab_elems * sizeof(uint16_t);
  const int by_budget = static_cast<int>(std::max<size_t>(1, kSlabBudget / slab_bytes));
  b.grid = std::max(1, std::min({c.sm_count * std::min(sh.per_sm, 4), by_budget, b.count}));
  return set_batch_attribute(b);
}

// Tuned shapes, per device, largest n and batch size (powers of two).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, Shape> g_tuned;
std::map<std::tuple<int, int, int>, int> g_tuned_thr;

// Runs the kernel over the sample table and returns its device time.
float time_shape(smp_batch &b, const Shape &sh, BatchInstance *sample, const int32_t *order, int k) {
  if (apply_shape(b, sh)) return 1e30f;
  Ctx &c = b.ctx->c;
  float best = 1e30f;
  for (int rep = 0; rep < 1; ++rep) {
    if (cudaMemsetAsync(b.d_queue.ptr, 0, sizeof(int), c.stream) != cudaSuccess ||
        cudaEventRecord(b.ev0, c.stream) != cudaSuccess ||
        launch_batch(b, c.stream, std::min(b.grid, k), order, k, 1, sample) != SMP_OK ||
        cudaEventRecord(b.ev1, c.stream) != cudaSuccess || cudaStreamSynchronize(c.stream) != cudaSuccess) {
      cudaGetLastError();
      return 1e30f;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b.ev0, b.ev1);
    best = std::min(best, ms);
  }
  return best;
}

// Coordinate descent over the shapes, timed on the batch itself (a sample
// would not do: the largest instances sit on single CTAs, and a sample's
// time is their span rather than the batch's throughput): window, then CTA
// size and count, then the shared rank region.  Fields the caller fixed are
// not searched.  Each candidate costs one batched run.
Shape autotune(smp_batch &b, Shape start, const smp_batch_cfg *cfg) {
  Ctx &c = b.ctx->c;
  BatchInstance *sample = b.d_table.as<BatchInstance>();
  const int32_t *order = b.d_order.as<int32_t>();
  const int k = b.count;
  Shape best = start;
  time_shape(b, best, sample, order, k);  // warm-up
  float best_t = time_shape(b, best, sample, order, k);
  const auto consider = [&](Shape sh) {
    if (!shape_fits(c, b.max_n, sh)) return;
    const float ms = time_shape(b, sh, sample, order, k);
    if (ms < best_t) {
      best_t = ms;
      best = sh;
    }
  };
  if (!(cfg && cfg->window > 0))
    for (int subs : {1, 2, 4, 8}) consider({best.block, best.per_sm, subs, best.rank_kb});
  if (!(cfg && (cfg->block_threads > 0 || cfg->ctas_per_sm > 0)))
    for (auto bp : {std::pair<int, int>{512, 1}, {512, 2}, {256, 2}, {256, 4}})
      consider({bp.first, bp.second, best.subs, best.rank_kb});
  if (!(cfg && cfg->rank_smem_kb != 0))
    for (int kb : {0, 32, 64}) consider({best.block, best.per_sm, best.subs, kb});
  return best;
}

// An instance the batch routed to the single-instance pipeline: its status
// and proposal count, from that pipeline's control block, into its table row
// (one thread; enqueued after the pipeline on the same stream).
__global__ void k_route_report(const Control *__restrict__ ctrl, BatchInstance *__restrict__ table, int idx) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int status = ctrl->status;
  table[idx].status = status;
  table[idx].proposals = status ? 0ull : ctrl->proposals;
}

// How many instances (largest first) have n above thr.
int routed_count(const smp_batch &b, int thr) {
  if (thr <= 0) return 0;
  int r = 0;
  while (r < b.count && b.inst[b.order[r]].n > thr) ++r;
  return r;
}

// Routes the instances above thr (thr <= 0: none).  The lanes are created on
// first use with every buffer a solve of the largest routed n takes, so that
// a captured step allocates nothing.
int set_threshold(smp_batch &b, int thr) {
  Ctx &c = b.ctx->c;
  b.threshold_n = thr > 0 ? thr : -1;
  b.routed = routed_count(b, thr);
  if (!b.routed) return SMP_OK;
  if (!b.ev_fork && cudaEventCreateWithFlags(&b.ev_fork, cudaEventDisableTiming) != cudaSuccess)
    return c.fail_cuda("route event");
  while (static_cast<int>(b.lanes.size()) < kRouteLanes) {
    smp_cfg lc = {};
    lc.device = c.device;
    smp_ctx *x = nullptr;
    int rc = smp_b200_create(&x, &lc);
    if (rc) return rc;
    b.lanes.push_back(x);
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return c.fail_cuda("route event");
    b.ev_join.push_back(e);
  }
  const int top = b.inst[b.order[0]].n;
  for (smp_ctx *x : b.lanes) {
    const int rc = reserve_buffers(x->c, top);
    if (rc) {
      c.last_error = x->c.last_error;
      return rc;
    }
  }
  return SMP_OK;
}

// The batched step: reset the queue; fork the routed instances to the lanes
// (each solve followed by k_route_report into its table row); run the
// persistent kernel on the rest; join; copy the table (statuses, proposals)
// back to pinned host memory.
int enqueue_step(smp_batch &b, cudaStream_t s) {
  Ctx &c = b.ctx->c;
  if (cudaMemsetAsync(b.d_queue.ptr, 0, sizeof(int), s) != cudaSuccess) return c.fail_cuda("queue reset");
  int rc = SMP_OK;
  const int lanes = std::min(b.routed, static_cast<int>(b.lanes.size()));
  if (lanes > 0) {
    if (cudaEventRecord(b.ev_fork, s) != cudaSuccess) return c.fail_cuda("route fork");
    for (int l = 0; l < lanes; ++l)
      if (cudaStreamWaitEvent(b.lanes[l]->c.stream, b.ev_fork, 0) != cudaSuccess) return c.fail_cuda("route fork");
    for (int k = 0; !rc && k < b.routed; ++k) {
      Ctx &lc = b.lanes[k % lanes]->c;
      const int i = b.order[k];
      const smp_instance &in = b.inst[i];
      rc = solve_enqueue(lc, in.pref_m, in.pref_w, in.n, in.match, SMP_F_DEVICE_PTRS);
      if (!rc) {
        k_route_report<<<1, 32, 0, lc.stream>>>(lc.d_ctrl.as<Control>(), b.d_table.as<BatchInstance>(), i);
        rc = lc.check_launch("k_route_report");
      }
      if (rc) c.last_error = lc.last_error;
    }
  }
  if (!rc && b.count > b.routed)
    rc = launch_batch(b, s, std::min(b.grid, b.count - b.routed), b.d_order.as<int32_t>() + b.routed,
                      b.count - b.routed, 1);
  // join every lane, even after an error: a capture must end joined
  for (int l = 0; l < lanes; ++l)
    if ((cudaEventRecord(b.ev_join[l], b.lanes[l]->c.stream) != cudaSuccess ||
         cudaStreamWaitEvent(s, b.ev_join[l], 0) != cudaSuccess) &&
        !rc)
      rc = c.fail_cuda("route join");
  if (rc) return rc;
  if (cudaMemcpyAsync(b.h_table, b.d_table.ptr, sizeof(smp_instance) * b.count, cudaMemcpyDeviceToHost, s) !=
      cudaSuccess)
    return c.fail_cuda("table readback");
  return SMP_OK;
}

// Device time of one uncaptured step (the best of two after a warm-up).
float time_step(smp_batch &b) {
  Ctx &c = b.ctx->c;
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    if (cudaEventRecord(b.ev0, c.stream) != cudaSuccess || enqueue_step(b, c.stream) != SMP_OK ||
        cudaEventRecord(b.ev1, c.stream) != cudaSuccess || cudaStreamSynchronize(c.stream) != cudaSuccess) {
      cudaGetLastError();
      return 1e30f;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b.ev0, b.ev1);
    if (rep > 0) best = std::min(best, ms);
  }
  return best;
}

// Routing none, or the largest 8, 32 or 128 instances (those above
// kRouteMinN), each timed as a whole step; returns the fastest threshold.
int tune_threshold(smp_batch &b) {
  std::vector<int> cands = {-1};
  for (int r : {8, 32, 128}) {
    if (r >= b.count) break;
    const int thr = std::max(b.inst[b.order[r]].n, kRouteMinN);  // at most r instances above it
    if (routed_count(b, thr) > 0 && std::find(cands.begin(), cands.end(), thr) == cands.end()) cands.push_back(thr);
  }
  int best_thr = -1;
  float best = 1e30f;
  for (int thr : cands) {
    if (set_threshold(b, thr)) continue;
    const float ms = time_step(b);
    if (ms < best) {
      best = ms;
      best_thr = thr;
    }
  }
  return best_thr;
}

void fill_batch_stats(const smp_batch &b, smp_instance *results, smp_batch_stats *st, float ms, int launches) {
  int failed = 0;
  long long props = 0;
  for (int i = 0; i < b.count; ++i) {
    if (b.h_table[i].status != SMP_OK) failed++;
    props += b.h_table[i].proposals;
  }
  if (results) std::memcpy(results, b.h_table, sizeof(smp_instance) * b.count);
  if (st) {
    *st = smp_batch_stats{};
    st->instances = b.count;
    st->failed = failed;
    st->proposals = props;
    st->ms = ms;
    st->launches = launches;
  }
}

}  // namespace

namespace smpb200 {

// Used by the serving loop: launch the batch kernel on a given stream for a
// table it owns (subs = look-ahead windows; the smem attribute is set here,
// outside any capture).
int launch_batch_kernel(Ctx &c, cudaStream_t s, int subs, BatchInstance *table, const int32_t *order, int count,
                        int *queue, uint16_t *slabs, size_t slab_elems, int max_n, int grid, int block,
                        int rank_smem_elems) {
  const size_t smem = batch_smem_bytes(max_n) + static_cast<size_t>(rank_smem_elems) * 2;
  cudaError_t e = cudaSuccess;
  switch (subs) {
    case 1:
      e = allow_dynamic_smem(c, k_batch<1>);
      if (e == cudaSuccess)
        k_batch<1><<<grid, block, smem, s>>>(table, order, count, queue, slabs, slab_elems, max_n, 1, rank_smem_elems);
      break;
    case 2:
      e = allow_dynamic_smem(c, k_batch<2>);
      if (e == cudaSuccess)
        k_batch<2><<<grid, block, smem, s>>>(table, order, count, queue, slabs, slab_elems, max_n, 1, rank_smem_elems);
      break;
    case 4:
      e = allow_dynamic_smem(c, k_batch<4>);
      if (e == cudaSuccess)
        k_batch<4><<<grid, block, smem, s>>>(table, order, count, queue, slabs, slab_elems, max_n, 1, rank_smem_elems);
      break;
    default:
      e = allow_dynamic_smem(c, k_batch<8>);
      if (e == cudaSuccess)
        k_batch<8><<<grid, block, smem, s>>>(table, order, count, queue, slabs, slab_elems, max_n, 1, rank_smem_elems);
      break;
  }
  if (e != cudaSuccess) return c.fail_cuda("k_batch smem attribute");
  return c.check_launch("k_batch");
}

}  // namespace smpb200

extern "C" {

int smp_b200_batch_create(smp_ctx *ctx, const smp_instance *inst, int32_t count, const smp_batch_cfg *cfg,
                          smp_batch **out) {
  if (!ctx || !inst || count <= 0 || !out) return SMP_ERR_INVALID_ARG;
  *out = nullptr;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  auto *b = new (std::nothrow) smp_batch();
  if (!b) return SMP_ERR_OOM;
  b->ctx = ctx;
  b->count = count;
  for (int i = 0; i < count; ++i) {
    if (!inst[i].pref_m || !inst[i].pref_w || !inst[i].match || inst[i].n <= 0 || inst[i].n > SMP_B200_BATCH_MAX_N) {
      delete b;
      c.last_error = "batch: null pointer or n out of range";
      return SMP_ERR_INVALID_ARG;
    }
    b->max_n = std::max(b->max_n, static_cast<int>(inst[i].n));
  }
  b->inst.assign(inst, inst + count);
  // Work queue order: largest instances first (longest-processing-time).
  b->order.resize(count);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return inst[x].n > inst[y].n; });

  // Shape: fixed fields from cfg, the rest tuned (or defaults with tune = -1).
  Shape sh{512, 2, 1, 32};  // the best shape on the 8192-instance mix
  if (cfg && cfg->block_threads > 0) sh.block = std::min(512, std::max(64, cfg->block_threads / 32 * 32));
  if (cfg && cfg->ctas_per_sm > 0) sh.per_sm = std::min(4, cfg->ctas_per_sm);
  else if (cfg && cfg->block_threads > 0) sh.per_sm = std::max(1, 1024 / sh.block);
  if (cfg && cfg->window > 0) sh.subs = subs_for_window(cfg->window);
  if (cfg && cfg->rank_smem_kb != 0) sh.rank_kb = std::max(0, cfg->rank_smem_kb);
  b->use_graph = !(cfg && cfg->use_graph < 0);
  const bool want_tune = !(cfg && cfg->tune < 0) &&
                         !(cfg && cfg->block_threads > 0 && cfg->ctas_per_sm > 0 && cfg->window > 0 &&
                           cfg->rank_smem_kb != 0);
  const bool want_thr = !(cfg && cfg->tune < 0) && !(cfg && cfg->threshold_n != 0);
  // Without tuning, shrink a default shape that does not fit (large max_n).
  while (!shape_fits(c, b->max_n, sh) && sh.rank_kb > 0) sh.rank_kb -= 32;
  if (!shape_fits(c, b->max_n, sh) && !(cfg && cfg->ctas_per_sm > 0)) sh.per_sm = 1;
  if (shape_smem(b->max_n, sh.rank_kb) > c.smem_optin) {
    delete b;
    return SMP_ERR_UNSUPPORTED;
  }
  b->slab_elems = static_cast<size_t>(b->max_n) * b->max_n;
  const size_t slab_bytes = b->slab_elems * sizeof(uint16_t);
  const int by_budget = static_cast<int>(std::max<size_t>(1, kSlabBudget / slab_bytes));
  const int max_grid = std::max(1, std::min({c.sm_count * 4, by_budget, count}));  // any tuned shape fits
  b->block = sh.block;
  b->per_sm = sh.per_sm;
  b->subs = sh.subs;
  b->rank_kb = sh.rank_kb;
  b->rank_smem_elems = sh.rank_kb * 512;
  b->smem = shape_smem(b->max_n, sh.rank_kb);
  b->grid = std::max(1, std::min({c.sm_count * sh.per_sm, by_budget, count}));

  int rc = b->d_table.ensure(sizeof(BatchInstance) * count);
  if (!rc) rc = b->d_order.ensure(sizeof(int32_t) * count);
  if (!rc) rc = b->d_queue.ensure(sizeof(int));
  if (!rc) rc = b->d_slabs.ensure(slab_bytes * max_grid);
  if (!rc && cudaMallocHost(reinterpret_cast<void **>(&b->h_table), sizeof(smp_instance) * count) != cudaSuccess) {
    cudaGetLastError();
    rc = SMP_ERR_OOM;
  }
  if (!rc && (cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)) rc = SMP_ERR_CUDA;
  if (rc) {
    smp_b200_batch_destroy(b);
    return rc;
  }
  std::memcpy(b->h_table, inst, sizeof(smp_instance) * count);
  for (int i = 0; i < count; ++i) {
    b->h_table[i].status = SMP_ERR_NOT_READY;
    b->h_table[i].proposals = 0;
  }
  if (cudaMemcpyAsync(b->d_table.ptr, b->h_table, sizeof(smp_instance) * count, cudaMemcpyHostToDevice, c.stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(b->d_order.ptr, b->order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, c.stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess) {
    c.fail_cuda("batch upload");
    smp_b200_batch_destroy(b);
    return SMP_ERR_CUDA;
  }
  if (want_tune) {
    const auto key = std::make_tuple(c.device, b->max_n, 31 - __builtin_clz(static_cast<unsigned>(count)));
    bool cached = false;
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) {
        sh = it->second;
        cached = true;
      }
    }
    if (!cached) {
      sh = autotune(*b, sh, cfg);
      std::lock_guard<std::mutex> lock(g_tune_mu);
      g_tuned[key] = sh;
    }
    b->tuned = true;
  }
  rc = apply_shape(*b, sh);
  if (rc) {
    smp_b200_batch_destroy(b);
    return rc;
  }
  // Routing to the all-SM pipeline: as configured, or timed on the batch.
  int thr = cfg && cfg->threshold_n > 0 ? cfg->threshold_n : -1;
  if (want_thr) {
    const auto key = std::make_tuple(c.device, b->max_n, 31 - __builtin_clz(static_cast<unsigned>(count)));
    bool cached = false;
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      auto it = g_tuned_thr.find(key);
      if (it != g_tuned_thr.end()) {
        thr = it->second;
        cached = true;
      }
    }
    if (!cached) {
      thr = tune_threshold(*b);
      std::lock_guard<std::mutex> lock(g_tune_mu);
      g_tuned_thr[key] = thr;
    }
    b->thr_tuned = true;
  }
  rc = set_threshold(*b, thr);
  // one uncaptured step first: kernel attributes are set outside the capture
  if (!rc && b->routed) {
    rc = enqueue_step(*b, c.stream);
    if (!rc) rc = c.sync("routed step");
  }
  if (rc) {
    smp_b200_batch_destroy(b);
    return rc;
  }
  if (b->use_graph) {
    // Capture the batched step once; every run replays it.
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      c.fail_cuda("batch capture");
      smp_b200_batch_destroy(b);
      return SMP_ERR_CUDA;
    }
    rc = enqueue_step(*b, c.stream);
    const cudaError_t end = cudaStreamEndCapture(c.stream, &graph);
    if (rc || end != cudaSuccess || cudaGraphInstantiate(&b->exec, graph, 0) != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (!rc) rc = c.fail_cuda("batch graph");
      smp_b200_batch_destroy(b);
      return rc;
    }
    cudaGraphDestroy(graph);
  }
  *out = b;
  return SMP_OK;
}

int smp_b200_batch_run(smp_batch *b, smp_instance *results, smp_batch_stats *st) {
  if (!b) return SMP_ERR_INVALID_ARG;
  Ctx &c = b->ctx->c;
  DeviceGuard g(c.device);
  if (cudaEventRecord(b->ev0, c.stream) != cudaSuccess) return c.fail_cuda("event");
  int rc = SMP_OK;
  if (b->exec) {
    if (cudaGraphLaunch(b->exec, c.stream) != cudaSuccess) rc = c.fail_cuda("batch graph launch");
  } else {
    rc = enqueue_step(*b, c.stream);
  }
  if (rc) return rc;
  if (cudaEventRecord(b->ev1, c.stream) != cudaSuccess) return c.fail_cuda("event");
  rc = c.sync("batch run");
  if (rc) return rc;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  fill_batch_stats(*b, results, st, ms, 1);
  return SMP_OK;
}

int smp_b200_batch_run_plain(smp_batch *b, smp_instance *results, smp_batch_stats *st) {
  if (!b) return SMP_ERR_INVALID_ARG;
  Ctx &c = b->ctx->c;
  DeviceGuard g(c.device);
  if (cudaEventRecord(b->ev0, c.stream) != cudaSuccess) return c.fail_cuda("event");
  // One launch per instance: grid of one CTA, its own instance, no queue.
  for (int k = 0; k < b->count; ++k) {
    const int rc = launch_batch(*b, c.stream, 1, b->d_order.as<int32_t>() + k, 1, 0);
    if (rc) return rc;
  }
  if (cudaMemcpyAsync(b->h_table, b->d_table.ptr, sizeof(smp_instance) * b->count, cudaMemcpyDeviceToHost,
                      c.stream) != cudaSuccess)
    return c.fail_cuda("table readback");
  if (cudaEventRecord(b->ev1, c.stream) != cudaSuccess) return c.fail_cuda("event");
  const int rc = c.sync("batch run plain");
  if (rc) return rc;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  fill_batch_stats(*b, results, st, ms, b->count);
  return SMP_OK;
}

int smp_b200_batch_config(const smp_batch *b, smp_batch_cfg *out) {
  if (!b || !out) return SMP_ERR_INVALID_ARG;
  *out = smp_batch_cfg{};
  out->block_threads = b->block;
  out->ctas_per_sm = b->per_sm;
  out->window = 32 * b->subs;
  out->use_graph = b->exec ? 1 : -1;
  out->rank_smem_kb = b->rank_kb > 0 ? b->rank_kb : -1;
  out->tune = b->tuned ? 1 : -1;
  out->threshold_n = b->threshold_n;
  return SMP_OK;
}

void smp_b200_batch_destroy(smp_batch *b) {
  if (!b) return;
  {
    DeviceGuard g(b->ctx->c.device);
    cudaStreamSynchronize(b->ctx->c.stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->h_table) cudaFreeHost(b->h_table);
    for (smp_ctx *x : b->lanes) smp_b200_destroy(x);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    for (cudaEvent_t e : b->ev_join) cudaEventDestroy(e);
    b->d_table.release();
    b->d_order.release();
    b->d_queue.release();
    b->d_slabs.release();
  }
  delete b;
}

int smp_b200_solve_batch(smp_ctx *ctx, smp_instance *inst, int32_t count, const smp_batch_cfg *cfg,
                         smp_batch_stats *st) {
  smp_batch *b = nullptr;
  smp_batch_cfg plain = cfg ? *cfg : smp_batch_cfg{};
  plain.use_graph = -1;  // a one-shot run gains nothing from capturing a graph
  int rc = smp_b200_batch_create(ctx, inst, count, &plain, &b);
  if (rc) return rc;
  rc = smp_b200_batch_run(b, inst, st);
  smp_b200_batch_destroy(b);
  return rc;
}

void smp_b200_batch_instance(uint64_t seed, uint32_t b, int32_t n_lo, int32_t n_hi, int32_t *n_out,
                             int32_t *kind_out) {
  // Philox counter (b, 0xFFFFFFFF, tag 12, 0): word 0 draws the size, word 1
  // the kind (the same stream the oracle restates).
  uint32_t o[4];
  philox4x32_10(b, 0xFFFFFFFFu, 12u, 0u, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), o);
  const double u = static_cast<double>(o[0]) * (1.0 / 4294967296.0);
  const double v = static_cast<double>(n_lo) * std::exp2(u * std::log2(static_cast<double>(n_hi) / n_lo));
  int32_t n = static_cast<int32_t>(std::floor(v));
  n = std::min(std::max(n, n_lo), n_hi);
  if (n_out) *n_out = n;
  if (kind_out) *kind_out = static_cast<int32_t>(o[1] % 3u);
}

}  // extern "C"
