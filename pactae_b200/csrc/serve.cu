// serve.cu -- the serving loop: single-instance requests of any size arrive
// at any time; a host thread admits them against an HBM budget and keeps the
// GPU busy with overlapping work (continuous batching):
//   - requests with n <= route_n are gathered into waves; each wave is one
//     launch of the batch kernel (one CTA per request) on its own stream, and
//     several waves are in flight at once, so a request that arrives while
//     others run starts in the next wave without waiting for them;
//   - larger requests go through the single-instance pipeline, several at
//     once (large_slots contexts, each with its own stream): one solve's
//     latency-bound chains and one-SM tail leave most SMs to the others
//     and to the waves.
// A request is admitted when its matrices (two n x n int32 lists and the
// n x n uint16 rank matrix: 10 n^2 bytes) fit in the budget; it releases
// them when it completes.  The reference has no serving layer.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <numeric>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch_kernels.cuh"
#include "common.cuh"
#include "internal.h"

using namespace smpb200;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
  int64_t ticket = 0;
  const int32_t *pm = nullptr;
  const int32_t *pw = nullptr;
  int32_t *match = nullptr;  // caller's output (host or device)
  int n = 0;
  uint32_t flags = 0;
  uint64_t bytes = 0;
  Clock::time_point t_submit, t_launch, t_done;
  int status = SMP_ERR_NOT_READY;
  int64_t proposals = 0;
  bool done = false;
  // device copies for host-pointer requests
  DeviceBuf d_pm, d_pw, d_match;
  const int32_t *dev_pm() const { return (flags & SMP_F_DEVICE_PTRS) ? pm : d_pm.as<int32_t>(); }
  const int32_t *dev_pw() const { return (flags & SMP_F_DEVICE_PTRS) ? pw : d_pw.as<int32_t>(); }
  int32_t *dev_match() const { return (flags & SMP_F_DEVICE_PTRS) ? match : d_match.as<int32_t>(); }
};

struct Wave {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  DeviceBuf table, order, queue, slabs;
  smp_instance *h_table = nullptr;  // pinned
  std::vector<Request *> reqs;
  bool busy = false;
};

}  // namespace

struct smp_server {
  smp_server_cfg cfg = {};
  smp_ctx *ctx = nullptr;        // device, sm count, error text for the waves
  struct LargeSlot {
    smp_ctx *ctx = nullptr;  // single-instance pipeline
    cudaEvent_t done = nullptr;
    Request *running = nullptr;
  };
  std::vector<LargeSlot> large;
  std::thread thread;
  std::mutex mu;
  std::condition_variable cv_submit, cv_done;
  std::deque<Request *> submitted;                 // guarded by mu
  std::unordered_map<int64_t, Request *> tickets;  // guarded by mu
  int64_t next_ticket = 1;                         // guarded by mu
  bool stop = false;                               // guarded by mu
  smp_server_stats stats = {};                     // guarded by mu
  // server-thread state
  std::deque<Request *> pending, small_q, large_q;
  std::vector<Wave> waves;
  uint64_t used = 0;
  cudaMemPool_t pool = nullptr;  // device_pool of the server's device
  int grid = 0;
  size_t slab_elems = 0;
};

namespace {

void finish(smp_server &s, Request *r, int status, int64_t proposals) {
  r->t_done = Clock::now();
  s.used -= r->bytes;
  r->d_pm.release();
  r->d_pw.release();
  r->d_match.release();
  std::lock_guard<std::mutex> lock(s.mu);
  r->status = status;
  r->proposals = proposals;
  r->done = true;
  s.stats.completed++;
  s.stats.admitted_bytes = static_cast<int64_t>(s.used);
  s.cv_done.notify_all();
}

// Host-pointer requests: device copies of the lists (and the output) on the
// given stream.  Returns the status.
int stage_request(Request *r, cudaStream_t st, cudaMemPool_t pool) {
  if (r->flags & SMP_F_DEVICE_PTRS) return SMP_OK;
  const size_t bytes = sizeof(int32_t) * static_cast<size_t>(r->n) * r->n;
  // allocated and freed in the order of the stream that runs the request
  for (DeviceBuf *b : {&r->d_pm, &r->d_pw, &r->d_match}) b->bind(pool, st);
  if (r->d_pm.ensure(bytes) || r->d_pw.ensure(bytes) || r->d_match.ensure(sizeof(int32_t) * r->n))
    return SMP_ERR_OOM;
  if (cudaMemcpyAsync(r->d_pm.ptr, r->pm, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(r->d_pw.ptr, r->pw, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) {
    cudaGetLastError();
    return SMP_ERR_CUDA;
  }
  return SMP_OK;
}

int unstage_request(Request *r, cudaStream_t st) {
  if (r->flags & SMP_F_DEVICE_PTRS) return SMP_OK;
  if (cudaMemcpyAsync(r->match, r->d_match.ptr, sizeof(int32_t) * r->n, cudaMemcpyDeviceToHost, st) !=
      cudaSuccess) {
    cudaGetLastError();
    return SMP_ERR_CUDA;
  }
  return SMP_OK;
}

void launch_wave(smp_server &s, Wave &w) {
  Ctx &c = s.ctx->c;
  const int count = static_cast<int>(w.reqs.size());
  int max_n = 0;
  for (Request *r : w.reqs) max_n = std::max(max_n, r->n);
  // (pageable source: cudaMemcpyAsync has copied it when it returns)
  std::vector<int32_t> order(count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return w.reqs[a]->n > w.reqs[b]->n; });
  int rc = SMP_OK;
  const auto now = Clock::now();
  for (int i = 0; i < count && !rc; ++i) {
    Request *r = w.reqs[i];
    r->t_launch = now;
    rc = stage_request(r, w.stream, s.pool);
    w.h_table[i] = smp_instance{r->dev_pm(), r->dev_pw(), r->dev_match(), r->n, SMP_ERR_NOT_READY, 0};
  }
  if (!rc && (cudaMemcpyAsync(w.table.ptr, w.h_table, sizeof(smp_instance) * count, cudaMemcpyHostToDevice,
                              w.stream) != cudaSuccess ||
              cudaMemcpyAsync(w.order.ptr, order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice,
                              w.stream) != cudaSuccess ||
              cudaMemsetAsync(w.queue.ptr, 0, sizeof(int), w.stream) != cudaSuccess))
    rc = c.fail_cuda("wave upload");
  const int block = s.cfg.block_threads > 0 ? s.cfg.block_threads : 512;
  // 32 KB of shared memory per CTA keeps the rank matrix of requests with
  // n <= 128 on chip, when it fits beside the bids; the look-ahead is one
  // window (the batch's best shape on its mix of sizes).
  const int rank_smem_elems = batch_smem_bytes(max_n) + (32u << 10) <= c.smem_optin ? (16 << 10) : 0;
  if (!rc)
    rc = launch_batch_kernel(c, w.stream, 1, w.table.as<BatchInstance>(), w.order.as<int32_t>(), count,
                             w.queue.as<int>(), w.slabs.as<uint16_t>(), s.slab_elems, max_n,
                             std::min(count, s.grid), block, rank_smem_elems);
  if (!rc && cudaMemcpyAsync(w.h_table, w.table.ptr, sizeof(smp_instance) * count, cudaMemcpyDeviceToHost,
                             w.stream) != cudaSuccess)
    rc = c.fail_cuda("wave readback");
  for (int i = 0; i < count && !rc; ++i) rc = unstage_request(w.reqs[i], w.stream);
  if (!rc && cudaEventRecord(w.done, w.stream) != cudaSuccess) rc = c.fail_cuda("wave event");
  if (rc) {
    cudaStreamSynchronize(w.stream);
    for (Request *r : w.reqs) finish(s, r, rc, 0);
    w.reqs.clear();
    return;
  }
  w.busy = true;
  std::lock_guard<std::mutex> lock(s.mu);
  s.stats.waves++;
}

void reap_wave(smp_server &s, Wave &w) {
  if (!w.busy || cudaEventQuery(w.done) != cudaSuccess) return;
  for (size_t i = 0; i < w.reqs.size(); ++i) finish(s, w.reqs[i], w.h_table[i].status, w.h_table[i].proposals);
  w.reqs.clear();
  w.busy = false;
}

void launch_large(smp_server &s, smp_server::LargeSlot &slot) {
  Request *r = s.large_q.front();
  s.large_q.pop_front();
  Ctx &lc = slot.ctx->c;
  r->t_launch = Clock::now();
  int rc = stage_request(r, lc.stream, s.pool);
  if (!rc) rc = solve_enqueue(lc, r->dev_pm(), r->dev_pw(), r->n, r->dev_match(), SMP_F_DEVICE_PTRS);
  if (!rc) rc = unstage_request(r, lc.stream);
  if (!rc && cudaEventRecord(slot.done, lc.stream) != cudaSuccess) rc = lc.fail_cuda("large event");
  if (rc) {
    cudaStreamSynchronize(lc.stream);
    finish(s, r, rc, 0);
    return;
  }
  slot.running = r;
  std::lock_guard<std::mutex> lock(s.mu);
  s.stats.large++;
}

void reap_large(smp_server &s, smp_server::LargeSlot &slot) {
  if (!slot.running || cudaEventQuery(slot.done) != cudaSuccess) return;
  Ctx &lc = slot.ctx->c;
  smp_stats st = {};
  const int rc = solve_finish(lc, SMP_F_DEVICE_PTRS, &st);
  finish(s, slot.running, rc, rc == SMP_OK ? st.proposals : 0);
  slot.running = nullptr;
}

void server_loop(smp_server *sp) {
  smp_server &s = *sp;
  cudaSetDevice(s.cfg.device);
  const int max_wave = s.cfg.max_wave > 0 ? s.cfg.max_wave : 256;
  for (;;) {
    {
      std::unique_lock<std::mutex> lock(s.mu);
      const bool idle =
          s.pending.empty() && s.small_q.empty() && s.large_q.empty() &&
          std::none_of(s.large.begin(), s.large.end(), [](const smp_server::LargeSlot &l) { return l.running; }) &&
          std::none_of(s.waves.begin(), s.waves.end(), [](const Wave &w) { return w.busy; });
      if (idle) s.cv_submit.wait_for(lock, std::chrono::microseconds(200), [&] { return s.stop || !s.submitted.empty(); });
      while (!s.submitted.empty()) {
        s.pending.push_back(s.submitted.front());
        s.submitted.pop_front();
      }
      if (s.stop && idle && s.pending.empty()) break;
    }
    // admission, first come first served
    while (!s.pending.empty()) {
      Request *r = s.pending.front();
      if (s.used > 0 && s.used + r->bytes > s.cfg.hbm_budget) break;
      s.pending.pop_front();
      s.used += r->bytes;
      (r->n > s.cfg.route_n ? s.large_q : s.small_q).push_back(r);
      std::lock_guard<std::mutex> lock(s.mu);
      s.stats.admitted_bytes = static_cast<int64_t>(s.used);
      s.stats.peak_bytes = std::max<int64_t>(s.stats.peak_bytes, static_cast<int64_t>(s.used));
    }
    for (auto &slot : s.large)
      if (!slot.running && !s.large_q.empty()) launch_large(s, slot);
    for (Wave &w : s.waves) {
      if (w.busy || s.small_q.empty()) continue;
      while (!s.small_q.empty() && static_cast<int>(w.reqs.size()) < max_wave) {
        w.reqs.push_back(s.small_q.front());
        s.small_q.pop_front();
      }
      launch_wave(s, w);
    }
    for (Wave &w : s.waves) reap_wave(s, w);
    for (auto &slot : s.large) reap_large(s, slot);
    // short pause while work is on the device
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

void destroy_server(smp_server *s) {
  if (!s) return;
  for (Wave &w : s->waves) {
    if (w.stream) {
      cudaStreamSynchronize(w.stream);
      cudaStreamDestroy(w.stream);
    }
    if (w.done) cudaEventDestroy(w.done);
    if (w.h_table) cudaFreeHost(w.h_table);
    w.table.release();
    w.order.release();
    w.queue.release();
    w.slabs.release();
  }
  for (auto &slot : s->large) {
    if (slot.done) cudaEventDestroy(slot.done);
    if (slot.ctx) smp_b200_destroy(slot.ctx);
  }
  if (s->ctx) smp_b200_destroy(s->ctx);  // also trims the device pool
  for (auto &kv : s->tickets) delete kv.second;
  delete s;
}

}  // namespace

extern "C" {

int smp_b200_server_create(const smp_server_cfg *cfg, smp_server **out) {
  if (!out) return SMP_ERR_INVALID_ARG;
  *out = nullptr;
  auto *s = new (std::nothrow) smp_server();
  if (!s) return SMP_ERR_OOM;
  if (cfg) s->cfg = *cfg;
  if (s->cfg.route_n <= 0) s->cfg.route_n = 1024;
  s->cfg.route_n = std::min(s->cfg.route_n, SMP_B200_BATCH_MAX_N);
  if (s->cfg.waves <= 0) s->cfg.waves = 2;
  if (s->cfg.hbm_budget == 0) s->cfg.hbm_budget = 64ull << 30;
  smp_cfg c1 = {};
  c1.device = s->cfg.device;
  int rc = smp_b200_create(&s->ctx, &c1);
  s->large.resize(static_cast<size_t>(s->cfg.large_slots > 0 ? std::min<uint64_t>(s->cfg.large_slots, 16) : 4));
  for (auto &slot : s->large)
    if (!rc) rc = smp_b200_create(&slot.ctx, &c1);
  if (rc) {
    destroy_server(s);
    return rc;
  }
  Ctx &c = s->ctx->c;
  DeviceGuard g(c.device);
  s->pool = device_pool(c.device);
  const int max_wave = s->cfg.max_wave > 0 ? s->cfg.max_wave : 256;
  const int per_sm = s->cfg.ctas_per_sm > 0 ? s->cfg.ctas_per_sm : 2;
  s->grid = std::max(1, std::min(max_wave, c.sm_count * per_sm));
  s->slab_elems = static_cast<size_t>(s->cfg.route_n) * s->cfg.route_n;
  s->waves.resize(s->cfg.waves);
  for (Wave &w : s->waves) {
    if (cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming) != cudaSuccess)
      rc = SMP_ERR_CUDA;
    if (!rc) rc = w.table.ensure(sizeof(BatchInstance) * max_wave);
    if (!rc) rc = w.order.ensure(sizeof(int32_t) * max_wave);
    if (!rc) rc = w.queue.ensure(sizeof(int));
    if (!rc) rc = w.slabs.ensure(sizeof(uint16_t) * s->slab_elems * s->grid);
    if (!rc && cudaMallocHost(reinterpret_cast<void **>(&w.h_table), sizeof(smp_instance) * max_wave) != cudaSuccess)
      rc = SMP_ERR_OOM;
    if (rc) break;
  }
  for (auto &slot : s->large)
    if (!rc && cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming) != cudaSuccess) rc = SMP_ERR_CUDA;
  // Each large slot holds the buffers of the largest request the budget
  // admits from the start: growing them while others run would stall the
  // burst that brought the first large requests.
  int reserve_n = SMP_B200_BATCH_MAX_N;
  while (reserve_n > s->cfg.route_n && 10ull * reserve_n * reserve_n > s->cfg.hbm_budget) reserve_n /= 2;
  if (reserve_n > s->cfg.route_n)
    for (auto &slot : s->large)
      if (!rc) rc = reserve_buffers(slot.ctx->c, reserve_n);
  if (rc) {
    cudaGetLastError();
    destroy_server(s);
    return rc;
  }
  s->thread = std::thread(server_loop, s);
  *out = s;
  return SMP_OK;
}

int smp_b200_submit(smp_server *s, const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *match_out,
                    uint32_t flags, int64_t *ticket) {
  if (!s || !pref_m || !pref_w || !match_out || !ticket || n <= 0 || n > SMP_B200_BATCH_MAX_N)
    return SMP_ERR_INVALID_ARG;
  const uint64_t bytes = 10ull * static_cast<uint64_t>(n) * static_cast<uint64_t>(n);
  if (bytes > s->cfg.hbm_budget) return SMP_ERR_BUSY;
  auto *r = new (std::nothrow) Request();
  if (!r) return SMP_ERR_OOM;
  r->pm = pref_m;
  r->pw = pref_w;
  r->match = match_out;
  r->n = n;
  r->flags = flags;
  r->bytes = bytes;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    r->ticket = s->next_ticket++;
    s->tickets[r->ticket] = r;
    s->submitted.push_back(r);
    s->stats.submitted++;
  }
  s->cv_submit.notify_one();
  *ticket = r->ticket;
  return SMP_OK;
}

int smp_b200_poll(smp_server *s, int64_t ticket, int32_t wait_ms, smp_result *result) {
  if (!s || !result) return SMP_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return SMP_ERR_INVALID_ARG;
  Request *r = it->second;
  if (!r->done) {
    if (wait_ms < 0)
      s->cv_done.wait(lock, [&] { return r->done; });
    else
      s->cv_done.wait_for(lock, std::chrono::milliseconds(wait_ms), [&] { return r->done; });
  }
  if (!r->done) return SMP_ERR_NOT_READY;
  result->status = r->status;
  result->n = r->n;
  result->proposals = r->proposals;
  result->queue_ms = ms_between(r->t_submit, r->t_launch);
  result->latency_ms = ms_between(r->t_submit, r->t_done);
  s->tickets.erase(it);
  delete r;
  return SMP_OK;
}

int smp_b200_server_stats(smp_server *s, smp_server_stats *st) {
  if (!s || !st) return SMP_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(s->mu);
  *st = s->stats;
  return SMP_OK;
}

void smp_b200_server_destroy(smp_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv_submit.notify_all();
  if (s->thread.joinable()) s->thread.join();
  destroy_server(s);
}

}  // extern "C"
