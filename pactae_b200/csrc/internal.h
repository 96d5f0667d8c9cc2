// internal.h -- host-side state shared by the translation units of
// libsmp_b200.so.  Not part of the public ABI (include/smp_b200.h is).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include <set>
#include <utility>
#include <array>
#include <string>

#include "smp_b200.h"

namespace smpb200 {

// The library's memory pool on a device (smp_b200.cu): created on first use,
// it keeps freed memory for later allocations until trim_device_pool.
cudaMemPool_t device_pool(int device);
void trim_device_pool(int device);

// Grow-only device allocation.  Bound to a pool and a stream, it allocates
// and frees in that stream's order (cudaMallocFromPoolAsync / cudaFreeAsync),
// so growing a buffer waits for nothing else on the device; cudaFree would
// wait for every stream.  Unbound, it uses cudaMalloc / cudaFree.
struct DeviceBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  cudaMemPool_t pool = nullptr;
  cudaStream_t stream = nullptr;

  void bind(cudaMemPool_t p, cudaStream_t s) {
    pool = p;
    stream = s;
  }
  int ensure(size_t need) {
    if (need <= bytes && ptr) return SMP_OK;
    release();
    if (need == 0) need = 16;
    if (!allocate(need)) {
      cudaGetLastError();  // clear the sticky-free allocation error
      if (pool) {
        // Memory freed on other streams may still sit in the pool: wait for
        // this stream, hand what is unused back and try once more.
        cudaStreamSynchronize(stream);
        cudaMemPoolTrimTo(pool, 0);
        if (allocate(need)) {
          bytes = need;
          return SMP_OK;
        }
        cudaGetLastError();
      }
      ptr = nullptr;
      bytes = 0;
      return SMP_ERR_OOM;
    }
    bytes = need;
    return SMP_OK;
  }
  void release() {
    if (ptr) {
      if (pool)
        cudaFreeAsync(ptr, stream);
      else
        cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
  }
  bool allocate(size_t need) {
    if (pool) return cudaMallocFromPoolAsync(&ptr, need, pool, stream) == cudaSuccess;
    return cudaMalloc(&ptr, need) == cudaSuccess;
  }
  template <typename T>
  T *as() const { return static_cast<T *>(ptr); }
};

// Makes the context's device current for the duration of an entry point and
// restores the caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Entries [begin, end) of src packed to uint16 in dst (host_pack.cpp).
void pack_u16(const int32_t *src, uint16_t *dst, size_t begin, size_t end, int n);

// A fixed set of host threads that run one job at a time: run(f) calls
// f(i, count) on every worker i and returns when all have finished; start(f)
// returns at once and wait() when the job has finished.  Started once per
// context, so a job costs a wake-up, not a thread creation.

class HostPool {
 public:
  explicit HostPool(int count) {
    for (int i = 0; i < count; ++i) threads_.emplace_back([this, i] { work(i); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : threads_) t.join();
  }
  int size() const { return static_cast<int>(threads_.size()); }
  void run(const std::function<void(int, int)> &f) {
    start(f);
    wait();
  }
  void start(std::function<void(int, int)> f) {
    std::unique_lock<std::mutex> lock(mu_);
    done_.wait(lock, [this] { return pending_ == 0; });
    owned_ = std::move(f);
    job_ = &owned_;
    pending_ = size();
    ++generation_;
    cv_.notify_all();
  }
  void wait() {
    std::unique_lock<std::mutex> lock(mu_);
    done_.wait(lock, [this] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  void work(int i) {
    unsigned seen = 0;
    for (;;) {
      const std::function<void(int, int)> *f;
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
        f = job_;
      }
      (*f)(i, size());
      std::lock_guard<std::mutex> lock(mu_);
      if (--pending_ == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  std::function<void(int, int)> owned_;
  const std::function<void(int, int)> *job_ = nullptr;
  unsigned generation_ = 0;
  int pending_ = 0;
  bool stop_ = false;
};

// Sends int32 host matrices to device memory packed to uint16, half the
// bytes on the host link.  Each of the pool's workers owns a CUDA stream and
// two pinned slots of kSlotEntries entries: it packs a piece of a matrix
// into one slot with ordinary stores -- the slot stays in the host's cache,
// where the copy engine reads it back, so the only host DRAM traffic is the
// read of the source -- and queues the slot's copy on its stream while it
// packs the next piece into the other.  Pieces are dealt to the workers in
// turn.  Each matrix is cut into row groups; when a worker has queued its
// pieces of a group it records the group's event on its stream, and
// wait_group makes a stream wait for every worker's event of that group, so
// device work on a group starts as soon as its rows have landed.
class HostLink {
 public:
  static constexpr size_t kSlotEntries = size_t{1} << 20;  // 2 MiB of uint16
  static constexpr int kMaxGroups = 32;
  struct Part {
    const int32_t *src;  // host, n columns
    uint16_t *dst;       // device, n columns
    int rows;            // rows sent: 0 .. rows-1, or row_ids[0 .. rows-1]
    const int32_t *row_ids = nullptr;  // host; rows to send, each a row of src and dst
  };
  HostLink() = default;
  HostLink(const HostLink &) = delete;
  HostLink &operator=(const HostLink &) = delete;
  ~HostLink();
  // Streams, events and pinned slots for the pool's workers.  SMP_OK, or
  // SMP_ERR_OOM / SMP_ERR_CUDA (the link is then unusable).
  int open(HostPool *pool);
  // Packs and sends parts[0..nparts) (at most two), each cut into `groups`
  // row groups; group g of part p is global group p * groups + g.  The
  // copies are queued after the work already queued on `after`.
  int start(const Part *parts, int nparts, int n, int groups, cudaStream_t after);
  // Rows [r0, r1) of global group g (indices into row_ids for a listed part).
  void group_rows(int g, int *part, int *r0, int *r1) const;
  // Blocks until every worker has queued its pieces of global group g, then
  // makes `stream` wait for them on the device.
  int wait_group(int g, cudaStream_t stream);
  // Waits for the workers and their copies; SMP_ERR_CUDA if a call failed.
  int finish();
  const std::string &error() const { return error_; }

 private:
  void work(int t);
  HostPool *pool_ = nullptr;
  int workers_ = 0;
  std::vector<cudaStream_t> streams_;
  std::vector<cudaEvent_t> slot_ev_;   // 2 per worker
  std::vector<cudaEvent_t> group_ev_;  // kMaxGroups per worker
  std::vector<uint16_t *> slots_;      // 2 per worker, pinned
  cudaEvent_t ready_ = nullptr;
  Part parts_[2] = {};
  int nparts_ = 0, n_ = 0, groups_ = 0;
  std::mutex mu_;
  std::condition_variable cv_;
  int queued_[kMaxGroups] = {};
  bool failed_ = false;
  bool running_ = false;
  std::string error_;
};

struct Control;  // common.cuh

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 148;
  size_t smem_optin = 0;  // max dynamic shared memory per block
  int prefix_k_cfg = 0;
  int tail_threshold_cfg = 0;
  int bulk_window_cfg = 0;
  int tail_window_cfg = 0;
  int mode_cfg = 0;
  int rank_bytes_cfg = 0;  // 4: int32 ranks at any n
  uint64_t hbm_budget = 64ull << 30;
  std::string last_error;

  // State of the staged solve.
  int n = 0;
  bool staged = false;
  const int32_t *pref_m = nullptr;  // device pointers the solve reads
  const int32_t *pref_w = nullptr;
  int K = 0;               // prefix width (0 = none)
  int tail_threshold = 0;  // 0 = tail kernel disabled; query-mode hand-over
  int tail_threshold_rank = 0;  // rank-mode hand-over (free women left)
  bool query_ok = false;   // the query mode may be chosen for this n
  int bulk_window = 256;   // look-ahead choices per warp step
  int tail_window = 256;
  int rank_bytes = 2;
  bool rank_valid = false;  // d_rank holds the inversion of pref_w
  bool tail_ran = false;
  bool swapped = false;  // the men share one list and the women proposed
  int phase = 0;            // 0 staged, 1 prechecked, 2 inited, 3 cored, 4 posted
  // The mode the host has read back from the precheck (kModeQuery / kModeRank),
  // or -1: the enqueue functions then skip the kernels that mode would gate
  // off.  -1 (unknown) enqueues everything and the device picks.
  int known_mode = -1;

  DeviceBuf d_pref_m, d_pref_w, d_rank, d_rankT, d_pr, d_prefix, d_bid, d_tailq, d_seen, d_ctrl, d_match;
  DeviceBuf d_pw16, d_pm16;  // pref_w and pref_m packed to uint16 (host-input solves)
  DeviceBuf d_swap_pos;  // women-proposing solves: position of each woman in the men's shared list
  // host-input women-proposing solves: which women's rows are whole on the
  // device, the women stopped at the end of theirs (two lists), row ids
  DeviceBuf d_swap_full, d_swap_over, d_swap_rows;
  // Host-input solves: the host threads that pack and screen, and the link
  // that sends packed rows through them (created on first use).
  std::unique_ptr<HostPool> pack_pool;
  std::unique_ptr<HostLink> link;
  DeviceBuf d_husband, d_prank;
  DeviceBuf d_qcnt, d_qlist;
  DeviceBuf gen_keys_a, gen_keys_b, gen_seg, gen_temp, gen_aux;
  Control *h_ctrl = nullptr;  // pinned host copy of the control block
  cudaEvent_t ev[10] = {};
  // Host-pointer solves: pref_w arrives on copy_stream in kCopyChunks row
  // chunks, each signalled by its event (created on first use).
  static constexpr int kCopyChunks = 16;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_chunk[kCopyChunks] = {};
  std::array<DeviceBuf *, 26> buffers() {
    return {&d_pref_m, &d_pref_w, &d_pw16, &d_pm16, &d_rank,    &d_rankT,    &d_pr,     &d_prefix, &d_bid,    &d_tailq,
            &d_seen,   &d_ctrl,   &d_match,   &d_husband,  &d_prank,  &d_qcnt,   &d_qlist,
            &gen_keys_a, &gen_keys_b, &gen_seg, &gen_temp, &gen_aux, &d_swap_pos, &d_swap_full, &d_swap_over,
            &d_swap_rows};
  }
  int launches = 0;  // kernels launched since the last stage / call
  smp_stats stats = {};

  int fail_cuda(const char *what) {
    const cudaError_t e = cudaGetLastError();
    last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return SMP_ERR_CUDA;
  }
  int check_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return SMP_OK;
    last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return SMP_ERR_CUDA;
  }
  int sync(const char *what) {
    const cudaError_t e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) return SMP_OK;
    last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return SMP_ERR_CUDA;
  }
};

// Lets a kernel launch with as much dynamic shared memory as the device
// allows beside its static shared memory.  The attribute is process-wide per
// kernel, so it is set once per kernel and device, to that one value, and
// never changed: setting it to each launch's own size would let a small
// launch on one thread (a solve) lower it under a larger launch another
// thread (the serving loop) is about to make, which then fails.
inline cudaError_t allow_dynamic_smem_ptr(const Ctx &c, const void *kernel) {
  static std::mutex mu;
  static std::set<std::pair<const void *, int>> done;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(kernel, c.device);
  if (done.count(key)) return cudaSuccess;
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, kernel);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(c.smem_optin - a.sharedSizeBytes));
  if (e == cudaSuccess) done.insert(key);
  return e;
}
template <typename Kernel>
inline cudaError_t allow_dynamic_smem(const Ctx &c, Kernel kernel) {
  return allow_dynamic_smem_ptr(c, reinterpret_cast<const void *>(kernel));
}

// smp_b200.cu: a whole solve split into its asynchronous part and its
// completion (the public smp_b200_solve is the two with a sync between).
int solve_enqueue(Ctx &c, const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *match_out,
                  uint32_t flags);
int solve_finish(Ctx &c, uint32_t flags, smp_stats *st);
int reserve_buffers(Ctx &c, int32_t n);

// batch.cu: the batch kernel on a caller's stream and table (serving loop).
struct BatchInstance;
int launch_batch_kernel(Ctx &c, cudaStream_t s, int subs, BatchInstance *table, const int32_t *order, int count,
                        int *queue, uint16_t *slabs, size_t slab_elems, int max_n, int grid, int block,
                        int rank_smem_elems);

// generate.cu
int generate_side(Ctx &c, int kind, int side, int n, uint64_t seed, uint32_t salt, int param,
                  int32_t *out);

}  // namespace smpb200

struct smp_ctx {
  smpb200::Ctx c;
};
