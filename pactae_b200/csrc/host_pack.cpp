// Host-side packing of int32 preference entries to uint16 for host-input
// solves of n <= 65535, whose lists then cross the host link at half size,
// and HostLink, the pipeline that packs and sends them.  An entry outside
// [0, n) becomes a value >= n (0xFFFF for negatives and for entries of 65536
// and up), which the device reports as invalid input, so a row that was not
// a permutation never packs into one.
#include <cstddef>
#include <cstdint>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include "internal.h"

namespace smpb200 {

namespace {

void pack_scalar(const int32_t *src, uint16_t *dst, size_t b, size_t e, int n) {
  for (size_t k = b; k < e; ++k) {
    const int32_t v = src[k];
    dst[k] = static_cast<unsigned>(v) < static_cast<unsigned>(n) ? static_cast<uint16_t>(v) : uint16_t{0xFFFFu};
  }
}

#if defined(__x86_64__)
// 16 entries per step: an unsigned min against 0xFFFF (negatives are large
// unsigned values) and a saturating pack.  Ordinary stores: the destination
// is a 2 MiB slot that the copy engine reads back while it is still in the
// host's cache (streaming stores would send it to DRAM and back).
__attribute__((target("avx2"))) void pack_avx2(const int32_t *src, uint16_t *dst, size_t b, size_t e, int n) {
  size_t k = b;
  while (k < e && (reinterpret_cast<uintptr_t>(dst + k) & 31u)) {
    pack_scalar(src, dst, k, k + 1, n);
    ++k;
  }
  const __m256i cap = _mm256_set1_epi32(0xFFFF);
  for (; k + 16 <= e; k += 16) {
    const __m256i lo = _mm256_min_epu32(_mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + k)), cap);
    const __m256i hi = _mm256_min_epu32(_mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + k + 8)), cap);
    // packus interleaves the 128-bit halves; the permute puts them in order
    const __m256i p = _mm256_permute4x64_epi64(_mm256_packus_epi32(lo, hi), 0xD8);
    _mm256_store_si256(reinterpret_cast<__m256i *>(dst + k), p);
  }
  pack_scalar(src, dst, k, e, n);
}

const bool kHaveAvx2 = __builtin_cpu_supports("avx2");
#endif

}  // namespace

void pack_u16(const int32_t *src, uint16_t *dst, size_t begin, size_t end, int n) {
#if defined(__x86_64__)
  if (kHaveAvx2) {
    pack_avx2(src, dst, begin, end, n);
    return;
  }
#endif
  pack_scalar(src, dst, begin, end, n);
}


// ---------------------------------------------------------------------------
// HostLink
// ---------------------------------------------------------------------------
HostLink::~HostLink() {
  if (running_) finish();
  for (cudaStream_t st : streams_) cudaStreamSynchronize(st);
  for (cudaEvent_t e : slot_ev_) cudaEventDestroy(e);
  for (cudaEvent_t e : group_ev_) cudaEventDestroy(e);
  if (ready_) cudaEventDestroy(ready_);
  for (cudaStream_t st : streams_) cudaStreamDestroy(st);
  for (uint16_t *h : slots_) cudaFreeHost(h);
}

int HostLink::open(HostPool *pool) {
  pool_ = pool;
  workers_ = pool->size();
  const auto fail = [&](const char *what) {
    error_ = std::string(what) + ": " + cudaGetErrorString(cudaGetLastError());
    return SMP_ERR_CUDA;
  };
  if (cudaEventCreateWithFlags(&ready_, cudaEventDisableTiming) != cudaSuccess) return fail("link event");
  for (int t = 0; t < workers_; ++t) {
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return fail("link stream");
    streams_.push_back(st);
    for (int k = 0; k < 2; ++k) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail("link slot event");
      slot_ev_.push_back(e);
      uint16_t *h = nullptr;
      if (cudaMallocHost(reinterpret_cast<void **>(&h), sizeof(uint16_t) * kSlotEntries) != cudaSuccess) {
        cudaGetLastError();
        error_ = "link slot: pinned host memory";
        return SMP_ERR_OOM;
      }
      slots_.push_back(h);
    }
    for (int g = 0; g < kMaxGroups; ++g) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail("link group event");
      group_ev_.push_back(e);
    }
  }
  return SMP_OK;
}

void HostLink::group_rows(int g, int *part, int *r0, int *r1) const {
  const int p = g / groups_, k = g % groups_;
  const int rows = parts_[p].rows;
  *part = p;
  *r0 = static_cast<int>(static_cast<int64_t>(rows) * k / groups_);
  *r1 = static_cast<int>(static_cast<int64_t>(rows) * (k + 1) / groups_);
}

int HostLink::start(const Part *parts, int nparts, int n, int groups, cudaStream_t after) {
  if (running_ || nparts < 1 || nparts > 2 || groups < 1 || nparts * groups > kMaxGroups) return SMP_ERR_INVALID_ARG;
  for (int p = 0; p < nparts; ++p) parts_[p] = parts[p];
  nparts_ = nparts;
  n_ = n;
  groups_ = groups;
  failed_ = false;
  error_.clear();
  for (int &q : queued_) q = 0;
  // the destinations may be fresh stream-ordered allocations on `after`
  if (cudaEventRecord(ready_, after) != cudaSuccess) {
    error_ = std::string("link start: ") + cudaGetErrorString(cudaGetLastError());
    return SMP_ERR_CUDA;
  }
  for (cudaStream_t st : streams_)
    if (cudaStreamWaitEvent(st, ready_, 0) != cudaSuccess) {
      error_ = std::string("link start: ") + cudaGetErrorString(cudaGetLastError());
      return SMP_ERR_CUDA;
    }
  running_ = true;
  pool_->start([this](int t, int) { work(t); });
  return SMP_OK;
}

void HostLink::work(int t) {
  cudaStream_t st = streams_[t];
  const int total = nparts_ * groups_;
  size_t piece = 0;  // pieces are dealt to the workers in turn, across groups
  int used = 0;
  bool ok = true;
  std::string why;
  // entries [b, e) of the part's matrices, in pieces of at most one slot
  const auto send = [&](const Part &P, size_t b, size_t e) {
    for (; b < e; b += kSlotEntries, ++piece) {
      if (static_cast<int>(piece % workers_) != t || !ok) continue;
      const int slot = 2 * t + (used & 1);
      if (used >= 2 && cudaEventSynchronize(slot_ev_[slot]) != cudaSuccess) {
        ok = false;
        why = "link slot wait";
        continue;
      }
      const size_t cnt = std::min(kSlotEntries, e - b);
      pack_u16(P.src + b, slots_[slot], 0, cnt, n_);
      if (cudaMemcpyAsync(P.dst + b, slots_[slot], sizeof(uint16_t) * cnt, cudaMemcpyHostToDevice, st) !=
              cudaSuccess ||
          cudaEventRecord(slot_ev_[slot], st) != cudaSuccess) {
        ok = false;
        why = "link copy";
        continue;
      }
      ++used;
    }
  };
  for (int g = 0; g < total; ++g) {
    int p, r0, r1;
    group_rows(g, &p, &r0, &r1);
    const Part &P = parts_[p];
    if (P.row_ids) {
      for (int i = r0; i < r1; ++i) {
        const size_t b = static_cast<size_t>(P.row_ids[i]) * n_;
        send(P, b, b + n_);
      }
    } else {
      send(P, static_cast<size_t>(r0) * n_, static_cast<size_t>(r1) * n_);
    }
    if (ok && cudaEventRecord(group_ev_[static_cast<size_t>(t) * kMaxGroups + g], st) != cudaSuccess) {
      ok = false;
      why = "link group event";
    }
    {
      std::lock_guard<std::mutex> lock(mu_);
      if (!ok && !failed_) {
        failed_ = true;
        error_ = why + ": " + cudaGetErrorString(cudaGetLastError());
      }
      ++queued_[g];
    }
    cv_.notify_all();
  }
  // the slots are reused by the next start: their copies must have finished
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    std::lock_guard<std::mutex> lock(mu_);
    if (!failed_) {
      failed_ = true;
      error_ = std::string("link stream: ") + cudaGetErrorString(cudaGetLastError());
    }
  }
}

int HostLink::wait_group(int g, cudaStream_t stream) {
  {
    std::unique_lock<std::mutex> lock(mu_);
    cv_.wait(lock, [&] { return queued_[g] == workers_; });
    if (failed_) return SMP_ERR_CUDA;
  }
  for (int t = 0; t < workers_; ++t)
    if (cudaStreamWaitEvent(stream, group_ev_[static_cast<size_t>(t) * kMaxGroups + g], 0) != cudaSuccess) {
      std::lock_guard<std::mutex> lock(mu_);
      failed_ = true;
      error_ = std::string("link group wait: ") + cudaGetErrorString(cudaGetLastError());
      return SMP_ERR_CUDA;
    }
  return SMP_OK;
}

int HostLink::finish() {
  if (!running_) return SMP_OK;
  pool_->wait();
  running_ = false;
  std::lock_guard<std::mutex> lock(mu_);
  return failed_ ? SMP_ERR_CUDA : SMP_OK;
}

}  // namespace smpb200
