// static_solve.cu -- smp_b200_solve_static: a whole solve that allocates
// nothing.
//
// Some callers cannot allocate device memory when they need a matching: a
// host application whose device memory is already reserved by its own
// caching allocator (a cudaMalloc from a library would fail or fragment that
// pool), a process running under a hard per-process device-memory limit
// whose budget is spent, or a latency-critical loop that must not stall on
// cudaMalloc/cudaFree (cudaFree synchronises the device).  For them this
// entry point takes device pointers to the two preference lists and to the
// output, and keeps all of its scratch -- the rank matrix and a small result
// header -- in one file-scope __device__ array compiled into the library.
// Every GPU that loads the library holds that array (kStaticScratchBytes,
// 2 MiB plus 256 bytes) until the process exits.
//
// Limits and rules (also stated in include/smp_b200.h):
//   - n <= SMP_B200_STATIC_MAX_N (1024); larger n is rejected with
//     SMP_ERR_UNSUPPORTED before anything runs.
//   - The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it.
//   - Every call is synchronous: it copies the result header back to the
//     host and waits on the stream, so no call can run on a stream under
//     capture.
//   - All calls share the one array, which keeps the last call's contents.
//     Each call overwrites the rank matrix and clears the header itself, but
//     calls whose work overlaps on the GPU (different streams, different host
//     threads without ordering) race on it: order them on one stream.
//
// The kernel is a one-CTA variant of the solve: warps invert the women's
// rows straight into the static rank matrix (checking each row is a
// permutation by reading it back), then follow proposal chains with the bid
// words and positions in shared memory, exactly as the tail kernel does, and
// finally write match[] and the proposal count.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "common.cuh"
#include "smp_b200.h"

namespace smpb200 {
namespace {

constexpr int kStaticMaxN = SMP_B200_STATIC_MAX_N;
constexpr size_t kHeaderBytes = 256;
constexpr size_t kStaticScratchBytes =
    kHeaderBytes + static_cast<size_t>(kStaticMaxN) * kStaticMaxN * sizeof(uint16_t);
constexpr int kMaxDevices = 64;

struct StaticHeader {
  int32_t status;
  int32_t bad_value;
  unsigned long long proposals;
};

// The scratch.  Host code must not take this name's address as a device
// pointer: in host code it is only a stand-in, so the entry point asks the
// runtime for the device address once per device.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

__device__ __forceinline__ void static_report(StaticHeader *h, int status, int value) {
  if (atomicCAS(&h->status, 0, status) == 0) h->bad_value = value;
}

__global__ void __launch_bounds__(1024, 1) k_solve_static(const int32_t *__restrict__ pref_m,
                                                          const int32_t *__restrict__ pref_w, int n,
                                                          int32_t *__restrict__ match, unsigned char *scratch) {
  StaticHeader *hdr = reinterpret_cast<StaticHeader *>(scratch);
  uint16_t *rank = reinterpret_cast<uint16_t *>(scratch + kHeaderBytes);
  __shared__ uint32_t sbid[kStaticMaxN];  // rank << 16 | man, 0xFFFFFFFF = free
  __shared__ uint16_t spos[kStaticMaxN];  // position of each man's current proposal
  __shared__ int s_next;
  __shared__ unsigned long long s_props;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;

  // The array keeps the previous call's contents: clear the header first.
  if (tid == 0) {
    hdr->status = 0;
    hdr->bad_value = 0;
    hdr->proposals = 0;
    s_next = 0;
    s_props = 0;
  }
  // Positions start at 0: a relaxed read of a displaced man's position that
  // races with his own store then returns 0 or an earlier position, never
  // leftover shared memory from another kernel (resuming early only repeats
  // proposals that are rejected again).
  for (int w = tid; w < n; w += blockDim.x) {
    sbid[w] = 0xFFFFFFFFu;
    spos[w] = 0;
  }
  __syncthreads();

  // 1. Inversion, one row per warp: scatter, then read back to check the row
  //    is a permutation (a duplicate leaves a slot whose rank is not its own).
  bool bad = false;
  for (int w = warp; w < n; w += nwarps) {
    const int32_t *row = pref_w + static_cast<size_t>(w) * n;
    uint16_t *out = rank + static_cast<size_t>(w) * n;
    for (int r = lane; r < n; r += 32) {
      const int m = row[r];
      if (static_cast<unsigned>(m) < static_cast<unsigned>(n)) {
        out[m] = static_cast<uint16_t>(r);
      } else {
        bad = true;
      }
    }
    __syncwarp();
    for (int r = lane; r < n; r += 32) {
      const int m = row[r];
      if (static_cast<unsigned>(m) < static_cast<unsigned>(n) && out[m] != r) bad = true;
    }
  }
  if (bad) static_report(hdr, SMP_ERR_INVALID_INPUT, -1);
  __syncthreads();
  if (*reinterpret_cast<volatile int32_t *>(&hdr->status)) return;

  // 2. Proposal chains, warp per free man, 32 choices per step.
  int m = -1, pos = 0;
  for (;;) {
    if (m < 0) {
      int i = 0;
      if (lane == 0) i = atomicAdd(&s_next, 1);
      i = __shfl_sync(kFullMask, i, 0);
      if (i >= n) break;
      m = i;
      pos = 0;
    }
    const int r = pos + lane;
    int w = 0;
    uint32_t rk = 0xFFFFFFFFu;
    bool ok = true;
    if (r < n) {
      w = pref_m[static_cast<size_t>(m) * n + r];
      ok = static_cast<unsigned>(w) < static_cast<unsigned>(n);
      if (ok) rk = rank[static_cast<size_t>(w) * n + m];
    }
    const unsigned badm = __ballot_sync(kFullMask, !ok);
    if (badm) {
      if (lane == __ffs(badm) - 1) static_report(hdr, SMP_ERR_INVALID_INPUT, w);
      break;
    }
    const uint32_t cur = (r < n) ? lds_relaxed_u32(sbid + w) : 0u;
    unsigned cand = __ballot_sync(kFullMask, r < n && rk < (cur >> 16));
    bool moved = false;
    while (cand) {
      const int j = __ffs(cand) - 1;
      uint32_t old = 0;
      int next_pos = 0;
      if (lane == j) {
        spos[m] = static_cast<uint16_t>(r);
        old = atom_min_relaxed_shared(sbid + w, (rk << 16) | static_cast<uint32_t>(m));
        if ((old >> 16) > rk && old != 0xFFFFFFFFu) next_pos = spos[old & 0xFFFFu] + 1;
      }
      old = __shfl_sync(kFullMask, old, j);
      next_pos = __shfl_sync(kFullMask, next_pos, j);
      const uint32_t rkj = __shfl_sync(kFullMask, rk, j);
      if ((old >> 16) > rkj) {
        m = (old == 0xFFFFFFFFu) ? -1 : static_cast<int>(old & 0xFFFFu);
        pos = next_pos;
        moved = true;
        break;
      }
      cand &= cand - 1;
    }
    if (!moved) {
      pos += 32;
      if (pos >= n) {  // rejected by every woman: the lists are not permutations
        if (lane == 0) static_report(hdr, SMP_ERR_INVALID_INPUT, m);
        break;
      }
    }
  }
  __syncthreads();
  if (*reinterpret_cast<volatile int32_t *>(&hdr->status)) return;

  // 3. match[m] = w and the proposal count.
  unsigned long long props = 0;
  for (int w = tid; w < n; w += blockDim.x) {
    const uint32_t b = sbid[w];
    if (b == 0xFFFFFFFFu) {
      static_report(hdr, SMP_ERR_INVALID_INPUT, w);
      continue;
    }
    match[b & 0xFFFFu] = w;
  }
  for (int mm = tid; mm < n; mm += blockDim.x) props += spos[mm] + 1ull;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) props += __shfl_down_sync(kFullMask, props, off);
  if (lane == 0) atomicAdd(&s_props, props);
  __syncthreads();
  if (tid == 0) hdr->proposals = s_props;
}

std::mutex g_setup_mutex;
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device (looked up once
// per device, with that device current).
int scratch_address(int device, void **out) {
  if (device < 0 || device >= kMaxDevices) return SMP_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return SMP_ERR_CUDA;
    }
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return SMP_OK;
}

}  // namespace
}  // namespace smpb200

extern "C" int smp_b200_solve_static(const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *match_out,
                                     int64_t *proposals, void *stream) {
  using namespace smpb200;
  if (!pref_m || !pref_w || !match_out || n <= 0) return SMP_ERR_INVALID_ARG;
  if (n > kStaticMaxN) return SMP_ERR_UNSUPPORTED;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return SMP_ERR_CUDA;
  }
  void *scratch = nullptr;
  int rc = scratch_address(device, &scratch);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_solve_static<<<1, 1024, 0, s>>>(pref_m, pref_w, n, match_out, static_cast<unsigned char *>(scratch));
  if (cudaGetLastError() != cudaSuccess) return SMP_ERR_CUDA;
  StaticHeader hdr = {};
  if (cudaMemcpyAsync(&hdr, scratch, sizeof(hdr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return SMP_ERR_CUDA;
  }
  if (hdr.status) return hdr.status;
  if (proposals) *proposals = static_cast<int64_t>(hdr.proposals);
  return SMP_OK;
}
