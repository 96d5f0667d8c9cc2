// common.cuh -- device-side building blocks shared by every kernel of the
// B200 stable-marriage solver: the per-solve control block, the packed bid
// word, relaxed/acquire-release PTX memory operations and Philox4x32-10.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace smpb200 {

constexpr unsigned kFullMask = 0xFFFFFFFFu;

// Status codes written by kernels; the values equal smp_status.
constexpr int kStatusOk = 0;
constexpr int kStatusInvalidInput = 2;

// Modes of one solve, chosen on the device by the precheck.
constexpr int kModeRank = 0;   // rank matrix, prefix gathered from it; any instance
constexpr int kModeQuery = 1;  // prefix answered straight from pref_w rows, no rank matrix

// Per-solve control block in device memory.  Kernels of one solve share it;
// the host writes its initial value (free_count = n, the allow_* switches)
// before the solve.
struct Control {
  int32_t status;         // first error a kernel saw (kStatus*), 0 if none
  int32_t perfect;        // precheck: every first choice distinct (and allowed)
  int32_t next_man;       // bulk kernel: next man that has not proposed yet
  int32_t free_count;     // women that have not received a proposal yet
  int32_t tail_count;     // men handed from the bulk kernel to the tail kernel
  int32_t tail_men;       // men the tail kernel started chains for
  int32_t bad_value;      // first out-of-range preference value seen
  int32_t mode;           // kModeRank or kModeQuery
  int32_t retry;          // query mode met a man beyond his prefix: rerun in rank mode
  int32_t allow_perfect;  // host switch: 0 disables the distinct-first-choices shortcut
  int32_t allow_query;    // host switch: 1 if the query mode may be chosen
  int32_t blocks_done;    // precheck: blocks that finished (the last one decides)
  int32_t distinct;       // precheck: number of distinct first choices
  int32_t distinct_w;     // k_wdistinct: distinct first choices of the women
  int32_t use_filter;     // k_wdistinct: k_bulk runs with its shared partner-rank filter
  int32_t swap_fail;      // k_swap_screen: a pref_m row differs from row 0
  unsigned long long proposals;        // sum over men of (final position + 1)
  unsigned long long blocking;         // checker: blocking pairs
  unsigned long long check_proposals;  // checker: proposals recounted from the matching
  unsigned long long bulk_proposals;   // proposals settled by k_bulk
  unsigned long long tail_proposals;   // proposals settled by k_tail
  unsigned int bulk_hops;              // accepted proposals in k_bulk
  unsigned int tail_hops;              // accepted proposals in k_tail
  // Chains k_tail handed to k_tail_coop (man, next position), at most one
  // per warp of the tail CTA; coop_count is 0 when none are waiting.
  int32_t coop_count;
  int32_t swap_next;      // k_swap_gs: next woman that has not proposed yet
  int32_t w_differ;       // k_swap_screen: a pref_w row differs from row 0
  int32_t swap_over;      // k_swap_gs: women stopped at the end of what the device holds of their rows
  int2 coop_chain[32];
};

__device__ __forceinline__ void report(Control *ctrl, int status, int value) {
  if (atomicCAS(&ctrl->status, 0, status) == 0) ctrl->bad_value = value;
}

// ---------------------------------------------------------------------------
// Bid word of a woman in global memory (64 bits):
//   rank of her current partner (21 bits) << 42 | partner (21) << 21 | the
//   position of this woman in the partner's list (21).
// A smaller word means a better partner for her (ranks of one woman are
// distinct), so atomicMin keeps the best proposal and returns the displaced
// one together with where that man resumes.  kFree (all ones) means no
// proposal yet.
// ---------------------------------------------------------------------------
constexpr unsigned long long kFree = ~0ull;
constexpr uint32_t kMask21 = (1u << 21) - 1;

__device__ __forceinline__ unsigned long long pack_bid(uint32_t rank, uint32_t man,
                                                       uint32_t pos) {
  return (static_cast<unsigned long long>(rank) << 42) |
         (static_cast<unsigned long long>(man) << 21) | pos;
}
__device__ __forceinline__ uint32_t bid_rank(unsigned long long b) {
  return static_cast<uint32_t>(b >> 42);
}
__device__ __forceinline__ uint32_t bid_man(unsigned long long b) {
  return static_cast<uint32_t>(b >> 21) & kMask21;
}
__device__ __forceinline__ uint32_t bid_pos(unsigned long long b) {
  return static_cast<uint32_t>(b) & kMask21;
}

// ---------------------------------------------------------------------------
// Memory operations with explicit PTX semantics.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_s32(const int *p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_volatile_s32(const int *p) {
  return *reinterpret_cast<const volatile int *>(p);
}

// Grid-strided L2 prefetch of [p, p + bytes), one request per 128-byte line.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
  const char *base = static_cast<const char *>(p);
  const size_t lines = (bytes + 127) / 128;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < lines; i += stride)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(base + i * 128));
}

// Shared-memory helpers for the single-CTA tail.
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t lds_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_addr(p)) : "memory");
  return v;
}
// Relaxed atomicMin on a shared word.  The proposals of the one-CTA kernels
// use it with no fence: a release would first wait for every load the thread
// has in flight, including the next man's window issued just before (Ahead),
// which puts a global round trip back on the chain of displacements.  The
// position a displaced man resumes from is read from a separate array after
// the atomic; without ordering that read can only return one of his earlier
// positions (only he writes it, and it only grows), and resuming there just
// repeats proposals that are rejected again, because every woman he proposed
// to since holds a partner she ranks above him.  The matching and the
// proposal count (taken from the final positions) do not change.
__device__ __forceinline__ uint32_t atom_min_relaxed_shared(uint32_t *p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.relaxed.cta.shared::cta.min.u32 %0, [%1], %2;"
               : "=r"(old) : "r"(smem_addr(p)), "r"(v) : "memory");
  return old;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the counter-based
// generator behind every seeded workload.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                       uint32_t c3, uint32_t k0, uint32_t k1,
                                                       uint32_t out[4]) {
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
    const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
    const uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c3 ^ k1;
    c1 = static_cast<uint32_t>(p1);
    c3 = static_cast<uint32_t>(p0);
    c0 = n0;
    c2 = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

}  // namespace smpb200
