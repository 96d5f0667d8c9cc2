// batch_kernels.cuh -- many independent instances in one persistent launch.
//
// The reference solves one instance per engine object
// (benchmark/smp_engine_exec.h:6-32); a batch here is a device table of
// instances that CTAs pull from a queue, largest first.  One CTA solves one
// instance at a time, start to finish:
//   1. inversion: warps invert the women's rows into a uint16 rank matrix --
//      in shared memory when it fits the CTA's rank region (small
//      instances), else in the CTA's own slab in global memory -- checking
//      each row is a permutation by reading it back;
//   2. proposals: the bid words (rank << 16 | man) and each man's position
//      live in shared memory, and warps follow displacement chains exactly as
//      the single-instance tail kernel does, looking ahead up to kMaxSub
//      windows of 32 choices per step;
//   3. match[m] = w, the proposal count and a status go back to the table.
// The same kernel launched with one instance per launch is the plain
// per-instance baseline the batched launch is measured against.
#pragma once

#include "common.cuh"
#include "smp_b200.h"
#include "step.cuh"

namespace smpb200 {

// Device-side row of the instance table (the host mirrors smp_instance).
struct BatchInstance {
  const int32_t *pref_m;
  const int32_t *pref_w;
  int32_t *match;
  int32_t n;
  int32_t status;
  unsigned long long proposals;
};

// Shared memory for one instance of size n: bids and positions, padded to
// 16 bytes; the rank region for small instances follows.
__host__ __device__ constexpr size_t batch_smem_bytes(int max_n) {
  return (static_cast<size_t>(max_n) * 4 + static_cast<size_t>(max_n) * 2 + 15) & ~static_cast<size_t>(15);
}

// Slab inversion in groups of rows through the shared rank region (free
// while the instance's matrix lives in the slab).  Scattering each woman's
// row straight into the slab cost a random 2-byte store and a random
// read-back per entry, two L2 sector transactions each: about 70 % of a
// batch.  Here the CTA takes G women at a time, G = rows of `slots` (16-byte
// aligned, with room for the destination's offset) that fit the region, at
// most one per warp; each woman's warps stream her row with 16-byte loads and
// scatter it into her shared row, placed at the destination row's offset from
// a 16-byte boundary; then all threads write the group out with 16-byte
// stores, checking that no slot stayed unset (a row that is not a
// permutation).
__device__ __forceinline__ int batch_row_slots(int n) { return ((n + 7) / 8) * 8 + 8; }

__device__ __forceinline__ void batch_scatter(uint16_t *srow, int m, int r, int n, bool &bad) {
  if (static_cast<unsigned>(m) < static_cast<unsigned>(n)) {
    srow[m] = static_cast<uint16_t>(r);
  } else {
    bad = true;
  }
}

__device__ __forceinline__ void batch_invert_slab(const int32_t *__restrict__ pref_w, uint16_t *slab, int n, int G,
                                                  uint16_t *buf, bool &bad, bool store = true) {
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int warp = tid >> 5;
  const int wpr = (nthr >> 5) / G;  // warps per woman
  const int g = warp / wpr;         // this warp's woman in the group (g >= G: none)
  const int sub = (warp % wpr) * 32 + (tid & 31);
  const int subn = wpr * 32;
  const int rs = batch_row_slots(n);
  const int cmax = rs / 8;
  uint4 *b4 = reinterpret_cast<uint4 *>(buf);
  for (int w0 = 0; w0 < n; w0 += G) {
    for (int c = tid; c < G * cmax; c += nthr) b4[c] = make_uint4(~0u, ~0u, ~0u, ~0u);
    __syncthreads();
    const int w = w0 + g;
    if (g < G && w < n) {
      const int32_t *row = pref_w + static_cast<size_t>(w) * n;
      const int pre = static_cast<int>((reinterpret_cast<uintptr_t>(slab + static_cast<size_t>(w) * n) & 15u) >> 1);
      uint16_t *srow = buf + g * rs + pre;
      const int head = min(n, static_cast<int>(((16u - (reinterpret_cast<uintptr_t>(row) & 15u)) & 15u) >> 2));
      if (sub < head) batch_scatter(srow, __ldcs(row + sub), sub, n, bad);
      const int nq = (n - head) >> 2;
      const int4 *rq = reinterpret_cast<const int4 *>(row + head);
      for (int i = sub; i < nq; i += subn) {
        const int4 q = __ldcs(rq + i);
        const int r = head + 4 * i;
        batch_scatter(srow, q.x, r, n, bad);
        batch_scatter(srow, q.y, r + 1, n, bad);
        batch_scatter(srow, q.z, r + 2, n, bad);
        batch_scatter(srow, q.w, r + 3, n, bad);
      }
      for (int t = head + 4 * nq + sub; t < n; t += subn) batch_scatter(srow, __ldcs(row + t), t, n, bad);
    }
    __syncthreads();
    for (int idx = tid; idx < G * cmax; idx += nthr) {
      const int gg = idx / cmax, c = idx - gg * cmax;
      const int ww = w0 + gg;
      if (ww >= n) continue;
      uint16_t *out = slab + static_cast<size_t>(ww) * n;
      const int pre = static_cast<int>((reinterpret_cast<uintptr_t>(out) & 15u) >> 1);
      if (c >= (pre + n + 7) / 8) continue;
      const uint4 v = b4[gg * cmax + c];
      const int first = c * 8 - pre;  // row element in the chunk's first slot
      if (first >= 0 && first + 8 <= n) {
        bad |= (__vcmpeq2(v.x, 0xFFFFFFFFu) | __vcmpeq2(v.y, 0xFFFFFFFFu) | __vcmpeq2(v.z, 0xFFFFFFFFu) |
                __vcmpeq2(v.w, 0xFFFFFFFFu)) != 0u;
        if (store) reinterpret_cast<uint4 *>(out - pre)[c] = v;
      } else {
        const uint16_t *vals = reinterpret_cast<const uint16_t *>(&v);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int e = first + k;
          if (e >= 0 && e < n) {
            bad |= vals[k] == 0xFFFFu;
            if (store) out[e] = vals[k];
          }
        }
      }
    }
    __syncthreads();
  }
}

// rank_smem_elems: uint16 slots of shared memory after the bids; an instance
// whose n*n rank matrix fits there keeps it on chip (small instances), the
// others use the CTA's slab in global memory.
template <int kMaxSub>
__global__ void __launch_bounds__(512, 2) k_batch(BatchInstance *__restrict__ table, const int32_t *__restrict__ order,
                                               int count, int *queue, uint16_t *__restrict__ slabs,
                                               size_t slab_elems, int max_n, int dynamic, int rank_smem_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *sbid = reinterpret_cast<uint32_t *>(smem_raw);
  uint16_t *spos = reinterpret_cast<uint16_t *>(smem_raw + static_cast<size_t>(max_n) * 4);
  uint16_t *srank = reinterpret_cast<uint16_t *>(smem_raw + batch_smem_bytes(max_n));
  __shared__ int s_idx;
  __shared__ int s_next_man;
  __shared__ int s_status;
  __shared__ int s_bad;
  __shared__ unsigned long long s_props;
  __shared__ int s_swap;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  uint16_t *const slab = slabs + static_cast<size_t>(blockIdx.x) * slab_elems;

  for (int round = 0;; ++round) {
    if (tid == 0) s_idx = dynamic ? atomicAdd(queue, 1) : (round == 0 ? static_cast<int>(blockIdx.x) : count);
    __syncthreads();
    const int k = s_idx;
    if (k >= count) return;
    BatchInstance *inst = table + order[k];
    const int n = inst->n;
    const int32_t *pref_m = inst->pref_m;
    const int32_t *pref_w = inst->pref_w;
    if (n <= 0 || n > max_n || n > 65535) {
      if (tid == 0) {
        inst->status = SMP_ERR_UNSUPPORTED;
        inst->proposals = 0;
      }
      __syncthreads();
      continue;
    }
    uint16_t *const rank =
        static_cast<long long>(n) * n <= static_cast<long long>(rank_smem_elems) ? srank : slab;
    if (tid == 0) {
      s_next_man = 0;
      s_status = 0;
      s_bad = 0;
      s_props = 0;
      s_swap = 2 * n <= rank_smem_elems && n >= 16;  // n >= 16: a row fits the bid words' memory
    }
    __syncthreads();

    // 0. Do all men share one list?  Then the stable matching is unique --
    // woman pi_1 gets her favourite man, pi_2 her favourite of the rest, ...
    // -- so the women-proposing run finds the same matching, with about
    // n ln n proposals instead of the men's n (n + 1) / 2; and the men's
    // proposal count is n (n + 1) / 2, each woman's place in the shared list
    // counted once.  The first choices are screened first; the full
    // comparison reads pref_m once.
    volatile int *swap_flag = &s_swap;
    if (*swap_flag) {
      const int first = __ldg(pref_m);
      for (int m = tid; m < n; m += blockDim.x)
        if (__ldg(pref_m + static_cast<size_t>(m) * n) != first) *swap_flag = 0;
    }
    __syncthreads();
    uint16_t *const inv = srank;      // inv[w] = her place in the shared list
    uint16_t *const row0 = srank + n;  // the shared list
    if (s_swap) {
      for (int w = tid; w < n; w += blockDim.x) inv[w] = 0xFFFFu;
      __syncthreads();
      for (int r = tid; r < n; r += blockDim.x) {
        const int w = __ldg(pref_m + r);
        if (static_cast<unsigned>(w) < static_cast<unsigned>(n)) {
          row0[r] = static_cast<uint16_t>(w);
          inv[w] = static_cast<uint16_t>(r);
        } else {
          *swap_flag = 0;  // the ordinary path reports it
        }
      }
      __syncthreads();
      for (int w = tid; w < n; w += blockDim.x)
        if (inv[w] == 0xFFFFu) *swap_flag = 0;  // not a permutation: the ordinary path reports it
      for (int m = 1 + warp; m < n; m += nwarps) {
        int go = 0;
        if (lane == 0) go = *swap_flag;
        if (!__shfl_sync(kFullMask, go, 0)) break;  // the whole warp leaves together
        const int32_t *row = pref_m + static_cast<size_t>(m) * n;
        bool same = true;
        for (int r = lane; r < n; r += 32) same &= __ldg(row + r) == static_cast<int>(row0[r]);
        if (!__all_sync(kFullMask, same) && lane == 0) *swap_flag = 0;
      }
      __syncthreads();
    }
    if (s_swap) {
      // the women's lists must be permutations too: checked in groups of
      // rows through the bid words' shared memory, which is free until now
      bool bad = false;
      const int G = min(static_cast<int>(batch_smem_bytes(max_n) / 2) / batch_row_slots(n), nwarps);
      batch_invert_slab(pref_w, slab, n, G, reinterpret_cast<uint16_t *>(smem_raw), bad, false);
      if (bad) s_status = SMP_ERR_INVALID_INPUT;
      __syncthreads();
      for (int m = tid; m < n; m += blockDim.x) {
        sbid[m] = 0xFFFFFFFFu;  // the men, holding no woman
        spos[m] = 0;            // the women's positions (a racing relaxed read sees 0, never leftovers)
      }
      __syncthreads();
      {
        // women propose down their lists; every man ranks a woman by her
        // place in the shared list
        const SharedBids bids{sbid, spos};
        const auto keep_going = [&]() { return *reinterpret_cast<volatile int *>(&s_status) == 0; };
        int m = -1, pos = 0, S = 1, bad_value = 0;
        Ahead ahead;
        unsigned long long settled = 0;
        unsigned int hops = 0;
        while (keep_going()) {
          if (m < 0) {
            int i = 0;
            if (lane == 0) i = atomicAdd(&s_next_man, 1);
            i = __shfl_sync(kFullMask, i, 0);
            if (i >= n) break;
            m = i;
            pos = 0;
            S = 1;
          }
          const int rc = man_step<kMaxSub, true, false, 1, 3>(bids, keep_going, pref_w,
                                                               static_cast<const uint16_t *>(inv),
                                                               static_cast<const uint32_t *>(nullptr), 0, n, false,
                                                               lane, m, pos, S, ahead, settled, hops, bad_value);
          if (rc == kStepMoved || rc == kStepMatchedFree) continue;
          if (rc == kStepBad && lane == 0) s_status = SMP_ERR_INVALID_INPUT;
          break;
        }
      }
      __syncthreads();
      if (!s_status)
        for (int m = tid; m < n; m += blockDim.x) {
          const uint32_t b = sbid[m];
          if (b == 0xFFFFFFFFu) {
            s_bad = 1;
            continue;
          }
          inst->match[m] = static_cast<int32_t>(b & 0xFFFFu);
        }
      __syncthreads();
      if (tid == 0) {
        inst->status = s_status ? s_status : (s_bad ? SMP_ERR_INVALID_INPUT : SMP_OK);
        inst->proposals = s_status || s_bad ? 0ull : static_cast<unsigned long long>(n) * (n + 1) / 2;
      }
      __syncthreads();
      continue;
    }
    // Positions start at 0, so a relaxed read of a displaced man's position
    // that races with his own store returns an earlier position (resuming
    // there only repeats rejected proposals), never leftover shared memory.
    for (int w = tid; w < n; w += blockDim.x) {
      sbid[w] = 0xFFFFFFFFu;
      spos[w] = 0;
    }
    __syncthreads();

    // 1. inversion: through the shared region in groups of rows when the
    // matrix lives in the slab, else one row per warp, checked by reading
    // the row back
    bool bad = false;
    const int groups = rank == slab ? min(rank_smem_elems / batch_row_slots(n), nwarps) : 0;
    if (groups >= 1) batch_invert_slab(pref_w, slab, n, groups, srank, bad);
    for (int w = groups >= 1 ? n : warp; w < n; w += nwarps) {
      const int32_t *row = pref_w + static_cast<size_t>(w) * n;
      uint16_t *out = rank + static_cast<size_t>(w) * n;
      for (int r = lane; r < n; r += 32) {
        const int m = __ldg(row + r);
        if (static_cast<unsigned>(m) < static_cast<unsigned>(n)) {
          out[m] = static_cast<uint16_t>(r);
        } else {
          bad = true;
        }
      }
      __syncwarp();
      for (int r = lane; r < n; r += 32) {
        const int m = __ldg(row + r);
        if (static_cast<unsigned>(m) < static_cast<unsigned>(n) && out[m] != r) bad = true;
      }
    }
    if (bad) s_status = SMP_ERR_INVALID_INPUT;
    __syncthreads();

    // 2. proposal chains, warp per free man (the step the tail kernel uses)
    {
      const SharedBids bids{sbid, spos};
      const auto keep_going = [&]() { return *reinterpret_cast<volatile int *>(&s_status) == 0; };
      int m = -1, pos = 0, S = 1, bad_value = 0;
      Ahead ahead;
      unsigned long long settled = 0;
      unsigned int hops = 0;
      while (keep_going()) {
        if (m < 0) {
          int i = 0;
          if (lane == 0) i = atomicAdd(&s_next_man, 1);
          i = __shfl_sync(kFullMask, i, 0);
          if (i >= n) break;
          m = i;
          pos = 0;
          S = 1;
        }
        const int rc = man_step<kMaxSub, true, false>(bids, keep_going, pref_m, static_cast<const uint16_t *>(rank),
                                                      static_cast<const uint32_t *>(nullptr),
                                         0, n, false, lane, m, pos, S, ahead, settled, hops, bad_value);
        if (rc == kStepMoved || rc == kStepMatchedFree) continue;
        if (rc == kStepBad && lane == 0) s_status = SMP_ERR_INVALID_INPUT;
        break;
      }
    }
    __syncthreads();

    // 3. outputs
    if (!s_status) {
      unsigned long long props = 0;
      for (int w = tid; w < n; w += blockDim.x) {
        const uint32_t b = sbid[w];
        if (b == 0xFFFFFFFFu) {
          s_bad = 1;
          continue;
        }
        inst->match[b & 0xFFFFu] = w;
      }
      for (int mm = tid; mm < n; mm += blockDim.x) props += spos[mm] + 1ull;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) props += __shfl_down_sync(kFullMask, props, off);
      if (lane == 0) atomicAdd(&s_props, props);
    }
    __syncthreads();
    if (tid == 0) {
      inst->status = s_status ? s_status : (s_bad ? SMP_ERR_INVALID_INPUT : SMP_OK);
      inst->proposals = s_status || s_bad ? 0ull : s_props;
    }
    __syncthreads();
  }
}

}  // namespace smpb200
