// Single solves whose men all share one list: the women propose.
//
// When every man ranks the women in the same order L, the stable matching is
// unique (each woman, taken in L's order, gets her best man not taken by a
// woman before her), so the women-proposing run returns the matching the
// men-proposing Gale-Shapley of the reference returns
// (src/smp/smp_engine_gs_1.cu:47-98).  The men's run would make n(n+1)/2
// proposals -- the man who ends with L[k] proposed to L[0..k] -- and needs the
// full rank matrix; the women's run makes about n ln n proposals and ranks
// every proposer by one inverted row, pos[w] = position of w in L.
//
//   k_swap_pos     pos = inverse of pref_m row 0; row 0 must be a permutation
//   k_swap_screen  every pref_m row equals row 0 (else swap_fail), and every
//                  pref_w row is a permutation (else the invalid-input status)
//   k_swap_gs      the women's proposals, one warp per chain
//   k_swap_rows_check, k_swap_mark_full
//                  host-input solves: the parts of pref_w sent, checked, and
//                  which rows are whole
//   k_swap_match   match[m] from the men's final bids; the men's proposal count
//   k_swap_direct  women who share one list M as well: match[M[k]] = L[k]
//                  (the k-th man of the women's list with the k-th woman of
//                  the men's), no proposals
#pragma once

#include "common.cuh"
#include "solve_kernels.cuh"

namespace smpb200 {

// pos[L[r]] = r, with pos preset to -1; an entry out of range or seen twice
// makes row 0 no permutation.
__global__ void k_swap_pos(const int32_t *__restrict__ pref_m, int32_t *__restrict__ pos, int n, Control *ctrl) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int w = __ldg(pref_m + r);
    if (static_cast<unsigned>(w) >= static_cast<unsigned>(n) || atomicCAS(pos + w, -1, r) != -1)
      report(ctrl, kStatusInvalidInput, w);
  }
}

// Rows t = 1 .. n-1 compare pref_m row t with row 0; rows t = n .. 2n-1
// check that pref_w row t-n is a permutation with a shared bitmap.  A solve
// whose men's rows were compared on the host (host-input solves) starts at
// t0 = n: only row 0 of pref_m is then on the device.  Row
// bodies move in 16-byte loads (row_span: rows start off 16-byte boundaries
// when n is not a multiple of 4).  Once a pref_m row differs, the solve
// takes the men's rank-mode pass, which checks pref_w itself: the CTAs stop.
// (One colour byte per man with plain stores and a check pass, instead of the
// bitmap's shared atomics, took 1.85 ms against 1.47 ms at n = 30000.)
__host__ __device__ constexpr size_t swap_screen_smem(int n) { return ((static_cast<size_t>(n) + 31) / 32) * 4; }

__global__ void __launch_bounds__(256) k_swap_screen(const int32_t *__restrict__ pref_m,
                                                     const int32_t *__restrict__ pref_w, int n, Control *ctrl,
                                                     int t0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *seen = reinterpret_cast<uint32_t *>(smem_raw);
  __shared__ int s_stop;
  __shared__ int s_wsame;  // no pref_w row has differed from row 0 yet
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int words = (n + 31) >> 5;
  bool bad = false;
  int bad_value = 0;
  for (int t = t0 + static_cast<int>(blockIdx.x); t < 2 * n; t += gridDim.x) {
    if (tid == 0) {
      s_stop = ld_volatile_s32(&ctrl->swap_fail) || ld_volatile_s32(&ctrl->status);
      s_wsame = !ld_volatile_s32(&ctrl->w_differ);
    }
    __syncthreads();
    if (s_stop) break;
    if (t < n) {
      // pref_m row t against row 0: chunk by chunk where both rows start at
      // the same 16-byte offset (all rows when n is a multiple of 4), else
      // each chunk against four entries of row 0
      const RowSpan s = row_span(pref_m, t, n);
      bool differs = false;
      if (s.head == row_span(pref_m, 0, n).head) {
        const int4 *q0 = reinterpret_cast<const int4 *>(pref_m + s.head);
        for (int i = tid; i < s.nq; i += nthr) {
          const int4 v = __ldcs(s.rq + i);
          const int4 u = __ldg(q0 + i);
          differs |= v.x != u.x || v.y != u.y || v.z != u.z || v.w != u.w;
        }
      } else {
        for (int i = tid; i < s.nq; i += nthr) {
          const int4 v = __ldcs(s.rq + i);
          const int c = s.head + 4 * i;
          differs |= v.x != __ldg(pref_m + c) || v.y != __ldg(pref_m + c + 1) || v.z != __ldg(pref_m + c + 2) ||
                     v.w != __ldg(pref_m + c + 3);
        }
      }
      if (tid < s.head) differs |= __ldcs(s.row + tid) != __ldg(pref_m + tid);
      const int c0 = s.head + 4 * s.nq;
      if (tid < s.tail) differs |= __ldcs(s.row + c0 + tid) != __ldg(pref_m + c0 + tid);
      if (__syncthreads_or(differs) && tid == 0) atomicExch(&ctrl->swap_fail, 1);
    } else {
      // pref_w row t - n: every value in range and seen once; while no
      // row has differed, also compared with row 0 (the women may share one
      // list as well)
      for (int i = tid; i < words; i += nthr) seen[i] = 0u;
      __syncthreads();
      const RowSpan s = row_span(pref_w, t - n, n);
      if (s_wsame && t > n) {
        bool differs = false;
        for (int i = tid; i < s.nq; i += nthr) {
          const int4 v = __ldcs(s.rq + i);
          const int c = s.head + 4 * i;
          differs |= v.x != __ldg(pref_w + c) || v.y != __ldg(pref_w + c + 1) || v.z != __ldg(pref_w + c + 2) ||
                     v.w != __ldg(pref_w + c + 3);
        }
        if (tid < s.head) differs |= __ldcs(s.row + tid) != __ldg(pref_w + tid);
        const int c0 = s.head + 4 * s.nq;
        if (tid < s.tail) differs |= __ldcs(s.row + c0 + tid) != __ldg(pref_w + c0 + tid);
        if (__syncthreads_or(differs) && tid == 0) atomicExch(&ctrl->w_differ, 1);  // one flag per CTA and row
      }
      const auto mark = [&](int v) {
        if (static_cast<unsigned>(v) >= static_cast<unsigned>(n)) {
          bad = true;
          bad_value = v;
          return;
        }
        const uint32_t bit = 1u << (v & 31);
        if (atomicOr(seen + (v >> 5), bit) & bit) {
          bad = true;
          bad_value = v;
        }
      };
      for (int i = tid; i < s.nq; i += nthr) {
        const int4 v = __ldcs(s.rq + i);
        mark(v.x);
        mark(v.y);
        mark(v.z);
        mark(v.w);
      }
      if (tid < s.head) mark(__ldcs(s.row + tid));
      if (tid < s.tail) mark(__ldcs(s.row + s.head + 4 * s.nq + tid));
      __syncthreads();  // the bitmap is cleared for the next row only after this one
    }
  }
  if (bad) report(ctrl, kStatusInvalidInput, bad_value);
}

// The women's proposals.  A man's bid word is pos[w] << 32 | r for the woman
// w he holds and her position r in her list (~0 while he is free), so
// atomicMin keeps the woman the men prefer and hands back the one it
// displaced together with where she resumes.  Each warp carries one woman:
// her next 32 men are read at once, the first man whose current word is
// worse than hers takes her proposal, and a displaced woman continues in the
// same warp.
//   Rows on the device: with full == nullptr every woman's whole row; else
// woman w's whole row where full[w] is set and her first `depth` entries
// otherwise (host-input solves send only those).  A woman who reaches the
// end of what the device holds of her row stops and is appended to `over`
// as (w, position), to resume once her row has been sent (start/start_count
// then list the women this launch resumes, instead of women 0..n-1 from
// position 0).  Gale-Shapley's result does not depend on that order.  An
// entry out of range is reported; a woman who runs out of her whole row
// (input that is not a permutation) too.
__global__ void __launch_bounds__(256) k_swap_gs(const int32_t *__restrict__ pref_m,
                                                 const int32_t *__restrict__ pref_w,
                                                 const int32_t *__restrict__ pos,
                                                 unsigned long long *__restrict__ bid, int n, Control *ctrl,
                                                 const uint8_t *__restrict__ full, int depth,
                                                 int2 *__restrict__ over, const int2 *__restrict__ start,
                                                 int start_count) {
  const int lane = threadIdx.x & 31;
  const int total = start ? start_count : n;
  int w = -1, r0 = 0;
  uint32_t key = 0;
  for (;;) {
    if (w < 0) {
      int i = 0;
      if (lane == 0) i = atomicAdd(&ctrl->swap_next, 1);
      i = __shfl_sync(kFullMask, i, 0);
      if (i >= total) break;
      if (start) {
        const int2 e = start[i];
        w = e.x;
        r0 = e.y;
      } else {
        w = i;
        r0 = 0;
      }
      key = static_cast<uint32_t>(__ldg(pos + w));
    }
    const int lim = (full == nullptr || full[w]) ? n : depth;  // entries of her row on the device
    if (r0 >= lim) {
      if (lane == 0) {
        if (lim >= n) {
          report(ctrl, kStatusInvalidInput, w);
        } else {
          // at most n: a woman who stops holds no man, so nothing sends her
          // back into this launch
          const int k = atomicAdd(&ctrl->swap_over, 1);
          if (k < n)
            over[k] = make_int2(w, r0);
          else
            report(ctrl, kStatusInvalidInput, w);
        }
      }
      w = -1;
      continue;
    }
    const int r = r0 + lane;
    const bool in_row = r < lim;
    const int m = in_row ? __ldg(pref_w + static_cast<size_t>(w) * n + r) : 0;
    const bool valid = static_cast<unsigned>(m) < static_cast<unsigned>(n);
    const bool open = in_row && valid && static_cast<uint32_t>(ld_relaxed_u64(bid + m) >> 32) > key;
    const unsigned hit = __ballot_sync(kFullMask, open);
    const unsigned bad = __ballot_sync(kFullMask, in_row && !valid);
    if (bad) {  // an entry out of range
      if (lane == __ffs(bad) - 1) report(ctrl, kStatusInvalidInput, m);
      w = -1;
      continue;
    }
    if (!hit) {
      r0 = min(r0 + 32, lim);
      continue;
    }
    const int f = __ffs(hit) - 1;
    unsigned long long old = 0;
    if (lane == f)
      old = atomicMin(bid + m, (static_cast<unsigned long long>(key) << 32) | static_cast<uint32_t>(r));
    old = __shfl_sync(kFullMask, old, f);
    if (static_cast<uint32_t>(old >> 32) < key) {  // a woman the men prefer got there first
      r0 += f + 1;
      continue;
    }
    if (old == ~0ull) {  // he was free: the chain ends
      w = -1;
      continue;
    }
    key = static_cast<uint32_t>(old >> 32);
    w = __ldg(pref_m + key);
    r0 = static_cast<int>(old & 0xFFFFFFFFull) + 1;
  }
}

// Host-input shared-list solves: checks the entries of pref_w the device
// holds -- the first `cols` of every row (rows == nullptr: rows 0..count-1)
// or of the listed rows -- are in range and name no man twice.  One row per
// CTA at a time, n bits of shared memory.
__global__ void __launch_bounds__(256) k_swap_rows_check(const int32_t *__restrict__ pref_w, int n,
                                                         const int32_t *__restrict__ rows, int count, int cols,
                                                         Control *ctrl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *seen = reinterpret_cast<uint32_t *>(smem_raw);
  const int words = (n + 31) >> 5;
  bool bad = false;
  int bad_value = 0;
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const int w = rows ? __ldg(rows + i) : i;
    for (int k = threadIdx.x; k < words; k += blockDim.x) seen[k] = 0u;
    __syncthreads();
    if (static_cast<unsigned>(w) < static_cast<unsigned>(n)) {
      const int32_t *row = pref_w + static_cast<size_t>(w) * n;
      for (int r = threadIdx.x; r < cols; r += blockDim.x) {
        const int v = __ldg(row + r);
        if (static_cast<unsigned>(v) >= static_cast<unsigned>(n)) {
          bad = true;
          bad_value = v;
          continue;
        }
        const uint32_t bit = 1u << (v & 31);
        if (atomicOr(seen + (v >> 5), bit) & bit) {
          bad = true;
          bad_value = v;
        }
      }
    } else if (threadIdx.x == 0) {
      bad = true;
      bad_value = w;
    }
    __syncthreads();  // the bitmap is cleared for the next row only after this one
  }
  if (bad) report(ctrl, kStatusInvalidInput, bad_value);
}

// full[rows[i]] = 1 for the rows now whole on the device.
__global__ void k_swap_mark_full(uint8_t *__restrict__ full, const int32_t *__restrict__ rows, int count, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int w = __ldg(rows + i);
    if (static_cast<unsigned>(w) < static_cast<unsigned>(n)) full[w] = 1;
  }
}

// match[m] = the woman m holds; the men's proposal count of the same
// matching is n(n+1)/2 (final positions 0 .. n-1 in the shared list).
__global__ void k_swap_match(const int32_t *__restrict__ pref_m, const unsigned long long *__restrict__ bid,
                             int32_t *__restrict__ match, int n, Control *ctrl) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    const unsigned long long b = bid[m];
    if (b == ~0ull) {
      report(ctrl, kStatusInvalidInput, m);
      match[m] = -1;
    } else {
      match[m] = __ldg(pref_m + static_cast<uint32_t>(b >> 32));
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctrl->proposals = static_cast<unsigned long long>(n) * (static_cast<unsigned long long>(n) + 1) / 2;
    ctrl->bulk_proposals = ctrl->proposals;
    ctrl->tail_proposals = 0;
  }
}

// Both sides share one list each (L for the men, M for the women): the k-th
// man of M and the k-th woman of L pair up.  The men's proposal count is
// again n(n+1)/2.
__global__ void k_swap_direct(const int32_t *__restrict__ pref_m, const int32_t *__restrict__ pref_w,
                              int32_t *__restrict__ match, int n, Control *ctrl) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    match[__ldg(pref_w + k)] = __ldg(pref_m + k);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctrl->proposals = static_cast<unsigned long long>(n) * (static_cast<unsigned long long>(n) + 1) / 2;
    ctrl->bulk_proposals = ctrl->proposals;
    ctrl->tail_proposals = 0;
  }
}

}  // namespace smpb200
