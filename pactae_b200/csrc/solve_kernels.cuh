// solve_kernels.cuh -- the sm_100a kernels of one Gale-Shapley solve.
//
//   k_precheck   distinct first choices?   (SmpEngineBamboo::IsPerfect,
//                                           include/smp/smp_engine_bamboo.h:25-33)
//   k_invert     rank[w][pref_w[w][r]] = r (F9RankMatrixInitKernel,
//                                           src/smp/kernel.cu:672-686)
//   k_prefix     per-man (woman, rank) pairs for the first K choices, the
//                part of the reference's PR matrix (kernel.cu:688-709) that a
//                solve actually reads
//   k_bulk       proposals on every SM      (La3F9CoreKernel, kernel.cu:633-670)
//   k_tail       the last chains in one CTA (MonitorProceture + LAProcedure,
//                                           src/smp/smp_engine_bamboo.cu:197-287)
//   k_match      match[m] = w               (SmpEngineBamboo::PostProc,
//                                           smp_engine_bamboo.cu:289-306)
//   k_check_*    stability checker (no counterpart in the reference)
//
// Layouts (all row-major, 64-bit offsets):
//   pref_m, pref_w  int32 [n][n]
//   rank            RankT [n][n], RankT = uint16_t for n <= 65535, else int32
//   prefix          uint32 [n][K] = woman << 16 | rank of the man for her
//   bid             u64 [n] (see common.cuh)
#pragma once

#include "common.cuh"

namespace smpb200 {

// When an inversion kernel runs, given the precheck's verdict.
constexpr int kInvertAlways = 0;
constexpr int kInvertUnlessPerfect = 1;  // the solve's own inversion
constexpr int kInvertIfPerfect = 2;      // the checker after a perfect solve

__device__ __forceinline__ bool invert_skipped(int mode, const Control *ctrl) {
  if (mode == kInvertAlways) return false;
  const int perfect = ld_volatile_s32(&ctrl->perfect);
  return mode == kInvertUnlessPerfect ? perfect != 0 : perfect == 0;
}

// Unset marker of a rank-matrix slot during inversion: never a valid rank
// (uint16 ranks are < n <= 65535; int32 ranks are >= 0).
template <typename RankT>
__device__ __forceinline__ RankT rank_unset();
template <>
__device__ __forceinline__ uint16_t rank_unset<uint16_t>() { return 0xFFFFu; }
template <>
__device__ __forceinline__ int32_t rank_unset<int32_t>() { return -1; }

// ---------------------------------------------------------------------------
// Precheck: ctrl->perfect stays 1 iff the n first choices are distinct.
// seen: ceil(n/32) zeroed words.
// ---------------------------------------------------------------------------
__global__ void k_precheck(const int32_t *__restrict__ pref_m, int n,
                           uint32_t *__restrict__ seen, Control *ctrl) {
  const int stride = gridDim.x * blockDim.x;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += stride) {
    const int w = __ldg(pref_m + static_cast<size_t>(m) * n);
    if (static_cast<unsigned>(w) >= static_cast<unsigned>(n)) {
      report(ctrl, kStatusInvalidInput, w);
      ctrl->perfect = 0;
      continue;
    }
    const uint32_t bit = 1u << (w & 31);
    if (atomicOr(seen + (w >> 5), bit) & bit) ctrl->perfect = 0;
  }
}

// ---------------------------------------------------------------------------
// Inversion.  One CTA inverts one row of pref_w at a time: the row streams in
// with 16-byte loads, each (r, m) is scattered into a shared-memory copy of
// the rank row, and the finished row streams out with 16-byte stores.  A
// slot still unset after the scatter means the row was not a permutation.
// Dynamic shared memory: n * sizeof(RankT) bytes, 16-byte aligned.
// ---------------------------------------------------------------------------
template <typename RankT>
__device__ __forceinline__ void scatter_one(RankT *srow, int m, int r, int n, bool &bad) {
  if (static_cast<unsigned>(m) < static_cast<unsigned>(n)) {
    srow[m] = static_cast<RankT>(r);
  } else {
    bad = true;
  }
}

template <typename RankT>
__device__ __forceinline__ void scatter4(RankT *srow, int4 q, int r, int n, bool &bad) {
  scatter_one(srow, q.x, r, n, bad);
  scatter_one(srow, q.y, r + 1, n, bad);
  scatter_one(srow, q.z, r + 2, n, bad);
  scatter_one(srow, q.w, r + 3, n, bad);
}

template <typename RankT>
__global__ void __launch_bounds__(512) k_invert(const int32_t *__restrict__ pref_w,
                                                RankT *__restrict__ rank, int n,
                                                Control *ctrl, int mode) {
  if (invert_skipped(mode, ctrl)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RankT *srow = reinterpret_cast<RankT *>(smem_raw);
  constexpr int kPerVec = 16 / sizeof(RankT);  // ranks per 16-byte store
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  bool bad = false;

  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    // 1. mark every slot unset (16-byte shared stores)
    {
      uint4 *s4 = reinterpret_cast<uint4 *>(srow);
      const int nvec = (n + kPerVec - 1) / kPerVec;
      const uint4 fill = make_uint4(~0u, ~0u, ~0u, ~0u);
      for (int i = tid; i < nvec; i += nthr) s4[i] = fill;
    }
    __syncthreads();

    // 2. stream the preference row in and scatter ranks
    const int32_t *row = pref_w + static_cast<size_t>(w) * n;
    const int head = min(n, static_cast<int>(((16u - (reinterpret_cast<uintptr_t>(row) & 15u)) & 15u) >> 2));
    if (tid < head) scatter_one(srow, __ldcs(row + tid), tid, n, bad);
    const int nq = (n - head) >> 2;
    const int4 *rq = reinterpret_cast<const int4 *>(row + head);
    int i = tid;
    for (; i + 3 * nthr < nq; i += 4 * nthr) {
      const int4 a = __ldcs(rq + i);
      const int4 b = __ldcs(rq + i + nthr);
      const int4 c = __ldcs(rq + i + 2 * nthr);
      const int4 d = __ldcs(rq + i + 3 * nthr);
      scatter4(srow, a, head + 4 * i, n, bad);
      scatter4(srow, b, head + 4 * (i + nthr), n, bad);
      scatter4(srow, c, head + 4 * (i + 2 * nthr), n, bad);
      scatter4(srow, d, head + 4 * (i + 3 * nthr), n, bad);
    }
    for (; i < nq; i += nthr) scatter4(srow, __ldcs(rq + i), head + 4 * i, n, bad);
    for (int t = head + 4 * nq + tid; t < n; t += nthr) scatter_one(srow, __ldcs(row + t), t, n, bad);
    __syncthreads();

    // 3. stream the rank row out, checking for unset slots
    RankT *out = rank + static_cast<size_t>(w) * n;
    const RankT unset = rank_unset<RankT>();
    const int ohead = min(n, static_cast<int>(((16u - (reinterpret_cast<uintptr_t>(out) & 15u)) & 15u) / sizeof(RankT)));
    for (int t = tid; t < ohead; t += nthr) {
      const RankT v = srow[t];
      bad |= (v == unset);
      __stcs(out + t, v);
    }
    const int nv = (n - ohead) / kPerVec;
    uint4 *o4 = reinterpret_cast<uint4 *>(out + ohead);
    for (int v = tid; v < nv; v += nthr) {
      RankT vals[kPerVec];
#pragma unroll
      for (int k = 0; k < kPerVec; ++k) {
        vals[k] = srow[ohead + v * kPerVec + k];
        bad |= (vals[k] == unset);
      }
      __stcs(o4 + v, *reinterpret_cast<const uint4 *>(vals));
    }
    for (int t = ohead + nv * kPerVec + tid; t < n; t += nthr) {
      const RankT v = srow[t];
      bad |= (v == unset);
      __stcs(out + t, v);
    }
    __syncthreads();
  }
  if (bad) report(ctrl, kStatusInvalidInput, -1);
}

// Inversion for rows that do not fit in shared memory: scatter straight to
// global memory, then verify rank[w][pref_w[w][r]] == r in a second pass.
__global__ void k_invert_global(const int32_t *__restrict__ pref_w, int32_t *__restrict__ rank,
                                int n, Control *ctrl, int mode) {
  if (invert_skipped(mode, ctrl)) return;
  const size_t total = static_cast<size_t>(n) * n;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int w = static_cast<int>(t / n);
    const int r = static_cast<int>(t - static_cast<size_t>(w) * n);
    const int m = __ldcs(pref_w + t);
    if (static_cast<unsigned>(m) < static_cast<unsigned>(n)) {
      rank[static_cast<size_t>(w) * n + m] = r;
    } else {
      report(ctrl, kStatusInvalidInput, m);
    }
  }
}
__global__ void k_invert_verify(const int32_t *__restrict__ pref_w, const int32_t *__restrict__ rank,
                                int n, Control *ctrl, int mode) {
  if (invert_skipped(mode, ctrl)) return;
  const size_t total = static_cast<size_t>(n) * n;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int w = static_cast<int>(t / n);
    const int r = static_cast<int>(t - static_cast<size_t>(w) * n);
    const int m = pref_w[t];
    if (static_cast<unsigned>(m) >= static_cast<unsigned>(n) ||
        rank[static_cast<size_t>(w) * n + m] != r) {
      report(ctrl, kStatusInvalidInput, m);
    }
  }
}

// ---------------------------------------------------------------------------
// Full validation (SMP_F_VALIDATE): every row of a preference matrix is a
// permutation of 0..n-1.  One CTA per row at a time with an n-bit shared
// bitmap; a value out of range or seen twice is reported.
// Dynamic shared memory: ceil(n/32) * 4 bytes.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_validate_rows(const int32_t *__restrict__ pref, int n, Control *ctrl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *seen = reinterpret_cast<uint32_t *>(smem_raw);
  const int words = (n + 31) >> 5;
  bool bad = false;
  int bad_value = 0;
  for (int row = blockIdx.x; row < n; row += gridDim.x) {
    for (int i = threadIdx.x; i < words; i += blockDim.x) seen[i] = 0u;
    __syncthreads();
    const int32_t *p = pref + static_cast<size_t>(row) * n;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const int v = __ldcs(p + r);
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
    __syncthreads();
  }
  if (bad) report(ctrl, kStatusInvalidInput, bad_value);
}

// ---------------------------------------------------------------------------
// Prefix gather: prefix[m][r] = pref_m[m][r] << 16 | rank[pref_m[m][r]][m]
// for r < K (uint16 ranks only).  An out-of-range woman is reported and her
// entry set to 0xFFFFFFFF.
// ---------------------------------------------------------------------------
__global__ void k_prefix(const int32_t *__restrict__ pref_m, const uint16_t *__restrict__ rank,
                         uint32_t *__restrict__ prefix, int n, int K, Control *ctrl) {
  if (ld_volatile_s32(&ctrl->perfect) || ld_volatile_s32(&ctrl->status)) return;
  const size_t total = static_cast<size_t>(n) * K;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int m = static_cast<int>(t / K);
    const int r = static_cast<int>(t - static_cast<size_t>(m) * K);
    const int w = __ldg(pref_m + static_cast<size_t>(m) * n + r);
    uint32_t e = 0xFFFFFFFFu;
    if (static_cast<unsigned>(w) < static_cast<unsigned>(n)) {
      e = (static_cast<uint32_t>(w) << 16) | __ldg(rank + static_cast<size_t>(w) * n + m);
    } else {
      report(ctrl, kStatusInvalidInput, w);
    }
    prefix[t] = e;
  }
}

// ---------------------------------------------------------------------------
// Window of 32 consecutive choices of one man, one per lane: lane l looks at
// position pos + l.  Returns false (and reports) for an out-of-range woman.
// ---------------------------------------------------------------------------
template <typename RankT>
__device__ __forceinline__ bool load_choice(const int32_t *__restrict__ pref_m,
                                            const RankT *__restrict__ rank,
                                            const uint32_t *__restrict__ prefix, int K, int n,
                                            int m, int r, int &w, uint32_t &rk) {
  if (r < K) {
    const uint32_t e = __ldg(prefix + static_cast<size_t>(m) * K + r);
    w = static_cast<int>(e >> 16);
    rk = e & 0xFFFFu;
    return e != 0xFFFFFFFFu;
  }
  w = __ldg(pref_m + static_cast<size_t>(m) * n + r);
  if (static_cast<unsigned>(w) >= static_cast<unsigned>(n)) return false;
  rk = static_cast<uint32_t>(__ldg(rank + static_cast<size_t>(w) * n + m));
  return true;
}

// ---------------------------------------------------------------------------
// Bulk proposals.  Each warp carries one free man at a time.  It looks at
// his next 32 choices at once; every woman whose current partner she ranks
// above him would reject him, so those proposals are settled by one relaxed
// read of her bid word.  For the first remaining candidate the warp proposes
// with a 64-bit atomicMin.  If accepted and she had a partner, the warp
// continues with the displaced man from the position stored in the returned
// word; if she was free, the number of free women drops and the warp takes a
// man who has not proposed yet.  Once no more than tail_threshold women are
// free, warps hand their man to the tail queue and stop.
// ---------------------------------------------------------------------------
template <typename RankT>
__global__ void __launch_bounds__(256) k_bulk(const int32_t *__restrict__ pref_m,
                                              const RankT *__restrict__ rank,
                                              const uint32_t *__restrict__ prefix, int K,
                                              unsigned long long *bid, Control *ctrl,
                                              int2 *tail_queue, int n, int tail_threshold) {
  if (ld_volatile_s32(&ctrl->perfect) || ld_volatile_s32(&ctrl->status)) return;
  const int lane = threadIdx.x & 31;
  int m = -1, pos = 0;
  unsigned long long settled = 0;  // proposals this warp decided (lane 0's copy is used)
  unsigned int hops = 0;           // proposals this warp saw accepted
  for (;;) {
    int free_now = 0;
    if (m < 0) {
      int v = n;
      if (lane == 0) {
        if (tail_threshold <= 0 || ld_relaxed_s32(&ctrl->free_count) > tail_threshold)
          v = atomicAdd(&ctrl->next_man, 1);
      }
      v = __shfl_sync(kFullMask, v, 0);
      if (v >= n) break;
      m = v;
      pos = 0;
    }
    if (tail_threshold > 0 && lane == 0) free_now = ld_relaxed_s32(&ctrl->free_count);

    const int r = pos + lane;
    const bool valid = r < n;
    int w = 0;
    uint32_t rk = 0xFFFFFFFFu;
    bool ok = true;
    if (valid) ok = load_choice(pref_m, rank, prefix, K, n, m, r, w, rk);
    const unsigned long long cur = (valid && ok) ? ld_relaxed_u64(bid + w) : 0ull;

    if (tail_threshold > 0) {
      free_now = __shfl_sync(kFullMask, free_now, 0);
      if (free_now <= tail_threshold) {
        if (lane == 0) {
          const int q = atomicAdd(&ctrl->tail_count, 1);
          tail_queue[q] = make_int2(m, pos);
        }
        break;
      }
    }
    const unsigned badmask = __ballot_sync(kFullMask, valid && !ok);
    if (badmask) {
      if (lane == __ffs(badmask) - 1) report(ctrl, kStatusInvalidInput, w);
      break;
    }

    unsigned cand = __ballot_sync(kFullMask, valid && rk < bid_rank(cur));
    bool moved = false;
    while (cand) {
      const int j = __ffs(cand) - 1;
      unsigned long long old = 0;
      if (lane == j) old = atomicMin(bid + w, pack_bid(rk, static_cast<uint32_t>(m), static_cast<uint32_t>(r)));
      old = __shfl_sync(kFullMask, old, j);
      const uint32_t rkj = __shfl_sync(kFullMask, rk, j);
      if (bid_rank(old) > rkj) {  // accepted: she was free or held a worse man
        settled += j + 1;
        hops++;
        if (old == kFree) {
          if (lane == 0) atomicSub(&ctrl->free_count, 1);
          m = -1;
        } else {
          m = static_cast<int>(bid_man(old));
          pos = static_cast<int>(bid_pos(old)) + 1;
        }
        moved = true;
        break;
      }
      cand &= cand - 1;  // someone better got there first
    }
    if (!moved) {
      settled += min(32, n - pos);
      pos += 32;
      if (pos >= n) {  // rejected by every woman: the lists are not permutations
        if (lane == 0) report(ctrl, kStatusInvalidInput, m);
        break;
      }
    }
  }
  if (lane == 0 && settled) {
    atomicAdd(&ctrl->bulk_proposals, settled);
    atomicAdd(&ctrl->bulk_hops, hops);
  }
}

// Largest n whose tail state (4-byte bid + 2-byte position per person) fits
// in one CTA's shared memory next to the tail's small bookkeeping.
constexpr int kTailSmemBytesMax = 227 * 1024;
__host__ __device__ constexpr size_t tail_smem_bytes(int n) {
  return static_cast<size_t>(n) * 4 + ((static_cast<size_t>(n) * 2 + 15) & ~static_cast<size_t>(15)) + 64;
}

__device__ __forceinline__ void write_perfect(const int32_t *__restrict__ pref_m, int32_t *match,
                                              int n, Control *ctrl) {
  const int stride = gridDim.x * blockDim.x;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += stride)
    match[m] = __ldg(pref_m + static_cast<size_t>(m) * n);
  if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->proposals = static_cast<unsigned long long>(n);
}

// ---------------------------------------------------------------------------
// Tail.  One CTA of 32 warps.  The bid words move into shared memory as
// rank << 16 | man (4 bytes; n <= 65535), and each man's position in his
// own list into a shared 2-byte array, written before every proposal and
// published by the acquire-release shared atomicMin.  Warps take men from the
// bulk kernel's queue and from the men that never proposed, and follow their
// chains exactly as k_bulk does, but every bid read and atomic stays inside
// the SM.  At the end the CTA writes match[] and the proposal count.
// ---------------------------------------------------------------------------
template <typename RankT>
__global__ void __launch_bounds__(1024, 1) k_tail(const int32_t *__restrict__ pref_m,
                                                  const RankT *__restrict__ rank,
                                                  const uint32_t *__restrict__ prefix, int K,
                                                  const unsigned long long *__restrict__ bid,
                                                  Control *ctrl, const int2 *__restrict__ tail_queue,
                                                  int32_t *__restrict__ match, int n) {
  if (ld_volatile_s32(&ctrl->perfect)) {
    write_perfect(pref_m, match, n, ctrl);
    return;
  }
  if (ld_volatile_s32(&ctrl->status)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *sbid = reinterpret_cast<uint32_t *>(smem_raw);
  uint16_t *spos = reinterpret_cast<uint16_t *>(smem_raw + static_cast<size_t>(n) * 4);
  __shared__ int s_next;
  __shared__ unsigned long long s_props;
  const int tid = threadIdx.x;
  const int lane = tid & 31;

  const int queued = ld_volatile_s32(&ctrl->tail_count);
  const int first_unstarted = min(ld_volatile_s32(&ctrl->next_man), n);
  const int total = queued + (n - first_unstarted);

  for (int w = tid; w < n; w += blockDim.x) {
    const unsigned long long b = bid[w];
    if (b == kFree) {
      sbid[w] = 0xFFFFFFFFu;
    } else {
      sbid[w] = (bid_rank(b) << 16) | bid_man(b);
      spos[bid_man(b)] = static_cast<uint16_t>(bid_pos(b));
    }
  }
  if (tid == 0) {
    s_next = 0;
    s_props = 0;
    ctrl->tail_men = total;
  }
  __syncthreads();

  int m = -1, pos = 0;
  unsigned long long settled = 0;
  unsigned int hops = 0;
  for (;;) {
    if (m < 0) {
      int i = 0;
      if (lane == 0) i = atomicAdd(&s_next, 1);
      i = __shfl_sync(kFullMask, i, 0);
      if (i >= total) break;
      if (i < queued) {
        const int2 e = tail_queue[i];
        m = e.x;
        pos = e.y;
      } else {
        m = first_unstarted + (i - queued);
        pos = 0;
      }
    }
    const int r = pos + lane;
    const bool valid = r < n;
    int w = 0;
    uint32_t rk = 0xFFFFFFFFu;
    bool ok = true;
    if (valid) ok = load_choice(pref_m, rank, prefix, K, n, m, r, w, rk);
    const unsigned badmask = __ballot_sync(kFullMask, valid && !ok);
    if (badmask) {
      if (lane == __ffs(badmask) - 1) report(ctrl, kStatusInvalidInput, w);
      break;
    }
    const uint32_t cur = valid ? lds_relaxed_u32(sbid + w) : 0u;
    unsigned cand = __ballot_sync(kFullMask, valid && rk < (cur >> 16));
    bool moved = false;
    while (cand) {
      const int j = __ffs(cand) - 1;
      uint32_t old = 0;
      int next_pos = 0;
      if (lane == j) {
        spos[m] = static_cast<uint16_t>(r);
        old = atom_min_acq_rel_shared(sbid + w, (rk << 16) | static_cast<uint32_t>(m));
        if ((old >> 16) > rk && old != 0xFFFFFFFFu) next_pos = spos[old & 0xFFFFu] + 1;
      }
      old = __shfl_sync(kFullMask, old, j);
      next_pos = __shfl_sync(kFullMask, next_pos, j);
      const uint32_t rkj = __shfl_sync(kFullMask, rk, j);
      if ((old >> 16) > rkj) {
        settled += j + 1;
        hops++;
        if (old == 0xFFFFFFFFu) {
          m = -1;
        } else {
          m = static_cast<int>(old & 0xFFFFu);
          pos = next_pos;
        }
        moved = true;
        break;
      }
      cand &= cand - 1;
    }
    if (!moved) {
      settled += min(32, n - pos);
      pos += 32;
      if (pos >= n) {
        if (lane == 0) report(ctrl, kStatusInvalidInput, m);
        break;
      }
    }
  }
  if (lane == 0 && settled) {
    atomicAdd(&ctrl->tail_proposals, settled);
    atomicAdd(&ctrl->tail_hops, hops);
  }
  __syncthreads();

  unsigned long long props = 0;
  for (int w = tid; w < n; w += blockDim.x) {
    const uint32_t b = sbid[w];
    if (b == 0xFFFFFFFFu) {
      report(ctrl, kStatusInvalidInput, w);
      continue;
    }
    match[b & 0xFFFFu] = w;
  }
  for (int mm = tid; mm < n; mm += blockDim.x) props += spos[mm] + 1ull;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) props += __shfl_down_sync(kFullMask, props, off);
  if (lane == 0) atomicAdd(&s_props, props);
  __syncthreads();
  if (tid == 0) ctrl->proposals = s_props;
}

// ---------------------------------------------------------------------------
// Matching from the global bid words (used when no tail kernel runs).
// ---------------------------------------------------------------------------
__global__ void k_match(const int32_t *__restrict__ pref_m, const unsigned long long *__restrict__ bid,
                        int32_t *__restrict__ match, int n, Control *ctrl) {
  if (ld_volatile_s32(&ctrl->perfect)) {
    write_perfect(pref_m, match, n, ctrl);
    return;
  }
  if (ld_volatile_s32(&ctrl->status)) return;
  unsigned long long props = 0;
  const int stride = gridDim.x * blockDim.x;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += stride) {
    const unsigned long long b = bid[w];
    if (b == kFree) {
      report(ctrl, kStatusInvalidInput, w);
      continue;
    }
    match[bid_man(b)] = w;
    props += bid_pos(b) + 1ull;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) props += __shfl_down_sync(kFullMask, props, off);
  if ((threadIdx.x & 31) == 0 && props) atomicAdd(&ctrl->proposals, props);
}

// ---------------------------------------------------------------------------
// Stability checker.
//   k_check_husband: husband[w] = m for match[m] = w (husband pre-filled
//     with -1); a woman matched twice or an out-of-range wife is reported.
//   k_check_prank:   prank[w] = rank[w][husband[w]].
//   k_check_scan:    warp per man; every woman before his wife in his list
//     is a blocking pair if she ranks him above her husband.  Also sums the
//     proposal count (position of the wife + 1).
// ---------------------------------------------------------------------------
__global__ void k_check_husband(const int32_t *__restrict__ match, int32_t *husband, int n,
                                Control *ctrl) {
  const int stride = gridDim.x * blockDim.x;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += stride) {
    const int w = match[m];
    if (static_cast<unsigned>(w) >= static_cast<unsigned>(n) || atomicExch(husband + w, m) != -1)
      report(ctrl, kStatusInvalidInput, w);
  }
}

template <typename RankT>
__global__ void k_check_prank(const int32_t *__restrict__ husband, const RankT *__restrict__ rank,
                              int32_t *__restrict__ prank, int n, Control *ctrl) {
  const int stride = gridDim.x * blockDim.x;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += stride) {
    const int h = husband[w];
    if (h < 0) {
      report(ctrl, kStatusInvalidInput, w);
      prank[w] = -1;
      continue;
    }
    prank[w] = static_cast<int32_t>(rank[static_cast<size_t>(w) * n + h]);
  }
}

template <typename RankT>
__global__ void k_check_scan(const int32_t *__restrict__ pref_m, const RankT *__restrict__ rank,
                             const int32_t *__restrict__ match, const int32_t *__restrict__ prank,
                             int n, Control *ctrl) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long blocking = 0, props = 0;
  for (int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; m < n; m += warps) {
    const int wife = match[m];
    const int32_t *row = pref_m + static_cast<size_t>(m) * n;
    bool found = false;
    for (int base = 0; base < n && !found; base += 32) {
      const int r = base + lane;
      const int w = r < n ? __ldg(row + r) : -1;
      const unsigned hit = __ballot_sync(kFullMask, r < n && w == wife);
      const int limit = hit ? (__ffs(hit) - 1) : 32;  // lanes before the wife
      if (lane < limit && r < n && static_cast<unsigned>(w) < static_cast<unsigned>(n)) {
        const int32_t pr = prank[w];
        if (pr >= 0 && static_cast<int32_t>(rank[static_cast<size_t>(w) * n + m]) < pr) blocking++;
      }
      if (hit) {
        found = true;
        if (lane == 0) props += static_cast<unsigned long long>(base + limit + 1);
      }
    }
    if (!found && lane == 0) report(ctrl, kStatusInvalidInput, m);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    blocking += __shfl_down_sync(kFullMask, blocking, off);
    props += __shfl_down_sync(kFullMask, props, off);
  }
  if (lane == 0) {
    if (blocking) atomicAdd(&ctrl->blocking, blocking);
    if (props) atomicAdd(&ctrl->check_proposals, props);
  }
}

}  // namespace smpb200
