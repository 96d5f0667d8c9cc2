// solve_kernels.cuh -- the sm_100a kernels of one Gale-Shapley solve.
//
//   k_precheck    distinct first choices; picks the mode  (SmpEngineBamboo::IsPerfect,
//                                                          include/smp/smp_engine_bamboo.h:25-33)
//   k_invert      rank[w][pref_w[w][r]] = r              (F9RankMatrixInitKernel,
//                                                          src/smp/kernel.cu:672-686)
//   k_pr          ranks by position, pr[m][r] = rank of m in his r-th choice's
//                 list, and each man's first K (woman, rank) pairs: the
//                 reference's PR matrix (kernel.cu:688-709) in uint16
//   k_q*          the same prefix answered straight from pref_w rows, without
//                 a rank matrix (query mode)
//   k_bulk        proposals on every SM                  (La3F9CoreKernel, kernel.cu:633-670)
//   k_tail        the last chains in one CTA             (MonitorProceture + LAProcedure,
//                                                          src/smp/smp_engine_bamboo.cu:197-287)
//   k_match       match[m] = w                           (SmpEngineBamboo::PostProc,
//                                                          smp_engine_bamboo.cu:289-306)
//   k_check_*     stability checker (no counterpart in the reference)
//
// Layouts (row-major, 64-bit offsets):
//   pref_m, pref_w  int32 [n][n]
//   rank            RankT [n][n], RankT = uint16_t for n <= 65535, else int32
//   prefix          uint32 [n][K] = woman << 16 | her rank of the man
//   qcnt, qlist     query index: the (man << 16 | position) pairs naming woman
//                   w among a man's first K choices are qlist[w*qcap ..] (qcnt[w])
//   bid             u64 [n] (see common.cuh)
//
// Every kernel opens with a gate (below) read from the control block, so the
// host enqueues the whole pipeline once and the device decides which parts
// run: no host round trip inside a solve.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "step.cuh"

namespace smpb200 {

// ---------------------------------------------------------------------------
// Gates.
// ---------------------------------------------------------------------------
enum Gate : int {
  kGateAlways = 0,
  kGateMain = 1,       // round 0 of a solve: not perfect, no error seen
  kGateModeRank = 2,   // round 0 in rank mode
  kGateModeQuery = 3,  // round 0 in query mode
  kGateRetry = 4,      // the rank-mode round after a query-mode abort
  kGateIfPerfect = 5,  // the checker after a perfect solve (needs its own inversion)
  kGateNoRank = 6,     // the checker after a solve that built no rank matrix
};

__device__ __forceinline__ bool gate_open(int gate, const Control *c) {
  if (gate == kGateAlways) return true;
  const int perfect = ld_volatile_s32(&c->perfect);
  if (gate == kGateIfPerfect) return perfect != 0;
  if (gate == kGateNoRank) return perfect != 0 || ld_volatile_s32(&c->mode) == kModeQuery;
  if (perfect || ld_volatile_s32(&c->status)) return false;
  switch (gate) {
    case kGateMain: return true;
    case kGateModeRank: return ld_volatile_s32(&c->mode) == kModeRank;
    case kGateModeQuery: return ld_volatile_s32(&c->mode) == kModeQuery;
    case kGateRetry: return ld_volatile_s32(&c->retry) != 0;
    default: return false;
  }
}

// Unset marker of a rank slot during inversion: never a valid rank (uint16
// ranks are < n <= 65535; int32 ranks are >= 0).
template <typename RankT>
__device__ __forceinline__ RankT rank_unset();
template <>
__device__ __forceinline__ uint16_t rank_unset<uint16_t>() { return 0xFFFFu; }
template <>
__device__ __forceinline__ int32_t rank_unset<int32_t>() { return -1; }

// Does a 16-byte chunk of ranks hold an unset slot?
template <typename RankT>
__device__ __forceinline__ bool any_unset(uint4 v);
template <>
__device__ __forceinline__ bool any_unset<uint16_t>(uint4 v) {
  return (__vcmpeq2(v.x, 0xFFFFFFFFu) | __vcmpeq2(v.y, 0xFFFFFFFFu) | __vcmpeq2(v.z, 0xFFFFFFFFu) |
          __vcmpeq2(v.w, 0xFFFFFFFFu)) != 0;
}
template <>
__device__ __forceinline__ bool any_unset<int32_t>(uint4 v) {
  return v.x == 0xFFFFFFFFu || v.y == 0xFFFFFFFFu || v.z == 0xFFFFFFFFu || v.w == 0xFFFFFFFFu;
}

// ---------------------------------------------------------------------------
// Precheck.  Marks each man's first choice in an n-bit bitmap (seen, zeroed
// by the host).  The last block to finish counts the distinct first choices
// and decides: perfect (all distinct, if allowed) and the mode -- query mode
// when at least a quarter of the first choices are distinct (proposals spread
// over the women, so each man stays within his prefix), rank mode otherwise
// (a few women draw most first proposals and men go deep into their lists).
// The control block arrives zeroed by a memset on the same stream (a copy
// from a host staging buffer would read whatever an earlier solve's readback
// left there by the time it ran, when solves are queued back to back or
// replayed from a graph); the switches come as arguments, and the precheck
// writes them and the free count into it.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_precheck(const int32_t *__restrict__ pref_m, int n,
                                                  uint32_t *__restrict__ seen, Control *ctrl, int allow_perfect,
                                                  int allow_query) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctrl->free_count = n;
    ctrl->allow_perfect = allow_perfect;
    ctrl->allow_query = allow_query;
  }
  const int stride = gridDim.x * blockDim.x;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += stride) {
    const int w = __ldg(pref_m + static_cast<size_t>(m) * n);
    if (static_cast<unsigned>(w) >= static_cast<unsigned>(n)) {
      report(ctrl, kStatusInvalidInput, w);
      continue;
    }
    atomicOr(seen + (w >> 5), 1u << (w & 31));
  }
  __shared__ int s_last;
  __shared__ int s_count;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&ctrl->blocks_done, 1) == static_cast<int>(gridDim.x) - 1;
    s_count = 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  int count = 0;
  const int words = (n + 31) >> 5;
  for (int i = threadIdx.x; i < words; i += blockDim.x) count += __popc(__ldcg(seen + i));
  atomicAdd(&s_count, count);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int distinct = s_count;
    ctrl->distinct = distinct;
    ctrl->perfect = (allow_perfect && distinct == n && ctrl->status == 0) ? 1 : 0;
    ctrl->mode = (allow_query && 4ll * distinct >= n) ? kModeQuery : kModeRank;
  }
}

// ---------------------------------------------------------------------------
// Row inversion in shared memory.  One CTA handles one row of pref_w at a
// time: 16-byte streaming loads, each (r, m) scattered into the shared rank
// row, then (k_invert) the row streams out with 16-byte stores, or
// (k_qinvert) the queries of that woman are answered from it.  The shared
// row is offset so that its 16-byte chunks line up with the 16-byte chunks of
// the destination row, which keeps both the shared reads and the global
// stores vectorised and free of bank conflicts.  A slot still unset after
// the scatter means the row was not a permutation.
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

// Shared bytes for one row with the alignment offset.
template <typename RankT>
__host__ __device__ constexpr size_t row_smem_bytes(int n) {
  return ((static_cast<size_t>(n) + 2 * (16 / sizeof(RankT))) * sizeof(RankT) + 15) & ~static_cast<size_t>(15);
}

// Clears the chunks [0, chunks) of sbuf, then streams row `row` of pref_w in
// and scatters it into srow (= sbuf + offset).  Ends with __syncthreads.
template <typename RankT>
__device__ __forceinline__ void load_row(const int32_t *__restrict__ row, RankT *sbuf, RankT *srow, int chunks,
                                         int n, bool &bad) {
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  uint4 *s4 = reinterpret_cast<uint4 *>(sbuf);
  const uint4 fill = make_uint4(~0u, ~0u, ~0u, ~0u);
  for (int i = tid; i < chunks; i += nthr) s4[i] = fill;
  __syncthreads();
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
}

template <typename RankT>
__global__ void __launch_bounds__(512) k_invert(const int32_t *__restrict__ pref_w, RankT *__restrict__ rank,
                                                int n, Control *ctrl, int gate) {
  if (!gate_open(gate, ctrl)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RankT *sbuf = reinterpret_cast<RankT *>(smem_raw);
  constexpr int kPerVec = 16 / sizeof(RankT);
  const RankT unset = rank_unset<RankT>();
  bool bad = false;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    RankT *out = rank + static_cast<size_t>(w) * n;
    const int pre = static_cast<int>((reinterpret_cast<uintptr_t>(out) & 15u) / sizeof(RankT));
    const int chunks = (pre + n + kPerVec - 1) / kPerVec;
    load_row(pref_w + static_cast<size_t>(w) * n, sbuf, sbuf + pre, chunks, n, bad);
    const uint4 *s4 = reinterpret_cast<const uint4 *>(sbuf);
    uint4 *o4 = reinterpret_cast<uint4 *>(reinterpret_cast<uintptr_t>(out) -
                                          static_cast<uintptr_t>(pre) * sizeof(RankT));
    for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
      const uint4 v = s4[c];
      const int first = c * kPerVec - pre;  // row element in the chunk's first slot
      if (first >= 0 && first + kPerVec <= n) {
        bad |= any_unset<RankT>(v);
        __stcs(o4 + c, v);
      } else {
        const RankT *vals = reinterpret_cast<const RankT *>(&v);
#pragma unroll
        for (int k = 0; k < kPerVec; ++k) {
          const int e = first + k;
          if (e >= 0 && e < n) {
            bad |= (vals[k] == unset);
            __stcs(out + e, vals[k]);
          }
        }
      }
    }
    __syncthreads();
  }
  if (bad) report(ctrl, kStatusInvalidInput, -1);
}

// int32 ranks (the reference's layout, smp_b200_invert) from a uint16
// shared row: ranks below 65536 fit 16 bits, so the row takes half the
// shared memory of an int32 one (three CTAs per SM at n = 30000 instead of
// one).  Each 16-byte output chunk is widened from 8 bytes of the row, which
// sits at the output row's offset from a 16-byte boundary.
__global__ void __launch_bounds__(512) k_invert_wide(const int32_t *__restrict__ pref_w, int32_t *__restrict__ rank,
                                                     int n, Control *ctrl, int gate) {
  if (!gate_open(gate, ctrl)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint16_t *sbuf = reinterpret_cast<uint16_t *>(smem_raw);
  bool bad = false;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    int32_t *out = rank + static_cast<size_t>(w) * n;
    const int pre = static_cast<int>((reinterpret_cast<uintptr_t>(out) & 15u) / sizeof(int32_t));
    const int chunks = (pre + n + 3) / 4;                   // 16-byte output chunks
    load_row(pref_w + static_cast<size_t>(w) * n, sbuf, sbuf + pre, (pre + n + 7) / 8, n, bad);
    const uint2 *s2 = reinterpret_cast<const uint2 *>(sbuf);
    uint4 *o4 = reinterpret_cast<uint4 *>(reinterpret_cast<uintptr_t>(out) -
                                          static_cast<uintptr_t>(pre) * sizeof(int32_t));
    for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
      const uint2 v = s2[c];
      const uint32_t vals[4] = {v.x & 0xFFFFu, v.x >> 16, v.y & 0xFFFFu, v.y >> 16};
      const int first = c * 4 - pre;  // row element in the chunk's first slot
      if (first >= 0 && first + 4 <= n) {
        bad |= (__vcmpeq2(v.x, 0xFFFFFFFFu) | __vcmpeq2(v.y, 0xFFFFFFFFu)) != 0;
        __stcs(o4 + c, make_uint4(vals[0], vals[1], vals[2], vals[3]));
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int e = first + k;
          if (e >= 0 && e < n) {
            bad |= (vals[k] == 0xFFFFu);
            __stcs(out + e, static_cast<int32_t>(vals[k]));
          }
        }
      }
    }
    __syncthreads();
  }
  if (bad) report(ctrl, kStatusInvalidInput, -1);
}

// Inversion for rows that do not fit in shared memory: scatter straight to
// global memory, then verify rank[w][pref_w[w][r]] == r in a second pass.
__global__ void k_invert_global(const int32_t *__restrict__ pref_w, int32_t *__restrict__ rank, int n,
                                Control *ctrl, int gate) {
  if (!gate_open(gate, ctrl)) return;
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
__global__ void k_invert_verify(const int32_t *__restrict__ pref_w, const int32_t *__restrict__ rank, int n,
                                Control *ctrl, int gate) {
  if (!gate_open(gate, ctrl)) return;
  const size_t total = static_cast<size_t>(n) * n;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int w = static_cast<int>(t / n);
    const int r = static_cast<int>(t - static_cast<size_t>(w) * n);
    const int m = pref_w[t];
    if (static_cast<unsigned>(m) >= static_cast<unsigned>(n) || rank[static_cast<size_t>(w) * n + m] != r)
      report(ctrl, kStatusInvalidInput, m);
  }
}

// ---------------------------------------------------------------------------
// Man-major copy of the rank matrix: rankT[m][w] = rank[w][m].  A solve's
// proposals read "her rank of him" for every candidate a man scans; in the
// woman-major matrix those reads fall in as many rows as candidates, in the
// man-major one they stay in the man's own row, which stays in cache while
// he scans.  Tiles of 64 x 64 go through shared memory so that both the
// reads and the writes are coalesced; a persistent grid walks the tiles.
// ---------------------------------------------------------------------------
// uint16 with n even: every row starts 4-byte aligned, so pairs of elements
// move as one 32-bit word and a warp reads or writes 128 bytes of a row.
__global__ void __launch_bounds__(512) k_transpose_u16x2(const uint16_t *__restrict__ src, uint16_t *__restrict__ dst,
                                                         int n, Control *ctrl, int gate) {
  if (!gate_open(gate, ctrl)) return;
  __shared__ uint16_t tile[64][66];
  const int lane = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 16
  const int tiles = (n + 63) / 64;
  const long long total = static_cast<long long>(tiles) * tiles;
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    const int r0 = static_cast<int>(t / tiles) * 64, c0 = static_cast<int>(t % tiles) * 64;
    const int c = c0 + 2 * lane;  // even, so c < n implies c + 1 < n
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = r0 + ty + 16 * k;
      if (r < n && c < n) {
        const uint32_t v = *reinterpret_cast<const uint32_t *>(src + static_cast<size_t>(r) * n + c);
        tile[ty + 16 * k][2 * lane] = static_cast<uint16_t>(v & 0xFFFFu);
        tile[ty + 16 * k][2 * lane + 1] = static_cast<uint16_t>(v >> 16);
      }
    }
    __syncthreads();
    const int oc = r0 + 2 * lane;  // output columns are source rows
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int orow = c0 + ty + 16 * k;  // output rows are source columns
      if (orow < n && oc < n) {
        const uint32_t v = static_cast<uint32_t>(tile[2 * lane][ty + 16 * k]) |
                           (static_cast<uint32_t>(tile[2 * lane + 1][ty + 16 * k]) << 16);
        *reinterpret_cast<uint32_t *>(dst + static_cast<size_t>(orow) * n + oc) = v;
      }
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(512) k_transpose(const T *__restrict__ src, T *__restrict__ dst, int n,
                                                   Control *ctrl, int gate) {
  if (!gate_open(gate, ctrl)) return;
  __shared__ T tile[64][65];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 16
  const int tiles = (n + 63) / 64;
  const long long total = static_cast<long long>(tiles) * tiles;
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    const int r0 = static_cast<int>(t / tiles) * 64, c0 = static_cast<int>(t % tiles) * 64;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int r = r0 + ty + 16 * k, c = c0 + tx + 32 * j;
        if (r < n && c < n) tile[ty + 16 * k][tx + 32 * j] = src[static_cast<size_t>(r) * n + c];
      }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int r = c0 + ty + 16 * k, c = r0 + tx + 32 * j;  // dst row = src column
        if (r < n && c < n) dst[static_cast<size_t>(r) * n + c] = tile[tx + 32 * j][ty + 16 * k];
      }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Full validation (SMP_F_VALIDATE): every row of a preference matrix is a
// permutation of 0..n-1.  One CTA per row at a time with an n-bit shared
// bitmap.  Dynamic shared memory: ceil(n/32) * 4 bytes.
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
// Query mode.  The prefix needs rank_w(m) only for the n*K pairs (w, m) with
// w among m's first K choices.  k_qscatter buckets those pairs by woman into
// fixed-capacity buckets (qlist[w * qcap + i], qcnt[w] of them): qcap =
// min(n, 1.5 K + 32) is far above the K a woman receives on average, and a
// bucket that would overflow sets the retry flag, so round 0 stops before any
// proposal and the rank-mode round solves the instance.  k_qinvert then
// streams each woman's row once, inverts it in shared memory and answers her
// bucket.  The rank matrix is never written: pref_w is read once and nothing
// n^2-sized is stored.  qcnt is zeroed by the host.
// ---------------------------------------------------------------------------
__global__ void k_qscatter(const int32_t *__restrict__ pref_m, int n, int K, int qcap, int32_t *__restrict__ qcnt,
                           uint32_t *__restrict__ qlist, Control *ctrl) {
  if (!gate_open(kGateModeQuery, ctrl)) return;
  const size_t total = static_cast<size_t>(n) * K;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int m = static_cast<int>(t / K);
    const int r = static_cast<int>(t - static_cast<size_t>(m) * K);
    const int w = __ldg(pref_m + static_cast<size_t>(m) * n + r);
    if (static_cast<unsigned>(w) >= static_cast<unsigned>(n)) {
      report(ctrl, kStatusInvalidInput, w);
      continue;
    }
    const int slot = atomicAdd(qcnt + w, 1);
    if (slot < qcap) {
      qlist[static_cast<size_t>(w) * qcap + slot] = (static_cast<uint32_t>(m) << 16) | static_cast<uint32_t>(r);
    } else if (slot == qcap) {
      atomicExch(&ctrl->retry, 1);  // a bucket overflowed: round 0 stops, the rank-mode round runs
    }
  }
}

// Rows [w0, w1) (the whole matrix, or one chunk of it as it arrives).
__global__ void __launch_bounds__(512) k_qinvert(const int32_t *__restrict__ pref_w, int n, int K, int qcap,
                                                 const int32_t *__restrict__ qcnt,
                                                 const uint32_t *__restrict__ qlist,
                                                 uint32_t *__restrict__ prefix, Control *ctrl, int w0, int w1) {
  if (!gate_open(kGateModeQuery, ctrl) || ld_volatile_s32(&ctrl->retry)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint16_t *srow = reinterpret_cast<uint16_t *>(smem_raw);
  const int chunks = (n + 7) / 8;
  bool bad = false;
  for (int w = w0 + static_cast<int>(blockIdx.x); w < w1; w += gridDim.x) {
    load_row(pref_w + static_cast<size_t>(w) * n, srow, srow, chunks, n, bad);
    // validation: every slot written
    const uint4 *s4 = reinterpret_cast<const uint4 *>(srow);
    for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
      uint4 v = s4[c];
      const int tailn = n - c * 8;
      if (tailn < 8) {  // slots past n keep the fill value; mask them out
        const auto keep = [tailn](uint32_t x, int half) -> uint32_t {
          return x & ((half < tailn ? 0x0000FFFFu : 0u) | (half + 1 < tailn ? 0xFFFF0000u : 0u));
        };
        v.x = keep(v.x, 0);
        v.y = keep(v.y, 2);
        v.z = keep(v.z, 4);
        v.w = keep(v.w, 6);
      }
      bad |= any_unset<uint16_t>(v);
    }
    const uint32_t *bucket = qlist + static_cast<size_t>(w) * qcap;
    const int count = min(__ldg(qcnt + w), qcap);
    for (int q = threadIdx.x; q < count; q += blockDim.x) {
      const uint32_t e = bucket[q];
      const uint32_t m = e >> 16, r = e & 0xFFFFu;
      prefix[static_cast<size_t>(m) * K + r] = (static_cast<uint32_t>(w) << 16) | srow[m];
    }
    __syncthreads();
  }
  if (bad) report(ctrl, kStatusInvalidInput, -1);
}

// Rows [w0, w1) for n <= kColorMaxN, written to keep pref_w streaming while a
// row is checked and answered.  Each CTA handles rows w0 + blockIdx.x + k *
// gridDim.x; the k-th row's slots are written as rank | (k & 1) << 15, so a
// slot this row did not write still carries the other colour (the row before
// it, or the fill at the start) and validation needs no clearing pass.  The
// next row's first batch of 16-byte loads is issued before the current row
// is validated and answered.  One barrier ends the scatter, one the answers.
// After a row that is not a permutation the colours may no longer tell, but
// that row has already reported the error.
constexpr int kColorMaxN = 32767;

struct RowSpan {
  const int32_t *row;  // first element
  const int4 *rq;      // first 16-byte aligned element (row + head)
  int head;            // scalars before rq (0..3)
  int nq;              // 16-byte chunks
  int tail;            // scalars after them (0..3)
};

__device__ __forceinline__ RowSpan row_span(const int32_t *pref_w, int w, int n) {
  RowSpan s;
  s.row = pref_w + static_cast<size_t>(w) * n;
  s.head = min(n, static_cast<int>(((16u - (reinterpret_cast<uintptr_t>(s.row) & 15u)) & 15u) >> 2));
  s.rq = reinterpret_cast<const int4 *>(s.row + s.head);
  s.nq = (n - s.head) >> 2;
  s.tail = n - s.head - 4 * s.nq;
  return s;
}

// Batch starting at chunk `base`: chunk base + tid + j * nthr into v[j].
__device__ __forceinline__ void row_batch_load(const RowSpan &s, int base, int4 (&v)[4]) {
  const int nthr = blockDim.x;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int i = base + static_cast<int>(threadIdx.x) + j * nthr;
    v[j] = i < s.nq ? __ldcs(s.rq + i) : make_int4(0, 0, 0, 0);
  }
}

__device__ __forceinline__ void scatter_c(uint16_t *srow, int m, int r, uint32_t cbit, int n, bool &bad) {
  if (static_cast<unsigned>(m) < static_cast<unsigned>(n)) {
    srow[m] = static_cast<uint16_t>(static_cast<uint32_t>(r) | cbit);
  } else {
    bad = true;
  }
}

// kThreads: 384 for long rows (n = 30000: 0.865 ms against 0.922 with 256),
// 256 for shorter ones (n = 12000: 0.198 ms against 0.204 with 384).
template <int kThreads>
__global__ void __launch_bounds__(kThreads) k_qinvert_c(const int32_t *__restrict__ pref_w, int n, int K, int qcap,
                                                      const int32_t *__restrict__ qcnt,
                                                      const uint32_t *__restrict__ qlist,
                                                      uint32_t *__restrict__ prefix, Control *ctrl, int w0, int w1) {
  if (!gate_open(kGateModeQuery, ctrl) || ld_volatile_s32(&ctrl->retry)) return;
  int w = w0 + static_cast<int>(blockIdx.x);
  if (w >= w1) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint16_t *srow = reinterpret_cast<uint16_t *>(smem_raw);
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int chunks = (n + 7) / 8;
  uint4 *s4 = reinterpret_cast<uint4 *>(srow);
  // colour 1 everywhere: the first row (colour 0) must write every slot
  for (int c = tid; c < chunks; c += nthr) s4[c] = make_uint4(~0u, ~0u, ~0u, ~0u);
  bool bad = false;
  RowSpan s = row_span(pref_w, w, n);
  int4 a[4];
  row_batch_load(s, 0, a);
  int edge_head = tid < s.head ? __ldcs(s.row + tid) : 0;
  int edge_tail = tid < s.tail ? __ldcs(s.row + s.head + 4 * s.nq + tid) : 0;
  __syncthreads();  // the fill before the first scatter
  for (int k = 0;; ++k) {
    const uint32_t cbit = static_cast<uint32_t>(k & 1) << 15;
    if (tid < s.head) scatter_c(srow, edge_head, tid, cbit, n, bad);
    if (tid < s.tail) scatter_c(srow, edge_tail, s.head + 4 * s.nq + tid, cbit, n, bad);
    for (int base = 0; base < s.nq; base += 4 * nthr) {
      if (base > 0) row_batch_load(s, base, a);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = base + tid + j * nthr;
        if (i < s.nq) {
          const int r = s.head + 4 * i;
          scatter_c(srow, a[j].x, r, cbit, n, bad);
          scatter_c(srow, a[j].y, r + 1, cbit, n, bad);
          scatter_c(srow, a[j].z, r + 2, cbit, n, bad);
          scatter_c(srow, a[j].w, r + 3, cbit, n, bad);
        }
      }
    }
    __syncthreads();  // row w complete in shared memory
    const int wn = w + static_cast<int>(gridDim.x);
    const RowSpan sn = row_span(pref_w, wn < w1 ? wn : w, n);
    if (wn < w1) {
      row_batch_load(sn, 0, a);
      edge_head = tid < sn.head ? __ldcs(sn.row + tid) : 0;
      edge_tail = tid < sn.tail ? __ldcs(sn.row + sn.head + 4 * sn.nq + tid) : 0;
    }
    // validation: every slot carries this row's colour
    const uint32_t want = cbit ? 0x80008000u : 0u;
    for (int c = tid; c < chunks; c += nthr) {
      const uint4 v = s4[c];
      const int tailn = n - c * 8;
      uint32_t m0 = 0x80008000u, m1 = 0x80008000u, m2 = 0x80008000u, m3 = 0x80008000u;
      if (tailn < 8) {  // halves past n keep the fill; leave them out
        const auto keep = [tailn](int half) -> uint32_t {
          return (half < tailn ? 0x00008000u : 0u) | (half + 1 < tailn ? 0x80000000u : 0u);
        };
        m0 = keep(0);
        m1 = keep(2);
        m2 = keep(4);
        m3 = keep(6);
      }
      bad |= (((v.x ^ want) & m0) | ((v.y ^ want) & m1) | ((v.z ^ want) & m2) | ((v.w ^ want) & m3)) != 0u;
    }
    const uint32_t *bucket = qlist + static_cast<size_t>(w) * qcap;
    const int count = min(__ldg(qcnt + w), qcap);
    for (int q = tid; q < count; q += nthr) {
      const uint32_t e = bucket[q];
      const uint32_t m = e >> 16, r = e & 0xFFFFu;
      prefix[static_cast<size_t>(m) * K + r] = (static_cast<uint32_t>(w) << 16) | (srow[m] & 0x7FFFu);
    }
    __syncthreads();  // answers read before the next row overwrites
    if (wn >= w1) break;
    w = wn;
    s = sn;
  }
  if (bad) report(ctrl, kStatusInvalidInput, -1);
}

// The layout rank-mode proposals read: by position (pr, uint16 ranks, n <=
// 65535) or man-major (rankT, int32 ranks).
template <typename RankT>
__host__ __device__ constexpr int rank_layout() {
  return std::is_same<RankT, uint16_t>::value ? 2 : 1;
}

// ---------------------------------------------------------------------------
// pr[m][r] = rankT[m][pref_m[m][r]]: the rank of man m in the list of his
// r-th choice, in the order he proposes (what the reference's PR matrix
// holds, kernel.cu:688-709, in uint16 and without the woman beside it).  A
// proposal then reads pref_m[m][r] and pr[m][r] side by side, sequentially,
// instead of a random rankT[m][w] that waits for pref_m[m][r]; in congested
// and correlated lists, where men reject hundreds of women per acceptance,
// that halves the round trips of a window.  The same pass writes each man's
// first K entries of the prefix table (woman << 16 | rank).  One CTA per man row at a time:
// his rankT row is staged in shared memory (16-byte loads over its aligned
// interior), his pref_m row streams in with 16-byte loads and gathers from
// it.  An out-of-range woman is reported.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_pr(const int32_t *__restrict__ pref_m, const uint16_t *__restrict__ rankT,
                                            uint16_t *__restrict__ pr, uint32_t *__restrict__ prefix, int K, int n,
                                            Control *ctrl, int gate) {
  if (!gate_open(gate, ctrl)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  bool bad = false;
  for (int m = blockIdx.x; m < n; m += gridDim.x) {
    const uint16_t *src = rankT + static_cast<size_t>(m) * n;
    const int pre = static_cast<int>((reinterpret_cast<uintptr_t>(src) & 15u) >> 1);
    uint16_t *srow = reinterpret_cast<uint16_t *>(smem_raw) + pre;  // same offset from 16 bytes as src
    const int a0 = min(n, (8 - pre) & 7);                           // first element on a 16-byte boundary
    const int nch = (n - a0) >> 3;
    for (int e = tid; e < a0; e += nthr) srow[e] = src[e];
    for (int c = tid; c < nch; c += nthr)
      reinterpret_cast<uint4 *>(srow + a0)[c] = __ldcs(reinterpret_cast<const uint4 *>(src + a0) + c);
    for (int e = a0 + 8 * nch + tid; e < n; e += nthr) srow[e] = src[e];
    __syncthreads();
    const RowSpan s = row_span(pref_m, m, n);
    uint16_t *out = pr + static_cast<size_t>(m) * n;
    uint32_t *pfx = prefix + static_cast<size_t>(m) * K;  // his first K choices, woman << 16 | rank
    const auto gather = [&](int w, int r) {
      if (static_cast<unsigned>(w) < static_cast<unsigned>(n)) {
        out[r] = srow[w];
        if (r < K) pfx[r] = (static_cast<uint32_t>(w) << 16) | srow[w];
      } else {
        bad = true;
        if (r < K) pfx[r] = 0xFFFFFFFFu;
      }
    };
    if (tid < s.head) gather(__ldcs(s.row + tid), tid);
    // 8-byte stores when the four outputs of a 16-byte load line up (they do
    // whenever pref_m starts on a 16-byte boundary); else one at a time
    const bool wide = ((reinterpret_cast<uintptr_t>(out + s.head)) & 7u) == 0;
    const auto rank_or_flag = [&](int w) -> uint32_t {
      if (static_cast<unsigned>(w) < static_cast<unsigned>(n)) return srow[w];
      bad = true;
      return 0u;
    };
    for (int i = tid; i < s.nq; i += nthr) {
      const int4 q = __ldcs(s.rq + i);
      const int r = s.head + 4 * i;
      if (wide && r >= K) {  // no prefix entry among the four
        const uint2 v = make_uint2(rank_or_flag(q.x) | (rank_or_flag(q.y) << 16),
                                   rank_or_flag(q.z) | (rank_or_flag(q.w) << 16));
        *reinterpret_cast<uint2 *>(out + r) = v;
      } else {
        gather(q.x, r);
        gather(q.y, r + 1);
        gather(q.z, r + 2);
        gather(q.w, r + 3);
      }
    }
    if (tid < s.tail) gather(__ldcs(s.row + s.head + 4 * s.nq + tid), s.head + 4 * s.nq + tid);
    __syncthreads();
  }
  if (bad) report(ctrl, kStatusInvalidInput, -1);
}

// The same inversion from rows packed to uint16 on the host (host-input
// solves stream pref_w in half the bytes): 16-byte loads hold 8 entries, and
// a row starts anywhere on a 2-byte boundary, so up to 7 entries before its
// first 16-byte boundary and 7 after its last are loaded one by one.
struct RowSpan16 {
  const uint16_t *row;
  const uint4 *rq;  // first 16-byte aligned entry
  int head, nq, tail;
};

__device__ __forceinline__ RowSpan16 row_span16(const uint16_t *pref16, int w, int n) {
  RowSpan16 s;
  s.row = pref16 + static_cast<size_t>(w) * n;
  s.head = min(n, static_cast<int>(((16u - (reinterpret_cast<uintptr_t>(s.row) & 15u)) & 15u) >> 1));
  s.rq = reinterpret_cast<const uint4 *>(s.row + s.head);
  s.nq = (n - s.head) >> 3;
  s.tail = n - s.head - 8 * s.nq;
  return s;
}

__global__ void __launch_bounds__(256) k_qinvert_p16(const uint16_t *__restrict__ pref16, int n, int K, int qcap,
                                                     const int32_t *__restrict__ qcnt,
                                                     const uint32_t *__restrict__ qlist,
                                                     uint32_t *__restrict__ prefix, Control *ctrl, int w0, int w1) {
  if (!gate_open(kGateModeQuery, ctrl) || ld_volatile_s32(&ctrl->retry)) return;
  int w = w0 + static_cast<int>(blockIdx.x);
  if (w >= w1) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint16_t *srow = reinterpret_cast<uint16_t *>(smem_raw);
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int chunks = (n + 7) / 8;
  uint4 *s4 = reinterpret_cast<uint4 *>(srow);
  for (int c = tid; c < chunks; c += nthr) s4[c] = make_uint4(~0u, ~0u, ~0u, ~0u);
  bool bad = false;
  RowSpan16 s = row_span16(pref16, w, n);
  const auto load = [&](const RowSpan16 &sp, int base, uint4 (&v)[2]) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int i = base + tid + j * nthr;
      v[j] = i < sp.nq ? __ldcs(sp.rq + i) : make_uint4(0, 0, 0, 0);
    }
  };
  const auto scatter8 = [&](uint4 v, int r, uint32_t cbit) {
    const uint32_t q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      scatter_c(srow, static_cast<int>(q[h] & 0xFFFFu), r + 2 * h, cbit, n, bad);
      scatter_c(srow, static_cast<int>(q[h] >> 16), r + 2 * h + 1, cbit, n, bad);
    }
  };
  uint4 a[2];
  load(s, 0, a);
  int edge = tid < s.head ? __ldcs(s.row + tid) : (tid < s.head + s.tail ? __ldcs(s.row + s.head + 8 * s.nq + (tid - s.head)) : 0);
  __syncthreads();  // the fill before the first scatter
  for (int k = 0;; ++k) {
    const uint32_t cbit = static_cast<uint32_t>(k & 1) << 15;
    if (tid < s.head) scatter_c(srow, edge, tid, cbit, n, bad);
    else if (tid < s.head + s.tail) scatter_c(srow, edge, s.head + 8 * s.nq + (tid - s.head), cbit, n, bad);
    for (int base = 0; base < s.nq; base += 2 * nthr) {
      if (base > 0) load(s, base, a);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int i = base + tid + j * nthr;
        if (i < s.nq) scatter8(a[j], s.head + 8 * i, cbit);
      }
    }
    __syncthreads();  // row w complete in shared memory
    const int wn = w + static_cast<int>(gridDim.x);
    const RowSpan16 sn = row_span16(pref16, wn < w1 ? wn : w, n);
    if (wn < w1) {
      load(sn, 0, a);
      edge = tid < sn.head ? __ldcs(sn.row + tid)
                           : (tid < sn.head + sn.tail ? __ldcs(sn.row + sn.head + 8 * sn.nq + (tid - sn.head)) : 0);
    }
    const uint32_t want = cbit ? 0x80008000u : 0u;
    for (int c = tid; c < chunks; c += nthr) {
      const uint4 v = s4[c];
      const int tailn = n - c * 8;
      uint32_t m0 = 0x80008000u, m1 = 0x80008000u, m2 = 0x80008000u, m3 = 0x80008000u;
      if (tailn < 8) {
        const auto keep = [tailn](int half) -> uint32_t {
          return (half < tailn ? 0x00008000u : 0u) | (half + 1 < tailn ? 0x80000000u : 0u);
        };
        m0 = keep(0);
        m1 = keep(2);
        m2 = keep(4);
        m3 = keep(6);
      }
      bad |= (((v.x ^ want) & m0) | ((v.y ^ want) & m1) | ((v.z ^ want) & m2) | ((v.w ^ want) & m3)) != 0u;
    }
    const uint32_t *bucket = qlist + static_cast<size_t>(w) * qcap;
    const int count = min(__ldg(qcnt + w), qcap);
    for (int q = tid; q < count; q += nthr) {
      const uint32_t e = bucket[q];
      const uint32_t m = e >> 16, r = e & 0xFFFFu;
      prefix[static_cast<size_t>(m) * K + r] = (static_cast<uint32_t>(w) << 16) | (srow[m] & 0x7FFFu);
    }
    __syncthreads();  // answers read before the next row overwrites
    if (wn >= w1) break;
    w = wn;
    s = sn;
  }
  if (bad) report(ctrl, kStatusInvalidInput, -1);
}

// Entries [begin, end) of a matrix packed to uint16 on the host, widened
// back to the int32 rows that rank-mode solves read.  A packed 0xFFFF -- what
// the packing makes of an entry outside [0, n) -- widens to 65535, still
// >= n (n <= 65535 here), so the kernels that read the entry report it.
// Eight entries per thread step: one 16-byte load and two 16-byte stores
// where all eight lie inside the span, one by one at its ragged ends.  Thread
// `first` of `stride` threads takes steps first, first + stride, ...
__device__ __forceinline__ void widen_span(const uint16_t *__restrict__ src, int32_t *__restrict__ dst, size_t begin,
                                           size_t end, size_t first, size_t stride) {
  const size_t base = begin & ~size_t{7};
  for (size_t i = base + first * 8; i < end; i += stride * 8) {
    if (i >= begin && i + 8 <= end) {
      const uint4 v = __ldcs(reinterpret_cast<const uint4 *>(src + i));
      const int4 lo = make_int4(static_cast<int>(v.x & 0xFFFFu), static_cast<int>(v.x >> 16),
                                static_cast<int>(v.y & 0xFFFFu), static_cast<int>(v.y >> 16));
      const int4 hi = make_int4(static_cast<int>(v.z & 0xFFFFu), static_cast<int>(v.z >> 16),
                                static_cast<int>(v.w & 0xFFFFu), static_cast<int>(v.w >> 16));
      int4 *out = reinterpret_cast<int4 *>(dst + i);
      out[0] = lo;
      out[1] = hi;
    } else {
      const size_t j1 = i + 8 < end ? i + 8 : end;
      for (size_t j = i < begin ? begin : i; j < j1; ++j) dst[j] = src[j];
    }
  }
}

__global__ void __launch_bounds__(256) k_widen16(const uint16_t *__restrict__ src, int32_t *__restrict__ dst,
                                                 size_t begin, size_t end) {
  widen_span(src, dst, begin, end, static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x,
             static_cast<size_t>(gridDim.x) * blockDim.x);
}

// The same for the listed rows rows[0 .. count) (ids already checked to lie
// in [0, n) on the host), one row per CTA at a time.
__global__ void __launch_bounds__(256) k_widen16_rows(const uint16_t *__restrict__ src, int32_t *__restrict__ dst,
                                                      const int32_t *__restrict__ rows, int count, int n) {
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const size_t b = static_cast<size_t>(__ldg(rows + i)) * n;
    widen_span(src, dst, b, b + n, threadIdx.x, blockDim.x);
  }
}

// ---------------------------------------------------------------------------
// Bulk proposals on every SM.  Each warp carries one free man at a time
// (man_step above, 64-bit bids in HBM).  A man accepted by a free woman
// lowers the count of free women and the warp takes a man who has not
// proposed yet; a displaced man continues in the same warp from the position
// stored in the returned bid.  Once no more than tail_threshold women are
// free, warps hand their man to the tail queue and stop.  In query mode a man
// whose next proposal lies beyond his prefix stops the solve for the
// rank-mode retry round.
// round 0: gate Main; round 1: gate Retry (rank mode).
// ---------------------------------------------------------------------------
// kFilter: bids go through FilteredBids, a per-CTA bound on each woman's
// partner rank in 4 n bytes of shared memory (one CTA of kFilterBlock threads
// per SM); else GlobalBids.  Both variants are enqueued and the device runs
// the one k_wdistinct chose (ctrl->use_filter).
constexpr int kFilterBlock = 768;
constexpr int kFilterMaxDistinct = 16;

// ---------------------------------------------------------------------------
// Chooses the bulk variant of a rank-mode round 0.  The filter pays off when
// the men's lists are nearly all alike (at most kFilterMaxDistinct distinct
// first choices: every man scans the same women) and the women's are not (at
// least n / 4 distinct first choices: most of those proposals are rejections
// by women who already hold a better man).  Where the women's lists are alike
// too, most proposals displace someone and the filter only adds work.  One
// CTA counts the women's distinct first choices in a shared bitmap.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_wdistinct(const int32_t *__restrict__ pref_w, int n, Control *ctrl) {
  extern __shared__ uint32_t seen[];
  if (!gate_open(kGateModeRank, ctrl) || ld_volatile_s32(&ctrl->distinct) > kFilterMaxDistinct) return;
  const int words = (n + 31) >> 5;
  for (int i = threadIdx.x; i < words; i += blockDim.x) seen[i] = 0u;
  __syncthreads();
  for (int w = threadIdx.x; w < n; w += blockDim.x) {
    const int m = __ldg(pref_w + static_cast<size_t>(w) * n);
    if (static_cast<unsigned>(m) < static_cast<unsigned>(n)) atomicOr(seen + (m >> 5), 1u << (m & 31));
  }
  __syncthreads();
  __shared__ int s_count;
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  int count = 0;
  for (int i = threadIdx.x; i < words; i += blockDim.x) count += __popc(seen[i]);
  atomicAdd(&s_count, count);
  __syncthreads();
  if (threadIdx.x == 0) {
    ctrl->distinct_w = s_count;
    ctrl->use_filter = 4ll * s_count >= n ? 1 : 0;
  }
}

template <typename RankT, int kMaxSub, bool kFilter = false>
__global__ void __launch_bounds__(kFilter ? kFilterBlock : 256)
    k_bulk(const int32_t *__restrict__ pref_m, const RankT *__restrict__ rank, const uint32_t *__restrict__ prefix,
           int K, unsigned long long *bid, Control *ctrl, int2 *tail_queue, int n, int tail_threshold_query,
           int tail_threshold_rank, int round, int only_mode = -1) {
  using Bids = typename std::conditional<kFilter, FilteredBids, GlobalBids>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *lrank = reinterpret_cast<uint32_t *>(smem_raw);
  if (kFilter) {
    // The gates are read once for the CTA: the retry flag may be raised by
    // another CTA while this one starts, and every thread must reach the
    // barrier.
    __shared__ int s_go;
    if (threadIdx.x == 0)
      s_go = round == 0 && ld_volatile_s32(&ctrl->use_filter) && gate_open(kGateMain, ctrl) &&
             !ld_volatile_s32(&ctrl->retry);
    __syncthreads();
    if (!s_go) return;
    for (int w = threadIdx.x; w < n; w += blockDim.x) lrank[w] = 0xFFFFFFFFu;
    __syncthreads();
  } else {
    if (!gate_open(round == 0 ? kGateMain : kGateRetry, ctrl)) return;
    if (round == 0 && ld_volatile_s32(&ctrl->retry)) return;  // a query bucket overflowed
    if (round == 0 && ld_volatile_s32(&ctrl->use_filter)) return;  // the filtered variant runs
    // enqueued for one mode only (the host has not read the precheck yet)
    if (round == 0 && only_mode >= 0 && ld_volatile_s32(&ctrl->mode) != only_mode) return;
  }
  const bool query = round == 0 && ld_volatile_s32(&ctrl->mode) == kModeQuery;
  // Free women left when the men move to the one-CTA tail: rank-mode
  // instances scan deep, which many SMs do faster, so they hand over later.
  const int tail_threshold = query ? tail_threshold_query : tail_threshold_rank;
  const int lane = threadIdx.x & 31;
  // Bring the whole prefix table into L2 (n*K*4 bytes, 23 MB at n = 30000):
  // it was written while pref_w streamed through L2, and every later step of
  // the solve -- this kernel and the one-SM tail -- is a chain of dependent
  // reads of it, so each miss would cost a DRAM round trip on the chain.
  if (prefix != nullptr) prefetch_l2(prefix, static_cast<size_t>(n) * K * sizeof(uint32_t));
  Bids bids;
  bids.bid = bid;
  if constexpr (kFilter) bids.lrank = lrank;
  int m = -1, pos = 0, S = 1, bad_value = 0;
  Ahead ahead;
  unsigned long long settled = 0;  // proposals this warp decided (lane 0's copy is used)
  unsigned int hops = 0;           // proposals this warp saw accepted
  for (;;) {
    if (m < 0) {
      int v = n;
      if (lane == 0 && ld_relaxed_s32(&ctrl->free_count) > tail_threshold) v = atomicAdd(&ctrl->next_man, 1);
      v = __shfl_sync(kFullMask, v, 0);
      if (v >= n) break;
      m = v;
      pos = 0;
      S = 1;
    }
    int free_now = 0;
    if (lane == 0) free_now = ld_relaxed_s32(&ctrl->free_count);  // consumed after the window loads
    const int hold_m = m, hold_pos = pos;
    const auto keep_going = [&]() { return __shfl_sync(kFullMask, free_now, 0) > tail_threshold; };
    const int rc = man_step<kMaxSub, true, true, 1, rank_layout<RankT>()>(bids, keep_going, pref_m, rank, prefix, K, n,
                                                                         query, lane, m,
                                                         pos, S, ahead, settled,
                                     hops, bad_value);
    if (rc == kStepMoved) continue;
    if (rc == kStepMatchedFree) {
      if (lane == 0) atomicSub(&ctrl->free_count, 1);
      continue;
    }
    if (rc == kStepHalt) {  // hand over (also how a retry stops everyone)
      // A round-0 abort drops the men: the retry round starts from scratch.
      if (lane == 0 && !(round == 0 && ld_volatile_s32(&ctrl->retry))) {
        const int q = atomicAdd(&ctrl->tail_count, 1);
        tail_queue[q] = make_int2(hold_m, hold_pos);
      }
      break;
    }
    if (rc == kStepBad) {
      if (lane == 0) report(ctrl, kStatusInvalidInput, bad_value);
    } else if (lane == 0) {  // kStepBeyond: query mode ran out of prefix
      atomicExch(&ctrl->retry, 1);
      atomicExch(&ctrl->free_count, -(1 << 30));
    }
    break;
  }
  if (lane == 0 && settled) {
    atomicAdd(&ctrl->bulk_proposals, settled);
    atomicAdd(&ctrl->bulk_hops, hops);
  }
}

// Shared memory of the tail: 4-byte bid and 2-byte position per person.
__host__ __device__ constexpr size_t tail_smem_bytes(int n) {
  return static_cast<size_t>(n) * 4 + ((static_cast<size_t>(n) * 2 + 15) & ~static_cast<size_t>(15)) + 64;
}

// The global bid words as shared ones (rank << 16 | man) plus each matched
// man's position; every other position starts at 0, so a relaxed read that
// races with a man's first store returns 0 (an earlier position), never
// leftover shared memory.  Called by the whole CTA; the caller synchronises.
__device__ __forceinline__ void tail_setup(const unsigned long long *__restrict__ bid, uint32_t *sbid,
                                           uint16_t *spos, int n) {
  for (int m = threadIdx.x; m < n; m += blockDim.x) spos[m] = 0;
  __syncthreads();
  for (int w = threadIdx.x; w < n; w += blockDim.x) {
    const unsigned long long b = bid[w];
    if (b == kFree) {
      sbid[w] = 0xFFFFFFFFu;
    } else {
      sbid[w] = (bid_rank(b) << 16) | bid_man(b);
      spos[bid_man(b)] = static_cast<uint16_t>(bid_pos(b));
    }
  }
}

// The tail's shared state into the bid buffer (4 n bytes of words, then 2 n
// bytes of positions; the buffer holds 8 n) and back.
__device__ __forceinline__ void coop_store(const uint32_t *sbid, const uint16_t *spos, unsigned long long *bid,
                                           int n) {
  uint32_t *gb = reinterpret_cast<uint32_t *>(bid);
  uint16_t *gp = reinterpret_cast<uint16_t *>(gb + n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    gb[i] = sbid[i];
    gp[i] = spos[i];
  }
}
__device__ __forceinline__ void coop_load(const unsigned long long *bid, uint32_t *sbid, uint16_t *spos, int n) {
  const uint32_t *gb = reinterpret_cast<const uint32_t *>(bid);
  const uint16_t *gp = reinterpret_cast<const uint16_t *>(gb + n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sbid[i] = gb[i];
    spos[i] = gp[i];
  }
}

// match[] and the proposal count (sum of final positions + 1) from the
// shared state, after every chain has ended.  Called by the whole CTA.
__device__ __forceinline__ void tail_finish(const uint32_t *sbid, const uint16_t *spos, int32_t *__restrict__ match,
                                            int n, Control *ctrl, unsigned long long *s_props) {
  unsigned long long props = 0;
  for (int w = threadIdx.x; w < n; w += blockDim.x) {
    const uint32_t b = sbid[w];
    if (b == 0xFFFFFFFFu) {
      report(ctrl, kStatusInvalidInput, w);
      continue;
    }
    match[b & 0xFFFFu] = w;
  }
  for (int mm = threadIdx.x; mm < n; mm += blockDim.x) props += spos[mm] + 1ull;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) props += __shfl_down_sync(kFullMask, props, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(s_props, props);
  __syncthreads();
  if (threadIdx.x == 0) ctrl->proposals = *s_props;
}

__device__ __forceinline__ void write_perfect(const int32_t *__restrict__ pref_m, int32_t *match, int n,
                                              Control *ctrl) {
  const int stride = gridDim.x * blockDim.x;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += stride)
    match[m] = __ldg(pref_m + static_cast<size_t>(m) * n);
  if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->proposals = static_cast<unsigned long long>(n);
}

// ---------------------------------------------------------------------------
// Tail.  One CTA of 32 warps.  The bid words move into shared memory as
// rank << 16 | man (n <= 65535), and each man's position into a shared
// 2-byte array (SharedBids).  Warps take men from the bulk kernel's queue and
// from the men that never proposed, and follow their chains with every bid
// read and atomic inside the SM.  At the end the CTA writes match[] and the
// proposal count.  In query mode a man beyond his prefix sets the retry flag
// and every warp stops.
// round 0: gate Main (and no retry pending); round 1: gate Retry.
// only_mode >= 0 runs the kernel only when the precheck chose that mode, so
// the host can enqueue a narrow and a wide variant and the device keeps one.
// ---------------------------------------------------------------------------
template <typename RankT, int kMaxSub>
__global__ void __launch_bounds__(1024, 1) k_tail(const int32_t *__restrict__ pref_m,
                                                  const RankT *__restrict__ rank,
                                                  const uint32_t *__restrict__ prefix, int K,
                                                  unsigned long long *bid, Control *ctrl,
                                                  const int2 *__restrict__ tail_queue,
                                                  int32_t *__restrict__ match, int n, int round,
                                                  int only_mode, int coop_chains) {
  if (only_mode >= 0 && round == 0 && ld_volatile_s32(&ctrl->mode) != only_mode) return;
  if (round == 0 && ld_volatile_s32(&ctrl->perfect)) {
    write_perfect(pref_m, match, n, ctrl);
    return;
  }
  if (!gate_open(round == 0 ? kGateMain : kGateRetry, ctrl)) return;
  if (round == 0 && ld_volatile_s32(&ctrl->retry)) return;
  const bool query = round == 0 && ld_volatile_s32(&ctrl->mode) == kModeQuery;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *sbid = reinterpret_cast<uint32_t *>(smem_raw);
  uint16_t *spos = reinterpret_cast<uint16_t *>(smem_raw + static_cast<size_t>(n) * 4);
  __shared__ int s_next;
  __shared__ int s_abort;
  __shared__ int s_busy;  // warps carrying a chain
  __shared__ unsigned long long s_props;
  const int tid = threadIdx.x;
  const int lane = tid & 31;

  const int queued = ld_volatile_s32(&ctrl->tail_count);
  const int first_unstarted = min(ld_volatile_s32(&ctrl->next_man), n);
  const int total = queued + (n - first_unstarted);
  tail_setup(bid, sbid, spos, n);
  if (tid == 0) {
    s_next = 0;
    s_abort = 0;
    s_busy = 0;
    s_props = 0;
    ctrl->tail_men = total;
  }
  __syncthreads();

  const SharedBids bids{sbid, spos};
  const auto keep_going = [&]() { return *reinterpret_cast<volatile int *>(&s_abort) == 0; };
  int m = -1, pos = 0, S = 1, bad_value = 0;
  Ahead ahead;
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
      S = 1;
      if (lane == 0) atomicAdd(&s_busy, 1);
    } else if (coop_chains > 0) {
      // Once no man waits and only a few chains are left, each goes to
      // k_tail_coop, which runs them one after another with the whole CTA
      // scanning (Gale-Shapley's result does not depend on the order).
      int hand = 0;
      if (lane == 0)
        hand = *reinterpret_cast<volatile int *>(&s_next) >= total &&
               *reinterpret_cast<volatile int *>(&s_busy) <= coop_chains;
      if (__shfl_sync(kFullMask, hand, 0)) {
        if (lane == 0) {
          const int e = atomicAdd(&ctrl->coop_count, 1);  // < 32: each warp hands over once
          ctrl->coop_chain[e] = make_int2(m, pos);
          atomicSub(&s_busy, 1);
        }
        break;
      }
    }
    const int rc = man_step<kMaxSub, (kMaxSub < 8), true, (kMaxSub == 8 ? 8 : 1), rank_layout<RankT>()>(
        bids, keep_going, pref_m, rank, prefix, K, n, query, lane, m, pos, S, ahead, settled,
                                     hops, bad_value);
    if (rc == kStepMatchedFree && lane == 0) atomicSub(&s_busy, 1);
    if (rc == kStepMoved || rc == kStepMatchedFree) continue;
    if (rc == kStepBad) {
      if (lane == 0) report(ctrl, kStatusInvalidInput, bad_value);
    } else if (rc == kStepBeyond && lane == 0) {
      s_abort = 1;
      atomicExch(&ctrl->retry, 1);
    }
    break;
  }
  if (lane == 0 && settled) {
    atomicAdd(&ctrl->tail_proposals, settled);
    atomicAdd(&ctrl->tail_hops, hops);
  }
  __syncthreads();
  if (s_abort || ld_volatile_s32(&ctrl->status)) return;
  if (ld_volatile_s32(&ctrl->coop_count) > 0) {
    // chains handed over: the shared state goes to k_tail_coop through the
    // bid buffer, which this kernel no longer reads
    coop_store(sbid, spos, bid, n);
    return;
  }
  tail_finish(sbid, spos, match, n, ctrl, &s_props);
}

// ---------------------------------------------------------------------------
// The chains k_tail handed over, one after another, each scanned by the
// whole CTA: 1024 threads test up to 8 choices each per step (widening from
// one while no candidate turns up), a CTA minimum picks the first woman who
// would accept him, and one thread records the proposal.  With one chain
// running nothing else changes a bid, so the first candidate always accepts
// and no atomic is needed.  Deep chains (correlated and congested lists, where
// a displaced man rejects hundreds of women before the next acceptance) move
// up to 8192 choices per round trip instead of one warp's 256.  Then the CTA
// writes match[] and the proposal count as k_tail would have.
// ---------------------------------------------------------------------------
template <typename RankT>
__global__ void __launch_bounds__(1024, 1) k_tail_coop(const int32_t *__restrict__ pref_m,
                                                       const RankT *__restrict__ rank,
                                                       const unsigned long long *__restrict__ bid, Control *ctrl,
                                                       int32_t *__restrict__ match, int n) {
  constexpr unsigned long long kNone = ~0ull;
  constexpr bool kByPos = rank_layout<RankT>() == 2;  // rank: pr[m][r], else rankT[m][w]
  const int chains = ld_volatile_s32(&ctrl->coop_count);
  if (chains <= 0 || ld_volatile_s32(&ctrl->status)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *sbid = reinterpret_cast<uint32_t *>(smem_raw);
  uint16_t *spos = reinterpret_cast<uint16_t *>(smem_raw + static_cast<size_t>(n) * 4);
  // Step t's first candidate in s_best[t % 3] as position << 32 | her bid
  // word when it was read, so every thread learns from the minimum whom she
  // drops; s_bad[t % 3]: an invalid entry was seen.  Three buffers: after
  // step t's barrier thread 0 clears the ones step t + 2 will use, which
  // every thread finished reading before that barrier.
  __shared__ unsigned long long s_best[3];
  __shared__ int s_bad[3];
  __shared__ unsigned long long s_props;
  const int tid = threadIdx.x;
  coop_load(bid, sbid, spos, n);
  if (tid == 0) {
    for (int i = 0; i < 3; ++i) {
      s_best[i] = kNone;
      s_bad[i] = 0;
    }
    s_props = 0;
  }
  __syncthreads();
  unsigned long long settled = 0;
  unsigned int hops = 0;
  int t = 0;
  bool stop = false;
  // Thread 0 records a proposal at the start of the next step, before that
  // step's barrier: the other threads took her old bid word from the
  // minimum, and the next man's span does not contain her (he scans his list
  // after her), so nothing reads her word or the proposer's position
  // meanwhile, and every step after sees them.
  bool pend = false;
  int pend_w = 0, pend_m = 0, pend_pos = 0;
  uint32_t pend_val = 0;
  int per_start = 1;  // spans of 1024 a man's scan starts with: what the last one needed
  int wv[8];
  for (int c = 0; c < chains && !stop; ++c) {
    const int2 ch = ctrl->coop_chain[c];
    int m = ch.x, pos = ch.y, per = per_start, from = pos;
    bool loaded = false;  // wv holds the span [pos, pos + 1024 per) of man m
    while (pos < n) {
      if (tid == 0 && pend) {
        sbid[pend_w] = pend_val;
        spos[pend_m] = static_cast<uint16_t>(pend_pos);
        pend = false;
      }
      const int *row = pref_m + static_cast<size_t>(m) * n;
      const RankT *rrow = rank + static_cast<size_t>(m) * n;
      if (!loaded) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int r = pos + tid + 1024 * j;
          wv[j] = (j < per && r < n) ? __ldg(row + r) : -1;
        }
      }
      loaded = false;
      uint32_t rv[8];
      bool bad = false;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        rv[j] = 0xFFFFFFFFu;
        if (wv[j] != -1) {
          if (static_cast<unsigned>(wv[j]) < static_cast<unsigned>(n)) {
            rv[j] = static_cast<uint32_t>(__ldg(rrow + (kByPos ? pos + tid + 1024 * j : wv[j])));
          } else {
            report(ctrl, kStatusInvalidInput, wv[j]);
            bad = true;
          }
        }
      }
      unsigned long long mine = kNone;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (mine == kNone && rv[j] != 0xFFFFFFFFu) {
          const uint32_t cur = sbid[wv[j]];
          if (rv[j] < (cur >> 16))
            mine = (static_cast<unsigned long long>(pos + tid + 1024 * j) << 32) | cur;
        }
      }
      const int b = t % 3;
      if (bad) s_bad[b] = 1;
      // one atomic per warp: positions are distinct, so one lane holds its minimum
      const uint32_t at = mine == kNone ? 0xFFFFFFFFu : static_cast<uint32_t>(mine >> 32);
      const uint32_t warp_min = __reduce_min_sync(kFullMask, at);  // every lane takes part
      if (mine != kNone && at == warp_min) atomicMin(&s_best[b], mine);
      __syncthreads();
      const unsigned long long key = s_best[b];
      const bool any_bad = s_bad[b] != 0;
      if (tid == 0) {
        s_best[(t + 2) % 3] = kNone;
        s_bad[(t + 2) % 3] = 0;
      }
      ++t;
      if (any_bad) {
        stop = true;
        break;
      }
      if (key == kNone) {  // rejected by every woman of the span
        const int end = min(n, pos + 1024 * per);
        settled += end - pos;
        pos = end;
        per = min(2 * per, 8);
        continue;
      }
      const int best = static_cast<int>(key >> 32);
      const uint32_t old = static_cast<uint32_t>(key);
      settled += best - pos + 1;
      hops++;
      per_start = min(8, (best - from) / 1024 + 1);
      if (tid == 0) {
        pend_w = row[best];
        pend_val = (static_cast<uint32_t>(rrow[kByPos ? best : pend_w]) << 16) | static_cast<uint32_t>(m);
        pend_m = m;
        pend_pos = best;
        pend = true;
      }
      if (old == 0xFFFFFFFFu) {  // she was free: the chain ends; the next one must see her taken
        if (tid == 0) {
          sbid[pend_w] = pend_val;
          spos[pend_m] = static_cast<uint16_t>(pend_pos);
          pend = false;
        }
        __syncthreads();
        break;
      }
      // the man she drops: issue his first span at once
      m = static_cast<int>(old & 0xFFFFu);
      if (m >= n) {  // not a man: the shared state is corrupt
        if (tid == 0) report(ctrl, kStatusInvalidInput, m);
        stop = true;
        break;
      }
      pos = spos[m] + 1;
      from = pos;
      per = per_start;
      const int *nrow = pref_m + static_cast<size_t>(m) * n;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int r = pos + tid + 1024 * j;
        wv[j] = (j < per && r < n) ? __ldg(nrow + r) : -1;
      }
      loaded = true;
    }
    if (!stop && pos >= n && tid == 0) report(ctrl, kStatusInvalidInput, m);  // rejected by every woman
  }
  if (tid == 0 && pend) {
    sbid[pend_w] = pend_val;
    spos[pend_m] = static_cast<uint16_t>(pend_pos);
  }
  if (tid == 0) {
    atomicAdd(&ctrl->tail_proposals, settled);
    atomicAdd(&ctrl->tail_hops, hops);
  }
  __syncthreads();
  if (ld_volatile_s32(&ctrl->status)) return;
  if (tid == 0) ctrl->coop_count = 0;
  tail_finish(sbid, spos, match, n, ctrl, &s_props);
}

// ---------------------------------------------------------------------------
// Query-mode tail.  The same job as k_tail for the mode uniform-like inputs
// take, where every choice a man reaches lies in his prefix, written for the
// shortest chain of dependent operations per displacement: the last free
// man's chain is the critical path of the whole solve (thousands of steps,
// one after the other, on one SM).  Per step, every lane
//   decodes its prefix word (woman, her rank of him), reads her bid word and
//   -- in parallel with the ballot -- the position of the man holding her;
// one 64-bit shuffle hands the first candidate's holder, his position and
// the proposer's rank to the warp, which issues the holder's next window at
// once, then proposes (one relaxed shared atomic) while that load is in
// flight.  If the atomic displaced exactly that holder the warp continues
// with the window already loaded; otherwise (a race, rare here) it reloads.
// The abort flag is read at the top of a step and tested at its end.  A man
// whose next choice lies beyond his prefix stops the solve for the rank-mode
// retry round, as in k_tail.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t prefix_word(const uint32_t *__restrict__ prefix, int K, int Kn, int m, int r) {
  return r < Kn ? __ldg(prefix + static_cast<size_t>(m) * K + r) : 0u;
}

__global__ void __launch_bounds__(1024, 1) k_tail_q(const int32_t *__restrict__ pref_m,
                                                    const uint32_t *__restrict__ prefix, int K,
                                                    const unsigned long long *__restrict__ bid, Control *ctrl,
                                                    const int2 *__restrict__ tail_queue,
                                                    int32_t *__restrict__ match, int n) {
  if (ld_volatile_s32(&ctrl->mode) != kModeQuery) return;
  if (ld_volatile_s32(&ctrl->perfect)) {
    write_perfect(pref_m, match, n, ctrl);
    return;
  }
  if (!gate_open(kGateMain, ctrl)) return;
  if (ld_volatile_s32(&ctrl->retry)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *sbid = reinterpret_cast<uint32_t *>(smem_raw);
  uint16_t *spos = reinterpret_cast<uint16_t *>(smem_raw + static_cast<size_t>(n) * 4);
  __shared__ int s_next;
  __shared__ int s_abort;
  __shared__ unsigned long long s_props;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int Kn = min(K, n);

  const int queued = ld_volatile_s32(&ctrl->tail_count);
  const int first_unstarted = min(ld_volatile_s32(&ctrl->next_man), n);
  const int total = queued + (n - first_unstarted);
  tail_setup(bid, sbid, spos, n);
  if (tid == 0) {
    s_next = 0;
    s_abort = 0;
    s_props = 0;
    ctrl->tail_men = total;
  }
  __syncthreads();

  int m = -1, pos = 0;
  uint32_t raw = 0;
  unsigned long long settled = 0;
  unsigned int hops = 0;
  // The warp's next man from the queue (false when none is left); called
  // before the loop and where a chain ends, not at the top of every step.
  const auto next_man = [&]() {
    int i = 0;
    if (lane == 0) i = atomicAdd(&s_next, 1);
    i = __shfl_sync(kFullMask, i, 0);
    if (i >= total) return false;
    if (i < queued) {
      const int2 e = tail_queue[i];
      m = e.x;
      pos = e.y;
    } else {
      m = first_unstarted + (i - queued);
      pos = 0;
    }
    raw = prefix_word(prefix, K, Kn, m, pos + lane);
    return true;
  };
  for (bool more = next_man(); more;) {
    const int aborted = *reinterpret_cast<volatile int *>(&s_abort);  // tested at the end of the step
    const int r = pos + lane;
    const bool ok = r < Kn && raw != 0xFFFFFFFFu;
    const int w = ok ? static_cast<int>(raw >> 16) : 0;
    const uint32_t rk = raw & 0xFFFFu;
    const uint32_t cur = ok ? lds_relaxed_u32(sbid + w) : 0u;
    const uint32_t hp = (ok && cur != 0xFFFFFFFFu) ? spos[cur & 0xFFFFu] : 0u;
    unsigned cm = __ballot_sync(kFullMask, ok && rk < (cur >> 16));
    const unsigned stop = __ballot_sync(kFullMask, r < n && !ok);
    if (stop) cm &= (1u << (__ffs(stop) - 1)) - 1u;
    if (cm == 0) {
      if (stop) {  // beyond the prefix (retry in rank mode) or an invalid entry
        if (lane == 0) {
          const int re = pos + __ffs(stop) - 1;
          if (re < Kn) {
            report(ctrl, kStatusInvalidInput, m);
          } else {
            s_abort = 1;
            atomicExch(&ctrl->retry, 1);
          }
        }
        break;
      }
      settled += min(32, n - pos);
      pos += 32;
      if (pos >= n) {  // rejected by every woman: the lists are not permutations
        if (lane == 0) report(ctrl, kStatusInvalidInput, m);
        break;
      }
      raw = prefix_word(prefix, K, Kn, m, pos + lane);
      if (aborted) break;
      continue;
    }
    const int j = __ffs(cm) - 1;
    const unsigned long long info = __shfl_sync(
        kFullMask, (static_cast<unsigned long long>(hp | (rk << 16)) << 32) | cur, j);
    const uint32_t hw = static_cast<uint32_t>(info);
    const int hm = static_cast<int>(hw & 0xFFFFu);
    const int hpos = static_cast<int>((info >> 32) & 0xFFFFu) + 1;
    const uint32_t rkj = static_cast<uint32_t>(info >> 48);
    uint32_t next_raw = 0;
    if (hw != 0xFFFFFFFFu) next_raw = prefix_word(prefix, K, Kn, hm, hpos + lane);
    uint32_t old = 0;
    if (lane == j) {
      spos[m] = static_cast<uint16_t>(pos + j);
      old = atom_min_relaxed_shared(sbid + w, (rk << 16) | static_cast<uint32_t>(m));
    }
    old = __shfl_sync(kFullMask, old, j);
    // The common step -- accepted, displacing the holder whose window is
    // already loading -- takes one branch; everything else the other side.
    if (old == hw && (old >> 16) > rkj && hw != 0xFFFFFFFFu && !aborted) {
      settled += j + 1;
      hops++;
      m = hm;
      pos = hpos;
      raw = next_raw;
      continue;
    }
    if ((old >> 16) <= rkj) {  // someone better got there first: read the bids again
      if (aborted) break;
      continue;
    }
    settled += j + 1;
    hops++;
    if (old == 0xFFFFFFFFu) {
      if (aborted) break;
      more = next_man();  // the chain ended at a free woman
      continue;
    } else if (old == hw) {
      m = hm;
      pos = hpos;
      raw = next_raw;
    } else {
      m = static_cast<int>(old & 0xFFFFu);
      pos = spos[m] + 1;
      raw = prefix_word(prefix, K, Kn, m, pos + lane);
    }
    if (aborted) break;
  }
  if (lane == 0 && settled) {
    atomicAdd(&ctrl->tail_proposals, settled);
    atomicAdd(&ctrl->tail_hops, hops);
  }
  __syncthreads();
  if (s_abort || ld_volatile_s32(&ctrl->status)) return;
  tail_finish(sbid, spos, match, n, ctrl, &s_props);
}

// ---------------------------------------------------------------------------
// Start of the rank-mode retry round: every woman free again, counters reset.
// One CTA.
// ---------------------------------------------------------------------------
__global__ void k_retry_reset(unsigned long long *bid, int n, Control *ctrl) {
  if (!gate_open(kGateRetry, ctrl)) return;
  for (int w = threadIdx.x; w < n; w += blockDim.x) bid[w] = kFree;
  if (threadIdx.x == 0) {
    ctrl->mode = kModeRank;
    ctrl->next_man = 0;
    ctrl->free_count = n;
    ctrl->tail_count = 0;
    ctrl->tail_men = 0;
    ctrl->bulk_proposals = 0;
    ctrl->tail_proposals = 0;
    ctrl->bulk_hops = 0;
    ctrl->tail_hops = 0;
    ctrl->coop_count = 0;
    ctrl->use_filter = 0;
  }
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
__global__ void k_check_husband(const int32_t *__restrict__ match, int32_t *husband, int n, Control *ctrl) {
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
                             const int32_t *__restrict__ match, const int32_t *__restrict__ prank, int n,
                             Control *ctrl) {
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
