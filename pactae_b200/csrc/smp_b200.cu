// smp_b200.cu -- the C ABI of include/smp_b200.h: context, phases of one
// solve, the whole-solve call, rank inversion, stability check and the
// seeded generator.  Host code only orchestrates; the work is in
// solve_kernels.cuh and generate.cu.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <type_traits>

#include "common.cuh"
#include "internal.h"
#include "solve_kernels.cuh"
#include "swap_kernels.cuh"

using namespace smpb200;

namespace {

constexpr int kDefaultPrefixK = 192;
constexpr int kDefaultTailThreshold = 96;      // query mode
constexpr int kDefaultRankTailThreshold = 32;  // rank mode (deep scans)
constexpr int kDefaultBulkWindow = 256;
constexpr int kDefaultTailWindow = 256;
// Query buckets hold up to 1.5 K + 32 pairs per woman (at most n).
int query_capacity(int n, int K) { return std::min(n, K + K / 2 + 32); }
// Host-pointer solves of at least this n stream their inputs (solve_streamed).
// Rank-mode host-input solves send each list in this many row groups.
constexpr int kRankGroups = 8;
constexpr int kStreamMinN = 4096;
constexpr int kRankTailWindow = 256;
// Chains left when k_tail hands the rest to k_tail_coop (one at a time, the
// whole CTA scanning each).
constexpr int kCoopChains = 4;
constexpr int kU16MaxN = 65535;
// From this n the colour-tagged query inversion runs 384-thread CTAs.
constexpr int kLongRowN = 16384;

inline bool valid_ctx(const smp_ctx *ctx) { return ctx != nullptr && ctx->c.stream != nullptr; }

// Phase-boundary events recorded on the context's stream.
enum Ev {
  kEvStageBegin = 0,
  kEvStageEnd = 1,     // = precheck begin
  kEvPrecheckEnd = 2,  // = init begin
  kEvInvertEnd = 3,
  kEvInitEnd = 4,      // = core begin
  kEvBulkEnd = 5,
  kEvCoreEnd = 6,      // = post begin
  kEvPostEnd = 7,
  kEvCheckBegin = 8,
  kEvCheckEnd = 9,
};

float elapsed(const Ctx &c, int a, int b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, c.ev[a], c.ev[b]) != cudaSuccess) {
    cudaGetLastError();
    return 0.f;
  }
  return ms;
}

int rank_bytes_for(int n) { return n <= kU16MaxN ? 2 : 4; }

// Blocks per SM that a kernel can keep resident at the given block size.
template <typename Kernel>
int resident_grid(const Ctx &c, Kernel kernel, int block) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 4;
  }
  return c.sm_count * std::max(per_sm, 1);
}

// Number of 32-choice windows for a configured look-ahead (choices).
int subs_for(int window) {
  if (window <= 32) return 1;
  if (window <= 64) return 2;
  if (window <= 128) return 4;
  return 8;
}

// --------------------------------------------------------------------------
// SMP_F_VALIDATE: both lists, every row a permutation.
int enqueue_validate(Ctx &c) {
  const int n = c.n;
  const size_t smem = ((static_cast<size_t>(n) + 31) / 32) * 4;
  if (smem > c.smem_optin) {
    c.last_error = "validate: n too large for the shared-memory bitmap";
    return SMP_ERR_UNSUPPORTED;
  }
  if (allow_dynamic_smem(c, k_validate_rows) !=
      cudaSuccess)
    return c.fail_cuda("k_validate_rows smem attribute");
  const int grid = std::min(n, c.sm_count * 4);
  k_validate_rows<<<grid, 512, smem, c.stream>>>(c.pref_m, n, c.d_ctrl.as<Control>());
  k_validate_rows<<<grid, 512, smem, c.stream>>>(c.pref_w, n, c.d_ctrl.as<Control>());
  c.launches += 2;
  return c.check_launch("k_validate_rows");
}

// Per-solve plan, fixed once n is known: rank width, prefix width, whether
// the query mode may run, and the tail threshold.
void plan(Ctx &c) {
  const int n = c.n;
  c.rank_bytes = c.rank_bytes_cfg == 4 ? 4 : rank_bytes_for(n);
  c.K = 0;
  if (c.rank_bytes == 2 && c.prefix_k_cfg >= 0) {
    const int want = c.prefix_k_cfg > 0 ? c.prefix_k_cfg : kDefaultPrefixK;
    c.K = std::min(want, n);
  }
  c.query_ok = c.mode_cfg != 1 && c.K > 0 && n <= kU16MaxN && row_smem_bytes<uint16_t>(n) <= c.smem_optin;
  c.bulk_window = c.bulk_window_cfg > 0 ? c.bulk_window_cfg : kDefaultBulkWindow;
  c.tail_window = c.tail_window_cfg > 0 ? c.tail_window_cfg : kDefaultTailWindow;
  c.tail_threshold = 0;
  if (c.tail_threshold_cfg >= 0 && n <= kU16MaxN && tail_smem_bytes(n) <= c.smem_optin)
    c.tail_threshold = c.tail_threshold_cfg > 0 ? c.tail_threshold_cfg : kDefaultTailThreshold;
  c.tail_threshold_rank = c.tail_threshold_cfg > 0 ? c.tail_threshold_cfg : kDefaultRankTailThreshold;
}

int enqueue_precheck(Ctx &c, bool allow_perfect) {
  const int n = c.n;
  // zeroed on the device, never copied from the host block (k_precheck)
  if (cudaMemsetAsync(c.d_ctrl.ptr, 0, sizeof(Control), c.stream) != cudaSuccess)
    return c.fail_cuda("control reset");
  const size_t words = (static_cast<size_t>(n) + 31) / 32;
  if (cudaMemsetAsync(c.d_seen.ptr, 0, words * 4, c.stream) != cudaSuccess) return c.fail_cuda("seen reset");
  const int grid = std::max(1, std::min(c.sm_count * 4, (n + 255) / 256));
  k_precheck<<<grid, 256, 0, c.stream>>>(c.pref_m, n, c.d_seen.as<uint32_t>(), c.d_ctrl.as<Control>(),
                                         allow_perfect ? 1 : 0, c.query_ok ? 1 : 0);
  c.launches++;
  return c.check_launch("k_precheck");
}

template <typename RankT>
int enqueue_invert(Ctx &c, const int32_t *pref_w, RankT *rank, int gate) {
  const int n = c.n;
  const size_t smem16 = row_smem_bytes<uint16_t>(n);  // n <= 65535: at most 131 KB
  if constexpr (std::is_same<RankT, int32_t>::value) {
    if (n <= kU16MaxN) {  // int32 output from a uint16 shared row
      if (allow_dynamic_smem(c, k_invert_wide) != cudaSuccess)
        return c.fail_cuda("k_invert_wide smem attribute");
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_invert_wide, 512, smem16) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 1;
      }
      const int grid = std::min(n, c.sm_count * std::max(per_sm, 1));
      k_invert_wide<<<grid, 512, smem16, c.stream>>>(pref_w, rank, n, c.d_ctrl.as<Control>(), gate);
      c.launches++;
      return c.check_launch("k_invert_wide");
    }
    // Rows of more than 65535 ranks do not fit a shared row: scatter straight
    // to global memory, then verify.
    k_invert_global<<<c.sm_count * 8, 256, 0, c.stream>>>(pref_w, rank, n, c.d_ctrl.as<Control>(), gate);
    c.launches++;
    int rc = c.check_launch("k_invert_global");
    if (rc) return rc;
    k_invert_verify<<<c.sm_count * 8, 256, 0, c.stream>>>(pref_w, rank, n, c.d_ctrl.as<Control>(), gate);
    c.launches++;
    return c.check_launch("k_invert_verify");
  } else {
    if (allow_dynamic_smem(c, k_invert<RankT>) != cudaSuccess) return c.fail_cuda("k_invert smem attribute");
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_invert<RankT>, 512, smem16) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 1;
    }
    const int grid = std::min(n, c.sm_count * std::max(per_sm, 1));
    k_invert<RankT><<<grid, 512, smem16, c.stream>>>(pref_w, rank, n, c.d_ctrl.as<Control>(), gate);
    c.launches++;
    return c.check_launch("k_invert");
  }
}

int enqueue_invert_any(Ctx &c, int gate) {
  return c.rank_bytes == 2 ? enqueue_invert<uint16_t>(c, c.pref_w, c.d_rank.as<uint16_t>(), gate)
                           : enqueue_invert<int32_t>(c, c.pref_w, c.d_rank.as<int32_t>(), gate);
}

// The rank matrix a solve's proposals read: inverted (woman-major, kept for
// the checker) and transposed to man-major (d_rankT).
int enqueue_rank(Ctx &c, int gate) {
  int rc = c.d_rankT.ensure(static_cast<size_t>(c.n) * c.n * c.rank_bytes);
  if (!rc) rc = enqueue_invert_any(c, gate);
  if (rc) return rc;
  const int tiles = (c.n + 63) / 64;
  const int grid = static_cast<int>(std::min<long long>(static_cast<long long>(c.sm_count) * 4,
                                                        static_cast<long long>(tiles) * tiles));
  if (c.rank_bytes == 2 && c.n % 2 == 0)
    k_transpose_u16x2<<<grid, 512, 0, c.stream>>>(c.d_rank.as<uint16_t>(), c.d_rankT.as<uint16_t>(), c.n,
                                                  c.d_ctrl.as<Control>(), gate);
  else if (c.rank_bytes == 2)
    k_transpose<uint16_t><<<grid, 512, 0, c.stream>>>(c.d_rank.as<uint16_t>(), c.d_rankT.as<uint16_t>(), c.n,
                                                      c.d_ctrl.as<Control>(), gate);
  else
    k_transpose<int32_t><<<grid, 512, 0, c.stream>>>(c.d_rank.as<int32_t>(), c.d_rankT.as<int32_t>(), c.n,
                                                     c.d_ctrl.as<Control>(), gate);
  c.launches++;
  rc = c.check_launch("k_transpose");
  if (rc || c.rank_bytes != 2) return rc;
  // uint16 ranks: proposals read them by position (pr)
  rc = c.d_pr.ensure(static_cast<size_t>(c.n) * c.n * 2);
  if (rc) return rc;
  const size_t smem = row_smem_bytes<uint16_t>(c.n);
  if (allow_dynamic_smem(c, k_pr) != cudaSuccess) return c.fail_cuda("k_pr smem attribute");
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pr, 512, smem) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  k_pr<<<std::min(c.n, c.sm_count * std::max(per_sm, 1)), 512, smem, c.stream>>>(
      c.pref_m, c.d_rankT.as<uint16_t>(), c.d_pr.as<uint16_t>(), c.K > 0 ? c.d_prefix.as<uint32_t>() : nullptr,
      c.K > 0 ? c.K : 0, c.n, c.d_ctrl.as<Control>(), gate);
  c.launches++;
  return c.check_launch("k_pr");
}

// The matrix rank-mode proposals read, as rank_layout<RankT>() says.
template <typename RankT>
const RankT *proposal_ranks(const Ctx &c) {
  return reinterpret_cast<const RankT *>(rank_layout<RankT>() == 2 ? c.d_pr.ptr : c.d_rankT.ptr);
}

// Query mode: bucket the (man, position) pairs of every man's first K
// choices by woman (enqueue_query_index), then answer them from each
// woman's row (enqueue_qinvert, for all rows or a chunk of them).
int enqueue_query_index(Ctx &c) {
  const int n = c.n;
  const int qcap = query_capacity(n, c.K);
  const size_t total = static_cast<size_t>(n) * c.K;
  int rc = c.d_qcnt.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (!rc) rc = c.d_qlist.ensure(sizeof(uint32_t) * static_cast<size_t>(n) * qcap);
  if (rc) return rc;
  if (cudaMemsetAsync(c.d_qcnt.ptr, 0, sizeof(int32_t) * static_cast<size_t>(n), c.stream) != cudaSuccess)
    return c.fail_cuda("qcnt reset");
  const int grid = static_cast<int>(std::min<size_t>(static_cast<size_t>(c.sm_count) * 16, (total + 255) / 256));
  k_qscatter<<<grid, 256, 0, c.stream>>>(c.pref_m, n, c.K, qcap, c.d_qcnt.as<int32_t>(), c.d_qlist.as<uint32_t>(),
                                         c.d_ctrl.as<Control>());
  c.launches++;
  return c.check_launch("k_qscatter");
}

int enqueue_qinvert(Ctx &c, int w0, int w1) {
  // n <= kColorMaxN: the pipelined kernel with colour-tagged slots;
  // larger n: the one with a clearing pass per row.
  const bool long_rows = c.n >= kLongRowN;
  const auto kernel = c.n > kColorMaxN ? k_qinvert : long_rows ? k_qinvert_c<384> : k_qinvert_c<256>;
  const size_t smem = row_smem_bytes<uint16_t>(c.n);
  if (allow_dynamic_smem(c, kernel) !=
      cudaSuccess)
    return c.fail_cuda("k_qinvert smem attribute");
  const int block = c.n > kColorMaxN ? 512 : long_rows ? 384 : 256;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int qgrid = std::max(1, std::min(w1 - w0, c.sm_count * std::max(per_sm, 1)));
  kernel<<<qgrid, block, smem, c.stream>>>(c.pref_w, c.n, c.K, query_capacity(c.n, c.K), c.d_qcnt.as<int32_t>(),
                                         c.d_qlist.as<uint32_t>(), c.d_prefix.as<uint32_t>(), c.d_ctrl.as<Control>(),
                                         w0, w1);
  c.launches++;
  return c.check_launch(c.n <= kColorMaxN ? "k_qinvert_c" : "k_qinvert");
}

// Rows [w0, w1) of pref_w packed to uint16 in d_pw16 (host-input solves).
int enqueue_qinvert16(Ctx &c, int w0, int w1) {
  const size_t smem = row_smem_bytes<uint16_t>(c.n);
  if (allow_dynamic_smem(c, k_qinvert_p16) != cudaSuccess) return c.fail_cuda("k_qinvert_p16 smem attribute");
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_qinvert_p16, 256, smem) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int qgrid = std::max(1, std::min(w1 - w0, c.sm_count * std::max(per_sm, 1)));
  k_qinvert_p16<<<qgrid, 256, smem, c.stream>>>(c.d_pw16.as<uint16_t>(), c.n, c.K, query_capacity(c.n, c.K),
                                                c.d_qcnt.as<int32_t>(), c.d_qlist.as<uint32_t>(),
                                                c.d_prefix.as<uint32_t>(), c.d_ctrl.as<Control>(), w0, w1);
  c.launches++;
  return c.check_launch("k_qinvert_p16");
}

int enqueue_query(Ctx &c) {
  const int rc = enqueue_query_index(c);
  return rc ? rc : enqueue_qinvert(c, 0, c.n);
}

// Buffers of init and core, and every woman free (SmpEngineBamboo::InitProc
// fills partner_rank with n, smp_engine_bamboo.cu:37).
int init_buffers(Ctx &c) {
  const int n = c.n;
  const size_t nn = static_cast<size_t>(n) * n;
  int rc = c.d_rank.ensure(nn * c.rank_bytes);
  if (!rc) rc = c.d_bid.ensure(sizeof(unsigned long long) * n);
  if (!rc && c.K > 0) rc = c.d_prefix.ensure(sizeof(uint32_t) * static_cast<size_t>(n) * c.K);
  if (!rc) rc = c.d_tailq.ensure(sizeof(int2) * static_cast<size_t>(n));
  if (!rc) rc = c.d_match.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (rc) return rc;
  if (cudaMemsetAsync(c.d_bid.ptr, 0xFF, sizeof(unsigned long long) * n, c.stream) != cudaSuccess)
    return c.fail_cuda("bid reset");
  return SMP_OK;
}

int enqueue_init(Ctx &c) {
  int rc = init_buffers(c);
  if (rc) return rc;
  if (c.query_ok && c.known_mode != kModeRank) {
    rc = enqueue_query(c);
    if (rc) return rc;
  }
  if (c.known_mode != kModeQuery) rc = enqueue_rank(c, kGateModeRank);
  if (rc) return rc;
  // (k_pr wrote the prefix beside the uint16 ranks; int32 ranks run without one)
  if (cudaEventRecord(c.ev[kEvInvertEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  return SMP_OK;
}

template <typename RankT, int kSub>
int launch_bulk(Ctx &c, int round) {
  const RankT *rank = proposal_ranks<RankT>(c);
  const uint32_t *prefix = c.K > 0 ? c.d_prefix.as<uint32_t>() : nullptr;
  const int rank_threshold = c.tail_threshold > 0 ? std::min(c.tail_threshold, c.tail_threshold_rank) : 0;
  const size_t filter = sizeof(uint32_t) * static_cast<size_t>(c.n);
  if (round == 0 && c.known_mode != kModeQuery && filter + 1024 <= c.smem_optin) {  // the filter fits
    // k_wdistinct decides on the device which of the two variants runs
    k_wdistinct<<<1, 1024, sizeof(uint32_t) * ((c.n + 31) / 32), c.stream>>>(c.pref_w, c.n, c.d_ctrl.as<Control>());
    c.launches++;
    int rc = c.check_launch("k_wdistinct");
    if (rc) return rc;
    const auto kernel = k_bulk<RankT, kSub, true>;
    if (allow_dynamic_smem(c, kernel) !=
        cudaSuccess)
      return c.fail_cuda("k_bulk smem attribute");
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kFilterBlock, filter) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 1;
    }
    kernel<<<c.sm_count * std::max(per_sm, 1), kFilterBlock, filter, c.stream>>>(
        c.pref_m, rank, prefix, c.K, c.d_bid.as<unsigned long long>(), c.d_ctrl.as<Control>(), c.d_tailq.as<int2>(),
        c.n, c.tail_threshold, rank_threshold, round, -1);
    c.launches++;
    rc = c.check_launch("k_bulk (filtered)");
    if (rc) return rc;
  }
  k_bulk<RankT, kSub><<<resident_grid(c, k_bulk<RankT, kSub>, 256), 256, 0, c.stream>>>(
      c.pref_m, rank, prefix, c.K, c.d_bid.as<unsigned long long>(), c.d_ctrl.as<Control>(), c.d_tailq.as<int2>(),
      c.n, c.tail_threshold, rank_threshold, round, c.known_mode);
  c.launches++;
  return c.check_launch("k_bulk");
}

template <typename RankT, int kSub>
int launch_tail(Ctx &c, int round, int only_mode) {
  const RankT *rank = proposal_ranks<RankT>(c);
  const uint32_t *prefix = c.K > 0 ? c.d_prefix.as<uint32_t>() : nullptr;
  const size_t smem = tail_smem_bytes(c.n);
  if (allow_dynamic_smem(c, k_tail<RankT, kSub>) != cudaSuccess) return c.fail_cuda("k_tail smem attribute");
  k_tail<RankT, kSub><<<1, 1024, smem, c.stream>>>(c.pref_m, rank, prefix, c.K, c.d_bid.as<unsigned long long>(),
                                                   c.d_ctrl.as<Control>(), c.d_tailq.as<int2>(),
                                                   c.d_match.as<int32_t>(), c.n, round, only_mode, kCoopChains);
  c.launches++;
  int rc = c.check_launch("k_tail");
  if (rc) return rc;
  // the last chains, if k_tail handed them over
  if (allow_dynamic_smem(c, k_tail_coop<RankT>) != cudaSuccess)
    return c.fail_cuda("k_tail_coop smem attribute");
  k_tail_coop<RankT><<<1, 1024, smem, c.stream>>>(c.pref_m, rank, c.d_bid.as<unsigned long long>(),
                                                  c.d_ctrl.as<Control>(), c.d_match.as<int32_t>(), c.n);
  c.launches++;
  return c.check_launch("k_tail_coop");
}

int launch_tail_query(Ctx &c) {
  const size_t smem = tail_smem_bytes(c.n);
  if (allow_dynamic_smem(c, k_tail_q) !=
      cudaSuccess)
    return c.fail_cuda("k_tail_q smem attribute");
  k_tail_q<<<1, 1024, smem, c.stream>>>(c.pref_m, c.d_prefix.as<uint32_t>(), c.K, c.d_bid.as<unsigned long long>(),
                                        c.d_ctrl.as<Control>(), c.d_tailq.as<int2>(), c.d_match.as<int32_t>(), c.n);
  c.launches++;
  return c.check_launch("k_tail_q");
}

template <typename RankT>
int launch_tail_window(Ctx &c, int window, int round, int only_mode) {
  switch (subs_for(window)) {
    case 1: return launch_tail<RankT, 1>(c, round, only_mode);
    case 2: return launch_tail<RankT, 2>(c, round, only_mode);
    case 4: return launch_tail<RankT, 4>(c, round, only_mode);
    default: return launch_tail<RankT, 8>(c, round, only_mode);
  }
}

template <typename RankT>
int enqueue_round(Ctx &c, int round) {
  int rc;
  switch (subs_for(c.bulk_window)) {
    case 1: rc = launch_bulk<RankT, 1>(c, round); break;
    case 2: rc = launch_bulk<RankT, 2>(c, round); break;
    case 4: rc = launch_bulk<RankT, 4>(c, round); break;
    default: rc = launch_bulk<RankT, 8>(c, round); break;
  }
  if (rc) return rc;
  if (round == 0 && cudaEventRecord(c.ev[kEvBulkEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  if (c.tail_threshold <= 0) return SMP_OK;
  if (round == 1 || !c.query_ok || c.tail_window_cfg > 0) return launch_tail_window<RankT>(c, c.tail_window, round, -1);
  // Query-mode instances end in short chains, every choice in the prefix
  // (k_tail_q); rank-mode ones in deep scans (wide look-ahead).  Both are
  // enqueued and the device runs the one for the mode the precheck chose.
  if (c.known_mode != kModeRank) rc = launch_tail_query(c);
  if (!rc && c.known_mode != kModeQuery) rc = launch_tail_window<RankT>(c, kRankTailWindow, round, kModeRank);
  return rc;
}

// Rank-mode retry round; every kernel of it returns at once unless the
// query mode stopped because a man went beyond his prefix.
template <typename RankT>
int enqueue_retry_round(Ctx &c) {
  k_retry_reset<<<1, 1024, 0, c.stream>>>(c.d_bid.as<unsigned long long>(), c.n, c.d_ctrl.as<Control>());
  c.launches++;
  int rc = c.check_launch("k_retry_reset");
  if (!rc) rc = enqueue_rank(c, kGateRetry);
  if (!rc) rc = enqueue_round<RankT>(c, 1);
  return rc;
}

template <typename RankT>
int enqueue_core_t(Ctx &c) {
  const int n = c.n;
  int rc = c.d_tailq.ensure(sizeof(int2) * static_cast<size_t>(n));
  if (!rc) rc = c.d_match.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (rc) return rc;
  c.tail_ran = c.tail_threshold > 0;
  rc = enqueue_round<RankT>(c, 0);
  // with the mode known, the caller enqueues the retry round if round 0 asks
  if (rc || !c.query_ok || c.known_mode >= 0) return rc;
  return enqueue_retry_round<RankT>(c);
}

int enqueue_core(Ctx &c) { return c.rank_bytes == 2 ? enqueue_core_t<uint16_t>(c) : enqueue_core_t<int32_t>(c); }

int enqueue_post(Ctx &c) {
  if (c.tail_ran) return SMP_OK;  // the tail kernel already wrote d_match
  const int n = c.n;
  int rc = c.d_match.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (rc) return rc;
  const int grid = std::max(1, std::min(c.sm_count * 4, (n + 255) / 256));
  k_match<<<grid, 256, 0, c.stream>>>(c.pref_m, c.d_bid.as<unsigned long long>(), c.d_match.as<int32_t>(), n,
                                      c.d_ctrl.as<Control>());
  c.launches++;
  return c.check_launch("k_match");
}

// Copy d_match out to the caller.
int copy_match_out(Ctx &c, int32_t *match_out, bool device) {
  const size_t bytes = sizeof(int32_t) * static_cast<size_t>(c.n);
  const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (cudaMemcpyAsync(match_out, c.d_match.ptr, bytes, kind, c.stream) != cudaSuccess)
    return c.fail_cuda("match copy");
  return SMP_OK;
}

int read_control(Ctx &c) {
  if (cudaMemcpyAsync(c.h_ctrl, c.d_ctrl.ptr, sizeof(Control), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
    return c.fail_cuda("control readback");
  return SMP_OK;
}

int control_status(Ctx &c) {
  const int s = c.h_ctrl->status;
  if (s != 0) {
    char buf[96];
    std::snprintf(buf, sizeof(buf), "invalid input detected on the device (value %d)", c.h_ctrl->bad_value);
    c.last_error = buf;
  }
  return s;
}

// Checker body: needs c.pref_m, c.d_rank valid for c.n.
template <typename RankT>
int enqueue_check_t(Ctx &c, const int32_t *match) {
  const int n = c.n;
  int rc = c.d_husband.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (!rc) rc = c.d_prank.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (rc) return rc;
  if (cudaMemsetAsync(c.d_husband.ptr, 0xFF, sizeof(int32_t) * static_cast<size_t>(n), c.stream) != cudaSuccess)
    return c.fail_cuda("husband reset");
  const int grid = std::max(1, std::min(c.sm_count * 4, (n + 255) / 256));
  k_check_husband<<<grid, 256, 0, c.stream>>>(match, c.d_husband.as<int32_t>(), n, c.d_ctrl.as<Control>());
  k_check_prank<RankT><<<grid, 256, 0, c.stream>>>(c.d_husband.as<int32_t>(), reinterpret_cast<const RankT *>(c.d_rank.ptr),
                                                  c.d_prank.as<int32_t>(), n, c.d_ctrl.as<Control>());
  const int sgrid = std::max(1, std::min(c.sm_count * 8, (n * 32 + 255) / 256));
  k_check_scan<RankT><<<sgrid, 256, 0, c.stream>>>(c.pref_m, reinterpret_cast<const RankT *>(c.d_rank.ptr), match,
                                                  c.d_prank.as<int32_t>(), n, c.d_ctrl.as<Control>());
  c.launches += 3;
  return c.check_launch("k_check");
}

int enqueue_check(Ctx &c, const int32_t *match) {
  return c.rank_bytes == 2 ? enqueue_check_t<uint16_t>(c, match) : enqueue_check_t<int32_t>(c, match);
}

// Per-solve state reset and plan for size n.
int stage_reset(Ctx &c, int32_t n) {
  c.n = n;
  c.staged = false;
  c.rank_valid = false;
  c.phase = 0;
  c.stats = smp_stats{};
  c.stats.n = n;
  c.stats.blocking_pairs = -1;
  c.launches = 0;
  c.known_mode = -1;
  c.swapped = false;
  plan(c);
  return SMP_OK;
}

// Bring the inputs onto the device (or adopt device pointers).
int do_stage(Ctx &c, const int32_t *pref_m, const int32_t *pref_w, int32_t n, uint32_t flags) {
  if (!pref_m || !pref_w || n <= 0 || n > SMP_B200_MAX_N) {
    c.last_error = "stage: null list or n out of range";
    return SMP_ERR_INVALID_ARG;
  }
  stage_reset(c, n);
  int rc = c.d_ctrl.ensure(sizeof(Control));
  if (!rc) rc = c.d_seen.ensure(((static_cast<size_t>(n) + 31) / 32) * 4);
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvStageBegin], c.stream) != cudaSuccess) return c.fail_cuda("event");
  if (flags & SMP_F_DEVICE_PTRS) {
    c.pref_m = pref_m;
    c.pref_w = pref_w;
  } else {
    const size_t bytes = sizeof(int32_t) * static_cast<size_t>(n) * n;
    rc = c.d_pref_w.ensure(bytes);
    if (!rc) rc = c.d_pref_m.ensure(bytes);
    if (rc) return rc;
    if (cudaMemcpyAsync(c.d_pref_w.ptr, pref_w, bytes, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
      return c.fail_cuda("pref_w copy");
    if (cudaMemcpyAsync(c.d_pref_m.ptr, pref_m, bytes, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
      return c.fail_cuda("pref_m copy");
    c.pref_m = c.d_pref_m.as<int32_t>();
    c.pref_w = c.d_pref_w.as<int32_t>();
  }
  if (cudaEventRecord(c.ev[kEvStageEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  c.staged = true;
  return SMP_OK;
}

void fill_stats(Ctx &c, bool timed_phases) {
  c.stats.proposals = static_cast<int64_t>(c.h_ctrl->proposals);
  c.stats.tail_proposals = static_cast<int64_t>(c.h_ctrl->tail_proposals);
  c.stats.bulk_hops = static_cast<int32_t>(c.h_ctrl->bulk_hops);
  c.stats.tail_hops = static_cast<int32_t>(c.h_ctrl->tail_hops);
  c.stats.perfect = c.h_ctrl->perfect;
  c.stats.mode = c.swapped ? 3 : c.h_ctrl->retry ? 2 : c.h_ctrl->mode;
  c.stats.tail_men = c.tail_ran && !c.swapped ? c.h_ctrl->tail_men : 0;
  c.stats.rank_bytes = c.rank_bytes;
  c.stats.kernel_launches = c.launches;
  if (timed_phases) {
    c.stats.stage_ms = elapsed(c, kEvStageBegin, kEvStageEnd);
    c.stats.precheck_ms = elapsed(c, kEvStageEnd, kEvPrecheckEnd);
    c.stats.init_ms = elapsed(c, kEvPrecheckEnd, kEvInitEnd);
    c.stats.core_ms = elapsed(c, kEvInitEnd, kEvCoreEnd);
    c.stats.post_ms = elapsed(c, kEvCoreEnd, kEvPostEnd);
    c.stats.total_ms = elapsed(c, kEvStageEnd, kEvPostEnd);
  }
  // Kernel-level times exist when the inversion and proposal kernels ran.
  if (c.phase >= 3 && !c.h_ctrl->perfect) {
    c.stats.invert_ms = elapsed(c, kEvPrecheckEnd, kEvInvertEnd);
    c.stats.bulk_ms = elapsed(c, kEvInitEnd, kEvBulkEnd);
    c.stats.tail_ms = c.tail_ran && !c.swapped ? elapsed(c, kEvBulkEnd, kEvCoreEnd) : 0.f;
  }
}

}  // namespace

namespace smpb200 {

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxDevices] = {};
}  // namespace

cudaMemPool_t device_pool(int device) {
  if (device < 0 || device >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pools[device]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;  // buffers then fall back to cudaMalloc
    }
    // Keep freed memory for the next allocation instead of returning it at
    // every synchronisation.
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[device] = pool;
  }
  return g_pools[device];
}

void trim_device_pool(int device) {
  if (device < 0 || device >= kMaxDevices) return;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (g_pools[device]) cudaMemPoolTrimTo(g_pools[device], 0);
}

// Allocates every buffer a device-pointer solve of size n uses, in either
// mode and with the checker, so that later solves up to n allocate nothing.
int reserve_buffers(Ctx &c, int32_t n) {
  if (n <= 0 || n > SMP_B200_MAX_N) return SMP_ERR_INVALID_ARG;
  stage_reset(c, n);
  const size_t nn = static_cast<size_t>(n) * n;
  int rc = c.d_ctrl.ensure(sizeof(Control));
  if (!rc) rc = c.d_seen.ensure(((static_cast<size_t>(n) + 31) / 32) * 4);
  if (!rc) rc = init_buffers(c);
  if (!rc) rc = c.d_rankT.ensure(nn * c.rank_bytes);
  if (!rc && c.rank_bytes == 2) rc = c.d_pr.ensure(nn * 2);
  if (!rc && c.query_ok) rc = c.d_qcnt.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (!rc && c.query_ok)
    rc = c.d_qlist.ensure(sizeof(uint32_t) * static_cast<size_t>(n) * query_capacity(n, c.K));
  if (!rc) rc = c.d_husband.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (!rc) rc = c.d_prank.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (!rc) rc = c.sync("reserve");
  c.n = 0;
  return rc;
}

// Enqueues a whole solve on c.stream with no host round trip (stage,
// precheck, init, core, post, the match copy, optional check, control
// readback).  The caller synchronises the stream, then calls solve_finish.
int solve_enqueue(Ctx &c, const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *match_out,
                  uint32_t flags) {
  int rc = do_stage(c, pref_m, pref_w, n, flags);
  if (rc) return rc;
  // One stream, no host round trips: kernels read the control block.
  rc = enqueue_precheck(c, (flags & SMP_F_NO_PRECHECK) == 0);
  if (!rc && (flags & SMP_F_VALIDATE)) rc = enqueue_validate(c);
  if (!rc && cudaEventRecord(c.ev[kEvPrecheckEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc) rc = enqueue_init(c);
  if (!rc && cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc) rc = enqueue_core(c);
  if (!rc && cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc) rc = enqueue_post(c);
  if (!rc && (flags & SMP_F_DEVICE_PTRS)) rc = copy_match_out(c, match_out, true);
  if (!rc && cudaEventRecord(c.ev[kEvPostEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc && !(flags & SMP_F_DEVICE_PTRS)) rc = copy_match_out(c, match_out, false);
  if (!rc && (flags & SMP_F_CHECK)) {
    if (cudaEventRecord(c.ev[kEvCheckBegin], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    // The checker reuses the solve's rank matrix; only a solve that built
    // none (perfect, or query mode) builds it here.
    if (!rc) rc = enqueue_invert_any(c, kGateNoRank);
    if (!rc) rc = enqueue_check(c, c.d_match.as<int32_t>());
    if (!rc && cudaEventRecord(c.ev[kEvCheckEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  }
  if (!rc) rc = read_control(c);
  return rc;
}

// The synchronous solve, in one pass when the precheck picks the query mode
// (uniform-like inputs): the pass enqueues only that mode's kernels -- the
// bulk restricted to it, so a rank-mode instance cannot start proposing
// before its ranks exist -- through the match copy, and the host waits once.
// If the precheck chose the rank mode, or a man went beyond his prefix, a
// second pass enqueues what remains and copies the match again.  Kernels a
// mode gates off would still cost a launch and a pass of every CTA over the
// gate: 14 of them took about 0.1 ms of a 2.6 ms uniform solve at
// n = 30000, where a wait for the precheck costs about 30 us.  The kernels
// keep their gates, so the device still decides what runs.  The checker
// (SMP_F_CHECK) must see the final matching: those solves take the fully
// gated pipeline.
int solve_swapped(Ctx &c, uint32_t flags, int32_t *match_out, bool &swapped, bool men_screened = false);

int solve_staged(Ctx &c, const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *match_out,
                 uint32_t flags, smp_stats *st) {
  // the checker, a disabled tail or a configured tail window (whose tail
  // kernel serves either mode) take the fully gated pipeline.  The tail is
  // this n's (plan), not the previous solve's: a fresh context's first solve
  // would otherwise always take the gated pipeline.
  if (n > 0 && n <= SMP_B200_MAX_N) {
    c.n = n;
    plan(c);
  }
  if ((flags & SMP_F_CHECK) || !(c.tail_threshold > 0) || c.tail_window_cfg > 0) {
    int rc = solve_enqueue(c, pref_m, pref_w, n, match_out, flags);
    if (!rc) rc = c.sync("solve");
    return rc ? rc : solve_finish(c, flags, st);
  }
  int rc = do_stage(c, pref_m, pref_w, n, flags);
  if (rc) return rc;
  const auto finish_pass = [&]() {
    int r = SMP_OK;
    if (cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess) r = c.fail_cuda("event");
    if (!r) r = enqueue_post(c);
    if (!r && (flags & SMP_F_DEVICE_PTRS)) r = copy_match_out(c, match_out, true);
    if (!r && cudaEventRecord(c.ev[kEvPostEnd], c.stream) != cudaSuccess) r = c.fail_cuda("event");
    if (!r && !(flags & SMP_F_DEVICE_PTRS)) r = copy_match_out(c, match_out, false);
    if (!r) r = read_control(c);
    if (!r) r = c.sync("solve");
    return r;
  };
  // pass 1: as if the precheck picks the query mode
  rc = enqueue_precheck(c, (flags & SMP_F_NO_PRECHECK) == 0);
  if (!rc && (flags & SMP_F_VALIDATE)) rc = enqueue_validate(c);
  if (!rc && cudaEventRecord(c.ev[kEvPrecheckEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  const bool speculate = c.query_ok;
  if (speculate) {
    c.known_mode = kModeQuery;
    if (!rc) rc = enqueue_init(c);
    if (!rc && cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    if (!rc) rc = enqueue_core(c);
    if (!rc) rc = finish_pass();
  } else {
    if (!rc) rc = read_control(c);
    if (!rc) rc = c.sync("precheck");
  }
  if (rc) return rc;
  const Control &h = *c.h_ctrl;
  const bool done = speculate && !h.status && (h.perfect || (h.mode == kModeQuery && !h.retry));
  if (!done && !h.status) {
    // pass 2: the rank mode, or the rank-mode retry of a query-mode round 0
    bool swapped = false;
    if (speculate && h.mode == kModeQuery && h.retry) {
      c.known_mode = -1;
      rc = c.rank_bytes == 2 ? enqueue_retry_round<uint16_t>(c) : enqueue_retry_round<int32_t>(c);
    } else {
      // one first choice for every man: perhaps one list for every man
      if (!h.perfect && h.mode == kModeRank && h.distinct == 1 && n >= 2 && c.mode_cfg == 0)
        rc = solve_swapped(c, flags, match_out, swapped);
      if (!rc && !swapped) {
        c.known_mode = h.perfect ? -1 : h.mode;
        rc = enqueue_init(c);
        if (!rc && cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
        if (!rc) rc = enqueue_core(c);
      }
    }
    if (!rc && !swapped) rc = finish_pass();
    if (rc) return rc;
  }
  return solve_finish(c, flags, st);
}

// A rank-mode solve whose men all make the same first choice may have men
// who share one list.  The screen checks that on all SMs (and that pref_w's
// rows are permutations); if so, the women propose and `swapped` is set,
// else the caller runs the men's rank-mode pass.  Stops after the screen,
// with `swapped` set, when it found invalid input.
int solve_swapped(Ctx &c, uint32_t flags, int32_t *match_out, bool &swapped, bool men_screened) {
  swapped = false;
  const int n = c.n;
  const size_t screen_smem = swap_screen_smem(n);
  if (screen_smem > c.smem_optin) return SMP_OK;
  int rc = c.d_swap_pos.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (!rc) rc = c.d_bid.ensure(sizeof(unsigned long long) * static_cast<size_t>(n));
  if (!rc) rc = c.d_match.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (rc) return rc;
  Control *ctrl = c.d_ctrl.as<Control>();
  int32_t *pos = c.d_swap_pos.as<int32_t>();
  unsigned long long *bid = c.d_bid.as<unsigned long long>();
  const int grid = std::max(1, std::min(c.sm_count * 4, (n + 255) / 256));
  if (cudaMemsetAsync(pos, 0xFF, sizeof(int32_t) * static_cast<size_t>(n), c.stream) != cudaSuccess)
    return c.fail_cuda("swap reset");
  k_swap_pos<<<grid, 256, 0, c.stream>>>(c.pref_m, pos, n, ctrl);
  if (allow_dynamic_smem(c, k_swap_screen) != cudaSuccess) return c.fail_cuda("k_swap_screen smem attribute");
  int per_sm = 0;  // one wave: every CTA resident
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_swap_screen, 256, screen_smem) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int t0 = men_screened ? n : 1;  // the host compared the men's rows already
  k_swap_screen<<<std::max(1, std::min(2 * n - t0, c.sm_count * std::max(per_sm, 1))), 256, screen_smem, c.stream>>>(
      c.pref_m, c.pref_w, n, ctrl, t0);
  c.launches += 2;
  rc = c.check_launch("k_swap_screen");
  if (!rc && cudaEventRecord(c.ev[kEvInvertEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc) rc = read_control(c);
  if (!rc) rc = c.sync("swap screen");
  if (rc) return rc;
  if (c.h_ctrl->status) {
    swapped = true;
    return SMP_OK;
  }
  if (c.h_ctrl->swap_fail) return SMP_OK;
  swapped = true;
  c.swapped = true;
  if (!c.h_ctrl->w_differ) {  // the women share one list too: pair rank for rank
    if (cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
    if (cudaEventRecord(c.ev[kEvBulkEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
    if (cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
    k_swap_direct<<<grid, 256, 0, c.stream>>>(c.pref_m, c.pref_w, c.d_match.as<int32_t>(), n, ctrl);
    c.launches++;
    rc = c.check_launch("k_swap_direct");
  } else {
    if (cudaMemsetAsync(bid, 0xFF, sizeof(unsigned long long) * static_cast<size_t>(n), c.stream) != cudaSuccess)
      return c.fail_cuda("swap bid reset");
    if (cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
    k_swap_gs<<<c.sm_count * 4, 256, 0, c.stream>>>(c.pref_m, c.pref_w, pos, bid, n, ctrl, nullptr, n, nullptr,
                                                    nullptr, 0);
    c.launches++;
    rc = c.check_launch("k_swap_gs");
    if (!rc && cudaEventRecord(c.ev[kEvBulkEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    if (!rc && cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    if (rc) return rc;
    k_swap_match<<<grid, 256, 0, c.stream>>>(c.pref_m, bid, c.d_match.as<int32_t>(), n, ctrl);
    c.launches++;
    rc = c.check_launch("k_swap_match");
  }
  if (!rc) rc = copy_match_out(c, match_out, (flags & SMP_F_DEVICE_PTRS) != 0);
  if (!rc && cudaEventRecord(c.ev[kEvPostEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc) rc = read_control(c);
  if (!rc) rc = c.sync("solve");
  return rc;
}

// Statistics and status of a solve whose stream has completed.
int solve_finish(Ctx &c, uint32_t flags, smp_stats *st) {
  c.phase = 3;
  fill_stats(c, true);
  c.phase = 4;
  if (flags & SMP_F_CHECK) {
    c.stats.blocking_pairs = static_cast<int64_t>(c.h_ctrl->blocking);
    c.stats.check_ms = elapsed(c, kEvCheckBegin, kEvCheckEnd);
    // The checker recounts the proposals from the matching itself.
    if (c.h_ctrl->check_proposals != c.h_ctrl->proposals && c.h_ctrl->status == 0) {
      c.last_error = "checker proposal count differs from the solve's";
      return SMP_ERR_CUDA;
    }
  }
  if (st) *st = c.stats;
  return control_status(c);
}

// Host-pointer solve that moves only what the solve reads, overlapped with
// the work.  A query-mode solve reads only each man's first K choices of
// pref_m (plus his first choice for the precheck), and pref_w row by row in
// the inversion.  So: copy the first K columns of pref_m, run the precheck
// and read its decision; in query mode send pref_w packed to uint16 in row
// groups and invert each group as it lands, and copy the rest of pref_m only
// if a man goes beyond his prefix (the rank-mode retry).  A rank-mode
// instance sends both lists packed and widens them on the device, unless
// the men may share one list: then pref_w crosses as it is while the host
// threads compare the men's rows, and only row 0 of pref_m follows if they
// are all alike.  A perfect instance copies nothing more.  Two host round
// trips (after the precheck and after round 0) are the price.
bool streamed_fits(const Ctx &c, uint32_t flags) {
  return !(flags & (SMP_F_DEVICE_PTRS | SMP_F_VALIDATE | SMP_F_CHECK)) && c.query_ok && c.K > 0 && c.K < c.n &&
         c.tail_threshold > 0 && c.n >= kStreamMinN;
}

// The context's host threads (created on first use): up to 16.  On a
// 16-core host, 8, 12 and 16 packed and sent an n = 30000 list in the same
// 37 ms, bound by reading it from host DRAM; comparing the men's rows with
// row 0 took 58, 53 and 44 ms.
HostPool *host_pool(Ctx &c) {
  if (!c.pack_pool) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    c.pack_pool.reset(new (std::nothrow) HostPool(static_cast<int>(std::min(hw, 16u))));
  }
  return c.pack_pool.get();
}

// Host-input solves send their lists packed to uint16 -- half the bytes on
// the host link, which is what a host-input solve of n = 30000 waits for --
// through the context's HostLink, when the host has threads to pack with.
// Sets up the packed device buffers (pref_w's, and pref_m's when both lists
// cross), the host threads and the link on first use; false if packing does
// not apply (the caller then copies int32 rows).
bool link_ready(Ctx &c, bool both) {
  const int n = c.n;
  if (n > 65535 || n < 8) return false;
  const unsigned hw = std::thread::hardware_concurrency();
  if (hw < 4) return false;
  const size_t bytes = sizeof(uint16_t) * static_cast<size_t>(n) * n;
  if (c.d_pw16.ensure(bytes)) return false;
  if (both && c.d_pm16.ensure(bytes)) return false;
  if (!host_pool(c)) return false;
  if (!c.link) {
    c.link.reset(new (std::nothrow) HostLink());
    if (!c.link || c.link->open(c.pack_pool.get()) != SMP_OK) {
      c.link.reset();
      return false;
    }
  }
  return true;
}

int enqueue_widen16(Ctx &c, const uint16_t *src, int32_t *dst, size_t begin, size_t end) {
  if (begin >= end) return SMP_OK;
  const size_t steps = (end - (begin & ~size_t{7}) + 7) / 8;
  const int grid = static_cast<int>(std::min<size_t>(static_cast<size_t>(c.sm_count) * 8, (steps + 255) / 256));
  k_widen16<<<grid, 256, 0, c.stream>>>(src, dst, begin, end);
  c.launches++;
  return c.check_launch("k_widen16");
}

// Sends parts through the link in `groups` row groups per part and, as each
// group lands, enqueues on c.stream what uses its rows (on_group(part, r0,
// r1)).  Returns after every copy has finished.
template <typename OnGroup>
int send_packed(Ctx &c, const HostLink::Part *parts, int nparts, int groups, OnGroup on_group) {
  HostLink &link = *c.link;
  int rc = link.start(parts, nparts, c.n, groups, c.stream);
  if (rc) {
    c.last_error = link.error();
    return rc;
  }
  for (int g = 0; !rc && g < nparts * groups; ++g) {
    int p = 0, r0 = 0, r1 = 0;
    link.group_rows(g, &p, &r0, &r1);
    rc = link.wait_group(g, c.stream);
    if (rc)
      c.last_error = link.error();
    else if (r0 < r1)
      rc = on_group(p, r0, r1);
  }
  // the workers read the caller's buffers: join them even after an error
  const int lr = link.finish();
  if (!rc && lr) {
    rc = lr;
    c.last_error = link.error();
  }
  return rc;
}

// Does every row of the host matrix pref_m equal row 0 (in its first `cols`
// entries; all of them by default)?  Rows are compared on the context's host
// threads, which stop at the first difference.
bool host_rows_equal_row0(Ctx &c, const int32_t *pref_m, int n, int cols = -1) {
  if (!host_pool(c)) return false;
  std::atomic<bool> differ{false};
  const size_t row_bytes = sizeof(int32_t) * static_cast<size_t>(cols < 0 ? n : cols);
  const auto job = [&](int i, int parts) {
    const int r0 = 1 + static_cast<int>(static_cast<int64_t>(n - 1) * i / parts);
    const int r1 = 1 + static_cast<int>(static_cast<int64_t>(n - 1) * (i + 1) / parts);
    for (int r = r0; r < r1 && !differ.load(std::memory_order_relaxed); ++r)
      if (std::memcmp(pref_m + static_cast<size_t>(r) * n, pref_m, row_bytes) != 0)
        differ.store(true, std::memory_order_relaxed);
  };
  c.pack_pool->run(job);
  return !differ.load();
}

// Host-input solve whose men all make the same first choice: perhaps one
// list L for every man.  Then the stable matching is unique, the women
// propose, and each woman reads her row only as far as the man she ends
// with.  The k-th woman of L ends where the k-1 before her have not taken
// her man, about n / (n - k + 1) entries in: only the last few hundred go
// past a short prefix.
//   1. Row 0 of pref_m and the first K entries of every woman's row cross
//      as int32 while the host threads compare every man's row with row 0.
//   2. A row differs: nothing more is sent here (shared = false); the caller
//      runs the men's rank mode, which needs both lists.
//   3. If every woman's row equals row 0 too (her first K entries first,
//      then the whole row, on the host threads), only row 0 of pref_w is
//      sent and the k-th man of that list pairs with the k-th woman of L.
//   4. Else the kSharedDeepRows women L ranks lowest are sent whole through
//      the link (packed, widened on the device), and the women propose.  A
//      woman who reaches the end of what the device holds of her row stops;
//      her row is sent and she resumes, until none stops.
// Every entry sent is checked on the device: in range, and no man twice in
// what was sent of a row.  Entries never sent are never read (as a
// query-mode solve never reads a man's choices beyond his prefix).
constexpr int kSharedDeepRows = 1024;

int solve_shared_host(Ctx &c, const int32_t *pref_m, const int32_t *pref_w, uint32_t flags, int32_t *match_out,
                      bool &shared) {
  const int n = c.n;
  shared = false;
  int32_t *dm = c.d_pref_m.as<int32_t>();
  int32_t *dw = c.d_pref_w.as<int32_t>();
  const size_t row = sizeof(int32_t) * static_cast<size_t>(n);
  const int kw = std::min(n, c.K);
  if (cudaMemcpyAsync(dm + c.K, pref_m + c.K, sizeof(int32_t) * (n - c.K), cudaMemcpyHostToDevice, c.stream) !=
      cudaSuccess)
    return c.fail_cuda("pref_m row 0 copy");
  if (cudaMemcpy2DAsync(dw, row, pref_w, row, sizeof(int32_t) * kw, n, cudaMemcpyHostToDevice, c.stream) !=
      cudaSuccess)
    return c.fail_cuda("pref_w prefix copy");
  if (!host_rows_equal_row0(c, pref_m, n)) return SMP_OK;
  shared = true;
  c.swapped = true;
  int rc = c.d_swap_pos.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (!rc) rc = c.d_bid.ensure(sizeof(unsigned long long) * static_cast<size_t>(n));
  if (!rc) rc = c.d_match.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (!rc) rc = c.d_swap_full.ensure(static_cast<size_t>(n));
  if (!rc) rc = c.d_swap_over.ensure(2 * sizeof(int2) * static_cast<size_t>(n));
  if (!rc) rc = c.d_swap_rows.ensure(sizeof(int32_t) * static_cast<size_t>(n));
  if (rc) return rc;
  Control *ctrl = c.d_ctrl.as<Control>();
  int32_t *pos = c.d_swap_pos.as<int32_t>();
  unsigned long long *bid = c.d_bid.as<unsigned long long>();
  uint8_t *full = c.d_swap_full.as<uint8_t>();
  int2 *over[2] = {c.d_swap_over.as<int2>(), c.d_swap_over.as<int2>() + n};
  int32_t *d_rows = c.d_swap_rows.as<int32_t>();
  const size_t check_smem = swap_screen_smem(n);
  const int grid = std::max(1, std::min(c.sm_count * 4, (n + 255) / 256));
  const int row_grid = std::max(1, std::min(c.sm_count * 8, n));

  // Sends the listed women's rows whole (ids in [0, n)), widens them into
  // dw, checks them and marks them whole.
  const auto send_rows = [&](const std::vector<int32_t> &rows) -> int {
    const int count = static_cast<int>(rows.size());
    if (!count) return SMP_OK;
    if (cudaMemcpyAsync(d_rows, rows.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, c.stream) !=
        cudaSuccess)
      return c.fail_cuda("row list copy");
    HostLink::Part part = {pref_w, c.d_pw16.as<uint16_t>(), count, rows.data()};
    int r = send_packed(c, &part, 1, 1, [&](int, int r0, int r1) {
      k_widen16_rows<<<std::max(1, std::min(r1 - r0, c.sm_count * 4)), 256, 0, c.stream>>>(
          c.d_pw16.as<uint16_t>(), dw, d_rows + r0, r1 - r0, n);
      c.launches++;
      return c.check_launch("k_widen16_rows");
    });
    if (r) return r;
    k_swap_rows_check<<<std::max(1, std::min(count, c.sm_count * 8)), 256, check_smem, c.stream>>>(
        dw, n, d_rows, count, n, ctrl);
    k_swap_mark_full<<<std::max(1, std::min(c.sm_count, (count + 255) / 256)), 256, 0, c.stream>>>(full, d_rows,
                                                                                                  count, n);
    c.launches += 2;
    return c.check_launch("k_swap_rows_check");
  };
  const auto reset_queue = [&]() -> int {  // swap_next, w_differ, swap_over
    return cudaMemsetAsync(reinterpret_cast<char *>(ctrl) + offsetof(Control, swap_next), 0, 3 * sizeof(int32_t),
                           c.stream) == cudaSuccess
               ? SMP_OK
               : c.fail_cuda("swap queue reset");
  };

  if (cudaEventRecord(c.ev[kEvPrecheckEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  // The women may share one list M as well (their first K entries first,
  // then every row on the host threads): the k-th man of M and the k-th
  // woman of L then pair up, no proposals.  Only row 0 of pref_w is sent;
  // it and L are checked before the pairing writes match[].
  if (host_rows_equal_row0(c, pref_w, n, kw) && host_rows_equal_row0(c, pref_w, n)) {
    if (cudaMemcpyAsync(dw + kw, pref_w + kw, sizeof(int32_t) * (n - kw), cudaMemcpyHostToDevice, c.stream) !=
            cudaSuccess ||
        cudaMemsetAsync(pos, 0xFF, sizeof(int32_t) * static_cast<size_t>(n), c.stream) != cudaSuccess ||
        cudaMemsetAsync(d_rows, 0, sizeof(int32_t), c.stream) != cudaSuccess)  // the row list {0}
      return c.fail_cuda("shared lists copy");
    k_swap_pos<<<grid, 256, 0, c.stream>>>(dm, pos, n, ctrl);
    k_swap_rows_check<<<1, 256, check_smem, c.stream>>>(dw, n, d_rows, 1, n, ctrl);
    c.launches += 2;
    rc = c.check_launch("k_swap_rows_check");
    if (!rc) rc = read_control(c);
    if (!rc) rc = c.sync("shared lists check");
    if (rc) return rc;
    if (!c.h_ctrl->status) {
      if (cudaEventRecord(c.ev[kEvInvertEnd], c.stream) != cudaSuccess ||
          cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess ||
          cudaEventRecord(c.ev[kEvBulkEnd], c.stream) != cudaSuccess ||
          cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess)
        return c.fail_cuda("event");
      k_swap_direct<<<grid, 256, 0, c.stream>>>(dm, dw, c.d_match.as<int32_t>(), n, ctrl);
      c.launches++;
      rc = c.check_launch("k_swap_direct");
      if (!rc) rc = copy_match_out(c, match_out, (flags & SMP_F_DEVICE_PTRS) != 0);
      if (!rc && cudaEventRecord(c.ev[kEvPostEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
      if (!rc) rc = read_control(c);
      if (!rc) rc = c.sync("solve");
    }
    return rc;
  }
  if (cudaMemsetAsync(pos, 0xFF, sizeof(int32_t) * static_cast<size_t>(n), c.stream) != cudaSuccess ||
      cudaMemsetAsync(full, 0, static_cast<size_t>(n), c.stream) != cudaSuccess ||
      cudaMemsetAsync(bid, 0xFF, sizeof(unsigned long long) * static_cast<size_t>(n), c.stream) != cudaSuccess)
    return c.fail_cuda("swap reset");
  k_swap_pos<<<grid, 256, 0, c.stream>>>(dm, pos, n, ctrl);
  k_swap_rows_check<<<row_grid, 256, check_smem, c.stream>>>(dw, n, nullptr, n, kw, ctrl);
  c.launches += 2;
  rc = c.check_launch("k_swap_rows_check");
  // the women L ranks lowest go deepest: their rows whole from the start
  std::vector<int32_t> rows;
  rows.reserve(kSharedDeepRows);
  for (int r = std::max(0, n - kSharedDeepRows); r < n; ++r)
    if (static_cast<unsigned>(pref_m[r]) < static_cast<unsigned>(n)) rows.push_back(pref_m[r]);
  if (!rc) rc = send_rows(rows);
  if (!rc && cudaEventRecord(c.ev[kEvInvertEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc && cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc) rc = reset_queue();
  if (rc) return rc;
  k_swap_gs<<<c.sm_count * 4, 256, 0, c.stream>>>(dm, dw, pos, bid, n, ctrl, full, kw, over[0], nullptr, 0);
  c.launches++;
  rc = c.check_launch("k_swap_gs");
  for (int round = 0; !rc; ++round) {
    rc = read_control(c);
    if (!rc) rc = c.sync("women's proposals");
    if (rc || c.h_ctrl->status) break;
    const int stopped = c.h_ctrl->swap_over;
    if (stopped <= 0 || stopped > n) break;
    std::vector<int2> list(stopped);
    if (cudaMemcpy(list.data(), over[round & 1], sizeof(int2) * stopped, cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = c.fail_cuda("stopped women");
      break;
    }
    rows.clear();
    for (const int2 &e : list)
      if (static_cast<unsigned>(e.x) < static_cast<unsigned>(n)) rows.push_back(e.x);
    rc = send_rows(rows);
    if (!rc) rc = reset_queue();
    if (rc) break;
    k_swap_gs<<<std::max(1, std::min(c.sm_count * 4, (stopped + 7) / 8)), 256, 0, c.stream>>>(
        dm, dw, pos, bid, n, ctrl, full, kw, over[(round + 1) & 1], over[round & 1], stopped);
    c.launches++;
    rc = c.check_launch("k_swap_gs");
  }
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvBulkEnd], c.stream) != cudaSuccess ||
      cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess)
    return c.fail_cuda("event");
  if (!c.h_ctrl->status) {
    k_swap_match<<<grid, 256, 0, c.stream>>>(dm, bid, c.d_match.as<int32_t>(), n, ctrl);
    c.launches++;
    rc = c.check_launch("k_swap_match");
    if (!rc) rc = copy_match_out(c, match_out, (flags & SMP_F_DEVICE_PTRS) != 0);
  }
  if (!rc && cudaEventRecord(c.ev[kEvPostEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
  if (!rc) rc = read_control(c);
  if (!rc) rc = c.sync("solve");
  return rc;
}

int solve_streamed(Ctx &c, const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *match_out,
                   uint32_t flags, smp_stats *st) {
  const size_t row = sizeof(int32_t) * static_cast<size_t>(n);
  int rc = c.d_ctrl.ensure(sizeof(Control));
  if (!rc) rc = c.d_seen.ensure(((static_cast<size_t>(n) + 31) / 32) * 4);
  if (!rc) rc = c.d_pref_m.ensure(row * n);
  if (!rc) rc = c.d_pref_w.ensure(row * n);
  if (rc) return rc;
  if (!c.copy_stream) {
    if (cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking) != cudaSuccess)
      return c.fail_cuda("copy stream");
    for (auto &e : c.ev_chunk)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return c.fail_cuda("chunk event");
  }
  int32_t *dm = c.d_pref_m.as<int32_t>();
  int32_t *dw = c.d_pref_w.as<int32_t>();
  c.pref_m = dm;
  c.pref_w = dw;
  if (cudaEventRecord(c.ev[kEvStageBegin], c.stream) != cudaSuccess) return c.fail_cuda("event");
  if (cudaMemcpy2DAsync(dm, row, pref_m, row, sizeof(int32_t) * c.K, n, cudaMemcpyHostToDevice, c.stream) !=
      cudaSuccess)
    return c.fail_cuda("pref_m prefix copy");
  if (cudaEventRecord(c.ev[kEvStageEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  c.staged = true;
  rc = enqueue_precheck(c, (flags & SMP_F_NO_PRECHECK) == 0);
  if (!rc) rc = read_control(c);
  if (!rc) rc = c.sync("precheck");
  if (rc) return rc;
  c.phase = 1;
  if (c.h_ctrl->status) return control_status(c);
  const auto copy_rest_of_m = [&]() {
    return cudaMemcpy2DAsync(dm + c.K, row, pref_m + c.K, row, sizeof(int32_t) * (n - c.K), n,
                             cudaMemcpyHostToDevice, c.stream) == cudaSuccess
               ? SMP_OK
               : c.fail_cuda("pref_m copy");
  };
  const bool query = c.h_ctrl->mode == kModeQuery && !c.h_ctrl->perfect;
  if (!c.h_ctrl->perfect) c.known_mode = c.h_ctrl->mode;  // enqueue only this mode's kernels
  bool swapped = false;
  if (!query) {
    // One first choice for every man: perhaps one list for every man.  Then
    // the host threads compare every man's row with row 0 while pref_w
    // crosses the link, and only row 0 of pref_m follows it: the
    // women-proposing pass reads nothing else of it.
    const bool try_shared = !c.h_ctrl->perfect && c.h_ctrl->mode == kModeRank && c.h_ctrl->distinct == 1 &&
                            c.mode_cfg == 0 && swap_screen_smem(n) <= c.smem_optin;
    bool shared = false;
    if (!c.h_ctrl->perfect) {
      bool screened = false;  // the men's rows were compared on the host already
      if (try_shared && link_ready(c, false)) {
        // completes the solve when the men share one list
        rc = solve_shared_host(c, pref_m, pref_w, flags, match_out, shared);
        screened = true;
        swapped = !rc && shared;
      }
      if (!rc && !swapped) {
        if ((!try_shared || screened) && link_ready(c, true)) {
          // Both lists cross packed, pref_w first; each row group is widened
          // back to int32 on the device as it lands.
          const HostLink::Part parts[2] = {{pref_w, c.d_pw16.as<uint16_t>(), n},
                                           {pref_m, c.d_pm16.as<uint16_t>(), n}};
          rc = send_packed(c, parts, 2, kRankGroups, [&](int p, int r0, int r1) {
            return enqueue_widen16(c, p ? c.d_pm16.as<uint16_t>() : c.d_pw16.as<uint16_t>(), p ? dm : dw,
                                   static_cast<size_t>(r0) * n, static_cast<size_t>(r1) * n);
          });
        } else {
          if (cudaMemcpyAsync(dw, pref_w, row * n, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
            rc = c.fail_cuda("pref_w copy");
          if (!rc && try_shared && !screened) {
            if (cudaMemcpyAsync(dm + c.K, pref_m + c.K, sizeof(int32_t) * (n - c.K), cudaMemcpyHostToDevice,
                                c.stream) != cudaSuccess)
              rc = c.fail_cuda("pref_m row 0 copy");
            if (!rc) shared = host_rows_equal_row0(c, pref_m, n);
          }
          if (!rc && !shared) rc = copy_rest_of_m();
        }
      }
    }
    if (!rc && !swapped && cudaEventRecord(c.ev[kEvPrecheckEnd], c.stream) != cudaSuccess)
      rc = c.fail_cuda("event");
    if (!rc && shared && !swapped) rc = solve_swapped(c, flags, match_out, swapped, true);
    if (!rc && !swapped) rc = enqueue_init(c);
    if (!rc && !swapped && cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    if (!rc && !swapped) rc = enqueue_core(c);
  } else {
    if (cudaEventRecord(c.ev[kEvPrecheckEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
    rc = init_buffers(c);
    if (!rc) rc = enqueue_query_index(c);
    const bool packed = !rc && n <= kColorMaxN && link_ready(c, false);
    if (packed) {
      // pref_w crosses packed in row groups; each group's inversion waits
      // only for its own rows
      const HostLink::Part part = {pref_w, c.d_pw16.as<uint16_t>(), n};
      rc = send_packed(c, &part, 1, Ctx::kCopyChunks,
                       [&](int, int r0, int r1) { return enqueue_qinvert16(c, r0, r1); });
    }
    for (int k = 0; !rc && !packed && k < Ctx::kCopyChunks; ++k) {
      const int r0 = static_cast<int>(static_cast<int64_t>(n) * k / Ctx::kCopyChunks);
      const int r1 = static_cast<int>(static_cast<int64_t>(n) * (k + 1) / Ctx::kCopyChunks);
      if (r0 == r1) continue;
      const size_t off = static_cast<size_t>(r0) * n;
      if (cudaMemcpyAsync(dw + off, pref_w + off, row * (r1 - r0), cudaMemcpyHostToDevice, c.copy_stream) !=
              cudaSuccess ||
          cudaEventRecord(c.ev_chunk[k], c.copy_stream) != cudaSuccess ||
          cudaStreamWaitEvent(c.stream, c.ev_chunk[k], 0) != cudaSuccess) {
        rc = c.fail_cuda("pref_w chunk copy");
        break;
      }
      rc = enqueue_qinvert(c, r0, r1);
    }
    if (!rc && cudaEventRecord(c.ev[kEvInvertEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    if (!rc && cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    c.tail_ran = true;
    if (!rc) rc = enqueue_round<uint16_t>(c, 0);
    if (!rc) rc = read_control(c);
    if (!rc) rc = c.sync("round 0");
    if (!rc && c.h_ctrl->retry && !c.h_ctrl->status) {
      c.known_mode = -1;
      rc = copy_rest_of_m();
      // the rank-mode retry inverts int32 rows: widen the packed ones
      if (!rc && packed)
        rc = enqueue_widen16(c, c.d_pw16.as<uint16_t>(), dw, 0, static_cast<size_t>(n) * n);
      if (!rc) rc = enqueue_retry_round<uint16_t>(c);
    }
  }
  if (!swapped) {  // the women-proposing pass has finished its solve
    if (!rc && cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    if (!rc) rc = enqueue_post(c);
    if (!rc && cudaEventRecord(c.ev[kEvPostEnd], c.stream) != cudaSuccess) rc = c.fail_cuda("event");
    if (!rc) rc = copy_match_out(c, match_out, false);
    if (!rc) rc = read_control(c);
  }
  // Both streams drain before returning, even after an error: the copies
  // read the caller's buffers.
  const int rs = c.sync("solve");
  if (cudaStreamSynchronize(c.copy_stream) != cudaSuccess && !rc && !rs) rc = c.fail_cuda("copy stream");
  if (rc) return rc;
  if (rs) return rs;
  return solve_finish(c, flags, st);
}

}  // namespace smpb200

// ===========================================================================
// Public ABI
// ===========================================================================
extern "C" {

const char *smp_b200_version(void) { return "smp_b200 0.1 (sm_100a)"; }

const char *smp_b200_strerror(int status) {
  switch (status) {
    case SMP_OK: return "ok";
    case SMP_ERR_INVALID_ARG: return "invalid argument";
    case SMP_ERR_INVALID_INPUT: return "invalid input: a preference row is not a permutation of 0..n-1";
    case SMP_ERR_OOM: return "out of device or pinned memory";
    case SMP_ERR_CUDA: return "CUDA error";
    case SMP_ERR_TIMEOUT: return "timed out (reserved: no call returns it)";
    case SMP_ERR_BUSY: return "no slot or HBM budget free";
    case SMP_ERR_NOT_READY: return "not finished yet";
    case SMP_ERR_UNSUPPORTED: return "unsupported request";
    case SMP_ERR_IO: return "a workload file could not be read or written";
    default: return "unknown status";
  }
}

const char *smp_b200_last_error(const smp_ctx *ctx) { return ctx ? ctx->c.last_error.c_str() : ""; }

int smp_b200_create(smp_ctx **out, const smp_cfg *cfg) {
  if (!out) return SMP_ERR_INVALID_ARG;
  *out = nullptr;
  smp_ctx *ctx = new (std::nothrow) smp_ctx();
  if (!ctx) return SMP_ERR_OOM;
  Ctx &c = ctx->c;
  if (cfg) {
    c.device = cfg->device;
    c.prefix_k_cfg = cfg->prefix_k;
    c.tail_threshold_cfg = cfg->tail_threshold;
    c.bulk_window_cfg = cfg->bulk_window;
    c.tail_window_cfg = cfg->tail_window;
    c.mode_cfg = cfg->mode;
    c.rank_bytes_cfg = cfg->rank_bytes;
    if (cfg->hbm_budget) c.hbm_budget = cfg->hbm_budget;
    if (cfg->rank_bytes != 0 && cfg->rank_bytes != 4) {
      delete ctx;
      return SMP_ERR_INVALID_ARG;
    }
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || c.device < 0 || c.device >= count) {
    cudaGetLastError();
    delete ctx;
    return SMP_ERR_CUDA;
  }
  DeviceGuard g(c.device);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, c.device) != cudaSuccess) {
    delete ctx;
    return SMP_ERR_CUDA;
  }
  c.sm_count = prop.multiProcessorCount;
  c.smem_optin = prop.sharedMemPerBlockOptin;
  if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return SMP_ERR_CUDA;
  }
  if (cudaMemPool_t pool = device_pool(c.device))
    for (DeviceBuf *b : c.buffers()) b->bind(pool, c.stream);
  for (auto &e : c.ev) {
    if (cudaEventCreate(&e) != cudaSuccess) {
      smp_b200_destroy(ctx);
      return SMP_ERR_CUDA;
    }
  }
  if (cudaMallocHost(reinterpret_cast<void **>(&c.h_ctrl), sizeof(Control)) != cudaSuccess) {
    cudaGetLastError();
    smp_b200_destroy(ctx);
    return SMP_ERR_OOM;
  }
  std::memset(c.h_ctrl, 0, sizeof(Control));
  *out = ctx;
  return SMP_OK;
}

void smp_b200_destroy(smp_ctx *ctx) {
  if (!ctx) return;
  Ctx &c = ctx->c;
  {
    DeviceGuard g(c.device);
    if (c.copy_stream) cudaStreamSynchronize(c.copy_stream);
    if (c.stream) cudaStreamSynchronize(c.stream);
    for (DeviceBuf *b : c.buffers()) b->release();
    if (c.stream) cudaStreamSynchronize(c.stream);
    trim_device_pool(c.device);
    for (auto &e : c.ev)
      if (e) cudaEventDestroy(e);
    for (auto &e : c.ev_chunk)
      if (e) cudaEventDestroy(e);
    if (c.copy_stream) cudaStreamDestroy(c.copy_stream);
    if (c.h_ctrl) cudaFreeHost(c.h_ctrl);
    c.link.reset();
    c.pack_pool.reset();
    if (c.stream) cudaStreamDestroy(c.stream);
  }
  delete ctx;
}

int smp_b200_stage(smp_ctx *ctx, const int32_t *pref_m, const int32_t *pref_w, int32_t n, uint32_t flags) {
  if (!valid_ctx(ctx)) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  int rc = do_stage(c, pref_m, pref_w, n, flags);
  if (rc) return rc;
  rc = c.sync("stage");
  if (rc) return rc;
  c.stats.stage_ms = elapsed(c, kEvStageBegin, kEvStageEnd);
  return SMP_OK;
}

int smp_b200_precheck(smp_ctx *ctx, int32_t *is_perfect) {
  if (!valid_ctx(ctx) || !ctx->c.staged) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  if (cudaEventRecord(c.ev[kEvStageEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  int rc = enqueue_precheck(c, true);
  if (!rc) rc = read_control(c);
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvPrecheckEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  rc = c.sync("precheck");
  if (rc) return rc;
  c.phase = 1;
  c.stats.precheck_ms = elapsed(c, kEvStageEnd, kEvPrecheckEnd);
  if (is_perfect) *is_perfect = c.h_ctrl->perfect;
  return control_status(c);
}

int smp_b200_init(smp_ctx *ctx) {
  if (!valid_ctx(ctx) || ctx->c.phase < 1) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  if (cudaEventRecord(c.ev[kEvPrecheckEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  int rc = enqueue_init(c);
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  rc = read_control(c);
  if (!rc) rc = c.sync("init");
  if (rc) return rc;
  c.phase = 2;
  c.stats.init_ms = elapsed(c, kEvPrecheckEnd, kEvInitEnd);
  return control_status(c);
}

int smp_b200_core(smp_ctx *ctx) {
  if (!valid_ctx(ctx) || ctx->c.phase < 2) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  if (cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  int rc = enqueue_core(c);
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  rc = read_control(c);
  if (!rc) rc = c.sync("core");
  if (rc) return rc;
  c.phase = 3;
  c.stats.core_ms = elapsed(c, kEvInitEnd, kEvCoreEnd);
  return control_status(c);
}

int smp_b200_post(smp_ctx *ctx, int32_t *match_out, uint32_t flags) {
  if (!valid_ctx(ctx) || !match_out || ctx->c.phase < 1) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  if (c.phase < 3) {
    // Precheck found the first choices distinct: the bulk and tail phases
    // were skipped (AbsSmpEngine skips InitProc/CoreProc, smp_engine_abs.h:16-33).
    if (!c.h_ctrl->perfect) return SMP_ERR_INVALID_ARG;
    c.tail_ran = false;
    int rc = c.d_match.ensure(sizeof(int32_t) * static_cast<size_t>(c.n));
    if (!rc) rc = c.d_bid.ensure(sizeof(unsigned long long) * static_cast<size_t>(c.n));
    if (rc) return rc;
  }
  if (cudaEventRecord(c.ev[kEvCoreEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  int rc = enqueue_post(c);
  if (!rc) rc = copy_match_out(c, match_out, (flags & SMP_F_DEVICE_PTRS) != 0);
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvPostEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  rc = read_control(c);
  if (!rc) rc = c.sync("post");
  if (rc) return rc;
  c.stats.post_ms = elapsed(c, kEvCoreEnd, kEvPostEnd);
  fill_stats(c, false);
  c.phase = 4;
  c.stats.total_ms = c.stats.precheck_ms + c.stats.init_ms + c.stats.core_ms + c.stats.post_ms;
  return control_status(c);
}

int smp_b200_stats(const smp_ctx *ctx, smp_stats *st) {
  if (!valid_ctx(ctx) || !st) return SMP_ERR_INVALID_ARG;
  *st = ctx->c.stats;
  return SMP_OK;
}

int smp_b200_solve(smp_ctx *ctx, const int32_t *pref_m, const int32_t *pref_w, int32_t n, int32_t *match_out,
                   uint32_t flags, smp_stats *st) {
  if (!valid_ctx(ctx) || !match_out) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  if (!(flags & SMP_F_DEVICE_PTRS) && pref_m && pref_w && n > 0 && n <= SMP_B200_MAX_N) {
    // The host-pointer solve moves only what it reads, overlapped with work.
    c.n = n;
    plan(c);
    if (smpb200::streamed_fits(c, flags)) {
      const int rc = stage_reset(c, n);
      return rc ? rc : smpb200::solve_streamed(c, pref_m, pref_w, n, match_out, flags, st);
    }
  }
  return smpb200::solve_staged(c, pref_m, pref_w, n, match_out, flags, st);
}

int smp_b200_invert(smp_ctx *ctx, const int32_t *pref_w, int32_t n, int32_t *rank_out, uint32_t flags) {
  if (!valid_ctx(ctx) || !pref_w || !rank_out || n <= 0 || n > SMP_B200_MAX_N) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  c.n = n;
  c.phase = 0;
  c.staged = false;
  c.rank_valid = false;
  const size_t bytes = sizeof(int32_t) * static_cast<size_t>(n) * n;
  int rc = c.d_ctrl.ensure(sizeof(Control));
  if (rc) return rc;
  const int32_t *src = pref_w;
  int32_t *dst = rank_out;
  if (!(flags & SMP_F_DEVICE_PTRS)) {
    rc = c.d_pref_w.ensure(bytes);
    if (!rc) rc = c.d_rank.ensure(bytes);
    if (rc) return rc;
    if (cudaMemcpyAsync(c.d_pref_w.ptr, pref_w, bytes, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
      return c.fail_cuda("pref_w copy");
    src = c.d_pref_w.as<int32_t>();
    dst = c.d_rank.as<int32_t>();
  }
  if (cudaMemsetAsync(c.d_ctrl.ptr, 0, sizeof(Control), c.stream) != cudaSuccess) return c.fail_cuda("control reset");
  if (cudaEventRecord(c.ev[kEvPrecheckEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  rc = enqueue_invert<int32_t>(c, src, dst, kGateAlways);
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvInitEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  if (!(flags & SMP_F_DEVICE_PTRS)) {
    if (cudaMemcpyAsync(rank_out, dst, bytes, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
      return c.fail_cuda("rank copy");
  }
  rc = read_control(c);
  if (!rc) rc = c.sync("invert");
  if (rc) return rc;
  c.stats = smp_stats{};
  c.stats.n = n;
  c.stats.blocking_pairs = -1;
  c.stats.rank_bytes = 4;
  c.stats.init_ms = elapsed(c, kEvPrecheckEnd, kEvInitEnd);
  return control_status(c);
}

int smp_b200_check(smp_ctx *ctx, const int32_t *pref_m, const int32_t *pref_w, int32_t n, const int32_t *match,
                   uint32_t flags, int64_t *blocking_pairs, int64_t *proposals) {
  if (!valid_ctx(ctx) || !match) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  int rc = do_stage(c, pref_m, pref_w, n, flags);
  if (rc) return rc;
  const int32_t *dmatch = match;
  if (!(flags & SMP_F_DEVICE_PTRS)) {
    rc = c.d_match.ensure(sizeof(int32_t) * static_cast<size_t>(n));
    if (rc) return rc;
    if (cudaMemcpyAsync(c.d_match.ptr, match, sizeof(int32_t) * static_cast<size_t>(n), cudaMemcpyHostToDevice,
                        c.stream) != cudaSuccess)
      return c.fail_cuda("match copy");
    dmatch = c.d_match.as<int32_t>();
  }
  rc = enqueue_precheck(c, false);
  if (rc) return rc;
  c.rank_bytes = c.rank_bytes_cfg == 4 ? 4 : rank_bytes_for(n);
  rc = c.d_rank.ensure(static_cast<size_t>(n) * n * c.rank_bytes);
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvCheckBegin], c.stream) != cudaSuccess) return c.fail_cuda("event");
  rc = enqueue_invert_any(c, kGateAlways);
  if (!rc) rc = enqueue_check(c, dmatch);
  if (rc) return rc;
  if (cudaEventRecord(c.ev[kEvCheckEnd], c.stream) != cudaSuccess) return c.fail_cuda("event");
  rc = read_control(c);
  if (!rc) rc = c.sync("check");
  if (rc) return rc;
  c.stats.check_ms = elapsed(c, kEvCheckBegin, kEvCheckEnd);
  const int s = control_status(c);
  if (blocking_pairs) *blocking_pairs = s == 0 ? static_cast<int64_t>(c.h_ctrl->blocking) : -1;
  if (proposals) *proposals = static_cast<int64_t>(c.h_ctrl->check_proposals);
  c.phase = 0;
  return s;
}

int smp_b200_generate(smp_ctx *ctx, int32_t kind, int32_t n, uint64_t seed, uint32_t salt, int32_t param,
                      int32_t *pref_m, int32_t *pref_w, uint32_t flags) {
  if (!valid_ctx(ctx) || !pref_m || !pref_w || n <= 0 || n > SMP_B200_MAX_N) return SMP_ERR_INVALID_ARG;
  if (kind < SMP_GEN_UNIFORM || kind > SMP_GEN_SOLO) return SMP_ERR_INVALID_ARG;
  if (kind == SMP_GEN_CORRELATED && (param < 0 || param > 10000)) return SMP_ERR_INVALID_ARG;
  if (kind == SMP_GEN_GROUPED && param <= 0) return SMP_ERR_INVALID_ARG;
  if (kind == SMP_GEN_SOLO && n < 3) return SMP_ERR_INVALID_ARG;
  Ctx &c = ctx->c;
  DeviceGuard g(c.device);
  const size_t bytes = sizeof(int32_t) * static_cast<size_t>(n) * n;
  int32_t *dm = pref_m, *dw = pref_w;
  if (!(flags & SMP_F_DEVICE_PTRS)) {
    int rc = c.d_pref_m.ensure(bytes);
    if (!rc) rc = c.d_pref_w.ensure(bytes);
    if (rc) return rc;
    dm = c.d_pref_m.as<int32_t>();
    dw = c.d_pref_w.as<int32_t>();
  }
  int rc = generate_side(c, kind, 0, n, seed, salt, param, dm);
  if (!rc) rc = generate_side(c, kind, 1, n, seed, salt, param, dw);
  if (rc) return rc;
  if (!(flags & SMP_F_DEVICE_PTRS)) {
    if (cudaMemcpyAsync(pref_m, dm, bytes, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
      return c.fail_cuda("pref_m copy");
    if (cudaMemcpyAsync(pref_w, dw, bytes, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess)
      return c.fail_cuda("pref_w copy");
  }
  c.staged = false;
  c.phase = 0;
  return c.sync("generate");
}

}  // extern "C"
