// step.cuh -- one proposal step of a man (load a window of his choices,
// settle rejections by reading bids, propose to the first candidate), shared
// by the single-instance bulk and tail kernels and the batch kernel.  Only
// inline device code and templates live here, so several translation units
// may include it.
#pragma once

#include "common.cuh"

namespace smpb200 {

// ---------------------------------------------------------------------------
// One choice of a man: his r-th woman and her rank of him, in two halves so
// that the first load can be issued early (see Ahead below).
// issue_choice: the raw word -- the packed prefix entry for r < K, else the
// woman from pref_m (rank mode), else nothing.
// finish_choice: decodes it (and reads the rank in rank mode).
//   0  ok
//   1  beyond the prefix while in query mode (rank unknown)
//   2  out-of-range woman (reported by the caller)
//   3  past the end of the list
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t issue_choice(const int32_t *__restrict__ pref_m,
                                                 const uint32_t *__restrict__ prefix, int K, int n, bool query,
                                                 int m, int r) {
  if (r >= n) return 0u;
  if (r < K) return __ldg(prefix + static_cast<size_t>(m) * K + r);
  if (query) return 0u;
  return static_cast<uint32_t>(__ldg(pref_m + static_cast<size_t>(m) * n + r));
}

// kLdg: the rank matrix is in global memory and read through the read-only
// path; false when it may be in shared memory (the batch kernel).
// kManMajor, the layout of the matrix a rank is read from:
//   0 (false)  woman-major, rank[w][m] = her rank of him;
//   1 (true)   man-major, rank[m][w], so a man's scan stays within his row;
//   2          by position, pr[m][r] = the rank of man m in the list of his
//              r-th choice: read at the index of his pref_m entry, so its
//              load does not wait for that one;
//   3          one rank per proposer, rank[m]: every receiver ranks the
//              proposers the same way (a batch instance solved with the
//              roles swapped because all men share one list).
template <bool kLdg = true, int kManMajor = 0, typename RankT>
__device__ __forceinline__ int finish_choice(uint32_t raw, const RankT *__restrict__ rank, int K, int n, bool query,
                                             int m, int r, int &w, uint32_t &rk) {
  if (r >= n) return 3;
  if (r < K) {
    w = static_cast<int>(raw >> 16);
    rk = raw & 0xFFFFu;
    return raw == 0xFFFFFFFFu ? 2 : 0;
  }
  if (query) return 1;
  w = static_cast<int>(raw);
  if (static_cast<unsigned>(w) >= static_cast<unsigned>(n)) return 2;
  const RankT *p = kManMajor == 3   ? rank + m
                   : kManMajor == 2 ? rank + static_cast<size_t>(m) * n + r
                   : kManMajor == 1 ? rank + static_cast<size_t>(m) * n + w
                                    : rank + static_cast<size_t>(w) * n + m;
  rk = static_cast<uint32_t>(kLdg ? __ldg(p) : *p);
  return 0;
}

template <bool kLdg = true, int kManMajor = 0, typename RankT>
__device__ __forceinline__ int load_choice(const int32_t *__restrict__ pref_m, const RankT *__restrict__ rank,
                                           const uint32_t *__restrict__ prefix, int K, int n, bool query, int m,
                                           int r, int &w, uint32_t &rk) {
  return finish_choice<kLdg, kManMajor>(issue_choice(pref_m, prefix, K, n, query, m, r), rank, K, n, query, m, r, w,
                                        rk);
}

// The window of the man a warp will carry next, loaded before it is known
// for certain.  When a warp picks its candidate, the bid word it read names
// the man who will be displaced and (directly, or through his stored
// position) where he resumes; his first window is issued then, so its load
// overlaps the atomic that confirms him.  man_step uses it only when the
// atomic displaced exactly that man at exactly that position; otherwise it is
// ignored and the window is loaded again, so a stale guess costs time only.
struct Ahead {
  int m = -1;        // whose window (warp-uniform); -1: none
  int pos = 0;       // its first position
  uint32_t raw = 0;  // this lane's issue_choice word
};

// ---------------------------------------------------------------------------
// One proposal step of a man, shared by the bulk, tail and batch kernels.
//
// A warp looks at the man's next S windows of 32 choices (S = 1 for a man
// just taken up, doubling up to kMaxSub while whole windows reject him).
// Every woman whose current partner she ranks above him would reject him, so
// those proposals are settled by one read of her bid; for the first remaining
// candidate the warp proposes with an atomicMin.  The common case -- accepted
// within the first window -- runs a tight single-window path; the wide path
// (S > 1) is only entered while galloping through a deep list, and after a
// lost race it moves on to the windows it already loaded.
//
// Bid storage is a policy: GlobalBids (64-bit words in HBM, the all-SM bulk
// kernel) or SharedBids (rank << 16 | man words and 2-byte positions in
// shared memory, one CTA).
// ---------------------------------------------------------------------------
constexpr int kStepMoved = 0;        // settled proposals; m / pos / S updated
constexpr int kStepMatchedFree = 1;  // accepted by a free woman: m = -1
constexpr int kStepBad = 2;          // invalid input (value in bad_value)
constexpr int kStepBeyond = 3;       // query mode: next choice beyond the prefix
constexpr int kStepHalt = 4;         // the caller's check asked to stop

struct GlobalBids {
  using Word = unsigned long long;
  static constexpr bool kFiltered = false;
  unsigned long long *bid;
  __device__ __forceinline__ Word word(int w) const { return ld_relaxed_u64(bid + w); }
  __device__ __forceinline__ static uint32_t rank_of(Word b) { return bid_rank(b); }
  __device__ __forceinline__ uint32_t cur_rank(int w) const { return bid_rank(ld_relaxed_u64(bid + w)); }
  // The man a bid word holds and where he would resume; false if free.
  __device__ __forceinline__ bool holder(Word b, int &hm, int &hp) const {
    if (b == kFree) return false;
    hm = static_cast<int>(bid_man(b));
    hp = static_cast<int>(bid_pos(b)) + 1;
    return true;
  }
  // Returns the replaced word if accepted, else 0 (an accepted word's rank is
  // above the proposer's, so it is never 0).
  __device__ __forceinline__ unsigned long long propose(int w, uint32_t rk, int m, int pos) const {
    const unsigned long long old =
        atomicMin(bid + w, pack_bid(rk, static_cast<uint32_t>(m), static_cast<uint32_t>(pos)));
    return bid_rank(old) > rk ? old : 0ull;
  }
  // true if she was free; else the displaced man and where he resumes
  __device__ __forceinline__ bool decode(unsigned long long res, int &m, int &pos) const {
    if (res == kFree) return true;
    m = static_cast<int>(bid_man(res));
    pos = static_cast<int>(bid_pos(res)) + 1;
    return false;
  }
};

struct SharedBids {
  using Word = uint32_t;
  static constexpr bool kFiltered = false;
  uint32_t *sbid;  // rank << 16 | man; 0xFFFFFFFF = free
  uint16_t *spos;  // each man's position of his current proposal
  __device__ __forceinline__ Word word(int w) const { return lds_relaxed_u32(sbid + w); }
  __device__ __forceinline__ static uint32_t rank_of(Word b) { return b >> 16; }
  __device__ __forceinline__ uint32_t cur_rank(int w) const { return lds_relaxed_u32(sbid + w) >> 16; }
  // The position read here is a guess (no ordering with the store that
  // published it); man_step checks it against the atomic's result.
  __device__ __forceinline__ bool holder(Word b, int &hm, int &hp) const {
    if (b == 0xFFFFFFFFu) return false;
    hm = static_cast<int>(b & 0xFFFFu);
    hp = static_cast<int>(spos[hm]) + 1;
    return true;
  }
  // The position is written before the atomic publishes the man; the
  // displaced man's position is read after it (a stale read is safe, see
  // atom_min_relaxed_shared).
  __device__ __forceinline__ unsigned long long propose(int w, uint32_t rk, int m, int pos) const {
    spos[m] = static_cast<uint16_t>(pos);
    const uint32_t old = atom_min_relaxed_shared(sbid + w, (rk << 16) | static_cast<uint32_t>(m));
    if ((old >> 16) <= rk) return 0ull;
    const uint32_t np = old != 0xFFFFFFFFu ? spos[old & 0xFFFFu] + 1u : 0u;
    return (static_cast<unsigned long long>(np) << 32) | old;
  }
  __device__ __forceinline__ bool decode(unsigned long long res, int &m, int &pos) const {
    const uint32_t old = static_cast<uint32_t>(res);
    if (old == 0xFFFFFFFFu) return true;
    m = static_cast<int>(old & 0xFFFFu);
    pos = static_cast<int>(res >> 32);
    return false;
  }
};

// GlobalBids behind a per-CTA filter in shared memory: lrank[w] is an upper
// bound on the rank of woman w's partner (all ones while unknown).  Every
// value written to it is a rank her partner had or a rank a proposal to her
// claimed, and her partner only ever improves, so it stays an upper bound
// even when two warps race on it (a lost update only loosens it): plain
// volatile loads and stores suffice.  A man she ranks above lrank[w] is
// rejected without touching L2 (check); every bid word the CTA reads lowers
// the bound (learn); a proposal first claims her locally, so only a warp that
// beats every rank its CTA knows for her sends the global atomic.  Where the
// men of many warps scan the same women (congested and correlated lists),
// this turns one L2 read per proposal into about one per woman and CTA, and
// the convoy of losing atomics on the first free woman into a few.
struct FilteredBids {
  using Word = unsigned long long;
  static constexpr bool kFiltered = true;
  unsigned long long *bid;
  volatile uint32_t *lrank;
  __device__ __forceinline__ Word word(int w) const { return ld_relaxed_u64(bid + w); }
  __device__ __forceinline__ static uint32_t rank_of(Word b) { return bid_rank(b); }
  __device__ __forceinline__ uint32_t cur_rank(int w) const { return bid_rank(ld_relaxed_u64(bid + w)); }
  // No side effects, so the loads of several windows can be in flight at once.
  __device__ __forceinline__ bool check(int w, uint32_t rk, Word &cw) const {
    if (rk > lrank[w]) {
      cw = kFree;
      return false;
    }
    cw = __ldcg(bid + w);
    return rk < bid_rank(cw);
  }
  __device__ __forceinline__ void learn(int w, Word cw) const {
    const uint32_t r = bid_rank(cw);
    if (r < lrank[w]) lrank[w] = r;
  }
  __device__ __forceinline__ bool holder(Word b, int &hm, int &hp) const {
    if (b == kFree) return false;
    hm = static_cast<int>(bid_man(b));
    hp = static_cast<int>(bid_pos(b)) + 1;
    return true;
  }
  __device__ __forceinline__ unsigned long long propose(int w, uint32_t rk, int m, int pos) const {
    if (lrank[w] < rk) return 0ull;  // her partner is better than him already
    lrank[w] = rk;
    const unsigned long long old =
        atomicMin(bid + w, pack_bid(rk, static_cast<uint32_t>(m), static_cast<uint32_t>(pos)));
    if (bid_rank(old) > rk) return old;
    learn(w, old);
    return 0ull;
  }
  __device__ __forceinline__ bool decode(unsigned long long res, int &m, int &pos) const {
    if (res == kFree) return true;
    m = static_cast<int>(bid_man(res));
    pos = static_cast<int>(bid_pos(res)) + 1;
    return false;
  }
};

// Candidates of one window (cm), stopped by the first bad / beyond lane (em).
// Returns kStepMoved / kStepMatchedFree with the acceptance lane in j_acc,
// kStepBad / kStepBeyond for a stop, or -1 if the window rejected him.
template <typename Bids>
__device__ __forceinline__ int try_window(const Bids &bids, int lane, int w, uint32_t rk, int st, unsigned cm,
                                          unsigned em, int m, int base, int &new_m, int &new_pos, int &j_acc,
                                          int &bad_value) {
  if (em) cm &= (1u << (__ffs(em) - 1)) - 1u;
  while (cm) {
    const int j = __ffs(cm) - 1;
    unsigned long long res = 0ull;
    if (lane == j) res = bids.propose(w, rk, m, base + j);
    res = __shfl_sync(kFullMask, res, j);
    if (res) {
      j_acc = j;
      return bids.decode(res, new_m, new_pos) ? kStepMatchedFree : kStepMoved;
    }
    cm &= cm - 1;  // someone better got there first
  }
  if (em) {
    const int e = __ffs(em) - 1;
    const int ste = __shfl_sync(kFullMask, st, e);
    bad_value = __shfl_sync(kFullMask, w, e);
    return ste == 2 ? kStepBad : kStepBeyond;
  }
  return -1;
}

// kSReset: the look-ahead (in windows) a man starts with after a move; 1 for
// chains that end within a few choices, kMaxSub where displaced men scan deep.
template <int kMaxSub, bool kAhead = true, bool kLdg = true, int kSReset = 1, int kManMajor = 0,
          typename RankT, typename Bids, typename Check>
__device__ __forceinline__ int man_step(const Bids &bids, Check keep_going, const int32_t *__restrict__ pref_m,
                                        const RankT *__restrict__ rank, const uint32_t *__restrict__ prefix, int K,
                                        int n, bool query, int lane, int &m, int &pos, int &S, Ahead &ahead,
                                        unsigned long long &settled, unsigned int &hops, int &bad_value) {
  int nm = -1, np = 0, j = 0;
  if (kMaxSub == 1 || S == 1) {
    int w0 = 0;
    uint32_t rk0 = 0xFFFFFFFFu;
    const int r = pos + lane;
    const uint32_t raw =
        (kAhead && ahead.m == m && ahead.pos == pos) ? ahead.raw : issue_choice(pref_m, prefix, K, n, query, m, r);
    if (kAhead) ahead.m = -1;
    const int st0 = finish_choice<kLdg, kManMajor>(raw, rank, K, n, query, m, r, w0, rk0);
    typename Bids::Word cw = 0;
    unsigned cm;
    if constexpr (Bids::kFiltered) {
      bool cand = false;
      if (st0 == 0) cand = bids.check(w0, rk0, cw);
      if (!keep_going()) return kStepHalt;
      cm = __ballot_sync(kFullMask, cand);
      if (st0 == 0) bids.learn(w0, cw);
    } else {
      uint32_t cr = 0u;
      if (st0 == 0) {
        cw = bids.word(w0);
        cr = Bids::rank_of(cw);
      }
      if (!keep_going()) return kStepHalt;
      cm = __ballot_sync(kFullMask, st0 == 0 && rk0 < cr);
    }
    const unsigned em = (pos + 32 > K) ? __ballot_sync(kFullMask, st0 == 1 || st0 == 2) : 0u;
    if (em) cm &= (1u << (__ffs(em) - 1)) - 1u;
    // Issue the window of the man the first candidate would displace.
    Ahead next;
    if (kAhead && cm) {
      const typename Bids::Word hw = __shfl_sync(kFullMask, cw, __ffs(cm) - 1);
      int hm = 0, hp = 0;
      if (bids.holder(hw, hm, hp)) {
        next.m = hm;
        next.pos = hp;
        next.raw = issue_choice(pref_m, prefix, K, n, query, hm, hp + lane);
      }
    }
    const int rc = try_window(bids, lane, w0, rk0, st0, cm, em, m, pos, nm, np, j, bad_value);
    if (rc == kStepMoved || rc == kStepMatchedFree) {
      settled += j + 1;
      hops++;
      m = rc == kStepMatchedFree ? -1 : nm;
      pos = np;
      S = kSReset;
      if (kAhead && rc == kStepMoved && next.m == nm && next.pos == np) ahead = next;
      return rc;
    }
    if (rc >= 0) return rc;
    settled += min(32, n - pos);
    pos += 32;
    if (pos >= n) {  // rejected by every woman: the lists are not permutations
      bad_value = m;
      return kStepBad;
    }
    S = min(2, kMaxSub);
    return kStepMoved;
  }
  // wide path
  int w[kMaxSub], st[kMaxSub];
  uint32_t rk[kMaxSub], cr[kMaxSub];
  bool cd[kMaxSub];  // FilteredBids: candidate
  if constexpr (Bids::kFiltered) {
    typename Bids::Word cws[kMaxSub];
#pragma unroll
    for (int s = 0; s < kMaxSub; ++s) {
      st[s] = 3;
      w[s] = 0;
      rk[s] = 0xFFFFFFFFu;
      cd[s] = false;
      cws[s] = 0;
      if (s < S) {
        const int r = pos + 32 * s + lane;
        if (r < n) {
          st[s] = load_choice<kLdg, kManMajor>(pref_m, rank, prefix, K, n, query, m, r, w[s], rk[s]);
          if (st[s] == 0) cd[s] = bids.check(w[s], rk[s], cws[s]);
        }
      }
    }
#pragma unroll
    for (int s = 0; s < kMaxSub; ++s)
      if (st[s] == 0) bids.learn(w[s], cws[s]);
  } else {
#pragma unroll
    for (int s = 0; s < kMaxSub; ++s) {
      st[s] = 3;
      w[s] = 0;
      rk[s] = 0xFFFFFFFFu;
      cr[s] = 0u;
      if (s < S) {
        const int r = pos + 32 * s + lane;
        if (r < n) {
          st[s] = load_choice<kLdg, kManMajor>(pref_m, rank, prefix, K, n, query, m, r, w[s], rk[s]);
          if (st[s] == 0) cr[s] = bids.cur_rank(w[s]);
        }
      }
    }
  }
  if (!keep_going()) return kStepHalt;
  const bool edge = pos + 32 * S > K;
  unsigned cm[kMaxSub], em[kMaxSub];
#pragma unroll
  for (int s = 0; s < kMaxSub; ++s) {
    cm[s] = 0u;
    em[s] = 0u;
    if (s < S) {
      cm[s] = __ballot_sync(kFullMask, Bids::kFiltered ? cd[s] : (st[s] == 0 && rk[s] < cr[s]));
      if (edge) em[s] = __ballot_sync(kFullMask, st[s] == 1 || st[s] == 2);
    }
  }
  for (int s0 = 0; s0 < S;) {
    int sstar = -1;
#pragma unroll
    for (int s = 0; s < kMaxSub; ++s)
      if (sstar < 0 && s >= s0 && s < S && (cm[s] | em[s])) sstar = s;
    if (sstar < 0) break;
    int ws = 0, sts = 3;
    uint32_t rks = 0xFFFFFFFFu;
    unsigned cms = 0u, ems = 0u;
#pragma unroll
    for (int s = 0; s < kMaxSub; ++s) {
      if (s == sstar) {
        ws = w[s];
        rks = rk[s];
        sts = st[s];
        cms = cm[s];
        ems = em[s];
      }
    }
    const int rc = try_window(bids, lane, ws, rks, sts, cms, ems, m, pos + 32 * sstar, nm, np, j, bad_value);
    if (rc == kStepMoved || rc == kStepMatchedFree) {
      settled += 32 * sstar + j + 1;
      hops++;
      m = rc == kStepMatchedFree ? -1 : nm;
      pos = np;
      S = kSReset;
      return rc;
    }
    if (rc >= 0) return rc;
    s0 = sstar + 1;
  }
  settled += min(32 * S, n - pos);
  pos += 32 * S;
  if (pos >= n) {
    bad_value = m;
    return kStepBad;
  }
  S = min(2 * S, kMaxSub);
  return kStepMoved;
}

}  // namespace smpb200
