// generate.cu -- seeded workload generator on the GPU.
//
// Recipe (shared with the CPU oracle, which restates it independently).
// Every row of a preference side (side 0 = men, 1 = women) is produced by
// giving each candidate column j a 64-bit key whose low 20 bits are j (so the
// keys of a row are distinct), sorting the keys ascending, and keeping the
// low 20 bits.  Keys are drawn from Philox4x32-10 with key (seed low 32 bits,
// seed high 32 bits) and counter (j, row, side << 8 | tag, salt); the row
// word is 0xFFFFFFFF for a side's shared draws.
//
//   UNIFORM      key = out[0] << 20 | j                            (tag 0)
//   CONGESTED    men: one UNIFORM-style row (tag 5, shared) copied to every
//                man; women: UNIFORM
//   CORRELATED   score[j] = out[0] of (j, shared, tag 1); noise = Irwin-Hall
//                sum of the 12 words of tags 2, 3, 4 (each >> 8), centred at
//                6 * 2^24, times 256 * sigma_e4 / 10000 (integer, truncating);
//                key = (2^36 - score - noise) << 20 | j  (higher total first)
//   PERFECT      first = shared UNIFORM row (tag 6); key = 0 for j = first[row],
//                else ((out[0] of tag 7) >> 1) + 1) << 20 | j
//                (include/utils/generate_workloads_flat.h:50-82)
//   REF_CONGESTED one shared UNIFORM-style row (tag 11) on every row, both
//                sides (generate_workloads_flat.h:14-47)
//   GROUPED      ids = shared UNIFORM row (tag 8); position p keyed by
//                (p / g) << 44 | (out[0] of tag 9 >> 8) << 20 | p, output
//                ids[p] (generate_workloads_flat.h:85-137)
//   SOLO         fixed anchor slots as in generate_workloads_flat.h:140-247;
//                the remaining values keyed like UNIFORM with tag 10
#include <cub/device/device_segmented_radix_sort.cuh>

#include "common.cuh"
#include "internal.h"

namespace smpb200 {
namespace {

constexpr uint32_t kRowShared = 0xFFFFFFFFu;
constexpr uint64_t kLow20 = 0xFFFFFull;

enum Tag : uint32_t {
  kTagUniform = 0,
  kTagScore = 1,
  kTagNoise = 2,
  kTagSharedRow = 5,
  kTagPerfectFirst = 6,
  kTagPerfectTail = 7,
  kTagGroupIds = 8,
  kTagGroupRow = 9,
  kTagSolo = 10,
  kTagRefCongested = 11,
};

struct GenParams {
  int kind;
  int side;
  int n;
  uint32_t k0, k1;  // Philox key
  uint32_t salt;
  int param;
};

__device__ __forceinline__ uint32_t draw0(const GenParams &p, uint32_t j, uint32_t row, uint32_t tag) {
  uint32_t o[4];
  philox4x32_10(j, row, (static_cast<uint32_t>(p.side) << 8) | tag, p.salt, p.k0, p.k1, o);
  return o[0];
}

// Anchor slots of a SOLO row: slot index and value (value -1 = unused),
// and the shuffled slot range [lo, lo + cnt).
struct SoloRow {
  int slot[3];
  int value[3];
  int lo;
  int cnt;
};
__device__ __forceinline__ SoloRow solo_row(int side, int n, int i) {
  SoloRow s;
  s.slot[0] = s.slot[1] = s.slot[2] = -1;
  s.value[0] = s.value[1] = s.value[2] = -1;
  if (side == 0) {
    const int m = (i == n - 1) ? n - 2 : i;
    s.slot[0] = 0;       s.value[0] = m;
    s.slot[1] = n - 2;   s.value[1] = (m - 1 + n - 1) % (n - 1);
    s.slot[2] = n - 1;   s.value[2] = n - 1;
    s.lo = 1;
    s.cnt = n - 3;
  } else if (i < n - 1) {
    const int a0 = (i + 1) % (n - 1);
    s.slot[0] = 0;       s.value[0] = a0;
    s.slot[1] = 1;       s.value[1] = (a0 + n - 1) % n;
    s.lo = 2;
    s.cnt = n - 2;
  } else {
    s.lo = 0;
    s.cnt = n;
  }
  return s;
}

// t-th value of 0..n-1 that is not an anchor value.
__device__ __forceinline__ int solo_value(const SoloRow &s, int t) {
  int v[3] = {s.value[0], s.value[1], s.value[2]};
  // sort the (at most three) anchor values ascending, -1 first
  if (v[0] > v[1]) { int x = v[0]; v[0] = v[1]; v[1] = x; }
  if (v[1] > v[2]) { int x = v[1]; v[1] = v[2]; v[2] = x; }
  if (v[0] > v[1]) { int x = v[0]; v[0] = v[1]; v[1] = x; }
  int j = t;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (v[k] >= 0 && j >= v[k]) ++j;
  return j;
}

// Keys of one row chunk: rows [row0, row0 + rows), row-local slot t at
// keys[(i - row0) * n + lo + t].  Also fills the segment offsets.
__global__ void k_gen_keys(GenParams p, int row0, int rows, uint32_t row_word_override,
                           const int32_t *__restrict__ aux, unsigned long long *__restrict__ keys,
                           int *__restrict__ seg_begin, int *__restrict__ seg_end) {
  const int n = p.n;
  const size_t total = static_cast<size_t>(rows) * n;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total; idx += stride) {
    const int li = static_cast<int>(idx / n);
    const int t = static_cast<int>(idx - static_cast<size_t>(li) * n);
    const int i = row0 + li;
    const uint32_t row = row_word_override != 0 ? row_word_override : static_cast<uint32_t>(i);
    int lo = 0, cnt = n;
    unsigned long long key = 0;
    switch (p.kind) {
      case SMP_GEN_UNIFORM:
      case SMP_GEN_CONGESTED: {  // (the shared men's row passes its own tag via aux == nullptr path)
        key = (static_cast<unsigned long long>(draw0(p, t, row, kTagUniform)) << 20) | t;
        break;
      }
      case SMP_GEN_CORRELATED: {
        long long ih = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          uint32_t o[4];
          philox4x32_10(t, row, (static_cast<uint32_t>(p.side) << 8) | (kTagNoise + k), p.salt, p.k0, p.k1, o);
          ih += static_cast<long long>(o[0] >> 8) + (o[1] >> 8) + (o[2] >> 8) + (o[3] >> 8);
        }
        const long long z = ih - 6ll * (1ll << 24);
        const long long noise = (z * 256ll * static_cast<long long>(p.param)) / 10000ll;
        const long long tot = static_cast<long long>(static_cast<uint32_t>(aux[t])) + noise;
        const unsigned long long inv = static_cast<unsigned long long>((1ll << 36) - tot);
        key = (inv << 20) | t;
        break;
      }
      case SMP_GEN_PERFECT: {
        const unsigned long long hi =
            (t == aux[i]) ? 0ull : static_cast<unsigned long long>(draw0(p, t, row, kTagPerfectTail) >> 1) + 1ull;
        key = (hi << 20) | t;
        break;
      }
      case SMP_GEN_GROUPED: {
        const unsigned long long grp = static_cast<unsigned long long>(t / p.param);
        key = (grp << 44) | (static_cast<unsigned long long>(draw0(p, t, row, kTagGroupRow) >> 8) << 20) | t;
        break;
      }
      case SMP_GEN_SOLO: {
        const SoloRow s = solo_row(p.side, n, i);
        lo = s.lo;
        cnt = s.cnt;
        if (t < cnt) {
          const int j = solo_value(s, t);
          key = (static_cast<unsigned long long>(draw0(p, j, row, kTagSolo)) << 20) | j;
        }
        break;
      }
      default:
        break;
    }
    if (t < cnt) keys[static_cast<size_t>(li) * n + lo + t] = key;
    if (t == 0) {
      seg_begin[li] = li * n + lo;
      seg_end[li] = li * n + lo + cnt;
    }
  }
}

// Shared single rows (one segment): tag chosen by the caller.
__global__ void k_gen_shared_keys(GenParams p, uint32_t tag, unsigned long long *__restrict__ keys,
                                  int *__restrict__ seg) {
  const int n = p.n;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    keys[t] = (static_cast<unsigned long long>(draw0(p, t, kRowShared, tag)) << 20) | t;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    seg[0] = 0;
    seg[1] = n;
  }
}

__global__ void k_gen_scores(GenParams p, int32_t *__restrict__ aux) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < p.n; t += gridDim.x * blockDim.x)
    aux[t] = static_cast<int32_t>(draw0(p, t, kRowShared, kTagScore));
}

__global__ void k_gen_emit(GenParams p, int row0, int rows, const int32_t *__restrict__ aux,
                           const unsigned long long *__restrict__ keys, int32_t *__restrict__ out) {
  const int n = p.n;
  const size_t total = static_cast<size_t>(rows) * n;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total; idx += stride) {
    const int li = static_cast<int>(idx / n);
    const int t = static_cast<int>(idx - static_cast<size_t>(li) * n);
    const int i = row0 + li;
    int32_t v;
    if (p.kind == SMP_GEN_SOLO) {
      const SoloRow s = solo_row(p.side, n, i);
      if (t == s.slot[0]) v = s.value[0];
      else if (t == s.slot[1]) v = s.value[1];
      else if (t == s.slot[2]) v = s.value[2];
      else v = static_cast<int32_t>(keys[idx] & kLow20);
    } else if (p.kind == SMP_GEN_GROUPED) {
      v = aux[keys[idx] & kLow20];
    } else {
      v = static_cast<int32_t>(keys[idx] & kLow20);
    }
    out[static_cast<size_t>(i) * n + t] = v;
  }
}

__global__ void k_gen_broadcast(const int32_t *__restrict__ row, int32_t *__restrict__ out, int n) {
  const size_t total = static_cast<size_t>(n) * n;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total; idx += stride)
    out[idx] = row[idx % n];
}

__global__ void k_gen_shared_emit(const unsigned long long *__restrict__ keys, int32_t *__restrict__ out,
                                  int n) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    out[t] = static_cast<int32_t>(keys[t] & kLow20);
}

int key_bits(int kind) {
  switch (kind) {
    case SMP_GEN_CORRELATED: return 60;
    case SMP_GEN_GROUPED: return 64;
    default: return 52;
  }
}

}  // namespace

// Sort `segments` segments of keys_in into keys_out.  Scratch comes from the
// context's generator buffers.
static int sort_segments(Ctx &c, const unsigned long long *keys_in, unsigned long long *keys_out,
                         size_t num_items, int segments, const int *seg_begin, const int *seg_end,
                         int bits) {
  size_t temp = 0;
  if (cub::DeviceSegmentedRadixSort::SortKeys(nullptr, temp, keys_in, keys_out, static_cast<int>(num_items),
                                              segments, seg_begin, seg_end, 0, bits, c.stream) != cudaSuccess)
    return c.fail_cuda("cub temp query");
  int rc = c.gen_temp.ensure(temp);
  if (rc) return rc;
  if (cub::DeviceSegmentedRadixSort::SortKeys(c.gen_temp.ptr, temp, keys_in, keys_out, static_cast<int>(num_items),
                                              segments, seg_begin, seg_end, 0, bits, c.stream) != cudaSuccess)
    return c.fail_cuda("cub segmented sort");
  return SMP_OK;
}

// One shared row (tag) into out[0..n).
static int shared_row(Ctx &c, const GenParams &p, uint32_t tag, int32_t *out) {
  const int n = p.n;
  int rc = c.gen_keys_a.ensure(sizeof(unsigned long long) * n);
  if (!rc) rc = c.gen_keys_b.ensure(sizeof(unsigned long long) * n);
  if (!rc) rc = c.gen_seg.ensure(sizeof(int) * 2);
  if (rc) return rc;
  auto *ka = static_cast<unsigned long long *>(c.gen_keys_a.ptr);
  auto *kb = static_cast<unsigned long long *>(c.gen_keys_b.ptr);
  int *seg = static_cast<int *>(c.gen_seg.ptr);
  k_gen_shared_keys<<<std::min(c.sm_count * 4, (n + 255) / 256), 256, 0, c.stream>>>(p, tag, ka, seg);
  rc = sort_segments(c, ka, kb, n, 1, seg, seg + 1, 52);
  if (rc) return rc;
  k_gen_shared_emit<<<std::min(c.sm_count * 4, (n + 255) / 256), 256, 0, c.stream>>>(kb, out, n);
  return c.check_launch("gen shared row");
}

int generate_side(Ctx &c, int kind, int side, int n, uint64_t seed, uint32_t salt, int param,
                  int32_t *out) {
  GenParams p;
  p.kind = kind;
  p.side = side;
  p.n = n;
  p.k0 = static_cast<uint32_t>(seed);
  p.k1 = static_cast<uint32_t>(seed >> 32);
  p.salt = salt;
  p.param = param;
  const int grid = c.sm_count * 8;

  // Sides made of one shared row.
  if ((kind == SMP_GEN_CONGESTED && side == 0) || kind == SMP_GEN_REF_CONGESTED) {
    const uint32_t tag = (kind == SMP_GEN_CONGESTED) ? kTagSharedRow : kTagRefCongested;
    int rc = c.gen_aux.ensure(sizeof(int32_t) * n);
    if (rc) return rc;
    int32_t *row = static_cast<int32_t *>(c.gen_aux.ptr);
    rc = shared_row(c, p, tag, row);
    if (rc) return rc;
    k_gen_broadcast<<<grid, 256, 0, c.stream>>>(row, out, n);
    return c.check_launch("gen broadcast");
  }

  int rc = c.gen_aux.ensure(sizeof(int32_t) * n);
  if (rc) return rc;
  int32_t *aux = static_cast<int32_t *>(c.gen_aux.ptr);
  if (kind == SMP_GEN_CORRELATED) {
    k_gen_scores<<<std::min(grid, (n + 255) / 256), 256, 0, c.stream>>>(p, aux);
    rc = c.check_launch("gen scores");
  } else if (kind == SMP_GEN_PERFECT) {
    rc = shared_row(c, p, kTagPerfectFirst, aux);
  } else if (kind == SMP_GEN_GROUPED) {
    rc = shared_row(c, p, kTagGroupIds, aux);
  }
  if (rc) return rc;

  // Rows in chunks of at most 2^26 keys.
  const size_t chunk_items = std::max<size_t>(static_cast<size_t>(n), static_cast<size_t>(1) << 26);
  const int rows_per_chunk = static_cast<int>(std::min<size_t>(n, chunk_items / n));
  const size_t keys_bytes = sizeof(unsigned long long) * static_cast<size_t>(rows_per_chunk) * n;
  rc = c.gen_keys_a.ensure(keys_bytes);
  if (!rc) rc = c.gen_keys_b.ensure(keys_bytes);
  if (!rc) rc = c.gen_seg.ensure(sizeof(int) * 2 * static_cast<size_t>(rows_per_chunk));
  if (rc) return rc;
  auto *ka = static_cast<unsigned long long *>(c.gen_keys_a.ptr);
  auto *kb = static_cast<unsigned long long *>(c.gen_keys_b.ptr);
  int *seg_begin = static_cast<int *>(c.gen_seg.ptr);
  int *seg_end = seg_begin + rows_per_chunk;
  const int bits = key_bits(kind);
  for (int row0 = 0; row0 < n; row0 += rows_per_chunk) {
    const int rows = std::min(rows_per_chunk, n - row0);
    const size_t items = static_cast<size_t>(rows) * n;
    k_gen_keys<<<grid, 256, 0, c.stream>>>(p, row0, rows, 0u, aux, ka, seg_begin, seg_end);
    rc = c.check_launch("gen keys");
    if (rc) return rc;
    rc = sort_segments(c, ka, kb, items, rows, seg_begin, seg_end, bits);
    if (rc) return rc;
    k_gen_emit<<<grid, 256, 0, c.stream>>>(p, row0, rows, aux, kb, out);
    rc = c.check_launch("gen emit");
    if (rc) return rc;
  }
  return SMP_OK;
}

}  // namespace smpb200
