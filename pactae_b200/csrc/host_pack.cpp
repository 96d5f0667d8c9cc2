// Host-side packing of int32 preference entries to uint16 for host-input
// solves of n <= 32767, whose lists then cross the host link at half size.
// An entry outside [0, n) becomes a value >= n (0xFFFF for negatives and
// for entries of 65536 and up), which the inversion reports as invalid
// input, so a row that was not a permutation never packs into one.
#include <cstddef>
#include <cstdint>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

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
// unsigned values), a saturating pack, and a streaming store -- the packed
// rows go to pinned staging that only the copy engine reads, so they skip
// the cache and its read-for-ownership.
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
    _mm256_stream_si256(reinterpret_cast<__m256i *>(dst + k), p);
  }
  _mm_sfence();
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

}  // namespace smpb200
