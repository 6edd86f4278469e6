// Host-side copies of the staging paths (pageable caller memory <-> page-locked
// staging).  Pieces of these sizes (tens of KB to MB) are below the size at
// which memcpy switches to non-temporal stores, so a plain memcpy first reads
// every destination line into the cache before overwriting it: a third of its
// memory traffic.  stream_copy writes with non-temporal AVX2 stores instead
// when the host has AVX2, and falls back to memcpy otherwise and for small
// pieces.
#include <immintrin.h>

#include <cstdint>
#include <cstring>

#include "wmh_internal.h"

namespace mhb {
namespace {

constexpr size_t kStreamMinBytes = static_cast<size_t>(64) << 10;

__attribute__((target("avx2"))) void stream_copy_avx2(char *d, const char *s, size_t bytes) {
  const size_t head = (32 - (reinterpret_cast<uintptr_t>(d) & 31u)) & 31u;
  memcpy(d, s, head);
  d += head;
  s += head;
  bytes -= head;
  const size_t blocks = bytes / 128;
  for (size_t i = 0; i < blocks; ++i, d += 128, s += 128) {
    const __m256i a0 = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s));
    const __m256i a1 = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + 32));
    const __m256i a2 = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + 64));
    const __m256i a3 = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + 96));
    _mm256_stream_si256(reinterpret_cast<__m256i *>(d), a0);
    _mm256_stream_si256(reinterpret_cast<__m256i *>(d + 32), a1);
    _mm256_stream_si256(reinterpret_cast<__m256i *>(d + 64), a2);
    _mm256_stream_si256(reinterpret_cast<__m256i *>(d + 96), a3);
  }
  memcpy(d, s, bytes - blocks * 128);
  _mm_sfence();  // the streamed lines are visible before the copy is used
}

// dst 32-byte aligned, n a multiple of 8.
__attribute__((target("avx2"))) void stream_f64_to_f32_avx2(float *dst, const double *src,
                                                             size_t n) {
  for (size_t i = 0; i < n; i += 8) {
    // cvtpd2ps rounds with the MXCSR mode, round-to-nearest by default: the
    // same as static_cast<float> and numpy's astype.
    const __m128 lo = _mm256_cvtpd_ps(_mm256_loadu_pd(src + i));
    const __m128 hi = _mm256_cvtpd_ps(_mm256_loadu_pd(src + i + 4));
    _mm256_stream_ps(dst + i, _mm256_set_m128(hi, lo));
  }
  _mm_sfence();
}

// 64-bit integers to uint32, values outside [0, 2^32) to 0xFFFFFFFF (both
// signed and unsigned sources: such a value has nonzero high 32 bits).  dst
// 32-byte aligned, n a multiple of 8.
__attribute__((target("avx2"))) void stream_i64_to_u32_avx2(uint32_t *dst, const uint64_t *src,
                                                             size_t n) {
  const __m256i zero = _mm256_setzero_si256();
  const __m256i ones = _mm256_set1_epi32(-1);
  const __m256i lows = _mm256_setr_epi32(0, 2, 4, 6, 0, 2, 4, 6);
  for (size_t i = 0; i < n; i += 8) {
    __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + i));
    __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + i + 4));
    a = _mm256_blendv_epi8(ones, a, _mm256_cmpeq_epi64(_mm256_srli_epi64(a, 32), zero));
    b = _mm256_blendv_epi8(ones, b, _mm256_cmpeq_epi64(_mm256_srli_epi64(b, 32), zero));
    const __m128i la = _mm256_castsi256_si128(_mm256_permutevar8x32_epi32(a, lows));
    const __m128i lb = _mm256_castsi256_si128(_mm256_permutevar8x32_epi32(b, lows));
    _mm256_stream_si256(reinterpret_cast<__m256i *>(dst + i), _mm256_set_m128i(lb, la));
  }
  _mm_sfence();
}

// Column packing, 16 entries per step: lo gets the low 16 bits of each column,
// hi the bits above, as bytes (HB = 8) or as nibbles two to a byte (HB = 4,
// even entry in the low nibble).  Non-temporal stores; lo 32-byte aligned and
// n a multiple of 16.  Returns the OR of every column shifted right by
// 16 + HB (nonzero: some column did not fit).
template <int HB>
__attribute__((target("avx2"))) uint32_t pack_cols_avx2(const uint32_t *src, size_t n,
                                                         uint16_t *lo, uint8_t *hi) {
  const __m256i mask16 = _mm256_set1_epi32(0xFFFF);
  __m256i over = _mm256_setzero_si256();
  for (size_t i = 0; i < n; i += 16) {
    const __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + i));
    const __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + i + 8));
    over = _mm256_or_si256(over, _mm256_or_si256(_mm256_srli_epi32(a, 16 + HB),
                                                 _mm256_srli_epi32(b, 16 + HB)));
    // 32 -> 16 bits; packus interleaves 128-bit lanes, permute restores order.
    const __m256i l = _mm256_permute4x64_epi64(
        _mm256_packus_epi32(_mm256_and_si256(a, mask16), _mm256_and_si256(b, mask16)), 0xD8);
    _mm256_stream_si256(reinterpret_cast<__m256i *>(lo + i), l);
    const __m256i h16 = _mm256_permute4x64_epi64(
        _mm256_packus_epi32(_mm256_srli_epi32(a, 16), _mm256_srli_epi32(b, 16)), 0xD8);
    const __m128i h8 = _mm_packus_epi16(_mm256_castsi256_si128(h16),
                                        _mm256_extracti128_si256(h16, 1));
    if (HB == 8) {
      _mm_storeu_si128(reinterpret_cast<__m128i *>(hi + i), h8);
    } else {
      // byte pairs (e, o) -> e + 16 * o, 16 bits each, then to bytes
      const __m128i pairs = _mm_maddubs_epi16(h8, _mm_set1_epi16(0x1001));
      const __m128i nib = _mm_packus_epi16(pairs, pairs);
      _mm_storel_epi64(reinterpret_cast<__m128i *>(hi + i / 2), nib);
    }
  }
  _mm_sfence();
  over = _mm256_or_si256(over, _mm256_srli_si256(over, 8));
  over = _mm256_or_si256(over, _mm256_srli_si256(over, 4));
  return static_cast<uint32_t>(_mm256_extract_epi32(over, 0) | _mm256_extract_epi32(over, 4));
}

bool host_has_avx2() {
  static const bool v = __builtin_cpu_supports("avx2");
  return v;
}

}  // namespace

void stream_copy(void *dst, const void *src, size_t bytes) {
  if (bytes >= kStreamMinBytes && host_has_avx2())
    stream_copy_avx2(static_cast<char *>(dst), static_cast<const char *>(src), bytes);
  else
    memcpy(dst, src, bytes);
}

void convert_f64_to_f32(float *dst, const double *src, size_t n) {
  size_t i = 0;
  if (n >= kStreamMinBytes / 4 && host_has_avx2()) {
    for (; i < n && (reinterpret_cast<uintptr_t>(dst + i) & 31u); ++i)
      dst[i] = static_cast<float>(src[i]);
    const size_t body = (n - i) & ~static_cast<size_t>(7);
    stream_f64_to_f32_avx2(dst + i, src + i, body);
    i += body;
  }
  for (; i < n; ++i) dst[i] = static_cast<float>(src[i]);
}

bool pack_cols(const uint32_t *src, size_t n, uint16_t *lo, uint8_t *hi, int hi_bits) {
  const int hb = hi_bits == 4 ? 4 : 8;
  const uint32_t limit_shift = 16 + hb;
  uint32_t over = 0;
  size_t i = 0;
  // Scalar head up to a 32-byte boundary of lo (an even count, so nibble
  // pairs stay whole), vector body, scalar tail.
  auto scalar = [&](size_t b, size_t e) {
    for (size_t k = b; k < e; ++k) {
      const uint32_t c = src[k];
      over |= c >> limit_shift;
      lo[k] = static_cast<uint16_t>(c);
      const uint8_t h = static_cast<uint8_t>(c >> 16);
      if (hb == 8) {
        hi[k] = h;
      } else if (k & 1) {
        hi[k / 2] = static_cast<uint8_t>(hi[k / 2] | ((h & 15u) << 4));
      } else {
        hi[k / 2] = static_cast<uint8_t>(h & 15u);
      }
    }
  };
  if (n >= 4096 && host_has_avx2()) {
    while (i < n && (reinterpret_cast<uintptr_t>(lo + i) & 31u)) i += 1;
    if (i & 1) ++i;
    if ((reinterpret_cast<uintptr_t>(lo + i) & 31u) == 0) {
      scalar(0, i);
      const size_t body = (n - i) & ~static_cast<size_t>(15);
      over |= hb == 8 ? pack_cols_avx2<8>(src + i, body, lo + i, hi + i)
                      : pack_cols_avx2<4>(src + i, body, lo + i, hi + i / 2);
      i += body;
    } else {
      i = 0;
    }
  }
  scalar(i, n);
  return over == 0;
}

void convert_i64_to_u32(uint32_t *dst, const uint64_t *src, size_t n) {
  size_t i = 0;
  if (n >= kStreamMinBytes / 4 && host_has_avx2()) {
    for (; i < n && (reinterpret_cast<uintptr_t>(dst + i) & 31u); ++i)
      dst[i] = (src[i] >> 32) ? 0xFFFFFFFFu : static_cast<uint32_t>(src[i]);
    const size_t body = (n - i) & ~static_cast<size_t>(7);
    stream_i64_to_u32_avx2(dst + i, src + i, body);
    i += body;
  }
  for (; i < n; ++i) dst[i] = (src[i] >> 32) ? 0xFFFFFFFFu : static_cast<uint32_t>(src[i]);
}

}  // namespace mhb
