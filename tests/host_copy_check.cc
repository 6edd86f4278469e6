// Checks the host staging helpers of minhashcuda_b200/csrc/host_copy.cc
// against memcpy and the scalar conversions, over random sizes, source and
// destination offsets, every float64 bit pattern class (NaN, inf,
// subnormal, huge) and out-of-range / negative 64-bit columns.  Prints "ok"
// and exits 0 when everything matches.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

namespace mhb {
void stream_copy(void *dst, const void *src, size_t bytes);
void convert_f64_to_f32(float *dst, const double *src, size_t n);
void convert_i64_to_u32(uint32_t *dst, const uint64_t *src, size_t n);
bool pack_cols(const uint32_t *src, size_t n, uint16_t *lo, uint8_t *hi, int hi_bits);
}  // namespace mhb

int main() {
  std::mt19937_64 g(7);
  // stream_copy == memcpy, including the bytes around the copied range.
  std::vector<unsigned char> src(3 << 20), a(3 << 20), b(3 << 20);
  for (auto &x : src) x = static_cast<unsigned char>(g());
  for (int t = 0; t < 300; ++t) {
    const size_t so = g() % 64, dof = g() % 64;
    size_t n = g() % (2 << 20);
    if (t % 3 == 0) n = (64 << 10) + g() % 300;
    memset(a.data(), 0x5A, a.size());
    memset(b.data(), 0x5A, b.size());
    mhb::stream_copy(a.data() + dof, src.data() + so, n);
    memcpy(b.data() + dof, src.data() + so, n);
    if (memcmp(a.data(), b.data(), a.size()) != 0) {
      printf("stream_copy mismatch: n=%zu\n", n);
      return 1;
    }
  }
  // Conversions == scalar casts.
  const size_t N = 1 << 20;
  std::vector<double> d(N + 16);
  std::vector<uint64_t> q(N + 16);
  for (size_t i = 0; i < d.size(); ++i) {
    uint64_t bits = g();
    double x;
    memcpy(&x, &bits, 8);
    if (i % 3 == 0) x = std::ldexp(static_cast<double>(g() >> 11), -static_cast<int>(g() % 80));
    d[i] = x;
    int64_t v = static_cast<int64_t>(g());
    if (i % 2) v = static_cast<int64_t>(g() % 0x100000000ull);
    if (i % 7 == 0) v = -static_cast<int64_t>(g() % 5);
    q[i] = static_cast<uint64_t>(v);
  }
  std::vector<float> f(N + 64);
  std::vector<uint32_t> u(N + 64);
  for (int t = 0; t < 40; ++t) {
    const size_t so = g() % 8, dof = g() % 8;
    const size_t n = (t % 2) ? N - g() % 1000 : g() % 70000;
    mhb::convert_f64_to_f32(f.data() + dof, d.data() + so, n);
    mhb::convert_i64_to_u32(u.data() + dof, q.data() + so, n);
    for (size_t i = 0; i < n; ++i) {
      const float want = static_cast<float>(d[so + i]);
      uint32_t x, y;
      memcpy(&x, &f[dof + i], 4);
      memcpy(&y, &want, 4);
      if (x != y && !(std::isnan(f[dof + i]) && std::isnan(want))) {
        printf("convert_f64_to_f32 mismatch at %zu\n", i);
        return 1;
      }
      const int64_t v = static_cast<int64_t>(q[so + i]);
      const uint32_t wu = (v < 0 || v > 0xFFFFFFFFll) ? 0xFFFFFFFFu : static_cast<uint32_t>(v);
      if (u[dof + i] != wu) {
        printf("convert_i64_to_u32 mismatch at %zu\n", i);
        return 1;
      }
    }
  }
  // pack_cols: low 16 bits and the bits above (bytes or nibbles) round-trip
  // every column below 2^(16 + hi_bits); a larger column is reported.
  for (int t = 0; t < 60; ++t) {
    const int hb = (t % 2) ? 4 : 8;
    const size_t lo_off = 2 * (g() % 20);  // even: nibble pairs stay whole
    const size_t n = (t % 3 == 0) ? (g() % 300) : (1 << 16) + g() % 70000;
    std::vector<uint32_t> c(n);
    for (auto &x : c) x = static_cast<uint32_t>(g() % (1ull << (16 + hb)));
    const bool plant = t % 5 == 4 && n > 0;
    if (plant) c[g() % n] = 1u << (16 + hb);
    std::vector<uint16_t> lo(n + 64, 0xAAAA);
    std::vector<uint8_t> hi(n + 64, 0xAA);
    const bool ok = mhb::pack_cols(c.data(), n, lo.data() + lo_off, hi.data() + lo_off, hb);
    if (ok == plant) {
      printf("pack_cols overflow report wrong (t=%d)\n", t);
      return 1;
    }
    if (plant) continue;
    for (size_t i = 0; i < n; ++i) {
      const uint8_t *h = hi.data() + lo_off;
      const uint32_t hv = hb == 8 ? h[i] : ((h[i / 2] >> ((i & 1) * 4)) & 15u);
      if ((static_cast<uint32_t>(lo[lo_off + i]) | (hv << 16)) != c[i]) {
        printf("pack_cols mismatch at %zu (t=%d)\n", i, t);
        return 1;
      }
    }
    if (lo[lo_off + n] != 0xAAAA) {
      printf("pack_cols wrote past lo (t=%d)\n", t);
      return 1;
    }
  }
  printf("ok\n");
  return 0;
}
