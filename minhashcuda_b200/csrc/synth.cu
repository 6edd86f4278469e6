// Synthetic CSR generators for the benchmark and the tests.  Not part
// of the hash path; the hash path never calls them.
//
// Every draw is keyed by the absolute row index (and the position in the row),
// so any row range can be regenerated on its own.  Row offsets are the
// caller's prefix sum of the row lengths.  Kernels:
//   mhs_row_nnz       per-row lengths from a few length laws,
//   mhs_lognormal_values  lognormal(mu, sigma) values,
//   mhs_zipf_cols     distinct Zipf(s)-ranked columns per row (without
//                     replacement), ranks mapped through a seeded affine
//                     permutation of [0, dim), sorted ascending;
//   mhs_uniform_cols  distinct uniform columns per row, sorted ascending.
// Zipf ranks use continuous power-law inversion (density x^-s on [1, dim+1)),
// an approximation of the discrete Zipf law; rows are sampled "without
// replacement" by drawing until the row holds its target number of distinct
// columns.  Uniform rows use exponential spacings (sorted uniforms as
// normalised partial sums of Exp(1) variates) mapped to [0, dim-n] and offset
// by the index, which yields n distinct sorted columns.
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Uniform in (0, 1).
__device__ __forceinline__ double unit(uint64_t seed, uint64_t a, uint64_t b) {
  const uint64_t x = mix64(seed ^ mix64(a * 0xD1B54A32D192ED03ull + b));
  return (static_cast<double>(x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

constexpr int kZipfThreads = 256;
constexpr int kZipfTable = 4096;  // hash-set slots (power of two)
constexpr int kZipfMaxRow = 2048; // longest row the Zipf generator fills

__device__ __forceinline__ uint32_t slot_of(uint32_t col) {
  return static_cast<uint32_t>(mix64(col) & (kZipfTable - 1));
}

__global__ void zipf_cols_kernel(uint32_t rows, uint64_t row0, const uint32_t *__restrict__ indptr,
                                 uint32_t dim, double s, uint64_t seed, uint64_t perm_a,
                                 uint64_t perm_b, uint32_t *__restrict__ cols,
                                 uint32_t *__restrict__ status) {
  __shared__ uint32_t table[kZipfTable];  // col + 1, 0 = empty (linear probing)
  __shared__ uint32_t owner[kZipfTable];  // lowest thread that drew the slot's col this round
  __shared__ uint32_t list[kZipfMaxRow];
  __shared__ uint32_t warp_new[kZipfThreads / 32];
  __shared__ uint32_t count;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const double one_minus_s = 1.0 - s;
  const double top = pow(static_cast<double>(dim) + 1.0, one_minus_s);
  for (uint32_t row = blockIdx.x; row < rows; row += gridDim.x) {
    const uint32_t start = indptr[row];
    const uint32_t n = indptr[row + 1] - start;
    if (n > kZipfMaxRow || n > dim) {
      if (tid == 0) atomicOr(status, 1u);
      continue;
    }
    for (int i = tid; i < kZipfTable; i += kZipfThreads) {
      table[i] = 0;
      owner[i] = 0xFFFFFFFFu;
    }
    if (tid == 0) count = 0;
    __syncthreads();
    // Draw rounds.  A round's new columns are accepted in the order of the
    // lowest thread that drew each of them, so the row's column set is a
    // pure function of (seed, row) regardless of atomic ordering.
    for (uint32_t round = 0;; ++round) {
      const uint32_t have = count;  // same snapshot in every thread
      __syncthreads();
      if (have >= n) break;
      if (round > 100000) {  // cannot happen for n <= dim; keeps the loop finite
        if (tid == 0) atomicOr(status, 2u);
        break;
      }
      const double u = unit(seed, ((row0 + row) << 20) ^ round, tid);
      const double x = pow(1.0 - u * (1.0 - top), 1.0 / one_minus_s);
      uint64_t rank = static_cast<uint64_t>(x) - 1;  // [0, dim)
      if (rank >= dim) rank = dim - 1;
      const uint32_t col = static_cast<uint32_t>((perm_a * rank + perm_b) % dim);
      const uint32_t key = col + 1u;
      // Phase 1: is the column already in the row (from earlier rounds)?
      bool old = false;
      uint32_t h = slot_of(col);
      for (int probe = 0; probe < kZipfTable; ++probe) {
        const uint32_t v = table[h];
        if (v == key) { old = true; break; }
        if (v == 0u) break;
        h = (h + 1) & (kZipfTable - 1);
      }
      __syncthreads();
      // Phase 2: insert new columns; every drawer of a column learns its slot.
      if (!old) {
        h = slot_of(col);
        for (int probe = 0; probe < kZipfTable; ++probe) {
          const uint32_t prev = atomicCAS(&table[h], 0u, key);
          if (prev == 0u || prev == key) break;
          h = (h + 1) & (kZipfTable - 1);
        }
        atomicMin(&owner[h], tid);
      }
      __syncthreads();
      // Phase 3: the owner of each new column takes a place in thread order.
      const bool rep = !old && owner[h] == tid;
      const unsigned ballot = __ballot_sync(0xFFFFFFFFu, rep);
      if (lane == 0) warp_new[warp] = __popc(ballot);
      __syncthreads();
      uint32_t before = __popc(ballot & ((1u << lane) - 1u)), total = 0;
      for (uint32_t w = 0; w < kZipfThreads / 32; ++w) {
        if (w < warp) before += warp_new[w];
        total += warp_new[w];
      }
      if (rep && have + before < n) list[have + before] = col;
      __syncthreads();
      if (rep) owner[h] = 0xFFFFFFFFu;
      if (tid == 0) count = min(n, have + total);
      __syncthreads();
    }
    __syncthreads();
    // Bitonic sort of list[0, P), P = next power of two >= n, padded high.
    uint32_t P = 1;
    while (P < n) P <<= 1;
    for (uint32_t i = n + threadIdx.x; i < P; i += kZipfThreads) list[i] = 0xFFFFFFFFu;
    __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = threadIdx.x; i < P; i += kZipfThreads) {
          const uint32_t l = i ^ j;
          if (l > i) {
            const uint32_t a = list[i], b = list[l];
            const bool up = (i & k) == 0;
            if ((a > b) == up) {
              list[i] = b;
              list[l] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    for (uint32_t i = threadIdx.x; i < n; i += kZipfThreads) cols[start + i] = list[i];
    __syncthreads();
  }
}

constexpr int kUniThreads = 256;

__global__ void uniform_cols_kernel(uint32_t rows, uint64_t row0,
                                    const uint32_t *__restrict__ indptr, uint32_t dim, uint64_t seed, uint32_t *__restrict__ cols,
                                    uint32_t *__restrict__ status) {
  __shared__ double part[kUniThreads];
  for (uint32_t row = blockIdx.x; row < rows; row += gridDim.x) {
    const uint32_t start = indptr[row];
    const uint32_t n = indptr[row + 1] - start;
    if (n > dim) {
      if (threadIdx.x == 0) atomicOr(status, 1u);
      continue;
    }
    if (n == 0) continue;
    // n + 1 exponential gaps; thread t owns gaps [t*k, (t+1)*k).
    const uint32_t k = (n + 1 + kUniThreads - 1) / kUniThreads;
    const uint32_t g0 = threadIdx.x * k;
    const uint32_t g1 = min(n + 1, g0 + k);
    const uint64_t rkey = ((row0 + row) << 1) | 1u;
    double sum = 0.0;
    for (uint32_t g = g0; g < g1; ++g) sum += -log(unit(seed, rkey, g));
    part[threadIdx.x] = sum;
    __syncthreads();
    // Inclusive scan of the per-thread sums (Hillis-Steele in shared memory).
    for (int off = 1; off < kUniThreads; off <<= 1) {
      const double v = threadIdx.x >= off ? part[threadIdx.x - off] : 0.0;
      __syncthreads();
      part[threadIdx.x] += v;
      __syncthreads();
    }
    const double total = part[kUniThreads - 1];
    double acc = threadIdx.x ? part[threadIdx.x - 1] : 0.0;
    const double span = static_cast<double>(dim - n) + 1.0;
    for (uint32_t g = g0; g < g1 && g < n; ++g) {
      acc += -log(unit(seed, rkey, g));
      double m = floor(acc / total * span);
      if (m > static_cast<double>(dim - n)) m = static_cast<double>(dim - n);
      cols[start + g] = static_cast<uint32_t>(m) + g;
    }
    __syncthreads();
  }
}

// Row lengths.  kind 0: Poisson(p1) through its normal approximation
// round(p1 + sqrt(p1) z); kind 1: round(lognormal(ln p1, p2)); kind 2:
// round(exp(U(ln p1, ln p2))) (log-uniform); kind 3: p1 * (1 + K), K >= 1 with
// P(K >= k) = k^(1 - p2) (a Zipf(p2) tail by continuous inversion).  Clipped to [lo, hi].
__global__ void row_nnz_kernel(uint32_t rows, uint64_t row0, int kind, double p1, double p2,
                               uint32_t lo, uint32_t hi, uint64_t seed, uint32_t *__restrict__ nnz) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const uint64_t r = row0 + i;
    const double u1 = unit(seed, r, 0x51u), u2 = unit(seed, r, 0x52u);
    const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    double v;
    switch (kind) {
      case 0: v = p1 + sqrt(p1) * z; break;
      case 1: v = exp(log(p1) + p2 * z); break;
      case 2: v = exp(log(p1) + u1 * (log(p2) - log(p1))); break;
      default: v = p1 * (1.0 + floor(pow(u1, -1.0 / (p2 - 1.0)))); break;
    }
    v = floor(v + 0.5);
    if (!(v >= lo)) v = lo;
    if (v > hi) v = hi;
    nnz[i] = static_cast<uint32_t>(v);
  }
}

// values[j] = exp(mu + sigma z) with z keyed by (row, position in row).
__global__ void lognormal_values_kernel(uint32_t rows, uint64_t row0,
                                        const uint32_t *__restrict__ indptr, double mu,
                                        double sigma, uint64_t seed, float *__restrict__ vals) {
  for (uint32_t row = blockIdx.x; row < rows; row += gridDim.x) {
    const uint32_t start = indptr[row], n = indptr[row + 1] - start;
    const uint64_t key = ((row0 + row) << 1);
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
      const double u1 = unit(seed, key, 2ull * j), u2 = unit(seed, key, 2ull * j + 1);
      const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
      vals[start + j] = static_cast<float>(exp(mu + sigma * z));
    }
  }
}

}  // namespace

extern "C" {

int mhs_row_nnz(uint32_t rows, uint64_t row0, int kind, double p1, double p2, uint32_t lo,
                uint32_t hi, uint64_t seed, uint32_t *d_nnz, void *stream) {
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (rows == 0) return 0;
  const uint32_t grid = std::min<uint32_t>((rows + 255) / 256, 65535u);
  row_nnz_kernel<<<grid, 256, 0, st>>>(rows, row0, kind, p1, p2, lo, hi, seed, d_nnz);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int mhs_lognormal_values(uint32_t rows, uint64_t row0, const uint32_t *d_indptr, double mu,
                         double sigma, uint64_t seed, float *d_vals, void *stream) {
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (rows == 0) return 0;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  lognormal_values_kernel<<<static_cast<uint32_t>(sms) * 16, 256, 0, st>>>(
      rows, row0, d_indptr, mu, sigma, seed, d_vals);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Returns 0 on success, 1 for rows longer than the generator supports or
// than dim, 2 for a launch or device error.  indptr is relative (starts at 0).
int mhs_zipf_cols(uint32_t rows, uint64_t row0, const uint32_t *d_indptr, uint32_t dim, double s, uint64_t seed,
                  uint32_t *d_cols, void *stream) {
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t *d_status = nullptr;
  if (cudaMalloc(&d_status, 4) != cudaSuccess) return 2;
  cudaMemsetAsync(d_status, 0, 4, st);
  // Seeded affine permutation rank -> (a*rank + b) mod dim with gcd(a, dim) = 1.
  uint64_t a = (seed * 0x9E3779B97F4A7C15ull) % dim;
  auto gcd = [](uint64_t x, uint64_t y) {
    while (y) {
      const uint64_t t = x % y;
      x = y;
      y = t;
    }
    return x;
  };
  if (a == 0) a = 1;
  while (gcd(a, dim) != 1) a = (a + 1) % dim ? (a + 1) % dim : 1;
  const uint64_t b = (seed * 0xC2B2AE3D27D4EB4Full) % dim;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t grid = static_cast<uint32_t>(sms) * 8;
  zipf_cols_kernel<<<grid, kZipfThreads, 0, st>>>(rows, row0, d_indptr, dim, s, seed, a, b, d_cols,
                                                  d_status);
  uint32_t h = 0;
  int rc = cudaGetLastError() == cudaSuccess ? 0 : 2;
  if (cudaMemcpyAsync(&h, d_status, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    rc = 2;
  cudaFree(d_status);
  if (rc == 0 && h) rc = 1;
  return rc;
}

int mhs_uniform_cols(uint32_t rows, uint64_t row0, const uint32_t *d_indptr, uint32_t dim, uint64_t seed,
                     uint32_t *d_cols, void *stream) {
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t *d_status = nullptr;
  if (cudaMalloc(&d_status, 4) != cudaSuccess) return 2;
  cudaMemsetAsync(d_status, 0, 4, st);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t grid = static_cast<uint32_t>(sms) * 8;
  uniform_cols_kernel<<<grid, kUniThreads, 0, st>>>(rows, row0, d_indptr, dim, seed, d_cols, d_status);
  uint32_t h = 0;
  int rc = cudaGetLastError() == cudaSuccess ? 0 : 2;
  if (cudaMemcpyAsync(&h, d_status, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    rc = 2;
  cudaFree(d_status);
  if (rc == 0 && h) rc = 1;
  return rc;
}

}  // extern "C"
