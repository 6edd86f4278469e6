// Downstream of the hash: LSH band keys and weighted-Jaccard estimates over
// device-resident hashes ([rows][samples][2] uint32, the layout mhcuda_calc
// returns).  The reference stops at the hashes; its tests consume them as
// datasketch's WeightedMinHash.jaccard does (test.py:104-106): the estimate
// for two rows is the fraction of samples whose (k, t) pairs are equal.
//
// Band key of band b (samples [b*w, (b+1)*w)) of a row:
//   h = 0x6A09E667F3BCC909 ^ b
//   for each sample s of the band: h = mix64(h ^ ((uint64)k_s << 32 | t_s))
// with mix64 the splitmix64 finaliser.  Rows whose keys agree in some band
// are candidate pairs (banded LSH).
#include <cstdint>

#include "../../include/minhashcuda.h"
#include "../../include/minhashcuda_b200.h"
#include "wmh_internal.h"

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// One thread per (row, band).
__global__ void band_keys_kernel(const uint2 *__restrict__ hashes, uint32_t rows, uint32_t samples,
                                 uint32_t width, uint32_t bands, uint64_t *__restrict__ keys) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= static_cast<uint64_t>(rows) * bands) return;
  const uint64_t row = i / bands;
  const uint32_t b = static_cast<uint32_t>(i - row * bands);
  const uint2 *h = hashes + row * samples + static_cast<uint64_t>(b) * width;
  uint64_t key = 0x6A09E667F3BCC909ull ^ b;
  for (uint32_t s = 0; s < width; ++s) {
    const uint2 v = h[s];
    key = mix64(key ^ ((static_cast<uint64_t>(v.x) << 32) | v.y));
  }
  keys[i] = key;
}

// One warp per pair: lanes compare samples, a warp reduction counts matches.
__global__ void jaccard_kernel(const uint2 *__restrict__ hashes, uint32_t rows, uint32_t samples,
                               const uint32_t *__restrict__ pairs, uint64_t npairs,
                               float *__restrict__ out) {
  const uint64_t p = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  if (p >= npairs) return;
  const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
  if (a >= rows || b >= rows) {
    if (lane == 0) out[p] = -1.0f;
    return;
  }
  const uint2 *ha = hashes + static_cast<uint64_t>(a) * samples;
  const uint2 *hb = hashes + static_cast<uint64_t>(b) * samples;
  uint32_t same = 0;
  for (uint32_t s = lane; s < samples; s += 32) {
    const uint2 x = ha[s], y = hb[s];
    same += (x.x == y.x && x.y == y.y) ? 1u : 0u;
  }
  for (int off = 16; off > 0; off >>= 1) same += __shfl_down_sync(0xFFFFFFFFu, same, off);
  if (lane == 0) out[p] = static_cast<float>(same) / static_cast<float>(samples);
}

}  // namespace

extern "C" {

enum MHCUDAResult mhcuda_lsh_bands(const MinhashCudaGenerator *gen, const uint32_t *d_hashes,
                                   uint32_t rows, uint32_t band_width, uint64_t *d_keys,
                                   void *stream) {
  mhb::GeneratorView g{};
  if (!mhb::generator_view(gen, &g) || !d_hashes || !d_keys || band_width == 0 ||
      band_width > g.samples)
    return mhcudaInvalidArguments;
  mhb::DeviceGuard on_device(g.device);
  if (!on_device.ok()) return mhcudaNoSuchDevice;
  const uint32_t bands = g.samples / band_width;
  const uint64_t n = static_cast<uint64_t>(rows) * bands;
  if (n == 0) return mhcudaSuccess;
  const cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g.stream;
  const uint64_t blocks = (n + 255) / 256;
  if (blocks > 0x7FFFFFFFull) return mhcudaInvalidArguments;
  band_keys_kernel<<<static_cast<unsigned>(blocks), 256, 0, st>>>(
      reinterpret_cast<const uint2 *>(d_hashes), rows, g.samples, band_width, bands, d_keys);
  if (cudaGetLastError() != cudaSuccess) return mhcudaRuntimeError;
  return cudaStreamSynchronize(st) == cudaSuccess ? mhcudaSuccess : mhcudaRuntimeError;
}

enum MHCUDAResult mhcuda_jaccard(const MinhashCudaGenerator *gen, const uint32_t *d_hashes,
                                 uint32_t rows, const uint32_t *d_pairs, uint64_t npairs,
                                 float *d_out, void *stream) {
  mhb::GeneratorView g{};
  if (!mhb::generator_view(gen, &g) || !d_hashes || !d_pairs || !d_out)
    return mhcudaInvalidArguments;
  mhb::DeviceGuard on_device(g.device);
  if (!on_device.ok()) return mhcudaNoSuchDevice;
  if (npairs == 0) return mhcudaSuccess;
  const cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g.stream;
  const uint64_t blocks = (npairs * 32 + 255) / 256;
  if (blocks > 0x7FFFFFFFull) return mhcudaInvalidArguments;
  jaccard_kernel<<<static_cast<unsigned>(blocks), 256, 0, st>>>(
      reinterpret_cast<const uint2 *>(d_hashes), rows, g.samples, d_pairs, npairs, d_out);
  if (cudaGetLastError() != cudaSuccess) return mhcudaRuntimeError;
  return cudaStreamSynchronize(st) == cudaSuccess ? mhcudaSuccess : mhcudaRuntimeError;
}

}  // extern "C"
