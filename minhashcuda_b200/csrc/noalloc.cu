// mhcuda_calc_device_noalloc: the device-resident hash for callers that must
// not allocate device memory.
//
// The ordinary device entry point (mhcuda_calc_device) grows a per-generator
// workspace with cudaMalloc whenever an input needs more scratch than the
// last one.  Some callers cannot allow that: a process whose device memory is
// already reserved in full by another allocator (a framework's caching
// allocator, for instance) would see the cudaMalloc fail, and a
// latency-critical loop cannot afford the device-wide synchronisation a
// cudaMalloc or cudaFree may cause.  This entry point therefore keeps its
// scratch -- the status word, the chunk table and the partial minima of rows
// that cross chunk boundaries -- in one fixed array in device memory that is
// part of the library image, and allocates nothing itself.
//
// Limits and sharing:
//  - the array holds kNoallocScratchBytes (8 MiB) on every device the library
//    is loaded on, until the process exits;
//  - an input needs 4 + 24 * s_pad bytes per chunk (s_pad = samples rounded up
//    to a multiple of 4) and chunks hold at most 2^20 nnz, so an input is
//    refused (mhcudaInvalidArguments) when
//        ceil(nnz / 2^20) > (8 MiB - 1 KiB) / (4 + 24 * s_pad);
//    with 128 samples that allows up to ~2.8e9 nnz, with 65535 samples 5 * 2^20;
//  - all calls on a device share the array, which keeps the last call's
//    contents; the status word is cleared at the start of every call and
//    every other byte a call reads is written by that call first.  Calls whose
//    work overlapped on the GPU would race on the array, so each call waits
//    for its own work to finish before returning and calls are serialised by a
//    process-wide lock;
//  - the first call on a device looks up the array's device address (with
//    that device current) and caches it.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/minhashcuda.h"
#include "../../include/minhashcuda_b200.h"
#include "wmh_internal.h"

namespace {

constexpr size_t kNoallocScratchBytes = static_cast<size_t>(8) << 20;
constexpr uint32_t kNoallocMaxChunk = 1u << 20;
constexpr int kMaxDevices = 64;

// The scratch itself.  In host code this name is only a stand-in: its device
// address comes from cudaGetSymbolAddress (noalloc_scratch_on below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_noalloc_mu;                  // serialises calls in this process
void *g_noalloc_addr[kMaxDevices] = {};   // device address of the array, per device

size_t round256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Device address of the scratch on `device` (which must be current); looked
// up once per device.  Caller holds g_noalloc_mu.
void *noalloc_scratch_on(int device) {
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return nullptr;
    }
    g_noalloc_addr[device] = p;
  }
  return g_noalloc_addr[device];
}

}  // namespace

extern "C" enum MHCUDAResult mhcuda_calc_device_noalloc(
    const MinhashCudaGenerator *gen, const float *d_weights, const uint32_t *d_cols,
    const uint32_t *d_rows, uint32_t length, uint32_t nnz, uint32_t *d_output, void *stream) {
  if (!gen || !d_rows || !d_output || length == 0 || (nnz && (!d_weights || !d_cols)))
    return mhcudaInvalidArguments;
  mhb::GeneratorView g{};
  if (!mhb::generator_view(gen, &g)) return mhcudaInvalidArguments;
  if (g.device < 0 || g.device >= kMaxDevices) return mhcudaNoSuchDevice;

  // Work decomposition that fits the fixed scratch.
  const uint32_t s_pad = g.s_pad;
  auto util = [&](uint32_t spl) {
    const uint32_t w = 32u * spl, tiles = (s_pad + w - 1) / w;
    return static_cast<double>(s_pad) / (static_cast<double>(tiles) * w);
  };
  mhb::HashPlan plan{};
  plan.spl = util(4) >= 0.75 ? 4 : (util(2) >= 0.75 ? 2 : 1);
  plan.minb = 4;
  plan.ntiles = (s_pad + 32u * plan.spl - 1) / (32u * plan.spl);
  const uint64_t per_chunk = 4 + 2 * static_cast<uint64_t>(s_pad) * (sizeof(float) + sizeof(uint2));
  const uint64_t max_chunks = (kNoallocScratchBytes - 1024) / per_chunk;
  const uint64_t warps = static_cast<uint64_t>(g.sm_count) * 4 * (mhb::kHashBlock / 32);
  uint64_t chunk = (static_cast<uint64_t>(nnz) * plan.ntiles + warps * 8 - 1) / (warps * 8);
  chunk = std::max<uint64_t>(chunk, (static_cast<uint64_t>(nnz) + max_chunks - 1) / max_chunks);
  chunk = std::max<uint64_t>(64, (chunk + 31) & ~31ull);
  if (max_chunks == 0 || chunk > kNoallocMaxChunk) {
    if (g.verbosity > 0)
      printf("mhcuda_calc_device_noalloc: %u nnz x %u samples needs more than the %zu-byte "
             "static scratch\n", nnz, g.samples, kNoallocScratchBytes);
    return mhcudaInvalidArguments;
  }
  plan.chunk = static_cast<uint32_t>(chunk);
  plan.nchunks = nnz == 0 ? 1u : static_cast<uint32_t>((nnz + chunk - 1) / chunk);
  const size_t off_rows = 256;
  const size_t off_ln = round256(off_rows + static_cast<size_t>(plan.nchunks) * 4);
  const size_t off_kt = round256(off_ln + static_cast<size_t>(plan.nchunks) * 2 * s_pad * 4);
  const size_t end = off_kt + static_cast<size_t>(plan.nchunks) * 2 * s_pad * 8;
  if (end > kNoallocScratchBytes) return mhcudaInvalidArguments;

  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  mhb::DeviceGuard on_device(g.device);
  if (!on_device.ok()) return mhcudaNoSuchDevice;
  char *scratch = static_cast<char *>(noalloc_scratch_on(g.device));
  if (!scratch) return mhcudaRuntimeError;
  const cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g.stream;
  const int bps = mhb::hash_blocks_per_sm(plan.spl, plan.minb, s_pad);
  const uint64_t items = static_cast<uint64_t>(plan.nchunks) * plan.ntiles;
  const uint64_t want = (items + mhb::kHashBlock / 32 - 1) / (mhb::kHashBlock / 32);
  plan.grid = static_cast<uint32_t>(
      std::max<uint64_t>(1, std::min<uint64_t>(want, static_cast<uint64_t>(g.sm_count) * bps)));

  mhb::HashArgs a{};
  a.params = g.params;
  a.dim = g.dim;
  a.samples = g.samples;
  a.s_pad = s_pad;
  a.weights = d_weights;
  a.cols = d_cols;
  a.indptr = d_rows;
  a.rows = length;
  a.nnz = nnz;
  a.chunk = plan.chunk;
  a.nchunks = plan.nchunks;
  a.ntiles = plan.ntiles;
  a.status = reinterpret_cast<uint32_t *>(scratch);
  a.chunk_row = reinterpret_cast<uint32_t *>(scratch + off_rows);
  a.part_ln = reinterpret_cast<float *>(scratch + off_ln);
  a.part_kt = reinterpret_cast<uint2 *>(scratch + off_kt);
  a.out = d_output;

  if (cudaMemsetAsync(a.status, 0, sizeof(uint32_t), st) != cudaSuccess ||
      mhb::launch_plan(a, st) != cudaSuccess || mhb::launch_hash(a, plan, st) != cudaSuccess ||
      (plan.nchunks > 1 && mhb::launch_finalize(a, st) != cudaSuccess)) {
    cudaGetLastError();
    return mhcudaRuntimeError;
  }
  uint32_t status = 0;
  if (cudaMemcpyAsync(&status, a.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return mhcudaRuntimeError;
  }
  return status ? mhcudaInvalidArguments : mhcudaSuccess;
}
