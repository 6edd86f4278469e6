// Host engine: generator lifetime, parameter init/IO, the calc drivers and
// the extern "C" entry points of include/minhashcuda.h and
// include/minhashcuda_b200.h.
//
// Replaces the reference's host runtime (minhashcuda.cc of
// src-d/minhashcuda) for one device:
//  - device choice: the lowest present device in the mask, no compute
//    capability filter (minhashcuda.cc:43-110 keeps several and drops CCs it
//    was not built for);
//  - no host binpacking (minhashcuda.cc:457-528): the hash launch cuts work
//    by nnz on the device (hash_kernels.cu);
//  - grow-only device workspace as in minhashcuda.cc:385-455, but sizes and
//    offsets are 64-bit and every launch is checked.
#include <algorithm>
#include <atomic>
#include <cinttypes>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>
#include <curand.h>

#include "../../include/minhashcuda.h"
#include "../../include/minhashcuda_b200.h"
#include "wmh_internal.h"

using mhb::HashArgs;
using mhb::HashPlan;
using mhb::stream_copy;

namespace {

#define MHB_INFO(gen, ...) \
  do { if ((gen)->verbosity > 0) { printf(__VA_ARGS__); fflush(stdout); } } while (0)
#define MHB_DEBUG(gen, ...) \
  do { if ((gen)->verbosity > 1) { printf(__VA_ARGS__); fflush(stdout); } } while (0)

// Makes the generator's device current until the enclosing function returns
// (mhb::DeviceGuard), or returns mhcudaNoSuchDevice.
#define MHB_ON_DEVICE(gen)                                \
  mhb::DeviceGuard device_guard__((gen)->device);         \
  if (!device_guard__.ok()) return mhcudaNoSuchDevice

// Returns `code` from the enclosing function when `call` fails.
#define MHB_CHECK(gen, call, code)                                                  \
  do {                                                                              \
    cudaError_t err__ = (call);                                                     \
    if (err__ != cudaSuccess) {                                                     \
      MHB_INFO(gen, "%s:%d -> %s\n", __FILE__, __LINE__, cudaGetErrorString(err__)); \
      return code;                                                                  \
    }                                                                               \
  } while (0)

struct DevBuf {
  void *ptr = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
  // Grow-only; contents are not preserved across growth.
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && ptr) return cudaSuccess;
    release();
    const size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
      ptr = nullptr;
      cudaGetLastError();
      return e;
    }
    cap = want;
    return cudaSuccess;
  }
  template <typename T>
  T *as() const { return static_cast<T *>(ptr); }
};

struct PinnedBuf {
  void *ptr = nullptr;
  size_t cap = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf &) = delete;
  PinnedBuf &operator=(const PinnedBuf &) = delete;
  ~PinnedBuf() { release(); }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
  }
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && ptr) return cudaSuccess;
    release();
    const size_t want = std::max<size_t>(bytes, 4096);
    cudaError_t e = cudaHostAlloc(&ptr, want, cudaHostAllocPortable);
    if (e != cudaSuccess) {
      ptr = nullptr;
      cudaGetLastError();
      return e;
    }
    cap = want;
    return cudaSuccess;
  }
  template <typename T>
  T *as() const { return static_cast<T *>(ptr); }
};

int env_int(const char *name, int fallback) {
  const char *v = getenv(name);
  if (!v || !*v) return fallback;
  return atoi(v);
}

// A hash-kernel configuration chosen by the autotuner: samples per lane,
// minimum resident blocks per SM (register budget) and items per resident
// warp (chunk granularity).
struct TuneChoice {
  uint32_t spl = 4;
  uint32_t minb = 4;
  uint32_t waves = 32;
};

// The autotuner's two choices for a shape class.  `alone` is the fastest
// candidate of all; `streamed` the fastest with the same samples per lane and
// 4 resident blocks per SM, for the mhcuda_calc pipeline, whose row blocks (up
// to 48M nnz) run beside host<->device copies.  There the budgets with fewer,
// longer-running warps lose: on a 2,000,000-row Zipf matrix that the 2-block
// kernel hashes fastest alone (385 against 415 ms), a pipelined call took
// 428-430 ms with 4 blocks per SM, 437-440 with 3 and 451-453 with 2.
struct TunedShape {
  TuneChoice alone, streamed;
};

// A captured plan/hash/finalize sequence, replayed for identical calls.
struct GraphEntry {
  std::vector<unsigned char> key;
  cudaGraphExec_t exec = nullptr;
};

// A device-resident batch seen by mhcuda_calc_batch_device: its matrix
// descriptors, copied to the device once, and the CUDA graph of its launches
// once the same batch has been hashed twice.
struct BatchEntry {
  std::vector<unsigned char> key;
  DevBuf desc;                    // BatchMatrix[count], then plan_base[count]
  PinnedBuf staging;              // host copy the descriptors were uploaded from
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t used = nullptr;     // after the last launch that read `desc`
  uint32_t seen = 0;
  ~BatchEntry() {
    if (used) cudaEventSynchronize(used);
    if (exec) cudaGraphExecDestroy(exec);
    if (used) cudaEventDestroy(used);
  }
};

}  // namespace

// The generator.  Opaque to callers (minhashcuda.h declares only the tag).
struct MinhashCudaGenerator_ {
  uint32_t dim = 0;
  uint16_t samples = 0;
  int verbosity = 0;
  int device = 0;
  uint32_t s_pad = 0;
  int sm_count = 0;
  float *params = nullptr;  // [dim][3][s_pad]
  cudaStream_t stream = nullptr;

  // Serialises calls on one generator (the reference's generator is not
  // re-entrant either: minhashcuda.cc:27-34 holds mutable buffers).
  mutable std::mutex mu;
  // Grow-only workspace.
  mutable DevBuf d_weights, d_cols, d_indptr, d_out, d_chunk_row, d_part_ln, d_part_kt, d_status;
  mutable PinnedBuf h_status;
  // Row-block pipelines of mhcuda_calc and mhcuda_calc_batch: three slots,
  // each a block's device CSR, hashes and (for pageable caller buffers)
  // pinned staging.
  struct Slot {
    DevBuf w, c, ip, out;
    PinnedBuf hw, hc, hip, hout;
    cudaEvent_t h2d = nullptr, done = nullptr, d2h = nullptr;
    bool busy = false;              // holds an enqueued block
    uint32_t *pending_out = nullptr;  // caller destination of a staged block of hashes
    size_t pending_bytes = 0;
  };
  // Pipelines: calc_pipelined and mhcuda_calc_batch use all three slots, so a
  // block's copy-in never waits for the copy-out of the block two before it
  // (and a batch group's host gather/scatter, as long as its device work,
  // overlaps the groups on either side).
  static constexpr int kPipeSlots = 3, kBatchSlots = 3;
  mutable Slot slots[kBatchSlots];
  mutable cudaStream_t s_in = nullptr, s_out = nullptr;
  // Autotuner results by shape class (see tune_key); read by every planner,
  // including the server's lane threads, hence its own lock.
  mutable std::mutex tune_mu;
  mutable std::unordered_map<uint64_t, TunedShape> tuned;
  // CUDA graphs of mhcuda_calc_device calls, most recent last.
  mutable std::vector<GraphEntry> graphs;
  // Device-resident batches, most recent last, and their batch-wide scratch.
  mutable std::vector<std::unique_ptr<BatchEntry>> batches;
  mutable DevBuf d_chunk_owner, d_batch_plan;
  // Optional timing of every hash-kernel launch with CUDA events recorded on
  // the launch stream (mhcuda_profile / mhcuda_profile_read).
  mutable bool profiling = false;
  mutable std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
  mutable size_t prof_used = 0;

  ~MinhashCudaGenerator_() {
    mhb::DeviceGuard on_device(device);
    if (stream) cudaStreamSynchronize(stream);
    batches.clear();  // waits for the launches that read each batch's descriptors
    d_weights.release(); d_cols.release(); d_indptr.release(); d_out.release();
    d_chunk_row.release(); d_part_ln.release(); d_part_kt.release(); d_status.release();
    h_status.release();
    for (auto &e : prof_events) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    for (auto &sl : slots) {
      if (sl.h2d) cudaEventDestroy(sl.h2d);
      if (sl.done) cudaEventDestroy(sl.done);
      if (sl.d2h) cudaEventDestroy(sl.d2h);
      sl.w.release(); sl.c.release(); sl.ip.release(); sl.out.release();
      sl.hw.release(); sl.hc.release(); sl.hip.release(); sl.hout.release();
    }
    if (s_in) cudaStreamDestroy(s_in);
    if (s_out) cudaStreamDestroy(s_out);
    for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
    d_chunk_owner.release(); d_batch_plan.release();
    if (params) cudaFree(params);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

using Gen = MinhashCudaGenerator_;

// Lowest device named by the mask that exists; mask 0 means device 0.
int pick_device(uint32_t devices) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return -1;
  }
  if (devices == 0) return 0;
  for (int d = 0; d < 32 && d < count; ++d) {
    if (devices & (1u << d)) return d;
  }
  return -1;
}

// Chooses samples-per-lane, chunk size and grid for one launch.
// Key of the autotuner's table: the shape class of a launch (log2 of nnz and
// of the mean row length).
uint64_t tune_key(uint64_t nnz, uint64_t rows) {
  auto lg = [](uint64_t x) {
    uint64_t b = 0;
    while (x > 1) {
      x >>= 1;
      ++b;
    }
    return b;
  };
  const uint64_t avg = rows ? (nnz + rows - 1) / rows : 1;
  return (lg(nnz + 1) << 8) | lg(avg + 1);
}

// The autotuner's choice for launches of this shape class, if it has one
// (streamed: the one for launches beside host<->device copies).
bool tuned_choice(const Gen *gen, uint64_t nnz, uint64_t rows, TuneChoice *out,
                  bool streamed = false) {
  std::lock_guard<std::mutex> lock(gen->tune_mu);
  const auto it = gen->tuned.find(tune_key(nnz, rows));
  if (it == gen->tuned.end()) return false;
  *out = streamed ? it->second.streamed : it->second.alone;
  return true;
}

// min_items: items per resident warp the chunk is capped to give (8 for the
// engine's own calls; the server asks for 2, its launches overlap).
HashPlan make_plan(const Gen *gen, uint64_t nnz, uint64_t rows, const TuneChoice *force = nullptr,
                   uint32_t min_items = 8) {
  HashPlan p{};
  const uint32_t s_pad = gen->s_pad;
  TuneChoice tuned{};
  bool have_tuned = false;
  if (force) {
    tuned = *force;
    have_tuned = true;
  } else {
    have_tuned = tuned_choice(gen, nnz, rows, &tuned);
  }
  int spl = env_int("MHCUDA_B200_SPL", 0);
  if (have_tuned && spl == 0) spl = static_cast<int>(tuned.spl);
  if (spl != 1 && spl != 2 && spl != 4) {
    // Wide tiles amortise the per-nnz overhead (shuffles, addressing, the
    // logf share); narrow tiles give small inputs more warps.  Keep lane
    // utilisation of the last tile >= 3/4.
    const uint64_t evals = nnz * static_cast<uint64_t>(gen->samples);
    spl = 4;
    auto util = [&](int s) {
      const uint32_t w = 32u * s;
      const uint32_t tiles = (s_pad + w - 1) / w;
      return static_cast<double>(s_pad) / (static_cast<double>(tiles) * w);
    };
    if (util(4) < 0.75) spl = util(2) >= 0.75 ? 2 : 1;
    if (evals < (1ull << 26) && spl > 1) spl = 1;  // small inputs: more items
  }
  p.spl = static_cast<uint32_t>(spl);
  p.minb = 4;
  if (p.spl == 4) {
    const int minb = env_int("MHCUDA_B200_MINB", have_tuned ? static_cast<int>(tuned.minb) : 4);
    p.minb = (minb == 3 || minb == 2) ? static_cast<uint32_t>(minb) : 4u;
  }
  const uint32_t tile_w = 32u * p.spl;
  p.ntiles = (s_pad + tile_w - 1) / tile_w;
  const int bps = mhb::hash_blocks_per_sm(p.spl, p.minb, s_pad);
  const uint64_t resident_warps =
      static_cast<uint64_t>(gen->sm_count) * bps * (mhb::kHashBlock / 32);
  const int waves = std::max(
      1, env_int("MHCUDA_B200_WAVES", have_tuned ? static_cast<int>(tuned.waves) : 32));
  const uint64_t target_items = resident_warps * waves;
  uint64_t chunk = (nnz * p.ntiles + target_items - 1) / target_items;
  // Rows shorter than a chunk finish inside it; aim for a few rows per chunk.
  const uint64_t avg_row = rows ? (nnz + rows - 1) / rows : 1;
  chunk = std::max<uint64_t>(chunk, std::min<uint64_t>(4 * avg_row, 1024));
  // Warps take items round-robin (static), so a launch with few items per
  // warp ends on a ragged last wave: keep at least min_items items per
  // resident warp even if rows then span chunks (their partials are merged
  // by finalize).
  {
    const uint64_t want = resident_warps * std::max<uint32_t>(1, min_items);
    chunk = std::min<uint64_t>(chunk, std::max<uint64_t>(64, (nnz * p.ntiles + want - 1) / want));
  }
  const int forced = env_int("MHCUDA_B200_CHUNK", 0);
  if (forced > 0) chunk = static_cast<uint64_t>(forced);
  chunk = std::max<uint64_t>(64, (chunk + 31) & ~31ull);
  chunk = std::min<uint64_t>(chunk, 1u << 24);
  p.chunk = static_cast<uint32_t>(chunk);
  const uint64_t nchunks = nnz == 0 ? 1 : (nnz + chunk - 1) / chunk;
  p.nchunks = static_cast<uint32_t>(nchunks);
  const uint64_t items = nchunks * p.ntiles;
  const uint64_t want_blocks = (items + (mhb::kHashBlock / 32) - 1) / (mhb::kHashBlock / 32);
  const uint64_t max_blocks = static_cast<uint64_t>(gen->sm_count) * bps;
  p.grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min(want_blocks, max_blocks)));
  return p;
}

// Ensures the per-launch workspace and fills the device-side arguments.
MHCUDAResult prepare_launch(const Gen *gen, uint32_t rows, uint32_t nnz, const HashPlan &plan,
                            HashArgs *a) {
  const size_t slots = static_cast<size_t>(plan.nchunks) * 2;
  MHB_CHECK(gen, gen->d_chunk_row.ensure(static_cast<size_t>(plan.nchunks) * 4),
            mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, gen->d_part_ln.ensure(slots * gen->s_pad * sizeof(float)),
            mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, gen->d_part_kt.ensure(slots * gen->s_pad * sizeof(uint2)),
            mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, gen->d_status.ensure(sizeof(uint32_t)), mhcudaMemoryAllocationFailure);
  a->params = gen->params;
  a->dim = gen->dim;
  a->samples = gen->samples;
  a->s_pad = gen->s_pad;
  a->rows = rows;
  a->nnz = nnz;
  a->chunk = plan.chunk;
  a->nchunks = plan.nchunks;
  a->ntiles = plan.ntiles;
  a->chunk_row = gen->d_chunk_row.as<uint32_t>();
  a->part_ln = gen->d_part_ln.as<float>();
  a->part_kt = gen->d_part_kt.as<uint2>();
  a->status = gen->d_status.as<uint32_t>();
  return mhcudaSuccess;
}

MHCUDAResult enqueue_hash(const Gen *gen, const HashArgs &a, const HashPlan &plan,
                          cudaStream_t stream, bool clear_status = true) {
  if (clear_status)
    MHB_CHECK(gen, cudaMemsetAsync(a.status, 0, sizeof(uint32_t), stream), mhcudaRuntimeError);
  MHB_CHECK(gen, mhb::launch_plan(a, stream), mhcudaRuntimeError);
  std::pair<cudaEvent_t, cudaEvent_t> *ev = nullptr;
  if (gen->profiling) {
    if (gen->prof_used == gen->prof_events.size()) {
      std::pair<cudaEvent_t, cudaEvent_t> e{nullptr, nullptr};
      MHB_CHECK(gen, cudaEventCreate(&e.first), mhcudaRuntimeError);
      MHB_CHECK(gen, cudaEventCreate(&e.second), mhcudaRuntimeError);
      gen->prof_events.push_back(e);
    }
    ev = &gen->prof_events[gen->prof_used++];
    MHB_CHECK(gen, cudaEventRecord(ev->first, stream), mhcudaRuntimeError);
  }
  MHB_CHECK(gen, mhb::launch_hash(a, plan, stream), mhcudaRuntimeError);
  if (ev) MHB_CHECK(gen, cudaEventRecord(ev->second, stream), mhcudaRuntimeError);
  if (plan.nchunks > 1) MHB_CHECK(gen, mhb::launch_finalize(a, stream), mhcudaRuntimeError);
  return mhcudaSuccess;
}

MHCUDAResult read_status(const Gen *gen, cudaStream_t stream) {
  MHB_CHECK(gen, gen->h_status.ensure(sizeof(uint32_t)), mhcudaMemoryAllocationFailure);
  uint32_t *h = gen->h_status.as<uint32_t>();
  MHB_CHECK(gen, cudaMemcpyAsync(h, gen->d_status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 stream),
            mhcudaMemoryCopyError);
  MHB_CHECK(gen, cudaStreamSynchronize(stream), mhcudaRuntimeError);
  if (*h != 0) {
    MHB_INFO(gen, "invalid CSR input (status 0x%x)\n", *h);
    return mhcudaInvalidArguments;
  }
  return mhcudaSuccess;
}

// True when `p` is page-locked host memory the copy engines can read directly.
bool is_pinned(const void *p) {
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeHost;
}

// Host threads for staging copies and conversions: one per core up to 16
// (a 16-core host stages pageable float64/int64 input 1.36x faster with 16
// than with 8); MHCUDA_B200_HOST_THREADS overrides.
unsigned host_threads() {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int forced = env_int("MHCUDA_B200_HOST_THREADS", 0);
  return forced > 0 ? static_cast<unsigned>(forced) : std::min(16u, hw);
}

// memcpy split over a few threads for large blocks (host bandwidth for the
// pinned staging of pageable caller buffers).
void par_memcpy(void *dst, const void *src, size_t bytes) {
  const size_t kSplit = static_cast<size_t>(8) << 20;
  const unsigned n = bytes < kSplit ? 1u : host_threads();
  if (n == 1) {
    stream_copy(dst, src, bytes);
    return;
  }
  const size_t part = (((bytes + n - 1) / n) + 4095) & ~static_cast<size_t>(4095);
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < n; ++t) {
    const size_t off = t * part;
    if (off >= bytes) break;
    const size_t len = std::min(part, bytes - off);
    pool.emplace_back([=]() {
      stream_copy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off, len);
    });
  }
  for (auto &th : pool) th.join();
}

// Creates the copy streams and slot events of the pipelines on first use.
cudaError_t batch_streams(const Gen *gen) {
  if (gen->s_in) return cudaSuccess;
  cudaError_t e = cudaStreamCreateWithFlags(&gen->s_in, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&gen->s_out, cudaStreamNonBlocking);
  for (auto &sl : gen->slots) {
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.h2d, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.d2h, cudaEventDisableTiming);
  }
  return e;
}

// Inputs with at least this many nnz go through the row-block pipeline.
constexpr uint64_t kPipelineMinNnz = 16ull << 20;

// mhcuda_calc for large inputs: rows are cut into blocks of about
// `block_nnz` entries; block i's hashes run on the generator stream while
// block i+1 is copied in on s_in and block i-1's hashes are copied out on
// s_out.  Caller buffers that are page-locked are copied directly; pageable
// ones go through pinned staging filled by host threads.
// A caller's host CSR: float32 or float64 weights, 32-bit (uint32/int32 bits)
// or 64-bit columns, uint32 offsets (absolute: weights[rows[0]] is the first
// entry).
struct HostCsr {
  const void *weights;
  bool w64;
  const void *cols;
  int cols64;  // 0: 32-bit, 1: int64, 2: uint64
  const uint32_t *rows;
  bool native() const { return !w64 && cols64 == 0; }
};

// Runs f(begin, end) over [0, n), split over up to 8 host threads once n
// reaches `split`.
template <typename F>
void par_for(size_t n, size_t split, F f) {
  const unsigned k = n < split ? 1u : host_threads();
  if (k == 1) {
    if (n) f(size_t{0}, n);
    return;
  }
  const size_t part = (((n + k - 1) / k) + 1023) & ~static_cast<size_t>(1023);
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < k; ++t) {
    const size_t b = t * part;
    if (b >= n) break;
    const size_t e = std::min(n, b + part);
    pool.emplace_back([=]() { f(b, e); });
  }
  for (auto &th : pool) th.join();
}

// Stages entries [b0, b0 + n) of the caller's weights and columns into the
// page-locked float32/uint32 buffers, converting on the way: float64 rounds
// to nearest; a 64-bit column outside [0, 2^32) becomes 0xFFFFFFFF, which no
// dim admits, so the device check rejects it instead of a wrapped value
// passing.
void stage_weights(const HostCsr &in, uint64_t b0, size_t n, float *w) {
  constexpr size_t kSplit = size_t{2} << 20;
  if (in.w64) {
    const double *src = static_cast<const double *>(in.weights) + b0;
    par_for(n, kSplit, [=](size_t b, size_t e) { mhb::convert_f64_to_f32(w + b, src + b, e - b); });
  } else {
    par_memcpy(w, static_cast<const float *>(in.weights) + b0, n * sizeof(float));
  }
}

void stage_cols(const HostCsr &in, uint64_t b0, size_t n, uint32_t *c) {
  constexpr size_t kSplit = size_t{2} << 20;
  if (in.cols64) {
    // int64 and uint64 alike: a negative int64 has its high bits set.
    const uint64_t *src = static_cast<const uint64_t *>(in.cols) + b0;
    par_for(n, kSplit, [=](size_t b, size_t e) { mhb::convert_i64_to_u32(c + b, src + b, e - b); });
  } else {
    par_memcpy(c, static_cast<const uint32_t *>(in.cols) + b0, n * sizeof(uint32_t));
  }
}

// Packs the caller's 32-bit columns [b0, b0 + n) into page-locked lo/hi
// arrays (mhb::pack_cols, split over host threads at even entries).  Returns
// false if some column needs more than 16 + hi_bits bits; the block then
// crosses the link unpacked.
bool stage_packed_cols(const HostCsr &in, uint64_t b0, size_t n, uint16_t *lo, uint8_t *hi,
                       int hi_bits) {
  constexpr size_t kSplit = size_t{2} << 20;
  const uint32_t *src = static_cast<const uint32_t *>(in.cols) + b0;
  std::atomic<bool> fits{true};
  par_for(n, kSplit, [&, src, lo, hi](size_t b, size_t e) {
    if (!mhb::pack_cols(src + b, e - b, lo + b, hi + (hi_bits == 4 ? b / 2 : b), hi_bits))
      fits.store(false, std::memory_order_relaxed);
  });
  return fits.load();
}

// Byte offset of the high parts behind `n` low halves in a packed-column
// buffer (16-byte aligned for the kernel's bulk copies).
size_t packed_hi_offset(size_t n) { return (2 * n + 255) & ~static_cast<size_t>(255); }

// Per-block timeline of calc_pipelined, written when MHCUDA_B200_PIPE_TRACE
// names a file: one CSV line per row block with its nnz and, in ms from the
// start of the call's first copy-in, the start and end of its copy-in,
// hashing (plan + hash + finalize) and copy-out, from CUDA events on the
// copy-in, generator and copy-out streams.  Lines are appended; `call`
// counts the traced calls of the process.
class PipeTrace {
 public:
  enum Point { kH2dStart, kH2dEnd, kHashStart, kHashEnd, kD2hStart, kD2hEnd, kPoints };
  explicit PipeTrace(size_t blocks) {
    const char *p = getenv("MHCUDA_B200_PIPE_TRACE");
    if (!p || !*p) return;
    path_ = p;
    ev_.assign(blocks * kPoints, nullptr);
    nnz_.assign(blocks, 0);
    for (auto &e : ev_)
      if (cudaEventCreate(&e) != cudaSuccess) {
        e = nullptr;
        path_.clear();  // no trace rather than a partial one
      }
  }
  ~PipeTrace() {
    for (auto &e : ev_)
      if (e) cudaEventDestroy(e);
  }
  bool on() const { return !path_.empty(); }
  void mark(size_t block, Point pt, cudaStream_t s) {
    if (on()) cudaEventRecord(ev_[block * kPoints + pt], s);
  }
  void nnz(size_t block, uint64_t n) {
    if (on()) nnz_[block] = n;
  }
  // After every block has been retired (their events have completed).
  void write(size_t issued) {
    if (!on() || issued == 0) return;
    static std::atomic<int> calls{0};
    const int call = calls++;
    FILE *f = fopen(path_.c_str(), "a");
    if (!f) return;
    if (ftell(f) == 0) fprintf(f, "call,block,nnz,h2d_start,h2d_end,hash_start,hash_end,d2h_start,d2h_end\n");
    for (size_t b = 0; b < issued; ++b) {
      fprintf(f, "%d,%zu,%" PRIu64, call, b, nnz_[b]);
      for (int pt = 0; pt < kPoints; ++pt) {
        float ms = -1.0f;
        if (cudaEventSynchronize(ev_[b * kPoints + pt]) != cudaSuccess ||
            cudaEventElapsedTime(&ms, ev_[0], ev_[b * kPoints + pt]) != cudaSuccess)
          ms = -1.0f;
        fprintf(f, ",%.3f", ms);
      }
      fprintf(f, "\n");
    }
    fclose(f);
  }

 private:
  std::string path_;
  std::vector<cudaEvent_t> ev_;
  std::vector<uint64_t> nnz_;
};

MHCUDAResult calc_pipelined(const Gen *gen, const HostCsr &in, uint32_t length,
                            uint32_t *output) {
  const cudaStream_t st = gen->stream;
  MHB_CHECK(gen, batch_streams(gen), mhcudaRuntimeError);
  const uint32_t *rows = in.rows;
  const uint64_t nnz = static_cast<uint64_t>(rows[length]) - rows[0];
  // Page-locked native arrays are copied straight from the caller; anything
  // else is staged (and converted) block by block.
  const bool pin_in = in.native() && is_pinned(in.weights) && is_pinned(in.cols) &&
                      is_pinned(rows);
  const bool pin_out = is_pinned(output);
  // Pageable 32-bit columns are staged by host threads anyway: they are
  // packed on the way (16 low bits plus 4 high bits when dim <= 2^20, 8 when
  // dim <= 2^24), which writes 2.5-3 instead of 4 bytes per entry to the
  // staging and sends 6.5-7 instead of 8 bytes per entry over the link.
  // Page-locked columns are copied by the DMA engine straight from the
  // caller: packing them would add host memory traffic the copy does not
  // have (measured on 2.8e9 entries: 448 ms per step unpacked, 462 / 472 /
  // 480 / 486 ms with 2, 4, 6 or 8 of every 8 blocks packed), so they cross
  // as they are.
  const int pack_bits =
      (in.cols64 == 0 && !pin_in && env_int("MHCUDA_B200_NO_PACK", 0) == 0)
          ? (gen->dim <= (1u << 20) ? 4 : (gen->dim <= (1u << 24) ? 8 : 0))
          : 0;
  // Block size once the pipeline has ramped up.  A block's copy-in (8 B per
  // nnz over a Gen5 x16 link) and its hashing (128 samples) take about as
  // long, so the kernel waits for every block that is larger than the one
  // before it; a smaller steady block shortens the ramp, a larger one has
  // fewer launch tails.  Measured on 2.8e9 page-locked nnz (ms per call):
  // 32M 434-437, 48M 428-432, 64M 429-436, 96M 438-441, and 447-450 for the
  // earlier blocks that grew by 8% up to 256M.  Pageable inputs go through
  // pinned staging, which is cheaper to allocate (and re-fill) in blocks of
  // at most 32M.
  uint64_t block_nnz =
      pin_in ? std::min<uint64_t>(std::max<uint64_t>(nnz / 8, 8ull << 20), 48ull << 20)
             : std::min<uint64_t>(std::max<uint64_t>(nnz / 16, 4ull << 20), 32ull << 20);
  const int forced = env_int("MHCUDA_B200_BLOCK_NNZ", 0);
  if (forced > 0) block_nnz = static_cast<uint64_t>(forced);
  const size_t row_bytes = static_cast<size_t>(gen->samples) * 2 * sizeof(uint32_t);
  MHB_CHECK(gen, gen->d_status.ensure(sizeof(uint32_t)), mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, cudaMemsetAsync(gen->d_status.ptr, 0, sizeof(uint32_t), st), mhcudaRuntimeError);
  // The blocks are cut from one matrix: a variant the autotuner chose for the
  // whole matrix's shape applies to each of them (their own, smaller shape
  // classes were never timed), its choice for launches beside copies.
  TuneChoice whole{};
  const TuneChoice *force = tuned_choice(gen, nnz, length, &whole, true) ? &whole : nullptr;

  // Finishes a slot: waits for its hashes and moves staged ones to the caller.
  auto retire = [&](Gen::Slot &sl) -> MHCUDAResult {
    if (!sl.busy) return mhcudaSuccess;
    MHB_CHECK(gen, cudaEventSynchronize(sl.d2h), mhcudaMemoryCopyError);
    if (sl.pending_out) par_memcpy(sl.pending_out, sl.hout.ptr, sl.pending_bytes);
    sl.pending_out = nullptr;
    sl.busy = false;
    return mhcudaSuccess;
  };

  // Blocks [r0, r1): as many rows as fit the block's nnz (at least one).
  // Hashing cannot start before the first block has crossed the bus, so the
  // first block is small -- 16M nnz, still a few waves of warp items -- and
  // later ones double up to block_nnz, where they stay.
  // MHCUDA_B200_BLOCK_NNZ gives constant blocks.
  struct Block {
    uint32_t r0, r1;
  };
  std::vector<Block> blocks;
  {
    uint64_t cur = forced > 0 ? block_nnz
                              : std::min(block_nnz, std::max<uint64_t>(block_nnz / 32, 16ull << 20));
    const double growth = forced > 0 ? 1.0 : 2.0;
    for (uint32_t r0 = 0; r0 < length;) {
      const uint64_t limit = static_cast<uint64_t>(rows[r0]) + cur;
      uint32_t r1 = static_cast<uint32_t>(
          std::upper_bound(rows + r0 + 1, rows + length + 1, limit,
                           [](uint64_t v, uint32_t x) { return v < x; }) - rows) - 1;
      r1 = std::max(r1, r0 + 1);
      blocks.push_back(Block{r0, r1});
      r0 = r1;
      cur = std::min<uint64_t>(block_nnz, static_cast<uint64_t>(static_cast<double>(cur) * growth));
    }
    // Only the last block's copy-out is left once hashing ends: end on a
    // small block.
    const uint64_t tail = std::max<uint64_t>(block_nnz / 16, 1ull << 20);
    const Block last = blocks.back();
    if (forced <= 0 && static_cast<uint64_t>(rows[last.r1]) - rows[last.r0] > 2 * tail) {
      const uint64_t target = static_cast<uint64_t>(rows[last.r1]) - tail;
      const uint32_t mid = static_cast<uint32_t>(
          std::upper_bound(rows + last.r0 + 1, rows + last.r1, target,
                           [](uint64_t v, uint32_t x) { return v < x; }) - rows);
      if (mid > last.r0 && mid < last.r1) {
        blocks.back().r1 = mid;
        blocks.push_back(Block{mid, last.r1});
      }
    }
  }
  // Size the slots and the launch scratch once for the largest block: growing
  // a buffer between blocks would free device memory, which waits for all
  // work in flight and stalls the pipeline.
  {
    uint64_t max_n = 0, max_len = 0;
    uint32_t max_chunks = 1;
    for (const Block &b : blocks) {
      const uint64_t n = static_cast<uint64_t>(rows[b.r1]) - rows[b.r0];
      max_n = std::max(max_n, n);
      max_len = std::max<uint64_t>(max_len, b.r1 - b.r0);
      max_chunks = std::max(max_chunks, make_plan(gen, n, b.r1 - b.r0, force).nchunks);
    }
    for (int k = 0; k < Gen::kPipeSlots; ++k) {
      Gen::Slot &sl = gen->slots[k];
      MHB_CHECK(gen, sl.w.ensure(max_n * 4 + 16), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.c.ensure(max_n * 4 + 512), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.ip.ensure((max_len + 1) * 4), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.out.ensure(max_len * row_bytes), mhcudaMemoryAllocationFailure);
      if (!pin_in) {
        MHB_CHECK(gen, sl.hw.ensure(max_n * 4), mhcudaMemoryAllocationFailure);
        MHB_CHECK(gen, sl.hip.ensure((max_len + 1) * 4), mhcudaMemoryAllocationFailure);
      }
      if (!pin_in || pack_bits)
        MHB_CHECK(gen, sl.hc.ensure(max_n * 4 + 512), mhcudaMemoryAllocationFailure);
      if (!pin_out) MHB_CHECK(gen, sl.hout.ensure(max_len * row_bytes), mhcudaMemoryAllocationFailure);
    }
    HashPlan big{};
    big.nchunks = max_chunks;
    HashArgs unused{};
    const MHCUDAResult pr = prepare_launch(gen, 0, 0, big, &unused);
    if (pr != mhcudaSuccess) return pr;
  }

  MHCUDAResult r = mhcudaSuccess;
  PipeTrace trace(blocks.size());
  size_t issued = 0;
  for (uint32_t i = 0; i < blocks.size() && r == mhcudaSuccess; ++i) {
    const uint32_t r0 = blocks[i].r0, r1 = blocks[i].r1;
    Gen::Slot &sl = gen->slots[i % Gen::kPipeSlots];
    r = retire(sl);
    if (r != mhcudaSuccess) break;
    const uint32_t len = r1 - r0;
    const uint32_t b0 = rows[r0];
    const uint32_t n = rows[r1] - b0;
    MHB_CHECK(gen, sl.w.ensure(static_cast<size_t>(n) * 4 + 16), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.c.ensure(static_cast<size_t>(n) * 4 + 512), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.ip.ensure((static_cast<size_t>(len) + 1) * 4), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.out.ensure(len * row_bytes), mhcudaMemoryAllocationFailure);
    const void *src_w = nullptr, *src_c = nullptr, *src_i = rows + r0;
    if (!pin_in || pack_bits)
      MHB_CHECK(gen, sl.hc.ensure(static_cast<size_t>(n) * 4 + 512), mhcudaMemoryAllocationFailure);
    const size_t hi_off = packed_hi_offset(n);
    const size_t hi_bytes = pack_bits == 4 ? (static_cast<size_t>(n) + 1) / 2 : n;
    const bool packed =
        pack_bits && n &&
        stage_packed_cols(in, b0, n, sl.hc.as<uint16_t>(), sl.hc.as<uint8_t>() + hi_off, pack_bits);
    if (pin_in) {
      src_w = static_cast<const float *>(in.weights) + b0;
      src_c = static_cast<const uint32_t *>(in.cols) + b0;
    } else {
      MHB_CHECK(gen, sl.hw.ensure(static_cast<size_t>(n) * 4), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.hip.ensure((static_cast<size_t>(len) + 1) * 4),
                mhcudaMemoryAllocationFailure);
      stage_weights(in, b0, n, static_cast<float *>(sl.hw.ptr));
      if (!packed) stage_cols(in, b0, n, static_cast<uint32_t *>(sl.hc.ptr));
      memcpy(sl.hip.ptr, src_i, (static_cast<size_t>(len) + 1) * 4);
      src_w = sl.hw.ptr;
      src_c = sl.hc.ptr;
      src_i = sl.hip.ptr;
    }
    trace.nnz(i, n);
    trace.mark(i, PipeTrace::kH2dStart, gen->s_in);
    MHB_CHECK(gen, cudaMemcpyAsync(sl.ip.ptr, src_i, (static_cast<size_t>(len) + 1) * 4,
                                   cudaMemcpyHostToDevice, gen->s_in),
              mhcudaMemoryCopyError);
    if (n) {
      MHB_CHECK(gen, cudaMemcpyAsync(sl.w.ptr, src_w, static_cast<size_t>(n) * 4,
                                     cudaMemcpyHostToDevice, gen->s_in),
                mhcudaMemoryCopyError);
      if (packed) {
        MHB_CHECK(gen, cudaMemcpyAsync(sl.c.ptr, sl.hc.ptr, static_cast<size_t>(n) * 2,
                                       cudaMemcpyHostToDevice, gen->s_in),
                  mhcudaMemoryCopyError);
        MHB_CHECK(gen, cudaMemcpyAsync(sl.c.as<char>() + hi_off, sl.hc.as<char>() + hi_off,
                                       hi_bytes, cudaMemcpyHostToDevice, gen->s_in),
                  mhcudaMemoryCopyError);
      } else {
        MHB_CHECK(gen, cudaMemcpyAsync(sl.c.ptr, src_c, static_cast<size_t>(n) * 4,
                                       cudaMemcpyHostToDevice, gen->s_in),
                  mhcudaMemoryCopyError);
      }
    }
    trace.mark(i, PipeTrace::kH2dEnd, gen->s_in);
    MHB_CHECK(gen, cudaEventRecord(sl.h2d, gen->s_in), mhcudaRuntimeError);
    MHB_CHECK(gen, cudaStreamWaitEvent(st, sl.h2d, 0), mhcudaRuntimeError);
    trace.mark(i, PipeTrace::kHashStart, st);
    const HashPlan plan = make_plan(gen, n, len, force);
    HashArgs a{};
    r = prepare_launch(gen, len, n, plan, &a);
    if (r != mhcudaSuccess) break;
    a.weights = sl.w.as<float>();
    if (packed) {
      a.cols_lo = sl.c.as<uint16_t>();
      a.cols_hi = sl.c.as<uint8_t>() + hi_off;
      a.col_hi_bits = static_cast<uint32_t>(pack_bits);
    } else {
      a.cols = sl.c.as<uint32_t>();
    }
    a.indptr = sl.ip.as<uint32_t>();
    a.out = sl.out.as<uint32_t>();
    r = enqueue_hash(gen, a, plan, st, /*clear_status=*/false);
    if (r != mhcudaSuccess) break;
    trace.mark(i, PipeTrace::kHashEnd, st);
    MHB_CHECK(gen, cudaEventRecord(sl.done, st), mhcudaRuntimeError);
    MHB_CHECK(gen, cudaStreamWaitEvent(gen->s_out, sl.done, 0), mhcudaRuntimeError);
    trace.mark(i, PipeTrace::kD2hStart, gen->s_out);
    uint32_t *dst = output + static_cast<size_t>(r0) * gen->samples * 2;
    if (pin_out) {
      MHB_CHECK(gen, cudaMemcpyAsync(dst, sl.out.ptr, len * row_bytes, cudaMemcpyDeviceToHost,
                                     gen->s_out),
                mhcudaMemoryCopyError);
    } else {
      MHB_CHECK(gen, sl.hout.ensure(len * row_bytes), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, cudaMemcpyAsync(sl.hout.ptr, sl.out.ptr, len * row_bytes,
                                     cudaMemcpyDeviceToHost, gen->s_out),
                mhcudaMemoryCopyError);
      sl.pending_out = dst;
      sl.pending_bytes = len * row_bytes;
    }
    trace.mark(i, PipeTrace::kD2hEnd, gen->s_out);
    MHB_CHECK(gen, cudaEventRecord(sl.d2h, gen->s_out), mhcudaRuntimeError);
    sl.busy = true;
    issued = i + 1;
    MHB_DEBUG(gen, "block %u: rows [%u, %u) nnz %u chunk %u\n", i, r0, r1, n, plan.chunk);
  }
  for (auto &sl : gen->slots) {
    const MHCUDAResult rr = retire(sl);
    if (r == mhcudaSuccess) r = rr;
  }
  if (r != mhcudaSuccess) {
    cudaDeviceSynchronize();
    return r;
  }
  trace.write(issued);
  return read_status(gen, st);
}

// Scratch per buffer when the [samples][dim] parameter streams are handled a
// block of sample rows at a time (init, retrieve, assign).
constexpr uint64_t kParamChunkBytes = 1ull << 30;

// Sample rows per block: about kParamChunkBytes of floats, whole 8-row groups
// (32-byte write segments in the table) when a block holds 8 rows or more.
// MHCUDA_B200_PARAM_CHUNK_ROWS overrides.
uint32_t param_chunk_rows(uint32_t dim, uint32_t samples) {
  const int forced = env_int("MHCUDA_B200_PARAM_CHUNK_ROWS", 0);
  uint64_t rows = forced > 0 ? static_cast<uint64_t>(forced)
                             : kParamChunkBytes / (static_cast<uint64_t>(dim) * sizeof(float));
  if (forced <= 0 && rows >= 8) rows &= ~uint64_t{7};
  return static_cast<uint32_t>(std::min<uint64_t>(std::max<uint64_t>(rows, 1), samples));
}

// Fills the table from `seed` as minhashcuda.cc:179-199 does: one cuRAND
// generator of type CURAND_RNG_PSEUDO_DEFAULT draws five runs of dim*samples
// uniforms U1..U5, and rs = -logf(U2*U1), ln_cs = logf(-logf(U3*U4)),
// betas = U5, each run in [samples][dim] order.  The runs are not
// materialised whole: two generators with that seed start at the absolute
// offsets of a run pair (curandSetGeneratorOffset: draws k and k+1 begin at
// k*n and (k+1)*n), each produces its run a block of sample rows at a time,
// and every block is combined and transposed into the table at once.  Values
// at an absolute offset do not depend on how the sequence is split into
// calls, so the table equals the reference's bit for bit with scratch of two
// blocks instead of two full runs (2 x 17 GB at 2^24 x 256).
MHCUDAResult init_params(Gen *gen, uint32_t seed) {
  const uint32_t D = gen->dim, S = gen->samples, P = gen->s_pad;
  const uint64_t n = static_cast<uint64_t>(D) * S;
  const uint32_t rows = param_chunk_rows(D, S);
  const size_t block = static_cast<size_t>(rows) * D;
  DevBuf a, b;
  MHB_CHECK(gen, a.ensure(block * sizeof(float)), mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, b.ensure(block * sizeof(float)), mhcudaMemoryAllocationFailure);
  curandGenerator_t rng[2] = {nullptr, nullptr};
  auto finish = [&](MHCUDAResult code) {
    for (curandGenerator_t g : rng)
      if (g) curandDestroyGenerator(g);
    return code;
  };
  for (curandGenerator_t &g : rng) {
    if (curandCreateGenerator(&g, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS) {
      g = nullptr;
      return finish(mhcudaRuntimeError);
    }
    if (curandSetStream(g, gen->stream) != CURAND_STATUS_SUCCESS ||
        curandSetPseudoRandomGeneratorSeed(g, seed) != CURAND_STATUS_SUCCESS)
      return finish(mhcudaRuntimeError);
  }
  struct Pass {
    mhb::PairOp op;
    uint32_t which;     // table slot: 0 rs, 1 ln_cs, 2 betas
    uint64_t first;     // index of the first uniform run it consumes
    bool pair;          // consumes runs first and first+1
  };
  const Pass passes[3] = {{mhb::PairOp::kGamma, 0, 0, true},
                          {mhb::PairOp::kLogGamma, 1, 2, true},
                          {mhb::PairOp::kCopy, 2, 4, false}};
  float *A = a.as<float>(), *B = b.as<float>();
  for (const Pass &p : passes) {
    if (curandSetGeneratorOffset(rng[0], p.first * n) != CURAND_STATUS_SUCCESS ||
        (p.pair && curandSetGeneratorOffset(rng[1], (p.first + 1) * n) != CURAND_STATUS_SUCCESS))
      return finish(mhcudaRuntimeError);
    for (uint32_t s0 = 0; s0 < S; s0 += rows) {
      const uint32_t cnt = std::min(rows, S - s0);
      const size_t len = static_cast<size_t>(cnt) * D;
      if (curandGenerateUniform(rng[0], A, len) != CURAND_STATUS_SUCCESS ||
          (p.pair && curandGenerateUniform(rng[1], B, len) != CURAND_STATUS_SUCCESS))
        return finish(mhcudaRuntimeError);
      if (mhb::launch_pack_params(A, p.pair ? B : nullptr, p.op, p.which, D, s0, cnt, P,
                                  gen->params, gen->stream) != cudaSuccess)
        return finish(mhcudaRuntimeError);
    }
  }
  if (cudaStreamSynchronize(gen->stream) != cudaSuccess) return finish(mhcudaRuntimeError);
  return finish(mhcudaSuccess);
}

}  // namespace

namespace mhb {

namespace {

// cuCtxGetCurrent / cuCtxSetCurrent, looked up through the runtime so that
// the library does not link the driver library directly.
using CtxGetFn = int (*)(void **);
using CtxSetFn = int (*)(void *);

struct CtxFns {
  CtxGetFn get = nullptr;
  CtxSetFn set = nullptr;
};

const CtxFns &ctx_fns() {
  static const CtxFns fns = []() {
    CtxFns f;
    void *g = nullptr, *s = nullptr;
    cudaDriverEntryPointQueryResult qg{}, qs{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &g, cudaEnableDefault, &qg) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxSetCurrent", &s, cudaEnableDefault, &qs) == cudaSuccess &&
        qg == cudaDriverEntryPointSuccess && qs == cudaDriverEntryPointSuccess) {
      f.get = reinterpret_cast<CtxGetFn>(g);
      f.set = reinterpret_cast<CtxSetFn>(s);
    }
    cudaGetLastError();
    return f;
  }();
  return fns;
}

}  // namespace

DeviceGuard::DeviceGuard(int device) {
  const CtxFns &f = ctx_fns();
  void *ctx = nullptr;
  if (f.get && f.get(&ctx) == 0) had_context_ = ctx != nullptr;
  if (cudaGetDevice(&prev_) != cudaSuccess) {
    cudaGetLastError();
    prev_ = -1;
  }
  if (prev_ == device && had_context_) {
    ok_ = true;
    return;
  }
  ok_ = cudaSetDevice(device) == cudaSuccess;
  if (!ok_) {
    cudaGetLastError();
    return;
  }
  changed_ = prev_ != device || !had_context_;
}

DeviceGuard::~DeviceGuard() {
  if (!changed_) return;
  const CtxFns &f = ctx_fns();
  if (!had_context_ && f.set) {
    f.set(nullptr);
  } else if (prev_ >= 0) {
    cudaSetDevice(prev_);
  }
  cudaGetLastError();
}

HashPlan plan_for_generator(const MinhashCudaGenerator_ *gen, uint64_t nnz, uint64_t rows,
                            uint32_t min_items) {
  return make_plan(gen, nnz, rows, nullptr, min_items);
}

bool generator_view(const MinhashCudaGenerator_ *gen, GeneratorView *view) {
  if (!gen || !view) return false;
  view->params = gen->params;
  view->dim = gen->dim;
  view->samples = gen->samples;
  view->s_pad = gen->s_pad;
  view->device = gen->device;
  view->sm_count = gen->sm_count;
  view->verbosity = gen->verbosity;
  view->stream = gen->stream;
  return true;
}

}  // namespace mhb

extern "C" {

MinhashCudaGenerator *mhcuda_init(uint32_t dim, uint16_t samples, uint32_t seed, int deferred,
                                  uint32_t devices, int verbosity, enum MHCUDAResult *status) {
  auto set = [&](MHCUDAResult r) {
    if (status) *status = r;
  };
  if (dim == 0 || samples == 0) {
    set(mhcudaInvalidArguments);
    return nullptr;
  }
  const int dev = pick_device(devices);
  if (dev < 0) {
    set(mhcudaNoSuchDevice);
    return nullptr;
  }
  mhb::DeviceGuard on_device(dev);
  if (!on_device.ok()) {
    set(mhcudaNoSuchDevice);
    return nullptr;
  }
  std::unique_ptr<Gen> gen(new Gen());
  gen->dim = dim;
  gen->samples = samples;
  gen->verbosity = verbosity;
  gen->device = dev;
  gen->s_pad = mhb::padded_samples(samples);
  if (cudaDeviceGetAttribute(&gen->sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    set(mhcudaNoSuchDevice);
    return nullptr;
  }
  MHB_DEBUG(gen.get(), "mhcuda_init: dim=%" PRIu32 " samples=%" PRIu16 " seed=%" PRIu32
            " deferred=%d device=%d\n", dim, samples, seed, deferred, dev);
  if (cudaStreamCreateWithFlags(&gen->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set(mhcudaRuntimeError);
    return nullptr;
  }
  const size_t table = static_cast<size_t>(dim) * 3 * gen->s_pad * sizeof(float);
  if (cudaMalloc(&gen->params, table) != cudaSuccess) {
    cudaGetLastError();
    gen->params = nullptr;
    MHB_INFO(gen.get(), "failed to allocate %zu bytes for the parameter table\n", table);
    set(mhcudaMemoryAllocationFailure);
    return nullptr;
  }
  // Zero fill: padding samples and, with `deferred`, the whole table.
  if (cudaMemsetAsync(gen->params, 0, table, gen->stream) != cudaSuccess) {
    set(mhcudaRuntimeError);
    return nullptr;
  }
  if (!deferred) {
    const MHCUDAResult r = init_params(gen.get(), seed);
    if (r != mhcudaSuccess) {
      set(r);
      return nullptr;
    }
  }
  if (cudaStreamSynchronize(gen->stream) != cudaSuccess) {
    set(mhcudaRuntimeError);
    return nullptr;
  }
  if (verbosity > 1) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    printf("GPU #%d memory: used %zu bytes, free %zu bytes, total %zu bytes\n", dev,
           total_b - free_b, free_b, total_b);
  }
  set(mhcudaSuccess);
  return gen.release();
}

MinhashCudaGeneratorParameters mhcuda_get_parameters(const MinhashCudaGenerator *gen) {
  if (!gen) return MinhashCudaGeneratorParameters{};
  MinhashCudaGeneratorParameters p{};
  p.dim = gen->dim;
  p.samples = gen->samples;
  p.verbosity = gen->verbosity;
  return p;
}

enum MHCUDAResult mhcuda_retrieve_random_vars(const MinhashCudaGenerator *gen, float *rs,
                                              float *ln_cs, float *betas) {
  if (!gen || !rs || !ln_cs || !betas) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  const uint32_t D = gen->dim, S = gen->samples;
  const uint32_t rows = param_chunk_rows(D, S);
  DevBuf tmp;
  MHB_CHECK(gen, tmp.ensure(static_cast<size_t>(rows) * D * sizeof(float)),
            mhcudaMemoryAllocationFailure);
  float *dst[3] = {rs, ln_cs, betas};
  // [samples][dim] host arrays, filled a block of sample rows at a time.
  for (uint32_t which = 0; which < 3; ++which) {
    for (uint32_t s0 = 0; s0 < S; s0 += rows) {
      const uint32_t cnt = std::min(rows, S - s0);
      const size_t len = static_cast<size_t>(cnt) * D;
      MHB_CHECK(gen, mhb::launch_unpack_params(gen->params, which, D, s0, cnt, gen->s_pad,
                                               tmp.as<float>(), gen->stream),
                mhcudaRuntimeError);
      MHB_CHECK(gen, cudaMemcpyAsync(dst[which] + static_cast<size_t>(s0) * D, tmp.ptr,
                                     len * sizeof(float), cudaMemcpyDeviceToHost, gen->stream),
                mhcudaMemoryCopyError);
    }
  }
  MHB_CHECK(gen, cudaStreamSynchronize(gen->stream), mhcudaMemoryCopyError);
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_assign_random_vars(const MinhashCudaGenerator *gen, const float *rs,
                                            const float *ln_cs, const float *betas) {
  if (!gen || !rs || !ln_cs || !betas) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  const uint32_t D = gen->dim, S = gen->samples;
  const uint32_t rows = param_chunk_rows(D, S);
  DevBuf tmp;
  MHB_CHECK(gen, tmp.ensure(static_cast<size_t>(rows) * D * sizeof(float)),
            mhcudaMemoryAllocationFailure);
  const float *src[3] = {rs, ln_cs, betas};
  for (uint32_t which = 0; which < 3; ++which) {
    for (uint32_t s0 = 0; s0 < S; s0 += rows) {
      const uint32_t cnt = std::min(rows, S - s0);
      const size_t len = static_cast<size_t>(cnt) * D;
      MHB_CHECK(gen, cudaMemcpyAsync(tmp.ptr, src[which] + static_cast<size_t>(s0) * D,
                                     len * sizeof(float), cudaMemcpyHostToDevice, gen->stream),
                mhcudaMemoryCopyError);
      MHB_CHECK(gen, mhb::launch_pack_params(tmp.as<float>(), nullptr, mhb::PairOp::kCopy, which,
                                             D, s0, cnt, gen->s_pad, gen->params, gen->stream),
                mhcudaRuntimeError);
    }
  }
  MHB_CHECK(gen, cudaStreamSynchronize(gen->stream), mhcudaMemoryCopyError);
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_calc(const MinhashCudaGenerator *gen, const float *weights,
                              const uint32_t *cols, const uint32_t *rows, uint32_t length,
                              uint32_t *output) {
  if (!gen || !weights || !cols || !rows || !output || length == 0) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  const uint32_t base = rows[0];
  if (rows[length] < base) return mhcudaInvalidArguments;
  const uint32_t nnz = rows[length] - base;
  const cudaStream_t st = gen->stream;
  const int min_override = env_int("MHCUDA_B200_PIPELINE_MIN_NNZ", 0);
  const uint64_t pipe_min = min_override > 0 ? static_cast<uint64_t>(min_override) : kPipelineMinNnz;
  if (nnz >= pipe_min && env_int("MHCUDA_B200_NO_PIPELINE", 0) == 0)
    return calc_pipelined(gen, HostCsr{weights, false, cols, 0, rows}, length, output);
  MHB_CHECK(gen, gen->d_weights.ensure(static_cast<size_t>(nnz) * 4 + 16),
            mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, gen->d_cols.ensure(static_cast<size_t>(nnz) * 4 + 16),
            mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, gen->d_indptr.ensure((static_cast<size_t>(length) + 1) * 4),
            mhcudaMemoryAllocationFailure);
  const size_t out_bytes = static_cast<size_t>(length) * gen->samples * 2 * sizeof(uint32_t);
  MHB_CHECK(gen, gen->d_out.ensure(out_bytes), mhcudaMemoryAllocationFailure);
  MHB_INFO(gen, "Preparing...\n");
  MHB_CHECK(gen, cudaMemcpyAsync(gen->d_indptr.ptr, rows, (static_cast<size_t>(length) + 1) * 4,
                                 cudaMemcpyHostToDevice, st),
            mhcudaMemoryCopyError);
  if (nnz) {
    MHB_CHECK(gen, cudaMemcpyAsync(gen->d_weights.ptr, weights + base,
                                   static_cast<size_t>(nnz) * 4, cudaMemcpyHostToDevice, st),
              mhcudaMemoryCopyError);
    MHB_CHECK(gen, cudaMemcpyAsync(gen->d_cols.ptr, cols + base, static_cast<size_t>(nnz) * 4,
                                   cudaMemcpyHostToDevice, st),
              mhcudaMemoryCopyError);
  }
  const HashPlan plan = make_plan(gen, nnz, length);
  HashArgs a{};
  MHCUDAResult r = prepare_launch(gen, length, nnz, plan, &a);
  if (r != mhcudaSuccess) return r;
  a.weights = gen->d_weights.as<float>();
  a.cols = gen->d_cols.as<uint32_t>();
  a.indptr = gen->d_indptr.as<uint32_t>();
  a.out = gen->d_out.as<uint32_t>();
  MHB_DEBUG(gen, "plan: spl=%u tiles=%u chunk=%u chunks=%u grid=%u\n", plan.spl, plan.ntiles,
            plan.chunk, plan.nchunks, plan.grid);
  MHB_INFO(gen, "Executing the CUDA kernel...\n");
  r = enqueue_hash(gen, a, plan, st);
  if (r != mhcudaSuccess) return r;
  MHB_CHECK(gen, cudaMemcpyAsync(output, gen->d_out.ptr, out_bytes, cudaMemcpyDeviceToHost, st),
            mhcudaMemoryCopyError);
  r = read_status(gen, st);
  if (r != mhcudaSuccess) return r;
  MHB_INFO(gen, "mhcuda - success\n");
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_calc_typed(const MinhashCudaGenerator *gen, const void *weights,
                                    int weights_type, const void *cols, int cols_type,
                                    const void *rows, int rows_type, uint32_t length,
                                    uint32_t *output) {
  if (!gen || !weights || !cols || !rows || !output || length == 0) return mhcudaInvalidArguments;
  if (weights_type != mhcudaFloat32 && weights_type != mhcudaFloat64) return mhcudaInvalidArguments;
  auto is_int = [](int t) {
    return t == mhcudaUInt32 || t == mhcudaInt32 || t == mhcudaInt64 || t == mhcudaUInt64;
  };
  if (!is_int(cols_type) || !is_int(rows_type)) return mhcudaInvalidArguments;
  const bool w64 = weights_type == mhcudaFloat64;
  const int cols64 = cols_type == mhcudaInt64 ? 1 : cols_type == mhcudaUInt64 ? 2 : 0;
  // 64-bit offsets are rebased to rows[0] (the caller's arrays are entered at
  // that entry); 32-bit ones stay absolute, as mhcuda_calc takes them.
  uint64_t base = 0;
  std::vector<uint32_t> rebased;
  const uint32_t *r32 = static_cast<const uint32_t *>(rows);
  if (rows_type == mhcudaInt64 || rows_type == mhcudaUInt64) {
    const bool sgn = rows_type == mhcudaInt64;
    auto at = [&](uint32_t i) -> uint64_t {
      return sgn ? static_cast<uint64_t>(static_cast<const int64_t *>(rows)[i])
                 : static_cast<const uint64_t *>(rows)[i];
    };
    if (sgn && static_cast<const int64_t *>(rows)[0] < 0) return mhcudaInvalidArguments;
    base = at(0);
    rebased.resize(static_cast<size_t>(length) + 1);
    uint64_t prev = base;
    for (uint32_t i = 0; i <= length; ++i) {
      const uint64_t v = at(i);
      if ((sgn && static_cast<int64_t>(v) < 0) || v < prev || v - base > 0xFFFFFFFFull)
        return mhcudaInvalidArguments;
      rebased[i] = static_cast<uint32_t>(v - base);
      prev = v;
    }
    r32 = rebased.data();
  }
  const size_t wsize = w64 ? sizeof(double) : sizeof(float);
  const size_t csize = cols64 ? sizeof(uint64_t) : sizeof(uint32_t);
  const void *w = static_cast<const char *>(weights) + base * wsize;
  const void *c = static_cast<const char *>(cols) + base * csize;
  if (!w64 && !cols64)
    return mhcuda_calc(gen, static_cast<const float *>(w), static_cast<const uint32_t *>(c), r32,
                       length, output);
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  if (r32[length] < r32[0]) return mhcudaInvalidArguments;
  return calc_pipelined(gen, HostCsr{w, w64, c, cols64, r32}, length, output);
}

enum MHCUDAResult mhcuda_calc_device(const MinhashCudaGenerator *gen, const float *d_weights,
                                     const uint32_t *d_cols, const uint32_t *d_rows,
                                     uint32_t length, uint32_t nnz, uint32_t *d_output,
                                     void *stream) {
  if (!gen || !d_rows || !d_output || length == 0 || (nnz && (!d_weights || !d_cols)))
    return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  const cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : gen->stream;
  const HashPlan plan = make_plan(gen, nnz, length);
  HashArgs a{};
  MHCUDAResult r = prepare_launch(gen, length, nnz, plan, &a);
  if (r != mhcudaSuccess) return r;
  a.weights = d_weights;
  a.cols = d_cols;
  a.indptr = d_rows;
  a.out = d_output;
  // Repeated calls with identical arguments replay a CUDA graph of the
  // memset + plan + hash + finalize sequence (one launch instead of four).
  // Not while profiling (per-launch events) or while the caller's stream is
  // itself being captured (the work then simply joins the caller's graph).
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  MHB_CHECK(gen, cudaStreamIsCapturing(st, &cap), mhcudaRuntimeError);
  if (gen->profiling || cap != cudaStreamCaptureStatusNone ||
      env_int("MHCUDA_B200_NO_GRAPHS", 0) != 0)
    return enqueue_hash(gen, a, plan, st);
  std::vector<unsigned char> key(sizeof(a) + sizeof(plan) + sizeof(st));
  memcpy(key.data(), &a, sizeof(a));
  memcpy(key.data() + sizeof(a), &plan, sizeof(plan));
  memcpy(key.data() + sizeof(a) + sizeof(plan), &st, sizeof(st));
  for (size_t i = 0; i < gen->graphs.size(); ++i) {
    if (gen->graphs[i].key == key) {
      MHB_CHECK(gen, cudaGraphLaunch(gen->graphs[i].exec, st), mhcudaRuntimeError);
      return mhcudaSuccess;
    }
  }
  cudaGraph_t graph = nullptr;
  MHB_CHECK(gen, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), mhcudaRuntimeError);
  r = enqueue_hash(gen, a, plan, st);
  const cudaError_t end = cudaStreamEndCapture(st, &graph);
  if (r != mhcudaSuccess || end != cudaSuccess) {
    cudaGetLastError();
    if (graph) cudaGraphDestroy(graph);
    return r != mhcudaSuccess ? r : mhcudaRuntimeError;
  }
  GraphEntry e;
  e.key = std::move(key);
  const cudaError_t inst = cudaGraphInstantiate(&e.exec, graph, 0);
  cudaGraphDestroy(graph);
  MHB_CHECK(gen, inst, mhcudaRuntimeError);
  constexpr size_t kMaxGraphs = 8;
  if (gen->graphs.size() == kMaxGraphs) {
    cudaGraphExecDestroy(gen->graphs.front().exec);
    gen->graphs.erase(gen->graphs.begin());
  }
  gen->graphs.push_back(std::move(e));
  MHB_CHECK(gen, cudaGraphLaunch(gen->graphs.back().exec, st), mhcudaRuntimeError);
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_calc_batch_device(const MinhashCudaGenerator *gen, uint32_t count,
                                           const float *const *d_weights,
                                           const uint32_t *const *d_cols,
                                           const uint32_t *const *d_rows, const uint32_t *lengths,
                                           uint32_t *const *d_outputs, void *stream) {
  if (!gen || (count && (!d_weights || !d_cols || !d_rows || !lengths || !d_outputs)))
    return mhcudaInvalidArguments;
  // Host descriptors: the CSR and output of every matrix with rows, and its
  // first thread in the batch's plan launch (rows + 1 threads per matrix).
  std::vector<mhb::BatchMatrix> mats(count);
  std::vector<uint32_t> plan_base(count);
  uint64_t plan_threads = 0;
  for (uint32_t m = 0; m < count; ++m) {
    mhb::BatchMatrix &d = mats[m];
    d = mhb::BatchMatrix{};
    plan_base[m] = static_cast<uint32_t>(std::min<uint64_t>(plan_threads, 0xFFFFFFFFull));
    if (!lengths[m]) continue;
    if (!d_weights[m] || !d_cols[m] || !d_rows[m] || !d_outputs[m]) return mhcudaInvalidArguments;
    d.weights = d_weights[m];
    d.cols = d_cols[m];
    d.indptr = d_rows[m];
    d.out = d_outputs[m];
    d.rows = lengths[m];
    plan_threads += static_cast<uint64_t>(lengths[m]) + 1;
  }
  if (plan_threads >= 0xFFFFFFFFull) return mhcudaInvalidArguments;
  if (plan_threads == 0) return mhcudaSuccess;  // no matrix has rows
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  const cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : gen->stream;

  // Kernel variant as for one large launch; the chunk size is chosen on the
  // device from the batch's nnz (batch_setup_kernel).
  const HashPlan vp = make_plan(gen, 1ull << 30, 1ull << 20);
  const int bps = mhb::hash_blocks_per_sm(vp.spl, vp.minb, gen->s_pad);
  const uint64_t resident_warps =
      static_cast<uint64_t>(gen->sm_count) * bps * (mhb::kHashBlock / 32);
  TuneChoice tc{};
  const int waves = std::max(1, env_int("MHCUDA_B200_WAVES", static_cast<int>(tc.waves)));
  const uint64_t max_chunks64 = count + resident_warps * 8 + 1;
  if (max_chunks64 >= 0xFFFFFFFFull) return mhcudaInvalidArguments;
  const uint32_t max_chunks = static_cast<uint32_t>(max_chunks64);
  HashPlan big{};
  big.nchunks = max_chunks;
  HashArgs base{};
  MHCUDAResult r = prepare_launch(gen, 0, 0, big, &base);
  if (r != mhcudaSuccess) return r;
  MHB_CHECK(gen, gen->d_chunk_owner.ensure(static_cast<size_t>(max_chunks) * 4),
            mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, gen->d_batch_plan.ensure(sizeof(mhb::BatchPlan)), mhcudaMemoryAllocationFailure);
  base.ntiles = vp.ntiles;

  // The batch's entry: descriptors on the device (uploaded once) and, from
  // its second call on, a CUDA graph of the launches.
  const size_t mats_bytes = static_cast<size_t>(count) * sizeof(mhb::BatchMatrix);
  const size_t desc_bytes = ((mats_bytes + 255) & ~static_cast<size_t>(255)) +
                            static_cast<size_t>(count) * sizeof(uint32_t);
  const void *batch_scratch[2] = {gen->d_chunk_owner.ptr, gen->d_batch_plan.ptr};
  std::vector<unsigned char> key(mats_bytes + count * sizeof(uint32_t) + sizeof(st) +
                                 sizeof(base) + sizeof(vp) + sizeof(batch_scratch));
  {
    unsigned char *k = key.data();
    memcpy(k, mats.data(), mats_bytes);
    k += mats_bytes;
    memcpy(k, plan_base.data(), count * sizeof(uint32_t));
    k += count * sizeof(uint32_t);
    memcpy(k, &st, sizeof(st));
    k += sizeof(st);
    memcpy(k, &base, sizeof(base));
    k += sizeof(base);
    memcpy(k, &vp, sizeof(vp));
    k += sizeof(vp);
    memcpy(k, batch_scratch, sizeof(batch_scratch));
  }
  BatchEntry *e = nullptr;
  for (auto &x : gen->batches)
    if (x->key == key) e = x.get();
  if (!e) {
    constexpr size_t kMaxBatches = 8;
    if (gen->batches.size() == kMaxBatches) gen->batches.erase(gen->batches.begin());
    std::unique_ptr<BatchEntry> ne(new BatchEntry());
    ne->key = std::move(key);
    MHB_CHECK(gen, cudaEventCreateWithFlags(&ne->used, cudaEventDisableTiming), mhcudaRuntimeError);
    MHB_CHECK(gen, ne->desc.ensure(desc_bytes), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, ne->staging.ensure(desc_bytes), mhcudaMemoryAllocationFailure);
    unsigned char *h = ne->staging.as<unsigned char>();
    memcpy(h, mats.data(), mats_bytes);
    memcpy(h + desc_bytes - count * sizeof(uint32_t), plan_base.data(), count * sizeof(uint32_t));
    MHB_CHECK(gen, cudaMemcpyAsync(ne->desc.ptr, h, desc_bytes, cudaMemcpyHostToDevice, st),
              mhcudaMemoryCopyError);
    gen->batches.push_back(std::move(ne));
    e = gen->batches.back().get();
  }
  mhb::BatchArgs b{};
  b.base = base;
  b.mats = e->desc.as<mhb::BatchMatrix>();
  b.plan_base = reinterpret_cast<const uint32_t *>(e->desc.as<unsigned char>() + desc_bytes -
                                                   count * sizeof(uint32_t));
  b.count = count;
  b.max_chunks = max_chunks;
  b.plan = gen->d_batch_plan.as<mhb::BatchPlan>();
  b.chunk_owner = gen->d_chunk_owner.as<uint32_t>();
  b.target_items = resident_warps * static_cast<uint64_t>(waves);
  b.want_items = resident_warps * 8;
  HashPlan lp = vp;
  lp.grid = static_cast<uint32_t>(static_cast<uint64_t>(gen->sm_count) * bps);
  const uint32_t pt = static_cast<uint32_t>(plan_threads);
  auto enqueue = [&]() -> MHCUDAResult {
    MHB_CHECK(gen, cudaMemsetAsync(base.status, 0, sizeof(uint32_t), st), mhcudaRuntimeError);
    MHB_CHECK(gen, mhb::launch_batch(b, lp, pt, st), mhcudaRuntimeError);
    return mhcudaSuccess;
  };
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  MHB_CHECK(gen, cudaStreamIsCapturing(st, &cap), mhcudaRuntimeError);
  const bool graphs = !gen->profiling && cap == cudaStreamCaptureStatusNone &&
                      env_int("MHCUDA_B200_NO_GRAPHS", 0) == 0;
  if (graphs && !e->exec && e->seen >= 1) {
    cudaGraph_t graph = nullptr;
    MHB_CHECK(gen, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), mhcudaRuntimeError);
    r = enqueue();
    const cudaError_t end = cudaStreamEndCapture(st, &graph);
    if (r != mhcudaSuccess || end != cudaSuccess) {
      cudaGetLastError();
      if (graph) cudaGraphDestroy(graph);
      return r != mhcudaSuccess ? r : mhcudaRuntimeError;
    }
    const cudaError_t inst = cudaGraphInstantiate(&e->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (inst != cudaSuccess) {
      e->exec = nullptr;
      MHB_CHECK(gen, inst, mhcudaRuntimeError);
    }
  }
  std::pair<cudaEvent_t, cudaEvent_t> *ev = nullptr;
  if (gen->profiling) {
    if (gen->prof_used == gen->prof_events.size()) {
      std::pair<cudaEvent_t, cudaEvent_t> pe{nullptr, nullptr};
      MHB_CHECK(gen, cudaEventCreate(&pe.first), mhcudaRuntimeError);
      MHB_CHECK(gen, cudaEventCreate(&pe.second), mhcudaRuntimeError);
      gen->prof_events.push_back(pe);
    }
    ev = &gen->prof_events[gen->prof_used++];
    MHB_CHECK(gen, cudaEventRecord(ev->first, st), mhcudaRuntimeError);
  }
  if (graphs && e->exec) {
    MHB_CHECK(gen, cudaGraphLaunch(e->exec, st), mhcudaRuntimeError);
  } else {
    r = enqueue();
    if (r != mhcudaSuccess) return r;
  }
  if (ev) MHB_CHECK(gen, cudaEventRecord(ev->second, st), mhcudaRuntimeError);
  ++e->seen;
  if (cap == cudaStreamCaptureStatusNone)
    MHB_CHECK(gen, cudaEventRecord(e->used, st), mhcudaRuntimeError);
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_autotune(const MinhashCudaGenerator *gen, const float *d_weights,
                                  const uint32_t *d_cols, const uint32_t *d_rows, uint32_t length,
                                  uint32_t nnz, uint32_t *d_output, void *stream,
                                  uint32_t *choice, double *best_ms) {
  if (!gen || !d_rows || !d_output || length == 0 || (nnz && (!d_weights || !d_cols)))
    return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  const cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : gen->stream;
  // Candidates: samples per lane (lane utilisation of the last tile >= 1/2),
  // register budget of the 4-sample variant (4, 3 or 2 resident blocks per SM:
  // fewer warps with more registers win where the gathers hit L2, more warps
  // where they stream from HBM), and chunk granularity.
  std::vector<TuneChoice> cands;
  for (uint32_t spl : {4u, 2u, 1u}) {
    const uint32_t w = 32u * spl, tiles = (gen->s_pad + w - 1) / w;
    if (static_cast<double>(gen->s_pad) / (static_cast<double>(tiles) * w) < 0.5) continue;
    for (uint32_t minb : spl == 4 ? std::vector<uint32_t>{4u, 3u, 2u} : std::vector<uint32_t>{4u})
      for (uint32_t waves : {8u, 32u, 128u}) cands.push_back(TuneChoice{spl, minb, waves});
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  MHB_CHECK(gen, cudaEventCreate(&e0), mhcudaRuntimeError);
  MHB_CHECK(gen, cudaEventCreate(&e1), mhcudaRuntimeError);
  TuneChoice best{};
  double best_t = 1e300;
  std::vector<double> times;
  MHCUDAResult r = mhcudaSuccess;
  for (const TuneChoice &c : cands) {
    const HashPlan plan = make_plan(gen, nnz, length, &c);
    HashArgs a{};
    r = prepare_launch(gen, length, nnz, plan, &a);
    if (r != mhcudaSuccess) break;
    a.weights = d_weights;
    a.cols = d_cols;
    a.indptr = d_rows;
    a.out = d_output;
    r = enqueue_hash(gen, a, plan, st);  // warm-up
    if (r != mhcudaSuccess) break;
    MHB_CHECK(gen, cudaEventRecord(e0, st), mhcudaRuntimeError);
    for (int k = 0; k < 2 && r == mhcudaSuccess; ++k) r = enqueue_hash(gen, a, plan, st);
    MHB_CHECK(gen, cudaEventRecord(e1, st), mhcudaRuntimeError);
    MHB_CHECK(gen, cudaEventSynchronize(e1), mhcudaRuntimeError);
    float ms = 0.0f;
    MHB_CHECK(gen, cudaEventElapsedTime(&ms, e0, e1), mhcudaRuntimeError);
    MHB_DEBUG(gen, "autotune spl=%u minb=%u waves=%u: %.3f ms\n", c.spl, c.minb, c.waves, ms / 2);
    times.push_back(ms / 2);
    if (ms / 2 < best_t) {
      best_t = ms / 2;
      best = c;
    }
  }
  // For the pipeline: the winner's samples per lane, 4 blocks per SM, the
  // fastest chunk granularity among those.
  TuneChoice best_streamed = best;
  double best_streamed_t = 1e300;
  for (size_t i = 0; i < times.size(); ++i) {
    const TuneChoice &c = cands[i];
    if (c.spl == best.spl && c.minb == 4 && times[i] < best_streamed_t) {
      best_streamed_t = times[i];
      best_streamed = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r != mhcudaSuccess) return r;
  {
    std::lock_guard<std::mutex> tl(gen->tune_mu);
    gen->tuned[tune_key(nnz, length)] = TunedShape{best, best_streamed};
  }
  if (choice) {
    choice[0] = best.spl;
    choice[1] = best.minb;
    choice[2] = best.waves;
  }
  if (best_ms) *best_ms = best_t;
  return read_status(gen, st);
}

enum MHCUDAResult mhcuda_device_status(const MinhashCudaGenerator *gen) {
  if (!gen) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  MHB_CHECK(gen, cudaDeviceSynchronize(), mhcudaRuntimeError);
  if (!gen->d_status.ptr) return mhcudaSuccess;
  const MHCUDAResult r = read_status(gen, gen->stream);
  MHB_CHECK(gen, cudaMemset(gen->d_status.ptr, 0, sizeof(uint32_t)), mhcudaRuntimeError);
  return r;
}

enum MHCUDAResult mhcuda_calc_batch(const MinhashCudaGenerator *gen, uint32_t count,
                                    const float *const *weights, const uint32_t *const *cols,
                                    const uint32_t *const *rows, const uint32_t *lengths,
                                    uint32_t *const *outputs) {
  if (!gen || !weights || !cols || !rows || !lengths || !outputs) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  // Per-matrix nnz; validated before any device work.
  std::vector<uint64_t> nnz_of(count, 0);
  for (uint32_t i = 0; i < count; ++i) {
    const uint64_t len = lengths[i];
    if (!len) continue;
    if (!weights[i] || !cols[i] || !rows[i] || !outputs[i]) return mhcudaInvalidArguments;
    if (rows[i][len] < rows[i][0]) return mhcudaInvalidArguments;
    nnz_of[i] = rows[i][len] - rows[i][0];
  }
  MHB_CHECK(gen, batch_streams(gen), mhcudaRuntimeError);
  const cudaStream_t st = gen->stream;
  const size_t row_bytes = static_cast<size_t>(gen->samples) * 2 * sizeof(uint32_t);
  // Groups of group_nnz (MHCUDA_B200_BATCH_GROUP_NNZ, or MHCUDA_B200_BLOCK_NNZ).
  // A group's host gather and scatter take about as long as its hashing, and
  // small groups keep them in the host's caches: measured on the 4096-matrix
  // batch (3.9e8 nnz, 256 samples), ms per call, constant groups of 8M / 12M /
  // 16M / 24M / 32M / 48M nnz: 202.5 / 204.4 / 203.4 / 222-231 / 218 / 235,
  // against 206.5 for groups growing from 2M to 16M and 219-220 for the
  // earlier groups growing from 8M to 64M (device-resident batch: 195-202).
  uint64_t group_nnz = 16ull << 20;
  const int cap = env_int("MHCUDA_B200_BATCH_GROUP_NNZ", 0);
  if (cap > 0) group_nnz = static_cast<uint64_t>(cap);
  const int forced = env_int("MHCUDA_B200_BLOCK_NNZ", 0);
  if (forced > 0) group_nnz = static_cast<uint64_t>(forced);
  const uint64_t group_rows = 1u << 20;
  MHB_CHECK(gen, gen->d_status.ensure(sizeof(uint32_t)), mhcudaMemoryAllocationFailure);
  MHB_CHECK(gen, cudaMemsetAsync(gen->d_status.ptr, 0, sizeof(uint32_t), st), mhcudaRuntimeError);
  const unsigned nth = host_threads();

  // A slot's staged hashes go back to their matrices once its copy is done.
  struct Pending {
    uint32_t first = 0, last = 0;  // matrices [first, last)
  };
  Pending pending[Gen::kBatchSlots];
  auto retire = [&](uint32_t k) -> MHCUDAResult {
    Gen::Slot &sl = gen->slots[k];
    if (!sl.busy) return mhcudaSuccess;
    MHB_CHECK(gen, cudaEventSynchronize(sl.d2h), mhcudaMemoryCopyError);
    const Pending pd = pending[k];
    const char *src = sl.hout.as<char>();
    std::vector<size_t> off(pd.last - pd.first + 1, 0);
    for (uint32_t i = pd.first; i < pd.last; ++i)
      off[i - pd.first + 1] = off[i - pd.first] + lengths[i] * row_bytes;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nth; ++t) {
      pool.emplace_back([&, t]() {
        for (uint32_t i = pd.first + t; i < pd.last; i += nth)
          if (lengths[i]) stream_copy(outputs[i], src + off[i - pd.first], lengths[i] * row_bytes);
      });
    }
    for (auto &th : pool) th.join();
    sl.busy = false;
    return mhcudaSuccess;
  };

  // Groups [m0, m1) of consecutive matrices, planned up front: up to
  // group_nnz entries and 2^20 rows each (a matrix larger than that is a
  // group of its own).
  struct Group {
    uint32_t m0, m1;
    uint64_t nnz, rows;
  };
  std::vector<Group> groups;
  {
    const uint64_t cur = group_nnz;
    for (uint32_t m0 = 0; m0 < count;) {
      uint32_t m1 = m0;
      uint64_t gn = 0, gr = 0;
      while (m1 < count) {
        const uint64_t n = nnz_of[m1], l = lengths[m1];
        if (m1 > m0 && (gn + n > cur || gr + l > group_rows)) break;
        if (gn + n >= 0xFFFFFFFFull || gr + l >= 0xFFFFFFFFull) {
          if (m1 == m0) return mhcudaInvalidArguments;
          break;
        }
        gn += n;
        gr += l;
        ++m1;
      }
      groups.push_back(Group{m0, m1, gn, gr});
      m0 = m1;
    }
  }
  // Slots and scratch sized once for the largest group (growing a buffer
  // mid-pipeline frees device memory, which waits for all work in flight).
  {
    uint64_t max_n = 0, max_r = 0;
    uint32_t max_chunks = 1;
    for (const Group &gp : groups) {
      max_n = std::max(max_n, gp.nnz);
      max_r = std::max(max_r, gp.rows);
      if (gp.rows) max_chunks = std::max(max_chunks, make_plan(gen, gp.nnz, gp.rows).nchunks);
    }
    for (Gen::Slot &sl : gen->slots) {
      MHB_CHECK(gen, sl.hw.ensure(max_n * 4), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.hc.ensure(max_n * 4), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.hip.ensure((max_r + 1) * 4), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.hout.ensure(max_r * row_bytes), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.w.ensure(max_n * 4 + 16), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.c.ensure(max_n * 4 + 16), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.ip.ensure((max_r + 1) * 4), mhcudaMemoryAllocationFailure);
      MHB_CHECK(gen, sl.out.ensure(max_r * row_bytes), mhcudaMemoryAllocationFailure);
    }
    HashPlan big{};
    big.nchunks = max_chunks;
    HashArgs unused{};
    const MHCUDAResult pr = prepare_launch(gen, 0, 0, big, &unused);
    if (pr != mhcudaSuccess) return pr;
  }

  MHCUDAResult r = mhcudaSuccess;
  for (uint32_t g = 0; g < groups.size() && r == mhcudaSuccess; ++g) {
    const uint32_t m0 = groups[g].m0, m1 = groups[g].m1;
    const uint64_t gn = groups[g].nnz, gr = groups[g].rows;
    const uint32_t k = g % Gen::kBatchSlots;
    Gen::Slot &sl = gen->slots[k];
    r = retire(k);
    if (r != mhcudaSuccess) break;
    if (gr == 0) continue;  // only empty matrices
    const uint32_t R = static_cast<uint32_t>(gr), N = static_cast<uint32_t>(gn);
    MHB_CHECK(gen, sl.hw.ensure(static_cast<size_t>(N) * 4), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.hc.ensure(static_cast<size_t>(N) * 4), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.hip.ensure((static_cast<size_t>(R) + 1) * 4), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.hout.ensure(static_cast<size_t>(R) * row_bytes), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.w.ensure(static_cast<size_t>(N) * 4 + 16), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.c.ensure(static_cast<size_t>(N) * 4 + 16), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.ip.ensure((static_cast<size_t>(R) + 1) * 4), mhcudaMemoryAllocationFailure);
    MHB_CHECK(gen, sl.out.ensure(static_cast<size_t>(R) * row_bytes), mhcudaMemoryAllocationFailure);
    // Gather the group into pinned staging: values and columns back to back,
    // row offsets rebased to the group's positions.
    std::vector<uint64_t> moff(m1 - m0 + 1, 0), roff(m1 - m0 + 1, 0);
    for (uint32_t i = m0; i < m1; ++i) {
      moff[i - m0 + 1] = moff[i - m0] + nnz_of[i];
      roff[i - m0 + 1] = roff[i - m0] + lengths[i];
    }
    float *sw = sl.hw.as<float>();
    uint32_t *sc = sl.hc.as<uint32_t>(), *si = sl.hip.as<uint32_t>();
    {
      std::vector<std::thread> pool;
      for (unsigned t = 0; t < nth; ++t) {
        pool.emplace_back([&, t]() {
          for (uint32_t i = m0 + t; i < m1; i += nth) {
            const uint64_t len = lengths[i];
            if (!len) continue;
            const uint32_t b = rows[i][0];
            const uint64_t po = moff[i - m0], ro = roff[i - m0];
            stream_copy(sw + po, weights[i] + b, nnz_of[i] * 4);
            stream_copy(sc + po, cols[i] + b, nnz_of[i] * 4);
            for (uint64_t x = 0; x < len; ++x)
              si[ro + x] = static_cast<uint32_t>(po + (rows[i][x] - b));
          }
        });
      }
      for (auto &th : pool) th.join();
    }
    si[R] = N;
    MHB_CHECK(gen, cudaMemcpyAsync(sl.ip.ptr, si, (static_cast<size_t>(R) + 1) * 4,
                                   cudaMemcpyHostToDevice, gen->s_in),
              mhcudaMemoryCopyError);
    if (N) {
      MHB_CHECK(gen, cudaMemcpyAsync(sl.w.ptr, sw, static_cast<size_t>(N) * 4,
                                     cudaMemcpyHostToDevice, gen->s_in),
                mhcudaMemoryCopyError);
      MHB_CHECK(gen, cudaMemcpyAsync(sl.c.ptr, sc, static_cast<size_t>(N) * 4,
                                     cudaMemcpyHostToDevice, gen->s_in),
                mhcudaMemoryCopyError);
    }
    MHB_CHECK(gen, cudaEventRecord(sl.h2d, gen->s_in), mhcudaRuntimeError);
    MHB_CHECK(gen, cudaStreamWaitEvent(st, sl.h2d, 0), mhcudaRuntimeError);
    const HashPlan plan = make_plan(gen, N, R);
    HashArgs a{};
    r = prepare_launch(gen, R, N, plan, &a);
    if (r != mhcudaSuccess) break;
    a.weights = sl.w.as<float>();
    a.cols = sl.c.as<uint32_t>();
    a.indptr = sl.ip.as<uint32_t>();
    a.out = sl.out.as<uint32_t>();
    r = enqueue_hash(gen, a, plan, st, /*clear_status=*/false);
    if (r != mhcudaSuccess) break;
    MHB_CHECK(gen, cudaEventRecord(sl.done, st), mhcudaRuntimeError);
    MHB_CHECK(gen, cudaStreamWaitEvent(gen->s_out, sl.done, 0), mhcudaRuntimeError);
    MHB_CHECK(gen, cudaMemcpyAsync(sl.hout.ptr, sl.out.ptr, static_cast<size_t>(R) * row_bytes,
                                   cudaMemcpyDeviceToHost, gen->s_out),
              mhcudaMemoryCopyError);
    MHB_CHECK(gen, cudaEventRecord(sl.d2h, gen->s_out), mhcudaRuntimeError);
    sl.busy = true;
    sl.pending_out = nullptr;
    pending[k] = Pending{m0, m1};
    MHB_DEBUG(gen, "batch group %u: matrices [%u, %u) rows %u nnz %u\n", g, m0, m1, R, N);
  }
  for (uint32_t k = 0; k < Gen::kBatchSlots; ++k) {
    const MHCUDAResult rr = retire(k);
    if (r == mhcudaSuccess) r = rr;
  }
  if (r != mhcudaSuccess) {
    cudaDeviceSynchronize();
    return r;
  }
  return read_status(gen, st);
}

enum MHCUDAResult mhcuda_host_register(uint32_t devices, const void *ptr, uint64_t bytes) {
  if (!ptr || bytes == 0) return mhcudaInvalidArguments;
  const int dev = pick_device(devices);
  if (dev < 0) return mhcudaNoSuchDevice;
  mhb::DeviceGuard on_device(dev);
  if (!on_device.ok()) return mhcudaNoSuchDevice;
  const cudaError_t e =
      cudaHostRegister(const_cast<void *>(ptr), static_cast<size_t>(bytes), cudaHostRegisterPortable);
  if (e == cudaSuccess) return mhcudaSuccess;
  cudaGetLastError();
  return e == cudaErrorHostMemoryAlreadyRegistered || e == cudaErrorInvalidValue
             ? mhcudaInvalidArguments
             : mhcudaMemoryAllocationFailure;
}

enum MHCUDAResult mhcuda_host_unregister(uint32_t devices, const void *ptr) {
  if (!ptr) return mhcudaInvalidArguments;
  const int dev = pick_device(devices);
  if (dev < 0) return mhcudaNoSuchDevice;
  mhb::DeviceGuard on_device(dev);
  if (!on_device.ok()) return mhcudaNoSuchDevice;
  if (cudaHostUnregister(const_cast<void *>(ptr)) != cudaSuccess) {
    cudaGetLastError();
    return mhcudaInvalidArguments;
  }
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_debug_device_logf(uint32_t devices, const float *in, float *out,
                                           uint64_t n) {
  if (!in || !out) return mhcudaInvalidArguments;
  const int dev = pick_device(devices);
  if (dev < 0) return mhcudaNoSuchDevice;
  mhb::DeviceGuard on_device(dev);
  if (!on_device.ok()) return mhcudaNoSuchDevice;
  if (n == 0) return mhcudaSuccess;
  DevBuf a, b;
  if (a.ensure(n * 4) != cudaSuccess || b.ensure(n * 4) != cudaSuccess)
    return mhcudaMemoryAllocationFailure;
  if (cudaMemcpy(a.ptr, in, n * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return mhcudaMemoryCopyError;
  if (mhb::launch_logf(a.as<float>(), b.as<float>(), n, nullptr) != cudaSuccess)
    return mhcudaRuntimeError;
  if (cudaMemcpy(out, b.ptr, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return mhcudaMemoryCopyError;
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_profile(const MinhashCudaGenerator *gen, int enable) {
  if (!gen) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  gen->profiling = enable != 0;
  gen->prof_used = 0;
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_profile_read(const MinhashCudaGenerator *gen, double *hash_ms,
                                      uint64_t *launches) {
  if (!gen || !hash_ms || !launches) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(gen->mu);
  MHB_ON_DEVICE(gen);
  double total = 0.0;
  for (size_t i = 0; i < gen->prof_used; ++i) {
    MHB_CHECK(gen, cudaEventSynchronize(gen->prof_events[i].second), mhcudaRuntimeError);
    float ms = 0.0f;
    MHB_CHECK(gen, cudaEventElapsedTime(&ms, gen->prof_events[i].first,
                                        gen->prof_events[i].second),
              mhcudaRuntimeError);
    total += ms;
  }
  *hash_ms = total;
  *launches = gen->prof_used;
  gen->prof_used = 0;
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_fini(MinhashCudaGenerator *gen) {
  delete gen;
  return mhcudaSuccess;
}

}  // extern "C"
