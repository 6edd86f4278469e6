// Internal declarations shared by the kernels (*.cu) and the host engine.
// Nothing here is part of the public ABI (include/minhashcuda*.h is).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

struct MinhashCudaGenerator_;

namespace mhb {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// Device status word bits (written by kernels, read by the host).
constexpr uint32_t kStatusBadColumn = 1u;  // a column index >= dim was seen
constexpr uint32_t kStatusBadIndptr = 2u;  // row offsets decrease or disagree with nnz
constexpr uint32_t kStatusStall = 4u;      // a bounded wait on a staging copy gave up

// Parameter table: one contiguous block per column d,
//   params[(d * 3 + 0) * s_pad + s] = r      (rs)
//   params[(d * 3 + 1) * s_pad + s] = ln_c   (ln_cs)
//   params[(d * 3 + 2) * s_pad + s] = beta   (betas)
// s_pad = samples rounded up to a multiple of 4, so every section starts on a
// 16-byte boundary and a lane can fetch 4 consecutive samples as one float4.
inline uint32_t padded_samples(uint32_t samples) { return (samples + 3u) & ~3u; }

// Work decomposition of one hash launch.
//
// The CSR's nnz positions [0, nnz) (relative to indptr[0]) are cut into
// `nchunks` chunks of `chunk` positions (a multiple of 32).  A row belongs to
// the chunk holding its first position (trailing empty rows to the last
// chunk).  A warp hashes one (chunk, sample-tile) item: it finishes every row
// that lies inside the chunk and leaves a partial arg-min for the row that
// runs in from the previous chunk ("head", slot 2c) and for the row that runs
// out past the chunk's end ("tail", slot 2c+1).  A finalize pass merges the
// partials of every row that crosses a chunk boundary, earlier positions
// winning ties exactly as the reference's strict '<' scan does.
struct HashPlan {
  uint32_t chunk;    // positions per chunk, multiple of 32
  uint32_t nchunks;  // >= 1
  uint32_t spl;      // samples per lane in one item: 1, 2 or 4
  uint32_t minb;     // kernel variant: minimum resident blocks per SM (4; 3 or 2 for spl 4)
  uint32_t ntiles;   // sample tiles of 32*spl samples
  uint32_t grid;     // persistent grid (blocks of kHashBlock threads)
};

constexpr int kHashBlock = 256;

struct HashArgs {
  const float *params;       // [dim][3][s_pad]
  uint32_t dim;
  uint32_t samples;
  uint32_t s_pad;
  const float *weights;      // CSR values, weights[p] for relative position p
  const uint32_t *cols;      // CSR column indices
  const uint32_t *indptr;    // rows+1 absolute offsets, indptr[0] = base
  uint32_t rows;
  uint32_t nnz;              // indptr[rows] - indptr[0]
  uint32_t chunk;
  uint32_t nchunks;
  uint32_t ntiles;
  uint32_t *chunk_row;       // [nchunks] first row owned by each chunk
  float *part_ln;            // [2*nchunks][s_pad] partial minima
  uint2 *part_kt;            // [2*nchunks][s_pad] partial (position of the minimum, 0)
  uint32_t *out;             // [rows][samples][2]
  uint32_t *status;          // device status word
  uint32_t host_csr;         // weights/cols/indptr/out are mapped host memory
  // Packed columns (col_hi_bits 4 or 8; cols unused): column p is
  // cols_lo[p] | hi(p) << 16, hi(p) the nibble p of cols_hi (4: entry p in
  // byte p/2, low nibble for even p) or its byte p (8).  Device memory, both
  // arrays 16-byte aligned.  col_hi_bits 0: the columns are `cols`.
  const uint16_t *cols_lo;
  const uint8_t *cols_hi;
  uint32_t col_hi_bits;
};

// One matrix of a device-resident batch (mhcuda_calc_batch_device).  The
// host fills the CSR pointers, rows and plan_base; batch_setup_kernel fills
// nnz, chunk_base and nchunks on the device.
struct BatchMatrix {
  const float *weights;    // weights[p] for relative position p
  const uint32_t *cols;
  const uint32_t *indptr;  // rows+1 absolute offsets, indptr[0] = offset of weights[0]
  uint32_t *out;           // [rows][samples][2]
  uint32_t rows;
  uint32_t nnz;
  uint32_t chunk_base;     // index of its first chunk in the batch's chunk space
  uint32_t nchunks;        // 0 for a matrix without rows
};

// Work decomposition of a batch, computed on the device.
struct BatchPlan {
  uint32_t chunk;    // positions per chunk, the same for every matrix
  uint32_t nchunks;  // chunks of all matrices
};

struct BatchArgs {
  HashArgs base;          // generator fields, ntiles, status and the batch-wide scratch
                          // (chunk_row, part_ln, part_kt indexed by batch chunk)
  BatchMatrix *mats;      // [count]
  const uint32_t *plan_base;  // [count] first plan thread of each matrix (rows+1 each)
  uint32_t count;
  uint32_t max_chunks;    // chunk slots the scratch holds
  BatchPlan *plan;
  uint32_t *chunk_owner;  // [max_chunks] matrix of each batch chunk
  uint64_t target_items;  // warp items to aim for (resident warps x waves)
  uint64_t want_items;    // items per launch below which chunks shrink (resident warps x 8)
};

// Launchers (hash_kernels.cu).  All enqueue on `stream` and return the launch
// error, if any.
cudaError_t launch_plan(const HashArgs &a, cudaStream_t stream);
cudaError_t launch_hash(const HashArgs &a, const HashPlan &plan, cudaStream_t stream);
cudaError_t launch_finalize(const HashArgs &a, cudaStream_t stream);
// A whole device-resident batch: setup (per-matrix nnz, chunk size, chunk
// tables), plan, one persistent hash launch over all matrices' chunks and
// finalize.  plan.spl/minb/ntiles/grid select the hash variant; plan_threads
// is the sum of rows+1 over the matrices that have rows.
cudaError_t launch_batch(const BatchArgs &b, const HashPlan &plan, uint32_t plan_threads,
                         cudaStream_t stream);
// Blocks per SM the hash kernel variant launched for (samples per lane,
// register budget, s_pad) reaches, and its registers per thread.
int hash_blocks_per_sm(uint32_t spl, uint32_t minb, uint32_t s_pad);
size_t hash_kernel_registers(uint32_t spl, uint32_t minb, uint32_t s_pad);

// Parameter kernels (param_kernels.cu).
enum class PairOp : int { kGamma = 0, kLogGamma = 1, kCopy = 2 };
// params[d][which][s_base + s] = op(a[s*dim + d], b[s*dim + d]) for s < samples.
cudaError_t launch_pack_params(const float *a, const float *b, PairOp op, uint32_t which,
                               uint32_t dim, uint32_t s_base, uint32_t samples, uint32_t s_pad,
                               float *params, cudaStream_t stream);
// dst[s*dim + d] = params[d][which][s_base + s] for s < samples.
cudaError_t launch_unpack_params(const float *params, uint32_t which, uint32_t dim,
                                 uint32_t s_base, uint32_t samples, uint32_t s_pad, float *dst,
                                 cudaStream_t stream);
cudaError_t launch_logf(const float *in, float *out, size_t n, cudaStream_t stream);

// memcpy for host staging moves: non-temporal stores for large pieces
// (host_copy.cc).
void stream_copy(void *dst, const void *src, size_t bytes);
// float64 -> float32 (round to nearest) and 64-bit -> uint32 (values outside
// [0, 2^32) become 0xFFFFFFFF), with non-temporal stores for large pieces.
void convert_f64_to_f32(float *dst, const double *src, size_t n);
void convert_i64_to_u32(uint32_t *dst, const uint64_t *src, size_t n);
// Packed columns for the host->device link: lo[i] = low 16 bits of src[i],
// hi = the bits above, as bytes (hi_bits 8: hi[i]) or nibbles (hi_bits 4:
// entry i in byte i/2, the low nibble for even i).  Returns false if some
// column needs more than 16 + hi_bits bits.  A range split across calls must
// be split at even entries.
bool pack_cols(const uint32_t *src, size_t n, uint16_t *lo, uint8_t *hi, int hi_bits);

// Makes `device` current for the calling thread while the guard lives and
// then gives the thread back the state it came with: its previous device, or
// no current context at all when it had none (restoring "device 0" there
// would create a context on device 0 that the caller never asked for).
// Every extern "C" entry point that works on a device holds one.
class DeviceGuard {
 public:
  explicit DeviceGuard(int device);
  ~DeviceGuard();
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
  bool ok() const { return ok_; }

 private:
  int prev_ = -1;
  bool had_context_ = true;
  bool changed_ = false;
  bool ok_ = false;
};

// Read-only view of a generator's fields for entry points that live outside
// engine.cu (engine.cu).
struct GeneratorView {
  const float *params;
  uint32_t dim;
  uint32_t samples;
  uint32_t s_pad;
  int device;
  int sm_count;
  int verbosity;
  cudaStream_t stream;
};
bool generator_view(const MinhashCudaGenerator_ *gen, GeneratorView *view);
// The engine's work decomposition for `nnz` entries in `rows` rows, with at
// least `min_items` warp items per resident warp where chunks allow.
HashPlan plan_for_generator(const MinhashCudaGenerator_ *gen, uint64_t nnz, uint64_t rows,
                            uint32_t min_items = 8);

}  // namespace mhb
