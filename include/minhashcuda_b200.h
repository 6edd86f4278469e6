/*
 * minhashcuda_b200.h -- entry points this engine adds beside the drop-in ABI
 * of minhashcuda.h.  All are extern "C", take plain pointers and sizes, and
 * return the same MHCUDAResult codes.  Device pointers must belong to the
 * generator's device; a `stream` argument is a cudaStream_t passed as void*
 * (NULL selects the generator's own stream).
 */
#ifndef MHCUDA_MINHASHCUDA_B200_H
#define MHCUDA_MINHASHCUDA_B200_H

#include <stddef.h>
#include <stdint.h>

#include "minhashcuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Device-resident counterpart of mhcuda_calc (minhashcuda.h:115-118): the
 * CSR (d_weights/d_cols with `nnz` entries, d_rows with length+1 offsets
 * whose first value is the offset of d_weights[0]) and d_output
 * (length*samples*2 uint32) already live in device memory.  The work is
 * enqueued on `stream` and the call returns without waiting; the generator's
 * scratch is reused by the next call on it, so calls on one generator must
 * be ordered on one stream.  Invalid CSR content (a column >= dim,
 * decreasing offsets) is detected on the device and reported by the next
 * mhcuda_device_status() call. */
enum MHCUDAResult mhcuda_calc_device(
    const MinhashCudaGenerator *gen, const float *d_weights,
    const uint32_t *d_cols, const uint32_t *d_rows, uint32_t length,
    uint32_t nnz, uint32_t *d_output, void *stream);

/* Autotuner: times the hash kernel's variants (samples per lane 1/2/4,
 * register budget, chunk granularity) on this device-resident CSR (same
 * arguments as mhcuda_calc_device; d_output receives the hashes), keeps the
 * fastest for launches of the same shape class (log2 of nnz and of the mean
 * row length) on this generator, and returns it in choice[3] = {samples per
 * lane, min blocks per SM, items per resident warp} and its time in *best_ms
 * (either may be NULL).  Results never depend on the choice.  Waits for
 * completion.  No counterpart in the reference (its launch shape is fixed by
 * host binpacking, minhashcuda.cc:457-528, and kernel.cu:155-160). */
enum MHCUDAResult mhcuda_autotune(
    const MinhashCudaGenerator *gen, const float *d_weights,
    const uint32_t *d_cols, const uint32_t *d_rows, uint32_t length,
    uint32_t nnz, uint32_t *d_output, void *stream, uint32_t *choice,
    double *best_ms);

/* Waits for the generator's device work and returns mhcudaInvalidArguments
 * if a preceding mhcuda_calc_device saw invalid CSR content (and clears the
 * flag), mhcudaRuntimeError on a CUDA error, else mhcudaSuccess.
 * No counterpart in the reference (its kernel launch is unchecked,
 * kernel.cu:166-170). */
enum MHCUDAResult mhcuda_device_status(const MinhashCudaGenerator *gen);

/* Allocation-free variant of mhcuda_calc_device, same arguments, for
 * callers that must not allocate device memory: processes whose device
 * memory another allocator (a framework's caching allocator, say) has
 * already reserved, where a cudaMalloc would fail, and latency-critical
 * loops that cannot take the device-wide synchronisation a cudaMalloc or
 * cudaFree may cause.  mhcuda_calc_device grows a workspace with cudaMalloc;
 * this call instead uses one fixed 8 MiB array of device memory that is part
 * of the library (every GPU that loads the library holds it until the process
 * exits) and calls no allocating routine.
 *  - Limit: an input needs 4 + 24*s_pad bytes per chunk of at most 2^20 nnz
 *    (s_pad = samples rounded up to a multiple of 4); it is refused with
 *    mhcudaInvalidArguments when ceil(nnz / 2^20) chunks do not fit in
 *    8 MiB - 1 KiB (about 2.8e9 nnz at 128 samples, 5*2^20 at 65535).
 *  - The first call on a device looks up the array's device address and
 *    caches it.
 *  - All calls share the array, which keeps the last call's contents: the
 *    status word is cleared by every call and everything else a call reads it
 *    writes first.  Calls whose work overlapped on the GPU would race on the
 *    array, so every call waits for its own work to finish before it returns
 *    and calls are serialised by a process-wide lock.
 *  - Returns mhcudaInvalidArguments for invalid CSR content (a column >= dim,
 *    decreasing offsets) as detected on the device.
 * No counterpart in the reference. */
enum MHCUDAResult mhcuda_calc_device_noalloc(
    const MinhashCudaGenerator *gen, const float *d_weights,
    const uint32_t *d_cols, const uint32_t *d_rows, uint32_t length,
    uint32_t nnz, uint32_t *d_output, void *stream);

/* Device-resident batch: hashes `count` CSR matrices that already live in
 * device memory against one generator in one persistent launch, whose warps
 * take (matrix, chunk of positions, sample tile) items from a table built on
 * the device.  The five arrays are host arrays of `count` entries; matrix i is
 * d_weights[i] and d_cols[i] (its entries), d_rows[i] (lengths[i]+1 offsets
 * whose first value is the offset of d_weights[i][0]) and d_outputs[i]
 * (lengths[i]*samples*2 uint32), all in the generator's device memory.  A
 * matrix with lengths[i] == 0 is skipped.  As with mhcuda_calc_device the work
 * is enqueued on `stream` and the call returns without waiting, calls on one
 * generator must be ordered on one stream, and invalid CSR content in any
 * matrix fails the whole batch as reported by the next
 * mhcuda_device_status().  A batch's descriptors are uploaded to the device
 * once (the last 8 distinct batches are kept per generator), and a batch
 * hashed again replays a CUDA graph of its launches.  Results equal one
 * mhcuda_calc (minhashcuda.h:115-118) per matrix, bit for bit; the reference
 * has no batch call (one launch per call, minhashcuda.cc:583-642). */
enum MHCUDAResult mhcuda_calc_batch_device(
    const MinhashCudaGenerator *gen, uint32_t count,
    const float *const *d_weights, const uint32_t *const *d_cols,
    const uint32_t *const *d_rows, const uint32_t *lengths,
    uint32_t *const *d_outputs, void *stream);

/* Element types accepted by mhcuda_calc_typed. */
enum MHCUDAElementType {
  mhcudaFloat32 = 0,
  mhcudaFloat64 = 1,
  mhcudaUInt32 = 2,
  mhcudaInt32 = 3,
  mhcudaInt64 = 4,
  mhcudaUInt64 = 5
};

/* mhcuda_calc (minhashcuda.h:115-118) for CSR arrays in the element types
 * scipy produces: float64 data, and int64 indices and offsets once a matrix
 * has 2^31 nnz or more.  weights: mhcudaFloat32/Float64; cols and rows: any
 * of the integer types.  The reference casts whole arrays to float32/uint32
 * on the host before its call (python.cc:310-327); here each block of rows is
 * converted while it is staged into page-locked memory on host threads, so
 * nothing is copied whole.  float64 -> float32 rounds to nearest (numpy's
 * astype).  Offsets are taken relative to rows[0], so a row range of a matrix
 * with more than 2^32 nnz works as long as the range itself has fewer.
 * Returns mhcudaInvalidArguments for an unknown type, an offset that
 * decreases or spans 2^32 or more, and a column outside [0, dim) (the
 * reference's cast wraps such values, python.cc:317-323).  Results equal
 * mhcuda_calc on the converted arrays. */
enum MHCUDAResult mhcuda_calc_typed(
    const MinhashCudaGenerator *gen, const void *weights, int weights_type,
    const void *cols, int cols_type, const void *rows, int rows_type,
    uint32_t length, uint32_t *output);

/* Hashes `count` independent CSR matrices (host buffers, as in mhcuda_calc)
 * against one generator in one device pass: the matrices are staged
 * back to back, one persistent launch walks a (matrix, row-chunk) work list
 * and each matrix's hashes land in outputs[i] (lengths[i]*samples*2 uint32).
 * Equivalent to `count` mhcuda_calc calls (minhashcuda.h:115-118), bit for
 * bit.  A matrix with lengths[i] == 0 is skipped. */
enum MHCUDAResult mhcuda_calc_batch(
    const MinhashCudaGenerator *gen, uint32_t count,
    const float *const *weights, const uint32_t *const *cols,
    const uint32_t *const *rows, const uint32_t *lengths,
    uint32_t *const *outputs);

/* Page-locks (registers) `bytes` of the caller's host memory at `ptr` for the
 * copy engines of every device (cudaHostRegisterPortable; the context of the
 * device selected like mhcuda_init's `devices` mask does the registering),
 * or releases such a registration.  mhcuda_calc then copies a CSR held in
 * registered memory straight to the device, with no staging copy on host
 * threads.  Registering runs at about the speed of one pageable copy of the
 * same bytes, so it pays for data hashed more than once (several generators,
 * repeated row-block passes); the Python module's minhash_cuda_pin uses it.
 * Returns mhcudaInvalidArguments for a range that is already registered.
 * No counterpart in the reference (its calls copy from pageable memory,
 * minhashcuda.cc:385-455). */
enum MHCUDAResult mhcuda_host_register(uint32_t devices, const void *ptr, uint64_t bytes);
enum MHCUDAResult mhcuda_host_unregister(uint32_t devices, const void *ptr);

/* Test hook: evaluates the device logf (the one the hash kernel applies to
 * every weight) on n host floats, on the device selected like mhcuda_init's
 * `devices` mask.  No counterpart in the reference. */
enum MHCUDAResult mhcuda_debug_device_logf(
    uint32_t devices, const float *in, float *out, uint64_t n);

/* Starts (enable != 0) or stops timing every hash-kernel launch of the
 * generator with CUDA events recorded on the launch stream, and clears the
 * accumulated figures.  No counterpart in the reference (its build
 * defines PROFILE, CMakeLists.txt:9-11, but no source reads it). */
enum MHCUDAResult mhcuda_profile(const MinhashCudaGenerator *gen, int enable);

/* Waits for the timed launches and returns their summed device time in ms
 * and their count since the last mhcuda_profile/mhcuda_profile_read call,
 * then clears them.  No counterpart in the reference. */
enum MHCUDAResult mhcuda_profile_read(const MinhashCudaGenerator *gen, double *hash_ms,
                                      uint64_t *launches);

/* ---- Downstream of the hash (device-resident hashes) ---------------------
 * d_hashes is [rows][samples][2] uint32 in the generator's device memory, as
 * mhcuda_calc_device writes it.  Both calls wait for their kernel.  No
 * counterpart in the reference, which returns the hashes to the host and
 * leaves their use to the caller (its tests estimate Jaccard similarity from
 * them, test.py:104-106). */

/* LSH band keys: d_keys[row][b] (samples/band_width bands of band_width
 * samples; trailing samples unused) is a 64-bit key of the band's (k, t)
 * pairs: h = 0x6A09E667F3BCC909 ^ b, then h = splitmix64(h ^ (k << 32 | t))
 * per sample.  Rows sharing a key in some band are candidate pairs. */
enum MHCUDAResult mhcuda_lsh_bands(const MinhashCudaGenerator *gen, const uint32_t *d_hashes,
                                   uint32_t rows, uint32_t band_width, uint64_t *d_keys,
                                   void *stream);

/* Weighted-Jaccard estimates: d_out[p] = fraction of samples whose (k, t)
 * pairs are equal for rows d_pairs[2p] and d_pairs[2p+1] (-1 for a pair
 * naming a row >= rows). */
enum MHCUDAResult mhcuda_jaccard(const MinhashCudaGenerator *gen, const uint32_t *d_hashes,
                                 uint32_t rows, const uint32_t *d_pairs, uint64_t npairs,
                                 float *d_out, void *stream);

/* ---- Serving: a continuous-batching request loop on one device ----------
 * No counterpart in the reference (every mhcuda_calc there is one blocking
 * launch per device, minhashcuda.cc:583-642).  `lanes` worker threads keep
 * batches in flight on their own streams; each request (a CSR and an output
 * buffer in host memory, as for mhcuda_calc, hashed against any generator on
 * the server's device) is scheduled shortest-remaining-work first: a free
 * lane batches the requests of one generator with the least work left, whole
 * where they fit and in row blocks otherwise.  Small batches run on a
 * high-priority stream straight from mapped host memory; at most lanes - 2
 * large batches are out at once.  Requests that arrive while others run join
 * the next batch a lane forms.  Device memory used by the server is
 * `hbm_budget_bytes` (split between the lanes at start; nothing grows later).
 * Results are bit-identical to mhcuda_calc. */
typedef struct MinhashCudaServer_ MinhashCudaServer;

/* Starts a server on the device selected like mhcuda_init's `devices`.
 * lanes: 1..16; hbm_budget_bytes >= 64 MiB. */
MinhashCudaServer *mhcuda_server_start(uint32_t devices, uint64_t hbm_budget_bytes,
                                       uint32_t lanes, int verbosity,
                                       enum MHCUDAResult *status);

/* Queues a request and returns its ticket.  The host buffers must stay valid
 * and unmodified until the request is waited for.  Refused with
 * mhcudaMemoryAllocationFailure if one row alone does not fit a lane. */
enum MHCUDAResult mhcuda_server_submit(MinhashCudaServer *srv, const MinhashCudaGenerator *gen,
                                       const float *weights, const uint32_t *cols,
                                       const uint32_t *rows, uint32_t length, uint32_t *output,
                                       uint64_t *ticket);

/* *done = 1 once the request's hashes are in its output buffer. */
enum MHCUDAResult mhcuda_server_poll(MinhashCudaServer *srv, uint64_t ticket, int *done);

/* Waits up to timeout_s for the request, then returns its result
 * (mhcudaInvalidArguments for invalid CSR, mhcudaRuntimeError if cancelled
 * or timed out) and, if latency_ms is not NULL, its submit-to-done time.
 * A finished ticket is released by this call. */
enum MHCUDAResult mhcuda_server_wait(MinhashCudaServer *srv, uint64_t ticket, double timeout_s,
                                     double *latency_ms);

/* Drops the request's blocks that have not started; it then completes with
 * mhcudaRuntimeError.  Returns mhcudaInvalidArguments for an unknown ticket or
 * a request that has already finished (its result stands). */
enum MHCUDAResult mhcuda_server_cancel(MinhashCudaServer *srv, uint64_t ticket);

/* Latency percentiles over completed requests and hashed nnz*samples per
 * second since start or the last reset. */
enum MHCUDAResult mhcuda_server_stats(MinhashCudaServer *srv, int reset, uint64_t *completed,
                                      double *p50_ms, double *p99_ms, double *p999_ms,
                                      double *evals_per_s);

/* Finishes queued work and frees the server. */
enum MHCUDAResult mhcuda_server_stop(MinhashCudaServer *srv);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* MHCUDA_MINHASHCUDA_B200_H */
