/*
 * minhashcuda.h -- drop-in C ABI of the B200 weighted-minhash engine.
 *
 * Every type and entry point below keeps the exact name, signature, struct
 * layout and enum values of src-d/minhashcuda's public header so that code
 * compiled against that header links against libmhcuda.so unchanged.  Each
 * declaration names the reference declaration it replaces.
 *
 * Semantics on this engine:
 *  - One generator lives on exactly one CUDA device (the lowest set bit of
 *    the `devices` mask that names a present device; mask 0 means device 0).
 *  - Parameters are kept on the device as one [dim][3][samples] table
 *    (r, ln_c, beta per column); the host-facing layout stays row-major
 *    [samples][dim] float32 for retrieve/assign.
 *  - All calls are synchronous: results are valid when the call returns.
 *  - One generator is not re-entrant; calls on one generator are serialised
 *    by an internal lock.  Different generators are independent (dim is a
 *    kernel argument, not device-global state).
 */
#ifndef MHCUDA_MINHASHCUDA_H
#define MHCUDA_MINHASHCUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifdef __GNUC__
#define MALLOC __attribute__((malloc))
#else
#define MALLOC
#endif

/* Opaque generator handle.  Replaces minhashcuda.h:41. */
typedef struct MinhashCudaGenerator_ MinhashCudaGenerator;

/* Parameters a generator was created with.  Replaces minhashcuda.h:44-48
 * (same members, same order). */
typedef struct {
  uint32_t dim;
  uint16_t samples;
  int verbosity;
} MinhashCudaGeneratorParameters;

/* Return codes.  Replaces minhashcuda.h:51-58 (same enumerators, same
 * values 0..5). */
enum MHCUDAResult {
  mhcudaSuccess,
  mhcudaInvalidArguments,
  mhcudaNoSuchDevice,
  mhcudaMemoryAllocationFailure,
  mhcudaRuntimeError,
  mhcudaMemoryCopyError
};
#ifndef __cplusplus
typedef enum MHCUDAResult MHCUDAResult;
#endif

/* Creates a generator of `samples` hashes over `dim`-dimensional rows.
 * Unless `deferred` is non-zero, rs ~ Gamma(2,1), ln_cs = ln(Gamma(2,1)) and
 * betas ~ U(0,1] are drawn from cuRAND's default pseudo-random generator with
 * `seed`, in the same draw order as the reference, so equal seeds give equal
 * parameters.  With `deferred`, the table is zero-filled and the caller is
 * expected to assign it.  samples may be any value in 1..65535.
 * On error returns NULL and stores the code in *status when status != NULL.
 * Replaces minhashcuda.h:74-76. */
MinhashCudaGenerator *mhcuda_init(
    uint32_t dim, uint16_t samples, uint32_t seed, int deferred,
    uint32_t devices, int verbosity, enum MHCUDAResult *status) MALLOC;

/* Returns {dim, samples, verbosity}; all zero for a NULL generator.
 * Replaces minhashcuda.h:81-82. */
MinhashCudaGeneratorParameters mhcuda_get_parameters(
    const MinhashCudaGenerator *gen);

/* Copies the parameters to three caller buffers of samples*dim floats each,
 * row-major [samples][dim].  Replaces minhashcuda.h:91-92. */
enum MHCUDAResult mhcuda_retrieve_random_vars(
    const MinhashCudaGenerator *gen, float *rs, float *ln_cs, float *betas);

/* Replaces the parameters with three caller buffers of samples*dim floats,
 * row-major [samples][dim].  Replaces minhashcuda.h:101-103. */
enum MHCUDAResult mhcuda_assign_random_vars(
    const MinhashCudaGenerator *gen, const float *rs,
    const float *ln_cs, const float *betas);

/* Hashes `length` CSR rows.  weights/cols are the CSR values and column
 * indices; rows holds length+1 offsets into them (rows[0] is normally 0; a
 * non-zero rows[0] is honoured as an absolute offset).  output receives
 * length*samples*2 uint32: for row i and sample s, output[(i*samples+s)*2]
 * is the arg-min column k and [..+1] is (uint32)(int32)t.  A (row, sample)
 * without any positive finite weight gets (0xFFFFFFFF, 0xFFFFFFFF).
 * Returns mhcudaInvalidArguments for NULL pointers, length == 0, a column
 * index >= dim or decreasing row offsets.  Host buffers may be pageable or
 * pinned.  Replaces minhashcuda.h:115-118. */
enum MHCUDAResult mhcuda_calc(
    const MinhashCudaGenerator *gen, const float *weights,
    const uint32_t *cols, const uint32_t *rows, uint32_t length,
    uint32_t *output);

/* Frees the generator and everything it holds on the device.  NULL is a
 * no-op.  Replaces minhashcuda.h:124. */
enum MHCUDAResult mhcuda_fini(MinhashCudaGenerator *gen);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* MHCUDA_MINHASHCUDA_H */
