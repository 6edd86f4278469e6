// Parameter-table kernels for sm_100a.
//
// Replace gamma_cuda / log_cuda (kernel.cu:18-36 of src-d/minhashcuda) and
// the layout the reference keeps its table in.  The reference runs
//   U1->rs, U2->ln_cs, U3->betas, rs=-logf(U2*U1), U4->ln_cs,
//   ln_cs=-logf(U3*U4), U5->betas, ln_cs=logf(ln_cs)        (minhashcuda.cc:186-200)
// as three element-wise kernels on [samples][dim] arrays, each followed by a
// device-wide synchronisation.  Here one pass per output array reads the two
// uniform streams in [samples][dim] order, applies the same float operations
// (each rounded to float as in the reference: -logf(a*b), then logf of that),
// and writes the result transposed into the [dim][3][s_pad] table through a
// shared-memory tile, so both the read and the write are coalesced.
#include <cstdint>

#include "wmh_internal.h"

namespace mhb {
namespace {

constexpr int kTile = 32;
constexpr int kRowsPerPass = 8;

__device__ __forceinline__ float pair_op(PairOp op, float a, float b) {
  switch (op) {
    case PairOp::kGamma:
      // kernel.cu:24 with v1 = b, v2 = a: -logf(v1 * v2).
      return -logf(b * a);
    case PairOp::kLogGamma: {
      // kernel.cu:24 then kernel.cu:35: logf(-logf(v1 * v2)).
      const float g = -logf(a * b);
      return logf(g);
    }
    default:
      return a;
  }
}

// Block (32, 8): tile of 32 samples x 32 columns.  a and b hold `samples`
// rows of `dim` values, the rows s_base.. of the [samples][dim] streams.
__global__ void pack_kernel(const float *__restrict__ a, const float *__restrict__ b, PairOp op,
                            uint32_t which, uint32_t dim, uint32_t s_base, uint32_t samples,
                            uint32_t s_pad, float *__restrict__ params) {
  __shared__ float tile[kTile][kTile + 1];
  const uint32_t d0 = blockIdx.x * kTile;
  const uint32_t s0 = blockIdx.y * kTile;
  // Read [s][d] rows, coalesced along d.
  for (int k = threadIdx.y; k < kTile; k += kRowsPerPass) {
    const uint32_t s = s0 + k, d = d0 + threadIdx.x;
    if (s < samples && d < dim) {
      const size_t i = static_cast<size_t>(s) * dim + d;
      tile[k][threadIdx.x] = pair_op(op, a[i], b ? b[i] : 0.0f);
    }
  }
  __syncthreads();
  // Write [d][which][s] rows, coalesced along s.
  for (int k = threadIdx.y; k < kTile; k += kRowsPerPass) {
    const uint32_t d = d0 + k, s = s0 + threadIdx.x;
    if (d < dim && s < samples)
      params[(static_cast<size_t>(d) * 3 + which) * s_pad + s_base + s] = tile[threadIdx.x][k];
  }
}

__global__ void unpack_kernel(const float *__restrict__ params, uint32_t which, uint32_t dim,
                              uint32_t s_base, uint32_t samples, uint32_t s_pad,
                              float *__restrict__ dst) {
  __shared__ float tile[kTile][kTile + 1];
  const uint32_t d0 = blockIdx.x * kTile;
  const uint32_t s0 = blockIdx.y * kTile;
  for (int k = threadIdx.y; k < kTile; k += kRowsPerPass) {
    const uint32_t d = d0 + k, s = s0 + threadIdx.x;
    if (d < dim && s < samples)
      tile[k][threadIdx.x] = params[(static_cast<size_t>(d) * 3 + which) * s_pad + s_base + s];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < kTile; k += kRowsPerPass) {
    const uint32_t s = s0 + k, d = d0 + threadIdx.x;
    if (s < samples && d < dim) dst[static_cast<size_t>(s) * dim + d] = tile[threadIdx.x][k];
  }
}

}  // namespace

cudaError_t launch_pack_params(const float *a, const float *b, PairOp op, uint32_t which,
                               uint32_t dim, uint32_t s_base, uint32_t samples, uint32_t s_pad,
                               float *params, cudaStream_t stream) {
  const dim3 block(kTile, kRowsPerPass);
  const dim3 grid((dim + kTile - 1) / kTile, (samples + kTile - 1) / kTile);
  if (grid.x == 0 || grid.y == 0) return cudaSuccess;
  pack_kernel<<<grid, block, 0, stream>>>(a, b, op, which, dim, s_base, samples, s_pad, params);
  return cudaGetLastError();
}

cudaError_t launch_unpack_params(const float *params, uint32_t which, uint32_t dim,
                                 uint32_t s_base, uint32_t samples, uint32_t s_pad, float *dst,
                                 cudaStream_t stream) {
  const dim3 block(kTile, kRowsPerPass);
  const dim3 grid((dim + kTile - 1) / kTile, (samples + kTile - 1) / kTile);
  if (grid.x == 0 || grid.y == 0) return cudaSuccess;
  unpack_kernel<<<grid, block, 0, stream>>>(params, which, dim, s_base, samples, s_pad, dst);
  return cudaGetLastError();
}

}  // namespace mhb
