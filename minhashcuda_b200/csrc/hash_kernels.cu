// Weighted-minhash hash kernels for sm_100a.
//
// Replaces weighted_minhash_cuda (kernel.cu:56-112 of src-d/minhashcuda) and
// the host-side binpacking that fed it (minhashcuda.cc:457-528).
//
// Per (row, sample) the value computed is the reference's (kernel.cu:95-110):
//   w = logf(weight); t = floorf(w / r + beta);
//   ln_a = ln_c - (t - beta) * r - r;  keep the first strict minimum.
// Each operation is spelled with an explicit round-to-nearest intrinsic so the
// compiler cannot re-associate or contract differently from the reference
// build: the multiply-subtract of kernel.cu:104-105 is one fused multiply-add
// (the form the reference build evaluates; pinned on a B200 by the tests).
//
// Layout and mapping (B200-first, not the reference's):
//  - parameters are [dim][3][s_pad]: one nnz's r / ln_c / beta for a tile of
//    32*SPL samples are three fully coalesced warp loads (SPL=4: 3 x 512 B),
//  - a warp owns one (chunk, sample tile) item; each lane keeps SPL running
//    minima in registers (no shared-memory spill as in kernel.cu:72-74),
//  - ln(weight) is evaluated once per nnz, lane-parallel over a 32-entry
//    block of the CSR (the reference evaluates it once per thread, :95), and
//    broadcast with warp shuffles,
//  - work is cut by nnz, not by rows, so one 50k-nnz row and many 5-nnz rows
//    cost the same per item; rows that cross a chunk boundary are merged by
//    a finalize pass (tie -> earlier position, as the strict '<' scan).
#include <cfloat>
#include <cstdint>

#include "wmh_internal.h"

namespace mhb {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

template <int SPL>
struct Lanes {
  float v[SPL];
  __device__ __forceinline__ void load(const float *__restrict__ p) {
    if constexpr (SPL == 4) {
      const float4 x = __ldg(reinterpret_cast<const float4 *>(p));
      v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else if constexpr (SPL == 2) {
      const float2 x = __ldg(reinterpret_cast<const float2 *>(p));
      v[0] = x.x; v[1] = x.y;
    } else {
      v[0] = __ldg(p);
    }
  }
};

// One (nnz, sample) evaluation, kernel.cu:101-109.
__device__ __forceinline__ void wmh_eval(float w, float r, float c, float b, uint32_t d,
                                         float &mn, uint32_t &kk, float &tf) {
  const float t = floorf(__fadd_rn(__fdiv_rn(w, r), b));
  const float tb = __fsub_rn(t, b);
  const float ln_a = __fsub_rn(__fmaf_rn(-tb, r, c), r);
  if (ln_a < mn) {
    mn = ln_a;
    kk = d;
    tf = t;
  }
}

__device__ __forceinline__ uint2 final_pair(uint32_t k, float t) {
  // (uint32)(int32)t as kernel.cu:108; the GPU conversion saturates.
  return k == kNone ? make_uint2(kNone, kNone)
                    : make_uint2(k, static_cast<uint32_t>(static_cast<int32_t>(t)));
}

// chunk_row[c] = first row whose first position is >= c*chunk (rows if none).
__global__ void plan_kernel(const HashArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > a.rows) return;
  const uint32_t base = a.indptr[0];
  uint32_t start, c_hi;
  if (i < a.rows) {
    const uint32_t s = a.indptr[i], e = a.indptr[i + 1];
    if (e < s || s < base) atomicOr(a.status, kStatusBadIndptr);
    start = s - base;
    c_hi = min(start / a.chunk, a.nchunks - 1);
  } else {
    if (a.indptr[a.rows] - base != a.nnz || a.indptr[a.rows] < base)
      atomicOr(a.status, kStatusBadIndptr);
    start = 0xFFFFFFFFu;
    c_hi = a.nchunks - 1;
  }
  uint32_t c_lo = 0;
  if (i > 0) {
    const uint32_t prev = a.indptr[i - 1] - base;
    c_lo = prev / a.chunk + 1;
  }
  for (uint32_t c = c_lo; c <= c_hi && c < a.nchunks; ++c) a.chunk_row[c] = i;
  (void)start;
}

template <int SPL>
struct RowState {
  float mn[SPL];
  uint32_t kk[SPL];
  float tf[SPL];
  __device__ __forceinline__ void reset() {
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
      mn[j] = FLT_MAX;
      kk[j] = kNone;
      tf[j] = 0.0f;
    }
  }
};

template <int SPL>
__device__ __forceinline__ void store_final(const HashArgs &a, uint32_t row, uint32_t s0,
                                            const RowState<SPL> &st) {
  uint32_t *o = a.out + (static_cast<size_t>(row) * a.samples + s0) * 2;
#pragma unroll
  for (int j = 0; j < SPL; ++j) {
    if (s0 + j < a.samples) *reinterpret_cast<uint2 *>(o + 2 * j) = final_pair(st.kk[j], st.tf[j]);
  }
}

template <int SPL>
__device__ __forceinline__ void store_partial(const HashArgs &a, uint32_t slot, uint32_t s0,
                                              const RowState<SPL> &st) {
  const size_t off = static_cast<size_t>(slot) * a.s_pad + s0;
#pragma unroll
  for (int j = 0; j < SPL; ++j) {
    a.part_ln[off + j] = st.mn[j];
    a.part_kt[off + j] = make_uint2(st.kk[j], __float_as_uint(st.tf[j]));
  }
}

template <int SPL>
__global__ void __launch_bounds__(kHashBlock, 3) hash_kernel(const HashArgs a) {
  if (*a.status & kStatusBadIndptr) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t base = a.indptr[0];
  const uint32_t items = a.nchunks * a.ntiles;
  const size_t col_stride = static_cast<size_t>(3) * a.s_pad;

  for (uint32_t item = gw; item < items; item += nw) {
    const uint32_t c = item / a.ntiles;
    const uint32_t tile = item - c * a.ntiles;
    const uint32_t s0 = tile * (32u * SPL) + lane * SPL;
    const bool active = s0 < a.s_pad;
    const uint32_t cs = c * a.chunk;
    const uint32_t ce = min(a.nnz, cs + a.chunk);
    uint32_t r_next = a.chunk_row[c];
    const uint32_t r_stop = (c + 1 < a.nchunks) ? a.chunk_row[c + 1] : a.rows;

    // The row being accumulated: kNone, the row running in from the previous
    // chunk (head), or an owned row.
    uint32_t row = kNone, row_end = cs;
    bool head = false;
    if (r_next > 0) {
      const uint32_t e = a.indptr[r_next] - base;
      if (e > cs) {
        row = r_next - 1;
        row_end = e;
        head = true;
      }
    }
    RowState<SPL> st;
    st.reset();

    auto flush = [&]() {
      if (row == kNone || !active) return;
      if (head) {
        store_partial<SPL>(a, 2 * c, s0, st);
      } else if (row_end > ce) {
        store_partial<SPL>(a, 2 * c + 1, s0, st);
      } else {
        store_final<SPL>(a, row, s0, st);
      }
    };

    // CSR block registers: lane l holds position blk + l.
    uint32_t blk = cs;
    float lw_cur;
    uint32_t col_cur;
    {
      const uint32_t p = blk + lane;
      const float wr = p < ce ? __ldg(a.weights + p) : 1.0f;
      col_cur = p < ce ? __ldg(a.cols + p) : 0u;
      lw_cur = logf(wr);
    }
    float w_nx = 1.0f;
    uint32_t col_nx = 0u;
    {
      const uint32_t p = blk + 32u + lane;
      if (p < ce) {
        w_nx = __ldg(a.weights + p);
        col_nx = __ldg(a.cols + p);
      }
    }

    Lanes<SPL> r_c, c_c, b_c;
    uint32_t d_cur = __shfl_sync(kFull, col_cur, 0);
    if (cs < ce && active && d_cur < a.dim) {
      const float *pp = a.params + d_cur * col_stride + s0;
      r_c.load(pp);
      c_c.load(pp + a.s_pad);
      b_c.load(pp + 2 * a.s_pad);
    }

    for (uint32_t p = cs; p < ce; ++p) {
      while (p >= row_end) {
        flush();
        // Owned rows start where the previous one ended; empty ones are
        // flushed here with no selection.
        if (r_next >= r_stop) {  // only reachable with inconsistent offsets
          if (lane == 0) atomicOr(a.status, kStatusBadIndptr);
          return;
        }
        row = r_next++;
        row_end = a.indptr[row + 1] - base;
        head = false;
        st.reset();
      }
      const uint32_t pn = p + 1;
      const uint32_t ln = pn & 31u;
      const uint32_t d_nx = __shfl_sync(kFull, ln ? col_cur : col_nx, ln);
      Lanes<SPL> r_n, c_n, b_n;
      if (pn < ce && active && d_nx < a.dim) {
        const float *pp = a.params + d_nx * col_stride + s0;
        r_n.load(pp);
        c_n.load(pp + a.s_pad);
        b_n.load(pp + 2 * a.s_pad);
      }
      const float w = __shfl_sync(kFull, lw_cur, p & 31u);
      if (d_cur < a.dim) {
#pragma unroll
        for (int j = 0; j < SPL; ++j)
          wmh_eval(w, r_c.v[j], c_c.v[j], b_c.v[j], d_cur, st.mn[j], st.kk[j], st.tf[j]);
      } else if (lane == 0) {
        atomicOr(a.status, kStatusBadColumn);
      }
      r_c = r_n;
      c_c = c_n;
      b_c = b_n;
      d_cur = d_nx;
      if (ln == 0 && pn < ce) {
        blk += 32u;
        lw_cur = logf(w_nx);
        col_cur = col_nx;
        const uint32_t q = blk + 32u + lane;
        w_nx = 1.0f;
        col_nx = 0u;
        if (q < ce) {
          w_nx = __ldg(a.weights + q);
          col_nx = __ldg(a.cols + q);
        }
      }
    }
    flush();
    // Remaining owned rows are empty and start at ce (only possible in the
    // last chunk: trailing empty rows).
    while (r_next < r_stop) {
      row = r_next++;
      row_end = ce;
      head = false;
      st.reset();
      flush();
    }
  }
}

// Merge the partials of every row that leaves its own chunk.
__global__ void finalize_kernel(const HashArgs a) {
  if (*a.status & kStatusBadIndptr) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t base = a.indptr[0];
  for (uint32_t c = gw; c < a.nchunks; c += nw) {
    const uint32_t r0 = a.chunk_row[c];
    const uint32_t r1 = (c + 1 < a.nchunks) ? a.chunk_row[c + 1] : a.rows;
    if (r1 <= r0) continue;
    const uint32_t row = r1 - 1;
    const uint32_t end = a.indptr[row + 1] - base;
    const uint32_t ce = min(a.nnz, c * a.chunk + a.chunk);
    if (end <= ce) continue;
    const uint32_t c_last = (end - 1) / a.chunk;
    uint32_t *o = a.out + static_cast<size_t>(row) * a.samples * 2;
    for (uint32_t s = lane; s < a.samples; s += 32) {
      size_t off = static_cast<size_t>(2 * c + 1) * a.s_pad + s;
      float mn = a.part_ln[off];
      uint2 kt = a.part_kt[off];
      for (uint32_t cc = c + 1; cc <= c_last; ++cc) {
        off = static_cast<size_t>(2 * cc) * a.s_pad + s;
        const float m2 = a.part_ln[off];
        if (m2 < mn) {
          mn = m2;
          kt = a.part_kt[off];
        }
      }
      *reinterpret_cast<uint2 *>(o + 2 * s) = final_pair(kt.x, __uint_as_float(kt.y));
    }
  }
}

__global__ void logf_kernel(const float *in, float *out, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[i] = logf(in[i]);
}

}  // namespace

cudaError_t launch_plan(const HashArgs &a, cudaStream_t stream) {
  const uint32_t threads = 256;
  const uint32_t blocks = (a.rows + 1 + threads - 1) / threads;
  plan_kernel<<<blocks, threads, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_hash(const HashArgs &a, const HashPlan &plan, cudaStream_t stream) {
  switch (plan.spl) {
    case 4: hash_kernel<4><<<plan.grid, kHashBlock, 0, stream>>>(a); break;
    case 2: hash_kernel<2><<<plan.grid, kHashBlock, 0, stream>>>(a); break;
    case 1: hash_kernel<1><<<plan.grid, kHashBlock, 0, stream>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_finalize(const HashArgs &a, cudaStream_t stream) {
  const uint32_t warps_per_block = 8;
  uint32_t blocks = (a.nchunks + warps_per_block - 1) / warps_per_block;
  if (blocks > 4096) blocks = 4096;
  finalize_kernel<<<blocks, 32 * warps_per_block, 0, stream>>>(a);
  return cudaGetLastError();
}

int hash_blocks_per_sm(uint32_t spl) {
  int n = 0;
  cudaError_t e = cudaErrorInvalidValue;
  switch (spl) {
    case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hash_kernel<4>, kHashBlock, 0); break;
    case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hash_kernel<2>, kHashBlock, 0); break;
    case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, hash_kernel<1>, kHashBlock, 0); break;
    default: break;
  }
  return e == cudaSuccess && n > 0 ? n : 1;
}

size_t hash_kernel_registers(uint32_t spl) {
  cudaFuncAttributes attr{};
  switch (spl) {
    case 4: cudaFuncGetAttributes(&attr, hash_kernel<4>); break;
    case 2: cudaFuncGetAttributes(&attr, hash_kernel<2>); break;
    case 1: cudaFuncGetAttributes(&attr, hash_kernel<1>); break;
    default: break;
  }
  return attr.numRegs;
}

cudaError_t launch_logf(const float *in, float *out, size_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  size_t blocks = (n + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  logf_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(in, out, n);
  return cudaGetLastError();
}

}  // namespace mhb
