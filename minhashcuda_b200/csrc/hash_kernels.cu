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
//    each with the position of its entry; (k, t) are recovered once per
//    (row, sample) at the row's end,
//  - each warp stages its CSR positions in 256-entry windows with TMA bulk
//    copies (cp.async.bulk, mbarrier completion, double-buffered), turns the
//    weights into ln(weight) in place once per nnz, lane-parallel (the
//    reference evaluates logf once per thread, :95), validates the window's
//    columns once, and reads them back as shared-memory broadcasts,
//  - parameters for the next nnz are loaded into a second register set while
//    the current one is evaluated (ping-pong, no register copies); the loop
//    has no branch per nnz, samples are evaluated in pairs with packed f32x2
//    arithmetic, and the running minimum is updated with selects,
//  - work is cut by nnz, not by rows, so one 50k-nnz row and many 5-nnz rows
//    cost the same per item; rows that cross a chunk boundary are merged by
//    a finalize pass (tie -> earlier position, as the strict '<' scan).
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstdlib>

#include "wmh_internal.h"

namespace mhb {
namespace {

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

// t of kernel.cu:103 exactly as the reference computes it: IEEE quotient,
// rounded sum, floor.
__device__ __forceinline__ float exact_t(float w, float r, float b) {
  return floorf(__fadd_rn(__fdiv_rn(w, r), b));
}

// Margin of the fast t below, relative to |w/r| + |beta| + 1.
constexpr float kTMargin = 0x1p-18f;

// Fast t.  Only floor(v) with v = RN(RN(w/r) + beta) is needed, and it only
// depends on the exact quotient when v lies close to an integer.  With
// y = rcp.approx(r) (documented error 1 ulp; 2^-22 relative assumed) and
// va = RN(RN(w*y) + beta):
//   |va - v| <= |w/r| * 2^-20.6 + |beta| * 2^-23 < m,
//   m = (|w*y| + |beta| + 1) * 2^-18,
// so when va is more than m away from every integer, floor(va) = floor(v).
// Returns false (t undecided) otherwise, and for every non-finite or
// flushed case (w = +-inf/NaN, r = 0/denormal/huge, |va| >= 2^22: m >= 16).
__device__ __forceinline__ bool fast_t(float w, float r, float b, float &t) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(r));
  const float qa = __fmul_rn(w, y);
  const float va = __fadd_rn(qa, b);
  t = floorf(va);
  const float f = __fsub_rn(va, t);  // exact for |va| >= 1; 1.0 or exact for va in (-1, 1)
  const float m = __fmaf_rn(__fadd_rn(fabsf(qa), fabsf(b)), kTMargin, kTMargin);
  return fabsf(__fsub_rn(f, 0.5f)) < __fsub_rn(0.5f, m);  // NaN -> false
}

// One (nnz, sample) evaluation, kernel.cu:101-109, given t: keeps the
// minimum and the position `p` it came from.
__device__ __forceinline__ void wmh_update(float t, float r, float c, float b, uint32_t p,
                                           float &mn, uint32_t &pos) {
  const float tb = __fsub_rn(t, b);
  const float ln_a = __fsub_rn(__fmaf_rn(-tb, r, c), r);
  const bool lt = ln_a < mn;
  mn = lt ? ln_a : mn;
  pos = lt ? p : pos;
}

// Column of relative position p in a packed CSR.
__device__ __forceinline__ uint32_t packed_col(const HashArgs &a, uint32_t p) {
  const uint32_t h = a.col_hi_bits == 4 ? (a.cols_hi[p >> 1] >> ((p & 1u) * 4)) & 15u
                                        : a.cols_hi[p];
  return static_cast<uint32_t>(a.cols_lo[p]) | (h << 16);
}

// The output pair of kernel.cu:108 for sample s whose minimum came from the
// entry at relative position `pos`: k = cols[pos] and t recomputed from the
// entry with the exact quotient.  Every evaluation used that same t (fast_t
// only decides t when it equals the exact one), so tracking the position
// instead of (k, t) changes nothing but the work per evaluation.
// (uint32)(int32)t as kernel.cu:108; the GPU conversion saturates.
// A position outside [0, nnz) (none found, or a partial that a failed launch
// left unwritten) yields kNone and reads nothing.
__device__ __forceinline__ uint2 resolve(const HashArgs &a, uint32_t pos, uint32_t s) {
  if (pos >= a.nnz) return make_uint2(kNone, kNone);
  const uint32_t k = a.col_hi_bits ? packed_col(a, pos) : a.cols[pos];
  // An invalid column was evaluated as column 0 and failed the call: keep
  // the parameter reads in bounds.
  if (k >= a.dim) return make_uint2(kNone, kNone);
  const float w = logf(a.weights[pos]);
  const float *col = a.params + static_cast<size_t>(k) * 3 * a.s_pad + s;
  const float t = exact_t(w, col[0], col[2 * static_cast<size_t>(a.s_pad)]);
  return make_uint2(k, static_cast<uint32_t>(static_cast<int32_t>(t)));
}

// chunk_row[c] = first row whose first position is >= c*chunk (rows if none),
// for the chunks whose first owned row is row i (i == rows: the chunks past
// the last row start); also validates the offsets.
__device__ __forceinline__ void plan_row(const HashArgs &a, uint32_t i) {
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

__global__ void plan_kernel(const HashArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= a.rows) plan_row(a, i);
}

template <int SPL>
struct RowState {
  float mn[SPL];
  uint32_t pos[SPL];  // relative position of the minimum, kNone if none
  __device__ __forceinline__ void reset() {
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
      mn[j] = FLT_MAX;
      pos[j] = kNone;
    }
  }
};

template <int SPL>
__device__ __forceinline__ void store_final(const HashArgs &a, uint32_t row, uint32_t s0,
                                            const RowState<SPL> &st) {
  uint32_t *o = a.out + (static_cast<size_t>(row) * a.samples + s0) * 2;
#pragma unroll
  for (int j = 0; j < SPL; ++j) {
    if (s0 + j < a.samples) *reinterpret_cast<uint2 *>(o + 2 * j) = resolve(a, st.pos[j], s0 + j);
  }
}

template <int SPL>
__device__ __forceinline__ void store_partial(const HashArgs &a, uint32_t slot, uint32_t s0,
                                              const RowState<SPL> &st) {
  const size_t off = static_cast<size_t>(slot) * a.s_pad + s0;
#pragma unroll
  for (int j = 0; j < SPL; ++j) {
    a.part_ln[off + j] = st.mn[j];
    a.part_kt[off + j] = make_uint2(st.pos[j], 0u);
  }
}

// ---- TMA bulk staging of the CSR (per warp, double-buffered) -------------

constexpr uint32_t kWin = 256;  // CSR positions per staged window
constexpr uint32_t kSpinLimit = 1u << 22;

// One warp's staging area: two windows of weights (turned into ln w in
// place) and column indices, each with its own transaction barrier.  Column
// slots n and n + 1 of a window of n positions hold column 0, so the loop may
// prefetch two positions past the window without a bounds branch (the row stride of c,
// kWin + 4 words, keeps both windows 16-byte aligned for the bulk copies).
struct alignas(16) WarpStage {
  float w[2][kWin];
  uint32_t c[2][kWin + 4];
  unsigned long long bar[2];
};

// Landing area of packed columns (HashArgs::col_hi_bits != 0): the low 16
// bits and the high nibbles or bytes of each window's columns, rebuilt into
// WarpStage::c by finish_window.
struct alignas(16) PackedStage {
  uint16_t lo[2][kWin];
  uint8_t hi[2][kWin];
};


__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Global -> this CTA's shared memory, completion counted on `bar`.  Both
// addresses 16-byte aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Positions of a window that arrive by bulk copy: a multiple of 4 (16 bytes
// of weights and of columns), or of 32 with packed columns (16 bytes of high
// nibbles); window starts are multiples of 32.
template <bool PACKED>
__device__ __forceinline__ uint32_t bulk_positions(uint32_t n, bool bulk_ok) {
  return bulk_ok ? (n & (PACKED ? ~31u : ~3u)) : 0u;
}

// Lane 0 starts the copy of positions [ws, ws + n) into buffer `b`: the
// 16-byte-aligned body by bulk copies, the ragged tail is left to
// finish_window's plain loads.
template <bool PACKED>
__device__ __forceinline__ void issue_window(const HashArgs &a, WarpStage &st, PackedStage *pk,
                                             uint32_t b, uint32_t ws, uint32_t n, bool bulk_ok,
                                             uint32_t lane) {
  // Order this warp's earlier generic accesses of the buffer before the
  // asynchronous writes that are about to land in it.
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncwarp();
  if (lane == 0) {
    const uint32_t nb = bulk_positions<PACKED>(n, bulk_ok);
    if (nb) {
      if constexpr (PACKED) {
        const uint32_t hi_bytes = a.col_hi_bits == 4 ? nb / 2 : nb;
        const uint32_t hi_off = a.col_hi_bits == 4 ? ws / 2 : ws;
        mbar_arrive_expect_tx(&st.bar[b], 6u * nb + hi_bytes);
        bulk_copy_g2s(st.w[b], a.weights + ws, 4u * nb, &st.bar[b]);
        bulk_copy_g2s(pk->lo[b], a.cols_lo + ws, 2u * nb, &st.bar[b]);
        bulk_copy_g2s(pk->hi[b], a.cols_hi + hi_off, hi_bytes, &st.bar[b]);
      } else {
        mbar_arrive_expect_tx(&st.bar[b], 8u * nb);
        bulk_copy_g2s(st.w[b], a.weights + ws, 4u * nb, &st.bar[b]);
        bulk_copy_g2s(st.c[b], a.cols + ws, 4u * nb, &st.bar[b]);
      }
    } else {
      mbar_arrive(&st.bar[b]);
    }
  }
}

// Waits for buffer `b` (bounded), loads the tail, turns weights into
// ln(weight) in place -- once per nnz, lane-parallel -- and validates the
// columns: a column >= dim flags kStatusBadColumn (the call then fails, its
// hashes are not valid output) and is replaced by column 0, so the
// evaluation loop reads only in-bounds parameters without a check per nnz.
// Returns false if the copy did not complete within the spin limit.
template <bool PACKED>
__device__ __forceinline__ bool finish_window(const HashArgs &a, WarpStage &st, PackedStage *pk,
                                              uint32_t b, uint32_t parity, uint32_t ws,
                                              uint32_t n, bool bulk_ok, uint32_t lane) {
  uint32_t spins = 0;
  while (!mbar_try_wait(&st.bar[b], parity)) {
    if (++spins > kSpinLimit) return false;
  }
  const uint32_t nb = bulk_positions<PACKED>(n, bulk_ok);
  bool bad = false;
  for (uint32_t i = lane; i < n; i += 32) {
    float x;
    uint32_t col;
    if constexpr (PACKED) {
      if (i < nb) {
        x = st.w[b][i];
        const uint32_t h = a.col_hi_bits == 4 ? (pk->hi[b][i >> 1] >> ((i & 1u) * 4)) & 15u
                                              : pk->hi[b][i];
        col = static_cast<uint32_t>(pk->lo[b][i]) | (h << 16);
      } else {
        x = __ldg(a.weights + ws + i);
        col = packed_col(a, ws + i);
      }
    } else if (i < nb) {
      x = st.w[b][i];
      col = st.c[b][i];
    } else if (a.host_csr) {  // mapped host memory: plain loads
      x = a.weights[ws + i];
      col = a.cols[ws + i];
    } else {
      x = __ldg(a.weights + ws + i);
      col = __ldg(a.cols + ws + i);
    }
    if (col >= a.dim) {
      bad = true;
      col = 0;
    }
    st.c[b][i] = col;
    st.w[b][i] = logf(x);
  }
  if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicOr(a.status, kStatusBadColumn);
  if (lane == 0) st.c[b][n] = st.c[b][n + 1] = 0;  // the prefetch slots past the window
  __syncwarp();
  return true;
}

template <int SPL>
struct Params {
  Lanes<SPL> r, c, b;
  __device__ __forceinline__ void load(const float *__restrict__ col_base, uint32_t s_pad) {
    r.load(col_base);
    c.load(col_base + s_pad);
    b.load(col_base + 2 * s_pad);
  }
};

// ---- Packed pairs of float32 (sm_100 f32x2 arithmetic) --------------------
// One add/sub/mul/fma.rn.f32x2 applies the IEEE round-to-nearest operation
// to both halves independently, so a pair computes exactly what two
// __fadd_rn / __fsub_rn / __fmul_rn / __fmaf_rn calls compute, in one issue.
struct F2 {
  unsigned long long v;
};
__device__ __forceinline__ F2 f2(float lo, float hi) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void split(F2 x, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x.v));
}
__device__ __forceinline__ F2 add2(F2 a, F2 b) {
  F2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 sub2(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 mul2(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

// Selects for samples j and j+1 given their ln_a pair (position p).
template <int SPL>
__device__ __forceinline__ void update_pair(F2 ln_a, uint32_t p, int j, RowState<SPL> &st) {
  float l0, l1;
  split(ln_a, l0, l1);
  const bool lt0 = l0 < st.mn[j], lt1 = l1 < st.mn[j + 1];
  st.mn[j] = lt0 ? l0 : st.mn[j];
  st.pos[j] = lt0 ? p : st.pos[j];
  st.mn[j + 1] = lt1 ? l1 : st.mn[j + 1];
  st.pos[j + 1] = lt1 ? p : st.pos[j + 1];
}

template <int SPL>
__device__ __forceinline__ void eval_all(const Params<SPL> &p, float w, uint32_t pos, bool active,
                                         RowState<SPL> &st) {
  float t[SPL];
  bool undecided = false;
  if constexpr (SPL % 2 == 0) {
    // fast_t on sample pairs.  The bound is fast_t's; the limit 0.5 - m is
    // one fma, (|qa| + |b|) * -2^-18 + (0.5 - 2^-18), whose single rounding
    // (<= 2^-26) is covered by the additive 2^-18 in m.
    const F2 ww = f2(w, w);
#pragma unroll
    for (int j = 0; j < SPL; j += 2) {
      float y0, y1;
      asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(p.r.v[j]));
      asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y1) : "f"(p.r.v[j + 1]));
      const F2 qa = mul2(ww, f2(y0, y1));
      const F2 va = add2(qa, f2(p.b.v[j], p.b.v[j + 1]));
      float q0, q1;
      split(qa, q0, q1);
      float v0, v1;
      split(va, v0, v1);
      t[j] = floorf(v0);
      t[j + 1] = floorf(v1);
      const F2 fr = sub2(va, f2(t[j], t[j + 1]));
      const F2 s = f2(__fadd_rn(fabsf(q0), fabsf(p.b.v[j])),
                      __fadd_rn(fabsf(q1), fabsf(p.b.v[j + 1])));
      const F2 lim = fma2(s, f2(-kTMargin, -kTMargin), f2(0.5f - kTMargin, 0.5f - kTMargin));
      const F2 dv = sub2(fr, f2(0.5f, 0.5f));
      float d0, d1, l0, l1;
      split(dv, d0, d1);
      split(lim, l0, l1);
      undecided |= !(fabsf(d0) < l0) || !(fabsf(d1) < l1);  // NaN -> undecided
    }
  } else {
#pragma unroll
    for (int j = 0; j < SPL; ++j) undecided |= !fast_t(w, p.r.v[j], p.b.v[j], t[j]);
  }
  // Rare: some lane's t sits within the margin of an integer; the warp takes
  // the exact quotient for all its samples (warp-uniform branch).
  if (__any_sync(0xFFFFFFFFu, undecided && active)) {
#pragma unroll
    for (int j = 0; j < SPL; ++j) t[j] = exact_t(w, p.r.v[j], p.b.v[j]);
  }
  if constexpr (SPL % 2 == 0) {
    // ln_a = fma(-(t - beta), r, ln_c) - r on pairs; beta - t is -(t - beta)
    // exactly (round-to-nearest is symmetric).
#pragma unroll
    for (int j = 0; j < SPL; j += 2) {
      const F2 rr = f2(p.r.v[j], p.r.v[j + 1]);
      const F2 nb = sub2(f2(p.b.v[j], p.b.v[j + 1]), f2(t[j], t[j + 1]));
      const F2 ln_a = sub2(fma2(nb, rr, f2(p.c.v[j], p.c.v[j + 1])), rr);
      update_pair<SPL>(ln_a, pos, j, st);
    }
  } else {
#pragma unroll
    for (int j = 0; j < SPL; ++j)
      wmh_update(t[j], p.r.v[j], p.c.v[j], p.b.v[j], pos, st.mn[j], st.pos[j]);
  }
}

// Per-warp state of the hash kernels: the staging buffers, their barrier
// phases and the launch-wide constants of the item loop.
struct WarpCtx {
  WarpStage *stg;
  PackedStage *pk;  // packed-column landing area (packed kernels only)
  uint32_t parity;  // bit b: phase parity to wait for on buffer b
  uint32_t lane;
};

__device__ __forceinline__ void warp_ctx_init(WarpCtx &w, WarpStage *stage_all,
                                              PackedStage *packed_all = nullptr) {
  w.lane = threadIdx.x & 31u;
  w.stg = &stage_all[threadIdx.x >> 5];
  w.pk = packed_all ? &packed_all[threadIdx.x >> 5] : nullptr;
  if (w.lane == 0) {
    mbar_init(&w.stg->bar[0], 1);
    mbar_init(&w.stg->bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  w.parity = 0;
}

// Parameter sets a warp keeps in registers for register budget MINB
// (resident blocks per SM).  The gathers are latency-bound; with 2 blocks per
// SM there are half the warps of the 4-block budget to hide them, and 128
// registers per thread, room for a third set (12 registers at 4 samples per
// lane) that keeps two positions' gathers in flight: 114-118 registers, no
// spills.  At 524,288 rows of the 1,000,000-dim Zipf(1.1) matrix this took
// the 2-block kernel from 107.6 to 101.9 ms (4 blocks: 105.6 ms); on uniform
// columns over 12,000,000 dims from 75.1 to 65.0 ms (4 blocks: 61.6 ms).  The
// 3- and 4-block budgets (85 and 64 registers) have no room for it.
__host__ __device__ constexpr int param_depth(int minb) { return minb == 2 ? 3 : 2; }

// One (chunk c, sample tile) item over the CSR of `a`: finishes the rows
// that lie inside chunk c and leaves partial minima for the rows that cross
// its ends.  Returns false after an error exit (status flagged, in-flight
// staging copies drained); the warp must then stop.
// SPAD: the generator's s_pad when it is known at compile time (0: read it
// from the arguments), which turns the parameter-block addressing into one
// wide multiply-add and immediate load offsets.
// DEPTH: parameter sets in registers, 2 (the next position is loaded while
// one is evaluated) or 3 (the next two are), see param_depth.
template <int SPL, int SPAD, bool PACKED, int DEPTH>
__device__ __forceinline__ bool hash_item(const HashArgs &a, uint32_t c, uint32_t tile,
                                          WarpCtx &wc) {
  const uint32_t lane = wc.lane;
  WarpStage &stg = *wc.stg;
  PackedStage *pk = wc.pk;
  uint32_t &parity = wc.parity;
  const uint32_t base = a.indptr[0];
  const uint32_t spad = SPAD ? static_cast<uint32_t>(SPAD) : a.s_pad;
  const size_t col_stride = static_cast<size_t>(3) * (SPAD ? static_cast<uint32_t>(SPAD) : a.s_pad);
  // Bulk copies only from device memory; mapped host CSR is read by the lanes.
  const uintptr_t col_addr =
      PACKED ? (reinterpret_cast<uintptr_t>(a.cols_lo) | reinterpret_cast<uintptr_t>(a.cols_hi))
             : reinterpret_cast<uintptr_t>(a.cols);
  const bool bulk_ok =
      !a.host_csr && ((reinterpret_cast<uintptr_t>(a.weights) | col_addr) & 15u) == 0;
  {
    const uint32_t s0 = tile * (32u * SPL) + lane * SPL;
    const bool active = s0 < spad;
    // Lanes past the last sample read the tile's first samples (in bounds)
    // and never store, so parameter loads need no branch.
    const float *__restrict__ pbase = a.params + (active ? s0 : tile * (32u * SPL));
    const uint32_t cs = c * a.chunk;
    const uint32_t ce = cs + min(a.chunk, a.nnz - cs);  // no uint32 overflow near 2^32
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

    const uint32_t nwin = (ce - cs + kWin - 1) / kWin;
    if (nwin > 0) issue_window<PACKED>(a, stg, pk, 0, cs, min(kWin, ce - cs), bulk_ok, lane);
    if (nwin > 1)
      issue_window<PACKED>(a, stg, pk, 1, cs + kWin, min(kWin, ce - cs - kWin), bulk_ok, lane);

    // Error exits wait (bounded) for the windows still in flight into this
    // warp's staging buffers before leaving: windows [from, min(from+2, nwin)).
    auto drain = [&](uint32_t from) {
      for (uint32_t kk = from; kk < nwin && kk < from + 2; ++kk) {
        const uint32_t bb = kk & 1u;
        for (uint32_t spins = 0; !mbar_try_wait(&stg.bar[bb], (parity >> bb) & 1u);)
          if (++spins > kSpinLimit) break;
        parity ^= 1u << bb;
      }
    };

    for (uint32_t k = 0; k < nwin; ++k) {
      const uint32_t b = k & 1u;
      const uint32_t ws = cs + k * kWin;
      const uint32_t n = min(kWin, ce - ws);
      if (!finish_window<PACKED>(a, stg, pk, b, (parity >> b) & 1u, ws, n, bulk_ok, lane)) {
        if (lane == 0) atomicOr(a.status, kStatusStall);
        drain(k);
        return false;
      }
      parity ^= 1u << b;
      const float *__restrict__ lw = stg.w[b];
      const uint32_t *__restrict__ cl = stg.c[b];

      // Columns in the window are < dim, and slots n and n + 1 hold column 0
      // (finish_window).
      if constexpr (DEPTH == 3) {
        // Three parameter sets: at each segment's start A holds position i
        // and B position i + 1; positions up to n + 1 read the zero column
        // slots past the window.
        Params<SPL> A, B, C;
        A.load(pbase + cl[0] * col_stride, spad);
        B.load(pbase + cl[1] * col_stride, spad);
        uint32_t i = 0;
        while (i < n) {
          while (ws + i >= row_end) {
            flush();
            if (r_next >= r_stop) {  // only reachable with inconsistent offsets
              if (lane == 0) atomicOr(a.status, kStatusBadIndptr);
              drain(k + 1);
              return false;
            }
            row = r_next++;
            row_end = a.indptr[row + 1] - base;
            head = false;
            st.reset();
          }
          const uint32_t seg = min(row_end - ws, n);
          while (i + 3 <= seg) {  // prefetches reach i + 4 <= n + 1
            C.load(pbase + cl[i + 2] * col_stride, spad);
            eval_all<SPL>(A, lw[i], ws + i, active, st);
            A.load(pbase + cl[i + 3] * col_stride, spad);
            eval_all<SPL>(B, lw[i + 1], ws + i + 1, active, st);
            B.load(pbase + cl[i + 4] * col_stride, spad);
            eval_all<SPL>(C, lw[i + 2], ws + i + 2, active, st);
            i += 3;
          }
          if (i + 2 == seg) {
            C.load(pbase + cl[i + 2] * col_stride, spad);
            eval_all<SPL>(A, lw[i], ws + i, active, st);
            eval_all<SPL>(B, lw[i + 1], ws + i + 1, active, st);
            i += 2;
            A = C;
            B.load(pbase + cl[i + 1] * col_stride, spad);
          } else if (i + 1 == seg) {
            eval_all<SPL>(A, lw[i], ws + i, active, st);
            i += 1;
            A = B;
            B.load(pbase + cl[i + 1] * col_stride, spad);
          }
        }
        if (k + 2 < nwin) {
          const uint32_t ws2 = ws + 2 * kWin;
          issue_window<PACKED>(a, stg, pk, b, ws2, min(kWin, ce - ws2), bulk_ok, lane);
        }
        continue;
      }
      Params<SPL> A, B;
      uint32_t dA = cl[0], dB = 0;
      A.load(pbase + dA * col_stride, spad);
      uint32_t i = 0;
      while (i < n) {
        // Row boundaries (warp-uniform): finish rows, start the next owned one.
        while (ws + i >= row_end) {
          flush();
          if (r_next >= r_stop) {  // only reachable with inconsistent offsets
            if (lane == 0) atomicOr(a.status, kStatusBadIndptr);
            drain(k + 1);
            return false;
          }
          row = r_next++;
          row_end = a.indptr[row + 1] - base;
          head = false;
          st.reset();
        }
        const uint32_t seg = min(row_end - ws, n);
        // Pairs: A holds position i, B is loaded for i+1 while A is
        // evaluated, A for i+2 while B is evaluated.
        while (i + 1 < seg) {  // i + 2 <= n
          dB = cl[i + 1];
          B.load(pbase + dB * col_stride, spad);
          eval_all<SPL>(A, lw[i], ws + i, active, st);
          dA = cl[i + 2];
          A.load(pbase + dA * col_stride, spad);
          eval_all<SPL>(B, lw[i + 1], ws + i + 1, active, st);
          i += 2;
        }
        if (i < seg) {  // i + 1 <= n
          dB = cl[i + 1];
          B.load(pbase + dB * col_stride, spad);
          eval_all<SPL>(A, lw[i], ws + i, active, st);
          ++i;
          A = B;
          dA = dB;
        }
      }
      if (k + 2 < nwin) {
        const uint32_t ws2 = ws + 2 * kWin;
        issue_window<PACKED>(a, stg, pk, b, ws2, min(kWin, ce - ws2), bulk_ok, lane);
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
  return true;
}

// PACKED: the columns arrive as cols_lo/cols_hi (HashArgs::col_hi_bits).
template <int SPL, int MINB, int SPAD, bool PACKED>
__global__ void __launch_bounds__(kHashBlock, MINB) hash_kernel(const HashArgs a) {
  __shared__ WarpStage stage_all[kHashBlock / 32];
  PackedStage *packed_all = nullptr;
  if constexpr (PACKED) {
    __shared__ PackedStage packed_stage[kHashBlock / 32];
    packed_all = packed_stage;
  }
  if (*a.status & kStatusBadIndptr) return;
  WarpCtx wc;
  warp_ctx_init(wc, stage_all, packed_all);
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t items = a.nchunks * a.ntiles;
  for (uint32_t item = gw; item < items; item += nw) {
    const uint32_t c = item / a.ntiles;
    if (!hash_item<SPL, SPAD, PACKED, param_depth(MINB)>(a, c, item - c * a.ntiles, wc)) return;
  }
}

// Merge the partials of every row that leaves its own chunk: one warp per
// (chunk owning such a row, tile of 32 samples), lanes over samples.  The
// chunks the row runs through are read in position order with unconditional
// loads, kFinalizeUnroll in flight (a row of 50,000 nnz cut into 64-nnz
// chunks has ~780 partials), and a strict '<' keeps the earliest position on
// ties, as the scan of kernel.cu:106 does.
constexpr uint32_t kFinalizeUnroll = 8;

// Merges, for sample s, the partials of the row that leaves chunk c (if one
// does) and writes its output pair.
__device__ __forceinline__ void finalize_item(const HashArgs &a, uint32_t c, uint32_t s) {
  const uint32_t base = a.indptr[0];
  const uint32_t r0 = a.chunk_row[c];
  const uint32_t r1 = (c + 1 < a.nchunks) ? a.chunk_row[c + 1] : a.rows;
  if (r1 <= r0) return;
  const uint32_t row = r1 - 1;
  const uint32_t end = a.indptr[row + 1] - base;
  const uint32_t ce = c * a.chunk + min(a.chunk, a.nnz - c * a.chunk);
  if (end <= ce || s >= a.samples) return;
  const uint32_t c_last = (end - 1) / a.chunk;
  const size_t stride = 2 * static_cast<size_t>(a.s_pad);  // one chunk's two slots
  size_t off = static_cast<size_t>(2 * c + 1) * a.s_pad + s;
  float mn = a.part_ln[off];
  uint32_t kp = a.part_kt[off].x;
  off = static_cast<size_t>(2 * (c + 1)) * a.s_pad + s;
  uint32_t cc = c + 1;
  for (; cc + kFinalizeUnroll - 1 <= c_last; cc += kFinalizeUnroll) {
    float m[kFinalizeUnroll];
    uint32_t k[kFinalizeUnroll];
#pragma unroll
    for (uint32_t u = 0; u < kFinalizeUnroll; ++u) {
      m[u] = a.part_ln[off + u * stride];
      k[u] = a.part_kt[off + u * stride].x;
    }
#pragma unroll
    for (uint32_t u = 0; u < kFinalizeUnroll; ++u) {
      const bool lt = m[u] < mn;
      mn = lt ? m[u] : mn;
      kp = lt ? k[u] : kp;
    }
    off += kFinalizeUnroll * stride;
  }
  for (; cc <= c_last; ++cc, off += stride) {
    const float m2 = a.part_ln[off];
    const uint32_t k2 = a.part_kt[off].x;
    const bool lt = m2 < mn;
    mn = lt ? m2 : mn;
    kp = lt ? k2 : kp;
  }
  uint32_t *o = a.out + (static_cast<size_t>(row) * a.samples + s) * 2;
  *reinterpret_cast<uint2 *>(o) = resolve(a, kp, s);
}

__global__ void finalize_kernel(const HashArgs a) {
  // Any failure (invalid CSR, a staging copy that gave up) fails the call;
  // the partials a failed hash launch left may be stale, so none is merged.
  if (*a.status != 0) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t gw = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nw = (gridDim.x * static_cast<uint64_t>(blockDim.x)) >> 5;
  const uint32_t stiles = (a.samples + 31) / 32;
  const uint64_t items = static_cast<uint64_t>(a.nchunks) * stiles;
  for (uint64_t it = gw; it < items; it += nw) {
    const uint32_t c = static_cast<uint32_t>(it / stiles);
    const uint32_t s = static_cast<uint32_t>(it - static_cast<uint64_t>(c) * stiles) * 32 + lane;
    finalize_item(a, c, s);
  }
}

// ---- Device-resident batches ----------------------------------------------
// Many CSR matrices hashed against one generator by one persistent launch.
// Every matrix is cut into chunks of the same size; the batch's chunks are
// numbered matrix after matrix, and a warp item is (batch chunk, sample
// tile).  chunk_owner maps a batch chunk to its matrix, whose CSR, output and
// slice of the chunk table and partials the item then works on exactly as a
// single-matrix launch would: results equal one launch per matrix bit for bit
// (a row's arg-min and its ties do not depend on how positions are cut).

// HashArgs of matrix m inside batch b.
__device__ __forceinline__ HashArgs matrix_view(const BatchArgs &b, const BatchMatrix &m,
                                                uint32_t chunk) {
  HashArgs v = b.base;
  v.weights = m.weights;
  v.cols = m.cols;
  v.indptr = m.indptr;
  v.out = m.out;
  v.rows = m.rows;
  v.nnz = m.nnz;
  v.chunk = chunk;
  v.nchunks = m.nchunks;
  v.chunk_row = b.base.chunk_row + m.chunk_base;
  v.part_ln = b.base.part_ln + static_cast<size_t>(2) * m.chunk_base * b.base.s_pad;
  v.part_kt = b.base.part_kt + static_cast<size_t>(2) * m.chunk_base * b.base.s_pad;
  return v;
}

constexpr int kSetupThreads = 1024;

// Exclusive prefix sum over the block of one value per thread; returns this
// thread's offset and writes the total to *total.
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t x, uint64_t *total) {
  __shared__ uint64_t warp_sums[kSetupThreads / 32];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint64_t incl = x;
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= static_cast<uint32_t>(o)) incl += y;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint64_t w = lane < kSetupThreads / 32 ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= static_cast<uint32_t>(o)) w += y;
    }
    warp_sums[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const uint64_t before_warp = warp ? warp_sums[warp - 1] : 0;
  *total = warp_sums[kSetupThreads / 32 - 1];
  __syncthreads();
  return before_warp + incl - x;
}

// One block of kSetupThreads: per-matrix nnz (validating the end offsets),
// the batch's chunk size (the planner's rule applied to the whole batch, and
// large enough that the chunks fit max_chunks), each matrix's chunk range
// and the chunk -> matrix table.
__global__ void __launch_bounds__(kSetupThreads) batch_setup_kernel(const BatchArgs b) {
  const uint32_t t = threadIdx.x;
  const uint32_t per = (b.count + kSetupThreads - 1) / kSetupThreads;
  const uint32_t m0 = min(b.count, t * per), m1 = min(b.count, m0 + per);
  uint64_t nnz_sum = 0, rows_sum = 0, nonempty = 0;
  for (uint32_t m = m0; m < m1; ++m) {
    BatchMatrix &mt = b.mats[m];
    uint32_t n = 0;
    if (mt.rows) {
      const uint32_t s0 = mt.indptr[0], e = mt.indptr[mt.rows];
      if (e < s0) {
        atomicOr(b.base.status, kStatusBadIndptr);
      } else {
        n = e - s0;
      }
      ++nonempty;
    }
    mt.nnz = n;
    nnz_sum += n;
    rows_sum += mt.rows;
  }
  uint64_t total_nnz, total_rows, total_nonempty;
  block_exclusive_scan(nnz_sum, &total_nnz);
  block_exclusive_scan(rows_sum, &total_rows);
  block_exclusive_scan(nonempty, &total_nonempty);
  __shared__ uint32_t s_chunk;
  if (t == 0) {
    const uint64_t ntiles = b.base.ntiles;
    uint64_t chunk = (total_nnz * ntiles + b.target_items - 1) / b.target_items;
    const uint64_t avg_row = total_rows ? (total_nnz + total_rows - 1) / total_rows : 1;
    chunk = max(chunk, min(4 * avg_row, static_cast<uint64_t>(1024)));
    chunk = min(chunk, max(static_cast<uint64_t>(64),
                           (total_nnz * ntiles + b.want_items - 1) / b.want_items));
    // sum over matrices of ceil(nnz_m / chunk) <= total_nnz / chunk + nonempty
    const uint64_t avail = b.max_chunks > total_nonempty ? b.max_chunks - total_nonempty : 1;
    chunk = max(chunk, (total_nnz + avail - 1) / avail);
    chunk = max(static_cast<uint64_t>(64), (chunk + 31) & ~static_cast<uint64_t>(31));
    if (chunk > (1u << 24)) {
      chunk = 1u << 24;
      if (total_nnz / chunk + total_nonempty > b.max_chunks) atomicOr(b.base.status, kStatusBadIndptr);
    }
    s_chunk = static_cast<uint32_t>(chunk);
  }
  __syncthreads();
  const uint32_t chunk = s_chunk;
  uint64_t my_chunks = 0;
  for (uint32_t m = m0; m < m1; ++m) {
    const BatchMatrix &mt = b.mats[m];
    if (mt.rows) my_chunks += max(static_cast<uint64_t>(1), (static_cast<uint64_t>(mt.nnz) + chunk - 1) / chunk);
  }
  uint64_t total_chunks;
  uint64_t cb = block_exclusive_scan(my_chunks, &total_chunks);
  const bool fits = total_chunks <= b.max_chunks;
  for (uint32_t m = m0; m < m1; ++m) {
    BatchMatrix &mt = b.mats[m];
    const uint32_t nc = mt.rows ? static_cast<uint32_t>(max(
        static_cast<uint64_t>(1), (static_cast<uint64_t>(mt.nnz) + chunk - 1) / chunk)) : 0u;
    mt.chunk_base = static_cast<uint32_t>(cb);
    mt.nchunks = fits ? nc : 0u;
    if (fits)
      for (uint32_t c = 0; c < nc; ++c) b.chunk_owner[cb + c] = m;
    cb += nc;
  }
  if (t == 0) {
    if (!fits) atomicOr(b.base.status, kStatusBadIndptr);
    b.plan->chunk = chunk;
    b.plan->nchunks = fits ? static_cast<uint32_t>(total_chunks) : 0u;
  }
}

// Matrix owning plan thread g: the last one whose plan_base is <= g (matrices
// without rows own no threads and share the next matrix's plan_base).
__device__ __forceinline__ uint32_t plan_owner(const BatchArgs &b, uint32_t g) {
  uint32_t lo = 0, hi = b.count;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (b.plan_base[mid] <= g) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void batch_plan_kernel(const BatchArgs b, uint32_t plan_threads) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= plan_threads || (*b.base.status & kStatusBadIndptr)) return;
  const uint32_t m = plan_owner(b, g);
  const BatchMatrix mt = b.mats[m];
  if (!mt.rows || !mt.nchunks) return;
  const HashArgs v = matrix_view(b, mt, b.plan->chunk);
  plan_row(v, g - b.plan_base[m]);
}

// The matrix view of an item is kept in shared memory, one per warp: its
// fields are read where the item needs them (per row or window), so the
// evaluation loop's registers are the single-matrix kernel's.
template <int SPL, int MINB, int SPAD>
__global__ void __launch_bounds__(kHashBlock, MINB) hash_batch_kernel(const BatchArgs b) {
  __shared__ WarpStage stage_all[kHashBlock / 32];
  __shared__ HashArgs views[kHashBlock / 32];
  if (*b.base.status & kStatusBadIndptr) return;
  WarpCtx wc;
  warp_ctx_init(wc, stage_all);
  HashArgs &view = views[threadIdx.x >> 5];
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t ntiles = b.base.ntiles;
  const uint32_t chunk = b.plan->chunk;
  const uint32_t items = b.plan->nchunks * ntiles;
  for (uint32_t item = gw; item < items; item += nw) {
    const uint32_t gc = item / ntiles;
    const uint32_t m = b.chunk_owner[gc];
    const uint32_t base = b.mats[m].chunk_base;
    __syncwarp();
    if (wc.lane == 0) view = matrix_view(b, b.mats[m], chunk);
    __syncwarp();
    if (!hash_item<SPL, SPAD, false, param_depth(MINB)>(view, gc - base, item - gc * ntiles, wc))
      return;
  }
}

__global__ void finalize_batch_kernel(const BatchArgs b) {
  if (*b.base.status != 0) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t gw = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nw = (gridDim.x * static_cast<uint64_t>(blockDim.x)) >> 5;
  const uint32_t stiles = (b.base.samples + 31) / 32;
  const uint32_t chunk = b.plan->chunk;
  const uint64_t items = static_cast<uint64_t>(b.plan->nchunks) * stiles;
  for (uint64_t it = gw; it < items; it += nw) {
    const uint32_t gc = static_cast<uint32_t>(it / stiles);
    const uint32_t s = static_cast<uint32_t>(it - static_cast<uint64_t>(gc) * stiles) * 32 + lane;
    const BatchMatrix mt = b.mats[b.chunk_owner[gc]];
    if (mt.nchunks < 2) continue;  // a matrix of one chunk has no partials to merge
    const HashArgs v = matrix_view(b, mt, chunk);
    finalize_item(v, gc - mt.chunk_base, s);
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

namespace {

using HashFn = void (*)(const HashArgs);
using BatchFn = void (*)(const BatchArgs);

BatchFn pick_batch(uint32_t spl, uint32_t minb, uint32_t s_pad) {
  switch (spl * 100000 + minb * 10000 + s_pad) {
    case 440128: return hash_batch_kernel<4, 4, 128>;
    case 430128: return hash_batch_kernel<4, 3, 128>;
    case 420128: return hash_batch_kernel<4, 2, 128>;
    case 440256: return hash_batch_kernel<4, 4, 256>;
    case 430256: return hash_batch_kernel<4, 3, 256>;
    case 420256: return hash_batch_kernel<4, 2, 256>;
    case 240064: return hash_batch_kernel<2, 4, 64>;
    default: break;
  }
  switch (spl * 10 + minb) {
    case 44: return hash_batch_kernel<4, 4, 0>;
    case 43: return hash_batch_kernel<4, 3, 0>;
    case 42: return hash_batch_kernel<4, 2, 0>;
    case 24: return hash_batch_kernel<2, 4, 0>;
    case 14: return hash_batch_kernel<1, 4, 0>;
    default: return nullptr;
  }
}

// Instantiated (samples per lane, minimum resident blocks per SM) variants,
// with s_pad compiled in for the common sample counts.
HashFn pick_hash(uint32_t spl, uint32_t minb, uint32_t s_pad, bool packed = false) {
  if (packed) {
    switch (spl * 100000 + minb * 10000 + s_pad) {
      case 440128: return hash_kernel<4, 4, 128, true>;
      case 430128: return hash_kernel<4, 3, 128, true>;
      case 420128: return hash_kernel<4, 2, 128, true>;
      case 440256: return hash_kernel<4, 4, 256, true>;
      case 430256: return hash_kernel<4, 3, 256, true>;
      case 420256: return hash_kernel<4, 2, 256, true>;
      case 240064: return hash_kernel<2, 4, 64, true>;
      default: break;
    }
    switch (spl * 10 + minb) {
      case 44: return hash_kernel<4, 4, 0, true>;
      case 43: return hash_kernel<4, 3, 0, true>;
      case 42: return hash_kernel<4, 2, 0, true>;
      case 24: return hash_kernel<2, 4, 0, true>;
      case 14: return hash_kernel<1, 4, 0, true>;
      default: return nullptr;
    }
  }
  switch (spl * 100000 + minb * 10000 + s_pad) {
    case 440128: return hash_kernel<4, 4, 128, false>;
    case 430128: return hash_kernel<4, 3, 128, false>;
    case 420128: return hash_kernel<4, 2, 128, false>;
    case 440256: return hash_kernel<4, 4, 256, false>;
    case 430256: return hash_kernel<4, 3, 256, false>;
    case 420256: return hash_kernel<4, 2, 256, false>;
    case 240064: return hash_kernel<2, 4, 64, false>;
    default: break;
  }
  switch (spl * 10 + minb) {
    case 44: return hash_kernel<4, 4, 0, false>;
    case 43: return hash_kernel<4, 3, 0, false>;
    case 42: return hash_kernel<4, 2, 0, false>;
    case 24: return hash_kernel<2, 4, 0, false>;
    case 14: return hash_kernel<1, 4, 0, false>;
    default: return nullptr;
  }
}

}  // namespace

cudaError_t launch_hash(const HashArgs &a, const HashPlan &plan, cudaStream_t stream) {
  const HashFn fn = pick_hash(plan.spl, plan.minb, a.s_pad, a.col_hi_bits != 0);
  if (!fn) return cudaErrorInvalidValue;
  fn<<<plan.grid, kHashBlock, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const HashArgs &a, cudaStream_t stream) {
  const uint64_t warps_per_block = 8;
  const uint64_t items = static_cast<uint64_t>(a.nchunks) * ((a.samples + 31) / 32);
  uint64_t blocks = (items + warps_per_block - 1) / warps_per_block;
  if (blocks > 8192) blocks = 8192;
  finalize_kernel<<<static_cast<unsigned>(blocks), 32 * warps_per_block, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_batch(const BatchArgs &b, const HashPlan &plan, uint32_t plan_threads,
                         cudaStream_t stream) {
  const BatchFn fn = pick_batch(plan.spl, plan.minb, b.base.s_pad);
  if (!fn || b.count == 0 || b.max_chunks == 0) return cudaErrorInvalidValue;
  batch_setup_kernel<<<1, kSetupThreads, 0, stream>>>(b);
  if (plan_threads)
    batch_plan_kernel<<<(plan_threads + 255) / 256, 256, 0, stream>>>(b, plan_threads);
  fn<<<plan.grid, kHashBlock, 0, stream>>>(b);
  const uint64_t stiles = (b.base.samples + 31) / 32;
  uint64_t blocks = (static_cast<uint64_t>(b.max_chunks) * stiles + 7) / 8;
  blocks = std::min<uint64_t>(std::max<uint64_t>(blocks, 1), 8192);
  finalize_batch_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(b);
  return cudaGetLastError();
}

int hash_blocks_per_sm(uint32_t spl, uint32_t minb, uint32_t s_pad) {
  const HashFn fn = pick_hash(spl, minb, s_pad);
  int n = 0;
  if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kHashBlock, 0) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return n > 0 ? n : 1;
}

size_t hash_kernel_registers(uint32_t spl, uint32_t minb, uint32_t s_pad) {
  const HashFn fn = pick_hash(spl, minb, s_pad);
  cudaFuncAttributes attr{};
  if (!fn || cudaFuncGetAttributes(&attr, fn) != cudaSuccess) return 0;
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
